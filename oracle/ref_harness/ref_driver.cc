// ref_driver.cc -- C-ABI harness around the reference's own executor.
//
// TEST INFRASTRUCTURE ONLY. This file is compiled together with the
// reference's executor sources (src/clifft/svm/*.cc,
// src/clifft/api/record_probabilities.cc) and bytecode passes
// (src/clifft/optimizer/{noise_block,multi_gate,expand_t,swap_meas,
// tile_axis_fusion,single_axis_fusion}_pass.cc), read in place from the
// reference tree by oracle/build_ref.sh, into oracle/_ref/libclifft_ref.so.
// Tests and the CPU-baseline leg of bench.py load that library to pin the
// oracle restatement and to time the reference executor. Nothing in the
// product links or calls it.
//
// The reference's `lower()` (src/clifft/backend/backend.cc) needs Stim and
// cannot be built offline, so the instruction factories it defines
// (src/clifft/backend/backend.cc:28-295) and that the bytecode passes call are
// supplied here: each one only fills the fields of the 32-byte Instruction the
// way the header contract (src/clifft/backend/backend.h:172-211) describes.

#include "clifft/backend/backend.h"
#include "clifft/optimizer/expand_t_pass.h"
#include "clifft/optimizer/multi_gate_pass.h"
#include "clifft/optimizer/noise_block_pass.h"
#include "clifft/optimizer/single_axis_fusion_pass.h"
#include "clifft/optimizer/swap_meas_pass.h"
#include "clifft/optimizer/tile_axis_fusion_pass.h"
#include "clifft/svm/svm.h"

#include "clifft_program_image.h"

#include <omp.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <memory>
#include <string>
#include <thread>
#include <vector>

using namespace clifft;

// ---------------------------------------------------------------------------
// Instruction factories (declared at src/clifft/backend/backend.h:172-211).
// ---------------------------------------------------------------------------
namespace clifft {
namespace {
Instruction blank(Opcode op) {
    Instruction i{};
    i.opcode = op;
    return i;
}
Instruction two_axis(Opcode op, uint16_t a, uint16_t b) {
    Instruction i = blank(op);
    i.axis_1 = a;
    i.axis_2 = b;
    return i;
}
Instruction one_axis(Opcode op, uint16_t a) {
    Instruction i = blank(op);
    i.axis_1 = a;
    return i;
}
Instruction pauli_payload(Opcode op, uint32_t a, uint32_t b) {
    Instruction i = blank(op);
    i.pauli.cp_mask_idx = a;
    i.pauli.condition_idx = b;
    return i;
}
}  // namespace

Instruction make_frame_cnot(uint16_t c, uint16_t t) { return two_axis(Opcode::OP_FRAME_CNOT, c, t); }
Instruction make_frame_cz(uint16_t a, uint16_t b) { return two_axis(Opcode::OP_FRAME_CZ, a, b); }
Instruction make_frame_h(uint16_t v) { return one_axis(Opcode::OP_FRAME_H, v); }
Instruction make_frame_s(uint16_t v) { return one_axis(Opcode::OP_FRAME_S, v); }
Instruction make_frame_s_dag(uint16_t v) { return one_axis(Opcode::OP_FRAME_S_DAG, v); }
Instruction make_frame_swap(uint16_t a, uint16_t b) { return two_axis(Opcode::OP_FRAME_SWAP, a, b); }
Instruction make_array_cnot(uint16_t c, uint16_t t) { return two_axis(Opcode::OP_ARRAY_CNOT, c, t); }
Instruction make_array_cz(uint16_t a, uint16_t b) { return two_axis(Opcode::OP_ARRAY_CZ, a, b); }
Instruction make_array_swap(uint16_t a, uint16_t b) { return two_axis(Opcode::OP_ARRAY_SWAP, a, b); }
Instruction make_array_multi_cnot(uint16_t target, uint64_t mask) {
    Instruction i = one_axis(Opcode::OP_ARRAY_MULTI_CNOT, target);
    i.multi_gate.mask = mask;
    return i;
}
Instruction make_array_multi_cz(uint16_t control, uint64_t mask) {
    Instruction i = one_axis(Opcode::OP_ARRAY_MULTI_CZ, control);
    i.multi_gate.mask = mask;
    return i;
}
Instruction make_array_h(uint16_t a) { return one_axis(Opcode::OP_ARRAY_H, a); }
Instruction make_array_s(uint16_t a) { return one_axis(Opcode::OP_ARRAY_S, a); }
Instruction make_array_s_dag(uint16_t a) { return one_axis(Opcode::OP_ARRAY_S_DAG, a); }
Instruction make_array_t(uint16_t a) { return one_axis(Opcode::OP_ARRAY_T, a); }
Instruction make_array_t_dag(uint16_t a) { return one_axis(Opcode::OP_ARRAY_T_DAG, a); }
Instruction make_array_rot(uint16_t a, double re, double im) {
    Instruction i = one_axis(Opcode::OP_ARRAY_ROT, a);
    i.math.weight_re = re;
    i.math.weight_im = im;
    return i;
}
Instruction make_array_u2(uint16_t a, uint32_t cp) {
    Instruction i = one_axis(Opcode::OP_ARRAY_U2, a);
    i.u2.cp_idx = cp;
    return i;
}
Instruction make_array_u4(uint16_t lo, uint16_t hi, uint32_t cp) {
    Instruction i = two_axis(Opcode::OP_ARRAY_U4, lo, hi);
    i.u4.cp_idx = cp;
    return i;
}
Instruction make_expand(uint16_t a) { return one_axis(Opcode::OP_EXPAND, a); }
Instruction make_expand_t(uint16_t a) { return one_axis(Opcode::OP_EXPAND_T, a); }
Instruction make_expand_t_dag(uint16_t a) { return one_axis(Opcode::OP_EXPAND_T_DAG, a); }
Instruction make_expand_rot(uint16_t a, double re, double im) {
    Instruction i = one_axis(Opcode::OP_EXPAND_ROT, a);
    i.math.weight_re = re;
    i.math.weight_im = im;
    return i;
}
Instruction make_swap_meas_interfere(uint16_t f, uint16_t t, uint32_t idx, bool sign) {
    Instruction i = two_axis(Opcode::OP_SWAP_MEAS_INTERFERE, f, t);
    i.classical.classical_idx = idx;
    if (sign) i.flags |= Instruction::FLAG_SIGN;
    return i;
}
Instruction make_meas(Opcode op, uint16_t a, uint32_t idx, bool sign) {
    Instruction i = one_axis(op, a);
    i.classical.classical_idx = idx;
    if (sign) i.flags |= Instruction::FLAG_SIGN;
    return i;
}
Instruction make_apply_pauli(uint32_t m, uint32_t c) { return pauli_payload(Opcode::OP_APPLY_PAULI, m, c); }
Instruction make_noise(uint32_t s) { return pauli_payload(Opcode::OP_NOISE, s, 0); }
Instruction make_noise_block(uint32_t s, uint32_t n) { return pauli_payload(Opcode::OP_NOISE_BLOCK, s, n); }
Instruction make_readout_noise(uint32_t e) { return pauli_payload(Opcode::OP_READOUT_NOISE, e, 0); }
Instruction make_detector(uint32_t l, uint32_t c, ExpectedParity e) {
    Instruction i = pauli_payload(Opcode::OP_DETECTOR, l, c);
    if (e == ExpectedParity::One) i.flags |= Instruction::FLAG_EXPECTED_ONE;
    return i;
}
Instruction make_postselect(uint32_t l, uint32_t c, ExpectedParity e) {
    Instruction i = pauli_payload(Opcode::OP_POSTSELECT, l, c);
    if (e == ExpectedParity::One) i.flags |= Instruction::FLAG_EXPECTED_ONE;
    return i;
}
Instruction make_observable(uint32_t l, uint32_t o) { return pauli_payload(Opcode::OP_OBSERVABLE, l, o); }
Instruction make_exp_val(uint32_t cp, uint32_t idx) {
    Instruction i = blank(Opcode::OP_EXP_VAL);
    i.exp_val.cp_exp_val_idx = cp;
    i.exp_val.exp_val_idx = idx;
    return i;
}
}  // namespace clifft

// The harness never expands a dense statevector through the final tableau;
// the one Stim call the executor TUs reference fails loudly if reached.
template <>
std::vector<std::complex<float>> stim::Tableau<64>::to_flat_unitary_matrix(bool) const {
    throw std::logic_error("Stim is not available in the reference harness");
}

// ---------------------------------------------------------------------------
// image <-> CompiledModule
// ---------------------------------------------------------------------------
namespace {

thread_local std::string g_err;

PauliMaskArena arena_from(uint32_t nq, uint32_t nw, uint32_t count, const uint64_t* x,
                          const uint64_t* z, const uint8_t* s) {
    PauliMaskArena a(nq, count);
    for (uint32_t i = 0; i < count; ++i) {
        auto v = a.mut_at(static_cast<PauliMaskHandle>(i));
        for (uint32_t w = 0; w < nw; ++w) {
            v.x().words[w] = x[size_t(i) * nw + w];
            v.z().words[w] = z[size_t(i) * nw + w];
        }
        v.set_sign(s ? s[i] != 0 : false);
    }
    return a;
}

std::unique_ptr<CompiledModule> module_from_image(const clifft_program_image* img) {
    auto m = std::make_unique<CompiledModule>();
    const uint32_t nw = img->num_words;
    if (nw != (img->num_qubits + 63) / 64) throw std::invalid_argument("num_words != ceil(n/64)");
    m->num_qubits = img->num_qubits;
    m->peak_rank = img->peak_rank;
    m->num_measurements = img->num_measurements;
    m->total_meas_slots = img->total_meas_slots;
    m->num_detectors = img->num_detectors;
    m->num_observables = img->num_observables;
    m->num_exp_vals = img->num_exp_vals;
    m->has_postselection = img->has_postselection != 0;
    m->bytecode.resize(img->num_instructions);
    if (img->num_instructions)
        std::memcpy(m->bytecode.data(), img->instructions, size_t(img->num_instructions) * 32);
    auto& cp = m->constant_pool;
    cp.global_weight = {img->global_weight_re, img->global_weight_im};
    cp.pauli_masks = arena_from(img->num_qubits, nw, img->num_pauli_masks, img->pauli_x,
                                img->pauli_z, img->pauli_sign);
    cp.exp_val_masks = arena_from(img->num_qubits, nw, img->num_exp_val_masks, img->exp_val_x,
                                  img->exp_val_z, img->exp_val_sign);
    cp.noise_channel_masks = arena_from(img->num_qubits, nw, img->num_noise_channels,
                                        img->noise_channel_x, img->noise_channel_z, nullptr);
    cp.noise_sites.resize(img->num_noise_sites);
    for (uint32_t s = 0; s < img->num_noise_sites; ++s) {
        for (uint32_t c = img->noise_site_offsets[s]; c < img->noise_site_offsets[s + 1]; ++c) {
            cp.noise_sites[s].channels.push_back(
                NoiseChannel{static_cast<PauliMaskHandle>(c), img->noise_channel_prob[c]});
        }
    }
    cp.noise_hazards.assign(img->noise_hazards, img->noise_hazards + img->num_noise_sites);
    for (uint32_t r = 0; r < img->num_readout_noise; ++r)
        cp.readout_noise.push_back(ReadoutNoiseEntry{img->readout_meas_idx[r], img->readout_prob[r]});
    for (uint32_t d = 0; d < img->num_detector_lists; ++d)
        cp.detector_targets.emplace_back(img->detector_targets + img->detector_offsets[d],
                                         img->detector_targets + img->detector_offsets[d + 1]);
    for (uint32_t d = 0; d < img->num_observable_lists; ++d)
        cp.observable_targets.emplace_back(img->observable_targets + img->observable_offsets[d],
                                           img->observable_targets + img->observable_offsets[d + 1]);
    cp.fused_u2_nodes.resize(img->num_u2);
    for (uint32_t n = 0; n < img->num_u2; ++n) {
        const double* d = img->u2_data + size_t(n) * CLIFFT_U2_DOUBLES_PER_NODE;
        auto& node = cp.fused_u2_nodes[n];
        for (int s = 0; s < 4; ++s) {
            for (int e = 0; e < 4; ++e) node.matrices[s][e] = {d[(s * 5 + e) * 2], d[(s * 5 + e) * 2 + 1]};
            node.gamma_multipliers[s] = {d[(s * 5 + 4) * 2], d[(s * 5 + 4) * 2 + 1]};
            node.out_states[s] = img->u2_out[n * 4 + s];
        }
    }
    cp.fused_u4_nodes.resize(img->num_u4);
    for (uint32_t n = 0; n < img->num_u4; ++n) {
        const double* d = img->u4_data + size_t(n) * CLIFFT_U4_DOUBLES_PER_NODE;
        auto& node = cp.fused_u4_nodes[n];
        for (int s = 0; s < 16; ++s) {
            const double* e = d + s * 34;
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c)
                    node.entries[s].matrix[r][c] = {e[(r * 4 + c) * 2], e[(r * 4 + c) * 2 + 1]};
            node.entries[s].gamma_multiplier = {e[32], e[33]};
            node.entries[s].out_state = img->u4_out[n * 16 + s];
        }
    }
    m->expected_observables.assign(img->expected_observables,
                                   img->expected_observables + img->num_expected_observables);
    return m;
}

// Owned storage for a module exported back to an image.
struct ExportedModule {
    std::unique_ptr<CompiledModule> mod;
    std::vector<uint8_t> instr;
    std::vector<uint64_t> px, pz, ex, ez, nx, nz;
    std::vector<uint8_t> ps, es;
    std::vector<uint32_t> site_off, ro_idx, det_off, det_t, obs_off, obs_t;
    std::vector<double> chan_p, ro_p, u2, u4;
    std::vector<uint8_t> u2o, u4o, exp_obs;
    clifft_program_image img{};
};

void export_arena(const PauliMaskArena& a, uint32_t nw, std::vector<uint64_t>& x,
                  std::vector<uint64_t>& z, std::vector<uint8_t>* s) {
    for (size_t i = 0; i < a.size(); ++i) {
        auto v = a.at(static_cast<PauliMaskHandle>(i));
        for (uint32_t w = 0; w < nw; ++w) {
            x.push_back(v.x().words[w]);
            z.push_back(v.z().words[w]);
        }
        if (s) s->push_back(v.sign() ? 1 : 0);
    }
}

void export_module(ExportedModule& e) {
    const CompiledModule& m = *e.mod;
    const auto& cp = m.constant_pool;
    const uint32_t nw = (m.num_qubits + 63) / 64;
    e.instr.resize(m.bytecode.size() * 32);
    if (!m.bytecode.empty()) std::memcpy(e.instr.data(), m.bytecode.data(), e.instr.size());
    export_arena(cp.pauli_masks, nw, e.px, e.pz, &e.ps);
    export_arena(cp.exp_val_masks, nw, e.ex, e.ez, &e.es);
    e.site_off.push_back(0);
    for (const auto& site : cp.noise_sites) {
        for (const auto& ch : site.channels) {
            auto v = cp.noise_channel_masks.at(ch.mask);
            for (uint32_t w = 0; w < nw; ++w) {
                e.nx.push_back(v.x().words[w]);
                e.nz.push_back(v.z().words[w]);
            }
            e.chan_p.push_back(ch.prob);
        }
        e.site_off.push_back(static_cast<uint32_t>(e.chan_p.size()));
    }
    for (const auto& r : cp.readout_noise) {
        e.ro_idx.push_back(r.meas_idx);
        e.ro_p.push_back(r.prob);
    }
    e.det_off.push_back(0);
    for (const auto& l : cp.detector_targets) {
        e.det_t.insert(e.det_t.end(), l.begin(), l.end());
        e.det_off.push_back(static_cast<uint32_t>(e.det_t.size()));
    }
    e.obs_off.push_back(0);
    for (const auto& l : cp.observable_targets) {
        e.obs_t.insert(e.obs_t.end(), l.begin(), l.end());
        e.obs_off.push_back(static_cast<uint32_t>(e.obs_t.size()));
    }
    for (const auto& node : cp.fused_u2_nodes) {
        for (int s = 0; s < 4; ++s) {
            for (int k = 0; k < 4; ++k) {
                e.u2.push_back(node.matrices[s][k].real());
                e.u2.push_back(node.matrices[s][k].imag());
            }
            e.u2.push_back(node.gamma_multipliers[s].real());
            e.u2.push_back(node.gamma_multipliers[s].imag());
            e.u2o.push_back(node.out_states[s]);
        }
    }
    for (const auto& node : cp.fused_u4_nodes) {
        for (int s = 0; s < 16; ++s) {
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c) {
                    e.u4.push_back(node.entries[s].matrix[r][c].real());
                    e.u4.push_back(node.entries[s].matrix[r][c].imag());
                }
            e.u4.push_back(node.entries[s].gamma_multiplier.real());
            e.u4.push_back(node.entries[s].gamma_multiplier.imag());
            e.u4o.push_back(node.entries[s].out_state);
        }
    }
    e.exp_obs = m.expected_observables;

    auto& i = e.img;
    i.num_qubits = m.num_qubits;
    i.peak_rank = m.peak_rank;
    i.num_measurements = m.num_measurements;
    i.total_meas_slots = m.total_meas_slots;
    i.num_detectors = m.num_detectors;
    i.num_observables = m.num_observables;
    i.num_exp_vals = m.num_exp_vals;
    i.has_postselection = m.has_postselection ? 1 : 0;
    i.num_instructions = static_cast<uint32_t>(m.bytecode.size());
    i.instructions = e.instr.data();
    i.num_words = nw;
    i.num_pauli_masks = static_cast<uint32_t>(cp.pauli_masks.size());
    i.pauli_x = e.px.data();
    i.pauli_z = e.pz.data();
    i.pauli_sign = e.ps.data();
    i.num_exp_val_masks = static_cast<uint32_t>(cp.exp_val_masks.size());
    i.exp_val_x = e.ex.data();
    i.exp_val_z = e.ez.data();
    i.exp_val_sign = e.es.data();
    i.num_noise_sites = static_cast<uint32_t>(cp.noise_sites.size());
    i.noise_site_offsets = e.site_off.data();
    i.num_noise_channels = static_cast<uint32_t>(e.chan_p.size());
    i.noise_channel_prob = e.chan_p.data();
    i.noise_channel_x = e.nx.data();
    i.noise_channel_z = e.nz.data();
    i.noise_hazards = cp.noise_hazards.data();
    i.num_readout_noise = static_cast<uint32_t>(e.ro_idx.size());
    i.readout_meas_idx = e.ro_idx.data();
    i.readout_prob = e.ro_p.data();
    i.num_detector_lists = static_cast<uint32_t>(cp.detector_targets.size());
    i.detector_offsets = e.det_off.data();
    i.detector_targets = e.det_t.data();
    i.num_observable_lists = static_cast<uint32_t>(cp.observable_targets.size());
    i.observable_offsets = e.obs_off.data();
    i.observable_targets = e.obs_t.data();
    i.num_u2 = static_cast<uint32_t>(cp.fused_u2_nodes.size());
    i.u2_data = e.u2.data();
    i.u2_out = e.u2o.data();
    i.num_u4 = static_cast<uint32_t>(cp.fused_u4_nodes.size());
    i.u4_data = e.u4.data();
    i.u4_out = e.u4o.data();
    i.num_expected_observables = static_cast<uint32_t>(e.exp_obs.size());
    i.expected_observables = e.exp_obs.data();
    i.global_weight_re = cp.global_weight.real();
    i.global_weight_im = cp.global_weight.imag();
}

template <typename F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    } catch (...) {
        g_err = "unknown exception";
        return -1;
    }
}

Opcode forced_variant(Opcode op) {
    switch (op) {
        case Opcode::OP_MEAS_DORMANT_STATIC: return Opcode::OP_MEAS_DORMANT_STATIC_FORCED;
        case Opcode::OP_MEAS_DORMANT_RANDOM: return Opcode::OP_MEAS_DORMANT_RANDOM_FORCED;
        case Opcode::OP_MEAS_ACTIVE_DIAGONAL: return Opcode::OP_MEAS_ACTIVE_DIAGONAL_FORCED;
        case Opcode::OP_MEAS_ACTIVE_INTERFERE: return Opcode::OP_MEAS_ACTIVE_INTERFERE_FORCED;
        case Opcode::OP_SWAP_MEAS_INTERFERE: return Opcode::OP_SWAP_MEAS_INTERFERE_FORCED;
        default: return op;
    }
}

bool is_forced_meas(Opcode op) {
    return op >= Opcode::OP_MEAS_DORMANT_STATIC_FORCED && op <= Opcode::OP_SWAP_MEAS_INTERFERE_FORCED;
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

const char* ref_svm_backend(void) { return svm_backend(); }

// clifft::sample (src/clifft/svm/svm.cc:191-255) with unpacked uint8 outputs.
int ref_sample(const clifft_program_image* img, uint32_t shots, uint64_t seed, uint8_t* meas,
               uint8_t* det, uint8_t* obs, double* exp_vals) {
    return guarded([&] {
        auto m = module_from_image(img);
        auto r = sample(*m, shots, seed);
        if (meas && !r.measurements.empty()) std::memcpy(meas, r.measurements.data(), r.measurements.size());
        if (det && !r.detectors.empty()) std::memcpy(det, r.detectors.data(), r.detectors.size());
        if (obs && !r.observables.empty()) std::memcpy(obs, r.observables.data(), r.observables.size());
        if (exp_vals && !r.exp_vals.empty())
            std::memcpy(exp_vals, r.exp_vals.data(), r.exp_vals.size() * sizeof(double));
        return 0;
    });
}

// clifft::sample_k (src/clifft/svm/svm.cc:548-613): every shot conditioned on
// exactly k faults. Throws (status -1, message) for strata without mass.
int ref_sample_k(const clifft_program_image* img, uint32_t shots, uint32_t k, uint64_t seed, uint8_t* meas,
                 uint8_t* det, uint8_t* obs, double* exp_vals) {
    return guarded([&] {
        auto m = module_from_image(img);
        auto r = sample_k(*m, shots, k, seed);
        if (meas && !r.measurements.empty()) std::memcpy(meas, r.measurements.data(), r.measurements.size());
        if (det && !r.detectors.empty()) std::memcpy(det, r.detectors.data(), r.detectors.size());
        if (obs && !r.observables.empty()) std::memcpy(obs, r.observables.data(), r.observables.size());
        if (exp_vals && !r.exp_vals.empty())
            std::memcpy(exp_vals, r.exp_vals.data(), r.exp_vals.size() * sizeof(double));
        return 0;
    });
}

// clifft::noise_site_probabilities (src/clifft/svm/svm.cc:356-369) into out
// (noise sites then readout entries); returns the count.
int64_t ref_noise_site_probabilities(const clifft_program_image* img, double* out, uint64_t cap) {
    int64_t n = -1;
    int rc = guarded([&] {
        auto m = module_from_image(img);
        auto p = noise_site_probabilities(*m);
        for (size_t i = 0; i < p.size() && i < cap; ++i) out[i] = p[i];
        n = int64_t(p.size());
        return 0;
    });
    return rc == 0 ? n : -1;
}

// clifft::sample_survivors (src/clifft/svm/svm.cc:266-345). counts[0..2] =
// total_shots, passed_shots, logical_errors. Record buffers must hold `shots`
// rows; the return value is the number of rows written.
int64_t ref_sample_survivors(const clifft_program_image* img, uint32_t shots, uint64_t seed,
                             int keep_records, uint64_t* counts, uint64_t* observable_ones,
                             uint8_t* meas, uint8_t* det, uint8_t* obs, double* exp_vals) {
    int64_t rows = -1;
    int rc = guarded([&] {
        auto m = module_from_image(img);
        auto r = sample_survivors(*m, shots, seed, keep_records != 0);
        counts[0] = r.total_shots;
        counts[1] = r.passed_shots;
        counts[2] = r.logical_errors;
        for (size_t i = 0; i < r.observable_ones.size(); ++i) observable_ones[i] = r.observable_ones[i];
        if (keep_records) {
            if (meas && !r.measurements.empty()) std::memcpy(meas, r.measurements.data(), r.measurements.size());
            if (det && !r.detectors.empty()) std::memcpy(det, r.detectors.data(), r.detectors.size());
            if (obs && !r.observables.empty()) std::memcpy(obs, r.observables.data(), r.observables.size());
            if (exp_vals && !r.exp_vals.empty())
                std::memcpy(exp_vals, r.exp_vals.data(), r.exp_vals.size() * sizeof(double));
        }
        rows = keep_records ? r.passed_shots : 0;
        return 0;
    });
    return rc == 0 ? rows : -1;
}

// Wall-clock timing of clifft::sample / sample_survivors on `threads` host
// threads, each running its own contiguous shot slice with seed `seed + t`
// (the shot-parallel CPU baseline). Returns elapsed seconds, < 0 on error.
double ref_time_sample_omp(const clifft_program_image* img, uint64_t shots, uint64_t seed,
                           int threads, int survivors, int omp_threads) {
    double secs = -1.0;
    guarded([&] {
        auto m = module_from_image(img);
        if (threads < 1) threads = 1;
        if (omp_threads < 1) omp_threads = 1;
        std::vector<std::thread> pool;
        std::vector<std::string> errs(threads);
        auto t0 = std::chrono::steady_clock::now();
        for (int t = 0; t < threads; ++t) {
            uint64_t lo = shots * t / threads, hi = shots * (t + 1) / threads;
            pool.emplace_back([&, t, lo, hi] {
                try {
                    // OpenMP team size of this worker's own parallel regions
                    // (the executor's intra-shot loops for large k)
                    omp_set_num_threads(omp_threads);
                    if (survivors)
                        (void)sample_survivors(*m, static_cast<uint32_t>(hi - lo), seed + t, false);
                    else
                        (void)sample(*m, static_cast<uint32_t>(hi - lo), seed + t);
                } catch (const std::exception& ex) {
                    errs[t] = ex.what();
                }
            });
        }
        for (auto& th : pool) th.join();
        auto t1 = std::chrono::steady_clock::now();
        for (auto& e : errs)
            if (!e.empty()) throw std::runtime_error(e);
        secs = std::chrono::duration<double>(t1 - t0).count();
        return 0;
    });
    return secs;
}

double ref_time_sample(const clifft_program_image* img, uint64_t shots, uint64_t seed, int threads,
                       int survivors) {
    return ref_time_sample_omp(img, shots, seed, threads, survivors, 1);
}

// Forced replay of `shots` trajectories, executed one instruction at a time.
//
// Measurements are rewritten to their *_FORCED variants (as
// src/clifft/api/record_probabilities.cc:96-118 does) and take their outcome
// from forced_meas[shot * total_meas_slots + slot]. Faults are injected through
// SchrodingerState::ForcedFaults (src/clifft/svm/svm.h:211-227): the fired
// noise sites of shot s are fault_sites[fault_offsets[s] .. fault_offsets[s+1])
// (ascending) and each fired site is patched to the single channel
// fault_channels[...] with probability 1, because exec_noise still draws a
// channel from the PRNG (src/clifft/svm/svm_kernels.inl:1899-1911). Readout
// flips are readout_entries[readout_offsets[s] .. readout_offsets[s+1]).
//
// Per shot outputs: meas (total_meas_slots bytes), det, obs (raw obs_record
// XOR expected_observables), exp_vals, meas_prob (probability of the forced
// outcome at each slot, NaN if the slot never executed), log_prob, reachable,
// discarded, final active_k, gamma (re, im), p_x / p_z (num_words each) and
// the first 2^final_k amplitudes of v (row stride 2^peak_rank complex).
int ref_forced_run(const clifft_program_image* img, uint32_t shots, const uint8_t* forced_meas,
                   const uint32_t* fault_offsets, const uint32_t* fault_sites,
                   const uint32_t* fault_channels, const uint32_t* readout_offsets,
                   const uint32_t* readout_entries, uint8_t* meas, uint8_t* det, uint8_t* obs,
                   double* exp_vals, double* meas_prob, double* log_prob, uint8_t* reachable,
                   uint8_t* discarded, uint32_t* final_k, double* gamma, uint64_t* px,
                   uint64_t* pz, double* v) {
    return guarded([&] {
        auto base = module_from_image(img);
        for (auto& ins : base->bytecode) ins.opcode = forced_variant(ins.opcode);
        const uint32_t slots = base->total_meas_slots;
        const uint32_t nw = img->num_words;
        const uint64_t vstride = uint64_t{1} << base->peak_rank;
        CompiledModule step;
        for (uint32_t s = 0; s < shots; ++s) {
            // Per-shot constant pool: fired sites collapse to their forced channel.
            step.constant_pool = base->constant_pool;
            step.num_qubits = base->num_qubits;
            step.peak_rank = base->peak_rank;
            step.num_measurements = base->num_measurements;
            step.total_meas_slots = base->total_meas_slots;
            step.num_detectors = base->num_detectors;
            step.num_observables = base->num_observables;
            step.num_exp_vals = base->num_exp_vals;
            step.has_postselection = base->has_postselection;
            SchrodingerState st({.peak_rank = base->peak_rank,
                                 .num_measurements = slots,
                                 .num_qubits = base->num_qubits,
                                 .num_detectors = base->num_detectors,
                                 .num_observables = base->num_observables,
                                 .num_exp_vals = base->num_exp_vals,
                                 .seed = 0});
            auto& ff = st.forced_faults;
            ff.active = true;
            if (fault_offsets) {
                for (uint32_t f = fault_offsets[s]; f < fault_offsets[s + 1]; ++f) {
                    uint32_t site = fault_sites[f];
                    auto& chans = step.constant_pool.noise_sites.at(site).channels;
                    NoiseChannel only = chans.at(fault_channels[f]);
                    only.prob = 1.0;
                    chans.assign(1, only);
                    ff.noise_indices.push_back(site);
                }
            }
            if (readout_offsets)
                for (uint32_t f = readout_offsets[s]; f < readout_offsets[s + 1]; ++f)
                    ff.readout_indices.push_back(readout_entries[f]);
            if (!ff.noise_indices.empty()) {
                st.next_noise_idx = ff.noise_indices[0];
                ff.noise_pos = 1;
            } else {
                st.next_noise_idx = static_cast<uint32_t>(-1);
            }
            std::vector<uint8_t> rec(forced_meas + size_t(s) * slots, forced_meas + size_t(s + 1) * slots);
            st.forced_record = std::span<const uint8_t>(rec);
            double* mp = meas_prob ? meas_prob + size_t(s) * slots : nullptr;
            if (mp)
                for (uint32_t k = 0; k < slots; ++k) mp[k] = std::nan("");
            step.bytecode.resize(1);
            for (const auto& ins : base->bytecode) {
                step.bytecode[0] = ins;
                double before = st.forced_log_probability;
                execute(step, st);
                if (is_forced_meas(ins.opcode) && mp && st.forced_reachable)
                    mp[ins.classical.classical_idx] = std::exp(st.forced_log_probability - before);
                if (!st.forced_reachable || st.discarded) break;
            }
            if (meas) std::memcpy(meas + size_t(s) * slots, st.meas_record.data(), slots);
            if (det && base->num_detectors)
                std::memcpy(det + size_t(s) * base->num_detectors, st.det_record.data(), base->num_detectors);
            if (obs)
                for (uint32_t i = 0; i < base->num_observables; ++i) {
                    uint8_t val = st.obs_record[i];
                    if (i < base->expected_observables.size() && base->expected_observables[i]) val ^= 1;
                    obs[size_t(s) * base->num_observables + i] = val;
                }
            if (exp_vals && base->num_exp_vals)
                std::memcpy(exp_vals + size_t(s) * base->num_exp_vals, st.exp_vals.data(),
                            base->num_exp_vals * sizeof(double));
            if (log_prob) log_prob[s] = st.forced_log_probability;
            if (reachable) reachable[s] = st.forced_reachable ? 1 : 0;
            if (discarded) discarded[s] = st.discarded ? 1 : 0;
            if (final_k) final_k[s] = st.active_k;
            if (gamma) {
                gamma[2 * s] = st.gamma().real();
                gamma[2 * s + 1] = st.gamma().imag();
            }
            for (uint32_t w = 0; w < nw; ++w) {
                if (px) px[size_t(s) * nw + w] = st.p_x[w];
                if (pz) pz[size_t(s) * nw + w] = st.p_z[w];
            }
            if (v) {
                double* row = v + size_t(s) * vstride * 2;
                for (uint64_t i = 0; i < vstride; ++i) {
                    auto a = i < st.v_size() ? st.v()[i] : std::complex<double>{0.0, 0.0};
                    row[2 * i] = a.real();
                    row[2 * i + 1] = a.imag();
                }
            }
        }
        return 0;
    });
}

// Run a subset of the reference's bytecode passes over a program. Bit i of
// `pass_mask` enables, in registry order (src/clifft/optimizer/pass_registry.h:67-95):
// 0 NoiseBlock, 1 MultiGate, 2 ExpandT, 3 ExpandRot, 4 SwapMeas,
// 5 TileAxisFusion, 6 SingleAxisFusion. The result is returned through an
// opaque handle whose image stays valid until ref_module_free.
void* ref_run_passes(const clifft_program_image* img, uint32_t pass_mask) {
    ExportedModule* out = nullptr;
    guarded([&] {
        auto e = std::make_unique<ExportedModule>();
        e->mod = module_from_image(img);
        BytecodePassManager pm;
        if (pass_mask & 1u) pm.add_pass(std::make_unique<NoiseBlockPass>());
        if (pass_mask & 2u) pm.add_pass(std::make_unique<MultiGatePass>());
        if (pass_mask & 4u) pm.add_pass(std::make_unique<ExpandTPass>());
        if (pass_mask & 8u) pm.add_pass(std::make_unique<ExpandRotPass>());
        if (pass_mask & 16u) pm.add_pass(std::make_unique<SwapMeasPass>());
        if (pass_mask & 32u) pm.add_pass(std::make_unique<TileAxisFusionPass>());
        if (pass_mask & 64u) pm.add_pass(std::make_unique<SingleAxisFusionPass>());
        pm.run(*e->mod);
        export_module(*e);
        out = e.release();
        return 0;
    });
    return out;
}

const clifft_program_image* ref_module_image(void* handle) {
    return handle ? &static_cast<ExportedModule*>(handle)->img : nullptr;
}

void ref_module_free(void* handle) { delete static_cast<ExportedModule*>(handle); }

}  // extern "C"
