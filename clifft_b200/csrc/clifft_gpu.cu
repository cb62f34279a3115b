// clifft_gpu.cu -- C ABI of the sm_100a Schrodinger-VM backend (include/clifft_gpu.h).
//
// Host side: program validation and upload, launch-shape selection, scratch
// and output management around the persistent interpreter kernel of
// svm_kernel.cuh.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <type_traits>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "clifft_gpu.h"
#include "svm_dispatch.h"
#include "svm_grad.h"
#include "svm_kernel.cuh"
#include "svm_sample_k.h"

using namespace cgpu;

namespace {

thread_local std::string g_last_error;

struct ApiError : std::runtime_error {
    int code;
    ApiError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CUDA_OK(expr)                                                                         \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess)                                                                \
            throw ApiError(_e == cudaErrorMemoryAllocation ? CLIFFT_GPU_ENOMEM : CLIFFT_GPU_ECUDA, \
                           std::string(#expr) + ": " + cudaGetErrorString(_e));               \
    } while (0)

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return CLIFFT_GPU_OK;
    } catch (const ApiError& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return CLIFFT_GPU_EINVAL;
    }
}

[[noreturn]] void invalid(const std::string& m) { throw ApiError(CLIFFT_GPU_EINVAL, m); }

constexpr uint32_t kMaxPeakRank = 34;  // 2^34 complex FP32 = 128 GiB: beyond one B200's HBM per shot
constexpr uint32_t kMaxWords = 4;      // frame width: num_qubits <= 256

uint16_t rd16(const uint8_t* p) {
    uint16_t v;
    std::memcpy(&v, p, 2);
    return v;
}
uint32_t rd32(const uint8_t* p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}
uint64_t rd64(const uint8_t* p) {
    uint64_t v;
    std::memcpy(&v, p, 8);
    return v;
}

// Checks the invariants the reference executor asserts
// (src/clifft/svm/svm_kernels.inl: axis < active_k for array ops, EXPAND on
// axis k, active measurements on axis k-1, pool indices in range) so that no
// launch can index outside the program or the statevector.
uint32_t validate(const clifft_program_image& im) {
    if (im.num_words != (im.num_qubits + 63) / 64 && !(im.num_qubits == 0 && im.num_words <= 1))
        invalid("num_words must equal ceil(num_qubits / 64)");
    if (im.num_words > kMaxWords) invalid("num_qubits > 256 is not supported by the CUDA backend");
    if (im.peak_rank > kMaxPeakRank) invalid("peak_rank too large for one GPU");
    if (im.total_meas_slots < im.num_measurements) invalid("total_meas_slots < num_measurements");
    if (im.num_instructions && !im.instructions) invalid("null instruction array");
    const uint32_t nq = std::max<uint32_t>(im.num_qubits, 1);
    const uint32_t frame_bits = std::max<uint32_t>(im.num_words, 1) * 64;
    for (uint32_t s = 0; s < im.num_noise_sites; ++s)
        if (im.noise_site_offsets[s] > im.noise_site_offsets[s + 1] ||
            im.noise_site_offsets[s + 1] > im.num_noise_channels)
            invalid("noise site offsets out of range");
    for (uint32_t d = 0; d < im.num_detector_lists; ++d)
        for (uint32_t i = im.detector_offsets[d]; i < im.detector_offsets[d + 1]; ++i)
            if (im.detector_targets[i] >= im.total_meas_slots) invalid("detector target out of range");
    for (uint32_t d = 0; d < im.num_observable_lists; ++d)
        for (uint32_t i = im.observable_offsets[d]; i < im.observable_offsets[d + 1]; ++i)
            if (im.observable_targets[i] >= im.total_meas_slots) invalid("observable target out of range");
    for (uint32_t r = 0; r < im.num_readout_noise; ++r)
        if (im.readout_meas_idx[r] >= im.total_meas_slots) invalid("readout entry out of range");
    for (uint32_t n = 0; n < im.num_u2 * 4; ++n)
        if (im.u2_out[n] > 3) invalid("U2 out state out of range");
    for (uint32_t n = 0; n < im.num_u4 * 16; ++n)
        if (im.u4_out[n] > 15) invalid("U4 out state out of range");

    uint32_t k = 0, peak = 0;
    for (uint32_t pc = 0; pc < im.num_instructions; ++pc) {
        const uint8_t* I = im.instructions + size_t(pc) * 32;
        uint32_t op = I[0];
        const uint32_t fl = I[2];
        const uint32_t a1 = rd16(I + 4), a2 = rd16(I + 6);
        const uint32_t p0 = rd32(I + 8), p1 = rd32(I + 12);
        auto bad = [&](const char* what) {
            char buf[160];
            std::snprintf(buf, sizeof buf, "instruction %u (opcode %u): %s (active_k=%u)", pc, I[0], what, k);
            invalid(buf);
        };
        if (op >= CLIFFT_OP_MEAS_DORMANT_STATIC_FORCED && op <= CLIFFT_OP_SWAP_MEAS_INTERFERE_FORCED)
            op -= CLIFFT_OP_MEAS_DORMANT_STATIC_FORCED - CLIFFT_OP_MEAS_DORMANT_STATIC;
        switch (op) {
            case CLIFFT_OP_FRAME_CNOT:
            case CLIFFT_OP_FRAME_CZ:
            case CLIFFT_OP_FRAME_SWAP:
                if (a1 >= frame_bits || a2 >= frame_bits) bad("axis beyond the frame");
                break;
            case CLIFFT_OP_FRAME_H:
            case CLIFFT_OP_FRAME_S:
            case CLIFFT_OP_FRAME_S_DAG:
                if (a1 >= frame_bits) bad("axis beyond the frame");
                break;
            case CLIFFT_OP_ARRAY_CNOT:
            case CLIFFT_OP_ARRAY_CZ:
            case CLIFFT_OP_ARRAY_SWAP:
                if (a1 >= k || a2 >= k || a1 == a2) bad("two-axis array op needs distinct active axes");
                break;
            case CLIFFT_OP_ARRAY_MULTI_CNOT:
            case CLIFFT_OP_ARRAY_MULTI_CZ: {
                uint64_t m = rd64(I + 8);
                if (a1 >= k) bad("multi-gate pivot axis not active");
                if (k < 64 && (m >> k)) bad("multi-gate mask has dormant axes");
                if ((m >> a1) & 1u) bad("multi-gate mask contains its own pivot");
                break;
            }
            case CLIFFT_OP_ARRAY_H:
            case CLIFFT_OP_ARRAY_S:
            case CLIFFT_OP_ARRAY_S_DAG:
                if (a1 >= k) bad("array op on a dormant axis");
                break;
            case CLIFFT_OP_ARRAY_T:
            case CLIFFT_OP_ARRAY_T_DAG:
            case CLIFFT_OP_ARRAY_ROT:
                if (a1 >= frame_bits) bad("axis beyond the frame");
                break;
            case CLIFFT_OP_ARRAY_U2:
                if (a1 >= frame_bits) bad("axis beyond the frame");
                if (p0 >= im.num_u2) bad("U2 constant-pool index out of range");
                break;
            case CLIFFT_OP_ARRAY_U4:
                if (!(a1 < a2 && a2 < k)) bad("U4 needs axis_lo < axis_hi < active_k");
                if (p0 >= im.num_u4) bad("U4 constant-pool index out of range");
                break;
            case CLIFFT_OP_EXPAND:
            case CLIFFT_OP_EXPAND_T:
            case CLIFFT_OP_EXPAND_T_DAG:
            case CLIFFT_OP_EXPAND_ROT:
                if (a1 != k) bad("EXPAND must target axis active_k");
                if (a1 >= frame_bits) bad("axis beyond the frame");
                ++k;
                peak = std::max(peak, k);
                if (k > im.peak_rank) bad("EXPAND exceeds peak_rank");
                break;
            case CLIFFT_OP_MEAS_DORMANT_STATIC:
            case CLIFFT_OP_MEAS_DORMANT_RANDOM:
                if (p0 >= im.total_meas_slots) bad("classical index out of range");
                if (!(fl & CLIFFT_FLAG_IDENTITY) && a1 >= frame_bits) bad("axis beyond the frame");
                break;
            case CLIFFT_OP_MEAS_ACTIVE_DIAGONAL:
            case CLIFFT_OP_MEAS_ACTIVE_INTERFERE:
                if (k == 0 || a1 != k - 1) bad("active measurement must target axis active_k-1");
                if (p0 >= im.total_meas_slots) bad("classical index out of range");
                --k;
                break;
            case CLIFFT_OP_SWAP_MEAS_INTERFERE:
                if (k == 0 || a2 != k - 1 || a1 > a2) bad("swap-measure must target axis active_k-1");
                if (p0 >= im.total_meas_slots) bad("classical index out of range");
                --k;
                break;
            case CLIFFT_OP_APPLY_PAULI:
                if (p0 >= im.num_pauli_masks) bad("Pauli mask index out of range");
                if (p1 >= im.total_meas_slots) bad("condition index out of range");
                break;
            case CLIFFT_OP_NOISE:
                if (p0 >= im.num_noise_sites) bad("noise site out of range");
                break;
            case CLIFFT_OP_NOISE_BLOCK:
                if (uint64_t(p0) + p1 > im.num_noise_sites) bad("noise block out of range");
                break;
            case CLIFFT_OP_READOUT_NOISE:
                if (p0 >= im.num_readout_noise) bad("readout entry out of range");
                break;
            case CLIFFT_OP_DETECTOR:
            case CLIFFT_OP_POSTSELECT:
                if (p0 >= im.num_detector_lists) bad("detector list out of range");
                if (p1 >= im.num_detectors) bad("detector index out of range");
                break;
            case CLIFFT_OP_OBSERVABLE:
                if (p0 >= im.num_observable_lists) bad("observable list out of range");
                if (p1 >= im.num_observables) bad("observable index out of range");
                break;
            case CLIFFT_OP_EXP_VAL:
                if (p0 >= im.num_exp_val_masks) bad("EXP_VAL mask out of range");
                if (p1 >= im.num_exp_vals) bad("EXP_VAL index out of range");
                break;
            default:
                bad("unknown opcode");
        }
    }
    (void)nq;
    return peak;
}


// Returns the current device's parked spare slab to the device (defined with
// the spare slabs below); true when there was one.
bool spare_release_current();
// A device allocation that, when the device is out of memory, returns the
// parked spare slab and tries once more.
template <class Alloc>
cudaError_t alloc_retry(Alloc&& alloc) {
    cudaError_t e = alloc();
    if (e == cudaErrorMemoryAllocation && spare_release_current()) {
        cudaGetLastError();  // clear the failed allocation's error
        e = alloc();
    }
    return e;
}

// Device-side scratch freed in stream order when the call ends.
struct StreamBuffers {
    cudaStream_t stream;
    std::vector<void*> ptrs;
    explicit StreamBuffers(cudaStream_t s) : stream(s) {}
    void* alloc(size_t bytes) {
        void* p = nullptr;
        if (bytes == 0) return nullptr;
        CUDA_OK(alloc_retry([&] { return cudaMallocAsync(&p, bytes, stream); }));
        ptrs.push_back(p);
        return p;
    }
    ~StreamBuffers() {
        for (void* p : ptrs) cudaFreeAsync(p, stream);
    }
};

}  // namespace

struct clifft_gpu_program {
    clifft_program_image meta{};  // counts only (host pointers dropped)
    DevProg dev{};
    void* blob = nullptr;
    size_t blob_bytes = 0;
    std::vector<uint8_t> expected_host;
    int device = 0;
    uint64_t content_hash = 0;  // FNV-1a of the device image and the launch-relevant counts
    std::vector<uint8_t> instr_host;  // the 32-byte instructions (host copy, for gradient programs)
    uint32_t num_rot_params = 0;      // ARRAY_ROT + EXPAND_ROT instructions
    std::vector<double> fault_probs;  // per noise site its total probability, then per readout entry its flip
                                      // probability (clifft::noise_site_probabilities order)
    // launch shapes already planned for this program (see plan_launch)
    mutable std::mutex plan_mu;
    mutable std::map<std::tuple<uint32_t, uint32_t, bool, uint32_t, uint32_t, uint32_t, bool>, std::vector<uint8_t>>
        plan_cache;
    // Statevector slab kept between calls (mapping tens of GB afresh on every
    // call costs more than a large-k launch's own setup). One call at a time
    // holds it; a concurrent call on the same handle allocates its own.
    std::mutex slab_mu;
    void* slab = nullptr;
    size_t slab_bytes = 0;
    bool slab_busy = false;
};

namespace {

// A call's use of the program's statevector slab: the first request takes the
// cached slab (growing it if needed); later requests of the same call reuse
// it, since the call's launches run one after another on one stream.
// One spare statevector slab per device, taken over by a program's first
// sampling call when it fits. Released programs free their slabs (parking
// them here made the 64-program batch graph 20x slower, cause not found), so
// the pool stays empty unless a caller fills it; clifft_gpu_trim empties it.
std::mutex g_spare_mu;
std::map<int, std::pair<void*, size_t>> g_spare;  // device -> (slab, bytes)

// takes the device's spare when it holds `bytes` without wasting more than
// as much again; a smaller spare is freed, a much larger one stays parked
// (an allocation that runs out of memory releases it)
void* spare_take(int device, size_t bytes, size_t* got) {
    void* ptr = nullptr;
    size_t have = 0;
    {
        std::lock_guard<std::mutex> lock(g_spare_mu);
        auto it = g_spare.find(device);
        if (it == g_spare.end()) return nullptr;
        have = it->second.second;
        if (have > 2 * bytes) return nullptr;
        ptr = it->second.first;
        g_spare.erase(it);
    }
    if (have >= bytes) {
        *got = have;
        return ptr;
    }
    cudaFree(ptr);
    return nullptr;
}
bool spare_release_current() {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return false;
    void* ptr = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_spare_mu);
        auto it = g_spare.find(device);
        if (it == g_spare.end()) return false;
        ptr = it->second.first;
        g_spare.erase(it);
    }
    cudaFree(ptr);
    return true;
}

struct SlabLease {
    clifft_gpu_program& prog;
    StreamBuffers& fallback;
    cudaStream_t stream;
    bool held = false;
    explicit SlabLease(clifft_gpu_program& p, StreamBuffers& b, cudaStream_t s) : prog(p), fallback(b), stream(s) {}
    void* get(size_t bytes) {
        if (bytes == 0) return nullptr;
        if (held && prog.slab_bytes >= bytes) return prog.slab;
        std::lock_guard<std::mutex> lock(prog.slab_mu);
        if (!held && prog.slab_busy) return fallback.alloc(bytes);  // another call holds it
        prog.slab_busy = held = true;
        if (prog.slab_bytes < bytes) {
            CUDA_OK(cudaStreamSynchronize(stream));  // earlier launches of this call may use the old slab
            if (prog.slab) cudaFree(prog.slab);
            prog.slab = nullptr;
            prog.slab_bytes = 0;
            size_t got = 0;
            if (void* sp = spare_take(prog.device, bytes, &got)) {
                prog.slab = sp;
                prog.slab_bytes = got;
            } else {
                CUDA_OK(alloc_retry([&] { return cudaMalloc(&prog.slab, bytes); }));
                prog.slab_bytes = bytes;
            }
        }
        return prog.slab;
    }
    ~SlabLease() {
        if (!held) return;
        cudaStreamSynchronize(stream);  // no launch of this call may still use it
        std::lock_guard<std::mutex> lock(prog.slab_mu);
        prog.slab_busy = false;
    }
};

}  // namespace

namespace {

struct BlobBuilder {
    std::vector<uint8_t> bytes;
    template <typename T>
    size_t put(const T* src, size_t count) {
        size_t off = (bytes.size() + 255) & ~size_t(255);
        bytes.resize(off + count * sizeof(T));
        if (count) std::memcpy(bytes.data() + off, src, count * sizeof(T));
        return off;
    }
};

template <typename T>
const T* at(void* base, size_t off) {
    return reinterpret_cast<const T*>(static_cast<uint8_t*>(base) + off);
}

// launch planning ---------------------------------------------------------
struct LaunchPlan {
    KernelFn fn;
    int G;             // lanes per shot (1..32), 0 = one CTA per shot
    int S;             // shots per warp region (1 for CTA groups)
    int threads;       // block size
    int regions;       // warp regions (or 1 CTA region) per block
    int blocks;
    size_t smem;
    bool state_in_smem;
    uint64_t state_stride;
    uint32_t nw_words;
    bool tiles;       // statevector passes stream through the bulk-copy tile engine
    bool fuse;        // ... and consecutive opcodes fuse into one pass
    uint32_t stages;  // tile buffers per CTA (2 / 3 let three 128-thread / two 256-thread CTAs share an SM)
    bool dense;       // the kernel instance with tensor-core dense blocks (FP32, CTA groups, three stages)
};

uint32_t nw_template(uint32_t nw) { return nw <= 1 ? 1 : 4; }

// CTA sizes (group_threads) of the warp-specialised CTA group: 256 or 512
// threads compute on tiles, one more warp issues every bulk copy of a fused
// block. The kernel instance fits in 96 registers, so two 288-thread CTAs
// share an SM.
constexpr uint32_t kWsThreads = 544, kWsThreadsHalf = 288;
bool ws_shape(uint32_t threads) { return threads == kWsThreads || threads == kWsThreadsHalf; }

// Shared-memory scratch of the tile engine for one shot group.
// dense: with the B operand of the tensor-core dense blocks (FP32 CTA groups
// with three stages only)
uint32_t tile_scratch_bytes(uint32_t precision, bool cta, uint32_t stages, bool dense = false) {
    if (precision == CLIFFT_GPU_FP32)
        return cta ? TileCfg<float, true>::smem_bytes(stages, dense) : TileCfg<float, false>::smem_bytes(stages);
    return cta ? TileCfg<double, true>::smem_bytes(stages) : TileCfg<double, false>::smem_bytes(stages);
}

// Shot-group width for one warp: about 32 amplitudes per lane, so each warp
// carries 32 / G shots whose statevectors interleave in 8 KiB (FP32) /
// 16 KiB (FP64) of shared memory.
int default_group(uint32_t peak) {
    uint64_t amps = uint64_t(1) << peak;
    int g = 1;
    while (g < 32 && uint64_t(g) * 32 < amps) g <<= 1;
    return g;
}

// Everything of a plan except the grid size, which depends on the shot count
// and (for global statevectors) on the free device memory at call time.
struct PlanShape {
    LaunchPlan L;
    int per_sm;
    int sms;
};

PlanShape plan_shape(const clifft_gpu_program& p, uint32_t precision, uint32_t group_req, uint32_t rec_words,
                     uint32_t det_words, uint32_t obs_words, bool allow_fusion, bool dense) {
    LaunchPlan L{};
    const size_t amp = precision == CLIFFT_GPU_FP32 ? 8 : 16;
    const uint64_t stride = uint64_t(1) << p.meta.peak_rank;
    const size_t state_bytes = stride * amp;
    int dev = 0;
    CUDA_OK(cudaGetDevice(&dev));
    int smem_optin = 0, sms = 0;
    CUDA_OK(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t smem_cap = size_t(smem_optin) - 1024;
    const size_t rec_bytes1 = size_t(rec_words + det_words + obs_words) * 4;

    // group_req: 0 = heuristic; 1..32 = lanes per shot; 64..1024 = CTA of that size
    int G;
    if (group_req >= 1 && group_req <= 32)
        G = int(group_req);
    else if (group_req > 32)
        G = 0;
    else
        G = (state_bytes <= 16384) ? default_group(p.meta.peak_rank) : (state_bytes <= (size_t(1) << 20) ? 32 : 0);
    if (G != 0 && (G & (G - 1))) invalid("group_threads below 32 must be a power of two");
    L.G = G;
    L.S = G ? 32 / G : 1;
    L.nw_words = nw_template(p.meta.num_words);
    // a CTA of 288 / 544 threads: 256 / 512 compute threads and one warp
    // that only moves the fused blocks' tiles (the warp-specialised kernel
    // instance, G = -1); the size is settled below for automatic requests
    auto pick_fn = [&](int kg) {
        L.fn = precision == CLIFFT_GPU_FP32 ? kernel_f32(kg, int(L.nw_words)) : kernel_f64(kg, int(L.nw_words));
        cudaFuncAttributes fa{};
        CUDA_OK(cudaFuncGetAttributes(&fa, (const void*)L.fn));
        return std::max(32, (fa.maxThreadsPerBlock / 32) * 32);
    };
    int max_threads = pick_fn(G);
    // one-shot groups (a CTA, or a warp of 32 lanes) stream global
    // statevectors through the tile engine: two 4 KiB buffers per warp keep
    // sixteen warps per SM (three buffers, twelve warps: 10 % slower at k = 14..17)
    L.stages = G == 32 ? 2 : 0;
    auto region_bytes = [&](bool in_smem) {
        size_t fuse = 0;  // tile-engine scratch of the group
        if ((G == 0 || G == 32) && !in_smem)
            fuse = tile_scratch_bytes(precision, G == 0, L.stages, dense && allow_fusion);
        return ((in_smem ? state_bytes * L.S : 0) + ((rec_bytes1 * L.S + 15) & ~size_t(15)) + fuse + 15) &
               ~size_t(15);
    };
    // block tail: reduction scratch for up to 32 warps, broadcast slot, control state
    auto tail = [&](int threads) { (void)threads; return size_t(3 * 8 * 32 + 64 + kCtlBytes); };
    if (G) {
        L.threads = std::min(128, max_threads);
        L.regions = L.threads / 32;
        // shared-memory statevectors only while at least 8 warps fit on an SM;
        // larger ones run from global memory (L2 / HBM) with full occupancy
        int smem_sm = 0;
        CUDA_OK(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
        L.state_in_smem = region_bytes(true) + tail(32) <= smem_cap && region_bytes(true) * 8 <= size_t(smem_sm);
        while (L.regions > 1 && region_bytes(L.state_in_smem) * L.regions + tail(L.threads) > smem_cap) {
            L.regions /= 2;
            L.threads = L.regions * 32;
        }
    } else {
        // default: 128 threads (three CTAs with two tile buffers each share an
        // SM) up to 8 MiB statevectors, else two CTAs with three buffers each:
        // 256 compute threads plus a copy warp when blocks fuse (k = 24: 98 vs
        // 107 ms), 256 threads without fusion
        int t = group_req > 32 ? int(group_req)
                               : (state_bytes <= (size_t(8) << 20) ? 128 : (allow_fusion ? int(kWsThreadsHalf) : 256));
        if (ws_shape(uint32_t(t))) max_threads = pick_fn(-1);
        L.threads = std::min(t, max_threads);
        L.regions = 1;
        L.stages = L.threads <= 128 ? 2 : (L.threads <= 256 || L.threads == int(kWsThreadsHalf) ? 3 : 4);
        L.state_in_smem = region_bytes(true) + tail(L.threads) <= smem_cap;
    }
    L.tiles = (G == 0 || G == 32) && !L.state_in_smem;
    if (!L.tiles) L.stages = 0;
    L.fuse = L.tiles && allow_fusion;
    // dense blocks: only in their own kernel instance (the others hold no
    // tcgen05 instruction), for FP32 CTA groups of 256 compute threads
    L.dense = dense && L.fuse && G == 0 && precision == CLIFFT_GPU_FP32 && L.stages == 3;
    if (L.dense) L.fn = kernel_f32(ws_shape(uint32_t(L.threads)) ? -1 : 0, int(L.nw_words), true);
    L.smem = region_bytes(L.state_in_smem) * L.regions + tail(L.threads);
    if (L.smem > smem_cap) invalid("measurement record too large for shared memory");
    {
        // only ever raised: launches planned earlier (a captured batch graph,
        // another host thread) keep a valid limit
        static std::mutex attr_mu;
        std::lock_guard<std::mutex> lock(attr_mu);
        cudaFuncAttributes cur{};
        CUDA_OK(cudaFuncGetAttributes(&cur, (const void*)L.fn));
        if (cur.maxDynamicSharedSizeBytes < int(L.smem))
            CUDA_OK(cudaFuncSetAttribute((const void*)L.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(L.smem)));
    }
    int per_sm = 0;
    CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)L.fn, L.threads, L.smem));
    if (per_sm < 1) invalid("kernel does not fit on an SM with this launch shape");
    L.state_stride = stride;
    return PlanShape{L, per_sm, sms};
}

static_assert(std::is_trivially_copyable<PlanShape>::value, "plan shapes are cached as bytes");

// Per host thread and device: the event pair that times a call's kernel.
struct CallEvents {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
};
CallEvents& call_events(int dev) {
    thread_local std::map<int, CallEvents> ev;
    CallEvents& c = ev[dev];
    if (!c.e0) {
        CUDA_OK(cudaEventCreate(&c.e0));
        CUDA_OK(cudaEventCreate(&c.e1));
    }
    return c;
}

// Calls allocate their scratch and staged records stream-ordered; the
// device's default pool keeps up to 1 GiB of freed memory instead of
// returning it at every synchronisation, so small repeated calls do not
// remap memory each time. Set once per device (never lowered).
void keep_pool_memory(int dev) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return;
    done.push_back(dev);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    uint64_t thr = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr) == cudaSuccess && thr < (1ull << 30)) {
        thr = 1ull << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
}

// The launch plan of one call. Shapes are planned once per (precision,
// group request, fusion, record widths) and program, so repeated calls skip
// the device queries; the grid is sized per call.
LaunchPlan plan_launch(const clifft_gpu_program& p, uint32_t precision, uint32_t group_req,
                       uint64_t shots, uint32_t rec_words, uint32_t det_words, uint32_t obs_words,
                       bool allow_fusion, uint32_t max_resident = 0, bool dense = false) {
    const auto key = std::make_tuple(precision, group_req, allow_fusion, rec_words, det_words, obs_words, dense);
    PlanShape ps;
    {
        std::lock_guard<std::mutex> lock(p.plan_mu);
        auto it = p.plan_cache.find(key);
        if (it != p.plan_cache.end()) {
            std::memcpy(&ps, it->second.data(), sizeof(PlanShape));
        } else {
            ps = plan_shape(p, precision, group_req, rec_words, det_words, obs_words, allow_fusion, dense);
            std::vector<uint8_t> blob(sizeof(PlanShape));
            std::memcpy(blob.data(), &ps, sizeof(PlanShape));
            p.plan_cache.emplace(key, std::move(blob));
        }
    }
    LaunchPlan L = ps.L;
    const int per_sm = ps.per_sm, sms = ps.sms;
    const uint64_t stride = L.state_stride;
    const size_t state_bytes = stride * (precision == CLIFFT_GPU_FP32 ? 8 : 16);
    const uint64_t shots_per_block = uint64_t(L.regions) * L.S;
    const uint64_t blocks_needed = (shots + shots_per_block - 1) / shots_per_block;
    uint64_t blocks = uint64_t(per_sm) * sms;
    if (!L.state_in_smem) {
        // global slabs: bound the resident state to ~half of free HBM
        size_t free_b = 0, total_b = 0;
        CUDA_OK(cudaMemGetInfo(&free_b, &total_b));
        uint64_t per_block_bytes = uint64_t(state_bytes) * shots_per_block;
        uint64_t max_blocks = std::max<uint64_t>(1, (free_b / 2) / std::max<uint64_t>(per_block_bytes, 1));
        blocks = std::min<uint64_t>(blocks, max_blocks);
    }
    if (max_resident) blocks = std::min<uint64_t>(blocks, std::max<uint64_t>(1, max_resident / shots_per_block));
    blocks = std::max<uint64_t>(1, std::min<uint64_t>(blocks, blocks_needed));
    L.blocks = int(blocks);
    return L;
}

// Launch shapes the autotuner tries (group_threads encoding): sub-warp groups
// around the heuristic width for shared-memory statevectors, warp or CTA
// groups for L2/HBM-resident ones up to 4 MiB, and for larger statevectors
// CTAs of 128 (two tile buffers, three CTAs per SM), 256 (three buffers, two
// per SM), 512 threads (four buffers) or 256 / 512 + a copy warp (three /
// four buffers, warp-specialised fused blocks). Up to 16 MiB a warp per shot
// is tried too: with thousands of shots resident (16 warps per SM) it beats
// every CTA shape (2368 shots: k = 20 715 vs 986 ms, k = 21 1353 vs 1797 ms),
// with fewer it loses (k = 20, 1184 shots: 563 vs 486 ms); from k = 22 on it
// loses at any count (k = 22: 4486 vs 3663 ms; k = 24: 789 vs 3074 shots/s).
// The trial runs on the call's own shots decide.
std::vector<uint32_t> tune_candidates(const clifft_gpu_program& p, uint32_t precision) {
    const size_t amp = precision == CLIFFT_GPU_FP32 ? 8 : 16;
    const size_t state_bytes = (size_t(1) << p.meta.peak_rank) * amp;
    std::vector<uint32_t> c;
    if (state_bytes <= 16384) {
        const int g = default_group(p.meta.peak_rank);
        for (int x : {g / 2, g, g * 2})
            if (x >= 1 && x <= 32) c.push_back(uint32_t(x));
    } else if (state_bytes <= (size_t(4) << 20)) {
        c = {32, 16, 64, 128, 256};
    } else if (state_bytes <= (size_t(16) << 20)) {
        c = {32, 128, 256, 512, kWsThreadsHalf, kWsThreads};
    } else {
        c = {128, 256, 512, kWsThreadsHalf, kWsThreads};
    }
    return c;
}

constexpr uint64_t kTuneMinShots = 1024;
constexpr uint32_t kSegHeaderBytes = 192;  // saved-state header of a shot between segments (svm_kernel.cuh)
constexpr uint32_t kMaxSegments = 8;

// Instruction cuts [0, c1, ..., n] for segmented survivor runs: each inner
// cut follows a POSTSELECT, at about equal numbers of POSTSELECTs per
// segment. Fewer than two POSTSELECTs give no inner cut.
std::vector<uint32_t> segment_cuts(const clifft_gpu_program& p) {
    std::vector<uint32_t> post;
    const uint32_t n = p.meta.num_instructions;
    for (uint32_t i = 0; i < n; ++i)
        if (p.instr_host[size_t(i) * 32] == CLIFFT_OP_POSTSELECT) post.push_back(i);
    std::vector<uint32_t> cuts{0};
    const uint32_t m = std::min<uint32_t>(kMaxSegments, uint32_t(post.size()));
    for (uint32_t j = 1; j < m; ++j) {
        const uint32_t c = post[size_t(j) * post.size() / m - 1] + 1;
        if (c > cuts.back() && c < n) cuts.push_back(c);
    }
    cuts.push_back(n);
    return cuts;
}

// Launch shapes picked by the autotuner, shared by every handle of the same
// program content in this process: (content hash, device, precision/mode).
std::mutex g_tune_mu;
std::map<std::tuple<uint64_t, int, uint32_t>, uint32_t> g_tuned;

uint64_t fnv1a(const uint8_t* p, size_t n, uint64_t h = 1469598103934665603ull) {
    for (size_t i = 0; i < n; ++i) h = (h ^ p[i]) * 1099511628211ull;
    return h;
}

// Least CUDA-core weight (U4 4, U2 2, any other micro-op 1) of a run that the
// dense-block path puts on the tensor cores: CLIFFT_GPU_DENSE_MIN_WEIGHT, else
// the default below.
uint32_t dense_min_weight() {
    static const uint32_t w = [] {
        const char* e = std::getenv("CLIFFT_GPU_DENSE_MIN_WEIGHT");
        const long v = e ? std::strtol(e, nullptr, 10) : 0;
        return v > 0 ? (uint32_t)v : 4u;
    }();
    return w;
}

// Persisted tuning results: with CLIFFT_GPU_TUNE_CACHE naming a file, every
// tuned shape is appended as "program-hash device-signature mode group" and
// earlier lines are consulted before timing trials. The device signature is
// the device name and SM count, so a cache file may travel between machines
// with the same GPU model.
std::map<std::tuple<uint64_t, uint64_t, uint32_t>, uint32_t> g_tune_file;
std::string g_tune_file_path;

uint64_t device_signature(int dev) {
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return fnv1a(reinterpret_cast<const uint8_t*>(prop.name), std::strlen(prop.name)) ^
           (uint64_t(prop.multiProcessorCount) << 48);
}

// caller holds g_tune_mu
bool tune_file_lookup(uint64_t hash, int dev, uint32_t key, uint32_t& group) {
    const char* path = std::getenv("CLIFFT_GPU_TUNE_CACHE");
    if (!path || !*path) return false;
    if (g_tune_file_path != path) {
        g_tune_file.clear();
        g_tune_file_path = path;
        if (FILE* f = std::fopen(path, "r")) {
            unsigned long long h = 0, sig = 0;
            unsigned m = 0, g = 0;
            while (std::fscanf(f, "%llx %llx %u %u", &h, &sig, &m, &g) == 4) g_tune_file[{h, sig, m}] = g;
            std::fclose(f);
        }
    }
    auto it = g_tune_file.find({hash, device_signature(dev), key});
    if (it == g_tune_file.end()) return false;
    group = it->second;
    return true;
}

// caller holds g_tune_mu
void tune_file_store(uint64_t hash, int dev, uint32_t key, uint32_t group) {
    const char* path = std::getenv("CLIFFT_GPU_TUNE_CACHE");
    if (!path || !*path) return;
    const uint64_t sig = device_signature(dev);
    if (FILE* f = std::fopen(path, "a")) {
        std::fprintf(f, "%016llx %016llx %u %u\n", (unsigned long long)hash, (unsigned long long)sig, key, group);
        std::fclose(f);
    }
    if (g_tune_file_path == path) g_tune_file[{hash, sig, key}] = group;
}

}  // namespace

extern "C" {

const char* clifft_gpu_last_error(void) { return g_last_error.c_str(); }

const char* clifft_gpu_backend_name(void) {
    static thread_local std::string name;
    int dev = 0;
    cudaDeviceProp prop{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        name = "unavailable:no CUDA device";
        return name.c_str();
    }
    if (prop.major != 10) {
        name = std::string("unavailable:sm_") + std::to_string(prop.major) + std::to_string(prop.minor) +
               " (this build targets sm_100a)";
        return name.c_str();
    }
    name = std::string("cuda:sm_100a:") + prop.name;
    return name.c_str();
}

int clifft_gpu_load(const clifft_program_image* image, clifft_gpu_program** out) {
    return guarded([&] {
        if (!image || !out) invalid("null argument");
        *out = nullptr;
        const clifft_program_image& im = *image;
        uint32_t peak = validate(im);
        (void)peak;
        auto p = std::make_unique<clifft_gpu_program>();
        p->meta = im;
        const uint32_t nw = std::max<uint32_t>(im.num_words, 1);
        const uint32_t nwt = nw_template(nw);
        // masks are widened to the kernel's template width (zero words above num_words)
        auto widen = [&](const uint64_t* src, uint32_t count) {
            std::vector<uint64_t> w(size_t(count) * nwt, 0);
            for (uint32_t i = 0; i < count; ++i)
                for (uint32_t j = 0; j < im.num_words; ++j) w[size_t(i) * nwt + j] = src[size_t(i) * im.num_words + j];
            return w;
        };
        std::vector<double> psum(im.num_noise_sites);
        for (uint32_t s = 0; s < im.num_noise_sites; ++s) {
            double acc = 0.0;  // same summation order as exec_noise (svm_kernels.inl:1898-1901)
            for (uint32_t c = im.noise_site_offsets[s]; c < im.noise_site_offsets[s + 1]; ++c)
                acc += im.noise_channel_prob[c];
            psum[s] = acc;
        }
        BlobBuilder b;
        size_t o_instr = b.put(im.instructions, size_t(im.num_instructions) * 32);
        auto px = widen(im.pauli_x, im.num_pauli_masks), pz = widen(im.pauli_z, im.num_pauli_masks);
        auto ex = widen(im.exp_val_x, im.num_exp_val_masks), ez = widen(im.exp_val_z, im.num_exp_val_masks);
        auto cx = widen(im.noise_channel_x, im.num_noise_channels);
        auto cz = widen(im.noise_channel_z, im.num_noise_channels);
        size_t o_px = b.put(px.data(), px.size()), o_pz = b.put(pz.data(), pz.size());
        size_t o_ps = b.put(im.pauli_sign, im.num_pauli_masks);
        size_t o_ex = b.put(ex.data(), ex.size()), o_ez = b.put(ez.data(), ez.size());
        size_t o_es = b.put(im.exp_val_sign, im.num_exp_val_masks);
        std::vector<uint32_t> site_off(im.noise_site_offsets, im.noise_site_offsets + im.num_noise_sites + 1);
        if (im.num_noise_sites == 0) site_off.assign(1, 0);
        size_t o_so = b.put(site_off.data(), site_off.size());
        size_t o_psum = b.put(psum.data(), psum.size());
        size_t o_cp = b.put(im.noise_channel_prob, im.num_noise_channels);
        size_t o_cx = b.put(cx.data(), cx.size()), o_cz = b.put(cz.data(), cz.size());
        size_t o_hz = b.put(im.noise_hazards, im.num_noise_sites);
        size_t o_rm = b.put(im.readout_meas_idx, im.num_readout_noise);
        size_t o_rp = b.put(im.readout_prob, im.num_readout_noise);
        std::vector<uint32_t> det_off(im.detector_offsets, im.detector_offsets + im.num_detector_lists + 1);
        std::vector<uint32_t> obs_off(im.observable_offsets, im.observable_offsets + im.num_observable_lists + 1);
        if (im.num_detector_lists == 0) det_off.assign(1, 0);
        if (im.num_observable_lists == 0) obs_off.assign(1, 0);
        size_t o_do = b.put(det_off.data(), det_off.size());
        size_t o_dt = b.put(im.detector_targets, det_off.back());
        size_t o_oo = b.put(obs_off.data(), obs_off.size());
        size_t o_ot = b.put(im.observable_targets, obs_off.back());
        size_t o_u2 = b.put(im.u2_data, size_t(im.num_u2) * CLIFFT_U2_DOUBLES_PER_NODE);
        size_t o_u2o = b.put(im.u2_out, size_t(im.num_u2) * 4);
        size_t o_u4 = b.put(im.u4_data, size_t(im.num_u4) * CLIFFT_U4_DOUBLES_PER_NODE);
        size_t o_u4o = b.put(im.u4_out, size_t(im.num_u4) * 16);
        p->expected_host.assign(im.expected_observables, im.expected_observables + im.num_expected_observables);
        size_t o_exo = b.put(p->expected_host.data(), p->expected_host.size());
        b.bytes.resize(b.bytes.size() + 256);
        CUDA_OK(cudaGetDevice(&p->device));
        {
            const uint32_t counts[] = {im.peak_rank, im.num_measurements, im.total_meas_slots, im.num_detectors,
                                       im.num_observables, im.num_exp_vals, im.num_words, im.num_instructions};
            p->content_hash = fnv1a(reinterpret_cast<const uint8_t*>(counts), sizeof(counts),
                                    fnv1a(b.bytes.data(), b.bytes.size()));
        }
        p->fault_probs.assign(psum.begin(), psum.end());
        for (uint32_t r = 0; r < im.num_readout_noise; ++r) p->fault_probs.push_back(im.readout_prob[r]);
        p->instr_host.assign(static_cast<const uint8_t*>(im.instructions),
                             static_cast<const uint8_t*>(im.instructions) + size_t(im.num_instructions) * 32);
        for (uint32_t i = 0; i < im.num_instructions; ++i) {
            const uint8_t op = p->instr_host[size_t(i) * 32];
            if (op == CLIFFT_OP_ARRAY_ROT || op == CLIFFT_OP_EXPAND_ROT) ++p->num_rot_params;
        }
        CUDA_OK(alloc_retry([&] { return cudaMalloc(&p->blob, b.bytes.size()); }));
        p->blob_bytes = b.bytes.size();
        CUDA_OK(cudaMemcpy(p->blob, b.bytes.data(), b.bytes.size(), cudaMemcpyHostToDevice));
        DevProg& d = p->dev;
        void* B = p->blob;
        d.instr = at<uint4>(B, o_instr);
        d.n_instr = im.num_instructions;
        d.nw = nwt;
        d.peak = im.peak_rank;
        d.num_meas = im.num_measurements;
        d.slots = im.total_meas_slots;
        d.num_det = im.num_detectors;
        d.num_obs = im.num_observables;
        d.num_exp = im.num_exp_vals;
        d.pauli_x = at<uint64_t>(B, o_px);
        d.pauli_z = at<uint64_t>(B, o_pz);
        d.pauli_sign = at<uint8_t>(B, o_ps);
        d.exp_x = at<uint64_t>(B, o_ex);
        d.exp_z = at<uint64_t>(B, o_ez);
        d.exp_sign = at<uint8_t>(B, o_es);
        d.n_sites = im.num_noise_sites;
        d.site_off = at<uint32_t>(B, o_so);
        d.site_psum = at<double>(B, o_psum);
        d.chan_prob = at<double>(B, o_cp);
        d.chan_x = at<uint64_t>(B, o_cx);
        d.chan_z = at<uint64_t>(B, o_cz);
        d.hazards = at<double>(B, o_hz);
        d.ro_meas = at<uint32_t>(B, o_rm);
        d.ro_prob = at<double>(B, o_rp);
        d.det_off = at<uint32_t>(B, o_do);
        d.det_tg = at<uint32_t>(B, o_dt);
        d.obs_off = at<uint32_t>(B, o_oo);
        d.obs_tg = at<uint32_t>(B, o_ot);
        d.u2 = at<double>(B, o_u2);
        d.u2_out = at<uint8_t>(B, o_u2o);
        d.u4 = at<double>(B, o_u4);
        d.u4_out = at<uint8_t>(B, o_u4o);
        d.n_expected = im.num_expected_observables;
        d.expected = at<uint8_t>(B, o_exo);
        // drop host pointers from the retained metadata
        clifft_program_image& m = p->meta;
        m.instructions = nullptr;
        m.pauli_x = m.pauli_z = m.exp_val_x = m.exp_val_z = m.noise_channel_x = m.noise_channel_z = nullptr;
        m.pauli_sign = m.exp_val_sign = m.u2_out = m.u4_out = m.expected_observables = nullptr;
        m.noise_site_offsets = m.readout_meas_idx = m.detector_offsets = m.detector_targets = nullptr;
        m.observable_offsets = m.observable_targets = nullptr;
        m.noise_channel_prob = m.noise_hazards = m.readout_prob = m.u2_data = m.u4_data = nullptr;
        *out = p.release();
    });
}

void clifft_gpu_free(clifft_gpu_program* prog) {
    if (!prog) return;
    if (prog->blob || prog->slab) {
        cudaDeviceSynchronize();
        if (prog->blob) cudaFree(prog->blob);
        if (prog->slab) cudaFree(prog->slab);
    }
    delete prog;
}

void clifft_gpu_trim(void) {
    std::map<int, std::pair<void*, size_t>> all;
    {
        std::lock_guard<std::mutex> lock(g_spare_mu);
        all.swap(g_spare);
    }
    for (auto& kv : all) cudaFree(kv.second.first);
}

uint32_t clifft_gpu_program_peak_rank(const clifft_gpu_program* prog) { return prog ? prog->meta.peak_rank : 0; }
uint64_t clifft_gpu_program_device_bytes(const clifft_gpu_program* prog) { return prog ? prog->blob_bytes : 0; }

}  // extern "C"

namespace {

// Device-resident per-shot fault lists prepared by the library itself
// (sample_k): begin offsets in args->fault_offsets / readout_offsets, end
// offsets here, every array a device pointer whatever args->flags says.
struct DeviceFaults {
    const uint32_t* fault_end = nullptr;
    const uint32_t* ro_end = nullptr;
};

// Message for the first device-side error code a launch recorded; `info`
// points at the launch's eight words of timeout diagnostics.
std::string device_error_message(int dev_err, const unsigned long long* info) {
    std::string msg = dev_err == DEV_ERR_ZERO_NORM    ? "active measurement on a zero-norm state"
                      : dev_err == DEV_ERR_TIMEOUT    ? "a bounded wait on a bulk-copy barrier timed out"
                      : dev_err == DEV_ERR_BAD_OPCODE ? "device reported an invalid opcode"
                                                      : "unknown device error " + std::to_string(dev_err);
    if (dev_err == DEV_ERR_TIMEOUT) {
        const unsigned long long* e = info;
        msg += " (pass " + std::to_string(e[0]) + ", instruction " + std::to_string(e[1]) + ", tile " +
               std::to_string(e[2]) + "/" + std::to_string(e[3]) + ", run log2 " + std::to_string(e[4]) + ", k " +
               std::to_string(e[5]) + ", barrier word " + std::to_string(e[6]) + ", waited " +
               std::to_string(e[7]) + " cycles)";
    }
    return msg;
}

// clifft_gpu_sample; `dfaults` non-null when the forced-fault lists live on
// the device (the outputs follow args->flags as usual).
void sample_impl(clifft_gpu_program* prog, const clifft_gpu_sample_args* args, clifft_gpu_outputs* out,
                 const DeviceFaults* dfaults) {
        if (!prog || !args || !out) invalid("null argument");
        const clifft_program_image& m = prog->meta;
        const uint64_t shots = args->shots;
        if (args->precision != CLIFFT_GPU_FP32 && args->precision != CLIFFT_GPU_FP64)
            invalid("precision must be CLIFFT_GPU_FP32 or CLIFFT_GPU_FP64");
        const uint32_t gt = args->group_threads;
        if (gt != 0 && !(gt <= 32 && (gt & (gt - 1)) == 0) && (gt % 32 != 0 || gt > 1024))
            invalid("group_threads must be 0, a power of two up to 32, or a multiple of 32 up to 1024");
        const bool dev_ptrs = (args->flags & CLIFFT_GPU_DEVICE_PTRS) != 0;
        const bool forced_meas = (args->flags & CLIFFT_GPU_FORCED_MEAS) != 0;
        const bool forced_faults = (args->flags & CLIFFT_GPU_FORCED_FAULTS) != 0;
        if (forced_meas && !args->forced_meas && m.total_meas_slots > 0)
            invalid("CLIFFT_GPU_FORCED_MEAS needs forced_meas");
        if (forced_faults && (!args->fault_offsets || !args->readout_offsets))
            invalid("CLIFFT_GPU_FORCED_FAULTS needs fault_offsets and readout_offsets");
        out->passed_shots = 0;
        out->logical_errors = 0;
        out->dust_clamps = 0;
        out->algorithmic_bytes = 0;
        out->streamed_bytes = 0;
        out->kernel_launches = 0;
        out->kernel_ms = 0.f;
        if (shots == 0) return;
        CUDA_OK(cudaSetDevice(prog->device));
        keep_pool_memory(prog->device);
        cudaStream_t st = static_cast<cudaStream_t>(args->stream);
        StreamBuffers buf(st);
        SlabLease slab(*prog, buf, st);

        // host-side validation of forced-fault inputs (bounds only)
        std::vector<uint32_t> h_foff, h_roff;
        if (forced_faults && !dev_ptrs && !dfaults) {
            for (uint64_t s = 0; s < shots; ++s) {
                if (args->fault_offsets[s] > args->fault_offsets[s + 1] ||
                    args->readout_offsets[s] > args->readout_offsets[s + 1])
                    invalid("forced-fault offsets must be non-decreasing");
                for (uint32_t f = args->fault_offsets[s]; f < args->fault_offsets[s + 1]; ++f) {
                    if (args->fault_sites[f] >= m.num_noise_sites) invalid("forced fault site out of range");
                    if (f > args->fault_offsets[s] && args->fault_sites[f] <= args->fault_sites[f - 1])
                        invalid("forced fault sites must be strictly ascending per shot");
                }
            }
        }

        const uint32_t rec_words = (m.total_meas_slots + 31) / 32;
        const uint32_t det_words = (m.num_detectors + 31) / 32;
        const uint32_t obs_words = (m.num_observables + 31) / 32;
        const bool allow_fusion = (args->flags & CLIFFT_GPU_NO_FUSION) == 0;
        // autotuned launch shape (group_threads == 0)
        const uint32_t tune_key = args->precision | (allow_fusion ? 2u : 0u) |
                                  (args->flags & CLIFFT_GPU_SURVIVORS ? 4u : 0u) | (forced_meas ? 8u : 0u) |
                                  (forced_faults ? 16u : 0u) | (args->flags & CLIFFT_GPU_TRACE ? 32u : 0u);
        uint32_t group_req = args->group_threads;
        std::vector<uint32_t> tune;
        const auto tune_id = std::make_tuple(prog->content_hash, prog->device, tune_key);
        if (group_req == 0 && !(args->flags & CLIFFT_GPU_NO_AUTOTUNE)) {
            std::lock_guard<std::mutex> lock(g_tune_mu);
            auto it = g_tuned.find(tune_id);
            uint32_t from_file = 0;
            if (it != g_tuned.end()) {
                group_req = it->second;
            } else if (tune_file_lookup(prog->content_hash, prog->device, tune_key, from_file)) {
                g_tuned[tune_id] = from_file;
                group_req = from_file;
            } else if (shots >= kTuneMinShots) {
                tune = tune_candidates(*prog, args->precision);
            }
        }
        const bool want_dense = (args->flags & CLIFFT_GPU_TENSOR_DENSE) && args->precision == CLIFFT_GPU_FP32;
        LaunchPlan L = plan_launch(*prog, args->precision, group_req, shots, rec_words, det_words, obs_words,
                                   allow_fusion, args->max_resident, want_dense);
        KParams K{};
        K.shots = shots;
        K.first_shot = args->first_shot;
        K.seed = args->seed;
        K.dust_eps = args->dust_eps > 0.0 ? args->dust_eps : (args->precision == CLIFFT_GPU_FP32 ? 1e-9 : 1e-18);
        K.flags = (args->flags & CLIFFT_GPU_SURVIVORS ? KF_SURVIVORS : 0) |
                  (forced_meas ? KF_FORCED_MEAS : 0) | (forced_faults ? KF_FORCED_FAULTS : 0) |
                  (args->flags & CLIFFT_GPU_TRACE ? KF_TRACE : 0) |
                  (args->flags & CLIFFT_GPU_RAW_PARITY ? KF_RAW_PARITY : 0) |
                  (args->flags & CLIFFT_GPU_TENSOR_DENSE ? KF_DENSE : 0);
        K.rec_words = rec_words;
        K.det_words = det_words;
        K.obs_words = obs_words;
        K.meas_out_words = (m.num_measurements + 63) / 64;
        K.det_out_words = (m.num_detectors + 63) / 64;
        K.obs_out_words = (m.num_observables + 63) / 64;
        const size_t amp = args->precision == CLIFFT_GPU_FP32 ? 8 : 16;
        // launch-shape dependent parameters (and the statevector slab)
        auto apply_plan = [&](KParams& Kx, const LaunchPlan& Lx) {
            Kx.flags = (K.flags & ~uint32_t(KF_FUSE)) | (Lx.fuse ? KF_FUSE : 0);
            // dense blocks on the tensor cores: FP32 CTA groups of 256 compute
            // threads (three tile stages) streaming fused blocks; other shapes
            // run the same blocks on the CUDA cores
            const bool dense_ok = Lx.dense;
            if (!dense_ok) Kx.flags &= ~uint32_t(KF_DENSE);
            Kx.fuse_bytes = Lx.tiles ? tile_scratch_bytes(args->precision, Lx.G == 0, Lx.stages, dense_ok) : 0;
            Kx.stages = Lx.stages;
            Kx.state_in_smem = Lx.state_in_smem ? 1 : 0;
            Kx.state_stride = Lx.state_stride;
            Kx.state_global = Lx.state_in_smem
                                  ? nullptr
                                  : slab.get(size_t(Lx.blocks) * Lx.regions * Lx.S * Lx.state_stride * amp);
            Kx.dense_min_weight = dense_min_weight();
        };
        const size_t n_counters = 5 + m.num_observables;
        const bool profile = (args->flags & CLIFFT_GPU_PROFILE) != 0;
        const size_t scratch_words = 2 + n_counters + (profile ? 8 : 0) + 8;
        auto* scratch = static_cast<unsigned long long*>(buf.alloc(scratch_words * 8 + 64));
        CUDA_OK(cudaMemsetAsync(scratch, 0, scratch_words * 8 + 64, st));
        K.phase_cycles = profile ? scratch + 2 + n_counters : nullptr;
        K.error_info = scratch + scratch_words - 8;
        K.work_counter = scratch;
        K.error_word = reinterpret_cast<int*>(scratch + 1);
        K.counters = scratch + 2;

        // inputs
        auto stage_in = [&](const void* src, size_t bytes) -> const void* {
            if (!src || bytes == 0) return nullptr;
            if (dev_ptrs) return src;
            void* d = buf.alloc(bytes);
            CUDA_OK(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, st));
            return d;
        };
        if (forced_meas)
            K.forced_meas = static_cast<const uint8_t*>(stage_in(args->forced_meas, shots * m.total_meas_slots));
        if (forced_faults && dfaults) {
            K.fault_off = args->fault_offsets;
            K.ro_off = args->readout_offsets;
            K.fault_end = dfaults->fault_end;
            K.ro_end = dfaults->ro_end;
            K.fault_sites = args->fault_sites;
            K.fault_chan = args->fault_channels;
            K.ro_entries = args->readout_entries;
        } else if (forced_faults) {
            uint64_t nf = dev_ptrs ? 0 : args->fault_offsets[shots];
            uint64_t nr = dev_ptrs ? 0 : args->readout_offsets[shots];
            K.fault_off = static_cast<const uint32_t*>(stage_in(args->fault_offsets, (shots + 1) * 4));
            K.ro_off = static_cast<const uint32_t*>(stage_in(args->readout_offsets, (shots + 1) * 4));
            if (dev_ptrs) {
                K.fault_sites = args->fault_sites;
                K.fault_chan = args->fault_channels;
                K.ro_entries = args->readout_entries;
            } else {
                K.fault_sites = static_cast<const uint32_t*>(stage_in(args->fault_sites, nf * 4));
                K.fault_chan = static_cast<const uint32_t*>(stage_in(args->fault_channels, nf * 4));
                K.ro_entries = static_cast<const uint32_t*>(stage_in(args->readout_entries, nr * 4));
            }
        }

        // outputs
        struct Out {
            void* host;
            void* dev;
            size_t bytes;
        };
        std::vector<Out> outs;
        auto stage_out = [&](void* host, size_t bytes) -> void* {
            if (!host || bytes == 0) return nullptr;
            if (dev_ptrs) return host;
            void* d = buf.alloc(bytes);
            outs.push_back({host, d, bytes});
            return d;
        };
        K.out_meas = static_cast<uint64_t*>(stage_out(out->meas, shots * K.meas_out_words * 8));
        K.out_det = static_cast<uint64_t*>(stage_out(out->det, shots * K.det_out_words * 8));
        K.out_obs = static_cast<uint64_t*>(stage_out(out->obs, shots * K.obs_out_words * 8));
        K.out_exp = static_cast<double*>(stage_out(out->exp_vals, shots * m.num_exp_vals * 8));
        K.out_survived = static_cast<uint8_t*>(stage_out(out->survived, shots));
        if (args->flags & CLIFFT_GPU_TRACE) {
            K.out_meas_prob = static_cast<double*>(stage_out(out->meas_prob, shots * m.total_meas_slots * 8));
            K.out_log_prob = static_cast<double*>(stage_out(out->log_prob, shots * 8));
            K.out_final_k = static_cast<uint32_t*>(stage_out(out->final_k, shots * 4));
            K.out_final_gamma = static_cast<double*>(stage_out(out->final_gamma, shots * 16));
            // px/pz are written at the kernel's template width; narrow below
            const uint32_t nwt = L.nw_words;
            K.out_final_px = static_cast<uint64_t*>(buf.alloc(out->final_px ? shots * nwt * 8 : 0));
            K.out_final_pz = static_cast<uint64_t*>(buf.alloc(out->final_pz ? shots * nwt * 8 : 0));
            K.dump_shots = std::min<uint64_t>(out->dump_shots, shots);
            K.out_final_v = static_cast<double*>(
                stage_out(out->final_v, K.dump_shots * (uint64_t(1) << m.peak_rank) * 16));
        }

        CallEvents& ce = call_events(prog->device);
        cudaEvent_t e0 = ce.e0, e1 = ce.e1;
        uint32_t launches = 0;
        if (!tune.empty()) {
            // Trial launches on the first shots of this call (their records are
            // rewritten by the real launch below): up to two resident waves per
            // candidate, fastest shots/s wins.
            float best_rate = -1.f;
            uint32_t best = 0;
            for (uint32_t cand : tune) {
                LaunchPlan Lc = plan_launch(*prog, args->precision, cand, shots, rec_words, det_words, obs_words,
                                            allow_fusion, args->max_resident, want_dense);
                const uint64_t wave = uint64_t(Lc.blocks) * Lc.regions * Lc.S;
                const uint64_t trial = std::min<uint64_t>(shots, 2 * wave);
                KParams Kc = K;
                apply_plan(Kc, Lc);
                Kc.shots = trial;
                auto* sc = static_cast<unsigned long long*>(buf.alloc(scratch_words * 8 + 64));
                CUDA_OK(cudaMemsetAsync(sc, 0, scratch_words * 8 + 64, st));
                Kc.work_counter = sc;
                Kc.error_word = reinterpret_cast<int*>(sc + 1);
                Kc.counters = sc + 2;
                Kc.phase_cycles = nullptr;
                Kc.error_info = sc + scratch_words - 8;
                CUDA_OK(cudaEventRecord(e0, st));
                Lc.fn<<<Lc.blocks, Lc.threads, Lc.smem, st>>>(prog->dev, Kc);
                CUDA_OK(cudaGetLastError());
                CUDA_OK(cudaEventRecord(e1, st));
                CUDA_OK(cudaEventSynchronize(e1));
                ++launches;
                float tms = 0.f;
                CUDA_OK(cudaEventElapsedTime(&tms, e0, e1));
                const float rate = float(trial) / std::max(tms, 1e-6f);
                if (rate > best_rate) {
                    best_rate = rate;
                    best = cand;
                }
            }
            {
                std::lock_guard<std::mutex> lock(g_tune_mu);
                g_tuned[tune_id] = best;
                tune_file_store(prog->content_hash, prog->device, tune_key, best);
            }
            L = plan_launch(*prog, args->precision, best, shots, rec_words, det_words, obs_words, allow_fusion,
                            args->max_resident, want_dense);
        }
        apply_plan(K, L);
        // Survivor runs of warp groups go segment by segment: the program is cut
        // after POSTSELECT opcodes, and only the shots still alive at a cut are
        // carried (state saved, ids compacted) into the next segment, so warps
        // are not left running lanes whose shot was already discarded.
        const std::vector<uint32_t> cuts =
            (args->flags & CLIFFT_GPU_SURVIVORS) && !(args->flags & CLIFFT_GPU_NO_SEGMENTS) && L.G > 0 &&
                    !(args->flags & CLIFFT_GPU_TRACE) && !profile &&
                    shots >= 4 * uint64_t(L.blocks) * L.regions * L.S && shots <= 0xffffffffull
                ? segment_cuts(*prog)
                : std::vector<uint32_t>();
        // segment buffers are set up ahead of the timed region
        const uint32_t nseg = cuts.size() < 3 ? 0u : uint32_t(cuts.size() - 1);
        uint32_t* lists[2] = {nullptr, nullptr};
        unsigned long long* segc = nullptr;
        if (nseg) {
            const uint32_t nwords = rec_words + det_words + obs_words;
            const uint64_t stride = (kSegHeaderBytes + ((nwords * 4u + 15u) & ~15u) +
                                     (uint64_t(1) << m.peak_rank) * amp + 15u) & ~uint64_t(15);
            K.seg_state = static_cast<unsigned char*>(buf.alloc(size_t(shots) * stride));
            K.seg_stride = stride;
            lists[0] = static_cast<uint32_t*>(buf.alloc(size_t(shots) * 4));
            lists[1] = static_cast<uint32_t*>(buf.alloc(size_t(shots) * 4));
            segc = static_cast<unsigned long long*>(buf.alloc(size_t(nseg) * 2 * 8));
            CUDA_OK(cudaMemsetAsync(segc, 0, size_t(nseg) * 2 * 8, st));
        }
        CUDA_OK(cudaEventRecord(e0, st));
        if (!nseg) {
            L.fn<<<L.blocks, L.threads, L.smem, st>>>(prog->dev, K);
            CUDA_OK(cudaGetLastError());
        } else {
            for (uint32_t sgi = 0; sgi < nseg; ++sgi) {
                KParams Ks = K;
                Ks.seg_flags = KSEG_ON | (sgi == 0 ? KSEG_FIRST : 0u) | (sgi + 1 == nseg ? KSEG_LAST : 0u);
                Ks.seg_begin = cuts[sgi];
                Ks.seg_end = cuts[sgi + 1];
                Ks.seg_in = sgi == 0 ? nullptr : lists[(sgi + 1) & 1];
                Ks.seg_count_in = sgi == 0 ? nullptr : segc + (sgi - 1);
                Ks.seg_out = lists[sgi & 1];
                Ks.seg_count_out = segc + sgi;
                if (sgi > 0) Ks.work_counter = segc + nseg + sgi;  // a fresh work counter per launch
                L.fn<<<L.blocks, L.threads, L.smem, st>>>(prog->dev, Ks);
                CUDA_OK(cudaGetLastError());
                ++launches;
            }
            --launches;  // the first segment is the call's regular launch
        }
        CUDA_OK(cudaEventRecord(e1, st));

        for (auto& o : outs) CUDA_OK(cudaMemcpyAsync(o.host, o.dev, o.bytes, cudaMemcpyDeviceToHost, st));
        std::vector<unsigned long long> hs(scratch_words);
        CUDA_OK(cudaMemcpyAsync(hs.data(), scratch, hs.size() * 8, cudaMemcpyDeviceToHost, st));
        std::vector<uint64_t> hpx, hpz;
        const uint32_t nwt = L.nw_words;
        if (K.out_final_px) {
            hpx.resize(shots * nwt);
            CUDA_OK(cudaMemcpyAsync(hpx.data(), K.out_final_px, hpx.size() * 8, cudaMemcpyDeviceToHost, st));
        }
        if (K.out_final_pz) {
            hpz.resize(shots * nwt);
            CUDA_OK(cudaMemcpyAsync(hpz.data(), K.out_final_pz, hpz.size() * 8, cudaMemcpyDeviceToHost, st));
        }
        CUDA_OK(cudaStreamSynchronize(st));
        float ms = 0.f;
        CUDA_OK(cudaEventElapsedTime(&ms, e0, e1));
        const uint32_t nwo = std::max<uint32_t>(m.num_words, 1);
        for (uint64_t s = 0; s < shots && !hpx.empty(); ++s)
            for (uint32_t w = 0; w < nwo; ++w) out->final_px[s * nwo + w] = hpx[s * nwt + w];
        for (uint64_t s = 0; s < shots && !hpz.empty(); ++s)
            for (uint32_t w = 0; w < nwo; ++w) out->final_pz[s * nwo + w] = hpz[s * nwt + w];
        const int dev_err = static_cast<int>(hs[1] & 0xffffffffu);
        if (dev_err != 0) throw ApiError(CLIFFT_GPU_EDEVICE, device_error_message(dev_err, hs.data() + scratch_words - 8));
        out->passed_shots = hs[2];
        out->logical_errors = hs[3];
        out->dust_clamps = hs[4];
        out->algorithmic_bytes = hs[5];
        out->streamed_bytes = hs[6];
        if (out->observable_ones)
            for (uint32_t i = 0; i < m.num_observables; ++i) out->observable_ones[i] = hs[7 + i];
        out->kernel_launches = launches + 1;
        out->kernel_ms = ms;
        out->group_threads = L.G ? uint32_t(L.G) : uint32_t(L.threads);
        out->state_in_smem = L.state_in_smem ? 1u : 0u;
        out->fused = L.fuse ? 1u : 0u;
        for (int i = 0; i < 5; ++i) out->phase_cycles[i] = profile ? hs[2 + n_counters + i] : 0;
}

}  // namespace

extern "C" {

int clifft_gpu_sample(clifft_gpu_program* prog, const clifft_gpu_sample_args* args, clifft_gpu_outputs* out) {
    return guarded([&] { sample_impl(prog, args, out, nullptr); });
}

}  // extern "C"

// ------------------------------------------------------ allocation-free sampling
// clifft_gpu_sample_noalloc keeps its launch scratch (work counter, error
// word, counters, timeout diagnostics) in this module's own device array
// instead of stream-ordered allocations. One array exists per device per
// process, so calls that overlap on one device race on it.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[CLIFFT_GPU_NOALLOC_SCRATCH_WORDS];

namespace {

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_ptr[kNoallocMaxDevices] = {};

// Address of g_noalloc_scratch on `dev` (which must be current), looked up
// once per device.
unsigned long long* noalloc_scratch(int dev) {
    if (dev < 0 || dev >= kNoallocMaxDevices) invalid("device ordinal out of range for the static scratch table");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        CUDA_OK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = static_cast<unsigned long long*>(p);
    }
    return g_noalloc_ptr[dev];
}

}  // namespace

extern "C" {

int clifft_gpu_sample_noalloc(clifft_gpu_program* prog, const clifft_gpu_sample_args* args,
                              clifft_gpu_outputs* out) {
    return guarded([&] {
        if (!prog || !args || !out) invalid("null argument");
        const clifft_program_image& m = prog->meta;
        const uint64_t shots = args->shots;
        if (args->precision != CLIFFT_GPU_FP32 && args->precision != CLIFFT_GPU_FP64)
            invalid("precision must be CLIFFT_GPU_FP32 or CLIFFT_GPU_FP64");
        const uint32_t gt = args->group_threads;
        if (gt != 0 && !(gt <= 32 && (gt & (gt - 1)) == 0) && (gt % 32 != 0 || gt > 1024))
            invalid("group_threads must be 0, a power of two up to 32, or a multiple of 32 up to 1024");
        if (!(args->flags & CLIFFT_GPU_DEVICE_PTRS))
            invalid("clifft_gpu_sample_noalloc needs CLIFFT_GPU_DEVICE_PTRS: every input and output "
                    "buffer must already be in device memory");
        if (args->flags & (CLIFFT_GPU_TRACE | CLIFFT_GPU_PROFILE))
            invalid("clifft_gpu_sample_noalloc does not support CLIFFT_GPU_TRACE or CLIFFT_GPU_PROFILE");
        const bool forced_meas = (args->flags & CLIFFT_GPU_FORCED_MEAS) != 0;
        const bool forced_faults = (args->flags & CLIFFT_GPU_FORCED_FAULTS) != 0;
        if (forced_meas && !args->forced_meas && m.total_meas_slots > 0)
            invalid("CLIFFT_GPU_FORCED_MEAS needs forced_meas");
        if (forced_faults && (!args->fault_offsets || !args->readout_offsets))
            invalid("CLIFFT_GPU_FORCED_FAULTS needs fault_offsets and readout_offsets");
        // scratch layout: work counter, error word, 5 totals, one counter per
        // observable, 8 words of timeout diagnostics
        const size_t n_counters = 5 + size_t(m.num_observables);
        const size_t words = 2 + n_counters + 8;
        if (words > CLIFFT_GPU_NOALLOC_SCRATCH_WORDS)
            invalid("clifft_gpu_sample_noalloc: a program with " + std::to_string(m.num_observables) +
                    " observables needs " + std::to_string(words) + " scratch words; the static scratch holds " +
                    std::to_string(CLIFFT_GPU_NOALLOC_SCRATCH_WORDS) + " (at most " +
                    std::to_string(CLIFFT_GPU_NOALLOC_SCRATCH_WORDS - 15) + " observables)");
        out->passed_shots = 0;
        out->logical_errors = 0;
        out->dust_clamps = 0;
        out->algorithmic_bytes = 0;
        out->streamed_bytes = 0;
        out->kernel_launches = 0;
        out->kernel_ms = 0.f;
        if (shots == 0) return;
        CUDA_OK(cudaSetDevice(prog->device));
        unsigned long long* scratch = noalloc_scratch(prog->device);
        cudaStream_t st = static_cast<cudaStream_t>(args->stream);

        const uint32_t rec_words = (m.total_meas_slots + 31) / 32;
        const uint32_t det_words = (m.num_detectors + 31) / 32;
        const uint32_t obs_words = (m.num_observables + 31) / 32;
        LaunchPlan L = plan_launch(*prog, args->precision, args->group_threads, shots, rec_words, det_words,
                                   obs_words, (args->flags & CLIFFT_GPU_NO_FUSION) == 0);
        if (!L.state_in_smem)
            invalid("clifft_gpu_sample_noalloc: the statevectors of this program (peak rank " +
                    std::to_string(m.peak_rank) +
                    ") do not fit in shared memory with this launch shape, and this entry point has no "
                    "global-memory statevector slab; use clifft_gpu_sample");
        KParams K{};
        K.shots = shots;
        K.first_shot = args->first_shot;
        K.seed = args->seed;
        K.dust_eps = args->dust_eps > 0.0 ? args->dust_eps : (args->precision == CLIFFT_GPU_FP32 ? 1e-9 : 1e-18);
        K.flags = (args->flags & CLIFFT_GPU_SURVIVORS ? KF_SURVIVORS : 0) | (forced_meas ? KF_FORCED_MEAS : 0) |
                  (forced_faults ? KF_FORCED_FAULTS : 0);
        K.fuse_bytes = 0;
        K.rec_words = rec_words;
        K.det_words = det_words;
        K.obs_words = obs_words;
        K.meas_out_words = (m.num_measurements + 63) / 64;
        K.det_out_words = (m.num_detectors + 63) / 64;
        K.obs_out_words = (m.num_observables + 63) / 64;
        K.state_in_smem = 1;
        K.state_stride = L.state_stride;
        K.state_global = nullptr;
        // every scratch word the kernel reads must start at zero: cleared on the
        // call's stream ahead of the launch
        CUDA_OK(cudaMemsetAsync(scratch, 0, words * 8, st));
        K.phase_cycles = nullptr;
        K.work_counter = scratch;
        K.error_word = reinterpret_cast<int*>(scratch + 1);
        K.counters = scratch + 2;
        K.error_info = scratch + words - 8;
        K.forced_meas = forced_meas ? args->forced_meas : nullptr;
        if (forced_faults) {
            K.fault_off = args->fault_offsets;
            K.ro_off = args->readout_offsets;
            K.fault_sites = args->fault_sites;
            K.fault_chan = args->fault_channels;
            K.ro_entries = args->readout_entries;
        }
        K.out_meas = K.meas_out_words ? out->meas : nullptr;
        K.out_det = K.det_out_words ? out->det : nullptr;
        K.out_obs = K.obs_out_words ? out->obs : nullptr;
        K.out_exp = m.num_exp_vals ? out->exp_vals : nullptr;
        K.out_survived = out->survived;

        L.fn<<<L.blocks, L.threads, L.smem, st>>>(prog->dev, K);
        CUDA_OK(cudaGetLastError());
        unsigned long long hs[CLIFFT_GPU_NOALLOC_SCRATCH_WORDS];
        CUDA_OK(cudaMemcpyAsync(hs, scratch, words * 8, cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        const int dev_err = static_cast<int>(hs[1] & 0xffffffffu);
        if (dev_err != 0) throw ApiError(CLIFFT_GPU_EDEVICE, device_error_message(dev_err, hs + words - 8));
        out->passed_shots = hs[2];
        out->logical_errors = hs[3];
        out->dust_clamps = hs[4];
        out->algorithmic_bytes = hs[5];
        out->streamed_bytes = hs[6];
        if (out->observable_ones)
            for (uint32_t i = 0; i < m.num_observables; ++i) out->observable_ones[i] = hs[7 + i];
        out->kernel_launches = 1;
        out->group_threads = L.G ? uint32_t(L.G) : uint32_t(L.threads);
        out->state_in_smem = 1;
        out->fused = 0;
        for (int i = 0; i < 5; ++i) out->phase_cycles[i] = 0;
    });
}

}  // extern "C"

// ---------------------------------------------------- multi-program batches
// A batch is an explicitly built CUDA graph with one (memset scratch ->
// sampling kernel) branch per program and no edges between branches, so one
// graph launch runs programs of different peak rank side by side, each with
// its own launch shape (autotuned by the warm-up call at creation).
struct clifft_gpu_batch {
    struct Item {
        clifft_gpu_program* prog = nullptr;
        clifft_gpu_outputs* out = nullptr;
        LaunchPlan L{};
        KParams K{};
        unsigned long long* scratch = nullptr;  // inside the batch's scratch block
        size_t scratch_words = 0;
        size_t scratch_at = 0;                  // word offset in the block
        void* slab = nullptr;
        cudaGraphNode_t kernel_node{};
        void* kargs[2] = {nullptr, nullptr};
    };
    std::vector<Item> items;
    int device = 0;
    unsigned long long* scratch_block = nullptr;
    size_t scratch_block_words = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<std::pair<KernelFn, size_t>> smem_limits;
};

namespace {

void batch_release(clifft_gpu_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    for (auto& it : b->items)
        if (it.slab) cudaFree(it.slab);
    if (b->scratch_block) cudaFree(b->scratch_block);
    delete b;
}

}  // namespace

extern "C" {

int clifft_gpu_batch_create(clifft_gpu_program* const* progs, const clifft_gpu_sample_args* args,
                            clifft_gpu_outputs* outs, uint32_t n, clifft_gpu_batch** out) {
    clifft_gpu_batch* b = nullptr;
    int rc = guarded([&] {
        if (!progs || !args || !outs || !out || n == 0) invalid("null argument or empty batch");
        *out = nullptr;
        b = new clifft_gpu_batch();
        b->device = progs[0]->device;
        CUDA_OK(cudaSetDevice(b->device));
        size_t slab_total = 0;
        for (uint32_t i = 0; i < n; ++i) {
            clifft_gpu_program* p = progs[i];
            const clifft_gpu_sample_args& a = args[i];
            if (!p) invalid("null program in batch");
            if (p->device != b->device) invalid("all programs of a batch must live on one device");
            if (!(a.flags & CLIFFT_GPU_DEVICE_PTRS))
                invalid("batch entries need CLIFFT_GPU_DEVICE_PTRS (outputs stay on the device)");
            if (a.flags & (CLIFFT_GPU_TRACE | CLIFFT_GPU_PROFILE))
                invalid("batch entries do not support CLIFFT_GPU_TRACE or CLIFFT_GPU_PROFILE");
            if (a.shots == 0) invalid("batch entries need at least one shot");
        }
        // warm-up call per program: full validation, the autotuned shape, kernel attributes
        for (uint32_t i = 0; i < n; ++i) {
            const int r = clifft_gpu_sample(progs[i], &args[i], &outs[i]);
            if (r != 0) throw ApiError(r, std::string("batch entry ") + std::to_string(i) + ": " + g_last_error);
        }
        b->items.resize(n);
        size_t words = 0;
        for (uint32_t i = 0; i < n; ++i) {
            auto& it = b->items[i];
            clifft_gpu_program* p = progs[i];
            const clifft_gpu_sample_args& a = args[i];
            const clifft_program_image& m = p->meta;
            it.prog = p;
            it.out = &outs[i];
            const uint32_t rec_words = (m.total_meas_slots + 31) / 32;
            const uint32_t det_words = (m.num_detectors + 31) / 32;
            const uint32_t obs_words = (m.num_observables + 31) / 32;
            const bool allow_fusion = (a.flags & CLIFFT_GPU_NO_FUSION) == 0;
            uint32_t group_req = a.group_threads;
            if (group_req == 0 && !(a.flags & CLIFFT_GPU_NO_AUTOTUNE)) {
                const bool fm = (a.flags & CLIFFT_GPU_FORCED_MEAS) != 0, ff = (a.flags & CLIFFT_GPU_FORCED_FAULTS) != 0;
                const uint32_t key = a.precision | (allow_fusion ? 2u : 0u) | (a.flags & CLIFFT_GPU_SURVIVORS ? 4u : 0u) |
                                     (fm ? 8u : 0u) | (ff ? 16u : 0u);
                std::lock_guard<std::mutex> lock(g_tune_mu);
                auto f = g_tuned.find(std::make_tuple(p->content_hash, p->device, key));
                if (f != g_tuned.end()) group_req = f->second;
            }
            it.L = plan_launch(*p, a.precision, group_req, a.shots, rec_words, det_words, obs_words, allow_fusion,
                               a.max_resident);
            KParams& K = it.K;
            K.shots = a.shots;
            K.first_shot = a.first_shot;
            K.seed = a.seed;
            K.dust_eps = a.dust_eps > 0.0 ? a.dust_eps : (a.precision == CLIFFT_GPU_FP32 ? 1e-9 : 1e-18);
            K.flags = (a.flags & CLIFFT_GPU_SURVIVORS ? KF_SURVIVORS : 0) |
                      (a.flags & CLIFFT_GPU_FORCED_MEAS ? KF_FORCED_MEAS : 0) |
                      (a.flags & CLIFFT_GPU_FORCED_FAULTS ? KF_FORCED_FAULTS : 0) | (it.L.fuse ? KF_FUSE : 0);
            K.fuse_bytes = it.L.tiles ? tile_scratch_bytes(a.precision, it.L.G == 0, it.L.stages) : 0;
            K.stages = it.L.stages;
            K.rec_words = rec_words;
            K.det_words = det_words;
            K.obs_words = obs_words;
            K.meas_out_words = (m.num_measurements + 63) / 64;
            K.det_out_words = (m.num_detectors + 63) / 64;
            K.obs_out_words = (m.num_observables + 63) / 64;
            K.state_in_smem = it.L.state_in_smem ? 1 : 0;
            K.state_stride = it.L.state_stride;
            K.forced_meas = (a.flags & CLIFFT_GPU_FORCED_MEAS) ? a.forced_meas : nullptr;
            if (a.flags & CLIFFT_GPU_FORCED_FAULTS) {
                K.fault_off = a.fault_offsets;
                K.ro_off = a.readout_offsets;
                K.fault_sites = a.fault_sites;
                K.fault_chan = a.fault_channels;
                K.ro_entries = a.readout_entries;
            }
            K.out_meas = K.meas_out_words ? outs[i].meas : nullptr;
            K.out_det = K.det_out_words ? outs[i].det : nullptr;
            K.out_obs = K.obs_out_words ? outs[i].obs : nullptr;
            K.out_exp = m.num_exp_vals ? outs[i].exp_vals : nullptr;
            K.out_survived = outs[i].survived;
            it.scratch_words = 2 + 5 + m.num_observables + 8;
            it.scratch_at = words;
            words += (it.scratch_words + 31) & ~size_t(31);
            if (!it.L.state_in_smem) {
                const size_t amp = a.precision == CLIFFT_GPU_FP32 ? 8 : 16;
                const size_t bytes = size_t(it.L.blocks) * it.L.regions * it.L.S * it.L.state_stride * amp;
                slab_total += bytes;
                CUDA_OK(alloc_retry([&] { return cudaMalloc(&it.slab, bytes); }));
                K.state_global = it.slab;
            }
        }
        (void)slab_total;
        CUDA_OK(alloc_retry([&] { return cudaMalloc(&b->scratch_block, words * 8); }));
        b->scratch_block_words = words;
        CUDA_OK(cudaGraphCreate(&b->graph, 0));
        for (auto& it : b->items) {
            it.scratch = b->scratch_block + it.scratch_at;
            KParams& K = it.K;
            K.work_counter = it.scratch;
            K.error_word = reinterpret_cast<int*>(it.scratch + 1);
            K.counters = it.scratch + 2;
            K.phase_cycles = nullptr;
            K.error_info = it.scratch + it.scratch_words - 8;
            cudaMemsetParams ms{};
            ms.dst = it.scratch;
            ms.value = 0;
            ms.elementSize = 1;
            ms.width = it.scratch_words * 8;
            ms.height = 1;
            ms.pitch = 0;
            cudaGraphNode_t mnode;
            CUDA_OK(cudaGraphAddMemsetNode(&mnode, b->graph, nullptr, 0, &ms));
            it.kargs[0] = &it.prog->dev;
            it.kargs[1] = &it.K;
            cudaKernelNodeParams kp{};
            kp.func = (void*)it.L.fn;
            kp.gridDim = dim3(it.L.blocks);
            kp.blockDim = dim3(it.L.threads);
            kp.sharedMemBytes = (unsigned)it.L.smem;
            kp.kernelParams = it.kargs;
            CUDA_OK(cudaGraphAddKernelNode(&it.kernel_node, b->graph, &mnode, 1, &kp));
            bool seen = false;
            for (auto& sl : b->smem_limits)
                if (sl.first == it.L.fn) {
                    sl.second = std::max(sl.second, it.L.smem);
                    seen = true;
                }
            if (!seen) b->smem_limits.push_back({it.L.fn, it.L.smem});
        }
        CUDA_OK(cudaGraphInstantiate(&b->exec, b->graph, 0));
        CUDA_OK(cudaEventCreate(&b->e0));
        CUDA_OK(cudaEventCreate(&b->e1));
        *out = b;
    });
    if (rc != 0) batch_release(b);
    return rc;
}

int clifft_gpu_batch_run(clifft_gpu_batch* b, const uint64_t* seeds, void* stream, float* graph_ms) {
    return guarded([&] {
        if (!b) invalid("null batch");
        CUDA_OK(cudaSetDevice(b->device));
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (seeds) {
            for (auto& it : b->items) {
                it.K.seed = seeds[&it - b->items.data()];
                cudaKernelNodeParams kp{};
                kp.func = (void*)it.L.fn;
                kp.gridDim = dim3(it.L.blocks);
                kp.blockDim = dim3(it.L.threads);
                kp.sharedMemBytes = (unsigned)it.L.smem;
                kp.kernelParams = it.kargs;
                CUDA_OK(cudaGraphExecKernelNodeSetParams(b->exec, it.kernel_node, &kp));
            }
        }
        for (auto& sl : b->smem_limits) {
            cudaFuncAttributes cur{};
            CUDA_OK(cudaFuncGetAttributes(&cur, (const void*)sl.first));
            if (cur.maxDynamicSharedSizeBytes < int(sl.second))
                CUDA_OK(cudaFuncSetAttribute((const void*)sl.first, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(sl.second)));
        }
        CUDA_OK(cudaEventRecord(b->e0, st));
        CUDA_OK(cudaGraphLaunch(b->exec, st));
        CUDA_OK(cudaEventRecord(b->e1, st));
        std::vector<unsigned long long> hs(b->scratch_block_words);
        CUDA_OK(cudaMemcpyAsync(hs.data(), b->scratch_block, hs.size() * 8, cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        float ms = 0.f;
        CUDA_OK(cudaEventElapsedTime(&ms, b->e0, b->e1));
        if (graph_ms) *graph_ms = ms;
        for (auto& it : b->items) {
            const unsigned long long* w = hs.data() + it.scratch_at;
            const int dev_err = static_cast<int>(w[1] & 0xffffffffu);
            if (dev_err != 0)
                throw ApiError(CLIFFT_GPU_EDEVICE, "batch entry " + std::to_string(&it - b->items.data()) +
                                                       ": device error " + std::to_string(dev_err));
            clifft_gpu_outputs* o = it.out;
            o->passed_shots = w[2];
            o->logical_errors = w[3];
            o->dust_clamps = w[4];
            o->algorithmic_bytes = w[5];
            o->streamed_bytes = w[6];
            if (o->observable_ones)
                for (uint32_t j = 0; j < it.prog->meta.num_observables; ++j) o->observable_ones[j] = w[7 + j];
            o->kernel_launches = 1;
            o->kernel_ms = ms;
            o->group_threads = it.L.G ? uint32_t(it.L.G) : uint32_t(it.L.threads);
            o->state_in_smem = it.L.state_in_smem ? 1u : 0u;
            o->fused = it.L.fuse ? 1u : 0u;
        }
    });
}

void clifft_gpu_batch_free(clifft_gpu_batch* b) { batch_release(b); }

}  // extern "C"

// ------------------------------------------------- expectation-value gradients
namespace {


const char* opcode_name(uint32_t op) {
    static const char* names[] = {
        "FRAME_CNOT", "FRAME_CZ", "FRAME_H", "FRAME_S", "FRAME_S_DAG", "FRAME_SWAP", "ARRAY_CNOT", "ARRAY_CZ",
        "ARRAY_SWAP", "ARRAY_MULTI_CNOT", "ARRAY_MULTI_CZ", "ARRAY_H", "ARRAY_S", "ARRAY_S_DAG", "ARRAY_T",
        "ARRAY_T_DAG", "ARRAY_ROT", "ARRAY_U2", "ARRAY_U4", "EXPAND", "EXPAND_T", "EXPAND_T_DAG", "EXPAND_ROT"};
    return op < sizeof(names) / sizeof(names[0]) ? names[op] : "a measurement / noise / classical opcode";
}

bool grad_supported(uint32_t op) {
    switch (op) {
        case CLIFFT_OP_FRAME_CNOT:
        case CLIFFT_OP_FRAME_CZ:
        case CLIFFT_OP_FRAME_H:
        case CLIFFT_OP_FRAME_S:
        case CLIFFT_OP_FRAME_S_DAG:
        case CLIFFT_OP_FRAME_SWAP:
        case CLIFFT_OP_ARRAY_CNOT:
        case CLIFFT_OP_ARRAY_CZ:
        case CLIFFT_OP_ARRAY_SWAP:
        case CLIFFT_OP_ARRAY_MULTI_CNOT:
        case CLIFFT_OP_ARRAY_MULTI_CZ:
        case CLIFFT_OP_ARRAY_H:
        case CLIFFT_OP_ARRAY_S:
        case CLIFFT_OP_ARRAY_S_DAG:
        case CLIFFT_OP_ARRAY_T:
        case CLIFFT_OP_ARRAY_T_DAG:
        case CLIFFT_OP_ARRAY_ROT:
        case CLIFFT_OP_EXPAND:
        case CLIFFT_OP_EXPAND_T:
        case CLIFFT_OP_EXPAND_T_DAG:
        case CLIFFT_OP_EXPAND_ROT:
        case CLIFFT_OP_EXP_VAL: return true;
        default: return false;
    }
}

}  // namespace

extern "C" {

uint32_t clifft_gpu_program_num_rot_params(const clifft_gpu_program* prog) {
    return prog ? prog->num_rot_params : 0;
}

int clifft_gpu_expval_grad(clifft_gpu_program* prog, const clifft_gpu_grad_args* args, double* exp_vals,
                           double* grads) {
    return guarded([&] {
        if (!prog || !args || !exp_vals) invalid("null argument");
        const clifft_program_image& m = prog->meta;
        if (args->precision != CLIFFT_GPU_FP32 && args->precision != CLIFFT_GPU_FP64)
            invalid("precision must be CLIFFT_GPU_FP32 or CLIFFT_GPU_FP64");
        const bool dev_ptrs = (args->flags & CLIFFT_GPU_DEVICE_PTRS) != 0;
        // the program: measurement-free, noise-free, rotations as ARRAY_ROT / EXPAND_ROT
        const uint32_t n = m.num_instructions;
        std::vector<int32_t> rot_index(n, -1);
        std::vector<uint32_t> exp_pc, exp_out;
        std::vector<uint8_t> seen_out(m.num_exp_vals, 0);
        uint32_t np = 0;
        for (uint32_t i = 0; i < n; ++i) {
            const uint8_t* ins = prog->instr_host.data() + size_t(i) * 32;
            const uint32_t op = ins[0];
            if (!grad_supported(op)) {
                std::string why = (op == CLIFFT_OP_ARRAY_U2 || op == CLIFFT_OP_ARRAY_U4)
                                      ? " (fused U2 / U4 nodes hide the rotation angles: compile gradient "
                                        "programs without the single-axis / tile-axis fusion passes)"
                                      : "";
                invalid("clifft_gpu_expval_grad needs a measurement-free, noise-free program: instruction " +
                        std::to_string(i) + " is " + opcode_name(op) + why);
            }
            if (op == CLIFFT_OP_ARRAY_ROT || op == CLIFFT_OP_EXPAND_ROT) rot_index[i] = int32_t(np++);
            if (op == CLIFFT_OP_EXP_VAL) {
                uint32_t out_idx = 0;
                std::memcpy(&out_idx, ins + 12, 4);
                if (out_idx >= m.num_exp_vals || seen_out[out_idx]) invalid("EXP_VAL output rows must be distinct");
                seen_out[out_idx] = 1;
                exp_pc.push_back(i);
                exp_out.push_back(out_idx);
            }
        }
        if (np != prog->num_rot_params) invalid("internal: rotation count mismatch");
        const uint64_t batch = args->batch;
        if (batch == 0 || exp_pc.empty()) return;
        if (np > 0 && !grads) invalid("grads output is null");
        CUDA_OK(cudaSetDevice(prog->device));
        cudaStream_t st = static_cast<cudaStream_t>(args->stream);
        StreamBuffers buf(st);
        auto up = [&](const void* src, size_t bytes) -> void* {
            void* d = buf.alloc(bytes);
            if (d) CUDA_OK(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, st));
            return d;
        };
        GradParams G{};
        G.batch = batch;
        G.n_exp = uint32_t(exp_pc.size());
        G.n_out = m.num_exp_vals;
        G.n_params = np;
        G.rot_index = static_cast<const int32_t*>(up(rot_index.data(), rot_index.size() * 4));
        G.exp_pc = static_cast<const uint32_t*>(up(exp_pc.data(), exp_pc.size() * 4));
        G.exp_out = static_cast<const uint32_t*>(up(exp_out.data(), exp_out.size() * 4));
        if (args->phases && np) {
            G.phases = dev_ptrs ? args->phases
                                : static_cast<const double*>(up(args->phases, size_t(batch) * np * 8));
        }
        const size_t out_e = size_t(batch) * m.num_exp_vals * 8, out_g = size_t(batch) * m.num_exp_vals * np * 8;
        G.out_exp = dev_ptrs ? exp_vals : static_cast<double*>(buf.alloc(out_e));
        G.out_grad = dev_ptrs ? grads : static_cast<double*>(buf.alloc(std::max<size_t>(out_g, 8)));
        // rows of EXP_VAL outputs no instruction writes stay zero
        CUDA_OK(cudaMemsetAsync(G.out_exp, 0, out_e, st));
        if (out_g) CUDA_OK(cudaMemsetAsync(G.out_grad, 0, out_g, st));
        const bool fp32 = args->precision == CLIFFT_GPU_FP32;
        ExpvalGradFn fn = expval_grad_kernel_fn(fp32);
        int per_sm = 0, sms = 0;
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, kExpvalGradThreads, 0));
        CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, prog->device));
        const uint64_t tasks = batch * G.n_exp;
        G.stride = uint64_t(1) << m.peak_rank;
        const size_t amp = fp32 ? 8 : 16;
        size_t free_b = 0, total_b = 0;
        CUDA_OK(cudaMemGetInfo(&free_b, &total_b));
        uint64_t blocks = std::min<uint64_t>(tasks, uint64_t(std::max(per_sm, 1)) * sms);
        blocks = std::max<uint64_t>(1, std::min<uint64_t>(blocks, (free_b / 2) / (2 * G.stride * amp)));
        G.slab = buf.alloc(size_t(blocks) * 2 * G.stride * amp);
        auto* work = static_cast<unsigned long long*>(buf.alloc(64));
        CUDA_OK(cudaMemsetAsync(work, 0, 64, st));
        G.work = work;
        fn<<<unsigned(blocks), kExpvalGradThreads, 0, st>>>(prog->dev, G);
        CUDA_OK(cudaGetLastError());
        if (!dev_ptrs) {
            CUDA_OK(cudaMemcpyAsync(exp_vals, G.out_exp, out_e, cudaMemcpyDeviceToHost, st));
            if (out_g) CUDA_OK(cudaMemcpyAsync(grads, G.out_grad, out_g, cudaMemcpyDeviceToHost, st));
        }
        CUDA_OK(cudaStreamSynchronize(st));
    });
}

}  // extern "C"

// ------------------------------------------------------ k-fault importance sampling
extern "C" {

int clifft_gpu_sample_k(clifft_gpu_program* prog, const clifft_gpu_sample_args* args, uint32_t k,
                        clifft_gpu_outputs* out) {
    return guarded([&] {
        if (!prog || !args || !out) invalid("null argument");
        if (args->flags & (CLIFFT_GPU_FORCED_MEAS | CLIFFT_GPU_FORCED_FAULTS))
            invalid("clifft_gpu_sample_k draws its own fault sets: forced outcomes / faults are not accepted");
        // the stratum must carry probability mass (src/clifft/svm/svm.cc:522-545)
        const std::vector<double>& probs = prog->fault_probs;
        const uint32_t n_total = uint32_t(probs.size());
        if (k > n_total)
            invalid("k (" + std::to_string(k) + ") exceeds total fault sites (" + std::to_string(n_total) + ")");
        uint32_t n_certain = 0, n_impossible = 0;
        for (double p : probs) {
            if (p <= 0.0)
                n_impossible++;
            else if (p >= 1.0)
                n_certain++;
        }
        if (k < n_certain || k > n_total - n_impossible)
            invalid("k-fault stratum k=" + std::to_string(k) + " has zero probability mass (" +
                    std::to_string(n_certain) + " sites have p=1, " + std::to_string(n_impossible) +
                    " sites have p=0)");
        const uint64_t shots = args->shots;
        if (shots == 0) {
            sample_impl(prog, args, out, nullptr);
            return;
        }
        const uint64_t stride = std::max<uint32_t>(k, 1);
        if (shots * stride > 0xffffffffull) invalid("shots x k exceeds 2^32 fault slots; split the call");
        // sampler tables: equal probabilities -> uniform k-subsets; else odds
        // ratios (scaled to mean 1) and the suffix subset-weight DP
        bool uniform = k <= kSampleKUniformMax;
        for (uint32_t i = 1; i < n_total && uniform; ++i) uniform = probs[i] == probs[0];
        std::vector<double> w, dp;
        if (!uniform) {
            w.resize(n_total);
            double sum_w = 0.0;
            for (uint32_t i = 0; i < n_total; ++i) {
                const double p = std::min(std::max(probs[i], 0.0), 1.0 - 1e-15);
                w[i] = p / (1.0 - p);
                sum_w += w[i];
            }
            if (sum_w > 0.0)
                for (double& x : w) x *= double(n_total) / sum_w;
            const uint32_t st = k + 1;
            dp.assign(size_t(n_total + 1) * st, 0.0);
            for (uint32_t i = 0; i <= n_total; ++i) dp[size_t(i) * st] = 1.0;
            for (int i = int(n_total) - 1; i >= 0; --i) {
                const uint32_t mx = std::min(n_total - uint32_t(i), k);
                for (uint32_t j = 1; j <= mx; ++j)
                    dp[size_t(i) * st + j] = dp[size_t(i + 1) * st + j] + w[i] * dp[size_t(i + 1) * st + (j - 1)];
            }
        }
        CUDA_OK(cudaSetDevice(prog->device));
        cudaStream_t st = static_cast<cudaStream_t>(args->stream);
        StreamBuffers buf(st);
        SampleKParams S{};
        S.shots = shots;
        S.first_shot = args->first_shot;
        S.seed = args->seed;
        S.k = k;
        S.n_total = n_total;
        S.n_q = prog->meta.num_noise_sites;
        S.uniform = uniform ? 1u : 0u;
        auto up = [&](const std::vector<double>& v) -> const double* {
            if (v.empty()) return nullptr;
            void* d = buf.alloc(v.size() * 8);
            CUDA_OK(cudaMemcpyAsync(d, v.data(), v.size() * 8, cudaMemcpyHostToDevice, st));
            return static_cast<const double*>(d);
        };
        S.w = up(w);
        S.dp = up(dp);
        auto u32 = [&](size_t n) { return static_cast<uint32_t*>(buf.alloc(n * 4)); };
        S.fault_off = u32(shots);
        S.fault_end = u32(shots);
        S.ro_off = u32(shots);
        S.ro_end = u32(shots);
        S.fault_sites = u32(shots * stride);
        S.fault_chan = u32(shots * stride);
        S.ro_entries = u32(shots * stride);
        launch_sample_k_prepare(prog->dev, S, st);
        CUDA_OK(cudaGetLastError());
        clifft_gpu_sample_args a = *args;
        a.flags |= CLIFFT_GPU_FORCED_FAULTS;
        a.fault_offsets = S.fault_off;
        a.fault_sites = S.fault_sites;
        a.fault_channels = S.fault_chan;
        a.readout_offsets = S.ro_off;
        a.readout_entries = S.ro_entries;
        DeviceFaults df;
        df.fault_end = S.fault_end;
        df.ro_end = S.ro_end;
        sample_impl(prog, &a, out, &df);
        out->kernel_launches += 1;
    });
}

}  // extern "C"
