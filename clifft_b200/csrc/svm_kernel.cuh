// svm_kernel.cuh -- persistent shot-parallel Schrodinger-VM interpreter for sm_100a.
//
// Work decomposition. A *shot group* of G lanes runs one shot of the
// reference's bytecode:
//   * G in {1, 2, 4, 8, 16, 32}: a warp carries S = 32 / G shots side by side
//     and walks the (shared, read-only) instruction stream in lockstep, so one
//     issued instruction advances S shots. Frame opcodes, noise, records and
//     detector logic cost one lane-instruction per shot instead of 32;
//     statevector sweeps are split over the G lanes of each shot. A warp takes
//     S shot indices at a time from a global work counter; a shot that stops
//     early (post-selection, unreachable forced outcome) parks its lanes until
//     the warp's other shots finish.
//   * G = 0: a whole CTA runs one shot (large k); sweeps use every thread and
//     the shot index comes from the work counter, so the CTA moves on as soon as
//     its shot ends.
// Statevectors live in shared memory when they fit and otherwise in a global
// slab per warp / CTA. Within a warp the S statevectors are interleaved
// (amplitude i of shot slot s at [i * S + s]) so lanes of different shots
// touching the same amplitude index hit consecutive banks / addresses.
//
// Per shot, the factored state |psi> = gamma * U_C * P * (|phi>_A (x) |0>_D)
// (src/clifft/svm/svm.h:92-103) is held as:
//   * the 2^k active amplitudes, complex FP32 or FP64;
//   * the Pauli frame p_x / p_z as NW 64-bit words in registers of every lane
//     of the group (updated redundantly: frame opcodes need no barrier);
//   * gamma as an FP64 complex in registers;
//   * measurement / detector / observable records as bit arrays in shared
//     memory.
// Branch probabilities and expectation values are reduced in FP64 with a fixed
// summation order, so every lane of a group derives the same outcome from the
// same counter-based Philox draw (identical control flow, no broadcast).
//
// Opcode semantics follow the reference kernels in
// src/clifft/svm/svm_kernels.inl and svm_forced_kernels.cc; each handler cites
// its source.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "clifft_program_image.h"

namespace cgpu {

// ------------------------------------------------------------------ program
struct DevProg {
    const uint4* instr;  // 2 x uint4 per instruction (32 bytes, verbatim)
    uint32_t n_instr;
    uint32_t nw;
    uint32_t peak;
    uint32_t num_meas;
    uint32_t slots;
    uint32_t num_det;
    uint32_t num_obs;
    uint32_t num_exp;
    const uint64_t* pauli_x;
    const uint64_t* pauli_z;
    const uint8_t* pauli_sign;
    const uint64_t* exp_x;
    const uint64_t* exp_z;
    const uint8_t* exp_sign;
    uint32_t n_sites;
    const uint32_t* site_off;
    const double* site_psum;  // sequential sum of the site's channel probs (same order as the reference)
    const double* chan_prob;
    const uint64_t* chan_x;
    const uint64_t* chan_z;
    const double* hazards;
    const uint32_t* ro_meas;
    const double* ro_prob;
    const uint32_t* det_off;
    const uint32_t* det_tg;
    const uint32_t* obs_off;
    const uint32_t* obs_tg;
    const double* u2;
    const uint8_t* u2_out;
    const double* u4;
    const uint8_t* u4_out;
    uint32_t n_expected;
    const uint8_t* expected;
};

// ------------------------------------------------------------- run params
struct KParams {
    uint64_t shots;
    uint64_t first_shot;
    uint64_t seed;
    double dust_eps;
    uint32_t flags;
    uint32_t rec_words;       // u32 words of measurement record per shot (>= ceil(slots/32))
    uint32_t det_words;       // u32 words of detector record per shot
    uint32_t obs_words;       // u32 words of observable record per shot
    uint32_t meas_out_words;  // u64 words per shot in outputs
    uint32_t det_out_words;
    uint32_t obs_out_words;
    uint32_t state_in_smem;
    uint64_t state_stride;    // amplitudes per shot slot (2^peak_rank)
    void* state_global;       // global slab base (when !state_in_smem)
    unsigned long long* work_counter;
    unsigned long long* counters;  // [0] passed, [1] logical errors, [2] dust clamps, [3] algorithmic bytes, [4] streamed bytes, [5..] observable ones
    int* error_word;               // first device-side error code (0 = none)
    unsigned long long* error_info;  // where a bounded wait gave up: site, pc, tile, tiles, r, k
    // forced inputs
    const uint8_t* forced_meas;
    const uint32_t* fault_off;
    const uint32_t* fault_sites;
    const uint32_t* fault_chan;
    const uint32_t* ro_off;
    const uint32_t* ro_entries;
    const uint32_t* fault_end;  // optional per-shot end offsets (else fault_off[shot + 1])
    const uint32_t* ro_end;     // optional per-shot end offsets (else ro_off[shot + 1])
    // outputs
    uint64_t* out_meas;
    uint64_t* out_det;
    uint64_t* out_obs;
    double* out_exp;
    uint8_t* out_survived;
    double* out_meas_prob;
    double* out_log_prob;
    uint32_t* out_final_k;
    double* out_final_gamma;
    uint64_t* out_final_px;
    uint64_t* out_final_pz;
    double* out_final_v;
    uint64_t dump_shots;
    uint32_t fuse_bytes;  // shared bytes per CTA reserved for fused tile sweeps (0 = off)
    uint32_t stages;      // tile buffers per CTA (2..kMaxStages) when fuse_bytes != 0
    uint32_t dense_min_weight;  // KF_DENSE: least CUDA-core weight of a run worth a GEMM (U4 4, U2 2, others 1)
    unsigned long long* phase_cycles;  // optional: SM cycles per executor phase (thread 0 of each group)
    // segmented execution (survivor runs of warp groups): this launch runs
    // instructions [seg_begin, seg_end) for the items of seg_in; shots alive
    // at seg_end save their state and append themselves to seg_out
    uint32_t seg_flags;                       // KSEG_* (0 = the whole program in one launch)
    uint32_t seg_begin, seg_end;
    const uint32_t* seg_in;                   // shot ids of this segment's items (null: item = shot)
    const unsigned long long* seg_count_in;   // number of items (null: shots)
    uint32_t* seg_out;
    unsigned long long* seg_count_out;
    unsigned char* seg_state;                 // per shot: saved state, seg_stride bytes
    uint64_t seg_stride;
};

enum : uint32_t {
    KF_SURVIVORS = 0x01u,
    KF_FORCED_MEAS = 0x02u,
    KF_FORCED_FAULTS = 0x04u,
    KF_TRACE = 0x10u,
    KF_FUSE = 0x20u,  // fused tile sweeps for global-memory statevectors (CTA groups)
    KF_RAW_PARITY = 0x40u,  // detectors / observables without expected parities, POSTSELECT records instead of discarding
    KF_DENSE = 0x80u,       // FP32 CTA groups of 256 compute threads: dense runs of fused blocks on tcgen05 (3xTF32)
};

enum : uint32_t {
    KSEG_ON = 0x1u,     // segmented launch
    KSEG_FIRST = 0x2u,  // shots start from the reset state
    KSEG_LAST = 0x4u,   // shots alive at the end are finished (records written)
};

enum : int {
    DEV_ERR_ZERO_NORM = 1,
    DEV_ERR_BAD_OPCODE = 2,
    DEV_ERR_TIMEOUT = 3,  // a bounded wait on a bulk-copy barrier gave up
};

// ----------------------------------------------------------------- complex
template <typename R>
struct Cx;
template <>
struct Cx<float> {
    using T = float2;
    static __device__ __forceinline__ T make(double re, double im) {
        return make_float2((float)re, (float)im);
    }
};
template <>
struct Cx<double> {
    using T = double2;
    static __device__ __forceinline__ T make(double re, double im) { return make_double2(re, im); }
};

// Complex arithmetic with every rounding step spelled out (explicit fma and
// round-to-nearest products / sums), so the compiler cannot contract
// differently in different inlining contexts: the fused tile path, the
// per-opcode sweeps and every launch shape perform bit-identical arithmetic.
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rn_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double rn_fma(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T>
__device__ __forceinline__ T cadd(T a, T b) {
    T r;
    r.x = rn_add(a.x, b.x);
    r.y = rn_add(a.y, b.y);
    return r;
}
template <typename T>
__device__ __forceinline__ T csub(T a, T b) {
    T r;
    r.x = rn_sub(a.x, b.x);
    r.y = rn_sub(a.y, b.y);
    return r;
}
// (a.x b.x - a.y b.y, a.x b.y + a.y b.x): one rounded product, one fma per part
template <typename T>
__device__ __forceinline__ T cmul(T a, T b) {
    T r;
    r.x = rn_fma(a.x, b.x, -rn_mul(a.y, b.y));
    r.y = rn_fma(a.x, b.y, rn_mul(a.y, b.x));
    return r;
}
// acc + a b, the sum step of a matrix row. FP64 rounds the product and then
// the sum (the reference's complex<double> arithmetic, which the oracle
// reproduces bit for bit); FP32 folds each part into two fused multiply-adds,
// which halves the instructions of the dense U2 / U4 nodes and rounds less.
__device__ __forceinline__ double2 cmac(double2 acc, double2 a, double2 b) { return cadd(acc, cmul(a, b)); }
__device__ __forceinline__ float2 cmac(float2 acc, float2 a, float2 b) {
    float2 r;
    r.x = rn_fma(a.x, b.x, rn_fma(-a.y, b.y, acc.x));
    r.y = rn_fma(a.x, b.y, rn_fma(a.y, b.x, acc.y));
    return r;
}
template <typename T, typename S>
__device__ __forceinline__ T cscale(T a, S s) {
    T r;
    r.x = rn_mul(a.x, s);
    r.y = rn_mul(a.y, s);
    return r;
}
template <typename T>
__device__ __forceinline__ T cneg(T a) {
    T r;
    r.x = -a.x;
    r.y = -a.y;
    return r;
}
template <typename T>
__device__ __forceinline__ double cnorm_d(T a) {
    double x = (double)a.x, y = (double)a.y;
    return __fma_rn(x, x, __dmul_rn(y, y));
}
__device__ __forceinline__ double2 dmul(double2 a, double2 b) {
    return make_double2(__fma_rn(a.x, b.x, -__dmul_rn(a.y, b.y)), __fma_rn(a.x, b.y, __dmul_rn(a.y, b.x)));
}

// kInvSqrt2 = std::numbers::sqrt2 / 2 (src/clifft/util/constants.h) and the
// separate 1.0 / std::sqrt(2.0) that EXPAND scales gamma by
// (src/clifft/svm/svm_kernels.inl:895).
#define CGPU_INV_SQRT2 0.70710678118654757
#define CGPU_EXPAND_SCALE 0.70710678118654746

// ---------------------------------------------------------------- philox
// Philox4x32-10 (Salmon et al., SC'11). Draw d of shot s uses counter
// (d >> 1, stream, s_lo, s_hi) and key (seed_lo, seed_hi); even draws take
// words (0, 1), odd draws words (2, 3); 53 high bits -> [0, 1) as the
// reference's random_double (src/clifft/svm/svm.h:150). Stream 0 feeds the
// executor; stream 1 the per-shot fault-site draws of sample_k.
__device__ __forceinline__ double philox_uniform(uint64_t seed, uint64_t shot, uint32_t draw,
                                                 uint32_t stream = 0u) {
    uint32_t c0 = draw >> 1, c1 = stream, c2 = (uint32_t)shot, c3 = (uint32_t)(shot >> 32);
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    uint64_t r = (draw & 1u) ? ((uint64_t)c3 << 32 | c2) : ((uint64_t)c1 << 32 | c0);
    return (double)(r >> 11) * 0x1.0p-53;
}

// ------------------------------------------------------------------ groups
// G lanes of one warp per shot (G = 1..32), S = 32 / G shots per warp.
template <int G>
struct Lanes {
    static constexpr bool kCta = false;
    static constexpr bool kWS = false;
    static constexpr int S = 32 / G;
    __device__ static __forceinline__ int size() { return G; }
    __device__ static __forceinline__ int rank() { return (int)(threadIdx.x & 31) & (G - 1); }
    __device__ static __forceinline__ int slot() { return (int)(threadIdx.x & 31) / G; }
    __device__ static __forceinline__ unsigned mask() {
        return G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(unsigned)(G - 1)));
    }
    __device__ static __forceinline__ void sync() {
        if (G > 1) __syncwarp(mask());
    }
};
// A whole CTA per shot.
struct CtaLanes {
    static constexpr bool kCta = true;
    static constexpr bool kWS = false;
    static constexpr int S = 1;
    __device__ static __forceinline__ int size() { return blockDim.x; }
    __device__ static __forceinline__ int rank() { return threadIdx.x; }
    __device__ static __forceinline__ int slot() { return 0; }
    __device__ static __forceinline__ unsigned mask() { return 0xffffffffu; }
    __device__ static __forceinline__ void sync() { __syncthreads(); }
};
template <int G>
struct GroupOf {
    using type = Lanes<G>;
};
template <>
struct GroupOf<0> {
    using type = CtaLanes;
};
// A whole CTA per shot whose last warp only moves tiles in fused blocks
// (warp-specialised tile engine); every other step runs on all its threads.
struct CtaLanesWS : CtaLanes {
    static constexpr bool kWS = true;
};
template <>
struct GroupOf<-1> {
    using type = CtaLanesWS;
};

__device__ __forceinline__ uint64_t ins0(uint64_t v, uint32_t pos) {
    uint64_t m = (1ull << pos) - 1;
    return (v & m) | ((v & ~m) << 1);
}
__device__ __forceinline__ uint64_t ins00(uint64_t v, uint32_t a, uint32_t b) {
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return ins0(ins0(v, lo), hi);
}
// the same on tile-local (32-bit) indices
__device__ __forceinline__ uint32_t ins0_32(uint32_t v, uint32_t pos) {
    const uint32_t m = (1u << pos) - 1u;
    return (v & m) | ((v & ~m) << 1);
}
__device__ __forceinline__ uint32_t ins00_32(uint32_t v, uint32_t a, uint32_t b) {
    const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return ins0_32(ins0_32(v, lo), hi);
}

// Frame words in registers. Axes are < 64 * NW by validation.
template <int NW>
struct Frame {
    uint64_t x[NW];
    uint64_t z[NW];
    __device__ __forceinline__ void clear() {
#pragma unroll
        for (int i = 0; i < NW; ++i) x[i] = z[i] = 0;
    }
    __device__ static __forceinline__ int get(const uint64_t* w, uint32_t a) {
        if (NW == 1) return (int)((w[0] >> (a & 63)) & 1u);
        uint64_t v = 0;
#pragma unroll
        for (int i = 0; i < NW; ++i)
            if ((uint32_t)i == (a >> 6)) v = w[i];
        return (int)((v >> (a & 63)) & 1u);
    }
    __device__ static __forceinline__ void put(uint64_t* w, uint32_t a, int b) {
#pragma unroll
        for (int i = 0; i < NW; ++i)
            if (NW == 1 || (uint32_t)i == (a >> 6)) {
                uint64_t m = 1ull << (a & 63);
                w[i] = b ? (w[i] | m) : (w[i] & ~m);
            }
    }
    __device__ static __forceinline__ void flip(uint64_t* w, uint32_t a, int b) {
#pragma unroll
        for (int i = 0; i < NW; ++i)
            if (NW == 1 || (uint32_t)i == (a >> 6)) w[i] ^= (uint64_t)(b & 1) << (a & 63);
    }
    __device__ __forceinline__ int px(uint32_t a) const { return get(x, a); }
    __device__ __forceinline__ int pz(uint32_t a) const { return get(z, a); }
};

// FP64 reduction of N values over one shot group with a fixed order (lane
// tree within the group, then warps in index order for a CTA). Every lane of
// the group returns the same bits.
template <class Grp, int N>
__device__ __forceinline__ void group_reduce(double (&v)[N], double* red) {
    if (!Grp::kCta) {
        constexpr int G = 32 / Grp::S;
        if (G > 1) {
            const unsigned m = Grp::mask();
#pragma unroll
            for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
                for (int j = 0; j < N; ++j) v[j] += __shfl_down_sync(m, v[j], off, G);
#pragma unroll
            for (int j = 0; j < N; ++j) v[j] = __shfl_sync(m, v[j], 0, G);
        }
        return;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int j = 0; j < N; ++j) v[j] += __shfl_down_sync(0xffffffffu, v[j], off);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < N; ++j) red[warp * N + j] = v[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < N; ++j) v[j] = 0.0;
    for (int w = 0; w < nwarps; ++w)
#pragma unroll
        for (int j = 0; j < N; ++j) v[j] += red[w * N + j];
    __syncthreads();
}

__device__ __forceinline__ int bit_of(const uint32_t* r, uint32_t i, int S) {
    return (int)((r[(i >> 5) * S] >> (i & 31)) & 1u);
}

// Per-lane totals flushed once per kernel.
struct Tally {
    unsigned long long passed = 0, logical = 0, dust = 0, bytes = 0, moved = 0;
};

// ------------------------------------------------------------- fused sweeps
// A fused block is a run of consecutive opcodes applied to the statevector in
// one streamed pass: tile by tile through shared memory, every micro-op of
// the block on a tile before it is written back. A tile covers the tile axes
// F (2^TILE_BITS amplitudes: every index with fixed values of the other,
// tile-global axes). The block's frame-dependent choices (conjugated phases,
// U2 / U4 variants, EXPAND phases) are resolved once per shot into micro-ops
// on tile-local bit positions; each amplitude sees the same arithmetic in the
// same order as the unfused opcode sequence.
//   * Axes an op moves amplitudes along (targets of CNOT / SWAP / H / U2 / U4,
//     the new axis of an EXPAND) must be tile axes. Control and parity axes
//     may be tile-global: their bits are constant over a tile and enter the
//     micro-op's condition through `greq` / `gpar`. Diagonal ops (CZ,
//     multi-CZ, phases) therefore fuse whatever their axes.
//   * EXPAND is a micro-op (copy the new axis' clear half onto its set half,
//     times the phase); the block loads only the runs of each tile whose new
//     axes are clear.
//   * An active measurement on axis k-1 ends a block: its two half-norms are
//     summed from the tile after the block's micro-ops (an X-basis
//     measurement first folds with an H micro-op, a fused swap with a SWAP
//     micro-op), and the collapse to the upper half flips the shot's address
//     label (`xo`) instead of copying it.
//   * With KF_DENSE (FP32 CTA groups) a run of micro-ops that stays on at
//     most four tile-local bits and holds an H / U2 / U4 is composed into one
//     16 x 16 complex matrix, applied as a batched GEMM on the tensor cores
//     (M_DENSE; the rest of the run becomes M_NOP).
enum : uint8_t { M_CNOT, M_CZ, M_SWAP, M_MCNOT, M_MCZ, M_H, M_PHASE, M_U2, M_U4, M_EXPAND, M_SCALE, M_DENSE, M_NOP };
enum : uint8_t {
    MF_PARITY = 0x1,  // the condition also needs odd parity of (index & par) ^ (global bits & gpar)
    MF_COPY = 0x2,    // EXPAND without a phase: a plain copy
};
template <typename T>
struct MicroOpT {
    uint8_t kind, a, b, flags;  // a, b: tile-local target bits
    uint32_t req;               // tile-local bits that must all be set
    uint32_t par;               // tile-local parity bits (MF_PARITY)
    uint32_t pad;
    uint64_t greq;              // tile-global index bits that must all be set
    uint64_t gpar;              // tile-global parity bits (MF_PARITY)
    T c[16];                    // coefficients, already in the statevector's precision
};
constexpr int kMaxStages = 4;      // tile buffers (tiles in flight) per shot group: 2..4, chosen per launch
constexpr int kMaxRunsLog2 = 6;    // at most 64 contiguous runs per tile
// Tile-engine geometry of a one-shot group. A CTA streams 32 KiB tiles and
// fuses up to 24 opcodes per pass; a warp running one shot streams 4 KiB
// tiles through two buffers and fuses up to 24 (FP32) / 16 (FP64), which
// leaves room for four 4-warp CTAs per SM (the register limit). Scratch
// layout of one group: [2 x kMaxStages mbarriers: tile loaded / tile computed]
// [dense-block slot: MMA mbarrier, TMEM address, phase][micro-ops][64 run
// offsets][64-byte axis -> local bit table][stages tile buffers, 128-B
// aligned][FP32 CTA groups with three stages: the dense block's B operand,
// 8 KiB].
template <typename R, bool CTA>
struct TileCfg {
    using MOp = MicroOpT<typename Cx<R>::T>;
    static constexpr int kBits = CTA ? (sizeof(R) == 4 ? 12 : 11) : (sizeof(R) == 4 ? 9 : 8);
    static constexpr int kMops = CTA ? 24 : (sizeof(R) == 4 ? 24 : 16);
    static constexpr uint32_t kBarOffset = 0;
    static constexpr uint32_t kDenseSlotOffset = 2u * kMaxStages * 8u;
    static constexpr uint32_t kMopsOffset = kDenseSlotOffset + 16u;
    static constexpr uint32_t kTablesOffset = kMopsOffset + kMops * (uint32_t)sizeof(MOp);
    static constexpr uint32_t kLbitOffset = kTablesOffset + 64u * 8u;
    static constexpr uint32_t kBufOffset = (kLbitOffset + 64u + 127u) & ~127u;
    static constexpr uint32_t kDenseBBytes = 8192u;  // B operand of a dense block: TF32 hi + lo, 32 x 32 each
    static __host__ __device__ constexpr bool dense_capable(uint32_t stages) {
        return CTA && sizeof(R) == 4 && stages == 3;
    }
    static __host__ __device__ constexpr uint32_t dense_b_offset(uint32_t stages) {
        return kBufOffset + stages * (1u << kBits) * 2u * (uint32_t)sizeof(R);
    }
    static __host__ __device__ constexpr uint32_t smem_bytes(uint32_t stages, bool dense = false) {
        return dense_b_offset(stages) + (dense && dense_capable(stages) ? kDenseBBytes : 0u);
    }
};

// ---- tensor-core primitives of the dense blocks (tcgen05, TMEM). A dense
// block U = Ur + i Ui acts on every 16-amplitude group x of a tile as one
// real product y = M x with the 32 x 32 matrix M = [[Ur, -Ui], [Ui, Ur]] in
// the interleaved order (index 2 d + 0 = Re, 2 d + 1 = Im): D = X M^T with
// the groups as the 128 rows of X (one TMEM lane each, the A operand), M^T
// as the K-major B operand in shared memory and D in TMEM. Both operands
// are split into a TF32 high part and the TF32 low part of the remainder;
// D = Xhi Mhi + Xlo Mhi + Xhi Mlo (3xTF32) keeps a product within a few
// FP32 ulps. One thread issues the MMAs; the group's threads read D back.
__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}
// x = hi + lo exactly (hi: x with its 13 low mantissa bits cleared); lo
// keeps its TF32 part
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
    hi = __float_as_uint(x) & 0xffffe000u;
    lo = __float_as_uint(x - __uint_as_float(hi)) & 0xffffe000u;
}
constexpr uint32_t kDenseTmemCols = 256;  // two 128-group chunks x (A hi 32 + A lo 32 + D 32) columns
// instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12
// = 2), both K-major, N = 32 (bits 17-22 = N / 8), M = 128 (bits 24-28 = M / 16)
constexpr uint32_t kDenseIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
// shared-memory descriptor of a K-major operand without swizzle: 8-row x
// 16-byte core matrices, LBO = 512 B between the two core matrices of an
// MMA's K = 8, SBO = 128 B between 8-row groups, version 1 (bits 46-47)
__device__ __forceinline__ uint64_t dense_b_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3fffu) | ((uint64_t)(512u >> 4) << 16) | ((uint64_t)(128u >> 4) << 32) |
           (1ull << 46);
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_alloc(uint32_t smem_dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_dst), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n" ::"r"(taddr),
                 "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
// D (+)= A B with A in TMEM, B by descriptor; accumulate = 0 overwrites D
__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %3, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %4, {%5, %5, %5, %5}, p;\n}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b_desc), "r"(accumulate), "r"(kDenseIdesc), "r"(z)
        : "memory");
}
// ---- bulk-copy (TMA, untiled) and mbarrier primitives. Every copy here reads
// or writes this GPU's own global memory; none uses cluster multicast.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ uint32_t mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok;
}
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst_smem)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void bulk_store(void* dst, const void* src_smem, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(smem_u32(src_smem)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// the mbarrier completes once every tcgen05.mma this thread issued has finished
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// barrier 1 over the first n threads of the CTA (the compute warps of a
// warp-specialised CTA group; barrier 0 is __syncthreads)
__device__ __forceinline__ void bar_sync_first(uint32_t n) { asm volatile("bar.sync 1, %0;\n" ::"r"(n) : "memory"); }
__device__ __forceinline__ bool bar_or_first(uint32_t n, bool pred) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n barrier.cta.red.or.pred q, 1, %2, p;\n selp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(n)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Scalar state the control warp of a CTA group hands to the worker warps
// before a statevector sweep.
template <int NW>
struct CtlState {
    uint64_t fx[NW], fz[NW];
    double2 gamma;
    double log_prob;
    unsigned long long dust, bytes, moved;
    uint32_t k, draw, next_noise, ff_pos, ff_end, ro_pos, ro_end, pc;
    uint32_t cmd;  // 0 = run the sweep at pc, 1 = shot finished
    uint32_t flags;
};
constexpr uint32_t kCtlBytes = 512;

// --------------------------------------------------------------- the shot
template <typename R, class Grp, int NW, bool DENSE = false>
struct Shot {
    using T = typename Cx<R>::T;
    static constexpr int S = Grp::S;
    // one-shot groups (a CTA, or a warp of 32 lanes) stream global
    // statevectors through the tile engine
    static constexpr bool kTiles = Grp::S == 1;
    using TC = TileCfg<R, Grp::kCta>;
    const DevProg& P;
    const KParams& K;
    T* v;           // slot base: amplitude i at v[i * S]
    uint32_t* rec;  // record words: word w at rec[w * S]
    uint32_t* det;
    uint32_t* obs;
    double* red;
    uint64_t shot;
    Frame<NW> f;
    double2 gamma;
    uint32_t k;
    uint32_t draw;
    uint32_t next_noise;
    uint32_t ff_pos, ff_end, ro_pos, ro_end;
    bool rec_dirty;
    bool stop;
    bool discarded;
    bool reachable;
    double log_prob;
    unsigned long long dust;
    unsigned long long bytes;  // algorithmic statevector bytes moved by this shot
    const uint8_t* forced;
    double* meas_prob;
    // fused-sweep state (one-shot groups with a global statevector)
    unsigned char* fuse;       // shared scratch: stage barriers, micro-ops, index tables, tile buffers
    uint32_t* bar_phase;       // CTA groups: bit st = parity of the phase stage st's barrier is in;
                               // bit 31 set once a wait timed out (the barriers are then unusable)
    bool resolving;            // true while a fused block's opcodes emit micro-ops
    bool solo;                 // CTA groups: only the control warp is executing
    int n_mops;
    unsigned long long moved;  // statevector bytes actually streamed
    // Address label of a one-shot group's global statevector: logical
    // amplitude i lives at v[i ^ xo]. A measurement that keeps the upper half
    // of axis k-1 flips bit k-1 instead of copying that half down. Its bits
    // are all above the tile bits, so the label maps every tile run to one
    // contiguous run.
    uint64_t xo;
    uint64_t tileF;  // tile axes of the fused block being resolved

    __device__ __forceinline__ Shot(const DevProg& p, const KParams& kp, T* vv, uint32_t* r, uint32_t* d,
                                    uint32_t* o, double* rd, unsigned char* fz, uint32_t* bp, uint64_t s)
        : P(p), K(kp), v(vv), rec(r), det(d), obs(o), red(rd), shot(s), fuse(fz), bar_phase(bp) {}

    __device__ __forceinline__ T& A(uint64_t i) { return v[(kTiles ? (i ^ xo) : i) * S]; }
    // algorithmic bytes of an opcode (per-opcode definition); streamed bytes
    // are counted separately because a fused block streams the state once
    __device__ __forceinline__ void account(uint64_t amps) {
        bytes += amps * sizeof(T);
        if (!resolving) moved += amps * sizeof(T);
    }
    __device__ __forceinline__ double uniform() { return philox_uniform(K.seed, K.first_shot + shot, draw++); }
    __device__ __forceinline__ void phase(double2 p) { gamma = dmul(gamma, p); }
    __device__ __forceinline__ void negate_gamma() { gamma = make_double2(-gamma.x, -gamma.y); }

    __device__ __forceinline__ void flush_records() {
        if (rec_dirty) {
            if (Grp::kCta && solo)
                __syncwarp();
            else
                Grp::sync();
            rec_dirty = false;
        }
    }
    __device__ __forceinline__ void write_meas(uint32_t idx, int bit, double prob) {
        if (Grp::rank() == 0) {
            uint32_t m = 1u << (idx & 31);
            uint32_t& w = rec[(idx >> 5) * S];
            w = bit ? (w | m) : (w & ~m);
            if (meas_prob) meas_prob[idx] = prob;
        }
        rec_dirty = true;
    }

    // SchrodingerState::scale_magnitude (src/clifft/svm/svm.h:177-186). The
    // lazy-renormalisation window is 1e+-100 in FP64 and 1e+-20 in FP32 so the
    // FP32 amplitudes never approach their exponent range.
    __device__ __forceinline__ void scale_magnitude(double s) {
        gamma.x *= s;
        gamma.y *= s;
        const double hi = sizeof(R) == 8 ? 1e100 : 1e20;
        const double lo = sizeof(R) == 8 ? 1e-100 : 1e-20;
        double g = hypot(gamma.x, gamma.y);
        if (g > hi || (g < lo && g > 0.0)) {
            uint64_t n = 1ull << k;
            if (kTiles && resolving) {
                // inside a fused block: the same scaling as a micro-op at this point
                const double c[2] = {g, 0.0};
                emit(M_SCALE, 0, 0, 0, 0, 0, c, 1);
                bytes += 2 * n * sizeof(T);
            } else {
                for (uint64_t i = Grp::rank(); i < n; i += Grp::size()) A(i) = cscale(A(i), (R)g);
                Grp::sync();
                account(2 * n);
            }
            gamma.x /= g;
            gamma.y /= g;
        }
    }

    // ---------------------------------------------------------- frame ops
    // src/clifft/svm/svm_kernels.inl:67-116,749-755
    __device__ __forceinline__ void frame_cnot(uint32_t c, uint32_t t) {
        int pxc = f.px(c), pzt = f.pz(t);
        Frame<NW>::flip(f.x, t, pxc);
        Frame<NW>::flip(f.z, c, pzt);
    }
    __device__ __forceinline__ void frame_cz(uint32_t c, uint32_t t) {
        int pxc = f.px(c), pxt = f.px(t);
        if (pxc & pxt) negate_gamma();
        Frame<NW>::flip(f.z, t, pxc);
        Frame<NW>::flip(f.z, c, pxt);
    }
    __device__ __forceinline__ void frame_h(uint32_t a) {
        int x = f.px(a), z = f.pz(a);
        if (x & z) negate_gamma();
        Frame<NW>::put(f.x, a, z);
        Frame<NW>::put(f.z, a, x);
    }
    __device__ __forceinline__ void frame_s(uint32_t a, bool dag) {
        int x = f.px(a);
        if (x) phase(make_double2(0.0, dag ? -1.0 : 1.0));
        Frame<NW>::flip(f.z, a, x);
    }
    __device__ __forceinline__ void frame_swap(uint32_t a, uint32_t b) {
        int xa = f.px(a), xb = f.px(b), za = f.pz(a), zb = f.pz(b);
        Frame<NW>::put(f.x, a, xb);
        Frame<NW>::put(f.x, b, xa);
        Frame<NW>::put(f.z, a, zb);
        Frame<NW>::put(f.z, b, za);
    }
    // A run of frame opcodes (FRAME_CNOT / CZ / H / S / S_DAG / SWAP: most of
    // a compiled Clifford circuit) executed with the frame and gamma in
    // registers and the next instruction word fetched one step ahead. The
    // updates and their order are those of the per-opcode handlers above.
    // Returns the first pc at or after `pc` that is not a frame opcode.
    __device__ __forceinline__ uint32_t frame_run(uint32_t pc, uint32_t n_instr) {
        if (pc >= n_instr) return pc;
        uint4 w = __ldg(P.instr + 2 * pc);
        if ((w.x & 0xffu) > CLIFFT_OP_FRAME_SWAP) return pc;
        Frame<NW> ff = f;
        double2 g = gamma;
        for (;;) {
            const uint32_t op = w.x & 0xffu;
            if (op > CLIFFT_OP_FRAME_SWAP) break;
            const uint32_t a = w.y & 0xffffu, b = w.y >> 16;
            const uint4 nxt = pc + 1 < n_instr ? __ldg(P.instr + 2 * (pc + 1)) : make_uint4(0xffu, 0u, 0u, 0u);
            const int xa = ff.px(a), xb = ff.px(b);
            switch (op) {
                case CLIFFT_OP_FRAME_CNOT:
                    Frame<NW>::flip(ff.x, b, xa);
                    Frame<NW>::flip(ff.z, a, ff.pz(b));
                    break;
                case CLIFFT_OP_FRAME_CZ:
                    if (xa & xb) g = make_double2(-g.x, -g.y);
                    Frame<NW>::flip(ff.z, b, xa);
                    Frame<NW>::flip(ff.z, a, xb);
                    break;
                case CLIFFT_OP_FRAME_H: {
                    const int za = ff.pz(a);
                    if (xa & za) g = make_double2(-g.x, -g.y);
                    Frame<NW>::put(ff.x, a, za);
                    Frame<NW>::put(ff.z, a, xa);
                    break;
                }
                case CLIFFT_OP_FRAME_S:
                case CLIFFT_OP_FRAME_S_DAG:
                    if (xa) g = dmul(g, make_double2(0.0, op == CLIFFT_OP_FRAME_S_DAG ? -1.0 : 1.0));
                    Frame<NW>::flip(ff.z, a, xa);
                    break;
                default: {  // FRAME_SWAP
                    const int za = ff.pz(a), zb = ff.pz(b);
                    Frame<NW>::put(ff.x, a, xb);
                    Frame<NW>::put(ff.x, b, xa);
                    Frame<NW>::put(ff.z, a, zb);
                    Frame<NW>::put(ff.z, b, za);
                    break;
                }
            }
            ++pc;
            w = nxt;
            if (pc >= n_instr) break;
        }
        f = ff;
        gamma = g;
        return pc;
    }

    // ---------------------------------------------------------- array ops
    // Generic sweeps (shared-memory statevectors, and global ones smaller than
    // a tile): one item per thread per step. Larger global statevectors stream
    // through the bulk-copy tile engine instead (stream_tiles), which keeps many
    // tiles in flight without holding them in registers.
    static constexpr int U = 1;

    template <class V, int UU = U, class Ld, class St>
    __device__ __forceinline__ void sweep(uint64_t n, Ld ld, St st) {
        const uint64_t step = (uint64_t)Grp::size();
        for (uint64_t i0 = Grp::rank(); i0 < n; i0 += step * UU) {
            V val[UU];
#pragma unroll
            for (int u = 0; u < UU; ++u)
                if (i0 + u * step < n) val[u] = ld(i0 + u * step);
#pragma unroll
            for (int u = 0; u < UU; ++u)
                if (i0 + u * step < n) st(val[u]);
        }
    }
    struct P2 {
        uint64_t i;
        T x, y;
    };
    struct P1 {
        uint64_t i;
        T x;
    };
    struct P4 {
        uint64_t i;
        T x0, x1, x2, x3;
    };

    // micro-op emission while resolving a fused block (thread 0 writes; every
    // thread computes the same values)
    using MOp = typename TC::MOp;
    __device__ __forceinline__ uint8_t local_bit(uint32_t axis) const {
        return reinterpret_cast<const uint8_t*>(fuse + fuse_lbit_offset())[axis];
    }
    static __host__ __device__ constexpr uint32_t fuse_bar_offset() { return TC::kBarOffset; }
    static __host__ __device__ constexpr uint32_t fuse_mops_offset() { return TC::kMopsOffset; }
    static __host__ __device__ constexpr uint32_t fuse_tables_offset() { return TC::kTablesOffset; }
    static __host__ __device__ constexpr uint32_t fuse_lbit_offset() { return TC::kLbitOffset; }
    // local image of an axis mask (its bits on tile axes)
    __device__ __forceinline__ uint32_t local_mask(uint64_t axes) const {
        uint32_t lm = 0;
        for (uint64_t w = axes & tileF; w; w &= w - 1) lm |= 1u << local_bit((uint32_t)__ffsll((long long)w) - 1);
        return lm;
    }
    // a, b: target axes (tile axes); req / par: condition axes (any);
    // coefficients c (nc complex values, converted to the statevector's
    // precision as the unfused handlers convert them)
    __device__ __forceinline__ void emit(uint8_t kind, uint32_t a, uint32_t b, uint64_t req, uint64_t par,
                                         uint8_t flags, const double* c, int nc) {
        MOp* m = reinterpret_cast<MOp*>(fuse + fuse_mops_offset()) + n_mops;
        if (Grp::rank() == 0) {
            m->kind = kind;
            m->a = local_bit(a);
            m->b = local_bit(b);
            m->flags = flags;
            m->req = local_mask(req);
            m->par = local_mask(par);
            m->greq = req & ~tileF;
            m->gpar = par & ~tileF;
        }
        // coefficients (up to 16 complex values of a U4 node) converted one
        // per thread: one global-load latency instead of a serial chain
        for (int j = Grp::rank(); j < nc; j += Grp::size()) m->c[j] = Cx<R>::make(c[2 * j], c[2 * j + 1]);
        n_mops++;
    }

    // exec_array_cnot (svm_kernels.inl:124-252)
    __device__ __forceinline__ void array_cnot(uint32_t c, uint32_t t) {
        const uint64_t n = 1ull << (k - 2), cb = 1ull << c, tb = 1ull << t;
        if (kTiles && resolving) {
            emit(M_CNOT, t, t, 1ull << c, 0, 0, nullptr, 0);
        } else {
            sweep<P2>(n, [&](uint64_t i) { P2 p; p.i = ins00(i, c, t) | cb; p.x = A(p.i); p.y = A(p.i | tb); return p; },
                      [&](const P2& p) { A(p.i) = p.y; A(p.i | tb) = p.x; });
            Grp::sync();
        }
        account(1ull << k);
        frame_cnot(c, t);
    }
    // exec_array_cz (svm_kernels.inl:255-365)
    __device__ __forceinline__ void array_cz(uint32_t c, uint32_t t) {
        const uint64_t n = 1ull << (k - 2), both = (1ull << c) | (1ull << t);
        if (kTiles && resolving) {
            emit(M_CZ, c, t, (1ull << c) | (1ull << t), 0, 0, nullptr, 0);
        } else {
            sweep<P1>(n, [&](uint64_t i) { P1 p; p.i = ins00(i, c, t) | both; p.x = A(p.i); return p; },
                      [&](const P1& p) { A(p.i) = cneg(p.x); });
            Grp::sync();
        }
        account(1ull << (k - 1));
        frame_cz(c, t);
    }
    // exec_array_swap (svm_kernels.inl:369-458)
    __device__ __forceinline__ void array_swap(uint32_t a, uint32_t b) {
        const uint64_t n = 1ull << (k - 2), ab = 1ull << a, bb = 1ull << b;
        if (kTiles && resolving) {
            emit(M_SWAP, a, b, 0, 0, 0, nullptr, 0);
        } else {
            sweep<P2>(n, [&](uint64_t i) { P2 p; p.i = ins00(i, a, b); p.x = A(p.i | ab); p.y = A(p.i | bb); return p; },
                      [&](const P2& p) { A(p.i | ab) = p.y; A(p.i | bb) = p.x; });
            Grp::sync();
        }
        account(1ull << k);
        frame_swap(a, b);
    }
    // exec_array_multi_cnot (svm_kernels.inl:464-550)
    __device__ __forceinline__ void array_multi_cnot(uint32_t t, uint64_t mask) {
        const uint64_t n = 1ull << (k - 1), tb = 1ull << t;
        if (kTiles && resolving) {
            emit(M_MCNOT, t, t, 0, mask & ~tb, MF_PARITY, nullptr, 0);
        } else {
            sweep<P2>(n,
                      [&](uint64_t i) {
                          P2 p;
                          p.i = ins0(i, t);
                          if (__popcll(p.i & mask) & 1) {
                              p.x = A(p.i);
                              p.y = A(p.i | tb);
                          } else {
                              p.i = ~0ull;
                          }
                          return p;
                      },
                      [&](const P2& p) {
                          if (p.i != ~0ull) {
                              A(p.i) = p.y;
                              A(p.i | tb) = p.x;
                          }
                      });
            Grp::sync();
        }
        account(1ull << k);
        for (uint32_t c = 0; c < k; ++c)
            if ((mask >> c) & 1ull) frame_cnot(c, t);
    }
    // exec_array_multi_cz (svm_kernels.inl:558-635)
    __device__ __forceinline__ void array_multi_cz(uint32_t c, uint64_t mask) {
        const uint64_t n = 1ull << (k - 1), cb = 1ull << c;
        if (kTiles && resolving) {
            emit(M_MCZ, c, c, cb, mask, MF_PARITY, nullptr, 0);
        } else {
            sweep<P1>(n,
                      [&](uint64_t i) {
                          P1 p;
                          p.i = ins0(i, c) | cb;
                          if (__popcll(p.i & mask) & 1)
                              p.x = A(p.i);
                          else
                              p.i = ~0ull;
                          return p;
                      },
                      [&](const P1& p) {
                          if (p.i != ~0ull) A(p.i) = cneg(p.x);
                      });
            Grp::sync();
        }
        account(1ull << k);
        for (uint32_t t = 0; t < k; ++t)
            if ((mask >> t) & 1ull) frame_cz(c, t);
    }
    // exec_array_h (svm_kernels.inl:639-744): (a +- b) / sqrt(2)
    __device__ __forceinline__ void array_h(uint32_t a) {
        const uint64_t n = 1ull << (k - 1), ab = 1ull << a;
        const R s = (R)CGPU_INV_SQRT2;
        if (kTiles && resolving) {
            emit(M_H, a, a, 0, 0, 0, nullptr, 0);
        } else {
            sweep<P2>(n, [&](uint64_t i) { P2 p; p.i = ins0(i, a); p.x = A(p.i); p.y = A(p.i | ab); return p; },
                      [&](const P2& p) {
                          A(p.i) = cscale(cadd(p.x, p.y), s);
                          A(p.i | ab) = cscale(csub(p.x, p.y), s);
                      });
            Grp::sync();
        }
        account(2ull << k);
        frame_h(a);
    }
    // apply_phase_waterfall (svm_kernels.inl:764-830)
    __device__ __forceinline__ void phase_sweep(uint32_t a, double re, double im) {
        const uint64_t n = 1ull << (k - 1), ab = 1ull << a;
        if (kTiles && resolving) {
            const double c[2] = {re, im};
            emit(M_PHASE, a, a, ab, 0, 0, c, 1);
        } else {
            const T ph = Cx<R>::make(re, im);
            sweep<P1>(n, [&](uint64_t i) { P1 p; p.i = ins0(i, a) | ab; p.x = A(p.i); return p; },
                      [&](const P1& p) { A(p.i) = cmul(p.x, ph); });
            Grp::sync();
        }
        account(1ull << k);
    }
    // exec_array_t / t_dag / rot (svm_kernels.inl:951-988,1044-1061)
    __device__ __forceinline__ void array_rot(uint32_t a, double zr, double zi) {
        int x = f.px(a);
        if (a >= k) {
            if (x) phase(make_double2(zr, zi));
            return;
        }
        if (x) {
            phase_sweep(a, zr, -zi);
            phase(make_double2(zr, zi));
        } else {
            phase_sweep(a, zr, zi);
        }
    }
    // Threads that compute on tiles in a fused block (the whole group, or
    // every warp but the copy warp of a warp-specialised CTA) and their barrier.
    static __device__ __forceinline__ int compute_threads() {
        return Grp::kWS ? (int)blockDim.x - 32 : Grp::size();
    }
    static __device__ __forceinline__ void csync() {
        if constexpr (Grp::kWS)
            bar_sync_first(blockDim.x - 32u);
        else
            Grp::sync();
    }
    // Statevector passes of a one-shot group with a global-memory statevector
    // larger than one tile go through the bulk-copy tile engine.
    __device__ __forceinline__ bool tiled(uint32_t kk) const {
        return kTiles && fuse != nullptr && kk > (uint32_t)TC::kBits;
    }
    // one run per tile covering the lowest TILE_BITS axes
    __device__ __forceinline__ void set_runs_low() {
        if (Grp::rank() == 0) reinterpret_cast<uint64_t*>(fuse + fuse_tables_offset())[0] = 0;
    }
    // run offsets of a tile over axes F (2^(TILE_BITS - r) runs of 2^r amplitudes)
    __device__ __forceinline__ void set_runs(uint64_t F, uint32_t r) {
        uint64_t* runoff = reinterpret_cast<uint64_t*>(fuse + fuse_tables_offset());
        for (int j = Grp::rank(); j < (1 << (TC::kBits - r)); j += Grp::size())
            runoff[j] = pdep((uint64_t)j << r, F);
    }

    // exec_expand / expand_with_phase / exec_expand_{t,t_dag,rot}
    // (svm_kernels.inl:876-1081)
    __device__ __forceinline__ void expand(uint32_t a, bool with_phase, double zr, double zi) {
        const uint64_t half = 1ull << k;
        int x = with_phase ? f.px(a) : 0;
        const T ph = Cx<R>::make(with_phase ? zr : 1.0, with_phase ? (x ? -zi : zi) : 0.0);
        if (kTiles && resolving) {
            // inside a fused block: the new axis is a tile axis and the copy a micro-op
            const double c[2] = {with_phase ? zr : 1.0, with_phase ? (x ? -zi : zi) : 0.0};
            emit(M_EXPAND, a, a, 0, 0, with_phase ? 0 : MF_COPY, c, 1);
            bytes += (2ull << k) * sizeof(T);
            k++;
            scale_magnitude(CGPU_EXPAND_SCALE);
            if (with_phase && x) phase(make_double2(zr, zi));
            return;
        }
        if (tiled(k)) {
            if constexpr (kTiles) {
                constexpr uint32_t MB = TC::kBits, TN = 1u << MB;
                set_runs_low();
                const int tid = Grp::rank(), nthr = Grp::size();
                cur_site = 1;
                stream_tiles(half >> MB, (half - 1) & ~(uint64_t)(TN - 1), MB, 0, half, 1, 0,
                             [&](T* buf, uint64_t, uint64_t) {
                    if (with_phase)
                        for (uint32_t l = tid; l < TN; l += nthr) buf[l] = cmul(buf[l], ph);
                    Grp::sync();
                });
                moved += (2ull << k) * sizeof(T);
                bytes += (2ull << k) * sizeof(T);
                k++;
                scale_magnitude(CGPU_EXPAND_SCALE);
                if (with_phase && x) phase(make_double2(zr, zi));
                return;
            }
        }
        if (!with_phase) {
            sweep<P1>(half, [&](uint64_t i) { P1 p; p.i = i; p.x = A(i); return p; },
                      [&](const P1& p) { A(half + p.i) = p.x; });
        } else {
            sweep<P1>(half, [&](uint64_t i) { P1 p; p.i = i; p.x = A(i); return p; },
                      [&](const P1& p) { A(half + p.i) = cmul(p.x, ph); });
        }
        Grp::sync();
        account(2ull << k);
        k++;
        scale_magnitude(CGPU_EXPAND_SCALE);
        if (with_phase && x) phase(make_double2(zr, zi));
    }
    // exec_array_u2 (svm_kernels.inl:1087-1297)
    __device__ __forceinline__ void array_u2(uint32_t a, uint32_t cp) {
        const double* node = P.u2 + (size_t)cp * CLIFFT_U2_DOUBLES_PER_NODE;
        int st = (f.pz(a) << 1) | f.px(a);
        const double* m = node + st * 10;
        phase(make_double2(m[8], m[9]));
        uint8_t out = P.u2_out[cp * 4 + st];
        Frame<NW>::put(f.x, a, out & 1);
        Frame<NW>::put(f.z, a, (out >> 1) & 1);
        if (a >= k) return;
        if (kTiles && resolving) {
            emit(M_U2, a, a, 0, 0, 0, m, 4);
            account(2ull << k);
            return;
        }
        const T m00 = Cx<R>::make(m[0], m[1]), m01 = Cx<R>::make(m[2], m[3]);
        const T m10 = Cx<R>::make(m[4], m[5]), m11 = Cx<R>::make(m[6], m[7]);
        const uint64_t n = 1ull << (k - 1), ab = 1ull << a;
        sweep<P2>(n, [&](uint64_t i) { P2 p; p.i = ins0(i, a); p.x = A(p.i); p.y = A(p.i | ab); return p; },
                  [&](const P2& p) {
                      A(p.i) = cmac(cmul(m00, p.x), m01, p.y);
                      A(p.i | ab) = cmac(cmul(m10, p.x), m11, p.y);
                  });
        Grp::sync();
        account(2ull << k);
    }
    // exec_array_u4 (svm_kernels.inl:1310-1531)
    __device__ __forceinline__ void array_u4(uint32_t lo, uint32_t hi, uint32_t cp) {
        const double* node = P.u4 + (size_t)cp * CLIFFT_U4_DOUBLES_PER_NODE;
        int st = (f.pz(hi) << 3) | (f.px(hi) << 2) | (f.pz(lo) << 1) | f.px(lo);
        const double* e = node + st * 34;
        phase(make_double2(e[32], e[33]));
        uint8_t out = P.u4_out[cp * 16 + st];
        Frame<NW>::put(f.x, lo, out & 1);
        Frame<NW>::put(f.z, lo, (out >> 1) & 1);
        Frame<NW>::put(f.x, hi, (out >> 2) & 1);
        Frame<NW>::put(f.z, hi, (out >> 3) & 1);
        if (kTiles && resolving) {
            emit(M_U4, lo, hi, 0, 0, 0, e, 16);
            account(2ull << k);
            return;
        }
        const uint64_t n = 1ull << (k - 2), lb = 1ull << lo, hb = 1ull << hi;
        T m[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) m[j] = Cx<R>::make(e[2 * j], e[2 * j + 1]);
        sweep<P4, (U > 2 ? 2 : U)>(n,
                  [&](uint64_t i) {
                      P4 p;
                      p.i = ins00(i, lo, hi);
                      p.x0 = A(p.i);
                      p.x1 = A(p.i | lb);
                      p.x2 = A(p.i | hb);
                      p.x3 = A(p.i | lb | hb);
                      return p;
                  },
                  [&](const P4& p) {
                      T y[4];
#pragma unroll
                      for (int r = 0; r < 4; ++r) {
                          T acc = cmul(m[r * 4 + 0], p.x0);
                          acc = cmac(acc, m[r * 4 + 1], p.x1);
                          acc = cmac(acc, m[r * 4 + 2], p.x2);
                          acc = cmac(acc, m[r * 4 + 3], p.x3);
                          y[r] = acc;
                      }
                      A(p.i) = y[0];
                      A(p.i | lb) = y[1];
                      A(p.i | hb) = y[2];
                      A(p.i | lb | hb) = y[3];
                  });
        Grp::sync();
        account(2ull << k);
    }

    // ------------------------------------------------------- measurements
    // Outcome selection shared by sampling and forced modes: sample_branch
    // (src/clifft/svm/svm_internal.h:65-79) and forced_log_increment
    // (src/clifft/svm/svm_forced_kernels.cc:42-60). `want` is the forced
    // branch or -1. Returns the branch, or -1 when the forced branch is
    // unreachable.
    __device__ __forceinline__ int choose(double p0, double p1, double total, int want, double* prob) {
        const double eps = K.dust_eps * total;
        if (p1 <= eps) {
            if (p1 > 0.0) dust++;
            *prob = 1.0;
            return want <= 0 ? 0 : -1;
        }
        if (p0 <= eps) {
            if (p0 > 0.0) dust++;
            *prob = 1.0;
            return (want < 0 || want == 1) ? 1 : -1;
        }
        if (want < 0) {
            double r = uniform();
            int b = (r * total < p0) ? 0 : 1;
            *prob = (b ? p1 : p0) / total;
            return b;
        }
        double pb = (want ? p1 : p0) / total;
        log_prob += log(pb);
        *prob = pb;
        return want;
    }

    __device__ __forceinline__ int forced_bit(uint32_t idx) const { return forced ? (int)forced[idx] : -1; }

    // exec_meas_dormant_static + FLAG_IDENTITY shortcut (svm_kernels.inl:1539-1545,
    // 2361-2369) and forced variants (svm_forced_kernels.cc:64-88)
    __device__ __forceinline__ void meas_dormant_static(uint32_t a, uint32_t idx, int sign, bool identity) {
        int det_bit = identity ? sign : (f.px(a) ^ sign);
        int want = forced_bit(idx);
        if (want >= 0 && want != det_bit) {
            reachable = false;
            stop = true;
            return;
        }
        write_meas(idx, det_bit, 1.0);
    }
    // exec_meas_dormant_random (svm_kernels.inl:1550-1566), forced
    // (svm_forced_kernels.cc:90-110)
    __device__ __forceinline__ void meas_dormant_random(uint32_t a, uint32_t idx, int sign) {
        int want = forced_bit(idx);
        int m_abs;
        if (want >= 0) {
            m_abs = want ^ sign;
            log_prob += log(0.5);
        } else {
            m_abs = uniform() < 0.5 ? 0 : 1;
        }
        if (f.px(a) && m_abs) negate_gamma();
        Frame<NW>::put(f.x, a, m_abs);
        Frame<NW>::put(f.z, a, 0);
        write_meas(idx, m_abs ^ sign, 0.5);
    }
    __device__ __forceinline__ bool zero_norm(double total) {
        if (!(total > 0.0)) {
            if (Grp::rank() == 0) atomicCAS(K.error_word, 0, DEV_ERR_ZERO_NORM);
            stop = true;
            return true;
        }
        return false;
    }
    // exec_meas_active_diagonal (svm_kernels.inl:1573-1627), forced
    // (svm_forced_kernels.cc:112-158)
    __device__ __forceinline__ void meas_diagonal(uint32_t a, uint32_t idx, int sign) {
        const uint64_t half = 1ull << (k - 1);
        double acc[2] = {0.0, 0.0};
        const bool tl = tiled(k);
        if (tl) {
            if constexpr (kTiles) {
                constexpr uint32_t MB = TC::kBits, TN = 1u << MB;
                set_runs_low();
                const int tid = Grp::rank(), nthr = Grp::size();
                const uint64_t ntiles = 1ull << (k - MB);
                cur_site = 2;
                stream_tiles(ntiles, ((1ull << k) - 1) & ~(uint64_t)(TN - 1), MB, 0, 0, 0, 0,
                             [&](T* buf, uint64_t t, uint64_t) {
                                 double q = 0.0;
                                 for (uint32_t l = tid; l < TN; l += nthr) q += cnorm_d(buf[l]);
                                 if (t >= ntiles / 2)
                                     acc[1] += q;
                                 else
                                     acc[0] += q;
                                 Grp::sync();
                             });
                moved += (1ull << k) * sizeof(T);
            }
        } else {
            const uint64_t step = (uint64_t)Grp::size();
            for (uint64_t i0 = Grp::rank(); i0 < half; i0 += step * U) {
                T x[U], y[U];
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (i0 + u * step < half) {
                        x[u] = A(i0 + u * step);
                        y[u] = A(i0 + u * step + half);
                    }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (i0 + u * step < half) {
                        acc[0] += cnorm_d(x[u]);
                        acc[1] += cnorm_d(y[u]);
                    }
            }
        }
        group_reduce<Grp, 2>(acc, red);
        if (tl)
            bytes += (1ull << k) * sizeof(T);
        else
            account(1ull << k);
        diag_tail(a, idx, sign, acc[0], acc[1], false);
    }
    // Outcome, collapse and bookkeeping of a diagonal measurement of axis
    // a = k-1 with half-norms p0 (bit a clear) and p1. relabel: the state
    // was summed by a fused block and the b = 1 half becomes the state by
    // flipping the address label; otherwise it is copied down (the
    // reference's step, counted in the algorithmic bytes either way).
    __device__ __forceinline__ void diag_tail(uint32_t a, uint32_t idx, int sign, double p0, double p1, bool relabel) {
        const uint64_t half = 1ull << (k - 1);
        const int pxv = f.px(a), pzv = f.pz(a);
        const double total = p0 + p1;
        if (zero_norm(total)) return;
        int want = forced_bit(idx);
        if (want >= 0) want = want ^ sign ^ pxv;
        double prob;
        int b = choose(p0, p1, total, want, &prob);
        if (b < 0) {
            reachable = false;
            stop = true;
            return;
        }
        int m_abs = b ^ pxv;
        if (b == 1 && pzv) negate_gamma();
        if (b == 1) {
            if (relabel) {
                if constexpr (kTiles) xo ^= half;
                bytes += (1ull << k) * sizeof(T);
            } else if (tiled(k)) {
                if constexpr (kTiles) {
                    constexpr uint32_t MB = TC::kBits, TN = 1u << MB;
                    set_runs_low();
                    cur_site = 3;
                    stream_tiles(half >> MB, (half - 1) & ~(uint64_t)(TN - 1), MB, half, 0, 1, 0,
                                 [&](T*, uint64_t, uint64_t) { Grp::sync(); });
                    moved += (1ull << k) * sizeof(T);
                    bytes += (1ull << k) * sizeof(T);
                }
            } else {
                sweep<P1>(half, [&](uint64_t i) { P1 p; p.i = i; p.x = A(i + half); return p; },
                          [&](const P1& p) { A(p.i) = p.x; });
                Grp::sync();
                account(1ull << k);
            }
        }
        k--;
        double pb = b ? p1 : p0;
        if (forced || pb > 0.0) scale_magnitude(sqrt(total / pb));
        Frame<NW>::put(f.x, a, m_abs);
        Frame<NW>::put(f.z, a, 0);
        write_meas(idx, m_abs ^ sign, prob);
    }
    // exec_meas_active_interfere (svm_kernels.inl:1634-1708) and
    // exec_swap_meas_interfere (svm_kernels.inl:1728-1804) with their forced
    // variants (svm_forced_kernels.cc:160-304). With a fused swap (f != t)
    // the fold runs in two passes over disjoint outputs (bit f clear, then
    // set) because the f-clear outputs read lower-half inputs that f-set
    // outputs overwrite; the reference serialises this loop instead.
    __device__ __forceinline__ void meas_interfere(uint32_t fa, uint32_t t, uint32_t idx, int sign) {
        const bool swapped = fa != t;
        if (swapped) frame_swap(fa, t);
        const uint64_t half = 1ull << t, fb = 1ull << fa;
        double acc[2] = {0.0, 0.0};
        // tiled path: the tile spans axes {fa, t} (t is its top local bit);
        // outputs are the tile positions with the t bit clear
        const bool tl = tiled(k);
        uint32_t tr = 0, lf = 0;
        uint64_t tC = 0;
        if (tl) {
            if constexpr (kTiles) {
                constexpr uint32_t MB = TC::kBits;
                const uint64_t F = tile_axes((1ull << t) | fb, tr);
                tC = ((1ull << k) - 1) & ~F;
                lf = (uint32_t)__popcll(F & (fb - 1));
                set_runs(F, tr);
                const int tid = Grp::rank(), nthr = Grp::size();
                const uint32_t lt = MB - 1, lfb = 1u << lf, HN = 1u << lt;
                cur_site = 4;
                stream_tiles(1ull << (k - MB), tC, tr, 0, 0, 0, 0, [&](T* buf, uint64_t, uint64_t) {
                    double qp = 0.0, qm = 0.0;
                    for (uint32_t l = tid; l < HN; l += nthr) {
                        uint32_t a0 = swapped ? ((l & ~lfb) | (((l >> lf) & 1u) << lt)) : l;
                        uint32_t a1 = swapped ? (a0 | lfb) : (l + HN);
                        T x = buf[a0], y = buf[a1];
                        qp += cnorm_d(cadd(x, y));
                        qm += cnorm_d(csub(x, y));
                    }
                    acc[0] += qp;
                    acc[1] += qm;
                    Grp::sync();
                });
                moved += (1ull << k) * sizeof(T);
            }
        } else {
            const uint64_t step = (uint64_t)Grp::size();
            for (uint64_t i0 = Grp::rank(); i0 < half; i0 += step * U) {
                T x[U], y[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint64_t i = i0 + u * step;
                    if (i < half) {
                        uint64_t a0 = swapped ? ((i & ~fb) | (((i >> fa) & 1ull) << t)) : i;
                        uint64_t a1 = swapped ? (a0 | fb) : (i + half);
                        x[u] = A(a0);
                        y[u] = A(a1);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (i0 + u * step < half) {
                        acc[0] += cnorm_d(cadd(x[u], y[u]));
                        acc[1] += cnorm_d(csub(x[u], y[u]));
                    }
            }
        }
        group_reduce<Grp, 2>(acc, red);
        if (tl)
            bytes += ((1ull << k) * 2 + (1ull << (k - 1))) * sizeof(T);
        else
            account((1ull << k) * 2 + (1ull << (k - 1)));
        const int pxv = f.px(t), pzv = f.pz(t);
        const double pp = acc[0], pm = acc[1], total = pp + pm;
        if (zero_norm(total)) return;
        int want = forced_bit(idx);
        if (want >= 0) want = want ^ sign ^ pzv;
        double prob;
        int bx = choose(pp, pm, total, want, &prob);
        if (bx < 0) {
            reachable = false;
            stop = true;
            return;
        }
        const R s = (R)CGPU_INV_SQRT2;
        if (tl) {
            if constexpr (kTiles) {
                constexpr uint32_t MB = TC::kBits;
                const int tid = Grp::rank(), nthr = Grp::size();
                const uint32_t lt = MB - 1, lfb = 1u << lf, HN = 1u << lt;
                const uint32_t nruns = 1u << (MB - tr);
                cur_site = 5;
                stream_tiles(1ull << (k - MB), tC, tr, 0, 0, nruns / 2, 0, [&](T* buf, uint64_t, uint64_t) {
                    if (!swapped) {
                        for (uint32_t l = tid; l < HN; l += nthr) {
                            T x = buf[l], y = buf[l + HN];
                            buf[l] = cscale(bx ? csub(x, y) : cadd(x, y), s);
                        }
                        Grp::sync();
                    } else {
                        // outputs with the fa bit clear read positions the fa-set outputs overwrite
                        for (int pass = 0; pass < 2; ++pass) {
                            for (uint32_t j = tid; j < HN / 2; j += nthr) {
                                uint32_t l = ins0_32(j, lf) | (pass ? lfb : 0u);
                                uint32_t a0 = pass ? ((l & ~lfb) | HN) : l;
                                T x = buf[a0], y = buf[a0 | lfb];
                                buf[l] = cscale(bx ? csub(x, y) : cadd(x, y), s);
                            }
                            Grp::sync();
                        }
                    }
                });
                moved += (1ull << k) * sizeof(T) + (1ull << (k - 1)) * sizeof(T);
            }
        } else if (!swapped) {
            sweep<P2>(half, [&](uint64_t i) { P2 p; p.i = i; p.x = A(i); p.y = A(i + half); return p; },
                      [&](const P2& p) { A(p.i) = cscale(bx ? csub(p.x, p.y) : cadd(p.x, p.y), s); });
            Grp::sync();
        } else {
            const uint64_t q = half >> 1;  // outputs with bit fa clear, then set
            for (int pass = 0; pass < 2; ++pass) {
                sweep<P2>(q,
                          [&](uint64_t j) {
                              P2 p;
                              p.i = ins0(j, fa) | (pass ? fb : 0ull);
                              uint64_t a0 = pass ? ((p.i & ~fb) | half) : p.i;
                              p.x = A(a0);
                              p.y = A(a0 | fb);
                              return p;
                          },
                          [&](const P2& p) { A(p.i) = cscale(bx ? csub(p.x, p.y) : cadd(p.x, p.y), s); });
                Grp::sync();
            }
        }
        interfere_tail(swapped, t, idx, sign, pxv, pzv, bx, pp, pm, prob);
    }
    // Bookkeeping of an X-basis measurement of axis t = k-1 after its fold:
    // branch bx with pp / pm the +/- branch weights.
    __device__ __forceinline__ void interfere_tail(bool swapped, uint32_t t, uint32_t idx, int sign, int pxv, int pzv,
                                                   int bx, double pp, double pm, double prob) {
        const int m_abs = bx ^ pzv;
        const double pb = bx ? pm : pp, total = pp + pm;
        if (!swapped) {
            if (pxv && m_abs) negate_gamma();
            k--;
            if (forced || pb > 0.0) scale_magnitude(sqrt(total / pb));
        } else {
            k--;
            if (forced || pb > 0.0) scale_magnitude(sqrt(total / pb));
            if (pxv && m_abs) negate_gamma();
        }
        Frame<NW>::put(f.x, t, m_abs);
        Frame<NW>::put(f.z, t, 0);
        write_meas(idx, m_abs ^ sign, prob);
    }
    // The measurement that ends a fused block: the block already applied the
    // fold's arithmetic as micro-ops (SWAP f<->t if fused, then H on t, so the
    // bit-t clear half holds (x + y) / sqrt2 and the set half (x - y) / sqrt2)
    // and summed the two halves' norms (w0 bit t clear, w1 set; each 1/2 of
    // the reference's |x +- y|^2 sums, which leaves every ratio unchanged).
    // Branch bx keeps the half with bit t = bx: the address label flips for
    // bx = 1. Diagonal measurements go to diag_tail.
    __device__ __forceinline__ void interfere_relabel(uint32_t fa, uint32_t t, uint32_t idx, int sign, double w0,
                                                      double w1) {
        const bool swapped = fa != t;
        if (swapped) frame_swap(fa, t);
        bytes += ((1ull << k) * 2 + (1ull << (k - 1))) * sizeof(T);
        const int pxv = f.px(t), pzv = f.pz(t);
        const double total = w0 + w1;
        if (zero_norm(total)) return;
        int want = forced_bit(idx);
        if (want >= 0) want = want ^ sign ^ pzv;
        double prob;
        const int bx = choose(w0, w1, total, want, &prob);
        if (bx < 0) {
            reachable = false;
            stop = true;
            return;
        }
        if (bx == 1) {
            if constexpr (kTiles) xo ^= 1ull << t;
        }
        interfere_tail(swapped, t, idx, sign, pxv, pzv, bx, w0, w1, prob);
    }

    // ------------------------------------------------- classical / noise
    // apply_pauli_to_frame (svm_kernels.inl:1812-1865)
    __device__ __forceinline__ void apply_pauli(const uint64_t* ex, const uint64_t* ez, int sign) {
        int par = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) par += __popcll(f.x[w] & __ldg(ez + w));
        if (par & 1) negate_gamma();
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            f.x[w] ^= __ldg(ex + w);
            f.z[w] ^= __ldg(ez + w);
        }
        if (sign) negate_gamma();
    }
    // SchrodingerState::draw_next_noise (src/clifft/svm/svm.h:231-248)
    __device__ __forceinline__ void draw_next_noise() {
        const uint32_t n = P.n_sites;
        if (n == 0 || next_noise >= n) {
            next_noise = 0xffffffffu;
            return;
        }
        double cur = next_noise == 0 ? 0.0 : __ldg(P.hazards + next_noise - 1);
        double gap = -log(1.0 - uniform());
        double target = cur + gap;
        uint32_t lo = next_noise, hi = n;  // hazards are cumulative: answer >= next_noise
        while (lo < hi) {
            uint32_t mid = lo + ((hi - lo) >> 1);
            if (__ldg(P.hazards + mid) > target)
                hi = mid;
            else
                lo = mid + 1;
        }
        next_noise = lo;
    }
    // exec_noise (svm_kernels.inl:1886-1921)
    __device__ __forceinline__ void noise(uint32_t site) {
        if (site != next_noise) return;
        const uint32_t c0 = __ldg(P.site_off + site), c1 = __ldg(P.site_off + site + 1);
        if (K.flags & KF_FORCED_FAULTS) {
            uint32_t c = c0 + K.fault_chan[ff_pos - 1];
            if (c < c1) apply_pauli(P.chan_x + (size_t)c * NW, P.chan_z + (size_t)c * NW, 0);
            next_noise = ff_pos < ff_end ? K.fault_sites[ff_pos++] : 0xffffffffu;
            return;
        }
        double r = uniform() * __ldg(P.site_psum + site), cum = 0.0;
        for (uint32_t c = c0; c < c1; ++c) {
            cum += __ldg(P.chan_prob + c);
            if (r < cum) {
                apply_pauli(P.chan_x + (size_t)c * NW, P.chan_z + (size_t)c * NW, 0);
                break;
            }
        }
        next_noise++;
        draw_next_noise();
    }
    // exec_readout_noise (svm_kernels.inl:1937-1959)
    __device__ __forceinline__ void readout_noise(uint32_t e) {
        bool fire = false;
        if (K.flags & KF_FORCED_FAULTS) {
            if (ro_pos < ro_end && K.ro_entries[ro_pos] == e) {
                fire = true;
                ro_pos++;
            }
        } else {
            fire = uniform() < __ldg(P.ro_prob + e);
        }
        if (fire) {
            flush_records();
            uint32_t mi = __ldg(P.ro_meas + e);
            if (Grp::rank() == 0) rec[(mi >> 5) * S] ^= 1u << (mi & 31);
            rec_dirty = true;
        }
    }
    __device__ __forceinline__ int list_parity(const uint32_t* off, const uint32_t* tg, uint32_t l) {
        int p = 0;
        const uint32_t e = __ldg(off + l + 1);
        for (uint32_t i = __ldg(off + l); i < e; ++i) p ^= bit_of(rec, __ldg(tg + i), S);
        return p;
    }
    // exec_exp_val (svm_kernels.inl:2031-2173)
    __device__ __forceinline__ void exp_val(uint32_t cp, uint32_t out_idx) {
        const uint64_t* mx = P.exp_x + (size_t)cp * NW;
        const uint64_t* mz = P.exp_z + (size_t)cp * NW;
        int fsign = P.exp_sign[cp] != 0;
        int par = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) par += __popcll(mx[w] & f.z[w]) + __popcll(mz[w] & f.x[w]);
        if (par & 1) fsign ^= 1;
        // any X / Y support on a dormant axis (>= k) gives <P> = 0
        bool dormant_x = false;
        const uint32_t full = k >> 6, rem = k & 63;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            if ((uint32_t)w < full) continue;
            uint64_t mw = mx[w];
            if ((uint32_t)w == full && rem) mw &= ~((1ull << rem) - 1);
            if (mw) dormant_x = true;
        }
        double result = 0.0;
        if (!dormant_x) {
            const uint64_t am = k == 64 ? ~0ull : ((1ull << k) - 1);
            const uint64_t xa = mx[0] & am, za = mz[0] & am;
            const int yz = __popcll(xa & za) & 3;
            double2 iph = make_double2(yz == 0 ? 1.0 : (yz == 2 ? -1.0 : 0.0),
                                       yz == 1 ? 1.0 : (yz == 3 ? -1.0 : 0.0));
            if (fsign) iph = make_double2(-iph.x, -iph.y);
            double acc[3] = {0.0, 0.0, 0.0};
            const uint64_t dim = 1ull << k;
            const uint64_t step = (uint64_t)Grp::size();
            for (uint64_t j0 = Grp::rank(); j0 < dim; j0 += step * U) {
                T av[U], bv[U];
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (j0 + u * step < dim) {
                        av[u] = A(j0 + u * step);
                        bv[u] = A((j0 + u * step) ^ xa);
                    }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint64_t j = j0 + u * step;
                    if (j < dim) {
                        double ar = (double)av[u].x, ai = (double)av[u].y;
                        double br = (double)bv[u].x, bi = -(double)bv[u].y;
                        acc[2] = __dadd_rn(acc[2], __fma_rn(ar, ar, __dmul_rn(ai, ai)));
                        double zs = (__popcll(j & za) & 1) ? -1.0 : 1.0;
                        ar *= zs;
                        ai *= zs;
                        acc[0] = __dadd_rn(acc[0], __fma_rn(br, ar, -__dmul_rn(bi, ai)));
                        acc[1] = __dadd_rn(acc[1], __fma_rn(br, ai, __dmul_rn(bi, ar)));
                    }
                }
            }
            group_reduce<Grp, 3>(acc, red);
            account(1ull << k);
            double2 num = dmul(make_double2(acc[0], acc[1]), iph);
            if (acc[2] > 0.0) result = num.x / acc[2];
            result = fmin(1.0, fmax(-1.0, result));
        }
        if (Grp::rank() == 0 && K.out_exp) K.out_exp[shot * P.num_exp + out_idx] = result;
    }

    // Executes instruction `pc` (the dispatch of execute_internal,
    // svm_kernels.inl:2183-2646; forced opcodes share the sampling handlers).
    __device__ __forceinline__ void exec(uint32_t pc) {
        cur_pc = pc;
        const uint4* ip = P.instr;
        const uint4 w0 = __ldg(ip + 2 * pc);
        uint32_t op = w0.x & 0xffu;
        const uint32_t fl = (w0.x >> 16) & 0xffu;
        const uint32_t a1 = w0.y & 0xffffu, a2 = w0.y >> 16;
        const uint32_t p0 = w0.z, p1 = w0.w;
        const int sign = (fl & CLIFFT_FLAG_SIGN) ? 1 : 0;
        if (op >= CLIFFT_OP_MEAS_DORMANT_STATIC_FORCED && op <= CLIFFT_OP_SWAP_MEAS_INTERFERE_FORCED)
            op -= CLIFFT_OP_MEAS_DORMANT_STATIC_FORCED - CLIFFT_OP_MEAS_DORMANT_STATIC;
            switch (op) {
            case CLIFFT_OP_FRAME_CNOT: frame_cnot(a1, a2); break;
            case CLIFFT_OP_FRAME_CZ: frame_cz(a1, a2); break;
            case CLIFFT_OP_FRAME_H: frame_h(a1); break;
            case CLIFFT_OP_FRAME_S: frame_s(a1, false); break;
            case CLIFFT_OP_FRAME_S_DAG: frame_s(a1, true); break;
            case CLIFFT_OP_FRAME_SWAP: frame_swap(a1, a2); break;
            case CLIFFT_OP_ARRAY_CNOT: array_cnot(a1, a2); break;
            case CLIFFT_OP_ARRAY_CZ: array_cz(a1, a2); break;
            case CLIFFT_OP_ARRAY_SWAP: array_swap(a1, a2); break;
            case CLIFFT_OP_ARRAY_MULTI_CNOT: array_multi_cnot(a1, ((uint64_t)p1 << 32) | p0); break;
            case CLIFFT_OP_ARRAY_MULTI_CZ: array_multi_cz(a1, ((uint64_t)p1 << 32) | p0); break;
            case CLIFFT_OP_ARRAY_H: array_h(a1); break;
            case CLIFFT_OP_ARRAY_S:
                phase_sweep(a1, 0.0, 1.0);
                frame_s(a1, false);
                break;
            case CLIFFT_OP_ARRAY_S_DAG:
                phase_sweep(a1, 0.0, -1.0);
                frame_s(a1, true);
                break;
            case CLIFFT_OP_ARRAY_T: array_rot(a1, CGPU_INV_SQRT2, CGPU_INV_SQRT2); break;
            case CLIFFT_OP_ARRAY_T_DAG: array_rot(a1, CGPU_INV_SQRT2, -CGPU_INV_SQRT2); break;
            case CLIFFT_OP_ARRAY_ROT: {
                const uint4 w1 = __ldg(ip + 2 * pc + 1);
                array_rot(a1, __longlong_as_double(((long long)p1 << 32) | p0),
                          __longlong_as_double(((long long)w1.y << 32) | w1.x));
                break;
            }
            case CLIFFT_OP_ARRAY_U2: array_u2(a1, p0); break;
            case CLIFFT_OP_ARRAY_U4: array_u4(a1, a2, p0); break;
            case CLIFFT_OP_EXPAND: expand(a1, false, 0.0, 0.0); break;
            case CLIFFT_OP_EXPAND_T: expand(a1, true, CGPU_INV_SQRT2, CGPU_INV_SQRT2); break;
            case CLIFFT_OP_EXPAND_T_DAG: expand(a1, true, CGPU_INV_SQRT2, -CGPU_INV_SQRT2); break;
            case CLIFFT_OP_EXPAND_ROT: {
                const uint4 w1 = __ldg(ip + 2 * pc + 1);
                expand(a1, true, __longlong_as_double(((long long)p1 << 32) | p0),
                       __longlong_as_double(((long long)w1.y << 32) | w1.x));
                break;
            }
            case CLIFFT_OP_MEAS_DORMANT_STATIC:
                meas_dormant_static(a1, p0, sign, (fl & CLIFFT_FLAG_IDENTITY) != 0);
                break;
            case CLIFFT_OP_MEAS_DORMANT_RANDOM: meas_dormant_random(a1, p0, sign); break;
            case CLIFFT_OP_MEAS_ACTIVE_DIAGONAL: meas_diagonal(a1, p0, sign); break;
            case CLIFFT_OP_MEAS_ACTIVE_INTERFERE: meas_interfere(a1, a1, p0, sign); break;
            case CLIFFT_OP_SWAP_MEAS_INTERFERE: meas_interfere(a1, a2, p0, sign); break;
            case CLIFFT_OP_APPLY_PAULI:
                flush_records();
                if (bit_of(rec, p1, S))
                    apply_pauli(P.pauli_x + (size_t)p0 * NW, P.pauli_z + (size_t)p0 * NW,
                                P.pauli_sign[p0] != 0);
                break;
            case CLIFFT_OP_NOISE: noise(p0); break;
            case CLIFFT_OP_NOISE_BLOCK:
                while (next_noise >= p0 && next_noise - p0 < p1) noise(next_noise);
                break;
            case CLIFFT_OP_READOUT_NOISE: readout_noise(p0); break;
            case CLIFFT_OP_DETECTOR: {
                flush_records();
                int par = ((fl & CLIFFT_FLAG_EXPECTED_ONE) && !(K.flags & KF_RAW_PARITY)) ? 1 : 0;
                par ^= list_parity(P.det_off, P.det_tg, p0);
                if (Grp::rank() == 0 && par) det[(p1 >> 5) * S] |= 1u << (p1 & 31);
                break;
            }
            case CLIFFT_OP_POSTSELECT: {
                flush_records();
                if (K.flags & KF_RAW_PARITY) {
                    // a reference-syndrome shot: the raw parity, recorded in the
                    // detector slot the instruction carries, no discard
                    const int par = list_parity(P.det_off, P.det_tg, p0);
                    if (Grp::rank() == 0 && par) det[(p1 >> 5) * S] |= 1u << (p1 & 31);
                    break;
                }
                int par = (fl & CLIFFT_FLAG_EXPECTED_ONE) ? 1 : 0;
                par ^= list_parity(P.det_off, P.det_tg, p0);
                if (par) {
                    discarded = true;
                    stop = true;
                }
                break;
            }
            case CLIFFT_OP_OBSERVABLE: {
                flush_records();
                int par = list_parity(P.obs_off, P.obs_tg, p0);
                if (Grp::rank() == 0 && par) obs[(p1 >> 5) * S] ^= 1u << (p1 & 31);
                break;
            }
            case CLIFFT_OP_EXP_VAL: exp_val(p0, p1); break;
            default:
                if (Grp::rank() == 0) atomicCAS(K.error_word, 0, DEV_ERR_BAD_OPCODE);
                stop = true;
                break;
        }
    }

    static __device__ __forceinline__ uint64_t pdep(uint64_t v, uint64_t mask) {
        uint64_t r = 0;
        for (uint64_t m = mask; m && v; m &= m - 1, v >>= 1)
            if (v & 1u) r |= m & (~m + 1);
        return r;
    }

    // Tile axes for a set of axes `uni` (|uni| < TILE_BITS): `uni` padded with
    // the lowest free axes. Returns F and sets `r` to the length (log2) of the
    // contiguous low run, so one tile is 2^(TILE_BITS - r) runs of 2^r
    // consecutive amplitudes.
    __device__ __forceinline__ uint64_t tile_axes(uint64_t uni, uint32_t& r) const {
        constexpr uint32_t MB = TC::kBits;
        uint64_t F = uni;
        for (uint32_t a = 0; (uint32_t)__popcll(F) < MB; ++a) F |= 1ull << a;
        r = (uint32_t)__ffsll((long long)~F) - 1;  // count of consecutive low axes in F
        return F;
    }

    // One streamed pass over 2^(k_pass) amplitudes in tiles of 2^TILE_BITS:
    // tile t covers the run offsets `runoff` (shared table, 2^(TILE_BITS - r)
    // runs of 2^r amplitudes) shifted by tbase = pdep(t, C). Loads come from
    // logical amplitudes load_add + ..., optional stores (the first
    // `store_runs` runs of each tile) go to store_add + ...; every logical
    // index is mapped through the address label (i ^ xo). Runs whose index
    // has a bit of `skip` set are not loaded (their contents are made by the
    // compute step). Bulk copies (TMA) run K.stages - 1 tiles ahead;
    // `compute(buf, t, tbase)` is called by every thread of the group and
    // must synchronise the group before it returns. Returns false after a
    // barrier timeout.
    uint32_t cur_pc = 0;   // instruction being executed (diagnostics)
    uint32_t cur_site = 0; // which statevector pass is streaming (diagnostics)
    template <class Compute>
    __device__ bool stream_tiles(uint64_t ntiles, uint64_t C, uint32_t r, uint64_t load_add, uint64_t store_add,
                                 uint32_t store_runs, uint32_t skip, Compute compute) {
        if constexpr (!Grp::kCta) {
            return stream_tiles_warp(ntiles, C, r, load_add, store_add, store_runs, skip, compute);
        }
        constexpr uint32_t MB = TC::kBits;
        constexpr uint32_t TN = 1u << MB;
        T* bufs = reinterpret_cast<T*>(fuse + TC::kBufOffset);
        uint64_t* bars = reinterpret_cast<uint64_t*>(fuse + fuse_bar_offset());
        const uint32_t nst = K.stages;
        const uint64_t* runoff = reinterpret_cast<const uint64_t*>(fuse + fuse_tables_offset());
        const uint32_t nruns = 1u << (MB - r);
        const uint32_t run_bytes = (1u << r) * (uint32_t)sizeof(T);
        const uint32_t load_bytes = (nruns >> __popc(skip)) * run_bytes;
        const uint64_t lx = xo;
        // the issuing warp: warp 0 of a CTA group, the shot's own warp otherwise
        const bool issuer = Grp::kCta ? (threadIdx.x >> 5) == 0 : true;
        const int lane = threadIdx.x & 31;
        // The stage barriers are initialised once per group (kernel entry);
        // each call continues from the phase every stage is in, tracked in
        // *bar_phase identically by every thread.
        uint32_t phase = *bar_phase;
        if (phase >> 31) {
            stop = true;
            return false;
        }
        // statevector writes made by ordinary stores must be visible to the copy engine
        fence_async_global();
        Grp::sync();
        // Tile bases and stages advance by running counters (a tile costs a
        // few hundred instructions at 4 KiB, so no division or bit-deposit
        // loop per tile): pdep(t + 1, C) = ((pdep(t, C) | ~C) + 1) & C.
        auto next_base = [C](uint64_t b) { return ((b | ~C) + 1) & C; };
        uint64_t issue_base = 0;  // pdep(next tile to load, C)
        uint32_t issue_st = 0;    // its stage
        auto issue_next = [&]() {
            if (lane == 0) mbar_expect_tx(&bars[issue_st], load_bytes);
            __syncwarp();
            const uint64_t base = load_add + issue_base;
            for (uint32_t j = lane; j < nruns; j += 32)
                if (!(j & skip))
                    bulk_load(bufs + issue_st * TN + (j << r), v + ((base + runoff[j]) ^ lx), run_bytes,
                              &bars[issue_st]);
            issue_base = next_base(issue_base);
            issue_st = issue_st + 1 == nst ? 0 : issue_st + 1;
        };
        if (issuer)
            for (uint64_t t = 0; t < ntiles && t < (uint64_t)(nst - 1); ++t) issue_next();
        bool ok_all = true;
        long long waited = 0;
        uint64_t t = 0;
        uint32_t st = 0;      // stage of tile t
        uint64_t tbase = 0;   // pdep(t, C)
        for (; t < ntiles; ++t, tbase = next_base(tbase), st = st + 1 == nst ? 0 : st + 1) {
            const uint32_t parity = (phase >> st) & 1u;
            uint32_t ok = 0;
            const long long w0 = clock64();
            for (uint32_t it = 0; it < (1u << 20) && !ok; ++it) ok = mbar_try_wait(&bars[st], parity);
            waited = clock64() - w0;
            const bool failed = Grp::kCta ? __syncthreads_or(!ok) != 0 : __any_sync(0xffffffffu, !ok) != 0;
            if (failed) {
                ok_all = false;
                break;
            }
            phase ^= 1u << st;
            // A pass without stores refills the stage that held tile t-1
            // before computing tile t (every thread finished tile t-1: compute
            // ends with a group barrier), so nst-1 tiles stay in flight during
            // the compute. With stores see below.
            if (issuer && !store_runs && t + nst - 1 < ntiles) {
                __syncwarp();
                issue_next();  // tile t + nst - 1
            }
            T* buf = bufs + st * TN;
            compute(buf, t, tbase);
            if (store_runs) {
                const uint64_t base = store_add + tbase;
                if constexpr (Grp::kCta) {
                    // bulk stores issued by warp 0 (32 KiB tiles)
                    fence_async_shared();
                    Grp::sync();
                    if (issuer) {
                        for (uint32_t j = lane; j < store_runs; j += 32)
                            bulk_store(v + ((base + runoff[j]) ^ lx), buf + (j << r), run_bytes);
                        bulk_commit();
                        // Refill the stage of tile t-1 once its store (one bulk
                        // group older than tile t's) has read the buffer: by now
                        // a whole compute has passed since it was issued. Waiting
                        // for it before the compute stalled the issuing warp for
                        // most of a store, and the CTA with it at its next barrier.
                        if (t + nst - 1 < ntiles) {
                            bulk_wait_read1();
                            __syncwarp();
                            issue_next();  // tile t + nst - 1
                        }
                    }
                }
            }
        }
        if (!ok_all) {
            // drain (bounded) every load still in flight before the buffers go away
            if (Grp::rank() == 0 && atomicCAS(K.error_word, 0, DEV_ERR_TIMEOUT) == 0 && K.error_info) {
                K.error_info[0] = cur_site;
                K.error_info[1] = cur_pc;
                K.error_info[2] = t;
                K.error_info[3] = ntiles;
                K.error_info[4] = r;
                K.error_info[5] = k;
                K.error_info[6] = *reinterpret_cast<volatile unsigned long long*>(&bars[st]);
                K.error_info[7] = (unsigned long long)waited;
            }
            // loads in flight at the failed wait: tiles t .. t+nst-2
            for (uint64_t q = t; q < ntiles && q < t + nst - 1; ++q) {
                const uint32_t sq = (uint32_t)(q % nst);
                for (uint32_t it = 0; it < (1u << 20); ++it)
                    if (mbar_try_wait(&bars[sq], (phase >> sq) & 1u)) break;
                phase ^= 1u << sq;
            }
            phase |= 1u << 31;
            stop = true;
        }
        if (issuer) {
            bulk_wait_all();
            fence_async_global();
        }
        *bar_phase = phase;
        Grp::sync();
        return ok_all;
    }

    // The same pass for a warp-specialised CTA group (fused blocks only;
    // loads from and stores to the same logical tiles): the last warp issues
    // every bulk load and store, the other warps only wait for loaded stages
    // and compute. Each stage has two mbarriers: `full` (the load's bytes
    // arrived) and `done` (the compute warps finished the tile; thread 0
    // arrives once). The copy warp refills a stage when its tile is done and
    // the tile's store has read the buffer, while the compute warps move on
    // to the next loaded stage. Every wait is bounded; a timeout on either
    // side is agreed on by the whole CTA, which drains its loads and stops.
    // In a completed pass every stage's two barriers complete once per tile
    // mapped to it, so every thread advances its copy of the phase bits the
    // same way.
    template <class Compute>
    __device__ bool stream_tiles_ws(uint64_t ntiles, uint64_t C, uint32_t r, uint32_t store_runs, uint32_t skip,
                                    Compute compute) {
        constexpr uint32_t MB = TC::kBits;
        constexpr uint32_t TN = 1u << MB;
        T* bufs = reinterpret_cast<T*>(fuse + TC::kBufOffset);
        uint64_t* full = reinterpret_cast<uint64_t*>(fuse + fuse_bar_offset());
        uint64_t* done = full + kMaxStages;
        const uint32_t nst = K.stages;
        const uint64_t* runoff = reinterpret_cast<const uint64_t*>(fuse + fuse_tables_offset());
        const uint32_t nruns = 1u << (MB - r);
        const uint32_t run_bytes = (1u << r) * (uint32_t)sizeof(T);
        const uint32_t load_bytes = (nruns >> __popc(skip)) * run_bytes;
        const uint64_t lx = xo;
        const uint32_t ncomp = blockDim.x - 32u;
        const bool copier = threadIdx.x >= ncomp;
        const uint32_t lane = threadIdx.x & 31u;
        uint32_t phase = *bar_phase;  // bits 0..3: full parity per stage, 8..11: done parity, 31: dead
        if (phase >> 31) {
            stop = true;
            return false;
        }
        auto next_base = [C](uint64_t b) { return ((b | ~C) + 1) & C; };
        // statevector writes made by ordinary stores must be visible to the copy engine
        fence_async_global();
        __syncthreads();
        bool ok = true;
        uint64_t t = 0;
        uint32_t loads[kMaxStages] = {0, 0, 0, 0};  // loads issued per stage (copy warp)
        long long waited = 0;
        if (copier) {
            uint64_t lbase = 0, lt = 0;
            auto load = [&](uint32_t st) {
                if (lane == 0) mbar_expect_tx(&full[st], load_bytes);
                __syncwarp();
                for (uint32_t j = lane; j < nruns; j += 32)
                    if (!(j & skip))
                        bulk_load(bufs + st * TN + (j << r), v + ((lbase + runoff[j]) ^ lx), run_bytes, &full[st]);
                loads[st]++;
                lbase = next_base(lbase);
                ++lt;
            };
            for (uint32_t st = 0; st < nst && lt < ntiles; ++st) load(st);
            uint64_t sbase = 0;
            uint32_t st = 0;
            for (; t < ntiles; ++t, st = st + 1 == nst ? 0 : st + 1) {
                const uint32_t parity = (phase >> (8 + st)) & 1u;
                uint32_t got = 0;
                const long long w0 = clock64();
                for (uint32_t it = 0; it < (1u << 20) && !got; ++it) got = mbar_try_wait(&done[st], parity);
                waited = clock64() - w0;
                if (__any_sync(0xffffffffu, !got)) {
                    ok = false;
                    break;
                }
                phase ^= 1u << (8 + st);
                if (store_runs) {
                    for (uint32_t j = lane; j < store_runs; j += 32)
                        bulk_store(v + ((sbase + runoff[j]) ^ lx), bufs + st * TN + (j << r), run_bytes);
                    bulk_commit();
                }
                sbase = next_base(sbase);
                if (lt < ntiles) {  // tile t + nst into this stage once its store has read it
                    if (store_runs) bulk_wait_read0();
                    __syncwarp();
                    load(st);
                }
            }
            bulk_wait_all();
            fence_async_global();
        } else {
            uint64_t tbase = 0;
            uint32_t st = 0;
            for (; t < ntiles; ++t, tbase = next_base(tbase), st = st + 1 == nst ? 0 : st + 1) {
                const uint32_t parity = (phase >> st) & 1u;
                uint32_t got = 0;
                const long long w0 = clock64();
                for (uint32_t it = 0; it < (1u << 20) && !got; ++it) got = mbar_try_wait(&full[st], parity);
                waited = clock64() - w0;
                if (bar_or_first(ncomp, !got)) {
                    ok = false;
                    break;
                }
                phase ^= 1u << st;
                compute(bufs + st * TN, t, tbase);  // ends with a compute-warp barrier
                // the tile's writes before the copy warp's bulk store reads them
                fence_async_shared();
                bar_sync_first(ncomp);
                if (threadIdx.x == 0) mbar_arrive(&done[st]);
            }
        }
        const bool failed = __syncthreads_or(!ok) != 0;
        if (!failed) {
            // every stage's barriers completed once per tile mapped to it
            phase = *bar_phase;
            for (uint32_t st = 0; st < nst; ++st)
                if (((ntiles + nst - 1 - st) / nst) & 1u) phase ^= (1u << st) | (1u << (8 + st));
        } else {
            if (threadIdx.x == 0 && atomicCAS(K.error_word, 0, DEV_ERR_TIMEOUT) == 0 && K.error_info) {
                K.error_info[0] = cur_site;
                K.error_info[1] = cur_pc;
                K.error_info[2] = t;
                K.error_info[3] = ntiles;
                K.error_info[4] = r;
                K.error_info[5] = k;
                K.error_info[6] = 1000 + (unsigned long long)copier;
                K.error_info[7] = (unsigned long long)waited;
            }
            if (copier) {
                // wait (bounded) for the last load issued into each stage
                const uint32_t p0 = *bar_phase;
                for (uint32_t st = 0; st < nst; ++st) {
                    if (!loads[st]) continue;
                    const uint32_t par = ((p0 >> st) ^ (loads[st] - 1u)) & 1u;
                    for (uint32_t it = 0; it < (1u << 20); ++it)
                        if (mbar_try_wait(&full[st], par)) break;
                }
            }
            phase |= 1u << 31;
            stop = true;
        }
        *bar_phase = phase;
        __syncthreads();
        return !failed;
    }

    // The same pass for a warp running one shot: two 4 KiB buffers filled by
    // 16-byte asynchronous copies from every lane (cp.async, waited for per
    // lane, then a warp barrier) and written back with 16-byte stores. Bulk
    // copies of 4 KiB tiles queue behind the SM's other copies; lane copies
    // keep the warp's loads in the load/store path. Nothing here spins: a
    // copy group always completes.
    template <class Compute>
    __device__ bool stream_tiles_warp(uint64_t ntiles, uint64_t C, uint32_t r, uint64_t load_add,
                                      uint64_t store_add, uint32_t store_runs, uint32_t skip, Compute compute) {
        constexpr uint32_t TN = 1u << TC::kBits;
        T* bufs = reinterpret_cast<T*>(fuse + TC::kBufOffset);
        const uint64_t* runoff = reinterpret_cast<const uint64_t*>(fuse + fuse_tables_offset());
        const uint32_t lane = threadIdx.x & 31;
        const uint32_t clog = r + (sizeof(T) == 8 ? 0u : 1u) - 1u;  // 16-B chunks per run, log2
        const uint32_t wmask = (1u << clog) - 1u;
        const uint32_t load_chunks = (1u << (TC::kBits - r)) << clog;
        const uint32_t store_chunks = store_runs << clog;
        const uint64_t lx = xo;
        auto next_base = [C](uint64_t b) { return ((b | ~C) + 1) & C; };
        auto load_tile = [&](T* dst, uint64_t tb) {
            const uint64_t base = load_add + tb;
            for (uint32_t c = lane; c < load_chunks; c += 32) {
                const uint32_t j = c >> clog, w = c & wmask;
                if (j & skip) continue;
                cp_async16(reinterpret_cast<uint4*>(dst + (j << r)) + w,
                           reinterpret_cast<const uint4*>(v + ((base + runoff[j]) ^ lx)) + w);
            }
            cp_async_commit();
        };
        // the run table was written by other lanes; statevector writes of
        // the previous pass must be visible before the copies read them
        __syncwarp();
        load_tile(bufs, 0);
        uint64_t tbase = 0;
        for (uint64_t t = 0; t < ntiles; ++t) {
            T* buf = bufs + (t & 1u) * TN;
            cp_async_wait<0>();
            __syncwarp();
            const uint64_t nb = next_base(tbase);
            if (t + 1 < ntiles) load_tile(bufs + ((t + 1) & 1u) * TN, nb);
            compute(buf, t, tbase);
            if (store_runs) {
                const uint64_t base = store_add + tbase;
                for (uint32_t c = lane; c < store_chunks; c += 32) {
                    const uint32_t j = c >> clog, w = c & wmask;
                    reinterpret_cast<uint4*>(v + ((base + runoff[j]) ^ lx))[w] =
                        reinterpret_cast<const uint4*>(buf + (j << r))[w];
                }
                __syncwarp();
            }
            tbase = nb;
        }
        return true;
    }

    // Fused block starting at `pc` (one-shot groups, statevector in global
    // memory, k > tile bits), ending before `limit`. With fusion (max_ops >
    // 1) EXPANDs join the block and an active measurement ends it. Returns
    // the number of instructions consumed, 0 when the opcode at `pc` does not
    // start a block worth streaming.
    // A fused block, in its dense-block instance when the launch asked for
    // tensor-core dense blocks: the default instance carries none of that
    // code, so its register allocation is the plain one. Kernels without
    // DENSE contain no tcgen05 instruction at all: the instance that holds a
    // TMEM allocation ran one CTA per SM at a time where shared memory and
    // registers fit two (296 shots took twice as long as 148), and merely
    // carrying that code slowed the default k = 24 path by 37 %.
    __device__ __forceinline__ uint32_t run_block(uint32_t pc, int max_ops, uint32_t limit) {
        if constexpr (kDenseOk) {
            if (K.flags & KF_DENSE) return fused_block<true>(pc, max_ops, limit);
        }
        return fused_block<false>(pc, max_ops, limit);
    }
    template <bool WITH_DENSE>
    __device__ uint32_t fused_block(uint32_t pc, int max_ops, uint32_t limit) {
        constexpr uint32_t MB = TC::kBits;
        const bool wide = max_ops > 1;
        uint64_t need = 0;   // axes that must be tile axes
        uint64_t fresh = 0;  // axes the block's EXPANDs create
        int slots = 0;       // micro-op slots (an EXPAND reserves one for a renormalisation)
        int nsweep = 0;      // array opcodes that touch the statevector
        uint32_t kk = k;     // k after the instructions admitted so far
        uint32_t end = pc;
        uint32_t term = 0;   // the terminating measurement's pc
        int term_kind = 0;   // 1 diagonal, 2 X-basis, 3 X-basis with a fused swap
        for (; end < limit; ++end) {
            const uint4 w0 = __ldg(P.instr + 2 * end);
            uint32_t op = w0.x & 0xffu;
            const uint32_t x1 = w0.y & 0xffffu, x2 = w0.y >> 16;
            if (op >= CLIFFT_OP_MEAS_DORMANT_STATIC_FORCED && op <= CLIFFT_OP_SWAP_MEAS_INTERFERE_FORCED)
                op -= CLIFFT_OP_MEAS_DORMANT_STATIC_FORCED - CLIFFT_OP_MEAS_DORMANT_STATIC;
            uint64_t nd = 0;
            int cost = 0, tk = 0;
            bool expand_op = false, ok = true;
            switch (op) {
                case CLIFFT_OP_FRAME_CNOT:
                case CLIFFT_OP_FRAME_CZ:
                case CLIFFT_OP_FRAME_H:
                case CLIFFT_OP_FRAME_S:
                case CLIFFT_OP_FRAME_S_DAG:
                case CLIFFT_OP_FRAME_SWAP: break;
                case CLIFFT_OP_ARRAY_CNOT: nd = 1ull << x2; cost = 1; break;          // the target moves
                case CLIFFT_OP_ARRAY_MULTI_CNOT: nd = 1ull << x1; cost = 1; break;    // the target moves
                case CLIFFT_OP_ARRAY_SWAP:
                case CLIFFT_OP_ARRAY_U4: nd = (1ull << x1) | (1ull << x2); cost = 1; break;
                case CLIFFT_OP_ARRAY_H: nd = 1ull << x1; cost = 1; break;
                case CLIFFT_OP_ARRAY_CZ:
                case CLIFFT_OP_ARRAY_MULTI_CZ:
                case CLIFFT_OP_ARRAY_S:
                case CLIFFT_OP_ARRAY_S_DAG: cost = 1; break;                           // diagonal: any axes
                case CLIFFT_OP_ARRAY_T:
                case CLIFFT_OP_ARRAY_T_DAG:
                case CLIFFT_OP_ARRAY_ROT: cost = x1 < kk ? 1 : 0; break;
                case CLIFFT_OP_ARRAY_U2:
                    if (x1 < kk) {
                        nd = 1ull << x1;
                        cost = 1;
                    }
                    break;
                case CLIFFT_OP_EXPAND:
                case CLIFFT_OP_EXPAND_T:
                case CLIFFT_OP_EXPAND_T_DAG:
                case CLIFFT_OP_EXPAND_ROT:
                    ok = wide;
                    nd = 1ull << kk;
                    cost = 2;
                    expand_op = true;
                    break;
                case CLIFFT_OP_MEAS_ACTIVE_DIAGONAL: ok = wide; tk = 1; break;
                case CLIFFT_OP_MEAS_ACTIVE_INTERFERE:
                    ok = wide;
                    tk = 2;
                    nd = 1ull << (kk - 1);
                    cost = 1;
                    break;
                case CLIFFT_OP_SWAP_MEAS_INTERFERE:
                    ok = wide;
                    tk = x1 != x2 ? 3 : 2;
                    nd = (1ull << x1) | (1ull << x2);
                    cost = tk == 3 ? 2 : 1;
                    break;
                default: ok = false;
            }
            if (!ok) break;
            const uint64_t cand = need | nd;
            if ((uint32_t)__popcll(cand) > MB || slots + cost > max_ops) break;
            if (nd) {
                uint32_t rr;
                tile_axes(cand, rr);
                if (MB - rr > (uint32_t)kMaxRunsLog2) break;
            }
            need = cand;
            slots += cost;
            if (expand_op) {
                fresh |= 1ull << kk;
                kk++;
            } else if (cost && !tk) {
                nsweep++;
            }
            if (tk) {
                term = end++;
                term_kind = tk;
                break;
            }
        }
        // a block of EXPANDs alone costs more than the plain expansions
        if (nsweep < 1 && !term_kind) return 0;
        uint32_t r;
        const uint64_t F = tile_axes(need, r);
        const uint64_t C = ((kk == 64) ? ~0ull : ((1ull << kk) - 1)) & ~F;
        uint8_t* lbit = reinterpret_cast<uint8_t*>(fuse + fuse_lbit_offset());
        if (Grp::rank() == 0) {
            uint32_t j = 0;
            for (uint32_t a = 0; a < 64; ++a) lbit[a] = ((F >> a) & 1u) ? (uint8_t)j++ : (uint8_t)0xff;
        }
        uint32_t skip = 0;  // run-index bits of the new axes: those runs are made, not loaded
        for (uint64_t w = fresh; w; w &= w - 1) {
            const uint32_t a = (uint32_t)__ffsll((long long)w) - 1;
            skip |= 1u << ((uint32_t)__popcll(F & ((1ull << a) - 1)) - r);
        }
        tileF = F;
        set_runs(F, r);
        Grp::sync();
        // resolve the block's frame-dependent choices into micro-ops
        resolving = true;
        n_mops = 0;
        const uint32_t rend = term_kind ? term : end;
        for (uint32_t q = pc; q < rend; ++q) exec(q);
        const int n_body = n_mops;  // the micro-ops before a terminator's own
        (void)n_body;
        uint32_t tfa = 0, tt = 0, tidx = 0;
        int tsign = 0;
        bool red_local = false;
        uint32_t red_bit = 0;
        if (term_kind) {
            const uint4 w0 = __ldg(P.instr + 2 * term);
            cur_pc = term;
            tfa = w0.y & 0xffffu;
            tt = term_kind == 3 ? (w0.y >> 16) : tfa;
            tidx = w0.z;
            tsign = (((w0.x >> 16) & 0xffu) & CLIFFT_FLAG_SIGN) ? 1 : 0;
            if (term_kind == 3) emit(M_SWAP, tfa, tt, 0, 0, 0, nullptr, 0);
            if (term_kind >= 2) emit(M_H, tt, tt, 0, 0, 0, nullptr, 0);
            red_local = ((F >> tt) & 1u) != 0;
            red_bit = red_local ? (uint32_t)__popcll(F & ((1ull << tt) - 1)) : tt;
        }
        resolving = false;
        if constexpr (kDenseOk && WITH_DENSE) {
            Grp::sync();  // the resolved micro-ops, read by every thread
            MOp* mm = reinterpret_cast<MOp*>(fuse + fuse_mops_offset());
            uint32_t dmask = 0;
            int j1 = 0;
            const int j0 = find_dense(mm, n_body, (int)K.dense_min_weight, local_mask(fresh), dmask, j1);
            if (j0 >= 0) {
                if (Grp::rank() < 16)
                    compose_dense(mm, j0, j1, dmask, Grp::rank(),
                                  reinterpret_cast<float*>(fuse + TC::dense_b_offset(K.stages)));
                fence_async_shared();  // the B operand, read by the tensor cores
                Grp::sync();
                if (Grp::rank() == 0) {
                    mm[j0].kind = M_DENSE;
                    mm[j0].req = dmask;
                    for (int j = j0 + 1; j < j1; ++j) mm[j].kind = M_NOP;
                }
            }
        }
        if (Grp::rank() == 0)
            compile_index_runs(reinterpret_cast<MOp*>(fuse + fuse_mops_offset()), n_mops,
                               (1u << MB) / (uint32_t)compute_threads());
        Grp::sync();
        const MOp* mops = reinterpret_cast<const MOp*>(fuse + fuse_mops_offset());
        const int tid = Grp::rank(), nthr = compute_threads();
        const int nm = n_mops;
        cur_site = 6;
        constexpr uint32_t TN = 1u << MB;
        const uint32_t rpt = TN / (uint32_t)nthr;  // amplitudes per thread in a register-staged run
        double acc[2] = {0.0, 0.0};
        const uint32_t nruns = 1u << (MB - r);
        // an X-basis terminator's H is the block's last micro-op: applied
        // together with the half-norm sums
        const int nmo = term_kind >= 2 ? nm - 1 : nm;
        auto body = [&](T* buf, uint64_t, uint64_t tbase) {
            for (int j = 0; j < nmo;) {
                if constexpr (kDenseOk && WITH_DENSE) {
                    if (mops[j].kind == M_NOP) {
                        ++j;
                        continue;
                    }
                    if (mops[j].kind == M_DENSE) {
                        apply_dense(mops[j].req, buf, tid);
                        csync();
                        ++j;
                        continue;
                    }
                }
                int e = j;
                while (e < nmo && index_map_kind(mops[e].kind)) ++e;
                if (e - j >= 2 && rpt <= kMaxRunAmps) {
                    if (kMaxRunAmps >= 16 && rpt == 16)
                        apply_index_run<(kMaxRunAmps >= 16 ? 16 : 8)>(mops, j, e, buf, tid, nthr, tbase);
                    else if (rpt == 8)
                        apply_index_run<8>(mops, j, e, buf, tid, nthr, tbase);
                    else
                        apply_index_run<4>(mops, j, e, buf, tid, nthr, tbase);
                    j = e;
                    continue;
                }
                apply_micro(mops[j], buf, tid, nthr, tbase);
                csync();
                ++j;
            }
            if (term_kind >= 2) {
                // H on the measured axis, summing the norms of both outputs
                const uint32_t a = red_bit, ab = 1u << a;
                const R s = (R)CGPU_INV_SQRT2;
                double q0 = 0.0, q1 = 0.0;
                for (uint32_t i = tid; i < (TN >> 1); i += nthr) {
                    const uint32_t i0 = ins0_32(i, a);
                    const T x = buf[i0], y = buf[i0 | ab];
                    const T u = cscale(cadd(x, y), s), w = cscale(csub(x, y), s);
                    buf[i0] = u;
                    buf[i0 | ab] = w;
                    q0 += cnorm_d(u);
                    q1 += cnorm_d(w);
                }
                acc[0] += q0;
                acc[1] += q1;
            } else if (term_kind) {
                // the measured axis' two half-norms of this tile
                double q0 = 0.0, q1 = 0.0;
                if (red_local) {
                    for (uint32_t l = tid; l < TN; l += nthr) {
                        const double q = cnorm_d(buf[l]);
                        if ((l >> red_bit) & 1u)
                            q1 += q;
                        else
                            q0 += q;
                    }
                } else {
                    for (uint32_t l = tid; l < TN; l += nthr) q0 += cnorm_d(buf[l]);
                    if ((tbase >> red_bit) & 1u) {
                        q1 = q0;
                        q0 = 0.0;
                    }
                }
                acc[0] += q0;
                acc[1] += q1;
            }
            csync();
        };
        if constexpr (Grp::kWS)
            stream_tiles_ws(1ull << (kk - MB), C, r, nm ? nruns : 0, skip, body);
        else
            stream_tiles(1ull << (kk - MB), C, r, 0, 0, nm ? nruns : 0, skip, body);
        moved += (((1ull << kk) >> __popcll(fresh)) + (nm ? (1ull << kk) : 0ull)) * sizeof(T);
        if (term_kind) {
            group_reduce<Grp, 2>(acc, red);
            if (!stop) {
                if (term_kind == 1) {
                    bytes += (1ull << k) * sizeof(T);
                    diag_tail(tt, tidx, tsign, acc[0], acc[1], true);
                } else {
                    interfere_relabel(tfa, tt, tidx, tsign, acc[0], acc[1]);
                }
            }
        }
        return end - pc;
    }

    // Micro-ops that map every amplitude to one position (CNOT, SWAP,
    // multi-CNOT: bit maps on the tile index) and / or multiply it by a
    // factor that depends on its position (CZ, multi-CZ, PHASE).
    static __device__ __forceinline__ bool index_map_kind(uint8_t kind) {
        return kind == M_CNOT || kind == M_SWAP || kind == M_MCNOT || kind == M_CZ || kind == M_MCZ ||
               kind == M_PHASE;
    }
    // Condition of a conditional micro-op at tile position p, given its
    // tile-global parity gp: every `req` bit set and, with MF_PARITY, odd
    // parity of the `par` bits and gp.
    static __device__ __forceinline__ bool micro_on(const MOp& m, uint32_t p, uint32_t gp) {
        return (p & m.req) == m.req && (!(m.flags & MF_PARITY) || ((__popc(p & m.par) ^ gp) & 1u));
    }
    static constexpr uint32_t kMaxRunAmps = sizeof(R) == 4 ? 16u : 8u;  // register budget of a staged run
    // A run of index-map micro-ops is compiled once per block into an affine
    // map over GF(2) of tile positions: after the run's first j ops an
    // amplitude that started at position p0 sits at P_j = L_j p0 ^ b_j, where
    // the linear part L_j depends only on the ops' tile-local bits and the
    // offset b_j also on the tile's global bits (global controls, the global
    // part of a multi gate's parity). CNOT / multi-CNOT / SWAP only update
    // (L, b); a diagonal op's condition is an AND of affine bits of P_j, each
    // the parity of p0 & row (the rows of L_j it reads) ^ a per-tile constant.
    // The rows of each diagonal op and the final map's columns are kept in
    // coefficient slots those ops do not use.
    struct RunRows {
        uint16_t row[3];
        uint8_t n, pad;
    };
    static __device__ __forceinline__ RunRows* run_rows(MOp& m) { return reinterpret_cast<RunRows*>(&m.c[1]); }
    static __device__ __forceinline__ const RunRows* run_rows(const MOp& m) {
        return reinterpret_cast<const RunRows*>(&m.c[1]);
    }
    static __device__ __forceinline__ uint16_t* run_cols(MOp& m) { return reinterpret_cast<uint16_t*>(&m.c[4]); }
    static __device__ __forceinline__ const uint16_t* run_cols(const MOp& m) {
        return reinterpret_cast<const uint16_t*>(&m.c[4]);
    }
    // Compiles every run the tile loop will stage (the same boundaries: at
    // least two consecutive index-map ops and rpt <= kMaxRunAmps). Run by one
    // thread.
    static __device__ void compile_index_runs(MOp* mops, int nm, uint32_t rpt) {
        constexpr uint32_t MB = TC::kBits;
        for (int j = 0; j < nm;) {
            int e = j;
            while (e < nm && index_map_kind(mops[e].kind)) ++e;
            if (!(e - j >= 2 && rpt <= kMaxRunAmps)) {
                ++j;
                continue;
            }
            uint16_t rows[MB];  // P bit i = parity(p0 & rows[i]) ^ b bit i
            for (uint32_t i = 0; i < MB; ++i) rows[i] = (uint16_t)(1u << i);
            for (int q = j; q < e; ++q) {
                MOp& m = mops[q];
                auto par_row = [&](uint32_t par) {
                    uint16_t x = 0;
                    for (uint32_t w = par; w; w &= w - 1) x ^= rows[__ffs(w) - 1];
                    return x;
                };
                switch (m.kind) {
                    case M_CNOT:
                        if (m.req) rows[m.a] ^= rows[__ffs(m.req) - 1];
                        break;
                    case M_MCNOT: rows[m.a] ^= par_row(m.par); break;
                    case M_SWAP: {
                        const uint16_t t = rows[m.a];
                        rows[m.a] = rows[m.b];
                        rows[m.b] = t;
                        break;
                    }
                    default: {  // M_CZ, M_MCZ, M_PHASE
                        RunRows* rr = run_rows(m);
                        int n = 0;
                        for (uint32_t w = m.req; w; w &= w - 1) rr->row[n++] = rows[__ffs(w) - 1];
                        if (m.flags & MF_PARITY) rr->row[n++] = par_row(m.par);
                        rr->n = (uint8_t)n;
                        break;
                    }
                }
            }
            uint16_t* fc = run_cols(mops[j]);
            for (uint32_t c = 0; c < MB; ++c) {
                uint32_t col = 0;
                for (uint32_t i = 0; i < MB; ++i) col |= ((rows[i] >> c) & 1u) << i;
                fc[c] = (uint16_t)col;
            }
            j = e;
        }
    }
    // A compiled run mops[j0, j1) in one pass over the tile: each thread
    // reads RPT amplitudes (positions tid + q * nthr) into registers, follows
    // the run's affine offset through its ops (scalar work per tile), applies
    // every diagonal factor in the run's order to the amplitudes it hits (the
    // same operations, in the same order, as one micro-op at a time), then
    // writes each amplitude at its final position. The barrier between the
    // read and write phases makes the in-place permutation safe.
    template <int RPT>
    static __device__ void apply_index_run(const MOp* mops, int j0, int j1, T* tile, int tid, int nthr,
                                           uint64_t tbase) {
        constexpr uint32_t MB = TC::kBits;
        constexpr uint32_t QB = RPT == 16 ? 4u : (RPT == 8 ? 3u : 2u);  // bits of the register index q
        constexpr uint32_t ALL = (1u << RPT) - 1u;
        const uint32_t lg = MB - QB;  // p0 = tid | q << lg
        T v[RPT];
#pragma unroll
        for (int q = 0; q < RPT; ++q) v[q] = tile[tid + q * nthr];
        // mask over q of parity(p0 & row) ^ k
        auto bits = [&](uint32_t row, uint32_t k) -> uint32_t {
            const uint32_t r = row >> lg;
            uint32_t m = ((r & 1u) ? (0xAAAAu & ALL) : 0u) ^ ((r & 2u) ? (0xCCCCu & ALL) : 0u);
            if (QB > 2) m ^= (r & 4u) ? (0xF0F0u & ALL) : 0u;
            if (QB > 3) m ^= (r & 8u) ? (0xFF00u & ALL) : 0u;
            const uint32_t t = ((uint32_t)__popc((uint32_t)tid & row & ((1u << lg) - 1u)) ^ k) & 1u;
            return m ^ (0u - t) & ALL;
        };
        uint32_t b = 0;  // the run's affine offset so far
        for (int j = j0; j < j1; ++j) {
            const MOp& m = mops[j];
            const uint64_t greq = m.greq;
            if ((tbase & greq) != greq) continue;  // the op is the identity on this tile
            const uint32_t kind = m.kind;
            if (kind == M_CNOT) {
                const uint32_t req = m.req;
                b ^= (req ? ((b >> (__ffs(req) - 1)) & 1u) : 1u) << m.a;
            } else if (kind == M_MCNOT) {
                b ^= (((uint32_t)__popc(b & m.par) ^ (uint32_t)__popcll(tbase & m.gpar)) & 1u) << m.a;
            } else if (kind == M_SWAP) {
                const uint32_t d = ((b >> m.a) ^ (b >> m.b)) & 1u;
                b ^= (0u - d) & ((1u << m.a) | (1u << m.b));
            } else {
                const RunRows rr = *run_rows(m);
                uint32_t hit = ALL;
                int n = 0;
                for (uint32_t w = m.req; w; w &= w - 1) hit &= bits(rr.row[n++], (b >> (__ffs(w) - 1)) & 1u);
                if (m.flags & MF_PARITY)
                    hit &= bits(rr.row[n], ((uint32_t)__popc(b & m.par) ^ (uint32_t)__popcll(tbase & m.gpar)) & 1u);
                if (kind == M_PHASE) {
                    const T ph = m.c[0];
#pragma unroll
                    for (int q = 0; q < RPT; ++q) {
                        const T w = cmul(v[q], ph);
                        v[q] = ((hit >> q) & 1u) ? w : v[q];
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < RPT; ++q) v[q] = ((hit >> q) & 1u) ? cneg(v[q]) : v[q];
                }
            }
        }
        // final positions: L p0 ^ b, L applied column by column
        const uint16_t* fc = run_cols(mops[j0]);
        uint32_t lt = b;
        for (uint32_t i = 0; i < lg; ++i) lt ^= ((tid >> i) & 1u) ? (uint32_t)fc[i] : 0u;
        uint32_t cq[QB];
#pragma unroll
        for (uint32_t i = 0; i < QB; ++i) cq[i] = fc[lg + i];
        csync();
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
            uint32_t pq = lt;
#pragma unroll
            for (uint32_t i = 0; i < QB; ++i)
                if ((q >> i) & 1) pq ^= cq[i];
            tile[pq] = v[q];
        }
        csync();
    }

    // One micro-op on a shared-memory tile of 2^TILE_BITS amplitudes whose
    // tile-global index bits are tbase; the arithmetic matches the unfused
    // opcode handlers exactly.
    static __device__ __forceinline__ void apply_micro(const MOp& m, T* tile, int tid, int nthr, uint64_t tbase) {
        constexpr uint32_t MB = TC::kBits;
        if ((tbase & m.greq) != m.greq) return;  // the op is the identity on this tile
        const uint32_t gp = (uint32_t)__popcll(tbase & m.gpar) & 1u;
        const uint32_t a = m.a, b = m.b;
        const uint32_t ab = 1u << a, bb = 1u << b;
        switch (m.kind) {
            case M_CNOT:
            case M_MCNOT:
                for (uint32_t i = tid; i < (1u << (MB - 1)); i += nthr) {
                    const uint32_t i0 = ins0_32(i, a);
                    if (micro_on(m, i0, gp)) {
                        T x = tile[i0];
                        tile[i0] = tile[i0 | ab];
                        tile[i0 | ab] = x;
                    }
                }
                break;
            case M_CZ:
            case M_MCZ:
            case M_PHASE: {
                // positions with every `req` bit set (at most two bits)
                const uint32_t nreq = (uint32_t)__popc(m.req);
                const uint32_t r0 = m.req ? (uint32_t)__ffs(m.req) - 1 : 0u;
                const uint32_t r1 = nreq > 1 ? (uint32_t)__ffs(m.req & (m.req - 1)) - 1 : 0u;
                const T ph = m.c[0];
                for (uint32_t i = tid; i < (1u << (MB - nreq)); i += nthr) {
                    const uint32_t idx = (nreq == 0 ? i : (nreq == 1 ? ins0_32(i, r0) : ins00_32(i, r0, r1))) | m.req;
                    if (!micro_on(m, idx, gp)) continue;
                    tile[idx] = m.kind == M_PHASE ? cmul(tile[idx], ph) : cneg(tile[idx]);
                }
                break;
            }
            case M_SWAP:
                for (uint32_t i = tid; i < (1u << (MB - 2)); i += nthr) {
                    uint32_t base = ins00_32(i, a, b);
                    T x = tile[base | ab];
                    tile[base | ab] = tile[base | bb];
                    tile[base | bb] = x;
                }
                break;
            case M_H: {
                const R s = (R)CGPU_INV_SQRT2;
                for (uint32_t i = tid; i < (1u << (MB - 1)); i += nthr) {
                    uint32_t i0 = ins0_32(i, a);
                    T x = tile[i0], y = tile[i0 | ab];
                    tile[i0] = cscale(cadd(x, y), s);
                    tile[i0 | ab] = cscale(csub(x, y), s);
                }
                break;
            }
            case M_U2: {
                const T m00 = m.c[0], m01 = m.c[1], m10 = m.c[2], m11 = m.c[3];
                for (uint32_t i = tid; i < (1u << (MB - 1)); i += nthr) {
                    uint32_t i0 = ins0_32(i, a);
                    T x = tile[i0], y = tile[i0 | ab];
                    tile[i0] = cmac(cmul(m00, x), m01, y);
                    tile[i0 | ab] = cmac(cmul(m10, x), m11, y);
                }
                break;
            }
            case M_U4: {
                // FP32: the 16 coefficients held in registers; FP64 reads them
                // from shared memory (its registers are spoken for)
                constexpr bool kHoist = sizeof(R) == 4;
                T cm[kHoist ? 16 : 1];
                if constexpr (kHoist) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) cm[j] = m.c[j];
                }
                auto coef = [&](int j) -> T {
                    if constexpr (kHoist)
                        return cm[j];
                    else
                        return m.c[j];
                };
                for (uint32_t i = tid; i < (1u << (MB - 2)); i += nthr) {
                    uint32_t q = ins00_32(i, a, b);
                    T x0 = tile[q], x1 = tile[q | ab], x2 = tile[q | bb], x3 = tile[q | ab | bb];
                    T y[4];
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        T acc = cmul(coef(4 * r), x0);
                        acc = cmac(acc, coef(4 * r + 1), x1);
                        acc = cmac(acc, coef(4 * r + 2), x2);
                        acc = cmac(acc, coef(4 * r + 3), x3);
                        y[r] = acc;
                    }
                    tile[q] = y[0];
                    tile[q | ab] = y[1];
                    tile[q | bb] = y[2];
                    tile[q | ab | bb] = y[3];
                }
                break;
            }
            case M_EXPAND: {
                // the new axis' set half from its clear half (x the phase)
                const T ph = m.c[0];
                const bool copy = (m.flags & MF_COPY) != 0;
                for (uint32_t i = tid; i < (1u << (MB - 1)); i += nthr) {
                    const uint32_t i0 = ins0_32(i, a);
                    tile[i0 | ab] = copy ? tile[i0] : cmul(tile[i0], ph);
                }
                break;
            }
            case M_SCALE: {
                const R g = m.c[0].x;
                for (uint32_t i = tid; i < (1u << MB); i += nthr) tile[i] = cscale(tile[i], g);
                break;
            }
            default: break;
        }
    }

    // ---- dense blocks on the tensor cores (KF_DENSE, FP32 CTA groups)
    // the dense-block code exists only in the kernel instances built for it
    static constexpr bool kDenseOk = DENSE && sizeof(R) == 4 && Grp::kCta;
    // Tile-local bits a micro-op moves or reads, or ~0u when it cannot join a
    // dense run (an expansion, a renormalisation, a condition on tile-global
    // bits).
    static __device__ __forceinline__ uint32_t dense_bits(const MOp& m) {
        if (m.greq || ((m.flags & MF_PARITY) && m.gpar)) return ~0u;
        const uint32_t cond = m.req | ((m.flags & MF_PARITY) ? m.par : 0u);
        switch (m.kind) {
            case M_H:
            case M_U2: return 1u << m.a;
            case M_SWAP:
            case M_U4: return (1u << m.a) | (1u << m.b);
            case M_CNOT:
            case M_MCNOT: return (1u << m.a) | cond;
            case M_CZ:
            case M_MCZ:
            case M_PHASE: return cond;
            default: return ~0u;
        }
    }
    // Work a micro-op costs on the CUDA cores, in passes over the tile
    static __device__ __forceinline__ int dense_weight(uint8_t kind) {
        return kind == M_U4 ? 4 : (kind == M_U2 ? 2 : 1);
    }
    // The heaviest run of micro-ops in [0, n) on at most four tile-local bits
    // that holds a mixing op (H, U2, U4) and is worth a GEMM (weight >=
    // min_weight; the first of equal weights): returns its first op (-1:
    // none), its end in j1 and its
    // four bits in dmask, padded with the highest free tile bits outside
    // `avoid`. The bits of axes the block creates are avoided: until their
    // EXPAND their set half of the tile is not loaded, and a GEMM would
    // multiply that memory (possibly NaN / Inf) by the zero coefficients of
    // the identity on a padding bit.
    static __device__ int find_dense(const MOp* mops, int n, int min_weight, uint32_t avoid, uint32_t& dmask,
                                     int& j1) {
        constexpr uint32_t MB = TC::kBits;
        int best = -1, best_w = min_weight - 1;
        uint32_t best_bits = 0;
        for (int j = 0; j < n; ++j) {
            uint32_t bits = 0;
            bool mix = false;
            int w = 0, e = j;
            for (; e < n; ++e) {
                const uint32_t b = dense_bits(mops[e]);
                if (b == ~0u || __popc(bits | b) > 4) break;
                bits |= b;
                mix |= mops[e].kind == M_H || mops[e].kind == M_U2 || mops[e].kind == M_U4;
                w += dense_weight(mops[e].kind);
            }
            if (e - j >= 2 && mix && w > best_w) {
                best = j;
                best_w = w;
                best_bits = bits;
                j1 = e;
            }
        }
        if (best >= 0) {
            // padding from the top: groups then vary in the low tile bits,
            // which spreads a warp's accesses over the shared-memory banks
            for (int q = (int)MB - 1; __popc(best_bits) < 4 && q >= 0; --q)
                if (!((avoid >> q) & 1u)) best_bits |= 1u << q;
            dmask = best_bits;
        }
        return best;
    }
    // Column `col` of the 16 x 16 matrix U of micro-ops [j0, j1) on the four
    // bits of dmask (index bit q = the q-th lowest bit of dmask), composed in
    // FP64 by applying each op to the basis vector e_col with the arithmetic
    // of its CUDA-core handler; written as its entries of M (rows n = 2 d + c
    // of the outputs, columns k = 2 col + c' of the inputs) into the K-major
    // B operand: element (n, k) at byte (k / 4) * 512 + (n / 8) * 128 +
    // (n % 8) * 16 + (k % 4) * 4, TF32 high parts first, low parts 4 KiB on.
    static __device__ __noinline__ void compose_dense(const MOp* mops, int j0, int j1, uint32_t dmask, int col,
                                                       float* bop) {
        uint32_t dbit[4];
        {
            uint32_t w = dmask;
            for (int q = 0; q < 4; ++q) {
                dbit[q] = (uint32_t)__ffs(w) - 1;
                w &= w - 1;
            }
        }
        auto dm = [&](uint32_t lm) {
            uint32_t r = 0;
            for (int q = 0; q < 4; ++q) r |= ((lm >> dbit[q]) & 1u) << q;
            return r;
        };
        double2 v[16];
        for (int i = 0; i < 16; ++i) v[i] = make_double2(i == col ? 1.0 : 0.0, 0.0);
        auto cd = [](const T& c) { return make_double2((double)c.x, (double)c.y); };
        auto mul = [](double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); };
        auto add = [](double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); };
        for (int j = j0; j < j1; ++j) {
            const MOp& m = mops[j];
            const bool use_par = (m.flags & MF_PARITY) != 0;
            const uint32_t req = dm(m.req), par = use_par ? dm(m.par) : 0u;
            auto on = [&](uint32_t i) { return (i & req) == req && (!use_par || (__popc(i & par) & 1)); };
            const uint32_t ab = dm(1u << (m.a & 31u)), bb = dm(1u << (m.b & 31u));
            switch (m.kind) {
                case M_CNOT:
                case M_MCNOT:
                    for (uint32_t i = 0; i < 16; ++i)
                        if (!(i & ab) && on(i)) {
                            const double2 t = v[i];
                            v[i] = v[i | ab];
                            v[i | ab] = t;
                        }
                    break;
                case M_CZ:
                case M_MCZ:
                    for (uint32_t i = 0; i < 16; ++i)
                        if (on(i)) v[i] = make_double2(-v[i].x, -v[i].y);
                    break;
                case M_PHASE: {
                    const double2 ph = cd(m.c[0]);
                    for (uint32_t i = 0; i < 16; ++i)
                        if (on(i)) v[i] = mul(v[i], ph);
                    break;
                }
                case M_SWAP:
                    for (uint32_t i = 0; i < 16; ++i)
                        if ((i & ab) && !(i & bb)) {
                            const uint32_t o = i ^ ab ^ bb;
                            const double2 t = v[i];
                            v[i] = v[o];
                            v[o] = t;
                        }
                    break;
                case M_H:
                    for (uint32_t i = 0; i < 16; ++i)
                        if (!(i & ab)) {
                            const double2 x = v[i], y = v[i | ab];
                            v[i] = make_double2((x.x + y.x) * CGPU_INV_SQRT2, (x.y + y.y) * CGPU_INV_SQRT2);
                            v[i | ab] = make_double2((x.x - y.x) * CGPU_INV_SQRT2, (x.y - y.y) * CGPU_INV_SQRT2);
                        }
                    break;
                case M_U2: {
                    const double2 m00 = cd(m.c[0]), m01 = cd(m.c[1]), m10 = cd(m.c[2]), m11 = cd(m.c[3]);
                    for (uint32_t i = 0; i < 16; ++i)
                        if (!(i & ab)) {
                            const double2 x = v[i], y = v[i | ab];
                            v[i] = add(mul(m00, x), mul(m01, y));
                            v[i | ab] = add(mul(m10, x), mul(m11, y));
                        }
                    break;
                }
                case M_U4:
                    for (uint32_t i = 0; i < 16; ++i)
                        if (!(i & ab) && !(i & bb)) {
                            const double2 x[4] = {v[i], v[i | ab], v[i | bb], v[i | ab | bb]};
                            double2 y[4];
                            for (int r = 0; r < 4; ++r) {
                                double2 acc = mul(cd(m.c[4 * r]), x[0]);
                                for (int c = 1; c < 4; ++c) acc = add(acc, mul(cd(m.c[4 * r + c]), x[c]));
                                y[r] = acc;
                            }
                            v[i] = y[0];
                            v[i | ab] = y[1];
                            v[i | bb] = y[2];
                            v[i | ab | bb] = y[3];
                        }
                    break;
                default: break;
            }
        }
        // M[2d][2col] = Re U[d][col], M[2d+1][2col] = Im, M[2d][2col+1] = -Im, M[2d+1][2col+1] = Re
        for (int d = 0; d < 16; ++d)
            for (int c = 0; c < 4; ++c) {
                const int n = 2 * d + (c & 1), k = 2 * col + (c >> 1);
                const double x = c == 0 ? v[d].x : (c == 1 ? v[d].y : (c == 2 ? -v[d].y : v[d].x));
                const float hi = __uint_as_float(to_tf32((float)x));
                const float lo = __uint_as_float(to_tf32((float)(x - (double)hi)));
                const int off = (k >> 2) * 128 + (n >> 3) * 32 + (n & 7) * 4 + (k & 3);  // in floats
                bop[off] = hi;
                bop[1024 + off] = lo;
            }
    }
    // y = U x on every 16-amplitude group of the tile (the groups vary the
    // four bits of dmask) on the tensor cores. The 256 groups form two
    // 128-row chunks; compute warp w writes rows 32 (w % 4) .. + 31 of chunk
    // w / 4 (its TMEM lane quarter) as TF32 hi / lo columns, thread 0 issues
    // the 24 MMAs (per chunk: 4 K-steps x 3 products) and commits them to the
    // dense mbarrier, every thread waits for it (bounded), reads its row of
    // D and writes its group back. The waits of all compute threads agree;
    // a wait that gives up records a device error and turns the dense path
    // off for the rest of the launch on this CTA.
    __device__ __noinline__ void apply_dense(uint32_t dmask, T* tile, int tid) {
        uint32_t* slot = reinterpret_cast<uint32_t*>(fuse + TC::kDenseSlotOffset);
        uint64_t* bar = reinterpret_cast<uint64_t*>(slot);
        const uint32_t state = slot[3];  // bit 0: the mbarrier's phase, bit 31: off after a timeout
        if (state >> 31) return;
        const uint32_t tmem = slot[2];
        const uint32_t w = (uint32_t)tid >> 5, lane = (uint32_t)tid & 31u, ch = w >> 2, qr = w & 3u;
        uint32_t dbit[4];
        {
            uint32_t m = dmask;
            for (int q = 0; q < 4; ++q) {
                dbit[q] = (uint32_t)__ffs(m) - 1;
                m &= m - 1;
            }
        }
        auto dpos = [&](uint32_t d) {
            return ((d & 1u) << dbit[0]) | (((d >> 1) & 1u) << dbit[1]) | (((d >> 2) & 1u) << dbit[2]) |
                   (((d >> 3) & 1u) << dbit[3]);
        };
        const uint32_t g = (ch << 7) | (qr << 5) | lane;
        const uint32_t base = ins0_32(ins0_32(ins0_32(ins0_32(g, dbit[0]), dbit[1]), dbit[2]), dbit[3]);
        const uint32_t cols = tmem + ((qr * 32u) << 16) + ch * 96u;  // this warp's lanes, the chunk's columns
        tc_fence_after();
#pragma unroll
        for (uint32_t p = 0; p < 4; ++p) {
            uint32_t hi[8], lo[8];
#pragma unroll
            for (uint32_t e = 0; e < 4; ++e) {
                const T x = tile[base | dpos(4 * p + e)];
                split_tf32(x.x, hi[2 * e], lo[2 * e]);
                split_tf32(x.y, hi[2 * e + 1], lo[2 * e + 1]);
            }
            tmem_st8(cols + 8 * p, hi);
            tmem_st8(cols + 32 + 8 * p, lo);
        }
        tmem_wait_st();
        tc_fence_before();
        csync();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t bsm = smem_u32(fuse + TC::dense_b_offset(K.stages));
#pragma unroll
            for (uint32_t c = 0; c < 2; ++c) {
                const uint32_t a = tmem + c * 96u, d = a + 64u;
#pragma unroll
                for (uint32_t st = 0; st < 4; ++st) umma_tf32(d, a + 8 * st, dense_b_desc(bsm + 1024 * st), st);
#pragma unroll
                for (uint32_t st = 0; st < 4; ++st) umma_tf32(d, a + 32 + 8 * st, dense_b_desc(bsm + 1024 * st), 1);
#pragma unroll
                for (uint32_t st = 0; st < 4; ++st)
                    umma_tf32(d, a + 8 * st, dense_b_desc(bsm + 4096 + 1024 * st), 1);
            }
            umma_commit(bar);
        }
        uint32_t got = 0;
        for (uint32_t it = 0; it < (1u << 20) && !got; ++it) got = mbar_try_wait(bar, state & 1u);
        bool failed;
        if constexpr (Grp::kWS)
            failed = bar_or_first(blockDim.x - 32u, !got);
        else
            failed = __syncthreads_or(!got) != 0;
        if (failed) {
            if (tid == 0) {
                slot[3] = state | (1u << 31);
                if (atomicCAS(K.error_word, 0, DEV_ERR_TIMEOUT) == 0 && K.error_info) {
                    K.error_info[0] = cur_site;
                    K.error_info[1] = cur_pc;
                    K.error_info[6] = 3000;  // the dense block's MMAs
                }
            }
            stop = true;
            return;
        }
        tc_fence_after();
        uint32_t y[32];
        tmem_ld32(cols + 64, y);
        tmem_wait_ld();
#pragma unroll
        for (uint32_t d = 0; d < 16; ++d)
            tile[base | dpos(d)] = make_float2(__uint_as_float(y[2 * d]), __uint_as_float(y[2 * d + 1]));
        tc_fence_before();
        if (tid == 0) slot[3] = state ^ 1u;  // read by the next call after the caller's barrier
    }

    // Whether instruction pc touches the statevector (needs every thread of a
    // CTA group) or only scalar state (frame, gamma, records, noise cursor).
    __device__ __forceinline__ bool needs_all(uint32_t pc) const {
        const uint4 w0 = __ldg(P.instr + 2 * pc);
        uint32_t op = w0.x & 0xffu;
        const uint32_t a1 = w0.y & 0xffffu;
        if (op >= CLIFFT_OP_MEAS_DORMANT_STATIC_FORCED && op <= CLIFFT_OP_SWAP_MEAS_INTERFERE_FORCED)
            op -= CLIFFT_OP_MEAS_DORMANT_STATIC_FORCED - CLIFFT_OP_MEAS_DORMANT_STATIC;
        switch (op) {
            case CLIFFT_OP_ARRAY_CNOT:
            case CLIFFT_OP_ARRAY_CZ:
            case CLIFFT_OP_ARRAY_SWAP:
            case CLIFFT_OP_ARRAY_MULTI_CNOT:
            case CLIFFT_OP_ARRAY_MULTI_CZ:
            case CLIFFT_OP_ARRAY_H:
            case CLIFFT_OP_ARRAY_S:
            case CLIFFT_OP_ARRAY_S_DAG:
            case CLIFFT_OP_ARRAY_U4:
            case CLIFFT_OP_EXPAND:
            case CLIFFT_OP_EXPAND_T:
            case CLIFFT_OP_EXPAND_T_DAG:
            case CLIFFT_OP_EXPAND_ROT:
            case CLIFFT_OP_MEAS_ACTIVE_DIAGONAL:
            case CLIFFT_OP_MEAS_ACTIVE_INTERFERE:
            case CLIFFT_OP_SWAP_MEAS_INTERFERE:
            case CLIFFT_OP_EXP_VAL: return true;
            case CLIFFT_OP_ARRAY_T:
            case CLIFFT_OP_ARRAY_T_DAG:
            case CLIFFT_OP_ARRAY_ROT:
            case CLIFFT_OP_ARRAY_U2: return a1 < k;
            default: return false;
        }
    }

    __device__ __forceinline__ CtlState<NW>* ctl() const {
        return reinterpret_cast<CtlState<NW>*>(reinterpret_cast<unsigned char*>(red) + 3 * 8 * 32 + 64);
    }
    __device__ __forceinline__ void publish(uint32_t pc, uint32_t cmd) {
        if (threadIdx.x == 0) {
            CtlState<NW>* c = ctl();
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                c->fx[w] = f.x[w];
                c->fz[w] = f.z[w];
            }
            c->gamma = gamma;
            c->log_prob = log_prob;
            c->dust = dust;
            c->bytes = bytes;
            c->moved = moved;
            c->k = k;
            c->draw = draw;
            c->next_noise = next_noise;
            c->ff_pos = ff_pos;
            c->ff_end = ff_end;
            c->ro_pos = ro_pos;
            c->ro_end = ro_end;
            c->pc = pc;
            c->cmd = cmd;
            c->flags = (stop ? 1u : 0u) | (discarded ? 2u : 0u) | (reachable ? 4u : 0u);
        }
    }
    __device__ __forceinline__ uint32_t adopt() {
        const CtlState<NW>* c = ctl();
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            f.x[w] = c->fx[w];
            f.z[w] = c->fz[w];
        }
        gamma = c->gamma;
        log_prob = c->log_prob;
        dust = c->dust;
        bytes = c->bytes;
        moved = c->moved;
        k = c->k;
        draw = c->draw;
        next_noise = c->next_noise;
        ff_pos = c->ff_pos;
        ff_end = c->ff_end;
        ro_pos = c->ro_pos;
        ro_end = c->ro_end;
        stop = (c->flags & 1u) != 0;
        discarded = (c->flags & 2u) != 0;
        reachable = (c->flags & 4u) != 0;
        rec_dirty = false;
        return c->pc | (c->cmd << 31);
    }
    // a statevector step executed by every thread (fused block or one opcode)
    __device__ __forceinline__ uint32_t run_all(uint32_t pc, bool fuse_on) {
        uint32_t used = 0;
        if (tiled(k)) used = run_block(pc, fuse_on ? TC::kMops : 1, P.n_instr);
        if (!used) {
            exec(pc);
            used = 1;
        }
        return used;
    }
    // CTA groups: warp 0 interprets the bytecode; the other warps join only
    // for statevector steps, receiving the scalar state through shared memory.
    // Every CTA-wide barrier is reached by all warps at the same program point.
    __device__ void run_cta(bool fuse_on, bool prof) {
        const uint32_t n_instr = P.n_instr;
        const bool ctrl = (threadIdx.x >> 5) == 0;
        uint32_t pc = 0;
        for (;;) {
            if (ctrl) {
                solo = true;
                const long long c0 = prof ? clock64() : 0;
                while (pc < n_instr && !stop) {
                    pc = frame_run(pc, n_instr);
                    if (pc >= n_instr || needs_all(pc)) break;
                    exec(pc);
                    ++pc;
                }
                flush_records();
                if (prof) atomicAdd(K.phase_cycles + 4, (unsigned long long)(clock64() - c0));
                publish(pc, (pc >= n_instr || stop) ? 1u : 0u);
            }
            __syncthreads();
            uint32_t word;
            if (ctrl) {
                word = (pc >= n_instr || stop) ? 0x80000000u : pc;
            } else {
                word = adopt();
            }
            solo = false;
            if (word >> 31) break;
            const long long c1 = prof ? clock64() : 0;
            const uint32_t used = run_all(word, fuse_on);
            __syncthreads();
            if (prof) {
                const uint32_t op = __ldg(P.instr + 2 * word).x & 0xffu;
                int cat = used > 1 ? 0 : 3;
                if ((op >= CLIFFT_OP_MEAS_ACTIVE_DIAGONAL && op <= CLIFFT_OP_SWAP_MEAS_INTERFERE) ||
                    (op >= CLIFFT_OP_MEAS_ACTIVE_DIAGONAL_FORCED && op <= CLIFFT_OP_SWAP_MEAS_INTERFERE_FORCED))
                    cat = 1;
                else if (op >= CLIFFT_OP_EXPAND && op <= CLIFFT_OP_EXPAND_ROT)
                    cat = 2;
                atomicAdd(K.phase_cycles + cat, (unsigned long long)(clock64() - c1));
            }
            pc = word + used;
        }
    }

    // ------------------------------------------------------------ driver
    __device__ __forceinline__ void run(Tally& tally) {
        const bool seg = (K.seg_flags & KSEG_ON) != 0;
        if (seg && !(K.seg_flags & KSEG_FIRST)) {
            load_state();
        } else {
            reset();
        }
        const uint32_t n_instr = P.n_instr;
        const bool fuse_on = Grp::kCta && (K.flags & KF_FUSE) != 0;
        const bool prof = K.phase_cycles != nullptr && Grp::rank() == 0;
        if (Grp::kCta) {
            run_cta(fuse_on, prof);
        } else {
            const uint32_t end = seg ? K.seg_end : n_instr;
            const int max_ops = (K.flags & KF_FUSE) ? TC::kMops : 1;
            for (uint32_t pc = seg ? K.seg_begin : 0; pc < end;) {
                pc = frame_run(pc, end);
                if (pc >= end) break;
                uint32_t used = 0;
                if constexpr (kTiles) {
                    // a warp running one shot streams its global statevector
                    // through the tile engine like a CTA group
                    if (tiled(k)) used = run_block(pc, max_ops, end);
                }
                if (!used) {
                    exec(pc);
                    used = 1;
                }
                pc += used;
                if (stop) break;
            }
        }
        Grp::sync();
        if (seg && !(K.seg_flags & KSEG_LAST) && !stop) {
            save_state();
            return;
        }
        finish(tally);
    }

    // Saved state of a shot between segments: frame, gamma, counters and
    // cursors, the packed records, and the 2^k active amplitudes.
    static __host__ __device__ constexpr uint32_t seg_header_bytes() { return 192u; }
    __device__ __forceinline__ void save_state() {
        flush_records();
        unsigned char* d = K.seg_state + shot * K.seg_stride;
        const int r = Grp::rank();
        if (r == 0) {
            uint64_t* w = reinterpret_cast<uint64_t*>(d);
#pragma unroll
            for (int i = 0; i < NW; ++i) {
                w[i] = f.x[i];
                w[NW + i] = f.z[i];
            }
            double* dd = reinterpret_cast<double*>(d + 64);
            dd[0] = gamma.x;
            dd[1] = gamma.y;
            dd[2] = log_prob;
            unsigned long long* u = reinterpret_cast<unsigned long long*>(d + 88);
            u[0] = dust;
            u[1] = bytes;
            u[2] = moved;
            uint32_t* q = reinterpret_cast<uint32_t*>(d + 112);
            q[0] = k;
            q[1] = draw;
            q[2] = next_noise;
            q[3] = ff_pos;
            q[4] = ff_end;
            q[5] = ro_pos;
            q[6] = ro_end;
            q[7] = (discarded ? 2u : 0u) | (reachable ? 4u : 0u);
        }
        uint32_t* words = reinterpret_cast<uint32_t*>(d + seg_header_bytes());
        const uint32_t nwords = K.rec_words + K.det_words + K.obs_words;
        for (uint32_t i = r; i < nwords; i += Grp::size()) words[i] = rec[i * S];
        T* amps = reinterpret_cast<T*>(d + seg_header_bytes() + ((nwords * 4u + 15u) & ~15u));
        for (uint64_t i = r; i < (1ull << k); i += Grp::size()) amps[i] = A(i);
        Grp::sync();
        if (r == 0) {
            const unsigned long long at = atomicAdd(K.seg_count_out, 1ull);
            K.seg_out[at] = (uint32_t)shot;
        }
    }
    __device__ __forceinline__ void load_state() {
        xo = 0;  // amplitudes come back in logical order
        tileF = 0;
        const unsigned char* d = K.seg_state + shot * K.seg_stride;
        const uint64_t* w = reinterpret_cast<const uint64_t*>(d);
#pragma unroll
        for (int i = 0; i < NW; ++i) {
            f.x[i] = w[i];
            f.z[i] = w[NW + i];
        }
        const double* dd = reinterpret_cast<const double*>(d + 64);
        gamma = make_double2(dd[0], dd[1]);
        log_prob = dd[2];
        const unsigned long long* u = reinterpret_cast<const unsigned long long*>(d + 88);
        dust = u[0];
        bytes = u[1];
        moved = u[2];
        const uint32_t* q = reinterpret_cast<const uint32_t*>(d + 112);
        k = q[0];
        draw = q[1];
        next_noise = q[2];
        ff_pos = q[3];
        ff_end = q[4];
        ro_pos = q[5];
        ro_end = q[6];
        stop = false;
        discarded = (q[7] & 2u) != 0;
        reachable = (q[7] & 4u) != 0;
        resolving = false;
        solo = false;
        n_mops = 0;
        rec_dirty = false;
        forced = (K.flags & KF_FORCED_MEAS) ? K.forced_meas + shot * P.slots : nullptr;
        meas_prob = nullptr;
        const int r = Grp::rank();
        const uint32_t* words = reinterpret_cast<const uint32_t*>(d + seg_header_bytes());
        const uint32_t nwords = K.rec_words + K.det_words + K.obs_words;
        for (uint32_t i = r; i < nwords; i += Grp::size()) rec[i * S] = words[i];
        const T* amps = reinterpret_cast<const T*>(d + seg_header_bytes() + ((nwords * 4u + 15u) & ~15u));
        for (uint64_t i = r; i < (1ull << k); i += Grp::size()) A(i) = amps[i];
        Grp::sync();
    }

    __device__ __forceinline__ void reset() {
        // SchrodingerState::reset (svm_state.cc:220-267): only v[0] needs a
        // value; every other amplitude is written by EXPAND before it is read.
        xo = 0;
        tileF = 0;
        f.clear();
        gamma = make_double2(1.0, 0.0);
        k = 0;
        draw = 0;
        stop = false;
        discarded = false;
        reachable = true;
        log_prob = 0.0;
        dust = 0;
        bytes = 0;
        moved = 0;
        resolving = false;
        solo = false;
        n_mops = 0;
        rec_dirty = false;
        forced = (K.flags & KF_FORCED_MEAS) ? K.forced_meas + shot * P.slots : nullptr;
        meas_prob = (K.flags & KF_TRACE) && K.out_meas_prob ? K.out_meas_prob + shot * P.slots : nullptr;
        for (uint32_t i = Grp::rank(); i < K.rec_words; i += Grp::size()) rec[i * S] = 0;
        for (uint32_t i = Grp::rank(); i < K.det_words; i += Grp::size()) det[i * S] = 0;
        for (uint32_t i = Grp::rank(); i < K.obs_words; i += Grp::size()) obs[i * S] = 0;
        if (meas_prob)
            for (uint32_t i = Grp::rank(); i < P.slots; i += Grp::size())
                meas_prob[i] = __longlong_as_double(0x7ff8000000000000ll);
        if (Grp::rank() == 0) A(0) = Cx<R>::make(1.0, 0.0);
        if (K.flags & KF_FORCED_FAULTS) {
            ff_pos = K.fault_off[shot];
            ff_end = K.fault_end ? K.fault_end[shot] : K.fault_off[shot + 1];
            ro_pos = K.ro_off[shot];
            ro_end = K.ro_end ? K.ro_end[shot] : K.ro_off[shot + 1];
            if (ff_pos < ff_end)
                next_noise = K.fault_sites[ff_pos++];
            else
                next_noise = 0xffffffffu;
        } else {
            next_noise = 0;
            draw_next_noise();
        }
        Grp::sync();
    }

    __device__ __forceinline__ void finish(Tally& tally) {
        const bool survived = !discarded && reachable;
        const int r = Grp::rank();
        // observables XOR expected_observables (svm.cc:236-245)
        if (r == 0 && !(K.flags & KF_RAW_PARITY))
            for (uint32_t i = 0; i < P.num_obs && i < P.n_expected; ++i)
                if (P.expected[i]) obs[(i >> 5) * S] ^= 1u << (i & 31);
        Grp::sync();
        if (K.out_meas)
            for (uint32_t w = r; w < K.meas_out_words; w += Grp::size()) {
                uint64_t lo = rec[2 * w * S];
                uint64_t hi = (2 * w + 1 < K.rec_words) ? rec[(2 * w + 1) * S] : 0u;
                uint64_t word = lo | (hi << 32);
                uint32_t base = w * 64;
                if (base + 64 > P.num_meas) {
                    uint32_t keep = P.num_meas > base ? P.num_meas - base : 0;
                    word &= keep >= 64 ? ~0ull : ((1ull << keep) - 1);
                }
                K.out_meas[shot * K.meas_out_words + w] = word;
            }
        if (K.out_det)
            for (uint32_t w = r; w < K.det_out_words; w += Grp::size()) {
                uint64_t lo = det[2 * w * S];
                uint64_t hi = (2 * w + 1 < K.det_words) ? det[(2 * w + 1) * S] : 0u;
                K.out_det[shot * K.det_out_words + w] = lo | (hi << 32);
            }
        if (K.out_obs)
            for (uint32_t w = r; w < K.obs_out_words; w += Grp::size()) {
                uint64_t lo = obs[2 * w * S];
                uint64_t hi = (2 * w + 1 < K.obs_words) ? obs[(2 * w + 1) * S] : 0u;
                K.out_obs[shot * K.obs_out_words + w] = lo | (hi << 32);
            }
        if (r == 0) {
            if (K.out_survived) K.out_survived[shot] = survived ? 1 : 0;
            if (K.out_log_prob) K.out_log_prob[shot] = log_prob;
            if (K.out_final_k) K.out_final_k[shot] = k;
            if (K.out_final_gamma) {
                K.out_final_gamma[2 * shot] = gamma.x;
                K.out_final_gamma[2 * shot + 1] = gamma.y;
            }
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                if (K.out_final_px) K.out_final_px[shot * NW + w] = f.x[w];
                if (K.out_final_pz) K.out_final_pz[shot * NW + w] = f.z[w];
            }
            if (survived && (K.flags & KF_SURVIVORS)) {
                tally.passed++;
                bool any = false;
                for (uint32_t i = 0; i < P.num_obs; ++i)
                    if ((obs[(i >> 5) * S] >> (i & 31)) & 1u) {
                        any = true;
                        atomicAdd(K.counters + 5 + i, 1ull);
                    }
                if (any) tally.logical++;
            }
            tally.dust += dust;
            tally.bytes += bytes;
            tally.moved += moved;
        }
        if (K.out_final_v && shot < K.dump_shots) {
            const uint64_t stride = 1ull << P.peak, n = 1ull << k;
            double* row = K.out_final_v + shot * stride * 2;
            for (uint64_t i = r; i < stride; i += Grp::size()) {
                double re = 0.0, im = 0.0;
                if (i < n) {
                    re = (double)A(i).x;
                    im = (double)A(i).y;
                }
                row[2 * i] = re;
                row[2 * i + 1] = im;
            }
        }
        Grp::sync();
    }
};

// ------------------------------------------------------------------ kernel
// Shared memory per warp (G > 0) or per CTA (G = 0):
//   [interleaved statevectors: 2^peak x S amplitudes, when state_in_smem]
//   [records: (rec_words + det_words + obs_words) x S u32, interleaved]
//   [tile-engine scratch (TileCfg), one-shot groups with global statevectors]
// then, for the whole block: 3 doubles per warp of reduction scratch and a
// broadcast slot.
template <int G>
__host__ __device__ constexpr int shots_per_group_region() {
    return G <= 0 ? 1 : 32 / G;
}

template <typename R, int G, int NW, bool DENSE = false>
__global__ void __launch_bounds__(G == 0 ? 512 : (G < 0 ? 544 : 128), G <= 0 ? 1 : 4)
    svm_sample_kernel(const DevProg P, const KParams K) {
    using Grp = typename GroupOf<G>::type;
    using T = typename Cx<R>::T;
    constexpr int S = Grp::S;
    extern __shared__ __align__(16) unsigned char smem[];
    const int region = Grp::kCta ? 0 : (int)(threadIdx.x >> 5);
    const int regions = Grp::kCta ? 1 : (int)(blockDim.x >> 5);
    const size_t state_bytes = K.state_in_smem ? (size_t)K.state_stride * S * sizeof(T) : 0;
    const size_t rec_bytes = ((size_t)(K.rec_words + K.det_words + K.obs_words) * S * 4 + 15) & ~(size_t)15;
    const size_t region_bytes = (state_bytes + rec_bytes + K.fuse_bytes + 15) & ~(size_t)15;
    unsigned char* rbase = smem + (size_t)region * region_bytes;
    unsigned char* tail = smem + (size_t)regions * region_bytes;
    double* red = reinterpret_cast<double*>(tail);
    unsigned long long* bcast =
        reinterpret_cast<unsigned long long*>(tail + 3 * sizeof(double) * (blockDim.x >> 5));
    uint32_t* rec = reinterpret_cast<uint32_t*>(rbase + state_bytes) + Grp::slot();
    uint32_t* det = rec + (size_t)K.rec_words * S;
    uint32_t* obs = det + (size_t)K.det_words * S;
    unsigned char* fz = K.fuse_bytes ? rbase + state_bytes + rec_bytes : nullptr;
    uint32_t bar_phase = 0;
    if (fz != nullptr) {
        // tile-engine stage barriers of each one-shot group (the CTA, or each
        // warp): initialised once, reused by every pass of every shot the
        // group runs
        if (Grp::rank() == 0) {
            uint64_t* bars = reinterpret_cast<uint64_t*>(fz + Shot<R, Grp, NW, DENSE>::fuse_bar_offset());
            for (int st = 0; st < 2 * kMaxStages; ++st) mbar_init(&bars[st], 1);
            mbar_fence_init();
        }
        __syncthreads();
    }
    // dense blocks: the MMA mbarrier and the CTA's TMEM columns, held for the
    // whole launch (two CTAs per SM use all 512 columns)
    constexpr bool kDenseKernel = DENSE && sizeof(R) == 4 && G <= 0;
    const bool dense = kDenseKernel && (K.flags & KF_DENSE) && fz != nullptr;
    uint32_t* dslot = dense ? reinterpret_cast<uint32_t*>(fz + TileCfg<R, true>::kDenseSlotOffset) : nullptr;
    if constexpr (kDenseKernel) {
        if (dense) {
            if (threadIdx.x == 0) {
                mbar_init(reinterpret_cast<uint64_t*>(dslot), 1);
                mbar_fence_init();
                dslot[3] = 0;
            }
            if (threadIdx.x < 32) {
                tmem_alloc(smem_u32(dslot + 2), kDenseTmemCols);
                tmem_relinquish();
            }
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
        }
    }
    T* v;
    if (K.state_in_smem) {
        v = reinterpret_cast<T*>(rbase) + Grp::slot();
    } else {
        const size_t gid = (size_t)blockIdx.x * regions + region;
        v = reinterpret_cast<T*>(K.state_global) + gid * K.state_stride * S + Grp::slot();
    }
    Tally tally;
    const unsigned long long n_items = K.seg_count_in ? *K.seg_count_in : K.shots;
    for (;;) {
        unsigned long long base = 0;
        if (Grp::kCta) {
            if (threadIdx.x == 0)
                *bcast = (bar_phase >> 31) ? ~0ull : atomicAdd(K.work_counter, 1ull);
            __syncthreads();
            base = *bcast;
            __syncthreads();
        } else {
            // a warp whose tile barriers timed out takes no further shots
            if ((threadIdx.x & 31) == 0)
                base = (bar_phase >> 31) ? ~0ull : atomicAdd(K.work_counter, (unsigned long long)S);
            base = __shfl_sync(0xffffffffu, base, 0);
        }
        if (base >= n_items) break;
        const unsigned long long item = base + Grp::slot();
        if (item < n_items) {
            const unsigned long long shot = K.seg_in ? (unsigned long long)K.seg_in[item] : item;
            Shot<R, Grp, NW, DENSE> s(P, K, v, rec, det, obs, red, fz, &bar_phase, shot);
            s.run(tally);
        }
        if (!Grp::kCta) __syncwarp();
    }
    if constexpr (kDenseKernel) {
        if (dense) {
            tc_fence_before();
            __syncthreads();
            if (threadIdx.x < 32) {
                // after a timed-out wait: wait (bounded) for the MMAs still in
                // flight before their TMEM columns are released
                const uint32_t st = dslot[3];
                if (st >> 31)
                    for (uint32_t it = 0; it < (1u << 20); ++it)
                        if (mbar_try_wait(reinterpret_cast<uint64_t*>(dslot), st & 1u)) break;
                __syncwarp();  // the dealloc is warp-aligned
                tc_fence_after();
                tmem_dealloc(dslot[2], kDenseTmemCols);
            }
        }
    }
    // flush per-lane totals (only group leaders hold non-zero values)
    if (tally.passed) atomicAdd(K.counters + 0, tally.passed);
    if (tally.logical) atomicAdd(K.counters + 1, tally.logical);
    if (tally.dust) atomicAdd(K.counters + 2, tally.dust);
    if (tally.bytes) atomicAdd(K.counters + 3, tally.bytes);
    if (tally.moved) atomicAdd(K.counters + 4, tally.moved);
}

}  // namespace cgpu
