// svm_kernel.cuh -- persistent shot-parallel Schrodinger-VM interpreter for sm_100a.
//
// One *shot group* (a warp, or a whole CTA) runs one shot of the reference's
// bytecode at a time and pulls the next shot index from a global work counter
// as soon as it finishes, so shots that die early (post-selection, unreachable
// forced outcomes) are replaced immediately (work-queue compaction).
//
// Per shot, the factored state |psi> = gamma * U_C * P * (|phi>_A (x) |0>_D)
// (src/clifft/svm/svm.h:92-103) is held as:
//   * the 2^k active amplitudes in shared memory (small k) or in a per-group
//     global slab (large k), complex FP32 or FP64;
//   * the Pauli frame p_x / p_z as NW 64-bit words in registers of every thread
//     of the group (updated redundantly, so frame opcodes cost no barrier);
//   * gamma as an FP64 complex in registers;
//   * measurement / detector / observable records as bit arrays in shared
//     memory.
// Branch probabilities and expectation values are reduced in FP64 with a fixed
// summation order, so every thread of the group derives the same outcome from
// the same counter-based Philox draw (identical control flow, no broadcast).
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
    uint32_t rec_words;   // u32 words of measurement record per group (>= ceil(slots/32))
    uint32_t det_words;   // u32 words of detector record
    uint32_t obs_words;   // u32 words of observable record
    uint32_t meas_out_words;  // u64 words per shot in outputs
    uint32_t det_out_words;
    uint32_t obs_out_words;
    uint32_t state_in_smem;
    uint64_t state_stride;  // amplitudes per group slab
    void* state_global;     // global slab base (when !state_in_smem)
    unsigned long long* work_counter;
    unsigned long long* counters;  // [0] passed, [1] logical errors, [2] dust clamps, [3] algorithmic bytes, [4..] observable ones
    int* error_word;               // first device-side error code (0 = none)
    // forced inputs
    const uint8_t* forced_meas;
    const uint32_t* fault_off;
    const uint32_t* fault_sites;
    const uint32_t* fault_chan;
    const uint32_t* ro_off;
    const uint32_t* ro_entries;
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
};

enum : uint32_t {
    KF_SURVIVORS = 0x01u,
    KF_FORCED_MEAS = 0x02u,
    KF_FORCED_FAULTS = 0x04u,
    KF_TRACE = 0x10u,
};

enum : int {
    DEV_ERR_ZERO_NORM = 1,
    DEV_ERR_BAD_OPCODE = 2,
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

template <typename T>
__device__ __forceinline__ T cadd(T a, T b) {
    T r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    return r;
}
template <typename T>
__device__ __forceinline__ T csub(T a, T b) {
    T r;
    r.x = a.x - b.x;
    r.y = a.y - b.y;
    return r;
}
template <typename T>
__device__ __forceinline__ T cmul(T a, T b) {
    T r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <typename T, typename S>
__device__ __forceinline__ T cscale(T a, S s) {
    T r;
    r.x = a.x * s;
    r.y = a.y * s;
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
    return x * x + y * y;
}
__device__ __forceinline__ double2 dmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// kInvSqrt2 = std::numbers::sqrt2 / 2 (src/clifft/util/constants.h) and the
// separate 1.0 / std::sqrt(2.0) that EXPAND scales gamma by
// (src/clifft/svm/svm_kernels.inl:895).
#define CGPU_INV_SQRT2 0.70710678118654757
#define CGPU_EXPAND_SCALE 0.70710678118654746

// ---------------------------------------------------------------- philox
// Philox4x32-10 (Salmon et al., SC'11). Draw d of shot s uses counter
// (d >> 1, 0, s_lo, s_hi) and key (seed_lo, seed_hi); even draws take words
// (0, 1), odd draws words (2, 3); 53 high bits -> [0, 1) as the reference's
// random_double (src/clifft/svm/svm.h:150).
__device__ __forceinline__ double philox_uniform(uint64_t seed, uint64_t shot, uint32_t draw) {
    uint32_t c0 = draw >> 1, c1 = 0u, c2 = (uint32_t)shot, c3 = (uint32_t)(shot >> 32);
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
struct WarpGroup {
    static constexpr bool kIsWarp = true;
    __device__ static __forceinline__ int size() { return 32; }
    __device__ static __forceinline__ int rank() { return threadIdx.x & 31; }
    __device__ static __forceinline__ int local() { return threadIdx.x >> 5; }
    __device__ static __forceinline__ int per_block() { return blockDim.x >> 5; }
    __device__ static __forceinline__ void sync() { __syncwarp(); }
};
struct CtaGroup {
    static constexpr bool kIsWarp = false;
    __device__ static __forceinline__ int size() { return blockDim.x; }
    __device__ static __forceinline__ int rank() { return threadIdx.x; }
    __device__ static __forceinline__ int local() { return 0; }
    __device__ static __forceinline__ int per_block() { return 1; }
    __device__ static __forceinline__ void sync() { __syncthreads(); }
};

__device__ __forceinline__ uint64_t ins0(uint64_t v, uint32_t pos) {
    uint64_t m = (1ull << pos) - 1;
    return (v & m) | ((v & ~m) << 1);
}
__device__ __forceinline__ uint64_t ins00(uint64_t v, uint32_t a, uint32_t b) {
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return ins0(ins0(v, lo), hi);
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
            if ((uint32_t)i == (a >> 6)) {
                uint64_t m = 1ull << (a & 63);
                w[i] = b ? (w[i] | m) : (w[i] & ~m);
            }
    }
    __device__ static __forceinline__ void flip(uint64_t* w, uint32_t a, int b) {
        if (b) {
#pragma unroll
            for (int i = 0; i < NW; ++i)
                if ((uint32_t)i == (a >> 6)) w[i] ^= 1ull << (a & 63);
        }
    }
    __device__ __forceinline__ int px(uint32_t a) const { return get(x, a); }
    __device__ __forceinline__ int pz(uint32_t a) const { return get(z, a); }
};

// Shared per-group scratch.
struct GroupShared {
    uint32_t* rec;     // rec_words
    uint32_t* det;     // det_words
    uint32_t* obs;     // obs_words
    double* red;       // reduction scratch: 3 * warps
    unsigned long long* bcast;
};

// FP64 group reduction of N values with a fixed order: warp tree to lane 0,
// warps combined in index order by every thread. All threads return the same
// bits.
template <class G, int N>
__device__ __forceinline__ void group_reduce(double (&v)[N], double* red) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int j = 0; j < N; ++j) v[j] += __shfl_down_sync(0xffffffffu, v[j], off);
    if (G::kIsWarp) {
#pragma unroll
        for (int j = 0; j < N; ++j) v[j] = __shfl_sync(0xffffffffu, v[j], 0);
        return;
    }
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

template <class G>
__device__ __forceinline__ unsigned long long group_next_shot(unsigned long long* counter,
                                                              unsigned long long* bcast) {
    unsigned long long s = 0;
    if (G::rank() == 0) s = atomicAdd(counter, 1ull);
    if (G::kIsWarp) return __shfl_sync(0xffffffffu, s, 0);
    if (G::rank() == 0) *bcast = s;
    __syncthreads();
    s = *bcast;
    __syncthreads();
    return s;
}

__device__ __forceinline__ int rec_get(const uint32_t* r, uint32_t i) { return (int)((r[i >> 5] >> (i & 31)) & 1u); }

// --------------------------------------------------------------- the shot
template <typename R, class G, int NW>
struct Shot {
    using T = typename Cx<R>::T;
    const DevProg& P;
    const KParams& K;
    T* v;
    GroupShared sh;
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

    __device__ Shot(const DevProg& p, const KParams& kp, T* vv, GroupShared s, uint64_t sh_idx)
        : P(p), K(kp), v(vv), sh(s), shot(sh_idx) {}

    // algorithmic bytes of one sweep touching `amps` amplitudes (read + write counted separately)
    __device__ __forceinline__ void account(uint64_t amps) { bytes += amps * sizeof(T); }

    __device__ __forceinline__ double uniform() { return philox_uniform(K.seed, K.first_shot + shot, draw++); }

    __device__ __forceinline__ void phase(double2 p) { gamma = dmul(gamma, p); }
    __device__ __forceinline__ void negate_gamma() { gamma = make_double2(-gamma.x, -gamma.y); }

    __device__ __forceinline__ void flush_records() {
        if (rec_dirty) {
            G::sync();
            rec_dirty = false;
        }
    }
    __device__ __forceinline__ void write_meas(uint32_t idx, int bit, double prob) {
        if (G::rank() == 0) {
            uint32_t m = 1u << (idx & 31);
            sh.rec[idx >> 5] = bit ? (sh.rec[idx >> 5] | m) : (sh.rec[idx >> 5] & ~m);
            if (meas_prob) meas_prob[idx] = prob;
        }
        rec_dirty = true;
    }

    // SchrodingerState::scale_magnitude (src/clifft/svm/svm.h:177-186). The
    // lazy-renormalisation window is 1e+-100 in FP64 and 1e+-20 in FP32 so the
    // FP32 amplitudes never approach their exponent range.
    __device__ void scale_magnitude(double s) {
        gamma.x *= s;
        gamma.y *= s;
        const double hi = sizeof(R) == 8 ? 1e100 : 1e20;
        const double lo = sizeof(R) == 8 ? 1e-100 : 1e-20;
        double g = hypot(gamma.x, gamma.y);
        if (g > hi || (g < lo && g > 0.0)) {
            uint64_t n = 1ull << k;
            for (uint64_t i = G::rank(); i < n; i += G::size()) v[i] = cscale(v[i], (R)g);
            G::sync();
            account(2 * n);
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

    // ---------------------------------------------------------- array ops
    // exec_array_cnot (svm_kernels.inl:124-252)
    __device__ void array_cnot(uint32_t c, uint32_t t) {
        const uint64_t n = 1ull << (k - 2), cb = 1ull << c, tb = 1ull << t;
        for (uint64_t i = G::rank(); i < n; i += G::size()) {
            uint64_t b0 = ins00(i, c, t) | cb;
            T a = v[b0], b = v[b0 | tb];
            v[b0] = b;
            v[b0 | tb] = a;
        }
        G::sync();
        account(1ull << k);
        frame_cnot(c, t);
    }
    // exec_array_cz (svm_kernels.inl:255-365)
    __device__ void array_cz(uint32_t c, uint32_t t) {
        const uint64_t n = 1ull << (k - 2), both = (1ull << c) | (1ull << t);
        for (uint64_t i = G::rank(); i < n; i += G::size()) {
            uint64_t idx = ins00(i, c, t) | both;
            v[idx] = cneg(v[idx]);
        }
        G::sync();
        account(1ull << (k - 1));
        frame_cz(c, t);
    }
    // exec_array_swap (svm_kernels.inl:369-458)
    __device__ void array_swap(uint32_t a, uint32_t b) {
        const uint64_t n = 1ull << (k - 2), ab = 1ull << a, bb = 1ull << b;
        for (uint64_t i = G::rank(); i < n; i += G::size()) {
            uint64_t base = ins00(i, a, b);
            T x = v[base | ab], y = v[base | bb];
            v[base | ab] = y;
            v[base | bb] = x;
        }
        G::sync();
        account(1ull << k);
        frame_swap(a, b);
    }
    // exec_array_multi_cnot (svm_kernels.inl:464-550)
    __device__ void array_multi_cnot(uint32_t t, uint64_t mask) {
        const uint64_t n = 1ull << (k - 1), tb = 1ull << t;
        for (uint64_t i = G::rank(); i < n; i += G::size()) {
            uint64_t a = ins0(i, t);
            if (__popcll(a & mask) & 1) {
                T x = v[a], y = v[a | tb];
                v[a] = y;
                v[a | tb] = x;
            }
        }
        G::sync();
        account(1ull << k);
        for (uint32_t c = 0; c < k; ++c)
            if ((mask >> c) & 1ull) frame_cnot(c, t);
    }
    // exec_array_multi_cz (svm_kernels.inl:558-635)
    __device__ void array_multi_cz(uint32_t c, uint64_t mask) {
        const uint64_t n = 1ull << (k - 1), cb = 1ull << c;
        for (uint64_t i = G::rank(); i < n; i += G::size()) {
            uint64_t a = ins0(i, c) | cb;
            if (__popcll(a & mask) & 1) v[a] = cneg(v[a]);
        }
        G::sync();
        account(1ull << k);
        for (uint32_t t = 0; t < k; ++t)
            if ((mask >> t) & 1ull) frame_cz(c, t);
    }
    // exec_array_h (svm_kernels.inl:639-744)
    __device__ void array_h(uint32_t a) {
        const uint64_t n = 1ull << (k - 1), ab = 1ull << a;
        const R s = (R)CGPU_INV_SQRT2;
        for (uint64_t i = G::rank(); i < n; i += G::size()) {
            uint64_t i0 = ins0(i, a), i1 = i0 | ab;
            T x = v[i0], y = v[i1];
            v[i0] = cscale(cadd(x, y), s);
            v[i1] = cscale(csub(x, y), s);
        }
        G::sync();
        account(2ull << k);
        frame_h(a);
    }
    // apply_phase_waterfall (svm_kernels.inl:764-830)
    __device__ void phase_sweep(uint32_t a, double re, double im) {
        const uint64_t n = 1ull << (k - 1), ab = 1ull << a;
        const T ph = Cx<R>::make(re, im);
        for (uint64_t i = G::rank(); i < n; i += G::size()) {
            uint64_t idx = ins0(i, a) | ab;
            v[idx] = cmul(v[idx], ph);
        }
        G::sync();
        account(1ull << k);
    }
    // exec_array_t / t_dag / rot (svm_kernels.inl:951-988,1044-1061)
    __device__ void array_rot(uint32_t a, double zr, double zi) {
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
    // exec_expand / expand_with_phase / exec_expand_{t,t_dag,rot}
    // (svm_kernels.inl:876-1081)
    __device__ void expand(uint32_t a, bool with_phase, double zr, double zi) {
        const uint64_t half = 1ull << k;
        int x = with_phase ? f.px(a) : 0;
        if (!with_phase) {
            for (uint64_t i = G::rank(); i < half; i += G::size()) v[half + i] = v[i];
        } else {
            const T ph = Cx<R>::make(zr, x ? -zi : zi);
            for (uint64_t i = G::rank(); i < half; i += G::size()) v[half + i] = cmul(v[i], ph);
        }
        G::sync();
        account(2ull << k);
        k++;
        scale_magnitude(CGPU_EXPAND_SCALE);
        if (with_phase && x) phase(make_double2(zr, zi));
    }
    // exec_array_u2 (svm_kernels.inl:1087-1297)
    __device__ void array_u2(uint32_t a, uint32_t cp) {
        const double* node = P.u2 + (size_t)cp * CLIFFT_U2_DOUBLES_PER_NODE;
        int st = (f.pz(a) << 1) | f.px(a);
        const double* m = node + st * 10;
        phase(make_double2(m[8], m[9]));
        uint8_t out = P.u2_out[cp * 4 + st];
        Frame<NW>::put(f.x, a, out & 1);
        Frame<NW>::put(f.z, a, (out >> 1) & 1);
        if (a >= k) return;
        const T m00 = Cx<R>::make(m[0], m[1]), m01 = Cx<R>::make(m[2], m[3]);
        const T m10 = Cx<R>::make(m[4], m[5]), m11 = Cx<R>::make(m[6], m[7]);
        const uint64_t n = 1ull << (k - 1), ab = 1ull << a;
        for (uint64_t i = G::rank(); i < n; i += G::size()) {
            uint64_t i0 = ins0(i, a), i1 = i0 | ab;
            T x = v[i0], y = v[i1];
            v[i0] = cadd(cmul(m00, x), cmul(m01, y));
            v[i1] = cadd(cmul(m10, x), cmul(m11, y));
        }
        G::sync();
        account(2ull << k);
    }
    // exec_array_u4 (svm_kernels.inl:1310-1531)
    __device__ void array_u4(uint32_t lo, uint32_t hi, uint32_t cp) {
        const double* node = P.u4 + (size_t)cp * CLIFFT_U4_DOUBLES_PER_NODE;
        int st = (f.pz(hi) << 3) | (f.px(hi) << 2) | (f.pz(lo) << 1) | f.px(lo);
        const double* e = node + st * 34;
        phase(make_double2(e[32], e[33]));
        uint8_t out = P.u4_out[cp * 16 + st];
        Frame<NW>::put(f.x, lo, out & 1);
        Frame<NW>::put(f.z, lo, (out >> 1) & 1);
        Frame<NW>::put(f.x, hi, (out >> 2) & 1);
        Frame<NW>::put(f.z, hi, (out >> 3) & 1);
        T m[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) m[j] = Cx<R>::make(e[2 * j], e[2 * j + 1]);
        const uint64_t n = 1ull << (k - 2), lb = 1ull << lo, hb = 1ull << hi;
        for (uint64_t i = G::rank(); i < n; i += G::size()) {
            uint64_t b = ins00(i, lo, hi);
            T x0 = v[b], x1 = v[b | lb], x2 = v[b | hb], x3 = v[b | lb | hb];
            T y[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                T acc = cmul(m[r * 4 + 0], x0);
                acc = cadd(acc, cmul(m[r * 4 + 1], x1));
                acc = cadd(acc, cmul(m[r * 4 + 2], x2));
                acc = cadd(acc, cmul(m[r * 4 + 3], x3));
                y[r] = acc;
            }
            v[b] = y[0];
            v[b | lb] = y[1];
            v[b | hb] = y[2];
            v[b | lb | hb] = y[3];
        }
        G::sync();
        account(2ull << k);
    }

    // ------------------------------------------------------- measurements
    // Outcome selection shared by sampling and forced modes: sample_branch
    // (src/clifft/svm/svm_internal.h:65-79) and forced_log_increment
    // (src/clifft/svm/svm_forced_kernels.cc:42-60). `want` is the forced
    // branch or -1. Returns the branch, or -1 when the forced branch is
    // unreachable.
    __device__ int choose(double p0, double p1, double total, int want, double* prob) {
        const double eps = K.dust_eps * total;
        if (want < 0) {
            if (p1 <= eps) {
                if (p1 > 0.0) dust++;
                *prob = 1.0;
                return 0;
            }
            if (p0 <= eps) {
                if (p0 > 0.0) dust++;
                *prob = 1.0;
                return 1;
            }
            double r = uniform();
            int b = (r * total < p0) ? 0 : 1;
            *prob = (b ? p1 : p0) / total;
            return b;
        }
        if (p1 <= eps) {
            if (p1 > 0.0) dust++;
            *prob = 1.0;
            return want == 0 ? 0 : -1;
        }
        if (p0 <= eps) {
            if (p0 > 0.0) dust++;
            *prob = 1.0;
            return want == 1 ? 1 : -1;
        }
        double pb = (want ? p1 : p0) / total;
        log_prob += log(pb);
        *prob = pb;
        return want;
    }

    __device__ __forceinline__ int forced_bit(uint32_t idx) const { return forced ? (int)forced[idx] : -1; }

    // exec_meas_dormant_static + FLAG_IDENTITY shortcut (svm_kernels.inl:1539-1545,
    // 2361-2369) and forced variants (svm_forced_kernels.cc:64-88)
    __device__ void meas_dormant_static(uint32_t a, uint32_t idx, int sign, bool identity) {
        int det = identity ? sign : (f.px(a) ^ sign);
        int want = forced_bit(idx);
        if (want >= 0 && want != det) {
            reachable = false;
            stop = true;
            return;
        }
        write_meas(idx, det, 1.0);
    }
    // exec_meas_dormant_random (svm_kernels.inl:1550-1566), forced
    // (svm_forced_kernels.cc:90-110)
    __device__ void meas_dormant_random(uint32_t a, uint32_t idx, int sign) {
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
    // exec_meas_active_diagonal (svm_kernels.inl:1573-1627), forced
    // (svm_forced_kernels.cc:112-158)
    __device__ void meas_diagonal(uint32_t a, uint32_t idx, int sign) {
        const uint64_t half = 1ull << (k - 1);
        int pxv = f.px(a), pzv = f.pz(a);
        double acc[2] = {0.0, 0.0};
        for (uint64_t i = G::rank(); i < half; i += G::size()) {
            acc[0] += cnorm_d(v[i]);
            acc[1] += cnorm_d(v[i + half]);
        }
        group_reduce<G, 2>(acc, sh.red);
        account(1ull << k);
        double p0 = acc[0], p1 = acc[1], total = p0 + p1;
        if (!(total > 0.0)) {
            if (G::rank() == 0) atomicCAS(K.error_word, 0, DEV_ERR_ZERO_NORM);
            stop = true;
            return;
        }
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
            for (uint64_t i = G::rank(); i < half; i += G::size()) v[i] = v[i + half];
            G::sync();
            account(1ull << k);
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
    __device__ void meas_interfere(uint32_t fa, uint32_t t, uint32_t idx, int sign) {
        const bool swapped = fa != t;
        if (swapped) frame_swap(fa, t);
        int pxv = f.px(t), pzv = f.pz(t);
        const uint64_t half = 1ull << t, fb = 1ull << fa;
        double acc[2] = {0.0, 0.0};
        for (uint64_t i = G::rank(); i < half; i += G::size()) {
            uint64_t a0, a1;
            if (swapped) {
                a0 = (i & ~fb) | (((i >> fa) & 1ull) << t);
                a1 = a0 | fb;
            } else {
                a0 = i;
                a1 = i + half;
            }
            T x = v[a0], y = v[a1];
            acc[0] += cnorm_d(cadd(x, y));
            acc[1] += cnorm_d(csub(x, y));
        }
        group_reduce<G, 2>(acc, sh.red);
        account((1ull << k) * 2 + (1ull << (k - 1)));
        double pp = acc[0], pm = acc[1], total = pp + pm;
        if (!(total > 0.0)) {
            if (G::rank() == 0) atomicCAS(K.error_word, 0, DEV_ERR_ZERO_NORM);
            stop = true;
            return;
        }
        int want = forced_bit(idx);
        if (want >= 0) want = want ^ sign ^ pzv;
        double prob;
        int bx = choose(pp, pm, total, want, &prob);
        if (bx < 0) {
            reachable = false;
            stop = true;
            return;
        }
        int m_abs = bx ^ pzv;
        const R s = (R)CGPU_INV_SQRT2;
        if (!swapped) {
            for (uint64_t i = G::rank(); i < half; i += G::size()) {
                T x = v[i], y = v[i + half];
                v[i] = cscale(bx ? csub(x, y) : cadd(x, y), s);
            }
            G::sync();
        } else {
            const uint64_t q = half >> 1;  // outputs with bit fa clear, then set
            for (int pass = 0; pass < 2; ++pass) {
                for (uint64_t j = G::rank(); j < q; j += G::size()) {
                    uint64_t i = ins0(j, fa) | (pass ? fb : 0ull);
                    uint64_t a0 = pass ? ((i & ~fb) | half) : i;
                    uint64_t a1 = a0 | fb;
                    T x = v[a0], y = v[a1];
                    v[i] = cscale(bx ? csub(x, y) : cadd(x, y), s);
                }
                G::sync();
            }
        }
        double pb = bx ? pm : pp;
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

    // ------------------------------------------------- classical / noise
    // apply_pauli_to_frame (svm_kernels.inl:1812-1865)
    __device__ void apply_pauli(const uint64_t* ex, const uint64_t* ez, int sign) {
        int par = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) par += __popcll(f.x[w] & ez[w]);
        if (par & 1) negate_gamma();
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            f.x[w] ^= ex[w];
            f.z[w] ^= ez[w];
        }
        if (sign) negate_gamma();
    }
    // SchrodingerState::draw_next_noise (src/clifft/svm/svm.h:231-248)
    __device__ void draw_next_noise() {
        const uint32_t n = P.n_sites;
        if (n == 0 || next_noise >= n) {
            next_noise = 0xffffffffu;
            return;
        }
        double cur = next_noise == 0 ? 0.0 : P.hazards[next_noise - 1];
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
    __device__ void noise(uint32_t site) {
        if (site != next_noise) return;
        const uint32_t c0 = P.site_off[site], c1 = P.site_off[site + 1];
        if (K.flags & KF_FORCED_FAULTS) {
            uint32_t c = c0 + K.fault_chan[ff_pos - 1];
            if (c < c1) apply_pauli(P.chan_x + (size_t)c * NW, P.chan_z + (size_t)c * NW, 0);
            next_noise = ff_pos < ff_end ? K.fault_sites[ff_pos++] : 0xffffffffu;
            return;
        }
        double r = uniform() * P.site_psum[site], cum = 0.0;
        for (uint32_t c = c0; c < c1; ++c) {
            cum += P.chan_prob[c];
            if (r < cum) {
                apply_pauli(P.chan_x + (size_t)c * NW, P.chan_z + (size_t)c * NW, 0);
                break;
            }
        }
        next_noise++;
        draw_next_noise();
    }
    // exec_readout_noise (svm_kernels.inl:1937-1959)
    __device__ void readout_noise(uint32_t e) {
        bool fire = false;
        if (K.flags & KF_FORCED_FAULTS) {
            if (ro_pos < ro_end && K.ro_entries[ro_pos] == e) {
                fire = true;
                ro_pos++;
            }
        } else {
            fire = uniform() < P.ro_prob[e];
        }
        if (fire) {
            flush_records();
            uint32_t mi = P.ro_meas[e];
            if (G::rank() == 0) sh.rec[mi >> 5] ^= 1u << (mi & 31);
            rec_dirty = true;
        }
    }
    __device__ __forceinline__ int list_parity(const uint32_t* off, const uint32_t* tg, uint32_t l) {
        int p = 0;
        for (uint32_t i = off[l]; i < off[l + 1]; ++i) p ^= rec_get(sh.rec, tg[i]);
        return p;
    }
    // exec_exp_val (svm_kernels.inl:2031-2173)
    __device__ void exp_val(uint32_t cp, uint32_t out_idx) {
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
            for (uint64_t j = G::rank(); j < dim; j += G::size()) {
                T a = v[j], b = v[j ^ xa];
                double ar = (double)a.x, ai = (double)a.y, br = (double)b.x, bi = -(double)b.y;
                acc[2] += ar * ar + ai * ai;
                double zs = (__popcll(j & za) & 1) ? -1.0 : 1.0;
                ar *= zs;
                ai *= zs;
                acc[0] += br * ar - bi * ai;
                acc[1] += br * ai + bi * ar;
            }
            group_reduce<G, 3>(acc, sh.red);
            account(1ull << k);
            double2 num = dmul(make_double2(acc[0], acc[1]), iph);
            if (acc[2] > 0.0) result = num.x / acc[2];
            result = fmin(1.0, fmax(-1.0, result));
        }
        if (G::rank() == 0 && K.out_exp) K.out_exp[shot * P.num_exp + out_idx] = result;
    }

    // ------------------------------------------------------------ driver
    __device__ void run() {
        // SchrodingerState::reset (svm_state.cc:220-267): only v[0] needs a
        // value; every other amplitude is written by EXPAND before it is read.
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
        rec_dirty = false;
        forced = (K.flags & KF_FORCED_MEAS) ? K.forced_meas + shot * P.slots : nullptr;
        meas_prob = (K.flags & KF_TRACE) && K.out_meas_prob ? K.out_meas_prob + shot * P.slots : nullptr;
        for (uint32_t i = G::rank(); i < K.rec_words; i += G::size()) sh.rec[i] = 0;
        for (uint32_t i = G::rank(); i < K.det_words; i += G::size()) sh.det[i] = 0;
        for (uint32_t i = G::rank(); i < K.obs_words; i += G::size()) sh.obs[i] = 0;
        if (meas_prob)
            for (uint32_t i = G::rank(); i < P.slots; i += G::size()) meas_prob[i] = __longlong_as_double(0x7ff8000000000000ll);
        if (G::rank() == 0) v[0] = Cx<R>::make(1.0, 0.0);
        if (K.flags & KF_FORCED_FAULTS) {
            ff_pos = K.fault_off[shot];
            ff_end = K.fault_off[shot + 1];
            ro_pos = K.ro_off[shot];
            ro_end = K.ro_off[shot + 1];
            if (ff_pos < ff_end)
                next_noise = K.fault_sites[ff_pos++];
            else
                next_noise = 0xffffffffu;
        } else {
            next_noise = 0;
            draw_next_noise();
        }
        G::sync();

        const uint4* ip = P.instr;
        for (uint32_t pc = 0; pc < P.n_instr && !stop; ++pc) {
            const uint4 w0 = __ldg(ip + 2 * pc), w1 = __ldg(ip + 2 * pc + 1);
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
                    if (k > a1) phase_sweep(a1, 0.0, 1.0);
                    frame_s(a1, false);
                    break;
                case CLIFFT_OP_ARRAY_S_DAG:
                    if (k > a1) phase_sweep(a1, 0.0, -1.0);
                    frame_s(a1, true);
                    break;
                case CLIFFT_OP_ARRAY_T: array_rot(a1, CGPU_INV_SQRT2, CGPU_INV_SQRT2); break;
                case CLIFFT_OP_ARRAY_T_DAG: array_rot(a1, CGPU_INV_SQRT2, -CGPU_INV_SQRT2); break;
                case CLIFFT_OP_ARRAY_ROT:
                    array_rot(a1, __longlong_as_double(((long long)p1 << 32) | p0),
                              __longlong_as_double(((long long)w1.y << 32) | w1.x));
                    break;
                case CLIFFT_OP_ARRAY_U2: array_u2(a1, p0); break;
                case CLIFFT_OP_ARRAY_U4: array_u4(a1, a2, p0); break;
                case CLIFFT_OP_EXPAND: expand(a1, false, 0.0, 0.0); break;
                case CLIFFT_OP_EXPAND_T: expand(a1, true, CGPU_INV_SQRT2, CGPU_INV_SQRT2); break;
                case CLIFFT_OP_EXPAND_T_DAG: expand(a1, true, CGPU_INV_SQRT2, -CGPU_INV_SQRT2); break;
                case CLIFFT_OP_EXPAND_ROT:
                    expand(a1, true, __longlong_as_double(((long long)p1 << 32) | p0),
                           __longlong_as_double(((long long)w1.y << 32) | w1.x));
                    break;
                case CLIFFT_OP_MEAS_DORMANT_STATIC:
                    meas_dormant_static(a1, p0, sign, (fl & CLIFFT_FLAG_IDENTITY) != 0);
                    break;
                case CLIFFT_OP_MEAS_DORMANT_RANDOM: meas_dormant_random(a1, p0, sign); break;
                case CLIFFT_OP_MEAS_ACTIVE_DIAGONAL: meas_diagonal(a1, p0, sign); break;
                case CLIFFT_OP_MEAS_ACTIVE_INTERFERE: meas_interfere(a1, a1, p0, sign); break;
                case CLIFFT_OP_SWAP_MEAS_INTERFERE: meas_interfere(a1, a2, p0, sign); break;
                case CLIFFT_OP_APPLY_PAULI:
                    flush_records();
                    if (rec_get(sh.rec, p1))
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
                    int par = (fl & CLIFFT_FLAG_EXPECTED_ONE) ? 1 : 0;
                    par ^= list_parity(P.det_off, P.det_tg, p0);
                    if (G::rank() == 0 && par) sh.det[p1 >> 5] |= 1u << (p1 & 31);
                    break;
                }
                case CLIFFT_OP_POSTSELECT: {
                    flush_records();
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
                    if (G::rank() == 0 && par) sh.obs[p1 >> 5] ^= 1u << (p1 & 31);
                    break;
                }
                case CLIFFT_OP_EXP_VAL: exp_val(p0, p1); break;
                default:
                    if (G::rank() == 0) atomicCAS(K.error_word, 0, DEV_ERR_BAD_OPCODE);
                    stop = true;
                    break;
            }
        }
        G::sync();
        finish();
    }

    __device__ void finish() {
        const bool survived = !discarded && reachable;
        const int r = G::rank();
        // observables XOR expected_observables (svm.cc:236-245)
        if (r == 0)
            for (uint32_t i = 0; i < P.num_obs && i < P.n_expected; ++i)
                if (P.expected[i]) sh.obs[i >> 5] ^= 1u << (i & 31);
        G::sync();
        if (K.out_meas)
            for (uint32_t w = r; w < K.meas_out_words; w += G::size()) {
                uint64_t lo = sh.rec[2 * w], hi = (2 * w + 1 < K.rec_words) ? sh.rec[2 * w + 1] : 0u;
                uint64_t word = lo | (hi << 32);
                uint32_t base = w * 64;
                if (base + 64 > P.num_meas) {
                    uint32_t keep = P.num_meas > base ? P.num_meas - base : 0;
                    word &= keep >= 64 ? ~0ull : ((1ull << keep) - 1);
                }
                K.out_meas[shot * K.meas_out_words + w] = word;
            }
        if (K.out_det)
            for (uint32_t w = r; w < K.det_out_words; w += G::size()) {
                uint64_t lo = sh.det[2 * w], hi = (2 * w + 1 < K.det_words) ? sh.det[2 * w + 1] : 0u;
                K.out_det[shot * K.det_out_words + w] = lo | (hi << 32);
            }
        if (K.out_obs)
            for (uint32_t w = r; w < K.obs_out_words; w += G::size()) {
                uint64_t lo = sh.obs[2 * w], hi = (2 * w + 1 < K.obs_words) ? sh.obs[2 * w + 1] : 0u;
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
                atomicAdd(K.counters + 0, 1ull);
                bool any = false;
                for (uint32_t i = 0; i < P.num_obs; ++i)
                    if ((sh.obs[i >> 5] >> (i & 31)) & 1u) {
                        any = true;
                        atomicAdd(K.counters + 4 + i, 1ull);
                    }
                if (any) atomicAdd(K.counters + 1, 1ull);
            }
            if (dust) atomicAdd(K.counters + 2, dust);
            if (bytes) atomicAdd(K.counters + 3, bytes);
        }
        if (K.out_final_v && shot < K.dump_shots) {
            const uint64_t stride = 1ull << P.peak, n = 1ull << k;
            double* row = K.out_final_v + shot * stride * 2;
            for (uint64_t i = r; i < stride; i += G::size()) {
                double re = 0.0, im = 0.0;
                if (i < n) {
                    re = (double)v[i].x;
                    im = (double)v[i].y;
                }
                row[2 * i] = re;
                row[2 * i + 1] = im;
            }
        }
        G::sync();
    }
};

// ------------------------------------------------------------------ kernel
template <typename R, class G, int NW>
__global__ void __launch_bounds__(1024) svm_sample_kernel(const DevProg P, const KParams K) {
    using T = typename Cx<R>::T;
    extern __shared__ __align__(16) unsigned char smem[];
    const int gl = G::local();
    const int per_block = G::per_block();
    // shared layout per group: [state (optional)] [rec] [det] [obs]; then
    // block-wide: reduction scratch (3 doubles per warp) + broadcast slot.
    const size_t state_bytes = K.state_in_smem ? (size_t)K.state_stride * sizeof(T) : 0;
    const size_t rec_bytes = (size_t)(K.rec_words + K.det_words + K.obs_words) * 4;
    const size_t group_bytes = (state_bytes + rec_bytes + 15) & ~(size_t)15;
    unsigned char* gbase = smem + (size_t)gl * group_bytes;
    unsigned char* tail = smem + (size_t)per_block * group_bytes;
    GroupShared sh;
    sh.rec = reinterpret_cast<uint32_t*>(gbase + state_bytes);
    sh.det = sh.rec + K.rec_words;
    sh.obs = sh.det + K.det_words;
    sh.red = reinterpret_cast<double*>(tail);
    sh.bcast = reinterpret_cast<unsigned long long*>(tail + 3 * sizeof(double) * (blockDim.x >> 5));
    T* v;
    if (K.state_in_smem) {
        v = reinterpret_cast<T*>(gbase);
    } else {
        const size_t gid = (size_t)blockIdx.x * per_block + gl;
        v = reinterpret_cast<T*>(K.state_global) + gid * K.state_stride;
    }
    for (;;) {
        unsigned long long shot = group_next_shot<G>(K.work_counter, sh.bcast);
        if (shot >= K.shots) break;
        Shot<R, G, NW> s(P, K, v, sh, shot);
        s.run();
    }
}

}  // namespace cgpu
