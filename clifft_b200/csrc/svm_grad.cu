// svm_grad.cu -- adjoint gradients of expectation values (clifft_gpu_expval_grad).
//
// For a measurement-free, noise-free program the statevector after
// instruction t is v_t = M_t v_{t-1}, with M_t a unitary on the active axes
// (array opcodes), an isometry that opens axis k (EXPAND*: the lower half
// copied to the upper half times a phase, here scaled by 1/sqrt(2) so v stays
// normalised) or the identity (frame opcodes, which only move the Pauli frame).
// An EXP_VAL at instruction t_e reads <P_e> = <v|O_e|v> / <v|v>, where O_e is
// the Pauli mask conjugated by the frame at t_e (the executor's exec_exp_val,
// src/clifft/svm/svm_kernels.inl:2031-2173, restated in svm_kernel.cuh).
//
// Adjoint method (one CTA per (parameter vector, EXP_VAL) pair): run forward
// to t_e, set lambda = O_e v, then walk the bytecode backwards. At a rotation
// t (ARRAY_ROT on an active axis a, or EXPAND_ROT opening axis a), whose phase
// e^{i s phi} multiplies the half with bit a set (s = -1 when the frame has X
// on a, as the executor conjugates the phase there),
//     d<P_e>/dphi = 2 Re <lambda_t | i s Pi_a v_t> / <v|v>
//                 = -2 s Im( sum_{j : bit a of j} conj(lambda_t[j]) v_t[j] ) / <v|v>,
// with v_t, lambda_t the states after instruction t. Then both are mapped
// back through M_t^dagger (= M_t^-1 for the unitary steps; E^dagger for an
// expansion), and the frame update of instruction t is undone (every frame
// update of these opcodes is its own inverse). Nothing is stored per
// instruction: the state is uncomputed with inverse gates. Sums are FP64.

#include <cuda_runtime.h>

#include <cstdint>

#include "svm_grad.h"
#include "svm_kernel.cuh"

namespace cgpu {

namespace {

constexpr int kGradThreads = kExpvalGradThreads;

__device__ __forceinline__ double block_sum(double x, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = x;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];  // fixed order
    __syncthreads();
    return t;
}

struct GFrame {
    uint64_t x[4], z[4];
    uint32_t nw;
    __device__ __forceinline__ int gx(uint32_t a) const { return (int)((x[a >> 6] >> (a & 63)) & 1u); }
    __device__ __forceinline__ int gz(uint32_t a) const { return (int)((z[a >> 6] >> (a & 63)) & 1u); }
    __device__ __forceinline__ void fx(uint32_t a, int b) { x[a >> 6] ^= (uint64_t)(b & 1) << (a & 63); }
    __device__ __forceinline__ void fz(uint32_t a, int b) { z[a >> 6] ^= (uint64_t)(b & 1) << (a & 63); }
    __device__ __forceinline__ void px(uint32_t a, int b) {
        const uint64_t m = 1ull << (a & 63);
        x[a >> 6] = b ? (x[a >> 6] | m) : (x[a >> 6] & ~m);
    }
    __device__ __forceinline__ void pz(uint32_t a, int b) {
        const uint64_t m = 1ull << (a & 63);
        z[a >> 6] = b ? (z[a >> 6] | m) : (z[a >> 6] & ~m);
    }
    // frame updates of the frame / array opcodes (svm_kernels.inl:67-116);
    // each is its own inverse on the (x, z) bits
    __device__ __forceinline__ void cnot(uint32_t c, uint32_t t) {
        const int xc = gx(c), zt = gz(t);
        fx(t, xc);
        fz(c, zt);
    }
    __device__ __forceinline__ void cz(uint32_t c, uint32_t t) {
        const int xc = gx(c), xt = gx(t);
        fz(t, xc);
        fz(c, xt);
    }
    __device__ __forceinline__ void h(uint32_t a) {
        const int xa = gx(a), za = gz(a);
        px(a, za);
        pz(a, xa);
    }
    __device__ __forceinline__ void s(uint32_t a) { fz(a, gx(a)); }
    __device__ __forceinline__ void swap(uint32_t a, uint32_t b) {
        const int xa = gx(a), xb = gx(b), za = gz(a), zb = gz(b);
        px(a, xb);
        px(b, xa);
        pz(a, zb);
        pz(b, za);
    }
};

template <typename R>
struct GradTask {
    using T = typename Cx<R>::T;
    const DevProg& P;
    const GradParams& G;
    T* v;
    T* lam;
    double* red;
    uint64_t shot;
    GFrame f;
    uint32_t k;

    __device__ GradTask(const DevProg& p, const GradParams& g, T* vv, T* ll, double* rd, uint64_t s)
        : P(p), G(g), v(vv), lam(ll), red(rd), shot(s), k(0) {
        for (int w = 0; w < 4; ++w) f.x[w] = f.z[w] = 0;
        f.nw = p.nw;
    }

    __device__ __forceinline__ uint4 word0(uint32_t pc) const { return __ldg(P.instr + 2 * pc); }
    // phase (re, im) of a T / ROT / EXPAND_T / EXPAND_ROT instruction
    __device__ __forceinline__ double2 phase_of(uint32_t pc, uint32_t op) const {
        if (op == CLIFFT_OP_ARRAY_T || op == CLIFFT_OP_EXPAND_T) return make_double2(CGPU_INV_SQRT2, CGPU_INV_SQRT2);
        if (op == CLIFFT_OP_ARRAY_T_DAG || op == CLIFFT_OP_EXPAND_T_DAG)
            return make_double2(CGPU_INV_SQRT2, -CGPU_INV_SQRT2);
        const int32_t pi = G.rot_index[pc];
        if (G.phases && pi >= 0) {
            double sn, cs;
            sincos(G.phases[shot * G.n_params + (uint32_t)pi], &sn, &cs);
            return make_double2(cs, sn);
        }
        const uint4 w0 = word0(pc), w1 = __ldg(P.instr + 2 * pc + 1);
        return make_double2(__longlong_as_double(((long long)w0.w << 32) | w0.z),
                            __longlong_as_double(((long long)w1.y << 32) | w1.x));
    }

    // ---- statevector primitives on one vector (CTA-wide, then a barrier)
    __device__ void swap_pairs2(T* x, uint32_t c, uint32_t t) {  // CNOT: swap |c=1,t=0> <-> |c=1,t=1>
        const uint64_t n = 1ull << (k - 2), cb = 1ull << c, tb = 1ull << t;
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t b0 = ins00(i, c, t) | cb;
            const T a = x[b0];
            x[b0] = x[b0 | tb];
            x[b0 | tb] = a;
        }
    }
    __device__ void neg11(T* x, uint32_t c, uint32_t t) {
        const uint64_t n = 1ull << (k - 2), both = (1ull << c) | (1ull << t);
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t j = ins00(i, c, t) | both;
            x[j] = cneg(x[j]);
        }
    }
    __device__ void swap_axes(T* x, uint32_t a, uint32_t b) {
        const uint64_t n = 1ull << (k - 2), ab = 1ull << a, bb = 1ull << b;
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t base = ins00(i, a, b);
            const T t0 = x[base | ab];
            x[base | ab] = x[base | bb];
            x[base | bb] = t0;
        }
    }
    __device__ void multi_cnot(T* x, uint32_t t, uint64_t mask) {
        const uint64_t n = 1ull << (k - 1), tb = 1ull << t;
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t i0 = ins0(i, t);
            if (__popcll(i0 & mask) & 1) {
                const T a = x[i0];
                x[i0] = x[i0 | tb];
                x[i0 | tb] = a;
            }
        }
    }
    __device__ void multi_cz(T* x, uint32_t c, uint64_t mask) {
        const uint64_t n = 1ull << (k - 1), cb = 1ull << c;
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t i0 = ins0(i, c) | cb;
            if (__popcll(i0 & mask) & 1) x[i0] = cneg(x[i0]);
        }
    }
    __device__ void hadamard(T* x, uint32_t a) {
        const uint64_t n = 1ull << (k - 1), ab = 1ull << a;
        const R s = (R)CGPU_INV_SQRT2;
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t i0 = ins0(i, a);
            const T p = x[i0], q = x[i0 | ab];
            x[i0] = cscale(cadd(p, q), s);
            x[i0 | ab] = cscale(csub(p, q), s);
        }
    }
    __device__ void phase_half(T* x, uint32_t a, double2 ph) {
        const uint64_t n = 1ull << (k - 1), ab = 1ull << a;
        const T p = Cx<R>::make(ph.x, ph.y);
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t j = ins0(i, a) | ab;
            x[j] = cmul(x[j], p);
        }
    }
    // k -> k + 1: x_hi = ph * x_lo / sqrt2, x_lo /= sqrt2
    __device__ void expand(T* x, double2 ph) {
        const uint64_t half = 1ull << k;
        const T p = Cx<R>::make(ph.x * CGPU_INV_SQRT2, ph.y * CGPU_INV_SQRT2);
        const R s = (R)CGPU_INV_SQRT2;
        for (uint64_t i = threadIdx.x; i < half; i += blockDim.x) {
            const T a = x[i];
            x[half + i] = cmul(a, p);
            x[i] = cscale(a, s);
        }
    }
    // adjoint of the expansion that made axis k-1: x_lo = (x_lo + conj(ph) x_hi) / sqrt2
    __device__ void unexpand(T* x, double2 ph) {
        const uint64_t half = 1ull << (k - 1);
        const T p = Cx<R>::make(ph.x * CGPU_INV_SQRT2, -ph.y * CGPU_INV_SQRT2);
        const R s = (R)CGPU_INV_SQRT2;
        for (uint64_t i = threadIdx.x; i < half; i += blockDim.x) x[i] = cadd(cscale(x[i], s), cmul(x[half + i], p));
    }
    // -2 s Im(sum over bit a set of conj(lam) v)
    __device__ double rot_term(uint32_t a, int s) {
        const uint64_t n = 1ull << (k - 1), ab = 1ull << a;
        double im = 0.0;
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t j = ins0(i, a) | ab;
            const double lr = (double)lam[j].x, li = (double)lam[j].y, vr = (double)v[j].x, vi = (double)v[j].y;
            im += lr * vi - li * vr;
        }
        return -2.0 * (double)s * block_sum(im, red);
    }

    // ---- one instruction, forward (dir = +1) or undone (dir = -1)
    __device__ void step(uint32_t pc, int dir, double inv_norm, double* grad_row) {
        const uint4 w0 = word0(pc);
        const uint32_t op = w0.x & 0xffu, a1 = w0.y & 0xffffu, a2 = w0.y >> 16;
        const uint64_t mask = ((uint64_t)w0.w << 32) | w0.z;
        const bool both = dir < 0;  // undoing: apply to lambda as well
        switch (op) {
            case CLIFFT_OP_FRAME_CNOT: f.cnot(a1, a2); break;
            case CLIFFT_OP_FRAME_CZ: f.cz(a1, a2); break;
            case CLIFFT_OP_FRAME_H: f.h(a1); break;
            case CLIFFT_OP_FRAME_S:
            case CLIFFT_OP_FRAME_S_DAG: f.s(a1); break;
            case CLIFFT_OP_FRAME_SWAP: f.swap(a1, a2); break;
            case CLIFFT_OP_ARRAY_CNOT:
                swap_pairs2(v, a1, a2);
                if (both) swap_pairs2(lam, a1, a2);
                __syncthreads();
                f.cnot(a1, a2);
                break;
            case CLIFFT_OP_ARRAY_CZ:
                neg11(v, a1, a2);
                if (both) neg11(lam, a1, a2);
                __syncthreads();
                f.cz(a1, a2);
                break;
            case CLIFFT_OP_ARRAY_SWAP:
                swap_axes(v, a1, a2);
                if (both) swap_axes(lam, a1, a2);
                __syncthreads();
                f.swap(a1, a2);
                break;
            case CLIFFT_OP_ARRAY_MULTI_CNOT:
                multi_cnot(v, a1, mask);
                if (both) multi_cnot(lam, a1, mask);
                __syncthreads();
                for (uint32_t c = 0; c < k; ++c)
                    if ((mask >> c) & 1ull) f.cnot(c, a1);
                break;
            case CLIFFT_OP_ARRAY_MULTI_CZ:
                multi_cz(v, a1, mask);
                if (both) multi_cz(lam, a1, mask);
                __syncthreads();
                for (uint32_t t = 0; t < k; ++t)
                    if ((mask >> t) & 1ull) f.cz(a1, t);
                break;
            case CLIFFT_OP_ARRAY_H:
                hadamard(v, a1);
                if (both) hadamard(lam, a1);
                __syncthreads();
                f.h(a1);
                break;
            case CLIFFT_OP_ARRAY_S:
            case CLIFFT_OP_ARRAY_S_DAG: {
                const double im = (op == CLIFFT_OP_ARRAY_S ? 1.0 : -1.0) * (double)dir;
                phase_half(v, a1, make_double2(0.0, im));
                if (both) phase_half(lam, a1, make_double2(0.0, im));
                __syncthreads();
                f.s(a1);
                break;
            }
            case CLIFFT_OP_ARRAY_T:
            case CLIFFT_OP_ARRAY_T_DAG:
            case CLIFFT_OP_ARRAY_ROT: {
                if (a1 >= k) break;  // dormant axis: a global phase only
                const int s = f.gx(a1) ? -1 : 1;
                double2 ph = phase_of(pc, op);
                ph.y *= (double)s;
                if (both) {
                    const int32_t pi = G.rot_index[pc];
                    if (op == CLIFFT_OP_ARRAY_ROT && pi >= 0) {
                        const double g = rot_term(a1, s) * inv_norm;
                        if (threadIdx.x == 0) grad_row[pi] += g;
                    }
                    ph.y = -ph.y;
                }
                phase_half(v, a1, ph);
                if (both) phase_half(lam, a1, ph);
                __syncthreads();
                break;
            }
            case CLIFFT_OP_EXPAND:
            case CLIFFT_OP_EXPAND_T:
            case CLIFFT_OP_EXPAND_T_DAG:
            case CLIFFT_OP_EXPAND_ROT: {
                double2 ph = make_double2(1.0, 0.0);
                if (op != CLIFFT_OP_EXPAND) {
                    ph = phase_of(pc, op);
                    if (f.gx(a1)) ph.y = -ph.y;
                }
                if (!both) {
                    expand(v, ph);
                    __syncthreads();
                    ++k;
                } else {
                    const int32_t pi = G.rot_index[pc];
                    if (op == CLIFFT_OP_EXPAND_ROT && pi >= 0) {
                        const double g = rot_term(k - 1, f.gx(a1) ? -1 : 1) * inv_norm;
                        if (threadIdx.x == 0) grad_row[pi] += g;
                    }
                    unexpand(v, ph);
                    unexpand(lam, ph);
                    __syncthreads();
                    --k;
                }
                break;
            }
            default: break;  // EXP_VAL of another observable: no state change
        }
    }

    // lambda = O_e v for the EXP_VAL at `pc`; returns <v|O_e|v> / <v|v> and
    // sets inv_norm, or returns 0 with dormant = true when the mask has X / Y
    // support on a dormant axis (the value and every derivative are 0).
    __device__ double apply_observable(uint32_t pc, double& inv_norm, bool& dormant) {
        const uint4 w0 = word0(pc);
        const uint32_t cp = w0.z;
        const uint32_t nw = P.nw;
        const uint64_t* mx = P.exp_x + (size_t)cp * nw;
        const uint64_t* mz = P.exp_z + (size_t)cp * nw;
        int fsign = P.exp_sign[cp] != 0;
        int par = 0;
        for (uint32_t w = 0; w < nw; ++w) par += __popcll(mx[w] & f.z[w]) + __popcll(mz[w] & f.x[w]);
        if (par & 1) fsign ^= 1;
        dormant = false;
        for (uint32_t w = 0; w < nw; ++w) {
            uint64_t m = mx[w];
            const uint32_t lo = w * 64;
            if (k >= lo + 64) continue;
            if (k > lo) m &= ~((1ull << (k - lo)) - 1);
            if (m) dormant = true;
        }
        if (dormant) return 0.0;
        const uint64_t am = k >= 64 ? ~0ull : ((1ull << k) - 1);
        const uint64_t xa = mx[0] & am, za = mz[0] & am;
        const int yz = __popcll(xa & za) & 3;
        double2 iph = make_double2(yz == 0 ? 1.0 : (yz == 2 ? -1.0 : 0.0), yz == 1 ? 1.0 : (yz == 3 ? -1.0 : 0.0));
        if (fsign) iph = make_double2(-iph.x, -iph.y);
        const T ip = Cx<R>::make(iph.x, iph.y);
        const uint64_t dim = 1ull << k;
        double nrm = 0.0, num = 0.0;
        for (uint64_t j = threadIdx.x; j < dim; j += blockDim.x) {
            T y = cmul(v[j], ip);
            if (__popcll(j & za) & 1) y = cneg(y);
            lam[j ^ xa] = y;
            const double vr = (double)v[j].x, vi = (double)v[j].y;
            nrm += vr * vr + vi * vi;
            // Re(conj(v[j ^ xa]) * y) accumulated at the partner index
            const double br = (double)v[j ^ xa].x, bi = (double)v[j ^ xa].y;
            num += br * (double)y.x + bi * (double)y.y;
        }
        __syncthreads();
        nrm = block_sum(nrm, red);
        num = block_sum(num, red);
        inv_norm = nrm > 0.0 ? 1.0 / nrm : 0.0;
        return num * inv_norm;
    }
};

template <typename R>
__global__ void __launch_bounds__(kGradThreads) expval_grad_kernel(const DevProg P, const GradParams G) {
    using T = typename Cx<R>::T;
    __shared__ double red[32];
    __shared__ unsigned long long task_s;
    T* v = reinterpret_cast<T*>(G.slab) + (size_t)blockIdx.x * 2 * G.stride;
    T* lam = v + G.stride;
    const uint64_t tasks = G.batch * G.n_exp;
    for (;;) {
        if (threadIdx.x == 0) task_s = atomicAdd(G.work, 1ull);
        __syncthreads();
        const unsigned long long task = task_s;
        __syncthreads();
        if (task >= tasks) break;
        const uint64_t shot = task / G.n_exp;
        const uint32_t e = (uint32_t)(task % G.n_exp);
        GradTask<R> t(P, G, v, lam, red, shot);
        if (threadIdx.x == 0) v[0] = Cx<R>::make(1.0, 0.0);
        __syncthreads();
        const uint32_t te = G.exp_pc[e];
        for (uint32_t pc = 0; pc < te; ++pc) t.step(pc, +1, 0.0, nullptr);
        double inv_norm = 0.0;
        bool dormant = false;
        const double val = t.apply_observable(te, inv_norm, dormant);
        const uint32_t row = G.exp_out[e];
        double* grad_row = G.out_grad + (shot * G.n_out + row) * (size_t)G.n_params;
        if (threadIdx.x == 0) G.out_exp[shot * G.n_out + row] = fmin(1.0, fmax(-1.0, val));
        for (uint32_t i = threadIdx.x; i < G.n_params; i += blockDim.x) grad_row[i] = 0.0;
        __syncthreads();
        if (!dormant)
            for (uint32_t pc = te; pc-- > 0;) t.step(pc, -1, inv_norm, grad_row);
        __syncthreads();
    }
}

}  // namespace

ExpvalGradFn expval_grad_kernel_fn(bool fp32) {
    return fp32 ? expval_grad_kernel<float> : expval_grad_kernel<double>;
}

}  // namespace cgpu
