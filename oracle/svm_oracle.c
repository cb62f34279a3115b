/*
 * svm_oracle.c -- CPU restatement of the reference Schrodinger-VM executor.
 *
 * TEST INFRASTRUCTURE ONLY (see svm_oracle.h). Each function names the
 * reference code it restates. Arithmetic follows the reference's portable
 * scalar path in double precision, including its two distinct 1/sqrt(2)
 * constants: kInvSqrt2 = sqrt(2)/2 for butterflies and phases
 * (src/clifft/util/constants.h) and 1.0/std::sqrt(2.0) for EXPAND's gamma
 * scale (src/clifft/svm/svm_kernels.inl:895).
 */
#include "svm_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static __thread char g_err[256];

const char* oracle_last_error(void) { return g_err; }

#define FAIL(...)                                         \
    do {                                                  \
        snprintf(g_err, sizeof g_err, __VA_ARGS__);       \
        return -1;                                        \
    } while (0)

typedef struct {
    double re, im;
} cplx;

static const double kInvSqrt2 = 1.4142135623730951 / 2.0; /* std::numbers::sqrt2 / 2 */

static inline cplx cmul(cplx a, cplx b) {
    cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static inline cplx cadd(cplx a, cplx b) {
    cplx r = {a.re + b.re, a.im + b.im};
    return r;
}
static inline cplx csub(cplx a, cplx b) {
    cplx r = {a.re - b.re, a.im - b.im};
    return r;
}
static inline cplx cscale(cplx a, double s) {
    cplx r = {a.re * s, a.im * s};
    return r;
}
static inline double cnorm(cplx a) { return a.re * a.re + a.im * a.im; }

/* ------------------------------------------------------------------ RNGs */

/* xoshiro256++ with SplitMix64 seeding (src/clifft/svm/svm.h:40-90). */
static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t splitmix64(uint64_t* s) {
    uint64_t z = (*s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static void xo_seed(uint64_t st[4], uint64_t seed) {
    uint64_t z = seed;
    for (int i = 0; i < 4; ++i) st[i] = splitmix64(&z);
}
static uint64_t xo_next(uint64_t s[4]) {
    const uint64_t result = rotl64(s[0] + s[3], 23) + s[0];
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return result;
}

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with a
 * Weyl-sequence key schedule. */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0;
        c1 = n1;
        c2 = n2;
        c3 = n3;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

/* ----------------------------------------------------------------- state */

typedef struct {
    const clifft_program_image* img;
    uint32_t nw;
    uint32_t k;
    cplx* v;
    uint64_t* px;
    uint64_t* pz;
    cplx gamma;
    uint8_t* meas;
    uint8_t* det;
    uint8_t* obs;
    double* exp;
    uint32_t next_noise;
    int discarded;
    /* forced mode */
    const uint8_t* forced;
    double log_prob;
    int reachable;
    int faults_active;
    const uint32_t* ff_sites;
    const uint32_t* ff_chan;
    uint32_t ff_n, ff_pos;
    const uint32_t* ro_idx;
    uint32_t ro_n, ro_pos;
    double* meas_prob;
    /* rng */
    int rng_kind;
    uint64_t xo[4];
    uint32_t key[2];
    uint64_t shot;
    uint64_t draw;
    uint64_t dust_clamps;
    double dust_eps;
} ostate;

/* random_double (src/clifft/svm/svm.h:150): 53 high bits times 2^-53. */
static double random_double(ostate* s) {
    uint64_t r;
    if (s->rng_kind == ORACLE_RNG_XOSHIRO) {
        r = xo_next(s->xo);
    } else {
        uint32_t ctr[4] = {(uint32_t)(s->draw >> 1), 0u, (uint32_t)s->shot,
                           (uint32_t)(s->shot >> 32)};
        uint32_t out[4];
        oracle_philox4x32_10(ctr, s->key, out);
        r = (s->draw & 1) ? ((uint64_t)out[3] << 32 | out[2]) : ((uint64_t)out[1] << 32 | out[0]);
        s->draw++;
    }
    return (double)(r >> 11) * 0x1.0p-53;
}

static inline int bget(const uint64_t* m, uint32_t i) { return (int)((m[i >> 6] >> (i & 63)) & 1u); }
static inline void bset(uint64_t* m, uint32_t i, int v) {
    uint64_t b = 1ULL << (i & 63);
    if (v)
        m[i >> 6] |= b;
    else
        m[i >> 6] &= ~b;
}
static inline void bxor(uint64_t* m, uint32_t i, int v) {
    if (v) m[i >> 6] ^= 1ULL << (i & 63);
}

static void multiply_phase(ostate* s, cplx p) { s->gamma = cmul(s->gamma, p); }
static const cplx kMinus1 = {-1.0, 0.0};

/* SchrodingerState::scale_magnitude (src/clifft/svm/svm.h:177-186). */
static void scale_magnitude(ostate* s, double scale) {
    s->gamma = cscale(s->gamma, scale);
    double g = hypot(s->gamma.re, s->gamma.im);
    if (g > 1e100 || (g < 1e-100 && g > 0.0)) {
        uint64_t sz = 1ULL << s->k;
        for (uint64_t i = 0; i < sz; ++i) s->v[i] = cscale(s->v[i], g);
        s->gamma.re /= g;
        s->gamma.im /= g;
    }
}

static inline uint64_t insert_zero_bit(uint64_t val, uint32_t pos) {
    uint64_t mask = (1ULL << pos) - 1;
    return (val & mask) | ((val & ~mask) << 1);
}
static inline uint64_t insert_zero_bits2(uint64_t val, uint32_t a, uint32_t b) {
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return insert_zero_bit(insert_zero_bit(val, lo), hi);
}

/* ------------------------------------------------------- frame opcodes */
/* src/clifft/svm/svm_kernels.inl:67-116,749-755 */
static void frame_cnot(ostate* s, uint32_t c, uint32_t t) {
    int pxc = bget(s->px, c), pzt = bget(s->pz, t);
    bxor(s->px, t, pxc);
    bxor(s->pz, c, pzt);
}
static void frame_cz(ostate* s, uint32_t c, uint32_t t) {
    int pxc = bget(s->px, c), pxt = bget(s->px, t);
    if (pxc && pxt) multiply_phase(s, kMinus1);
    bxor(s->pz, t, pxc);
    bxor(s->pz, c, pxt);
}
static void frame_h(ostate* s, uint32_t v) {
    int px = bget(s->px, v), pz = bget(s->pz, v);
    if (px && pz) multiply_phase(s, kMinus1);
    bset(s->px, v, pz);
    bset(s->pz, v, px);
}
static void frame_s(ostate* s, uint32_t v, int dag) {
    int px = bget(s->px, v);
    if (px) {
        cplx ph = {0.0, dag ? -1.0 : 1.0};
        multiply_phase(s, ph);
    }
    bxor(s->pz, v, px);
}
static void frame_swap(ostate* s, uint32_t a, uint32_t b) {
    int xa = bget(s->px, a), xb = bget(s->px, b);
    if (xa != xb) {
        bxor(s->px, a, 1);
        bxor(s->px, b, 1);
    }
    int za = bget(s->pz, a), zb = bget(s->pz, b);
    if (za != zb) {
        bxor(s->pz, a, 1);
        bxor(s->pz, b, 1);
    }
}

/* ------------------------------------------------------- array opcodes */
/* exec_array_cnot scalar path (svm_kernels.inl:238-251) */
static void array_cnot(ostate* s, uint32_t c, uint32_t t) {
    uint64_t iters = 1ULL << (s->k - 2), cb = 1ULL << c, tb = 1ULL << t;
    for (uint64_t i = 0; i < iters; ++i) {
        uint64_t b0 = insert_zero_bits2(i, c, t) | cb;
        cplx tmp = s->v[b0];
        s->v[b0] = s->v[b0 | tb];
        s->v[b0 | tb] = tmp;
    }
    frame_cnot(s, c, t);
}
/* exec_array_cz scalar path (svm_kernels.inl:343-364) */
static void array_cz(ostate* s, uint32_t c, uint32_t t) {
    uint64_t iters = 1ULL << (s->k - 2), both = (1ULL << c) | (1ULL << t);
    for (uint64_t i = 0; i < iters; ++i) {
        uint64_t idx = insert_zero_bits2(i, c, t) | both;
        s->v[idx].re = -s->v[idx].re;
        s->v[idx].im = -s->v[idx].im;
    }
    frame_cz(s, c, t);
}
/* exec_array_swap scalar path (svm_kernels.inl:444-457) */
static void array_swap(ostate* s, uint32_t a, uint32_t b) {
    uint64_t iters = 1ULL << (s->k - 2), ab = 1ULL << a, bb = 1ULL << b;
    for (uint64_t i = 0; i < iters; ++i) {
        uint64_t base = insert_zero_bits2(i, a, b);
        cplx tmp = s->v[base | ab];
        s->v[base | ab] = s->v[base | bb];
        s->v[base | bb] = tmp;
    }
    frame_swap(s, a, b);
}
/* exec_array_multi_cnot (svm_kernels.inl:464-550): flip target where the
 * parity of the control bits is odd; frame CNOT per control. */
static void array_multi_cnot(ostate* s, uint32_t target, uint64_t mask) {
    uint64_t tb = 1ULL << target, half = 1ULL << (s->k - 1);
    for (uint64_t i = 0; i < half; ++i) {
        uint64_t a = insert_zero_bit(i, target);
        if (__builtin_popcountll(a & mask) & 1) {
            cplx tmp = s->v[a];
            s->v[a] = s->v[a | tb];
            s->v[a | tb] = tmp;
        }
    }
    for (uint32_t c = 0; c < s->k; ++c)
        if (mask & (1ULL << c)) frame_cnot(s, c, target);
}
/* exec_array_multi_cz (svm_kernels.inl:558-635) */
static void array_multi_cz(ostate* s, uint32_t control, uint64_t mask) {
    uint64_t cb = 1ULL << control, half = 1ULL << (s->k - 1);
    for (uint64_t i = 0; i < half; ++i) {
        uint64_t a = insert_zero_bit(i, control) | cb;
        if (__builtin_popcountll(a & mask) & 1) {
            s->v[a].re = -s->v[a].re;
            s->v[a].im = -s->v[a].im;
        }
    }
    for (uint32_t t = 0; t < s->k; ++t)
        if (mask & (1ULL << t)) frame_cz(s, control, t);
}
/* exec_array_h scalar path (svm_kernels.inl:730-744) */
static void array_h(ostate* s, uint32_t v) {
    uint64_t iters = 1ULL << (s->k - 1), vb = 1ULL << v;
    for (uint64_t i = 0; i < iters; ++i) {
        uint64_t i0 = insert_zero_bit(i, v), i1 = i0 | vb;
        cplx a = s->v[i0], b = s->v[i1];
        s->v[i0] = cscale(cadd(a, b), kInvSqrt2);
        s->v[i1] = cscale(csub(a, b), kInvSqrt2);
    }
    frame_h(s, v);
}
/* apply_phase_waterfall scalar path (svm_kernels.inl:822-829) */
static void phase_waterfall(ostate* s, uint32_t v, double re, double im) {
    uint64_t iters = 1ULL << (s->k - 1), vb = 1ULL << v;
    cplx ph = {re, im};
    for (uint64_t i = 0; i < iters; ++i) {
        uint64_t idx = insert_zero_bit(i, v) | vb;
        s->v[idx] = cmul(s->v[idx], ph);
    }
}
/* exec_array_s / s_dag (svm_kernels.inl:833-846) */
static void array_s(ostate* s, uint32_t v, int dag) {
    phase_waterfall(s, v, 0.0, dag ? -1.0 : 1.0);
    frame_s(s, v, dag);
}
/* exec_array_t / t_dag / rot (svm_kernels.inl:951-988,1044-1061): dormant axis
 * contributes a gamma phase only; an X frame bit conjugates the array phase
 * and gamma absorbs the original one. */
static void array_rot(ostate* s, uint32_t v, double zre, double zim) {
    int px = bget(s->px, v);
    cplx z = {zre, zim};
    if (v >= s->k) {
        if (px) multiply_phase(s, z);
        return;
    }
    if (px) {
        phase_waterfall(s, v, zre, -zim);
        multiply_phase(s, z);
    } else {
        phase_waterfall(s, v, zre, zim);
    }
}
/* exec_expand / expand_with_phase / exec_expand_{t,t_dag,rot}
 * (svm_kernels.inl:876-1081). */
static void expand_phase(ostate* s, uint32_t v, double zre, double zim, int with_phase) {
    uint64_t half = 1ULL << s->k;
    int px = with_phase ? bget(s->px, v) : 0;
    (void)v;
    if (!with_phase) {
        memcpy(s->v + half, s->v, half * sizeof(cplx));
    } else {
        cplx ph = {zre, px ? -zim : zim};
        for (uint64_t i = 0; i < half; ++i) s->v[half + i] = cmul(s->v[i], ph);
    }
    s->k++;
    scale_magnitude(s, 1.0 / sqrt(2.0));
    if (with_phase && px) {
        cplx z = {zre, zim};
        multiply_phase(s, z);
    }
}
/* exec_array_u2 scalar path (svm_kernels.inl:1087-1297) */
static void array_u2(ostate* s, uint32_t axis, uint32_t cp) {
    const double* node = s->img->u2_data + (size_t)cp * CLIFFT_U2_DOUBLES_PER_NODE;
    int st = (bget(s->pz, axis) ? 2 : 0) | (bget(s->px, axis) ? 1 : 0);
    const double* m = node + st * 10;
    cplx g = {m[8], m[9]};
    multiply_phase(s, g);
    uint8_t out = s->img->u2_out[cp * 4 + st];
    bset(s->px, axis, out & 1);
    bset(s->pz, axis, (out >> 1) & 1);
    if (axis >= s->k) return;
    cplx m00 = {m[0], m[1]}, m01 = {m[2], m[3]}, m10 = {m[4], m[5]}, m11 = {m[6], m[7]};
    uint64_t iters = 1ULL << (s->k - 1), vb = 1ULL << axis;
    for (uint64_t i = 0; i < iters; ++i) {
        uint64_t i0 = insert_zero_bit(i, axis), i1 = i0 | vb;
        cplx a = s->v[i0], b = s->v[i1];
        s->v[i0] = cadd(cmul(m00, a), cmul(m01, b));
        s->v[i1] = cadd(cmul(m10, a), cmul(m11, b));
    }
}
/* exec_array_u4 scalar path (svm_kernels.inl:1310-1531) */
static void array_u4(ostate* s, uint32_t lo, uint32_t hi, uint32_t cp) {
    const double* node = s->img->u4_data + (size_t)cp * CLIFFT_U4_DOUBLES_PER_NODE;
    int st = (bget(s->pz, hi) << 3) | (bget(s->px, hi) << 2) | (bget(s->pz, lo) << 1) |
             bget(s->px, lo);
    const double* e = node + st * 34;
    cplx g = {e[32], e[33]};
    multiply_phase(s, g);
    uint8_t out = s->img->u4_out[cp * 16 + st];
    bset(s->px, lo, out & 1);
    bset(s->pz, lo, (out >> 1) & 1);
    bset(s->px, hi, (out >> 2) & 1);
    bset(s->pz, hi, (out >> 3) & 1);
    cplx m[4][4];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            m[r][c].re = e[(r * 4 + c) * 2];
            m[r][c].im = e[(r * 4 + c) * 2 + 1];
        }
    uint64_t lb = 1ULL << lo, hb = 1ULL << hi, iters = 1ULL << (s->k - 2);
    for (uint64_t i = 0; i < iters; ++i) {
        uint64_t b = insert_zero_bits2(i, lo, hi);
        uint64_t ix[4] = {b, b | lb, b | hb, b | lb | hb};
        cplx x[4];
        for (int j = 0; j < 4; ++j) x[j] = s->v[ix[j]];
        for (int r = 0; r < 4; ++r) {
            cplx acc = cmul(m[r][0], x[0]);
            acc = cadd(acc, cmul(m[r][1], x[1]));
            acc = cadd(acc, cmul(m[r][2], x[2]));
            acc = cadd(acc, cmul(m[r][3], x[3]));
            s->v[ix[r]] = acc;
        }
    }
}

/* ------------------------------------------------------- measurements */

/* sample_branch (src/clifft/svm/svm_internal.h:65-79) */
static int sample_branch(ostate* s, double p0, double p1, double total, double* prob_out) {
    double eps = s->dust_eps * total;
    if (p1 <= eps) {
        if (p1 > 0.0) s->dust_clamps++;
        *prob_out = 1.0;
        return 0;
    }
    if (p0 <= eps) {
        if (p0 > 0.0) s->dust_clamps++;
        *prob_out = 1.0;
        return 1;
    }
    double r = random_double(s);
    int b = (r * total < p0) ? 0 : 1;
    *prob_out = (b ? p1 : p0) / total;
    return b;
}

/* forced_log_increment (src/clifft/svm/svm_forced_kernels.cc:42-60). Returns
 * reachability; *inc is the log increment. */
static int forced_branch(ostate* s, double p0, double p1, double total, int b, double* inc) {
    double eps = s->dust_eps * total;
    *inc = 0.0;
    if (p1 <= eps) {
        if (p1 > 0.0) s->dust_clamps++;
        return b == 0;
    }
    if (p0 <= eps) {
        if (p0 > 0.0) s->dust_clamps++;
        return b == 1;
    }
    *inc = log((b ? p1 : p0) / total);
    return 1;
}

static void record_prob(ostate* s, uint32_t idx, double p) {
    if (s->meas_prob) s->meas_prob[idx] = p;
}

/* Returns 0 to continue, 1 to stop the shot (unreachable forced outcome). */
static int meas_dormant_static(ostate* s, uint32_t v, uint32_t idx, int sign, int identity) {
    uint8_t det = identity ? (uint8_t)(sign ? 1 : 0) : (uint8_t)(bget(s->px, v) ^ sign);
    if (s->forced) {
        /* svm_forced_kernels.cc:64-88 */
        if (s->forced[idx] != det) {
            s->reachable = 0;
            return 1;
        }
    }
    s->meas[idx] = det;
    record_prob(s, idx, 1.0);
    return 0;
}

static int meas_dormant_random(ostate* s, uint32_t v, uint32_t idx, int sign) {
    int m_abs;
    if (s->forced) {
        /* svm_forced_kernels.cc:90-110 */
        m_abs = s->forced[idx] ^ sign;
        s->log_prob += log(0.5);
    } else {
        /* svm_kernels.inl:1550-1566 */
        m_abs = random_double(s) < 0.5 ? 0 : 1;
    }
    if (bget(s->px, v) && m_abs) multiply_phase(s, kMinus1);
    bset(s->px, v, m_abs);
    bset(s->pz, v, 0);
    s->meas[idx] = (uint8_t)(m_abs ^ sign);
    record_prob(s, idx, 0.5);
    return 0;
}

/* exec_meas_active_diagonal (svm_kernels.inl:1573-1627) and its forced
 * variant (svm_forced_kernels.cc:112-158). */
static int meas_active_diagonal(ostate* s, uint32_t v, uint32_t idx, int sign) {
    uint64_t half = 1ULL << (s->k - 1);
    int pxv = bget(s->px, v), pzv = bget(s->pz, v);
    double p0 = 0.0, p1 = 0.0;
    for (uint64_t i = 0; i < half; ++i) {
        p0 += cnorm(s->v[i]);
        p1 += cnorm(s->v[i + half]);
    }
    double total = p0 + p1;
    int b;
    double prob;
    if (s->forced) {
        int m_abs = s->forced[idx] ^ sign;
        b = m_abs ^ pxv;
        double inc;
        if (!forced_branch(s, p0, p1, total, b, &inc)) {
            s->reachable = 0;
            return 1;
        }
        s->log_prob += inc;
        prob = exp(inc);
    } else {
        b = sample_branch(s, p0, p1, total, &prob);
    }
    int m_abs = b ^ pxv;
    if (b == 1 && pzv) multiply_phase(s, kMinus1);
    if (b == 1) memmove(s->v, s->v + half, half * sizeof(cplx));
    s->k--;
    double pb = b ? p1 : p0;
    if (s->forced || pb > 0.0) scale_magnitude(s, sqrt(total / pb));
    bset(s->px, v, m_abs);
    bset(s->pz, v, 0);
    s->meas[idx] = (uint8_t)(m_abs ^ sign);
    record_prob(s, idx, prob);
    return 0;
}

/* exec_meas_active_interfere (svm_kernels.inl:1634-1708), exec_swap_meas_interfere
 * (svm_kernels.inl:1728-1804) and their forced variants
 * (svm_forced_kernels.cc:160-304). `f` == `t` means no fused swap. */
static int meas_interfere(ostate* s, uint32_t f, uint32_t t, uint32_t idx, int sign) {
    int swapped = (f != t);
    if (swapped) frame_swap(s, f, t);
    int pxv = bget(s->px, t), pzv = bget(s->pz, t);
    uint64_t half = 1ULL << t, fb = 1ULL << f;
    double pp = 0.0, pm = 0.0;
    for (uint64_t i = 0; i < half; ++i) {
        uint64_t a, c;
        if (swapped) {
            uint64_t bf = (i >> f) & 1;
            a = (i & ~fb) | (bf << t);
            c = a | fb;
        } else {
            a = i;
            c = i + half;
        }
        pp += cnorm(cadd(s->v[a], s->v[c]));
        pm += cnorm(csub(s->v[a], s->v[c]));
    }
    double total = pp + pm;
    int bx;
    double prob;
    if (s->forced) {
        int m_abs = s->forced[idx] ^ sign;
        bx = m_abs ^ pzv;
        double inc;
        if (!forced_branch(s, pp, pm, total, bx, &inc)) {
            s->reachable = 0;
            return 1;
        }
        s->log_prob += inc;
        prob = exp(inc);
    } else {
        bx = sample_branch(s, pp, pm, total, &prob);
    }
    int m_abs = bx ^ pzv;
    for (uint64_t i = 0; i < half; ++i) {
        uint64_t a, c;
        if (swapped) {
            uint64_t bf = (i >> f) & 1;
            a = (i & ~fb) | (bf << t);
            c = a | fb;
        } else {
            a = i;
            c = i + half;
        }
        s->v[i] = cscale(bx ? csub(s->v[a], s->v[c]) : cadd(s->v[a], s->v[c]), kInvSqrt2);
    }
    double pb = bx ? pm : pp;
    if (!swapped) {
        if (pxv && m_abs) multiply_phase(s, kMinus1);
        s->k--;
        if (s->forced || pb > 0.0) scale_magnitude(s, sqrt(total / pb));
    } else {
        s->k--;
        if (s->forced || pb > 0.0) scale_magnitude(s, sqrt(total / pb));
        if (pxv && m_abs) multiply_phase(s, kMinus1);
    }
    bset(s->px, t, m_abs);
    bset(s->pz, t, 0);
    s->meas[idx] = (uint8_t)(m_abs ^ sign);
    record_prob(s, idx, prob);
    return 0;
}

/* ------------------------------------------------- classical / noise */

/* apply_pauli_to_frame (svm_kernels.inl:1812-1865) */
static void apply_pauli(ostate* s, const uint64_t* ex, const uint64_t* ez, int sign) {
    int parity = 0;
    for (uint32_t w = 0; w < s->nw; ++w) parity += __builtin_popcountll(s->px[w] & ez[w]);
    if (parity & 1) multiply_phase(s, kMinus1);
    for (uint32_t w = 0; w < s->nw; ++w) {
        s->px[w] ^= ex[w];
        s->pz[w] ^= ez[w];
    }
    if (sign) multiply_phase(s, kMinus1);
}

/* SchrodingerState::draw_next_noise (src/clifft/svm/svm.h:231-248) */
static void draw_next_noise(ostate* s) {
    uint32_t n = s->img->num_noise_sites;
    const double* hz = s->img->noise_hazards;
    if (n == 0 || s->next_noise >= n) {
        s->next_noise = UINT32_MAX;
        return;
    }
    double cur = s->next_noise == 0 ? 0.0 : hz[s->next_noise - 1];
    double gap = -log(1.0 - random_double(s));
    double target = cur + gap;
    uint32_t lo = 0, hi = n; /* upper_bound: first hz[i] > target */
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2;
        if (hz[mid] > target)
            hi = mid;
        else
            lo = mid + 1;
    }
    s->next_noise = lo;
}

/* exec_noise (svm_kernels.inl:1886-1921) */
static void noise_site(ostate* s, uint32_t site) {
    if (site != s->next_noise) return;
    const clifft_program_image* im = s->img;
    uint32_t c0 = im->noise_site_offsets[site], c1 = im->noise_site_offsets[site + 1];
    if (s->faults_active) {
        uint32_t c = c0 + s->ff_chan[s->ff_pos - 1];
        if (c < c1)
            apply_pauli(s, im->noise_channel_x + (size_t)c * s->nw,
                        im->noise_channel_z + (size_t)c * s->nw, 0);
        s->next_noise = s->ff_pos < s->ff_n ? s->ff_sites[s->ff_pos++] : UINT32_MAX;
        return;
    }
    double psum = 0.0;
    for (uint32_t c = c0; c < c1; ++c) psum += im->noise_channel_prob[c];
    double r = random_double(s) * psum, cum = 0.0;
    for (uint32_t c = c0; c < c1; ++c) {
        cum += im->noise_channel_prob[c];
        if (r < cum) {
            apply_pauli(s, im->noise_channel_x + (size_t)c * s->nw,
                        im->noise_channel_z + (size_t)c * s->nw, 0);
            break;
        }
    }
    s->next_noise++;
    draw_next_noise(s);
}

/* exec_readout_noise (svm_kernels.inl:1937-1959) */
static void readout_noise(ostate* s, uint32_t e) {
    int fire = 0;
    if (s->faults_active) {
        if (s->ro_pos < s->ro_n && s->ro_idx[s->ro_pos] == e) {
            fire = 1;
            s->ro_pos++;
        }
    } else {
        fire = random_double(s) < s->img->readout_prob[e];
    }
    if (fire) s->meas[s->img->readout_meas_idx[e]] ^= 1;
}

static uint8_t list_parity(const uint8_t* meas, const uint32_t* off, const uint32_t* tg, uint32_t l) {
    uint8_t p = 0;
    for (uint32_t i = off[l]; i < off[l + 1]; ++i) p ^= meas[tg[i]];
    return p;
}

/* exec_exp_val (svm_kernels.inl:2031-2173) */
static void exp_val(ostate* s, uint32_t cp, uint32_t out_idx) {
    const clifft_program_image* im = s->img;
    const uint64_t* mx = im->exp_val_x + (size_t)cp * s->nw;
    const uint64_t* mz = im->exp_val_z + (size_t)cp * s->nw;
    int fsign = im->exp_val_sign[cp] != 0;
    int parity = 0;
    for (uint32_t w = 0; w < s->nw; ++w) {
        parity += __builtin_popcountll(mx[w] & s->pz[w]);
        parity += __builtin_popcountll(mz[w] & s->px[w]);
    }
    if (parity & 1) fsign = !fsign;
    uint32_t k = s->k;
    uint32_t full = k / 64, rem = k % 64;
    int dormant_x = 0;
    if (rem > 0 && full < s->nw && (mx[full] & ~((1ULL << rem) - 1))) dormant_x = 1;
    for (uint32_t w = (rem == 0 ? full : full + 1); w < s->nw && !dormant_x; ++w)
        if (mx[w]) dormant_x = 1;
    if (dormant_x) {
        s->exp[out_idx] = 0.0;
        return;
    }
    uint64_t xa = 0, za = 0;
    if (k > 0) {
        uint64_t am = (k == 64) ? ~0ULL : ((1ULL << k) - 1);
        xa = mx[0] & am;
        za = mz[0] & am;
    }
    int yz = __builtin_popcountll(xa & za) & 3;
    cplx iph = {yz == 0 ? 1.0 : (yz == 2 ? -1.0 : 0.0), yz == 1 ? 1.0 : (yz == 3 ? -1.0 : 0.0)};
    if (fsign) {
        iph.re = -iph.re;
        iph.im = -iph.im;
    }
    uint64_t dim = 1ULL << k;
    double nre = 0.0, nim = 0.0, den = 0.0;
    for (uint64_t j = 0; j < dim; ++j) {
        cplx a = s->v[j];
        den += cnorm(a);
        cplx b = s->v[j ^ xa];
        double zs = (__builtin_popcountll(j & za) & 1) ? -1.0 : 1.0;
        cplx sa = {zs * a.re, zs * a.im};
        cplx cb = {b.re, -b.im};
        cplx t = cmul(cb, sa);
        nre += t.re;
        nim += t.im;
    }
    cplx num = {nre, nim};
    num = cmul(num, iph);
    double r = 0.0;
    if (den > 0.0) r = num.re / den;
    if (r > 1.0) r = 1.0;
    if (r < -1.0) r = -1.0;
    s->exp[out_idx] = r;
}

/* ----------------------------------------------------------- dispatch */

static inline uint32_t rd_u32(const uint8_t* p) {
    uint32_t v;
    memcpy(&v, p, 4);
    return v;
}
static inline uint16_t rd_u16(const uint8_t* p) {
    uint16_t v;
    memcpy(&v, p, 2);
    return v;
}
static inline uint64_t rd_u64(const uint8_t* p) {
    uint64_t v;
    memcpy(&v, p, 8);
    return v;
}
static inline double rd_f64(const uint8_t* p) {
    double v;
    memcpy(&v, p, 8);
    return v;
}

/* execute_internal (svm_kernels.inl:2183-2646). Forced opcodes behave like
 * their sampling counterparts with s->forced set. */
static int execute(ostate* s) {
    const clifft_program_image* im = s->img;
    for (uint32_t pc = 0; pc < im->num_instructions; ++pc) {
        const uint8_t* I = im->instructions + (size_t)pc * 32;
        uint8_t op = I[0], fl = I[2];
        uint32_t a1 = rd_u16(I + 4), a2 = rd_u16(I + 6);
        uint32_t p0 = rd_u32(I + 8), p1 = rd_u32(I + 12);
        int sign = (fl & CLIFFT_FLAG_SIGN) != 0;
        if (op >= CLIFFT_OP_MEAS_DORMANT_STATIC_FORCED && op <= CLIFFT_OP_SWAP_MEAS_INTERFERE_FORCED) {
            if (!s->forced) FAIL("forced measurement opcode without a forced record");
            op = (uint8_t)(op - (CLIFFT_OP_MEAS_DORMANT_STATIC_FORCED - CLIFFT_OP_MEAS_DORMANT_STATIC));
        }
        switch (op) {
            case CLIFFT_OP_FRAME_CNOT: frame_cnot(s, a1, a2); break;
            case CLIFFT_OP_FRAME_CZ: frame_cz(s, a1, a2); break;
            case CLIFFT_OP_FRAME_H: frame_h(s, a1); break;
            case CLIFFT_OP_FRAME_S: frame_s(s, a1, 0); break;
            case CLIFFT_OP_FRAME_S_DAG: frame_s(s, a1, 1); break;
            case CLIFFT_OP_FRAME_SWAP: frame_swap(s, a1, a2); break;
            case CLIFFT_OP_ARRAY_CNOT: array_cnot(s, a1, a2); break;
            case CLIFFT_OP_ARRAY_CZ: array_cz(s, a1, a2); break;
            case CLIFFT_OP_ARRAY_SWAP: array_swap(s, a1, a2); break;
            case CLIFFT_OP_ARRAY_MULTI_CNOT: array_multi_cnot(s, a1, rd_u64(I + 8)); break;
            case CLIFFT_OP_ARRAY_MULTI_CZ: array_multi_cz(s, a1, rd_u64(I + 8)); break;
            case CLIFFT_OP_ARRAY_H: array_h(s, a1); break;
            case CLIFFT_OP_ARRAY_S: array_s(s, a1, 0); break;
            case CLIFFT_OP_ARRAY_S_DAG: array_s(s, a1, 1); break;
            case CLIFFT_OP_ARRAY_T: array_rot(s, a1, kInvSqrt2, kInvSqrt2); break;
            case CLIFFT_OP_ARRAY_T_DAG: array_rot(s, a1, kInvSqrt2, -kInvSqrt2); break;
            case CLIFFT_OP_ARRAY_ROT: array_rot(s, a1, rd_f64(I + 8), rd_f64(I + 16)); break;
            case CLIFFT_OP_ARRAY_U2: array_u2(s, a1, p0); break;
            case CLIFFT_OP_ARRAY_U4: array_u4(s, a1, a2, p0); break;
            case CLIFFT_OP_EXPAND: expand_phase(s, a1, 0, 0, 0); break;
            case CLIFFT_OP_EXPAND_T: expand_phase(s, a1, kInvSqrt2, kInvSqrt2, 1); break;
            case CLIFFT_OP_EXPAND_T_DAG: expand_phase(s, a1, kInvSqrt2, -kInvSqrt2, 1); break;
            case CLIFFT_OP_EXPAND_ROT: expand_phase(s, a1, rd_f64(I + 8), rd_f64(I + 16), 1); break;
            case CLIFFT_OP_MEAS_DORMANT_STATIC:
                if (meas_dormant_static(s, a1, p0, sign, (fl & CLIFFT_FLAG_IDENTITY) != 0)) return 1;
                break;
            case CLIFFT_OP_MEAS_DORMANT_RANDOM:
                if (meas_dormant_random(s, a1, p0, sign)) return 1;
                break;
            case CLIFFT_OP_MEAS_ACTIVE_DIAGONAL:
                if (meas_active_diagonal(s, a1, p0, sign)) return 1;
                break;
            case CLIFFT_OP_MEAS_ACTIVE_INTERFERE:
                if (meas_interfere(s, a1, a1, p0, sign)) return 1;
                break;
            case CLIFFT_OP_SWAP_MEAS_INTERFERE:
                if (meas_interfere(s, a1, a2, p0, sign)) return 1;
                break;
            case CLIFFT_OP_APPLY_PAULI:
                if (s->meas[p1])
                    apply_pauli(s, im->pauli_x + (size_t)p0 * s->nw, im->pauli_z + (size_t)p0 * s->nw,
                                im->pauli_sign[p0] != 0);
                break;
            case CLIFFT_OP_NOISE: noise_site(s, p0); break;
            case CLIFFT_OP_NOISE_BLOCK:
                while (s->next_noise >= p0 && s->next_noise < p0 + p1) noise_site(s, s->next_noise);
                break;
            case CLIFFT_OP_READOUT_NOISE: readout_noise(s, p0); break;
            case CLIFFT_OP_DETECTOR: {
                uint8_t par = (fl & CLIFFT_FLAG_EXPECTED_ONE) ? 1 : 0;
                par ^= list_parity(s->meas, im->detector_offsets, im->detector_targets, p0);
                s->det[p1] = par;
                break;
            }
            case CLIFFT_OP_POSTSELECT: {
                uint8_t par = (fl & CLIFFT_FLAG_EXPECTED_ONE) ? 1 : 0;
                par ^= list_parity(s->meas, im->detector_offsets, im->detector_targets, p0);
                s->det[p1] = 0;
                if (par) {
                    s->discarded = 1;
                    return 1;
                }
                break;
            }
            case CLIFFT_OP_OBSERVABLE:
                s->obs[p1] ^= list_parity(s->meas, im->observable_offsets, im->observable_targets, p0);
                break;
            case CLIFFT_OP_EXP_VAL: exp_val(s, p0, p1); break;
            default: FAIL("unknown opcode %u at instruction %u", op, pc);
        }
    }
    return 0;
}

int oracle_run(const clifft_program_image* img, const oracle_args* a, oracle_outputs* o) {
    if (img->peak_rank >= 40) FAIL("oracle: peak_rank %u too large", img->peak_rank);
    const uint32_t nw = img->num_words;
    const uint32_t slots = img->total_meas_slots;
    const uint64_t vdim = 1ULL << img->peak_rank;
    ostate s;
    memset(&s, 0, sizeof s);
    s.img = img;
    s.nw = nw;
    s.v = (cplx*)calloc(vdim, sizeof(cplx));
    s.px = (uint64_t*)calloc(nw ? nw : 1, 8);
    s.pz = (uint64_t*)calloc(nw ? nw : 1, 8);
    s.meas = (uint8_t*)calloc(slots + 1, 1);
    s.det = (uint8_t*)calloc(img->num_detectors + 1, 1);
    s.obs = (uint8_t*)calloc(img->num_observables + 1, 1);
    s.exp = (double*)calloc(img->num_exp_vals + 1, sizeof(double));
    if (!s.v || !s.px || !s.pz || !s.meas || !s.det || !s.obs || !s.exp) FAIL("oracle: out of memory");
    s.rng_kind = (int)a->rng_kind;
    s.dust_eps = a->dust_eps;
    if (s.rng_kind == ORACLE_RNG_XOSHIRO) xo_seed(s.xo, a->seed);
    s.key[0] = (uint32_t)a->seed;
    s.key[1] = (uint32_t)(a->seed >> 32);
    int rc = 0;
    for (uint32_t shot = 0; shot < a->shots && rc == 0; ++shot) {
        /* SchrodingerState::reset (src/clifft/svm/svm_state.cc:220-267) */
        memset(s.v, 0, (size_t)vdim * sizeof(cplx));
        s.v[0].re = 1.0;
        memset(s.px, 0, nw * 8);
        memset(s.pz, 0, nw * 8);
        s.gamma.re = 1.0;
        s.gamma.im = 0.0;
        s.k = 0;
        memset(s.meas, 0, slots);
        memset(s.det, 0, img->num_detectors);
        memset(s.obs, 0, img->num_observables);
        memset(s.exp, 0, img->num_exp_vals * sizeof(double));
        s.discarded = 0;
        s.reachable = 1;
        s.log_prob = 0.0;
        s.shot = a->first_shot + shot;
        s.draw = 0;
        s.forced = a->forced_meas ? a->forced_meas + (size_t)shot * slots : NULL;
        s.meas_prob = o->meas_prob ? o->meas_prob + (size_t)shot * slots : NULL;
        if (s.meas_prob)
            for (uint32_t i = 0; i < slots; ++i) s.meas_prob[i] = NAN;
        s.faults_active = (a->fault_offsets != NULL) || (a->readout_offsets != NULL);
        if (s.faults_active) {
            /* prepare_forced_shot cursor setup (src/clifft/svm/svm.cc:497-520) */
            if (a->fault_offsets) {
                s.ff_sites = a->fault_sites + a->fault_offsets[shot];
                s.ff_chan = a->fault_channels + a->fault_offsets[shot];
                s.ff_n = a->fault_offsets[shot + 1] - a->fault_offsets[shot];
            } else {
                s.ff_n = 0;
            }
            s.ff_pos = 0;
            if (s.ff_n) {
                s.next_noise = s.ff_sites[0];
                s.ff_pos = 1;
            } else {
                s.next_noise = UINT32_MAX;
            }
            if (a->readout_offsets) {
                s.ro_idx = a->readout_entries + a->readout_offsets[shot];
                s.ro_n = a->readout_offsets[shot + 1] - a->readout_offsets[shot];
            } else {
                s.ro_n = 0;
            }
            s.ro_pos = 0;
        } else {
            /* sample() per-shot noise seeding (src/clifft/svm/svm.cc:225-226) */
            s.next_noise = 0;
            draw_next_noise(&s);
        }
        rc = execute(&s);
        if (rc == 1) rc = 0; /* early stop (postselect / unreachable) is not an error */
        if (rc < 0) break;
        if (o->meas && img->num_measurements)
            memcpy(o->meas + (size_t)shot * img->num_measurements, s.meas, img->num_measurements);
        if (o->det && img->num_detectors)
            memcpy(o->det + (size_t)shot * img->num_detectors, s.det, img->num_detectors);
        if (o->obs)
            for (uint32_t i = 0; i < img->num_observables; ++i) {
                uint8_t val = s.obs[i];
                if (i < img->num_expected_observables && img->expected_observables[i]) val ^= 1;
                o->obs[(size_t)shot * img->num_observables + i] = val;
            }
        if (o->exp_vals && img->num_exp_vals)
            memcpy(o->exp_vals + (size_t)shot * img->num_exp_vals, s.exp, img->num_exp_vals * sizeof(double));
        if (o->discarded) o->discarded[shot] = (uint8_t)s.discarded;
        if (o->log_prob) o->log_prob[shot] = s.log_prob;
        if (o->reachable) o->reachable[shot] = (uint8_t)s.reachable;
        if (o->final_k) o->final_k[shot] = s.k;
        if (o->final_gamma) {
            o->final_gamma[2 * shot] = s.gamma.re;
            o->final_gamma[2 * shot + 1] = s.gamma.im;
        }
        if (o->final_px) memcpy(o->final_px + (size_t)shot * nw, s.px, nw * 8);
        if (o->final_pz) memcpy(o->final_pz + (size_t)shot * nw, s.pz, nw * 8);
        if (o->final_v) {
            double* row = o->final_v + (size_t)shot * vdim * 2;
            memset(row, 0, (size_t)vdim * 2 * sizeof(double));
            memcpy(row, s.v, ((size_t)1 << s.k) * sizeof(cplx));
        }
    }
    o->dust_clamps = s.dust_clamps;
    free(s.v);
    free(s.px);
    free(s.pz);
    free(s.meas);
    free(s.det);
    free(s.obs);
    free(s.exp);
    return rc < 0 ? -1 : 0;
}
