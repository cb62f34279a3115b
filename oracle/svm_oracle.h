/*
 * svm_oracle.h -- CPU restatement of the reference Schrodinger-VM executor.
 *
 * TEST INFRASTRUCTURE. This library is the checker for the CUDA backend: the
 * parity tests, the import-time smoke check and the CPU-baseline leg of the
 * benchmark may load it; the product never does. It restates, in plain C and
 * double precision, the scalar code path of the reference executor
 * (src/clifft/svm/svm_kernels.inl, svm_forced_kernels.cc, svm_state.cc,
 * svm.cc:191-345) and is pinned against the reference itself, built from its
 * own sources by oracle/build_ref.sh (tests/test_oracle_vs_reference.py).
 *
 * Two random streams are provided:
 *   ORACLE_RNG_XOSHIRO  the reference's single xoshiro256++ stream seeded once
 *                       by SplitMix64 and streamed across shots
 *                       (src/clifft/svm/svm.h:40-90,150); reproduces
 *                       clifft::sample bit for bit;
 *   ORACLE_RNG_PHILOX   the CUDA backend's per-shot counter stream
 *                       (Philox4x32-10, key = seed, counter = (draw/2, 0,
 *                       shot_lo, shot_hi), two 53-bit uniforms per block);
 *                       reproduces the GPU's free sampling bit for bit.
 */
#ifndef CLIFFT_SVM_ORACLE_H
#define CLIFFT_SVM_ORACLE_H

#include <stdint.h>

#include "../include/clifft_program_image.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_RNG_XOSHIRO = 0, ORACLE_RNG_PHILOX = 1 };

typedef struct oracle_args {
    uint32_t shots;
    uint64_t seed;
    uint32_t rng_kind;
    uint64_t first_shot;           /* Philox shot index of shot 0 */
    double dust_eps;               /* relative dust threshold; reference 1e-18 */
    const uint8_t* forced_meas;    /* NULL or shots x total_meas_slots bytes */
    const uint32_t* fault_offsets; /* NULL or shots + 1: forced noise faults */
    const uint32_t* fault_sites;   /* ascending per shot */
    const uint32_t* fault_channels;
    const uint32_t* readout_offsets; /* NULL or shots + 1: forced readout flips */
    const uint32_t* readout_entries; /* ascending per shot */
} oracle_args;

typedef struct oracle_outputs {
    uint8_t* meas;        /* shots x num_measurements (visible slots) */
    uint8_t* det;         /* shots x num_detectors */
    uint8_t* obs;         /* shots x num_observables, XOR expected_observables */
    double* exp_vals;     /* shots x num_exp_vals */
    uint8_t* discarded;   /* shots */
    double* meas_prob;    /* shots x total_meas_slots; NaN where not executed */
    double* log_prob;     /* shots: forced-mode log probability */
    uint8_t* reachable;   /* shots */
    uint32_t* final_k;    /* shots */
    double* final_gamma;  /* shots x 2 */
    uint64_t* final_px;   /* shots x num_words */
    uint64_t* final_pz;
    double* final_v;      /* shots x 2^peak_rank x 2 (zero beyond 2^final_k) */
    uint64_t dust_clamps; /* out: total over shots */
} oracle_outputs;

int oracle_run(const clifft_program_image* img, const oracle_args* args, oracle_outputs* out);
const char* oracle_last_error(void);

/* Philox4x32-10 block, for known-answer tests of the stream. */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

#ifdef __cplusplus
}
#endif

#endif
