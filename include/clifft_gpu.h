/*
 * clifft_gpu.h -- C ABI of the B200 (sm_100a) Schrodinger-VM backend.
 *
 * The backend executes the reference compiler's bytecode unchanged: a program
 * is handed over as a `clifft_program_image` (the flat form of
 * clifft::CompiledModule, src/clifft/backend/backend.h:324-344), uploaded once,
 * and then sampled in batches of shots by persistent CUDA kernels.
 *
 * Mapping onto the reference interface:
 *   clifft_gpu_load          replaces handing a `const CompiledModule&` to the
 *                            SVM (src/clifft/svm/svm.h:331,358); validates the
 *                            bytecode against the executor's invariants
 *                            (axis ranges, EXPAND on axis k, active measurement
 *                            on axis k-1, pool indices) before anything runs;
 *   clifft_gpu_sample        replaces clifft::sample (svm.h:331-332,
 *                            src/clifft/svm/svm.cc:191-255) and, with
 *                            CLIFFT_GPU_SURVIVORS, clifft::sample_survivors
 *                            (svm.h:358-360, svm.cc:266-345); with
 *                            CLIFFT_GPU_FORCED it is the batched form of the
 *                            forced-outcome replay behind
 *                            clifft::record_probabilities (svm.h:405-406,
 *                            src/clifft/api/record_probabilities.cc:122-191)
 *                            and of the forced-fault cursors of sample_k
 *                            (svm.cc:497-520);
 *   clifft_gpu_backend_name  mirrors clifft::svm_backend (svm.h:316);
 *   clifft_gpu_last_error    carries the message the reference would throw
 *                            (std::invalid_argument / std::runtime_error).
 *
 * Every entry point returns 0 on success or a negative status and never throws
 * across the ABI. Calls are re-entrant: each call uses its own stream-ordered
 * scratch, so concurrent host threads may sample the same program. A sampling
 * call returns after its stream has finished the call's work. Statevectors
 * that do not fit in shared memory live in a device slab kept on the program
 * handle between calls (one call at a time uses it; a concurrent call
 * allocates its own for the call's duration). Per-call scratch and staged
 * records come from the device's default stream-ordered memory pool, whose
 * release threshold the library raises to 1 GiB on first use of a device so
 * freed memory is reused instead of remapped by every call.
 */
#ifndef CLIFFT_GPU_H
#define CLIFFT_GPU_H

#include <stddef.h>
#include <stdint.h>

#include "clifft_program_image.h"

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CLIFFT_GPU_OK 0
#define CLIFFT_GPU_EINVAL (-1)   /* invalid argument / malformed bytecode (ValueError) */
#define CLIFFT_GPU_ECUDA (-2)    /* CUDA runtime failure (RuntimeError) */
#define CLIFFT_GPU_EDEVICE (-3)  /* kernel reported a device-side error (RuntimeError) */
#define CLIFFT_GPU_ENOMEM (-4)   /* device allocation failed (MemoryError) */

/* precision of the statevector (probability sums, gamma and renormalisation
 * are always FP64) */
#define CLIFFT_GPU_FP64 0u
#define CLIFFT_GPU_FP32 1u

/* sample flags */
#define CLIFFT_GPU_SURVIVORS 0x01u      /* count survivors; shots stop at the first failing POSTSELECT */
#define CLIFFT_GPU_FORCED_MEAS 0x02u    /* outcomes from forced_meas (record_probabilities semantics) */
#define CLIFFT_GPU_FORCED_FAULTS 0x04u  /* fault sites / channels / readout flips from the CSR inputs */
#define CLIFFT_GPU_DEVICE_PTRS 0x08u    /* every input/output pointer is a device pointer */
#define CLIFFT_GPU_TRACE 0x10u          /* fill meas_prob and the final-state dump */
#define CLIFFT_GPU_NO_FUSION 0x20u      /* plain executor: one statevector pass per opcode */
#define CLIFFT_GPU_FORCE_FUSION 0x40u   /* reserved (fusion is on unless CLIFFT_GPU_NO_FUSION) */
#define CLIFFT_GPU_PROFILE 0x80u        /* fill phase_cycles (adds timing atomics; not for benchmarks) */
#define CLIFFT_GPU_NO_AUTOTUNE 0x100u   /* group_threads == 0: use the built-in heuristic, no trial launches */
#define CLIFFT_GPU_NO_SEGMENTS 0x200u   /* survivor runs: one launch, no compaction between POSTSELECT segments */
#define CLIFFT_GPU_RAW_PARITY 0x400u   /* detectors and observables without their expected parities, POSTSELECT
                                         recorded as a detector instead of discarding: the reference-syndrome
                                         shot of compute_reference_syndrome (src/clifft/api/reference_syndrome.cc:9-30) */
#define CLIFFT_GPU_TENSOR_DENSE 0x800u /* FP32, one CTA per shot, fusion on: runs of fused micro-ops on at most four
                                         tile-local bits holding an H / U2 / U4 are composed into one 16x16 complex
                                         matrix and applied on the tensor cores (3xTF32 MMAs). Probabilities and
                                         amplitudes stay within FP32 tolerance but are not bit-identical to the
                                         CUDA-core path, hence opt-in */

typedef struct clifft_gpu_program clifft_gpu_program;

typedef struct clifft_gpu_sample_args {
    uint64_t shots;
    uint64_t seed;          /* Philox key; shot s uses counter (draw/2, 0, first_shot + s) */
    uint64_t first_shot;    /* global index of shot 0 (multi-GPU shards, resumption) */
    uint32_t precision;     /* CLIFFT_GPU_FP64 or CLIFFT_GPU_FP32 */
    uint32_t flags;
    uint32_t group_threads; /* 0 = automatic (autotuned, see below); 1,2,4..32 = lanes per shot
                               (32/G shots per warp); 64..1024 = one CTA of that size per shot;
                               288 / 544 = one CTA of 256 / 512 compute threads plus a warp that
                               issues the tile copies of fused blocks */
    uint32_t max_resident;  /* upper bound on shots whose statevectors are resident at once (shots run
                               in waves of at most this many); 0 = as many as one wave of the launch holds */
    double dust_eps;        /* relative dust threshold; 0 = 1e-18 (FP64) / 1e-9 (FP32) */
    /* CLIFFT_GPU_FORCED_MEAS: shots x total_meas_slots bytes (0/1) */
    const uint8_t* forced_meas;
    /* CLIFFT_GPU_FORCED_FAULTS: per-shot CSR over fired noise sites (ascending)
     * with the fired channel (index within the site), and readout entries. */
    const uint32_t* fault_offsets;   /* shots + 1 */
    const uint32_t* fault_sites;
    const uint32_t* fault_channels;
    const uint32_t* readout_offsets; /* shots + 1 */
    const uint32_t* readout_entries;
    void* stream;                    /* cudaStream_t; NULL = the legacy default stream */
} clifft_gpu_sample_args;

typedef struct clifft_gpu_outputs {
    /* Per-shot bit-packed records, little-endian bit order inside u64 words:
     * bit i of row s is word[s * words + i / 64] >> (i % 64). Any may be NULL. */
    uint64_t* meas;       /* shots x ceil(num_measurements / 64) */
    uint64_t* det;        /* shots x ceil(num_detectors / 64) */
    uint64_t* obs;        /* shots x ceil(num_observables / 64), XOR expected_observables */
    double* exp_vals;     /* shots x num_exp_vals */
    uint8_t* survived;    /* shots: 1 unless discarded by POSTSELECT / unreachable */
    /* CLIFFT_GPU_TRACE */
    double* meas_prob;    /* shots x total_meas_slots: probability of the realised outcome, NaN if not executed */
    double* log_prob;     /* shots: forced-mode log probability (record_probabilities) */
    uint32_t* final_k;    /* shots */
    double* final_gamma;  /* shots x 2 */
    uint64_t* final_px;   /* shots x num_words */
    uint64_t* final_pz;
    double* final_v;      /* dump_shots x 2^peak_rank x 2 (complex FP64) */
    uint64_t dump_shots;  /* rows of final_v to fill (shots 0 .. dump_shots-1) */
    /* host-side results (always host memory) */
    uint64_t passed_shots;
    uint64_t logical_errors;
    uint64_t* observable_ones; /* num_observables counters, may be NULL */
    uint64_t dust_clamps;
    uint64_t algorithmic_bytes; /* statevector bytes the executed opcodes must move, opcode by opcode */
    uint64_t streamed_bytes;    /* statevector bytes actually streamed (a fused block streams once) */
    uint32_t kernel_launches;  /* kernels this call launched */
    float kernel_ms;           /* device time of the sampling kernel(s) */
    uint32_t group_threads;    /* shot-group size that ran */
    uint32_t state_in_smem;    /* 1 if the statevectors lived in shared memory */
    uint32_t fused;            /* 1 if fused tile sweeps were enabled */
    uint64_t phase_cycles[5];  /* CLIFFT_GPU_PROFILE: SM cycles in fused blocks, measurements, expansions,
                                  unfused array sweeps, other opcodes (summed over CTA shot groups;
                                  zero when shots run on warps) */
} clifft_gpu_outputs;

/* Upload + validate a program. *out receives an opaque handle. */
int clifft_gpu_load(const clifft_program_image* image, clifft_gpu_program** out);
/* Release a handle (waits for the device) and the statevector slab that
 * sampling calls keep on it between calls. */
void clifft_gpu_free(clifft_gpu_program* prog);
/* Return any spare statevector slab the library holds to the device. */
void clifft_gpu_trim(void);
/* Sample. See the flags above for survivors / forced / trace behaviour.
 * Survivor compaction: with CLIFFT_GPU_SURVIVORS, at least four resident waves
 * of shots and one warp (or less) per shot, the program is cut into up to 8
 * segments after POSTSELECT opcodes; shots still alive at a cut save their
 * state and are compacted into the next segment's launch, so warps carry only
 * live shots. Records and counters are those of a single launch.
 * Autotuning: with group_threads == 0 and no CLIFFT_GPU_NO_AUTOTUNE, the
 * first call of a (precision, mode) pair on a program with at least 1024
 * shots times a few candidate launch shapes (lanes per shot, or CTA size)
 * on up to two resident waves of this call's own shots, keeps the fastest
 * for every handle of the same program content on this device (for the rest
 * of the process), and uses it from then on. With the environment variable
 * CLIFFT_GPU_TUNE_CACHE naming a file, results are also appended there and
 * read back by later processes (keyed by program content, GPU model and
 * mode), so trials run once per program and GPU model. Results do not depend on
 * the launch shape: every shot draws from its own Philox stream and every
 * reduction has a fixed order. Trial launches are counted in
 * kernel_launches but not in kernel_ms. */
int clifft_gpu_sample(clifft_gpu_program* prog, const clifft_gpu_sample_args* args,
                      clifft_gpu_outputs* out);
/* "cuda:sm_100a" when a B200-class device is current; "unavailable:<why>" otherwise. */
const char* clifft_gpu_backend_name(void);
/* Message of the last failing call on this host thread. */
const char* clifft_gpu_last_error(void);
/*
 * clifft_gpu_sample_noalloc -- clifft_gpu_sample without any device memory
 * allocation. No counterpart in the reference (its CPU executor allocates
 * per call); this entry point exists for callers that cannot allocate device
 * memory while they sample: a process whose free device memory is owned by
 * another allocator (a framework's caching allocator that reserved it), or a
 * decoding loop with a fixed device-memory budget in which an allocation that
 * fails mid-run is not acceptable.
 *
 * It runs the same kernel as clifft_gpu_sample and returns the same records
 * and counters for the same arguments. Differences and limits:
 *  - CLIFFT_GPU_DEVICE_PTRS is required: every input and output buffer is a
 *    device buffer the caller owns. CLIFFT_GPU_TRACE and CLIFFT_GPU_PROFILE
 *    are rejected. kernel_ms is not measured (0).
 *  - The program's statevectors must fit in shared memory with the chosen
 *    launch shape (there is no global-memory statevector slab); otherwise the
 *    call returns CLIFFT_GPU_EINVAL and clifft_gpu_sample must be used.
 *  - Launch scratch lives in a file-scope device array of
 *    CLIFFT_GPU_NOALLOC_SCRATCH_WORDS 64-bit words (4 KiB) per device: work
 *    counter, error word, 5 totals, one counter per observable and 8 words of
 *    diagnostics, so a program may have at most
 *    CLIFFT_GPU_NOALLOC_SCRATCH_WORDS - 15 observables; larger programs get
 *    CLIFFT_GPU_EINVAL. Those words must start at zero: the call clears them
 *    itself on args->stream before its launch, so nothing needs to be zeroed
 *    beforehand.
 *  - There is one such array per device per process. Calls that overlap on
 *    the same device (other streams or other host threads) race on it and
 *    their results are undefined: serialise them. The call synchronises its
 *    stream before it returns.
 *  - The first call on each device looks up the array's device address with
 *    that device current (cudaGetSymbolAddress); make that first call before
 *    any stream capture begins on that device.
 */
#define CLIFFT_GPU_NOALLOC_SCRATCH_WORDS 512u
int clifft_gpu_sample_noalloc(clifft_gpu_program* prog, const clifft_gpu_sample_args* args,
                              clifft_gpu_outputs* out);
/*
 * k-fault importance sampling: clifft::sample_k / sample_k_survivors
 * (src/clifft/svm/svm.h:366-372, src/clifft/svm/svm.cc:356-711). Every shot
 * is conditioned on exactly k fault events among the noise sites and readout
 * entries (clifft::noise_site_probabilities order: sites, then readout
 * entries), drawn on the device per shot from the exact conditional
 * Poisson-binomial distribution (uniform k-subsets when every probability is
 * equal); a fired site's channel is drawn as the NOISE opcode draws it. Same
 * arguments and outputs as clifft_gpu_sample (CLIFFT_GPU_SURVIVORS selects
 * sample_k_survivors); forced outcomes / faults are rejected. Strata without
 * probability mass are rejected with the reference's messages. The draws use
 * Philox stream 1 of each shot's counter space, the executor stream 0.
 */
int clifft_gpu_sample_k(clifft_gpu_program* prog, const clifft_gpu_sample_args* args, uint32_t k,
                        clifft_gpu_outputs* out);

/*
 * Multi-program batches (the batched form of clifft::sample over many
 * programs, e.g. a sweep of circuits with different peak rank). A batch is a
 * CUDA graph with one independent branch per program (clear scratch, sampling
 * kernel), so a single graph launch runs all programs side by side, each with
 * its own launch shape.
 *
 *   clifft_gpu_batch_create  n programs, n argument blocks and n output blocks.
 *                            Every entry needs CLIFFT_GPU_DEVICE_PTRS (its inputs
 *                            and records stay in device buffers the caller keeps
 *                            alive for the batch's lifetime); TRACE / PROFILE are
 *                            rejected. Creation runs each entry once through
 *                            clifft_gpu_sample (validation, autotuning), then
 *                            allocates the batch's own statevector slabs and
 *                            scratch and instantiates the graph.
 *   clifft_gpu_batch_run     replays the graph on `stream` (seeds[i] replaces
 *                            entry i's seed when `seeds` is non-NULL), waits, and
 *                            fills each entry's host-side counters (passed_shots,
 *                            observable_ones, ... of the output blocks given at
 *                            creation); *graph_ms = device time of the replay.
 *   clifft_gpu_batch_free    releases the graph, slabs and scratch.
 *
 * No counterpart in the reference (its sample() runs one program per call).
 */
typedef struct clifft_gpu_batch clifft_gpu_batch;
int clifft_gpu_batch_create(clifft_gpu_program* const* progs, const clifft_gpu_sample_args* args,
                            clifft_gpu_outputs* outs, uint32_t n, clifft_gpu_batch** out);
int clifft_gpu_batch_run(clifft_gpu_batch* batch, const uint64_t* seeds, void* stream, float* graph_ms);
void clifft_gpu_batch_free(clifft_gpu_batch* batch);
/*
 * Gradients of expectation values by the adjoint method (d<P>/dtheta for
 * every continuous rotation of a measurement-free, noise-free program). No
 * counterpart in the reference, which has no differentiation.
 *
 * Parameters are the rotation instructions (ARRAY_ROT and EXPAND_ROT) in
 * program order, clifft_gpu_program_num_rot_params of them; parameter j is the
 * phase angle phi_j (radians) of its payload (cos phi, sin phi), the phase the
 * executor puts on the |1> half of the rotated axis. For each of `batch`
 * parameter vectors (args->phases, batch x num_rot_params, or NULL to use the
 * program's own payloads for every row) the call returns every EXP_VAL row
 * (exp_vals, batch x num_exp_vals) and its derivatives (grads, batch x
 * num_exp_vals x num_rot_params). The kernel runs each (vector, EXP_VAL) pair
 * forward to the EXP_VAL, then back through the bytecode, undoing each
 * instruction with its inverse (no per-instruction state is stored) and
 * accumulating the derivatives in FP64; args->precision selects the
 * statevector precision. Programs with measurements, noise, classical records
 * or fused U2 / U4 nodes are rejected (CLIFFT_GPU_EINVAL).
 */
typedef struct clifft_gpu_grad_args {
    uint64_t batch;        /* parameter vectors */
    uint32_t precision;    /* CLIFFT_GPU_FP64 or CLIFFT_GPU_FP32 statevector */
    uint32_t flags;        /* CLIFFT_GPU_DEVICE_PTRS: phases, exp_vals and grads are device pointers */
    const double* phases;  /* batch x num_rot_params, or NULL */
    void* stream;          /* cudaStream_t; NULL = the legacy default stream */
} clifft_gpu_grad_args;
uint32_t clifft_gpu_program_num_rot_params(const clifft_gpu_program* prog);
int clifft_gpu_expval_grad(clifft_gpu_program* prog, const clifft_gpu_grad_args* args, double* exp_vals,
                           double* grads);
/* Program metadata accessors (host memory). */
uint32_t clifft_gpu_program_peak_rank(const clifft_gpu_program* prog);
uint64_t clifft_gpu_program_device_bytes(const clifft_gpu_program* prog);

#ifdef __cplusplus
}
#endif

#endif /* CLIFFT_GPU_H */
