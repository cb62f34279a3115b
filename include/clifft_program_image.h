/*
 * clifft_program_image.h -- flat, pointer-and-count description of a compiled
 * Clifft program (bytecode + constant pool + metadata).
 *
 * This is the serialisation of the reference's `clifft::CompiledModule`
 * (src/clifft/backend/backend.h:324-344) and its `ConstantPool`
 * (src/clifft/backend/backend.h:255-300) into plain arrays, so that a
 * program can cross a C ABI without C++ types:
 *
 *   - instructions are the reference's 32-byte `Instruction` records
 *     (src/clifft/backend/backend.h:95-163), copied byte for byte;
 *   - every Pauli mask arena (PauliMaskArena, src/clifft/util/pauli_arena.h:63-110)
 *     becomes parallel x / z word arrays of `num_words` u64 per mask plus a
 *     sign byte per mask;
 *   - noise sites (NoiseSite / NoiseChannel, src/clifft/frontend/hir.h:68-75)
 *     become CSR: channel range [site_offsets[s], site_offsets[s+1]) with one
 *     probability and one x/z mask per channel (the channel's handle into
 *     noise_channel_masks is resolved at export time);
 *   - detector / observable target lists become CSR as well;
 *   - FusedU2Node (backend.h:224-234) is 4 frame states x {4 matrix entries,
 *     gamma multiplier} complex doubles = 40 doubles per node, plus 4 out-state
 *     bytes; FusedU4Node (backend.h:240-253) is 16 frame states x {16 matrix
 *     entries (row-major), gamma multiplier} = 544 doubles per node, plus 16
 *     out-state bytes.
 *
 * All pointers are host pointers owned by the caller; a consumer copies what it
 * needs before the call returns.
 */
#ifndef CLIFFT_PROGRAM_IMAGE_H
#define CLIFFT_PROGRAM_IMAGE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CLIFFT_INSTRUCTION_BYTES 32
#define CLIFFT_U2_DOUBLES_PER_NODE 40  /* 4 states x 5 complex */
#define CLIFFT_U4_DOUBLES_PER_NODE 544 /* 16 states x 17 complex */

typedef struct clifft_program_image {
    /* CompiledModule metadata (backend.h:327-334) */
    uint32_t num_qubits;
    uint32_t peak_rank;
    uint32_t num_measurements;   /* visible measurements */
    uint32_t total_meas_slots;   /* visible + hidden */
    uint32_t num_detectors;
    uint32_t num_observables;
    uint32_t num_exp_vals;
    uint32_t has_postselection;

    /* bytecode */
    uint32_t num_instructions;
    const uint8_t* instructions; /* num_instructions * 32 bytes */

    /* width of every Pauli mask in 64-bit words: ceil(num_qubits / 64) */
    uint32_t num_words;

    /* OP_APPLY_PAULI masks (ConstantPool::pauli_masks) */
    uint32_t num_pauli_masks;
    const uint64_t* pauli_x; /* num_pauli_masks * num_words */
    const uint64_t* pauli_z;
    const uint8_t* pauli_sign; /* num_pauli_masks */

    /* OP_EXP_VAL masks (ConstantPool::exp_val_masks) */
    uint32_t num_exp_val_masks;
    const uint64_t* exp_val_x;
    const uint64_t* exp_val_z;
    const uint8_t* exp_val_sign;

    /* OP_NOISE / OP_NOISE_BLOCK sites (ConstantPool::noise_sites) */
    uint32_t num_noise_sites;
    const uint32_t* noise_site_offsets; /* num_noise_sites + 1 */
    uint32_t num_noise_channels;
    const double* noise_channel_prob;  /* num_noise_channels */
    const uint64_t* noise_channel_x;   /* num_noise_channels * num_words */
    const uint64_t* noise_channel_z;
    const double* noise_hazards;       /* num_noise_sites (cumulative) */

    /* OP_READOUT_NOISE entries (ConstantPool::readout_noise) */
    uint32_t num_readout_noise;
    const uint32_t* readout_meas_idx;
    const double* readout_prob;

    /* detector and observable target lists (CSR) */
    uint32_t num_detector_lists;
    const uint32_t* detector_offsets; /* num_detector_lists + 1 */
    const uint32_t* detector_targets;
    uint32_t num_observable_lists;
    const uint32_t* observable_offsets;
    const uint32_t* observable_targets;

    /* fused nodes */
    uint32_t num_u2;
    const double* u2_data;     /* num_u2 * 40 doubles */
    const uint8_t* u2_out;     /* num_u2 * 4 */
    uint32_t num_u4;
    const double* u4_data;     /* num_u4 * 544 doubles */
    const uint8_t* u4_out;     /* num_u4 * 16 */

    /* CompiledModule::expected_observables (backend.h:339) */
    uint32_t num_expected_observables;
    const uint8_t* expected_observables;

    /* ConstantPool::global_weight (backend.h:261) */
    double global_weight_re;
    double global_weight_im;
} clifft_program_image;

/* Opcode numbering of the reference's `enum class Opcode`
 * (src/clifft/backend/backend.h:25-86). */
enum clifft_opcode {
    CLIFFT_OP_FRAME_CNOT = 0,
    CLIFFT_OP_FRAME_CZ,
    CLIFFT_OP_FRAME_H,
    CLIFFT_OP_FRAME_S,
    CLIFFT_OP_FRAME_S_DAG,
    CLIFFT_OP_FRAME_SWAP,
    CLIFFT_OP_ARRAY_CNOT,
    CLIFFT_OP_ARRAY_CZ,
    CLIFFT_OP_ARRAY_SWAP,
    CLIFFT_OP_ARRAY_MULTI_CNOT,
    CLIFFT_OP_ARRAY_MULTI_CZ,
    CLIFFT_OP_ARRAY_H,
    CLIFFT_OP_ARRAY_S,
    CLIFFT_OP_ARRAY_S_DAG,
    CLIFFT_OP_ARRAY_T,
    CLIFFT_OP_ARRAY_T_DAG,
    CLIFFT_OP_ARRAY_ROT,
    CLIFFT_OP_ARRAY_U2,
    CLIFFT_OP_ARRAY_U4,
    CLIFFT_OP_EXPAND,
    CLIFFT_OP_EXPAND_T,
    CLIFFT_OP_EXPAND_T_DAG,
    CLIFFT_OP_EXPAND_ROT,
    CLIFFT_OP_MEAS_DORMANT_STATIC,
    CLIFFT_OP_MEAS_DORMANT_RANDOM,
    CLIFFT_OP_MEAS_ACTIVE_DIAGONAL,
    CLIFFT_OP_MEAS_ACTIVE_INTERFERE,
    CLIFFT_OP_SWAP_MEAS_INTERFERE,
    CLIFFT_OP_MEAS_DORMANT_STATIC_FORCED,
    CLIFFT_OP_MEAS_DORMANT_RANDOM_FORCED,
    CLIFFT_OP_MEAS_ACTIVE_DIAGONAL_FORCED,
    CLIFFT_OP_MEAS_ACTIVE_INTERFERE_FORCED,
    CLIFFT_OP_SWAP_MEAS_INTERFERE_FORCED,
    CLIFFT_OP_APPLY_PAULI,
    CLIFFT_OP_NOISE,
    CLIFFT_OP_NOISE_BLOCK,
    CLIFFT_OP_READOUT_NOISE,
    CLIFFT_OP_DETECTOR,
    CLIFFT_OP_POSTSELECT,
    CLIFFT_OP_OBSERVABLE,
    CLIFFT_OP_EXP_VAL,
    CLIFFT_NUM_OPCODES
};

/* Instruction flag bits (backend.h:97-101). */
#define CLIFFT_FLAG_SIGN 0x01u
#define CLIFFT_FLAG_HIDDEN 0x02u
#define CLIFFT_FLAG_IDENTITY 0x04u
#define CLIFFT_FLAG_EXPECTED_ONE 0x08u

/* Byte offsets inside one 32-byte instruction (backend.h:103-160). */
#define CLIFFT_INSTR_OFF_OPCODE 0
#define CLIFFT_INSTR_OFF_FLAGS 2
#define CLIFFT_INSTR_OFF_AXIS1 4
#define CLIFFT_INSTR_OFF_AXIS2 6
#define CLIFFT_INSTR_OFF_PAYLOAD 8

#ifdef __cplusplus
}
#endif

#endif /* CLIFFT_PROGRAM_IMAGE_H */
