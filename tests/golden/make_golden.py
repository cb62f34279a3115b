"""Generates the golden fixtures in tests/golden/ from the reference executor.

Run in a container where the reference tree is available and
oracle/build_ref.sh has built oracle/_ref/libclifft_ref.so:

    python tests/golden/make_golden.py

Each fixture `<case>.npz` holds one program (after the reference's own
bytecode passes, so U2 / U4 / MULTI / SWAP_MEAS / NOISE_BLOCK nodes are the
reference's) together with reference outputs:
  * `sample_*`  -- clifft::sample(program, SAMPLE_SHOTS, seed) records;
  * `forced_*`  -- step-wise forced replay (forced outcomes, injected faults,
                   readout flips): records, per-measurement probabilities,
                   log probability, reachability, final k / gamma / frame / v.
The parity tests on the GPU machine (where the reference tree does not exist)
read only these files.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from clifft_b200 import workloads as W  # noqa: E402
from oracle import pyoracle as O  # noqa: E402
from _programs import random_forced_inputs, random_program  # noqa: E402

SAMPLE_SHOTS = 256
FORCED_SHOTS = 24


def cases():
    out = []
    for seed in range(12):
        out.append((f"fuzz{seed:02d}", random_program(seed, n=10, length=180, max_k=6,
                                                      postselect=(seed % 4 == 3))))
    out.append(("fuzz_k9", random_program(100, n=12, length=260, max_k=9)))
    out.append(("fuzz_w2", random_program(101, n=70, length=200, max_k=6)))
    out.append(("fuzz_k16", random_program(102, n=24, length=260, max_k=16, noise=True,
                                           expand_bias=0.45)))
    out.append(("cfg0", W.lower(W.config0())))
    c2 = W.config2_circuits()
    out.append(("cfg2_s105", W.lower(c2[5])))
    out.append(("cfg2_s100", W.lower(c2[0])))
    c4, _ = W.config4()
    out.append(("cfg4", W.lower(c4)))
    return out


def main():
    if not O.ref_available():
        raise SystemExit("reference harness missing: run oracle/build_ref.sh first")
    for name, raw in cases():
        prog = O.ref_passes(raw, O.PASS_ALL)
        shots_forced = 6 if prog.peak_rank > 12 else FORCED_SHOTS
        prog.name = name
        d = {f"prog_{k}": v for k, v in prog.to_npz_dict().items()}
        d["ref_backend"] = np.array(O.ref_backend())
        seed = 1000 + len(name)
        if not prog.has_postselection:
            s = O.ref_sample(prog, SAMPLE_SHOTS, seed)
            d.update({f"sample_{k}": v for k, v in s.items()})
        else:
            s = O.ref_sample_survivors(prog, SAMPLE_SHOTS, seed, keep_records=True)
            d.update({f"surv_{k}": np.asarray(v) for k, v in s.items()})
        d["sample_seed"] = np.array(seed)
        # forced inputs: random faults and readout flips, and outcomes sampled
        # by the oracle under those same faults (every 5th record flipped to
        # exercise unreachable outcomes)
        faults, ros = random_forced_inputs(prog, shots_forced, seed + 2, fault_rate=0.2)
        o = O.run(prog, shots_forced, seed=seed + 1, rng=O.RNG_PHILOX, faults=faults,
                  readout_faults=ros)
        fm = np.zeros((shots_forced, prog.total_meas_slots), np.uint8)
        fm[:, :prog.num_measurements] = o["meas"]
        fm[::5] ^= 1
        f = O.ref_forced(prog, fm, faults, ros)
        d["forced_meas_in"] = fm
        fo = np.zeros(shots_forced + 1, np.uint32)
        flat_s, flat_c = [], []
        for i, sh in enumerate(faults):
            flat_s += [x[0] for x in sh]
            flat_c += [x[1] for x in sh]
            fo[i + 1] = len(flat_s)
        ro = np.zeros(shots_forced + 1, np.uint32)
        flat_r = []
        for i, sh in enumerate(ros):
            flat_r += sh
            ro[i + 1] = len(flat_r)
        d.update(fault_offsets=fo, fault_sites=np.array(flat_s, np.uint32),
                 fault_channels=np.array(flat_c, np.uint32), readout_offsets=ro,
                 readout_entries=np.array(flat_r, np.uint32))
        for k, v in f.items():
            d[f"forced_{k}"] = v
        if prog.peak_rank > 12:
            # large statevectors: keep the first 2^12 amplitudes of each final state
            d["forced_final_v"] = f["final_v"][:, :1 << 12]
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **d)
        print(name, prog.summary()["ops"].get("ARRAY_U2", 0), prog.summary()["ops"].get("ARRAY_U4", 0),
              prog.peak_rank, prog.num_instructions)


def dense_program():
    """A k = 20 program dense in single- and two-axis unitaries (the
    reference's passes turn its gate runs into U2 / U4 nodes): the workload
    of the tensor-core dense blocks, which the configured programs (CNOT, CZ,
    SWAP and phase gates only) never form."""
    return random_program(500, n=24, length=900, max_k=20, noise=False, classical=False, expvals=False,
                          readout=False, expand_bias=0.2)


def bench_programs():
    """Benchmark programs (reference bytecode passes applied) for bench.py:
    programs/<name>.npz for configs 0, 1, 3, the 64 programs of config 2 and
    the dense k = 20 program."""
    outdir = os.path.join(HERE, "programs")
    os.makedirs(outdir, exist_ok=True)
    items = [("cfg0", W.lower(W.config0())),
             ("cfg1", W.lower(W.config1(), postselect_all=True)),
             ("cfg3", W.lower(W.config3()))]
    for i, c in enumerate(W.config2_circuits()):
        items.append((f"cfg2_{i:02d}", W.lower(c)))
    c4, theta = W.config4()
    items.append(("cfg4", W.lower(c4)))
    items.append(("dense_k20", dense_program()))
    for name, raw in items:
        prog = O.ref_passes(raw, O.PASS_ALL)
        prog.name = name
        prog.save(os.path.join(outdir, f"{name}.npz"))


def load_case(path):
    """(program, dict of arrays) from a fixture file."""
    from clifft_b200.program import Program
    with np.load(path, allow_pickle=False) as z:
        d = {k: z[k] for k in z.files}
    prog = Program.from_npz_dict({k[5:]: v for k, v in d.items() if k.startswith("prog_")})
    return prog, d


def unflatten(d):
    """Forced-fault lists from a fixture's CSR arrays."""
    fo, fs, fc = d["fault_offsets"], d["fault_sites"], d["fault_channels"]
    ro, re_ = d["readout_offsets"], d["readout_entries"]
    n = fo.shape[0] - 1
    faults = [[(int(fs[j]), int(fc[j])) for j in range(fo[i], fo[i + 1])] for i in range(n)]
    ros = [[int(re_[j]) for j in range(ro[i], ro[i + 1])] for i in range(n)]
    return faults, ros


if __name__ == "__main__":
    main()
    bench_programs()
