"""Test infrastructure: times the reference's own GPU J/K route on this device beside
the product's build of the same workload, and checks that the two agree.

    make -C oracle refgpu                      # once, where the reference tree is
    python oracle/ref_gpu_bench.py [--workload h2o8_sto3g] [--max-unit-gb 4]

The reference route (oracle/ref_gpu_shim.cu) runs the full four-set product of every
ordered ShellSet 4-tuple: one thread per shell quartet, every integral written to a
device buffer, then digested with two FP64 atomics per integral.  It has no
screening and no permutational symmetry.  Units whose integral buffer exceeds
--max-unit-gb are skipped, and the line then says so (for (H2O)64/cc-pVDZ a single
(dd|dd) unit needs 174 GB, so the reference route cannot run that workload whole).

Prints one JSON line: the reference's device time (CUDA events around its launches),
shell quartets and quartets/s; the product's device time for the same J/K (Schwarz
threshold 0, and the workload's own threshold); and max |dJ|, |dK| between the two
when every unit ran.
"""
import argparse
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="h2o8_sto3g")
    ap.add_argument("--max-unit-gb", type=float, default=4.0)
    args = ap.parse_args()
    lai = importlib.import_module("libaccint-public_b200")
    w = lai.workloads.make(args.workload)
    rb = oracle.RefGpuBasis(w.basis)
    cap = args.max_unit_gb * 1e9 / 8
    units = [u for u in range(rb.nunits) if rb.unit_size(u)[1] <= cap]
    full = len(units) == rb.nunits

    # warm-up: Boys table, local-memory reservation, module load
    rb.jk(w.D, units[0], units[0] + 1)
    if full:
        Jr, Kr, ref_ms, ref_q = rb.jk(w.D)
    else:
        ref_ms, ref_q = 0.0, 0
        for u in units:
            _, _, ms, q = rb.jk(w.D, u, u + 1)
            ref_ms += ms
            ref_q += q

    out = {"workload": args.workload, "nbf": w.nbf,
           "reference_gpu": {"device_ms": ref_ms, "shell_quartets": ref_q,
                             "shell_quartets_per_s": ref_q / (ref_ms * 1e-3) if ref_ms > 0 else None,
                             "units_run": len(units), "units_total": rb.nunits,
                             "route": "every ordered ShellSet 4-tuple, full product, integrals "
                                      "materialized, plain FP64-atomic digestion"}}
    for key, thr in (("ours_threshold0", 0.0), ("ours_default", w.thr)):
        eng = lai.Engine(w.basis, threshold=thr)
        eng.jk(w.D)
        J, K, rep = eng.jk(w.D)
        out[key] = {"device_ms": rep.seconds_device * 1e3, "canonical_quartets": rep.quartets_fp64,
                    "schwarz": thr}
        if full:
            out[key]["max_abs_dJ_vs_reference_gpu"] = float(np.max(np.abs(J - Jr)))
            out[key]["max_abs_dK_vs_reference_gpu"] = float(np.max(np.abs(K - Kr)))
        if full and ref_ms > 0:
            out[key]["speedup_vs_reference_gpu"] = ref_ms / (rep.seconds_device * 1e3)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
