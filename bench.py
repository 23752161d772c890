#!/usr/bin/env python
"""J+K build benchmark: (H2O)64 / cc-pVDZ, plain FP64, Schwarz 1e-12, on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full Coulomb + exchange build (every canonical shell quartet that
passes Schwarz 1e-12, 6.38e9 quartets) from a density already in HBM.  The
metric is canonical shell quartets per second (whole job); ``jk_build_s`` is the
matching J+K build time.  The set-up (outside the timed region) creates the
engine and runs the project's launch autotuner (lai_engine_autotune, about a
minute on this workload; ``--no-autotune`` keeps the built-in heuristics).
N > 1 (one process per GPU under torchrun): every rank
computes an equal slice of every quartet block and one NCCL all-reduce sums J
and K (strong scaling, total work fixed).

``--workload rhf_<system>`` (e.g. rhf_h2o16_ccpvdz) times a whole device-resident
RHF calculation instead (one-electron integrals, the J/K build of every iteration,
DIIS and diagonalization); its metric is seconds per converged SCF.

``--workload df_<system>`` (e.g. df_h2o16_ccpvdz) times density-fitted J+K builds
(auxiliary basis: the reference's built-in cc-pVDZ-RI) after the one-time metric and
three-centre set-up; its metric is seconds per J+K build.

``--impl reference`` times the reference's own CPU implementation (the
unmodified LibAccInt sources compiled into oracle/_ref: compute_2e_shell_quartet
+ FockBuilder::accumulate_symmetric, OpenMP over all host cores) on a seeded
uniform sample of the same canonical quartets, each step a bounded sample.
"""
import argparse
import datetime
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "h2o64_ccpvdz"
METRIC = "jk_quartets_per_s"
UNIT = "quartets/s"

SYSTEMS = {
    "h2o64_ccpvdz": "(H2O)64 4x4x4 grid, cc-pVDZ (Cartesian)",
    "h2o16_ccpvdz": "(H2O)16 2x2x4 grid, cc-pVDZ (Cartesian)",
    "h2o8_sto3g": "(H2O)8 2x2x2 grid, built-in STO-3G",
    "c12h26_ccpvtz": "all-trans C12H26, cc-pVTZ (Cartesian, s..f)",
    "c12h26_ccpvqz": "all-trans C12H26, cc-pVQZ (Cartesian, s..g)",
}

# DRAM bytes (read + write) per launch of a class kernel, averaged over the launches of
# one timed step in a one-pass ncu capture (dram__bytes_read.sum + dram__bytes_write.sum);
# the capture and its command are summarised under profiles/.
TRAFFIC_PER_LAUNCH = {
    ("h2o64_ccpvdz", "(ps|ss)"): 25.50e6,  # profiles/eri_small_psss_h2o64_dram.txt
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="target CPU time of the reference sample (per step for --impl reference)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations (0, 2, 3, 4) timed after the headline workload")
    ap.add_argument("--no-autotune", action="store_true",
                    help="J/K workloads: skip lai_engine_autotune in the set-up (built-in launch heuristics)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ----------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(device_index)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# reference CPU path (oracle/_ref) on a uniform sample of the canonical quartets
# ----------------------------------------------------------------------------
def reference_sampler(w):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if oracle.reference() is None:
        return None
    R = oracle.RefBasis(w.basis)
    Q = R.schwarz_parallel(0)
    cq = oracle.CanonicalQuartets(Q, w.thr)
    return R, cq


def time_reference(R, cq, D, target_s, seed, nthreads=0):
    """quartets/s of the reference CPU path on a uniform sample sized to ~target_s
    (nthreads 0 = all host cores)."""
    n = 4000 if nthreads != 1 else 1000
    t = R.time_quartets(D, cq.sample(n, seed), nthreads)[0]
    rate = n / max(t, 1e-6)
    n = int(min(max(rate * target_s, 1000), 5e7))
    t = R.time_quartets(D, cq.sample(n, seed + 1), nthreads)[0]
    return n / t, n, t


def jk_config(args, w, total_q, ws, **extra):
    """The config block both arms print (identically) for a single-system J/K workload."""
    cfg = {"workload": args.workload, "system": SYSTEMS.get(args.workload, args.workload),
           "nbf": w.nbf, "shells": w.basis.n_shells, "quartets": int(total_q), "schwarz": w.thr,
           "nocc": w.nocc, "parallelism": f"quartet shards x{ws}" + (" + NCCL all-reduce" if ws > 1 else ""),
           "l2": "GPU arm: L2 flushed (256 MB write) between timed steps"}
    cfg.update(extra)
    return cfg


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    if args.workload.startswith(("rhf_", "df_")) or args.workload == "clusters256":
        print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the J/K build of a "
                          "single system; use --workload h2o64_ccpvdz (default)"}))
        return 0
    lai = importlib.import_module("libaccint-public_b200")
    w = lai.workloads.make(args.workload)
    s = reference_sampler(w)
    if s is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_oracle.so not built"}))
        return 0
    R, cq = s
    cores = host_cores()
    # every step is one fixed-size sample of the canonical quartets, sized in the
    # warm-up to about step_target seconds on all host cores
    step_target = max(2.0, args.cpu_seconds / 2)
    rate0, _, _ = time_reference(R, cq, w.D, step_target / 4, 1000)
    n_step = int(min(max(rate0 * step_target, 1000), 5e7))
    for i in range(args.warmup):
        R.time_quartets(w.D, cq.sample(max(1000, n_step // 4), 1100 + i), 0)
    walls, kern = [], []
    for i in range(args.steps):
        smp = cq.sample(n_step, 2000 + 17 * i)
        t0 = time.perf_counter()
        kern.append(R.time_quartets(w.D, smp, 0)[0])
        walls.append(time.perf_counter() - t0)
    value = n_step * args.steps / sum(kern)
    sample = (f"{n_step} canonical quartets per step drawn uniformly (seeded) from the {cq.total} of "
              f"{args.workload}; compute_2e_shell_quartet + accumulate_symmetric, OpenMP {cores} threads")
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(walls), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": jk_config(args, w, cq.total, ws),
        "schedule": "reference CPU path (OpenMP, all host cores)",
        "quartets_per_step": n_step,
        "jk_build_s": cq.total / value, "jk_build_s_kind": "extrapolated from the sample",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


# ----------------------------------------------------------------------------
# batched workload: 256 independent water clusters in one batched engine
# ----------------------------------------------------------------------------
def run_batched(args):
    """Every shell-quartet class of all clusters as one persistent launch (batched
    engine), plain FP64 and mixed precision (FP32 below Q_ij Q_kl max|D| = 1e-7)."""
    import torch
    import torch.distributed as dist

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    lai = importlib.import_module("libaccint-public_b200")
    cl = lai.workloads.clusters(256)
    t0 = time.perf_counter()
    eng = lai.BatchedEngine([w.basis for w in cl], device=local)
    setup_s = time.perf_counter() - t0
    off, nbfs = eng.layout()
    dev = torch.device("cuda", local)
    Dh = eng.pack([w.D for w in cl])
    D = torch.from_numpy(Dh).to(dev)
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream()  # graph capture needs a stream other than the legacy default
    torch.cuda.set_stream(stream)
    shard = (rank, ws)
    cut = 1e-7

    def step(fp32_cut):
        # one CUDA graph per precision setting: captured at the first warm-up step
        rep = eng.jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), stream=stream.cuda_stream,
                            fp32_cut=fp32_cut, shard=shard, graph=True)
        if ws > 1:
            dist.all_reduce(J)
            dist.all_reduce(K)
        return rep

    def timed(fp32_cut):
        for _ in range(args.warmup):
            step(fp32_cut)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        reps = []
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(stream)
            reps.append(step(fp32_cut))
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        tot = torch.tensor([sum(a.elapsed_time(b) for a, b in ev)], dtype=torch.float64, device=dev)
        if ws > 1:
            dist.all_reduce(tot, op=dist.ReduceOp.MAX)
        return tot.item() / args.steps, reps[-1]

    clocks = ClockSampler(local)
    ms64, rep64 = timed(0.0)
    J64, K64 = eng.unpack(J.cpu().numpy()), eng.unpack(K.cpu().numpy())
    ms32, rep32 = timed(cut)
    clk = clocks.stop()
    J32, K32 = eng.unpack(J.cpu().numpy()), eng.unpack(K.cpu().numpy())
    nq = rep64.quartets_fp64 + rep64.quartets_fp32
    if ws > 1:
        t = torch.tensor([nq], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        nq = int(t.item())
    dE = [lai.molecules.energy(w.D, a, b) - lai.molecules.energy(w.D, c, d)
          for w, a, b, c, d in zip(cl, J32, K32, J64, K64)]
    # end to end through the host entry point (pinned host buffers)
    e2e_ms = []
    if ws == 1:
        Jh = np.empty_like(Dh)
        Kh = np.empty_like(Dh)
        Dp = torch.from_numpy(Dh).pin_memory()
        Jp = torch.from_numpy(Jh).pin_memory()
        Kp = torch.from_numpy(Kh).pin_memory()
        opts = eng._opts(cut, False, (0, 1), False)
        L = lai.lib()
        import ctypes
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            rep = lai._lib.JKReport()
            lai._lib.check(L.lai_jk_build_batched(eng._h, ctypes.c_void_p(Dp.data_ptr()),
                                                  ctypes.c_void_p(Jp.data_ptr()), ctypes.c_void_p(Kp.data_ptr()),
                                                  ctypes.byref(opts), ctypes.byref(rep)))
            e2e_ms.append((time.perf_counter() - t1) * 1e3)
    if rank == 0:
        n_el = int(off[-1])
        out = {
            "metric": METRIC, "value": nq / (ms32 * 1e-3), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
            "config": {"workload": "clusters256", "system": "256 water clusters, U{1..12} waters (seeded), cc-pVDZ",
                       "clusters": len(cl), "nbf_total": int(nbfs.sum()), "quartets": nq, "schwarz": 1e-12,
                       "fp32_cut": cut, "launch": "one persistent launch per shell-quartet class for all "
                                                  "clusters, the whole build replayed as one CUDA graph",
                       "parallelism": f"quartet shards x{ws}",
                       "l2": "flushed (256 MB write) between timed steps"},
            "jk_build_s": ms32 * 1e-3,
            "fp64": {"value": nq / (ms64 * 1e-3), "ms_per_step": ms64},
            "mixed_speedup_vs_fp64": ms64 / ms32,
            "quartets_fp32_fraction": rep32.quartets_fp32 / max(1, rep32.quartets_fp32 + rep32.quartets_fp64),
            "per_cluster_max_abs_dE": float(np.max(np.abs(dE))),
            "clocks": clk, "gpu_launches": rep32.kernel_launches, "setup_s": setup_s,
        }
        if e2e_ms:
            out["e2e"] = {"value": nq / (statistics.mean(e2e_ms) * 1e-3), "unit": UNIT,
                          "h2d_bytes_per_step": 8 * n_el, "d2h_bytes_per_step": 16 * n_el,
                          "ms_per_step": statistics.mean(e2e_ms)}
        print(json.dumps(out))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------
def run_rhf(args):
    """Whole RHF calculations (1 GPU; rank 0 only under torchrun): the device
    driver of libaccint-public_b200/scf.py from the core-Hamiltonian guess to
    convergence (|dE| < 1e-12, max |dD| < 1e-10)."""
    import torch
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    lai = importlib.import_module("libaccint-public_b200")
    name = args.workload[len("rhf_"):]
    w = lai.workloads.make(name)
    rhf = lai.scf.RHF(w.basis, threshold=w.thr, device=local)
    for _ in range(args.warmup):
        rhf.run()
    clk = ClockSampler(local)
    runs = [rhf.run() for _ in range(args.steps)]
    clk = clk.stop()
    dev_s = [(r.one_e_ms + sum(r.iter_ms) + r.jk_ms[-1]) * 1e-3 for r in runs]
    jk_s = [sum(r.jk_ms) * 1e-3 for r in runs]
    r0 = runs[-1]
    out = {
        "metric": "rhf_seconds", "value": statistics.mean(dev_s), "unit": "s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(dev_s),
        "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "system": SYSTEMS.get(name, name), "nbf": w.nbf,
                   "electrons": rhf.n_electrons, "schwarz": w.thr,
                   "convergence": "|dE| < 1e-12 and max |dD| < 1e-10", "diis": 6,
                   "l2": "inputs larger than L2 for the J/K build (pair data, D/J/K scattered)"},
        "energy": r0.total_energy, "iterations": r0.iterations, "converged": r0.converged,
        "jk_share": statistics.mean(j / d for j, d in zip(jk_s, dev_s)),
        "jk_ms_per_build": statistics.mean(jk_s) * 1e3 / (r0.iterations + 1),
        "one_electron_ms": r0.one_e_ms,
        "clocks": clk,
    }
    print(json.dumps(out))
    return 0


def run_df(args):
    """Density-fitted J+K builds (1 GPU; rank 0 only under torchrun)."""
    import torch
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    lai = importlib.import_module("libaccint-public_b200")
    name = args.workload[len("df_"):]
    w = lai.workloads.make(name)
    aux = lai.BasisSet.from_atoms(w.Z, w.xyz, "cc-pvdz-ri")
    eng = lai.Engine(w.basis, threshold=w.thr, device=local)
    dev = torch.device("cuda", local)
    D = torch.from_numpy(w.D).to(dev)
    # the first set-up also initializes cuSOLVER/cuBLAS; the second one is timed
    lai.df.DFFockBuilder(eng, aux).initialize()
    df = lai.df.DFFockBuilder(eng, aux)
    df.set_density(D)
    df.initialize()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    s = torch.cuda.current_stream()
    # the occupied orbitals of the synthetic density (D = C C^T, rank nocc), as an
    # SCF step hands them over; factored once on the host, outside the timing
    lam, U = np.linalg.eigh(w.D)
    C = torch.from_numpy(U[:, -w.nocc:] * np.sqrt(np.maximum(lam[-w.nocc:], 0.0))).to(dev)

    def step(orbitals):
        # one SCF step's J and K: a new density each time (its factors are not reused)
        if orbitals:
            df.set_orbitals(C, 1.0)
        else:
            df.set_density(D)
        return df.compute_coulomb(), df.compute_exchange()

    def timed(orbitals, n):
        ms = []
        for _ in range(n):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            JK = step(orbitals)
            b.record(s)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        return ms, JK

    for _ in range(args.warmup):
        step(True)
        step(False)
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    ms, (J, K) = timed(True, args.steps)
    ms_d, _ = timed(False, args.steps)
    clk = clk.stop()
    E = lai.molecules.energy(w.D, J.cpu().numpy(), K.cpu().numpy())
    # the exact four-centre build of the same density, for the fitting error and the time
    J4 = torch.empty_like(D)
    K4 = torch.empty_like(D)
    eng.jk_device(D.data_ptr(), J4.data_ptr(), K4.data_ptr(), stream=s.cuda_stream)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    eng.jk_device(D.data_ptr(), J4.data_ptr(), K4.data_ptr(), stream=s.cuda_stream)
    b.record(s)
    torch.cuda.synchronize()
    E4 = lai.molecules.energy(w.D, J4.cpu().numpy(), K4.cpu().numpy())
    out = {
        "metric": "df_jk_seconds", "value": statistics.mean(ms) * 1e-3, "unit": "s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(ms),
        "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "system": SYSTEMS.get(name, name), "nbf": w.nbf,
                   "aux": "cc-pVDZ-RI (built-in set of the reference)", "naux": aux.nbf,
                   "l2": "flushed (256 MB write) between timed steps"},
        "step": "set_orbitals(C_occ) + compute_coulomb + compute_exchange (a new density each step)",
        "density_path_ms": statistics.mean(ms_d),
        "density_path": "set_density(D) + J + K: D factored by one eigendecomposition per step",
        "setup_ms": df.init_ms, "energy": E, "energy_four_center": E4, "fitting_error": E - E4,
        "four_center_jk_ms": a.elapsed_time(b),
        "clocks": clk,
    }
    print(json.dumps(out))
    return 0


MIXED_CUT = 1e-7  # FP32 for quartets with Q_ij Q_kl max|D| below this
MIXED_FAST_CUT, MIXED_FAST_REL = 1e-5, 1e-6  # lai_jk_opts.fp32_cut, fp32_prim_rel


def mixed_leg(eng, D, J64, K64, flush, stream, steps, fp64_ms, cut=MIXED_CUT, prim_rel=0.0):
    """The same build in mixed precision (FP32 below Q_ij Q_kl max|D| = cut), outside
    the timed region: device ms per build (CUDA events on the launching stream, L2
    flushed before each build, as in the timed FP64 steps), the FP32 share, and the
    errors of J, K and E = tr(DJ)/2 - tr(DK)/4 against the FP64 J64/K64 of the same
    density.  The engine reads max|D| once per mixed build (one stream
    synchronisation), and that is inside the timed interval."""
    import torch
    Jm = torch.empty_like(J64)
    Km = torch.empty_like(K64)
    s = stream.cuda_stream
    rep = eng.jk_device(D.data_ptr(), Jm.data_ptr(), Km.data_ptr(), stream=s, fp32_cut=cut,
                        fp32_prim_rel=prim_rel)  # warm-up
    ms = []
    for _ in range(steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rep = eng.jk_device(D.data_ptr(), Jm.data_ptr(), Km.data_ptr(), stream=s, fp32_cut=cut,
                            fp32_prim_rel=prim_rel)
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))

    # dE = tr(D dJ)/2 - tr(D dK)/4 from the differences themselves: differencing two
    # energies of ~4.5e3 Eh would bottom out at their rounding (~1e-12 Eh)
    dE = float(0.5 * torch.sum(D * (Jm - J64)).item() - 0.25 * torch.sum(D * (Km - K64)).item())
    m = sum(ms) / len(ms)
    n32, n64 = int(rep.quartets_fp32), int(rep.quartets_fp64)
    return {"fp32_cut": cut, "fp32_prim_rel": prim_rel, "ms_per_build": m, "speedup_vs_fp64": fp64_ms / m,
            "quartets_fp32": n32, "quartets_fp64": n64, "fp32_fraction": n32 / max(1, n32 + n64),
            "max_abs_dJ": float(torch.max(torch.abs(Jm - J64)).item()),
            "max_abs_dK": float(torch.max(torch.abs(Km - K64)).item()),
            "abs_dE": abs(dE), "dE": dE,
            "bar": "|dE| < 1e-8 Eh against the FP64 build"}



def _device_ms(fn, flush, stream, steps):
    """Mean device time (ms) of fn() over `steps` calls after one warm-up call:
    CUDA events on `stream`, L2 flushed before each call (outside the events)."""
    import torch
    fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    return statistics.mean(ms)


def side_configs(lai, dev, flush, stream, steps, cpu_baseline=True):
    """The other configurations of the benchmark set, each timed once in the default
    run (device time per build, L2 flushed; one GPU): config 0 against the reference's
    own CPU FockBuilder build in full, config 2 (C12H26/cc-pVTZ) plain FP64 and mixed,
    config 3 (256 clusters, batched engine, CUDA graph) plain FP64 and mixed, config 4
    (the (H2O)16 nuclear gradient)."""
    import ctypes
    import torch
    s = stream.cuda_stream
    out = {}

    def dev_mats(n):
        return (torch.empty((n, n), dtype=torch.float64, device=dev),
                torch.empty((n, n), dtype=torch.float64, device=dev))

    # config 0: (H2O)8 / STO-3G, plain FP64
    w = lai.workloads.make("h2o8_sto3g")
    eng = lai.Engine(w.basis, threshold=w.thr, device=dev.index)
    D = torch.from_numpy(w.D).to(dev)
    J, K = dev_mats(w.nbf)
    ms = _device_ms(lambda: eng.jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), stream=s), flush, stream, steps)
    nq = eng.quartet_count()
    c0 = {"system": SYSTEMS["h2o8_sto3g"], "nbf": w.nbf, "quartets": nq, "schwarz": w.thr, "dtype": "f64",
          "ms_per_build": ms, "quartets_per_s": nq / (ms * 1e-3)}
    if cpu_baseline:
        # the reference's own CPU path in full: Engine::compute(coulomb, FockBuilder),
        # N^4 without screening, OpenMP on all host cores (oracle/_ref)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        if oracle.reference() is not None:
            R = oracle.RefBasis(builtin_sto3g=(w.Z, w.xyz))
            Jr, Kr, t = R.jk_full(w.D, 0)
            c0["cpu_baseline"] = {"kind": "reference", "cores": host_cores(), "full_build_s": t,
                                  "sample": "the whole build: Engine::compute(coulomb, FockBuilder), full N^4",
                                  "speedup_vs_reference_cpu": t / (ms * 1e-3),
                                  "max_abs_dJ": float(np.max(np.abs(J.cpu().numpy() - Jr))),
                                  "max_abs_dK": float(np.max(np.abs(K.cpu().numpy() - Kr)))}
    out["cfg0_h2o8_sto3g"] = c0
    del eng

    # config 2: C12H26 / cc-pVTZ, plain FP64 and mixed (FP32 below Q_ij Q_kl max|D| = 1e-7)
    w = lai.workloads.make("c12h26_ccpvtz")
    eng = lai.Engine(w.basis, threshold=w.thr, device=dev.index)
    D = torch.from_numpy(w.D).to(dev)
    J, K = dev_mats(w.nbf)
    J2, K2 = dev_mats(w.nbf)
    ms64 = _device_ms(lambda: eng.jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), stream=s), flush, stream, steps)
    rep = [None]

    def mixed():
        rep[0] = eng.jk_device(D.data_ptr(), J2.data_ptr(), K2.data_ptr(), stream=s, fp32_cut=MIXED_CUT)
    ms32 = _device_ms(mixed, flush, stream, steps)
    dE = float(0.5 * torch.sum(D * (J2 - J)).item() - 0.25 * torch.sum(D * (K2 - K)).item())
    nq = eng.quartet_count()
    out["cfg2_c12h26_ccpvtz"] = {
        "system": SYSTEMS["c12h26_ccpvtz"], "nbf": w.nbf, "quartets": nq, "fp64_ms_per_build": ms64,
        "fp64_quartets_per_s": nq / (ms64 * 1e-3), "mixed_ms_per_build": ms32, "fp32_cut": MIXED_CUT,
        "mixed_speedup_vs_fp64": ms64 / ms32,
        "fp32_fraction": rep[0].quartets_fp32 / max(1, rep[0].quartets_fp32 + rep[0].quartets_fp64),
        "abs_dE": abs(dE), "max_abs_dJ": float(torch.max(torch.abs(J2 - J)).item()),
        "max_abs_dK": float(torch.max(torch.abs(K2 - K)).item())}
    del eng

    # config 3: 256 clusters in one batched engine, every class one launch for all
    # clusters, the build replayed as a CUDA graph; plain FP64 and mixed
    cl = lai.workloads.clusters(256)
    eng = lai.BatchedEngine([c.basis for c in cl], device=dev.index)
    Dp = torch.from_numpy(eng.pack([c.D for c in cl])).to(dev)
    Jp, Kp = torch.empty_like(Dp), torch.empty_like(Dp)
    Jq, Kq = torch.empty_like(Dp), torch.empty_like(Dp)
    reps = {}
    gs = torch.cuda.Stream(device=dev)  # graph capture needs a stream other than the legacy default
    torch.cuda.synchronize()

    def batched(cut, Jo, Ko):
        reps[cut] = eng.jk_device(Dp.data_ptr(), Jo.data_ptr(), Ko.data_ptr(), stream=gs.cuda_stream,
                                  fp32_cut=cut, graph=True)
    ms64 = _device_ms(lambda: batched(0.0, Jp, Kp), flush, gs, steps)
    ms32 = _device_ms(lambda: batched(MIXED_CUT, Jq, Kq), flush, gs, steps)
    off, _ = eng.layout()
    Dh, dJ, dK = Dp.cpu().numpy(), (Jq - Jp).cpu().numpy(), (Kq - Kp).cpu().numpy()
    dE = [0.5 * float(np.dot(Dh[a:b], dJ[a:b])) - 0.25 * float(np.dot(Dh[a:b], dK[a:b]))
          for a, b in zip(off[:-1], off[1:])]
    r = reps[MIXED_CUT]
    nq = r.quartets_fp32 + r.quartets_fp64
    out["cfg3_clusters256"] = {
        "system": "256 water clusters, U{1..12} waters (seeded), cc-pVDZ", "quartets": int(nq),
        "fp64_ms_per_build": ms64, "mixed_ms_per_build": ms32, "fp32_cut": MIXED_CUT,
        "mixed_speedup_vs_fp64": ms64 / ms32, "mixed_quartets_per_s": nq / (ms32 * 1e-3),
        "fp32_fraction": r.quartets_fp32 / max(1, nq), "per_cluster_max_abs_dE": float(np.max(np.abs(dE)))}
    del eng

    # config 4: (H2O)16 / cc-pVDZ nuclear gradient of E = tr(DJ)/2 - tr(DK)/4 (FP64)
    w = lai.workloads.make("h2o16_ccpvdz")
    eng = lai.Engine(w.basis, threshold=w.thr, device=dev.index)
    D = torch.from_numpy(w.D).to(dev)
    G = torch.empty((eng.natom(), 3), dtype=torch.float64, device=dev)
    J, K = dev_mats(w.nbf)
    lib = lai.lib()

    def grad():
        lai._lib.check(lib.lai_jk_gradient_device(eng._h, ctypes.c_void_p(D.data_ptr()),
                                                  ctypes.c_void_p(G.data_ptr()), ctypes.c_void_p(s)))
    msg = _device_ms(grad, flush, stream, 1)
    msj = _device_ms(lambda: eng.jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), stream=s), flush, stream, steps)
    out["cfg4_h2o16_gradient"] = {
        "system": SYSTEMS["h2o16_ccpvdz"], "natom": int(G.shape[0]), "gradient_ms": msg, "jk_build_ms": msj,
        "translational_invariance": float(torch.max(torch.abs(G.sum(dim=0))).item())}
    return out

def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "clusters256":
        return run_batched(args)
    if args.workload.startswith("rhf_"):
        return run_rhf(args)
    if args.workload.startswith("df_"):
        return run_df(args)
    import torch
    import torch.distributed as dist

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    lai = importlib.import_module("libaccint-public_b200")
    w = lai.workloads.make(args.workload)
    n = w.nbf
    t0 = time.perf_counter()
    eng = lai.Engine(w.basis, threshold=w.thr, device=local)
    setup_s = time.perf_counter() - t0
    total_q = eng.quartet_count()
    shard = (rank, ws)

    dev = torch.device("cuda", local)
    D = torch.from_numpy(w.D).to(dev)
    J = torch.empty((n, n), dtype=torch.float64, device=dev)
    K = torch.empty((n, n), dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
    stream = torch.cuda.current_stream()

    # set-up, outside the timed region: the project's autotuner times each
    # class-pair launch under its kernel families and launch shapes on this
    # density and keeps the fastest (every rank tunes its own engine)
    tune = None
    if not args.no_autotune:
        t0 = time.perf_counter()
        tb, ta = eng.autotune(D.data_ptr(), stream=stream.cuda_stream)
        torch.cuda.synchronize()
        tune = {"seconds": time.perf_counter() - t0, "launch_ms_before": tb, "launch_ms_after": ta}

    def step(profile=False):
        rep = eng.jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), stream=stream.cuda_stream,
                            shard=shard, profile=profile)
        if ws > 1:
            dist.all_reduce(J)
            dist.all_reduce(K)
        return rep

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- timed region: K steps, L2 flushed between steps (outside the events) ----
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    launches = 0
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record(stream)
        rep = step()
        ev[i][1].record(stream)
        launches += rep.kernel_launches
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    tot = torch.tensor([sum(step_ms)], dtype=torch.float64, device=dev)
    if ws > 1:
        dist.all_reduce(tot, op=dist.ReduceOp.MAX)
    ms_per_step = tot.item() / args.steps
    value = total_q / (ms_per_step * 1e-3)
    E = lai.molecules.energy(w.D, J.cpu().numpy(), K.cpu().numpy())

    # ---- end to end through the public C ABI with host buffers ----
    pin = lambda a: torch.from_numpy(a).pin_memory()  # noqa: E731
    D_h = pin(w.D)
    J_h = torch.empty((n, n), dtype=torch.float64).pin_memory()
    K_h = torch.empty((n, n), dtype=torch.float64).pin_memory()
    e2e_ms = []
    for i in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        t = time.perf_counter()
        if ws == 1:
            eng.jk(D_h.numpy(), out=(J_h.numpy(), K_h.numpy()))
        else:
            Dd = D_h.to(dev, non_blocking=True)
            eng.jk_device(Dd.data_ptr(), J.data_ptr(), K.data_ptr(), stream=stream.cuda_stream, shard=shard)
            dist.all_reduce(J)
            dist.all_reduce(K)
            J_h.copy_(J, non_blocking=True)
            K_h.copy_(K, non_blocking=True)
            torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t) * 1e3)
    et = torch.tensor([sum(e2e_ms)], dtype=torch.float64, device=dev)
    if ws > 1:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    e2e_value = total_q / (et.item() / args.steps * 1e-3)
    E2 = lai.molecules.energy(w.D, J_h.numpy(), K_h.numpy())

    # ---- per-launch profile (one extra build, outside the timed region) ----
    torch.cuda.synchronize()
    step(profile=True)
    torch.cuda.synchronize()
    pr = eng.last_profile()

    # ---- mixed precision on the same density (one GPU only: no collectives) ----
    mixed = None
    if ws == 1:
        try:
            mixed = mixed_leg(eng, D, J, K, flush, stream, args.steps, ms_per_step)
            # the fastest setting measured inside the 1e-8 Eh bar on this workload:
            # more quartets in FP32 and their primitives screened relative to the quartet
            mixed["fast"] = mixed_leg(eng, D, J, K, flush, stream, args.steps, ms_per_step,
                                      cut=MIXED_FAST_CUT, prim_rel=MIXED_FAST_REL)
        except Exception as ex:  # report, do not lose the FP64 line
            mixed = {"error": f"{type(ex).__name__}: {ex}"}
    configs = None
    if ws == 1 and not args.no_configs and args.workload == WORKLOAD:
        try:
            configs = side_configs(lai, dev, flush, stream, min(args.steps, 2),
                                   cpu_baseline=not args.no_cpu_baseline)
        except Exception as ex:  # report, do not lose the headline line
            configs = {"error": f"{type(ex).__name__}: {ex}"}
    pms, pfl, pfx, pcl = pr["ms"], pr["alg_flops"], pr["alg_flops_executed"], pr["lclass"]
    peak = lai.probe_fp64_peak(local)
    roof_all = float(np.sum(pfx) / (np.sum(pms) * 1e-3) / 1e12)
    roof_all_nominal = float(np.sum(pfl) / (np.sum(pms) * 1e-3) / 1e12)
    by_class = {}
    for ms, fl, cl, nq, npq in zip(pms, pfx, pcl, pr["quartets"], pr["prim_quartets"]):
        key = "(%s%s|%s%s)" % tuple("spdfg"[x] for x in cl)
        a = by_class.setdefault(key, [0.0, 0.0, 0, 0, 0])
        a[0] += ms
        a[1] += fl
        a[2] += 1
        a[3] += int(nq)
        a[4] += int(npq)
    # dominant kernel = the class kernel with the largest share of device time
    dom_key, (dom_ms, dom_fl, dom_n, _, _) = max(by_class.items(), key=lambda kv: kv[1][0])
    dom_tf = float(dom_fl / (dom_ms * 1e-3) / 1e12)
    traffic = TRAFFIC_PER_LAUNCH.get((args.workload, dom_key))
    prim_exec = int(np.sum(pr["prim_quartets"]))

    out = None
    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            s = reference_sampler(w)
            if s is not None:
                R, cq = s
                rate, ns, ts = time_reference(R, cq, w.D, args.cpu_seconds, 7)
                cpu = {"value": rate, "unit": UNIT, "cores": host_cores(), "kind": "reference",
                       "sample": f"{ns} canonical quartets drawn uniformly (seeded) from the "
                                 f"{cq.total} of {args.workload}, {ts:.1f} s on all host cores; "
                                 f"full-build estimate {cq.total / rate:.0f} s"}
                # the serial screened-symmetric path (one thread), the best correct
                # single-core figure of the reference
                r1, n1, t1 = time_reference(R, cq, w.D, max(2.0, args.cpu_seconds / 3), 11, nthreads=1)
                cpu["value_1thread"] = r1
                cpu["sample_1thread"] = f"{n1} canonical quartets, {t1:.1f} s on one host core"
        top_cls = sorted(by_class.items(), key=lambda kv: -kv[1][0])
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": jk_config(args, w, total_q, ws),
            "schedule": "autotuned in the set-up (lai_engine_autotune)" if tune else "built-in launch heuristics",
            "jk_build_s": ms_per_step * 1e-3,
            "energy": E, "energy_e2e": E2,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * n * n,
                    "d2h_bytes_per_step": 16 * n * n, "ms_per_step": et.item() / args.steps},
            "roofline": {"bound": "fp64", "achieved": dom_tf, "peak": peak, "unit": "TFLOP/s",
                         "frac": dom_tf / peak, "traffic": traffic,
                         "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                         "kernel": "class %s kernel: %d launches, %.1f ms of the step (largest share)" % (
                             dom_key, dom_n, dom_ms),
                         "all_kernels_achieved": roof_all, "all_kernels_frac": roof_all / peak,
                         "work": "algorithmic FP64 work of the primitive quartets executed "
                                 "(those passing the primitive Schwarz cut); counting all nonzero "
                                 "primitives instead gives %.2f TFLOP/s" % roof_all_nominal,
                         "prim_quartets_executed": prim_exec,
                         "peak_source": "measured in-run: register-resident FP64 FMA loop "
                                        "(MEASURED_PEAKS.json has no FP64 entry)"},
            "classes": {"columns": ["ms", "TFLOP/s executed", "quartets", "primitive quartets executed"],
                        **{k: [round(v[0], 2), round(v[1] / (v[0] * 1e-3) / 1e12, 2), v[3], v[4]]
                           for k, v in top_cls}},
            "clocks": clk,
            "gpu_launches": launches,
            "setup_s": setup_s,
            "autotune": tune,
            "mixed": mixed,
            "configs": configs,
        }
        if cpu:
            out["cpu_baseline"] = cpu
        print(json.dumps(out))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
