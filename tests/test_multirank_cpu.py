"""The multi-GPU protocol on CPU ranks (gloo, world size 2): every rank takes its
slice of each quartet block from lai_shard_range (the partition the device build
uses for shard_index/shard_count), computes the partial J/K of its slice, and one
all-reduce sums them.  The partial J/K here come from the oracle restatement (the
ranks have no GPU); the result must equal the single-process build.  A rank that
raises makes the others fail with an error, not hang (short process-group timeout)."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _canonical_blocks(oracle, basis, thr):
    """Canonical Schwarz-screened quartets grouped by (la, lb, lc, ld) class,
    standing in for the engine's class-pair blocks."""
    Q = oracle.orc_schwarz(basis)
    ls = [s.l for s in basis.shells]
    n = len(ls)
    blocks = {}
    for i in range(n):
        for j in range(i, n):
            for k in range(i, n):
                for m in range(j if k == i else k, n):
                    if Q[i, j] * Q[k, m] >= thr:
                        blocks.setdefault((ls[i], ls[j], ls[k], ls[m]), []).append((i, j, k, m))
    return [np.array(v, dtype=np.int32) for _, v in sorted(blocks.items())]


def _rank_main(rank, world, port, result_path, fail_rank):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ctypes
    import importlib

    import torch
    import torch.distributed as dist
    import oracle

    lai = importlib.import_module("libaccint-public_b200")
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        w = lai.workloads.make("h2o2_sto3g")
        blocks = _canonical_blocks(oracle, w.basis, w.thr)
        J = np.zeros((w.nbf, w.nbf))
        K = np.zeros((w.nbf, w.nbf))
        L = lai.lib()
        for b in blocks:
            lo, hi = ctypes.c_int64(), ctypes.c_int64()
            lai._lib.check(L.lai_shard_range(len(b), rank, world, ctypes.byref(lo), ctypes.byref(hi)))
            if rank == fail_rank:
                raise RuntimeError("injected failure on this rank")
            oracle.orc_jk_list(w.basis, w.D, b[lo.value:hi.value], J, K)
        Jt = torch.from_numpy(J)
        Kt = torch.from_numpy(K)
        dist.all_reduce(Jt)
        dist.all_reduce(Kt)
        if rank == 0:
            np.savez(result_path, J=Jt.numpy(), K=Kt.numpy())
    finally:
        dist.destroy_process_group()


def _spawn(tmp_path, fail_rank=-1):
    import torch.multiprocessing as mp
    out = str(tmp_path / "jk.npz")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out, fail_rank)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    return out, codes


def test_sharded_jk_two_ranks_matches_single(tmp_path, lai, oracle):
    out, codes = _spawn(tmp_path)
    assert codes == [0, 0]
    r = np.load(out)
    w = lai.workloads.make("h2o2_sto3g")
    J0, K0, _ = oracle.orc_jk(w.basis, w.D, w.thr)
    assert np.max(np.abs(r["J"] - J0)) < 1e-12
    assert np.max(np.abs(r["K"] - K0)) < 1e-12


def test_failing_rank_is_reported_not_hung(tmp_path):
    out, codes = _spawn(tmp_path, fail_rank=1)
    assert codes[1] != 0          # the failing rank exits with an error
    assert codes[0] is not None   # and the other one ended (error or not), no hang


def test_shard_ranges_tile_every_block(lai):
    import ctypes
    L = lai.lib()
    for total in (0, 1, 7, 1000003, 6381126924):
        for count in (1, 2, 3, 8):
            got = []
            for i in range(count):
                lo, hi = ctypes.c_int64(), ctypes.c_int64()
                assert L.lai_shard_range(total, i, count, ctypes.byref(lo), ctypes.byref(hi)) == 0
                got.append((lo.value, hi.value))
            assert got[0][0] == 0 and got[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            assert max(h - l for l, h in got) - min(h - l for l, h in got) <= 1
    lo, hi = ctypes.c_int64(), ctypes.c_int64()
    assert L.lai_shard_range(10, 2, 2, ctypes.byref(lo), ctypes.byref(hi)) == -1
