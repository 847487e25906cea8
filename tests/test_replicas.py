"""The N > 1 path on CPU: two ranks over gloo (one process each, 127.0.0.1), each optimising
its own seeded replica mesh with the oracle's f32 restatement as a stand-in for the GPU step,
the barrier around the timed region, the maximum of the ranks' times and the whole-job rate
(volumesurfacediscretemeshoptimization_b200/replicas.py, as bench.py uses them over NCCL);
and the reference arm's rank rule (rank 0 alone runs)."""
import hashlib
import os
import socket
import sys
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from volumesurfacediscretemeshoptimization_b200 import meshgen as G, replicas
    r, w, _ = replicas.rank_info()
    dist = replicas.init("gloo", timeout_s=60)
    xyz, tets = G.tet_cube(5, seed=replicas.replica_seed(r))
    om = O.OracleMesh(2, xyz, tets)
    x = om.xyz
    replicas.barrier(dist)
    t0 = time.perf_counter()
    for v0, v1 in om.color_ranges():
        x = om.dmo_color_f32(x, v0, v1, nthreads=1)
    ms = (time.perf_counter() - t0) * 1e3 + 1000.0 * r     # rank 1 made the slower one, whatever the load
    replicas.barrier(dist)
    ms_max = replicas.max_over_ranks(ms, dist)
    n_inner = om.info["nV"] - om.info["nSurf"]
    rate = replicas.whole_job_rate(n_inner, ms_max, w)
    out.put((r, ms, ms_max, rate, n_inner, float(np.abs(x - om.xyz).sum()), hashlib.sha1(xyz.tobytes()).hexdigest()))
    replicas.finish(dist)


def test_two_replicas_over_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=180) for _ in range(2)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, ms0, max0, rate0, n0, moved0, x0), (r1, ms1, max1, rate1, n1, moved1, x1) = res
    # both ranks hold the slowest rank's time and the same whole-job rate
    assert max0 == max1 == max(ms0, ms1) and ms1 > ms0
    assert rate0 == rate1 == pytest.approx(2 * n0 / (max0 / 1e3))
    # each rank optimised its own mesh: different jitter, both moved
    assert n0 == n1 and x0 != x1 and moved0 > 0 and moved1 > 0


def test_single_process_needs_no_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    from volumesurfacediscretemeshoptimization_b200 import replicas
    assert replicas.rank_info() == (0, 1, 0)
    assert replicas.init("gloo") is None
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.whole_job_rate(1000, 500.0, 1) == 2000.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun every rank starts the reference arm; ranks other than 0 exit 0 at once."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        warmup, steps, gpus = 1, 1, 2
    t0 = time.perf_counter()
    assert bench.run_reference(A) == 0
    assert time.perf_counter() - t0 < 5.0
    assert capsys.readouterr().out == ""
