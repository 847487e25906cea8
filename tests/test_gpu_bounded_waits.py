"""The bounded device waits expire, report VSDMO_E_TIMEOUT, and leave the handle usable.

The test-only entry point vsdmo_debug_set_wait_limit_ns lowers the limit of the waits that
report an expiry: the colour-class waits of the batched persistent iteration, the stage waits
of the tensor-core GEMM and the weight / MMA waits of the proposal inference. A limit of 0 makes
the GEMM and inference waits expire at once and a batch colour wait as soon as it is entered;
nothing faults and nothing spins: the kernel records the expiry, lets its copies and MMAs in
flight land (those drains keep the 1 s limit), releases its tensor memory and returns. Each test
forces an expiry, checks the status, restores the default and runs the same handle normally.
"""
import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu
TRI = 0
E_TIMEOUT = 6


@pytest.fixture
def wait_limit(vsdmo):
    yield vsdmo.debug_set_wait_limit_ns
    vsdmo.debug_set_wait_limit_ns(-1)


def test_wait_limit_argument_checks(vsdmo, wait_limit):
    with pytest.raises(vsdmo.VSDMOError) as e:
        wait_limit(2_000_000_000)   # only lowering is allowed
    assert e.value.status == 1
    wait_limit(1_000_000_000)
    wait_limit(-1)


def test_batch_colour_wait_expires_then_recovers(vsdmo, wait_limit):
    # one mesh of 40,000 vertices: its colour-1 items are taken while colour-0 items are still
    # being searched, so their waits are entered
    xyz, el = G.tri_grid(200, seed=5, jitter=0.4)
    b = vsdmo.BatchDMO([(TRI, xyz, el)])
    b.set_config([8], [3], [32])
    x0 = b.positions()
    wait_limit(0)
    with pytest.raises(vsdmo.VSDMOError) as e:
        b.iterate(1)
    assert e.value.status == E_TIMEOUT
    wait_limit(-1)
    x1 = b.positions()
    assert np.all(np.isfinite(x1))
    moved = np.any(x1 != x0, axis=1)
    # the expired items were skipped: part of the mesh moved, not all of what a full pass moves
    b.iterate(1)
    x2 = b.positions()
    mn, mean, below = b.stats(2)
    assert below[0] == 0
    mn1, _, _ = b.stats(1)
    assert mn[0] >= mn1[0] - 1e-6
    # the same pass from the same positions on a fresh handle gives the same positions
    ref = vsdmo.BatchDMO([(TRI, xyz, el)])
    ref.set_config([8], [3], [32])
    ref.set_positions(x1)
    ref.iterate(1)
    assert np.array_equal(ref.positions(), x2)
    full = vsdmo.BatchDMO([(TRI, xyz, el)])
    full.set_config([8], [3], [32])
    full.iterate(1)
    assert int(moved.sum()) < int(np.any(full.positions() != x0, axis=1).sum())


def test_gemm_stage_wait_expires_then_recovers(vsdmo, wait_limit):
    # K = 512: 16 chunks through the 4-stage ring, so both kinds of stage wait are on the path
    r = np.random.default_rng(0)
    A = r.standard_normal((300, 512)).astype(np.float32)
    B = r.standard_normal((64, 512)).astype(np.float32)
    wait_limit(0)
    with pytest.raises(vsdmo.VSDMOError) as e:
        vsdmo.debug_gemm_bf16(A, B)
    assert e.value.status == E_TIMEOUT
    wait_limit(-1)
    D = vsdmo.debug_gemm_bf16(A, B)

    def bf16(x):
        u = x.view(np.uint32).astype(np.uint64)
        u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
        return u.astype(np.uint32).view(np.float32)

    ref = bf16(A).astype(np.float64) @ bf16(B).astype(np.float64).T
    assert np.abs(D - ref).max() < 1e-3 * np.abs(ref).max()


def test_inference_wait_expires_then_recovers(vsdmo, wait_limit):
    xyz, tets = G.tet_cube(12, seed=2)
    mesh = vsdmo.DMOMeshTet(xyz, tets)
    opt = vsdmo.DMOTetClass(mesh, n_iter=4)
    model = vsdmo.ProposalModel(seed=4)
    opt.set_model(model, 4, 2, 0.05)
    opt.iterate(1)
    wait_limit(0)
    with pytest.raises(vsdmo.VSDMOError) as e:
        opt.iterate(1)
    assert e.value.status == E_TIMEOUT
    wait_limit(-1)
    assert np.all(np.isfinite(mesh.positions()))
    opt.iterate(2)
    mn, _ = opt.history()
    assert len(mn) == 5
    assert np.all(np.diff(mn) >= -1e-6)
    # the network runs again: its proposals equal those of the same model on a fresh handle
    # from the same positions
    y = opt.proposals(0)
    mesh2 = vsdmo.DMOMeshTet(mesh.positions(original_order=True), tets)
    opt2 = vsdmo.DMOTetClass(mesh2, n_iter=1)
    opt2.set_model(model, 4, 2, 0.05)
    y2 = opt2.proposals(0)
    assert np.all(np.isfinite(y)) and np.array_equal(y, y2)
