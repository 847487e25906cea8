"""GPU tests of the learned proposal: the tcgen05 BF16 GEMM, the network's forward pass and
gradients against the CPU oracle (oracle/mlp_oracle.py), training, training-pair collection
from plain DMO, and the learned optimiser mode (monotone, and what training gains over an
untrained network)."""
import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mo():
    from oracle import mlp_oracle
    return mlp_oracle


@pytest.mark.parametrize("M,N,K", [(128, 128, 32), (300, 16, 96), (257, 96, 256), (128, 64, 128),
                                   (1000, 128, 128), (128, 32, 4096)])
def test_tensor_core_gemm(vsdmo, mo, M, N, K):
    r = np.random.default_rng(M + N + K)
    A = r.uniform(-1, 1, size=(M, K)).astype(np.float32)
    B = r.uniform(-1, 1, size=(N, K)).astype(np.float32)
    D = vsdmo.debug_gemm_bf16(A, B)
    ref = mo.bf16(A) @ mo.bf16(B).T
    bound = (np.abs(mo.bf16(A)) @ np.abs(mo.bf16(B)).T) * 2e-6 + 1e-6   # FP32 accumulation
    assert np.all(np.abs(D - ref) <= bound), float(np.abs(D - ref).max())


def test_forward_matches_oracle(vsdmo, mo):
    m = vsdmo.ProposalModel(seed=3)
    p = m.get_params()
    r = np.random.default_rng(1)
    P = mo.unflatten(p)
    for k in ("b1", "b2", "b3"):
        P[k] = r.uniform(-0.1, 0.1, size=P[k].shape)
    P["b4"][:3] = r.uniform(-0.1, 0.1, size=3)
    p = mo.flatten(P).astype(np.float32)
    m.set_params(p)
    assert np.array_equal(m.get_params(), p)
    X = r.uniform(-1, 1, size=(300, 96)).astype(np.float32)
    Y = m.forward(X)
    Yr, _ = mo.forward(p, X)
    err = np.abs(Y - Yr).max()
    assert err <= 2e-2 * np.abs(Yr).max() + 1e-4, err


def test_gradients_match_oracle(vsdmo, mo):
    m = vsdmo.ProposalModel(seed=5)
    r = np.random.default_rng(2)
    P = mo.unflatten(m.get_params())
    for k in ("b1", "b2", "b3"):
        P[k] = r.uniform(0.0, 0.1, size=P[k].shape)
    p = mo.flatten(P).astype(np.float32)
    m.set_params(p)
    X = r.uniform(-1, 1, size=(256, 96)).astype(np.float32)
    T = r.uniform(-0.5, 0.5, size=(256, 3)).astype(np.float32)
    loss, g = m.gradients(X, T)
    loss_r, g_r = mo.loss_and_grad(p, X, T)
    assert abs(loss - loss_r) <= 1e-4 * abs(loss_r) + 1e-7
    o = 0
    for name, shape in mo.SHAPES:
        n = int(np.prod(shape))
        a, b = g[o:o + n], g_r[o:o + n]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert rel < 2e-2, (name, rel)
        o += n


def test_training_reduces_loss(vsdmo):
    r = np.random.default_rng(7)
    X = r.uniform(-1, 1, size=(8192, 96)).astype(np.float32)
    Wt = r.normal(0, 0.15, size=(96, 3))
    T = np.tanh(X @ Wt).astype(np.float32) * 0.3
    m = vsdmo.ProposalModel(seed=1)
    hist = m.train(X, T, steps=300, batch=512, lr=2e-3, seed=4)
    assert np.all(np.isfinite(hist))
    assert hist[-20:].mean() < 0.2 * hist[:5].mean(), (hist[:5].mean(), hist[-20:].mean())


def _ring_features(xyz, hf_rowptr, hf, v):
    """Network input of vertex v, restated with the same float32 operations as the kernel."""
    c0 = xyz[v]
    tri = hf.reshape(-1, 3)[hf_rowptr[v]:hf_rowptr[v + 1]]
    nb, mm = [], np.float32(0)
    for t in tri:
        for u in t:
            mm = max(mm, np.float32(np.abs(xyz[u] - c0).max()))
            if u not in nb and len(nb) < 32:
                nb.append(int(u))
    inv = np.float32(1) / mm
    f = np.zeros(96, np.float32)
    for a, u in enumerate(nb):
        f[3 * a:3 * a + 3] = (xyz[u] - c0) * inv
    return f, mm


def test_collect_pairs_first_colour_exact(vsdmo):
    import torch
    xyz, tets = G.tet_cube(9, seed=11)
    mesh = vsdmo.DMOMeshTet(xyz, tets)
    opt = vsdmo.DMOTetClass(mesh, n_iter=1)
    x_before = mesh.positions()
    cap = 4096
    f = torch.zeros(cap * 96, dtype=torch.float32, device="cuda")
    t = torch.zeros(cap * 3, dtype=torch.float32, device="cuda")
    n = opt.collect_pairs(1, f.data_ptr(), t.data_ptr(), cap)
    assert n == mesh.info["nV"] - mesh.info["nSurf"]
    F = f.cpu().numpy().reshape(cap, 96)
    Tt = t.cpu().numpy().reshape(cap, 3)
    rp, hf = mesh.array(vsdmo.A_HF_ROWPTR), mesh.array(vsdmo.A_HALFFACES)
    off = mesh.array(vsdmo.A_COL_INNER)
    x_after = mesh.positions()
    moved = 0
    for i, v in enumerate(range(off[0], off[1])):
        fr, mm = _ring_features(x_before, rp, hf, v)
        assert np.array_equal(F[i], fr), v
        tr = (x_after[v] - x_before[v]) * (np.float32(1) / mm)
        assert np.array_equal(Tt[i], tr.astype(np.float32)), v
        moved += int(np.any(tr != 0))
    assert moved > 0


def test_fused_inference_matches_gemm_path(vsdmo):
    """The fused features + network kernel of the learned search against the per-layer GEMM
    path fed with the collected FP32 features of the same vertices."""
    import torch
    xyz, tets = G.tet_cube(12, seed=2)
    mesh = vsdmo.DMOMeshTet(xyz, tets)
    opt = vsdmo.DMOTetClass(mesh, n_iter=1)
    model = vsdmo.ProposalModel(seed=4)
    r = np.random.default_rng(0)
    p = model.get_params()
    p[mlp_bias_slice()] = r.uniform(-0.05, 0.05, size=p[mlp_bias_slice()].shape)
    model.set_params(p)
    opt.set_model(model, 4, 2, 0.05)
    y_fused = opt.proposals(0)
    cap = 4096
    f = torch.zeros(cap * 96, dtype=torch.float32, device="cuda")
    t = torch.zeros(cap * 3, dtype=torch.float32, device="cuda")
    opt.set_model(None)
    opt.collect_pairs(1, f.data_ptr(), t.data_ptr(), cap)
    n = len(y_fused)
    feats = f.cpu().numpy().reshape(cap, 96)[:n]
    y_gemm = model.forward(feats)
    # same BF16 inputs and weights; accumulation order inside the tensor cores may differ
    assert np.abs(y_fused - y_gemm).max() <= 1e-3 * max(1.0, np.abs(y_gemm).max())


def mlp_bias_slice():
    from oracle import mlp_oracle as mo
    o = mo.IN * mo.HID
    return slice(o, o + mo.HID)


def _train_on_plain_pairs(vsdmo, seed, n_cells=14, iters=8, steps=400):
    import torch
    xyz, tets = G.tet_cube(n_cells, seed=seed)
    mesh = vsdmo.DMOMeshTet(xyz, tets)
    opt = vsdmo.DMOTetClass(mesh, n_iter=iters)
    cap = (mesh.info["nV"] - mesh.info["nSurf"]) * iters
    f = torch.zeros(cap * 96, dtype=torch.float32, device="cuda")
    t = torch.zeros(cap * 3, dtype=torch.float32, device="cuda")
    n = opt.collect_pairs(iters, f.data_ptr(), t.data_ptr(), cap)
    model = vsdmo.ProposalModel(seed=seed)
    hist = model.train(None, None, steps=steps, batch=1024, lr=1e-3, seed=seed,
                       device_ptrs=(f.data_ptr(), t.data_ptr()), n_rows=n)
    return model, hist


def test_learned_mode_monotone_and_gain(vsdmo):
    trained, hist = _train_on_plain_pairs(vsdmo, seed=21)
    assert hist[-20:].mean() < hist[:5].mean()
    untrained = vsdmo.ProposalModel(seed=99)
    res = {}
    for name, model in (("trained", trained), ("untrained", untrained)):
        xyz, tets = G.tet_cube(14, seed=5)
        mesh = vsdmo.DMOMeshTet(xyz, tets)
        opt = vsdmo.DMOTetClass(mesh, n_iter=6)
        q0 = opt.getQuality()
        opt.set_model(model, 4, 2, 0.012)
        opt.optimize()
        mn, mean = opt.history()
        assert np.all(np.diff(mn) >= -1e-6)          # the fallback keeps the minimum monotone
        assert mn[-1] > q0 and mean[-1] > mean[0]
        acc, fb, fb_moved, skipped = opt.learned_counters()
        assert acc + fb == 6 * (mesh.info["nV"] - mesh.info["nSurf"])
        res[name] = (acc, fb, mean[-1])
    # what training gains: more updates accepted from the cheap reduced search
    assert res["trained"][0] > 2 * res["untrained"][0] + 100, res


def test_learned_proposals_once_per_iteration(vsdmo):
    """One network launch per iteration (stale proposals for later colour classes): the
    reduced search and the fallback judge the current ring, so the minimum stays monotone."""
    trained, _ = _train_on_plain_pairs(vsdmo, seed=22)
    xyz, tets = G.tet_cube(14, seed=6)
    mesh = vsdmo.DMOMeshTet(xyz, tets)
    opt = vsdmo.DMOTetClass(mesh, n_iter=5)
    q0 = opt.getQuality()
    opt.set_model(trained, 4, 2, 0.012)
    opt.set_proposal_schedule(2)          # iterations 0, 1 per colour class, then once
    opt.optimize()
    mn, mean = opt.history()
    assert np.all(np.diff(mn) >= -1e-6)
    assert mn[-1] > q0 and mean[-1] > mean[0]
    acc, fb, _, _ = opt.learned_counters()
    assert acc + fb == 5 * (mesh.info["nV"] - mesh.info["nSurf"]) and acc > fb
    # the whole run with one launch per iteration
    opt2 = vsdmo.DMOTetClass(vsdmo.DMOMeshTet(xyz, tets), n_iter=1)
    opt2.set_model(trained, 4, 2, 0.012)
    opt2.set_proposal_schedule(0)
    opt2.iterate(1)
    assert opt2.learned_counters()[0] > 0


def test_learned_colour_launches_match_oracle(vsdmo, oracle_mod):
    """Learned mode, colour class by colour class, bitwise against the oracle's f32
    restatement (or_dmo_tet_learned_f32): the reduced 4^3 x 2 search around the network's
    proposals, then the plain search for the vertices it did not move."""
    trained, _ = _train_on_plain_pairs(vsdmo, seed=23)
    xyz, tets = G.tet_cube(10, seed=7)
    mesh = vsdmo.DMOMeshTet(xyz, tets)
    om = oracle_mod.OracleMesh(2, xyz, tets)
    assert mesh.info == om.info
    opt = vsdmo.DMOTetClass(mesh, n_iter=2)
    opt.set_model(trained, 4, 2, 0.012)
    x = mesh.positions()
    queued_total = 0
    for sweep in range(2):
        for c, (v0, v1) in enumerate(om.color_ranges()):
            Y = opt.proposals(c)
            xo, queued = om.dmo_tet_learned_f32(x, v0, v1, Y, 4, 2, 0.012)
            opt.run_color(c)
            g = mesh.positions()
            assert np.array_equal(g.view(np.uint32), xo.view(np.uint32)), (sweep, c)
            queued_total += int(queued.sum())
            x = g
    acc, fb, _, _ = opt.learned_counters()
    assert fb == queued_total and acc + fb == 2 * (mesh.info["nV"] - mesh.info["nSurf"]) and acc > fb
