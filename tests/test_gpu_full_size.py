"""The full-size benchmark workloads against the FP64 oracle (final minimum and mean within 1e-4).

tests/golden/full_size_fp64.json holds the FP64 restatement's minimum and mean element quality
after every iteration of each workload (generated by tests/golden/make_full_size.py on the CPU:
config 2 alone is about 8 CPU-minutes). The library runs the same workload on the GPU:

* config 1: 64x64 flat triangle grid, 10 iterations, boundary fixed;
* config 2: 48^3 Kuhn tet cube, 20 iterations, boundary fixed (the bench's workload);
* config 2 hex: 32^3 hex cube, 20 iterations, the reference's shape metric;
* config 3: the icosphere of level 7 and the 512 x 256 torus with the specified noise
  (tangential 0.35 l, normal N(0, 1e-3)), 15 iterations, feature vertices sliding on their
  curves (the reference's DMOTriClass / DMOQuadClass loop).

The final mean is within 1e-4 of the FP64 run on every workload, and so is the final minimum
except on config 2: there every FP32 implementation of the search drifts from the FP64
trajectory once near-tie decisions compound (the oracle's float restatement, bitwise equal to
the library, is within 1e-6 of FP64 through iteration 5, up to 3.1e-3 off at iteration 7 and
4.4e-4 below it after 20; the mean stays within 8e-6 throughout), so its minimum is held to 1e-4
through iteration 4 and to 1e-3 at the end. On config 2 the first iteration is also compared vertex by
vertex, colour by colour from the same state: positions within 1e-5 h wherever the FP64
decision margin exceeds 1e-5.
"""
import json
import os

import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "full_size_fp64.json")))
TRI, QUAD, TET, HEX = 0, 1, 2, 3


def _library_run(vsdmo, name):
    g = GOLDEN[name]
    xyz, el = eval(g["generator"], {"meshgen": G})
    if name == "config1":
        m = vsdmo.DMOMeshTri(xyz, el)
        o = vsdmo.DMOTriFlatClass(m, n_iter=g["iterations"])
    elif name == "config2":
        m = vsdmo.DMOMeshTet(xyz, el)
        o = vsdmo.DMOTetClass(m, n_iter=g["iterations"])
    elif name == "config2_hex":
        m = vsdmo.DMOMeshHex(xyz, el)
        o = vsdmo.DMOHexClass(m, n_iter=g["iterations"])
    elif name == "config3_tri":
        m = vsdmo.DMOMeshTri(xyz, el)
        o = vsdmo.DMOTriClass(m, n_iter=g["iterations"])
    else:
        m = vsdmo.DMOMeshQuad(xyz, el)
        o = vsdmo.DMOQuadClass(m, n_iter=g["iterations"])
    # feature vertices come from a 20 degree dihedral rule evaluated with acosf; on config 3 one
    # edge lies within an ulp of the threshold, where CUDA's acosf and the host's differ
    assert abs(m.info["nFeature"] - g["feature_vertices"]) <= 2
    return m, o


@pytest.mark.parametrize("name", ["config1", "config2", "config2_hex", "config3_tri", "config3_quad"])
def test_full_size_final_quality_against_fp64(vsdmo, name):
    g = GOLDEN[name]
    m, o = _library_run(vsdmo, name)
    q_min0, q_mean0 = o.quality_stats()
    assert abs(q_min0 - g["initial_min"]) < 1e-6 and abs(q_mean0 - g["initial_mean"]) < 1e-6
    o.optimize()
    mn, mean = o.history()
    assert len(mn) == g["iterations"] + 1
    dmin = np.abs(np.asarray(mn[1:]) - g["min"])
    dmean = np.abs(np.asarray(mean[1:]) - g["mean"])
    assert dmean[-1] < 1e-4, (mean[-1], g["mean"][-1], float(dmean.max()))
    assert np.all(dmean < 2e-4), float(dmean.max())
    if name == "config2":
        assert np.all(dmin[:4] < 1e-4), dmin[:4]
        assert dmin[-1] < 1e-3, (mn[-1], g["min"][-1])
    else:
        assert dmin[-1] < 1e-4, (mn[-1], g["min"][-1], float(dmin.max()))
    assert np.all(np.diff(mn) >= -1e-6)


def test_config2_first_iteration_positions_against_fp64(oracle_mod, vsdmo):
    xyz, el = G.config2()
    h = 1.0 / 48
    om = oracle_mod.OracleMesh(oracle_mod.TET, xyz, el)
    gm = vsdmo.DMOMeshTet(xyz, el)
    opt = vsdmo.DMOTetClass(gm, n_iter=1)
    x = om.xyz
    checked = total = 0
    for c, (v0, v1) in enumerate(om.color_ranges()):
        x64, margin = om.dmo_color_f64(x.astype(np.float64), v0, v1, nthreads=os.cpu_count() or 1)
        opt.run_color(c)
        g = gm.positions()
        clear = margin > 1e-5
        d = np.abs(g[v0:v1].astype(np.float64) - x64[v0:v1]).max(1)
        assert np.all(d[clear] < 1e-5 * h), (c, float(d[clear].max()))
        checked += int(clear.sum())
        total += v1 - v0
        x = g
    assert total == 103823 and checked > 0.5 * total
