"""Generates the golden fixtures in tests/golden/ from the CPU oracle.

The reference repository ships no tests, fixtures or sample meshes, so these fixtures pin
the oracle's own restatement (connectivity, colouring and DMO results on small seeded
meshes) against drift; tests/test_oracle_golden.py re-derives them and compares, and the
GPU parity tests compare the CUDA library against the same oracle.

Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from volumesurfacediscretemeshoptimization_b200 import meshgen as G  # noqa: E402

CASES = {
    "tri_grid8": dict(kind=O.TRI, gen=lambda: G.tri_grid(8, seed=3, jitter=0.4), iters=3),
    "tet_cube4": dict(kind=O.TET, gen=lambda: G.tet_cube(4, seed=5, jitter=0.3), iters=2),
}


def make(name):
    c = CASES[name]
    xyz, el = c["gen"]()
    m = O.OracleMesh(c["kind"], xyz, el, color_seed=1)
    out = {"in_xyz": xyz, "in_elems": el}
    for k, v in m.arrays().items():
        out[k] = v
    x0 = m.xyz
    x32, mn32, me32 = m.optimize_f32(x0, c["iters"])
    x64, mn64, me64 = m.optimize_f64(x0, c["iters"])
    out.update(dmo_f32_xyz=x32, dmo_f32_min=mn32, dmo_f32_mean=me32,
               dmo_f64_xyz=x64, dmo_f64_min=mn64, dmo_f64_mean=me64,
               info=np.array([m.info[k] for k in O.I_NAMES], dtype=np.int64))
    return out


def main():
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **make(name))
        print("wrote", name)


if __name__ == "__main__":
    main()
