"""Generates tests/golden/full_size_fp64.json: the FP64 oracle's minimum and mean element
quality after every iteration of the full-size benchmark workloads, the yardstick of the -m gpu
test tests/test_gpu_full_size.py (the library's final minimum and mean within 1e-4 of them).

    python tests/golden/make_full_size.py [--threads N] [--only NAME ...]

The FP64 restatements are the oracle's literal double versions of the reference kernels
(oracle/or_dmo.c, or_hex.c, or_surf.c, or_feat.c), run here on the CPU with OpenMP; config 2
takes about 8 minutes on 8 cores. Each entry records the generator call, the optimiser settings
and the colouring (the library's default hashed priorities, color_seed 1).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from volumesurfacediscretemeshoptimization_b200 import meshgen as G  # noqa: E402

OUT = os.path.join(HERE, "full_size_fp64.json")

# name: (generator call, kind, iterations, optimiser settings, runner)
WORKLOADS = {
    "config1": ("meshgen.config1()", O.TRI, 10, "DMOTriFlatClass, mean ratio, 8x8, 3 levels, boundary fixed"),
    "config2": ("meshgen.config2()", O.TET, 20, "DMOTetClass, mean ratio, 8x8x8, 3 levels, boundary fixed"),
    "config2_hex": ("meshgen.config2_hex()", O.HEX, 20, "DMOHexClass, shape metric, 8x8x8, 3 levels, boundary fixed"),
    "config3_tri": ("meshgen.config3_tri()", O.TRI, 15,
                    "DMOTriClass, mean ratio, 8x8, 3 levels, 1-ring quadrics, feature vertices slide"),
    "config3_quad": ("meshgen.config3_quad()", O.QUAD, 15,
                     "DMOQuadClass, mean ratio, 8x8, 3 levels, 1-ring quadrics, feature vertices slide"),
}


def run(name, threads):
    call, kind, iters, settings = WORKLOADS[name]
    xyz, el = eval(call, {"meshgen": G})
    om = O.OracleMesh(kind, xyz, el, color_seed=1)
    t0 = time.time()
    q0 = om.element_qualities_f64(om.xyz)
    if kind in (O.TRI, O.QUAD) and om.is_surface:
        _, mn, mean = om.optimize_surf_features_f64(om.xyz, iters, nthreads=threads)
    else:
        _, mn, mean = om.optimize_f64(om.xyz, iters, nthreads=threads)
    return {"generator": call, "iterations": iters, "settings": settings, "color_seed": 1,
            "vertices": om.info["nV"], "elements": om.info["nE"], "feature_vertices": om.info["nFeature"],
            "initial_min": float(q0.min()), "initial_mean": float(q0.mean()),
            "min": [float(v) for v in mn], "mean": [float(v) for v in mean],
            "cpu_seconds": round(time.time() - t0, 1)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", nargs="*")
    args = ap.parse_args()
    O.build()
    data = json.load(open(OUT)) if os.path.exists(OUT) else {}
    for name in args.only or WORKLOADS:
        print(f"{name} ...", flush=True)
        data[name] = run(name, args.threads)
        print(f"  {data[name]['min'][-1]:.6f} / {data[name]['mean'][-1]:.6f} in {data[name]['cpu_seconds']} s",
              flush=True)
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
