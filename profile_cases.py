"""Small, self-contained workloads of each kernel family, for profiling one family at a time
(``ncu -k <kernel> python profile_cases.py <case>``).

Every case builds its mesh, runs one warm-up iteration (graph capture) and then ``--iters``
iterations, and prints one line with the case's time per iteration (CUDA events on the
library stream, not under a profiler's replay).

    tri2d       flat triangle grid 64^2 (4,096 vertices), k_dmo_tri2d
    flat_quad   flat quad grid 181^2 (32,761 vertices), k_dmo_flat<4>
    surf_tri    icosphere level 7 with surface noise (163,842 vertices), k_dmo_surf<3>
    surf_quad   torus 512x256 quads with surface noise (131,072 vertices), k_dmo_surf<4>
                (surface cases: --fit-ring 2 fits the quadrics over the 2-ring)
    tet         Kuhn tet cube 48^3 (117,649 vertices), k_dmo_tet
    hex         hex cube 32^3 (35,937 vertices), k_dmo_hex (--quality CONDITION: k_dmo_hex_cond)
    learned     Kuhn tet cube 100^3 (1,030,301 vertices) with the proposal network (trained
                first with --train, else untrained): k_mlp_tet_infer, k_dmo_tet_learned,
                k_dmo_tet_list
    batched     --meshes flat tri / quad grids of 500-50,000 vertices in one persistent
                launch per iteration, k_batch_iter
    build       the connectivity build of the tet cube 48^3 from pinned host arrays (radix
                sorts, CSR, colouring); --iters builds after one warm-up build
"""
from __future__ import annotations

import argparse
import json
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["tri2d", "flat_quad", "surf_tri", "surf_quad", "tet", "hex", "learned", "batched",
                                     "build"])
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--meshes", type=int, default=256)
    ap.add_argument("--train", action="store_true", help="learned: train the network first (else untrained)")
    ap.add_argument("--quality", default="MEAN_RATIO", help="QualityCriterium name (e.g. CONDITION for hex)")
    ap.add_argument("--fit-ring", type=int, default=1, help="surface cases: quadric fit over the 1- or 2-ring")
    a = ap.parse_args(argv)
    import torch
    import volumesurfacediscretemeshoptimization_b200 as V
    from volumesurfacediscretemeshoptimization_b200 import meshgen as G

    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    c = a.case
    if c == "build":
        # the connectivity build of the 48^3 tet cube from pinned host arrays, --iters times
        # after one warm-up build
        import ctypes as C
        from volumesurfacediscretemeshoptimization_b200 import _capi
        xyz, el = G.config2()
        lib = _capi.lib()
        px = torch.from_numpy(xyz).pin_memory()
        pe = torch.from_numpy(el).pin_memory()
        ms = []
        for rep in range(a.iters + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            with torch.cuda.stream(stream):
                e0.record(stream)
                h = C.c_void_p()
                _capi.check(lib.vsdmo_mesh_create(_capi.TET, C.c_void_p(px.data_ptr()), len(xyz), C.c_void_p(pe.data_ptr()),
                                                  len(el), _capi.HOST, 1, C.c_void_p(sp), C.byref(h)))
                e1.record(stream)
            torch.cuda.synchronize()
            lib.vsdmo_mesh_destroy(h)
            if rep:
                ms.append(e0.elapsed_time(e1))
        print(json.dumps({"case": c, "iters": a.iters, "ms_per_build": sum(ms) / len(ms)}), flush=True)
        return 0
    if c == "batched":
        opt = V.BatchDMO(G.config4(count=a.meshes), stream=sp)
        it = lambda n: opt.iterate(n)
    else:
        if c == "tri2d":
            xyz, el = G.config1()
            mesh, cls = V.DMOMeshTri(xyz, el, stream=sp), V.DMOTriFlatClass
        elif c == "flat_quad":
            xyz, el = G.quad_grid(181, seed=0, jitter=0.4)
            mesh, cls = V.DMOMeshQuad(xyz, el, stream=sp), V.DMOQuadFlatClass
        elif c == "surf_tri":
            xyz, el = G.config3_tri()
            mesh, cls = V.DMOMeshTri(xyz, el, stream=sp), V.DMOTriClass
        elif c == "surf_quad":
            xyz, el = G.config3_quad()
            mesh, cls = V.DMOMeshQuad(xyz, el, stream=sp), V.DMOQuadClass
        elif c == "tet":
            xyz, el = G.config2()
            mesh, cls = V.DMOMeshTet(xyz, el, stream=sp), V.DMOTetClass
        elif c == "hex":
            xyz, el = G.config2_hex()
            mesh, cls = V.DMOMeshHex(xyz, el, stream=sp), V.DMOHexClass
        else:
            xyz, el = G.config5()
            mesh, cls = V.DMOMeshTet(xyz, el, stream=sp), V.DMOTetClass
        kw = {"fit_ring": a.fit_ring} if c in ("surf_tri", "surf_quad") else {}
        opt = cls(mesh, qualityCriterium=getattr(V.QualityCriterium, a.quality), n_iter=10 ** 6, **kw)
        if c == "learned":
            from volumesurfacediscretemeshoptimization_b200.learned import DEFAULTS, train_proposal
            model = train_proposal(stream)[0] if a.train else V.ProposalModel(seed=0, stream=sp)
            opt.set_model(model, DEFAULTS["reduced_n"], DEFAULTS["reduced_depth"], DEFAULTS["reduced_scale"])
        it = lambda n: opt.iterate(n)
    it(1)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        e0.record(stream)
        it(a.iters)
        e1.record(stream)
    torch.cuda.synchronize()
    line = {"case": c, "iters": a.iters, "ms_per_iteration": e0.elapsed_time(e1) / a.iters,
            "wall_s": time.perf_counter() - t0}
    if c != "batched":
        line.update(quality=a.quality, min_quality=opt.getQuality(), fit_ring=a.fit_ring)
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
