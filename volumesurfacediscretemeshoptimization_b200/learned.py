"""Training of the proposal network from plain DMO runs.

Pairs (one-ring features, DMO displacement) are collected on the GPU from plain iterations
of a seeded tet cube (``DMOTetClass.collect_pairs``) and the network is trained on the GPU by
the library's own forward / backward / Adam kernels (``ProposalModel.train``). Device buffers
come from torch (allocation only).
"""
from __future__ import annotations

import time

# training and reduced-search settings used for the 100^3 tet cube measurements: one level of
# 4^3 candidates at 0.0175 of the plain search's first extent (measured against 1-3 levels,
# 3^3-5^3 candidates and scales 0.008-0.05 on that cube and on the same cube jittered with
# another seed: the fewest milliseconds to plain's final minimum on both)
DEFAULTS = {"reduced_n": 4, "reduced_depth": 1, "reduced_scale": 0.0175,
            "train_steps": (20000, 6000), "train_lr": (1e-3, 2e-4), "batch": 8192,
            "pairs_mesh": "tet cube 48^3, jitter 0.3h", "pairs_seed": 1000, "pairs_iterations": 20}


def train_proposal(stream=None, cfg=DEFAULTS, model_seed: int = 0):
    """Collects training pairs and trains a new ProposalModel on the GPU.

    Returns (model, info) where info holds the pair count, final loss, target variance and
    the host times of the two phases."""
    import torch
    import volumesurfacediscretemeshoptimization_b200 as V
    from volumesurfacediscretemeshoptimization_b200 import meshgen as G

    dev = torch.device("cuda", torch.cuda.current_device())
    sp = stream.cuda_stream if stream is not None else None
    t0 = time.perf_counter()
    xyz, tets = G.config2(seed=cfg["pairs_seed"])
    tm = V.DMOMeshTet(xyz, tets, stream=sp)
    topt = V.DMOTetClass(tm, n_iter=cfg["pairs_iterations"])
    cap = (tm.info["nV"] - tm.info["nSurf"]) * cfg["pairs_iterations"]
    feats = torch.empty(cap * 96, dtype=torch.float32, device=dev)
    targ = torch.empty(cap * 3, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    n_pairs = topt.collect_pairs(cfg["pairs_iterations"], feats.data_ptr(), targ.data_ptr(), cap)
    t_collect = time.perf_counter() - t0
    model = V.ProposalModel(seed=model_seed, stream=sp)
    t1 = time.perf_counter()
    losses = []
    for k, (steps, lr) in enumerate(zip(cfg["train_steps"], cfg["train_lr"])):
        h = model.train(None, None, steps=steps, batch=cfg["batch"], lr=lr, seed=k,
                        device_ptrs=(feats.data_ptr(), targ.data_ptr()), n_rows=n_pairs)
        losses.append(float(h[-50:].mean()))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    tvar = float(targ.view(-1, 3)[:n_pairs].var(0).mean().item())
    topt.close()
    tm.close()
    info = {"pairs": n_pairs, "source": f"{cfg['pairs_iterations']} plain iterations, {cfg['pairs_mesh']} "
                                        f"seed {cfg['pairs_seed']}",
            "steps": list(cfg["train_steps"]), "lr": list(cfg["train_lr"]), "batch": cfg["batch"],
            "final_mse": losses[-1], "target_variance": tvar, "collect_s": t_collect, "train_s": t_train}
    return model, info
