"""CPU restatement of the learned proposal network (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline may use this module, and only
as the checker. The network has no counterpart in the reference (it is the project's learned
proposal): 96 -> 128 -> 128 -> 128 -> 3 with ReLU, parameters in one flat array
(W1 [128x96] b1 W2 [128x128] b2 W3 [128x128] b3 W4 [16x128] b4 [16], rows 3..15 of W4 / b4
zero). This module restates what the CUDA kernels compute, including where they round to
BF16: the inputs, the weights, every hidden activation after the ReLU, the output gradient
and every pre-activation gradient. Products and sums are taken in float64 here (the tensor
cores accumulate in FP32), so results agree to FP32 accumulation error, except where an
FP32 value sits on a BF16 rounding boundary.

With bf16=False the same functions are the plain float64 network; `finite_difference_check`
pins the backward formulas against central differences of the loss in that mode.
"""
import numpy as np

IN, HID, OUT, OUTP = 96, 128, 3, 16
SHAPES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)),
          ("b3", (HID,)), ("W4", (OUTP, HID)), ("b4", (OUTP,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unflatten(p):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def flatten(d):
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SHAPES])


def _r(x, on):
    return bf16(x.astype(np.float32)) if on else np.asarray(x, np.float64)


def forward(p, X, bf=True):
    """Returns (Y [n x 3], cache)."""
    P = unflatten(p)
    Xb = _r(X, bf)
    W = {k: _r(P[k], bf) for k in ("W1", "W2", "W3", "W4")}
    H1 = _r(np.maximum(Xb @ W["W1"].T + P["b1"], 0.0), bf)
    H2 = _r(np.maximum(H1 @ W["W2"].T + P["b2"], 0.0), bf)
    H3 = _r(np.maximum(H2 @ W["W3"].T + P["b3"], 0.0), bf)
    Y = H3 @ W["W4"].T + P["b4"]
    return Y[:, :OUT], dict(Xb=Xb, W=W, H1=H1, H2=H2, H3=H3, Y=Y)


def loss_and_grad(p, X, T, bf=True):
    """Mean squared error over the 3 outputs and its gradient (flat, like the parameters)."""
    B = len(X)
    _, c = forward(p, X, bf)
    Y, W = c["Y"], c["W"]
    e = Y[:, :OUT] - T
    loss = float((e * e).sum() / (3.0 * B))
    dY = np.zeros((B, OUTP))
    dY[:, :OUT] = 2.0 * e / (3.0 * B)
    dY = _r(dY, bf)
    g = {"b4": dY.sum(0), "W4": dY.T @ c["H3"]}
    dZ3 = _r((dY @ W["W4"]) * (c["H3"] > 0), bf)
    g["b3"] = dZ3.sum(0)
    g["W3"] = dZ3.T @ c["H2"]
    dZ2 = _r((dZ3 @ W["W3"]) * (c["H2"] > 0), bf)
    g["b2"] = dZ2.sum(0)
    g["W2"] = dZ2.T @ c["H1"]
    dZ1 = _r((dZ2 @ W["W2"]) * (c["H1"] > 0), bf)
    g["b1"] = dZ1.sum(0)
    g["W1"] = dZ1.T @ c["Xb"]
    g["W4"][OUT:] = 0.0
    g["b4"][OUT:] = 0.0
    return loss, flatten(g)


def init_params(seed=0):
    """He-uniform weights and zero biases, the same scheme the library uses (different RNG)."""
    r = np.random.default_rng(seed)
    d = {}
    for name, shape in SHAPES:
        if name.startswith("W"):
            a = np.sqrt(6.0 / shape[1])
            d[name] = r.uniform(-a, a, size=shape)
        else:
            d[name] = np.zeros(shape)
    d["W4"][OUT:] = 0.0
    return flatten(d)


def finite_difference_check(seed=0, n=16, eps=1e-6, n_probe=40):
    """Max relative error between loss_and_grad (float64 mode) and central differences at
    n_probe random parameters (biases shifted so that ReLUs are not at their kinks)."""
    r = np.random.default_rng(seed)
    p = init_params(seed)
    P = unflatten(p)
    for k in ("b1", "b2", "b3"):
        P[k] = r.uniform(0.05, 0.2, size=P[k].shape)
    p = flatten(P)
    X = r.uniform(-1, 1, size=(n, IN))
    T = r.uniform(-0.3, 0.3, size=(n, OUT))
    _, g = loss_and_grad(p, X, T, bf=False)
    valid = np.ones(N_PARAMS, bool)
    o = sum(int(np.prod(s)) for nm, s in SHAPES[:6])
    valid[o + OUT * HID:o + OUTP * HID] = False          # padded rows of W4
    valid[N_PARAMS - (OUTP - OUT):] = False              # padded b4
    idx = r.choice(np.flatnonzero(valid), size=n_probe, replace=False)
    worst = 0.0
    for i in idx:
        q = p.copy(); q[i] += eps
        lp, _ = loss_and_grad(q, X, T, bf=False)
        q[i] -= 2 * eps
        lm, _ = loss_and_grad(q, X, T, bf=False)
        fd = (lp - lm) / (2 * eps)
        worst = max(worst, abs(fd - g[i]) / max(1e-6, abs(fd) + abs(g[i])))
    return worst
