"""CPU tests of the network oracle (oracle/mlp_oracle.py): BF16 rounding and the backward
formulas against central finite differences."""
import numpy as np

from oracle import mlp_oracle as mo


def test_bf16_rounding_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-30, 3.0e38], np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # halfway, rounds to the even mantissa
    assert r[2] == 1.0 + 2 ** -6            # halfway, rounds up to even
    assert r[3] == -2.5
    u = r.astype(np.float32).view(np.uint32)
    assert np.all(u & 0xFFFF == 0)


def test_backward_matches_finite_differences():
    assert mo.finite_difference_check(seed=0) < 1e-5
    assert mo.finite_difference_check(seed=1) < 1e-5


def test_padded_outputs_carry_no_gradient():
    r = np.random.default_rng(0)
    p = mo.init_params(3)
    X = r.uniform(-1, 1, size=(64, mo.IN))
    T = r.uniform(-1, 1, size=(64, mo.OUT))
    _, g = mo.loss_and_grad(p, X, T)
    G = mo.unflatten(g)
    assert np.all(G["W4"][mo.OUT:] == 0) and np.all(G["b4"][mo.OUT:] == 0)
    assert np.abs(G["W1"]).sum() > 0
