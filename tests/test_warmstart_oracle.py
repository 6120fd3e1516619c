"""The FP64 restatement of the warm-start network (oracle/warmnet_ref.py):
its backward pass against central finite differences, and the BF16 rounding
it applies to the weights."""
import numpy as np
import pytest

from oracle.warmnet_ref import WarmNetRef, bf16_round


def test_bf16_rounding_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 3.140625], dtype=np.float32)
    r = bf16_round(x)
    # 7 stored mantissa bits: 1 + 2^-8 is a tie -> even (1.0), 1 + 2^-9 rounds down,
    # 1 + 3*2^-9 rounds up to 1 + 2^-7
    np.testing.assert_array_equal(r, [1.0, 1.0, 1.0, 1.0 + 2 ** -7, -2.5, 3.140625])


@pytest.mark.parametrize("levels,channels", [(1, (2, 2)), (2, (4, 2, 2))])
def test_backward_matches_finite_differences(levels, channels):
    rng = np.random.default_rng(3)
    net = WarmNetRef(8, 8, 4, levels, channels, hidden=6, n_inputs=4)
    w = rng.uniform(-0.5, 0.5, net.n_weights)
    x = rng.uniform(-1, 1, (2, 4))
    t = rng.uniform(0, 1, (2, 8 * 8 * 4))
    _, g = net.loss_and_grad(w, x, t, round_weights=False)
    h = 1e-6
    for i in rng.choice(net.n_weights, 60, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (net.loss_and_grad(wp, x, t, round_weights=False)[0] -
              net.loss_and_grad(wm, x, t, round_weights=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(g[i])) + 1e-10, (i, fd, g[i])


def test_pretrained_weights_file():
    """The stored network (BF16 bit patterns) matches the architecture the
    FP64 restatement lays out for it."""
    import os

    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gpesolver_b200", "data",
                        "warmstart_128x128x32.npz")
    with np.load(path) as f:
        ref = WarmNetRef(int(f["nx"]), int(f["ny"]), int(f["nz"]), int(f["levels"]),
                         [int(c) for c in f["channels"]], int(f["hidden"]), int(f["n_inputs"]))
        w = (f["weights_bf16"].astype(np.uint32) << 16).view(np.float32)
    assert w.size == ref.n_weights and np.all(np.isfinite(w))
