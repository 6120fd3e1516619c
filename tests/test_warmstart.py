"""The warm-start network on the GPU: gradients of its CUDA forward and
backward kernels against the FP64 NumPy restatement (oracle/warmnet_ref.py,
itself pinned against finite differences), and what a trained network gains:
imaginary time from its prediction reaches the ground-state energy tolerance
in fewer iterations than from the Gaussian start, on solves it was not
trained on."""
import numpy as np
import pytest

import gpesolver_b200 as G
from gpesolver_b200 import sweep, warmstart as W
from oracle.warmnet_ref import WarmNetRef

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("dims,levels,channels", [((16, 16, 8), 2, (4, 4, 2)), ((16, 16, 8), 1, (8, 2)),
                                                   ((32, 32, 32), 2, (4, 8, 8))])
def test_gradients_match_fp64_restatement(dims, levels, channels):
    """(32^3: the large layers take the tiled forward convolution.)"""
    import torch

    nx, ny, nz = dims
    cfg = W.WarmConfig(nx=nx, ny=ny, nz=nz, levels=levels, channels=channels, hidden=8, max_batch=3)
    net = W.WarmStartNet(cfg, seed=5)
    ref = WarmNetRef(nx, ny, nz, levels, channels, hidden=8)
    assert net.n_weights == ref.n_weights
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, (3, 4)).astype(np.float32)
    t = rng.uniform(0, 2, (3, nx * ny * nz)).astype(np.float32)
    td = torch.tensor(t, device="cuda")
    loss, g = net.gradients(x, td.data_ptr())
    rloss, rg = ref.loss_and_grad(net.get_weights(), x, t)
    assert abs(loss - rloss) <= 1e-5 * abs(rloss)
    for name, (o, n) in ref.off.items():
        assert _rel(g[o:o + n], rg[o:o + n]) < 2e-4, name
    # forward: the amplitudes themselves
    amp = torch.empty(3 * nx * ny * nz, device="cuda")
    net.forward(x, amp.data_ptr())
    net.close()


def test_trained_network_shortens_imaginary_time():
    import torch

    grids = ((64, 64, 16),)
    train_p = sweep.sweep_params(count=128, seed=11, grids=grids)
    held_p = sweep.sweep_params(count=6, seed=12, grids=grids)
    targets, _ = W.ground_states(train_p, iters=3000)
    cfg = W.WarmConfig(nx=64, ny=64, nz=16, levels=3, channels=(16, 16, 8, 4), hidden=64, max_batch=8)
    net = W.WarmStartNet(cfg, seed=1)
    hist = W.train(net, train_p, targets, epochs=40, batch=8, lr=1e-3, lr_final=3e-5)
    assert hist[-1] < 0.5 * hist[0]
    gain, same = [], 0
    for p in held_p:
        with G.B200GrossPitaevskiSolver(p) as a, G.B200GrossPitaevskiSolver(p) as b:
            for s in (a, b):
                s.init_pote()
            a.init_buffer("GAUSS")
            net.predict_into(b)
            ia, _, ea = W.time_to_ground_state(a)
            ib, _, eb = W.time_to_ground_state(b)
            # the same ground state: both stop about 1e-6 (relative) above it;
            # another (metastable) state differs by 1e-4 and more
            if abs(ea - eb) <= 1e-5 * abs(ea):
                same += 1
                gain.append(ia / ib)
    net.close()
    del targets
    torch.cuda.empty_cache()
    # most predictions lead imaginary time to the Gaussian start's ground state,
    # in fewer iterations
    assert same >= len(held_p) // 2, same
    assert np.median(gain) > 1.2, gain


def test_committed_network_shortens_imaginary_time_at_128():
    """The committed 128x128x32 network (gpesolver_b200/data) on the first 8
    held-out solves of the warm-start study (SplitMix64 seed 2000, CYLINDRICAL,
    edd, n_atoms, omega_r, omega_z / omega_r over the sweep ranges): imaginary
    time from its prediction and from the Gaussian start both run to dE/E <
    1e-8 between checks 10 iterations apart.  On a B200 the warm starts took
    2.0-4.1x fewer iterations (median 3.1x) and all reached the Gaussian start's
    state; over all 32 held-out solves the median time ratio was 2.35x (29 of
    32 in the same state), short of the 3x target.  Held here: the same state
    for at least 7 of 8, a median iteration ratio of at least 2.5, none below
    1.5."""
    grids = ((128, 128, 32),)
    held_p = sweep.sweep_params(count=8, seed=2000, grids=grids)
    net = W.WarmStartNet.pretrained()
    ratios, same = [], 0
    for p in held_p:
        with G.B200GrossPitaevskiSolver(p) as a, G.B200GrossPitaevskiSolver(p) as b:
            for s in (a, b):
                s.init_pote()
            a.init_buffer("GAUSS")
            net.predict_into(b)
            ia, _, ea = W.time_to_ground_state(a)
            ib, _, eb = W.time_to_ground_state(b)
            if abs(ea - eb) <= 1e-5 * abs(ea):
                same += 1
                ratios.append(ia / ib)
    net.close()
    assert same >= 7, same
    assert np.median(ratios) >= 2.5, ratios
    assert min(ratios) >= 1.5, ratios
