"""FP64 NumPy restatement of the warm-start network -- TEST INFRASTRUCTURE ONLY.

The checker for gpesolver_b200/csrc/warmstart.cu: the same layers, weight
layout and loss, with the weights rounded to BF16 (round to nearest even) as
the CUDA forward and backward passes use them, evaluated in FP64.  Its own
backward pass is pinned against central finite differences in
tests/test_warmstart_oracle.py.

Layout of the flat weight vector (the CUDA layout): dense 1 weights
[hidden][n_inputs], bias [hidden]; dense 2 weights [latent][hidden], bias
[latent]; then per convolution weights [cout][cin][27] (tap t = 9 dx + 3 dy +
dz over offsets -1..1), bias [cout].  Volumes are [channel][x][y][z].
"""
from __future__ import annotations

import numpy as np


def bf16_round(w: np.ndarray) -> np.ndarray:
    """FP32 -> BF16 (round to nearest, ties to even) -> FP64."""
    f = np.asarray(w, dtype=np.float32).copy()
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r.astype(np.uint32)).view(np.float32).astype(np.float64)


class WarmNetRef:
    def __init__(self, nx, ny, nz, levels, channels, hidden, n_inputs=4):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.levels, self.channels, self.hidden, self.n_inputs = levels, list(channels), hidden, n_inputs
        f = 1 << levels
        self.g0 = (nx // f, ny // f, nz // f)
        self.latent = channels[0] * self.g0[0] * self.g0[1] * self.g0[2]
        off = 0
        self.off = {}

        def take(name, n):
            nonlocal off
            self.off[name] = (off, n)
            off += n

        take("d1w", hidden * n_inputs)
        take("d1b", hidden)
        take("d2w", self.latent * hidden)
        take("d2b", self.latent)
        self.convs = []
        for s in range(levels + 1):
            cin = channels[s]
            cout = channels[s + 1] if s < levels else 1
            take(f"c{s}w", cout * cin * 27)
            take(f"c{s}b", cout)
            self.convs.append((cin, cout, s < levels))
        self.n_weights = off

    def _get(self, w, name, shape):
        o, n = self.off[name]
        return w[o:o + n].reshape(shape)

    @staticmethod
    def _up(x):
        return x.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)

    @staticmethod
    def _conv(u, Wc, bc):
        """u [cin][X][Y][Z], Wc [cout][cin][27] -> [cout][X][Y][Z], zero padding."""
        cin, X, Y, Z = u.shape
        p = np.zeros((cin, X + 2, Y + 2, Z + 2))
        p[:, 1:-1, 1:-1, 1:-1] = u
        out = np.zeros((Wc.shape[0], X, Y, Z)) + bc[:, None, None, None]
        for t in range(27):
            dx, dy, dz = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
            sh = p[:, 1 + dx:1 + dx + X, 1 + dy:1 + dy + Y, 1 + dz:1 + dz + Z]
            out += np.tensordot(Wc[:, :, t], sh, axes=(1, 0))
        return out

    @staticmethod
    def _conv_back(u, Wc, gy):
        """gradients of the convolution: dW [cout][cin][27], db [cout], du."""
        cin, X, Y, Z = u.shape
        p = np.zeros((cin, X + 2, Y + 2, Z + 2))
        p[:, 1:-1, 1:-1, 1:-1] = u
        dW = np.zeros_like(Wc)
        dp = np.zeros_like(p)
        for t in range(27):
            dx, dy, dz = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
            sl = (slice(None), slice(1 + dx, 1 + dx + X), slice(1 + dy, 1 + dy + Y), slice(1 + dz, 1 + dz + Z))
            dW[:, :, t] = np.tensordot(gy, p[sl], axes=([1, 2, 3], [1, 2, 3]))
            dp[sl] += np.tensordot(Wc[:, :, t], gy, axes=(0, 0))
        return dW, gy.sum(axis=(1, 2, 3)), dp[:, 1:-1, 1:-1, 1:-1]

    @staticmethod
    def _silu(y):
        return y / (1 + np.exp(-y))

    @staticmethod
    def _silu_grad(y):
        s = 1 / (1 + np.exp(-y))
        return s * (1 + y * (1 - s))

    def loss_and_grad(self, w32, inputs, targets, round_weights: bool = True):
        """Mean squared amplitude error over the batch and its gradient (FP64),
        with the weights rounded to BF16 (round_weights=False: used as given,
        for finite-difference checks of the backward pass)."""
        w = bf16_round(w32) if round_weights else np.asarray(w32, dtype=np.float64)
        B = inputs.shape[0]
        H, L = self.hidden, self.latent
        d1w, d1b = self._get(w, "d1w", (H, self.n_inputs)), self._get(w, "d1b", (H,))
        d2w, d2b = self._get(w, "d2w", (L, H)), self._get(w, "d2b", (L,))
        grad = np.zeros(self.n_weights)
        loss = 0.0
        N = self.nx * self.ny * self.nz
        for b in range(B):
            x = np.asarray(inputs[b], dtype=np.float64)
            h1p = d1w @ x + d1b
            h1 = self._silu(h1p)
            h2p = d2w @ h1 + d2b
            h2 = self._silu(h2p)
            vol = h2.reshape((self.channels[0],) + self.g0)
            cache = []
            for s, (cin, cout, up) in enumerate(self.convs):
                Wc = self._get(w, f"c{s}w", (cout, cin, 27))
                bc = self._get(w, f"c{s}b", (cout,))
                u = self._up(vol) if up else vol
                y = self._conv(u, Wc, bc)
                cache.append((vol, u, y))
                vol = self._silu(y) if s < self.levels else y
            u_out = vol[0]  # the amplitude (linear output)
            t = np.asarray(targets[b], dtype=np.float64).reshape(u_out.shape)
            d = u_out - t
            loss += float((d * d).sum())
            g = (2 * d / (B * N))[None]
            for s in range(self.levels, -1, -1):
                cin, cout, up = self.convs[s]
                vin, u, y = cache[s]
                if s < self.levels:
                    g = g * self._silu_grad(y)
                Wc = self._get(w, f"c{s}w", (cout, cin, 27))
                dW, db, du = self._conv_back(u, Wc, g)
                o, n = self.off[f"c{s}w"]
                grad[o:o + n] += dW.reshape(-1)
                o, n = self.off[f"c{s}b"]
                grad[o:o + n] += db
                if up:
                    du = du.reshape(cin, du.shape[1] // 2, 2, du.shape[2] // 2, 2, du.shape[3] // 2, 2).sum(
                        axis=(2, 4, 6))
                g = du
            g2 = g.reshape(-1) * self._silu_grad(h2p)
            o, n = self.off["d2w"]
            grad[o:o + n] += np.outer(g2, h1).reshape(-1)
            o, n = self.off["d2b"]
            grad[o:o + n] += g2
            g1 = (d2w.T @ g2) * self._silu_grad(h1p)
            o, n = self.off["d1w"]
            grad[o:o + n] += np.outer(g1, x).reshape(-1)
            o, n = self.off["d1b"]
            grad[o:o + n] += g1
        return loss / (B * N), grad
