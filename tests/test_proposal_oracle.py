"""The CPU oracle of the proposal network checked against finite differences (CPU).

With bf16 rounding switched off, the oracle's analytic gradients of the loss with respect to
sampled entries of every weight and bias must match central differences of its own forward
pass and loss; this pins the oracle that the GPU gradients are compared with."""
import numpy as np

from oracle import proposal_oracle as PO


def _setup(n=6, seed=0):
    rng = np.random.default_rng(seed)
    lay, P = {}, {}
    shapes = {"w1": (32, 18), "w2": (32, 288), "w3": (32, 288), "w4": (32, 288), "f1": (128, 304),
              "f2": (128, 128), "f3": (16, 128)}
    for k, (r, c) in shapes.items():
        P[k] = rng.normal(0, np.sqrt(2.0 / c), (r, c))
    for k, r in (("b1", 32), ("b2", 32), ("b3", 32), ("b4", 32), ("bf1", 128), ("bf2", 128), ("bf3", 16)):
        P[k] = rng.normal(0, 0.1, r)
    feat = rng.uniform(-1, 1, (n, 24, 24, 2))
    pred16 = np.zeros((n, 16))
    pred16[:, :14] = rng.integers(-40, 41, (n, 14)) / 64.0
    tmv = rng.integers(-25, 26, (n, 2))
    tskip = (rng.random(n) < 0.5).astype(np.uint8)
    return P, feat, pred16, tmv, tskip


def _loss(P, feat, pred16, tmv, tskip):
    o, _ = PO.forward(P, feat, pred16)
    return PO.head_loss(o, tmv, tskip)[0]


def test_oracle_gradients_match_finite_differences():
    PO.ROUND = False
    try:
        P, feat, pred16, tmv, tskip = _setup()
        o, acts = PO.forward(P, feat, pred16)
        _, dO = PO.head_loss(o, tmv, tskip)
        G = PO.backward(P, acts, dO)
        rng = np.random.default_rng(1)
        eps = 1e-6
        for name, w in P.items():
            for _ in range(4):
                idx = tuple(int(rng.integers(0, s)) for s in w.shape)
                old = w[idx]
                w[idx] = old + eps
                lp = _loss(P, feat, pred16, tmv, tskip)
                w[idx] = old - eps
                lm = _loss(P, feat, pred16, tmv, tskip)
                w[idx] = old
                fd = (lp - lm) / (2 * eps)
                assert abs(fd - G[name][idx]) <= 1e-5 + 1e-4 * abs(fd), (name, idx, fd, G[name][idx])
    finally:
        PO.ROUND = True
