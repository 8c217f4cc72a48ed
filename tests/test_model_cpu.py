"""The double-precision MLP reference against finite differences (CPU)."""
import numpy as np

import oracle


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.1, oracle.MLP_PARAMS).astype(np.float32)
    X = rng.uniform(0, 8, (48, 8)).astype(np.float32)
    Y = rng.uniform(0, 10, 48).astype(np.float32)
    g, _ = oracle.mlp_grad(p, X, Y)

    def loss(q):
        return float(((oracle.mlp_forward(q, X) - Y) ** 2).mean())

    for i in (0, 37, 520, 700, 2900, 4650, 4799, 4800):
        eps = 1e-3
        qp, qm = p.copy(), p.copy()
        qp[i] += eps
        qm[i] -= eps
        fd = (loss(qp) - loss(qm)) / (float(qp[i]) - float(qm[i]))
        assert abs(fd - g[i]) <= 1e-3 * max(1.0, abs(g[i])), (i, fd, g[i])
