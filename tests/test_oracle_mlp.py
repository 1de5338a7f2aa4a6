"""CPU checks of the oracle's FP64 MLP gradient (learned walk budget): the
analytic gradient agrees with central finite differences of the loss."""
import numpy as np

import oracle_binding as ob


def test_mlp_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(7)
    n = 16
    params = (rng.standard_normal(5258) * 0.2).astype(np.float32)
    X = rng.standard_normal((n, 6)).astype(np.float32)
    count = rng.integers(2, 11, n).astype(np.uint8)
    length = rng.uniform(20, 80, n).astype(np.float32)
    g, loss = ob.mlp_loss_grad(params, X, count, length)
    assert np.isfinite(loss) and loss > 0
    # parameters are FP32 in the interface; the step is the FP32 difference
    # actually taken, small enough that no ReLU input crosses zero
    # a few coordinates of every block: W1 0..383, b1 ..447, W2 ..4543, b2 ..4607, W3 ..5247, b3 ..5257
    for i in [0, 100, 383, 389, 465, 4543, 4550, 4611, 5000, 5247, 5250, 5257]:
        h = 1e-4
        p1, p2 = params.copy(), params.copy()
        p1[i] += np.float32(h)
        p2[i] -= np.float32(h)
        _, l1 = ob.mlp_loss_grad(p1, X, count, length)
        _, l2 = ob.mlp_loss_grad(p2, X, count, length)
        fd = (l1 - l2) / (float(p1[i]) - float(p2[i]))
        assert abs(fd - g[i]) <= 1e-4 * max(1.0, abs(g[i])) + 1e-5, (i, fd, g[i])
