"""Pin the CPU restatement of the warm-start MLP: its backward pass matches
finite differences (float64, no BF16 rounding), and its BF16 rounding matches
torch's."""
import numpy as np
import torch

from oracle import mlp


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(1).normal(scale=10.0, size=4096).astype(np.float32)
    ref = torch.tensor(x).bfloat16().float().numpy()
    np.testing.assert_array_equal(mlp.bf16(x), ref)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(2)
    dims = [5, 7, 6, 3]
    W = [rng.normal(size=(dims[l + 1], dims[l])) for l in range(3)]
    b = [rng.normal(size=dims[l + 1]) * 0.1 for l in range(3)]
    X = rng.normal(size=(4, 5))
    T = rng.normal(size=(4, 3))

    def loss(W_, b_):
        Y, _ = mlp.forward(W_, b_, X, rounding=False)
        return 0.5 * np.sum((Y - T) ** 2)

    Y, cache = mlp.forward(W, b, X, rounding=False)
    gW, gb = mlp.backward(W, cache, Y - T)
    eps = 1e-6
    for l in range(3):
        for (i, j) in [(0, 0), (1, 2), (dims[l + 1] - 1, dims[l] - 1)]:
            Wp = [w.copy() for w in W]
            Wm = [w.copy() for w in W]
            Wp[l][i, j] += eps
            Wm[l][i, j] -= eps
            fd = (loss(Wp, b) - loss(Wm, b)) / (2 * eps)
            assert abs(fd - gW[l][i, j]) <= 1e-6 * max(1.0, abs(fd))
        bp = [v.copy() for v in b]
        bm = [v.copy() for v in b]
        bp[l][0] += eps
        bm[l][0] -= eps
        fd = (loss(W, bp) - loss(W, bm)) / (2 * eps)
        assert abs(fd - gb[l][0]) <= 1e-6 * max(1.0, abs(fd))
