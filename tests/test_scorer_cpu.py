"""The learned block order on the CPU: the scorer oracle's backward pass against finite
differences, its BF16 rounding, and the library's host-side block features against the
oracle's restatement (bit-exact)."""
import numpy as np
import pytest

import scorer_oracle as SO
from ltlb200 import api


def _data(seed, n=96):
    rng = np.random.default_rng(seed)
    X = rng.random((n, SO.NF)).astype(np.float32)
    Y = (rng.random(n) < 0.3).astype(np.float32)
    return X, Y


def test_layout_matches_abi():
    assert SO.PARAMS == api.SCORER_PARAMS == 6337
    assert SO.NF == api.SCORER_FEATURES


@pytest.mark.parametrize("pos_weight", [1.0, 4.0])
def test_exact_gradient_vs_finite_differences(pos_weight):
    X, Y = _data(1)
    p = SO.init_params(3).astype(np.float64)
    p[SO.B1:SO.W2] = 0.05  # biases away from zero so ReLU kinks are rare
    p[SO.B2:SO.W3] = 0.05
    g = SO.grad_exact(p, X, Y, pos_weight)
    rng = np.random.default_rng(7)
    idx = np.concatenate([rng.choice(np.arange(SO.W1, SO.B1), 12), rng.choice(np.arange(SO.B1, SO.W2), 4),
                          rng.choice(np.arange(SO.W2, SO.B2), 12), rng.choice(np.arange(SO.B2, SO.W3), 4),
                          rng.choice(np.arange(SO.W3, SO.B3), 6), [SO.B3]])
    eps = 1e-6
    for i in idx:
        a, b = p.copy(), p.copy()
        a[i] += eps
        b[i] -= eps
        fd = (SO.loss_exact(a, X, Y, pos_weight) - SO.loss_exact(b, X, Y, pos_weight)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_rounded_gradient_close_to_exact():
    X, Y = _data(2, 256)
    p = SO.init_params(5)
    g, loss = SO.grad(p, X, Y, 2.0)
    ge = SO.grad_exact(p, X, Y, 2.0)
    assert np.linalg.norm(g - ge) <= 0.05 * np.linalg.norm(ge)
    assert abs(loss - SO.loss_exact(p, X, Y, 2.0)) <= 0.02 * abs(loss)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-39, 65504.0], dtype=np.float32)
    r = SO.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0          # tie rounds to even (mantissa ...0)
    assert r[2] == 1.0078125    # above the tie rounds up
    assert r[3] == -2.5
    assert (r.view(np.uint32) & 0xFFFF == 0).all()


def _random_info(rng):
    op = int(rng.integers(7))
    cost = int(rng.integers(3, 20))
    un = op in (0, 3, 4, 5)
    lcost = int(rng.integers(1, cost))
    rcost = 0 if un else int(rng.integers(1, cost))
    big = lambda: int(rng.integers(0, 1 << int(rng.integers(1, 40))))
    return dict(op=op, cost=cost, c1=1, lcost=lcost, rcost=rcost, position=int(rng.integers(0, 40)),
                nblocks=int(rng.integers(1, 60)), lrows=big(), rrows=1 if un else big(), candidates=big(),
                level_cands=big(), lstat=[big() for _ in range(2)], rstat=[0] * 2 if un else [big() for _ in range(2)],
                npos=int(rng.integers(0, 5000)), nneg=int(rng.integers(0, 5000)), nalpha=int(rng.integers(1, 27)))


def test_block_features_bit_exact():
    rng = np.random.default_rng(11)
    for _ in range(500):
        info = _random_info(rng)
        got = api.block_features(**info)
        want = SO.block_features(**info)
        assert got.view(np.uint32).tolist() == want.view(np.uint32).tolist(), info


def test_scorer_symbols_exported():
    L = api.lib()
    for name in ("ltlg_block_features", "ltlg_engine_set_scorer", "ltlg_batch_set_scorer",
                 "ltlg_engine_label_blocks", "ltlg_scorer_forward", "ltlg_scorer_grad", "ltlg_scorer_train"):
        assert hasattr(L, name)
