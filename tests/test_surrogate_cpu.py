"""CPU checks of the learned-conduction surrogate's oracle and host logic:
the numpy restatement's backward pass against finite differences, the
adjoint identity behind backward-data-as-flipped-convolution, bf16 rounding,
and the window metrics of the plain-RKL2 re-check."""
import numpy as np
import pytest

from oracle import surrogate_ref as R


def small_net(seed=1):
    W, B = R.init_params(seed)
    rng = np.random.default_rng(seed + 7)
    for l in range(4):
        B[l] = (rng.standard_normal(B[l].shape) * 0.05).astype(np.float32)
    # the last layer's weights are small at init; make them O(1) so every
    # gradient term is visible in the finite differences
    W[3] = W[3] * 10.0
    return [w.astype(np.float64) for w in W], [b.astype(np.float64) for b in B]


def test_reference_gradients_match_finite_differences():
    W, B = small_net()
    rng = np.random.default_rng(3)
    x = np.zeros((2, 11, 11, 11, 16))
    x[..., :5] = rng.uniform(0.0, 1.0, (2, 11, 11, 11, 5))
    tgt = rng.standard_normal((2, 3, 3, 3)) * 0.1
    loss, dW, dB = R.loss_and_grads(W, B, x, tgt, rounding=False)
    h = 1e-6
    for l, idx in [(0, (4, 3, 2)), (1, (13, 7, 30)), (2, (26, 0, 5)), (3, (9, 0, 17)), (3, (0, 0, 0))]:
        Wp = [w.copy() for w in W]
        Wm = [w.copy() for w in W]
        Wp[l][idx] += h
        Wm[l][idx] -= h
        lp, _, _ = R.loss_and_grads(Wp, B, x, tgt, rounding=False)
        lm, _, _ = R.loss_and_grads(Wm, B, x, tgt, rounding=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - dW[l][idx]) <= 1e-6 * max(1e-3, abs(fd)) + 1e-10, (l, idx, fd, dW[l][idx])
    for l, c in [(0, 3), (2, 31), (3, 0)]:
        Bp = [b.copy() for b in B]
        Bm = [b.copy() for b in B]
        Bp[l][c] += h
        Bm[l][c] -= h
        fd = (R.loss_and_grads(W, Bp, x, tgt, False)[0] - R.loss_and_grads(W, Bm, x, tgt, False)[0]) / (2 * h)
        assert abs(fd - dB[l][c]) <= 1e-6 * max(1e-3, abs(fd)) + 1e-10, (l, c, fd, dB[l][c])


def test_padded_channels_get_zero_gradient():
    W, B = small_net()
    rng = np.random.default_rng(5)
    x = np.zeros((1, 10, 10, 10, 16))
    x[..., :5] = rng.uniform(0.0, 1.0, (1, 10, 10, 10, 5))
    tgt = rng.standard_normal((1, 2, 2, 2))
    _, dW, dB = R.loss_and_grads(W, B, x, tgt, rounding=True)
    assert np.all(dW[0][:, :, 5:] == 0.0)          # input channels 5..15 are zero
    assert np.all(dW[3][:, 1:, :] == 0.0)          # only output channel 0 is trained
    assert np.all(dB[3][1:] == 0.0)


def test_backward_data_is_the_adjoint_of_the_forward_conv():
    rng = np.random.default_rng(9)
    x = rng.standard_normal((2, 7, 7, 7, 16))
    w = rng.standard_normal((27, 32, 16))
    y = rng.standard_normal((2, 5, 5, 5, 32))
    lhs = np.sum(R.conv(x, w) * y)
    rhs = np.sum(x * R.conv(y, R.flip(w), pad=2))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -3.140625, 1e-40, 65504.0])
    r = R.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0                                # tie -> even
    assert r[2] == 1.0 + 2.0 ** -6                    # tie -> even (up)
    assert r[3] == -3.140625
    assert r[5] == 65536.0


def test_window_metrics_repeat_on_a_power_of_two_grid():
    from lare3d_b200.grid import grid
    from lare3d_b200.surrogate import window_metrics
    n = 64
    m = grid(n, n, n)
    for x0 in (0, -20, 44):
        w = window_metrics(m, n, x0, 104, "x")
        assert np.all(w["dxb"] == m["dxb"][2]) and np.all(w["dxc"] == m["dxc"][2])
    # a general grid: values follow the wrapped grid index
    m2 = grid(48, 48, 48, (0.0, 0.7))
    w = window_metrics(m2, 48, 45, 10, "x")
    for i in range(-1, 13):
        gi = ((45 + i - 1) % 48) + 1
        assert w["dxb"][i + 1] == m2["dxb"][gi + 1]


def test_surrogate_refuses_a_per_cell_neutral_fraction():
    """The network and its exact re-check take the temperature with one xi_n
    for the whole grid, so a partially ionised deck is refused up front."""
    from types import SimpleNamespace
    from lare3d_b200 import surrogate
    from lare3d_b200.abi import EOS_ION
    sim = SimpleNamespace(params=SimpleNamespace(eos_number=EOS_ION), nx=64, ny=64, nz=64)
    with pytest.raises(ValueError, match="EOS_IDEAL"):
        surrogate.SurrogateConduction(sim, None, None, 1.0)
