"""GPU checks of the learned-conduction surrogate: every kernel of the
forward and backward pass against the numpy oracle (oracle/surrogate_ref.py),
training on the engine's own RKL2 pairs, what the trained network gains over
the method without it, and the plain-RKL2 arbiter (exact column re-check,
patch-wise rejection and whole-grid fallback)."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import surrogate_ref as R

pytestmark = pytest.mark.gpu


def torch_mod():
    import torch
    return torch


def to_bf16_dev(a):
    torch = torch_mod()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to("cuda").to(torch.bfloat16).flatten()


def rand_bf16(rng, shape, scale=1.0):
    return R.bf16(rng.standard_normal(shape) * scale)


@pytest.fixture(params=[1, 0], ids=["tcgen05", "mma_sync"])
def engine(request, built):
    """Run a test on both convolution engines; the tensor-core one is the
    default and is restored afterwards."""
    from lare3d_b200 import surrogate as S
    S.lib().set_engine(request.param)
    yield request.param
    assert S.lib().status(True) == 0
    S.lib().set_engine(1)


@pytest.mark.parametrize("cin,cout,pad,masked", [(16, 32, 0, False), (32, 32, 0, False), (32, 8, 0, False),
                                                 (32, 1, 0, False), (16, 32, 2, True), (32, 32, 2, True)])
@pytest.mark.parametrize("din", [9, 24])
def test_conv_kernel_fp32_output(engine, cin, cout, pad, masked, din):
    """lare_sur_conv with FP32 output against float64 on bf16 operands
    (products are exact; only the FP32 accumulation order differs)."""
    torch = torch_mod()
    from lare3d_b200 import surrogate as S
    rng = np.random.default_rng(cin * 100 + cout + pad + din)
    nb = 3 if din < 20 else 2
    dout = din - 2 + 2 * pad
    x = rand_bf16(rng, (nb, din, din, din, cin))
    w = rand_bf16(rng, (27, cout, cin), 0.2)
    bias = rng.standard_normal(cout).astype(np.float32)
    ref = R.conv(x, w, bias.astype(np.float64), pad=pad)
    # device copies stay referenced until the kernels have run
    xd, wd, bd = to_bf16_dev(x), to_bf16_dev(w), torch.from_numpy(bias).cuda()
    y = torch.empty(nb * dout ** 3 * cout, dtype=torch.float32, device="cuda")
    S.lib().conv(cin, cout, 0, 1, xd.data_ptr(), din, pad, wd.data_ptr(), bd.data_ptr(), y.data_ptr(), dout, nb,
                 None, None)
    got = y.cpu().numpy().reshape(ref.shape)
    assert rel_l2(got, ref) <= 1e-6
    if masked:
        # bf16 output with ReLU mask: exact up to the final bf16 rounding
        mask = rand_bf16(rng, ref.shape)
        md = to_bf16_dev(mask)
        yb = torch.empty(nb * dout ** 3 * cout, dtype=torch.bfloat16, device="cuda")
        S.lib().conv(cin, cout, 0, 0, xd.data_ptr(), din, pad, wd.data_ptr(), None, yb.data_ptr(), dout, nb,
                     md.data_ptr(), None)
        got = yb.float().cpu().numpy().reshape(ref.shape)
        want = R.conv(x, w, pad=pad, mask=mask)
        assert np.all(got[mask <= 0] == 0)
        assert rel_l2(got, want) <= 4e-3


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 32), (32, 16)])
def test_wgrad_kernel(built, cin, cout):
    torch = torch_mod()
    from lare3d_b200 import surrogate as S
    rng = np.random.default_rng(cin + 3 * cout)
    nb, dout = 3, 13          # 6591 voxels: several chunks and a ragged tail
    x = rand_bf16(rng, (nb, dout + 2, dout + 2, dout + 2, cin))
    dy = rand_bf16(rng, (nb, dout, dout, dout, cout))
    dw_ref, db_ref = R.wgrad(dy, x)
    L = S.lib()
    work = torch.empty(L.wgrad_work(cin, cout, dout, nb), dtype=torch.float32, device="cuda")
    dw = torch.empty(27 * cout * cin, dtype=torch.float32, device="cuda")
    db = torch.empty(cout, dtype=torch.float32, device="cuda")
    dyd, xd = to_bf16_dev(dy), to_bf16_dev(x)
    L.conv_wgrad(cin, cout, dyd.data_ptr(), xd.data_ptr(), dout + 2, dout, nb, work.data_ptr(), dw.data_ptr(),
                 db.data_ptr(), None)
    assert rel_l2(dw.cpu().numpy().reshape(dw_ref.shape), dw_ref) <= 1e-6
    assert rel_l2(db.cpu().numpy(), db_ref) <= 1e-6
    # deterministic: a second call gives the same bits
    dw2 = dw.clone()
    L.conv_wgrad(cin, cout, dyd.data_ptr(), xd.data_ptr(), dout + 2, dout, nb, work.data_ptr(), dw.data_ptr(),
                 db.data_ptr(), None)
    assert torch.equal(dw, dw2)


def test_network_gradients_match_oracle(engine):
    """Whole forward + backward (MSE loss) on 24^3 windows against the numpy
    oracle with the same bf16 rounding points."""
    torch = torch_mod()
    from lare3d_b200.surrogate import Network, LAYERS
    W, B = R.init_params(4)
    rng = np.random.default_rng(11)
    B = [(rng.standard_normal(b.shape) * 0.05).astype(np.float32) for b in B]
    W[3] = W[3] * 10.0
    nb, win = 2, 24
    x = np.zeros((nb, win, win, win, 16))
    x[..., :5] = rng.uniform(0.0, 1.0, (nb, win, win, win, 5))
    x = R.bf16(x)
    tgt = rng.standard_normal((nb, 16, 16, 16)).astype(np.float32) * 0.1
    loss, dW, dB = R.loss_and_grads(W, B, x, tgt.astype(np.float64), rounding=True)
    net = Network(seed=0)
    net.set_params(W, B)
    b = net.buffers(nb, win, True)
    b["x"].copy_(to_bf16_dev(x))
    b["tgt"].copy_(torch.from_numpy(tgt.ravel()).cuda())
    net.forward(b, nb)
    net.backward(b, nb)
    torch.cuda.synchronize()
    assert abs(net.loss.item() - loss) <= 1e-3 * loss
    for l in range(len(LAYERS)):
        assert rel_l2(net.wgrad(l).cpu().numpy(), dW[l]) <= 2e-2, l
        assert rel_l2(net.bgrad(l).cpu().numpy(), dB[l]) <= 2e-2, l


@pytest.fixture(scope="module")
def trained(built):
    """A network trained on 64^3 conduction decks (8 seeds x 4 RKL2 steps)."""
    torch = torch_mod()
    from lare3d_b200 import surrogate as S
    store, dT, dt = S.generate([1, 2, 3, 4, 5, 6, 7, 8], n=64, steps=4)
    net = S.Network(seed=0)
    net.meta["dt_scale"] = S.dt_scale_of(dT)
    net.meta["dt"] = dt
    hist = S.train(net, store, dT, iters=4000, nb=32, lr=5e-4, log_every=100)
    torch.cuda.synchronize()
    return net, dt, hist


def plain_and_surrogate(net, dt, seed, bound=1e-3, check=False):
    from lare3d_b200 import decks, gpu
    from lare3d_b200 import surrogate as S
    d = decks.conduction(64, seed=seed)
    ref = gpu.simulation(d, precision=32)
    ref.start(d.state)
    e0 = ref.get_field("energy")
    ref.conduct_heat(dt)
    sim = gpu.simulation(d, precision=32)
    sim.start(d.state)
    sc = S.SurrogateConduction(sim, d, net, dt, bound=bound, col=16, check=check, seed=seed)
    info = sc.step()
    g = (d.params.gamma - 1.0) / 2.0
    T_ref = g * ref.get_field("energy")[2:-2, 2:-2, 2:-2]
    T_sur = g * sim.get_field("energy")[2:-2, 2:-2, 2:-2]
    T_zero = g * e0[2:-2, 2:-2, 2:-2]
    sc.close()
    return T_ref, T_sur, T_zero, info


def test_training_reduces_loss(trained):
    net, dt, hist = trained
    tail = np.mean([v for _, v in hist[-5:]])
    assert tail < 0.2 * hist[0][1], hist


def test_trained_network_beats_no_network(trained):
    """What the network gains: on a held-out seed, the surrogate step's
    temperature error against plain RKL2 is far below that of the method
    without it (no conduction update, dT = 0)."""
    net, dt, _ = trained
    T_ref, T_sur, T_zero, _ = plain_and_surrogate(net, dt, seed=9)
    r_net = np.abs(T_sur - T_ref) / T_ref
    r_zero = np.abs(T_zero - T_ref) / T_ref
    e_net, e_zero = np.sqrt(np.mean(r_net ** 2)), np.sqrt(np.mean(r_zero ** 2))
    f_net, f_zero = np.mean(r_net > 1e-3), np.mean(r_zero > 1e-3)
    assert e_net < 0.5 * e_zero, (e_net, e_zero)
    assert f_net < 0.6 * f_zero, (f_net, f_zero)


def test_training_is_what_gains(trained):
    """The same network untrained (its initial weights, the trained output
    scale) against the trained one on a held-out seed: training, not the
    architecture, brings the error down (to a third, measured, for this
    short 64^3 training run).  (Against plain RKL2 the network
    gains no time at this size: RKL2 at this dt needs s >= 14 stages to be
    stable, so no cheaper plain step exists to compare at equal cost, and
    the network step itself is slower than those stages; bench.py reports
    both times.)"""
    from lare3d_b200 import surrogate as S
    net, dt, _ = trained
    raw = S.Network(seed=0)
    raw.meta.update(net.meta)
    T_ref, T_sur, _z, _ = plain_and_surrogate(net, dt, seed=9)
    _r, T_raw, _z2, _ = plain_and_surrogate(raw, dt, seed=9)
    e_net = np.sqrt(np.mean((np.abs(T_sur - T_ref) / T_ref) ** 2))
    e_raw = np.sqrt(np.mean((np.abs(T_raw - T_ref) / T_ref) ** 2))
    assert e_net < 0.5 * e_raw, (e_net, e_raw)


def test_column_recheck_is_exact_rkl2(built):
    """The window engine's RKL2 on a column plus an s+2 halo reproduces the
    whole-grid RKL2 bit for bit inside the column."""
    from lare3d_b200 import decks, gpu
    from lare3d_b200 import surrogate as S
    torch = torch_mod()
    d = decks.conduction(64, seed=5)
    ref = gpu.simulation(d, precision=32)
    ref.start(d.state)
    net = S.Network(seed=0)
    sim = gpu.simulation(d, precision=32)
    sim.start(d.state)
    sc = S.SurrogateConduction(sim, d, net, d.dt_fixed, bound=1e-3, col=16, seed=2)
    s = sim.conduction_stages(d.dt_fixed)
    sc._window(s)
    x0 = 16 - sc.halo_w
    fs, fw = S._fields(sim), S._fields(sc.win)
    import ctypes as C
    names = ("energy", "rho", "bx", "by", "bz")
    src = (C.c_void_p * 5)(*[fs[k][0] for k in names])
    dst = (C.c_void_p * 5)(*[fw[k][0] for k in names])
    _e, sx, sxy, eb = fs["energy"]
    _w, wsx, wsxy, _ = fw["energy"]
    S.lib().copy_column(eb, src, sx, sxy, 64, 64, dst, wsx, wsxy, sc.wn, sc.wn, 64, x0, x0, 5, sc.stream)
    torch.cuda.synchronize()
    sc.win.boundary_conditions()
    sc.win.conduct_heat_stages(d.dt_fixed, s)
    assert ref.conduct_heat(d.dt_fixed) == s
    e_ref = ref.get_field("energy")
    e_win = sc.win.get_field("energy")
    h = sc.halo_w
    # grid cells 16..31 (Fortran 17..32) are window cells h+1..h+16
    # energy arrays start at Fortran index -1
    a = e_ref[18:34, 18:34, 2:66]
    b = e_win[h + 2:h + 18, h + 2:h + 18, 2:66]
    assert np.array_equal(a, b)
    sc.close()


def test_rejection_and_fallback_give_plain_rkl2(built):
    """An untrained network misses the 1e-3 bound everywhere: every checked
    patch is rejected, the step falls back to plain RKL2, and the result is
    the plain RKL2 step bit for bit."""
    from lare3d_b200 import surrogate as S
    net = S.Network(seed=0)
    net.meta["dt_scale"] = 1.0
    from lare3d_b200 import decks
    d = decks.conduction(64, seed=6)
    T_ref, T_sur, _T0, info = plain_and_surrogate(net, d.dt_fixed, seed=6, check=True)
    assert info.checked == 4 and info.rejected == info.checked and info.fallback
    assert np.array_equal(T_ref, T_sur)


def test_patchwise_rejection_replaces_only_bad_patches(trained):
    """With a trained network and a loose bound some patches pass; the ones
    rejected carry the RKL2 values exactly and the accepted ones are within
    the bound."""
    net, dt, _ = trained
    T_ref, T_sur, _T0, info = plain_and_surrogate(net, dt, seed=9, bound=3e-3, check=True)
    assert info.checked == 4 and not info.fallback
    cx, cy = info.column
    for p in range(info.checked):
        a, b, c = p % 1, (p // 1) % 1, p
        sl = (slice(cx * 16, cx * 16 + 16), slice(cy * 16, cy * 16 + 16), slice(c * 16, c * 16 + 16))
        err = np.max(np.abs(T_sur[sl] - T_ref[sl]) / np.abs(T_ref[sl]))
        if info.errs[p] > 3e-3:
            assert err == 0.0
        else:
            assert err <= 3e-3 * (1 + 1e-5)
