"""Learned DROP initializer: tensor-core convolutions, network gradients and training.

The oracle (oracle/unet_oracle.py) states the network in numpy.  On the CPU its analytic
gradients are pinned against central finite differences (float64 mode).  On the GPU, through the
C ABI:
  * one convolution (tcgen05 implicit GEMM) against the oracle's convolution of the same bf16
    inputs: within one bf16 rounding of the fp32 result (2^-7 relative + 1e-3);
  * its weight gradient (fp32 accumulation over voxels): 1e-4 relative to the largest entry;
  * the whole network's parameter gradients against the oracle in bf16-emulating mode: 3e-2
    relative L2 error per layer (bf16 activations round differently when fp32 sums differ in
    order), and the loss to 1e-3 relative;
  * Adam steps on one volume lower the loss.
"""
import numpy as np
import pytest

from oracle.unet_oracle import (LAYERS, UNetOracle, bf16, bf16_bits, conv3d, conv3d_dgrad, conv3d_wgrad,
                                param_layout)


def random_params(rng, output_scale=0.3):
    offs, n = param_layout()
    p = np.zeros(n, np.float32)
    for l, (cin, cout, *_) in enumerate(LAYERS):
        o, b = offs[l]
        w = rng.normal(0, np.sqrt(2 / (27 * (2 if l == 0 else cin))), (cout, 27, cin)).astype(np.float32)
        if l == 0:
            w[:, :, 2:] = 0
        if l == len(LAYERS) - 1:
            w[1:] = 0
            w *= output_scale
        p[o:b] = w.reshape(-1)
        if l < len(LAYERS) - 1:
            p[b:b + cout] = rng.normal(0, 0.05, cout)
    return p


def volume(rng, shape):
    V = int(np.prod(shape))
    x0 = rng.uniform(0.5, 1.5, V).astype(np.float32)
    hull = (rng.uniform(size=V) < 0.7).astype(np.uint8)
    target = (x0 + rng.normal(0, 0.1, V)).astype(np.float32)
    return x0, hull, target


def test_oracle_conv_matches_direct_sum():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(3, 4, 5, 16))
    w = rng.normal(size=(16, 27, 16))
    out = conv3d(x, w)
    z, y, xx, co = 1, 0, 4, 3
    s = 0.0
    for t in range(27):
        dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
        if 0 <= z + dz < 3 and 0 <= y + dy < 4 and 0 <= xx + dx < 5:
            s += w[co, t] @ x[z + dz, y + dy, xx + dx]
    assert out[z, y, xx, co] == pytest.approx(s, rel=1e-12)
    # the data gradient is the adjoint of the convolution: <conv(x), g> = <x, dgrad(g)>
    g = rng.normal(size=out.shape)
    assert np.sum(out * g) == pytest.approx(np.sum(x * conv3d_dgrad(g, w)), rel=1e-10)
    # and the weight gradient is its adjoint in w
    assert np.sum(out * g) == pytest.approx(np.sum(w * conv3d_wgrad(x, g)), rel=1e-10)


def test_bf16_rounding_is_nearest_even():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1.0 + 2 ** -9], np.float32)
    np.testing.assert_array_equal(bf16(a), np.array([1.0, 1.0, 1.0 + 2 ** -6, -2.5, 1.0], np.float32))


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    shape = (8, 8, 8)
    p = random_params(rng).astype(np.float64)
    x0, hull, target = volume(rng, shape)
    _, g = UNetOracle(p, quantize=False).loss_and_gradients(x0, hull, target, shape)
    offs, _ = param_layout()
    picks = []
    for l in range(len(LAYERS)):  # a few parameters with nonzero gradient from every layer
        o, b = offs[l]
        nz = np.nonzero(g[o:b + LAYERS[l][1]])[0]
        picks += list(o + rng.choice(nz, min(3, len(nz)), replace=False))
    eps = 1e-6
    for i in picks:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (UNetOracle(pp, False).loss_and_gradients(x0, hull, target, shape)[0]
              - UNetOracle(pm, False).loss_and_gradients(x0, hull, target, shape)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-4 * np.abs(g).max() + 1e-4 * abs(fd), (i, fd, g[i])


# ------------------------------------------------------------------------------------- GPU --

def _to_bf16(t_np, dev):
    import torch
    return torch.from_numpy(bf16_bits(t_np).view(np.int16)).to(dev).view(torch.bfloat16)


def _from_bf16(t):
    import torch  # noqa: F401
    return (t.view(__import__("torch").int16).cpu().numpy().view(np.uint16).astype(np.uint32) << 16).view(np.float32)


CONV_CASES = [(16, 16, 0, 0, 0, 0), (16, 32, 0, 1, 0, 1), (32, 16, 0, 0, 1, 0), (64, 128, 0, 0, 0, 1),
              (128, 64, 1, 1, 0, 1), (32, 64, 1, 0, 0, 0), (128, 128, 0, 0, 1, 1), (64, 32, 1, 1, 1, 1)]


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,up,res,msk,relu", CONV_CASES)
def test_conv3d_and_weight_gradient_match_oracle(cin, cout, up, res, msk, relu):
    import torch
    from pct_reconstruction_b200.learned import conv3d as gconv, conv3d_wgrad as gwgrad
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(cin * 1000 + cout + 7 * up)
    shape = (8, 14, 20)  # 2240 voxels: 17.5 tiles of 128, so the last tile is partial
    ishape = tuple(s // 2 for s in shape) if up else shape
    x = bf16(rng.normal(0, 1, ishape + (cin,)).astype(np.float32))
    w = bf16(rng.normal(0, 0.1, (cout, 27, cin)).astype(np.float32))
    b = rng.normal(0, 0.1, cout).astype(np.float32)
    r = bf16(rng.normal(0, 1, shape + (cout,)).astype(np.float32))
    m = bf16(rng.normal(0, 1, shape + (cout,)).astype(np.float32))
    ref = conv3d(x, w, bool(up)).astype(np.float32) + b
    if res:
        ref = ref + r
    if relu:
        ref = np.maximum(ref, 0)
    if msk:
        ref = np.where(m > 0, ref, 0)
    out = gconv(_to_bf16(x, dev), cin, shape, _to_bf16(w, dev), cout, upsample=up, bias=torch.from_numpy(b).to(dev),
                residual=_to_bf16(r, dev) if res else None, mask=_to_bf16(m, dev) if msk else None, relu=relu)
    got = _from_bf16(out).reshape(shape + (cout,))
    np.testing.assert_array_less(np.abs(got - bf16(ref)), 2 ** -7 * np.abs(ref) + 1e-3)
    dz = bf16(rng.normal(0, 1, shape + (cout,)).astype(np.float32))
    dw = gwgrad(_to_bf16(x, dev), cin, shape, _to_bf16(dz, dev), cout, upsample=up).cpu().numpy()
    rw = conv3d_wgrad(x, dz, bool(up)).reshape(-1)
    assert np.abs(dw - rw).max() <= 1e-4 * np.abs(rw).max()


@pytest.mark.gpu
def test_network_gradients_match_oracle():
    import torch
    from pct_reconstruction_b200.learned import UNet
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5)
    shape = (8, 16, 24)
    p = random_params(rng)
    x0, hull, target = volume(rng, shape)
    with UNet(shape[2], shape[1], shape[0], seed=1) as net:
        net.set_params(p)
        np.testing.assert_array_equal(net.get_params(), p)
        T = [torch.from_numpy(a).to(dev) for a in (x0, hull, target)]
        loss, g = net.gradients(*T)
        y = net.forward(T[0], T[1]).cpu().numpy()
    o = UNetOracle(p, quantize=True)
    lo, go = o.loss_and_gradients(x0, hull, target, shape)
    assert loss == pytest.approx(lo, rel=1e-3)
    np.testing.assert_allclose(y, o.y.reshape(-1), atol=1e-2)
    np.testing.assert_array_equal(y[hull == 0], x0[hull == 0])  # outside the hull the start is kept
    offs, _ = param_layout()
    for l in range(len(LAYERS)):
        a, b = offs[l]
        e = b + LAYERS[l][1]
        err = np.linalg.norm(g[a:e] - go[a:e]) / np.linalg.norm(go[a:e])
        assert err < 3e-2, (l, err)


@pytest.mark.gpu
def test_untrained_network_returns_x0_and_training_lowers_loss():
    import torch
    from pct_reconstruction_b200.learned import UNet
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(9)
    shape = (8, 16, 16)
    x0, hull, _ = volume(rng, shape)
    target = (0.8 * x0 + 0.3).astype(np.float32)  # a learnable map (the noisy target has a noise floor)
    T = [torch.from_numpy(a).to(dev) for a in (x0, hull, target)]
    with UNet(shape[2], shape[1], shape[0], seed=2) as net:
        np.testing.assert_array_equal(net.forward(T[0], T[1]).cpu().numpy(), x0)  # zero output layer
        losses = [net.train_step(*T, 1e-3) for _ in range(60)]
    assert losses[-1] < 0.2 * losses[0]


WEIGHTS = __import__("pathlib").Path(__file__).resolve().parents[1] / "pct_reconstruction_b200" / "weights" / \
    "unet_200x200x32.bin"


@pytest.mark.gpu
def test_trained_network_beats_the_fbp_start_on_a_held_out_phantom():
    """What the trained network gains: on a phantom outside its training seeds (1000..1255) the
    learned start is within 1% of the FBP-started 12-iteration DROP image before any iteration,
    the FBP start is not, and the learned start's error is under a third of the FBP start's."""
    import torch
    from pct_reconstruction_b200 import Config
    from pct_reconstruction_b200 import learned as L
    cfg = Config(**L.scan_config())
    with L.UNet(cfg.COLUMNS, cfg.ROWS, cfg.SLICES) as net:
        net.load(WEIGHTS)
        _, td = L.scan_phantom(cfg, 900_123, 20_000_000, torch.device("cuda", 0))
        r = L.evaluate_scan(cfg, td, net, 12, 0.01)
    fbp0, learned0 = r["fbp"]["rel_rmse"][0], r["learned"]["rel_rmse"][0]
    print(f"start error: FBP {fbp0:.4f}, learned {learned0:.4f}; FBP needs "
          f"{r['fbp']['iterations_to_tolerance']} iterations to 1%")
    assert r["learned"]["iterations_to_tolerance"] == 0
    assert r["fbp"]["iterations_to_tolerance"] >= 1
    assert learned0 < fbp0 / 3


@pytest.mark.gpu
def test_non_finite_network_output_keeps_the_fbp_start(c1_params):
    from pct_reconstruction_b200 import Config, Context
    from pct_reconstruction_b200 import phantoms as P
    from pct_reconstruction_b200.engine import PCTError
    from pct_reconstruction_b200.learned import UNet
    cfg = Config(**dict(c1_params, SC_ON=1, SC_LOWER_THRESHOLD=-10.0, SC_UPPER_THRESHOLD=0.0))
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 40000, seed=33, continuous_angles=False,
                           angle_interval_deg=4.0, t_extent=16.0, v_extent=3.5)
    td = {k: v.numpy() for k, v in P.tracker_data(tr).items()}
    with Context(cfg) as ctx, UNet(cfg.COLUMNS, cfg.ROWS, cfg.SLICES) as net:
        ctx.preprocessing(td, integer_angles=True)
        x0 = ctx.x_GPU_2_host()
        p = net.get_params()
        p[-16:] = np.nan  # the output layer's bias
        net.set_params(p)
        with pytest.raises(PCTError):
            net.initial_iterate(ctx)
        np.testing.assert_array_equal(ctx.x_GPU_2_host(), x0)
        net.set_params(np.zeros_like(p))  # zero network: the estimate is x_0 itself
        net.initial_iterate(ctx)
        np.testing.assert_array_equal(ctx.x_GPU_2_host(), x0)
