"""The learned p' preconditioner on the GPU against its numpy specification
(oracle/unet.py).

Forward: the device rounds to BF16 at the same points as the oracle and
accumulates in FP32, so outputs agree to about 1e-3 relative; the
tolerance is 2e-2 on the norm of the difference.  Backward: every layer's
weight and bias gradients agree with the oracle's to 5e-2 relative in norm
(BF16 dZ; FP32 atomics in the weight gradient).  The p' adapters are FP64
or FP32 element-wise arithmetic: 1e-6 relative.  The flexible solve keeps
plain MSI bitwise whenever the network's correction is rejected.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import unet as U  # noqa: E402

from mach2d_b200 import unet  # noqa: E402

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch, torch.device("cuda:0")


def _params(seed):
    rng = np.random.default_rng(seed)
    p = U.init_params(seed)
    layers, _, _ = U.split(np.arange(p.size))
    for _, b in layers:
        p[b] = rng.standard_normal(b.size) * 0.1
    p[-17:] = rng.standard_normal(17) * 0.3
    return p


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("n,H,W", [(2, 16, 32), (1, 24, 40)])
def test_forward_matches_oracle(n, H, W):
    torch, dev = _torch()
    p = _params(1)
    feat = np.random.default_rng(2).standard_normal((n, 11, H, W)).astype(np.float32)
    net = unet.UNet(n, H, W, params=p)
    out = torch.zeros(n, H, W, dtype=torch.float32, device=dev)
    net.forward(torch.from_numpy(feat).to(dev), out)
    torch.cuda.synchronize()
    ref, _ = U.forward(p.astype(np.float64), feat.astype(np.float64))
    assert _rel(out.cpu().numpy(), ref) < 2e-2
    net.close()


def test_tcgen05_and_mma_sync_paths_agree():
    """With every convolution that fits on the tcgen05 kernel (images 256 and
    128 wide here) against none: the mma.sync kernel accumulates the same
    16-channel, per-tap products in the same order, so the forward outputs
    agree bitwise, and the gradients up to the atomics' order."""
    torch, dev = _torch()
    n, H, W = 2, 16, 256
    p = _params(11)
    rng = np.random.default_rng(12)
    feat = torch.from_numpy(rng.standard_normal((n, 11, H, W)).astype(np.float32)).to(dev)
    t = torch.from_numpy(rng.standard_normal((n, H, W)).astype(np.float32)).to(dev)
    m = torch.ones(n, H, W, dtype=torch.float32, device=dev)
    net = unet.UNet(n, H, W, params=p)
    outs, grads, losses = [], [], []
    try:
        for mode in (2, 0):
            unet.set_tensor_path(mode)
            o = torch.zeros(n, H, W, dtype=torch.float32, device=dev)
            net.forward(feat, o)
            outs.append(o.cpu().numpy())
            losses.append(net.loss_grad(feat, t, m))
            grads.append(net.grads())
            assert net.status() == 0
    finally:
        unet.set_tensor_path(1)
    assert np.array_equal(outs[0], outs[1])
    assert abs(losses[0] / losses[1] - 1) < 1e-6      # the loss is summed with atomics
    assert _rel(grads[0], grads[1]) < 1e-5          # weight gradients use FP32 atomics
    ref, _ = U.forward(p.astype(np.float64), feat.cpu().numpy().astype(np.float64))
    assert _rel(outs[0], ref) < 2e-2
    net.close()


def test_gradients_match_oracle():
    torch, dev = _torch()
    n, H, W = 2, 16, 32
    p = _params(3)
    rng = np.random.default_rng(4)
    feat = rng.standard_normal((n, 11, H, W)).astype(np.float32)
    t = rng.standard_normal((n, H, W)).astype(np.float32)
    m = np.ones((n, H, W), dtype=np.float32)
    m[:, 13:, :] = 0.0
    m[:, :, 29:] = 0.0
    net = unet.UNet(n, H, W, params=p)
    loss = net.loss_grad(torch.from_numpy(feat).to(dev), torch.from_numpy(t).to(dev), torch.from_numpy(m).to(dev))
    g = net.grads()
    lo, go, _ = U.loss_grad(p.astype(np.float64), feat.astype(np.float64), t, m, 1.0 / m.sum())
    assert abs(loss - lo) <= 2e-2 * lo
    layers, _, _ = U.split(np.arange(p.size))
    for k, (w, b) in enumerate(layers):
        assert _rel(g[w.reshape(-1)], go[w.reshape(-1)]) < 5e-2, ("W", k)
        assert _rel(g[b], go[b]) < 5e-2, ("b", k)
    assert _rel(g[-17:], go[-17:]) < 5e-2
    net.close()


def test_training_fits_a_fixed_batch():
    torch, dev = _torch()
    n, H, W = 4, 16, 32
    rng = np.random.default_rng(5)
    feat = torch.from_numpy(rng.standard_normal((n, 11, H, W)).astype(np.float32)).to(dev)
    # a smooth target that depends on the input: a blurred first plane
    f0 = feat[:, 0].cpu().numpy()
    tt = (f0 + np.roll(f0, 1, 1) + np.roll(f0, -1, 1) + np.roll(f0, 1, 2) + np.roll(f0, -1, 2)) / 5
    t = torch.from_numpy(tt.astype(np.float32)).to(dev)
    m = torch.ones(n, H, W, dtype=torch.float32, device=dev)
    net = unet.UNet(n, H, W, seed=6)
    first = net.loss_grad(feat, t, m)
    for _ in range(150):
        net.loss_grad(feat, t, m)
        net.adam(2e-3)
    last = net.loss_grad(feat, t, m)
    assert last < 0.1 * first
    net.close()


def _pprime_system(nxr=40, nyr=20, iters=3):
    from mach2d_b200.simplec import Simplec, euler_cosine_case
    g = Simplec(euler_cosine_case(nxr, nyr))
    for _ in range(iters):
        g.iterate()
    out = g.nx, g.ny, g.field("ap"), g.field("bp"), g.field("Jp")
    g.close()
    return out


def test_adapters_match_oracle():
    torch, dev = _torch()
    nx, ny, a, b, Jp = _pprime_system()
    H, W = unet.image_shape(nx, ny)
    x = np.random.default_rng(7).standard_normal(nx * ny) * 1e-3
    da, db, dx, dJ = (torch.from_numpy(v).to(dev) for v in (a, b, x, Jp))
    r = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
    rr = torch.zeros(1, dtype=torch.float64, device=dev)
    unet.residual5(nx, ny, da, db, dx, r, rr)
    ro = U.residual5(nx, ny, a, b, x)
    assert _rel(r.cpu().numpy(), ro) < 1e-12 and abs(rr.item() / np.sum(ro * ro) - 1) < 1e-12
    feat = torch.zeros(11, H, W, dtype=torch.float32, device=dev)
    stats = torch.zeros(16, dtype=torch.float64, device=dev)
    unet.features(nx, ny, H, W, da, r, dJ, feat, stats)
    fo, (sig, mean, std) = U.features(nx, ny, H, W, a, ro, Jp)
    s = stats.cpu().numpy()
    assert abs(s[4] / sig - 1) < 1e-12 and abs(s[5] - mean) < 1e-12 * abs(mean) + 1e-12 and abs(s[6] / std - 1) < 1e-10
    assert np.max(np.abs(feat.cpu().numpy() - fo)) < 1e-6 * max(1.0, np.max(np.abs(fo)))
    y = torch.from_numpy(np.random.default_rng(8).standard_normal((H, W)).astype(np.float32)).to(dev)
    xo = torch.zeros_like(dx)
    unet.apply(nx, ny, H, W, da, db, y, stats, dx, xo)
    ref = U.apply(nx, ny, H, W, a, b, y.cpu().numpy().astype(np.float64), s[4], x)
    xg = xo.cpu().numpy()
    real = np.zeros((ny, nx), bool)
    real[1:-1, 1:-1] = True
    real = real.reshape(-1)
    assert np.array_equal(xg[real], ref[real])
    assert np.max(np.abs(xg[~real] - ref[~real])) <= 1e-13 * np.max(np.abs(ref))
    # the boundary rows carry no residual after the correction (up to ghost-ghost couplings)
    rg = U.residual5(nx, ny, a, b, xg).reshape(ny, nx)
    assert np.max(np.abs(rg[0, 1:-1])) <= 1e-12 * np.max(np.abs(b)) + 1e-300
    t = torch.zeros(H, W, dtype=torch.float32, device=dev)
    m = torch.zeros(H, W, dtype=torch.float32, device=dev)
    unet.target(nx, ny, H, W, dx, stats, t, m)
    to = np.zeros((H, W))
    to[:ny - 2, :nx - 2] = x.reshape(ny, nx)[1:-1, 1:-1] / s[4]
    assert np.max(np.abs(t.cpu().numpy() - to)) <= 1e-6 * np.max(np.abs(to))
    assert m.sum().item() == (nx - 2) * (ny - 2)


def test_flexible_solve_keeps_plain_msi_when_the_correction_is_rejected():
    torch, dev = _torch()
    nx, ny, a, b, Jp = _pprime_system()
    H, W = unet.image_shape(nx, ny)
    da, db, dJ = (torch.from_numpy(v).to(dev) for v in (a, b, Jp))
    L = unet._bind()
    work = torch.empty(L.m2d_msi_workspace_doubles(5, nx, ny), dtype=torch.float64, device=dev)
    nit = torch.zeros(2, dtype=torch.int32, device=dev)
    x_plain = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
    unet.msi5(nx, ny, 20, 1e-2, da, db, x_plain, work, nit)
    net = unet.UNet(1, H, W, seed=9)
    # a huge constant correction raises |r|: rejected
    p = net.params()
    p[-17:-1] = 0.0
    p[-1] = 1e6
    net.set_params(p)
    x = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
    rep = net.solve(nx, ny, 20, 1e-2, da, db, x, dJ, work)
    torch.cuda.synchronize()
    assert rep.accepted == 0 and rep.r1 > rep.r0
    assert torch.equal(x, x_plain)
    assert rep.nit == int(nit[0].item())
    net.close()
