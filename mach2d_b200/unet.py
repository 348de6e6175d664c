"""The learned p' preconditioner (no counterpart in the reference) behind the
C ABI: the U-Net of csrc/m2d_unet.cu, its training loop and the flexible
pressure-correction solve.

Device memory comes from torch tensors (plumbing only); every computation
is a kernel of libmach2d_b200.so.  Training pairs are harvested from the
solver itself: the p' systems the SIMPLEC iteration assembles, each paired
with its converged MSI solution.
"""
import ctypes

import numpy as np

from ._lib import check, lib

_vp, _int, _f, _d = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
CHANNELS = (16, 32, 64, 128)
# (cin, cout) of the 14 convolutions in network order
LAYERS = ((16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128), (192, 64), (64, 64),
          (96, 32), (32, 32), (48, 16), (16, 16))


class LearnedReport(ctypes.Structure):
    _fields_ = [("accepted", _int), ("r0", _d), ("r1", _d), ("nit", _int)]


def _bind():
    L = lib()
    if getattr(L, "_unet_bound", False):
        return L
    L.m2d_unet_param_count.restype = ctypes.c_long
    L.m2d_unet_create.argtypes = [_int, _int, _int, _int, ctypes.POINTER(_vp)]
    L.m2d_unet_destroy.argtypes = [_vp]
    L.m2d_unet_set_params.argtypes = [_vp, ctypes.POINTER(_f), ctypes.c_long]
    L.m2d_unet_get_params.argtypes = [_vp, ctypes.POINTER(_f), ctypes.c_long]
    L.m2d_unet_get_grads.argtypes = [_vp, ctypes.POINTER(_f), ctypes.c_long]
    L.m2d_unet_forward.argtypes = [_vp, _int, _vp, _vp, _vp]
    L.m2d_unet_loss_grad.argtypes = [_vp, _int, _vp, _vp, _vp, _f, ctypes.POINTER(_f), _vp]
    L.m2d_unet_adam.argtypes = [_vp, _f, _f, _f, _f, _vp]
    L.m2d_residual5.argtypes = [_int, _int, _vp, _vp, _vp, _vp, _vp, _vp]
    L.m2d_pprime_features.argtypes = [_int] * 4 + [_vp] * 5 + [_vp]
    L.m2d_pprime_apply.argtypes = [_int] * 4 + [_vp] * 6 + [_vp]
    L.m2d_pprime_target.argtypes = [_int] * 4 + [_vp] * 4 + [_vp]
    L.m2d_pprime_solve_learned.argtypes = [_vp, _int, _int, _int, _d] + [_vp] * 5 + [_int, _vp,
                                                                                        ctypes.POINTER(LearnedReport)]
    L.m2d_pprime_solve_cycles.argtypes = [_vp, _int, _int, _int, _int, _d] + [_vp] * 5 + [_int, _vp,
                                                                                     ctypes.POINTER(LearnedReport)]
    L.m2d_unet_set_tensor_path.argtypes = [_int]
    L.m2d_unet_status.argtypes = [_vp, ctypes.POINTER(_int)]
    L.m2d_msi_workspace_doubles.restype = ctypes.c_long
    L.m2d_msi_workspace_doubles.argtypes = [_int] * 3
    L.m2d_msi_solve_device_ws.argtypes = [_int] * 4 + [_d] + [_vp] * 4 + [ctypes.c_long, _vp, _vp, _vp, _int]
    L._unet_bound = True
    return L


def set_tensor_path(mode):
    """Which convolutions run on the tcgen05 kernel: 0 none (mma.sync); 1 (the
    default) or 2 every one whose image shape allows it (even height, width a
    multiple of 128)."""
    check(_bind().m2d_unet_set_tensor_path(int(mode)))


def param_count():
    return int(_bind().m2d_unet_param_count())


def init_params(seed):
    """He-normal convolution weights, zero biases, small head (FP32)."""
    rng = np.random.default_rng(seed)
    out = []
    for ci, co in LAYERS:
        out.append(rng.standard_normal(co * 9 * ci) * np.sqrt(2.0 / (9 * ci)))
        out.append(np.zeros(co))
    out.append(rng.standard_normal(16) * 0.25)
    out.append([0.0])
    return np.concatenate(out).astype(np.float32)


def image_shape(nx, ny):
    """Smallest H x W (multiples of 8) holding the real cells of an nx x ny system."""
    return -(-(ny - 2) // 8) * 8, -(-(nx - 2) // 8) * 8


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class UNet:
    """One network with buffers for up to `bmax` H x W images on a device."""

    def __init__(self, bmax, H, W, device=0, params=None, seed=0):
        L = _bind()
        self.bmax, self.H, self.W, self.device = bmax, H, W, device
        self._h = _vp()
        check(L.m2d_unet_create(bmax, H, W, device, ctypes.byref(self._h)))
        self.nparam = param_count()
        self.set_params(init_params(seed) if params is None else params)

    def close(self):
        if self._h:
            lib().m2d_unet_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def status(self):
        """Synchronises and returns the device error word (0: no wait ran out)."""
        flags = _int()
        lib().m2d_unet_status(self._h, ctypes.byref(flags))
        return flags.value

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().m2d_unet_set_params(self._h, p.ctypes.data_as(ctypes.POINTER(_f)), p.size))

    def _get(self, fn):
        out = np.empty(self.nparam, dtype=np.float32)
        check(fn(self._h, out.ctypes.data_as(ctypes.POINTER(_f)), out.size))
        return out

    def params(self):
        return self._get(lib().m2d_unet_get_params)

    def grads(self):
        return self._get(lib().m2d_unet_get_grads)

    def forward(self, feat, out, nimg=None, stream=None):
        """feat: device tensor [n, 11, H, W] float32; out: [n, H, W] float32."""
        n = feat.shape[0] if nimg is None else nimg
        check(lib().m2d_unet_forward(self._h, n, _ptr(feat), _ptr(out), stream))

    def loss_grad(self, feat, target, mask=None, scale=None, nimg=None, stream=None):
        n = feat.shape[0] if nimg is None else nimg
        if scale is None:
            scale = 1.0 / float(mask[:n].sum()) if mask is not None else 1.0 / (n * self.H * self.W)
        loss = _f()
        check(lib().m2d_unet_loss_grad(self._h, n, _ptr(feat), _ptr(target), _ptr(mask), float(scale),
                                       ctypes.byref(loss), stream))
        return loss.value

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        check(lib().m2d_unet_adam(self._h, lr, beta1, beta2, eps, stream))

    def solve(self, nx, ny, nitm, tol, a, b, x, Jp, work, prec=0, stream=None):
        """Flexible p' solve (m2d_pprime_solve_learned) on device tensors."""
        rep = LearnedReport()
        check(lib().m2d_pprime_solve_learned(self._h, nx, ny, nitm, tol, _ptr(a), _ptr(b), _ptr(x), _ptr(Jp),
                                             _ptr(work), prec, stream, ctypes.byref(rep)))
        return rep

    def solve_cycles(self, nx, ny, m, max_cycles, tol, a, b, x, Jp, work, prec=0, stream=None):
        """Two-level cycles (m2d_pprime_solve_cycles) on device tensors."""
        rep = LearnedReport()
        check(lib().m2d_pprime_solve_cycles(self._h, nx, ny, m, max_cycles, tol, _ptr(a), _ptr(b), _ptr(x), _ptr(Jp),
                                            _ptr(work), prec, stream, ctypes.byref(rep)))
        return rep


def features(nx, ny, H, W, a, r, Jp, feat, stats, stream=None):
    check(_bind().m2d_pprime_features(nx, ny, H, W, _ptr(a), _ptr(r), _ptr(Jp), _ptr(feat), _ptr(stats), stream))


def apply(nx, ny, H, W, a, b, y, stats, x, xout, stream=None):
    check(_bind().m2d_pprime_apply(nx, ny, H, W, _ptr(a), _ptr(b), _ptr(y), _ptr(stats), _ptr(x), _ptr(xout), stream))


def target(nx, ny, H, W, delta, stats, t, mask, stream=None):
    check(_bind().m2d_pprime_target(nx, ny, H, W, _ptr(delta), _ptr(stats), _ptr(t), _ptr(mask), stream))


def residual5(nx, ny, a, b, x, r, rr=None, stream=None):
    check(_bind().m2d_residual5(nx, ny, _ptr(a), _ptr(b), _ptr(x), _ptr(r), _ptr(rr), stream))


def msi5(nx, ny, nitm, tol, a, b, x, work, nit, prec=0, stream=None):
    """Plain device MSI solve of a 5-diagonal system (m2d_msi_solve_device_ws)."""
    L = _bind()
    check(L.m2d_msi_solve_device_ws(5, nx, ny, nitm, tol, _ptr(a), _ptr(b), _ptr(x), _ptr(work),
                                    work.numel(), stream, _ptr(nit), None, prec))


class PairSet:
    """Training pairs on the device: features [n, 11, H, W], targets and masks [n, H, W]."""

    def __init__(self, capacity, H, W, device=0):
        import torch
        dev = torch.device("cuda", device)
        self.H, self.W, self.n = H, W, 0
        self.feat = torch.zeros(capacity, 11, H, W, dtype=torch.float32, device=dev)
        self.t = torch.zeros(capacity, H, W, dtype=torch.float32, device=dev)
        self.mask = torch.zeros(capacity, H, W, dtype=torch.float32, device=dev)

    @property
    def capacity(self):
        return self.feat.shape[0]


def harvest(sim, pairs, iters_between=1, count=None, tight_nitm=400, tight_tol=1e-10, held_out=None):
    """Runs the SIMPLEC context `sim` and stores, after every `iters_between`
    outer iterations, its last p' system (ap, bp) with the converged MSI
    solution of ap delta = bp as one training pair.  With `held_out` (a
    list), the systems themselves are kept there as (ap, bp) device copies."""
    import torch
    nx, ny = sim.nx, sim.ny
    dev = pairs.feat.device
    N = nx * ny
    L = _bind()
    work = torch.empty(L.m2d_msi_workspace_doubles(5, nx, ny), dtype=torch.float64, device=dev)
    nit = torch.zeros(2, dtype=torch.int32, device=dev)
    delta = torch.zeros(N, dtype=torch.float64, device=dev)
    stats = torch.zeros(16, dtype=torch.float64, device=dev)
    Jp = torch.from_numpy(sim.field("Jp")).to(dev)
    count = pairs.capacity - pairs.n if count is None else count
    for _ in range(count):
        for _ in range(iters_between):
            sim.iterate()
        a = torch.from_numpy(sim.field("ap")).to(dev)
        b = torch.from_numpy(sim.field("bp")).to(dev)
        delta.zero_()
        msi5(nx, ny, tight_nitm, tight_tol, a, b, delta, work, nit)
        k = pairs.n
        features(nx, ny, pairs.H, pairs.W, a, b, Jp, pairs.feat[k], stats)
        target(nx, ny, pairs.H, pairs.W, delta, stats, pairs.t[k], pairs.mask[k])
        pairs.n += 1
        if held_out is not None:
            held_out.append((a, b))
    torch.cuda.synchronize(dev)
    return pairs


def harvest_systems(systems, nx, ny, Jp, pairs, tight_nitm=2000, tight_tol=1e-10):
    """Training pairs from given 5-diagonal systems [(a, b)] (device
    tensors): the features of each system's initial residual r = b (zero
    guess) and, as the target, its MSI solution to tight_tol."""
    import torch
    dev = pairs.feat.device
    L = _bind()
    work = torch.empty(L.m2d_msi_workspace_doubles(5, nx, ny), dtype=torch.float64, device=dev)
    nit = torch.zeros(2, dtype=torch.int32, device=dev)
    delta = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
    stats = torch.zeros(16, dtype=torch.float64, device=dev)
    for a, b in systems:
        if pairs.n >= pairs.capacity:
            break
        delta.zero_()
        msi5(nx, ny, tight_nitm, tight_tol, a, b, delta, work, nit)
        k = pairs.n
        features(nx, ny, pairs.H, pairs.W, a, b, Jp, pairs.feat[k], stats)
        target(nx, ny, pairs.H, pairs.W, delta, stats, pairs.t[k], pairs.mask[k])
        pairs.n += 1
    torch.cuda.synchronize(dev)
    return pairs


def train(net, pairs, steps, batch=None, lr=1e-3, seed=0, lr_final=None, log=None):
    """Adam on random minibatches of the pairs; returns the loss history."""
    import torch
    batch = min(net.bmax, pairs.n) if batch is None else batch
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    dev = pairs.feat.device
    fb = torch.empty(batch, 11, pairs.H, pairs.W, dtype=torch.float32, device=dev)
    tb = torch.empty(batch, pairs.H, pairs.W, dtype=torch.float32, device=dev)
    mb = torch.empty(batch, pairs.H, pairs.W, dtype=torch.float32, device=dev)
    for s in range(steps):
        idx = torch.randint(0, pairs.n, (batch,), generator=g).to(dev)
        torch.index_select(pairs.feat[:pairs.n], 0, idx, out=fb)
        torch.index_select(pairs.t[:pairs.n], 0, idx, out=tb)
        torch.index_select(pairs.mask[:pairs.n], 0, idx, out=mb)
        rate = lr if lr_final is None else lr * (lr_final / lr) ** (s / max(1, steps - 1))
        hist.append(net.loss_grad(fb, tb, mb))
        net.adam(rate)
        if log and (s % log == 0 or s == steps - 1):
            print(f"step {s} loss {hist[-1]:.4e}")
    return hist


def _flops_per_image(H, W):
    lv = (0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0)
    return sum(2 * (H >> l) * (W >> l) * ci * co * 9 for (ci, co), l in zip(LAYERS, lv))


def main(argv=None):
    """Times the network's kernels on random inputs:
    python -m mach2d_b200.unet {forward,train} --batch B --height H --width W --path MODE --reps K"""
    import argparse

    import torch
    ap = argparse.ArgumentParser(prog="python -m mach2d_b200.unet")
    ap.add_argument("what", choices=["forward", "train"])
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--height", type=int, default=256)
    ap.add_argument("--width", type=int, default=512)
    ap.add_argument("--path", type=int, default=1, help="tensor-path mode (set_tensor_path)")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args(argv)
    dev = torch.device("cuda:0")
    set_tensor_path(a.path)
    net = UNet(a.batch, a.height, a.width, seed=1)
    g = torch.Generator(device=dev).manual_seed(1)
    feat = torch.randn(a.batch, 11, a.height, a.width, device=dev, generator=g)
    out = torch.zeros(a.batch, a.height, a.width, device=dev)
    t = torch.randn(a.batch, a.height, a.width, device=dev, generator=g)
    m = torch.ones(a.batch, a.height, a.width, device=dev)

    def step():
        if a.what == "forward":
            net.forward(feat, out)
        else:
            net.loss_grad(feat, t, m, stream=None)
            net.adam(1e-4)
    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(1, a.reps)
    fl = a.batch * _flops_per_image(a.height, a.width) * (1 if a.what == "forward" else 3)
    print(f"{a.what} {a.batch}x{a.height}x{a.width} path {a.path}: {ms:.3f} ms, {fl / ms / 1e9:.1f} TFLOP/s, "
          f"status {net.status()}")
    net.close()


if __name__ == "__main__":
    main()
