"""Failure detection without a GPU fault: a device-side wait that runs out.

Every wait of the MSI cluster kernel (warp-to-warp hand-offs, staged copies)
and of the tcgen05 convolution is bounded in %globaltimer time; when one runs
out the kernel records ERR_SPIN_TIMEOUT, stops waiting and runs to its end,
and the host call returns M2D_ERR_TIMEOUT (4) -- the reference's only
failure check is the NaN test that stops the run (src/mach2d_main.f90:
424-436).  The test hook m2d_test_wait_hook makes the next launches of one
kernel wait once more on an mbarrier that nothing completes, bounded by a
short limit, so that this wait runs out.  The hook's wait sits where no copy
can be left in flight (the MSI kernel's other warps keep their own, much
longer bounds; the convolution's CTA has issued nothing yet), so the context
stays usable: the next call without the hook must return bitwise the result
of a call made before the fault.  Nothing here traps, faults or hangs a GPU.
"""
import ctypes

import numpy as np
import pytest

from _oracle import call as orc
from _systems import dirichlet_system
from mach2d_b200 import M2DError
from mach2d_b200._lib import call, check, lib

pytestmark = pytest.mark.gpu
LIMIT_S = 0.02


def _hook(kernel, limit_s):
    L = lib()
    L.m2d_test_wait_hook.argtypes = [ctypes.c_int, ctypes.c_double]
    check(L.m2d_test_wait_hook(kernel, limit_s))


@pytest.mark.parametrize("nd", [9, 5])
def test_msi_wait_runs_out_then_context_recovers(nd):
    nx, ny = 130, 66                       # three row groups: the cluster kernel
    a, b = dirichlet_system(nd, nx, ny, seed=41)
    name = f"m2d_msi{nd}_solve"
    x_ref = np.zeros(nx * ny)
    nit = orc(f"msi{nd}_solve", nx, ny, 20, 1e-8, a, b, x_ref)
    _hook(1, LIMIT_S)
    try:
        x = np.zeros(nx * ny)
        with pytest.raises(M2DError) as e:
            call(name, nx, ny, 20, 1e-8, a, b, x)
        assert e.value.code == 4 and "wait ran out" in str(e.value)
    finally:
        _hook(0, 0.0)
    x = np.zeros(nx * ny)
    call(name, nx, ny, 20, 1e-8, a, b, x)
    assert np.array_equal(x, x_ref) and nit >= 2


def test_iteration_reports_wait_timeout_and_continues():
    from mach2d_b200.simplec import Simplec, euler_cosine_case
    case = euler_cosine_case(60, 30)
    g, ref = Simplec(case), Simplec(case)
    r0 = ref.iterate()
    _hook(1, LIMIT_S)
    try:
        with pytest.raises(M2DError) as e:
            g.iterate()
        assert e.value.code == 4
    finally:
        _hook(0, 0.0)
    # a fresh context on the same device runs bitwise like the one before
    h = Simplec(case)
    r1 = h.iterate()
    assert (r1.it, r1.itp_used, r1.normpl, r1.norm) == (r0.it, r0.itp_used, r0.normpl, r0.norm)
    assert np.array_equal(h.field("p"), ref.field("p"))
    for s in (g, ref, h):
        s.close()


def test_tcgen05_convolution_wait_runs_out_then_recovers():
    import torch
    from mach2d_b200 import unet
    dev = torch.device("cuda:0")
    n, H, W = 1, 16, 256                   # level-0 and level-1 layers run on the tcgen05 kernel
    rng = np.random.default_rng(5)
    feat = torch.from_numpy(rng.standard_normal((n, 11, H, W)).astype(np.float32)).to(dev)
    net = unet.UNet(n, H, W, seed=3)
    unet.set_tensor_path(1)
    ref = torch.zeros(n, H, W, dtype=torch.float32, device=dev)
    net.forward(feat, ref)
    assert net.status() == 0
    _hook(2, LIMIT_S)
    try:
        out = torch.zeros(n, H, W, dtype=torch.float32, device=dev)
        net.forward(feat, out)
        assert net.status() == 8                    # ERR_SPIN_TIMEOUT, and the word is cleared
    finally:
        _hook(0, 0.0)
    out = torch.zeros(n, H, W, dtype=torch.float32, device=dev)
    net.forward(feat, out)
    assert net.status() == 0
    assert torch.equal(out, ref)
    net.close()
