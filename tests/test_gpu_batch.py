"""Batches of nozzle instances (m2d_batch_*): no counterpart in the reference.

Each instance is a full context on its own stream, so the batch must give
every instance exactly the results it gets when run alone (same kernels, same
order of operations), whatever the number of host workers; and a failing
instance must stop alone without disturbing the others.  The instances are
set up by the same worker threads; a set-up failure fails the whole batch.
"""
import numpy as np
import pytest

from mach2d_b200 import M2DError
from mach2d_b200.simplec import Batch, Simplec, euler_cosine_case, n01_case

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "p", "T", "ro", "Uce", "Vcn")
REPORT = ("it", "dt", "norm", "normpl", "rmass", "fmi", "fme", "Fd", "itp_used")


def _cases():
    # uneven grids and operating points, as in the batched workload
    return [euler_cosine_case(64, 32, p0=8.0e5, T0=900.0),
            euler_cosine_case(96, 40, Rin=2.2, Rout=1.6),
            n01_case(),
            euler_cosine_case(130, 48, Lc=1.5, Ld=3.0, p0=2.0e6, T0=1200.0),
            euler_cosine_case(48, 32)]


@pytest.mark.parametrize("workers", [1, 3, 0])
def test_batch_instances_equal_solo_runs(workers):
    iters = 12
    b = Batch(_cases(), workers=workers)
    reps = b.iterate(iters)
    for k, case in enumerate(_cases()):
        solo = Simplec(case)
        for _ in range(iters):
            r = solo.iterate()
        for c in REPORT:
            assert getattr(reps[k], c) == getattr(r, c), (k, c)
        for f in FIELDS:
            assert np.array_equal(b.instances[k].field(f), solo.field(f)), (k, f)
        assert b.instances[k].integrals()[3] == solo.integrals()[3]
        solo.close()
    b.close()


def test_batch_failure_stays_in_its_instance():
    b = Batch(_cases()[:3], workers=2)
    b.iterate(1)
    g = b.instances[2]                                  # the N01 deck
    u = g.field("u")
    u[g.nx * 5 + 7] = np.nan
    g.set_field("u", u)
    with pytest.raises(M2DError) as e:
        b.iterate(3)
    assert e.value.code == 3 and "instance 2" in str(e.value)
    import ctypes
    from mach2d_b200._lib import lib
    st = ctypes.c_int()
    for k, want in ((0, 0), (1, 0), (2, 3)):
        lib().m2d_batch_status(b._b, k, ctypes.byref(st))
        assert st.value == want, (k, st.value)
    reps = None
    with pytest.raises(M2DError):
        reps = b.iterate(2)                             # instance 2 stays stopped, others go on
    assert reps is None
    assert b.instances[0].scalar("it") == 6 and b.instances[1].scalar("it") == 6
    b.close()


def test_batch_set_up_failure_names_the_instance_and_keeps_none():
    # the instances are set up by the worker threads; one that cannot be
    # set up (fewer than 3 real volumes) fails the whole batch
    cases = _cases()
    cases[3].nxr = 2
    with pytest.raises(M2DError) as e:
        Batch(cases, workers=3)
    assert e.value.code == 2 and "instance 3" in str(e.value)
    b = Batch(_cases()[:2], workers=2)                  # the device is still usable
    assert b.iterate(1)[1].it == 1
    b.close()


def test_concurrent_captured_batch_equals_solo_runs():
    """Every instance's captured iteration in flight at once (graph mode):
    each instance still gets bitwise the results of running it alone."""
    iters = 10
    b = Batch(_cases(), workers=1)
    for s in b.instances:
        s.set_graph(True)
    reps = b.iterate(iters)
    for k, case in enumerate(_cases()):
        solo = Simplec(case)
        for _ in range(iters):
            r = solo.iterate()
        for c in REPORT:
            assert getattr(reps[k], c) == getattr(r, c), (k, c)
        for f in FIELDS:
            assert np.array_equal(b.instances[k].field(f), solo.field(f)), (k, f)
        solo.close()
    b.close()


@pytest.mark.parametrize("solver,variants", [(0, (0, 1, 2, 3)), (2, (0, 1, 2))])
def test_msi_schedules_give_the_same_iterates(solver, variants):
    case = euler_cosine_case(96, 70, solver=solver)          # three row groups of 32
    runs = []
    for v in variants:
        g = Simplec(case)
        g.set_msi_schedule(v)
        g.set_graph(v % 2 == 0)
        reps = [g.iterate() for _ in range(6)]
        runs.append(([tuple(getattr(r, c) for c in REPORT) for r in reps], [g.field(f) for f in FIELDS]))
        g.close()
    for hist, fields in runs[1:]:
        assert hist == runs[0][0]
        for a, b in zip(fields, runs[0][1]):
            assert np.array_equal(a, b)


def test_autotuned_batch_equals_untuned_batch():
    cases = _cases()
    tuned = Batch(cases, workers=2)
    plain = Batch(cases, workers=2)
    for s in tuned.instances + plain.instances:
        s.set_graph(True)
    chosen, ms = tuned.autotune(1)
    assert chosen in ms and set(ms) == {1, 2, 3}
    done = int(tuned.instances[0].scalar("it"))
    assert done == 2 * len(ms)
    r_t = tuned.iterate(4)
    r_p = plain.iterate(done + 4)
    for k in range(len(cases)):
        for c in REPORT:
            assert getattr(r_t[k], c) == getattr(r_p[k], c), (k, c)
        for f in FIELDS:
            assert np.array_equal(tuned.instances[k].field(f), plain.instances[k].field(f)), (k, f)
        assert tuned.instances[k].scalar("msi_schedule") == chosen
    tuned.close()
    plain.close()
