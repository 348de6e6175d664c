"""The captured iteration (m2d_ctx_set_graph): each outer iteration is one
CUDA graph whose p' loop is a conditional WHILE node, with the loop exit,
p_avg, the outer norm and the next time step computed on the device.  The
kernels and the arithmetic are those of the default mode, so every report
column and every field must agree bitwise, for each solver, time stepper
and thermophysical model, and when the two modes alternate in one run."""
import json
import os

import numpy as np
import pytest

from mach2d_b200.simplec import Simplec, euler_cosine_case, n01_case
from mach2d_b200.thermo import mixture_init

pytestmark = pytest.mark.gpu
COLS = ("it", "dt", "norm", "normpl", "rmass", "fmi", "fme", "Fd", "itp_used")
FIELDS = ("u", "v", "p", "T", "ro", "pl", "Uce", "Vcn", "roe", "ron", "cp", "vle", "kn")


def _air():
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "air_species.json")))
    return mixture_init(d["base"], d["fractions"], d["Mi"], d["cpi"], d["mui"], d["kpi"])


CASES = {
    "n01_euler": lambda: n01_case(),
    "cosine_ns_ramp": lambda: euler_cosine_case(30, 14, modvis=1, Twall=900.0, dtmodel=0, dt1=1e-7, dt2=1e-6, it1=3,
                                                it2=10),
    "mixture_ns": lambda: euler_cosine_case(30, 14, modvis=1, Twall=-1.0, ktm=1, mix=_air()),
    "tdma": lambda: n01_case(solver=1, nitm_u=3, nitm_p=5),
    "fp32_sweeps": lambda: euler_cosine_case(40, 20, solver=2),
    "two_itm": lambda: n01_case(itmmax=2),
}


@pytest.mark.parametrize("name", list(CASES))
def test_graph_mode_is_bitwise_the_default_mode(name):
    a, b = Simplec(CASES[name]()), Simplec(CASES[name]())
    b.set_graph(True)
    for _ in range(25):
        ra, rb = a.iterate(), b.iterate()
        assert [getattr(ra, k) for k in COLS] == [getattr(rb, k) for k in COLS], (name, ra.it)
    for f in FIELDS:
        assert np.array_equal(a.field(f), b.field(f)), (name, f)
    for k in ("dt", "normpl", "p_avg", "it"):
        assert a.scalar(k) == b.scalar(k), k
    a.close(), b.close()


def test_modes_alternate_within_one_run():
    a, b = Simplec(n01_case()), Simplec(n01_case())
    for k in range(30):
        b.set_graph(k % 10 < 5)
        ra, rb = a.iterate(), b.iterate()
        assert [getattr(ra, c) for c in COLS] == [getattr(rb, c) for c in COLS], k
    a.close(), b.close()


def test_graph_run_stops_where_the_default_run_stops():
    a, b = Simplec(n01_case()), Simplec(n01_case())
    b.set_graph(True)
    ra, rb = a.run(3000), b.run(3000)
    assert ra.it == rb.it and ra.normpl == rb.normpl
    assert a.integrals()[3] == b.integrals()[3]
    a.close(), b.close()


def test_run_with_two_iterations_in_flight_equals_single_iterations():
    """m2d_run in graph mode queues each captured iteration before the
    previous one's scalars come back; its reports, fields and stopping
    iteration are those of one m2d_iterate at a time."""
    a = Simplec(euler_cosine_case(30, 14))
    b = Simplec(euler_cosine_case(30, 14))
    a.set_graph(True)
    b.set_graph(True)
    for _ in range(3):              # the two modes mix
        a.iterate(), b.iterate()
    ra = [a.iterate() for _ in range(37)]
    rb = b.run(37)
    assert rb.it == ra[-1].it == 40
    for c in ("dt", "norm", "normpl", "rmass", "fmi", "fme", "Fd", "itp_used"):
        assert getattr(rb, c) == getattr(ra[-1], c), c
    for f in ("u", "v", "p", "T", "ro"):
        assert np.array_equal(a.field(f), b.field(f)), f
    assert b.iterate().normpl == a.iterate().normpl
    assert a.scalar("launches") == b.scalar("launches")
    a.close(), b.close()


def test_run_stops_at_the_reference_stopping_iteration_in_graph_mode():
    c = euler_cosine_case(20, 10, tolt=1e-6)
    a, b = Simplec(c), Simplec(c)
    a.set_graph(True)
    b.set_graph(True)
    for _ in range(100000):
        r = a.iterate()
        if a.scalar("it_stop") == r.it:
            break
    assert a.scalar("it_stop") == r.it
    rb = b.run(100000)
    assert rb.it == r.it and rb.normpl == r.normpl
    assert np.array_equal(a.field("p"), b.field("p"))
    a.close(), b.close()
