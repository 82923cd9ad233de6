"""Failure detection on the GPU, without faulting, trapping or hanging it.

* Bounded waits: every streaming kernel waits on its shared-memory load ring for at most a
  fixed number of polls.  The test switch solar_gpu_inject_wait_timeout makes the chosen kernel issue
  no loads and give up after a few polls, so its first wait runs out with nothing in flight; the
  call must return SOLAR_ERR_TIMEOUT naming the kernel, and the same context (and a fresh
  one) must give the correct results afterwards.
* NaN/Inf watchdog: a non-finite value placed in the host state passed to set_state makes a
  stepping call return SOLAR_ERR_NAN naming the step; with the watchdog off the call
  succeeds, as the reference does.
* The per-step norm loop (solar_gpu_rk4_norms) gives the same values as RK4 + norm per step.
"""
import numpy as np
import pytest

from solar_b200 import _lib, configs
from solar_b200.solver import Solver

pytestmark = pytest.mark.gpu

WAIT_POLLS = 1000    # bound of the injected waits (polls of mbarrier.try_wait)


def smooth_state(cfg, seed):
    rng = np.random.default_rng(seed)
    q = np.zeros((6, 5, cfg.nr, cfg.nx, cfg.nx))
    with Solver(cfg) as s:
        for f in range(5):
            s.set_state(np.zeros_like(q))
            for _ in range(3):
                d = configs.unit_vectors(rng, 1)[0] * rng.uniform(0.6, 0.95)
                s.add_gaussian(configs.Source(tuple(d), 0.1, rng.uniform(0.5, 1.5)))
            q[:, f] = s.get_state()[:, 4]
    return q


@pytest.fixture(scope="module")
def cfg():
    return configs.c1(nx=32, nr=32)


@pytest.fixture(scope="module")
def q0(cfg):
    return smooth_state(cfg, 7)


def inject(s, kernels, polls=WAIT_POLLS):
    _lib.check(s.lib.solar_gpu_inject_wait_timeout(s._h, kernels, polls))


CASES = [
    (_lib.SOLAR_KERNEL_EDGE, "compute_rhs", "edge kernel"),
    (_lib.SOLAR_KERNEL_STAGE, "compute_rhs", "stage kernel"),
    (_lib.SOLAR_KERNEL_FILTER, "filter_exp", "filter kernel"),
    (_lib.SOLAR_KERNEL_ADJ_STAGE, "rhs_adjoint", "transposed stage kernel"),
]


@pytest.mark.parametrize("kernel,op,name", CASES, ids=[c[2].replace(" ", "_") for c in CASES])
@pytest.mark.parametrize("precision,nf", [("fp64", 5), ("fp32", 4)])
def test_wait_timeout_reported_and_context_recovers(cfg, q0, kernel, op, name, precision, nf):
    with Solver(cfg, precision=precision, nfields=nf) as s:
        want = getattr(s, op)(q0)
        inject(s, kernel)
        with pytest.raises(_lib.SolarError) as e:
            getattr(s, op)(q0)
        assert e.value.status == _lib.SOLAR_ERR_TIMEOUT
        assert name in str(e.value)
        inject(s, 0, 0)
        again = getattr(s, op)(q0)
    with Solver(cfg, precision=precision, nfields=nf) as fresh:
        fresh_out = getattr(fresh, op)(q0)
    if op == "rhs_adjoint":           # the transposed exchange adds with atomics
        tol = 1e-12 if precision == "fp64" else 1e-5
        assert np.linalg.norm(again - want) <= tol * np.linalg.norm(want)
        assert np.linalg.norm(fresh_out - want) <= tol * np.linalg.norm(want)
    else:
        np.testing.assert_array_equal(again, want)
        np.testing.assert_array_equal(fresh_out, want)


def test_wait_timeout_in_the_step_graph(cfg, q0):
    with Solver(cfg) as s:
        s.set_state(q0)
        s.rk4(2)
        want = s.get_state()
        s.set_state(q0)
        inject(s, _lib.SOLAR_KERNEL_STAGE | _lib.SOLAR_KERNEL_FILTER)
        with pytest.raises(_lib.SolarError) as e:
            s.rk4(1)
        assert e.value.status == _lib.SOLAR_ERR_TIMEOUT
        inject(s, 0, 0)
        s.set_state(q0)
        s.rk4(2)                                  # graph captured again with normal waits
        np.testing.assert_array_equal(s.get_state(), want)


def test_inject_rejects_bad_arguments(cfg):
    with Solver(cfg) as s:
        assert s.lib.solar_gpu_inject_wait_timeout(s._h, 64, 100) == _lib.SOLAR_ERR_ARG
        assert s.lib.solar_gpu_inject_wait_timeout(s._h, 1, 0) == _lib.SOLAR_ERR_ARG


@pytest.mark.parametrize("precision,nf", [("fp64", 5), ("fp32", 4)])
def test_watchdog_reports_nonfinite_state(cfg, q0, precision, nf):
    bad = q0.copy()
    bad[2, 4, 10, 5, 7] = np.nan
    with Solver(cfg, precision=precision, nfields=nf) as s:
        s.set_state(q0)
        s.set_watchdog(1)
        s.rk4(3)                                  # clean state: no report
        s.set_watchdog(0)
        s.set_state(bad)
        s.rk4(2)                                  # watchdog off: the reference's behaviour
        assert s.diag()["nonfinite"]
        s.set_state(bad)
        s.set_watchdog(2)
        with pytest.raises(_lib.SolarError) as e:
            s.rk4(3)                              # context steps 6, 7, 8: checks after 6 and 8
        assert e.value.status == _lib.SOLAR_ERR_NAN
        assert "after step 6" in str(e.value)
        s.set_state(q0)
        s.rk4(2)                                  # the report is cleared once read


def test_watchdog_rejects_negative_interval(cfg):
    with Solver(cfg) as s:
        assert s.lib.solar_gpu_set_watchdog(s._h, -1) == _lib.SOLAR_ERR_ARG


@pytest.mark.parametrize("precision,nf", [("fp64", 5), ("fp32", 4)])
def test_rk4_norms_equal_step_by_step_norms(cfg, q0, precision, nf):
    with Solver(cfg, precision=precision, nfields=nf) as a, Solver(cfg, precision=precision, nfields=nf) as b:
        a.set_state(q0)
        b.set_state(q0)
        got = a.rk4_norms(6, field=4)
        want = []
        for _ in range(6):
            b.rk4(1)
            want.append(b.norm(4))
        np.testing.assert_array_equal(got, np.array(want))
        np.testing.assert_array_equal(a.get_state(), b.get_state())
        if nf == 4:                               # rho is not stored: its norm is 0
            assert np.all(a.rk4_norms(2, field=1) == 0.0)
