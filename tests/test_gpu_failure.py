"""Failure paths on the GPU, made on the host (no fault, trap or hang):
a solve stopped by its iteration limit, a NaN in the input, and a served
request that fails at run time while the others carry on.

The reference's PETSc solve returns its last iterate when it stops early
(mo_petsc.f90:216-232); OCVTOT_NH then applies it.  The library does the
same and says so: ORCTM_E_NOT_CONVERGED with the residual in
orctm_solve_stats, the state updated from the iterate it has."""
import ctypes as Cc
import time

import numpy as np
import pytest

import oracle as O
from helpers import assert_close, instance
from orctm_b200 import _lib, grid
from orctm_b200 import configs as C
from orctm_b200.api import Instance
from orctm_b200.serve import Job, Server

pytestmark = pytest.mark.gpu


def _solve_status(gpu):
    s = _lib.SolveStats()
    st = gpu.lib.orctm_ocvtot_nh(gpu.h, Cc.byref(s))
    return st, s.as_dict()


@pytest.mark.parametrize("mode", ["fp64", "fp32_refined"])
def test_iteration_limit_returns_not_converged_and_updates_state(mode):
    inst = instance("c2s")
    gpu = Instance(inst)
    st = C.copy_state(inst)
    gpu.upload_state(st)
    gpu.set_solver(mode, rtol=1e-12, maxit=3)
    status, stats = _solve_status(gpu)
    assert status == _lib.ORCTM_E_NOT_CONVERGED
    assert stats["converged"] == 0
    assert 1 <= stats["iterations"] <= 3 + 1, stats
    assert np.isfinite(stats["relres"]) and 1e-12 < stats["relres"] < stats["relres_initial"]
    # the iterate was applied: PNH, the corrected velocities and WNO are the
    # oracle's post-solve update of that same pressure
    pnh = gpu.download("pnh")
    assert np.isfinite(pnh).all() and np.abs(pnh).max() > 0
    O.Oracle(inst).ocvtot_nh(st, pnh=pnh)
    for k in ("pnh", "uoo", "voe", "wno", "uoo1", "voe1", "wno1", "wo"):
        assert_close(gpu.download(k), st[k], 1e-12, k)
    assert b"residual target" in _lib.load().orctm_status_string(status)


@pytest.mark.parametrize("field", ["uoo", "pnh"])
def test_nan_input_stops_the_solve(field):
    """A NaN in a velocity (right-hand side) or in the warm start (the
    residual) stops the solve at once with a non-zero status; it neither
    spins to the iteration limit nor reports convergence."""
    inst = instance("c2s")
    gpu = Instance(inst)
    st = C.copy_state(inst)
    bad = np.array(st[field], order="F")
    bad[bad.shape[0] // 2, bad.shape[1] // 2, 1] = np.nan
    st[field] = bad
    gpu.upload_state(st)
    gpu.set_solver("fp64", rtol=1e-10, maxit=5000)
    t = time.time()
    status, stats = _solve_status(gpu)
    assert status == _lib.ORCTM_E_NOT_CONVERGED
    assert stats["converged"] == 0
    assert stats["iterations"] == 0, stats
    assert not (stats["relres"] <= 1e-10)
    assert time.time() - t < 10.0
    # the handle stays usable: a clean state converges afterwards
    gpu.upload_state(C.copy_state(inst))
    status, stats = _solve_status(gpu)
    assert status == 0 and stats["converged"] == 1


def test_served_request_failing_at_run_time_is_isolated():
    """A request whose state holds a NaN fails in its first step (status
    ORCTM_E_NOT_CONVERGED, no step completed) while the requests beside it
    complete bit-identical to running alone."""
    specs = [dict(nx=40, ny=33, nz=24), dict(nx=57, ny=21, nz=31), dict(nx=33, ny=48, nz=17)]
    insts = [C.make_instance("c4", index=k, builder=grid.build_grid, **sp)
             for k, sp in enumerate(specs)]
    nsteps = 2

    def alone(inst):
        g = Instance(inst)
        g.upload_state(C.copy_state(inst))
        g.set_solver("fp64", rtol=1e-10, maxit=5000)
        for _ in range(nsteps):
            g.step_hotpath()
        out = {k: g.download(k) for k in ("uoo", "voe", "wno", "pnh")}
        g.close()
        return out

    want = [alone(i) for i in insts[:2]]
    bad_state = C.copy_state(insts[2])
    u = np.array(bad_state["uoo"], order="F")
    u[u.shape[0] // 2, u.shape[1] // 2, 0] = np.nan
    bad_state["uoo"] = u
    with Server(slots=3, solver="fp64", rtol=1e-10, maxit=5000) as srv:
        good = [srv.submit(Job(i, C.copy_state(i), nsteps)) for i in insts[:2]]
        bad = srv.submit(Job(insts[2], bad_state, nsteps))
        for j in good + [bad]:
            srv.wait(j)
        tot = srv.stats()
    assert bad.stats["status"] == _lib.ORCTM_E_NOT_CONVERGED
    assert bad.stats["steps_done"] == 0
    assert tot["failed"] == 1 and tot["completed"] == 2
    for j, w in zip(good, want):
        assert j.stats["status"] == 0
        for k, v in w.items():
            assert np.array_equal(j.outputs()[k], v), k
