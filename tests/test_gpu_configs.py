"""Parity at the configurations' own shapes and at the drop-in's
tolerances (fields within 1e-12 per step, the pressure within 1e-9 of the
exact solution at the 1e-10 residual target).

* The solve isolated: the oracle, given the pressure the GPU found, must
  reproduce every field the GPU's step writes (UOO, VOE, WNO, PNH and each
  tracer) within 1e-12 relative max-norm.  The stencils and the post-solve
  update are then checked apart from the solver, whose own bound follows.
* The solve: at the production target (relative residual 1e-10) the
  pressure must lie within 1e-9 (relative max-norm) of the exact solution of
  the same operator, for both solver forms.  The exact solution is the GPU
  solve driven to a 1e-15 residual (its outer residual is accumulated in
  double-double against the exact FP64 operator, so it converges to the
  solution, not to a conditioning-sized neighbourhood of it); on c1 and c2
  it is itself checked against the oracle's FGMRES at 1e-13 and, on c1,
  against a sparse direct solve.
* c1 (512x1x60): 200 steps, each step checked against the oracle started
  from the GPU's state with the GPU's pressure (1e-12), and the free-running
  trajectories of GPU and oracle compared step by step.
* c2 (256x256x60) and c3 (1024x1024x80): one step routine by routine in the
  driver's order, each routine's outputs at 1e-12 (c3 also gets the solve
  bound above).
"""
import numpy as np
import pytest

import oracle as O
from helpers import relerr
from orctm_b200 import configs as C
from orctm_b200 import grid
from orctm_b200.api import Instance

pytestmark = pytest.mark.gpu
TOL = 1e-12
SOLVE_TOL = 1e-9
PRODUCTION_RTOL = 1e-10
STEP_FIELDS = ("uoo", "voe", "wno", "pnh")


def _make(name, **over):
    return C.make_instance(name, builder=grid.build_grid, **over)


def _state_copy(st):
    return {k: ([t.copy() for t in v] if k == "tracers" else v.copy()) for k, v in st.items()}


def _step_errors(got, want):
    e = {k: relerr(got[k], want[k]) for k in STEP_FIELDS}
    for n, (a, b) in enumerate(zip(got["tracers"], want["tracers"])):
        e[f"tracer{n}"] = relerr(a, b)
    return e


@pytest.mark.parametrize("name,over", [("c1", {}), ("c2", {}), ("c4", dict(index=5))])
@pytest.mark.parametrize("mode", ["fp64", "fp32_refined"])
def test_step_with_solve_isolated(name, over, mode):
    """One production step (rtol 1e-10) on the GPU; the oracle steps the same
    state with the GPU's pressure: every written field within 1e-12."""
    inst = _make(name, **over)
    st = C.copy_state(inst)
    gpu = Instance(inst)
    gpu.upload_state(st)
    gpu.set_solver(mode, rtol=PRODUCTION_RTOL, maxit=20000)
    for _ in range(2):
        before = gpu.download_state()
        stats = gpu.step_hotpath()
        assert stats["converged"] == 1 and stats["relres"] <= PRODUCTION_RTOL, stats
        got = gpu.download_state()
        O.Oracle(inst).step_hotpath(before, pnh=got["pnh"])
        err = _step_errors(got, before)
        print(name, mode, {k: f"{v:.1e}" for k, v in err.items()})
        assert max(err.values()) <= TOL, err
    gpu.close()


def _exact_pressure(inst):
    g = Instance(inst)
    g.upload_state(C.copy_state(inst))
    g.set_solver("fp64", rtol=1e-15, maxit=100000)
    s = g.ocvtot_nh()
    p = g.download("pnh")
    g.close()
    return p, s


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_exact_pressure_agrees_with_oracle_krylov(name):
    inst = _make(name)
    p, s = _exact_pressure(inst)
    assert s["relres"] <= 1e-14, s
    st = C.copy_state(inst)
    orc = O.Oracle(inst)
    info = orc.ocvtot_nh(st, solver="fgmres", rtol=1e-13)
    assert info["relres"] <= 1e-13
    e = relerr(st["pnh"], p)
    print(name, "oracle FGMRES(1e-13) vs GPU exact", f"{e:.2e}")
    assert e <= 1e-10, e
    if name == "c1":
        st = C.copy_state(inst)
        orc.ocvtot_nh(st, solver="direct")
        e = relerr(st["pnh"], p)
        print(name, "direct vs GPU exact", f"{e:.2e}")
        assert e <= 1e-11, e


def _solution_errors(inst):
    exact, _ = _exact_pressure(inst)
    out = {}
    for mode in ("fp64", "fp32_refined"):
        g = Instance(inst)
        g.upload_state(C.copy_state(inst))
        g.set_solver(mode, rtol=PRODUCTION_RTOL, maxit=20000)
        s = g.ocvtot_nh()
        p = g.download("pnh")
        g.close()
        assert s["converged"] == 1 and s["relres"] <= PRODUCTION_RTOL, (mode, s)
        out[mode] = relerr(p, exact)
        print(inst["name"], mode, "relres", f"{s['relres']:.2e}", "its", s["iterations"],
              "error", f"{out[mode]:.2e}")
    return out


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_solution_within_1e9_at_production_rtol(name):
    errs = _solution_errors(_make(name))
    assert max(errs.values()) <= SOLVE_TOL, errs


def test_c1_slice_200_steps():
    """c1 at its own size: 200 production steps.  Each step equals the
    oracle's step from the GPU's state with the GPU's pressure (1e-12); the
    free-running GPU and oracle (sparse direct solve) trajectories are
    compared every step and stay within the solve's bound."""
    inst = _make("c1")
    orc = O.Oracle(inst)
    gpu = Instance(inst)
    gpu.upload_state(C.copy_state(inst))
    gpu.set_solver("fp64", rtol=PRODUCTION_RTOL, maxit=20000)
    free = C.copy_state(inst)
    worst_iso, worst_free, curve = 0.0, 0.0, []
    for n in range(200):
        before = gpu.download_state()
        stats = gpu.step_hotpath()
        assert stats["converged"] == 1, (n, stats)
        got = gpu.download_state()
        orc.step_hotpath(before, pnh=got["pnh"])
        iso = max(_step_errors(got, before).values())
        orc.step_hotpath(free, solver="direct")
        fr = max(_step_errors(got, free).values())
        worst_iso, worst_free = max(worst_iso, iso), max(worst_free, fr)
        curve.append(fr)
    print("c1 200 steps: worst per-step", f"{worst_iso:.2e}", "free-running at steps 1, 10, 50, 100, 200:",
          " ".join(f"{curve[k]:.1e}" for k in (0, 9, 49, 99, 199)))
    assert worst_iso <= TOL, worst_iso
    assert worst_free <= 1e-8, worst_free


def _routines_one_step(inst):
    """The step's routines in the driver's order on GPU and oracle, each
    routine's outputs compared; returns the worst error per routine."""
    orc = O.Oracle(inst)
    st = C.copy_state(inst)
    gpu = Instance(inst)
    gpu.upload_state(st)
    gpu.set_solver("fp64", rtol=PRODUCTION_RTOL, maxit=20000)
    errs = {}

    def cmp(routine, fields):
        e = 0.0
        for k in fields:
            if k.startswith("tracer"):
                e = max(e, relerr(gpu.download(k), st["tracers"][int(k[6:])]))
            else:
                e = max(e, relerr(gpu.download(k), st[k]))
        errs[routine] = e

    ntr = len(st["tracers"])
    trs = [f"tracer{n}" for n in range(ntr)]
    gpu.ocuad()
    orc.ocuad(st["uoo"], st["uko"], st["vke"], st["wo"])
    cmp("ocuad", ["uoo"])
    gpu.ocvad()
    orc.ocvad(st["voe"], st["uko"], st["vke"], st["wo"])
    cmp("ocvad", ["voe"])
    gpu.ocwad()
    orc.ocwad(st["wno"], st["uko"], st["vke"], st["wo"], st["zo"])
    cmp("ocwad", ["wno"])
    gpu.ocadpo_all()
    for t in st["tracers"]:
        orc.ocadpo(t, st["uko"], st["vke"], st["wo"], st["zo"])
    cmp("ocadpo", trs)
    gpu.octdiff()
    orc.octdiff(st["tracers"], st["dvo"], st["zo"])
    cmp("octdiff", trs)
    gpu.octimf()
    orc.octimf(st["uoo"], st["voe"], st["uko"], st["vke"])
    gpu.ocvisc()
    orc.ocvisc(st["uoo"], st["voe"], st["wno"], st["uko"], st["vke"], st["avo"])
    cmp("ocvisc", ["uoo", "voe", "wno", "uko", "vke"])
    stats = gpu.ocvtot_nh()
    assert stats["converged"] == 1, stats
    orc.ocvtot_nh(st, pnh=gpu.download("pnh"))
    cmp("ocvtot_nh (post-solve)", ["pnh", "uoo", "voe", "wno", "uoo1", "voe1", "wno1", "wo"])
    gpu.close()
    return errs


def test_c2_routines_at_full_shape():
    errs = _routines_one_step(_make("c2"))
    print("c2", {k: f"{v:.1e}" for k, v in errs.items()})
    assert max(errs.values()) <= TOL, errs


def test_c3_full_shape():
    """c3, 1024x1024x80 (84 M cells): the solution bound of both solver
    forms, then one step routine by routine (one instance generated)."""
    inst = _make("c3")
    errs = _solution_errors(inst)
    assert max(errs.values()) <= SOLVE_TOL, errs
    errs = _routines_one_step(inst)
    print("c3", {k: f"{v:.1e}" for k, v in errs.items()})
    assert max(errs.values()) <= TOL, errs
