"""CUDA path against the CPU restatement (oracle), routine by routine.

Tolerances: the stencil routines are compared at 1e-12 relative max-norm
(the target; both sides evaluate the reference's operation order in IEEE
binary64 without contraction, and differ by a few ulp because the kernels
divide by Newton-Raphson refinement and multiply by reciprocal metrics).  The
Poisson solve is compared with a sparse direct solve of the same operator:
relative residual <= 1e-10 and solution within 1e-9.
"""
import numpy as np
import pytest

import oracle as O
from orctm_b200 import configs as C
from orctm_b200.api import Instance

from helpers import SMALL, assert_close, instance

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module", params=sorted(SMALL))
def case(request):
    inst = instance(request.param)
    return request.param, inst


def _pair(inst):
    orc = O.Oracle(inst)
    gpu = Instance(inst)
    st = C.copy_state(inst)
    gpu.upload_state(st)
    return orc, gpu, st


def test_upload_download_roundtrip(case):
    _, inst = case
    _, gpu, st = _pair(inst)
    back = gpu.download_state()
    for k in ("uoo", "voe", "wno", "pnh", "zo", "dvo", "avo"):
        assert np.array_equal(back[k], st[k]), k
    for a, b in zip(back["tracers"], st["tracers"]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("routine", ["ocuad", "ocvad", "ocwad"])
def test_momentum_advection(case, routine):
    _, inst = case
    orc, gpu, st = _pair(inst)
    field = {"ocuad": "uoo", "ocvad": "voe", "ocwad": "wno"}[routine]
    getattr(gpu, routine)()
    if routine == "ocwad":
        orc.ocwad(st["wno"], st["uko"], st["vke"], st["wo"], st["zo"])
    else:
        getattr(orc, routine)(st[field], st["uko"], st["vke"], st["wo"])
    assert_close(gpu.download(field), st[field], TOL, routine)


def test_tracer_advection(case):
    _, inst = case
    orc, gpu, st = _pair(inst)
    for n, t in enumerate(st["tracers"]):
        gpu.ocadpo(n)
        orc.ocadpo(t, st["uko"], st["vke"], st["wo"], st["zo"])
        assert_close(gpu.download(f"tracer{n}"), t, TOL, f"ocadpo tracer {n}")


def test_tracer_advection_all_equals_one_by_one(case):
    """The fused advection of every tracer equals OCADPO called per tracer,
    bit for bit (same arithmetic per tracer; shared transports and volumes)."""
    _, inst = case
    _, one, st = _pair(inst)
    _, fused, _ = _pair(inst)
    for n in range(len(st["tracers"])):
        one.ocadpo(n)
    fused.ocadpo_all()
    for n in range(len(st["tracers"])):
        assert np.array_equal(one.download(f"tracer{n}"), fused.download(f"tracer{n}")), n


def test_async_copies_and_step_outputs_equal_synchronous(case):
    """Uploads queued on the copy stream, outputs downloaded while the step
    still runs: the same state, bit for bit, as synchronous copies."""
    _, inst = case
    _, ref, st = _pair(inst)
    ref.set_solver("fp64", rtol=1e-12, maxit=20000)
    asy = Instance(inst)
    asy.set_solver("fp64", rtol=1e-12, maxit=20000)
    src = C.copy_state(inst)
    for k in ("uoo", "voe", "wno", "uko", "vke", "wo", "uoo1", "voe1", "wno1", "pnh", "zo",
              "dvo", "avo"):
        asy.upload_async(k, np.asfortranarray(src[k]))
    for n, t in enumerate(src["tracers"]):
        asy.upload_async(f"tracer{n}", np.asfortranarray(t))
    outs = {k: np.zeros(asy.shape(k), order="F") for k in ("uoo", "voe", "wno", "pnh")}
    for n in range(asy.ntr):
        outs[f"tracer{n}"] = np.zeros(asy.shape("pnh"), order="F")
    asy.set_step_outputs(outs)
    for _ in range(2):
        ref.step_hotpath()
        asy.step_hotpath()
        asy.wait_copies()
    for k, a in outs.items():
        assert np.array_equal(a, ref.download(k)), k
    back = np.zeros(asy.shape("voe1"), order="F")
    asy.download_async("voe1", back)
    asy.wait_copies()
    assert np.array_equal(back, ref.download("voe1"))


def test_tracer_diffusion(case):
    _, inst = case
    orc, gpu, st = _pair(inst)
    gpu.octdiff()
    orc.octdiff(st["tracers"], st["dvo"], st["zo"])
    for n, t in enumerate(st["tracers"]):
        assert_close(gpu.download(f"tracer{n}"), t, TOL, f"octdiff tracer {n}")


def test_momentum_diffusion(case):
    _, inst = case
    orc, gpu, st = _pair(inst)
    gpu.ocvisc()
    orc.ocvisc(st["uoo"], st["voe"], st["wno"], st["uko"], st["vke"], st["avo"])
    for k in ("uoo", "voe", "wno", "uko", "vke"):
        assert_close(gpu.download(k), st[k], TOL, f"ocvisc {k}")


@pytest.mark.parametrize("mode", ["fp64", "fp32_refined"])
def test_nh_correction(case, mode):
    name, inst = case
    orc, gpu, st = _pair(inst)
    # the outer residual is accumulated in double-double, so a 1e-12 residual
    # target gives a solution within ~1e-12 of the direct solve
    gpu.set_solver(mode, rtol=1e-12, maxit=20000)
    stats = gpu.ocvtot_nh()
    orc.ocvtot_nh(st, solver="direct")
    assert stats["converged"] == 1 and stats["relres"] <= 1e-12, stats
    x_gpu = gpu.download("pnh")
    assert_close(x_gpu, st["pnh"], 1e-9, f"pnh ({mode})")
    for k in ("uoo", "voe", "wno", "uoo1", "voe1", "wno1", "wo"):
        assert_close(gpu.download(k), st[k], 1e-9, f"{k} after OCVTOT_NH ({mode})")


def test_solver_residual_target(case):
    """At the production target (1e-10) both solver forms reach the residual;
    the solution error is then bounded by the conditioning (checked at 1e-6
    in the relative 2-norm; the 1e-9 solution bound is checked at the 1e-12
    target by test_nh_correction)."""
    _, inst = case
    ref = None
    for mode in ("fp64", "fp32_refined"):
        orc, gpu, st = _pair(inst)
        gpu.set_solver(mode, rtol=1e-10, maxit=20000)
        stats = gpu.ocvtot_nh()
        assert stats["converged"] == 1 and stats["relres"] <= 1e-10, (mode, stats)
        if ref is None:
            orc.ocvtot_nh(st, solver="direct")
            ref = st["pnh"]
        x = gpu.download("pnh")
        err = np.linalg.norm(x - ref) / np.linalg.norm(ref)
        assert err <= 1e-6, (mode, err)


def test_step_hotpath(case):
    _, inst = case
    orc, gpu, st = _pair(inst)
    gpu.set_solver("fp64", rtol=1e-13, maxit=20000)
    for _ in range(2):
        gpu.step_hotpath()
        orc.step_hotpath(st, solver="direct")
    got = gpu.download_state()
    for k in ("uoo", "voe", "wno", "pnh"):
        assert_close(got[k], st[k], 1e-8, f"step {k}")
    for n, t in enumerate(st["tracers"]):
        assert_close(got["tracers"][n], t, 1e-10, f"step tracer {n}")


@pytest.mark.parametrize("mode", ["fp64", "fp32_refined"])
@pytest.mark.parametrize("case_name", ["c2s", "c1s", "c4deep"])
def test_solver_variants_bit_identical(case_name, mode):
    """Every column-kernel and stencil-kernel variant the autotuner chooses
    between gives the same pressure bit for bit, with the same iteration
    count, as the autotuned solve."""
    inst = instance(case_name)
    combos = [(-1, -1)] + [(c, 0) for c in range(6)] + [(0, s) for s in range(1, 9)]
    ref = None
    for c, s in combos:
        gpu = Instance(inst)
        gpu.upload_state(C.copy_state(inst))
        gpu.set_solver(mode, rtol=1e-12, maxit=20000)
        gpu.set_tuning(c, s)
        stats = gpu.ocvtot_nh()
        used = gpu.tuning(mode)
        assert all(v >= 0 for v in used), used
        if c >= 0:
            assert used == (c, s) or (c >= 2 and used[0] == 0), (used, c, s)
        got = (gpu.download("pnh"), stats["iterations"], stats["outer_iterations"])
        if ref is None:
            ref = got
        else:
            assert np.array_equal(got[0], ref[0]), (c, s)
            assert got[1:] == ref[1:], (c, s, got[1:], ref[1:])


def test_extra_snapshot_of_device_fields(case, tmp_path):
    """orctm_write_extra writes the device-resident fields in the reference's
    EXTRA layout: per level the oracle reader finds IDATE, ICODE, KCODE =
    INT(TIESTU/TIESTW) and the values rounded to float32."""
    _, inst = case
    _, gpu, st = _pair(inst)
    gpu.step_hotpath()
    fields = ["tracer0", "uko", "vke", "wo", "zo"]
    path = str(tmp_path / "snap.ext")
    gpu.write_extra(path, fields, idate=20261203)
    recs = O.read_extra(path)
    ke = inst["ke"]
    exp = []
    for k in fields:
        a = gpu.download(k)
        if k == "zo":
            exp.append((gpu.EXTRA_CODES[k], -100, a))
            continue
        nk = a.shape[2]
        for l in range(nk):
            kc = int(inst["tiestw"][l]) if k == "wo" else int(inst["tiestu"][l])
            exp.append((gpu.EXTRA_CODES[k], kc, a[:, :, l]))
    assert len(recs) == len(exp) == 4 * ke + 1 + 1
    for (idate, code, kcode, v), (ecode, ekc, ea) in zip(recs, exp):
        assert (idate, code, kcode) == (20261203, ecode, ekc)
        assert np.array_equal(v, ea.ravel(order="F").astype(np.float32))


def test_extra_restart_round_trip(case, tmp_path):
    """A snapshot written by one instance and read into another (the AUFW /
    AUFR pair): the second instance holds the first one's fields rounded to
    float32."""
    _, inst = case
    _, a, _ = _pair(inst)
    a.step_hotpath()
    _, b, _ = _pair(inst)
    fields = ["tracer0", "tracer1", "uko", "vke", "zo", "wo", "dvo", "avo"]
    path = str(tmp_path / "restart.ext")
    a.write_extra(path, fields, idate=1)
    b.read_extra(path, fields)
    for k in fields:
        want = a.download(k).astype(np.float32).astype(np.float64)
        assert np.array_equal(b.download(k), want), k
