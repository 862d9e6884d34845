"""OCTHER, OCMODMOM and OCCLIT on the GPU against the oracle, bit for bit
(IEEE binary64 without contraction on both sides; the grid-angle cosines and
the wind-mixing EXP are the host's), on a c1 slice, c2 boxes (UNESCO and
linear equations of state, with sea ice) and a c4 member; then whole steps
(orctm_step_full) against the oracle's whole step: one step with the
oracle fed the GPU's pressure (so the comparison excludes the two solvers'
differences) to 1e-12, and a c1 slice over 20 steps with both sides solving."""
import numpy as np
import pytest

import oracle as O
from orctm_b200 import configs as C
from orctm_b200 import grid
from orctm_b200.api import Instance

pytestmark = pytest.mark.gpu

CASES = [("c1", dict(nx=96, nz=30), 1, False), ("c2", dict(nx=40, ny=33, nz=24), 0, False),
         ("c2", dict(nx=37, ny=29, nz=18), 0, True), ("c4", dict(nx=50, ny=41, nz=31), 1, True)]
B = dict(O.BARO_DEFAULTS, niter=60)


def _thermo(inst, eos, ice):
    t = C.make_thermo(inst, eos=eos)
    if ice:
        g = C.rng(inst["seed"] + 5)
        shp = (inst["ie"], inst["je"])
        t.update(sicomo=np.asfortranarray(g.uniform(0, 0.9, shp)),
                 sictho=np.asfortranarray(g.uniform(0, 0.5, shp)),
                 sicsno=np.asfortranarray(g.uniform(0, 0.1, shp)))
    return t


def _setup(inst, t, b=B):
    """GPU instance with the state, the thermodynamics, the Coriolis inputs and
    the barotropic set-up; the oracle's state dict and tables."""
    orc = O.Oracle(inst)
    mv = C.barotropic_minvalue(inst)
    deuto, deute, deutio, deutie = orc.deut(inst["depto"], mv)
    st = C.copy_state(inst)
    st["kcondep"] = C.initial_kcondep(inst)
    gpu = Instance(inst)
    gpu.upload_state(C.copy_state(inst))
    gpu.set_thermo(**{k: v for k, v in t.items()})
    cor = C.make_coriolis(inst)
    gpu.set_coriolis(cor["ftwou"], cor["ftwov"], cor["gila"], cor["giph"], cor["omega"])
    gpu.set_barotropic(deuto, deute, mv, sorpar=b["sorpar"], niter=b["niter"],
                       eta_forc=bool(b["eta_forc"]))
    return gpu, orc, st, cor, (deuto, deute, deutio, deutie)


def _eq(gpu_arr, want, name):
    assert gpu_arr.shape == want.shape, name
    bad = np.argwhere(gpu_arr != want)
    assert bad.size == 0, f"{name}: {len(bad)} points differ, first at {bad[0]}"


@pytest.mark.parametrize("name,over,eos,ice", CASES)
def test_octher_ocmodmom_occlit_bit_identical(name, over, eos, ice):
    inst = C.make_instance(name, builder=grid.build_grid, **over)
    t = _thermo(inst, eos, ice)
    gpu, orc, st, cor, (deuto, deute, deutio, deutie) = _setup(inst, t)
    # an unstable pair of levels: the convection counter moves
    st["tracers"][0][:, :, 1] += 3.0
    gpu.upload("tracer0", st["tracers"][0])
    gpu.octher()
    orc.octher(t, st)
    for n in (0, 1):
        _eq(gpu.download(f"tracer{n}"), st["tracers"][n], f"tracer{n}")
    for k in ("zo", "avo", "dvo"):
        _eq(gpu.download(k), st[k], k)
    for k in ("po", "stabio", "rhoo", "eminpo", "rivrun"):
        _eq(gpu.download_baroclinic(k), st[k], k)
    _eq(gpu.download_baroclinic("kcondep"), st["kcondep"].astype(np.float64), "kcondep")
    gpu.octimf()
    orc.octimf(st["uoo"], st["voe"], st["uko"], st["vke"])
    gpu.ocmodmom()
    orc.ocmodmom(B, cor, deutio, deutie, st)
    for k in ("uko", "vke", "wno"):
        _eq(gpu.download(k), st[k], k)
    for k in ("uk1o", "vk1e", "po", "stabio"):
        _eq(gpu.download_baroclinic(k), st[k], k)
    for k in ("u1o", "uso", "v1e", "vse"):
        _eq(gpu.download_barotropic(k), st[k], k)
    # UOO kept its own values although UKO shared its buffer after OCTIMF
    _eq(gpu.download("uoo"), st["uoo"], "uoo")
    contra = gpu.occlit()
    want = orc.occlit(B, deutio, deutie, st)
    for k in ("uko", "vke", "wo"):
        _eq(gpu.download(k), st[k], k)
    for k in ("uk1o", "vk1e", "stabio"):
        _eq(gpu.download_baroclinic(k), st[k], k)
    # CONTRA is summed in another order on the device
    assert abs(contra - want) <= 1e-12 * max(abs(want), 1e-300)
    gpu.close()


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name,over", [("c2", dict(nx=40, ny=33, nz=24)), ("c1", dict(nx=128, nz=40))])
def test_step_full_against_oracle_with_the_gpu_pressure(name, over):
    inst = C.make_instance(name, builder=grid.build_grid, **over)
    t = _thermo(inst, None, False)
    b = dict(B, niter=80)
    gpu, orc, st, cor, (deuto, deute, deutio, deutie) = _setup(inst, t, b)
    wind = C.make_wind(inst)
    gpu.ocwind(**wind)           # the forcing the step reuses; UOO / VOE get it once here
    orc.ocwind(wind["txo"], wind["tye"], wind["sicomu"], wind["sicomv"], wind["tauwatu"],
               wind["tauwatv"], st["uoo"], st["voe"])
    gpu.set_solver("fp64", rtol=1e-12)
    tables = orc.itprep(b, deuto, deute)
    info = gpu.step_full(1)
    pnh = gpu.download("pnh")
    want = orc.step_full(st, t, b, cor, (deutio, deutie), tables, 1, wind=wind, pnh=pnh)
    assert info["converged"] and info["contra"] < 1e-3
    assert abs(info["contra"] - want["contra"]) <= 1e-12 * max(want["contra"], 1e-300)
    for k in ("uoo", "voe", "wno", "uko", "vke", "wo", "zo"):
        assert _rel(gpu.download(k), st[k]) <= 1e-12, k
    for n in (0, 1):
        assert _rel(gpu.download(f"tracer{n}"), st["tracers"][n]) <= 1e-12, n
    for k in ("po", "stabio", "rhoo"):
        assert _rel(gpu.download_baroclinic(k), st[k]) <= 1e-12, k
    gpu.close()


def test_step_full_c1_twenty_steps():
    """The vertical slice over 20 whole steps, each side with its own solve
    (GPU PCG to 1e-12, oracle sparse LU): the fields stay within 1e-8."""
    inst = C.make_instance("c1", builder=grid.build_grid)
    t = C.make_thermo(inst)
    b = dict(B, niter=250)
    gpu, orc, st, cor, (deuto, deute, deutio, deutie) = _setup(inst, t, b)
    gpu.set_solver("fp64", rtol=1e-12)
    tables = orc.itprep(b, deuto, deute)
    worst = {}
    for step in range(1, 21):
        info = gpu.step_full(step)
        orc.step_full(st, t, b, cor, (deutio, deutie), tables, step)
        assert info["converged"]
        for k in ("uoo", "wno", "pnh", "zo"):
            worst[k] = max(worst.get(k, 0.0), _rel(gpu.download(k), st[k]))
        worst["tho"] = max(worst.get("tho", 0.0), _rel(gpu.download("tracer0"), st["tracers"][0]))
    assert all(np.isfinite(v) for v in worst.values())
    assert max(worst.values()) <= 1e-8, worst
    gpu.close()
