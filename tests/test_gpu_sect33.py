"""The reference's own Sect. 3.3 experiment (verification/Sect.3.3: its grid,
initial temperature and salinity, forcing and namelist constants, from
tests/golden/sect33/sect33.npz) on the GPU against the oracle: OCTHER,
OCMODMOM and OCCLIT bit for bit; whole steps (orctm_step_full) from the
experiment's initial state, 1 and then 20, the oracle given the GPU's
pressure, every field within 1e-12."""
import numpy as np
import pytest

import helpers as H
import oracle as O
from orctm_b200 import configs as C
from orctm_b200 import grid
from orctm_b200.api import Instance

pytestmark = pytest.mark.gpu
B = dict(O.BARO_DEFAULTS)


def _setup():
    inst = H.sect33_instance()
    thermo, cor = H.sect33_forcing()
    orc = O.Oracle(inst)
    mv = C.barotropic_minvalue(inst)
    deuto, deute = grid.uv_depths(inst["depto"])
    gpu = Instance(inst)
    gpu.upload_state(C.copy_state(inst))
    gpu.set_thermo(**thermo)
    gpu.set_coriolis(cor["ftwou"], cor["ftwov"], cor["gila"], cor["giph"], cor["omega"])
    gpu.set_barotropic(deuto, deute, mv, sorpar=B["sorpar"], niter=B["niter"])
    gpu.set_solver("fp64", rtol=1e-12)
    st = C.copy_state(inst)
    st["kcondep"] = C.initial_kcondep(inst)
    _, _, deutio, deutie = orc.deut(inst["depto"], mv)
    return inst, orc, gpu, st, thermo, cor, (deuto, deute, deutio, deutie)


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_routines_bit_identical():
    inst, orc, gpu, st, thermo, cor, (deuto, deute, deutio, deutie) = _setup()
    gpu.octher()
    orc.octher(thermo, st)
    for k in ("po", "stabio", "rhoo"):
        assert np.array_equal(gpu.download_baroclinic(k), st[k]), k
    for k in ("avo", "dvo", "zo"):
        assert np.array_equal(gpu.download(k), st[k]), k
    gpu.octimf()
    orc.octimf(st["uoo"], st["voe"], st["uko"], st["vke"])
    gpu.ocmodmom()
    orc.ocmodmom(B, cor, deutio, deutie, st)
    for k in ("uko", "vke", "wno"):
        assert np.array_equal(gpu.download(k), st[k]), k
    for k in ("uk1o", "vk1e", "po", "stabio"):
        assert np.array_equal(gpu.download_baroclinic(k), st[k]), k
    gpu.occlit()
    orc.occlit(B, deutio, deutie, st)
    for k in ("uko", "vke", "wo"):
        assert np.array_equal(gpu.download(k), st[k]), k
    gpu.close()


def test_whole_step_with_the_gpu_pressure_and_twenty_steps():
    inst, orc, gpu, st, thermo, cor, (deuto, deute, deutio, deutie) = _setup()
    tables = orc.itprep(B, deuto, deute)
    info = gpu.step_full(1)
    want = orc.step_full(st, thermo, B, cor, (deutio, deutie), tables, 1, pnh=gpu.download("pnh"))
    assert info["converged"] and info["contra"] < 1e-3
    for k in ("uoo", "voe", "wno", "wo", "zo"):
        assert _rel(gpu.download(k), st[k]) <= 1e-12, k
    for n in (0, 1):
        assert _rel(gpu.download(f"tracer{n}"), st["tracers"][n]) <= 1e-12
    gpu.close()
    # twenty steps from the initial state, the oracle given the GPU's pressure
    # at every step (the tank's 1-2 mm cells make the operator ill-conditioned
    # enough that a 1e-12 residual leaves ~1e-6 of the pressure open, so two
    # independent solves would part by that much)
    inst, orc, gpu, st, thermo, cor, (deuto, deute, deutio, deutie) = _setup()
    worst = {}
    for step in range(1, 21):
        info = gpu.step_full(step)
        orc.step_full(st, thermo, B, cor, (deutio, deutie), tables, step, pnh=gpu.download("pnh"))
        assert info["converged"]
        for k in ("uoo", "wno", "zo"):
            worst[k] = max(worst.get(k, 0.0), _rel(gpu.download(k), st[k]))
        worst["sao"] = max(worst.get("sao", 0.0), _rel(gpu.download("tracer1"), st["tracers"][1]))
    assert max(worst.values()) <= 1e-12, worst
    assert np.abs(st["uoo"]).max() > 0
    gpu.close()
