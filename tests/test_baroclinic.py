"""OCTHER (with both equations of state), OCMODMOM and OCCLIT on the host:
the C oracle's restatement against an independent numpy restatement
(tests/np_restate.py), bit for bit, on a c1 slice, a c2 box and a c4 member;
the equation of state against its published check values.  CPU only."""
import ctypes as Cty

import numpy as np
import pytest

import np_restate as R
import oracle as O
from orctm_b200 import configs as C
from orctm_b200 import grid

CASES = {"c1": ("c1", dict(nx=48, nz=20)), "c2": ("c2", dict(nx=26, ny=21, nz=14)),
         "c4": ("c4", dict(nx=23, ny=29, nz=9))}
B = dict(O.BARO_DEFAULTS)


def test_equation_of_state_check_values():
    lib = O.lib()
    lib.og_adisit.restype = Cty.c_double
    lib.og_rho1.restype = Cty.c_double
    d = Cty.c_double
    # adisitj.f90:48-51: potential temperature 8.4678516 at S = 25, p = 1000
    # bar is 10 degC in situ, to 0.2 microkelvin
    assert abs(lib.og_adisit(d(8.4678516), d(25.), d(1000.)) - 10.0) < 2e-7
    # the UNESCO (1981) equation of state that RHO1J evaluates (Gill, 1982,
    # appendix 3): 1062.53817 kg/m^3 at S = 35, T = 25 degC, p = 1000 bar and
    # 1023.34306 at p = 0
    assert abs(lib.og_rho1(d(25.), d(35.), d(1000.)) - 1062.53817) < 1e-5
    assert abs(lib.og_rho1(d(25.), d(35.), d(0.)) - 1023.34306) < 1e-5
    # the numpy restatement gives the same values bit for bit
    t = np.array([8.4678516, 0.5, 29.0])
    s_ = np.array([25.0, 34.0, 36.5])
    p = np.array([1000.0, 12.3, 450.0])
    for i in range(3):
        a = lib.og_adisit(d(t[i]), d(s_[i]), d(p[i]))
        assert a == R.adisit(t[i:i + 1], s_[i:i + 1], p[i:i + 1])[0]
        assert lib.og_rho1(d(a), d(s_[i]), d(p[i])) == R.rho1(np.array([a]), s_[i:i + 1], p[i:i + 1])[0]


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    name, over = CASES[request.param]
    inst = C.make_instance(name, builder=grid.build_grid, **over)
    return inst, O.Oracle(inst)


def _g(inst):
    keys = ("ie", "je", "ke", "dt", "almzer", "dzw", "dz", "di", "tiestu", "tiestw", "dlxp", "dlyp",
            "dlxu", "dlyu", "dlxv", "dlyv", "dtdxpo", "dtdyo", "dtdxuo", "dpye", "weto", "ddpo",
            "amsuo", "amsue", "dduo", "ddue")
    return {k: inst[k] for k in keys}


def _forcing(inst, eos, ice):
    t = C.make_thermo(inst, eos=eos)
    if ice:  # sea ice exercises the EISREST / REDWMICE terms
        g = C.rng(inst["seed"] + 5)
        shp = (inst["ie"], inst["je"])
        t.update(sicomo=np.asfortranarray(g.uniform(0, 0.9, shp)),
                 sictho=np.asfortranarray(g.uniform(0, 0.5, shp)),
                 sicsno=np.asfortranarray(g.uniform(0, 0.1, shp)))
    return t


@pytest.mark.parametrize("eos,ice", [(0, False), (1, False), (0, True)])
def test_octher(case, eos, ice):
    inst, orc = case
    t = _forcing(inst, eos, ice)
    tv = O.thermo_values(inst, t)
    st = C.copy_state(inst)
    st["kcondep"] = C.initial_kcondep(inst)
    # an unstable pair of levels so that the convection counter moves
    st["tracers"][0][:, :, 1] += 3.0
    orc.octher(t, st)
    ws = C.copy_state(inst)
    ws["tracers"][0][:, :, 1] += 3.0
    kc = C.initial_kcondep(inst)
    tho, sao = ws["tracers"][0], ws["tracers"][1]
    em, rr = R.octher_surface(_g(inst), tv, tho, sao, ws["zo"])
    po, stab, rho = R.octher_column(_g(inst), tv, tho, sao, ws["zo"], ws["uko"], ws["vke"],
                                    ws["avo"], ws["dvo"], kc)
    for a, b in ((st["eminpo"], em), (st["rivrun"], rr), (st["po"], po), (st["stabio"], stab),
                 (st["rhoo"], rho), (st["tracers"][0], tho), (st["tracers"][1], sao),
                 (st["zo"], ws["zo"]), (st["avo"], ws["avo"]), (st["dvo"], ws["dvo"]),
                 (st["kcondep"], kc)):
        assert np.array_equal(a, b)
    assert (st["kcondep"] > 1).any()
    assert np.abs(st["rivrun"]).max() > 0 and np.all(st["stabio"] >= 0)


def _modmom_inputs(inst, orc):
    t = C.make_thermo(inst)
    st = C.copy_state(inst)
    st["kcondep"] = C.initial_kcondep(inst)
    orc.octher(t, st)
    orc.octimf(st["uoo"], st["voe"], st["uko"], st["vke"])
    _, _, deutio, deutie = orc.deut(inst["depto"], C.barotropic_minvalue(inst))
    return st, deutio, deutie


def test_ocmodmom(case):
    inst, orc = case
    st, deutio, deutie = _modmom_inputs(inst, orc)
    cor = C.make_coriolis(inst)
    ws = {k: np.array(v, order="F", copy=True) for k, v in st.items() if isinstance(v, np.ndarray)}
    orc.ocmodmom(B, cor, deutio, deutie, st)
    out = R.ocmodmom(_g(inst), B, cor, deutio, deutie, ws["zo"], ws["uoo"], ws["voe"], ws["uko"],
                     ws["vke"], ws["wno"], ws["po"], ws["stabio"])
    for k, a in zip(("uk1o", "vk1e", "u1o", "uso", "v1e", "vse"), out):
        assert np.array_equal(st[k], a), k
    for k in ("uko", "vke", "wno", "po", "stabio"):
        assert np.array_equal(st[k], ws[k]), k
    assert np.abs(st["uso"]).max() > 0


def test_occlit(case):
    inst, orc = case
    st, deutio, deutie = _modmom_inputs(inst, orc)
    orc.ocmodmom(B, C.make_coriolis(inst), deutio, deutie, st)
    ws = {k: np.array(st[k], order="F", copy=True) for k in ("uko", "vke", "uk1o", "vk1e", "wo", "stabio")}
    contra = orc.occlit(B, deutio, deutie, st)
    c2 = R.occlit(_g(inst), B, deutio, deutie, ws["uko"], ws["vke"], ws["uk1o"], ws["vk1e"],
                  ws["wo"], ws["stabio"])
    for k in ws:
        assert np.array_equal(st[k], ws[k]), k
    assert contra == c2
    assert 0 <= contra < 1e-3


@pytest.mark.parametrize("name,over", [("c1", dict(nx=48, nz=20)),
                                       ("c2", dict(nx=26, ny=21, nz=14, closed=True)),
                                       ("c2", dict(nx=26, ny=21, nz=14, dt=2.0)),
                                       ("c4", dict(nx=23, ny=29, nz=9, closed=True))])
def test_whole_steps_stay_bounded(name, over):
    """Twelve whole steps (the driver's order, the oracle) with wind: the
    surface stays bounded and CONTRA below the reference's 1e-3.  The c2-c5
    boxes at their own time steps (10 s on 500 m cells over 4000 m) are run
    closed: with their west and south sides open, TRONEU's explicit boundary
    row Z1O = B1O / XX (troneu.f90:67-102) makes the elevation grow tenfold per
    step there, a property of the reference's scheme; open at 2 s it is stable."""
    inst = C.make_instance(name, builder=grid.build_grid, **over)
    orc = O.Oracle(inst)
    st = C.copy_state(inst)
    st["kcondep"] = C.initial_kcondep(inst)
    t = C.make_thermo(inst)
    b = dict(B, niter=250)
    deuto, deute, deutio, deutie = orc.deut(inst["depto"], C.barotropic_minvalue(inst))
    tables = orc.itprep(b, deuto, deute)
    z0 = float(np.abs(st["zo"]).max())
    for step in range(1, 13):
        info = orc.step_full(st, t, b, C.make_coriolis(inst), (deutio, deutie), tables, step,
                             wind=C.make_wind(inst))
        assert info["contra"] < 1e-3
    assert float(np.abs(st["zo"]).max()) < 5 * z0 + 0.5
    for k in ("uoo", "voe", "wno", "pnh"):
        assert np.isfinite(st[k]).all(), k
    assert np.isfinite(st["tracers"][0]).all()
