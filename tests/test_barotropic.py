"""The barotropic (free-surface) solve on the host: the C oracle's
restatement of BODEN's u/v depths, ITPREP, TRONEU, OCVTRO and OCVTOT against
an independent numpy restatement (tests/np_restate.py), bit for bit, on a
c1 slice, a c2 box and a c4 member.  CPU only."""
import numpy as np
import pytest

import np_restate as R
import oracle as O
from orctm_b200 import configs as C
from orctm_b200 import grid

CASES = {"c1": ("c1", dict(nx=64)), "c2": ("c2", dict(nx=30, ny=23, nz=12)),
         "c4": ("c4", dict(nx=27, ny=35, nz=9))}
B = dict(O.BARO_DEFAULTS, niter=60)


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    name, over = CASES[request.param]
    inst = C.make_instance(name, builder=grid.build_grid, **over)
    return inst, O.Oracle(inst), C.make_barotropic(inst)


def _g(inst):
    return {k: inst[k] for k in ("ie", "je", "ke", "dt", "dlxp", "dlyp", "dlxu", "dlyu", "dlxv",
                                 "dlyv", "dtdxpo", "dtdyo", "dtdxuo", "dpye", "weto", "amsuo",
                                 "amsue", "dduo", "ddue")}


def test_depths_and_itprep(case):
    inst, orc, _ = case
    mv = C.barotropic_minvalue(inst)
    got = orc.deut(inst["depto"], mv)
    want = R.deut(_g(inst), inst["depto"], mv)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    got = orc.itprep(B, got[0], got[1])
    want = R.itprep(_g(inst), B, want[0], want[1])
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    assert np.all(got[3] > 0)                       # FF = 1 / (XX + ...) with XX > 0


@pytest.mark.parametrize("eta_forc", [0, 1])
def test_troneu(case, eta_forc):
    inst, orc, bt = case
    b = dict(B, eta_forc=eta_forc)
    deuto, deute, _, _ = orc.deut(inst["depto"], C.barotropic_minvalue(inst))
    tab = orc.itprep(b, deuto, deute)
    b1o, z1o = orc.troneu(b, *tab, bt["u1o"], bt["v1e"], bt["uzo"], bt["vze"])
    b1w, z1w = R.troneu(_g(inst), b, *tab, bt["u1o"], bt["v1e"], bt["uzo"], bt["vze"])
    assert np.array_equal(b1o, b1w)
    assert np.array_equal(z1o, z1w)
    assert np.abs(z1o).max() > 0
    if eta_forc:
        assert not z1o[0, :].any() and not z1o[:, -1].any()


def test_sor_converges_to_the_elevation_equation(case):
    """Enough sweeps solve XX z - UF/VF couplings = B1O on the interior."""
    inst, orc, bt = case
    b = dict(B, niter=4000, sorpar=1.5)
    deuto, deute, _, _ = orc.deut(inst["depto"], C.barotropic_minvalue(inst))
    xx, uf, vf, ff = orc.itprep(b, deuto, deute)
    b1o, z = orc.troneu(b, xx, uf, vf, ff, bt["u1o"], bt["v1e"], bt["uzo"], bt["vze"])
    I, J = slice(1, -1), slice(1, -1)
    lhs = z[I, J] / ff[I, J] - (uf[2:-1, J] * z[2:, J] + uf[1:-2, J] * z[:-2, J]
                                + vf[I, 2:-1] * z[I, 2:] + vf[I, 1:-2] * z[I, :-2])
    assert np.abs(lhs - b1o[I, J]).max() <= 1e-8 * max(np.abs(b1o).max(), 1e-30)


def test_ocvtro_and_ocvtot(case):
    inst, orc, bt = case
    deuto, deute, deutio, deutie = orc.deut(inst["depto"], C.barotropic_minvalue(inst))
    tab = orc.itprep(B, deuto, deute)
    _, z1o = orc.troneu(B, *tab, bt["u1o"], bt["v1e"], bt["uzo"], bt["vze"])
    st = C.copy_state(inst)
    uzo, vze, zo = bt["uzo"].copy(order="F"), bt["vze"].copy(order="F"), st["zo"].copy(order="F")
    uso, vse = orc.ocvtro(B, deutio, deutie, z1o, uzo, vze, zo)
    w = R.ocvtro(_g(inst), B, deutio, deutie, z1o, bt["uzo"], bt["vze"], st["zo"])
    for a, b in zip((uzo, vze, uso, vse, zo), w):
        assert np.array_equal(a, b)
    ref = R.ocvtot(_g(inst), B, uso, vse, st["uoo"], st["voe"], st["uko"], st["vke"])
    orc.ocvtot(B, uso, vse, st["uoo"], st["voe"], st["uko"], st["vke"], st["wo"])
    for k, b in zip(("uoo", "voe", "uko", "vke", "wo"), ref):
        assert np.array_equal(st[k], b), k


def test_ocbarp_and_ocwind(case):
    inst, orc, _ = case
    st = C.copy_state(inst)
    g = _g(inst)
    g["dzw"] = inst["dzw"]
    rng = np.random.default_rng(5)
    uso = np.asfortranarray(rng.standard_normal((inst["ie"] + 1, inst["je"])))
    vse = np.asfortranarray(rng.standard_normal((inst["ie"], inst["je"] + 1)))
    want = R.ocbarp(g, uso, vse)
    uzo, vze = np.zeros_like(uso), np.zeros_like(vse)
    u, v = uso.copy(order="F"), vse.copy(order="F")
    orc.ocbarp(u, v, uzo, vze)
    for a, b in zip((u, v, uzo, vze), want):
        assert np.array_equal(a, b)
    w = C.make_wind(inst)
    wu, wv = R.ocwind(g, w["txo"], w["tye"], w["sicomu"], w["sicomv"], w["tauwatu"],
                      w["tauwatv"], st["uoo"], st["voe"])
    orc.ocwind(w["txo"], w["tye"], w["sicomu"], w["sicomv"], w["tauwatu"], w["tauwatv"],
               st["uoo"], st["voe"])
    assert np.array_equal(st["uoo"], wu) and np.array_equal(st["voe"], wv)
    assert not np.array_equal(wu, C.copy_state(inst)["uoo"])


def test_trotest(case):
    """TROTEST's SORPAR: the oracle and the numpy restatement agree exactly
    (fewer tries and sweeps than the reference's 200 x 200, to stay fast)."""
    inst, orc, _ = case
    deuto, deute, _, _ = orc.deut(inst["depto"], C.barotropic_minvalue(inst))
    tab = orc.itprep(B, deuto, deute)
    got = orc.trotest(B, *tab, ntry=25, niter=30)
    want = R.trotest(_g(inst), B, *tab, ntry=25, niter=30)
    assert got == want
    assert 1.75 < got <= 1.775 + 1e-12
