"""The barotropic solve on the GPU against the oracle, bit for bit (the
kernels evaluate the reference's expressions in IEEE binary64 without
contraction, as the oracle does): ITPREP + TRONEU's SOR (Z1O, B1O), OCVTRO
(USO, VSE, UZO, VZE, ZO), OCVTOT (UOO, VOE, UKO, VKE, WO), OCBARP and OCWIND,
on a c1 slice,
c2 boxes (with and without OBC_ETA_FORC) and a c4 member; then c2 at its own
size, 256x256x60, with the reference's 250 sweeps."""
import numpy as np
import pytest

import oracle as O
from orctm_b200 import configs as C
from orctm_b200 import grid
from orctm_b200.api import Instance

pytestmark = pytest.mark.gpu

CASES = [("c1", dict(nx=96), 0), ("c2", dict(nx=40, ny=33, nz=24), 0),
         ("c2", dict(nx=37, ny=29, nz=18), 1), ("c4", dict(nx=50, ny=41, nz=31), 0),
         ("c2", dict(), 0)]


@pytest.mark.parametrize("name,over,eta_forc", CASES)
def test_barotropic_solve_bit_identical(name, over, eta_forc):
    inst = C.make_instance(name, builder=grid.build_grid, **over)
    orc = O.Oracle(inst)
    bt = C.make_barotropic(inst)
    mv = C.barotropic_minvalue(inst)
    b = dict(O.BARO_DEFAULTS, eta_forc=eta_forc, sorpar=1.7)
    deuto, deute, deutio, deutie = orc.deut(inst["depto"], mv)
    tab = orc.itprep(b, deuto, deute)
    st = C.copy_state(inst)
    gpu = Instance(inst)
    gpu.upload_state(st)
    gpu.set_barotropic(deuto, deute, mv, sorpar=b["sorpar"], niter=b["niter"],
                       eta_forc=bool(eta_forc))
    for rep in range(2):                      # the second call replays the SOR graph
        gpu.troneu(bt["u1o"], bt["v1e"], bt["uzo"], bt["vze"])
    b1o, z1o = orc.troneu(b, *tab, bt["u1o"], bt["v1e"], bt["uzo"], bt["vze"])
    assert np.array_equal(gpu.download_barotropic("b1o"), b1o)
    assert np.array_equal(gpu.download_barotropic("z1o"), z1o)
    gpu.ocvtro()
    uzo, vze = bt["uzo"].copy(order="F"), bt["vze"].copy(order="F")
    uso, vse = orc.ocvtro(b, deutio, deutie, z1o, uzo, vze, st["zo"])
    for k, want in (("uso", uso), ("vse", vse), ("uzo", uzo), ("vze", vze)):
        assert np.array_equal(gpu.download_barotropic(k), want), k
    assert np.array_equal(gpu.download("zo"), st["zo"])
    gpu.ocvtot()
    orc.ocvtot(b, uso, vse, st["uoo"], st["voe"], st["uko"], st["vke"], st["wo"])
    for k in ("uoo", "voe", "uko", "vke", "wo"):
        assert np.array_equal(gpu.download(k), st[k]), k
    # OCBARP on the USO / VSE that OCVTRO left, then OCWIND after OCTIMF
    # (UKO shares UOO's buffer there: the in-place update must not touch UKO)
    gpu.ocbarp()
    uzo2, vze2 = np.zeros_like(uso), np.zeros_like(vse)
    orc.ocbarp(uso, vse, uzo2, vze2)
    for k, want in (("uso", uso), ("vse", vse), ("uzo", uzo2), ("vze", vze2)):
        assert np.array_equal(gpu.download_barotropic(k), want), k
    gpu.octimf()
    orc.octimf(st["uoo"], st["voe"], st["uko"], st["vke"])
    w = C.make_wind(inst)
    gpu.ocwind(w["txo"], w["tye"], w["sicomu"], w["sicomv"], w["tauwatu"], w["tauwatv"])
    uko_before = st["uko"].copy()
    orc.ocwind(w["txo"], w["tye"], w["sicomu"], w["sicomv"], w["tauwatu"], w["tauwatv"],
               st["uoo"], st["voe"])
    for k in ("uoo", "voe"):
        assert np.array_equal(gpu.download(k), st[k]), k
    assert np.array_equal(gpu.download("uko"), uko_before)
    gpu.close()


def test_barotropic_requires_setup_and_checks_arguments():
    inst = C.make_instance("c2", builder=grid.build_grid, nx=20, ny=17, nz=8)
    gpu = Instance(inst)
    gpu.upload_state(C.copy_state(inst))
    bt = C.make_barotropic(inst)
    with pytest.raises(Exception):
        gpu.troneu(bt["u1o"], bt["v1e"], bt["uzo"], bt["vze"])
    with pytest.raises(Exception):
        gpu.ocvtot()
    d = O.Oracle(inst).deut(inst["depto"], C.barotropic_minvalue(inst))
    with pytest.raises(Exception):
        gpu.set_barotropic(d[0], d[1], 0.2, sorpar=2.5)
    with pytest.raises(ValueError):
        gpu.set_barotropic(d[1], d[0], 0.2)
    gpu.set_barotropic(d[0], d[1], 0.2)
    with pytest.raises(ValueError):
        gpu.troneu(bt["v1e"], bt["u1o"], bt["uzo"], bt["vze"])


@pytest.mark.parametrize("name,over,ntry,niter", [("c2", dict(nx=40, ny=33, nz=8), 200, 200),
                                                   ("c1", dict(nx=96), 60, 80),
                                                   ("c4", dict(nx=50, ny=41, nz=9), 40, 50)])
def test_trotest_chooses_the_oracles_sorpar(name, over, ntry, niter):
    """TROTEST on the device (the reference's 200 x 200 on a c2 box): the same
    SORPAR as the oracle, bit for bit, and TRONEU then uses it."""
    inst = C.make_instance(name, builder=grid.build_grid, **over)
    orc = O.Oracle(inst)
    mv = C.barotropic_minvalue(inst)
    deuto, deute, _, _ = orc.deut(inst["depto"], mv)
    tab = orc.itprep(O.BARO_DEFAULTS, deuto, deute)
    want = orc.trotest(O.BARO_DEFAULTS, *tab, ntry=ntry, niter=niter)
    gpu = Instance(inst)
    gpu.upload_state(C.copy_state(inst))
    gpu.set_barotropic(deuto, deute, mv)
    got = gpu.trotest(ntry, niter)
    assert got == want, (got, want)
    bt = C.make_barotropic(inst)
    gpu.troneu(bt["u1o"], bt["v1e"], bt["uzo"], bt["vze"])
    _, z1o = orc.troneu(dict(O.BARO_DEFAULTS, sorpar=want), *tab, bt["u1o"], bt["v1e"], bt["uzo"],
                        bt["vze"])
    assert np.array_equal(gpu.download_barotropic("z1o"), z1o)
