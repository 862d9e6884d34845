"""The reference's own Sect. 3.3 experiment (an internal wave over a
Gaussian ridge in a laboratory tank; verification/Sect.3.3) on the host:
the fixture equals the reference's input files (when they are present), the
record reader refuses damaged files, the C oracle's OCTHER (UNESCO EOS, the
experiment's namelist constants), OCMODMOM and OCCLIT equal the independent
numpy restatement bit for bit on it, and whole oracle steps from its initial
state stay bounded.  CPU only."""
import os

import numpy as np
import pytest

import helpers as H
import np_restate as R
import oracle as O
from orctm_b200 import configs as C
from orctm_b200.api import read_model_records

REF = "/root/reference"
B = dict(O.BARO_DEFAULTS)


def _g(inst):
    keys = ("ie", "je", "ke", "dt", "almzer", "dzw", "dz", "di", "tiestu", "tiestw", "dlxp", "dlyp",
            "dlxu", "dlyu", "dlxv", "dlyv", "dtdxpo", "dtdyo", "dtdxuo", "dpye", "weto", "ddpo",
            "amsuo", "amsue", "dduo", "ddue")
    return {k: inst[k] for k in keys}


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "ORCTM", "verification", "Sect.3.3")),
                    reason="the reference's files are not here")
def test_fixture_equals_the_reference_files():
    import importlib.util

    spec = importlib.util.spec_from_file_location(
        "mk33", os.path.join(os.path.dirname(H.SECT33), "make_fixture.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    raw = mk.load(REF)
    f = np.load(H.SECT33)
    assert sorted(raw) == sorted(f.files)
    for k in raw:
        assert np.array_equal(np.asarray(raw[k]), f[k]), k
    # what mkgrid.f90 writes: 2 mm cells (ddx = 2.E-3), no rotation, 100 levels of 1 mm
    assert np.all(f["dlxp"] == 2.E-3) and np.all(f["dlyv"] == 2.E-3)
    assert not f["ftwou"].any() and not f["ftwov"].any()
    assert np.all(f["dzw"] == 1.E-3) and float(f["ctl_dt"]) == 2.5E-4
    assert set(np.unique(f["sao"])) == {5.0, 35.0} and np.all(f["tho"] == 10.0)


def test_reader_refuses_damaged_files(tmp_path):
    good = tmp_path / "good"
    hdr = np.array([0, 507, -100, 3], dtype=">i8").tobytes()
    vals = np.array([1.0, 2.0, 3.0], dtype=">f8").tobytes()
    rec = lambda b: np.array([len(b)], ">i4").tobytes() + b + np.array([len(b)], ">i4").tobytes()
    good.write_bytes(rec(hdr) + rec(vals))
    (h, v), = read_model_records(str(good))
    assert h == (0, 507, -100, 3) and list(v) == [1.0, 2.0, 3.0]
    bad = tmp_path / "bad"
    bad.write_bytes(rec(hdr) + rec(vals)[:-3])          # truncated
    with pytest.raises(ValueError):
        read_model_records(str(bad))
    bad.write_bytes(rec(hdr) + rec(vals[:16]))          # fewer values than the header says
    with pytest.raises(ValueError):
        read_model_records(str(bad))


@pytest.fixture(scope="module")
def sect33():
    inst = H.sect33_instance()
    thermo, cor = H.sect33_forcing()
    return inst, O.Oracle(inst), thermo, cor


def test_routines_bit_for_bit_against_numpy(sect33):
    inst, orc, thermo, cor = sect33
    tv = O.thermo_values(inst, thermo)
    st = C.copy_state(inst)
    st["kcondep"] = C.initial_kcondep(inst)
    orc.octher(thermo, st)
    ws = C.copy_state(inst)
    kc = C.initial_kcondep(inst)
    tho, sao = ws["tracers"]
    em, rr = R.octher_surface(_g(inst), tv, tho, sao, ws["zo"])
    po, stab, rho = R.octher_column(_g(inst), tv, tho, sao, ws["zo"], ws["uko"], ws["vke"],
                                    ws["avo"], ws["dvo"], kc)
    for a, b in ((st["po"], po), (st["stabio"], stab), (st["rhoo"], rho), (st["avo"], ws["avo"]),
                 (st["dvo"], ws["dvo"]), (st["kcondep"], kc), (st["tracers"][1], sao)):
        assert np.array_equal(a, b)
    # the salinity contrast makes a horizontal pressure gradient
    assert np.ptp(st["po"][:, 2, -1]) > 0
    orc.octimf(st["uoo"], st["voe"], st["uko"], st["vke"])
    _, _, deutio, deutie = orc.deut(inst["depto"], C.barotropic_minvalue(inst))
    w2 = {k: np.array(v, order="F", copy=True) for k, v in st.items() if isinstance(v, np.ndarray)}
    orc.ocmodmom(B, cor, deutio, deutie, st)
    out = R.ocmodmom(_g(inst), B, cor, deutio, deutie, w2["zo"], w2["uoo"], w2["voe"], w2["uko"],
                     w2["vke"], w2["wno"], w2["po"], w2["stabio"])
    for k, a in zip(("uk1o", "vk1e", "u1o", "uso", "v1e", "vse"), out):
        assert np.array_equal(st[k], a), k
    assert np.abs(st["uk1o"]).max() > 0
    w3 = {k: np.array(st[k], order="F", copy=True) for k in ("uko", "vke", "uk1o", "vk1e", "wo", "stabio")}
    contra = orc.occlit(B, deutio, deutie, st)
    c2 = R.occlit(_g(inst), B, deutio, deutie, w3["uko"], w3["vke"], w3["uk1o"], w3["vk1e"],
                  w3["wo"], w3["stabio"])
    for k in w3:
        assert np.array_equal(st[k], w3[k]), k
    assert contra == c2 < 1e-3


def test_whole_steps_from_the_initial_state_stay_bounded(sect33):
    inst, orc, thermo, cor = sect33
    st = C.copy_state(inst)
    st["kcondep"] = C.initial_kcondep(inst)
    b = dict(B)
    deuto, deute, deutio, deutie = orc.deut(inst["depto"], C.barotropic_minvalue(inst))
    tables = orc.itprep(b, deuto, deute)
    for step in range(1, 6):
        info = orc.step_full(st, thermo, b, cor, (deutio, deutie), tables, step)
        assert info["contra"] < 1e-3
    # the density contrast of the tank starts to move the water, slowly
    assert 0 < np.abs(st["uoo"]).max() < 0.01 and np.abs(st["zo"]).max() < 1e-3
    for k in ("uoo", "wno", "pnh", "zo"):
        assert np.isfinite(st[k]).all(), k
