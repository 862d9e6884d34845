"""Open-boundary tide forcing and sponge on the GPU (orctm_set_obc,
orctm_obc_eta, orctm_obc_uv, orctm_obc_ts, orctm_set_obc_sponge_exp)
against the oracle's restatement of mo_obcs.f90, on the reference's W+S
layout and on every-side layouts with crossing, uneven, unsponged and
zero-relaxation bands, in the 1/x and the exponential form.  The kernels and the
oracle evaluate the same expressions in the same order; they differ only
through COS (CUDA's cos against the C library's), hence the 1e-13 bound.
Also: a buffer shared with UKO after OCTIMF, and pending downloads, keep
their contents."""
import numpy as np
import pytest

import oracle as O
from helpers import assert_close
from orctm_b200 import configs as C
from orctm_b200.api import Instance
from test_obc import CASES, _case, _exp_case

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _pair(inst, obc):
    orc = O.Oracle(inst)
    gpu = Instance(inst)
    st = C.copy_state(inst)
    gpu.upload_state(st)
    gpu.set_obc(obc)
    return orc, gpu, st


@pytest.mark.parametrize("kind", CASES)
def test_obc_uv_parity(kind):
    inst, obc = _case(kind)
    orc, gpu, st = _pair(inst, obc)
    for step in (1, 4321, 100000):
        gpu.obc_uv(step)
        orc.obc_uv(obc, step, st["uoo"], st["voe"])
        assert_close(gpu.download("uoo"), st["uoo"], TOL, f"UOO step {step}")
        assert_close(gpu.download("voe"), st["voe"], TOL, f"VOE step {step}")


@pytest.mark.parametrize("kind", CASES)
def test_obc_eta_parity(kind):
    inst, obc = _case(kind)
    orc, gpu, st = _pair(inst, obc)
    for step in (3, 86400):
        gpu.obc_eta(step)
        orc.obc_eta(obc, step, st["zo"])
        assert_close(gpu.download("zo"), st["zo"], TOL, f"ZO step {step}")


def test_obc_then_step_matches_oracle():
    """The driver's order (orctm.f90:1358-1369, 1454-1562): sponge, OCTIMF,
    then the hot path, on the c2 layout."""
    inst, obc = _case("reference")
    orc, gpu, st = _pair(inst, obc)
    gpu.obc_uv(10)
    gpu.octimf()
    orc.obc_uv(obc, 10, st["uoo"], st["voe"])
    orc.octimf(st["uoo"], st["voe"], st["uko"], st["vke"])
    for k in ("uoo", "voe", "uko", "vke"):
        assert_close(gpu.download(k), st[k], TOL, k)
    gpu.set_solver("fp64", rtol=1e-13, maxit=20000)
    gpu.step_hotpath()
    orc.step_hotpath(st, solver="direct")
    for k in ("uoo", "voe", "wno", "pnh"):
        assert_close(gpu.download(k), st[k], 1e-8, k)


def test_shared_and_held_buffers_keep_their_contents():
    inst, obc = _case("crossing")
    _, gpu, st = _pair(inst, obc)
    gpu.octimf()                       # UKO, VKE now share UOO's, VOE's buffers
    u_before = gpu.download("uoo")
    held = np.zeros(gpu.shape("voe"), order="F")
    gpu.download_async("voe", held)    # pending download of VOE
    z_held = np.zeros(gpu.shape("zo"), order="F")
    gpu.download_async("zo", z_held)   # pending download of ZO
    gpu.obc_uv(50)
    gpu.obc_eta(50)
    gpu.wait_copies()
    assert np.array_equal(gpu.download("uko"), u_before)
    assert np.array_equal(held, st["voe"])
    assert np.array_equal(z_held, st["zo"])
    assert not np.array_equal(gpu.download("uoo"), u_before)
    assert not np.array_equal(gpu.download("zo"), st["zo"])


def test_set_obc_rejects_bad_arguments():
    inst, obc = _case("reference")
    gpu = Instance(inst)
    with pytest.raises(Exception):
        gpu.obc_uv(1)                  # constants not set
    bad = dict(obc, width=[0, 1, 1, 1])
    with pytest.raises(Exception):
        gpu.set_obc(bad)
    bad = dict(obc, width=[inst["ie"] + 1, 1, 1, 1])
    with pytest.raises(Exception):
        gpu.set_obc(bad)
    bad = dict(obc, ntide=9)
    with pytest.raises(Exception):
        gpu.set_obc(bad)
    amp = [list(r) for r in obc["amp"]]
    amp[0][1] = None
    with pytest.raises(Exception):
        gpu.set_obc(dict(obc, amp=amp))
    with pytest.raises(Exception):
        gpu.set_obc_sponge_exp(3600.0)     # constants not set
    gpu.set_obc(obc)
    with pytest.raises(Exception):
        gpu.set_obc_sponge_exp(float("inf"))


@pytest.mark.parametrize("kind", CASES)
def test_obc_ts_parity(kind):
    """FORC_OBCS_TS + SPONGE_OBCS_TS on THO and SAO: the same expressions as
    the oracle and no transcendental function, so equal bit for bit."""
    inst, obc = _case(kind)
    orc, gpu, st = _pair(inst, obc)
    cli = [C.make_obc_ts(inst, n) for n in (0, 1)]
    for n in (0, 1):
        gpu.set_obc_ts(n, cli[n])
    for _ in range(2):
        gpu.obc_ts()
        for n in (0, 1):
            orc.obc_ts(obc, cli[n], st["tracers"][n])
    for n in (0, 1):
        got = gpu.download(f"tracer{n}")
        assert np.array_equal(got, st["tracers"][n]), (n, float(np.abs(got - st["tracers"][n]).max()))
    # the passive tracer has no boundary forcing
    assert np.array_equal(gpu.download("tracer2"), st["tracers"][2])


def test_obc_ts_keeps_pending_download_and_needs_records():
    inst, obc = _case("reference")
    _, gpu, st = _pair(inst, obc)
    with pytest.raises(Exception):
        gpu.obc_ts()                   # no record set
    gpu.set_obc_ts(0, C.make_obc_ts(inst, 0))
    held = np.zeros(gpu.shape("pnh"), order="F")
    gpu.download_async("tracer0", held)
    gpu.obc_ts()
    gpu.wait_copies()
    assert np.array_equal(held, st["tracers"][0])
    assert not np.array_equal(gpu.download("tracer0"), st["tracers"][0])
    gpu.set_obc(obc)                   # discards the records
    with pytest.raises(Exception):
        gpu.obc_ts()


def test_reference_sect35_files_drive_the_sponges():
    """The reference's own Sect. 3.5 boundary files (tests/golden/sect35)
    on a grid of that experiment's size (IE = 4000, JE = 5, KE = 300; W and
    E open, 30-cell sponges, relaxation times of its OCECTL): the u/v tide
    sponge and the T/S climatology sponge accept them and match the oracle
    (1e-13 for u/v, whose tidal sums call COS; bit for bit for T/S)."""
    from orctm_b200 import api, grid
    from test_reference_fixtures import HERE, JE, KE, NTIDE, OB, PERIODS

    inst = C.make_instance("c2", builder=grid.build_grid, nx=4000 - 2, ny=JE - 2, nz=KE)
    inst["ob"] = dict(OB)
    amp, pha = api.read_obc_files(HERE, inst["ie"], inst["je"], OB, NTIDE, variables=(1, 2))
    for b in (0, 1):             # OBC_ETA_FORC off: the elevation constants stay zero
        amp[b][0] = np.zeros((JE, NTIDE), order="F")
        pha[b][0] = np.zeros((JE, NTIDE), order="F")
    obc = {"ntide": NTIDE, "period": np.array(PERIODS), "sponge": [1, 1, 0, 0],
           "width": [30, 30, 1, 1], "relax_inner": 44714.1643, "relax_bound": 2.0,
           "amp": amp, "pha": pha}
    orc, gpu, st = _pair(inst, obc)
    for step in (1, 7200, 43200):
        gpu.obc_uv(step)
        orc.obc_uv(obc, step, st["uoo"], st["voe"])
    assert_close(gpu.download("uoo"), st["uoo"], TOL, "UOO")
    assert_close(gpu.download("voe"), st["voe"], TOL, "VOE")
    for n in (0, 1):
        cli = [api.read_obc_ts_record(HERE, s, n, JE, KE, 3) for s in (0, 1)] + [None, None]
        gpu.set_obc_ts(n, cli)
    gpu.obc_ts()
    for n in (0, 1):
        cli = [api.read_obc_ts_record(HERE, s, n, JE, KE, 3) for s in (0, 1)] + [None, None]
        orc.obc_ts(obc, cli, st["tracers"][n])
        assert np.array_equal(gpu.download(f"tracer{n}"), st["tracers"][n]), n


@pytest.mark.parametrize("kind", CASES)
def test_obc_exp_sponge_parity(kind):
    """OBC_SPONGE_EXP (SPONGE_OBCS_UV_EXP, _ETA_EXP, _TS_EXP): UOO, VOE and ZO
    against the oracle within the COS bound; THO (record set before the
    switch) and SAO (set after it), whose south band has its own rate, bit
    for bit, as the rates come from the same host EXP; TAO = 0 returns to
    the 1/x form.  Stretched metrics, so that the band lengths' summation
    order matters."""
    inst, obc = _exp_case(kind)
    orc, gpu, st = _pair(inst, obc)
    cli = [C.make_obc_ts(inst, n) for n in (0, 1)]
    gpu.set_obc_ts(0, cli[0])
    gpu.set_obc_sponge_exp(obc["tao"])
    gpu.set_obc_ts(1, cli[1])
    for step in (1, 4321):
        gpu.obc_uv(step)
        orc.obc_uv(obc, step, st["uoo"], st["voe"])
        gpu.obc_eta(step)
        orc.obc_eta(obc, step, st["zo"])
    for k in ("uoo", "voe", "zo"):
        assert_close(gpu.download(k), st[k], TOL, k)
    inv = dict(obc, tao=0.0)
    for form in (obc, inv):
        gpu.obc_ts()
        for n in (0, 1):
            orc.obc_ts(form, cli[n], st["tracers"][n], salinity=n == 1)
        for n in (0, 1):
            got = gpu.download(f"tracer{n}")
            assert np.array_equal(got, st["tracers"][n]), (n, float(np.abs(got - st["tracers"][n]).max()))
        gpu.set_obc_sponge_exp(0.0)
    gpu.obc_uv(99)
    orc.obc_uv(inv, 99, st["uoo"], st["voe"])
    assert_close(gpu.download("uoo"), st["uoo"], TOL, "UOO after the switch back")

