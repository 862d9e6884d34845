"""Open-boundary tide forcing and sponge on the CPU: the C oracle
(og_obc_eta / og_obc_uv, a loop-by-loop restatement of mo_obcs.f90) against
an independent numpy restatement in per-cell distance form, on the
reference's own layout (W+S open) and on cases that open every side with
bands that cross, differ in width, are switched off or have zero relaxation
times, in the 1/x form and in the exponential form of OBC_SPONGE_EXP (on
stretched metrics, so that the band lengths' summation order shows); the
harmonic-constant files round trip.  No GPU."""
import numpy as np
import pytest

import np_restate as NR
import oracle as O
from helpers import assert_close, instance
from orctm_b200 import api, configs

TOL = 1e-14  # numpy's and the C library's COS may differ in the last bit


def _case(kind):
    inst = instance("c2s")
    if kind == "reference":                      # W + S open (the c2 layout)
        return inst, configs.make_obc(inst)
    inst = dict(inst)
    inst["ob"] = {"west": True, "east": True, "north": True, "south": True}
    IE, JE = inst["ie"], inst["je"]
    if kind == "crossing":                       # W/E and N/S bands overlap
        obc = configs.make_obc(inst, width=max(IE, JE))
        obc["width"] = [IE - 10, 14, JE - 9, 12]
    elif kind == "uneven":
        obc = configs.make_obc(inst)
        obc["width"] = [3, 5, 2, 4]
    elif kind == "one_off":                      # north open but not sponged
        obc = configs.make_obc(inst)
        obc["sponge"] = [1, 1, 0, 1]
    elif kind == "zero_relax":                   # lambda = 0 rows (mo_obcs.f90:1580-1583)
        obc = configs.make_obc(inst, relax_bound=0.0)
        obc["width"] = [1, 4, 1, 6]
    else:
        raise ValueError(kind)
    return inst, obc


CASES = ("reference", "crossing", "uneven", "one_off", "zero_relax")
TOL_EXP = 1e-14  # numpy's EXP and the C library's may differ in the last bit too


def _exp_case(kind):
    """_case with the exponential sponge (TAO = 5 DT) and every metric
    stretched by seeded factors in [0.7, 1.3]."""
    inst, obc = _case(kind)
    inst = dict(inst)
    g = np.random.default_rng(4242)
    for k in ("dlxp", "dlyp", "dlxu", "dlyu", "dlxv", "dlyv"):
        a = np.asarray(inst[k], dtype=np.float64)
        inst[k] = np.asfortranarray(a * g.uniform(0.7, 1.3, a.shape))
    return inst, dict(obc, tao=5.0 * inst["dt"])


@pytest.mark.parametrize("kind", CASES)
@pytest.mark.parametrize("step", [1, 4321])
def test_oracle_uv_equals_numpy(kind, step):
    inst, obc = _case(kind)
    o = O.Oracle(inst)
    st = configs.copy_state(inst)
    u0, v0 = st["uoo"].copy(), st["voe"].copy()
    o.obc_uv(obc, step, st["uoo"], st["voe"])
    assert_close(st["uoo"], NR.obc_sponge(inst, obc, step, u0, "u"), TOL, "UOO")
    assert_close(st["voe"], NR.obc_sponge(inst, obc, step, v0, "v"), TOL, "VOE")
    assert not np.array_equal(st["uoo"], u0)


@pytest.mark.parametrize("kind", CASES)
def test_oracle_eta_equals_numpy(kind):
    inst, obc = _case(kind)
    o = O.Oracle(inst)
    zo = np.array(inst["zo"], order="F", copy=True)
    z0 = zo.copy()
    o.obc_eta(obc, 777, zo)
    assert_close(zo, NR.obc_sponge(inst, obc, 777, z0, "z"), TOL, "ZO")


def test_outside_bands_unchanged():
    inst, obc = _case("uneven")
    o = O.Oracle(inst)
    st = configs.copy_state(inst)
    u0 = st["uoo"].copy()
    o.obc_uv(obc, 5, st["uoo"], st["voe"])
    w = obc["width"]
    # u-points: west band i = 0..w0-1, east i = IE-w1+1..IE, north j = 1..w2,
    # south j = JE-w3+1..JE (array index j-1)
    IE, JE = inst["ie"], inst["je"]
    inner = (slice(w[0], IE - w[1] + 1), slice(w[2], JE - w[3]))
    assert np.array_equal(st["uoo"][inner], u0[inner])


def test_boundary_cell_takes_tidal_value():
    """With the boundary relaxation time equal to DT the west boundary u-cell
    (d = 1, away from the corners) is set to the tidal value."""
    inst, obc = _case("reference")
    o = O.Oracle(inst)
    st = configs.copy_state(inst)
    step = 1000
    o.obc_uv(obc, step, st["uoo"], st["voe"])
    pi = 4.0 * np.arctan(1.0)
    t = step * inst["dt"]
    am, ph = obc["amp"][0][1], obc["pha"][0][1]
    m1 = inst["amsuo"][0, :, 0]
    tide = sum(am[:, td] * m1 * np.cos(2 * pi * (t - ph[:, td]) / obc["period"][td])
               for td in range(obc["ntide"]))
    JE, w = inst["je"], obc["width"]
    rows = slice(0, JE - w[3])          # south band rows excluded (north closed)
    for k in range(inst["ke"]):
        mk = inst["amsuo"][0, rows, k]
        want = tide[rows] * mk
        got = st["uoo"][0, rows, k]
        wet = mk > 0
        assert np.allclose(got[wet], want[wet], rtol=1e-13, atol=1e-15)


def test_obc_files_round_trip(tmp_path):
    inst, obc = _case("crossing")
    api.write_obc_files(str(tmp_path), obc["amp"], obc["pha"])
    amp, pha = api.read_obc_files(str(tmp_path), inst["ie"], inst["je"], inst["ob"],
                                  obc["ntide"])
    for b in range(4):
        for v in range(3):
            assert np.array_equal(amp[b][v], obc["amp"][b][v])
            assert np.array_equal(pha[b][v], obc["pha"][b][v])
    # 8-byte big-endian reals, ntide columns of n values (FORM='BINARY')
    raw = (tmp_path / "OB_West_v_Amp.bin").read_bytes()
    n = configs.obc_points(inst["ie"], inst["je"], 0, 2)
    assert len(raw) == 8 * n * obc["ntide"]
    assert np.frombuffer(raw[8 * n:8 * n + 8], dtype=">f8")[0] == obc["amp"][0][2][0, 1]


def test_obc_points_match_reference_dimensions():
    # mo_obcs.f90:124-138: W/E z, u (1:je) and v (0:je); N/S z, v (1:ie) and u (0:ie)
    ie, je = 30, 20
    assert [configs.obc_points(ie, je, 0, v) for v in range(3)] == [je, je, je + 1]
    assert [configs.obc_points(ie, je, 3, v) for v in range(3)] == [ie, ie + 1, ie]


@pytest.mark.parametrize("kind", CASES)
@pytest.mark.parametrize("tracer", [0, 1])
def test_oracle_ts_equals_numpy(kind, tracer):
    inst, obc = _case(kind)
    cli = configs.make_obc_ts(inst, tracer)
    o = O.Oracle(inst)
    t = np.array(inst["tracers"][tracer], order="F", copy=True)
    t0 = t.copy()
    o.obc_ts(obc, cli, t)
    assert_close(t, NR.obc_sponge_ts(inst, obc, cli, t0), 0.0, "tracer")
    assert not np.array_equal(t, t0)


def test_obc_ts_records_round_trip(tmp_path):
    inst, _ = _case("reference")
    ie, je, ke = inst["ie"], inst["je"], inst["ke"]
    recs = [configs.make_obc_ts(inst, 0, seed=s)[0] for s in (1, 2, 3)]   # west, 3 times
    api.write_obc_ts_records(str(tmp_path), 0, 0, recs)
    for r in range(3):
        assert np.array_equal(api.read_obc_ts_record(str(tmp_path), 0, 0, je, ke, r), recs[r])
    raw = (tmp_path / "OB_West_T.bin").read_bytes()
    assert len(raw) == 3 * 8 * je * ke
    # level 2 of record 1 starts after record 0 and level 1 of record 1
    off = 8 * (je * ke + je)
    assert np.frombuffer(raw[off:off + 8], dtype=">f8")[0] == recs[1][0, 1]
    with pytest.raises(ValueError):
        api.read_obc_ts_record(str(tmp_path), 0, 0, je, ke, 3)


@pytest.mark.parametrize("kind", CASES)
def test_oracle_exp_sponge_equals_numpy(kind):
    """SPONGE_OBCS_UV_EXP, _ETA_EXP and _TS_EXP (mo_obcs.f90:2588-3222)."""
    inst, obc = _exp_case(kind)
    o = O.Oracle(inst)
    st = configs.copy_state(inst)
    u0, v0, z0 = st["uoo"].copy(), st["voe"].copy(), st["zo"].copy()
    o.obc_uv(obc, 4321, st["uoo"], st["voe"])
    assert_close(st["uoo"], NR.obc_sponge(inst, obc, 4321, u0, "u"), TOL_EXP, "UOO")
    assert_close(st["voe"], NR.obc_sponge(inst, obc, 4321, v0, "v"), TOL_EXP, "VOE")
    assert not np.array_equal(st["uoo"], u0)
    o.obc_eta(obc, 777, st["zo"])
    assert_close(st["zo"], NR.obc_sponge(inst, obc, 777, z0, "z"), TOL_EXP, "ZO")
    for tracer in (0, 1):
        cli = configs.make_obc_ts(inst, tracer)
        t = np.array(inst["tracers"][tracer], order="F", copy=True)
        t0 = t.copy()
        o.obc_ts(obc, cli, t, salinity=tracer == 1)
        want = NR.obc_sponge_ts(inst, obc, cli, t0, salinity=tracer == 1)
        assert_close(t, want, TOL_EXP, f"tracer {tracer}")
        assert not np.array_equal(t, t0)


def test_exp_sponge_differs_from_one_over_x_and_sao_south_band():
    """The exponential form changes the bands only, and differs from the 1/x
    form there.  SAO's south-band loop reads the rate T's loop ended with
    (Ms_s from Lt_s, mo_obcs.f90:2976): given THO's record and field, SAO
    differs from THO in the south band only, and not in its innermost row,
    whose rate is that one."""
    inst, obc = _exp_case("reference")
    o = O.Oracle(inst)
    cli = configs.make_obc_ts(inst, 0)
    t0 = np.array(inst["tracers"][0], order="F", copy=True)
    res = {}
    for name, ob, sal in (("exp", obc, False), ("sao", obc, True),
                          ("inv", dict(obc, tao=0.0), False)):
        t = np.array(t0, order="F", copy=True)
        o.obc_ts(ob, cli, t, salinity=sal)
        res[name] = t
    JE, w = inst["je"], obc["width"]
    inner = (slice(w[0], None), slice(0, JE - w[3]))   # outside the west and south bands
    assert np.array_equal(res["exp"][inner], t0[inner])
    assert not np.array_equal(res["exp"], t0)
    assert not np.array_equal(res["exp"], res["inv"])
    rows = np.nonzero((res["exp"] != res["sao"]).any(axis=(0, 2)))[0]  # j - 1
    assert rows.size > 0
    assert rows.min() >= JE - w[3] + 1 and rows.max() <= JE - 1, rows

