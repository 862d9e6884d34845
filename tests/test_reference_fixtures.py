"""The reference's own input files for the path, read by this package's
readers: the open-boundary harmonic constants and T/S boundary climatology
of the Sect. 3.5 experiment (OB_{East,West}_{u,v}_{Amp,Gph}.bin,
OB_{East,West}_{T,S}.bin, written by its Gen_Boundary.m and read by
INI_OBCS, mo_obcs.f90:263-506) and the stratification profiles TRef.bin /
SRef.bin (BT_forc/mkgrid.f90:222-233).  Copies live in tests/golden/sect35
(copy_fixtures.py).  That experiment is IE_G = 4000, JE_G = 5, KE = 300
(Sect.3.5/src_orctm/mo_param1.f90:24-25 with -DVERSIONGR03, :32 with
-DLEVELS40, Sect.3.5/src_orctm/Makefile:42), two tidal constituents
(tidalPeriod in Sect.3.5/OCECTL), W and E open, OBC_ETA_FORC off
(Makefile:49: -DZZOBC_ETA_FORC).  CPU only."""
import os

import numpy as np
import pytest

from orctm_b200 import api

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sect35")
IE, JE, KE, NTIDE = 4000, 5, 300, 2
OB = {"west": True, "east": True, "north": False, "south": False}
PERIODS = (44714.1643, 86164.0906)
NREC = 10     # climatology records in the T/S files


def _raw(name):
    return np.fromfile(os.path.join(HERE, name), dtype=">f8")


def test_harmonic_constants_read_as_stored():
    amp, pha = api.read_obc_files(HERE, IE, JE, OB, NTIDE, variables=(1, 2))
    for b, side in ((0, "West"), (1, "East")):
        for v, var, n in ((1, "u", JE), (2, "v", JE + 1)):
            for arr, q in ((amp, "Amp"), (pha, "Gph")):
                a = arr[b][v]
                assert a.shape == (n, NTIDE)
                # n values of constituent 1, then n of constituent 2
                assert np.array_equal(a.ravel(order="F"), _raw(f"OB_{side}_{var}_{q}.bin"))
        assert amp[b][0] is None and pha[b][0] is None
        # values of the experiment's generator: u amplitudes 0.05 (M2) and
        # 0.04 (K1) m/s, phases a quarter period, no v forcing
        assert np.array_equal(amp[b][1], np.tile([0.05, 0.04], (JE, 1)))
        assert np.allclose(pha[b][1], np.tile([PERIODS[0] / 4, PERIODS[1] / 4], (JE, 1)),
                           rtol=1e-15, atol=0)
        assert not amp[b][2].any() and not pha[b][2].any()
    for b in (2, 3):
        assert all(amp[b][v] is None for v in range(3))


def test_harmonic_constants_wrong_shape_refused():
    with pytest.raises(ValueError):
        api.read_obc_files(HERE, IE, JE + 1, OB, NTIDE, variables=(1, 2))
    with pytest.raises(ValueError):
        api.read_obc_files(HERE, IE, JE, OB, 3, variables=(1, 2))
    with pytest.raises(FileNotFoundError):
        api.read_obc_files(HERE, IE, JE, OB, NTIDE)        # no z files: ETA forcing off


@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("tracer", [0, 1])
def test_ts_climatology_records(side, tracer):
    """Each record is KE levels of JE values (the file holds exactly NREC);
    every record of this experiment is the TRef/SRef profile, level by level,
    along the whole boundary."""
    name = f"OB_{api.OBC_SIDES[side]}_{'TS'[tracer]}.bin"
    raw = _raw(name)
    assert raw.size == NREC * JE * KE
    prof = api.read_ts_profile(os.path.join(HERE, ("TRef.bin", "SRef.bin")[tracer]), KE)
    for r in range(NREC):
        rec = api.read_obc_ts_record(HERE, side, tracer, JE, KE, r)
        assert rec.shape == (JE, KE)
        assert np.array_equal(rec.ravel(order="F"), raw[r * JE * KE:(r + 1) * JE * KE])
        assert np.array_equal(rec, np.tile(prof, (JE, 1)))
    with pytest.raises(ValueError):
        api.read_obc_ts_record(HERE, side, tracer, JE, KE, NREC)


def test_stratification_profiles():
    t = api.read_ts_profile(os.path.join(HERE, "TRef.bin"), KE)
    s = api.read_ts_profile(os.path.join(HERE, "SRef.bin"), KE)
    assert np.array_equal(t, _raw("TRef.bin")) and np.array_equal(s, _raw("SRef.bin"))
    # warm, fresher surface over cold, saltier depths
    assert t[0] > t[-1] and s[0] < s[-1]
    assert np.all(np.diff(t) <= 0)
    with pytest.raises(ValueError):
        api.read_ts_profile(os.path.join(HERE, "TRef.bin"), KE + 1)


def test_writers_reproduce_the_reference_files(tmp_path):
    """The package's writers give back the reference's bytes."""
    amp, pha = api.read_obc_files(HERE, IE, JE, OB, NTIDE, variables=(1, 2))
    api.write_obc_files(str(tmp_path), amp, pha)
    for side in ("West", "East"):
        for var in ("u", "v"):
            for q in ("Amp", "Gph"):
                n = f"OB_{side}_{var}_{q}.bin"
                assert (tmp_path / n).read_bytes() == open(os.path.join(HERE, n), "rb").read()
    for side in (0, 1):
        for tr in (0, 1):
            recs = [api.read_obc_ts_record(HERE, side, tr, JE, KE, r) for r in range(NREC)]
            api.write_obc_ts_records(str(tmp_path), side, tr, recs)
            n = f"OB_{api.OBC_SIDES[side]}_{'TS'[tr]}.bin"
            assert (tmp_path / n).read_bytes() == open(os.path.join(HERE, n), "rb").read()
