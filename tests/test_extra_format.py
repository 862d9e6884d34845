"""EXTRA-format output (the reference's restart/output records) against the
oracle's restatement of write_slice + the EXTRA header: byte-identical files
from the library's host writer, and a round trip through the reader.  CPU."""
import ctypes as C

import numpy as np

import oracle as O
from orctm_b200 import _lib

_D = C.POINTER(C.c_double)


def _host_write(path, idate, code, kcodes, data, append=False):
    lib = _lib.load()
    data = np.asfortranarray(data, dtype=np.float64)
    nlev = len(kcodes)
    kc = (C.c_int * nlev)(*kcodes)
    st = lib.orctm_write_extra_host(str(path).encode(), int(append), idate, code, nlev, kc,
                                    data.size // nlev, data.ctypes.data_as(_D))
    assert st == 0


def test_host_writer_equals_oracle_bytes(tmp_path):
    g = np.random.Generator(np.random.PCG64(20261203))
    ie, je, ke = 13, 9, 5
    tho = g.normal(10.0, 5.0, (ie, je, ke))
    uko = g.normal(0.0, 0.3, (ie + 1, je, ke))
    zo = g.normal(0.0, 0.2, (ie, je))
    tiestu = [1, 3, 7, 15, 31]
    a, b = tmp_path / "lib.ext", tmp_path / "oracle.ext"
    _host_write(a, 20261203, 2, tiestu, tho)
    _host_write(a, 20261203, 3, tiestu, uko, append=True)
    _host_write(a, 20261203, 1, [-100], zo, append=True)
    recs = [(20261203, 2, tiestu[k], tho[:, :, k]) for k in range(ke)]
    recs += [(20261203, 3, tiestu[k], uko[:, :, k]) for k in range(ke)]
    recs += [(20261203, 1, -100, zo)]
    O.write_extra(b, recs)
    assert a.read_bytes() == b.read_bytes()
    back = O.read_extra(a)
    assert [(r[1], r[2]) for r in back] == [(r[1], r[2]) for r in recs]
    for (_, _, _, v), (_, _, _, ref) in zip(back, recs):
        assert np.array_equal(v, np.asarray(ref, np.float64).ravel(order="F").astype(np.float32))


def test_extra_record_layout(tmp_path):
    """One level of a 2 x 2 field: 4-byte big-endian markers around a 16-byte
    header and a 16-byte float32 payload."""
    p = tmp_path / "one.ext"
    _host_write(p, 7, 5, [3], np.array([[1.0, 2.0], [3.0, 4.0]]))
    raw = p.read_bytes()
    assert len(raw) == (4 + 16 + 4) + (4 + 16 + 4)
    assert np.frombuffer(raw[:4], ">i4")[0] == 16
    assert list(np.frombuffer(raw[4:20], ">i4")) == [7, 5, 3, 4]
    assert list(np.frombuffer(raw[28:44], ">f4")) == [1.0, 3.0, 2.0, 4.0]  # column-major


def test_host_reader_reads_oracle_file(tmp_path):
    g = np.random.Generator(np.random.PCG64(7))
    a = g.normal(0.0, 1.0, (11, 6, 4))
    b = g.normal(0.0, 1.0, (11, 6))
    p = tmp_path / "r.ext"
    recs = [(1, 2, 10 * k, a[:, :, k]) for k in range(4)] + [(1, 1, -100, b)]
    O.write_extra(p, recs)
    lib = _lib.load()
    out = np.zeros(11 * 6 * 4)
    kc = (C.c_int * 4)()
    assert lib.orctm_read_extra_host(str(p).encode(), 2, 4, 66, out.ctypes.data_as(_D), kc) == 0
    assert list(kc) == [0, 10, 20, 30]
    assert np.array_equal(out.reshape((11, 6, 4), order="F"), a.astype(np.float32).astype(np.float64))
    one = np.zeros(66)
    assert lib.orctm_read_extra_host(str(p).encode(), 1, 1, 66, one.ctypes.data_as(_D), None) == 0
    assert np.array_equal(one, b.ravel(order="F").astype(np.float32).astype(np.float64))
    # a code that is not there, or too few levels
    assert lib.orctm_read_extra_host(str(p).encode(), 5, 1, 66, one.ctypes.data_as(_D), None) != 0
    assert lib.orctm_read_extra_host(str(p).encode(), 1, 2, 66, out.ctypes.data_as(_D), None) != 0


def test_gridinfo_equals_oracle_bytes(tmp_path):
    """GRID_INFO.ext (wrte_gridinfo.f90:52-172): the library's writer against
    the oracle's record restatement in the reference's record order."""
    from orctm_b200 import api, configs

    inst = configs.make_instance("c2", nx=11, ny=8, nz=5)
    ie, je, ke = inst["ie"], inst["je"], inst["ke"]
    g = np.random.Generator(np.random.PCG64(7))
    lon = {"p": g.uniform(110, 120, (ie, je)), "u": g.uniform(110, 120, (ie + 1, je)),
           "v": g.uniform(110, 120, (ie, je + 1))}
    lat = {"p": g.uniform(10, 20, (ie, je)), "u": g.uniform(10, 20, (ie + 1, je)),
           "v": g.uniform(10, 20, (ie, je + 1))}
    deuto = g.uniform(0, 4000, (ie + 1, je))
    deute = g.uniform(0, 4000, (ie, je + 1))
    a, b = tmp_path / "lib.ext", tmp_path / "oracle.ext"
    api.write_gridinfo(str(a), inst, lon, lat, deuto, deute)
    flat = [(110, lon["p"]), (120, lat["p"]), (111, lon["u"]), (121, lat["u"]),
            (112, lon["v"]), (122, lat["v"]), (200, inst["depto"]), (201, deuto),
            (202, deute), (410, inst["dlxp"]), (411, inst["dlxu"]), (412, inst["dlxv"]),
            (420, inst["dlyp"]), (421, inst["dlyu"]), (422, inst["dlyv"])]
    recs = [(0, code, -100, v) for code, v in flat]
    for code, key in ((300, "weto"), (301, "amsuo"), (302, "amsue"), (430, "ddpo"),
                      (431, "dduo"), (432, "ddue")):
        recs += [(0, code, k + 1, inst[key][:, :, k]) for k in range(ke)]
    O.write_extra(b, recs)
    assert a.read_bytes() == b.read_bytes()
    back = O.read_extra(a)
    assert len(back) == 15 + 6 * ke
    assert [r[1] for r in back[:3]] == [110, 120, 111]
