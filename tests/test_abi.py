"""The C ABI without a GPU: the library loads, exports every function the
header declares, the host-side BELEG/BODEN builder equals the oracle's, and
argument checks fail cleanly.  CPU only."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle as O
from orctm_b200 import _lib, configs, grid

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "orctm_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(orctm_[a-z0-9_]+)\s*\(", src)))


def test_header_functions_exported():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_python_export_list_matches_header():
    names = set(declared_functions())
    assert set(_lib.EXPORTS) <= names


@pytest.mark.parametrize("name,over", [("c1", dict(nx=40)), ("c2", dict(nx=30, ny=22, nz=17)),
                                       ("c4", dict()), ("c3", dict(nx=48, ny=40))])
def test_grid_builder_equals_oracle(name, over):
    r = configs.raw_instance(name, **over)
    args = (r["ie"], r["je"], r["ke"], r["dt"], r["dzw"], r["depto_raw"], r["dlxp"], r["dlyp"],
            r["dlxu"], r["dlyu"], r["dlxv"], r["dlyv"])
    d1, g1 = O.build_grid(*args)
    d2, g2 = grid.build_grid(*args)
    assert np.array_equal(d1, d2)
    for k in g1:
        assert np.array_equal(g1[k], g2[k]), k


def test_status_strings():
    lib = _lib.load()
    for s in range(0, -9, -1):
        assert lib.orctm_status_string(s)
    assert lib.orctm_abi_version() == 1


def test_argument_checks_without_device():
    lib = _lib.load()
    d = _lib.Desc()
    d.ie, d.je, d.ke, d.ntracers = 2, 2, 1, 2
    h = C.c_void_p()
    assert lib.orctm_create(C.byref(d), C.byref(h)) == -1          # grid too small
    d.ie, d.je, d.ke, d.ntracers = 10, 10, 5, 1
    assert lib.orctm_create(C.byref(d), C.byref(h)) == -1          # too few tracers
    d.ntracers, d.dt, d.ah00, d.almzer = 2, 1.0, 1.0, 1e-19
    assert lib.orctm_create(C.byref(d), C.byref(h)) == -6          # harmonic diffusion
    n = C.c_size_t()
    assert lib.orctm_field_size(None, 0, C.byref(n)) == -1
    assert lib.orctm_ocuad(None) == -1
    assert lib.orctm_set_solver(None, 0, 1e-10, 10) == -1


def test_create_reports_missing_device():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    inst = configs.make_instance("c2", builder=grid.build_grid, nx=12, ny=10, nz=6)
    from orctm_b200.api import Instance

    with pytest.raises(_lib.OrctmError) as e:
        Instance(inst)
    assert e.value.status in (-7, -2)


def test_open_boundary_and_gridinfo_argument_checks(tmp_path):
    """Null handles and missing arrays fail with ORCTM_E_ARG before any device
    call; the GRID_INFO writer is host-only and refuses missing arrays."""
    from orctm_b200 import api

    lib = _lib.load()
    o = _lib.Obc()
    assert lib.orctm_set_obc(None, C.byref(o)) == -1
    assert lib.orctm_obc_uv(None, 1) == -1
    assert lib.orctm_obc_eta(None, 1) == -1
    assert lib.orctm_obc_ts(None) == -1
    assert lib.orctm_set_obc_ts(None, 0, None) == -1
    assert lib.orctm_set_obc_sponge_exp(None, 3600.0) == -1
    inst = configs.make_instance("c2", builder=grid.build_grid, nx=9, ny=7, nz=4)
    d, keep = api.make_desc(inst)
    g = _lib.GridInfo()                      # every coordinate pointer NULL
    path = str(tmp_path / "GRID_INFO.ext").encode()
    assert lib.orctm_write_gridinfo(path, C.byref(d), C.byref(g)) == -1
    assert lib.orctm_write_gridinfo(None, C.byref(d), C.byref(g)) == -1
    assert not (tmp_path / "GRID_INFO.ext").exists()


FORTRAN = os.path.join(ROOT, "orctm_b200", "fortran", "orctm_gpu_mod.f90")


def _fortran_type_fields(src, name):
    body = re.search(r"type, bind\(c\) :: %s\n(.*?)end type %s" % (name, name), src, re.S).group(1)
    fields = []
    for line in body.splitlines():
        line = line.split("!")[0]
        if "::" not in line:
            continue
        decl = re.sub(r"\([^)]*\)", "", line.split("::")[1])   # drop dimensions
        fields += [f.strip() for f in decl.split(",") if f.strip()]
    return fields


def _c_struct_fields(src, name):
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), src, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        decl = re.sub(r"^(const\s+)?(int|double|size_t)\s*\**", "", decl)
        for f in decl.split(","):
            fields.append(re.sub(r"[\[\*].*|\s", "", f.replace("*", "")))
    return [f for f in fields if f]


def test_fortran_module_binds_exported_symbols_and_matching_types():
    """The ISO_C_BINDING module (no Fortran compiler here): every bound name
    exists in the library and every bind(c) type lists the C struct's fields
    in the same order."""
    lib = _lib.load()
    src = open(FORTRAN).read()
    names = re.findall(r'bind\(c, name="(orctm_[a-z0-9_]+)"\)', src)
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
        assert n in declared_functions(), n
    hdr = open(HEADER).read()
    for t in ("orctm_desc", "orctm_solve_stats", "orctm_obc", "orctm_gridinfo", "orctm_barotropic",
              "orctm_thermo", "orctm_coriolis"):
        assert _fortran_type_fields(src, t) == _c_struct_fields(hdr, t), t


_NOALLOC_PTRS = ("tracer_in", "tracer_out", "dvo", "ddpo", "weto", "di", "dzw", "dlxp", "dlyp",
                 "dlxu", "dlyu", "dlxv", "dlyv", "zo")


def _noalloc_args():
    a = _lib.NoAllocArgs()
    a.ie, a.je, a.ke = 10, 9, 5
    a.dt, a.almzer, a.aulapts, a.ah00 = 10.0, 1e-19, 1e3, 0.0
    # distinct non-null placeholders: every refusal below happens before the
    # entry point touches a device, so they are never dereferenced
    for n, k in enumerate(_NOALLOC_PTRS):
        setattr(a, k, 0x100000 + 0x1000 * n)
    return a


@pytest.mark.parametrize("change,status,words", [
    (dict(ke=1), -1, b"grid size"),
    (dict(ke=321), -1, b"grid size"),
    (dict(ie=2), -1, b"grid size"),
    (dict(ie=2050, je=2050, ke=10), -8, b"no-allocation limit"),
    (dict(zo=None), -1, b"missing device pointer"),
    (dict(dvo=None), -1, b"missing device pointer"),
    (dict(tracer_out=0x100000), -1, b"different buffers"),
    (dict(ah00=1.0), -6, b"harmonic"),
])
def test_noalloc_refusals_carry_a_message(change, status, words):
    """orctm_octdiff_noalloc refuses bad sizes, missing or aliased arrays and
    harmonic diffusion before any device work, and orctm_last_error(NULL)
    then says why."""
    lib = _lib.load()
    a = _noalloc_args()
    for k, v in change.items():
        setattr(a, k, v)
    assert lib.orctm_octdiff_noalloc(C.byref(a)) == status
    assert words in lib.orctm_last_error(None)
    assert lib.orctm_octdiff_noalloc(None) == -1
    assert b"null argument" in lib.orctm_last_error(None)


def test_extra_reader_rejects_corrupt_record_markers(tmp_path):
    """A record marker that does not match the header's size (a corrupt or
    wrong-endian file) is refused before a buffer is sized from it."""
    lib = _lib.load()
    good = tmp_path / "good.ext"
    O.write_extra(str(good), [(1, 2, 3, np.arange(6.0))])
    out = np.zeros(6)
    assert lib.orctm_read_extra_host(str(good).encode(), 2, 1, 6, _lib_ptr(out), None) == 0
    assert np.array_equal(out, np.arange(6.0))
    raw = bytearray(good.read_bytes())
    for bad in (b"\xff\xff\xff\xf0", raw[0:4][::-1]):      # huge marker; little-endian marker
        b = bytearray(raw)
        b[0:4] = bad
        p = tmp_path / "bad.ext"
        p.write_bytes(bytes(b))
        assert lib.orctm_read_extra_host(str(p).encode(), 2, 1, 6, _lib_ptr(out), None) == -1
    b = bytearray(raw)
    b[24:28] = b"\x7f\xff\xff\xff"                          # data marker disagrees with IEDIM
    p = tmp_path / "bad2.ext"
    p.write_bytes(bytes(b))
    assert lib.orctm_read_extra_host(str(p).encode(), 2, 1, 6, _lib_ptr(out), None) == -1


def _lib_ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))
