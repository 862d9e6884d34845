"""Host side of the batch/serve API without a GPU: argument checks, the
memory estimate, and request marshalling."""
import ctypes as C

import numpy as np
import pytest

from orctm_b200 import _lib, configs, grid
from orctm_b200 import serve as S


@pytest.fixture(scope="module")
def inst():
    return configs.make_instance("c4", index=1, builder=grid.build_grid, nx=20, ny=17, nz=9)


def test_estimate_grows_with_size_and_solver(inst):
    e64 = S.estimate_device_bytes(inst, "fp64")
    e32 = S.estimate_device_bytes(inst, "fp32_refined")
    assert e32 > e64 > 0
    big = dict(inst)
    big["ke"] = inst["ke"] * 2
    assert S.estimate_device_bytes(big, "fp64") > e64


def test_estimate_rejects_bad_desc(inst):
    lib = S._bind(_lib.load())
    d, keep = S.make_desc(inst)
    d.ntracers = 1
    b = C.c_ulonglong()
    assert lib.orctm_estimate_device_bytes(C.byref(d), 0, C.byref(b)) == _lib.ORCTM_E_ARG


@pytest.mark.parametrize("kw", [dict(slots=0), dict(memory_fraction=0.0),
                                dict(memory_fraction=1.5), dict(rtol=0.0), dict(maxit=0)])
def test_serve_create_rejects_bad_options(kw):
    lib = S._bind(_lib.load())
    o = S.opts(**kw)
    h = C.c_void_p()
    assert lib.orctm_serve_create(C.byref(o), C.byref(h)) == _lib.ORCTM_E_ARG


def test_serve_create_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = S._bind(_lib.load())
    h = C.c_void_p()
    assert lib.orctm_serve_create(C.byref(S.opts()), C.byref(h)) == -7  # ORCTM_E_NODEVICE


def test_job_marshalling(inst):
    st = configs.copy_state(inst)
    j = S.Job(inst, st, nsteps=4)
    r = j.req
    assert r.nsteps == 4 and r.nin == 13 + len(st["tracers"])
    ids = [r.in_fields[k] for k in range(r.nin)]
    assert sorted(ids) == sorted(set(ids))
    # outputs: uoo, voe, wno, pnh and every tracer, in the reference layouts
    assert r.nout == 4 + inst["ntracers"]
    assert j.out["uoo"].shape == (inst["ie"] + 1, inst["je"], inst["ke"])
    assert j.out["voe"].shape == (inst["ie"], inst["je"] + 1, inst["ke"])
    assert j.out["wno"].shape == (inst["ie"], inst["je"], inst["ke"] + 1)
    assert j.out["pnh"].shape == (inst["ie"], inst["je"], inst["ke"])
    assert j.out["uoo"].flags.f_contiguous
    # the input pointers address the job's own Fortran-ordered copies
    a = np.ctypeslib.as_array(r.in_data[0], shape=(st["uoo"].size,))
    assert np.array_equal(a, st["uoo"].ravel(order="F"))
    out = j.outputs()
    assert len(out["tracers"]) == inst["ntracers"]


def test_serve_submit_rejects_bad_request():
    lib = S._bind(_lib.load())
    assert lib.orctm_serve_submit(None, None, None) == _lib.ORCTM_E_ARG
