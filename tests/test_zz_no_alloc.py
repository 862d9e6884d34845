"""orctm_octdiff_noalloc, the scratch-free entry point, against orctm_octdiff
and against the oracle.

The entry point exists for callers that may not allocate device memory (code
under CUDA graph capture, hosts whose device memory belongs to another
runtime); it keeps its scratch in a fixed array inside the library.  This
test allocates the input and output arrays itself (with torch), calls the
entry point through the C ABI twice in a row for every tracer -- the second
call reuses the scratch array the first one left behind -- and compares each
result with the handle-based orctm_octdiff and with the oracle's OCTDIFF at
the tolerance of the other parity tests, on a c2 box and a c1 slice, and
on the c2 box without the biharmonic part (AULAPTS <= ALMZER).  It
also checks that a grid beyond the fixed limit is refused.  This file is
collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from orctm_b200 import _lib
from orctm_b200 import configs
from orctm_b200.api import Instance

from helpers import assert_close, instance

pytestmark = pytest.mark.gpu
TOL = 1e-12
ORCTM_E_TOO_LARGE = -8
_D = C.POINTER(C.c_double)


class Args(C.Structure):
    _fields_ = [("ie", C.c_int), ("je", C.c_int), ("ke", C.c_int),
                ("dt", C.c_double), ("almzer", C.c_double), ("aulapts", C.c_double),
                ("ah00", C.c_double),
                ("tracer_in", C.c_void_p), ("tracer_out", C.c_void_p), ("dvo", C.c_void_p),
                ("ddpo", C.c_void_p), ("weto", C.c_void_p), ("di", C.c_void_p),
                ("dzw", C.c_void_p), ("dlxp", C.c_void_p), ("dlyp", C.c_void_p),
                ("dlxu", C.c_void_p), ("dlyu", C.c_void_p), ("dlxv", C.c_void_p),
                ("dlyv", C.c_void_p), ("zo", C.c_void_p), ("stream", C.c_void_p)]


@pytest.mark.parametrize("case,vertical_only", [("c2s", False), ("c1s", False), ("c2s", True)])
def test_octdiff_noalloc_matches_handle_path_and_oracle(case, vertical_only):
    import torch

    lib = _lib.load()
    lib.orctm_octdiff_noalloc.argtypes = [C.POINTER(Args)]
    inst = instance(case)
    if vertical_only:  # AULAPTS <= ALMZER: the vertical solve writes the output directly
        inst["aulapts"] = 0.0
    st = configs.copy_state(inst)
    with Instance(inst) as gpu:
        gpu.upload_state(st)
        gpu.octdiff()
        want = [gpu.download(f"tracer{n}") for n in range(gpu.ntr)]
    # the oracle's OCTDIFF_BASE + OCTDIFF_TS on the same inputs
    ref = [np.array(t, order="F", copy=True) for t in st["tracers"]]
    O.Oracle(inst).octdiff(ref, np.asfortranarray(st["dvo"]), np.asfortranarray(st["zo"]))

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(np.ravel(a, order="F"))).to("cuda")

    keep = {k: dev(inst[k]) for k in ("ddpo", "weto", "di", "dzw", "dlxp", "dlyp", "dlxu",
                                      "dlyu", "dlxv", "dlyv")}
    keep["dvo"] = dev(st["dvo"])
    keep["zo"] = dev(st["zo"])
    a = Args()
    a.ie, a.je, a.ke = inst["ie"], inst["je"], inst["ke"]
    a.dt, a.almzer, a.aulapts, a.ah00 = inst["dt"], inst["almzer"], inst["aulapts"], inst["ah00"]
    for k, t in keep.items():
        setattr(a, k, t.data_ptr())
    a.stream = None
    shape = (inst["ie"], inst["je"], inst["ke"])
    for call in range(2):
        for n, tr in enumerate(st["tracers"]):
            tin = dev(tr)
            tout = torch.full_like(tin, float("nan"))
            a.tracer_in, a.tracer_out = tin.data_ptr(), tout.data_ptr()
            status = lib.orctm_octdiff_noalloc(C.byref(a))
            assert status == 0, lib.orctm_status_string(status)
            torch.cuda.synchronize()
            got = tout.cpu().numpy().reshape(shape, order="F")
            assert_close(got, want[n], TOL, f"call {call}, tracer {n}")
            assert_close(got, ref[n], TOL, f"call {call}, tracer {n} against the oracle")

    big = Args()
    C.pointer(big)[0] = a
    big.ie, big.je, big.ke = 2050, 2050, 10
    assert lib.orctm_octdiff_noalloc(C.byref(big)) == ORCTM_E_TOO_LARGE
