"""Shared helpers of the parity tests (the oracle is the checker)."""
import numpy as np

import oracle as O
from orctm_b200 import configs as C
from orctm_b200 import grid

# Cases the oracle finishes in seconds.  (name, overrides, cfl)
SMALL = {
    "c1s": ("c1", dict(nx=96), None),
    "c2s": ("c2", dict(nx=40, ny=33, nz=24), None),
    "c2cfl": ("c2", dict(nx=37, ny=29, nz=18), 0.45),
    "c4m": ("c4", dict(nx=50, ny=41, nz=31), None),
    # deep columns: the shared-memory solver variants need the opt-in above 48 KB
    "c4deep": ("c4", dict(nx=37, ny=29, nz=97), None),
}


def instance(case: str, index: int = 0):
    name, over, cfl = SMALL[case]
    return C.make_instance(name, index=index, builder=grid.build_grid, cfl=cfl, **over)


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def assert_close(got, want, tol, what=""):
    e = relerr(got, want)
    assert e <= tol, f"{what}: relative max-norm error {e:.3e} > {tol:.1e}"
    return e
