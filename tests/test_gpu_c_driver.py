"""The ABI from plain C on the GPU: the C driver's results equal the Python
(ctypes) path's bit for bit on the same inputs."""
import subprocess

import numpy as np
import pytest

from orctm_b200 import configs as C
from orctm_b200 import grid
from orctm_b200.api import Instance

from c_driver_support import build_driver, write_input

pytestmark = pytest.mark.gpu


def test_c_driver_equals_python_path(tmp_path):
    inst = C.make_instance("c4", index=3, builder=grid.build_grid, nx=40, ny=33, nz=24)
    st = C.copy_state(inst)
    exe = build_driver(str(tmp_path))
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    write_input(str(inp), inst, st, 2, 0, 1e-10)
    r = subprocess.run([exe, str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    gpu = Instance(inst)
    gpu.upload_state(C.copy_state(inst))
    gpu.set_solver("fp64", rtol=1e-10, maxit=20000)
    for _ in range(2):
        gpu.step_hotpath()
    got = np.fromfile(out, dtype=np.float64)
    pos = 0
    for k in ["uoo", "voe", "wno", "pnh"] + [f"tracer{n}" for n in range(gpu.ntr)]:
        want = gpu.download(k).ravel(order="F")
        assert np.array_equal(got[pos:pos + want.size], want), k
        pos += want.size
    assert pos == got.size
