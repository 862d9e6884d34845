"""The ABI from plain C: the driver compiles as C99 against the header and
links against the library; without a GPU, creating a handle fails cleanly
with ORCTM_E_NODEVICE.  CPU only (the GPU run is in test_gpu_c_driver.py)."""
import subprocess

import pytest

from orctm_b200 import configs as C
from orctm_b200 import grid

from c_driver_support import build_driver, write_input


def test_c_driver_builds_and_reports_no_device(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    exe = build_driver(str(tmp_path))
    inst = C.make_instance("c2", builder=grid.build_grid, nx=12, ny=10, nz=6)
    inp = tmp_path / "in.bin"
    write_input(str(inp), inst, C.copy_state(inst), 1, 0, 1e-10)
    r = subprocess.run([exe, str(inp), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 2
    assert "create status -7" in r.stderr
