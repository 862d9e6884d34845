"""Builds the plain C ABI driver (tests/c_driver/orctm_c_driver.c) and writes
its input files from an instance dict."""
import os
import subprocess

import numpy as np

from orctm_b200 import _lib
from orctm_b200.api import FIELDS, GEOMETRY_KEYS, field_id

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_driver(outdir: str) -> str:
    exe = os.path.join(outdir, "orctm_c_driver")
    libdir = os.path.dirname(_lib.SO)
    _lib.load()  # builds the library if it is missing
    subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_driver", "orctm_c_driver.c"),
                    "-L", libdir, "-lorctm_gpu", f"-Wl,-rpath,{libdir}", "-o", exe],
                   check=True)
    return exe


def write_input(path: str, inst: dict, state: dict, nsteps: int, solver: int, rtol: float):
    ob = inst["ob"]
    ntr = len(state["tracers"])
    head = np.array([inst["ie"], inst["je"], inst["ke"], ntr, int(ob["west"]), int(ob["east"]),
                     int(ob["north"]), int(ob["south"]), nsteps, solver], dtype=np.int32)
    dv = np.array([inst["dt"], inst["almzer"], inst["aulapts"], inst["aulapuv"], inst["ah00"],
                   rtol], dtype=np.float64)
    with open(path, "wb") as f:
        f.write(head.tobytes())
        f.write(dv.tobytes())
        for k in GEOMETRY_KEYS:
            f.write(np.asarray(inst[k], dtype=np.float64).ravel(order="F").tobytes())
        by_id = {field_id(k): state[k] for k in FIELDS}
        by_id.update({field_id(f"tracer{n}"): t for n, t in enumerate(state["tracers"])})
        for fid in range(field_id("tracer0") + ntr):
            f.write(np.asarray(by_id[fid], dtype=np.float64).ravel(order="F").tobytes())
