"""Regenerates tests/golden/oracle_golden.npz from the CPU restatement.

The reference ships no golden outputs (parity unpinned), so these fixtures
freeze the oracle's own results on small seeded instances: every hot-path
routine applied once to the initial state, the assembled operator, the RHS
and two full hot-path steps.  tests/test_oracle.py recomputes them and
requires exact equality, so any change to the oracle's arithmetic shows up.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from orctm_b200 import configs as C  # noqa: E402

CASES = {
    "c1": ("c1", dict(nx=32), None),
    "c2": ("c2", dict(nx=16, ny=12, nz=10), None),
    "c2cfl": ("c2", dict(nx=14, ny=11, nz=9), 0.45),
}


def run_case(case):
    name, over, cfl = CASES[case]
    inst = C.make_instance(name, builder=O.build_grid, cfl=cfl, **over)
    orc = O.Oracle(inst)
    out = {}
    for k in ("ddpo", "weto", "dduo", "amsuo", "ddue", "amsue", "depto"):
        out[f"geo_{k}"] = inst[k]
    st = C.copy_state(inst)
    orc.ocuad(st["uoo"], st["uko"], st["vke"], st["wo"])
    out["ocuad_uoo"] = st["uoo"]
    st = C.copy_state(inst)
    orc.ocvad(st["voe"], st["uko"], st["vke"], st["wo"])
    out["ocvad_voe"] = st["voe"]
    st = C.copy_state(inst)
    orc.ocwad(st["wno"], st["uko"], st["vke"], st["wo"], st["zo"])
    out["ocwad_wno"] = st["wno"]
    st = C.copy_state(inst)
    for n, t in enumerate(st["tracers"]):
        orc.ocadpo(t, st["uko"], st["vke"], st["wo"], st["zo"])
        out[f"ocadpo_t{n}"] = t
    st = C.copy_state(inst)
    orc.octdiff(st["tracers"], st["dvo"], st["zo"])
    for n, t in enumerate(st["tracers"]):
        out[f"octdiff_t{n}"] = t
    st = C.copy_state(inst)
    orc.ocvisc(st["uoo"], st["voe"], st["wno"], st["uko"], st["vke"], st["avo"])
    for k in ("uoo", "voe", "wno"):
        out[f"ocvisc_{k}"] = st[k]
    st = C.copy_state(inst)
    out["nh_rhs"] = orc.nh_rhs(st["uoo"], st["uoo1"], st["voe"], st["voe1"], st["wno"],
                               st["wno1"], st["zo"])
    A = orc.matrix()
    out["matrix_indptr"], out["matrix_indices"], out["matrix_data"] = A.indptr, A.indices, A.data
    st = C.copy_state(inst)
    for _ in range(2):
        orc.step_hotpath(st, solver="direct")
    for k in ("uoo", "voe", "wno", "pnh"):
        out[f"step2_{k}"] = st[k]
    for n, t in enumerate(st["tracers"]):
        out[f"step2_t{n}"] = t
    return out


def main():
    arrays = {}
    for case in CASES:
        for k, v in run_case(case).items():
            arrays[f"{case}/{k}"] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, "oracle_golden.npz"), **arrays)
    print(len(arrays), "arrays")


if __name__ == "__main__":
    main()
