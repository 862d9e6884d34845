"""Builds sect33.npz next to this script from the reference's own inputs of
its Sect. 3.3 verification experiment (an internal wave shoaling over a
Gaussian ridge in a laboratory tank, ORCTM/verification/Sect.3.3/): the grid
file arcgri and coordinates anta, the initial temperature and salinity
INITEM / INISAL, the wind-speed and river forcing GIU10 / GIRIV (all written
by the experiment's BT_forc/mkgrid.f90), and the constants of its namelist
OCECTL.  The fields are stored as they are in the files (compressed: they
are mostly constant), so tests can build the experiment without the
reference.  Run once, in a checkout that has the reference next to it:
    python tests/golden/sect33/make_fixture.py [reference root]
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", ".."))
from orctm_b200.api import read_model_records  # noqa: E402

IE, JE, KE = 1004, 5, 100  # BT_forc/mkgrid.f90:13


def load(root: str) -> dict:
    base = os.path.join(root, "ORCTM", "verification", "Sect.3.3")
    bt = os.path.join(base, "BT_forc")
    out = {}
    codes = {507: "depto", 85: "dlxp", 185: "dlxu", 285: "dlxv", 86: "dlyp", 186: "dlyu",
             286: "dlyv", 175: "ftwou", 176: "ftwov"}  # mkgrid.f90:66-83
    shapes = {"depto": (IE, JE), "dlxp": (IE, JE), "dlyp": (IE, JE), "dlxu": (IE + 1, JE),
              "dlyu": (IE + 1, JE), "ftwou": (IE + 1, JE), "dlxv": (IE, JE + 1),
              "dlyv": (IE, JE + 1), "ftwov": (IE, JE + 1)}
    for h, v in read_model_records(os.path.join(bt, "arcgri")):
        k = codes[h[1]]
        out[k] = v.reshape(shapes[k], order="F")
    anta = {h[1]: v for h, v in read_model_records(os.path.join(bt, "anta"))}
    out["gila_full"] = anta[54].reshape((2 * IE + 1, 2 * JE + 1), order="F")  # GILA_G (coriol.f90:35)
    out["giph_full"] = anta[55].reshape((2 * IE + 1, 2 * JE + 1), order="F")
    for name, key in (("INITEM", "tho"), ("INISAL", "sao")):
        recs = read_model_records(os.path.join(bt, name))
        assert len(recs) == KE
        out[key] = np.stack([v.reshape((IE, JE), order="F") for _, v in recs], axis=2)
    for name, key in (("GIU10", "fu10"), ("GIRIV", "giriv")):
        (h, v), = read_model_records(os.path.join(bt, name))
        out[key] = v.reshape((IE, JE), order="F")
    text = open(os.path.join(base, "OCECTL")).read()

    def num(key):
        m = re.search(r"\b%s\s*=\s*([-+0-9.Ee]+)" % key, text)
        return float(m.group(1))

    for key in ("DT", "CAULAPTS", "CAULAPUV", "AUS", "CAH00", "DV0", "AV0", "CWT", "CSTABEPS",
                "DBACK", "ABACK", "CRELSAL", "CRELTEM", "CDVOCON", "CAVOCON"):
        out["ctl_" + key.lower()] = np.float64(num(key))
    m = re.search(r"DZW\s*=\s*(\d+)\*([-+0-9.Ee]+)", text)
    out["dzw"] = np.full(int(m.group(1)), float(m.group(2)))
    return out


def main(root: str) -> None:
    out = load(root)
    np.savez_compressed(os.path.join(HERE, "sect33.npz"), **out)
    print({k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
