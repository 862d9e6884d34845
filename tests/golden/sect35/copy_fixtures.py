"""Copies the reference's own open-boundary and stratification input files
of its Sect. 3.5 verification experiment (ORCTM/verification/Sect.3.5/obcs/
and BT_forc/) next to this script, as test fixtures.

These are the only artefacts the reference ships for the path (it has no
tests and no outputs).  They are produced by the reference's own
Gen_Boundary.m and read by INI_OBCS (mo_obcs.f90:263-506) and mkgrid.f90
(TRef.bin / SRef.bin, BT_forc/mkgrid.f90:222-233).  Run once, in a checkout
that has the reference next to it:
    python tests/golden/sect35/copy_fixtures.py [reference root]
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = {
    "obcs": [f"OB_{s}_{v}_{q}.bin" for s in ("East", "West") for v in ("u", "v")
             for q in ("Amp", "Gph")] + [f"OB_{s}_{t}.bin" for s in ("East", "West")
                                         for t in ("T", "S")],
    "BT_forc": ["TRef.bin", "SRef.bin"],
}


def main(root: str) -> None:
    base = os.path.join(root, "ORCTM", "verification", "Sect.3.5")
    for sub, names in FILES.items():
        for n in names:
            shutil.copyfile(os.path.join(base, sub, n), os.path.join(HERE, n))
            print(n)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
