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


# ------------------------------------------------ Sect. 3.3 (the reference's) --
SECT33 = __import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "sect33",
                                    "sect33.npz")


def sect33_instance():
    """The reference's Sect. 3.3 experiment (verification/Sect.3.3: grid
    arcgri, initial INITEM / INISAL, namelist OCECTL) as an instance dict,
    from tests/golden/sect33/sect33.npz: the grid through BELEG + BODEN, T and
    S from the initial files, the fluid at rest (ISTART = 0), AULAPTS /
    AULAPUV = C* DT / 3600 and AH00 = CAH00 / 4e5 (orctm.f90:500-502)."""
    f = np.load(SECT33)
    ie, je = f["depto"].shape
    ke = f["dzw"].size
    dt = float(f["ctl_dt"])
    inst = {"name": "sect33", "seed": 0, "ie": ie, "je": je, "ke": ke, "nx": ie - 2, "ny": je - 2,
            "nz": ke, "dt": dt, "dzw": np.ascontiguousarray(f["dzw"]),
            "depto_raw": np.asfortranarray(f["depto"]),
            "ob": {"west": False, "east": False, "north": False, "south": False},
            "almzer": C.ALMZER, "aulapts": float(f["ctl_caulapts"]) * dt / 3600.0,
            "aulapuv": float(f["ctl_caulapuv"]) * dt / 3600.0,
            "ah00": float(f["ctl_cah00"]) / 4.E5, "ntracers": 2, "tide": None}
    for k in ("dlxp", "dlyp", "dlxu", "dlyu", "dlxv", "dlyv"):
        inst[k] = np.asfortranarray(f[k])
    depto, geo = grid.build_grid(ie, je, ke, dt, inst["dzw"], inst["depto_raw"], inst["dlxp"],
                                 inst["dlyp"], inst["dlxu"], inst["dlyu"], inst["dlxv"],
                                 inst["dlyv"])
    inst["depto"] = depto
    inst.update(geo)
    z = lambda *s: np.zeros(s, order="F")
    inst.update({"uoo": z(ie + 1, je, ke), "voe": z(ie, je + 1, ke), "wno": z(ie, je, ke + 1),
                 "uko": z(ie + 1, je, ke), "vke": z(ie, je + 1, ke), "wo": z(ie, je, ke + 1),
                 "uoo1": z(ie + 1, je, ke), "voe1": z(ie, je + 1, ke), "wno1": z(ie, je, ke + 1),
                 "pnh": z(ie, je, ke), "zo": z(ie, je), "dvo": z(ie, je, ke + 1),
                 "avo": z(ie, je, ke + 1),
                 "tracers": [np.asfortranarray(f["tho"]), np.asfortranarray(f["sao"])]})
    return inst


def sect33_forcing():
    """OCTHER's constants and forcing of Sect. 3.3 (OCECTL; GIU10, GIRIV),
    OCMODMOM's Coriolis inputs (arcgri's FTWOU / FTWOV, anta's GILA / GIPH as
    coriol.f90:46-47 takes them on one rank)."""
    f = np.load(SECT33)
    ie, je = f["depto"].shape
    dzw1 = float(f["dzw"][0])
    thermo = {"eos": 0, "crelsal": float(f["ctl_crelsal"]), "creltem": float(f["ctl_creltem"]),
              "relsal": float(f["ctl_crelsal"]) * 20. / dzw1,
              "reltem": float(f["ctl_creltem"]) * 20. / dzw1,
              "wt": float(f["ctl_cwt"]) / (6.0 ** 3), "cstabeps": float(f["ctl_cstabeps"]),
              "dv0": float(f["ctl_dv0"]), "av0": float(f["ctl_av0"]),
              "cavocon": float(f["ctl_cavocon"]), "cdvocon": float(f["ctl_cdvocon"]),
              "dback": float(f["ctl_dback"]), "aback": float(f["ctl_aback"]),
              "fu10": np.asfortranarray(f["fu10"]), "giriv": np.asfortranarray(f["giriv"])}
    cor = {"ftwou": np.asfortranarray(f["ftwou"]), "ftwov": np.asfortranarray(f["ftwov"]),
           "gila": np.asfortranarray(f["gila_full"][:2 * ie, :2 * je]),
           "giph": np.asfortranarray(f["giph_full"][:2 * ie, :2 * je]), "omega": 7.292E-5}
    return thermo, cor
