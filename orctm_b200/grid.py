"""BELEG + BODEN geometry through the library's orctm_build_grid."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

GEOM_KEYS = ("tiestu", "tiestw", "dz", "di", "dtdxpo", "dtdyo", "dtdxuo", "dpyo", "dtdxue",
             "dpye", "ddpo", "weto", "dduo", "amsuo", "ddue", "amsue")


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def build_grid(ie, je, ke, dt, dzw, depto, dlxp, dlyp, dlxu, dlyu, dlxv, dlyv):
    """Returns (depto adjusted by BODEN, geometry dict) in the reference layouts."""
    f = lambda s: np.zeros(s, dtype=np.float64, order="F")
    depto = np.array(depto, dtype=np.float64, order="F", copy=True)
    g = {
        "tiestu": f(ke + 1), "tiestw": f(ke + 1), "dz": f(ke + 1), "di": f(ke + 1),
        "dtdxpo": f((ie, je)), "dtdyo": f((ie, je)), "dtdxuo": f((ie + 1, je)),
        "dpyo": f((ie + 1, je)), "dtdxue": f((ie, je + 1)), "dpye": f((ie, je + 1)),
        "ddpo": f((ie, je, ke)), "weto": f((ie, je, ke)), "dduo": f((ie + 1, je, ke)),
        "amsuo": f((ie + 1, je, ke)), "ddue": f((ie, je + 1, ke)), "amsue": f((ie, je + 1, ke)),
    }
    dzw = np.ascontiguousarray(dzw, dtype=np.float64)
    m = [np.asfortranarray(a, dtype=np.float64) for a in (dlxp, dlyp, dlxu, dlyu, dlxv, dlyv)]
    st = _lib.load().orctm_build_grid(ie, je, ke, C.c_double(dt), _p(dzw), _p(depto),
                                      *[_p(a) for a in m], *[_p(g[k]) for k in GEOM_KEYS])
    _lib.check(st)
    return depto, g


def uv_depths(depto):
    """BODEN's u- and v-point depths (boden.f90:116-131): DEUTO (IE+1, JE) =
    MIN of the two neighbouring DEPTO, the first and last column copied from
    their neighbours; DEUTE (IE, JE+1) likewise in j.  ``depto`` is the
    BODEN-adjusted (IE, JE) depth."""
    d = np.asarray(depto, dtype=np.float64)
    ie, je = d.shape
    deuto = np.zeros((ie + 1, je), order="F")
    deuto[1:ie, :] = np.where(d[1:, :] < d[:-1, :], d[1:, :], d[:-1, :])
    deuto[0, :] = deuto[1, :]
    deuto[ie, :] = deuto[ie - 1, :]
    deute = np.zeros((ie, je + 1), order="F")
    deute[:, 1:je] = np.where(d[:, 1:] < d[:, :-1], d[:, 1:], d[:, :-1])
    deute[:, 0] = deute[:, 1]
    deute[:, je] = deute[:, je - 1]
    return deuto, deute
