"""ctypes front end of the CPU restatement (oracle) of ORCTM's NH hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, and only as the checker or the timed CPU
baseline.  PARITY PINNED ONLY IN PART: the reference (Fortran/PETSc) cannot
run here and ships no golden outputs; its check values and input files pin
what they cover (see orctm_oracle.h).

Arrays are numpy float64 in Fortran order with the reference's shapes
(single-rank domain, I_start = J_start = 0):
    p-points (IE, JE, KE)      u-points (IE+1, JE, KE)
    v-points (IE, JE+1, KE)    w-points (IE, JE, KE+1)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liborctm_oracle.so")
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def build(force: bool = False) -> str:
    """Compiles liborctm_oracle.so with the Makefile next to this file."""
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(
        os.path.join(_HERE, "orctm_oracle.c")
    ):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return _SO


class _Grid(C.Structure):
    _fields_ = [
        ("ie", C.c_int), ("je", C.c_int), ("ke", C.c_int),
        ("ob_west", C.c_int), ("ob_east", C.c_int), ("ob_north", C.c_int), ("ob_south", C.c_int),
        ("dt", C.c_double), ("almzer", C.c_double), ("aulapts", C.c_double),
        ("aulapuv", C.c_double), ("ah00", C.c_double),
        ("dzw", _D), ("di", _D), ("dz", _D), ("tiestu", _D), ("tiestw", _D),
        ("dlxp", _D), ("dlyp", _D), ("dtdxpo", _D), ("dtdyo", _D),
        ("dlxu", _D), ("dlyu", _D), ("dtdxuo", _D), ("dpyo", _D),
        ("dlxv", _D), ("dlyv", _D), ("dtdxue", _D), ("dpye", _D),
        ("ddpo", _D), ("weto", _D), ("dduo", _D), ("amsuo", _D), ("ddue", _D), ("amsue", _D),
    ]


class _Obc(C.Structure):
    _fields_ = [
        ("ntide", C.c_int), ("period", _D), ("sponge", C.c_int * 4), ("width", C.c_int * 4),
        ("relax_inner", C.c_double), ("relax_bound", C.c_double),
        ("amp", (_D * 3) * 4), ("pha", (_D * 3) * 4),
        ("tao", C.c_double), ("salinity", C.c_int),
    ]


def obc_struct(obc: dict):
    """og_obc of an open-boundary dict (orctm_b200.configs.make_obc); returns
    the structure and the arrays it points into."""
    keep = [np.ascontiguousarray(obc["period"], dtype=np.float64)]
    o = _Obc()
    o.ntide = int(obc["ntide"])
    o.period = _p(keep[0])
    for b in range(4):
        o.sponge[b] = int(obc["sponge"][b])
        o.width[b] = int(obc["width"][b])
        for v in range(3):
            for dst, src in ((o.amp, obc["amp"]), (o.pha, obc["pha"])):
                a = src[b][v]
                if a is None:
                    dst[b][v] = _D()
                else:
                    a = np.asfortranarray(a, dtype=np.float64)
                    keep.append(a)
                    dst[b][v] = _p(a)
    o.relax_inner = float(obc["relax_inner"])
    o.relax_bound = float(obc["relax_bound"])
    o.tao = float(obc.get("tao", 0.0))  # 0: the 1/x sponge
    return o, keep


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.og_matrix_nnz.restype = C.c_size_t
        _lib.og_solve.restype = C.c_int
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1), a.flags
    return a.ctypes.data_as(_D)


GEOM_KEYS = ("tiestu", "tiestw", "dz", "di", "dtdxpo", "dtdyo", "dtdxuo", "dpyo", "dtdxue",
             "dpye", "ddpo", "weto", "dduo", "amsuo", "ddue", "amsue")


def build_grid(ie, je, ke, dt, dzw, depto, dlxp, dlyp, dlxu, dlyu, dlxv, dlyv):
    """BELEG + BODEN restated: returns (depto_adjusted, geometry dict)."""
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
    args = [np.asfortranarray(a, dtype=np.float64) for a in (dlxp, dlyp, dlxu, dlyu, dlxv, dlyv)]
    lib().og_build_grid(ie, je, ke, C.c_double(dt), _p(dzw), _p(depto), *[_p(a) for a in args],
                        *[_p(g[k]) for k in GEOM_KEYS])
    return depto, g


class _Baro(C.Structure):
    _fields_ = [("grav", C.c_double), ("stabn", C.c_double), ("conn", C.c_double),
                ("rlsa1", C.c_double), ("sorpar", C.c_double), ("niter", C.c_int),
                ("eta_forc", C.c_int)]


# the reference driver's constants (orctm.f90:352-353, 657-661, 680) and the
# SOR sweeps of troneu.f90:104; SORPAR is TROTEST's choice at run time
BARO_DEFAULTS = {"grav": 9.806, "stabn": 0.6, "conn": 0.5, "rlsa1": 1.0 - 0.085,
                 "sorpar": 1.75, "niter": 250, "eta_forc": 0}


def baro_struct(b: dict):
    v = dict(BARO_DEFAULTS, **b)
    return _Baro(v["grav"], v["stabn"], v["conn"], v["rlsa1"], v["sorpar"], int(v["niter"]),
                 int(v["eta_forc"]))


class _Thermo(C.Structure):
    _fields_ = [("eos", C.c_int), ("rho0", C.c_double), ("drdt", C.c_double),
                ("drds", C.c_double), ("t0", C.c_double), ("s0", C.c_double),
                ("grav", C.c_double), ("relsal", C.c_double), ("reltem", C.c_double),
                ("rhoicwa", C.c_double), ("rhosnwa", C.c_double), ("wt", C.c_double),
                ("cstabeps", C.c_double), ("dv0", C.c_double), ("av0", C.c_double),
                ("cavocon", C.c_double), ("cdvocon", C.c_double),
                ("preff", _D), ("dbackv", _D), ("abackv", _D),
                ("sicomo", _D), ("sictho", _D), ("sicsno", _D), ("relsao", _D), ("reltho", _D),
                ("giriv", _D), ("fu10", _D)]


# the reference driver's OCTHER constants (orctm.f90:311-330, 503, 561-569,
# 739-743); eos 0 = ADISITJ + RHO1J, 1 = linear (rho0 + drdt (T - t0) + drds (S - s0))
THERMO_DEFAULTS = {"eos": 0, "rho0": 1025.0, "drdt": -0.2, "drds": 0.78, "t0": 10.0, "s0": 35.0,
                   "grav": 9.806, "crelsal": 3.E-7, "creltem": 0.0,
                   "rhoicwa": 0.91E+03 / 1.025E+03, "rhosnwa": 0.33E+03 / 1.025E+03,
                   "wt": 0.5E-3 / (6.0 ** 3), "cstabeps": 0.05, "dv0": 0.5E-2, "av0": 0.5E-2,
                   "cavocon": 0.0, "cdvocon": 20.0, "aback": 5.E-5, "dback": 5.E-5}
THERMO_2D = ("sicomo", "sictho", "sicsno", "relsao", "reltho", "giriv", "fu10")


def thermo_values(inst: dict, t: dict) -> dict:
    """The full OCTHER parameter set of an instance: THERMO_DEFAULTS updated by
    ``t``; RELSAL / RELTEM from CRELSAL / CRELTEM (orctm.f90:561, 569), PREFF
    = 0.1026 TIESTU (beleg.f90:127), DBACKV / ABACKV constant (orctm.f90:515-519)."""
    v = dict(THERMO_DEFAULTS, **t)
    ke = inst["ke"]
    dzw1 = float(np.asarray(inst["dzw"])[0])
    v.setdefault("relsal", v["crelsal"] * 20. / dzw1)
    v.setdefault("reltem", v["creltem"] * 20. / dzw1)
    if "preff" not in v:
        v["preff"] = 0.1026 * np.asarray(inst["tiestu"], dtype=np.float64)[:ke]
    if "dbackv" not in v:
        v["dbackv"] = np.full(ke + 1, v["dback"])
    if "abackv" not in v:
        v["abackv"] = np.full(ke + 1, v["aback"])
    return v


def thermo_struct(inst: dict, t: dict):
    v = thermo_values(inst, t)
    keep = []

    def arr(a):
        if a is None:
            return _D()
        a = np.asfortranarray(a, dtype=np.float64)
        keep.append(a)
        return _p(a)

    s = _Thermo(int(v["eos"]), v["rho0"], v["drdt"], v["drds"], v["t0"], v["s0"], v["grav"],
                v["relsal"], v["reltem"], v["rhoicwa"], v["rhosnwa"], v["wt"], v["cstabeps"],
                v["dv0"], v["av0"], v["cavocon"], v["cdvocon"], arr(v["preff"]), arr(v["dbackv"]),
                arr(v["abackv"]), *[arr(v.get(k)) for k in THERMO_2D])
    return s, keep


class _Coriolis(C.Structure):
    _fields_ = [("ftwou", _D), ("ftwov", _D), ("gila", _D), ("giph", _D), ("omega", C.c_double)]


def coriolis_struct(c: dict):
    keep = [np.asfortranarray(c[k], dtype=np.float64) for k in ("ftwou", "ftwov", "gila", "giph")]
    return _Coriolis(*[_p(a) for a in keep], float(c.get("omega", 7.292E-5))), keep


class Oracle:
    """Holds one instance's geometry and exposes the restated routines."""

    def __init__(self, inst: dict):
        self.inst = inst
        self.ie, self.je, self.ke = inst["ie"], inst["je"], inst["ke"]
        self._keep = {}
        gr = _Grid()
        gr.ie, gr.je, gr.ke = self.ie, self.je, self.ke
        ob = inst["ob"]
        gr.ob_west, gr.ob_east, gr.ob_north, gr.ob_south = (int(ob[k]) for k in ("west", "east", "north", "south"))
        gr.dt = inst["dt"]
        gr.almzer = inst["almzer"]
        gr.aulapts = inst["aulapts"]
        gr.aulapuv = inst["aulapuv"]
        gr.ah00 = inst["ah00"]
        for k in ("dzw", "di", "dz", "tiestu", "tiestw", "dlxp", "dlyp", "dtdxpo", "dtdyo", "dlxu",
                  "dlyu", "dtdxuo", "dpyo", "dlxv", "dlyv", "dtdxue", "dpye", "ddpo", "weto",
                  "dduo", "amsuo", "ddue", "amsue"):
            a = np.asfortranarray(inst[k], dtype=np.float64)
            self._keep[k] = a
            setattr(gr, k, _p(a))
        self.g = gr

    # -- stencils ---------------------------------------------------------
    def ocadpo(self, trf, uko, vke, wo, zo):
        lib().og_ocadpo(C.byref(self.g), _p(trf), _p(uko), _p(vke), _p(wo), _p(zo))

    def ocuad(self, uoo, uko, vke, wo):
        lib().og_ocuad(C.byref(self.g), _p(uoo), _p(uko), _p(vke), _p(wo))

    def ocvad(self, voe, uko, vke, wo):
        lib().og_ocvad(C.byref(self.g), _p(voe), _p(uko), _p(vke), _p(wo))

    def ocwad(self, wno, uko, vke, wo, zo):
        lib().og_ocwad(C.byref(self.g), _p(wno), _p(uko), _p(vke), _p(wo), _p(zo))

    def octdiff(self, tracers, dvo, zo):
        arr = (_D * len(tracers))(*[_p(t) for t in tracers])
        lib().og_octdiff(C.byref(self.g), len(tracers), arr, _p(dvo), _p(zo))

    def ocvisc(self, uoo, voe, wno, uko, vke, avo):
        lib().og_ocvisc(C.byref(self.g), _p(uoo), _p(voe), _p(wno), _p(uko), _p(vke), _p(avo))

    # -- open boundaries (mo_obcs.f90) ---------------------------------------
    def obc_eta(self, obc, step, zo):
        o, keep = obc_struct(obc)
        lib().og_obc_eta(C.byref(self.g), C.byref(o), int(step), _p(zo))

    def obc_uv(self, obc, step, uoo, voe):
        o, keep = obc_struct(obc)
        lib().og_obc_uv(C.byref(self.g), C.byref(o), int(step), _p(uoo), _p(voe))

    def obc_ts(self, obc, cli, trf, salinity=False):
        """FORC_OBCS_TS + SPONGE_OBCS_TS on one tracer; cli[b] is side b's
        climatology record (n, KE) or None; salinity: the tracer is SAO
        (matters in the exponential form only)."""
        o, keep = obc_struct(obc)
        o.salinity = 1 if salinity else 0
        arrs = [None if c is None else np.asfortranarray(c, dtype=np.float64) for c in cli]
        ptrs = (_D * 4)(*[_D() if a is None else _p(a) for a in arrs])
        lib().og_obc_ts(C.byref(self.g), C.byref(o), ptrs, _p(trf))

    def octimf(self, uoo, voe, uko, vke):
        lib().og_octimf(C.byref(self.g), _p(uoo), _p(voe), _p(uko), _p(vke))

    # -- barotropic solve (boden.f90, itprep.f90, troneu.f90, ocvtro.f90, ocvtot.f90)
    def _f2(self, kind):
        ie, je = self.ie, self.je
        return np.zeros({"p": (ie, je), "u": (ie + 1, je), "v": (ie, je + 1)}[kind], order="F")

    def deut(self, depto, minvalue):
        """(DEUTO, DEUTE, DEUTIO, DEUTIE) from the BODEN-adjusted DEPTO."""
        out = [self._f2("u"), self._f2("v"), self._f2("u"), self._f2("v")]
        lib().og_deut(C.byref(self.g), _p(np.asfortranarray(depto, dtype=np.float64)),
                      C.c_double(minvalue), *[_p(a) for a in out])
        return tuple(out)

    def itprep(self, b, deuto, deute):
        out = [self._f2("p"), self._f2("u"), self._f2("v"), self._f2("p")]
        lib().og_itprep(C.byref(self.g), C.byref(baro_struct(b)), _p(deuto), _p(deute),
                        *[_p(a) for a in out])
        return tuple(out)  # xx, uf, vf, ff

    def trotest(self, b, xx, uf, vf, ff, ntry=200, niter=200):
        """TROTEST's choice of SORPAR."""
        lib().og_trotest.restype = C.c_double
        return lib().og_trotest(C.byref(self.g), C.byref(baro_struct(b)), _p(xx), _p(uf), _p(vf),
                                _p(ff), int(ntry), int(niter))

    def troneu(self, b, xx, uf, vf, ff, u1o, v1e, uzo, vze):
        b1o, z1o = self._f2("p"), self._f2("p")
        lib().og_troneu(C.byref(self.g), C.byref(baro_struct(b)), _p(xx), _p(uf), _p(vf), _p(ff),
                        _p(u1o), _p(v1e), _p(uzo), _p(vze), _p(b1o), _p(z1o))
        return b1o, z1o

    def ocvtro(self, b, deutio, deutie, z1o, uzo, vze, zo):
        """In place on uzo, vze, zo; returns (uso, vse)."""
        uso, vse = self._f2("u"), self._f2("v")
        lib().og_ocvtro(C.byref(self.g), C.byref(baro_struct(b)), _p(deutio), _p(deutie),
                        _p(z1o), _p(uzo), _p(vze), _p(uso), _p(vse), _p(zo))
        return uso, vse

    def ocbarp(self, uso, vse, uzo, vze):
        """In place on uso, vse, uzo, vze."""
        lib().og_ocbarp(C.byref(self.g), _p(uso), _p(vse), _p(uzo), _p(vze))

    def ocwind(self, txo, tye, sicomu, sicomv, tauwatu, tauwatv, uoo, voe):
        """In place on uoo, voe (level 1)."""
        arrs = [np.asfortranarray(a, dtype=np.float64)
                for a in (txo, tye, sicomu, sicomv, tauwatu, tauwatv)]
        lib().og_ocwind(C.byref(self.g), *[_p(a) for a in arrs], _p(uoo), _p(voe))

    def ocvtot(self, b, uso, vse, uoo, voe, uko, vke, wo):
        """In place on uoo, voe, uko, vke, wo."""
        lib().og_ocvtot(C.byref(self.g), C.byref(baro_struct(b)), _p(uso), _p(vse), _p(uoo),
                        _p(voe), _p(uko), _p(vke), _p(wo))

    # -- OCTHER, OCMODMOM, OCCLIT --------------------------------------------
    def octher_surface(self, t, tho, sao, zo):
        """OCTHER part A in place on tho, sao, zo; returns (eminpo, rivrun)."""
        ts, keep = thermo_struct(self.inst, t)
        eminpo, rivrun = self._f2("p"), self._f2("p")
        lib().og_octher_surface(C.byref(self.g), C.byref(ts), _p(tho), _p(sao), _p(zo),
                                _p(eminpo), _p(rivrun))
        return eminpo, rivrun

    def octher_column(self, t, tho, sao, zo, uko, vke, avo, dvo, kcondep):
        """OCTHER parts C, D in place on tho, sao, avo, dvo, kcondep (int32,
        (IE, JE)); returns (po, stabio, rhoo)."""
        ts, keep = thermo_struct(self.inst, t)
        shp = (self.ie, self.je, self.ke)
        po, stabio, rhoo = (np.zeros(shp, order="F") for _ in range(3))
        assert kcondep.dtype == np.int32 and kcondep.flags.f_contiguous
        lib().og_octher_column(C.byref(self.g), C.byref(ts), _p(tho), _p(sao), _p(zo), _p(uko),
                               _p(vke), _p(po), _p(stabio), _p(rhoo), _p(avo), _p(dvo),
                               kcondep.ctypes.data_as(_I))
        return po, stabio, rhoo

    def octher(self, t, st, obc=None, cli=None):
        """Whole OCTHER (octher.f90:1-455) on a state dict: part A, the T/S
        boundary forcing of tracers 0 and 1 when ``obc`` and ``cli`` (cli[n]
        the four side records of tracer n) are given, parts C and D.  Sets
        st's eminpo, rivrun, po, stabio, rhoo."""
        tho, sao = st["tracers"][0], st["tracers"][1]
        st["eminpo"], st["rivrun"] = self.octher_surface(t, tho, sao, st["zo"])
        if obc is not None and cli is not None:
            for n in (0, 1):
                if cli[n] is not None:
                    self.obc_ts(obc, cli[n], st["tracers"][n], salinity=n == 1)
        st["po"], st["stabio"], st["rhoo"] = self.octher_column(
            t, tho, sao, st["zo"], st["uko"], st["vke"], st["avo"], st["dvo"], st["kcondep"])

    def ocmodmom(self, b, c, deutio, deutie, st):
        """OCMODMOM on a state dict (in place on uko, vke, wno, po, stabio; sets
        uk1o, vk1e, wn1o, u1o, uso, v1e, vse)."""
        cs, keep = coriolis_struct(c)
        ie, je, ke = self.ie, self.je, self.ke
        st["uk1o"] = np.zeros((ie + 1, je, ke), order="F")
        st["vk1e"] = np.zeros((ie, je + 1, ke), order="F")
        st["wn1o"] = np.zeros((ie, je, ke + 1), order="F")
        for k in ("u1o", "uso"):
            st[k] = self._f2("u")
        for k in ("v1e", "vse"):
            st[k] = self._f2("v")
        lib().og_ocmodmom(C.byref(self.g), C.byref(baro_struct(b)), C.byref(cs), _p(deutio),
                          _p(deutie), _p(st["zo"]), _p(st["uoo"]), _p(st["voe"]), _p(st["uko"]),
                          _p(st["vke"]), _p(st["uk1o"]), _p(st["vk1e"]), _p(st["wno"]),
                          _p(st["wn1o"]), _p(st["po"]), _p(st["stabio"]), _p(st["u1o"]),
                          _p(st["uso"]), _p(st["v1e"]), _p(st["vse"]))

    def occlit(self, b, deutio, deutie, st):
        """OCCLIT on a state dict (in place on uko, vke, uk1o, vk1e, wo,
        stabio); returns CONTRA."""
        lib().og_occlit.restype = C.c_double
        return lib().og_occlit(C.byref(self.g), C.byref(baro_struct(b)), _p(deutio), _p(deutie),
                               _p(st["uko"]), _p(st["vke"]), _p(st["uk1o"]), _p(st["vk1e"]),
                               _p(st["wo"]), _p(st["stabio"]))

    def step_full(self, st, t, b, c, deut, tables, ldtrun, wind=None, obc=None, cli=None,
                  solver="direct", rtol=1e-13, pnh=None):
        """One whole step in the driver's order (orctm.f90:1327-1562) on a state
        dict: OCTHER, OCWIND, the open-boundary forcing, OCTIMF, OCMODMOM,
        OCBARP, OCCLIT, TRONEU, OCVTRO, OCVTOT, STABIO times 1000/DZ, the hot
        path.  deut = (DEUTIO, DEUTIE), tables = ITPREP's (XX, UF, VF, FF).
        Returns the hot path's solve info with "contra"."""
        deutio, deutie = deut
        self.octher(t, st, obc=obc, cli=cli)
        if wind is not None:
            self.ocwind(wind["txo"], wind["tye"], wind["sicomu"], wind["sicomv"],
                        wind["tauwatu"], wind["tauwatv"], st["uoo"], st["voe"])
        if obc is not None:
            if dict(BARO_DEFAULTS, **b)["eta_forc"]:
                self.obc_eta(obc, ldtrun, st["zo"])
            self.obc_uv(obc, ldtrun, st["uoo"], st["voe"])
        self.octimf(st["uoo"], st["voe"], st["uko"], st["vke"])
        self.ocmodmom(b, c, deutio, deutie, st)
        st["uzo"], st["vze"] = self._f2("u"), self._f2("v")
        self.ocbarp(st["uso"], st["vse"], st["uzo"], st["vze"])
        contra = self.occlit(b, deutio, deutie, st)
        st["b1o"], st["z1o"] = self.troneu(b, *tables, st["u1o"], st["v1e"], st["uzo"], st["vze"])
        st["uso"], st["vse"] = self.ocvtro(b, deutio, deutie, st["z1o"], st["uzo"], st["vze"], st["zo"])
        self.ocvtot(b, st["uso"], st["vse"], st["uoo"], st["voe"], st["uko"], st["vke"], st["wo"])
        dz = np.asarray(self.inst["dz"], dtype=np.float64)
        for k in range(self.ke):
            st["stabio"][:, :, k] = (1000. / dz[k]) * st["stabio"][:, :, k]
        info = self.step_hotpath(st, solver=solver, rtol=rtol, pnh=pnh)
        info["contra"] = contra
        return info

    # -- OCVTOT_NH ----------------------------------------------------------
    @property
    def nunk(self):
        return (self.ie - 2) * (self.je - 2) * self.ke

    def nh_rhs(self, uoo, uoo1, voe, voe1, wno, wno1, zo):
        b = np.zeros(self.nunk)
        lib().og_nh_rhs(C.byref(self.g), _p(uoo), _p(uoo1), _p(voe), _p(voe1), _p(wno), _p(wno1),
                        _p(zo), _p(b))
        return b

    def matrix(self):
        """compute_matrix as a scipy CSR matrix (DMDA natural order)."""
        import scipy.sparse as sp

        nnz = lib().og_matrix_nnz(C.byref(self.g))
        rp = np.zeros(self.nunk + 1, dtype=np.int32)
        ci = np.zeros(nnz, dtype=np.int32)
        v = np.zeros(nnz)
        lib().og_matrix_csr(C.byref(self.g), rp.ctypes.data_as(_I), ci.ctypes.data_as(_I), _p(v))
        return sp.csr_matrix((v, ci, rp), shape=(self.nunk, self.nunk))

    def solve(self, A, b, x0=None, rtol=1e-13, maxit=5000):
        """FGMRES + column preconditioner (CPU).  Returns (x, its, relres)."""
        x = np.zeros(self.nunk) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        rp = np.ascontiguousarray(A.indptr, dtype=np.int32)
        ci = np.ascontiguousarray(A.indices, dtype=np.int32)
        v = np.ascontiguousarray(A.data, dtype=np.float64)
        rel = C.c_double(0.0)
        its = lib().og_solve(C.byref(self.g), rp.ctypes.data_as(_I), ci.ctypes.data_as(_I), _p(v),
                             _p(np.ascontiguousarray(b)), _p(x), C.c_double(rtol), maxit,
                             C.byref(rel))
        return x, its, rel.value

    @staticmethod
    def direct_solve(A, b):
        """Sparse LU solve (SuperLU): the stand-in for PETSc's FGMRES + one-level
        PCMG, whose single level is a direct factorisation."""
        import scipy.sparse.linalg as spl

        return spl.spsolve(A.tocsc(), b)

    def nh_post(self, x, pnh, uoo, voe, wno, uoo1, voe1, wno1, wo):
        lib().og_nh_post(C.byref(self.g), _p(np.ascontiguousarray(x)), _p(pnh), _p(uoo), _p(voe),
                         _p(wno), _p(uoo1), _p(voe1), _p(wno1), _p(wo))

    def ocvtot_nh(self, st, solver="direct", rtol=1e-13, pnh=None):
        """Whole OCVTOT_NH on a state dict (in place).  Returns solve info.

        ``pnh`` (a p-point array, e.g. the pressure another implementation
        found) replaces the solve: its interior is used as the solution, so
        that the post-solve update can be checked apart from the solver."""
        b = self.nh_rhs(st["uoo"], st["uoo1"], st["voe"], st["voe1"], st["wno"], st["wno1"], st["zo"])
        if pnh is not None:
            x = np.asarray(pnh)[1:-1, 1:-1, :].reshape(-1, order="F").copy()
            self.nh_post(x, st["pnh"], st["uoo"], st["voe"], st["wno"], st["uoo1"], st["voe1"],
                         st["wno1"], st["wo"])
            return {"its": 0, "relres": None, "b": b, "x": x}
        A = self.matrix()
        x0 = st["pnh"][1:-1, 1:-1, :].reshape(-1, order="F").copy()
        if solver == "direct":
            x = self.direct_solve(A, b)
            its, rel = 1, float(np.linalg.norm(b - A @ x) / max(np.linalg.norm(b), 1e-300))
        else:
            x, its, rel = self.solve(A, b, x0=x0, rtol=rtol)
        self.nh_post(x, st["pnh"], st["uoo"], st["voe"], st["wno"], st["uoo1"], st["voe1"],
                     st["wno1"], st["wo"])
        return {"its": its, "relres": rel, "b": b, "x": x}

    def step_hotpath(self, st, solver="direct", rtol=1e-13, pnh=None):
        """One pass of the hot path in the driver's order (orctm.f90:1454-1562);
        ``pnh`` as in ocvtot_nh."""
        self.ocuad(st["uoo"], st["uko"], st["vke"], st["wo"])
        self.ocvad(st["voe"], st["uko"], st["vke"], st["wo"])
        self.ocwad(st["wno"], st["uko"], st["vke"], st["wo"], st["zo"])
        for t in st["tracers"]:
            self.ocadpo(t, st["uko"], st["vke"], st["wo"], st["zo"])
        self.octdiff(st["tracers"], st["dvo"], st["zo"])
        self.octimf(st["uoo"], st["voe"], st["uko"], st["vke"])
        self.ocvisc(st["uoo"], st["voe"], st["wno"], st["uko"], st["vke"], st["avo"])
        info = self.ocvtot_nh(st, solver=solver, rtol=rtol, pnh=pnh)
        self.octimf(st["uoo"], st["voe"], st["uko"], st["vke"])
        return info


# ------------------------------------------------------------------ EXTRA ---
def write_extra(path, records, append=False):
    """EXTRA-format records as the reference writes them: for each
    (idate, code, kcode, values) a header record of four big-endian int32
    (IDATE, ICODE, KCODE, IEDIM) and a record of the values as big-endian
    float32 (REAL(x, sp)), each record framed by its big-endian int32 length
    (Fortran sequential unformatted, -convert big_endian: write_slice,
    mo_parallel.f90:733-779; aufw.f90:54-160; Makefile:75)."""
    with open(path, "ab" if append else "wb") as f:
        for idate, code, kcode, values in records:
            v = np.asarray(values, dtype=np.float64).ravel(order="F").astype(">f4")
            hdr = np.array([idate, code, kcode, v.size], dtype=">i4").tobytes()
            for payload in (hdr, v.tobytes()):
                m = np.array([len(payload)], dtype=">i4").tobytes()
                f.write(m + payload + m)


def read_extra(path):
    """The records of an EXTRA file: [(idate, code, kcode, float32 values)]."""
    out = []
    data = open(path, "rb").read()
    pos = 0

    def record():
        nonlocal pos
        n = int(np.frombuffer(data, ">i4", 1, pos)[0])
        payload = data[pos + 4:pos + 4 + n]
        tail = int(np.frombuffer(data, ">i4", 1, pos + 4 + n)[0])
        assert tail == n, "record markers differ"
        pos += n + 8
        return payload

    while pos < len(data):
        hdr = np.frombuffer(record(), ">i4")
        vals = np.frombuffer(record(), ">f4")
        assert vals.size == hdr[3]
        out.append((int(hdr[0]), int(hdr[1]), int(hdr[2]), vals.astype(np.float32)))
    return out
