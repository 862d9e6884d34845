"""Host-side mirror of the reference's hot-path interface.

``Instance`` owns one device-resident regional domain and exposes the
reference's subroutine names (OCUAD, OCVAD, OCWAD, OCADPO, OCTDIFF_BASE +
OCTDIFF_TS, OCTIMF, OCVISC, OCVTOT_NH) as methods that call the C ABI of
liborctm_gpu.so.  Arrays are numpy float64 in the reference's Fortran layouts
(see orctm_b200.configs).  Every call goes to the CUDA library; there is no
host fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (F_AVO, F_DVO, F_PNH, F_THO, F_UKO, F_UOO, F_UOO_1, F_VKE, F_VOE, F_VOE_1,
                   F_WNO, F_WNO_1, F_WO, F_ZO, SOLVER_FP32_REFINED, SOLVER_FP64, SolveStats)

_D = C.POINTER(C.c_double)

FIELDS = {"uoo": F_UOO, "voe": F_VOE, "wno": F_WNO, "uko": F_UKO, "vke": F_VKE, "wo": F_WO,
          "uoo1": F_UOO_1, "voe1": F_VOE_1, "wno1": F_WNO_1, "pnh": F_PNH, "zo": F_ZO,
          "dvo": F_DVO, "avo": F_AVO}
SHAPES = {"uoo": "u", "voe": "v", "wno": "w", "uko": "u", "vke": "v", "wo": "w", "uoo1": "u",
          "voe1": "v", "wno1": "w", "pnh": "p", "zo": "2", "dvo": "w", "avo": "w"}


def _p(a):
    return a.ctypes.data_as(_D)


GEOMETRY_KEYS = ("dzw", "di", "dlxp", "dlyp", "dtdxpo", "dtdyo", "dlxu", "dlyu", "dtdxuo", "dlxv",
                 "dlyv", "dpye", "ddpo", "weto", "dduo", "amsuo", "ddue", "amsue")


def make_desc(inst: dict, device: int = 0):
    """The orctm_desc of an instance dict, and the arrays its pointers refer
    to (keep them alive while the descriptor is in use)."""
    d = _lib.Desc()
    d.ie, d.je, d.ke = inst["ie"], inst["je"], inst["ke"]
    d.i_start = d.j_start = 0
    d.ntracers = int(inst.get("ntracers", len(inst.get("tracers", [])) or 2))
    ob = inst["ob"]
    d.ob_west, d.ob_east, d.ob_north, d.ob_south = (int(ob[k]) for k in
                                                    ("west", "east", "north", "south"))
    d.dt, d.almzer, d.aulapts, d.aulapuv, d.ah00 = (inst["dt"], inst["almzer"], inst["aulapts"],
                                                    inst["aulapuv"], inst["ah00"])
    keep = []
    for k in GEOMETRY_KEYS:
        a = np.asfortranarray(inst[k], dtype=np.float64)
        keep.append(a)
        setattr(d, k, _p(a))
    d.device = device
    return d, keep


OBC_SIDES = ("West", "East", "North", "South")
OBC_VARS = ("z", "u", "v")


def make_obc(obc: dict):
    """The orctm_obc of an open-boundary dict (keys ntide, period, sponge,
    width, relax_inner, relax_bound, amp, pha as orctm_b200.configs.make_obc
    returns them; amp[s][v] / pha[s][v] are (n, ntide) arrays or None), and
    the arrays its pointers refer to."""
    o = _lib.Obc()
    keep = [np.ascontiguousarray(obc["period"], dtype=np.float64)]
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
                    continue
                a = np.asfortranarray(a, dtype=np.float64)
                keep.append(a)
                dst[b][v] = _p(a)
    o.relax_inner = float(obc["relax_inner"])
    o.relax_bound = float(obc["relax_bound"])
    return o, keep


def obc_file_name(side: int, var: int, phase: bool) -> str:
    """The file INI_OBCS reads one array from (mo_obcs.f90:270-398), e.g.
    OB_West_u_Amp.bin / OB_West_u_Gph.bin."""
    return f"OB_{OBC_SIDES[side]}_{OBC_VARS[var]}_{'Gph' if phase else 'Amp'}.bin"


def read_obc_files(dirname: str, ie: int, je: int, ob: dict, ntide: int, variables=(0, 1, 2)):
    """amp[s][v], pha[s][v] from the reference's harmonic-constant files of the
    open sides: unformatted stream files (FORM='BINARY') of ntide columns of
    n values, 8-byte big-endian reals (-r8, -convert big_endian, Makefile:75).
    ``variables`` lists the ones to read (0 z, 1 u, 2 v): INI_OBCS reads the z
    files only with OBC_ETA_FORC and the u/v files only with OBC_UV_FORC
    (mo_obcs.f90:266-398); the others stay None."""
    import os

    from .configs import OBC_BOUNDARIES, obc_points

    amp = [[None] * 3 for _ in range(4)]
    pha = [[None] * 3 for _ in range(4)]
    for b, name in enumerate(OBC_BOUNDARIES):
        if not ob[name]:
            continue
        for v in variables:
            n = obc_points(ie, je, b, v)
            for dst, ph in ((amp, False), (pha, True)):
                path = os.path.join(dirname, obc_file_name(b, v, ph))
                a = np.fromfile(path, dtype=">f8")
                if a.size != n * ntide:
                    raise ValueError(f"{path}: {a.size} values, expected {n} x {ntide}")
                dst[b][v] = np.asfortranarray(a.astype(np.float64).reshape((n, ntide), order="F"))
    return amp, pha


def read_model_records(path: str):
    """The records of a model input file as the reference's experiments write
    them (grid file arcgri, coordinates anta, initial INITEM / INISAL, daily
    forcing GI*; BT_forc/mkgrid.f90): Fortran sequential unformatted records,
    big-endian (-convert big_endian, Makefile:75), in pairs of a header of
    four 8-byte integers (IDATE, CODE, LEVEL, N) and N 8-byte reals.  Returns
    [((idate, code, level, n), values)]."""
    data = open(path, "rb").read()
    pos = 0

    def record():
        nonlocal pos
        if pos + 4 > len(data):
            raise ValueError(f"{path}: truncated record marker at byte {pos}")
        n = int(np.frombuffer(data, ">i4", 1, pos)[0])
        if n < 0 or pos + 8 + n > len(data):
            raise ValueError(f"{path}: record of {n} bytes at byte {pos} runs past the end")
        tail = int(np.frombuffer(data, ">i4", 1, pos + 4 + n)[0])
        if tail != n:
            raise ValueError(f"{path}: record markers differ at byte {pos}")
        payload = data[pos + 4:pos + 4 + n]
        pos += n + 8
        return payload

    out = []
    while pos < len(data):
        hdr = record()
        if len(hdr) != 32:
            raise ValueError(f"{path}: header record of {len(hdr)} bytes, expected 32")
        h = tuple(int(v) for v in np.frombuffer(hdr, ">i8"))
        vals = record()
        if len(vals) != 8 * h[3]:
            raise ValueError(f"{path}: {len(vals)} bytes of values, header says {h[3]} reals")
        out.append((h, np.frombuffer(vals, ">f8").astype(np.float64)))
    return out


def read_ts_profile(path: str, ke: int) -> np.ndarray:
    """A reference stratification profile (TRef.bin / SRef.bin): KE values,
    one per level from the surface down, each read by its own READ of a
    FORM='BINARY' file, i.e. a stream of 8-byte big-endian reals
    (BT_forc/mkgrid.f90:222-233 of the Sect. 3.5 experiment)."""
    a = np.fromfile(path, dtype=">f8")
    if a.size != ke:
        raise ValueError(f"{path}: {a.size} values, expected KE = {ke}")
    return a.astype(np.float64)


def write_obc_files(dirname: str, amp, pha) -> None:
    """Writes amp / pha in the layout read_obc_files (and INI_OBCS) reads."""
    import os

    for b in range(4):
        for v in range(3):
            for src, ph in ((amp, False), (pha, True)):
                a = src[b][v]
                if a is not None:
                    np.asarray(a, dtype=np.float64).ravel(order="F").astype(">f8").tofile(
                        os.path.join(dirname, obc_file_name(b, v, ph)))


def write_gridinfo(path: str, inst: dict, lon: dict, lat: dict, deuto, deute) -> None:
    """GRID_INFO.ext of an instance (WRTE_GRIDINFO, wrte_gridinfo.f90):
    lon / lat map "p", "u", "v" to the coordinates (degrees) at those points
    in the reference layouts; deuto / deute are the depths at u and v points
    (DEPTO comes from the instance).  Host only."""
    d, keep = make_desc(inst)
    g = _lib.GridInfo()
    arrs = {"lonp": lon["p"], "latp": lat["p"], "lonu": lon["u"], "latu": lat["u"],
            "lonv": lon["v"], "latv": lat["v"], "depto": inst["depto"], "deuto": deuto,
            "deute": deute}
    shapes = {"p": (inst["ie"], inst["je"]), "u": (inst["ie"] + 1, inst["je"]),
              "v": (inst["ie"], inst["je"] + 1)}
    for k, a in arrs.items():
        a = np.asfortranarray(a, dtype=np.float64)
        want = shapes["p" if k == "depto" else k[-1] if k.startswith(("lon", "lat")) else
                      {"deuto": "u", "deute": "v"}[k]]
        if a.shape != want:
            raise ValueError(f"{k}: shape {a.shape}, expected {want}")
        keep.append(a)
        setattr(g, k, _p(a))
    _lib.check(_lib.load().orctm_write_gridinfo(path.encode(), C.byref(d), C.byref(g)))


def read_obc_ts_record(dirname: str, side: int, tracer: int, n: int, ke: int, record: int):
    """Record `record` (0-based: the one FORC_OBCS_TS reads at its
    record-th call, mo_obcs.f90:937-960) of OB_<Side>_T.bin (tracer 0) or
    OB_<Side>_S.bin (tracer 1): a stream file of 8-byte big-endian reals in
    which each record is KE levels of n values (n = JE west/east, IE
    north/south).  Returns the (n, KE) array set_obc_ts takes."""
    import os

    path = os.path.join(dirname, f"OB_{OBC_SIDES[side]}_{'TS'[tracer]}.bin")
    count = n * ke
    a = np.fromfile(path, dtype=">f8", count=count, offset=8 * count * record)
    if a.size != count:
        raise ValueError(f"{path}: record {record} is incomplete")
    return np.asfortranarray(a.astype(np.float64).reshape((n, ke), order="F"))


def write_obc_ts_records(dirname: str, side: int, tracer: int, records) -> None:
    """Writes (n, KE) records in the layout read_obc_ts_record reads."""
    import os

    path = os.path.join(dirname, f"OB_{OBC_SIDES[side]}_{'TS'[tracer]}.bin")
    with open(path, "wb") as f:
        for r in records:
            f.write(np.asarray(r, dtype=np.float64).ravel(order="F").astype(">f8").tobytes())


def field_id(name) -> int:
    if isinstance(name, int):
        return name
    if name.startswith("tracer"):
        return F_THO + int(name[6:])
    return FIELDS[name]


class Instance:
    """One regional domain resident on a GPU (an orctm_handle)."""

    def __init__(self, inst: dict, device: int = 0):
        self.lib = _lib.load()
        self.ie, self.je, self.ke = inst["ie"], inst["je"], inst["ke"]
        self.dzw1 = float(np.asarray(inst["dzw"])[0])
        self.ntr = int(inst.get("ntracers", len(inst.get("tracers", [])) or 2))
        d, keep = make_desc(inst, device)
        h = C.c_void_p()
        st = self.lib.orctm_create(C.byref(d), C.byref(h))
        del keep
        _lib.check(st, None)
        self.h = h
        self._inflight = []
        self._step_out = {}

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.orctm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- data movement ------------------------------------------------------
    def shape(self, name: str):
        ie, je, ke = self.ie, self.je, self.ke
        return {"p": (ie, je, ke), "u": (ie + 1, je, ke), "v": (ie, je + 1, ke),
                "w": (ie, je, ke + 1), "2": (ie, je)}[SHAPES.get(name, "p")]

    def _fid(self, name):
        return field_id(name)

    def upload(self, name, arr: np.ndarray):
        a = np.asfortranarray(arr, dtype=np.float64)
        _lib.check(self.lib.orctm_upload(self.h, self._fid(name), _p(a), a.size), self.h)

    def download(self, name, out: np.ndarray | None = None) -> np.ndarray:
        shp = self.shape(name if isinstance(name, str) and not name.startswith("tracer") else "pnh")
        a = np.zeros(shp, dtype=np.float64, order="F") if out is None else out
        _lib.check(self.lib.orctm_download(self.h, self._fid(name), _p(a), a.size), self.h)
        return a

    # -- asynchronous copies (page-locked host arrays; see orctm_gpu.h) -------
    def upload_async(self, name, arr: np.ndarray):
        """Queues the upload of a Fortran-ordered float64 array; the array must
        stay alive and unchanged until wait_copies()."""
        if not (arr.flags.f_contiguous and arr.dtype == np.float64):
            raise ValueError("upload_async needs a Fortran-contiguous float64 array")
        self._inflight.append(arr)
        _lib.check(self.lib.orctm_upload_async(self.h, self._fid(name), _p(arr), arr.size), self.h)

    def download_async(self, name, out: np.ndarray):
        if not (out.flags.f_contiguous and out.dtype == np.float64):
            raise ValueError("download_async needs a Fortran-contiguous float64 array")
        self._inflight.append(out)
        _lib.check(self.lib.orctm_download_async(self.h, self._fid(name), _p(out), out.size),
                   self.h)

    def set_step_outputs(self, outputs: dict):
        """{field name: Fortran-ordered float64 array}: downloaded by each
        step_hotpath as soon as the field is final (empty dict: none)."""
        names = list(outputs)
        ids = (C.c_int * max(len(names), 1))(*[self._fid(k) for k in names])
        ptrs = (_D * max(len(names), 1))(*[_p(outputs[k]) for k in names])
        sizes = (C.c_size_t * max(len(names), 1))(*[outputs[k].size for k in names])
        self._step_out = dict(outputs)
        _lib.check(self.lib.orctm_set_step_outputs(self.h, len(names), ids, ptrs, sizes), self.h)

    def wait_copies(self):
        _lib.check(self.lib.orctm_wait_copies(self.h), self.h)
        self._inflight = []

    # reference output format; codes from ORCTM/code_output.txt
    EXTRA_CODES = {"tracer0": 2, "tracer1": 5, "uko": 3, "vke": 4, "uoo": 3, "voe": 4, "zo": 1,
                   "wo": 7, "wno": 7, "dvo": 111, "avo": 110}

    def write_extra(self, path: str, fields, codes=None, idate: int = 0, append: bool = False):
        """Writes device-resident fields to an EXTRA file (orctm_write_extra)."""
        fields = list(fields)
        codes = list(codes) if codes is not None else [self.EXTRA_CODES[k] for k in fields]
        ids = (C.c_int * len(fields))(*[self._fid(k) for k in fields])
        cs = (C.c_int * len(codes))(*codes)
        _lib.check(self.lib.orctm_write_extra(self.h, path.encode(), int(append), idate,
                                              len(fields), ids, cs), self.h)

    def read_extra(self, path: str, fields, codes=None):
        """Uploads fields from an EXTRA file (orctm_read_extra)."""
        fields = list(fields)
        codes = list(codes) if codes is not None else [self.EXTRA_CODES[k] for k in fields]
        ids = (C.c_int * len(fields))(*[self._fid(k) for k in fields])
        cs = (C.c_int * len(codes))(*codes)
        _lib.check(self.lib.orctm_read_extra(self.h, path.encode(), len(fields), ids, cs), self.h)

    def upload_state(self, st: dict):
        for k in FIELDS:
            if k in st:
                self.upload(k, st[k])
        for n, t in enumerate(st.get("tracers", [])):
            self.upload(f"tracer{n}", t)

    def download_state(self) -> dict:
        out = {k: self.download(k) for k in FIELDS}
        out["tracers"] = [self.download(f"tracer{n}") for n in range(self.ntr)]
        return out

    # -- the reference's routines -----------------------------------------
    def ocuad(self):
        _lib.check(self.lib.orctm_ocuad(self.h), self.h)

    def ocvad(self):
        _lib.check(self.lib.orctm_ocvad(self.h), self.h)

    def ocwad(self):
        _lib.check(self.lib.orctm_ocwad(self.h), self.h)

    def ocadpo(self, tracer: int):
        _lib.check(self.lib.orctm_ocadpo(self.h, tracer), self.h)

    def ocadpo_all(self):
        """OCADPO for every tracer at once (shared transports and volumes)."""
        _lib.check(self.lib.orctm_ocadpo_all(self.h), self.h)

    def octdiff(self):
        _lib.check(self.lib.orctm_octdiff(self.h), self.h)

    def octimf(self):
        _lib.check(self.lib.orctm_octimf(self.h), self.h)

    # -- open boundaries (mo_obcs.f90) -----------------------------------------
    def set_obc(self, obc: dict):
        """INI_OBCS: tidal constants and sponge parameters to the device."""
        o, keep = make_obc(obc)
        _lib.check(self.lib.orctm_set_obc(self.h, C.byref(o)), self.h)

    def obc_eta(self, ldtrun: int):
        """FORC_OBCS_ETA + SPONGE_OBCS_ETA(ZO) at time step ldtrun."""
        _lib.check(self.lib.orctm_obc_eta(self.h, int(ldtrun)), self.h)

    def set_obc_ts(self, tracer: int, cli):
        """FORC_OBCS_TS: side s's climatology record cli[s], (n, KE) or None."""
        arrs = [None if c is None else np.asfortranarray(c, dtype=np.float64) for c in cli]
        ptrs = (_D * 4)(*[_D() if a is None else _p(a) for a in arrs])
        _lib.check(self.lib.orctm_set_obc_ts(self.h, int(tracer), ptrs), self.h)

    def obc_ts(self):
        """SPONGE_OBCS_TS(THO, SAO) towards the records of set_obc_ts."""
        _lib.check(self.lib.orctm_obc_ts(self.h), self.h)

    def set_obc_sponge_exp(self, tao: float):
        """OBC_SPONGE_EXP: the exponential sponge (SPONGE_OBCS_*_EXP) with the
        namelist TAO in s from now on; 0 returns to the 1/x form."""
        _lib.check(self.lib.orctm_set_obc_sponge_exp(self.h, C.c_double(tao)), self.h)

    def obc_uv(self, ldtrun: int):
        """FORC_OBCS_UV + UPGRADE_OBCS_UV + SPONGE_OBCS_UV(UOO, VOE) at time step ldtrun."""
        _lib.check(self.lib.orctm_obc_uv(self.h, int(ldtrun)), self.h)

    def ocvisc(self):
        _lib.check(self.lib.orctm_ocvisc(self.h), self.h)

    # -- barotropic solve (itprep.f90, troneu.f90, ocvtro.f90, ocvtot.f90) -------
    BARO_FIELDS = {"z1o": ("p", _lib.B_Z1O), "b1o": ("p", _lib.B_B1O), "uso": ("u", _lib.B_USO),
                   "vse": ("v", _lib.B_VSE), "uzo": ("u", _lib.B_UZO), "vze": ("v", _lib.B_VZE),
                   "u1o": ("u", _lib.B_U1O), "v1e": ("v", _lib.B_V1E)}

    # OCTHER's constants as the reference driver sets them (orctm.f90:311-330,
    # 503, 561-569, 739-743); eos "unesco" = ADISITJ + RHO1J, "linear" =
    # rho0 + drdt (T - t0) + drds (S - s0)
    THERMO_DEFAULTS = {"eos": "unesco", "rho0": 1025.0, "drdt": -0.2, "drds": 0.78, "t0": 10.0,
                       "s0": 35.0, "grav": 9.806, "crelsal": 3.E-7, "creltem": 0.0,
                       "rhoicwa": 0.91E+03 / 1.025E+03, "rhosnwa": 0.33E+03 / 1.025E+03,
                       "wt": 0.5E-3 / (6.0 ** 3), "cstabeps": 0.05, "dv0": 0.5E-2, "av0": 0.5E-2,
                       "cavocon": 0.0, "cdvocon": 20.0, "aback": 5.E-5, "dback": 5.E-5}
    THERMO_2D = ("sicomo", "sictho", "sicsno", "relsao", "reltho", "giriv", "fu10")
    BAROCLINIC = {"po": ("p3", _lib.C_PO), "stabio": ("p3", _lib.C_STABIO),
                  "rhoo": ("p3", _lib.C_RHOO), "uk1o": ("u3", _lib.C_UK1O),
                  "vk1e": ("v3", _lib.C_VK1E), "eminpo": ("p", _lib.C_EMINPO),
                  "rivrun": ("p", _lib.C_RIVRUN), "kcondep": ("p", _lib.C_KCONDEP)}

    def set_thermo(self, **kw):
        """OCTHER's constants and forcing (orctm_set_thermo).  Keys as
        THERMO_DEFAULTS plus relsal / reltem (default CRELSAL 20 / DZW(1)),
        preff (KE), dbackv / abackv (KE+1) and the (IE, JE) forcing arrays
        THERMO_2D (absent = 0); ``eos`` is "unesco", "linear" or 0 / 1."""
        v = dict(self.THERMO_DEFAULTS, **kw)
        eos = {"unesco": _lib.EOS_UNESCO, "linear": _lib.EOS_LINEAR}.get(v["eos"], v["eos"])
        dzw1 = self.dzw1
        relsal = v.get("relsal", v["crelsal"] * 20. / dzw1)
        reltem = v.get("reltem", v["creltem"] * 20. / dzw1)
        ke = self.ke
        keep = []

        def arr(a, shape=None):
            if a is None:
                return None
            a = np.asfortranarray(a, dtype=np.float64)
            if shape is not None and a.shape != shape:
                raise ValueError(f"OCTHER input shape {a.shape}, expected {shape}")
            keep.append(a)
            return _p(a)

        dbackv = arr(v.get("dbackv", np.full(ke + 1, v["dback"])), (ke + 1,))
        abackv = arr(v.get("abackv", np.full(ke + 1, v["aback"])), (ke + 1,))
        preff = arr(v.get("preff"), (ke,))
        t = _lib.Thermo(int(eos), v["rho0"], v["drdt"], v["drds"], v["t0"], v["s0"], v["grav"],
                        relsal, reltem, v["rhoicwa"], v["rhosnwa"], v["wt"], v["cstabeps"],
                        v["dv0"], v["av0"], v["cavocon"], v["cdvocon"], preff, dbackv, abackv,
                        *[arr(v.get(k), (self.ie, self.je)) for k in self.THERMO_2D])
        _lib.check(self.lib.orctm_set_thermo(self.h, C.byref(t)), self.h)

    def set_coriolis(self, ftwou, ftwov, gila, giph, omega: float = 7.292E-5):
        """OCMODMOM's Coriolis inputs: FTWOU (IE+1, JE), FTWOV (IE, JE+1),
        GILA / GIPH (2 IE, 2 JE)."""
        ie, je = self.ie, self.je
        arrs = [np.asfortranarray(a, dtype=np.float64) for a in (ftwou, ftwov, gila, giph)]
        for a, w in zip(arrs, [(ie + 1, je), (ie, je + 1), (2 * ie, 2 * je), (2 * ie, 2 * je)]):
            if a.shape != w:
                raise ValueError(f"Coriolis input shape {a.shape}, expected {w}")
        c = _lib.Coriolis(*[_p(a) for a in arrs], float(omega))
        _lib.check(self.lib.orctm_set_coriolis(self.h, C.byref(c)), self.h)

    def octher(self):
        _lib.check(self.lib.orctm_octher(self.h), self.h)

    def ocmodmom(self):
        _lib.check(self.lib.orctm_ocmodmom(self.h), self.h)

    def occlit(self) -> float:
        """OCCLIT; returns CONTRA (raises above 1e-3, as the reference aborts)."""
        v = C.c_double()
        _lib.check(self.lib.orctm_occlit(self.h, C.byref(v)), self.h)
        return v.value

    def _baroclinic_shape(self, name):
        kind, which = self.BAROCLINIC[name]
        ie, je, ke = self.ie, self.je, self.ke
        return {"p3": (ie, je, ke), "u3": (ie + 1, je, ke), "v3": (ie, je + 1, ke),
                "p": (ie, je)}[kind], which

    def download_baroclinic(self, name: str) -> np.ndarray:
        shp, which = self._baroclinic_shape(name)
        a = np.zeros(shp, dtype=np.float64, order="F")
        _lib.check(self.lib.orctm_download_baroclinic(self.h, which, _p(a), a.size), self.h)
        return a

    def upload_baroclinic(self, name: str, a):
        shp, which = self._baroclinic_shape(name)
        a = np.asfortranarray(a, dtype=np.float64)
        if a.shape != shp:
            raise ValueError(f"{name} shape {a.shape}, expected {shp}")
        _lib.check(self.lib.orctm_upload_baroclinic(self.h, which, _p(a), a.size), self.h)

    def step_full(self, ldtrun: int, check_contra: bool = True) -> dict:
        """One whole step (orctm_step_full); the solve's statistics and CONTRA.
        With check_contra False a CONTRA above 1e-3 (ORCTM_E_UNSTABLE, where
        the reference aborts) is reported in the result instead of raised."""
        s = SolveStats()
        v = C.c_double()
        allow = (_lib.ORCTM_E_NOT_CONVERGED,) + (() if check_contra else (_lib.E_UNSTABLE,))
        st = _lib.check(self.lib.orctm_step_full(self.h, int(ldtrun), C.byref(s), C.byref(v)),
                        self.h, allow=allow)
        d = s.as_dict()
        d["contra"] = v.value
        d["unstable"] = st == _lib.E_UNSTABLE
        return d

    def set_barotropic(self, deuto, deute, minvalue: float, grav=9.806, stabn=0.6, conn=0.5,
                       rlsa1=1.0 - 0.085, sorpar=1.75, niter=250, eta_forc=False):
        """ITPREP: the SOR coefficients and inverse depths on the device from
        the u/v depths DEUTO (IE+1, JE) and DEUTE (IE, JE+1)."""
        du = np.asfortranarray(deuto, dtype=np.float64)
        dv = np.asfortranarray(deute, dtype=np.float64)
        if du.shape != (self.ie + 1, self.je) or dv.shape != (self.ie, self.je + 1):
            raise ValueError("DEUTO must be (IE+1, JE) and DEUTE (IE, JE+1)")
        b = _lib.Barotropic(_p(du), _p(dv), minvalue, grav, stabn, conn, rlsa1, sorpar,
                            int(niter), int(bool(eta_forc)))
        _lib.check(self.lib.orctm_set_barotropic(self.h, C.byref(b)), self.h)

    def trotest(self, ntry: int = 200, niter: int = 200) -> float:
        """TROTEST: chooses SORPAR (kept for TRONEU) and returns it."""
        v = C.c_double()
        _lib.check(self.lib.orctm_trotest(self.h, int(ntry), int(niter), C.byref(v)), self.h)
        return v.value

    def troneu(self, u1o=None, v1e=None, uzo=None, vze=None):
        """TRONEU: B1O and Z1O from the transports (u: (IE+1, JE), v: (IE, JE+1));
        with none given, from the device's (OCMODMOM's U1O, V1E, OCBARP's UZO, VZE)."""
        if u1o is None and v1e is None and uzo is None and vze is None:
            _lib.check(self.lib.orctm_troneu(self.h, None, None, None, None), self.h)
            return
        arrs = [np.asfortranarray(a, dtype=np.float64) for a in (u1o, v1e, uzo, vze)]
        for a, k in zip(arrs, "uvuv"):
            want = (self.ie + 1, self.je) if k == "u" else (self.ie, self.je + 1)
            if a.shape != want:
                raise ValueError(f"transport shape {a.shape}, expected {want}")
        _lib.check(self.lib.orctm_troneu(self.h, *[_p(a) for a in arrs]), self.h)

    def ocvtro(self):
        _lib.check(self.lib.orctm_ocvtro(self.h), self.h)

    def ocvtot(self):
        _lib.check(self.lib.orctm_ocvtot(self.h), self.h)

    def ocbarp(self):
        _lib.check(self.lib.orctm_ocbarp(self.h), self.h)

    def ocwind(self, txo=None, tye=None, sicomu=None, sicomv=None, tauwatu=None, tauwatv=None):
        """OCWIND: TXO (IE+1, JE), TYE (IE, JE+1), the rest (IE, JE); with none
        given, the forcing of the previous call."""
        if all(a is None for a in (txo, tye, sicomu, sicomv, tauwatu, tauwatv)):
            _lib.check(self.lib.orctm_ocwind(self.h, None, None, None, None, None, None), self.h)
            return
        ie, je = self.ie, self.je
        want = [(ie + 1, je), (ie, je + 1)] + [(ie, je)] * 4
        arrs = [np.asfortranarray(a, dtype=np.float64)
                for a in (txo, tye, sicomu, sicomv, tauwatu, tauwatv)]
        for a, w in zip(arrs, want):
            if a.shape != w:
                raise ValueError(f"OCWIND forcing shape {a.shape}, expected {w}")
        _lib.check(self.lib.orctm_ocwind(self.h, *[_p(a) for a in arrs]), self.h)

    def download_barotropic(self, name: str) -> np.ndarray:
        kind, which = self.BARO_FIELDS[name]
        shp = {"p": (self.ie, self.je), "u": (self.ie + 1, self.je),
               "v": (self.ie, self.je + 1)}[kind]
        a = np.zeros(shp, dtype=np.float64, order="F")
        _lib.check(self.lib.orctm_download_barotropic(self.h, which, _p(a), a.size), self.h)
        return a

    def ocvtot_nh(self) -> dict:
        s = SolveStats()
        _lib.check(self.lib.orctm_ocvtot_nh(self.h, C.byref(s)), self.h,
                   allow=(_lib.ORCTM_E_NOT_CONVERGED,))
        return s.as_dict()

    def step_hotpath(self) -> dict:
        s = SolveStats()
        _lib.check(self.lib.orctm_step_hotpath(self.h, C.byref(s)), self.h,
                   allow=(_lib.ORCTM_E_NOT_CONVERGED,))
        return s.as_dict()

    def set_solver(self, mode: str | int = "fp64", rtol: float = 1e-10, maxit: int = 5000):
        m = {"fp64": SOLVER_FP64, "fp32_refined": SOLVER_FP32_REFINED}.get(mode, mode)
        _lib.check(self.lib.orctm_set_solver(self.h, int(m), float(rtol), int(maxit)), self.h)

    def synchronize(self):
        _lib.check(self.lib.orctm_synchronize(self.h), self.h)

    def set_tuning(self, col: int = -1, spmv: int = -1):
        """Forces the Poisson kernel variants (-1: autotune on the first solve)."""
        _lib.check(self.lib.orctm_set_tuning(self.h, col, spmv), self.h)

    def tuning(self, precision: str = "fp64") -> tuple:
        c, s = C.c_int(), C.c_int()
        pr = 1 if precision == "fp32_refined" else 0
        _lib.check(self.lib.orctm_get_tuning(self.h, pr, C.byref(c), C.byref(s)), self.h)
        return c.value, s.value

    def device_bytes(self) -> int:
        """Device bytes this instance holds (state, tables, solver vectors)."""
        n = C.c_ulonglong()
        _lib.check(self.lib.orctm_device_bytes(self.h, C.byref(n)), self.h)
        return int(n.value)

    # -- device timing -------------------------------------------------------
    def timer_start(self):
        _lib.check(self.lib.orctm_timer_start(self.h), self.h)

    def timer_stop(self) -> float:
        ms = C.c_double()
        _lib.check(self.lib.orctm_timer_stop(self.h, C.byref(ms)), self.h)
        return ms.value

    def set_profiling(self, on: bool):
        _lib.check(self.lib.orctm_set_profiling(self.h, int(bool(on))), self.h)

    def profile(self) -> dict:
        out = {}
        for k, name in enumerate(_lib.PROF_KINDS):
            n, ms = C.c_longlong(), C.c_double()
            _lib.check(self.lib.orctm_profile_get(self.h, k, C.byref(n), C.byref(ms)), self.h)
            out[name] = {"launches": n.value, "ms": ms.value}
        return out

    @staticmethod
    def kernel_launches() -> int:
        return int(_lib.load().orctm_kernel_launches())
