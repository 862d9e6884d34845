"""Seeded synthetic instances of the five benchmark configurations.

No public dataset is involved: every input is generated here from
``numpy.random.Generator(PCG64(seed))`` with base seed 20261203 (instance seed
= base + index).  An instance is a dict holding the reference's model inputs
in its own Fortran layouts (single-rank domain, halos included):

    p-points (IE, JE, KE)      u-points (IE+1, JE, KE)
    v-points (IE, JE+1, KE)    w-points (IE, JE, KE+1)

plus the geometry produced by a BELEG/BODEN grid builder that the caller
passes in (the library's ``orctm_b200.grid.build_grid`` by default).

Configurations (interior sizes; IE = nx + 2, JE = ny + 2):
  c1  512 x 1 x 60 ISW slice, dx = 25 m, dz geometric from 2 m to 1200 m,
      Gaussian sill 900 m tall, 2 km wide at x = 6 km, dt = 2 s
  c2  256 x 256 x 60 tidal box, dx = 500 m, 4000 m plain with filtered-noise
      ridges, ~15 % land, W+S open boundaries, passive tracer, dt = 10 s
  c3  1024 x 1024 x 80, dx = 1852 m (1/60 deg), same generators, dt = 20 s
  c4  ensemble members: nx, ny ~ U[96,512], nz ~ U[40,100], dt = 10 s
  c5  served requests: c4-like members up to 768 x 768 x 80
"""
from __future__ import annotations

import math

import numpy as np

BASE_SEED = 20261203

# Namelist constants of the verification runs (verification/Sect.3.5/OCECTL)
# and of orctm.f90:240, 500-502.
CAULAPTS = 0.0002
CAULAPUV = 0.00375
ALMZER = 1.0e-19


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def geometric_dz(nz: int, dz0: float, total: float) -> np.ndarray:
    """Layer thicknesses growing geometrically from dz0 and summing to total."""
    lo, hi = 1.0 + 1e-12, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        s = dz0 * (r ** nz - 1.0) / (r - 1.0)
        lo, hi = (r, hi) if s < total else (lo, r)
    r = 0.5 * (lo + hi)
    dz = dz0 * r ** np.arange(nz)
    dz *= total / dz.sum()
    return np.round(dz, 6)


def _gauss_filter2d(a: np.ndarray, sigma: float) -> np.ndarray:
    """Periodic Gaussian filter via FFT (input generation only)."""
    nx, ny = a.shape
    kx = np.fft.fftfreq(nx)[:, None]
    ky = np.fft.fftfreq(ny)[None, :]
    h = np.exp(-2.0 * (math.pi * sigma) ** 2 * (kx ** 2 + ky ** 2))
    return np.real(np.fft.ifft2(np.fft.fft2(a) * h))


def _f(shape) -> np.ndarray:
    return np.zeros(shape, dtype=np.float64, order="F")


def _metrics(ie: int, je: int, dx: float, dy: float):
    return {
        "dlxp": np.full((ie, je), dx, order="F"), "dlyp": np.full((ie, je), dy, order="F"),
        "dlxu": np.full((ie + 1, je), dx, order="F"), "dlyu": np.full((ie + 1, je), dy, order="F"),
        "dlxv": np.full((ie, je + 1), dx, order="F"), "dlyv": np.full((ie, je + 1), dy, order="F"),
    }


def _bathymetry_box(g: np.random.Generator, nx: int, ny: int, depth: float = 4000.0,
                    land_frac: float = 0.15) -> np.ndarray:
    """4000 m plain plus white noise Gaussian-filtered (sigma = 8 cells).  The
    positive anomalies are scaled into ridges so that the (1 - land_frac)
    quantile sits at 10 m depth: about land_frac of the cells become land
    (depth < 10 m) and the ridge flanks pass through every depth between."""
    n = _gauss_filter2d(g.standard_normal((nx, ny)), 8.0)
    n = (n - n.mean()) / n.std()
    q_land = np.quantile(n, 1.0 - land_frac)
    r = np.clip(n / q_land, 0.0, None)
    return np.clip(depth - (depth - 10.0) * r, 0.0, depth)


def raw_instance(name: str, index: int = 0, seed: int | None = None, **over) -> dict:
    """Model inputs before the grid builder runs (depth, metrics, dz, dt, ...).
    ``closed=True`` makes every side land (whole steps of c2-c5: the
    reference's open-boundary elevation row in TRONEU, Z1O = B1O / XX,
    troneu.f90:67-102, is explicit and grows at these time steps)."""
    s = BASE_SEED + index if seed is None else seed
    g = rng(s)
    ob = {"west": False, "east": False, "north": False, "south": False}
    tracers = 2
    if name == "c1":
        nx, ny, nz = over.get("nx", 512), over.get("ny", 1), over.get("nz", 60)
        dx, dt = 25.0, 2.0
        dzw = geometric_dz(nz, 2.0, 1200.0)
        x = (np.arange(nx + 2) - 0.5) * dx
        depth = 1200.0 - 900.0 * np.exp(-(((x - 6000.0) / 1000.0) ** 2))
        depto = np.repeat(depth[:, None], ny + 2, axis=1)
        depto[0, :] = 0.0          # closed west (land column i = 1)
        depto[-1, :] = 0.0         # closed east (land column i = IE)
        depto[:, 0] = 0.0          # land rows j = 1, JE: a vertical slice
        depto[:, -1] = 0.0
        tide = None
    elif name in ("c2", "c3", "c4", "c5"):
        if name == "c2":
            nx, ny, nz, dx, dt = 256, 256, 60, 500.0, 10.0
        elif name == "c3":
            nx, ny, nz, dx, dt = 1024, 1024, 80, 1852.0, 20.0
        else:
            hi = 512 if name == "c4" else 768
            nx, ny = int(g.integers(96, hi + 1)), int(g.integers(96, hi + 1))
            nz = int(g.integers(40, (100 if name == "c4" else 80) + 1))
            dx, dt = 500.0, 10.0
        nx, ny, nz = over.get("nx", nx), over.get("ny", ny), over.get("nz", nz)
        dx = over.get("dx", dx)
        dzw = geometric_dz(nz, 2.0, 4000.0)
        depto = np.zeros((nx + 2, ny + 2))
        depto[:, :] = np.pad(_bathymetry_box(g, nx, ny), 1, mode="edge")
        # closed north (j = 1) and east (i = IE): land halo; W and S open
        depto[-1, :] = 0.0
        depto[:, 0] = 0.0
        ob["west"] = ob["south"] = True
        tracers = 3
        tide = {"period": 44712.0,
                "amplitude": 1.0 if name in ("c2", "c3") else float(g.uniform(0.5, 1.5)),
                "phase": 0.0 if name in ("c2", "c3") else float(g.uniform(0.0, 2 * math.pi))}
    else:
        raise ValueError(f"unknown configuration {name!r}")
    if over.get("closed"):
        # every side land: the open west and south of c2-c5 closed
        depto[0, :] = depto[-1, :] = 0.0
        depto[:, 0] = depto[:, -1] = 0.0
        ob = {k: False for k in ob}
    dt = over.get("dt", dt)
    ie, je, ke = nx + 2, ny + 2, nz
    inst = {"name": name, "seed": s, "ie": ie, "je": je, "ke": ke, "nx": nx, "ny": ny, "nz": nz,
            "dt": float(dt), "dzw": np.ascontiguousarray(dzw, dtype=np.float64),
            "depto_raw": np.asfortranarray(depto, dtype=np.float64), "ob": ob,
            "almzer": ALMZER, "aulapts": CAULAPTS * dt / 3600.0,
            "aulapuv": CAULAPUV * dt / 3600.0, "ah00": 0.0, "ntracers": tracers, "tide": tide}
    inst.update(_metrics(ie, je, dx, dx))
    return inst


def default_builder():
    from . import grid

    return grid.build_grid


def make_instance(name: str, index: int = 0, seed: int | None = None, builder=None,
                  cfl: float | None = None, cfl_w="auto", **over) -> dict:
    """Raw inputs + geometry (via ``builder``) + a seeded initial state.

    ``cfl`` rescales the horizontal velocities to that Courant number (kernel
    stress tests); by default velocities are O(0.1-0.3 m/s).  ``cfl_w`` caps
    the vertical Courant number of the initial w (the scheme is stable below
    1): by default at VERTICAL_CFL unless ``cfl`` is given; None leaves it
    uncapped."""
    inst = raw_instance(name, index=index, seed=seed, **over)
    builder = builder or default_builder()
    depto, geo = builder(inst["ie"], inst["je"], inst["ke"], inst["dt"], inst["dzw"],
                         inst["depto_raw"], inst["dlxp"], inst["dlyp"], inst["dlxu"],
                         inst["dlyu"], inst["dlxv"], inst["dlyv"])
    inst["depto"] = depto
    inst.update(geo)
    inst.update(initial_state(inst, cfl=cfl, cfl_w=cfl_w))
    return inst


# Open-boundary namelist OCEOBC of the verification runs
# (verification/Sect.3.5/OCECTL): sponge widths, relaxation times and the two
# tidal periods (semidiurnal and diurnal, s).
OBC_WIDTH = 30
OBC_RELAX_INNER = 44714.1643
OBC_PERIODS = (44714.1643, 86164.0906)
OBC_BOUNDARIES = ("west", "east", "north", "south")


def obc_points(ie: int, je: int, b: int, v: int) -> int:
    """Points along boundary b (0 W, 1 E, 2 N, 3 S) of variable v (0 z, 1 u,
    2 v), as the reference dimensions OB{W,E,N,S}{Z,U,V}am (mo_obcs.f90:124-138)."""
    if b < 2:
        return je + 1 if v == 2 else je
    return ie + 1 if v == 1 else ie


def make_obc(inst: dict, seed: int | None = None, width: int | None = None,
             relax_bound: float | None = None) -> dict:
    """Seeded tidal harmonic constants and 1/x sponge parameters for the open
    boundaries of ``inst`` (the inputs INI_OBCS reads from OB_*_Amp.bin /
    OB_*_Gph.bin and namelist OCEOBC, mo_obcs.f90:263-506).

    Amplitudes vary smoothly along each boundary around the instance's tide
    amplitude (elevation, m) and its shallow-water velocity (m/s); phases are
    times (s) that lag along the boundary like a progressive wave.  The
    boundary relaxation time defaults to DT, so that the sponge sets the
    outermost cell to the tidal value."""
    ie, je = inst["ie"], inst["je"]
    g = rng((inst["seed"] if seed is None else seed) + 7919)
    tide = inst.get("tide") or {"amplitude": 1.0, "phase": 0.0}
    ntide = len(OBC_PERIODS)
    amp = [[None] * 3 for _ in range(4)]
    pha = [[None] * 3 for _ in range(4)]
    depth = float(np.max(inst["depto"])) if "depto" in inst else 4000.0
    uscale = math.sqrt(9.81 / max(depth, 1.0))
    for b, name in enumerate(OBC_BOUNDARIES):
        if not inst["ob"][name]:
            continue
        for v in range(3):
            n = obc_points(ie, je, b, v)
            s = np.linspace(0.0, 1.0, n)
            a = np.empty((n, ntide), order="F")
            p = np.empty((n, ntide), order="F")
            for td, per in enumerate(OBC_PERIODS):
                base = tide["amplitude"] * (1.0 if td == 0 else 0.3) * (1.0 if v == 0 else uscale)
                a[:, td] = base * (1.0 + 0.2 * np.sin(2 * math.pi * (s + g.uniform())))
                p[:, td] = (tide["phase"] / (2 * math.pi) + 0.25 * s + g.uniform(0, 0.05)) * per
            amp[b][v], pha[b][v] = a, p
    w = width if width is not None else min(OBC_WIDTH, max(1, (ie - 2) // 3), max(1, (je - 2) // 3))
    return {"ntide": ntide, "period": np.array(OBC_PERIODS, dtype=np.float64),
            "sponge": [int(inst["ob"][k]) for k in OBC_BOUNDARIES], "width": [w] * 4,
            "relax_inner": OBC_RELAX_INNER,
            "relax_bound": float(inst["dt"] if relax_bound is None else relax_bound),
            "amp": amp, "pha": pha}


def make_obc_ts(inst: dict, tracer: int, seed: int | None = None) -> list:
    """Seeded boundary climatology of one tracer (0 temperature, 1 salinity):
    per open side an (n, KE) record (n = JE west/east, IE north/south) as
    FORC_OBCS_TS reads from OB_<Side>_T.bin / OB_<Side>_S.bin
    (mo_obcs.f90:932-1012), near the instance's own profile with a smooth
    along-boundary variation; None for closed sides."""
    ie, je, ke = inst["ie"], inst["je"], inst["ke"]
    g = rng((inst["seed"] if seed is None else seed) + 104729 + tracer)
    t = inst["tracers"][tracer]
    prof = np.array([float(np.mean(t[:, :, k])) for k in range(ke)])
    out = []
    for b, name in enumerate(OBC_BOUNDARIES):
        if not inst["ob"][name]:
            out.append(None)
            continue
        n = je if b < 2 else ie
        s = np.linspace(0.0, 1.0, n)[:, None]
        amp = 0.5 if tracer == 0 else 0.1
        c = prof[None, :] + amp * np.sin(2 * math.pi * (s + g.uniform())) \
            + g.normal(0.0, 0.01 * amp, (n, ke))
        out.append(np.asfortranarray(c))
    return out


# default cap on the vertical Courant number |w| dt / DDPO of initial states
VERTICAL_CFL = 0.5


def _wdiag(inst: dict, u: np.ndarray, v: np.ndarray) -> np.ndarray:
    """w from continuity, bottom-up (the form of ocvtot_nh.f90:215-236)."""
    ie, je, ke = inst["ie"], inst["je"], inst["ke"]
    w = _f((ie, je, ke + 1))
    area = inst["dlxp"] * inst["dlyp"]
    fu = u * inst["dduo"] * inst["dlyu"][:, :, None]
    fv = v * inst["ddue"] * inst["dlxv"][:, :, None]
    for k in range(ke - 1, -1, -1):
        div = (fu[:-1, :, k] - fu[1:, :, k]) + (fv[:, 1:, k] - fv[:, :-1, k])
        w[:, :, k] = w[:, :, k + 1] + inst["weto"][:, :, k] * div / area
    return w


def initial_state(inst: dict, cfl: float | None = None, cfl_w="auto") -> dict:
    # cfl_w: cap on the vertical Courant number of the initial w; "auto" is
    # 0.5 for workloads (many steps) and no cap for kernel stress cases that
    # set a horizontal Courant number (single routine applications)
    if cfl_w == "auto":
        cfl_w = None if cfl is not None else VERTICAL_CFL
    g = rng(inst["seed"] + 7919)
    ie, je, ke, dt = inst["ie"], inst["je"], inst["ke"], inst["dt"]
    dx = float(inst["dlxp"][0, 0])
    z = -inst["tiestu"][:ke]                                   # cell-centre height
    x = (np.arange(ie) - 0.5) * dx
    # interface depression (c1) / none, and the tanh stratification
    if inst["name"] == "c1":
        eta = -30.0 / np.cosh((x - 2000.0) / 500.0) ** 2
    else:
        eta = np.zeros(ie)
    tho = 15.0 + 5.0 * np.tanh((z[None, None, :] + 50.0 - eta[:, None, None]) / 10.0)
    tho = np.broadcast_to(tho, (ie, je, ke)).copy(order="F")
    tho += 1e-4 * g.standard_normal((ie, je, ke))
    sao = np.full((ie, je, ke), 35.0, order="F")
    tracers = [np.asfortranarray(tho), sao]
    if inst["ntracers"] >= 3:
        tracers.append(np.asfortranarray(g.uniform(0.0, 1.0, (ie, je, ke))))

    def smooth3(shape, sig):
        a = g.standard_normal(shape)
        out = np.empty(shape)
        for k in range(shape[2]):
            out[:, :, k] = _gauss_filter2d(a[:, :, k], sig) if min(shape[:2]) > 4 else a[:, :, k]
        return out / max(np.abs(out).max(), 1e-30)

    prof = 0.6 + 0.4 * np.cos(np.linspace(0.0, math.pi, ke))[None, None, :]
    u = (0.25 * prof * smooth3((ie + 1, je, ke), 6.0) + 0.02 * g.standard_normal((ie + 1, je, ke)))
    v = (0.25 * prof * smooth3((ie, je + 1, ke), 6.0) + 0.02 * g.standard_normal((ie, je + 1, ke)))
    if inst["ny"] == 1:
        v[:] = 0.0
    if cfl is not None:
        s = cfl * dx / dt / max(np.abs(u).max(), np.abs(v).max(), 1e-30)
        u *= s
        v *= s
    u = np.asfortranarray(u * inst["amsuo"])
    v = np.asfortranarray(v * inst["amsue"])
    w = _wdiag(inst, u, v)
    if cfl_w is not None:
        # The smooth random (u, v) are not divergence-free, and w integrated
        # from continuity over thousands of metres can reach tenths of m/s;
        # across the thin upper layers that exceeds the limited advection's
        # stability limit (vertical Courant number 1).  Scale (u, v) -- and
        # with them w, which is linear in them -- so that |w| dt / DDPO stays
        # below cfl_w on both cells of every interface.
        d = inst["ddpo"]
        thin = np.where(d > 0.0, d, np.inf)
        lim = np.minimum(thin[:, :, :-1], thin[:, :, 1:])
        cz = max(float((np.abs(w[:, :, 1:ke]) * dt / lim).max()),
                 float((np.abs(w[:, :, 0]) * dt / thin[:, :, 0]).max()))
        if cz > cfl_w:
            s = cfl_w / cz
            u = np.asfortranarray(u * s)
            v = np.asfortranarray(v * s)
            w = np.asfortranarray(w * s)
    # synthetic hydrostatic increment: the state one step before (drives the NH RHS)
    du = 1e-3 * smooth3((ie + 1, je, ke), 4.0) * inst["amsuo"]
    dv = 1e-3 * smooth3((ie, je + 1, ke), 4.0) * inst["amsue"]
    if inst["ny"] == 1:
        dv[:] = 0.0
    u1 = np.asfortranarray(u - du)
    v1 = np.asfortranarray(v - dv)
    w1 = _wdiag(inst, u1, v1)
    zo = np.asfortranarray(0.2 * g.standard_normal((ie, je)) * inst["weto"][:, :, 0])
    kep = ke + 1
    lev = np.arange(kep)
    dvo = np.asfortranarray(np.broadcast_to(2e-5 + 1e-3 * np.exp(-lev / 5.0), (ie, je, kep)).copy())
    dvo *= 1.0 + 0.1 * g.uniform(-1, 1, (ie, je, kep))
    avo = np.asfortranarray(np.broadcast_to(2e-4 + 5e-3 * np.exp(-lev / 5.0), (ie, je, kep)).copy())
    avo *= 1.0 + 0.1 * g.uniform(-1, 1, (ie, je, kep))
    # OCTHER masks both with WETO (octher.f90:382-393) and zeroes DVO(KEP)
    dvo[:, :, :ke] *= inst["weto"]
    avo[:, :, :ke] *= inst["weto"]
    dvo[:, :, 0] = 0.0
    dvo[:, :, -1] = 0.0
    return {
        "uoo": u, "voe": v, "wno": np.asfortranarray(w.copy()),
        "uko": np.asfortranarray(u.copy()), "vke": np.asfortranarray(v.copy()),
        "wo": np.asfortranarray(w.copy()),
        "uoo1": u1, "voe1": v1, "wno1": w1,
        "pnh": _f((ie, je, ke)), "zo": zo,
        "tracers": tracers, "dvo": np.asfortranarray(dvo), "avo": np.asfortranarray(avo),
    }


STATE_KEYS = ("uoo", "voe", "wno", "uko", "vke", "wo", "uoo1", "voe1", "wno1", "pnh", "zo",
              "dvo", "avo")


def copy_state(inst: dict) -> dict:
    st = {k: np.array(inst[k], order="F", copy=True) for k in STATE_KEYS}
    st["tracers"] = [np.array(t, order="F", copy=True) for t in inst["tracers"]]
    return st


def barotropic_minvalue(inst: dict) -> float:
    """BODEN's small thickness threshold MIN(1, DZW(1)/10) (boden.f90)."""
    return min(1.0, float(inst["dzw"][0]) / 10.0)


def make_barotropic(inst: dict, seed: int | None = None) -> dict:
    """Seeded inputs of the barotropic solve (TRONEU, OCVTRO, OCVTOT): the
    previous and the new vertically integrated transports U1O/UZO (u-points,
    (IE+1, JE), m^2/s) and V1E/VZE (v-points, (IE, JE+1)), smooth, of the
    size of the instance's velocities times its depths, zero where the
    column is dry."""
    ie, je = inst["ie"], inst["je"]
    g = rng((inst["seed"] if seed is None else seed) + 31337)
    depth = np.asarray(inst["depto"], dtype=np.float64)
    du = np.zeros((ie + 1, je))
    du[1:ie, :] = np.minimum(depth[:-1, :], depth[1:, :])
    dv = np.zeros((ie, je + 1))
    dv[:, 1:je] = np.minimum(depth[:, :-1], depth[:, 1:])

    def smooth(shape, amp):
        a = g.standard_normal(shape)
        a = _gauss_filter2d(a, 3.0) if min(shape) > 8 else a
        return np.asfortranarray(amp * a / max(np.abs(a).max(), 1e-30))

    out = {}
    for k, shp, d in (("u1o", (ie + 1, je), du), ("uzo", (ie + 1, je), du),
                      ("v1e", (ie, je + 1), dv), ("vze", (ie, je + 1), dv)):
        out[k] = np.asfortranarray(smooth(shp, 0.1) * d)
    return out


def make_wind(inst: dict, seed: int | None = None) -> dict:
    """Seeded surface forcing of OCWIND: wind stress TXO (u-points, (IE+1,
    JE)) and TYE (v-points, (IE, JE+1)) in N/m^2 / (rho) units of m^2/s^2,
    the open-water fractions SICOMU / SICOMV in [0, 1] and the ice-ocean
    stresses TAUWATU / TAUWATV, both (IE, JE) as the reference declares them
    (mo_commo1.f90:160-167)."""
    ie, je = inst["ie"], inst["je"]
    g = rng((inst["seed"] if seed is None else seed) + 4242)
    return {"txo": np.asfortranarray(1e-4 * g.standard_normal((ie + 1, je))),
            "tye": np.asfortranarray(1e-4 * g.standard_normal((ie, je + 1))),
            "sicomu": np.asfortranarray(g.uniform(0.0, 1.0, (ie, je))),
            "sicomv": np.asfortranarray(g.uniform(0.0, 1.0, (ie, je))),
            "tauwatu": np.asfortranarray(1e-4 * g.standard_normal((ie, je))),
            "tauwatv": np.asfortranarray(1e-4 * g.standard_normal((ie, je)))}


def make_thermo(inst: dict, seed: int | None = None, eos: int | None = None) -> dict:
    """Seeded surface forcing and switches of OCTHER: restoring targets RELSAO
    / RELTHO near the surface tracers, 10 m wind speed FU10 (m/s), a few river
    inflow points GIRIV (m/s), and no sea ice.  The vertical slice c1 uses the
    linear equation of state its description asks for; the other workloads
    the reference's UNESCO EOS.  Constants not given default to the
    reference driver's (oracle.THERMO_DEFAULTS, also in orctm_b200.api)."""
    ie, je = inst["ie"], inst["je"]
    g = rng((inst["seed"] if seed is None else seed) + 2718)
    tr = inst["tracers"]
    w1 = inst["weto"][:, :, 0]
    giriv = np.zeros((ie, je))
    wet = np.argwhere(w1 > 0.5)
    if len(wet):
        for q in g.choice(len(wet), size=min(3, len(wet)), replace=False):
            i, j = wet[q]
            giriv[i, j] = 1e-4 * g.uniform(0.5, 1.5)
    return {"eos": (1 if inst["name"] == "c1" else 0) if eos is None else eos,
            "relsao": np.asfortranarray(tr[1][:, :, 0] + 0.1 * g.standard_normal((ie, je))),
            "reltho": np.asfortranarray(tr[0][:, :, 0] + 0.5 * g.standard_normal((ie, je))),
            "creltem": 1e-7,
            "fu10": np.asfortranarray(g.uniform(2.0, 12.0, (ie, je))),
            "giriv": np.asfortranarray(giriv)}


def make_coriolis(inst: dict, lat0: float = 20.5, seed: int | None = None) -> dict:
    """Coriolis inputs of OCMODMOM for a plane grid near latitude lat0 (deg):
    FTWOU / FTWOV = 2 OMEGA sin(lat) at u- / v-points and the double-resolution
    longitudes / latitudes GILA / GIPH (2 IE, 2 JE), radians, with a slight
    seeded rotation so that both of their differences are non-zero."""
    ie, je = inst["ie"], inst["je"]
    g = rng((inst["seed"] if seed is None else seed) + 1618)
    omega, radius = 7.292E-5, 6.371E6
    dx = float(inst["dlxp"][0, 0])
    rot = g.uniform(0.05, 0.15)
    ii, jj = np.meshgrid(np.arange(1, 2 * ie + 1), np.arange(1, 2 * je + 1), indexing="ij")
    x, y = 0.5 * dx * ii, 0.5 * dx * jj
    xr, yr = x * math.cos(rot) - y * math.sin(rot), x * math.sin(rot) + y * math.cos(rot)
    lat = math.radians(lat0) + yr / radius
    lon = xr / (radius * math.cos(math.radians(lat0)))
    # u-point (i, j) sits at the double-resolution index (2 i + 1, 2 j), v at (2 i, 2 j + 1)
    ftwou = np.zeros((ie + 1, je))
    ftwov = np.zeros((ie, je + 1))
    for i in range(ie + 1):
        ftwou[i, :] = 2.0 * omega * np.sin(lat[min(2 * i, 2 * ie - 1), 1::2])
    for j in range(je + 1):
        ftwov[:, j] = 2.0 * omega * np.sin(lat[1::2, min(2 * j, 2 * je - 1)])
    return {"ftwou": np.asfortranarray(ftwou), "ftwov": np.asfortranarray(ftwov),
            "gila": np.asfortranarray(lon), "giph": np.asfortranarray(lat), "omega": omega}


def initial_kcondep(inst: dict) -> np.ndarray:
    """KCONDEP as BODEN initialises it (boden.f90:261): 1 wet, -99 dry."""
    w = inst["weto"][:, :, 0]
    return np.asfortranarray(np.where(w > 0.5, 1, -99).astype(np.int32))
