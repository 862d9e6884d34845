"""Independent numpy restatements used to cross-check the C oracle.

Written from the reference Fortran, not from oracle/orctm_oracle.c, and
vectorised over (i, j): OCADPO (ocadpo.f90:94-348) and the operator of
compute_matrix (mo_petsc.f90:543-782).  Test infrastructure only.
Arrays are 0-based numpy views of the Fortran arrays: p-point index
i-1 <-> Fortran I, u-point index i <-> Fortran I (I_start = 0).
"""
import math

import numpy as np
import scipy.sparse as sp


def ocadpo(g, trf, uko, vke, wo, zo):
    """Returns the advected tracer (float64, same layout as trf)."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    dt = g["dt"]
    weto, ddpo = g["weto"], g["ddpo"]
    dlxp, dlyp = g["dlxp"], g["dlyp"]
    dduo, dlyu, ddue, dlxv = g["dduo"], g["dlyu"], g["ddue"], g["dlxv"]
    T = trf.copy()
    s1o = weto * dlxp[:, :, None] * dlyp[:, :, None] * ddpo
    s1o[:, :, 0] = s1o[:, :, 0] + dlxp * dlyp * weto[:, :, 0] * (zo - wo[:, :, 0] * dt)
    I = slice(1, ie - 1)
    J = slice(1, je - 1)
    # vertical
    trp = np.zeros((ie, je, ke + 1))   # index k-1 <-> TRP(K), K = 1..KEP
    wtp = np.zeros((ie, je, ke + 1))
    trm = np.zeros((ie, je, ke + 1))   # index k   <-> TRM(K), K = 0..KE
    wtm = np.zeros((ie, je, ke + 1))
    for k in range(ke):
        kup, klo = max(k - 1, 0), min(k + 1, ke - 1)
        t, tu, tl = T[I, J, k], T[I, J, kup], T[I, J, klo]
        abl = np.abs(tu - tl)
        zwabl = np.abs(tu + tl - 2. * t)
        c = 0.5 * dt * dlyp[I, J] * dlxp[I, J]
        up = c * (wo[I, J, k] + np.abs(wo[I, J, k]))
        um = c * (np.abs(wo[I, J, k + 1]) - wo[I, J, k + 1])
        scha = np.where(0. > (abl - zwabl) / (abl + 1e-20), 0., (abl - zwabl) / (abl + 1e-20))
        x = scha * s1o[I, J, k] / (up + um + 1e-20)
        w = weto[I, J, klo]
        sch = np.where(x < w, x, w)
        if k == 0 or k == ke - 1:
            sch = np.zeros_like(sch)
        schi = 1. - sch
        trp[I, J, k] = up * (schi * t + sch * 0.5 * (t + tu))
        trm[I, J, k + 1] = um * (schi * t + sch * 0.5 * (t + tl))
        wtp[I, J, k] = up
        wtm[I, J, k + 1] = um
    new = T.copy()
    for k in range(ke):
        m = weto[I, J, k] > 0.5
        rn = s1o[I, J, k] + wtp[I, J, k + 1] - wtp[I, J, k] - wtm[I, J, k + 1] + wtm[I, J, k]
        t1 = (T[I, J, k] * s1o[I, J, k] + trp[I, J, k + 1] - trp[I, J, k] - trm[I, J, k + 1]
              + trm[I, J, k]) / np.where(m, rn, 1.0)
        new[I, J, k] = np.where(m, t1, T[I, J, k])
        s1o[I, J, k] = np.where(m, rn, s1o[I, J, k])
    T = new
    # x: face arrays indexed by p-index
    for direction in ("x", "y"):
        trp = np.zeros((ie, je, ke))
        trm = np.zeros((ie, je, ke))
        wtp = np.zeros((ie, je, ke))
        wtm = np.zeros((ie, je, ke))
        if direction == "x":
            t, tp_, tm_ = T[I, J, :], T[2:, J, :], T[:-2, J, :]   # tp_: I+1, tm_: I-1
            u0 = uko[2:ie, J, :]        # u-point I   (u index I)
            um1 = uko[1:ie - 1, J, :]   # u-point I-1
            up = 0.5 * dt * dduo[2:ie, J, :] * dlyu[2:ie, J][:, :, None] * (u0 + np.abs(u0))
            um = 0.5 * dt * dduo[1:ie - 1, J, :] * (np.abs(um1) - um1) * dlyu[1:ie - 1, J][:, :, None]
            mask = weto[I, J, :] * weto[2:, J, :] * weto[:-2, J, :]
        else:
            t, tp_, tm_ = T[I, J, :], T[I, :-2, :], T[I, 2:, :]   # tp_: J-1, tm_: J+1
            vn = vke[I, 1:je - 1, :]    # v-point J-1 (v index J-1)
            vs = vke[I, 2:je, :]        # v-point J
            up = 0.5 * dt * ddue[I, 1:je - 1, :] * dlxv[I, 1:je - 1][:, :, None] * (vn + np.abs(vn))
            um = 0.5 * dt * ddue[I, 2:je, :] * dlxv[I, 2:je][:, :, None] * (np.abs(vs) - vs)
            mask = weto[I, J, :] * weto[I, :-2, :] * weto[I, 2:, :]
        abl = np.abs(tp_ - tm_)
        zwabl = np.abs(tp_ + tm_ - 2. * t)
        q = (abl - zwabl) / (abl + 1e-20)
        if direction == "x":
            scha = np.where(0. > q, 0., q) * weto[I, J, :] * weto[2:, J, :] * weto[:-2, J, :]
        else:
            scha = np.where(0. > q, 0., q) * weto[I, J, :] * weto[I, :-2, :] * weto[I, 2:, :]
        x = scha * s1o[I, J, :] / (up + um + 1e-20)
        sch = np.where(x < 1., x, 1.)
        schi = 1. - sch
        trp[I, J, :] = up * (schi * t + sch * 0.5 * (t + tp_))
        trm[I, J, :] = um * (schi * t + sch * 0.5 * (t + tm_))
        wtp[I, J, :] = up
        wtm[I, J, :] = um
        if direction == "x":
            rn = s1o[I, J] + wtp[:-2, J] - wtp[I, J] - wtm[I, J] + wtm[2:, J]
            t1 = (T[I, J] * s1o[I, J] + trp[:-2, J] - trp[I, J] - trm[I, J] + trm[2:, J])
        else:
            rn = s1o[I, J] + wtp[I, 2:] - wtp[I, J] - wtm[I, J] + wtm[I, :-2]
            t1 = (T[I, J] * s1o[I, J] + trp[I, 2:] - trp[I, J] - trm[I, J] + trm[I, :-2])
        m = weto[I, J, :] > 0.5
        new = T.copy()
        new[I, J, :] = np.where(m, t1 / np.where(m, rn, 1.0), T[I, J, :])
        s1o[I, J, :] = np.where(m, rn, s1o[I, J, :])
        T = new
    return T


def _zw(ddpo, dzw):
    ie, je, ke = ddpo.shape
    zw = np.zeros((ie, je, ke + 1))
    for K in range(1, ke + 2):
        if K == 1:
            d = np.where(ddpo[:, :, 0] == 0, dzw[0] / 2.0, ddpo[:, :, 0] / 2.0)
        elif K == ke + 1:
            d = np.where(ddpo[:, :, ke - 1] == 0, dzw[ke - 1], ddpo[:, :, ke - 1])
        else:
            a, b = ddpo[:, :, K - 2], ddpo[:, :, K - 1]
            d = np.where(a == 0, (dzw[K - 1] + dzw[K - 2]) / 2.0, np.where(b == 0, a, (a + b) / 2.0))
        zw[:, :, K - 1] = 1.0 / d
    return zw


def matrix(g):
    """compute_matrix as scipy CSR (single rank, no cyclic boundaries)."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    nx, ny = ie - 2, je - 2
    w = g["weto"]
    zw = _zw(g["ddpo"], g["dzw"])
    zp = 1.0 / ((1.0 / zw[:, :, :-1] + 1.0 / zw[:, :, 1:]) / 2.0)
    xu = 1.0 / g["dlxu"][1:, :]      # XU(I,J), I = 1..IE
    xp = 1.0 / g["dlxp"]
    yv = 1.0 / g["dlyv"][:, 1:]      # YV(I,J), J = 1..JE
    yp = 1.0 / g["dlyp"]
    rows, cols, vals = [], [], []
    idx = lambda i, j, k: (i - 1) + nx * ((j - 1) + ny * k)   # i, j: p-index 1..nx
    for k in range(ke):
        for j in range(1, je - 1):
            for i in range(1, ie - 1):
                r = idx(i, j, k)
                XW = xu[i - 1, j] * xp[i, j]; XC = (xu[i - 1, j] + xu[i, j]) * xp[i, j]; XE = xu[i, j] * xp[i, j]
                YN = yv[i, j - 1] * yp[i, j]; YC = (yv[i, j - 1] + yv[i, j]) * yp[i, j]; YS = yv[i, j] * yp[i, j]
                ZU = zw[i, j, k] * zp[i, j, k]; ZC = (zw[i, j, k] + zw[i, j, k + 1]) * zp[i, j, k]
                ZD = zw[i, j, k + 1] * zp[i, j, k]
                if w[i, j, k] == 0:
                    rows.append(r); cols.append(r); vals.append(-(XC + YC + ZC))
                    continue
                if w[i - 1, j, k] == 0 and w[i + 1, j, k] == 1:
                    XW = 0.0; XC = xu[i, j] * xp[i, j]
                elif w[i - 1, j, k] == 1 and w[i + 1, j, k] == 0:
                    XE = 0.0; XC = xu[i - 1, j] * xp[i, j]
                elif w[i - 1, j, k] == 0 and w[i + 1, j, k] == 0:
                    XW = XE = XC = 0.0
                if w[i, j - 1, k] == 0 and w[i, j + 1, k] == 1:
                    YN = 0.0; YC = yv[i, j] * yp[i, j]
                elif w[i, j - 1, k] == 1 and w[i, j + 1, k] == 0:
                    YS = 0.0; YC = yv[i, j - 1] * yp[i, j]
                elif w[i, j - 1, k] == 0 and w[i, j + 1, k] == 0:
                    YN = YS = YC = 0.0
                if k == 0:
                    ZU = 0.0
                elif k == ke - 1 or w[i, j, k + 1] == 0:
                    ZD = 0.0; ZC = zw[i, j, k] * zp[i, j, k]
                ent = []
                if w[i - 1, j, k] == 1 and i - 1 != 0: ent.append((r - 1, XW))
                if w[i, j - 1, k] == 1 and j - 1 != 0: ent.append((r - nx, YN))
                if k != 0: ent.append((r - nx * ny, ZU))
                ent.append((r, -(XC + YC + ZC)))
                if k != ke - 1 and w[i, j, k + 1] == 1: ent.append((r + nx * ny, ZD))
                if w[i, j + 1, k] == 1 and j - 1 != ny - 1: ent.append((r + nx, YS))
                if w[i + 1, j, k] == 1 and i - 1 != nx - 1: ent.append((r + 1, XE))
                for c, v in ent:
                    rows.append(r); cols.append(c); vals.append(v)
    n = nx * ny * ke
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def obc_sponge_ts(g, obc, cli, x, salinity=False):
    """FORC_OBCS_TS + SPONGE_OBCS_TS (mo_obcs.f90:932-1272) on one tracer in
    the same per-cell distance form as obc_sponge, the boundary value of
    level k being cli[b][q, k] times the boundary cell's WETO at level k.
    salinity: the tracer is SAO (SPONGE_OBCS_TS_EXP's south band)."""
    return obc_sponge(g, obc, 0, x, "t", cli=cli, salinity=salinity)


def _exp_rates(g, obc, kind, w, ni, nj, salinity):
    """OBC_SPONGE_EXP's rate EXP(-4 L/Lsp)/TAO per cell and side, (ni, nj)
    arrays in the staggering's array indices; L sums the metric from the
    boundary cell to the cell in ascending index order, one row at a time
    (sequential, like Fortran's SUM over the index range), Lsp is L of the
    band's innermost cell; SAO's south band takes Lsp for every cell
    (mo_obcs.f90:2976)."""
    st = {"z": "p", "t": "p", "u": "u", "v": "v"}[kind]
    dx, dy = np.asarray(g["dlx" + st]), np.asarray(g["dly" + st])
    tao = float(obc["tao"])
    rates = []
    for b in range(4):
        L = np.zeros((ni, nj))
        if b == 0:
            acc = np.zeros(nj)
            for a in range(ni):
                acc = acc + dx[a, :]
                L[a, :] = acc
            lsp = L[min(w[b], ni) - 1, :][None, :]
        elif b == 1:
            for a in range(ni):
                acc = np.zeros(nj)
                for x in range(a, ni):
                    acc = acc + dx[x, :]
                L[a, :] = acc
            lsp = L[ni - w[b], :][None, :]
        elif b == 2:
            acc = np.zeros(ni)
            for c in range(nj):
                acc = acc + dy[:, c]
                L[:, c] = acc
            lsp = L[:, min(w[b], nj) - 1][:, None]
        else:
            for c in range(nj):
                acc = np.zeros(ni)
                for y in range(c, nj):
                    acc = acc + dy[:, y]
                L[:, c] = acc
            lsp = L[:, nj - w[b]][:, None]
            if salinity:
                L = np.broadcast_to(lsp, (ni, nj))
        rates.append(np.exp(-(4.0 * L / lsp)) / tao)
    return rates


def obc_sponge(g, obc, step, x, kind, cli=None, salinity=False):
    """Open-boundary tide forcing + 1/x sponge (mo_obcs.f90:569-642 and
    1561-1720 for kind "z" on ZO; 1881-2032 and 2295-2582 for "u" / "v" on
    UOO / VOE), restated per cell from the cell's distance d to each side's
    boundary cell: band weights s1 = w - d + 1, s2 = d - 1, and in the
    corners the band with the smaller d (the later corner loop on equal d).
    With a nonzero obc["tao"], the exponential sponge of OBC_SPONGE_EXP
    (mo_obcs.f90:2588-3222): the band term is MASK * MASK * DT * M *
    (boundary - X).  Returns the relaxed copy of x."""
    IE, JE = g["ie"], g["je"]
    ilo = 0 if kind == "u" else 1
    jlo = 0 if kind == "v" else 1
    mask = {"z": g["weto"], "t": g["weto"], "u": g["amsuo"], "v": g["amsue"]}[kind]
    v = "zuv".index(kind) if kind != "t" else 0
    x = np.array(x, dtype=np.float64, copy=True)
    x3 = x[:, :, None] if kind == "z" else x
    ni, nj, nk = x3.shape
    I = np.arange(ni)[:, None] + ilo          # Fortran indices
    J = np.arange(nj)[None, :] + jlo
    d = [np.broadcast_to(I + 1 if kind == "u" else I, (ni, nj)),
         np.broadcast_to(IE - I + 1, (ni, nj)),
         np.broadcast_to(J + 1 if kind == "v" else J, (ni, nj)),
         np.broadcast_to(JE - J + 1, (ni, nj))]
    ob = g["ob"]
    on = [bool(ob[s]) and bool(obc["sponge"][b])
          for b, s in enumerate(("west", "east", "north", "south"))]
    w = [int(obc["width"][b]) for b in range(4)]
    inb = [on[b] & (d[b] <= w[b]) for b in range(4)]
    pi = 4.0 * np.arctan(1.0)
    t = float(step) * g["dt"]

    # boundary-cell masks as (ni, nj) arrays for level k (array indices)
    def bmask(b, k):
        m = mask[:, :, k]
        if b == 0:
            return np.broadcast_to(m[0:1, :], (ni, nj))
        if b == 1:
            return np.broadcast_to(m[ni - 1:ni, :], (ni, nj))
        if b == 2:
            return np.broadcast_to(m[:, 0:1], (ni, nj))
        return np.broadcast_to(m[:, nj - 1:nj], (ni, nj))

    # tidal boundary values (level-1 mask of the boundary cell)
    zb = []
    for b in range(4):
        if kind == "t":
            zb.append(None)
            continue
        if not on[b]:
            zb.append(np.zeros((ni, nj)))
            continue
        am, ph = obc["amp"][b][v], obc["pha"][b][v]
        m1 = bmask(b, 0)[:, 0] if b >= 2 else bmask(b, 0)[0, :]
        s = np.zeros(m1.shape)
        for td in range(int(obc["ntide"])):
            s = s + am[:, td] * m1 * np.cos(2.0 * pi * (t - ph[:, td]) / obc["period"][td])
        zb.append(np.broadcast_to(s[None, :] if b < 2 else s[:, None], (ni, nj)))
    s1 = [(w[b] - d[b] + 1).astype(np.float64) for b in range(4)]
    s2 = [(d[b] - 1).astype(np.float64) for b in range(4)]
    lam = []
    for b in range(4):
        l = (s1[b] * obc["relax_bound"] + s2[b] * obc["relax_inner"]) / float(w[b])
        with np.errstate(divide="ignore"):
            lam.append(np.where(l != 0.0, g["dt"] / np.where(l != 0.0, l, 1.0), 0.0))
    expo = float(obc.get("tao", 0.0)) != 0.0
    if expo:
        rate = _exp_rates(g, obc, kind, w, ni, nj, salinity)
    anyb = inb[0] | inb[1] | inb[2] | inb[3]
    for k in range(nk):
        X = x3[:, :, k]
        mi = mask[:, :, k]
        f = []
        for b in range(4):
            mb = bmask(b, k)
            if kind == "t":
                if not on[b]:
                    f.append(np.zeros((ni, nj)))
                    continue
                c = cli[b][:, k]
                obk = np.broadcast_to(c[None, :] if b < 2 else c[:, None], (ni, nj)) * mb
            else:
                obk = zb[b] if kind == "z" else zb[b] * mb
            if expo:
                f.append(np.where(inb[b], mb * mi * g["dt"] * rate[b] * (obk - X), 0.0))
                continue
            xr = (s1[b] * obk + s2[b] * X) / float(w[b])
            f.append(np.where(inb[b], mb * mi * lam[b] * (xr - X), 0.0))
        fo = f[0] + f[1] + f[2] + f[3]
        fo = np.where(inb[0] & inb[2], np.where(d[0] < d[2], f[0], f[2]), fo)
        fo = np.where(inb[0] & inb[3], np.where(d[0] < d[3], f[0], f[3]), fo)
        fo = np.where(inb[1] & inb[2], np.where(d[1] < d[2], f[1], f[2]), fo)
        fo = np.where(inb[1] & inb[3], np.where(d[1] < d[3], f[1], f[3]), fo)
        x3[:, :, k] = np.where(anyb, X + fo, X)
    return x


def octdiff(g, tracers, dvo, zo):
    """OCTDIFF_BASE (tracer-independent factors, octdiff_base.f90:178-226)
    and OCTDIFF_TS (octdiff_ts.f90:294-404) with AH00 <= ALMZER and no sea
    ice: implicit vertical diffusion by the pre-eliminated tridiagonal
    TRIDSY, then the explicit biharmonic term when AULAPTS > ALMZER.
    Returns the diffused copies of the tracers."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    dt, almzer, aulapts = g["dt"], g["almzer"], g["aulapts"]
    weto, ddpo, di, dzw = g["weto"], g["ddpo"], g["di"], g["dzw"]
    dlxp, dlyp, dlxu, dlyu = g["dlxp"], g["dlyp"], g["dlxu"], g["dlyu"]
    dlxv, dlyv = g["dlxv"], g["dlyv"]
    I, J = slice(1, ie - 1), slice(1, je - 1)          # I = 2..IE1, J = 2..JE1
    zzsurf = np.zeros(ke)
    zzsurf[0] = 1.0
    ice = 0.0                                          # RHOICWA*SICTHO + RHOSNWA*SICSNO
    # TRIDSY, octdiff_base.f90:182-201
    t1 = np.zeros((ie - 2, je - 2, ke))
    t2 = np.zeros((ie - 2, je - 2, ke))
    t3 = np.zeros((ie - 2, je - 2, ke))
    for k in range(ke):
        den = ddpo[I, J, k] + zzsurf[k] * (zo[I, J] - ice - ice) + almzer
        t1[:, :, k] = -dt * dvo[I, J, k] * weto[I, J, k] * di[k] / den
        t3[:, :, k] = -dt * dvo[I, J, k + 1] * di[k + 1] / den
        t2[:, :, k] = 1. - t1[:, :, k] - t3[:, :, k]
    for k in range(1, ke):
        a = t1[:, :, k].copy()
        t1[:, :, k - 1] = a / t2[:, :, k - 1]
        t2[:, :, k] = t2[:, :, k] - t3[:, :, k - 1] * a / t2[:, :, k - 1]
    out = []
    for tr in tracers:
        x = np.array(tr, dtype=np.float64, copy=True)
        # implicit vertical diffusion, octdiff_ts.f90:296-323
        r = x[I, J, :].copy()
        for k in range(1, ke):
            r[:, :, k] = r[:, :, k] - t1[:, :, k - 1] * r[:, :, k - 1]
        y = np.zeros_like(r)
        y[:, :, ke - 1] = r[:, :, ke - 1] / t2[:, :, ke - 1]
        for l in range(ke - 2, -1, -1):
            y[:, :, l] = (r[:, :, l] - t3[:, :, l] * y[:, :, l + 1]) / t2[:, :, l]
        x[I, J, :] = y
        x[I, J, :] = x[I, J, :] + 0.0                 # THTEN = 0 (AH00 <= ALMZER)
        if aulapts > almzer:
            # AULX(I,J) = AULAPTS*DLXU(I,J)**4, AULY(I,J) = AULAPTS*DLYV(I,J)**4
            # (octdiff_base.f90:208-219), the power as (x*x)*(x*x).  u arrays are
            # indexed by Fortran I (I_start = 0), v arrays by Fortran J.
            aulx = aulapts * ((dlxu * dlxu) * (dlxu * dlxu))
            auly = aulapts * ((dlyv * dlyv) * (dlyv * dlyv))
            Im, Ip, Jm, Jp = slice(0, ie - 2), slice(2, ie), slice(0, je - 2), slice(2, je)
            uW, uE = slice(1, ie - 1), slice(2, ie)      # u-point I-1 and I of p-cell I
            vS, vN = slice(1, je - 1), slice(2, je)      # v-point J-1 and J of p-cell J
            # Laplacian, octdiff_ts.f90:344-358 (T1O stays 0 outside 2..IE1 x 2..JE1)
            lap = np.zeros_like(x)
            for k in range(ke):
                c = x[I, J, k]
                ex = (weto[Im, J, k] * (x[Im, J, k] - c) / dlxu[uW, J]
                      + weto[Ip, J, k] * (x[Ip, J, k] - c) / dlxu[uE, J]) / dlxp[I, J]
                ey = (weto[I, Jm, k] * (x[I, Jm, k] - c) / dlyv[I, vS]
                      + weto[I, Jp, k] * (x[I, Jp, k] - c) / dlyv[I, vN]) / dlyp[I, J]
                lap[I, J, k] = weto[I, J, k] * (ex + ey)
            # biharmonic update, octdiff_ts.f90:366-392
            for k in range(ke):
                L = lap[:, :, k]
                c = L[I, J]
                den = (ddpo[I, J, k] + almzer + zzsurf[k] * (zo[I, J] - ice - ice)) \
                    * dlxp[I, J] * dlyp[I, J]
                s = (weto[Im, J, k] * aulx[uW, J] * dlyu[uW, J] * (L[Im, J] - c) / dlxu[uW, J]
                     + weto[Ip, J, k] * aulx[uE, J] * dlyu[uE, J] * (L[Ip, J] - c) / dlxu[uE, J]
                     + weto[I, Jm, k] * auly[I, vS] * dlxv[I, vS] * (L[I, Jm] - c) / dlyv[I, vS]
                     + weto[I, Jp, k] * auly[I, vN] * dlxv[I, vN] * (L[I, Jp] - c) / dlyv[I, vN])
                x[I, J, k] = x[I, J, k] - (weto[I, J, k] / den) * dzw[k] * s
        out.append(x)
    return out


def _mx0(x):
    """MAX(0., x) as the Fortran intrinsic evaluates it for non-NaN x."""
    return np.where(0.0 > x, 0.0, x)


def _mn1(x):
    """MIN(1., x) for non-NaN x."""
    return np.where(x < 1.0, x, 1.0)


def _limited(t, ta, tb, up, um, vol):
    """The limited upwind pair of ocuad.f90:41-52 (TRP uses ta, TRM tb)."""
    abl = np.abs(ta - tb)
    zwabl = np.abs(ta + tb - 2. * t)
    with np.errstate(divide="ignore", invalid="ignore"):
        scha = _mx0((abl - zwabl) / (abl + 1.E-20))
        sch = _mn1(scha * vol / (up + um + 1.E-20))
    schi = 1. - sch
    return up * (schi * t + sch * 0.5 * (t + ta)), um * (schi * t + sch * 0.5 * (t + tb))


def ocuad(g, uoo, uko, vke, wo):
    """OCUAD (ocuad.f90:1-271) on u-points: the vertical, x and y sweeps of
    the limited scheme with the boundary faces at I = 0, IE and J = 1, JE.
    Arrays: u (IE+1, JE, KE) indexed by Fortran I and J-1; p and w by I-1,
    J-1; v by I-1, J.  Returns the advected copy of uoo."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    dt = g["dt"]
    amsuo, dduo, ddue = g["amsuo"], g["dduo"], g["ddue"]
    dlxu, dlyu, dlxp, dlyp, dlxv = g["dlxu"], g["dlyu"], g["dlxp"], g["dlyp"], g["dlxv"]
    trf = np.array(uoo, dtype=np.float64, copy=True)
    trvol = amsuo * dlxu[:, :, None] * dlyu[:, :, None] * dduo
    I, J = slice(1, ie), slice(1, je - 1)        # Fortran I = 1..IE1, J = 2..JE1
    wet = amsuo[I, J, :] > 0.5

    def update(rn, num):
        with np.errstate(divide="ignore", invalid="ignore"):
            tr1 = num / rn
        trf[I, J, :] = np.where(wet, tr1, trf[I, J, :])
        trvol[I, J, :] = np.where(wet, rn, trvol[I, J, :])

    # vertical sweep (ocuad.f90:33-83); TRP(K) at index K-1, TRM(K) at index K
    trp = np.zeros((ie - 1, je - 2, ke + 1))
    trm = np.zeros((ie - 1, je - 2, ke + 1))
    wtp = np.zeros((ie - 1, je - 2, ke + 1))
    wtm = np.zeros((ie - 1, je - 2, ke + 1))
    c = 0.5 * dt * dlyp[0:ie - 1, J] * dlxp[0:ie - 1, J]     # DLYP(I,J), DLXP(I,J)
    for k in range(ke):
        kup, klo = max(k - 1, 0), min(k + 1, ke - 1)
        t = trf[I, J, k]
        wup = 0.5 * (wo[0:ie - 1, J, k] + wo[1:ie, J, k])
        wlo = 0.5 * (wo[0:ie - 1, J, k + 1] + wo[1:ie, J, k + 1])
        up = c * (wup + np.abs(wup))
        um = c * (np.abs(wlo) - wlo)
        p, m = _limited(t, trf[I, J, kup], trf[I, J, klo], up, um, trvol[I, J, k])
        trp[:, :, k], trm[:, :, k + 1], wtp[:, :, k], wtm[:, :, k + 1] = p, m, up, um
    V = trvol[I, J, :]
    rn = V + wtp[:, :, 1:] - wtp[:, :, :ke] - wtm[:, :, 1:] + wtm[:, :, :ke]
    update(rn, trf[I, J, :] * V + trp[:, :, 1:] - trp[:, :, :ke] - trm[:, :, 1:] + trm[:, :, :ke])

    # x sweep (ocuad.f90:92-175): faces at u-points I = 0..IE
    trp = np.zeros((ie + 1, je - 2, ke))
    trm = np.zeros((ie + 1, je - 2, ke))
    wtp = np.zeros((ie + 1, je - 2, ke))
    wtm = np.zeros((ie + 1, je - 2, ke))
    ud = uko[:, J, :] * dduo[:, J, :]
    uos = 0.5 * (ud[1:ie] + ud[2:ie + 1])
    uwe = 0.5 * (ud[0:ie - 1] + ud[1:ie])
    up = 0.5 * dt * dlyp[1:ie, J][:, :, None] * (uos + np.abs(uos))
    um = 0.5 * dt * (np.abs(uwe) - uwe) * dlyp[0:ie - 1, J][:, :, None]
    p, m = _limited(trf[I, J, :], trf[2:ie + 1, J, :], trf[0:ie - 1, J, :], up, um,
                    trvol[I, J, :])
    trp[1:ie], trm[1:ie], wtp[1:ie], wtm[1:ie] = p, m, up, um
    for i, uos_, uwe_, dyp, dyu in (
            (0, 0.5 * (ud[0] + ud[1]), ud[0], dlyp[0, J], dlyu[0, J]),
            (ie, ud[ie], 0.5 * (ud[ie - 1] + ud[ie]), dlyp[ie - 1, J], dlyu[ie, J])):
        upb = 0.5 * dt * dyp[:, None] * (uos_ + np.abs(uos_))
        umb = 0.5 * dt * (np.abs(uwe_) - uwe_) * dyu[:, None]
        trp[i], trm[i], wtp[i], wtm[i] = upb * trf[i, J, :], umb * trf[i, J, :], upb, umb
    V = trvol[I, J, :]
    rn = V + wtp[0:ie - 1] - wtp[1:ie] - wtm[1:ie] + wtm[2:ie + 1]
    update(rn, trf[I, J, :] * V + trp[0:ie - 1] - trp[1:ie] - trm[1:ie] + trm[2:ie + 1])

    # y sweep (ocuad.f90:187-255): faces at J = 1..JE (index J-1)
    trp = np.zeros((ie - 1, je, ke))
    trm = np.zeros((ie - 1, je, ke))
    wtp = np.zeros((ie - 1, je, ke))
    wtm = np.zeros((ie - 1, je, ke))
    vd = vke[:, :, :] * ddue                       # v index (I-1, J)
    dx = 0.5 * (dlxv[0:ie - 1, :] + dlxv[1:ie, :])  # 0.5*(DLXV(I,J)+DLXV(I+1,J)), J = 0..JE
    vs = 0.5 * (vd[0:ie - 1] + vd[1:ie])           # 0.5*(VKE(I,J)DDUE(I,J)+VKE(I+1,J)DDUE(I+1,J))
    for jj in range(1, je + 1):                    # Fortran J = 1..JE
        vsu, vno = vs[:, jj], vs[:, jj - 1]
        upj = 0.5 * dt * dx[:, jj - 1][:, None] * (vno + np.abs(vno))
        umj = 0.5 * dt * dx[:, jj][:, None] * (np.abs(vsu) - vsu)
        t = trf[I, jj - 1, :]
        if 2 <= jj <= je - 1:
            p, m = _limited(t, trf[I, jj - 2, :], trf[I, jj, :], upj, umj, trvol[I, jj - 1, :])
        else:
            p, m = upj * t, umj * t
        trp[:, jj - 1], trm[:, jj - 1], wtp[:, jj - 1], wtm[:, jj - 1] = p, m, upj, umj
    V = trvol[I, J, :]
    rn = V + wtp[:, 2:je] - wtp[:, 1:je - 1] - wtm[:, 1:je - 1] + wtm[:, 0:je - 2]
    update(rn, trf[I, J, :] * V + trp[:, 2:je] - trp[:, 1:je - 1] - trm[:, 1:je - 1]
           + trm[:, 0:je - 2])
    return trf


def ocvad(g, voe, uko, vke, wo):
    """OCVAD (ocvad.f90:1-271) on v-points, the transposed OCUAD with its own
    edge faces at I = 1, IE and J = 0, JE.  The J = 0 face reads DLXU(I,0),
    outside DLXU (ocvad.f90:211); as in the oracle, DLXV(I,0) stands in.
    Arrays: v (IE, JE+1, KE) indexed by I-1 and Fortran J; u by I and J-1;
    p and w by I-1, J-1.  Returns the advected copy of voe."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    dt = g["dt"]
    amsue, dduo, ddue = g["amsue"], g["dduo"], g["ddue"]
    dlxv, dlyv, dlxp, dlyp, dlyu, dlxu = (g["dlxv"], g["dlyv"], g["dlxp"], g["dlyp"],
                                          g["dlyu"], g["dlxu"])
    trf = np.array(voe, dtype=np.float64, copy=True)
    trvol = amsue * dlxv[:, :, None] * dlyv[:, :, None] * ddue
    I, J = slice(1, ie - 1), slice(1, je)        # Fortran I = 2..IE1, J = 1..JE1
    pI, pJ = slice(1, ie - 1), slice(0, je - 1)  # p-point I-1, J-1 of those cells
    wet = amsue[I, J, :] > 0.5

    def update(rn, num):
        with np.errstate(divide="ignore", invalid="ignore"):
            tr1 = num / rn
        trf[I, J, :] = np.where(wet, tr1, trf[I, J, :])
        trvol[I, J, :] = np.where(wet, rn, trvol[I, J, :])

    # vertical sweep: TRP(K) at index K-1, TRM(K) at index K
    trp = np.zeros((ie - 2, je - 1, ke + 1))
    trm = np.zeros((ie - 2, je - 1, ke + 1))
    wtp = np.zeros((ie - 2, je - 1, ke + 1))
    wtm = np.zeros((ie - 2, je - 1, ke + 1))
    c = 0.5 * dt * dlyp[pI, pJ] * dlxp[pI, pJ]
    for k in range(ke):
        kup, klo = max(k - 1, 0), min(k + 1, ke - 1)
        wup = 0.5 * (wo[pI, 0:je - 1, k] + wo[pI, 1:je, k])
        wlo = 0.5 * (wo[pI, 0:je - 1, k + 1] + wo[pI, 1:je, k + 1])
        up = c * (wup + np.abs(wup))
        um = c * (np.abs(wlo) - wlo)
        p, m = _limited(trf[I, J, k], trf[I, J, kup], trf[I, J, klo], up, um, trvol[I, J, k])
        trp[:, :, k], trm[:, :, k + 1], wtp[:, :, k], wtm[:, :, k + 1] = p, m, up, um
    V = trvol[I, J, :]
    rn = V + wtp[:, :, 1:] - wtp[:, :, :ke] - wtm[:, :, 1:] + wtm[:, :, :ke]
    update(rn, trf[I, J, :] * V + trp[:, :, 1:] - trp[:, :, :ke] - trm[:, :, 1:] + trm[:, :, :ke])

    # x sweep: faces at v-point I = 1..IE (index I-1)
    trp = np.zeros((ie, je - 1, ke))
    trm = np.zeros((ie, je - 1, ke))
    wtp = np.zeros((ie, je - 1, ke))
    wtm = np.zeros((ie, je - 1, ke))
    ud = uko * dduo                                   # u index (I, J-1)
    uu = 0.5 * (ud[:, 0:je - 1] + ud[:, 1:je])        # at v-row J: UKO(I,J), UKO(I,J+1)
    dyu = 0.5 * (dlyu[:, 0:je - 1] + dlyu[:, 1:je])   # 0.5*(DLYU(I,J)+DLYU(I,J+1))
    for ii in range(1, ie + 1):                        # Fortran I = 1..IE
        uos, uwe = uu[ii], uu[ii - 1]
        upi = 0.5 * dt * dyu[ii][:, None] * (uos + np.abs(uos))
        umi = 0.5 * dt * (np.abs(uwe) - uwe) * dyu[ii - 1][:, None]
        t = trf[ii - 1, J, :]
        if 2 <= ii <= ie - 1:
            p, m = _limited(t, trf[ii, J, :], trf[ii - 2, J, :], upi, umi, trvol[ii - 1, J, :])
        else:
            p, m = upi * t, umi * t
        trp[ii - 1], trm[ii - 1], wtp[ii - 1], wtm[ii - 1] = p, m, upi, umi
    V = trvol[I, J, :]
    rn = V + wtp[0:ie - 2] - wtp[1:ie - 1] - wtm[1:ie - 1] + wtm[2:ie]
    update(rn, trf[I, J, :] * V + trp[0:ie - 2] - trp[1:ie - 1] - trm[1:ie - 1] + trm[2:ie])

    # y sweep: faces at v-point J = 0..JE
    trp = np.zeros((ie - 2, je + 1, ke))
    trm = np.zeros((ie - 2, je + 1, ke))
    wtp = np.zeros((ie - 2, je + 1, ke))
    wtm = np.zeros((ie - 2, je + 1, ke))
    vd = vke[I] * ddue[I]                              # (IE-2, JE+1, KE), index Fortran J
    for jj in range(0, je + 1):
        t = trf[I, jj, :]
        if jj == 0:
            vno = vd[:, 0]
            vsu = 0.5 * (vd[:, 0] + vd[:, 1])
            upj = 0.5 * dt * dlxv[I, 0][:, None] * (vno + np.abs(vno))     # DLXU(I,0) in ref
            umj = 0.5 * dt * dlxp[pI, 0][:, None] * (np.abs(vsu) - vsu)
        elif jj == je:
            vno = 0.5 * (vd[:, je] + vd[:, je - 1])
            vsu = vd[:, je]
            upj = 0.5 * dt * dlxp[pI, je - 1][:, None] * (vno + np.abs(vno))
            umj = 0.5 * dt * dlxu[2:ie, je - 1][:, None] * (np.abs(vsu) - vsu)
        else:
            vno = 0.5 * (vd[:, jj] + vd[:, jj - 1])
            vsu = 0.5 * (vd[:, jj] + vd[:, jj + 1])
            upj = 0.5 * dt * dlxp[pI, jj - 1][:, None] * (vno + np.abs(vno))
            umj = 0.5 * dt * dlxp[pI, jj][:, None] * (np.abs(vsu) - vsu)
        if 1 <= jj <= je - 1:
            p, m = _limited(t, trf[I, jj - 1, :], trf[I, jj + 1, :], upj, umj, trvol[I, jj, :])
        else:
            p, m = upj * t, umj * t
        trp[:, jj], trm[:, jj], wtp[:, jj], wtm[:, jj] = p, m, upj, umj
    V = trvol[I, J, :]
    rn = V + wtp[:, 2:je + 1] - wtp[:, 1:je] - wtm[:, 1:je] + wtm[:, 0:je - 1]
    update(rn, trf[I, J, :] * V + trp[:, 2:je + 1] - trp[:, 1:je] - trm[:, 1:je]
           + trm[:, 0:je - 1])
    return trf


def ocwad(g, wno, uko, vke, wo, zo):
    """OCWAD (ocwad.f90:1-238) on w-points, levels 2..KE updated.  The
    limiter's MIN(WETO(I,J,KLO), ...) reads WETO(KEP), one level past WETO
    (ocwad.f90:63); as in the oracle it is taken as 0.  The x and y sweeps
    reuse the flux arrays of the vertical step, whose edge faces (I = 1, IE;
    J = 1, JE) are 0 on levels 2..KE.  Arrays: w (IE, JE, KE+1) and p by
    I-1, J-1; u by I, J-1; v by I-1, J.  Returns the advected copy of wno."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    dt = g["dt"]
    weto, ddpo, dduo, ddue = g["weto"], g["ddpo"], g["dduo"], g["ddue"]
    dlxp, dlyp, dlyu, dlxv = g["dlxp"], g["dlyp"], g["dlyu"], g["dlxv"]
    trf = np.array(wno, dtype=np.float64, copy=True)
    I, J = slice(1, ie - 1), slice(1, je - 1)        # Fortran 2..IE1, 2..JE1
    wet_k = np.concatenate([weto, np.zeros((ie, je, 1))], axis=2)  # WETO(KEP) := 0
    # S1O, ocwad.f90:24-36
    a = weto * dlxp[:, :, None] * dlyp[:, :, None]
    s1o = np.empty((ie, je, ke))
    s1o[:, :, 0] = a[:, :, 0] * (ddpo[:, :, 0] + zo) / 2.0
    if ke > 1:
        s1o[:, :, 1] = a[:, :, 1] * (ddpo[:, :, 0] + ddpo[:, :, 1] + zo) / 2.0
    for k in range(2, ke):
        s1o[:, :, k] = a[:, :, k] * (ddpo[:, :, k - 1] + ddpo[:, :, k]) / 2.0

    def update(k, rn, num):
        wet = weto[I, J, k] > 0.5
        with np.errstate(divide="ignore", invalid="ignore"):
            t1 = num / rn
        trf[I, J, k] = np.where(wet, t1, trf[I, J, k])
        s1o[I, J, k] = np.where(wet, rn, s1o[I, J, k])

    # vertical (ocwad.f90:44-103): TRP(K), WTP(K) at index K-1 (K = 1..KEP);
    # TRM(K), WTM(K) at index K (K = 0..KE); all zero but what is set below
    trp = np.zeros((ie, je, ke + 1))
    trm = np.zeros((ie, je, ke + 1))
    wtp = np.zeros((ie, je, ke + 1))
    wtm = np.zeros((ie, je, ke + 1))
    c = 0.5 * dt * dlyp * dlxp
    for k in range(1, ke):                          # Fortran K = 2..KE
        kup, klo = k - 1, k + 1
        t, tu, tl = trf[I, J, k], trf[I, J, kup], trf[I, J, klo]
        abl = np.abs(tu - tl)
        zwabl = np.abs(tu + tl - 2. * t)
        wup = 0.5 * (wo[I, J, k] + wo[I, J, kup])
        wum = 0.5 * (wo[I, J, k] + wo[I, J, klo])
        up = c[I, J] * (wup + np.abs(wup))
        um = c[I, J] * (np.abs(wum) - wum)
        with np.errstate(divide="ignore", invalid="ignore"):
            scha = _mx0((abl - zwabl) / (abl + 1.E-20))
            x = scha * s1o[I, J, k] / (up + um + 1.E-20)
        cap = wet_k[I, J, klo]
        sch = np.where(x < cap, x, cap)
        schi = 1. - sch
        trp[I, J, k] = up * (schi * t + sch * 0.5 * (t + tu))
        trm[I, J, k + 1] = um * (schi * t + sch * 0.5 * (t + tl))
        wtp[I, J, k], wtm[I, J, k + 1] = up, um
    wup = 0.5 * (wo[:, :, ke] + wo[:, :, ke - 1])
    up = c * (wup + np.abs(wup))
    trp[:, :, ke] = up * (0.5 * (trf[:, :, ke - 1] + trf[:, :, ke]))
    wtp[:, :, ke] = up
    wum = 0.5 * (wo[:, :, 0] + wo[:, :, 1])
    um = c * (np.abs(wum) - wum)
    trm[:, :, 1] = um * (0.5 * (trf[:, :, 0] + trf[:, :, 1]))
    wtm[:, :, 1] = um
    for k in range(1, ke):
        rn = s1o[I, J, k] + wtp[I, J, k + 1] - wtp[I, J, k] - wtm[I, J, k + 1] + wtm[I, J, k]
        update(k, rn, trf[I, J, k] * s1o[I, J, k] + trp[I, J, k + 1] - trp[I, J, k]
               - trm[I, J, k + 1] + trm[I, J, k])

    # x sweep (ocwad.f90:110-164): interior faces overwrite the arrays
    trp, trm, wtp, wtm = trp[:, :, :ke], trm[:, :, 1:], wtp[:, :, :ke], wtm[:, :, 1:]
    trp, trm, wtp, wtm = (np.array(a_, copy=True) for a_ in (trp, trm, wtp, wtm))
    for arr in (trp, trm, wtp, wtm):               # levels 2..KE: edges are 0
        arr[0, :, 1:] = 0.0
        arr[ie - 1, :, 1:] = 0.0
    ud = uko * dduo
    for k in range(1, ke):
        t, te, tw = trf[I, J, k], trf[2:ie, J, k], trf[0:ie - 2, J, k]
        abl = np.abs(te - tw)
        zwabl = np.abs(te + tw - 2. * t)
        uos = 0.5 * (ud[2:ie, J, k] + ud[2:ie, J, k - 1])
        uwe = 0.5 * (ud[1:ie - 1, J, k] + ud[1:ie - 1, J, k - 1])
        up = 0.5 * dt * dlyu[2:ie, J] * (uos + np.abs(uos))
        um = 0.5 * dt * dlyu[1:ie - 1, J] * (np.abs(uwe) - uwe)
        with np.errstate(divide="ignore", invalid="ignore"):
            scha = _mx0((abl - zwabl) / (abl + 1.E-20)) * weto[I, J, k] \
                * weto[2:ie, J, k] * weto[0:ie - 2, J, k]
            sch = _mn1(scha * s1o[I, J, k] / (up + um + 1.E-20))
        schi = 1. - sch
        trp[I, J, k] = up * (schi * t + sch * 0.5 * (t + te))
        trm[I, J, k] = um * (schi * t + sch * 0.5 * (t + tw))
        wtp[I, J, k], wtm[I, J, k] = up, um
    for k in range(1, ke):
        rn = s1o[I, J, k] + wtp[0:ie - 2, J, k] - wtp[I, J, k] - wtm[I, J, k] + wtm[2:ie, J, k]
        update(k, rn, trf[I, J, k] * s1o[I, J, k] + trp[0:ie - 2, J, k] - trp[I, J, k]
               - trm[I, J, k] + trm[2:ie, J, k])

    # y sweep (ocwad.f90:171-227)
    for arr in (trp, trm, wtp, wtm):
        arr[:, 0, 1:] = 0.0
        arr[:, je - 1, 1:] = 0.0
    vd = vke * ddue
    for k in range(1, ke):
        t, tn, ts = trf[I, J, k], trf[I, 0:je - 2, k], trf[I, 2:je, k]
        abl = np.abs(tn - ts)
        zwabl = np.abs(tn + ts - 2. * t)
        vsu = 0.5 * (vd[I, 2:je, k] + vd[I, 2:je, k - 1])
        vno = 0.5 * (vd[I, 1:je - 1, k] + vd[I, 1:je - 1, k - 1])
        up = 0.5 * dt * dlxv[I, 1:je - 1] * (vno + np.abs(vno))
        um = 0.5 * dt * dlxv[I, 2:je] * (np.abs(vsu) - vsu)
        with np.errstate(divide="ignore", invalid="ignore"):
            scha = _mx0((abl - zwabl) / (abl + 1.E-20)) * weto[I, J, k] \
                * weto[I, 0:je - 2, k] * weto[I, 2:je, k]
            sch = _mn1(scha * s1o[I, J, k] / (up + um + 1.E-20))
        schi = 1. - sch
        trp[I, J, k] = up * (schi * t + sch * 0.5 * (t + tn))
        trm[I, J, k] = um * (schi * t + sch * 0.5 * (t + ts))
        wtp[I, J, k], wtm[I, J, k] = up, um
    for k in range(1, ke):
        rn = s1o[I, J, k] + wtp[I, 2:je, k] - wtp[I, J, k] - wtm[I, J, k] + wtm[I, 0:je - 2, k]
        update(k, rn, trf[I, J, k] * s1o[I, J, k] + trp[I, 2:je, k] - trp[I, J, k]
               - trm[I, J, k] + trm[I, 0:je - 2, k])
    return trf


def nh_rhs(g, uoo, uoo1, voe, voe1, wno, wno1, zo):
    """OCVTOT_NH up to the solve (ocvtot_nh.f90:11-62) and ComputeRHS with
    CG2D4NONHY off (mo_petsc.f90:298-376): DIVG*WETO over I = 2..IE1,
    J = 2..JE1, K = 1..KE in DMDA natural order (x fastest)."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    dt = g["dt"]
    gu = (uoo - uoo1) / dt
    gv = (voe - voe1) / dt
    gw = (wno - wno1) / dt
    divgu = (gu[1:ie + 1] - gu[0:ie]) / g["dlxp"][:, :, None]
    divgv = (gv[:, 0:je] - gv[:, 1:je + 1]) / g["dlyp"][:, :, None]
    dd = np.maximum(g["ddpo"], 1.E-3)
    divgw = np.empty((ie, je, ke))
    divgw[:, :, 1:] = (gw[:, :, 1:ke] - gw[:, :, 2:ke + 1]) / dd[:, :, 1:]
    divgw[:, :, 0] = (gw[:, :, 0] - gw[:, :, 1]) / (dd[:, :, 0] + zo)
    divg = divgu + divgv + divgw
    rhs = divg[1:ie - 1, 1:je - 1, :] * g["weto"][1:ie - 1, 1:je - 1, :]
    return rhs.reshape(-1, order="F")


def nh_post(g, x, pnh, uoo, voe):
    """OCVTOT_NH after the solve (ocvtot_nh.f90:150-255; mo_petsc.f90:223-227
    writes the solution into PNH's interior): open-boundary fill of PNH, u/v
    corrected by the PNH gradient, WNO re-integrated from the bottom, and the
    rotation UOO_1 = UOO, VOE_1 = VOE, WNO_1 = WO = WNO.  Returns (pnh, uoo,
    voe, wno) as new arrays."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    ob = g["ob"]
    pnh = np.array(pnh, copy=True)
    uoo = np.array(uoo, copy=True)
    voe = np.array(voe, copy=True)
    pnh[1:ie - 1, 1:je - 1, :] = np.asarray(x).reshape((ie - 2, je - 2, ke), order="F")
    if ob["west"]:
        pnh[0, 1:je - 1, :] = pnh[1, 1:je - 1, :]
    if ob["east"]:
        pnh[ie - 1, 1:je - 1, :] = pnh[ie - 2, 1:je - 1, :]
    if ob["north"]:
        pnh[:, 0, :] = pnh[:, 1, :]
    if ob["south"]:
        pnh[:, je - 1, :] = pnh[:, je - 2, :]
    J = slice(1, je - 1)
    uoo[1:ie, J, :] = uoo[1:ie, J, :] + g["amsuo"][1:ie, J, :] * g["dtdxuo"][1:ie, J][:, :, None] \
        * (pnh[0:ie - 1, J, :] - pnh[1:ie, J, :])
    I = slice(1, ie - 1)
    voe[I, 1:je, :] = voe[I, 1:je, :] + g["amsue"][I, 1:je, :] * g["dpye"][I, 1:je][:, :, None] \
        * (pnh[I, 1:je, :] - pnh[I, 0:je - 1, :])
    dti = 1. / g["dt"]
    ud = uoo * g["dduo"] * g["dlyu"][:, :, None]
    vd = voe * g["ddue"] * g["dlxv"][:, :, None]
    wno = np.zeros((ie, je, ke + 1))
    weto = g["weto"]
    for k in range(ke - 1, -1, -1):
        t1 = dti * weto[:, :, k] * (g["dtdxpo"] * (ud[0:ie, :, k] - ud[1:ie + 1, :, k]) / g["dlyp"])
        t2 = dti * weto[:, :, k] * (+ g["dtdyo"] * (vd[:, 1:je + 1, k] - vd[:, 0:je, k]) / g["dlxp"])
        wno[:, :, k] = wno[:, :, k + 1] + t1 + t2
    return pnh, uoo, voe, wno


def _fmx(a, b):
    """Fortran MAX(a, b) for non-NaN operands (a when not b > a)."""
    return np.where(a > b, a, b)


def _col_solve(t1, t2, t3, rhs, mask, k0):
    """Pre-eliminated tridiagonal column solve of ocvisc.f90:142-160 over
    levels k0..KE-1 (0-based): t1, t2, t3 (..., KE) are TRIDSY(:,1..3) after
    the elimination; returns the solution times the masks as the reference
    forms it."""
    ke = rhs.shape[-1]
    r = rhs.copy()
    for k in range(k0 + 1, ke):
        r[..., k] = r[..., k] - t1[..., k - 1] * r[..., k - 1]
    x = np.zeros_like(r)
    x[..., ke - 1] = mask[..., ke - 1] * r[..., ke - 1] / t2[..., ke - 1]
    for l in range(ke - 2, k0 - 1, -1):
        x[..., l] = (r[..., l] - t3[..., l] * x[..., l + 1]) * mask[..., l] / t2[..., l]
    return x


def _eliminate(t1, t2, t3, k0):
    ke = t1.shape[-1]
    for k in range(k0 + 1, ke):
        a = t1[..., k].copy()
        t1[..., k - 1] = a / t2[..., k - 1]
        t2[..., k] = t2[..., k] - t3[..., k - 1] * a / t2[..., k - 1]


def ocvisc(g, uoo, voe, wno, uko, vke, avo):
    """OCVISC with FREESLIP and NON_HYDROSTATIC (ocvisc.f90:37-767): bottom
    speeds, implicit vertical diffusion of u, v (with quadratic bottom
    friction) and w, biharmonic horizontal diffusion, then OCTIMF.  Returns
    (uoo, voe, wno, uko, vke) as new arrays.  u arrays are indexed by
    Fortran I and J-1, v by I-1 and J, p and w by I-1 and J-1."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    dt, almzer, aulapuv = g["dt"], g["almzer"], g["aulapuv"]
    amsuo, amsue, weto = g["amsuo"], g["amsue"], g["weto"]
    dduo, ddue, ddpo, di = g["dduo"], g["ddue"], g["ddpo"], g["di"]
    dlxp, dlyp, dlxu, dlyu, dlxv, dlyv = (g["dlxp"], g["dlyp"], g["dlxu"], g["dlyu"],
                                          g["dlxv"], g["dlyv"])
    uoo = np.array(uoo, copy=True)
    voe = np.array(voe, copy=True)
    wno = np.array(wno, copy=True)
    uko = np.array(uko, copy=True)
    vke = np.array(vke, copy=True)
    mv10 = g["dzw"][0] / 10.0
    minvalue = mv10 if mv10 < 1.0 else 1.0              # MIN(1.0, DZW(1)/10.0)
    bofric = rayfric = 3.E-3

    # bottom speeds (ocvisc.f90:49-102): SPEEDU on u-points I = 1..IE1,
    # J = 2..JE1; SPEEDV on v-points I = 2..IE1, J = 1..JE1
    speedu = np.zeros((ie + 1, je))
    speedv = np.zeros((ie, je + 1))
    uI, uJ = slice(1, ie), slice(1, je - 1)
    for k in range(ke):
        bot = amsuo[uI, uJ, k] > 0.5 if k == ke - 1 else \
            (amsuo[uI, uJ, k] - amsuo[uI, uJ, k + 1]) > 0.5
        q = 0.25 * (voe[0:ie - 1, 2:je, k] + voe[1:ie, 2:je, k] + voe[0:ie - 1, 1:je - 1, k]
                    + voe[1:ie, 1:je - 1, k])
        u = uoo[uI, uJ, k]
        s = _fmx(np.sqrt(u * u + q * q), 1.E-3)
        speedu[uI, uJ] = np.where(bot, s, speedu[uI, uJ])
    vI, vJ = slice(1, ie - 1), slice(1, je)
    for k in range(ke):
        bot = amsue[vI, vJ, k] > 0.5 if k == ke - 1 else \
            (amsue[vI, vJ, k] - amsue[vI, vJ, k + 1]) > 0.5
        q = 0.25 * (uoo[2:ie, 0:je - 1, k] + uoo[1:ie - 1, 0:je - 1, k] + uoo[2:ie, 1:je, k]
                    + uoo[1:ie - 1, 1:je, k])
        v = voe[vI, vJ, k]
        s = _fmx(np.sqrt(v * v + q * q), 1.E-3)
        speedv[vI, vJ] = np.where(bot, s, speedv[vI, vJ])

    def uv_tridsy(avo_a, avo_b, m, dd, sp):
        """TRIDSY of ocvisc.f90:113-140 / 165-190 for one staggering."""
        n = m.shape[:-1]
        t1, t2, t3 = np.zeros(n + (ke,)), np.zeros(n + (ke,)), np.zeros(n + (ke,))
        for k in range(ke):
            avup = 0.5 * (avo_a[..., k] + avo_b[..., k]) * m[..., k]
            if k < ke - 1:
                avlo = 0.5 * (avo_a[..., k + 1] + avo_b[..., k + 1]) * m[..., k + 1] \
                    + (bofric + rayfric * dd[..., k] * sp) * (m[..., k] - m[..., k + 1])
            else:
                avlo = (bofric + rayfric * dd[..., k] * sp) * m[..., k]
            den = almzer + dd[..., k]
            t1[..., k] = -dt * avup * m[..., k] * di[k] / den
            t3[..., k] = -dt * avlo * m[..., k] * di[k + 1] / den
            t2[..., k] = 1. - t1[..., k] - t3[..., k]
            t3[..., k] = t3[..., k] * m[..., k + 1] if k < ke - 1 else 0.0
        _eliminate(t1, t2, t3, 0)
        return t1, t2, t3

    # V (ocvisc.f90:108-164): v-points I = 2..IE1, J = 1..JE1
    t1, t2, t3 = uv_tridsy(avo[1:ie - 1, 0:je - 1, :], avo[1:ie - 1, 1:je, :], amsue[vI, vJ, :],
                           ddue[vI, vJ, :], speedv[vI, vJ])
    vke[vI, vJ, :] = _col_solve(t1, t2, t3, voe[vI, vJ, :], amsue[vI, vJ, :], 0)
    # U (ocvisc.f90:166-215): u-points I = 1..IE1, J = 2..JE1
    t1, t2, t3 = uv_tridsy(avo[0:ie - 1, uJ, :], avo[1:ie, uJ, :], amsuo[uI, uJ, :],
                           dduo[uI, uJ, :], speedu[uI, uJ])
    uko[uI, uJ, :] = _col_solve(t1, t2, t3, uoo[uI, uJ, :], amsuo[uI, uJ, :], 0)
    # W (ocvisc.f90:223-271): p-points I = 2..IE1, J = 2..JE1, levels 2..KE
    pI, pJ = slice(1, ie - 1), slice(1, je - 1)
    a, w, dp = avo[pI, pJ, :], weto[pI, pJ, :], ddpo[pI, pJ, :]
    n = w.shape[:-1]
    t1, t2, t3 = np.zeros(n + (ke,)), np.zeros(n + (ke,)), np.zeros(n + (ke,))
    for k in range(1, ke):
        avup = 0.5 * (a[..., k - 1] + a[..., k]) * w[..., k - 1]
        avlo = 0.5 * (a[..., k + 1] + a[..., k]) * w[..., k] if k < ke - 1 else 0.0
        den = 2.0 * almzer + dp[..., k - 1] + dp[..., k]
        t1[..., k] = -2.0 * dt * avup * w[..., k] * di[k - 1] / den
        t3[..., k] = -2.0 * dt * avlo * w[..., k] * di[k] / den
        t2[..., k] = 1. - t1[..., k] - t3[..., k]
        if k == ke - 1:
            t3[..., k] = 0.0
    _eliminate(t1, t2, t3, 1)
    wnew = _col_solve(t1, t2, t3, wno[pI, pJ, :ke], w, 1)
    wno[pI, pJ, 1:ke] = wnew[..., 1:ke]

    # psi-point widths and coefficients (ocvisc.f90:286-339)
    dlypsi = np.zeros((ie + 1, je))
    dlypsi[1:ie] = 0.5 * (dlyv[0:ie - 1, 1:je + 1] + dlyv[1:ie, 1:je + 1])
    dlypsi[0] = dlyv[0, 1:je + 1]
    dlypsi[ie] = dlyv[ie - 1, 1:je + 1]
    dlxpsi = np.zeros((ie, je + 1))
    dlxpsi[:, 1:je] = 0.5 * (dlxu[1:ie + 1, 0:je - 1] + dlxu[1:ie + 1, 1:je])
    dlxpsi[:, 0] = dlxu[1:ie + 1, 0]
    dlxpsi[:, je] = dlxu[1:ie + 1, je - 1]
    p4 = lambda x: (x * x) * (x * x)
    mv = np.float64(minvalue)
    aulux = aulapuv * p4(_fmx(dlxp, mv))
    auluy = aulapuv * p4(_fmx(mv, dlypsi[1:ie + 1, :]))
    aulvy = aulapuv * p4(_fmx(mv, dlyp))
    aulvx = aulapuv * p4(_fmx(dlxpsi[:, 1:je + 1], mv))
    aulwx = aulapuv * p4(_fmx(dlxu[1:ie + 1, :], mv))
    aulwy = aulapuv * p4(_fmx(dlyv[:, 1:je + 1], mv))
    dzu = _fmx(dduo[1:ie + 1], mv)            # p-shaped (IE, JE, KE)
    dzv = _fmx(ddue[:, 1:je + 1], mv)
    dzp = _fmx(ddpo, mv)

    # Laplacians (FREESLIP, ocvisc.f90:347-430), every level
    uk1o = np.zeros_like(uko)
    vk1e = np.zeros_like(vke)
    for k in range(ke):
        U, M = uko[:, :, k], amsuo[:, :, k]
        # interior u-points I = 1..IE1, J = 2..JE1
        i0, j0 = uI, uJ
        xt = (M[2:ie + 1, j0] * (U[2:ie + 1, j0] - U[i0, j0]) / dlxp[1:ie, j0]
              - M[0:ie - 1, j0] * (U[i0, j0] - U[0:ie - 1, j0]) / dlxp[0:ie - 1, j0]) / dlxu[i0, j0]
        yt = (M[i0, 0:je - 2] * (U[i0, 0:je - 2] - U[i0, j0]) / dlypsi[i0, 0:je - 2]
              - M[i0, 2:je] * (U[i0, j0] - U[i0, 2:je]) / dlypsi[i0, j0]) / dlyu[i0, j0]
        uk1o[i0, j0, k] = M[i0, j0] * (xt + yt)
        # I = 0 and I = IE, J = 2..JE1
        ytI = lambda i: (M[i, 0:je - 2] * (U[i, 0:je - 2] - U[i, j0]) / dlypsi[i, 0:je - 2]
                         - M[i, 2:je] * (U[i, j0] - U[i, 2:je]) / dlypsi[i, j0]) / dlyu[i, j0]
        uk1o[0, j0, k] = M[0, j0] * ((M[1, j0] * (U[1, j0] - U[0, j0]) / dlxp[0, j0]) / dlxu[0, j0]
                                     + ytI(0))
        uk1o[ie, j0, k] = M[ie, j0] * ((-M[ie - 1, j0] * (U[ie, j0] - U[ie - 1, j0])
                                        / dlxp[ie - 1, j0]) / dlxu[ie, j0] + ytI(ie))
        # J = 1 and J = JE, I = 1..IE1
        xtJ = lambda j: (M[2:ie + 1, j] * (U[2:ie + 1, j] - U[i0, j]) / dlxp[1:ie, j]
                         - M[0:ie - 1, j] * (U[i0, j] - U[0:ie - 1, j]) / dlxp[0:ie - 1, j]) \
            / dlxu[i0, j]
        uk1o[i0, 0, k] = M[i0, 0] * (xtJ(0) + (-M[i0, 1] * (U[i0, 0] - U[i0, 1]) / dlypsi[i0, 0])
                                     / dlyu[i0, 0])
        uk1o[i0, je - 1, k] = M[i0, je - 1] * (xtJ(je - 1) + (M[i0, je - 2] * (
            U[i0, je - 2] - U[i0, je - 1]) / dlypsi[i0, je - 2]) / dlyu[i0, je - 1])

        V, N = vke[:, :, k], amsue[:, :, k]
        # interior v-points I = 2..IE1, J = 1..JE1 (array rows 1..IE-2, cols 1..JE-1)
        a0, b0 = slice(1, ie - 1), slice(1, je)
        xt = (N[2:ie, b0] * (V[2:ie, b0] - V[a0, b0]) / dlxpsi[a0, b0]
              - N[0:ie - 2, b0] * (V[a0, b0] - V[0:ie - 2, b0]) / dlxpsi[0:ie - 2, b0]) / dlxv[a0, b0]
        yt = (N[a0, 0:je - 1] * (V[a0, 0:je - 1] - V[a0, b0]) / dlyp[a0, 0:je - 1]
              - N[a0, 2:je + 1] * (V[a0, b0] - V[a0, 2:je + 1]) / dlyp[a0, 1:je]) / dlyv[a0, b0]
        vk1e[a0, b0, k] = N[a0, b0] * (xt + yt)
        ytV = lambda r: (N[r, 0:je - 1] * (V[r, 0:je - 1] - V[r, b0]) / dlyp[r, 0:je - 1]
                         - N[r, 2:je + 1] * (V[r, b0] - V[r, 2:je + 1]) / dlyp[r, 1:je]) / dlyv[r, b0]
        # I = 1 (row 0) and I = IE (row IE-1), J = 1..JE1
        vk1e[0, b0, k] = N[0, b0] * ((N[1, b0] * (V[1, b0] - V[0, b0]) / dlxpsi[0, b0])
                                     / dlxv[0, b0] + ytV(0))
        vk1e[ie - 1, b0, k] = N[ie - 1, b0] * ((-N[ie - 2, b0] * (V[ie - 1, b0] - V[ie - 2, b0])
                                                / dlxpsi[ie - 2, b0]) / dlxv[ie - 1, b0]
                                               + ytV(ie - 1))
        # J = 0 and J = JE, I = 2..IE1
        xtV = lambda c: (N[2:ie, c] * (V[2:ie, c] - V[a0, c]) / dlxpsi[a0, c]
                         - N[0:ie - 2, c] * (V[a0, c] - V[0:ie - 2, c]) / dlxpsi[0:ie - 2, c]) \
            / dlxv[a0, c]
        vk1e[a0, 0, k] = N[a0, 0] * (xtV(0) + (-N[a0, 1] * (V[a0, 0] - V[a0, 1]) / dlyp[a0, 0])
                                     / dlyv[a0, 0])
        vk1e[a0, je, k] = N[a0, je] * (xtV(je) + (N[a0, je - 1] * (V[a0, je - 1] - V[a0, je])
                                                   / dlyp[a0, je - 1]) / dlyv[a0, je])

    # biharmonic updates of UOO and VOE (ocvisc.f90:435-478)
    for k in range(ke):
        L, M = uk1o[:, :, k], amsuo[:, :, k]
        i0, j0 = uI, uJ
        area = dlxu[i0, j0] * dlyu[i0, j0]
        t = (aulux[1:ie, j0] * dlyp[1:ie, j0] * M[2:ie + 1, j0] * (L[2:ie + 1, j0] - L[i0, j0])
             / dlxp[1:ie, j0]
             - aulux[0:ie - 1, j0] * dlyp[0:ie - 1, j0] * M[0:ie - 1, j0]
             * (L[i0, j0] - L[0:ie - 1, j0]) / dlxp[0:ie - 1, j0]
             + auluy[0:ie - 1, 0:je - 2] * dlxpsi[0:ie - 1, 1:je - 1] * M[i0, 0:je - 2]
             * (L[i0, 0:je - 2] - L[i0, j0]) / dlypsi[i0, 0:je - 2]
             - auluy[0:ie - 1, j0] * dlxpsi[0:ie - 1, 2:je] * M[i0, 2:je]
             * (L[i0, j0] - L[i0, 2:je]) / dlypsi[i0, j0])
        uoo[i0, j0, k] = (M[i0, j0] / area) * (dlxu[i0, j0] * dlyu[i0, j0] * uko[i0, j0, k] - t)

        L, N = vk1e[:, :, k], amsue[:, :, k]
        a0, b0 = slice(1, ie - 1), slice(1, je)
        area = dlxv[a0, b0] * dlyv[a0, b0]
        t = (aulvx[a0, 0:je - 1] * dlypsi[2:ie, 0:je - 1] * N[2:ie, b0] * (L[2:ie, b0] - L[a0, b0])
             / dlxpsi[a0, b0]
             - aulvx[0:ie - 2, 0:je - 1] * dlypsi[1:ie - 1, 0:je - 1] * N[0:ie - 2, b0]
             * (L[a0, b0] - L[0:ie - 2, b0]) / dlxpsi[0:ie - 2, b0]
             + aulvy[a0, 0:je - 1] * dlxp[a0, 0:je - 1] * N[a0, 0:je - 1]
             * (L[a0, 0:je - 1] - L[a0, b0]) / dlyp[a0, 0:je - 1]
             - aulvy[a0, 1:je] * dlxp[a0, 1:je] * N[a0, 2:je + 1]
             * (L[a0, b0] - L[a0, 2:je + 1]) / dlyp[a0, 1:je])
        voe[a0, b0, k] = (N[a0, b0] / area) * (dlxv[a0, b0] * dlyv[a0, b0] * vke[a0, b0, k] - t)

    # w: Laplacian with its edge rows, then the biharmonic update
    # (FREESLIP + NON_HYDROSTATIC, ocvisc.f90:616-687), levels 1..KE
    wn1o = np.zeros((ie, je, ke))
    for k in range(ke):
        W, E = wno[:, :, k], weto[:, :, k]
        xtW = lambda r, c: (E[r + 1, c] * (W[r + 1, c] - W[r, c]) / dlxu[r + 1, c]
                            - E[r - 1, c] * (W[r, c] - W[r - 1, c]) / dlxu[r, c]) / dlxp[r, c]
        ytW = lambda r, c: (E[r, c - 1] * (W[r, c - 1] - W[r, c]) / dlyv[r, c]
                            - E[r, c + 1] * (W[r, c] - W[r, c + 1]) / dlyv[r, c + 1]) / dlyp[r, c]
        r, c = np.meshgrid(np.arange(1, ie - 1), np.arange(1, je - 1), indexing="ij")
        wn1o[1:ie - 1, 1:je - 1, k] = E[r, c] * (xtW(r, c) + ytW(r, c))
        cJ = np.arange(1, je - 1)
        wn1o[0, 1:je - 1, k] = E[0, cJ] * ((E[1, cJ] * (W[1, cJ] - W[0, cJ]) / dlxu[1, cJ])
                                           / dlxp[0, cJ] + ytW(0, cJ))
        wn1o[ie - 1, 1:je - 1, k] = E[ie - 1, cJ] * ((-E[ie - 2, cJ] * (W[ie - 1, cJ] - W[ie - 2, cJ])
                                                     / dlxu[ie - 1, cJ]) / dlxp[ie - 1, cJ]
                                                    + ytW(ie - 1, cJ))
        rI = np.arange(1, ie - 1)
        wn1o[1:ie - 1, 0, k] = E[rI, 0] * (xtW(rI, 0) + (-E[rI, 1] * (W[rI, 0] - W[rI, 1])
                                                        / dlyv[rI, 1]) / dlyp[rI, 0])
        wn1o[1:ie - 1, je - 1, k] = E[rI, je - 1] * (xtW(rI, je - 1) + (
            E[rI, je - 2] * (W[rI, je - 2] - W[rI, je - 1]) / dlyv[rI, je - 1]) / dlyp[rI, je - 1])
    for k in range(ke):
        L, E = wn1o[:, :, k], weto[:, :, k]
        r, c = pI, pJ
        vol = dlxp[r, c] * dlyp[r, c] * dzp[r, c, k]
        t = (+aulwx[r, c] * dlyu[2:ie, c] * dzu[r, c, k] * E[2:ie, c] * (L[2:ie, c] - L[r, c])
             / dlxu[2:ie, c]
             - aulwx[0:ie - 2, c] * dlyu[1:ie - 1, c] * dzu[0:ie - 2, c, k] * E[0:ie - 2, c]
             * (L[r, c] - L[0:ie - 2, c]) / dlxu[1:ie - 1, c]
             + aulwy[r, 0:je - 2] * dlxv[r, 1:je - 1] * dzv[r, 0:je - 2, k] * E[r, 0:je - 2]
             * (L[r, 0:je - 2] - L[r, c]) / dlyv[r, 1:je - 1]
             - aulwy[r, c] * dlxv[r, 2:je] * dzv[r, c, k] * E[r, 2:je]
             * (L[r, c] - L[r, 2:je]) / dlyv[r, 2:je])
        wno[r, c, k] = (E[r, c] / vol) * (dlxp[r, c] * dlyp[r, c] * dzp[r, c, k] * wno[r, c, k] - t)
    # OCTIMF (ocvisc.f90:767)
    return uoo, voe, wno, uoo.copy(), voe.copy()


# --------------------------------------------------------------- barotropic ---
# Written from boden.f90:117-128, 264-274, itprep.f90:15-40, troneu.f90:48-134,
# ocvtro.f90:1-62 and ocvtot.f90:13-96.  2D arrays: p (IE, JE), u (IE+1, JE)
# with index i <-> I, v (IE, JE+1) with index j <-> J.

def deut(g, depto, minvalue):
    ie, je = g["ie"], g["je"]
    deuto = np.zeros((ie + 1, je))
    deuto[1:ie, :] = np.minimum(depto[:-1, :], depto[1:, :])
    deuto[0, :] = deuto[1, :]
    deuto[ie, :] = deuto[ie - 1, :]
    deute = np.zeros((ie, je + 1))
    deute[:, 1:je] = np.minimum(depto[:, :-1], depto[:, 1:])
    deute[:, 0] = deute[:, 1]
    deute[:, je] = deute[:, je - 1]
    with np.errstate(divide="ignore"):
        deutio = np.where(deuto > minvalue, 1.0 / np.where(deuto > minvalue, deuto, 1.0), 0.0)
        deutie = np.where(deute > minvalue, 1.0 / np.where(deute > minvalue, deute, 1.0), 0.0)
    return deuto, deute, deutio, deutie


def itprep(g, b, deuto, deute):
    dt = g["dt"]
    xx = g["dlxp"] * g["dlyp"]
    uf = deuto * g["dlyu"] / g["dlxu"] * b["grav"] * b["conn"] * b["stabn"] * (dt * dt)
    vf = deute * g["dlxv"] / g["dlyv"] * b["grav"] * b["conn"] * b["stabn"] * (dt * dt)
    ff = 1.0 / (xx + uf[1:, :] + uf[:-1, :] + vf[:, 1:] + vf[:, :-1])
    return xx, uf, vf, ff


def troneu(g, b, xx, uf, vf, ff, u1o, v1e, uzo, vze):
    ie, je = g["ie"], g["je"]
    conn = b["conn"]
    cono = 1.0 - conn
    fu = (cono * u1o + uzo * conn) * g["dlyu"]           # the west face term at I-1 ...
    fu2 = (u1o * cono + uzo * conn) * g["dlyu"]          # ... and the east face term at I
    fv = (v1e * cono + conn * vze) * g["dlxv"]
    b1o = g["weto"][:, :, 0] * (g["dtdxpo"] * (fu[:-1, :] - fu2[1:, :]) / g["dlyp"]
                                + g["dtdyo"] * (fv[:, 1:] - fv[:, :-1]) / g["dlxp"])
    b1o = b1o * xx
    z = np.zeros((ie, je))
    if not b["eta_forc"]:
        z[0, :] = b1o[0, :] / xx[0, :]
        z[ie - 1, :] = b1o[ie - 1, :] / xx[ie - 1, :]
        z[:, 0] = b1o[:, 0] / xx[:, 0]
        z[:, je - 1] = b1o[:, je - 1] / xx[:, je - 1]
    # red-black masks over the interior I = 2..IE-1, J = 2..JE-1 (0-based 1..)
    I, J = np.meshgrid(np.arange(1, ie + 1), np.arange(1, je + 1), indexing="ij")
    inner = (I >= 2) & (I <= ie - 1) & (J >= 2) & (J <= je - 1)
    colour = [inner & ((I + J) % 2 == 0), inner & ((I + J) % 2 == 1)]
    sorpar = b["sorpar"]
    sorpai = 1.0 - sorpar
    ufe = np.zeros((ie, je)); ufw = np.zeros((ie, je))
    vfs = np.zeros((ie, je)); vfn = np.zeros((ie, je))
    ufe[:, :] = uf[1:, :]       # UF(I,J)
    ufw[:, :] = uf[:-1, :]      # UF(I-1,J)
    vfs[:, :] = vf[:, 1:]       # VF(I,J)
    vfn[:, :] = vf[:, :-1]      # VF(I,J-1)
    for _ in range(b["niter"]):
        for m in colour:
            ze = np.zeros_like(z); zw = np.zeros_like(z); zs = np.zeros_like(z); zn = np.zeros_like(z)
            ze[:-1, :] = z[1:, :]
            zw[1:, :] = z[:-1, :]
            zs[:, :-1] = z[:, 1:]
            zn[:, 1:] = z[:, :-1]
            new = sorpar * ff * (b1o + ufe * ze + ufw * zw + vfs * zs + vfn * zn) + sorpai * z
            z = np.where(m, new, z)
    return b1o, z


def ocvtro(g, b, deutio, deutie, z1o, uzo, vze, zo):
    ie, je = g["ie"], g["je"]
    c = b["rlsa1"] * b["grav"] * b["stabn"]
    uzo = uzo * deutio
    vze = vze * deutie
    uso = uzo.copy()
    vse = vze.copy()
    # USO: I = 1..IE-1, J = 2..JE-1
    uso[1:ie, 1:je - 1] = (uzo[1:ie, 1:je - 1] + c * g["dtdxuo"][1:ie, 1:je - 1]
                           * (z1o[0:ie - 1, 1:je - 1] - z1o[1:ie, 1:je - 1])
                           * g["amsuo"][1:ie, 1:je - 1, 0])
    # VSE: I = 2..IE-1, J = 1..JE-1
    vse[1:ie - 1, 1:je] = (vze[1:ie - 1, 1:je] + c * g["dpye"][1:ie - 1, 1:je]
                           * (z1o[1:ie - 1, 1:je] - z1o[1:ie - 1, 0:je - 1])
                           * g["amsue"][1:ie - 1, 1:je, 0])
    return uzo, vze, uso, vse, zo + z1o


def ocvtot(g, b, uso, vse, uoo, voe, uko, vke):
    conn = b["conn"]
    cono = 1.0 - conn
    dti = 1.0 / g["dt"]
    uk = g["amsuo"] * (uso[:, :, None] + uko)
    vk = g["amsue"] * (vse[:, :, None] + vke)
    uko_n = conn * uk + uoo * cono
    vke_n = conn * vk + voe * cono
    uoo_n, voe_n = uk, vk
    fu = uko_n * g["dduo"] * g["dlyu"][:, :, None]
    fv = vke_n * g["ddue"] * g["dlxv"][:, :, None]
    tx = dti * g["weto"] * (g["dtdxpo"][:, :, None] * (fu[:-1] - fu[1:]) / g["dlyp"][:, :, None])
    ty = dti * g["weto"] * (g["dtdyo"][:, :, None] * (fv[:, 1:] - fv[:, :-1]) / g["dlxp"][:, :, None])
    ke = g["ke"]
    wo = np.zeros(g["weto"].shape[:2] + (ke + 1,))
    for k in range(ke - 1, -1, -1):
        wo[:, :, k] = wo[:, :, k + 1] + tx[:, :, k] + ty[:, :, k]
    return uoo_n, voe_n, uko_n, vke_n, wo


def ocbarp(g, uso, vse):
    """ocbarp.f90:10-45: returns (uso, vse, uzo, vze)."""
    uzo = uso * g["amsuo"][:, :, 0]
    vze = vse * g["amsue"][:, :, 0]
    return uso * g["amsuo"][:, :, 0], vse * g["amsue"][:, :, 0], uzo, vze


def ocwind(g, txo, tye, sicomu, sicomv, tauwatu, tauwatv, uoo, voe):
    """ocwind.f90:20-38 on copies of uoo, voe.  p-shaped ice fields are
    indexed [I-1, J-1]; u arrays [I, J-1]; v arrays [I-1, J]."""
    ie, je = g["ie"], g["je"]
    dtdect = g["dt"] / g["dzw"][0]
    uoo, voe = uoo.copy(), voe.copy()
    a = g["amsuo"][1:ie, 1:je - 1, 0]                      # I = 1..IE-1, J = 2..JE-1
    ur = sicomu[0:ie - 1, 1:je - 1]
    uoo[1:ie, 1:je - 1, 0] = uoo[1:ie, 1:je - 1, 0] + dtdect * a * (
        txo[1:ie, 1:je - 1] * ur + (1. - ur) * a * tauwatu[0:ie - 1, 1:je - 1])
    b = g["amsue"][1:ie - 1, 1:je, 0]                      # I = 2..IE-1, J = 1..JE-1
    vr = sicomv[1:ie - 1, 0:je - 1]
    voe[1:ie - 1, 1:je, 0] = voe[1:ie - 1, 1:je, 0] + dtdect * b * (
        tye[1:ie - 1, 1:je] * vr + (1. - vr) * b * tauwatv[1:ie - 1, 0:je - 1])
    return uoo, voe


def trotest(g, b, xx, uf, vf, ff, ntry=200, niter=200):
    """trotest.f90:24-115 with SQRTRND (sqrtrnd.f90:1-8), one rank.  The SOR
    colours are vectorised (updates within a colour are independent); the sum
    of squared changes is accumulated serially in the reference's loop order
    (colour 1 then colour 2, J outer, I inner) with a cumulative sum."""
    import math
    ie, je = g["ie"], g["je"]
    d = 0.34679201245
    rnd = np.zeros((ie, je))
    for jj in range(je):
        for ii in range(ie):
            c = math.sqrt(34251. * d)
            d = c - int(c)
            rnd[ii, jj] = d
    b1o = (rnd - 0.5) * g["weto"][:, :, 0] * xx
    I, J = np.meshgrid(np.arange(1, ie + 1), np.arange(1, je + 1), indexing="ij")
    inner = (I >= 2) & (I <= ie - 1) & (J >= 2) & (J <= je - 1)
    colours = [inner & ((I + J) % 2 == 0), inner & ((I + J) % 2 == 1)]
    order = []  # (J, I)-ordered flat positions of each colour, Fortran order
    for m in colours:
        jj, ii = np.nonzero(m.T)
        order.append(ii + ie * jj)
    ufe, ufw, vfs, vfn = uf[1:, :], uf[:-1, :], vf[:, 1:], vf[:, :-1]
    sorpar, convmin, sorpmin = 1.75, 9e99, 1.75
    for _ in range(ntry):
        sorpar = sorpar + 0.001
        sorpai = 1. - sorpar
        z = np.zeros((ie, je))
        chabas = sumcha = 0.0
        for kiter in range(1, niter + 1):
            parts = []
            for m, pos in zip(colours, order):
                ze = np.zeros_like(z); zw = np.zeros_like(z); zs = np.zeros_like(z); zn = np.zeros_like(z)
                ze[:-1, :] = z[1:, :]; zw[1:, :] = z[:-1, :]; zs[:, :-1] = z[:, 1:]; zn[:, 1:] = z[:, :-1]
                new = sorpar * ff * (b1o + ufe * ze + ufw * zw + vfs * zs + vfn * zn) + sorpai * z
                dz = (z - new).ravel(order="F")[pos]
                parts.append(dz * dz)
                z = np.where(m, new, z)
            s = np.concatenate(parts)
            sumcha = float(np.cumsum(s)[-1]) if s.size else 0.0
            if kiter == 1:
                chabas = sumcha
        contric = sumcha / chabas
        if contric < convmin:
            sorpmin, convmin = sorpar, contric
    return sorpmin


# --------------------------------------------------------------- OCTHER ---
# Written from octher.f90, adisitj.f90 and rho1j.f90 as the reference is
# built (EISREST, REDWMICE, NURDIF); vectorised over (i, j).
def adisit(th, sh, pa):
    a1, a2, a3, a4 = 3.6504E-4, 8.3198E-5, 5.4065E-7, 4.0274E-9
    b1, b2, c1, c2 = 1.7439E-5, 2.9778E-7, 8.9309E-7, 3.1628E-8
    c3, d, e1, e2 = 2.1987E-10, 4.1057E-9, 1.6056E-10, 5.0484E-12
    pr = pa
    qc = pr * (a1 + pr * (c1 - e1 * pr))
    qv = pr * (b1 - d * pr)
    dc = 1. + pr * (-a2 + pr * (c2 - e2 * pr))
    dv = b2 * pr
    qnq = -pr * (-a3 + pr * c3)
    qn3 = -pr * a4
    qvs = qv * (sh - 35.) + qc
    dvs = dv * (sh - 35.) + dc
    tpo = th
    th = (th + qvs) / dvs
    t = th
    fne = -qvs + t * (dvs + t * (qnq + t * qn3)) - tpo
    fst = dvs + t * (2 * qnq + 3 * qn3 * t)
    return th - fne / fst


def rho1(t, s, p):
    B = (8.24493E-1, -4.0899E-3, 7.6438E-5, -8.2467E-7, 5.3875E-9)
    Cc = (-5.72466E-3, 1.0227E-4, -1.6546E-6)
    d0 = 4.8314E-4
    A = (999.8426, 6.793952E-2, -9.095290E-3, 1.001685E-4, -1.120083E-6, 6.536332E-9)
    F = (54.6746, -0.603459, 1.09987E-2, -6.1670E-5)
    Gg = (7.944E-2, 1.6483E-2, -5.3009E-4)
    AI = (2.2838E-3, -1.0981E-5, -1.6078E-6)
    aj0 = 1.91075E-4
    AM = (-9.9348E-7, 2.0816E-8, 9.1697E-10)
    E = (19652.21, 148.4206, -2.327105, 1.360477E-2, -5.155288E-5)
    H = (3.239908, 1.43713E-3, 1.16092E-4, -5.77905E-7)
    AK = (8.50935E-5, -6.12293E-6, 5.2787E-8)
    s = np.where(s > 28., s, 28.)
    s3h = np.sqrt(s * s * s)
    num = (A[0] + t * (A[1] + t * (A[2] + t * (A[3] + t * (A[4] + t * A[5]))))
           + s * (B[0] + t * (B[1] + t * (B[2] + t * (B[3] + t * B[4])))) + d0 * (s * s)
           + s3h * (Cc[0] + t * (Cc[1] + Cc[2] * t)))
    kk = (p * (H[0] + t * (H[1] + t * (H[2] + t * H[3])) + s * (AI[0] + t * (AI[1] + AI[2] * t))
               + aj0 * s3h + (AK[0] + t * (AK[1] + t * AK[2]) + s * (AM[0] + t * (AM[1] + t * AM[2]))) * p)
          + E[0] + t * (E[1] + t * (E[2] + t * (E[3] + t * E[4])))
          + s * (F[0] + t * (F[1] + t * (F[2] + t * F[3]))) + s3h * (Gg[0] + t * (Gg[1] + Gg[2] * t)))
    return num / (1. - p / kk)


def density(th_, t, s, p):
    if th_["eos"] == 1:
        return th_["rho0"] + th_["drdt"] * (t - th_["t0"]) + th_["drds"] * (s - th_["s0"])
    return rho1(adisit(t, s, p), s, p)


def _z2(th_, k, shape):
    a = th_.get(k)
    return np.zeros(shape) if a is None else np.asarray(a, dtype=np.float64)


def octher_surface(g, th_, tho, sao, zo):
    """octher.f90:43-107 in place on tho, sao, zo; returns (eminpo, rivrun)."""
    shp = zo.shape
    dt = g["dt"]
    sicomo, sictho, sicsno = (_z2(th_, k, shp) for k in ("sicomo", "sictho", "sicsno"))
    relsao, reltho, giriv = (_z2(th_, k, shp) for k in ("relsao", "reltho", "giriv"))
    reiscon = 1. - sicomo
    oldso = sao[:, :, 0].copy()
    sao[:, :, 0] = sao[:, :, 0] + dt * th_["relsal"] * reiscon * (relsao - sao[:, :, 0])
    tho[:, :, 0] = tho[:, :, 0] + dt * th_["reltem"] * (reltho - tho[:, :, 0])
    ddpo1 = g["ddpo"][:, :, 0]
    eminpo = ((ddpo1 + zo - sictho * th_["rhoicwa"] - sicsno * th_["rhosnwa"])
              * (np.where(oldso > 1.E-3, oldso, 1.E-3) / np.where(sao[:, :, 0] > 1.E-3, sao[:, :, 0], 1.E-3) - 1.))
    zo[:] = (zo + eminpo) * g["weto"][:, :, 0]
    eminpo = eminpo * (1. / dt)
    z = ddpo1 + zo - sictho * th_["rhoicwa"] - sicsno * th_["rhosnwa"]
    zzzdz = np.where(g["almzer"] > z, g["almzer"], z)
    driv = giriv * dt
    sao[:, :, 0] = sao[:, :, 0] * zzzdz / (zzzdz + driv)
    zo[:] = zo + driv
    return eminpo, driv / dt


def octher_column(g, th_, tho, sao, zo, uko, vke, avo, dvo, kcondep):
    """octher.f90:139-451 in place on tho, sao, avo, dvo, kcondep; returns
    (po, stabio, rhoo)."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    shp = (ie, je)
    G = th_["grav"]
    preff, dz, di, dzw = th_["preff"], g["dz"], g["di"], g["dzw"]
    weto, ddpo = g["weto"], g["ddpo"]
    sicomo, sictho, sicsno, fu10 = (_z2(th_, k, shp) for k in ("sicomo", "sictho", "sicsno", "fu10"))
    po = np.zeros((ie, je, ke), order="F")
    stab = np.zeros((ie, je, ke), order="F")
    rhoo = np.zeros((ie, je, ke), order="F")
    rh = density(th_, tho[:, :, 0], sao[:, :, 0], preff[0])
    po[:, :, 0] = G * g["tiestu"][0] * 0.00097 * rh
    for k in range(1, ke):                      # Fortran K = k + 1
        disti = 1. / dz[k]
        rh = density(th_, tho[:, :, k], sao[:, :, k], preff[k])
        rup = density(th_, tho[:, :, k - 1], sao[:, :, k - 1], preff[k])
        stab[:, :, k] = disti * (rh - rup)
        po[:, :, k] = po[:, :, k - 1] + G * dz[k] * 0.00049 * (rh + rup)
        zs = 1. if k == 1 else 0.
        surf = zs * (zo - sictho * th_["rhoicwa"] - sicsno * th_["rhosnwa"])
        den = ddpo[:, :, k] + ddpo[:, :, k - 1] + surf + (1. - weto[:, :, k])
        tq = ((ddpo[:, :, k - 1] + surf) * tho[:, :, k - 1] + ddpo[:, :, k] * tho[:, :, k]) / den
        sq = ((ddpo[:, :, k - 1] + surf) * sao[:, :, k - 1] + ddpo[:, :, k] * sao[:, :, k]) / den
        st = stab[:, :, k]
        q = -st / (1.E-11 + np.abs(st))
        switc = np.where(0. > q, 0., q) * weto[:, :, k]
        helpswi = switc
        sw = 0.
        tho[:, :, k - 1] = tq * sw + (1. - sw) * tho[:, :, k - 1]
        tho[:, :, k] = tq * sw + (1. - sw) * tho[:, :, k]
        sao[:, :, k - 1] = sq * sw + (1. - sw) * sao[:, :, k - 1]
        sao[:, :, k] = sq * sw + (1. - sw) * sao[:, :, k]
        st = (1. - sw) * st
        stab[:, :, k] = np.where(st > 0., st, 0.)
        kcondep += ((kcondep == k) & (helpswi >= 0.5)).astype(kcondep.dtype)
    # D on I = 1..IE-1, J = 1..JE-1 (0-based p index 0..IE-2)
    relne = 0.4
    relax = 1. - relne
    gor = G / 1025.
    P = (slice(0, ie - 1), slice(0, je - 1))
    Uw, Ue = (slice(0, ie - 1), slice(0, je - 1)), (slice(1, ie), slice(0, je - 1))
    Vs, Vn = (slice(0, ie - 1), slice(0, je - 1)), (slice(0, ie - 1), slice(1, je))
    ice = 1. - sicomo[P]
    f = fu10[P]
    t1 = th_["wt"] * (ice * ice) * (f * f * f)
    s1 = th_["wt"] * (ice * ice) * (f * f * f)
    amsuo, amsue = g["amsuo"], g["amsue"]
    for k in range(1, ke):
        ko = k - 1
        stabeps = th_["cstabeps"] / dzw[ko]
        wtdecay = math.exp(-float(dzw[ko]) / 40.)
        zs = 1. if ko == 0 else 0.
        sk, sko = stab[P + (k,)], stab[P + (ko,)]
        t1 = t1 * wtdecay * stabeps / (stabeps + 0.5 * (sk + (1. - zs) * sko))
        s1 = s1 * wtdecay * stabeps / (stabeps + 0.5 * (sk + (1. - zs) * sko))
        du1 = uko[Uw + (k,)] - uko[Uw + (ko,)]
        du2 = uko[Ue + (k,)] - uko[Ue + (ko,)]
        dv1 = vke[Vs + (k,)] - vke[Vs + (ko,)]
        dv2 = vke[Vn + (k,)] - vke[Vn + (ko,)]
        w = weto[P + (k,)]
        dudo = g["almzer"] + w * (di[k] * di[k]) * (du1 * du1 + du2 * du2 + dv1 * dv1 + dv2 * dv2) * 0.5
        hho = w * (amsuo[Ue + (k,)] + amsuo[Uw + (k,)] + amsue[Vs + (k,)] + amsue[Vn + (k,)]) * 0.25
        r = gor * sk / dudo
        rinumo = hho * np.where(r > 0., r, 0.)
        xd, xa = 1. + 5. * rinumo, 1. + 5. * rinumo
        dv, av = dvo[P + (k,)], avo[P + (k,)]
        m = th_["dv0"] + s1
        dv = (relax * np.where(m < dv, m, dv) + relne * (s1 + th_["dv0"] / (xd * xd * xd) + th_["dbackv"][k] + 0.0)) * w
        m = th_["av0"] + th_["abackv"][k]
        av = (relax * np.where(m < av, m, av) + relne * (t1 + th_["av0"] / (xa * xa) + th_["abackv"][k] + 0.0)) * w
        ca = th_["cavocon"] * (1.E-11 - sk) / (1.E-11 + np.abs(sk))
        av = w * np.where(ca > av, ca, av)
        cd = th_["cdvocon"] * (1.E-11 - sk) / (1.E-11 + np.abs(sk))
        dv = w * np.where(cd > dv, cd, dv)
        dvo[P + (k,)] = dv
        avo[P + (k,)] = av
    avo[:, :, ke] = 0.
    dvo[:, :, ke] = 0.
    for k in range(1, ke):
        land = weto[:, :, k] < 0.5
        tho[:, :, k] = np.where(land, tho[:, :, k - 1], tho[:, :, k])
        sao[:, :, k] = np.where(land, sao[:, :, k - 1], sao[:, :, k])
    for k in range(ke):
        rhoo[:, :, k] = density(th_, tho[:, :, k], sao[:, :, k], preff[k])
    return po, stab, rhoo


# ------------------------------------------------------------- OCMODMOM ---
# Written from ocmodmom.f90 (NON_HYDROSTATIC); vectorised over (i, j), with
# the grid angles evaluated by math.cos / math.sqrt point by point.
def ocmodmom(g, b, c, deutio, deutie, zo, uoo, voe, uko, vke, wno, po, stabio):
    """In place on uko, vke, wno, po, stabio; returns (uk1o, vk1e, u1o, uso, v1e, vse)."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    G, stabn, dt, almzer = b["grav"], b["stabn"], g["dt"], g["almzer"]
    stabo = 1. - stabn
    dduo, ddue, amsuo, amsue = g["dduo"], g["ddue"], g["amsuo"], g["amsue"]
    gila, giph, omega = c["gila"], c["giph"], c["omega"]
    GI = lambda a, ii, jj: float(a[ii - 1, jj - 1])
    for k in range(ke):
        stabio[:, :, k] = 0.001 * g["dz"][k] * stabio[:, :, k] * g["weto"][:, :, k]
        po[:, :, k] = po[:, :, k] + G * zo * b["rlsa1"]
    for k in range(ke):
        uko[:, :, k] = uko[:, :, k] * dduo[:, :, k]
        vke[:, :, k] = vke[:, :, k] * ddue[:, :, k]
    uk1o, vk1e = uko.copy(order="F"), vke.copy(order="F")
    wn1o = wno.copy(order="F")
    # grid-angle factors (Fortran I, J -> 0-based u index I, p index I-1)
    fu = {}
    for j in range(2, je):
        for i in range(1, ie):
            dlon = (GI(gila, 2 * i + 2, 2 * j) - GI(gila, 2 * i + 1, 2 * j)) * math.cos(GI(gila, 2 * i + 1, 2 * j))
            dlat = GI(giph, 2 * i + 2, 2 * j) - GI(giph, 2 * i + 1, 2 * j)
            fu[i, j] = (dlon, math.sqrt(dlon * dlon + dlat * dlat) + almzer,
                        2 * omega * math.cos(GI(giph, 2 * i + 1, 2 * j)))
    fv = {}
    for j in range(1, je):
        for i in range(2, ie):
            dlon = (GI(gila, 2 * i, 2 * j) - GI(gila, 2 * i, 2 * j + 1)) * math.cos(GI(gila, 2 * i, 2 * j + 1))
            dlat = GI(giph, 2 * i, 2 * j) - GI(giph, 2 * i, 2 * j + 1)
            fv[i, j] = (dlon, math.sqrt(dlon * dlon + dlat * dlat) + almzer,
                        2 * omega * math.cos(GI(giph, 2 * i, 2 * j + 1)))
    fw = {}
    for j in range(2, je):
        for i in range(2, ie):
            dlon = (GI(gila, 2 * i + 1, 2 * j) - GI(gila, 2 * i, 2 * j)) * math.cos(GI(gila, 2 * i, 2 * j))
            dlat = GI(giph, 2 * i, 2 * j - 1) - GI(giph, 2 * i, 2 * j)
            fw[i, j] = (dlon, dlat, math.sqrt(dlon * dlon + dlat * dlat) + almzer,
                        2 * omega * math.cos(GI(giph, 2 * i, 2 * j)))

    def tab(d, lo_i, hi_i, lo_j, hi_j, q):
        return np.array([[d[i, j][q] for j in range(lo_j, hi_j + 1)] for i in range(lo_i, hi_i + 1)])

    dlon_u, dist_u, f1_u = (tab(fu, 1, ie - 1, 2, je - 1, q) for q in range(3))
    dlon_v, dist_v, f1_v = (tab(fv, 2, ie - 1, 1, je - 1, q) for q in range(3))
    dlon_w, dlat_w, dist_w, f1_w = (tab(fw, 2, ie - 1, 2, je - 1, q) for q in range(4))
    # index maps: u(I, J) -> [I, J-1]; v(I, J) -> [I-1, J]; p(I, J) -> [I-1, J-1]
    Iu, Ju = slice(1, ie), slice(1, je - 1)            # u interior I 1..IE-1, J 2..JE-1
    for _ in range(12):
        ucor = stabn * uk1o + stabo * uko
        vcor = stabn * vk1e + stabo * vke
        wcor = stabn * wn1o + stabo * wno
        for k in range(ke):
            # u: VCOR(I,J), (I+1,J), (I,J-1), (I+1,J-1) -> v array [I-1, J], [I, J], [I-1, J-1], [I, J-1]
            vc = vcor[:, :, k]
            vcor_u = 0.25 * (vc[0:ie - 1, 2:je] + vc[1:ie, 2:je] + vc[0:ie - 1, 1:je - 1] + vc[1:ie, 1:je - 1])
            pk = po[:, :, k]
            new_u = (uko[Iu, Ju, k] + g["dtdxuo"][Iu, Ju] * (pk[0:ie - 1, 1:je - 1] - pk[1:ie, 1:je - 1]) * dduo[Iu, Ju, k]
                     + dt * c["ftwou"][Iu, Ju] * vcor_u * amsuo[Iu, Ju, k])
            # v: UCOR(I,J), (I-1,J), (I,J+1), (I-1,J+1) for I 2..IE-1, J 1..JE-1
            uc = ucor[:, :, k]
            ucor_v = 0.25 * (uc[2:ie, 0:je - 1] + uc[1:ie - 1, 0:je - 1] + uc[2:ie, 1:je] + uc[1:ie - 1, 1:je])
            new_v = (vke[1:ie - 1, 1:je, k] + g["dpye"][1:ie - 1, 1:je] * (pk[1:ie - 1, 1:je] - pk[1:ie - 1, 0:je - 1])
                     * ddue[1:ie - 1, 1:je, k] - dt * c["ftwov"][1:ie - 1, 1:je] * ucor_v * amsue[1:ie - 1, 1:je, k])
            # NH u: WCOR at p (I, J) and (I+1, J), J 2..JE-1 -> p [I-1, J-1], [I, J-1]
            wa, wb = wcor[:, :, k], wcor[:, :, k + 1]
            dlxp, dlyp = g["dlxp"], g["dlyp"]
            wcor_u = 0.25 * ((wa[0:ie - 1, 1:je - 1] + wb[0:ie - 1, 1:je - 1]) * dlxp[0:ie - 1, 1:je - 1]
                             + (wa[1:ie, 1:je - 1] + wb[1:ie, 1:je - 1]) * dlxp[1:ie, 1:je - 1]) / g["dlxu"][Iu, Ju]
            new_u = new_u - dt * f1_u * wcor_u * dduo[Iu, Ju, k] * dlon_u / dist_u
            # NH v: p (I, J), (I, J+1) for I 2..IE-1, J 1..JE-1 -> p [I-1, J-1], [I-1, J]
            wcor_v = 0.25 * ((wa[1:ie - 1, 0:je - 1] + wb[1:ie - 1, 0:je - 1]) * dlyp[1:ie - 1, 0:je - 1]
                             + (wa[1:ie - 1, 1:je] + wb[1:ie - 1, 1:je]) * dlyp[1:ie - 1, 1:je]) / g["dlyv"][1:ie - 1, 1:je]
            new_v = new_v - dt * f1_v * wcor_v * ddue[1:ie - 1, 1:je, k] * dlon_v / dist_v
            uk1o[Iu, Ju, k] = new_u
            vk1e[1:ie - 1, 1:je, k] = new_v
            if k >= 1:
                # p I, J 2..IE-1 / 2..JE-1 -> [1:ie-1, 1:je-1]; u(I), u(I-1) -> [I], [I-1]; v(J), v(J-1)
                dd = g["ddpo"][1:ie - 1, 1:je - 1, k] + almzer
                ddm = g["ddpo"][1:ie - 1, 1:je - 1, k - 1] + almzer
                ucor_w = 0.25 * ((uko[2:ie, 1:je - 1, k] + uko[1:ie - 1, 1:je - 1, k]) / dd
                                 + (uko[2:ie, 1:je - 1, k - 1] + uko[1:ie - 1, 1:je - 1, k - 1]) / ddm)
                vcor_w = 0.25 * ((vke[1:ie - 1, 2:je, k] + vke[1:ie - 1, 1:je - 1, k]) / dd
                                 + (vke[1:ie - 1, 2:je, k - 1] + vke[1:ie - 1, 1:je - 1, k - 1]) / ddm)
                wn1o[1:ie - 1, 1:je - 1, k] = (wno[1:ie - 1, 1:je - 1, k] + dt * g["weto"][1:ie - 1, 1:je - 1, k]
                                               * (f1_w * dlon_w / dist_w * ucor_w - f1_w * dlat_w / dist_w * vcor_w))
        wno[:] = wn1o
    u1o = np.zeros((ie + 1, je))
    uso = np.zeros((ie + 1, je))
    v1e = np.zeros((ie, je + 1))
    vse = np.zeros((ie, je + 1))
    for k in range(ke):
        po[:, :, k] = po[:, :, k] - G * zo * b["rlsa1"]
        u1o = u1o + dduo[:, :, k] * uoo[:, :, k]
        uso = uso + uk1o[:, :, k]
        v1e = v1e + ddue[:, :, k] * voe[:, :, k]
        vse = vse + vk1e[:, :, k]
    for k in range(ke):
        uko[:, :, k] = uoo[:, :, k] - amsuo[:, :, k] * deutio * u1o
        uk1o[:, :, k] = uk1o[:, :, k] * (amsuo[:, :, k] / (almzer + dduo[:, :, k])) - amsuo[:, :, k] * deutio * uso
        vke[:, :, k] = voe[:, :, k] - amsue[:, :, k] * deutie * v1e
        vk1e[:, :, k] = vk1e[:, :, k] * (amsue[:, :, k] / (almzer + ddue[:, :, k])) - amsue[:, :, k] * deutie * vse
    return uk1o, vk1e, u1o, uso, v1e, vse


# --------------------------------------------------------------- OCCLIT ---
def _occlit_div(g, uko, vke, k, below):
    """occlit.f90:108-112 / 250-254 over all p-points at level k."""
    ie, je = g["ie"], g["je"]
    dti = 1. / g["dt"]
    return below + dti * g["weto"][:, :, k] * (
        g["dtdxpo"] * (uko[0:ie, :, k] * g["dlyu"][0:ie, :] - uko[1:ie + 1, :, k] * g["dlyu"][1:ie + 1, :]) / g["dlyp"]
        + g["dtdyo"] * (vke[:, 1:je + 1, k] * g["dlxv"][:, 1:je + 1] - vke[:, 0:je, k] * g["dlxv"][:, 0:je]) / g["dlxp"])


def occlit(g, b, deutio, deutie, uko, vke, uk1o, vk1e, wo, stabio):
    """In place on uko, vke, uk1o, vk1e, wo, stabio; returns CONTRA."""
    ie, je, ke = g["ie"], g["je"], g["ke"]
    G, stabn, conn, dt, almzer = b["grav"], b["stabn"], b["conn"], g["dt"], g["almzer"]
    dduo, ddue, amsuo, amsue = g["dduo"], g["ddue"], g["amsuo"], g["amsue"]
    stabio[:, :, 0] = 0.
    bruva = np.zeros((ie, je))
    for k in range(ke):
        bruva = bruva + g["tiestw"][k + 1] * stabio[:, :, k]
    uko *= dduo
    uk1o *= dduo
    vke *= ddue
    vk1e *= ddue
    for k in range(ke - 1, -1, -1):
        wo[:, :, k] = _occlit_div(g, uko, vke, k, wo[:, :, k + 1])
    wpo = np.zeros((ie, je, ke))
    slow = np.zeros((ie, je))
    for k in range(ke):
        slow = slow + stabio[:, :, k] * dt * wo[:, :, k]
        wpo[:, :, k] = slow
    under = 0.
    contrij = np.zeros((ie, je))
    dtdxuo_p = g["dtdxuo"][1:ie + 1, :]          # DTDXUO(I, J) at p-index I
    for it in range(1, 9):
        px = np.zeros((ie + 1, je))
        py = np.zeros((ie, je + 1))
        for k in range(ke):
            px[1:ie, :] = px[1:ie, :] + dduo[1:ie, :, k] * g["dtdxuo"][1:ie, :] * (wpo[1:ie, :, k] - wpo[0:ie - 1, :, k]) * amsuo[1:ie, :, k]
            py[:, 1:je] = py[:, 1:je] + ddue[:, 1:je, k] * g["dpye"][:, 1:je] * (wpo[:, 0:je - 1, k] - wpo[:, 1:je, k]) * amsue[:, 1:je, k]
        px[1:ie, :] = px[1:ie, :] * deutio[1:ie, :]
        py[:, 1:je] = py[:, 1:je] * deutie[:, 1:je]
        ucos = np.zeros((ie + 1, je))
        vcos = np.zeros((ie, je + 1))
        U = (slice(1, ie), slice(1, je - 1))          # I 1..IE-1, J 2..JE-1
        V = (slice(1, ie - 1), slice(1, je))          # I 2..IE-1, J 1..JE-1
        for k in range(ke):
            dw = wpo[1:ie, 1:je - 1, k] - wpo[0:ie - 1, 1:je - 1, k]
            u = uk1o[U + (k,)] + stabn * (px[U] - g["dtdxuo"][U] * dw) * dduo[U + (k,)]
            ucos[U] = ucos[U] + u
            uko[U + (k,)] = u * amsuo[U + (k,)]
            dwv = wpo[1:ie - 1, 0:je - 1, k] - wpo[1:ie - 1, 1:je, k]
            v = vk1e[V + (k,)] + stabn * (py[V] - g["dpye"][V] * dwv) * ddue[V + (k,)]
            vcos[V] = vcos[V] + v
            vke[V + (k,)] = v * amsue[V + (k,)]
        for k in range(ke):
            uko[U + (k,)] = uko[U + (k,)] - ucos[U] * deutio[U] * dduo[U + (k,)]
            vke[V + (k,)] = vke[V + (k,)] - vcos[V] * deutie[V] * ddue[V + (k,)]
        if it == 8:
            break
        t1o = np.zeros((ie, je, ke))
        slow = np.zeros((ie, je))
        for k in range(ke - 1, -1, -1):
            t1o[:, :, k] = _occlit_div(g, uko, vke, k, slow)
            slow = t1o[:, :, k]
        tlow = np.zeros((ie, je))
        contrij = np.zeros((ie, je))
        for k in range(1, ke):
            ove = wpo[:, :, k].copy()
            tlow = tlow + G * stabio[:, :, k] * dt * (conn * t1o[:, :, k] + wo[:, :, k])
            speed = 2. * G * bruva * (dtdxuo_p * dtdxuo_p + g["dtdyo"] * g["dtdyo"])
            brems = under * speed * conn * stabn / (1. + speed)
            vorw = 1. - brems
            wpo[:, :, k] = vorw * tlow + brems * wpo[:, :, k]
            d = ove - wpo[:, :, k]
            contrij = contrij + d * d
        under = 1.
    for k in range(ke):
        uko[:, :, k] = uko[:, :, k] * amsuo[:, :, k] / (almzer + dduo[:, :, k])
        uk1o[:, :, k] = uk1o[:, :, k] * amsuo[:, :, k] / (almzer + dduo[:, :, k])
        vke[:, :, k] = vke[:, :, k] * amsue[:, :, k] / (almzer + ddue[:, :, k])
        vk1e[:, :, k] = vk1e[:, :, k] * amsue[:, :, k] / (almzer + ddue[:, :, k])
    return float(np.add.accumulate(contrij.T.ravel())[-1])  # J outer, I inner, in order
