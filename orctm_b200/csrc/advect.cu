// Mass-conserving limited advection (Maier-Reimer scheme) of tracers and of
// the u, v, w momenta: OCADPO (ocadpo.f90:94-348), OCUAD (ocuad.f90:1-271),
// OCVAD (ocvad.f90:1-271) and OCWAD (ocwad.f90:1-238).
//
// Each routine is three direction-split sweeps z -> x -> y.  Per sweep a cell
// volume V and the field T are updated from face transports
//     RN = V + WTP(-) - WTP(0) - WTM(0) + WTM(+)
//     T' = (T*V + TRP(-) - TRP(0) - TRM(0) + TRM(+)) / RN
// The z sweep runs one thread per column marching down the column with the
// transports of the level below carried in registers; the x and y sweeps
// compute each face's transports once per block into shared memory and then
// update one cell per thread.  Every sweep writes a fresh buffer (never in place), so
// neighbouring columns always read the previous sweep's values.  Arithmetic is
// IEEE binary64 in the reference's operation order (built with --fmad=false),
// except that the three divisions of a face and a cell use div_nr (within
// 1 ulp of IEEE division), so results match the CPU restatement to a few ulp.
#include "common.cuh"
#include "ops.h"

namespace orctm {

namespace {

struct Fl { double trp, trm, wtp, wtm; };

#define AT(a, i, j, K) (a)[G.L.at((i), (j), (K)-1)]
#define A2(a, i, j) (a)[G.L.at2((i), (j))]

// the same without a mask factor (OCUAD/OCVAD forms: SCHA has no WETO product)
__device__ __forceinline__ Fl limited_nm(double up, double um, double t, double tprev, double tnext,
                                         double vol, double cap) {
  const double abl = fabs(tprev - tnext);
  const double zwabl = fabs(tprev + tnext - 2. * t);
  const double scha = fmx(0., div_nr(abl - zwabl, abl + 1.E-20));
  const double sch = fmn(cap, div_nr(scha * vol, up + um + 1.E-20));
  const double schi = 1. - sch;
  Fl f;
  f.trp = up * (schi * t + sch * 0.5 * (t + tprev));
  f.trm = um * (schi * t + sch * 0.5 * (t + tnext));
  f.wtp = up;
  f.wtm = um;
  return f;
}

__device__ __forceinline__ Fl upwind(double up, double um, double t) {
  Fl f;
  f.trp = up * t;
  f.trm = um * t;
  f.wtp = up;
  f.wtm = um;
  return f;
}

__device__ __forceinline__ Fl zero_fl() { return Fl{0., 0., 0., 0.}; }

// update from the transports of the previous (m) / own (c) / next (p) faces
__device__ __forceinline__ void apply(double t, double v, const Fl& m, const Fl& c, const Fl& p,
                                      double& tn, double& vn) {
  const double rn = v + m.wtp - c.wtp - c.wtm + p.wtm;
  tn = div_nr(t * v + m.trp - c.trp - c.trm + p.trm, rn);
  vn = rn;
}

// vertical update: RN = V + WTP(K+1) - WTP(K) - WTM(K) + WTM(K-1)
__device__ __forceinline__ void apply_z(double t, double v, const Fl& fm, const Fl& fc,
                                        const Fl& fp, double& tn, double& vn) {
  const double rn = v + fp.wtp - fc.wtp - fc.wtm + fm.wtm;
  tn = div_nr(t * v + fp.trp - fc.trp - fc.trm + fm.trm, rn);
  vn = rn;
}

// ---------------------------------------------------------------- OCADPO ---
// vertical sweep, ocadpo.f90:94-173; one thread per p-column
__global__ void k_adpo_z(Geo G, const double* __restrict__ T, const double* __restrict__ wo,
                         const double* __restrict__ zo, double* __restrict__ To,
                         double* __restrict__ Vo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const int ij = G.L.at2(i, j);
  const double dlxp = G.dlxp[ij], dlyp = G.dlyp[ij];
  auto v0 = [&](int K) {
    double s = wet(G.gp, ij, K) * dlxp * dlyp * thick(G.gp, G.dzw, ij, K);
    if (K == 1) s = s + dlxp * dlyp * wet(G.gp, ij, 1) * (zo[ij] - AT(wo, i, j, 1) * G.dt);
    return s;
  };
  const bool interior = i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1;
  if (!interior) {
    for (int K = 1; K <= KE; ++K) {
      AT(To, i, j, K) = AT(T, i, j, K);
      AT(Vo, i, j, K) = v0(K);
    }
    return;
  }
  const double cdt = 0.5 * G.dt * dlyp * dlxp;
  auto flux = [&](int K, double vol) {
    const int klo = K + 1 < KE ? K + 1 : KE;
    const int kup = K - 1 > 1 ? K - 1 : 1;
    const double t = AT(T, i, j, K), tu = AT(T, i, j, kup), tl = AT(T, i, j, klo);
    const double w0 = AT(wo, i, j, K), w1 = AT(wo, i, j, K + 1);
    const double up = cdt * (w0 + fabs(w0));
    const double um = cdt * (fabs(w1) - w1);
    const double abl = fabs(tu - tl);
    const double zwabl = fabs(tu + tl - 2. * t);
    const double scha = fmx(0., div_nr(abl - zwabl, abl + 1.E-20));
    double sch = fmn(wet(G.gp, ij, klo), div_nr(scha * vol, up + um + 1.E-20));
    if (K == 1 || K == KE) sch = 0.;
    const double schi = 1. - sch;
    Fl f;
    f.trp = up * (schi * t + sch * 0.5 * (t + tu));
    f.trm = um * (schi * t + sch * 0.5 * (t + tl));
    f.wtp = up;
    f.wtm = um;
    return f;
  };
  Fl fm = zero_fl();               // transports of level K-1 (TRM/WTM(0) = 0)
  double vk = v0(1);
  Fl fc = flux(1, vk);
  for (int K = 1; K <= KE; ++K) {
    double vn = 0.;
    Fl fp = zero_fl();             // TRP/WTP(KEP) = 0
    if (K < KE) {
      vn = v0(K + 1);
      fp = flux(K + 1, vn);
    }
    const double t = AT(T, i, j, K);
    double tn = t, vv = vk;
    if (wetb(G.gp, ij, K)) apply_z(t, vk, fm, fc, fp, tn, vv);
    AT(To, i, j, K) = tn;
    AT(Vo, i, j, K) = vv;
    fm = fc;
    fc = fp;
    vk = vn;
  }
}

// x-direction transports at p-column q of row j (ocadpo.f90:203-232)
__device__ __forceinline__ Fl adpo_xflux(const Geo& G, const double* T, const double* V,
                                         const double* uko, int q, int j, int K) {
  if (q < 2 || q > G.L.ie - 1) return zero_fl();
  const double u0 = AT(uko, q, j, K), um1 = AT(uko, q - 1, j, K);
  const int ij = G.L.at2(q, j), ijm = G.L.at2(q - 1, j);
  const double up = 0.5 * G.dt * thick(G.gu, G.dzw, ij, K) * G.dlyu[ij] * (u0 + fabs(u0));
  const double um = 0.5 * G.dt * thick(G.gu, G.dzw, ijm, K) * (fabs(um1) - um1) * G.dlyu[ijm];
  // SCHA = MAX(...)*WETO(I)*WETO(I+1)*WETO(I-1), factors applied in that order
  const double t = AT(T, q, j, K), te = AT(T, q + 1, j, K), tw = AT(T, q - 1, j, K);
  const double abl = fabs(te - tw);
  const double zwabl = fabs(te + tw - 2. * t);
  const double scha = fmx(0., div_nr(abl - zwabl, abl + 1.E-20)) * wet(G.gp, ij, K) *
                      wet(G.gp, G.L.at2(q + 1, j), K) * wet(G.gp, G.L.at2(q - 1, j), K);
  const double sch = fmn(1., div_nr(scha * AT(V, q, j, K), up + um + 1.E-20));
  const double schi = 1. - sch;
  Fl f;
  f.trp = up * (schi * t + sch * 0.5 * (t + te));
  f.trm = um * (schi * t + sch * 0.5 * (t + tw));
  f.wtp = up;
  f.wtm = um;
  return f;
}

__device__ __forceinline__ Fl adpo_yflux(const Geo& G, const double* T, const double* V,
                                         const double* vke, int i, int q, int K) {
  if (q < 2 || q > G.L.je - 1) return zero_fl();
  const int ijn = G.L.at2(i, q - 1), ij = G.L.at2(i, q);
  const double vn = AT(vke, i, q - 1, K), vs = AT(vke, i, q, K);
  const double up = 0.5 * G.dt * thick(G.gv, G.dzw, ijn, K) * G.dlxv[ijn] * (vn + fabs(vn));
  const double um = 0.5 * G.dt * thick(G.gv, G.dzw, ij, K) * G.dlxv[ij] * (fabs(vs) - vs);
  const double t = AT(T, i, q, K), tn = AT(T, i, q - 1, K), ts = AT(T, i, q + 1, K);
  const double abl = fabs(tn - ts);
  const double zwabl = fabs(tn + ts - 2. * t);
  const double scha = fmx(0., div_nr(abl - zwabl, abl + 1.E-20)) * wet(G.gp, ij, K) *
                      wet(G.gp, G.L.at2(i, q - 1), K) * wet(G.gp, G.L.at2(i, q + 1), K);
  const double sch = fmn(1., div_nr(scha * AT(V, i, q, K), up + um + 1.E-20));
  const double schi = 1. - sch;
  Fl f;
  f.trp = up * (schi * t + sch * 0.5 * (t + tn));
  f.trm = um * (schi * t + sch * 0.5 * (t + ts));
  f.wtp = up;
  f.wtm = um;
  return f;
}


// ----------------------------------------------------------------- OCUAD ---
// vertical sweep, ocuad.f90:20-86; u-columns i in [0, IE]
__global__ void k_uad_z(Geo G, const double* __restrict__ T, const double* __restrict__ wo,
                        double* __restrict__ To, double* __restrict__ Vo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const int ij = G.L.at2(i, j);
  auto v0 = [&](int K) {
    return wet(G.gu, ij, K) * G.dlxu[ij] * G.dlyu[ij] * thick(G.gu, G.dzw, ij, K);
  };
  const bool interior = i >= 1 && i <= IE - 1 && j >= 2 && j <= JE - 1;
  if (!interior) {
    for (int K = 1; K <= KE; ++K) {
      AT(To, i, j, K) = AT(T, i, j, K);
      AT(Vo, i, j, K) = v0(K);
    }
    return;
  }
  const int ijp = G.L.at2(i, j);
  const double cdt = 0.5 * G.dt * G.dlyp[ijp] * G.dlxp[ijp];
  auto flux = [&](int K, double vol) {
    const int klo = K + 1 < KE ? K + 1 : KE;
    const int kup = K - 1 > 1 ? K - 1 : 1;
    const double wup = 0.5 * (AT(wo, i, j, K) + AT(wo, i + 1, j, K));
    const double wlo = 0.5 * (AT(wo, i, j, K + 1) + AT(wo, i + 1, j, K + 1));
    const double up = cdt * (wup + fabs(wup));
    const double um = cdt * (fabs(wlo) - wlo);
    return limited_nm(up, um, AT(T, i, j, K), AT(T, i, j, kup), AT(T, i, j, klo), vol, 1.);
  };
  Fl fm = zero_fl();
  double vk = v0(1);
  Fl fc = flux(1, vk);
  for (int K = 1; K <= KE; ++K) {
    double vn = 0.;
    Fl fp = zero_fl();
    if (K < KE) {
      vn = v0(K + 1);
      fp = flux(K + 1, vn);
    }
    const double t = AT(T, i, j, K);
    double tn = t, vv = vk;
    if (wetb(G.gu, ij, K)) apply_z(t, vk, fm, fc, fp, tn, vv);
    AT(To, i, j, K) = tn;
    AT(Vo, i, j, K) = vv;
    fm = fc;
    fc = fp;
    vk = vn;
  }
}

// x-face transports of u-cell q, ocuad.f90:99-148
__device__ __forceinline__ Fl uad_xflux(const Geo& G, const double* T, const double* V,
                                        const double* uko, int q, int j, int K) {
  const int IE = G.L.ie;
  auto ud = [&](int ii) { return AT(uko, ii, j, K) * thick(G.gu, G.dzw, G.L.at2(ii, j), K); };
  if (q >= 1 && q <= IE - 1) {
    const double uos = 0.5 * (ud(q) + ud(q + 1));
    const double uwe = 0.5 * (ud(q - 1) + ud(q));
    const double up = 0.5 * G.dt * G.dlyp[G.L.at2(q + 1, j)] * (uos + fabs(uos));
    const double um = 0.5 * G.dt * (fabs(uwe) - uwe) * G.dlyp[G.L.at2(q, j)];
    return limited_nm(up, um, AT(T, q, j, K), AT(T, q + 1, j, K), AT(T, q - 1, j, K),
                      AT(V, q, j, K), 1.);
  }
  if (q == 0) {
    const double uos = 0.5 * (ud(0) + ud(1));
    const double uwe = ud(0);
    const double up = 0.5 * G.dt * G.dlyp[G.L.at2(1, j)] * (uos + fabs(uos));
    const double um = 0.5 * G.dt * (fabs(uwe) - uwe) * G.dlyu[G.L.at2(0, j)];
    return upwind(up, um, AT(T, 0, j, K));
  }
  if (q == IE) {
    const double uos = ud(IE);
    const double uwe = 0.5 * (ud(IE - 1) + ud(IE));
    const double up = 0.5 * G.dt * G.dlyp[G.L.at2(IE, j)] * (uos + fabs(uos));
    const double um = 0.5 * G.dt * (fabs(uwe) - uwe) * G.dlyu[G.L.at2(IE, j)];
    return upwind(up, um, AT(T, IE, j, K));
  }
  return zero_fl();
}

// y-face transports of u-cell (i, q), ocuad.f90:184-233
__device__ __forceinline__ Fl uad_yflux(const Geo& G, const double* T, const double* V,
                                        const double* vke, int i, int q, int K) {
  const int JE = G.L.je;
  if (q < 1 || q > JE) return zero_fl();
  auto vd = [&](int ii, int jj) { return AT(vke, ii, jj, K) * thick(G.gv, G.dzw, G.L.at2(ii, jj), K); };
  const double vsu = 0.5 * (vd(i, q) + vd(i + 1, q));
  const double vno = 0.5 * (vd(i, q - 1) + vd(i + 1, q - 1));
  const double up = 0.5 * G.dt * (0.5 * (G.dlxv[G.L.at2(i, q - 1)] + G.dlxv[G.L.at2(i + 1, q - 1)])) *
                    (vno + fabs(vno));
  const double um = 0.5 * G.dt * (0.5 * (G.dlxv[G.L.at2(i, q)] + G.dlxv[G.L.at2(i + 1, q)])) *
                    (fabs(vsu) - vsu);
  if (q == 1 || q == JE) return upwind(up, um, AT(T, i, q, K));
  return limited_nm(up, um, AT(T, i, q, K), AT(T, i, q - 1, K), AT(T, i, q + 1, K),
                    AT(V, i, q, K), 1.);
}


// ----------------------------------------------------------------- OCVAD ---
// vertical sweep, ocvad.f90:20-86; v-columns j in [0, JE]
__global__ void k_vad_z(Geo G, const double* __restrict__ T, const double* __restrict__ wo,
                        double* __restrict__ To, double* __restrict__ Vo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const int ij = G.L.at2(i, j);
  auto v0 = [&](int K) {
    return wet(G.gv, ij, K) * G.dlxv[ij] * G.dlyv[ij] * thick(G.gv, G.dzw, ij, K);
  };
  const bool interior = i >= 2 && i <= IE - 1 && j >= 1 && j <= JE - 1;
  if (!interior) {
    for (int K = 1; K <= KE; ++K) {
      AT(To, i, j, K) = AT(T, i, j, K);
      AT(Vo, i, j, K) = v0(K);
    }
    return;
  }
  const double cdt = 0.5 * G.dt * G.dlyp[ij] * G.dlxp[ij];
  auto flux = [&](int K, double vol) {
    const int klo = K + 1 < KE ? K + 1 : KE;
    const int kup = K - 1 > 1 ? K - 1 : 1;
    const double wup = 0.5 * (AT(wo, i, j, K) + AT(wo, i, j + 1, K));
    const double wlo = 0.5 * (AT(wo, i, j, K + 1) + AT(wo, i, j + 1, K + 1));
    const double up = cdt * (wup + fabs(wup));
    const double um = cdt * (fabs(wlo) - wlo);
    return limited_nm(up, um, AT(T, i, j, K), AT(T, i, j, kup), AT(T, i, j, klo), vol, 1.);
  };
  Fl fm = zero_fl();
  double vk = v0(1);
  Fl fc = flux(1, vk);
  for (int K = 1; K <= KE; ++K) {
    double vn = 0.;
    Fl fp = zero_fl();
    if (K < KE) {
      vn = v0(K + 1);
      fp = flux(K + 1, vn);
    }
    const double t = AT(T, i, j, K);
    double tn = t, vv = vk;
    if (wetb(G.gv, ij, K)) apply_z(t, vk, fm, fc, fp, tn, vv);
    AT(To, i, j, K) = tn;
    AT(Vo, i, j, K) = vv;
    fm = fc;
    fc = fp;
    vk = vn;
  }
}

// x-face transports of v-cell (q, j), ocvad.f90:99-148
__device__ __forceinline__ Fl vad_xflux(const Geo& G, const double* T, const double* V,
                                        const double* uko, int q, int j, int K) {
  const int IE = G.L.ie;
  if (q < 1 || q > IE) return zero_fl();
  auto ud = [&](int ii, int jj) { return AT(uko, ii, jj, K) * thick(G.gu, G.dzw, G.L.at2(ii, jj), K); };
  const double uos = 0.5 * (ud(q, j) + ud(q, j + 1));
  const double uwe = 0.5 * (ud(q - 1, j) + ud(q - 1, j + 1));
  const double up = 0.5 * G.dt * (0.5 * (G.dlyu[G.L.at2(q, j)] + G.dlyu[G.L.at2(q, j + 1)])) *
                    (uos + fabs(uos));
  const double um = 0.5 * G.dt * (fabs(uwe) - uwe) *
                    (0.5 * (G.dlyu[G.L.at2(q - 1, j)] + G.dlyu[G.L.at2(q - 1, j + 1)]));
  if (q == 1 || q == IE) return upwind(up, um, AT(T, q, j, K));
  return limited_nm(up, um, AT(T, q, j, K), AT(T, q + 1, j, K), AT(T, q - 1, j, K),
                    AT(V, q, j, K), 1.);
}

// y-face transports of v-cell (i, q), ocvad.f90:184-233.  The J = 0 edge
// reads DLXU(I,0) in the reference, outside DLXU's bounds; DLXV(I,0) is used.
__device__ __forceinline__ Fl vad_yflux(const Geo& G, const double* T, const double* V,
                                        const double* vke, int i, int q, int K) {
  const int JE = G.L.je;
  auto vd = [&](int jj) { return AT(vke, i, jj, K) * thick(G.gv, G.dzw, G.L.at2(i, jj), K); };
  if (q >= 1 && q <= JE - 1) {
    const double vno = 0.5 * (vd(q) + vd(q - 1));
    const double vsu = 0.5 * (vd(q) + vd(q + 1));
    const double up = 0.5 * G.dt * G.dlxp[G.L.at2(i, q)] * (vno + fabs(vno));
    const double um = 0.5 * G.dt * G.dlxp[G.L.at2(i, q + 1)] * (fabs(vsu) - vsu);
    return limited_nm(up, um, AT(T, i, q, K), AT(T, i, q - 1, K), AT(T, i, q + 1, K),
                      AT(V, i, q, K), 1.);
  }
  if (q == 0) {
    const double vno = vd(0);
    const double vsu = 0.5 * (vd(0) + vd(1));
    const double up = 0.5 * G.dt * G.dlxv[G.L.at2(i, 0)] * (vno + fabs(vno));
    const double um = 0.5 * G.dt * G.dlxp[G.L.at2(i, 1)] * (fabs(vsu) - vsu);
    return upwind(up, um, AT(T, i, 0, K));
  }
  if (q == JE) {
    const double vno = 0.5 * (vd(JE) + vd(JE - 1));
    const double vsu = vd(JE);
    const double up = 0.5 * G.dt * G.dlxp[G.L.at2(i, JE)] * (vno + fabs(vno));
    const double um = 0.5 * G.dt * G.dlxu[G.L.at2(i, JE)] * (fabs(vsu) - vsu);
    return upwind(up, um, AT(T, i, JE, K));
  }
  return zero_fl();
}


// ----------------------------------------------------------------- OCWAD ---
// vertical sweep, ocwad.f90:14-102; w-columns, levels 1..KEP.  WETO(KEP),
// read one level past WETO in the reference (ocwad.f90:63), is taken as 0.
__global__ void k_wad_z(Geo G, const double* __restrict__ T, const double* __restrict__ wo,
                        const double* __restrict__ zo, double* __restrict__ To,
                        double* __restrict__ Vo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const int ij = G.L.at2(i, j);
  const double dlxp = G.dlxp[ij], dlyp = G.dlyp[ij];
  auto v0 = [&](int K) {
    const double a = wet(G.gp, ij, K) * dlxp * dlyp;
    if (K == 1) return a * (thick(G.gp, G.dzw, ij, 1) + zo[ij]) / 2.0;
    if (K == 2)
      return a * (thick(G.gp, G.dzw, ij, 1) + thick(G.gp, G.dzw, ij, 2) + zo[ij]) / 2.0;
    return a * (thick(G.gp, G.dzw, ij, K - 1) + thick(G.gp, G.dzw, ij, K)) / 2.0;
  };
  const bool interior = i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1;
  AT(To, i, j, KE + 1) = AT(T, i, j, KE + 1);
  AT(To, i, j, 1) = AT(T, i, j, 1);
  AT(Vo, i, j, 1) = v0(1);
  if (!interior || KE < 2) {
    for (int K = 2; K <= KE; ++K) {
      AT(To, i, j, K) = AT(T, i, j, K);
      AT(Vo, i, j, K) = v0(K);
    }
    return;
  }
  const double cdt = 0.5 * G.dt * dlyp * dlxp;
  auto flux = [&](int K, double vol) {
    const double wup = 0.5 * (AT(wo, i, j, K) + AT(wo, i, j, K - 1));
    const double wum = 0.5 * (AT(wo, i, j, K) + AT(wo, i, j, K + 1));
    const double up = cdt * (wup + fabs(wup));
    const double um = cdt * (fabs(wum) - wum);
    const double cap = K + 1 <= KE ? wet(G.gp, ij, K + 1) : 0.0;
    return limited_nm(up, um, AT(T, i, j, K), AT(T, i, j, K - 1), AT(T, i, j, K + 1), vol, cap);
  };
  // edge transports, ocwad.f90:72-83
  Fl fm;  // level 1: only TRM/WTM used
  {
    const double wum = 0.5 * (AT(wo, i, j, 1) + AT(wo, i, j, 2));
    const double um = cdt * (fabs(wum) - wum);
    fm = Fl{0., um * (0.5 * (AT(T, i, j, 1) + AT(T, i, j, 2))), 0., um};
  }
  Fl fkep;
  {
    const double wup = 0.5 * (AT(wo, i, j, KE + 1) + AT(wo, i, j, KE));
    const double up = cdt * (wup + fabs(wup));
    fkep = Fl{up * (0.5 * (AT(T, i, j, KE) + AT(T, i, j, KE + 1))), 0., up, 0.};
  }
  double vk = v0(2);
  Fl fc = flux(2, vk);
  for (int K = 2; K <= KE; ++K) {
    double vn = 0.;
    Fl fp = fkep;
    if (K < KE) {
      vn = v0(K + 1);
      fp = flux(K + 1, vn);
    }
    const double t = AT(T, i, j, K);
    double tn = t, vv = vk;
    if (wetb(G.gp, ij, K)) apply_z(t, vk, fm, fc, fp, tn, vv);
    AT(To, i, j, K) = tn;
    AT(Vo, i, j, K) = vv;
    fm = fc;
    fc = fp;
    vk = vn;
  }
}

__device__ __forceinline__ Fl wad_xflux(const Geo& G, const double* T, const double* V,
                                        const double* uko, int q, int j, int K) {
  if (q < 2 || q > G.L.ie - 1) return zero_fl();
  auto ud = [&](int ii, int KK) { return AT(uko, ii, j, KK) * thick(G.gu, G.dzw, G.L.at2(ii, j), KK); };
  const double uos = 0.5 * (ud(q, K) + ud(q, K - 1));
  const double uwe = 0.5 * (ud(q - 1, K) + ud(q - 1, K - 1));
  const double up = 0.5 * G.dt * G.dlyu[G.L.at2(q, j)] * (uos + fabs(uos));
  const double um = 0.5 * G.dt * G.dlyu[G.L.at2(q - 1, j)] * (fabs(uwe) - uwe);
  const double t = AT(T, q, j, K), te = AT(T, q + 1, j, K), tw = AT(T, q - 1, j, K);
  const double abl = fabs(te - tw);
  const double zwabl = fabs(te + tw - 2. * t);
  const double scha = fmx(0., div_nr(abl - zwabl, abl + 1.E-20)) * wet(G.gp, G.L.at2(q, j), K) *
                      wet(G.gp, G.L.at2(q + 1, j), K) * wet(G.gp, G.L.at2(q - 1, j), K);
  const double sch = fmn(1., div_nr(scha * AT(V, q, j, K), up + um + 1.E-20));
  const double schi = 1. - sch;
  return Fl{up * (schi * t + sch * 0.5 * (t + te)), um * (schi * t + sch * 0.5 * (t + tw)), up, um};
}

__device__ __forceinline__ Fl wad_yflux(const Geo& G, const double* T, const double* V,
                                        const double* vke, int i, int q, int K) {
  if (q < 2 || q > G.L.je - 1) return zero_fl();
  auto vd = [&](int jj, int KK) { return AT(vke, i, jj, KK) * thick(G.gv, G.dzw, G.L.at2(i, jj), KK); };
  const double vsu = 0.5 * (vd(q, K) + vd(q, K - 1));
  const double vno = 0.5 * (vd(q - 1, K) + vd(q - 1, K - 1));
  const double up = 0.5 * G.dt * G.dlxv[G.L.at2(i, q - 1)] * (vno + fabs(vno));
  const double um = 0.5 * G.dt * G.dlxv[G.L.at2(i, q)] * (fabs(vsu) - vsu);
  const double t = AT(T, i, q, K), tn = AT(T, i, q - 1, K), ts = AT(T, i, q + 1, K);
  const double abl = fabs(tn - ts);
  const double zwabl = fabs(tn + ts - 2. * t);
  const double scha = fmx(0., div_nr(abl - zwabl, abl + 1.E-20)) * wet(G.gp, G.L.at2(i, q), K) *
                      wet(G.gp, G.L.at2(i, q - 1), K) * wet(G.gp, G.L.at2(i, q + 1), K);
  const double sch = fmn(1., div_nr(scha * AT(V, i, q, K), up + um + 1.E-20));
  const double schi = 1. - sch;
  return Fl{up * (schi * t + sch * 0.5 * (t + tn)), um * (schi * t + sch * 0.5 * (t + ts)), up, um};
}



// ---------------------------------------------------- horizontal sweeps ---
// One kernel per (routine, direction).  A block of one level first computes,
// one thread per position, the face transports of every position its cells
// need (its own cells plus one halo position on each side along the sweep)
// into shared memory; then each cell applies RN / T' from its neighbours'
// entries (block shapes in Sweep below).
enum { V_ADPO = 0, V_UAD = 1, V_VAD = 2, V_WAD = 3 };

template <int VAR> struct Rng;
template <> struct Rng<V_ADPO> { static constexpr int i0 = 1, j0 = 1, iL = 2, jL = 2, iH = 1, jH = 1, kL = 1; };
template <> struct Rng<V_UAD>  { static constexpr int i0 = 0, j0 = 1, iL = 1, jL = 2, iH = 1, jH = 1, kL = 1; };
template <> struct Rng<V_VAD>  { static constexpr int i0 = 1, j0 = 0, iL = 2, jL = 1, iH = 1, jH = 1, kL = 1; };
template <> struct Rng<V_WAD>  { static constexpr int i0 = 1, j0 = 1, iL = 2, jL = 2, iH = 1, jH = 1, kL = 2; };
// (iH, jH: the update range ends at IE - iH, JE - jH)

template <int VAR, int DIR>
__device__ __forceinline__ Fl face(const Geo& G, const double* T, const double* V,
                                   const double* vel, int qi, int qj, int K) {
  if (VAR == V_ADPO) return DIR == 0 ? adpo_xflux(G, T, V, vel, qi, qj, K) : adpo_yflux(G, T, V, vel, qi, qj, K);
  if (VAR == V_UAD) return DIR == 0 ? uad_xflux(G, T, V, vel, qi, qj, K) : uad_yflux(G, T, V, vel, qi, qj, K);
  if (VAR == V_VAD) return DIR == 0 ? vad_xflux(G, T, V, vel, qi, qj, K) : vad_yflux(G, T, V, vel, qi, qj, K);
  return DIR == 0 ? wad_xflux(G, T, V, vel, qi, qj, K) : wad_yflux(G, T, V, vel, qi, qj, K);
}

template <int VAR>
__device__ __forceinline__ bool wet_var(const Geo& G, int ij, int K) {
  if (VAR == V_UAD) return wetb(G.gu, ij, K);
  if (VAR == V_VAD) return wetb(G.gv, ij, K);
  return wetb(G.gp, ij, K);
}

constexpr int kSx = 32, kSy = 8;

// Block shape of a sweep: one thread per face position, so the face phase
// is a single pass.  x sweeps: (kSx + 2) x kSy threads hold the faces of
// kSx + 2 columns and update the kSx cells between them; y sweeps: kSx x kSy
// threads hold kSy rows of faces and update the kSy - 2 rows between them.
template <int DIR>
struct Sweep {
  static constexpr int BX = DIR == 0 ? kSx + 2 : kSx, BY = kSy;  // threads = faces
  static constexpr int CX = kSx, CY = DIR == 0 ? kSy : kSy - 2;  // cells
};

template <int DIR>
inline dim3 sweep_block() {
  return dim3(Sweep<DIR>::BX, Sweep<DIR>::BY);
}
template <int DIR>
inline dim3 sweep_grid(int nx, int ny, int nz) {
  using S = Sweep<DIR>;
  return dim3((nx + S::CX - 1) / S::CX, (ny + S::CY - 1) / S::CY, nz);
}

template <int VAR, int DIR>
__global__ void __launch_bounds__(Sweep<DIR>::BX * Sweep<DIR>::BY)
    k_hsweep(Geo G, const double* __restrict__ T, const double* __restrict__ V,
             const double* __restrict__ vel, double* __restrict__ To, double* __restrict__ Vo) {
  using R = Rng<VAR>;
  using S = Sweep<DIR>;
  __shared__ Fl fl[S::BY][S::BX];
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  const int K = blockIdx.z + 1;
  const int ib = blockIdx.x * S::CX + R::i0, jb = blockIdx.y * S::CY + R::j0;
  const int iLo = R::iL, iHi = IE - R::iH, jLo = R::jL, jHi = JE - R::jH;
  const bool klev = K >= R::kL && K <= KE;
  const int hx = threadIdx.x, hy = threadIdx.y;
  if (klev) {
    const int qi = ib + hx - (DIR == 0), qj = jb + hy - (DIR == 1);
    // only positions a cell in the update range reads
    const bool need = DIR == 0 ? (qj >= jLo && qj <= jHi) : (qi >= iLo && qi <= iHi);
    fl[hy][hx] = need ? face<VAR, DIR>(G, T, V, vel, qi, qj, K) : zero_fl();
  }
  __syncthreads();
  const int ci = hx - (DIR == 0), cj = hy - (DIR == 1);  // the thread's cell in the tile
  if (ci < 0 || ci >= S::CX || cj < 0 || cj >= S::CY) return;
  const int i = ib + ci, j = jb + cj;
  const int iMax = VAR == V_UAD ? IE : IE, jMax = JE;
  if (i > iMax || j > jMax) return;
  const double t = AT(T, i, j, K);
  double tn = t;
  const bool hasv = K <= KE;
  double v = hasv ? AT(V, i, j, K) : 0.0, vn = v;
  if (klev && i >= iLo && i <= iHi && j >= jLo && j <= jHi && wet_var<VAR>(G, G.L.at2(i, j), K)) {
    if (DIR == 0)  // RN = V + WTP(I-1) - WTP(I) - WTM(I) + WTM(I+1)
      apply(t, v, fl[hy][hx - 1], fl[hy][hx], fl[hy][hx + 1], tn, vn);
    else           // RN = V + WTP(J+1) - WTP(J) - WTM(J) + WTM(J-1)
      apply(t, v, fl[hy + 1][hx], fl[hy][hx], fl[hy - 1][hx], tn, vn);
  }
  AT(To, i, j, K) = tn;
  if (Vo && hasv) AT(Vo, i, j, K) = vn;
}

// ---------------------------------------------------- OCADPO, all tracers ---
// The driver calls OCADPO once per tracer with unchanged velocities
// (orctm.f90:1459-1460 and the passive tracers after them).  The transports
// WTP/WTM, the volumes RN and the geometry factors depend on the velocities
// and the geometry only, so these sweeps form them once and advect up to
// kMaxFused tracers with them.  Each tracer's arithmetic is, expression for
// expression, that of k_adpo_z, adpo_xflux / adpo_yflux and apply, so the
// results equal separate OCADPO calls bit for bit.
constexpr int kMaxFused = 4;

struct TrIO {
  const double* in[kMaxFused];
  double* out[kMaxFused];
};

template <int NT>
struct FlN {
  double wtp, wtm;
  double trp[NT], trm[NT];
};

template <int NT>
__device__ __forceinline__ FlN<NT> zero_fln() {
  FlN<NT> f;
  f.wtp = f.wtm = 0.;
#pragma unroll
  for (int n = 0; n < NT; ++n) f.trp[n] = f.trm[n] = 0.;
  return f;
}

template <int NT>
__device__ __forceinline__ Fl pick(const FlN<NT>& f, int n) {
  return Fl{f.trp[n], f.trm[n], f.wtp, f.wtm};
}

template <int NT>
__global__ void k_adpo_z_all(Geo G, TrIO io, const double* __restrict__ wo,
                             const double* __restrict__ zo, double* __restrict__ Vo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const int ij = G.L.at2(i, j);
  const double dlxp = G.dlxp[ij], dlyp = G.dlyp[ij];
  auto v0 = [&](int K) {
    double s = wet(G.gp, ij, K) * dlxp * dlyp * thick(G.gp, G.dzw, ij, K);
    if (K == 1) s = s + dlxp * dlyp * wet(G.gp, ij, 1) * (zo[ij] - AT(wo, i, j, 1) * G.dt);
    return s;
  };
  const bool interior = i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1;
  if (!interior) {
    for (int K = 1; K <= KE; ++K) {
#pragma unroll
      for (int n = 0; n < NT; ++n) AT(io.out[n], i, j, K) = AT(io.in[n], i, j, K);
      AT(Vo, i, j, K) = v0(K);
    }
    return;
  }
  const double cdt = 0.5 * G.dt * dlyp * dlxp;
  auto flux = [&](int K, double vol) {
    const int klo = K + 1 < KE ? K + 1 : KE;
    const int kup = K - 1 > 1 ? K - 1 : 1;
    const double w0 = AT(wo, i, j, K), w1 = AT(wo, i, j, K + 1);
    const double up = cdt * (w0 + fabs(w0));
    const double um = cdt * (fabs(w1) - w1);
    const double cap = wet(G.gp, ij, klo);
    FlN<NT> f;
    f.wtp = up;
    f.wtm = um;
#pragma unroll
    for (int n = 0; n < NT; ++n) {
      const double* T = io.in[n];
      const double t = AT(T, i, j, K), tu = AT(T, i, j, kup), tl = AT(T, i, j, klo);
      const double abl = fabs(tu - tl);
      const double zwabl = fabs(tu + tl - 2. * t);
      const double scha = fmx(0., div_nr(abl - zwabl, abl + 1.E-20));
      double sch = fmn(cap, div_nr(scha * vol, up + um + 1.E-20));
      if (K == 1 || K == KE) sch = 0.;
      const double schi = 1. - sch;
      f.trp[n] = up * (schi * t + sch * 0.5 * (t + tu));
      f.trm[n] = um * (schi * t + sch * 0.5 * (t + tl));
    }
    return f;
  };
  FlN<NT> fm = zero_fln<NT>();
  double vk = v0(1);
  FlN<NT> fc = flux(1, vk);
  for (int K = 1; K <= KE; ++K) {
    double vn = 0.;
    FlN<NT> fp = zero_fln<NT>();
    if (K < KE) {
      vn = v0(K + 1);
      fp = flux(K + 1, vn);
    }
    const bool w = wetb(G.gp, ij, K);
    double vv = vk;
#pragma unroll
    for (int n = 0; n < NT; ++n) {
      const double t = AT(io.in[n], i, j, K);
      double tn = t, vt = vk;
      if (w) apply_z(t, vk, pick(fm, n), pick(fc, n), pick(fp, n), tn, vt);
      AT(io.out[n], i, j, K) = tn;
      vv = vt;
    }
    AT(Vo, i, j, K) = vv;
    fm = fc;
    fc = fp;
    vk = vn;
  }
}

// the face transports of adpo_xflux (DIR 0) / adpo_yflux (DIR 1) for NT tracers
template <int NT, int DIR>
__device__ __forceinline__ FlN<NT> adpo_face_all(const Geo& G, const TrIO& io,
                                                 const double* V, const double* vel, int qi,
                                                 int qj, int K) {
  const int q = DIR == 0 ? qi : qj;
  const int qmax = DIR == 0 ? G.L.ie - 1 : G.L.je - 1;
  if (q < 2 || q > qmax) return zero_fln<NT>();
  const int i = qi, j = qj;
  double up, um;
  int ij, ijp, ijm;  // the cell, its neighbour in +DIR and in -DIR
  if (DIR == 0) {
    const double u0 = AT(vel, q, j, K), um1 = AT(vel, q - 1, j, K);
    ij = G.L.at2(q, j);
    ijm = G.L.at2(q - 1, j);
    ijp = G.L.at2(q + 1, j);
    up = 0.5 * G.dt * thick(G.gu, G.dzw, ij, K) * G.dlyu[ij] * (u0 + fabs(u0));
    um = 0.5 * G.dt * thick(G.gu, G.dzw, ijm, K) * (fabs(um1) - um1) * G.dlyu[ijm];
  } else {
    const int ijn = G.L.at2(i, q - 1);
    ij = G.L.at2(i, q);
    const double vn = AT(vel, i, q - 1, K), vs = AT(vel, i, q, K);
    up = 0.5 * G.dt * thick(G.gv, G.dzw, ijn, K) * G.dlxv[ijn] * (vn + fabs(vn));
    um = 0.5 * G.dt * thick(G.gv, G.dzw, ij, K) * G.dlxv[ij] * (fabs(vs) - vs);
    ijp = G.L.at2(i, q - 1);  // factor order of adpo_yflux: WETO(J), WETO(J-1), WETO(J+1)
    ijm = G.L.at2(i, q + 1);
  }
  const double w1 = wet(G.gp, ij, K), w2 = wet(G.gp, ijp, K), w3 = wet(G.gp, ijm, K);
  const double vol = AT(V, i, j, K);
  FlN<NT> f;
  f.wtp = up;
  f.wtm = um;
#pragma unroll
  for (int n = 0; n < NT; ++n) {
    const double* T = io.in[n];
    // x: t, east, west (TRP uses the east value); y: t, north (q-1), south (q+1)
    const double t = AT(T, i, j, K);
    const double ta = DIR == 0 ? AT(T, q + 1, j, K) : AT(T, i, q - 1, K);
    const double tb = DIR == 0 ? AT(T, q - 1, j, K) : AT(T, i, q + 1, K);
    const double abl = fabs(ta - tb);
    const double zwabl = fabs(ta + tb - 2. * t);
    const double scha = fmx(0., div_nr(abl - zwabl, abl + 1.E-20)) * w1 * w2 * w3;
    const double sch = fmn(1., div_nr(scha * vol, up + um + 1.E-20));
    const double schi = 1. - sch;
    f.trp[n] = up * (schi * t + sch * 0.5 * (t + ta));
    f.trm[n] = um * (schi * t + sch * 0.5 * (t + tb));
  }
  return f;
}

template <int NT, int DIR>
__global__ void __launch_bounds__(Sweep<DIR>::BX * Sweep<DIR>::BY)
    k_hsweep_adpo_all(Geo G, TrIO io, const double* __restrict__ V,
                      const double* __restrict__ vel, double* __restrict__ Vo) {
  using R = Rng<V_ADPO>;
  using S = Sweep<DIR>;
  __shared__ FlN<NT> fl[S::BY][S::BX];
  const int IE = G.L.ie, JE = G.L.je;
  const int K = blockIdx.z + 1;
  const int ib = blockIdx.x * S::CX + R::i0, jb = blockIdx.y * S::CY + R::j0;
  const int iLo = R::iL, iHi = IE - R::iH, jLo = R::jL, jHi = JE - R::jH;
  const int hx = threadIdx.x, hy = threadIdx.y;
  {
    const int qi = ib + hx - (DIR == 0), qj = jb + hy - (DIR == 1);
    const bool need = DIR == 0 ? (qj >= jLo && qj <= jHi) : (qi >= iLo && qi <= iHi);
    fl[hy][hx] = need ? adpo_face_all<NT, DIR>(G, io, V, vel, qi, qj, K) : zero_fln<NT>();
  }
  __syncthreads();
  const int ci = hx - (DIR == 0), cj = hy - (DIR == 1);  // the thread's cell in the tile
  if (ci < 0 || ci >= S::CX || cj < 0 || cj >= S::CY) return;
  const int i = ib + ci, j = jb + cj;
  if (i > IE || j > JE) return;
  const double v = AT(V, i, j, K);
  double vn = v;
  const bool upd = i >= iLo && i <= iHi && j >= jLo && j <= jHi && wetb(G.gp, G.L.at2(i, j), K);
#pragma unroll
  for (int n = 0; n < NT; ++n) {
    const double t = AT(io.in[n], i, j, K);
    double tn = t, vt = v;
    if (upd) {
      if (DIR == 0)  // RN = V + WTP(I-1) - WTP(I) - WTM(I) + WTM(I+1)
        apply(t, v, pick(fl[hy][hx - 1], n), pick(fl[hy][hx], n), pick(fl[hy][hx + 1], n), tn, vt);
      else           // RN = V + WTP(J+1) - WTP(J) - WTM(J) + WTM(J-1)
        apply(t, v, pick(fl[hy + 1][hx], n), pick(fl[hy][hx], n), pick(fl[hy - 1][hx], n), tn, vt);
    }
    AT(io.out[n], i, j, K) = tn;
    vn = vt;
  }
  if (Vo) AT(Vo, i, j, K) = vn;
}

inline dim3 grid2(int nx, int ny, dim3 b) { return dim3((nx + b.x - 1) / b.x, (ny + b.y - 1) / b.y, 1); }

}  // namespace

// T -> out through the z, x and y sweeps; tA, vA, vB: scratch fields
void launch_ocadpo(const Geo& G, const double* T, const double* uko, const double* vke,
                   const double* wo, const double* zo, double* out, double* tA, double* vA,
                   double* vB, cudaStream_t st) {
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  const dim3 bc(32, 4);
  k_adpo_z<<<grid2(IE, JE, bc), bc, 0, st>>>(G, T, wo, zo, out, vA);
  count_launch();
  k_hsweep<V_ADPO, 0><<<sweep_grid<0>(IE, JE, KE), sweep_block<0>(), 0, st>>>(G, out, vA, uko, tA, vB);
  count_launch();
  k_hsweep<V_ADPO, 1><<<sweep_grid<1>(IE, JE, KE), sweep_block<1>(), 0, st>>>(G, tA, vB, vke, out, nullptr);
  count_launch();
}

namespace {
template <int NT>
void adpo_all_group(const Geo& G, TrIO zio, TrIO xio, TrIO yio, const double* uko,
                    const double* vke, const double* wo, const double* zo, double* vA, double* vB,
                    cudaStream_t st) {
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  const dim3 bc(32, 4);
  k_adpo_z_all<NT><<<grid2(IE, JE, bc), bc, 0, st>>>(G, zio, wo, zo, vA);
  count_launch();
  k_hsweep_adpo_all<NT, 0><<<sweep_grid<0>(IE, JE, KE), sweep_block<0>(), 0, st>>>(G, xio, vA, uko, vB);
  count_launch();
  k_hsweep_adpo_all<NT, 1><<<sweep_grid<1>(IE, JE, KE), sweep_block<1>(), 0, st>>>(G, yio, vB, vke, nullptr);
  count_launch();
}
}  // namespace

int adpo_max_fused() { return kMaxFused; }

// ntr tracers T[n] -> out[n] through the z, x and y sweeps, kMaxFused at a
// time; mid[n]: the x-sweep outputs; vA, vB: scratch volumes
void launch_ocadpo_all(const Geo& G, int ntr, const double* const* T, double* const* out,
                       double* const* mid, const double* uko, const double* vke,
                       const double* wo, const double* zo, double* vA, double* vB,
                       cudaStream_t st) {
  for (int n0 = 0; n0 < ntr; n0 += kMaxFused) {
    const int nt = ntr - n0 < kMaxFused ? ntr - n0 : kMaxFused;
    TrIO zio{}, xio{}, yio{};
    for (int n = 0; n < nt; ++n) {
      zio.in[n] = T[n0 + n];
      zio.out[n] = out[n0 + n];
      xio.in[n] = out[n0 + n];
      xio.out[n] = mid[n0 + n];
      yio.in[n] = mid[n0 + n];
      yio.out[n] = out[n0 + n];
    }
    switch (nt) {
      case 1: adpo_all_group<1>(G, zio, xio, yio, uko, vke, wo, zo, vA, vB, st); break;
      case 2: adpo_all_group<2>(G, zio, xio, yio, uko, vke, wo, zo, vA, vB, st); break;
      case 3: adpo_all_group<3>(G, zio, xio, yio, uko, vke, wo, zo, vA, vB, st); break;
      default: adpo_all_group<4>(G, zio, xio, yio, uko, vke, wo, zo, vA, vB, st); break;
    }
  }
}

void launch_ocuad(const Geo& G, const double* T, const double* uko, const double* vke,
                  const double* wo, double* out, double* tA, double* vA, double* vB,
                  cudaStream_t st) {
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  const dim3 b(32, 4);
  k_uad_z<<<grid2(IE + 1, JE, b), b, 0, st>>>(G, T, wo, out, vA);
  count_launch();
  k_hsweep<V_UAD, 0><<<sweep_grid<0>(IE + 1, JE, KE), sweep_block<0>(), 0, st>>>(G, out, vA, uko, tA, vB);
  count_launch();
  k_hsweep<V_UAD, 1><<<sweep_grid<1>(IE + 1, JE, KE), sweep_block<1>(), 0, st>>>(G, tA, vB, vke, out, nullptr);
  count_launch();
}

void launch_ocvad(const Geo& G, const double* T, const double* uko, const double* vke,
                  const double* wo, double* out, double* tA, double* vA, double* vB,
                  cudaStream_t st) {
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  const dim3 b(32, 4);
  k_vad_z<<<grid2(IE, JE + 1, b), b, 0, st>>>(G, T, wo, out, vA);
  count_launch();
  k_hsweep<V_VAD, 0><<<sweep_grid<0>(IE, JE + 1, KE), sweep_block<0>(), 0, st>>>(G, out, vA, uko, tA, vB);
  count_launch();
  k_hsweep<V_VAD, 1><<<sweep_grid<1>(IE, JE + 1, KE), sweep_block<1>(), 0, st>>>(G, tA, vB, vke, out, nullptr);
  count_launch();
}

void launch_ocwad(const Geo& G, const double* T, const double* uko, const double* vke,
                  const double* wo, const double* zo, double* out, double* tA, double* vA,
                  double* vB, cudaStream_t st) {
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  const dim3 b(32, 4);
  k_wad_z<<<grid2(IE, JE, b), b, 0, st>>>(G, T, wo, zo, out, vA);
  count_launch();
  k_hsweep<V_WAD, 0><<<sweep_grid<0>(IE, JE, KE + 1), sweep_block<0>(), 0, st>>>(G, out, vA, uko, tA, vB);
  count_launch();
  k_hsweep<V_WAD, 1><<<sweep_grid<1>(IE, JE, KE + 1), sweep_block<1>(), 0, st>>>(G, tA, vB, vke, out, nullptr);
  count_launch();
}

}  // namespace orctm
