// Tracer diffusion (OCTDIFF_BASE + OCTDIFF_TS: octdiff_base.f90:182-221,
// octdiff_ts.f90:51-59, 294-407) and momentum diffusion with quadratic
// bottom drag (OCVISC, FREESLIP branch: ocvisc.f90:37-478, 615-688).
//
// Implicit vertical diffusion is one Thomas solve per water column, one
// thread per column.  The tracers' horizontal biharmonic operator is one
// fused pass (the first Laplacian formed per level in shared memory, never
// stored); the momentum one is two passes (a Laplacian into a scratch field,
// then the flux-form update).  Arithmetic follows the reference's operation order in IEEE binary64,
// with two changes that stay within a few ulp: the stencils multiply by
// reciprocal metrics and per-face coefficients computed once at set-up
// instead of dividing by the metrics, and the remaining divisions (by
// thicknesses and Thomas pivots) use div_nr (within 1 ulp of IEEE division).
#include "common.cuh"
#include "ops.h"

namespace orctm {

namespace {

#define AT(a, i, j, K) (a)[G.L.at((i), (j), (K)-1)]

inline dim3 grid2(int nx, int ny, dim3 b) { return dim3((nx + b.x - 1) / b.x, (ny + b.y - 1) / b.y, 1); }

// ------------------------------------------------------------- OCTDIFF ----
// Implicit vertical diffusion of ntr tracers (TRIDSY built once per column).
// Columns outside i in [2,IE1], j in [2,JE1] are copied unchanged.
struct TrPtrs {
  const double* in[8];
  double* out[8];
};

// The eliminated diagonals of a column solve are kept per thread (local
// memory, cached in L1/L2).  Keeping them in shared memory instead was
// measured 2.1-2.5x slower on c3: 640 B per column limits a B200 SM to about
// 350 resident columns, too few to hide the solves' memory latency.
constexpr int kVertBlock = 64;

__global__ void __launch_bounds__(kVertBlock) k_tdiff_vert(Geo G, TrPtrs tp, int ntr,
                                                           const double* __restrict__ dvo,
                                                           const double* __restrict__ zo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const bool interior = i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1;
  if (!interior) {
    for (int n = 0; n < ntr; ++n)
      for (int K = 1; K <= KE; ++K) AT(tp.out[n], i, j, K) = AT(tp.in[n], i, j, K);
    return;
  }
  const int ij = G.L.at2(i, j);
  const double zij = zo[ij];
  // TRIDSY(K,1..3) of octdiff_base.f90:188-194; only the eliminated diagonal
  // is kept per level, TRIDSY(K,3) is recomputed by the same expression
  auto den = [&](int K) {
    const double zzsurf = K == 1 ? 1. : 0.;
    return thick(G.gp, G.dzw, ij, K) + zzsurf * (zij) + G.almzer;
  };
  auto tri3 = [&](int K, double dn) { return div_nr(-G.dt * AT(dvo, i, j, K + 1) * G.di[K], dn); };
  double t2p[kMaxKe];
  double ylast[8];
  double t2prev = 1.0, t3prev = 0.0;
  for (int K = 1; K <= KE; ++K) {
    const double dn = den(K);
    const double t1 = div_nr(-G.dt * AT(dvo, i, j, K) * wet(G.gp, ij, K) * G.di[K - 1], dn);
    const double t3 = tri3(K, dn);
    double t2 = 1. - t1 - t3;
    double m = 0.0;
    if (K >= 2) {
      m = div_nr(t1, t2prev);                       // TRIDSY(K-1,1) after elimination
      t2 = t2 - div_nr(t3prev * t1, t2prev);        // TRIDSY(K,2) after elimination
    }
    t2p[K - 1] = t2;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      if (n >= ntr) break;
      const double tk = AT(tp.in[n], i, j, K);
      const double y = K == 1 ? tk : tk - m * ylast[n];  // T1O(K)
      AT(tp.out[n], i, j, K) = y;
      ylast[n] = y;
    }
    t2prev = t2;
    t3prev = t3;
  }
  double nxt[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    if (n >= ntr) break;
    nxt[n] = div_nr(AT(tp.out[n], i, j, KE), t2p[KE - 1]);
    AT(tp.out[n], i, j, KE) = nxt[n];
  }
  for (int l = KE - 1; l >= 1; --l) {
    const double t3 = tri3(l, den(l));
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      if (n >= ntr) break;
      nxt[n] = div_nr(AT(tp.out[n], i, j, l) - t3 * nxt[n], t2p[l - 1]);
      AT(tp.out[n], i, j, l) = nxt[n];
    }
  }
}

// The same solve with the tracer count known at compile time and the loads
// of U levels issued together before they are used: the input and output
// arrays may alias as far as the compiler knows, so the one-level form above
// waits a full memory latency per level in each sweep.  Every value is
// formed by the same expressions in the same order, so the results equal
// k_tdiff_vert's bit for bit.
template <int NTR, int U>
__global__ void __launch_bounds__(kVertBlock) k_tdiff_vert_b(Geo G, TrPtrs tp,
                                                             const double* __restrict__ dvo,
                                                             const double* __restrict__ zo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const int pl = G.L.plane;
  const int base = G.L.at(i, j, 0);
  const bool interior = i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1;
  if (!interior) {
    for (int K0 = 1; K0 <= KE; K0 += U) {
      double v[NTR][U];
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int n = 0; n < NTR; ++n)
          v[n][u] = K0 + u <= KE ? tp.in[n][base + (K0 + u - 1) * pl] : 0.0;
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int n = 0; n < NTR; ++n)
          if (K0 + u <= KE) tp.out[n][base + (K0 + u - 1) * pl] = v[n][u];
    }
    return;
  }
  const int ij = G.L.at2(i, j);
  const double zij = zo[ij];
  auto den = [&](int K) {
    const double zzsurf = K == 1 ? 1. : 0.;
    return thick(G.gp, G.dzw, ij, K) + zzsurf * (zij) + G.almzer;
  };
  double t2p[kMaxKe];
  double ylast[NTR];
  double t2prev = 1.0, t3prev = 0.0;
  // forward elimination, U levels per batch: DVO(K..K+U) and the tracers of
  // K..K+U-1 are loaded first
  for (int K0 = 1; K0 <= KE; K0 += U) {
    double lt[NTR][U], ld[U + 1];
#pragma unroll
    for (int u = 0; u <= U; ++u) ld[u] = K0 + u <= KE + 1 ? dvo[base + (K0 + u - 1) * pl] : 0.0;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int n = 0; n < NTR; ++n)
        lt[n][u] = K0 + u <= KE ? tp.in[n][base + (K0 + u - 1) * pl] : 0.0;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int K = K0 + u;
      if (K > KE) break;
      const double dn = den(K);
      const double t1 = div_nr(-G.dt * ld[u] * wet(G.gp, ij, K) * G.di[K - 1], dn);
      const double t3 = div_nr(-G.dt * ld[u + 1] * G.di[K], dn);
      double t2 = 1. - t1 - t3;
      double m = 0.0;
      if (K >= 2) {
        m = div_nr(t1, t2prev);
        t2 = t2 - div_nr(t3prev * t1, t2prev);
      }
      t2p[K - 1] = t2;
#pragma unroll
      for (int n = 0; n < NTR; ++n) {
        const double tk = lt[n][u];
        const double y = K == 1 ? tk : tk - m * ylast[n];
        tp.out[n][base + (K - 1) * pl] = y;
        ylast[n] = y;
      }
      t2prev = t2;
      t3prev = t3;
    }
  }
  // back substitution, U levels per batch: the forward values and DVO of
  // l-U+1..l loaded first
  double nxt[NTR];
#pragma unroll
  for (int n = 0; n < NTR; ++n) {
    nxt[n] = div_nr(ylast[n], t2p[KE - 1]);
    tp.out[n][base + (KE - 1) * pl] = nxt[n];
  }
  for (int l0 = KE - 1; l0 >= 1; l0 -= U) {
    double ly[NTR][U], ld[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int l = l0 - u;
      ld[u] = l >= 1 ? dvo[base + l * pl] : 0.0;  // DVO(l+1)
#pragma unroll
      for (int n = 0; n < NTR; ++n) ly[n][u] = l >= 1 ? tp.out[n][base + (l - 1) * pl] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int l = l0 - u;
      if (l < 1) break;
      const double t3 = div_nr(-G.dt * ld[u] * G.di[l], den(l));
#pragma unroll
      for (int n = 0; n < NTR; ++n) {
        nxt[n] = div_nr(ly[n][u] - t3 * nxt[n], t2p[l - 1]);
        tp.out[n][base + (l - 1) * pl] = nxt[n];
      }
    }
  }
}

// Laplacian and biharmonic update fused (octdiff_ts.f90:342-399), all
// tracers in one launch.  A block of 32 x 8 cells marches down the levels;
// per level it stages the 36 x 12 tile of the vertically diffused tracer in
// shared memory, forms the masked Laplacian T1O on the 34 x 10 positions its
// cells need, and applies the biharmonic update, so the Laplacian never goes
// to HBM.  The geometry a thread needs (wet-level counts, reciprocal metrics,
// face terms) is loaded once for all levels and tracers, and the loads of the
// next level are issued before the current one is computed.  The Laplacian
// (0 outside the interior) and the biharmonic factor W / ((DDPO + ALMZER +
// ZZSURF ZO) DLXP DLYP) DZW use 1/(DLXP DLYP), reciprocal metrics and the
// face terms AULX DLYU / DLXU and AULY DLXV / DLYV precomputed, multiplied in
// the reference's order.  The blocks cover i in [1, IE], j in [1, JE]: cells
// outside the interior are copied.  (Measured on c3: one launch per level,
// reloading the geometry each time, was 2.1x slower than this form.)
constexpr int kHbX = 32, kHbY = 8;
constexpr int kHbTx = kHbX + 4, kHbTy = kHbY + 4;   // tracer tile
constexpr int kHbLx = kHbX + 2, kHbLy = kHbY + 2;   // Laplacian tile
constexpr int kHbT = kHbTx * kHbTy, kHbL = kHbLx * kHbLy, kHbN = kHbX * kHbY;
constexpr int kHbTf = (kHbT + kHbN - 1) / kHbN, kHbLf = (kHbL + kHbN - 1) / kHbN;

__global__ void __launch_bounds__(kHbN) k_tdiff_hbih(Geo G, TrPtrs tp, int ntr,
                                                     const double* __restrict__ zo) {
  __shared__ double ts[kHbT];
  __shared__ double ls[kHbL];
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kHbX * ty;
  const int i0 = blockIdx.x * kHbX + 1, j0 = blockIdx.y * kHbY + 1;
  const int plane = G.L.plane;
  // tracer-tile entries this thread loads (element (i0-2+hx, j0-2+hy));
  // entries outside the field's plane [0, IE] x [0, JE] are not loaded and
  // hold 0 (no Laplacian or update that is formed reads them)
  int toff[kHbTf];
  bool tval[kHbTf], tin[kHbTf];
#pragma unroll
  for (int f = 0; f < kHbTf; ++f) {
    const int e = tid + f * kHbN;
    const int hy = e / kHbTx, hx = e - hy * kHbTx;
    const int ii = i0 - 2 + hx, jj = j0 - 2 + hy;
    tval[f] = e < kHbT;
    tin[f] = tval[f] && ii >= 0 && ii <= IE && jj >= 0 && jj <= JE;
    toff[f] = tin[f] ? G.L.at2(ii, jj) : 0;
  }
  // Laplacian positions this thread forms, with their level-independent data
  struct LapPos {
    int e, c, kb, w, ea, n, s;
    bool in;
    double rxw, rxe, rxp, ryn, rys, ryp;
  };
  LapPos lp[kHbLf];
#pragma unroll
  for (int f = 0; f < kHbLf; ++f) {
    LapPos& L = lp[f];
    L.e = tid + f * kHbN;
    const int hy = L.e / kHbLx, hx = L.e - hy * kHbLx;
    const int i = i0 - 1 + hx, j = j0 - 1 + hy;
    L.in = L.e < kHbL && i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1;
    L.c = (hy + 1) * kHbTx + (hx + 1);
    if (L.in) {
      const int ij = G.L.at2(i, j);
      L.kb = G.gp.kb[ij];
      L.w = G.gp.kb[G.L.at2(i - 1, j)];
      L.ea = G.gp.kb[G.L.at2(i + 1, j)];
      L.n = G.gp.kb[G.L.at2(i, j - 1)];
      L.s = G.gp.kb[G.L.at2(i, j + 1)];
      L.rxw = G.rdlxu[G.L.at2(i - 1, j)];
      L.rxe = G.rdlxu[ij];
      L.rxp = G.rdlxp[ij];
      L.ryn = G.rdlyv[G.L.at2(i, j - 1)];
      L.rys = G.rdlyv[ij];
      L.ryp = G.rdlyp[ij];
    }
  }
  // this thread's cell
  const int i = i0 + tx, j = j0 + ty;
  const bool cell = i <= IE && j <= JE;
  const bool inner = cell && i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1;
  int kbc = 0, kbw = 0, kbe = 0, kbn = 0, kbs = 0;
  double tfw = 0, tfe = 0, tfn = 0, tfs = 0, rar = 0, bot = 0, zc = 0;
  if (inner) {
    const int ijc = G.L.at2(i, j);
    kbc = G.gp.kb[ijc];
    kbw = G.gp.kb[G.L.at2(i - 1, j)];
    kbe = G.gp.kb[G.L.at2(i + 1, j)];
    kbn = G.gp.kb[G.L.at2(i, j - 1)];
    kbs = G.gp.kb[G.L.at2(i, j + 1)];
    tfw = G.tfx[G.L.at2(i - 1, j)];
    tfe = G.tfx[ijc];
    tfn = G.tfy[G.L.at2(i, j - 1)];
    tfs = G.tfy[ijc];
    rar = G.rareap[ijc];
    bot = G.gp.bot[ijc];
    zc = zo[ijc];
  }
  const int me_t = (ty + 2) * kHbTx + (tx + 2), me_l = (ty + 1) * kHbLx + (tx + 1);
  const int own = cell ? G.L.at(i, j, 0) : 0;
  auto wet_at = [](int kb, int K) { return K <= kb ? 1.0 : 0.0; };
  for (int n = 0; n < ntr; ++n) {
    const double* __restrict__ T = tp.in[n];
    double* __restrict__ O = tp.out[n];
    double nx[kHbTf];
#pragma unroll
    for (int f = 0; f < kHbTf; ++f) nx[f] = tin[f] ? T[toff[f]] : 0.0;
    for (int K = 1; K <= KE; ++K) {
      __syncthreads();  // the previous level's tiles are no longer read
#pragma unroll
      for (int f = 0; f < kHbTf; ++f)
        if (tval[f]) ts[tid + f * kHbN] = nx[f];
      if (K < KE) {
#pragma unroll
        for (int f = 0; f < kHbTf; ++f)
          if (tin[f]) nx[f] = T[toff[f] + plane * K];
      }
      __syncthreads();
#pragma unroll
      for (int f = 0; f < kHbLf; ++f) {
        const LapPos& L = lp[f];
        if (L.e >= kHbL) continue;
        double r = 0.0;
        if (L.in) {
          const double c = ts[L.c];
          r = wet_at(L.kb, K) *
              ((wet_at(L.w, K) * (ts[L.c - 1] - c) * L.rxw +
                wet_at(L.ea, K) * (ts[L.c + 1] - c) * L.rxe) *
                   L.rxp +
               (wet_at(L.n, K) * (ts[L.c - kHbTx] - c) * L.ryn +
                wet_at(L.s, K) * (ts[L.c + kHbTx] - c) * L.rys) *
                   L.ryp);
        }
        ls[L.e] = r;
      }
      __syncthreads();
      if (cell) {
        const double t = ts[me_t];
        double r = t;
        if (inner) {
          const double zzsurf = K == 1 ? 1. : 0.;
          const double c = ls[me_l];
          const double th = K < kbc ? G.dzw[K - 1] : (K == kbc ? bot : 0.0);
          const double fac = div_nr(wet_at(kbc, K) * rar, th + G.almzer + zzsurf * (zc));
          r = t - fac * G.dzw[K - 1] *
                      (wet_at(kbw, K) * tfw * (ls[me_l - 1] - c) +
                       wet_at(kbe, K) * tfe * (ls[me_l + 1] - c) +
                       wet_at(kbn, K) * tfn * (ls[me_l - kHbLx] - c) +
                       wet_at(kbs, K) * tfs * (ls[me_l + kHbLx] - c));
        }
        O[own + plane * (K - 1)] = r;
      }
    }
  }
}

// -------------------------------------------------------------- OCVISC ----
// bottom speeds SPEEDU/SPEEDV (ocvisc.f90:53-104): evaluated at the single
// level where the mask drops from 1 to 0 (or at KE when the column is full)
__global__ void k_visc_speed(Geo G, const double* __restrict__ uoo, const double* __restrict__ voe,
                             double* __restrict__ spu, double* __restrict__ spv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int IE = G.L.ie, JE = G.L.je;
  if (i > IE || j > JE) return;
  const int ij = G.L.at2(i, j);
  double su = 0., sv = 0.;
  if (i >= 1 && i <= IE - 1 && j >= 2 && j <= JE - 1) {
    const int K = G.gu.kb[ij];
    if (K >= 1) {
      const double a = 0.25 * (AT(voe, i, j, K) + AT(voe, i + 1, j, K) + AT(voe, i, j - 1, K) +
                               AT(voe, i + 1, j - 1, K));
      const double u = AT(uoo, i, j, K);
      su = fmx(sqrt(u * u + a * a), 1.E-3);
    }
  }
  if (i >= 2 && i <= IE - 1 && j >= 1 && j <= JE - 1) {
    const int K = G.gv.kb[ij];
    if (K >= 1) {
      const double a = 0.25 * (AT(uoo, i, j, K) + AT(uoo, i - 1, j, K) + AT(uoo, i, j + 1, K) +
                               AT(uoo, i - 1, j + 1, K));
      const double v = AT(voe, i, j, K);
      sv = fmx(sqrt(v * v + a * a), 1.E-3);
    }
  }
  spu[ij] = su;
  spv[ij] = sv;
}

// implicit vertical diffusion of u (DIR = 0, ocvisc.f90:168-218) or v
// (DIR = 1, ocvisc.f90:114-165) with quadratic bottom drag in the last row
template <int DIR>
__global__ void __launch_bounds__(kVertBlock) k_visc_uv(Geo G, const double* __restrict__ X,
                                                        const double* __restrict__ keep,
                                                        const double* __restrict__ avo,
                                                        const double* __restrict__ speed,
                                                        double* __restrict__ O) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const bool interior = DIR == 0 ? (i >= 1 && i <= IE - 1 && j >= 2 && j <= JE - 1)
                                 : (i >= 2 && i <= IE - 1 && j >= 1 && j <= JE - 1);
  const bool valid = DIR == 0 ? (j >= 1) : (i >= 1);
  if (!valid) return;
  if (!interior) {
    for (int K = 1; K <= KE; ++K) AT(O, i, j, K) = AT(keep, i, j, K);
    return;
  }
  const ColGeo& cg = DIR == 0 ? G.gu : G.gv;
  const int ij = G.L.at2(i, j);
  const int ij2 = DIR == 0 ? G.L.at2(i + 1, j) : G.L.at2(i, j + 1);
  const double BOFRIC = 3.E-3, RAYFRIC = 3.E-3;
  const double sp = speed[ij];
  auto avo_at = [&](int q, int K) { return avo[q + G.L.plane * (K - 1)]; };
  // TRIDSY(K,1) and TRIDSY(K,3) (after the AMS(K+1) factor) of
  // ocvisc.f90:117-140 / 171-193
  auto tri = [&](int K, double& t1, double& t3) {
    const double am = wet(cg, ij, K), dd = thick(cg, G.dzw, ij, K);
    const double avup = 0.5 * (avo_at(ij, K) + avo_at(ij2, K)) * am;
    if (K < KE) {
      const double am1 = wet(cg, ij, K + 1);
      const double avlo = 0.5 * (avo_at(ij, K + 1) + avo_at(ij2, K + 1)) * am1 +
                          (BOFRIC + RAYFRIC * dd * sp) * (am - am1);
      t1 = div_nr(-G.dt * avup * am * G.di[K - 1], G.almzer + dd);
      t3 = div_nr(-G.dt * avlo * am * G.di[K], G.almzer + dd);
    } else {
      const double avlo = (BOFRIC + RAYFRIC * dd * sp) * am;
      t1 = div_nr(-G.dt * avup * am * G.di[K - 1], G.almzer + dd);
      t3 = div_nr(-G.dt * avlo * am * G.di[K], G.almzer + dd);
    }
  };
  double t2p[kMaxKe];
  double t2prev = 1.0, t3prev = 0.0, yprev = 0.0;
  for (int K = 1; K <= KE; ++K) {
    double t1, t3;
    tri(K, t1, t3);
    double t2 = 1. - t1 - t3;
    t3 = K < KE ? t3 * wet(cg, ij, K + 1) : 0.;
    const double xk = AT(X, i, j, K);
    double y = xk;
    if (K >= 2) {
      const double m = div_nr(t1, t2prev);
      t2 = t2 - div_nr(t3prev * t1, t2prev);
      y = xk - m * yprev;
    }
    t2p[K - 1] = t2;
    AT(O, i, j, K) = y;
    yprev = y;
    t2prev = t2;
    t3prev = t3;
  }
  double nxt = div_nr(wet(cg, ij, KE) * AT(O, i, j, KE), t2p[KE - 1]);
  AT(O, i, j, KE) = nxt;
  for (int l = KE - 1; l >= 1; --l) {
    double t1, t3;
    tri(l, t1, t3);
    t3 = t3 * wet(cg, ij, l + 1);
    nxt = div_nr((AT(O, i, j, l) - t3 * nxt) * wet(cg, ij, l), t2p[l - 1]);
    AT(O, i, j, l) = nxt;
  }
}

// k_visc_uv with the loads of U levels issued together before they are used
// (X and AVO of both columns in the forward sweep, the forward values and AVO
// in the backward one); the same expressions in the same order, so the
// results equal k_visc_uv's bit for bit.
template <int DIR, int U>
__global__ void __launch_bounds__(kVertBlock) k_visc_uv_b(Geo G, const double* __restrict__ X,
                                                          const double* __restrict__ keep,
                                                          const double* __restrict__ avo,
                                                          const double* __restrict__ speed,
                                                          double* __restrict__ O) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const bool interior = DIR == 0 ? (i >= 1 && i <= IE - 1 && j >= 2 && j <= JE - 1)
                                 : (i >= 2 && i <= IE - 1 && j >= 1 && j <= JE - 1);
  const bool valid = DIR == 0 ? (j >= 1) : (i >= 1);
  if (!valid) return;
  const int pl = G.L.plane;
  const int base = G.L.at(i, j, 0);
  if (!interior) {
    for (int K = 1; K <= KE; ++K) O[base + (K - 1) * pl] = keep[base + (K - 1) * pl];
    return;
  }
  const ColGeo& cg = DIR == 0 ? G.gu : G.gv;
  const int ij = G.L.at2(i, j);
  const int ij2 = DIR == 0 ? G.L.at2(i + 1, j) : G.L.at2(i, j + 1);
  const double BOFRIC = 3.E-3, RAYFRIC = 3.E-3;
  const double sp = speed[ij];
  // TRIDSY(K,1) and TRIDSY(K,3) from AVO of levels K (a0, b0) and K+1 (a1, b1)
  // of the two columns, as k_visc_uv's tri
  auto tri = [&](int K, double a0, double b0, double a1, double b1, double& t1, double& t3) {
    const double am = wet(cg, ij, K), dd = thick(cg, G.dzw, ij, K);
    const double avup = 0.5 * (a0 + b0) * am;
    if (K < KE) {
      const double am1 = wet(cg, ij, K + 1);
      const double avlo = 0.5 * (a1 + b1) * am1 + (BOFRIC + RAYFRIC * dd * sp) * (am - am1);
      t1 = div_nr(-G.dt * avup * am * G.di[K - 1], G.almzer + dd);
      t3 = div_nr(-G.dt * avlo * am * G.di[K], G.almzer + dd);
    } else {
      const double avlo = (BOFRIC + RAYFRIC * dd * sp) * am;
      t1 = div_nr(-G.dt * avup * am * G.di[K - 1], G.almzer + dd);
      t3 = div_nr(-G.dt * avlo * am * G.di[K], G.almzer + dd);
    }
  };
  double t2p[kMaxKe];
  double t2prev = 1.0, t3prev = 0.0, yprev = 0.0;
  for (int K0 = 1; K0 <= KE; K0 += U) {
    double la[U + 1], lb[U + 1], lx[U];
#pragma unroll
    for (int u = 0; u <= U; ++u) {
      const bool ok = K0 + u <= KE;
      la[u] = ok ? avo[ij + (K0 + u - 1) * pl] : 0.0;
      lb[u] = ok ? avo[ij2 + (K0 + u - 1) * pl] : 0.0;
      if (u < U) lx[u] = ok ? X[base + (K0 + u - 1) * pl] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int K = K0 + u;
      if (K > KE) break;
      double t1, t3;
      tri(K, la[u], lb[u], la[u + 1], lb[u + 1], t1, t3);
      double t2 = 1. - t1 - t3;
      t3 = K < KE ? t3 * wet(cg, ij, K + 1) : 0.;
      const double xk = lx[u];
      double y = xk;
      if (K >= 2) {
        const double m = div_nr(t1, t2prev);
        t2 = t2 - div_nr(t3prev * t1, t2prev);
        y = xk - m * yprev;
      }
      t2p[K - 1] = t2;
      O[base + (K - 1) * pl] = y;
      yprev = y;
      t2prev = t2;
      t3prev = t3;
    }
  }
  double nxt = div_nr(wet(cg, ij, KE) * yprev, t2p[KE - 1]);
  O[base + (KE - 1) * pl] = nxt;
  for (int l0 = KE - 1; l0 >= 1; l0 -= U) {
    double la[U], lb[U], la1[U], lb1[U], ly[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int l = l0 - u;
      const bool ok = l >= 1;
      la[u] = ok ? avo[ij + (l - 1) * pl] : 0.0;
      lb[u] = ok ? avo[ij2 + (l - 1) * pl] : 0.0;
      la1[u] = ok ? avo[ij + l * pl] : 0.0;
      lb1[u] = ok ? avo[ij2 + l * pl] : 0.0;
      ly[u] = ok ? O[base + (l - 1) * pl] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int l = l0 - u;
      if (l < 1) break;
      double t1, t3;
      tri(l, la[u], lb[u], la1[u], lb1[u], t1, t3);
      t3 = t3 * wet(cg, ij, l + 1);
      nxt = div_nr((ly[u] - t3 * nxt) * wet(cg, ij, l), t2p[l - 1]);
      O[base + (l - 1) * pl] = nxt;
    }
  }
}

// implicit vertical diffusion of w, levels 2..KE (ocvisc.f90:225-270).  One
// forward sweep forms each level's coefficients, eliminates (the multiplier
// TRIDSY(K-1,1)/TRIDSY(K-1,2) and the new diagonal, in the reference's
// operation order) and substitutes; only the eliminated diagonal is kept per
// level, and the backward sweep recomputes TRIDSY(K,3) by the same expression.
// The loads of U levels are issued together (the results do not depend on U).
template <int U>
__global__ void __launch_bounds__(kVertBlock) k_visc_w_b(Geo G, const double* __restrict__ W,
                                                         const double* __restrict__ avo,
                                                         double* __restrict__ O) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const int pl = G.L.plane;
  const int base = G.L.at(i, j, 0);
  const bool interior = i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1 && KE >= 2;
  if (!interior) {
    for (int K = 1; K <= KE + 1; ++K) O[base + (K - 1) * pl] = W[base + (K - 1) * pl];
    return;
  }
  const int ij = G.L.at2(i, j);
  auto den = [&](int K) {
    return 2.0 * G.almzer + thick(G.gp, G.dzw, ij, K - 1) + thick(G.gp, G.dzw, ij, K);
  };
  // AVO of levels K-1 (am), K (a0), K+1 (a1)
  auto tri1 = [&](int K, double dn, double am, double a0) {
    const double avup = 0.5 * (am + a0) * wet(G.gp, ij, K - 1);
    return div_nr(-2.0 * G.dt * avup * wet(G.gp, ij, K) * G.di[K - 2], dn);
  };
  auto tri3 = [&](int K, double dn, double a0, double a1) {
    const double avlo = K < KE ? 0.5 * (a1 + a0) * wet(G.gp, ij, K) : 0.0;
    return div_nr(-2.0 * G.dt * avlo * wet(G.gp, ij, K) * G.di[K - 1], dn);
  };
  double t2p[kMaxKe];
  O[base] = W[base];
  O[base + KE * pl] = W[base + KE * pl];
  double prev = 0.0, t2prev = 1.0, t3prev = 0.0;
  for (int K0 = 2; K0 <= KE; K0 += U) {
    double la[U + 2], lw[U];
#pragma unroll
    for (int u = 0; u < U + 2; ++u) {
      const int K = K0 - 1 + u;  // K0-1 .. K0+U
      la[u] = K <= KE ? avo[base + (K - 1) * pl] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) lw[u] = K0 + u <= KE ? W[base + (K0 + u - 1) * pl] : 0.0;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int K = K0 + u;
      if (K > KE) break;
      const double dn = den(K);
      const double t1 = tri1(K, dn, la[u], la[u + 1]), t3 = tri3(K, dn, la[u + 1], la[u + 2]);
      double t2 = 1. - t1 - t3;
      double y = lw[u];
      if (K >= 3) {
        const double m = div_nr(t1, t2prev);
        t2 = t2 - div_nr(t3prev * t1, t2prev);
        y = y - m * prev;
      }
      t2p[K - 1] = t2;
      O[base + (K - 1) * pl] = y;
      prev = y;
      t2prev = t2;
      t3prev = K < KE ? t3 : 0.;
    }
  }
  double nxt = div_nr(wet(G.gp, ij, KE) * prev, t2p[KE - 1]);
  O[base + (KE - 1) * pl] = nxt;
  for (int K0 = KE - 1; K0 >= 2; K0 -= U) {
    double la[U], la1[U], ly[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int K = K0 - u;
      const bool ok = K >= 2;
      la[u] = ok ? avo[base + (K - 1) * pl] : 0.0;
      la1[u] = ok ? avo[base + K * pl] : 0.0;
      ly[u] = ok ? O[base + (K - 1) * pl] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int K = K0 - u;
      if (K < 2) break;
      const double t3 = tri3(K, den(K), la[u], la1[u]);
      nxt = div_nr((ly[u] - t3 * nxt) * wet(G.gp, ij, K), t2p[K - 1]);
      O[base + (K - 1) * pl] = nxt;
    }
  }
}

__device__ __forceinline__ double rdlypsi(const Geo& G, int i, int j) { return G.rdlypsi[G.L.at2(i, j)]; }
__device__ __forceinline__ double rdlxpsi(const Geo& G, int i, int j) { return G.rdlxpsi[G.L.at2(i, j)]; }

// first Laplacians UK1O (u), VK1E (v), WN1O (w), ocvisc.f90:350-438, 617-669.
// (Fusing this pass with the next through shared-memory tiles, as the tracer
// kernel above does, was measured on c3 and not kept: with the geometry of
// the edge cases reloaded every level the fused form was 5% slower, and one
// launch per level 1.7x slower, than these two level-parallel passes.)
__global__ void k_visc_lap(Geo G, const double* __restrict__ uk, const double* __restrict__ vk,
                           const double* __restrict__ wn, double* __restrict__ u1,
                           double* __restrict__ v1, double* __restrict__ w1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int K = blockIdx.z + 1;
  const int IE = G.L.ie, JE = G.L.je;
  if (i > IE || j > JE) return;
  // ---- u-points
  if (j >= 1) {
    auto AO = [&](int ii, int jj) { return wet(G.gu, G.L.at2(ii, jj), K); };
    auto UK = [&](int ii, int jj) { return AT(uk, ii, jj, K); };
    const bool jin = j >= 2 && j <= JE - 1, iin = i >= 1 && i <= IE - 1;
    double r = 0.0;
    auto ypart = [&]() {
      return (AO(i, j - 1) * (UK(i, j - 1) - UK(i, j)) * rdlypsi(G, i, j - 1) -
              AO(i, j + 1) * (UK(i, j) - UK(i, j + 1)) * rdlypsi(G, i, j)) *
             G.rdlyu[G.L.at2(i, j)];
    };
    auto xpart = [&]() {
      return (AO(i + 1, j) * (UK(i + 1, j) - UK(i, j)) * G.rdlxp[G.L.at2(i + 1, j)] -
              AO(i - 1, j) * (UK(i, j) - UK(i - 1, j)) * G.rdlxp[G.L.at2(i, j)]) *
             G.rdlxu[G.L.at2(i, j)];
    };
    if (jin && iin) {
      r = AO(i, j) * (xpart() + ypart());
    } else if (jin && i == 0) {
      r = AO(i, j) * ((AO(i + 1, j) * (UK(i + 1, j) - UK(i, j)) * G.rdlxp[G.L.at2(i + 1, j)]) *
                          G.rdlxu[G.L.at2(i, j)] +
                      ypart());
    } else if (jin && i == IE) {
      r = AO(i, j) * ((-AO(i - 1, j) * (UK(i, j) - UK(i - 1, j)) * G.rdlxp[G.L.at2(i, j)]) *
                          G.rdlxu[G.L.at2(i, j)] +
                      ypart());
    } else if (iin && j == 1) {
      r = AO(i, j) * (xpart() + (-AO(i, j + 1) * (UK(i, j) - UK(i, j + 1)) * rdlypsi(G, i, j)) *
                                    G.rdlyu[G.L.at2(i, j)]);
    } else if (iin && j == JE) {
      r = AO(i, j) * (xpart() + (AO(i, j - 1) * (UK(i, j - 1) - UK(i, j)) * rdlypsi(G, i, j - 1)) *
                                    G.rdlyu[G.L.at2(i, j)]);
    }
    AT(u1, i, j, K) = r;
  }
  // ---- v-points
  if (i >= 1) {
    auto AE = [&](int ii, int jj) { return wet(G.gv, G.L.at2(ii, jj), K); };
    auto VK = [&](int ii, int jj) { return AT(vk, ii, jj, K); };
    const bool jin = j >= 1 && j <= JE - 1, iin = i >= 2 && i <= IE - 1;
    double r = 0.0;
    auto xpart = [&]() {
      return (AE(i + 1, j) * (VK(i + 1, j) - VK(i, j)) * rdlxpsi(G, i, j) -
              AE(i - 1, j) * (VK(i, j) - VK(i - 1, j)) * rdlxpsi(G, i - 1, j)) *
             G.rdlxv[G.L.at2(i, j)];
    };
    auto ypart = [&]() {
      return (AE(i, j - 1) * (VK(i, j - 1) - VK(i, j)) * G.rdlyp[G.L.at2(i, j)] -
              AE(i, j + 1) * (VK(i, j) - VK(i, j + 1)) * G.rdlyp[G.L.at2(i, j + 1)]) *
             G.rdlyv[G.L.at2(i, j)];
    };
    if (jin && iin) {
      r = AE(i, j) * (xpart() + ypart());
    } else if (jin && i == 1) {
      r = AE(i, j) * ((AE(i + 1, j) * (VK(i + 1, j) - VK(i, j)) * rdlxpsi(G, i, j)) *
                          G.rdlxv[G.L.at2(i, j)] +
                      ypart());
    } else if (jin && i == IE) {
      r = AE(i, j) * ((-AE(i - 1, j) * (VK(i, j) - VK(i - 1, j)) * rdlxpsi(G, i - 1, j)) *
                          G.rdlxv[G.L.at2(i, j)] +
                      ypart());
    } else if (iin && j == 0) {
      r = AE(i, j) * (xpart() + (-AE(i, j + 1) * (VK(i, j) - VK(i, j + 1)) * G.rdlyp[G.L.at2(i, j + 1)]) *
                                    G.rdlyv[G.L.at2(i, j)]);
    } else if (iin && j == JE) {
      r = AE(i, j) * (xpart() + (AE(i, j - 1) * (VK(i, j - 1) - VK(i, j)) * G.rdlyp[G.L.at2(i, j)]) *
                                    G.rdlyv[G.L.at2(i, j)]);
    }
    AT(v1, i, j, K) = r;
  }
  // ---- w-points (levels 1..KE)
  if (i >= 1 && j >= 1) {
    auto WE = [&](int ii, int jj) { return wet(G.gp, G.L.at2(ii, jj), K); };
    auto WN = [&](int ii, int jj) { return AT(wn, ii, jj, K); };
    const bool jin = j >= 2 && j <= JE - 1, iin = i >= 2 && i <= IE - 1;
    double r = 0.0;
    auto xpart = [&]() {
      return (WE(i + 1, j) * (WN(i + 1, j) - WN(i, j)) * G.rdlxu[G.L.at2(i, j)] -
              WE(i - 1, j) * (WN(i, j) - WN(i - 1, j)) * G.rdlxu[G.L.at2(i - 1, j)]) *
             G.rdlxp[G.L.at2(i, j)];
    };
    auto ypart = [&]() {
      return (WE(i, j - 1) * (WN(i, j - 1) - WN(i, j)) * G.rdlyv[G.L.at2(i, j - 1)] -
              WE(i, j + 1) * (WN(i, j) - WN(i, j + 1)) * G.rdlyv[G.L.at2(i, j)]) *
             G.rdlyp[G.L.at2(i, j)];
    };
    if (jin && iin) {
      r = WE(i, j) * (xpart() + ypart());
    } else if (jin && i == 1) {
      r = WE(i, j) * ((WE(i + 1, j) * (WN(i + 1, j) - WN(i, j)) * G.rdlxu[G.L.at2(i, j)]) *
                          G.rdlxp[G.L.at2(i, j)] +
                      ypart());
    } else if (jin && i == IE) {
      r = WE(i, j) * ((-WE(i - 1, j) * (WN(i, j) - WN(i - 1, j)) * G.rdlxu[G.L.at2(i - 1, j)]) *
                          G.rdlxp[G.L.at2(i, j)] +
                      ypart());
    } else if (iin && j == 1) {
      r = WE(i, j) * (xpart() + (-WE(i, j + 1) * (WN(i, j) - WN(i, j + 1)) * G.rdlyv[G.L.at2(i, j)]) *
                                    G.rdlyp[G.L.at2(i, j)]);
    } else if (iin && j == JE) {
      r = WE(i, j) * (xpart() + (WE(i, j - 1) * (WN(i, j - 1) - WN(i, j)) * G.rdlyv[G.L.at2(i, j - 1)]) *
                                    G.rdlyp[G.L.at2(i, j)]);
    }
    AT(w1, i, j, K) = r;
  }
}

// second passes, ocvisc.f90:445-477 (u, v) and 673-688 (w)
__global__ void k_visc_bih(Geo G, const double* __restrict__ uoo, const double* __restrict__ voe,
                           const double* __restrict__ uk, const double* __restrict__ vk,
                           const double* __restrict__ wn, const double* __restrict__ u1,
                           const double* __restrict__ v1, const double* __restrict__ w1,
                           double* __restrict__ uo, double* __restrict__ vo,
                           double* __restrict__ wo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int K = blockIdx.z + 1;  // 1..KE+1
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const double mv = G.minvalue;
  // The face terms AUL.. * width / length of ocvisc.f90:445-477, 673-688 are
  // precomputed per face (G.ugx .. G.wgy) and the cell areas' reciprocals per
  // cell, so a cell needs no division except by its thickness (w).
  if (K <= KE) {
    // ---- u
    if (j >= 1) {
      double r = AT(uoo, i, j, K);
      if (i >= 1 && i <= IE - 1 && j >= 2 && j <= JE - 1) {
        auto AO = [&](int ii, int jj) { return wet(G.gu, G.L.at2(ii, jj), K); };
        auto U1 = [&](int ii, int jj) { return AT(u1, ii, jj, K); };
        const int ij = G.L.at2(i, j);
        r = (AO(i, j) * G.rareau[ij]) *
            (G.dlxu[ij] * G.dlyu[ij] * AT(uk, i, j, K) -
             (G.ugx[G.L.at2(i + 1, j)] * AO(i + 1, j) * (U1(i + 1, j) - U1(i, j)) -
              G.ugx[ij] * AO(i - 1, j) * (U1(i, j) - U1(i - 1, j)) +
              G.ugy[G.L.at2(i, j - 1)] * AO(i, j - 1) * (U1(i, j - 1) - U1(i, j)) -
              G.ugy[ij] * AO(i, j + 1) * (U1(i, j) - U1(i, j + 1))));
      }
      AT(uo, i, j, K) = r;
    }
    // ---- v
    if (i >= 1) {
      double r = AT(voe, i, j, K);
      if (i >= 2 && i <= IE - 1 && j >= 1 && j <= JE - 1) {
        auto AE = [&](int ii, int jj) { return wet(G.gv, G.L.at2(ii, jj), K); };
        auto V1 = [&](int ii, int jj) { return AT(v1, ii, jj, K); };
        const int ij = G.L.at2(i, j);
        r = (AE(i, j) * G.rareav[ij]) *
            (G.dlxv[ij] * G.dlyv[ij] * AT(vk, i, j, K) -
             (G.vgx[ij] * AE(i + 1, j) * (V1(i + 1, j) - V1(i, j)) -
              G.vgx[G.L.at2(i - 1, j)] * AE(i - 1, j) * (V1(i, j) - V1(i - 1, j)) +
              G.vgy[ij] * AE(i, j - 1) * (V1(i, j - 1) - V1(i, j)) -
              G.vgy[G.L.at2(i, j + 1)] * AE(i, j + 1) * (V1(i, j) - V1(i, j + 1))));
      }
      AT(vo, i, j, K) = r;
    }
  }
  // ---- w (levels 1..KE updated, KEP carried)
  if (i >= 1 && j >= 1) {
    double r = AT(wn, i, j, K);
    if (K <= KE && i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1) {
      auto WE = [&](int ii, int jj) { return wet(G.gp, G.L.at2(ii, jj), K); };
      auto W1 = [&](int ii, int jj) { return AT(w1, ii, jj, K); };
      auto dzu = [&](int ii, int jj) { return fmx(thick(G.gu, G.dzw, G.L.at2(ii, jj), K), mv); };
      auto dzv = [&](int ii, int jj) { return fmx(thick(G.gv, G.dzw, G.L.at2(ii, jj), K), mv); };
      const int ij = G.L.at2(i, j);
      const double dzp = fmx(thick(G.gp, G.dzw, ij, K), mv);
      r = div_nr(WE(i, j) * G.rareap[ij], dzp) *
          (G.dlxp[ij] * G.dlyp[ij] * dzp * AT(wn, i, j, K) -
           (G.wgx[ij] * dzu(i, j) * WE(i + 1, j) * (W1(i + 1, j) - W1(i, j)) -
            G.wgx[G.L.at2(i - 1, j)] * dzu(i - 1, j) * WE(i - 1, j) * (W1(i, j) - W1(i - 1, j)) +
            G.wgy[G.L.at2(i, j - 1)] * dzv(i, j - 1) * WE(i, j - 1) * (W1(i, j - 1) - W1(i, j)) -
            G.wgy[ij] * dzv(i, j) * WE(i, j + 1) * (W1(i, j) - W1(i, j + 1))));
    }
    AT(wo, i, j, K) = r;
  }
}

}  // namespace

void launch_octdiff_vert(const Geo& G, int ntr, const double* const* in, double* const* out,
                         const double* dvo, const double* zo, cudaStream_t st) {
  TrPtrs tp{};
  for (int n = 0; n < ntr; ++n) {
    tp.in[n] = in[n];
    tp.out[n] = out[n];
  }
  const dim3 b(32, kVertBlock / 32);
  const dim3 gr = grid2(G.L.ie, G.L.je, b);
  switch (ntr) {
    case 1: k_tdiff_vert_b<1, 4><<<gr, b, 0, st>>>(G, tp, dvo, zo); break;
    case 2: k_tdiff_vert_b<2, 4><<<gr, b, 0, st>>>(G, tp, dvo, zo); break;
    case 3: k_tdiff_vert_b<3, 4><<<gr, b, 0, st>>>(G, tp, dvo, zo); break;
    case 4: k_tdiff_vert_b<4, 4><<<gr, b, 0, st>>>(G, tp, dvo, zo); break;
    default: k_tdiff_vert<<<gr, b, 0, st>>>(G, tp, ntr, dvo, zo); break;
  }
  count_launch();
}

void launch_octdiff_hbih(const Geo& G, int ntr, const double* const* in, double* const* out,
                         const double* zo, cudaStream_t st) {
  TrPtrs tp{};
  for (int n = 0; n < ntr; ++n) {
    tp.in[n] = in[n];
    tp.out[n] = out[n];
  }
  const dim3 b(kHbX, kHbY);
  k_tdiff_hbih<<<grid2(G.L.ie, G.L.je, b), b, 0, st>>>(G, tp, ntr, zo);
  count_launch();
}

void launch_ocvisc(const Geo& G, const double* uoo, const double* voe, const double* wno,
                   const double* uko, const double* vke, const double* avo, double* spu,
                   double* spv, double* ukv, double* vkv, double* wnv, double* u1, double* v1,
                   double* w1, double* uo, double* vo, double* wo, cudaStream_t st) {
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  const dim3 b2(32, 4), bc(32, kVertBlock / 32), b3(32, 4);
  k_visc_speed<<<grid2(IE + 1, JE + 1, b2), b2, 0, st>>>(G, uoo, voe, spu, spv);
  count_launch();
  k_visc_uv_b<0, 4><<<grid2(IE + 1, JE + 1, bc), bc, 0, st>>>(G, uoo, uko, avo, spu, ukv);
  count_launch();
  k_visc_uv_b<1, 4><<<grid2(IE + 1, JE + 1, bc), bc, 0, st>>>(G, voe, vke, avo, spv, vkv);
  count_launch();
  k_visc_w_b<4><<<grid2(IE, JE, bc), bc, 0, st>>>(G, wno, avo, wnv);
  count_launch();
  dim3 gl = grid2(IE + 1, JE + 1, b3);
  gl.z = KE;
  k_visc_lap<<<gl, b3, 0, st>>>(G, ukv, vkv, wnv, u1, v1, w1);
  count_launch();
  gl.z = KE + 1;
  k_visc_bih<<<gl, b3, 0, st>>>(G, uoo, voe, ukv, vkv, wnv, u1, v1, w1, uo, vo, wo);
  count_launch();
}

}  // namespace orctm
