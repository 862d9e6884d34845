// Barotropic (free-surface) solve and total velocities, the part of the
// reference step that runs just before the hot path (orctm.f90:1342-1431):
// OCWIND's surface stress (ocwind.f90:1-42), OCBARP's barotropic transports
// (ocbarp.f90:1-48), ITPREP's SOR coefficients (itprep.f90:15-40) and
// TROTEST's choice of the SOR parameter (trotest.f90:1-118), with the inverse u/v depths
// (boden.f90:264-274), TRONEU's right-hand side and red-black SOR for the
// elevation change Z1O (troneu.f90:48-134), OCVTRO's barotropic velocities
// and ZO update (ocvtro.f90:1-62), and OCVTOT's total velocities, time
// filter and WO (ocvtot.f90:13-96).
//
// The 2D fields live in the padded plane layout of common.cuh.  Every
// expression is the reference's, term for term, in IEEE binary64 (the
// library is built with --fmad=false and IEEE division), so the results equal
// the CPU restatement bit for bit.  One SOR colour is one kernel (a grid-wide
// dependency separates the colours); the 2 x niter launches are replayed as a
// CUDA graph by the caller.
#include "common.cuh"
#include "ops.h"

namespace orctm {

namespace {

#define AT(a, i, j, K) (a)[G.L.at((i), (j), (K)-1)]
#define A2(a, i, j) (a)[G.L.at2((i), (j))]

inline dim3 grid2(int nx, int ny, dim3 b) { return dim3((nx + b.x - 1) / b.x, (ny + b.y - 1) / b.y, 1); }

// ITPREP and the inverse depths; one thread per (i, j) in [0, IE] x [0, JE]
__global__ void k_itprep(Geo G, BaroArgs a, const double* __restrict__ deuto,
                         const double* __restrict__ deute, BaroFields f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int IE = G.L.ie, JE = G.L.je;
  if (i > IE || j > JE) return;
  const double dt = G.dt;
  const int ij = G.L.at2(i, j);
  if (j >= 1) {  // u-points I in [0, IE]: UF, DEUTIO
    f.uf[ij] = deuto[ij] * G.dlyu[ij] / G.dlxu[ij] * a.grav * a.conn * a.stabn * (dt * dt);
    f.deutio[ij] = deuto[ij] > a.minvalue ? 1. / deuto[ij] : 0.0;
  }
  if (i >= 1) {  // v-points J in [0, JE]: VF, DEUTIE
    f.vf[ij] = deute[ij] * G.dlxv[ij] / G.dlyv[ij] * a.grav * a.conn * a.stabn * (dt * dt);
    f.deutie[ij] = deute[ij] > a.minvalue ? 1. / deute[ij] : 0.0;
  }
  if (i >= 1 && j >= 1) f.xx[ij] = G.dlxp[ij] * G.dlyp[ij];
}

// FF needs the UF / VF of the neighbouring faces: a second pass
__global__ void k_itprep_ff(Geo G, BaroFields f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (i > G.L.ie || j > G.L.je) return;
  const int ij = G.L.at2(i, j);
  f.ff[ij] = 1. / (f.xx[ij] + f.uf[ij] + f.uf[G.L.at2(i - 1, j)] + f.vf[ij] + f.vf[G.L.at2(i, j - 1)]);
}

// B1O (troneu.f90:48-60) and, unless OBC_ETA_FORC, the boundary Z1O
// (troneu.f90:67-102); Z1O is zero elsewhere (cleared before the launch)
__global__ void k_troneu_rhs(Geo G, BaroArgs a, BaroFields f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int IE = G.L.ie, JE = G.L.je;
  if (i > IE || j > JE) return;
  const double conn = a.conn, cono = 1. - a.conn;
  const int ij = G.L.at2(i, j), iw = G.L.at2(i - 1, j), jn = G.L.at2(i, j - 1);
  const double v =
      wet(G.gp, ij, 1) *
      (G.dtdxpo[ij] *
           ((cono * f.u1o[iw] + f.uzo[iw] * conn) * G.dlyu[iw] -
            (f.u1o[ij] * cono + f.uzo[ij] * conn) * G.dlyu[ij]) /
           G.dlyp[ij] +
       G.dtdyo[ij] *
           ((f.v1e[ij] * cono + conn * f.vze[ij]) * G.dlxv[ij] -
            (f.v1e[jn] * cono + conn * f.vze[jn]) * G.dlxv[jn]) /
           G.dlxp[ij]);
  const double b = v * f.xx[ij];
  f.b1o[ij] = b;
  if (!a.eta_forc && (i == 1 || i == IE || j == 1 || j == JE)) f.z1o[ij] = b / f.xx[ij];
}

// one SOR colour (troneu.f90:108-127): J in [2, JE-1], I = IS, IS+2, ..,
// IE-1 with IS = MOD(J + parity, 2) + 2 (p_ioff = p_joff = 0 on one rank)
__global__ void k_sor(Geo G, BaroArgs a, BaroFields f, int parity) {
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int IE = G.L.ie, JE = G.L.je;
  if (j > JE - 1) return;
  const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + (j + parity) % 2 + 2;
  if (i > IE - 1) return;
  const int ij = G.L.at2(i, j);
  const double sorpai = 1. - a.sorpar;
  double* z = f.z1o;
  z[ij] = a.sorpar * f.ff[ij] *
              (f.b1o[ij] + f.uf[ij] * z[G.L.at2(i + 1, j)] + f.uf[G.L.at2(i - 1, j)] * z[G.L.at2(i - 1, j)] +
               f.vf[ij] * z[G.L.at2(i, j + 1)] + f.vf[G.L.at2(i, j - 1)] * z[G.L.at2(i, j - 1)]) +
          sorpai * z[ij];
}

// TROTEST's right-hand side B1O = (RND - 0.5) WETO(.,.,1) XX from the
// pseudo-random values the host drew (trotest.f90:43-55), in place on b1o
__global__ void k_trotest_rhs(Geo G, BaroFields f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (i > G.L.ie || j > G.L.je) return;
  const int ij = G.L.at2(i, j);
  f.b1o[ij] = (f.b1o[ij] - 0.5) * wet(G.gp, ij, 1) * f.xx[ij];
}

// one SOR colour of TROTEST (trotest.f90:62-91): SORPAR from device memory
// (the trials replay one captured graph); the squared change of each point,
// ZALT - Z1O, goes to d2 when d2 is not null
__global__ void k_sor_trial(Geo G, BaroFields f, const double* __restrict__ sorpar, double* d2,
                            int parity) {
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int IE = G.L.ie, JE = G.L.je;
  if (j > JE - 1) return;
  const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + (j + parity) % 2 + 2;
  if (i > IE - 1) return;
  const int ij = G.L.at2(i, j);
  const double sp = *sorpar, sorpai = 1. - sp;
  double* z = f.z1o;
  const double zalt = z[ij];
  const double zn = sp * f.ff[ij] *
                        (f.b1o[ij] + f.uf[ij] * z[G.L.at2(i + 1, j)] + f.uf[G.L.at2(i - 1, j)] * z[G.L.at2(i - 1, j)] +
                         f.vf[ij] * z[G.L.at2(i, j + 1)] + f.vf[G.L.at2(i, j - 1)] * z[G.L.at2(i, j - 1)]) +
                    sorpai * zalt;
  z[ij] = zn;
  if (d2) {
    const double dz = zalt - zn;
    d2[ij] = dz * dz;
  }
}

// OCVTRO; one thread per (i, j) in [0, IE] x [0, JE]
__global__ void k_ocvtro(Geo G, BaroArgs a, BaroFields f, double* __restrict__ zo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int IE = G.L.ie, JE = G.L.je;
  if (i > IE || j > JE) return;
  const int ij = G.L.at2(i, j);
  const double c = a.rlsa1 * a.grav * a.stabn;
  if (j >= 1) {  // u-points: ocvtro.f90:11-16, 34-39
    const double uz = f.uzo[ij] * f.deutio[ij];
    f.uzo[ij] = uz;
    double us = uz;
    if (i >= 1 && i <= IE - 1 && j >= 2 && j <= JE - 1)
      us = uz + c * G.dtdxuo[ij] * (f.z1o[ij] - f.z1o[G.L.at2(i + 1, j)]) * wet(G.gu, ij, 1);
    f.uso[ij] = us;
  }
  if (i >= 1) {  // v-points: ocvtro.f90:18-23, 42-48
    const double vz = f.vze[ij] * f.deutie[ij];
    f.vze[ij] = vz;
    double vs = vz;
    if (i >= 2 && i <= IE - 1 && j >= 1 && j <= JE - 1)
      vs = vz + c * G.dpye[ij] * (f.z1o[G.L.at2(i, j + 1)] - f.z1o[ij]) * wet(G.gv, ij, 1);
    f.vse[ij] = vs;
  }
  if (i >= 1 && j >= 1) zo[ij] = zo[ij] + f.z1o[ij];  // ocvtro.f90:53-57
}

// OCVTOT; one thread per column (i, j) in [0, IE] x [0, JE].  The filtered
// UKO / VKE of the west and north neighbours that WO needs are re-formed
// from the inputs by the same expressions, so no thread waits on another.
__global__ void k_ocvtot(Geo G, BaroArgs a, const double* __restrict__ uso,
                         const double* __restrict__ vse, const double* __restrict__ uoo,
                         const double* __restrict__ voe, const double* __restrict__ uko,
                         const double* __restrict__ vke, double* __restrict__ uoo_o,
                         double* __restrict__ voe_o, double* __restrict__ uko_o,
                         double* __restrict__ vke_o, double* __restrict__ wo_o) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const double conn = a.conn, cono = 1. - a.conn, dti = 1. / G.dt;
  // ocvtot.f90:13-29 then 43-61: UAKO = AMSUO (USO + UKO); UKO = CONN UAKO + UOO CONO
  auto ukf = [&](int ii, int K, double& unf) {
    const int q = G.L.at2(ii, j);
    unf = wet(G.gu, q, K) * (uso[q] + AT(uko, ii, j, K));
    return conn * unf + AT(uoo, ii, j, K) * cono;
  };
  auto vkf = [&](int jj, int K, double& vnf) {
    const int q = G.L.at2(i, jj);
    vnf = wet(G.gv, q, K) * (vse[q] + AT(vke, i, jj, K));
    return conn * vnf + AT(voe, i, jj, K) * cono;
  };
  if (j >= 1)
    for (int K = 1; K <= KE; ++K) {
      double unf;
      const double uk = ukf(i, K, unf);
      AT(uko_o, i, j, K) = uk;
      AT(uoo_o, i, j, K) = unf;
    }
  if (i >= 1)
    for (int K = 1; K <= KE; ++K) {
      double vnf;
      const double vk = vkf(j, K, vnf);
      AT(vke_o, i, j, K) = vk;
      AT(voe_o, i, j, K) = vnf;
    }
  if (i >= 1 && j >= 1) {  // ocvtot.f90:73-93
    const int ij = G.L.at2(i, j), iw = G.L.at2(i - 1, j), jn = G.L.at2(i, j - 1);
    double w = 0.0;
    AT(wo_o, i, j, KE + 1) = w;
    for (int K = KE; K >= 1; --K) {
      double d;
      const double uw = ukf(i - 1, K, d), ue = ukf(i, K, d);
      const double vs = vkf(j, K, d), vn = vkf(j - 1, K, d);
      const double we = wet(G.gp, ij, K);
      w = w +
          dti * we *
              (G.dtdxpo[ij] *
               (uw * thick(G.gu, G.dzw, iw, K) * G.dlyu[iw] - ue * thick(G.gu, G.dzw, ij, K) * G.dlyu[ij]) /
               G.dlyp[ij]) +
          dti * we *
              (+G.dtdyo[ij] *
               (vs * thick(G.gv, G.dzw, ij, K) * G.dlxv[ij] - vn * thick(G.gv, G.dzw, jn, K) * G.dlxv[jn]) /
               G.dlxp[ij]);
      AT(wo_o, i, j, K) = w;
    }
  }
}

// OCBARP (ocbarp.f90:10-45); one thread per (i, j) in [0, IE] x [0, JE]
__global__ void k_ocbarp(Geo G, BaroFields f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int IE = G.L.ie, JE = G.L.je;
  if (i > IE || j > JE) return;
  const int ij = G.L.at2(i, j);
  if (j >= 1) {
    const double u = f.uso[ij], a = wet(G.gu, ij, 1);
    f.uzo[ij] = u * a;
    f.uso[ij] = u * a;
  }
  if (i >= 1) {
    const double v = f.vse[ij], a = wet(G.gv, ij, 1);
    f.vze[ij] = v * a;
    f.vse[ij] = v * a;
  }
}

// OCWIND (ocwind.f90:20-38): the surface stress on level 1 of UOO and VOE
__global__ void k_ocwind(Geo G, WindFields w, double* __restrict__ uoo, double* __restrict__ voe) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int IE = G.L.ie, JE = G.L.je;
  if (i > IE || j > JE) return;
  const int ij = G.L.at2(i, j);
  const double dtdect = G.dt / G.dzw[0];
  if (i >= 1 && i <= IE - 1 && j >= 2 && j <= JE - 1) {
    const double ur = w.sicomu[ij], a = wet(G.gu, ij, 1);
    uoo[ij] = uoo[ij] + dtdect * a * (w.txo[ij] * ur + (1. - ur) * a * w.tauwatu[ij]);
  }
  if (i >= 2 && i <= IE - 1 && j >= 1 && j <= JE - 1) {
    const double vr = w.sicomv[ij], a = wet(G.gv, ij, 1);
    voe[ij] = voe[ij] + dtdect * a * (w.tye[ij] * vr + (1. - vr) * a * w.tauwatv[ij]);
  }
}

const dim3 kB2(32, 8);

}  // namespace

void launch_trotest_rhs(const Geo& G, const BaroFields& f, cudaStream_t st) {
  k_trotest_rhs<<<grid2(G.L.ie, G.L.je, kB2), kB2, 0, st>>>(G, f);
  count_launch();
}

void launch_sor_trial(const Geo& G, const BaroFields& f, const double* sorpar, double* d2,
                      int parity, cudaStream_t st) {
  const int nx = (G.L.ie - 2 + 1) / 2, ny = G.L.je - 2;
  if (nx < 1 || ny < 1) return;
  k_sor_trial<<<grid2(nx, ny, kB2), kB2, 0, st>>>(G, f, sorpar, d2, parity);
  count_launch();
}

void launch_ocbarp(const Geo& G, const BaroFields& f, cudaStream_t st) {
  k_ocbarp<<<grid2(G.L.ie + 1, G.L.je + 1, kB2), kB2, 0, st>>>(G, f);
  count_launch();
}

void launch_ocwind(const Geo& G, const WindFields& w, double* uoo, double* voe, cudaStream_t st) {
  k_ocwind<<<grid2(G.L.ie + 1, G.L.je + 1, kB2), kB2, 0, st>>>(G, w, uoo, voe);
  count_launch();
}

void launch_itprep(const Geo& G, const BaroArgs& a, const double* deuto, const double* deute,
                   const BaroFields& f, cudaStream_t st) {
  k_itprep<<<grid2(G.L.ie + 1, G.L.je + 1, kB2), kB2, 0, st>>>(G, a, deuto, deute, f);
  count_launch();
  k_itprep_ff<<<grid2(G.L.ie, G.L.je, kB2), kB2, 0, st>>>(G, f);
  count_launch();
}

void launch_troneu_rhs(const Geo& G, const BaroArgs& a, const BaroFields& f, cudaStream_t st) {
  k_troneu_rhs<<<grid2(G.L.ie, G.L.je, kB2), kB2, 0, st>>>(G, a, f);
  count_launch();
}

void launch_sor(const Geo& G, const BaroArgs& a, const BaroFields& f, int parity, cudaStream_t st) {
  const int nx = (G.L.ie - 2 + 1) / 2, ny = G.L.je - 2;
  if (nx < 1 || ny < 1) return;
  k_sor<<<grid2(nx, ny, kB2), kB2, 0, st>>>(G, a, f, parity);
  count_launch();
}

void launch_ocvtro(const Geo& G, const BaroArgs& a, const BaroFields& f, double* zo,
                   cudaStream_t st) {
  k_ocvtro<<<grid2(G.L.ie + 1, G.L.je + 1, kB2), kB2, 0, st>>>(G, a, f, zo);
  count_launch();
}

void launch_ocvtot(const Geo& G, const BaroArgs& a, const double* uso, const double* vse,
                   const double* uoo, const double* voe, const double* uko, const double* vke,
                   double* uoo_o, double* voe_o, double* uko_o, double* vke_o, double* wo_o,
                   cudaStream_t st) {
  const dim3 b(32, 4);
  k_ocvtot<<<grid2(G.L.ie + 1, G.L.je + 1, b), b, 0, st>>>(G, a, uso, vse, uoo, voe, uko, vke,
                                                            uoo_o, voe_o, uko_o, vke_o, wo_o);
  count_launch();
}

}  // namespace orctm
