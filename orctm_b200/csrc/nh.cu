// Nonhydrostatic pressure correction OCVTOT_NH (ocvtot_nh.f90:1-259) around
// the Poisson solve (poisson.cu): the right-hand side DIVG*WETO
// (ocvtot_nh.f90:11-62, ComputeRHS mo_petsc.f90:298-376) and, after the
// solve, the open-boundary PNH fill, the u/v pressure-gradient correction and
// the continuity re-diagnosis of WNO (ocvtot_nh.f90:150-236).
#include <algorithm>

#include "common.cuh"
#include "ops.h"

namespace orctm {

namespace {

#define AT(a, i, j, K) (a)[G.L.at((i), (j), (K)-1)]

inline dim3 grid2(int nx, int ny, dim3 b) { return dim3((nx + b.x - 1) / b.x, (ny + b.y - 1) / b.y, 1); }
inline dim3 grid3(int nx, int ny, int nz, dim3 b) {
  return dim3((nx + b.x - 1) / b.x, (ny + b.y - 1) / b.y, nz);
}

// ------------------------------------------------------------ RHS --------
// b = DIVG * WETO for the interior cells (ocvtot_nh.f90:11-62,
// mo_petsc.f90:298-376); other entries of b are left untouched (zero).
__global__ void k_nh_rhs(Geo G, const double* __restrict__ uoo, const double* __restrict__ uoo1,
                         const double* __restrict__ voe, const double* __restrict__ voe1,
                         const double* __restrict__ wno, const double* __restrict__ wno1,
                         const double* __restrict__ zo, double* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int K = blockIdx.z + 1;
  const int IE = G.L.ie, JE = G.L.je;
  if (i > IE - 1 || j > JE - 1) return;
  const double DT = G.dt;
  const int ij = G.L.at2(i, j);
  const double gu0 = (AT(uoo, i, j, K) - AT(uoo1, i, j, K)) / DT;
  const double gum = (AT(uoo, i - 1, j, K) - AT(uoo1, i - 1, j, K)) / DT;
  const double divgu = (gu0 - gum) / G.dlxp[ij];
  const double gvm = (AT(voe, i, j - 1, K) - AT(voe1, i, j - 1, K)) / DT;
  const double gv0 = (AT(voe, i, j, K) - AT(voe1, i, j, K)) / DT;
  const double divgv = (gvm - gv0) / G.dlyp[ij];
  const double gw0 = (AT(wno, i, j, K) - AT(wno1, i, j, K)) / DT;
  const double gw1 = (AT(wno, i, j, K + 1) - AT(wno1, i, j, K + 1)) / DT;
  double divgw;
  if (K >= 2)
    divgw = (gw0 - gw1) / fmx(thick(G.gp, G.dzw, ij, K), 1.E-3);
  else
    divgw = (gw0 - gw1) / (fmx(thick(G.gp, G.dzw, ij, 1), 1.E-3) + zo[ij]);
  const double divg = divgu + divgv + divgw;
  AT(b, i, j, K) = divg * wet(G.gp, ij, K);
}

// ------------------------------------------------------- post solve -----
// PNH: interior from the solution, open-boundary halo copied from the first
// interior row/column (ocvtot_nh.f90:154-186), the rest kept.
__global__ void k_nh_pnh(Geo G, const double* __restrict__ x, const double* __restrict__ pold,
                         double* __restrict__ pnh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int K = blockIdx.z + 1;
  const int IE = G.L.ie, JE = G.L.je;
  if (i > IE || j > JE) return;
  auto inner = [&](int ii, int jj) { return ii >= 2 && ii <= IE - 1 && jj >= 2 && jj <= JE - 1; };
  // value after the west/east fill (J = 2..JE1)
  auto we_fill = [&](int ii, int jj) -> double {
    if (inner(ii, jj)) return AT(x, ii, jj, K);
    if (jj >= 2 && jj <= JE - 1) {
      if (ii == 1 && G.ob_w) return AT(x, 2, jj, K);
      if (ii == IE && G.ob_e) return AT(x, IE - 1, jj, K);
    }
    return AT(pold, ii, jj, K);
  };
  double v = we_fill(i, j);
  if (j == 1 && G.ob_n) v = we_fill(i, 2);
  if (j == JE && G.ob_s) v = we_fill(i, JE - 1);
  AT(pnh, i, j, K) = v;
}

// u/v correction by the pressure gradient (ocvtot_nh.f90:189-203)
__global__ void k_nh_uv(Geo G, const double* __restrict__ pnh, const double* __restrict__ uoo,
                        const double* __restrict__ voe, double* __restrict__ uo,
                        double* __restrict__ vo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int K = blockIdx.z + 1;
  const int IE = G.L.ie, JE = G.L.je;
  if (i > IE || j > JE) return;
  if (j >= 1) {
    double u = AT(uoo, i, j, K);
    if (i >= 1 && i <= IE - 1 && j >= 2 && j <= JE - 1) {
      const int ij = G.L.at2(i, j);
      u = u + wet(G.gu, ij, K) * G.dtdxuo[ij] * (AT(pnh, i, j, K) - AT(pnh, i + 1, j, K));
    }
    AT(uo, i, j, K) = u;
  }
  if (i >= 1) {
    double v = AT(voe, i, j, K);
    if (i >= 2 && i <= IE - 1 && j >= 1 && j <= JE - 1) {
      const int ij = G.L.at2(i, j);
      v = v + wet(G.gv, ij, K) * G.dpye[ij] * (AT(pnh, i, j + 1, K) - AT(pnh, i, j, K));
    }
    AT(vo, i, j, K) = v;
  }
}

// WNO re-diagnosed from continuity, bottom up (ocvtot_nh.f90:215-236)
__global__ void k_nh_w(Geo G, const double* __restrict__ uoo, const double* __restrict__ voe,
                       double* __restrict__ wno) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  if (i > IE || j > JE) return;
  const int ij = G.L.at2(i, j), ijw = G.L.at2(i - 1, j), ijn = G.L.at2(i, j - 1);
  double w = 0.0;
  AT(wno, i, j, KE + 1) = 0.0;
  for (int K = KE; K >= 1; --K) {
    const double we = wet(G.gp, ij, K);
    w = w +
        G.dti * we *
            (G.dtdxpo[ij] *
             (AT(uoo, i - 1, j, K) * thick(G.gu, G.dzw, ijw, K) * G.dlyu[ijw] -
              AT(uoo, i, j, K) * thick(G.gu, G.dzw, ij, K) * G.dlyu[ij]) /
             G.dlyp[ij]) +
        G.dti * we *
            (+G.dtdyo[ij] *
             (AT(voe, i, j, K) * thick(G.gv, G.dzw, ij, K) * G.dlxv[ij] -
              AT(voe, i, j - 1, K) * thick(G.gv, G.dzw, ijn, K) * G.dlxv[ijn]) /
             G.dlxp[ij]);
    AT(wno, i, j, K) = w;
  }
}

}  // namespace

void launch_nh_rhs(const Geo& G, const double* uoo, const double* uoo1, const double* voe,
                   const double* voe1, const double* wno, const double* wno1, const double* zo,
                   double* b, cudaStream_t st) {
  const dim3 bk(32, 4);
  k_nh_rhs<<<grid3(G.L.ie - 2, G.L.je - 2, G.L.ke, bk), bk, 0, st>>>(G, uoo, uoo1, voe, voe1, wno,
                                                                     wno1, zo, b);
  count_launch();
}


void launch_nh_post(const Geo& G, const double* x, const double* pold, double* pnh,
                    const double* uoo, const double* voe, double* uo, double* vo, double* wno,
                    cudaStream_t st) {
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  const dim3 b3(32, 4), b2(32, 4);
  k_nh_pnh<<<grid3(IE, JE, KE, b3), b3, 0, st>>>(G, x, pold, pnh);
  count_launch();
  k_nh_uv<<<grid3(IE + 1, JE + 1, KE, b3), b3, 0, st>>>(G, pnh, uoo, voe, uo, vo);
  count_launch();
  k_nh_w<<<grid2(IE, JE, b2), b2, 0, st>>>(G, uo, vo, wno);
  count_launch();
}

}  // namespace orctm
