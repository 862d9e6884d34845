// Open-boundary tide forcing and 1/x sponge relaxation, as mo_obcs.f90 runs
// them with OBC_TIDE on and OBC_SPONGE_EXP off (Makefile:49-50):
//   FORC_OBCS_ETA + SPONGE_OBCS_ETA(ZO)              mo_obcs.f90:569-642, 1561-1720
//   FORC_OBCS_UV + UPGRADE_OBCS_UV + SPONGE_OBCS_UV  mo_obcs.f90:1881-2032, 2295-2582
//   FORC_OBCS_TS + SPONGE_OBCS_TS                    mo_obcs.f90:932-1272
// and, with ObcArgs::expo, the exponential sponge of OBC_SPONGE_EXP
// (SPONGE_OBCS_ETA_EXP, _UV_EXP, _TS_EXP, mo_obcs.f90:2588-3222): the same
// bands and corner rule, each band term mask * mask * DT * M * (boundary -
// X) with the rate M = EXP(-4 L/Lsp)/TAO of a table the host forms.
//
// The reference forms the boundary values (tidal sums), then per open side a
// correction array over its sponge band, sums the four arrays and lets the
// nearer band win in the corners.  Here one thread owns kLz levels of one
// (i, j) column of a staggering and does all of that for its own cells (the
// columns' levels are split over gridDim.z): a cell's position in a
// band is its distance d = 1, 2, ... from the boundary cell of that side
// (west: i + 1 for u-points, i for v- and p-points; north: j + 1 for v-points,
// j otherwise; east IE - i + 1; south JE - j + 1), which gives the weights
// s1 = width - d + 1, s2 = d - 1 of every band loop and the corner rule
// "the band with the smaller d wins, the later corner loop on ties of
// bands" of mo_obcs.f90:1646-1714 and 2453-2566.  Each expression keeps the
// reference's operation order, so the result differs from the CPU
// restatement only through COS (CUDA's cos against the C library's).
// Columns outside every band are not written (the reference adds 0 there).
#include <cuda_runtime.h>

#include "common.cuh"
#include "ops.h"

namespace orctm {
namespace {

enum { FK_P = 0, FK_U = 1, FK_V = 2 };

// One tidal boundary value: sum over td of AM(q,td) * MASK * COS(2 PI (t -
// PH(q,td)) / T(td)) (mo_obcs.f90:578-584, 1893-1899 and the like).
__device__ double tide_sum(const ObcSide& s, int q, double mask, const ObcArgs& a) {
  double v = 0.0;
  for (int td = 0; td < a.ntide; ++td) {
    const int e = q + s.n * td;
    v = v + s.amp[e] * mask * cos(2.0 * a.pi * (a.t - s.pha[e]) / a.period[td]);
  }
  return v;
}

// lambda of a band row (mo_obcs.f90:1578-1583)
__device__ __forceinline__ double band_lambda(double s1, double s2, int w, const ObcArgs& a) {
  const double l = (s1 * a.relb + s2 * a.reli) / (double)w;
  return l != 0.0 ? a.dt / l : 0.0;
}

// levels per thread: the band columns are few, so the levels are spread
// over gridDim.z; a thread forms its columns' tidal sums once for kLz levels
constexpr int kLz = 4;

// CLI: the boundary values are climatology records (FORC_OBCS_TS,
// mo_obcs.f90:964-1012: side.amp holds CLI_T?G as (n, KE), and the value at
// level K is CLI_T?G(q, K) * WETO of the boundary cell at K) instead of tidal
// sums; the field is a 3D p-point tracer (SPONGE_OBCS_TS, mo_obcs.f90:1019-1272).
template <int FK, bool CLI>
__global__ void k_obc_sponge(Geo G, ObcArgs a, double* __restrict__ x) {
  const int IE = G.L.ie, JE = G.L.je;
  const int ilo = FK == FK_U ? 0 : 1, jlo = FK == FK_V ? 0 : 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + ilo;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + jlo;
  if (i > IE || j > JE) return;
  // distances from the four boundary cells of this staggering
  const int dW = FK == FK_U ? i + 1 : i, dE = IE - i + 1;
  const int dN = FK == FK_V ? j + 1 : j, dS = JE - j + 1;
  const bool inW = a.on[0] && dW <= a.width[0], inE = a.on[1] && dE <= a.width[1];
  const bool inN = a.on[2] && dN <= a.width[2], inS = a.on[3] && dS <= a.width[3];
  if (!(inW || inE || inN || inS)) return;
  const ColGeo& c = FK == FK_U ? G.gu : FK == FK_V ? G.gv : G.gp;
  const int iW = ilo, jN = jlo;  // the boundary cells: (iW, j), (IE, j), (i, jN), (i, JE)
  const int ijW = G.L.at2(iW, j), ijE = G.L.at2(IE, j), ijN = G.L.at2(i, jN), ijS = G.L.at2(i, JE);
  const int ij = G.L.at2(i, j);
  // boundary values (FORC_OBCS_*): level-1 masks of the boundary cells
  double zW = 0., zE = 0., zN = 0., zS = 0.;
  if (!CLI) {
    if (inW) zW = tide_sum(a.side[0], j - jlo, wet(c, ijW, 1), a);
    if (inE) zE = tide_sum(a.side[1], j - jlo, wet(c, ijE, 1), a);
    if (inN) zN = tide_sum(a.side[2], i - ilo, wet(c, ijN, 1), a);
    if (inS) zS = tide_sum(a.side[3], i - ilo, wet(c, ijS, 1), a);
  }
  // band weights and relaxation rates
  double s1[4], s2[4], lam[4];
  const int d[4] = {dW, dE, dN, dS};
  const bool in[4] = {inW, inE, inN, inS};
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    s1[b] = (double)(a.width[b] - d[b] + 1);
    s2[b] = (double)(d[b] - 1);
    lam[b] = in[b] && !a.expo ? band_lambda(s1[b], s2[b], a.width[b], a) : 0.0;
  }
  constexpr bool k2d = FK == FK_P && !CLI;  // ZO
  const int nk = k2d ? 1 : G.L.ke;
  const int k0 = (int)blockIdx.z * kLz + 1, k1 = min(nk, k0 + kLz - 1);
  const int q[4] = {j - jlo, j - jlo, i - ilo, i - ilo};  // position along each side
  for (int K = k0; K <= k1; ++K) {
    double* px = k2d ? x + ij : x + G.L.at(i, j, K - 1);
    const double X = *px;
    // the mask products use level K of the cell and its boundary cell; ZO
    // (2D) uses WETO(.,.,1)
    const double mi = wet(c, ij, K);
    const double mb[4] = {wet(c, ijW, K), wet(c, ijE, K), wet(c, ijN, K), wet(c, ijS, K)};
    const double zb[4] = {zW, zE, zN, zS};
    double f[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      f[b] = 0.0;
      if (!in[b]) continue;
      // UPGRADE_OBCS_UV: obc_u*(.,k) = obc_uz*(.) * mask of the boundary cell at
      // k; FORC_OBCS_TS: obc_t*(.,k) = CLI_T*G(.,k) * WETO of the boundary cell
      double ob;
      if (CLI)
        ob = a.side[b].amp[q[b] + a.side[b].n * (K - 1)] * mb[b];
      else
        ob = FK == FK_P ? zb[b] : zb[b] * mb[b];
      if (a.expo) {
        // OBC_SPONGE_EXP: mask * mask * DT * EXP(-4 L/Lsp)/TAO * (boundary - X)
        // (mo_obcs.f90:2641, 2906, 3108 and the like)
        const double m = a.side[b].wexp[q[b] + a.side[b].n * (d[b] - 1)];
        f[b] = mb[b] * mi * a.dt * m * (ob - X);
      } else {
        const double xr = (s1[b] * ob + s2[b] * X) / (double)a.width[b];
        f[b] = mb[b] * mi * lam[b] * (xr - X);
      }
    }
    double fo = f[0] + f[1] + f[2] + f[3];
    if (inW && inN) fo = dW < dN ? f[0] : f[2];
    if (inW && inS) fo = dW < dS ? f[0] : f[3];
    if (inE && inN) fo = dE < dN ? f[1] : f[2];
    if (inE && inS) fo = dE < dS ? f[1] : f[3];
    *px = X + fo;
  }
}

template <int FK, bool CLI = false>
void launch_one(const Geo& G, const ObcArgs& a, double* x, cudaStream_t st) {
  const int ni = FK == FK_U ? G.L.ie + 1 : G.L.ie, nj = FK == FK_V ? G.L.je + 1 : G.L.je;
  const int nk = FK == FK_P && !CLI ? 1 : G.L.ke;
  const dim3 b(32, 8);
  k_obc_sponge<FK, CLI>
      <<<dim3((ni + 31) / 32, (nj + 7) / 8, (nk + kLz - 1) / kLz), b, 0, st>>>(G, a, x);
  count_launch();
}

}  // namespace

void launch_obc_eta(const Geo& G, const ObcArgs& a, double* zo, cudaStream_t st) {
  launch_one<FK_P>(G, a, zo, st);
}

void launch_obc_uv(const Geo& G, const ObcArgs& au, const ObcArgs& av, double* uoo, double* voe,
                   cudaStream_t st) {
  launch_one<FK_U>(G, au, uoo, st);
  launch_one<FK_V>(G, av, voe, st);
}

void launch_obc_ts(const Geo& G, const ObcArgs& a, double* tracer, cudaStream_t st) {
  launch_one<FK_P, true>(G, a, tracer, st);
}

}  // namespace orctm
