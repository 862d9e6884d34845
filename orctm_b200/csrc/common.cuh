// Device layout, geometry views and helpers shared by every kernel.
//
// Every 3D field lives on the device in one padded layout that covers the
// union of the reference's p-, u-, v- and w-point index ranges on a
// single-rank domain:
//     i in [0, IE]   (u-points start at I_start = 0, p/v/w at 1)
//     j in [0, JE]   (v-points start at J_start = 0)
//     level l in [0, KE]  (l = Fortran K-1; w-points use all KE+1 levels)
// offset(i, j, l) = i + P * (j + JN * l), P = IE+1 rounded up to 32 doubles
// (rows start 256-byte aligned, i is the coalescing axis), JN = JE + 1.
// 2D fields use the same (i, j) plane.  Slots a field does not use (i = 0 of
// a p-point field, say) are carried along untouched.
//
// Geometry is stored compressed: BODEN makes every thickness/mask column
// monotone (wet from the surface down to a bottom level, then land), so
//     DDPO(i,j,K) = K <  kb(i,j) ? DZW(K) : K == kb(i,j) ? bot(i,j) : 0
//     WETO(i,j,K) = K <= kb(i,j)
// and likewise DDUO/AMSUO and DDUE/AMSUE: 3D geometry costs no HBM traffic.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace orctm {

constexpr int kMaxKe = 320;  // longest column a handle accepts (the reference runs KE = 300)

struct Layout {
  int ie, je, ke;   // IE, JE, KE (halos included)
  int P, JN;        // pitch (elements) and rows per level
  // Offsets are 32-bit: orctm_create rejects a padded field of 2^31 elements
  // or more, so every offset (and the small negative ones a stencil forms at
  // an array's edge, which land in the allocation's guard zone) fits an int.
  int plane;  // P * JN
  __host__ __device__ int at(int i, int j, int l) const { return i + P * (j + JN * l); }
  __host__ __device__ int at2(int i, int j) const { return i + P * j; }
  __host__ __device__ long long n3() const { return (long long)plane * (ke + 1); }
};

// Compressed column geometry of one staggering (p, u or v points).
struct ColGeo {
  const int* kb;      // number of wet levels (0 = land column)
  const double* bot;  // thickness of the deepest wet level
};

// Read-only geometry view passed by value to kernels.
struct Geo {
  Layout L;
  double dt, dti, almzer, aulapts, aulapuv, minvalue;
  int ob_w, ob_e, ob_n, ob_s;
  ColGeo gp, gu, gv;
  const double* dzw;   // [KE]     DZW(K) at index K-1
  const double* di;    // [KE+1]   DI(K)  at index K-1
  // 2D metrics, padded plane layout
  const double *dlxp, *dlyp, *dlxu, *dlyu, *dlxv, *dlyv;
  const double *dtdxpo, *dtdyo, *dtdxuo, *dpye;
  // biharmonic coefficients and psi-point widths, computed once at set-up
  // exactly as octdiff_base.f90:210-219 and ocvisc.f90:286-327 compute them
  const double *aulx, *auly;                          // AULAPTS*DLXU**4, AULAPTS*DLYV**4 (p plane)
  const double *aulux, *auluy, *aulvx, *aulvy, *aulwx, *aulwy;  // (p plane)
  const double *dlypsi;                               // u-points, i in [0,IE]
  const double *dlxpsi;                               // v-points, j in [0,JE]
  // reciprocals of the metrics (0 where a metric is undefined), so the
  // Laplacian and biharmonic stencils multiply instead of dividing
  const double *rdlxp, *rdlyp, *rdlxu, *rdlyu, *rdlxv, *rdlyv, *rdlxpsi, *rdlypsi;
  // per-face biharmonic coefficients, each shared by the two cells of a face:
  //   tfx = AULX DLYU / DLXU, tfy = AULY DLXV / DLYV           (tracers)
  //   ugx = AULUX DLYP / DLXP, ugy = AULUY DLXPSI / DLYPSI      (u)
  //   vgx = AULVX DLYPSI / DLXPSI, vgy = AULVY DLXP / DLYP      (v)
  //   wgx = AULWX DLYU / DLXU, wgy = AULWY DLXV / DLYV          (w, times DZ)
  // and reciprocal cell areas 1/(DLXU DLYU), 1/(DLXV DLYV), 1/(DLXP DLYP)
  const double *tfx, *tfy, *ugx, *ugy, *vgx, *vgy, *wgx, *wgy;
  const double *rareau, *rareav, *rareap;
};

__device__ __forceinline__ double thick(const ColGeo& c, const double* dzw, int ij, int K) {
  const int kb = c.kb[ij];
  return K < kb ? dzw[K - 1] : (K == kb ? c.bot[ij] : 0.0);
}
__device__ __forceinline__ double wet(const ColGeo& c, int ij, int K) {
  return K <= c.kb[ij] ? 1.0 : 0.0;
}
__device__ __forceinline__ bool wetb(const ColGeo& c, int ij, int K) { return K <= c.kb[ij]; }

// a / b by Newton-Raphson refinement of a hardware reciprocal estimate
// (rcp.approx.ftz.f64), two iterations r <- r + r (1 - b r), then one
// residual correction q <- q + r (a - b q) (the quotient refinement of
// P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Develop. 34 (1990) 111-119).  The
// result is within 1 ulp of the correctly rounded quotient (checked against
// IEEE division by orctm_check_division).  Denominators that are zero,
// subnormal, infinite or NaN take the IEEE division.
__device__ __forceinline__ double div_nr(double a, double b) {
  const double ab = fabs(b);
  if (!(ab >= 1e-300 && ab <= 1e300)) return a / b;
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
  double e = __fma_rn(-b, r, 1.0);
  r = __fma_rn(r, e, r);
  e = __fma_rn(-b, r, 1.0);
  r = __fma_rn(r, e, r);
  const double q = a * r;
  return __fma_rn(r, __fma_rn(-b, q, a), q);
}

// Fortran MAX/MIN for non-NaN operands, evaluated exactly as the oracle does.
__device__ __forceinline__ double fmx(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double fmn(double a, double b) { return b < a ? b : a; }

}  // namespace orctm

#define ORCTM_CUDA_OK(expr)                                   \
  do {                                                        \
    cudaError_t e_ = (expr);                                  \
    if (e_ != cudaSuccess) return orctm::cuda_status(e_);     \
  } while (0)
