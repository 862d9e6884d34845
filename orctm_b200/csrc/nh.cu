// Nonhydrostatic pressure correction OCVTOT_NH (ocvtot_nh.f90:1-259) with the
// Poisson solve that the reference hands to PETSc (petsc_solve_3D,
// ComputeRHS, compute_matrix: mo_petsc.f90:211-397, 543-782).
//
// The operator is never assembled.  Each kernel regenerates the 7-point
// coefficients of compute_matrix from 2D data: the neighbours' wet-level
// counts (the land/Neumann/Dirichlet cases), the 2D reciprocal metrics XU, XP,
// YV, YP and the vertical factors ZW/ZP, which equal 1D tables except at the
// three levels around each column's bottom, stored per column.  The matrix
// therefore costs no HBM traffic.
//
// The solve is iterative refinement: the outer residual r = b - A x is
// accumulated in double-double (error-free FMA products) against the exact
// FP64 matrix entries, and each correction A d = r is solved by
// preconditioned conjugate gradients (FP64, or FP32 for the refined form) on
// the row-scaled operator B = diag(1/ZP) A, whose vertical couplings become
// the symmetric ZW(K) and whose residual asymmetry is confined to horizontal
// couplings at partial bottom cells.  The preconditioner is the exact
// column-tridiagonal (line) solve, per thread, with the column's
// factorisation in shared memory.  Dot products are reduced
// deterministically: every block writes a partial sum and the last block to
// finish (atomic ticket) adds the partials in block order and updates the
// solver scalars on the device, so an iteration needs no host round trip.
// A device flag marks convergence; later kernels of an already converged
// solve return at once.
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
  const long long ij = G.L.at2(i, j);
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

// ------------------------------------------------------- coefficients ----
struct Coef {
  double dc, w, e, n, s, u, d;  // diagonal, west, east, north, south, up, down
};

__device__ __forceinline__ double zw_at(const PoissonGeo& P, int kb, long long ij, int K) {
  if (kb >= 1) {
    if (K == kb) return P.zwa[ij];
    if (K == kb + 1) return P.zwb[ij];
  }
  return P.zwn[K - 1];
}
__device__ __forceinline__ double zp_at(const PoissonGeo& P, int kb, long long ij, int K) {
  if (kb >= 1) {
    if (K == kb - 1) return P.zpa[ij];
    if (K == kb) return P.zpb[ij];
    if (K == kb + 1) return P.zpc[ij];
  }
  return P.zpn[K - 1];
}
__device__ __forceinline__ double izp_at(const PoissonGeo& P, int kb, long long ij, int K) {
  if (kb >= 1) {
    if (K == kb - 1) return P.iza[ij];
    if (K == kb) return P.izb[ij];
    if (K == kb + 1) return P.izc[ij];
  }
  return P.izn[K - 1];
}

// Row (i,j,K) of compute_matrix (mo_petsc.f90:607-767).  Entries that the
// reference does not insert are returned as 0.  With SCALED the row of
// B = diag(1/ZP) A is returned instead: vertical entries ZW(K), ZW(K+1) and
// horizontal entries (and X_C, Y_C) times 1/ZP.
template <bool SCALED>
__device__ __forceinline__ Coef coef(const Geo& G, const PoissonGeo& P, int i, int j, int K) {
  const int IE = G.L.ie, JE = G.L.je, KE = G.L.ke;
  const long long ij = G.L.at2(i, j);
  const int kb = G.gp.kb[ij];
  const double xuw = P.xu[G.L.at2(i - 1, j)], xue = P.xu[ij], xp = P.xp[ij];
  const double yvn = P.yv[G.L.at2(i, j - 1)], yvs = P.yv[ij], yp = P.yp[ij];
  const double zw0 = zw_at(P, kb, ij, K), zw1 = zw_at(P, kb, ij, K + 1);
  const double zp = SCALED ? 1.0 : zp_at(P, kb, ij, K);
  const double hs = SCALED ? izp_at(P, kb, ij, K) : 1.0;  // horizontal row scale
  Coef c;
  double X_C = (xuw + xue) * xp, Y_C = (yvn + yvs) * yp, Z_C = (zw0 + zw1) * zp;
  c.w = c.e = c.n = c.s = c.u = c.d = 0.0;
  if (K > kb) {  // land row: diagonal only
    c.dc = SCALED ? -((X_C + Y_C) * hs + Z_C) : -(X_C + Y_C + Z_C);
    return c;
  }
  const bool ww = K <= G.gp.kb[G.L.at2(i - 1, j)], we = K <= G.gp.kb[G.L.at2(i + 1, j)];
  const bool wn = K <= G.gp.kb[G.L.at2(i, j - 1)], ws = K <= G.gp.kb[G.L.at2(i, j + 1)];
  if (!ww && we) X_C = xue * xp;
  else if (ww && !we) X_C = xuw * xp;
  else if (!ww && !we) X_C = 0.0;
  if (!wn && ws) Y_C = yvs * yp;
  else if (wn && !ws) Y_C = yvn * yp;
  else if (!wn && !ws) Y_C = 0.0;
  const bool wd = K + 1 <= kb;
  if (K == 1) {
  } else if (K == KE || !wd) {
    Z_C = zw0 * zp;
  }
  c.dc = SCALED ? -((X_C + Y_C) * hs + Z_C) : -(X_C + Y_C + Z_C);
  if (i > 2 && ww) c.w = xuw * xp * hs;
  if (i < IE - 1 && we) c.e = xue * xp * hs;
  if (j > 2 && wn) c.n = yvn * yp * hs;
  if (j < JE - 1 && ws) c.s = yvs * yp * hs;
  if (K != 1) c.u = zw0 * zp;
  if (K != KE && wd) c.d = zw1 * zp;
  return c;
}

template <typename T>
__device__ __forceinline__ double apply_row(const Geo& G, const Coef& c, const T* x, int i, int j,
                                            int K, double xm, double x0, double xp) {
  // CSR column order: up, north, west, centre, east, south, down
  double s = 0.0;
  if (c.u != 0.0) s += c.u * xm;
  if (c.n != 0.0) s += c.n * (double)AT(x, i, j - 1, K);
  if (c.w != 0.0) s += c.w * (double)AT(x, i - 1, j, K);
  s += c.dc * x0;
  if (c.e != 0.0) s += c.e * (double)AT(x, i + 1, j, K);
  if (c.s != 0.0) s += c.s * (double)AT(x, i, j + 1, K);
  if (c.d != 0.0) s += c.d * xp;
  return s;
}

// ------------------------------------------------------- reductions ------
// Stores this block's partials; returns true in the last block to finish, in
// which thread 0 holds the totals (added in block order) in v.
template <int NV>
__device__ bool grid_sum(double (&v)[NV], SolverState* S) {
  __shared__ double sh[NV * 32];
  __shared__ bool last;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  // flatten the thread index for the warp-level reduction
  const int lane = tid & 31, warp = tid >> 5;
  const int nthreads = blockDim.x * blockDim.y;
  const int nw = (nthreads + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[q * 32 + warp] = x;
  }
  __syncthreads();
  const unsigned nb = gridDim.x * gridDim.y;
  const unsigned bid = blockIdx.x + gridDim.x * blockIdx.y;
  if (tid == 0) {
    for (int q = 0; q < NV; ++q) {
      double x = 0.0;
      for (int w = 0; w < nw; ++w) x += sh[q * 32 + w];
      S->partials[(size_t)q * S->max_blocks + bid] = x;
    }
    __threadfence();
    const unsigned t = atomicAdd(&S->ticket, 1u);
    last = (t == nb - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // last block: add partials in block order (deterministic)
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = 0.0;
    for (unsigned b = tid; b < nb; b += nthreads) x += ((volatile double*)S->partials)[(size_t)q * S->max_blocks + b];
    // fixed-order tree over the strided partial sums
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    __syncthreads();
    if (lane == 0) sh[q * 32 + warp] = x;
    __syncthreads();
    if (tid == 0) {
      double y = 0.0;
      for (int w = 0; w < nw; ++w) y += sh[q * 32 + w];
      v[q] = y;
    }
  }
  if (tid == 0) S->ticket = 0;
  return tid == 0;
}

// ------------------------------------------------------- PCG kernels -----
// Column kernel: optional residual update, then z = M^-1 r with the exact
// column tridiagonal solve, then the dots r.z and r.r.
// All on the scaled operator B = diag(1/ZP) A:
//   MODE 0 (init, x given): r = b - B x
//   MODE 1 (init, x = 0):   r = b / ZP   (the right-hand side of B x = b / ZP)
//   MODE 2 (iteration):     x += alpha p ; r -= alpha q
template <typename T, typename TX, int MODE>
__global__ void __launch_bounds__(64) k_pcg_col(Geo G, PoissonGeo P, SolverState* S,
                                                const T* __restrict__ b, TX* __restrict__ x,
                                                T* __restrict__ r, const T* __restrict__ p,
                                                const T* __restrict__ q, T* __restrict__ z) {
  extern __shared__ unsigned char smraw[];
  if (S->converged) return;
  const int KE = G.L.ke, IE = G.L.ie, JE = G.L.je;
  const int tx = threadIdx.x, bw = blockDim.x;
  const int i = blockIdx.x * blockDim.x + tx + 2;
  const int j = blockIdx.y + 2;
  const bool act = i <= IE - 1 && j <= JE - 1;
  T* ys = (T*)smraw;                 // y'(K) per column, [KE][bw]
  T* dv = ys + (size_t)KE * bw;      // 1/d'(K)
  double alpha = 0.0;
  if (MODE == 2) alpha = S->alpha;
  double rz = 0.0, rr = 0.0, bb = 0.0;
  if (act) {
    const long long ij = G.L.at2(i, j);
    const int kb = G.gp.kb[ij];
    double yprev = 0.0, dprev = 1.0, cprev = 0.0;
    double xm = 0.0, x0 = 0.0, xp = 0.0;
    if (MODE == 0) {
      x0 = (double)AT(x, i, j, 1);
    }
    for (int K = 1; K <= KE; ++K) {
      const Coef c = coef<true>(G, P, i, j, K);
      double rk;
      if (MODE == 0) {
        xp = K < KE ? (double)AT(x, i, j, K + 1) : 0.0;
        const double ax = apply_row(G, c, x, i, j, K, xm, x0, xp);
        const double bk = (double)AT(b, i, j, K);
        rk = bk - ax;
        bb += bk * bk;
        xm = x0;
        x0 = xp;
      } else if (MODE == 1) {
        rk = (double)AT(b, i, j, K) * izp_at(P, kb, ij, K);
        bb += rk * rk;
      } else {
        const double pk = (double)AT(p, i, j, K), qk = (double)AT(q, i, j, K);
        AT(x, i, j, K) = (TX)((double)AT(x, i, j, K) + alpha * pk);
        rk = (double)AT(r, i, j, K) - alpha * qk;
      }
      const T rkt = (T)rk;
      AT(r, i, j, K) = rkt;
      rk = (double)rkt;
      rr += rk * rk;
      // forward elimination: a = up coupling, c(K-1) = down coupling of K-1
      double y, d;
      if (K == 1) {
        d = c.dc;
        y = rk;
      } else {
        const double m = c.u * dprev;  // a(K) / d'(K-1)
        d = c.dc - m * cprev;
        y = rk - m * yprev;
      }
      const double dinv = 1.0 / d;
      ys[(size_t)(K - 1) * bw + tx] = (T)y;
      dv[(size_t)(K - 1) * bw + tx] = (T)dinv;
      yprev = y;
      dprev = dinv;
      cprev = c.d;
    }
    // back substitution z(K) = (y'(K) - c(K) z(K+1)) / d'(K)
    double znext = 0.0;
    for (int K = KE; K >= 1; --K) {
      const Coef c = coef<true>(G, P, i, j, K);
      const double zk = ((double)ys[(size_t)(K - 1) * bw + tx] - c.d * znext) *
                        (double)dv[(size_t)(K - 1) * bw + tx];
      const T zt = (T)zk;
      AT(z, i, j, K) = zt;
      znext = (double)zt;
      rz += (double)AT(r, i, j, K) * (double)zt;
    }
  }
  double v[3] = {rz, rr, bb};
  if (grid_sum<3>(v, S)) {
    if (MODE == 2) {
      S->beta = v[0] / S->rho;
    } else {
      S->bb = v[2];
      S->beta = 0.0;
    }
    S->rho = v[0];
    S->rr = v[1];
    S->iter += (MODE == 2);
    if (sqrt(v[1]) <= S->tol * sqrt(S->bb) || S->bb == 0.0) S->converged = 1;
    if (!(v[0] == v[0]) || !(v[1] == v[1])) S->converged = 2;  // NaN: stop
  }
}

// Stencil kernel: p = z + beta p_old (first iteration: p = z), q = A p, and
// the dot p.q; alpha = rho / (p.q).
template <typename T>
__global__ void __launch_bounds__(128) k_pcg_spmv(Geo G, PoissonGeo P, SolverState* S,
                                                  const T* __restrict__ z,
                                                  const T* __restrict__ pold, T* __restrict__ pnew,
                                                  T* __restrict__ q, int first) {
  if (S->converged) return;
  const int KE = G.L.ke, IE = G.L.ie, JE = G.L.je;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const double beta = first ? 0.0 : S->beta;
  double pq = 0.0;
  if (i <= IE - 1 && j <= JE - 1) {
    auto pv = [&](int ii, int jj, int K) -> double {
      const double zz = (double)AT(z, ii, jj, K);
      return first ? zz : (double)(T)(zz + beta * (double)AT(pold, ii, jj, K));
    };
    double pm = 0.0, p0 = pv(i, j, 1), pp = 0.0;
    for (int K = 1; K <= KE; ++K) {
      pp = K < KE ? pv(i, j, K + 1) : 0.0;
      const Coef c = coef<true>(G, P, i, j, K);
      double s = 0.0;
      if (c.u != 0.0) s += c.u * pm;
      if (c.n != 0.0) s += c.n * pv(i, j - 1, K);
      if (c.w != 0.0) s += c.w * pv(i - 1, j, K);
      s += c.dc * p0;
      if (c.e != 0.0) s += c.e * pv(i + 1, j, K);
      if (c.s != 0.0) s += c.s * pv(i, j + 1, K);
      if (c.d != 0.0) s += c.d * pp;
      AT(pnew, i, j, K) = (T)p0;
      const T qt = (T)s;
      AT(q, i, j, K) = qt;
      pq += p0 * (double)qt;
      pm = p0;
      p0 = pp;
    }
  }
  double v[1] = {pq};
  if (grid_sum<1>(v, S)) {
    S->pq = v[0];
    S->alpha = S->rho / v[0];
    if (!(v[0] > 0.0) && !(v[0] < 0.0)) S->converged = 3;  // breakdown
  }
}

// r = b - A x with the exact FP64 entries of compute_matrix, accumulated in
// double-double (products split exactly with an FMA), then rounded once; and
// ||r||^2, ||b||^2.  This is the outer residual of the refinement loop and
// the reported residual.
struct DD {
  double hi, lo;
};
__device__ __forceinline__ void dd_sub_prod(DD& s, double c, double x) {
  const double p = c * x;
  const double pe = __fma_rn(c, x, -p);  // c*x = p + pe exactly
  const double t = s.hi - p;             // two-sum of s.hi and -p
  const double bv = t - s.hi;
  const double e = (s.hi - (t - bv)) + (-p - bv);
  const double lo = s.lo + e - pe;
  const double hi = t + lo;
  s.lo = lo - (hi - t);
  s.hi = hi;
}

__global__ void __launch_bounds__(128) k_resid(Geo G, PoissonGeo P, SolverState* S,
                                               const double* __restrict__ b,
                                               const double* __restrict__ x,
                                               double* __restrict__ r) {
  const int KE = G.L.ke, IE = G.L.ie, JE = G.L.je;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  double rr = 0.0, bb = 0.0;
  if (i <= IE - 1 && j <= JE - 1) {
    double xm = 0.0, x0 = AT(x, i, j, 1), xp = 0.0;
    for (int K = 1; K <= KE; ++K) {
      xp = K < KE ? AT(x, i, j, K + 1) : 0.0;
      const Coef c = coef<false>(G, P, i, j, K);
      const double bk = AT(b, i, j, K);
      DD s{bk, 0.0};
      if (c.u != 0.0) dd_sub_prod(s, c.u, xm);
      if (c.n != 0.0) dd_sub_prod(s, c.n, AT(x, i, j - 1, K));
      if (c.w != 0.0) dd_sub_prod(s, c.w, AT(x, i - 1, j, K));
      dd_sub_prod(s, c.dc, x0);
      if (c.e != 0.0) dd_sub_prod(s, c.e, AT(x, i + 1, j, K));
      if (c.s != 0.0) dd_sub_prod(s, c.s, AT(x, i, j + 1, K));
      if (c.d != 0.0) dd_sub_prod(s, c.d, xp);
      const double rk = s.hi + s.lo;
      if (r) AT(r, i, j, K) = rk;
      rr += rk * rk;
      bb += bk * bk;
      xm = x0;
      x0 = xp;
    }
  }
  double v[2] = {rr, bb};
  if (grid_sum<2>(v, S)) {
    S->res_rr = v[0];
    S->res_bb = v[1];
  }
}

// refinement helpers
__global__ void k_scale_to_f32(Geo G, const double* __restrict__ r, const SolverState* S,
                               float* __restrict__ r32) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int K = blockIdx.z + 1;
  if (i > G.L.ie - 1 || j > G.L.je - 1) return;
  const double s = S->res_rr > 0.0 ? 1.0 / sqrt(S->res_rr) : 0.0;
  AT(r32, i, j, K) = (float)(AT(r, i, j, K) * s);
}

__global__ void k_axpy_f32(Geo G, const float* __restrict__ d, const SolverState* S,
                           double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int K = blockIdx.z + 1;
  if (i > G.L.ie - 1 || j > G.L.je - 1) return;
  const double s = sqrt(S->res_rr);
  AT(x, i, j, K) = AT(x, i, j, K) + s * (double)AT(d, i, j, K);
}

__global__ void k_axpy_f64(Geo G, const double* __restrict__ d, double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int K = blockIdx.z + 1;
  if (i > G.L.ie - 1 || j > G.L.je - 1) return;
  AT(x, i, j, K) = AT(x, i, j, K) + AT(d, i, j, K);
}

__global__ void k_reset(SolverState* S, double tol, int keep_bb) {
  S->converged = 0;
  S->iter = 0;
  S->ticket = 0;
  S->tol = tol;
  S->beta = 0.0;
  if (!keep_bb) S->bb = 0.0;
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
      const long long ij = G.L.at2(i, j);
      u = u + wet(G.gu, ij, K) * G.dtdxuo[ij] * (AT(pnh, i, j, K) - AT(pnh, i + 1, j, K));
    }
    AT(uo, i, j, K) = u;
  }
  if (i >= 1) {
    double v = AT(voe, i, j, K);
    if (i >= 2 && i <= IE - 1 && j >= 1 && j <= JE - 1) {
      const long long ij = G.L.at2(i, j);
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
  const long long ij = G.L.at2(i, j), ijw = G.L.at2(i - 1, j), ijn = G.L.at2(i, j - 1);
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

// columns per block of the column kernel: 64, or 32 when 64 columns of
// factorisation would not fit in shared memory
static int pcg_col_width(const Geo& G, bool f32) {
  const size_t per = (size_t)2 * G.L.ke * (f32 ? sizeof(float) : sizeof(double));
  return per * 64 <= 200 * 1024 ? 64 : 32;
}

size_t pcg_col_smem(const Geo& G, bool f32) {
  return (size_t)2 * G.L.ke * pcg_col_width(G, f32) * (f32 ? sizeof(float) : sizeof(double));
}

template <typename T, typename TX, int MODE>
static void launch_col_mode(const Geo& G, const PoissonGeo& P, SolverState* S, const T* b, TX* x,
                            T* r, const T* p, const T* q, T* z, cudaStream_t st) {
  static int attr_dev = -1;
  static size_t attr_bytes = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t sm = pcg_col_smem(G, sizeof(T) == 4);
  if (attr_dev != dev || sm > attr_bytes) {
    cudaFuncSetAttribute(k_pcg_col<T, TX, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)std::max<size_t>(sm, 48 * 1024));
    attr_dev = dev;
    attr_bytes = std::max<size_t>(sm, 48 * 1024);
  }
  const int bw = pcg_col_width(G, sizeof(T) == 4);
  const dim3 blk(bw, 1);
  const dim3 grd((G.L.ie - 2 + bw - 1) / bw, G.L.je - 2, 1);
  k_pcg_col<T, TX, MODE><<<grd, blk, sm, st>>>(G, P, S, b, x, r, p, q, z);
  count_launch();
}

template <typename T, typename TX>
void launch_pcg_col(const Geo& G, const PoissonGeo& P, SolverState* S, int mode, const T* b, TX* x,
                    T* r, const T* p, const T* q, T* z, cudaStream_t st) {
  if (mode == 0)
    launch_col_mode<T, TX, 0>(G, P, S, b, x, r, p, q, z, st);
  else if (mode == 1)
    launch_col_mode<T, TX, 1>(G, P, S, b, x, r, p, q, z, st);
  else
    launch_col_mode<T, TX, 2>(G, P, S, b, x, r, p, q, z, st);
}
template void launch_pcg_col<double, double>(const Geo&, const PoissonGeo&, SolverState*, int,
                                             const double*, double*, double*, const double*,
                                             const double*, double*, cudaStream_t);
template void launch_pcg_col<float, float>(const Geo&, const PoissonGeo&, SolverState*, int,
                                           const float*, float*, float*, const float*,
                                           const float*, float*, cudaStream_t);

template <typename T>
void launch_pcg_spmv(const Geo& G, const PoissonGeo& P, SolverState* S, const T* z, const T* pold,
                     T* pnew, T* q, int first, cudaStream_t st) {
  const dim3 blk(32, 4);
  k_pcg_spmv<T><<<grid2(G.L.ie - 2, G.L.je - 2, blk), blk, 0, st>>>(G, P, S, z, pold, pnew, q,
                                                                     first);
  count_launch();
}
template void launch_pcg_spmv<double>(const Geo&, const PoissonGeo&, SolverState*, const double*,
                                      const double*, double*, double*, int, cudaStream_t);
template void launch_pcg_spmv<float>(const Geo&, const PoissonGeo&, SolverState*, const float*,
                                     const float*, float*, float*, int, cudaStream_t);

void launch_resid(const Geo& G, const PoissonGeo& P, SolverState* S, const double* b,
                  const double* x, double* r, cudaStream_t st) {
  const dim3 blk(32, 4);
  k_resid<<<grid2(G.L.ie - 2, G.L.je - 2, blk), blk, 0, st>>>(G, P, S, b, x, r);
  count_launch();
}

void launch_scale_to_f32(const Geo& G, const double* r, const SolverState* S, float* r32,
                         cudaStream_t st) {
  const dim3 blk(32, 4);
  k_scale_to_f32<<<grid3(G.L.ie - 2, G.L.je - 2, G.L.ke, blk), blk, 0, st>>>(G, r, S, r32);
  count_launch();
}

void launch_axpy_f32(const Geo& G, const float* d, const SolverState* S, double* x,
                     cudaStream_t st) {
  const dim3 blk(32, 4);
  k_axpy_f32<<<grid3(G.L.ie - 2, G.L.je - 2, G.L.ke, blk), blk, 0, st>>>(G, d, S, x);
  count_launch();
}

void launch_axpy_f64(const Geo& G, const double* d, double* x, cudaStream_t st) {
  const dim3 blk(32, 4);
  k_axpy_f64<<<grid3(G.L.ie - 2, G.L.je - 2, G.L.ke, blk), blk, 0, st>>>(G, d, x);
  count_launch();
}

void launch_solver_reset(SolverState* S, double tol, int keep_bb, cudaStream_t st) {
  k_reset<<<1, 1, 0, st>>>(S, tol, keep_bb);
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
