// Matrix-free Poisson solve of the nonhydrostatic pressure correction
// (petsc_solve_3D / ComputeRHS / compute_matrix, mo_petsc.f90:211-397,
// 543-782).
//
// The operator is never assembled.  Each thread owns one water column and
// loads the column's 2D data once (the neighbours' wet-level counts, which
// decide the land/Neumann/Dirichlet cases, the products of the reciprocal
// metrics XU, XP, YV, YP, and the column's bottom values of ZW, ZP, 1/ZP);
// the per-level coefficients of compute_matrix then follow from 1D tables.
// The matrix costs no HBM traffic.
//
// The solve is iterative refinement: the outer residual r = b - A x is
// accumulated in double-double (error-free FMA products) against the exact
// FP64 matrix entries, and each correction A d = r is solved by
// preconditioned conjugate gradients (FP64, or FP32 for the refined form) on
// the row-scaled operator B = diag(1/ZP) A, whose vertical couplings become
// the symmetric ZW(K) and whose remaining asymmetry is confined to horizontal
// couplings at partial bottom cells.  The preconditioner is the exact
// column-tridiagonal (line) solve of B; its pivots are constant and are
// factorised once at set-up.  A thread applies it to its own column: the
// forward sweep leaves y' in the output vector (L2-resident) and the
// backward sweep overwrites it with z.
//
// Dot products are reduced deterministically: every block writes a partial
// sum and the last block to finish (atomic ticket) adds the partials in
// block order and updates the solver scalars on the device, so an iteration
// needs no host round trip.  A device flag marks convergence; kernels of an
// already converged solve return at once.
#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "ops.h"

namespace orctm {

namespace {

#define AT(a, i, j, K) (a)[G.L.at((i), (j), (K)-1)]

inline dim3 grid2(int nx, int ny, dim3 b) { return dim3((nx + b.x - 1) / b.x, (ny + b.y - 1) / b.y, 1); }
inline dim3 grid3(int nx, int ny, int nz, dim3 b) {
  return dim3((nx + b.x - 1) / b.x, (ny + b.y - 1) / b.y, nz);
}

// ------------------------------------------------------- coefficients ----
struct Coef {
  double dc, w, e, n, s, u, d;  // diagonal, west, east, north, south, up, down
};

// 2D data of one column (i, j), i in [2, IE-1], j in [2, JE-1]
struct ColC {
  long long ij;
  int kb, kbw, kbe, kbn, kbs;
  int kreg;                            // levels 2..kreg have the regular (all-wet) row
  bool iw, ie, in, is;                 // couplings the DMDA allows (not at the domain edge)
  double cw, ce, cn, cs, xcf, ycf;     // XU(I-1)XP, XU(I)XP, YV(J-1)YP, YV(J)YP, sums
  double zwa, zwb, zpa, zpb, zpc, iza, izb, izc;
};

__device__ __forceinline__ ColC load_col(const Geo& G, const PoissonGeo& P, int i, int j) {
  ColC c;
  const int IE = G.L.ie, JE = G.L.je;
  c.ij = G.L.at2(i, j);
  c.kb = G.gp.kb[c.ij];
  c.kbw = G.gp.kb[G.L.at2(i - 1, j)];
  c.kbe = G.gp.kb[G.L.at2(i + 1, j)];
  c.kbn = G.gp.kb[G.L.at2(i, j - 1)];
  c.kbs = G.gp.kb[G.L.at2(i, j + 1)];
  c.iw = i > 2;
  c.ie = i < IE - 1;
  c.in = j > 2;
  c.is = j < JE - 1;
  const double xuw = P.xu[G.L.at2(i - 1, j)], xue = P.xu[c.ij], xp = P.xp[c.ij];
  const double yvn = P.yv[G.L.at2(i, j - 1)], yvs = P.yv[c.ij], yp = P.yp[c.ij];
  c.cw = xuw * xp;
  c.ce = xue * xp;
  c.cn = yvn * yp;
  c.cs = yvs * yp;
  c.xcf = (xuw + xue) * xp;
  c.ycf = (yvn + yvs) * yp;
  c.zwa = P.zwa[c.ij]; c.zwb = P.zwb[c.ij];
  c.zpa = P.zpa[c.ij]; c.zpb = P.zpb[c.ij]; c.zpc = P.zpc[c.ij];
  c.iza = P.iza[c.ij]; c.izb = P.izb[c.ij]; c.izc = P.izc[c.ij];
  // below kreg every neighbour is wet and ZW/ZP are the 1D tables: K < kb - 1
  // keeps K, K+1 and the ZP selections away from the bottom specials
  const int km = min(min(c.kbw, c.kbe), min(c.kbn, c.kbs));
  c.kreg = min(km, c.kb - 2);
  return c;
}

__device__ __forceinline__ double zw_of(const ColC& c, const PoissonGeo& P, int K) {
  if (c.kb >= 1) {
    if (K == c.kb) return c.zwa;
    if (K == c.kb + 1) return c.zwb;
  }
  return P.zwn[K - 1];
}
__device__ __forceinline__ double zp_of(const ColC& c, const PoissonGeo& P, int K) {
  if (c.kb >= 1) {
    if (K == c.kb - 1) return c.zpa;
    if (K == c.kb) return c.zpb;
    if (K == c.kb + 1) return c.zpc;
  }
  return P.zpn[K - 1];
}
__device__ __forceinline__ double izp_of(const ColC& c, const PoissonGeo& P, int K) {
  if (c.kb >= 1) {
    if (K == c.kb - 1) return c.iza;
    if (K == c.kb) return c.izb;
    if (K == c.kb + 1) return c.izc;
  }
  return P.izn[K - 1];
}

// Row K of compute_matrix (mo_petsc.f90:607-767) for the column, entries the
// reference does not insert returned as 0.  With SCALED the row of
// B = diag(1/ZP) A: vertical entries ZW(K), ZW(K+1); horizontal entries and
// X_C, Y_C multiplied by 1/ZP.
template <bool SCALED>
__device__ __forceinline__ Coef row(const ColC& c, const PoissonGeo& P, int K, int KE) {
  const double zw0 = zw_of(c, P, K), zw1 = zw_of(c, P, K + 1);
  const double zp = SCALED ? 1.0 : zp_of(c, P, K);
  const double hs = SCALED ? izp_of(c, P, K) : 1.0;
  Coef r;
  double X_C = c.xcf, Y_C = c.ycf, Z_C = (zw0 + zw1) * zp;
  r.w = r.e = r.n = r.s = r.u = r.d = 0.0;
  if (K > c.kb) {  // land row: diagonal only
    r.dc = SCALED ? -((X_C + Y_C) * hs + Z_C) : -(X_C + Y_C + Z_C);
    return r;
  }
  const bool ww = K <= c.kbw, we = K <= c.kbe, wn = K <= c.kbn, ws = K <= c.kbs;
  if (!ww && we) X_C = c.ce;
  else if (ww && !we) X_C = c.cw;
  else if (!ww && !we) X_C = 0.0;
  if (!wn && ws) Y_C = c.cs;
  else if (wn && !ws) Y_C = c.cn;
  else if (!wn && !ws) Y_C = 0.0;
  const bool wd = K + 1 <= c.kb;
  if (K == 1) {
  } else if (K == KE || !wd) {
    Z_C = zw0 * zp;
  }
  r.dc = SCALED ? -((X_C + Y_C) * hs + Z_C) : -(X_C + Y_C + Z_C);
  if (c.iw && ww) r.w = c.cw * hs;
  if (c.ie && we) r.e = c.ce * hs;
  if (c.in && wn) r.n = c.cn * hs;
  if (c.is && ws) r.s = c.cs * hs;
  if (K != 1) r.u = zw0 * zp;
  if (K != KE && wd) r.d = zw1 * zp;
  return r;
}

// Row K of B for a regular level (2 <= K <= kreg): all six neighbours wet,
// vertical factors from the 1D tables.  Same values as row<true>.
__device__ __forceinline__ Coef row_regular(const ColC& c, const double* zw, const double* iz,
                                            int K) {
  const double zw0 = zw[K - 1], zw1 = zw[K], hs = iz[K - 1];
  Coef r;
  r.u = zw0;
  r.d = zw1;
  r.w = c.iw ? c.cw * hs : 0.0;
  r.e = c.ie ? c.ce * hs : 0.0;
  r.n = c.in ? c.cn * hs : 0.0;
  r.s = c.is ? c.cs * hs : 0.0;
  r.dc = -((c.xcf + c.ycf) * hs + (zw0 + zw1));
  return r;
}

// vertical entries only (the preconditioner's tridiagonal)
template <bool SCALED>
__device__ __forceinline__ double down_of(const ColC& c, const PoissonGeo& P, int K, int KE) {
  if (K > c.kb || K == KE || K + 1 > c.kb) return 0.0;
  const double zw1 = zw_of(c, P, K + 1);
  return SCALED ? zw1 : zw1 * zp_of(c, P, K);
}

// ------------------------------------------------------- reductions ------
// Stores this block's partials; returns true in thread 0 of the last block
// to finish, which then holds the totals (added in block order) in v.
template <int NV>
__device__ bool grid_sum(double (&v)[NV], SolverState* S) {
  __shared__ double sh[NV * 32];
  __shared__ bool last;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
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
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = 0.0;
    for (unsigned b = tid; b < nb; b += nthreads)
      x += ((volatile double*)S->partials)[(size_t)q * S->max_blocks + b];
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

// ------------------------------------------------------- set-up ---------
// Pivots of the column tridiagonal of B (constant): dinv(K) = 1/d'(K) with
// d'(1) = d(1), d'(K) = d(K) - a(K) c(K-1) / d'(K-1).
__global__ void k_factor(Geo G, PoissonGeo P, double* __restrict__ dinv64,
                         float* __restrict__ dinv32) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int KE = G.L.ke;
  if (i > G.L.ie - 1 || j > G.L.je - 1) return;
  const ColC c = load_col(G, P, i, j);
  double dprev = 1.0, cprev = 0.0;
  for (int K = 1; K <= KE; ++K) {
    const Coef r = row<true>(c, P, K, KE);
    const double d = K == 1 ? r.dc : r.dc - (r.u * dprev) * cprev;
    const double di = 1.0 / d;
    AT(dinv64, i, j, K) = di;
    AT(dinv32, i, j, K) = (float)di;
    dprev = di;
    cprev = r.d;
  }
}

// ------------------------------------------------------- PCG kernels -----

// Column kernel: residual update, z = M^-1 r (exact column tridiagonal of B),
// dots r.z and r.r.
//   MODE 1 (init, x = 0):   r = b / ZP   (the right-hand side of B x = b / ZP)
//   MODE 2 (iteration):     x += alpha p ; r -= alpha q
template <typename T, int MODE>
__global__ void __launch_bounds__(128) k_pcg_col(Geo G, PoissonGeo P, SolverState* S,
                                                 const T* __restrict__ b, T* __restrict__ x,
                                                 T* __restrict__ r, const T* __restrict__ p,
                                                 const T* __restrict__ q, T* __restrict__ z) {
  if (S->converged) return;
  const int KE = G.L.ke, IE = G.L.ie, JE = G.L.je;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const double alpha = MODE == 2 ? S->alpha : 0.0;
  // pivots rounded to FP32 in both precisions: a fixed preconditioner that
  // moves half the bytes (the operator apply and the vectors keep precision T)
  const float* __restrict__ dinv = P.dinv32;
  double rz = 0.0, rr = 0.0, bb = 0.0;
  if (i <= IE - 1 && j <= JE - 1) {
    const ColC c = load_col(G, P, i, j);
    double yprev = 0.0, dprev = 0.0;
    const long long base = G.L.at(i, j, 0), plane = G.L.plane;
    constexpr int U = 4;  // levels whose loads are issued together
    for (int K0 = 1; K0 <= KE; K0 += U) {
      double lb[U], lr[U], lp[U], lq[U], lx[U], ld[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int K = K0 + u;
        lb[u] = lr[u] = lp[u] = lq[u] = lx[u] = ld[u] = 0.0;
        if (K <= KE) {
          const long long o = base + plane * (K - 1);
          if (MODE == 1) {
            lb[u] = (double)b[o];
          } else {
            lr[u] = (double)r[o];
            lp[u] = (double)p[o];
            lq[u] = (double)q[o];
            lx[u] = (double)x[o];
          }
          ld[u] = (double)dinv[o];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int K = K0 + u;
        if (K > KE) break;
        const long long o = base + plane * (K - 1);
        double rk;
        if (MODE == 1) {
          rk = lb[u] * izp_of(c, P, K);
          bb += rk * rk;
        } else {
          x[o] = (T)(lx[u] + alpha * lp[u]);
          rk = lr[u] - alpha * lq[u];
        }
        const T rkt = (T)rk;
        r[o] = rkt;
        rk = (double)rkt;
        rr += rk * rk;
        const double up = (K == 1 || K > c.kb) ? 0.0 : zw_of(c, P, K);  // a(K) of B
        const double y = rk - (up * dprev) * yprev;
        z[o] = (T)y;  // y' kept in z until the backward sweep
        yprev = (double)(T)y;
        dprev = ld[u];
      }
    }
    double znext = 0.0;
    for (int K1 = KE; K1 >= 1; K1 -= U) {
      double ly[U], ld[U], lr[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int K = K1 - u;
        ly[u] = ld[u] = lr[u] = 0.0;
        if (K >= 1) {
          const long long o = base + plane * (K - 1);
          ly[u] = (double)z[o];
          ld[u] = (double)dinv[o];
          lr[u] = (double)r[o];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int K = K1 - u;
        if (K < 1) break;
        const double dn = down_of<true>(c, P, K, KE);
        const double zk = (ly[u] - dn * znext) * ld[u];
        const T zt = (T)zk;
        z[base + plane * (K - 1)] = zt;
        znext = (double)zt;
        rz += lr[u] * znext;
      }
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

// Stencil kernel: p = z + beta p_old (first iteration: p = z), q = B p, and
// the dot p.q; alpha = rho / (p.q).  A block of 32 x 4 columns marches down
// the levels; p of its 34 x 6 halo tile is formed once per level into a
// three-level shared-memory ring, and the 7-point product reads the ring.
constexpr int kTx = 32, kTy = 4, kHx = kTx + 2, kHy = kTy + 2;

template <typename T>
__global__ void __launch_bounds__(128) k_pcg_spmv(Geo G, PoissonGeo P, SolverState* S,
                                                  const T* __restrict__ z,
                                                  const T* __restrict__ pold, T* __restrict__ pnew,
                                                  T* __restrict__ q, int first) {
  constexpr int kH = kHx * kHy, kNt = kTx * kTy, kF = (kH + kNt - 1) / kNt;
  __shared__ T ring[3][kH];
  __shared__ double szw[kMaxKe + 1], siz[kMaxKe];
  if (S->converged) return;
  for (int e = threadIdx.x + kTx * threadIdx.y; e <= G.L.ke; e += kTx * kTy) {
    szw[e] = P.zwn[e];
    if (e < G.L.ke) siz[e] = P.izn[e];
  }
  const int KE = G.L.ke, IE = G.L.ie, JE = G.L.je;
  const long long plane = G.L.plane;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kTx * ty;
  const int i0 = blockIdx.x * kTx + 2, j0 = blockIdx.y * kTy + 2;
  const int i = i0 + tx, j = j0 + ty;
  const bool act = i <= IE - 1 && j <= JE - 1;
  const double beta = first ? 0.0 : S->beta;
  // halo-tile entries this thread fills: offsets at level 1, validity
  long long fo[kF];
  int fs[kF];
  bool fv[kF];
#pragma unroll
  for (int f = 0; f < kF; ++f) {
    const int e = tid + f * kNt;
    const int hy = e / kHx, hx = e - hy * kHx;
    const int ii = i0 - 1 + hx, jj = j0 - 1 + hy;
    fs[f] = e < kH ? e : -1;
    fv[f] = e < kH && ii >= 2 && ii <= IE - 1 && jj >= 2 && jj <= JE - 1;
    fo[f] = fv[f] ? G.L.at(ii, jj, 0) : 0;
  }
  // the halo values of two levels ahead are held in registers, so the loads of
  // level K+3 are in flight while level K is computed
  double qz[2][kF], qp[2][kF];
  auto load = [&](int slot, int K) {
#pragma unroll
    for (int f = 0; f < kF; ++f) {
      qz[slot][f] = 0.0;
      qp[slot][f] = 0.0;
      if (fv[f] && K <= KE) {
        const long long o = fo[f] + plane * (K - 1);
        qz[slot][f] = (double)z[o];
        if (!first) qp[slot][f] = (double)pold[o];
      }
    }
  };
  auto store = [&](T* dst, int slot) {
#pragma unroll
    for (int f = 0; f < kF; ++f)
      if (fs[f] >= 0)
        dst[fs[f]] = first ? (T)qz[slot][f] : (T)(qz[slot][f] + beta * qp[slot][f]);
  };
  ColC c;
  if (act) c = load_col(G, P, i, j);
  const long long own = act ? G.L.at(i, j, 0) : 0;
  const int me = (ty + 1) * kHx + (tx + 1);
  T* prv = ring[0];
  T* cur = ring[1];
  T* nxt = ring[2];
  for (int e = threadIdx.x + kTx * threadIdx.y; e < kH; e += kNt) prv[e] = (T)0;
  load(0, 1);
  store(cur, 0);
  load(0, 2);
  load(1, 3);
  double pq = 0.0;
  // one level; SA (the register slot holding level K+1) is a literal at every
  // call so the register queue is never indexed dynamically
  auto level = [&](int K, auto sa_c) {
    constexpr int SA = decltype(sa_c)::value;
    __syncthreads();  // the slot of level K-2 is free; level K is complete
    store(nxt, SA);
    load(SA, K + 3);
    __syncthreads();
    if (act) {
      const Coef rw = (K >= 2 && K <= c.kreg) ? row_regular(c, szw, siz, K) : row<true>(c, P, K, KE);
      const double p0 = (double)cur[me];
      // entries that are not inserted are exactly 0 and their neighbours finite
      double s = rw.dc * p0;
      s = __fma_rn(rw.u, (double)prv[me], s);
      s = __fma_rn(rw.n, (double)cur[me - kHx], s);
      s = __fma_rn(rw.w, (double)cur[me - 1], s);
      s = __fma_rn(rw.e, (double)cur[me + 1], s);
      s = __fma_rn(rw.s, (double)cur[me + kHx], s);
      s = __fma_rn(rw.d, (double)nxt[me], s);
      const long long o = own + plane * (K - 1);
      pnew[o] = (T)p0;
      const T qt = (T)s;
      q[o] = qt;
      pq += p0 * (double)qt;
    }
    T* t = prv;
    prv = cur;
    cur = nxt;
    nxt = t;
  };
  for (int K = 1; K <= KE; K += 2) {
    level(K, std::integral_constant<int, 0>{});
    if (K + 1 <= KE) level(K + 1, std::integral_constant<int, 1>{});
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
    const ColC c = load_col(G, P, i, j);
    double xm = 0.0, x0 = AT(x, i, j, 1), xp = 0.0;
    for (int K = 1; K <= KE; ++K) {
      xp = K < KE ? AT(x, i, j, K + 1) : 0.0;
      const Coef rw = row<false>(c, P, K, KE);
      const double bk = AT(b, i, j, K);
      DD s{bk, 0.0};
      if (rw.u != 0.0) dd_sub_prod(s, rw.u, xm);
      if (rw.n != 0.0) dd_sub_prod(s, rw.n, AT(x, i, j - 1, K));
      if (rw.w != 0.0) dd_sub_prod(s, rw.w, AT(x, i - 1, j, K));
      dd_sub_prod(s, rw.dc, x0);
      if (rw.e != 0.0) dd_sub_prod(s, rw.e, AT(x, i + 1, j, K));
      if (rw.s != 0.0) dd_sub_prod(s, rw.s, AT(x, i, j + 1, K));
      if (rw.d != 0.0) dd_sub_prod(s, rw.d, xp);
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

const dim3 kColBlock(32, 4);

}  // namespace

void launch_factor(const Geo& G, const PoissonGeo& P, double* dinv64, float* dinv32,
                   cudaStream_t st) {
  k_factor<<<grid2(G.L.ie - 2, G.L.je - 2, kColBlock), kColBlock, 0, st>>>(G, P, dinv64, dinv32);
  count_launch();
}

template <typename T, typename TX>
void launch_pcg_col(const Geo& G, const PoissonGeo& P, SolverState* S, int mode, const T* b, TX* x,
                    T* r, const T* p, const T* q, T* z, cudaStream_t st) {
  const dim3 grd = grid2(G.L.ie - 2, G.L.je - 2, kColBlock);
  if (mode == 1)
    k_pcg_col<T, 1><<<grd, kColBlock, 0, st>>>(G, P, S, b, x, r, p, q, z);
  else
    k_pcg_col<T, 2><<<grd, kColBlock, 0, st>>>(G, P, S, b, x, r, p, q, z);
  count_launch();
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
  const dim3 blk(kTx, kTy);
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
  k_resid<<<grid2(G.L.ie - 2, G.L.je - 2, kColBlock), kColBlock, 0, st>>>(G, P, S, b, x, r);
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

size_t solver_max_blocks(const Geo& G) {
  const dim3 g = grid2(G.L.ie - 2, G.L.je - 2, kColBlock);
  return (size_t)g.x * g.y;
}

}  // namespace orctm
