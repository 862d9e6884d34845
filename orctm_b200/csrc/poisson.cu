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
#include "tma.cuh"

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
  int ij;
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

// vertical entries only (the preconditioner's tridiagonal)
template <bool SCALED>
__device__ __forceinline__ double down_of(const ColC& c, const PoissonGeo& P, int K, int KE) {
  if (K > c.kb || K == KE || K + 1 > c.kb) return 0.0;
  const double zw1 = zw_of(c, P, K + 1);
  return SCALED ? zw1 : zw1 * zp_of(c, P, K);
}

// ------------------------------------------------------- reductions ------
// Every kernel that reduces has blocks of 32 x BY threads, a warp being 32
// consecutive columns i of one row j.  Each warp writes one partial sum at
// its canonical index (row j, 32-column chunk), and the last block to finish
// (atomic ticket) adds the partials in index order with a fixed 64-thread
// pattern, so the totals do not depend on the block shape of the variant that
// ran.  Returns true in thread 0 of the last block, which then holds the
// totals in v.
template <int NV>
__device__ bool grid_sum(double (&v)[NV], SolverState* S) {
  __shared__ double sh[NV * 2];
  __shared__ bool last;
  const int lane = threadIdx.x, tid = threadIdx.x + 32 * threadIdx.y;
  const unsigned nchunk = gridDim.x;
  const unsigned nrow = (unsigned)S->rows;  // JE - 2 rows of unknowns
  const unsigned row = blockIdx.y * blockDim.y + threadIdx.y;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0 && row < nrow) S->partials[(size_t)q * S->max_blocks + row * nchunk + blockIdx.x] = x;
  }
  __threadfence();
  __syncthreads();
  const unsigned nb = gridDim.x * gridDim.y;
  if (tid == 0) {
    const unsigned t = atomicAdd(&S->ticket, 1u);
    last = (t == nb - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  const unsigned n = nrow * nchunk;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = 0.0;
    if (tid < 64)
      for (unsigned b = tid; b < n; b += 64)
        x += ((volatile double*)S->partials)[(size_t)q * S->max_blocks + b];
    if (tid < 64) {
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) sh[q * 2 + (tid >> 5)] = x;
    }
  }
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = sh[q * 2] + sh[q * 2 + 1];
    S->ticket = 0;
  }
  return tid == 0;
}

// The same reduction for blocks whose warps are identified by (row, chunk)
// directly (blocks wider than 32 columns, or with a warp that owns no
// columns: writes = false).  The partial index and the summation order are
// those of grid_sum, so every form's totals agree bit for bit.
template <int NV>
__device__ bool grid_sum_rows(double (&v)[NV], SolverState* S, unsigned row, unsigned chunk,
                              unsigned nchunk, bool writes) {
  __shared__ double sh[NV * 2];
  __shared__ bool last;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y, lane = tid & 31;
  const unsigned nrow = (unsigned)S->rows;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (writes && lane == 0 && row < nrow && chunk < nchunk)
      S->partials[(size_t)q * S->max_blocks + row * nchunk + chunk] = x;
  }
  __threadfence();
  __syncthreads();
  const unsigned nb = gridDim.x * gridDim.y;
  if (tid == 0) {
    const unsigned t = atomicAdd(&S->ticket, 1u);
    last = (t == nb - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  const unsigned n = nrow * nchunk;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = 0.0;
    if (tid < 64)
      for (unsigned b = tid; b < n; b += 64)
        x += ((volatile double*)S->partials)[(size_t)q * S->max_blocks + b];
    if (tid < 64) {
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) sh[q * 2 + (tid >> 5)] = x;
    }
  }
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = sh[q * 2] + sh[q * 2 + 1];
    S->ticket = 0;
  }
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
// The column tridiagonal is symmetric (a(K+1) = c(K) = ZW(K+1)), so
// M = L D L^T with y = L^-1 r from the forward sweep and r.z = sum dinv y^2:
// the dot needs no second pass over r.  With SM the forward values y are
// kept in shared memory ([level][thread], blockDim.x * blockDim.y * KE
// elements) for the backward sweep; otherwise they go through z.
template <typename T, int MODE, bool SM, int U>
__global__ void __launch_bounds__(128) k_pcg_col(Geo G, PoissonGeo P, SolverState* S,
                                                 const T* __restrict__ b, T* __restrict__ x,
                                                 T* __restrict__ r, const T* __restrict__ p,
                                                 const T* __restrict__ q, T* __restrict__ z) {
  extern __shared__ __align__(16) unsigned char col_smem[];
  T* ys = reinterpret_cast<T*>(col_smem);
  __shared__ T szw[kMaxKe + 1];
  if (S->converged) return;
  const int KE = G.L.ke, IE = G.L.ie, JE = G.L.je;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y, nt = blockDim.x * blockDim.y;
  for (int e = tid; e <= KE; e += nt) szw[e] = (T)P.zwn[e];
  __syncthreads();
  // arithmetic in T: the FP32 inner solve computes in FP32 (dots summed in T
  // over U levels, then in FP64)
  const T alpha = MODE == 2 ? (T)S->alpha : T(0);
  // pivots rounded to FP32 in both precisions: a fixed preconditioner that
  // moves half the bytes (the operator apply and the vectors keep precision T)
  const float* __restrict__ dinv = P.dinv32;
  double rz = 0.0, rr = 0.0, bb = 0.0;
  if (i <= IE - 1 && j <= JE - 1) {
    const ColC c = load_col(G, P, i, j);
    const T zwa = (T)c.zwa;
    const int kb = c.kb;
    T yprev = 0, dprev = 0;
    const unsigned base = (unsigned)G.L.at(i, j, 0), plane = (unsigned)G.L.plane;
    // U: levels whose loads are issued together.  Levels below the bottom
    // (K > kb) are land rows: decoupled, right-hand side 0, so every vector
    // holds exact zeros there (k_resid clears x) and their dot terms are +0;
    // they are neither loaded nor stored, while the lanes of a warp still
    // march the levels together (their loads stay coalesced).
    for (int K0 = 1; K0 <= KE; K0 += U) {
      T lb[U], lr[U], lp[U], lq[U], lx[U], ld[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int K = K0 + u;
        lb[u] = lr[u] = lp[u] = lq[u] = lx[u] = ld[u] = T(0);
        if (K <= kb) {
          const unsigned o = base + plane * (unsigned)(K - 1);
          if (MODE == 1) {
            lb[u] = b[o];
          } else {
            lr[u] = r[o];
            lp[u] = p[o];
            lq[u] = q[o];
            lx[u] = x[o];
          }
          ld[u] = (T)dinv[o];
        }
      }
      // partial dots are flushed to FP64 at every fourth level (K = 4, 8, ...)
      // and at the end, whatever U is
      T rzt = 0, rrt = 0, bbt = 0;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int K = K0 + u;
        if (K > KE) break;
        if (u == 4) {
          rz += (double)rzt;
          rr += (double)rrt;
          bb += (double)bbt;
          rzt = rrt = bbt = 0;
        }
        const unsigned o = base + plane * (unsigned)(K - 1);
        T rk;
        const bool wetk = K <= kb;
        if (MODE == 1) {
          rk = (T)((double)lb[u] * izp_of(c, P, K));
          bbt = fma(rk, rk, bbt);
        } else {
          if (wetk) x[o] = fma(alpha, lp[u], lx[u]);
          rk = fma(-alpha, lq[u], lr[u]);
        }
        if (wetk) r[o] = rk;
        rrt = fma(rk, rk, rrt);
        // a(K) of B: ZW(K) above a wet level below the surface
        const T up = (K == 1 || K > kb) ? T(0) : (K == kb ? zwa : szw[K - 1]);
        const T yt = fma(-(up * dprev), yprev, rk);
        if (SM) ys[(K - 1) * nt + tid] = yt;
        else if (wetk) z[o] = yt;  // y kept in z until the backward sweep
        yprev = yt;
        dprev = ld[u];
        rzt = fma(yt * yt, dprev, rzt);
      }
      rz += (double)rzt;
      rr += (double)rrt;
      bb += (double)bbt;
    }
    T znext = 0;
    for (int K1 = KE; K1 >= 1; K1 -= U) {
      T ly[U], ld[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int K = K1 - u;
        ly[u] = ld[u] = T(0);
        if (K >= 1 && K <= kb) {
          const unsigned o = base + plane * (unsigned)(K - 1);
          ly[u] = SM ? ys[(K - 1) * nt + tid] : z[o];
          ld[u] = (T)dinv[o];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int K = K1 - u;
        if (K < 1) break;
        // c(K) of B: ZW(K+1) when level K+1 is wet
        const T dn = (K >= kb || K == KE) ? T(0) : (K + 1 == kb ? zwa : szw[K]);
        const T zt = fma(-dn, znext, ly[u]) * ld[u];
        if (K <= kb) z[base + plane * (unsigned)(K - 1)] = zt;
        znext = zt;
      }
    }
  }
  double v[3] = {rz, rr, bb};
  // warp (row, 32-column chunk) of this thread, for blocks of any width
  const unsigned row = blockIdx.y * blockDim.y + threadIdx.y;
  const unsigned chunk = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
  if (grid_sum_rows<3>(v, S, row, chunk, (unsigned)((IE - 2 + 31) / 32), true)) {
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
// the dot p.q; alpha = rho / (p.q).  A block of 32 x kTy columns marches down
// the levels; p of its 34 x (kTy+2) halo tile is formed once per level into a
// three-level shared-memory ring, and the 7-point product reads the ring.
// Arithmetic is in the storage type T (the FP32 inner solve computes in
// FP32; the dot is accumulated per thread in T over 8 levels, then in FP64).
// Offsets are 32-bit: a padded field has fewer than 2^31 elements
// (checked when the handle is created).
constexpr int kTx = 32;

template <typename T, int kTy>
__global__ void __launch_bounds__(kTx * kTy) k_pcg_spmv(Geo G, PoissonGeo P, SolverState* S,
                                                       const T* __restrict__ z,
                                                       const T* __restrict__ pold,
                                                       T* __restrict__ pnew, T* __restrict__ q,
                                                       int first) {
  constexpr int kHx = kTx + 2, kHy = kTy + 2;
  constexpr int kH = kHx * kHy, kNt = kTx * kTy, kF = (kH + kNt - 1) / kNt;
  __shared__ T ring[3][kH];
  __shared__ T szw[kMaxKe + 1], siz[kMaxKe];
  if (S->converged) return;
  const int KE = G.L.ke, IE = G.L.ie, JE = G.L.je;
  const unsigned plane = (unsigned)G.L.plane;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kTx * ty;
  for (int e = tid; e <= KE; e += kNt) {
    szw[e] = (T)P.zwn[e];
    if (e < KE) siz[e] = (T)P.izn[e];
  }
  const int i0 = blockIdx.x * kTx + 2, j0 = blockIdx.y * kTy + 2;
  const int i = i0 + tx, j = j0 + ty;
  const bool act = i <= IE - 1 && j <= JE - 1;
  const T beta = first ? T(0) : (T)S->beta;
  // the deepest wet level of the block's columns: below it every cell of the
  // block is a land row, whose p and q are exact zeros already in memory and
  // whose dot terms are +0, so the march stops there (loads go one level
  // further, for the level below the deepest wet row)
  __shared__ int skmax;
  if (tid == 0) skmax = 0;
  __syncthreads();
  if (act) atomicMax(&skmax, (int)G.gp.kb[G.L.at2(i, j)]);
  __syncthreads();
  const int kmax = skmax, klim = min(KE, kmax + 1);
  // halo-tile entries this thread fills: offsets at level 1, validity, and
  // the entry's wet levels (below them the values are exact zeros)
  unsigned fo[kF];
  int fs[kF], fk[kF];
  bool fv[kF];
#pragma unroll
  for (int f = 0; f < kF; ++f) {
    const int e = tid + f * kNt;
    const int hy = e / kHx, hx = e - hy * kHx;
    const int ii = i0 - 1 + hx, jj = j0 - 1 + hy;
    fs[f] = e < kH ? e : -1;
    fv[f] = e < kH && ii >= 2 && ii <= IE - 1 && jj >= 2 && jj <= JE - 1;
    fo[f] = fv[f] ? (unsigned)G.L.at(ii, jj, 0) : 0u;
    fk[f] = fv[f] ? (int)G.gp.kb[G.L.at2(ii, jj)] : 0;
  }
  // the halo values of two levels ahead are held in registers, so the loads of
  // level K+3 are in flight while level K is computed
  T qz[2][kF], qp[2][kF];
  auto load = [&](int slot, int K) {
#pragma unroll
    for (int f = 0; f < kF; ++f) {
      qz[slot][f] = T(0);
      qp[slot][f] = T(0);
      if (fv[f] && K <= klim && K <= fk[f]) {
        const unsigned o = fo[f] + plane * (unsigned)(K - 1);
        qz[slot][f] = z[o];
        if (!first) qp[slot][f] = pold[o];
      }
    }
  };
  auto store = [&](T* dst, int slot) {
#pragma unroll
    for (int f = 0; f < kF; ++f)
      if (fs[f] >= 0) dst[fs[f]] = first ? qz[slot][f] : fma(beta, qp[slot][f], qz[slot][f]);
  };
  ColC c;
  T cw = 0, ce = 0, cn = 0, cs = 0, xyc = 0;
  int kreg = 0;
  if (act) {
    c = load_col(G, P, i, j);
    cw = c.iw ? (T)c.cw : T(0);
    ce = c.ie ? (T)c.ce : T(0);
    cn = c.in ? (T)c.cn : T(0);
    cs = c.is ? (T)c.cs : T(0);
    xyc = (T)(c.xcf + c.ycf);
    kreg = c.kreg;
  }
  const unsigned own = act ? (unsigned)G.L.at(i, j, 0) : 0u;
  const int kown = act ? (int)c.kb : 0;
  const int me = (ty + 1) * kHx + (tx + 1);
  T* prv = ring[0];
  T* cur = ring[1];
  T* nxt = ring[2];
  for (int e = tid; e < kH; e += kNt) prv[e] = T(0);
  load(0, 1);
  store(cur, 0);
  load(0, 2);
  load(1, 3);
  double pq = 0.0;
  T pqt = T(0);
  // one level; SA (the register slot holding level K+1) is a literal at every
  // call so the register queue is never indexed dynamically
  auto level = [&](int K, auto sa_c) {
    constexpr int SA = decltype(sa_c)::value;
    __syncthreads();  // the slot of level K-2 is free; level K is complete
    store(nxt, SA);
    load(SA, K + 3);
    __syncthreads();
    // land rows of this column (K > kown): p = 0, q = 0 stays in memory and
    // the dot term is +0, so nothing is formed there
    if (act && K <= kown) {
      const T p0 = cur[me];
      const T pu = prv[me], pn = cur[me - kHx], pw = cur[me - 1], pe = cur[me + 1];
      const T ps = cur[me + kHx], pd = nxt[me];
      T s;
      if (K >= 2 && K <= kreg) {
        // regular row: all six neighbours wet, vertical factors from the tables;
        // B p = hs (cw pw + ce pe + cn pn + cs ps - (xcf+ycf) p0)
        //       + zw0 (pu - p0) + zw1 (pd - p0)
        const T zw0 = szw[K - 1], zw1 = szw[K], hs = siz[K - 1];
        T h = cw * pw;
        h = fma(ce, pe, h);
        h = fma(cn, pn, h);
        h = fma(cs, ps, h);
        h = fma(-xyc, p0, h);
        s = zw0 * (pu - p0);
        s = fma(zw1, pd - p0, s);
        s = fma(hs, h, s);
      } else {
        // entries that are not inserted are exactly 0 and their neighbours finite
        const Coef rw = row<true>(c, P, K, KE);
        s = (T)rw.dc * p0;
        s = fma((T)rw.u, pu, s);
        s = fma((T)rw.n, pn, s);
        s = fma((T)rw.w, pw, s);
        s = fma((T)rw.e, pe, s);
        s = fma((T)rw.s, ps, s);
        s = fma((T)rw.d, pd, s);
      }
      const unsigned o = own + plane * (unsigned)(K - 1);
      pnew[o] = p0;
      q[o] = s;
      pqt = fma(p0, s, pqt);
      if ((K & 7) == 0) {
        pq += (double)pqt;
        pqt = T(0);
      }
    }
    T* t = prv;
    prv = cur;
    cur = nxt;
    nxt = t;
  };
  for (int K = 1; K <= kmax; K += 2) {
    level(K, std::integral_constant<int, 0>{});
    if (K + 1 <= kmax) level(K + 1, std::integral_constant<int, 1>{});
  }
  pq += (double)pqt;
  double v[1] = {pq};
  if (grid_sum<1>(v, S)) {
    S->pq = v[0];
    S->alpha = S->rho / v[0];
    if (!(v[0] > 0.0) && !(v[0] < 0.0)) S->converged = 3;  // breakdown
  }
}

// The same product without shared memory or barriers: every thread forms p
// of its own column and of its four horizontal neighbours from z and p_old
// (the neighbours' lines are shared by the warps of a block through L1), and
// keeps its own p of levels K-1, K, K+1 in registers.  Neighbours outside the
// unknowns hold zeros (the solver vectors are zeroed at allocation and only
// unknowns are written) and meet zero coefficients.
template <typename T, int BY>
__global__ void __launch_bounds__(32 * BY) k_pcg_spmv_l1(Geo G, PoissonGeo P, SolverState* S,
                                                        const T* __restrict__ z,
                                                        const T* __restrict__ pold,
                                                        T* __restrict__ pnew, T* __restrict__ q,
                                                        int first) {
  __shared__ T szw[kMaxKe + 1], siz[kMaxKe];
  if (S->converged) return;
  const int KE = G.L.ke, IE = G.L.ie, JE = G.L.je;
  const unsigned plane = (unsigned)G.L.plane, pitch = (unsigned)G.L.P;
  const int tid = threadIdx.x + 32 * threadIdx.y;
  for (int e = tid; e <= KE; e += 32 * BY) {
    szw[e] = (T)P.zwn[e];
    if (e < KE) siz[e] = (T)P.izn[e];
  }
  __syncthreads();
  const int i = blockIdx.x * 32 + threadIdx.x + 2, j = blockIdx.y * BY + threadIdx.y + 2;
  const bool act = i <= IE - 1 && j <= JE - 1;
  const T beta = first ? T(0) : (T)S->beta;
  double pq = 0.0;
  if (act) {
    const ColC c = load_col(G, P, i, j);
    const T cw = c.iw ? (T)c.cw : T(0), ce = c.ie ? (T)c.ce : T(0);
    const T cn = c.in ? (T)c.cn : T(0), cs = c.is ? (T)c.cs : T(0);
    const T xyc = (T)(c.xcf + c.ycf);
    const int kreg = c.kreg;
    const unsigned o0 = (unsigned)G.L.at(i, j, 0);
    auto pv = [&](unsigned o) -> T { return first ? z[o] : fma(beta, pold[o], z[o]); };
    T pu = T(0), p0 = pv(o0);
    T pqt = T(0);
    for (int K = 1; K <= KE; ++K) {
      const unsigned o = o0 + plane * (unsigned)(K - 1);
      const T pd = K < KE ? pv(o + plane) : T(0);
      const T pw = pv(o - 1), pe = pv(o + 1), pn = pv(o - pitch), ps = pv(o + pitch);
      T s;
      if (K >= 2 && K <= kreg) {
        const T zw0 = szw[K - 1], zw1 = szw[K], hs = siz[K - 1];
        T h = cw * pw;
        h = fma(ce, pe, h);
        h = fma(cn, pn, h);
        h = fma(cs, ps, h);
        h = fma(-xyc, p0, h);
        s = zw0 * (pu - p0);
        s = fma(zw1, pd - p0, s);
        s = fma(hs, h, s);
      } else {
        const Coef rw = row<true>(c, P, K, KE);
        s = (T)rw.dc * p0;
        s = fma((T)rw.u, pu, s);
        s = fma((T)rw.n, pn, s);
        s = fma((T)rw.w, pw, s);
        s = fma((T)rw.e, pe, s);
        s = fma((T)rw.s, ps, s);
        s = fma((T)rw.d, pd, s);
      }
      pnew[o] = p0;
      q[o] = s;
      pqt = fma(p0, s, pqt);
      if ((K & 7) == 0) {
        pq += (double)pqt;
        pqt = T(0);
      }
      pu = p0;
      p0 = pd;
    }
    pq += (double)pqt;
  }
  double v[1] = {pq};
  if (grid_sum<1>(v, S)) {
    S->pq = v[0];
    S->alpha = S->rho / v[0];
    if (!(v[0] > 0.0) && !(v[0] < 0.0)) S->converged = 3;  // breakdown
  }
}

// Warp-row form: a warp holds 32 consecutive columns of one row j and keeps
// its own p of levels K-1, K, K+1 in registers; the west and east neighbours
// come from the adjacent lanes by shuffle (the two edge lanes load theirs),
// the north and south neighbours are formed from z and p_old of rows j-1 and
// j+1 (shared with the neighbouring warps through L1).  No shared-memory tile
// and no barrier in the level loop.  The arithmetic is that of the other
// forms, so the results are the same bit for bit.
template <typename T, int BY>
__global__ void __launch_bounds__(32 * BY) k_pcg_spmv_wr(Geo G, PoissonGeo P, SolverState* S,
                                                        const T* __restrict__ z,
                                                        const T* __restrict__ pold,
                                                        T* __restrict__ pnew, T* __restrict__ q,
                                                        int first) {
  __shared__ T szw[kMaxKe + 1], siz[kMaxKe];
  if (S->converged) return;
  const int KE = G.L.ke, IE = G.L.ie, JE = G.L.je;
  const unsigned plane = (unsigned)G.L.plane, pitch = (unsigned)G.L.P;
  const int lane = threadIdx.x, tid = threadIdx.x + 32 * threadIdx.y;
  for (int e = tid; e <= KE; e += 32 * BY) {
    szw[e] = (T)P.zwn[e];
    if (e < KE) siz[e] = (T)P.izn[e];
  }
  __syncthreads();
  const int i = blockIdx.x * 32 + lane + 2, j = blockIdx.y * BY + threadIdx.y + 2;
  const bool row_ok = j <= JE - 1;           // the same for the whole warp
  const bool in_arr = row_ok && i <= IE;     // column i = IE holds zeros (not an unknown)
  const bool act = row_ok && i <= IE - 1;
  const T beta = first ? T(0) : (T)S->beta;
  double pq = 0.0;
  if (row_ok) {
    ColC c;
    T cw = 0, ce = 0, cn = 0, cs = 0, xyc = 0;
    int kreg = 0;
    if (act) {
      c = load_col(G, P, i, j);
      cw = c.iw ? (T)c.cw : T(0);
      ce = c.ie ? (T)c.ce : T(0);
      cn = c.in ? (T)c.cn : T(0);
      cs = c.is ? (T)c.cs : T(0);
      xyc = (T)(c.xcf + c.ycf);
      kreg = c.kreg;
    }
    const unsigned o0 = in_arr ? (unsigned)G.L.at(i, j, 0) : 0u;
    auto pv = [&](unsigned o) -> T { return first ? z[o] : fma(beta, pold[o], z[o]); };
    T pu = T(0), p0 = in_arr ? pv(o0) : T(0);
    T pqt = T(0);
    for (int K = 1; K <= KE; ++K) {
      const unsigned o = o0 + plane * (unsigned)(K - 1);
      const T pd = (in_arr && K < KE) ? pv(o + plane) : T(0);
      T pn = T(0), ps = T(0);
      if (act) {
        pn = pv(o - pitch);
        ps = pv(o + pitch);
      }
      T pw = __shfl_up_sync(0xffffffffu, p0, 1);
      T pe = __shfl_down_sync(0xffffffffu, p0, 1);
      if (act && lane == 0) pw = pv(o - 1);
      if (act && lane == 31) pe = pv(o + 1);
      if (act) {
        T s;
        if (K >= 2 && K <= kreg) {
          const T zw0 = szw[K - 1], zw1 = szw[K], hs = siz[K - 1];
          T h = cw * pw;
          h = fma(ce, pe, h);
          h = fma(cn, pn, h);
          h = fma(cs, ps, h);
          h = fma(-xyc, p0, h);
          s = zw0 * (pu - p0);
          s = fma(zw1, pd - p0, s);
          s = fma(hs, h, s);
        } else {
          const Coef rw = row<true>(c, P, K, KE);
          s = (T)rw.dc * p0;
          s = fma((T)rw.u, pu, s);
          s = fma((T)rw.n, pn, s);
          s = fma((T)rw.w, pw, s);
          s = fma((T)rw.e, pe, s);
          s = fma((T)rw.s, ps, s);
          s = fma((T)rw.d, pd, s);
        }
        pnew[o] = p0;
        q[o] = s;
        pqt = fma(p0, s, pqt);
        if ((K & 7) == 0) {
          pq += (double)pqt;
          pqt = T(0);
        }
      }
      pu = p0;
      p0 = pd;
    }
    pq += (double)pqt;
  }
  double v[1] = {pq};
  if (grid_sum<1>(v, S)) {
    S->pq = v[0];
    S->alpha = S->rho / v[0];
    if (!(v[0] > 0.0) && !(v[0] < 0.0)) S->converged = 3;  // breakdown
  }
}

// TMA-staged form.  A block of TX x TY consumer threads (one column each)
// and one producer warp marches down the levels.  The producer's first lane
// issues, for every level, tiled bulk-tensor loads of the (TX+4) x (TY+2)
// halo tiles of z and p_old into an NS-stage shared-memory ring (the tile
// starts two columns west of the block so that its first element is 16-byte
// aligned); a stage is refilled once every consumer warp has released it, so
// up to NS-2 levels are in flight ahead of the two the consumers read.
// Consumers form p = z + beta p_old for their column and its four horizontal
// neighbours from the tile, keep p of the level above in a register and read
// the level below from the next stage.  No block-wide barrier in the level
// loop; waits on the stage barriers are bounded (a timeout stops the solve
// with converged = 4).  Positions outside the unknowns hold zeros (the solver
// vectors are zeroed at allocation and only unknowns are written; loads past
// the field's extent are zero-filled) and meet zero coefficients, and the
// arithmetic and dot order equal the other forms', so the results are the
// same bit for bit.
template <typename T, int TX, int TY, int NS>
struct SpmvTma {
  static constexpr int HX = TX + 4, HY = TY + 2;
  static constexpr int kArrBytes = HX * HY * (int)sizeof(T);
  static constexpr int kArrPitch = (kArrBytes + 127) / 128 * 128;
  static constexpr int kStage = 2 * kArrPitch;
  static constexpr int kSmem = NS * kStage + 128;  // + alignment slack
  static constexpr int kConsumers = TX * TY;
  static constexpr int kThreads = kConsumers + 32;
  static_assert(TX % 32 == 0, "a warp covers 32 columns of one row");
  static_assert((HX * sizeof(T)) % 16 == 0, "TMA box rows are whole 16-byte units");
  static_assert(NS >= 3, "two stages are read while at least one loads");
};

// Partial of one warp row (row j, 32-column chunk) at its canonical index,
// summed with the shuffle pattern of grid_sum (a warp's lanes are 32
// consecutive columns).
__device__ __forceinline__ void warp_partial(double x, SolverState* S, unsigned row,
                                             unsigned chunk, unsigned nchunk, int lane) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  if (lane == 0 && row < (unsigned)S->rows && chunk < nchunk)
    S->partials[row * nchunk + chunk] = x;
}

// Totals over all partials by the last block to finish (grid_sum's second
// half): the same index order and 64-thread pattern.
__device__ bool grid_total1(double& v, SolverState* S) {
  __shared__ double sh[2];
  __shared__ bool last;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y, lane = tid & 31;
  __threadfence();
  __syncthreads();
  const unsigned nb = gridDim.x * gridDim.y;
  if (tid == 0) last = (atomicAdd(&S->ticket, 1u) == nb - 1);
  __syncthreads();
  if (!last) return false;
  __threadfence();
  const unsigned n = (unsigned)S->rows * (unsigned)((S->max_blocks) / S->rows);
  double x = 0.0;
  if (tid < 64)
    for (unsigned b = tid; b < n; b += 64) x += ((volatile double*)S->partials)[b];
  if (tid < 64) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[tid >> 5] = x;
  }
  __syncthreads();
  if (tid == 0) {
    v = sh[0] + sh[1];
    S->ticket = 0;
  }
  return tid == 0;
}

// The block walks tiles t = blockIdx.x, blockIdx.x + gridDim.x, ... (one
// tile per block when the grid has a block per tile; a persistent grid of a
// block or two per SM otherwise, so that the producer streams the next
// tile's first levels while the consumers finish the current one and the
// block's set-up is paid once).
template <typename T, int TX, int TY, int NS>
__global__ void __launch_bounds__(TX * TY + 32, 1)
    k_pcg_spmv_tma(Geo G, PoissonGeo P, SolverState* S, const __grid_constant__ CUtensorMap mz,
                   const __grid_constant__ CUtensorMap mpo, T* __restrict__ pnew,
                   T* __restrict__ q, int first) {
  using C = SpmvTma<T, TX, TY, NS>;
  extern __shared__ unsigned char spmv_dsm[];
  __shared__ __align__(8) uint64_t full[NS], empty[NS];
  __shared__ T szw[kMaxKe + 1], siz[kMaxKe];
  if (S->converged) return;
  const int KE = G.L.ke, IE = G.L.ie, JE = G.L.je;
  const unsigned plane = (unsigned)G.L.plane;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntx = (IE - 2 + TX - 1) / TX, nty = (JE - 2 + TY - 1) / TY, ntiles = ntx * nty;
  const unsigned nchunk = (unsigned)((IE - 2 + 31) / 32);
  unsigned char* ring = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(spmv_dsm) + 127) & ~uintptr_t(127));
  auto zt = [&](int s) { return reinterpret_cast<T*>(ring + s * C::kStage); };
  auto pt = [&](int s) { return reinterpret_cast<T*>(ring + s * C::kStage + C::kArrPitch); };
  for (int e = tid; e <= KE; e += C::kThreads) {
    szw[e] = (T)P.zwn[e];
    if (e < KE) siz[e] = (T)P.izn[e];
  }
  if (tid == 0) {
    for (int s = 0; s < NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], C::kConsumers / 32);
    }
    mbar_init_fence();
  }
  __syncthreads();
  bool ok = true;
  if (warp == C::kConsumers / 32) {
    // ---- producer: the whole warp walks the (tile, level) steps so that it
    // reaches the block's later barriers together; its first lane issues
    const uint32_t bytes = (first ? 1u : 2u) * (uint32_t)C::kArrBytes;
    if (lane == 0) {
      tma_prefetch_desc(&mz);
      if (!first) tma_prefetch_desc(&mpo);
    }
    long long g = 0;  // steps issued
    for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
      const int i0 = (t % ntx) * TX + 2, j0 = (t / ntx) * TY + 2;
      for (int K = 1; K <= KE; ++K, ++g) {
        const int s = (int)(g % NS);
        const long long n = g / NS;
        if (n > 0 && !__all_sync(0xffffffffu, mbar_wait(&empty[s], (unsigned)((n - 1) & 1)))) {
          ok = false;
          break;
        }
        if (lane == 0) {
          mbar_arrive_expect_tx(&full[s], bytes);
          tma_load_3d(zt(s), &mz, i0 - 2, j0 - 1, K - 1, &full[s]);
          if (!first) tma_load_3d(pt(s), &mpo, i0 - 2, j0 - 1, K - 1, &full[s]);
        }
        __syncwarp();
      }
    }
    // the block does not exit with copies in flight into its shared memory
    for (long long h = g - NS > 0 ? g - NS : 0; h < g; ++h)
      ok = __all_sync(0xffffffffu, mbar_wait(&full[h % NS], (unsigned)((h / NS) & 1))) && ok;
  } else {
    // ---- consumers
    const int tx = tid % TX, ty = tid / TX;
    const T beta = first ? T(0) : (T)S->beta;
    const int me = (ty + 1) * C::HX + (tx + 2);
    auto pv = [&](int s, int e) -> T {
      return first ? zt(s)[e] : fma(beta, pt(s)[e], zt(s)[e]);
    };
    long long g = 0;  // steps consumed
    for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
      const int i0 = (t % ntx) * TX + 2, j0 = (t / ntx) * TY + 2;
      const int i = i0 + tx, j = j0 + ty;
      const bool act = i <= IE - 1 && j <= JE - 1;
      ColC c;
      T cw = 0, ce = 0, cn = 0, cs = 0, xyc = 0;
      int kreg = 0;
      if (act) {
        c = load_col(G, P, i, j);
        cw = c.iw ? (T)c.cw : T(0);
        ce = c.ie ? (T)c.ce : T(0);
        cn = c.in ? (T)c.cn : T(0);
        cs = c.is ? (T)c.cs : T(0);
        xyc = (T)(c.xcf + c.ycf);
        kreg = c.kreg;
      }
      const unsigned own = act ? (unsigned)G.L.at(i, j, 0) : 0u;
      double pq = 0.0;
      ok = __all_sync(0xffffffffu, mbar_wait(&full[g % NS], (unsigned)((g / NS) & 1)));
      T pu = T(0), p0 = ok ? pv((int)(g % NS), me) : T(0);
      T pqt = T(0);
      for (int K = 1; K <= KE && ok; ++K, ++g) {
        const int s = (int)(g % NS);
        T pd = T(0);
        if (K < KE) {
          const int s1 = (int)((g + 1) % NS);
          if (!__all_sync(0xffffffffu, mbar_wait(&full[s1], (unsigned)(((g + 1) / NS) & 1)))) {
            ok = false;
            break;
          }
          pd = pv(s1, me);
        }
        if (act) {
          const T pw = pv(s, me - 1), pe = pv(s, me + 1);
          const T pn = pv(s, me - C::HX), ps = pv(s, me + C::HX);
          T sv;
          if (K >= 2 && K <= kreg) {
            const T zw0 = szw[K - 1], zw1 = szw[K], hs = siz[K - 1];
            T h = cw * pw;
            h = fma(ce, pe, h);
            h = fma(cn, pn, h);
            h = fma(cs, ps, h);
            h = fma(-xyc, p0, h);
            sv = zw0 * (pu - p0);
            sv = fma(zw1, pd - p0, sv);
            sv = fma(hs, h, sv);
          } else {
            const Coef rw = row<true>(c, P, K, KE);
            sv = (T)rw.dc * p0;
            sv = fma((T)rw.u, pu, sv);
            sv = fma((T)rw.n, pn, sv);
            sv = fma((T)rw.w, pw, sv);
            sv = fma((T)rw.e, pe, sv);
            sv = fma((T)rw.s, ps, sv);
            sv = fma((T)rw.d, pd, sv);
          }
          const unsigned o = own + plane * (unsigned)(K - 1);
          pnew[o] = p0;
          q[o] = sv;
          pqt = fma(p0, sv, pqt);
          if ((K & 7) == 0) {
            pq += (double)pqt;
            pqt = T(0);
          }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        pu = p0;
        p0 = pd;
      }
      pq += (double)pqt;
      // this tile's warp-row partial (a warp is 32 columns of one row)
      warp_partial(pq, S, (unsigned)(j0 - 2 + ty), (unsigned)((i0 - 2 + tx) / 32), nchunk, lane);
    }
  }
  if (!ok) atomicExch(&S->converged, 4);  // a stage wait timed out: stop the solve
  double v = 0.0;
  if (grid_total1(v, S)) {
    S->pq = v;
    S->alpha = S->rho / v;
    if (S->converged == 0 && !(v > 0.0) && !(v < 0.0)) S->converged = 3;  // breakdown
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
                                               double* __restrict__ x,
                                               double* __restrict__ r) {
  const int KE = G.L.ke, IE = G.L.ie, JE = G.L.je;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  double rr = 0.0, bb = 0.0;
  if (i <= IE - 1 && j <= JE - 1) {
    const ColC c = load_col(G, P, i, j);
    // land rows (K > kb): diagonal only with a zero right-hand side, so the
    // solution there is 0; x is set to it and r (0) is not stored, which
    // keeps every solver vector exactly 0 on land for the PCG kernels
    for (int K = c.kb + 1; K <= KE; ++K)
      if (AT(x, i, j, K) != 0.0) AT(x, i, j, K) = 0.0;
    double xm = 0.0, x0 = AT(x, i, j, 1), xp = 0.0;
    for (int K = 1; K <= c.kb; ++K) {
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

__global__ void k_set_limit(SolverState* S, int limit) { S->limit = limit; }

// the last node of the device-side PCG loop's body
__global__ void k_pcg_continue(cudaGraphConditionalHandle hc, const SolverState* S, int chunk) {
  cudaGraphSetConditional(hc, (S->converged == 0 && S->iter + chunk <= S->limit) ? 1u : 0u);
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

// ---------------------------------------------------------- tensor maps
namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (the library does not link libcuda)
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}

constexpr int kTmaTx = 64, kTmaTy = 8, kTmaNs = 6;      // variant 6
constexpr int kTmaTx2 = 32, kTmaTy2 = 8, kTmaNs2 = 8;   // variant 7

template <typename T, int TX, int TY, int NS>
cudaError_t tma_optin() {
  return cudaFuncSetAttribute(k_pcg_spmv_tma<T, TX, TY, NS>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              SpmvTma<T, TX, TY, NS>::kSmem);
}

// persistent: a grid of one block per SM (the kernels fit one block per SM),
// otherwise a block per tile
template <typename T, int TX, int TY, int NS>
int tma_launch(const Geo& G, const PoissonGeo& P, SolverState* S, const T* z, const T* pold,
               T* pnew, T* q, int first, bool persistent, cudaStream_t st) {
  using C = SpmvTma<T, TX, TY, NS>;
  CUtensorMap mz, mp;
  const int e1 = encode_field_map(&mz, z, (int)sizeof(T), G.L.P, G.L.JN, G.L.ke, C::HX, C::HY);
  const int e2 = encode_field_map(&mp, first ? z : pold, (int)sizeof(T), G.L.P, G.L.JN, G.L.ke,
                                  C::HX, C::HY);
  if (e1 || e2) return e1 ? e1 : e2;
  const int ntiles = ((G.L.ie - 2 + TX - 1) / TX) * ((G.L.je - 2 + TY - 1) / TY);
  int nblk = ntiles;
  if (persistent) {
    static int nsm = 0;
    if (!nsm) {
      int dev = 0;
      if (cudaGetDevice(&dev) != cudaSuccess ||
          cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        nsm = 148;
    }
    nblk = ntiles < nsm ? ntiles : nsm;
  }
  k_pcg_spmv_tma<T, TX, TY, NS><<<nblk, C::kThreads, C::kSmem, st>>>(G, P, S, mz, mp, pnew, q,
                                                                      first);
  return 0;
}

}  // namespace

int encode_field_map(CUtensorMap* map, const void* base, int elem_bytes, int P, int JN, int nlev,
                     int bx, int by) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return (int)CUDA_ERROR_NOT_FOUND;
  const cuuint64_t dims[3] = {(cuuint64_t)P, (cuuint64_t)JN, (cuuint64_t)nlev};
  const cuuint64_t strides[2] = {(cuuint64_t)P * elem_bytes, (cuuint64_t)P * JN * elem_bytes};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return (int)fn(map, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

namespace {

// Variants of the column kernel (chosen per handle by the autotuner):
// forward values through the output vector or in shared memory, the number
// of levels whose loads are issued together, and blocks of 32 x 4 columns or
// of 128 consecutive columns of one row (each warp's segment then adjoins its
// neighbours', the same DRAM pages).
struct ColVariant {
  bool sm;
  int u;
  dim3 blk;
};
constexpr int kNumColVariants = 6;
const ColVariant kColVariants[kNumColVariants] = {
    {false, 4, dim3(32, 4)}, {false, 8, dim3(32, 4)}, {true, 4, dim3(32, 2)}, {true, 8, dim3(32, 2)},
    {false, 4, dim3(128, 1)}, {false, 8, dim3(128, 1)}};
// a shared-memory variant is usable while its block's forward values fit here
constexpr size_t kColSmemMax = 96 * 1024;

template <typename T, int MODE, bool SM, int U>
void col_launch(dim3 blk, size_t smem, const Geo& G, const PoissonGeo& P, SolverState* S,
                const T* b, T* x, T* r, const T* p, const T* q, T* z, cudaStream_t st) {
  k_pcg_col<T, MODE, SM, U><<<grid2(G.L.ie - 2, G.L.je - 2, blk), blk, smem, st>>>(G, P, S, b, x,
                                                                                  r, p, q, z);
}

template <typename T, int MODE, int U>
cudaError_t col_optin() {
  return cudaFuncSetAttribute(k_pcg_col<T, MODE, true, U>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kColSmemMax);
}

template <typename T, int SM, int U>
void col_mode(int mode, dim3 blk, size_t smem, const Geo& G, const PoissonGeo& P, SolverState* S,
              const T* b, T* x, T* r, const T* p, const T* q, T* z, cudaStream_t st) {
  if (mode == 1)
    col_launch<T, 1, SM, U>(blk, smem, G, P, S, b, x, r, p, q, z, st);
  else
    col_launch<T, 2, SM, U>(blk, smem, G, P, S, b, x, r, p, q, z, st);
}

}  // namespace

template <typename T>
bool pcg_col_variant_ok(const Geo& G, int variant) {
  if (variant < 0 || variant >= kNumColVariants) return false;
  const ColVariant& v = kColVariants[variant];
  return !v.sm || (size_t)v.blk.x * v.blk.y * G.L.ke * sizeof(T) <= kColSmemMax;
}
template bool pcg_col_variant_ok<double>(const Geo&, int);
template bool pcg_col_variant_ok<float>(const Geo&, int);
int pcg_col_variants() { return kNumColVariants; }

// The shared-memory variants' dynamic shared memory (plus about 2.6 KB of
// static) may exceed the 48 KB default, so their opt-in is raised to the
// variants' fixed maximum on the current device.  Every caller sets the same
// value (the attribute is process-wide per kernel), so handles created on
// several threads never lower it under one another's launches.
cudaError_t pcg_prepare_device() {
  const cudaError_t e[] = {col_optin<double, 1, 4>(), col_optin<double, 2, 4>(),
                           col_optin<double, 1, 8>(), col_optin<double, 2, 8>(),
                           col_optin<float, 1, 4>(),  col_optin<float, 2, 4>(),
                           col_optin<float, 1, 8>(),  col_optin<float, 2, 8>(),
                           tma_optin<double, kTmaTx, kTmaTy, kTmaNs>(),
                           tma_optin<float, kTmaTx, kTmaTy, kTmaNs>(),
                           tma_optin<double, kTmaTx2, kTmaTy2, kTmaNs2>(),
                           tma_optin<float, kTmaTx2, kTmaTy2, kTmaNs2>()};
  for (cudaError_t x : e)
    if (x != cudaSuccess) return x;
  return cudaSuccess;
}

template <typename T, typename TX>
void launch_pcg_col(const Geo& G, const PoissonGeo& P, SolverState* S, int mode, const T* b, TX* x,
                    T* r, const T* p, const T* q, T* z, int variant, cudaStream_t st) {
  if (!pcg_col_variant_ok<T>(G, variant)) variant = 0;
  const ColVariant& v = kColVariants[variant];
  const size_t smem = v.sm ? (size_t)v.blk.x * v.blk.y * G.L.ke * sizeof(T) : 0;
  switch (variant) {
    case 0: case 4: col_mode<T, false, 4>(mode, v.blk, smem, G, P, S, b, x, r, p, q, z, st); break;
    case 1: case 5: col_mode<T, false, 8>(mode, v.blk, smem, G, P, S, b, x, r, p, q, z, st); break;
    case 2: col_mode<T, true, 4>(mode, v.blk, smem, G, P, S, b, x, r, p, q, z, st); break;
    default: col_mode<T, true, 8>(mode, v.blk, smem, G, P, S, b, x, r, p, q, z, st); break;
  }
  count_launch();
}
template void launch_pcg_col<double, double>(const Geo&, const PoissonGeo&, SolverState*, int,
                                             const double*, double*, double*, const double*,
                                             const double*, double*, int, cudaStream_t);
template void launch_pcg_col<float, float>(const Geo&, const PoissonGeo&, SolverState*, int,
                                           const float*, float*, float*, const float*,
                                           const float*, float*, int, cudaStream_t);

// Variants of the stencil kernel: shared-memory ring with 32 x 8 or 32 x 4
// tiles, the barrier-free L1 form, or the warp-row form, each with 32 x 8 or
// 32 x 4 blocks; and the TMA-staged form with 64 x 8 (6 stages) or 32 x 8
// (8 stages) columns per block, a block per tile, and the 64 x 8 form with a
// persistent grid of one block per SM.
int pcg_spmv_variants() { return 9; }

bool pcg_spmv_variant_ok(int variant) {
  if (variant < 0 || variant >= pcg_spmv_variants()) return false;
  return variant < 6 || encode_tiled() != nullptr;
}

// Returns cudaErrorInvalidValue (nothing launched) when a TMA variant's
// tensor maps cannot be encoded.
template <typename T>
cudaError_t launch_pcg_spmv(const Geo& G, const PoissonGeo& P, SolverState* S, const T* z,
                            const T* pold, T* pnew, T* q, int first, int variant,
                            cudaStream_t st) {
  const int nx = G.L.ie - 2, ny = G.L.je - 2;
  switch (variant) {
    case 6:
      if (tma_launch<T, kTmaTx, kTmaTy, kTmaNs>(G, P, S, z, pold, pnew, q, first, false, st))
        return cudaErrorInvalidValue;
      break;
    case 7:
      if (tma_launch<T, kTmaTx2, kTmaTy2, kTmaNs2>(G, P, S, z, pold, pnew, q, first, false, st))
        return cudaErrorInvalidValue;
      break;
    case 8:
      if (tma_launch<T, kTmaTx, kTmaTy, kTmaNs>(G, P, S, z, pold, pnew, q, first, true, st))
        return cudaErrorInvalidValue;
      break;
    case 1:
      k_pcg_spmv<T, 4><<<grid2(nx, ny, dim3(kTx, 4)), dim3(kTx, 4), 0, st>>>(G, P, S, z, pold,
                                                                              pnew, q, first);
      break;
    case 2:
      k_pcg_spmv_l1<T, 8><<<grid2(nx, ny, dim3(32, 8)), dim3(32, 8), 0, st>>>(G, P, S, z, pold,
                                                                               pnew, q, first);
      break;
    case 3:
      k_pcg_spmv_l1<T, 4><<<grid2(nx, ny, dim3(32, 4)), dim3(32, 4), 0, st>>>(G, P, S, z, pold,
                                                                               pnew, q, first);
      break;
    case 4:
      k_pcg_spmv_wr<T, 8><<<grid2(nx, ny, dim3(32, 8)), dim3(32, 8), 0, st>>>(G, P, S, z, pold,
                                                                               pnew, q, first);
      break;
    case 5:
      k_pcg_spmv_wr<T, 4><<<grid2(nx, ny, dim3(32, 4)), dim3(32, 4), 0, st>>>(G, P, S, z, pold,
                                                                               pnew, q, first);
      break;
    default:
      k_pcg_spmv<T, 8><<<grid2(nx, ny, dim3(kTx, 8)), dim3(kTx, 8), 0, st>>>(G, P, S, z, pold,
                                                                              pnew, q, first);
      break;
  }
  count_launch();
  return cudaSuccess;
}
template cudaError_t launch_pcg_spmv<double>(const Geo&, const PoissonGeo&, SolverState*,
                                             const double*, const double*, double*, double*, int,
                                             int, cudaStream_t);
template cudaError_t launch_pcg_spmv<float>(const Geo&, const PoissonGeo&, SolverState*,
                                            const float*, const float*, float*, float*, int, int,
                                            cudaStream_t);

void launch_resid(const Geo& G, const PoissonGeo& P, SolverState* S, const double* b, double* x,
                  double* r, cudaStream_t st) {
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

void launch_set_limit(SolverState* S, int limit, cudaStream_t st) {
  k_set_limit<<<1, 1, 0, st>>>(S, limit);
  count_launch();
}

void launch_pcg_continue(cudaGraphConditionalHandle hc, const SolverState* S, int chunk,
                         cudaStream_t st) {
  k_pcg_continue<<<1, 1, 0, st>>>(hc, S, chunk);
  count_launch();
}

size_t solver_max_blocks(const Geo& G) {
  // one partial per warp row: 32-column chunks x rows of unknowns
  return (size_t)((G.L.ie - 2 + 31) / 32) * (size_t)(G.L.je - 2);
}

}  // namespace orctm
