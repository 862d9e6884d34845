// Kernel launchers shared between the kernel files and the handle code.
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

#include "common.cuh"

namespace orctm {

// Vertical factors and reciprocal metrics of the matrix-free Poisson operator.
struct PoissonGeo {
  const double *xu, *xp, *yv, *yp;             // 1/DLXU, 1/DLXP, 1/DLYV, 1/DLYP (2D)
  const double *zwa, *zwb;                     // ZW at levels kb and kb+1 (2D)
  const double *zpa, *zpb, *zpc;               // ZP at levels kb-1, kb, kb+1 (2D)
  const double *zwn, *zpn;                     // ZW(K), K=1..KE+1 and ZP(K), K=1..KE elsewhere
  const double *iza, *izb, *izc, *izn;         // 1/ZP = (1/ZW(K) + 1/ZW(K+1))/2, same selection
  const double* dinv64;                        // pivots 1/d'(K) of the column tridiagonal of B (3D)
  const float* dinv32;                         // the same rounded to FP32
};

// Device-resident scalars of one Krylov solve.
struct SolverState {
  double rho, beta, alpha, pq, rr, bb, tol, res_rr, res_bb;
  int converged;  // 0 running, 1 converged, 2 NaN, 3 breakdown, 4 a stage wait timed out
  int iter;
  int limit;      // iteration limit of the device-side loop (orctm handle's maxit)
  unsigned ticket;
  int rows;          // JE - 2: rows of unknowns, the reduction's row count
  int max_blocks;    // partial sums per quantity: 32-column chunks x rows
  double* partials;  // [4 * max_blocks]
};

// Open-boundary tidal constants of one side for one variable (device arrays,
// (n, ntide) column-major: OB{W,E,N,S}{Z,U,V}am / ...ph of mo_obcs.f90:40-46).
constexpr int kObcMaxTides = 8;
struct ObcSide {
  const double* amp;
  const double* pha;
  int n;  // points along the side
  // the exponential sponge's rates (OBC_SPONGE_EXP): wexp[q + n * (d - 1)] =
  // EXP(-4 L/Lsp) / TAO of the band cell at distance d = 1..width from the
  // boundary in row q (mo_obcs.f90:2640 and the like); null in the 1/x form
  const double* wexp;
};
// Arguments of one open-boundary sponge launch (one staggering), by value.
struct ObcArgs {
  int ntide;
  double period[kObcMaxTides];
  double pi, t, dt, relb, reli;  // PI, i_step * DT, DT, rel_*b, rel_*i
  int on[4];                     // west, east, north, south: open and sponged
  int width[4];                  // spongew, spongee, spongen, sponges
  int expo;                      // the exponential sponge (side[b].wexp) instead of 1/x
  ObcSide side[4];
};

// barotropic.cu: constants of the barotropic solve and its 2D device fields
// (padded plane layout)
struct BaroArgs {
  double grav, stabn, conn, rlsa1, sorpar, minvalue;
  int niter, eta_forc;
};
struct BaroFields {
  double *xx, *ff, *b1o, *z1o;            // p-points
  double *uf, *deutio, *u1o, *uzo, *uso;  // u-points
  double *vf, *deutie, *v1e, *vze, *vse;  // v-points
};
// surface forcing of OCWIND (2D, padded plane layout)
struct WindFields {
  double *txo, *tye, *sicomu, *sicomv, *tauwatu, *tauwatv;
};
void launch_ocbarp(const Geo& G, const BaroFields& f, cudaStream_t st);
void launch_trotest_rhs(const Geo& G, const BaroFields& f, cudaStream_t st);
void launch_sor_trial(const Geo& G, const BaroFields& f, const double* sorpar, double* d2,
                      int parity, cudaStream_t st);
void launch_ocwind(const Geo& G, const WindFields& w, double* uoo, double* voe, cudaStream_t st);
void launch_itprep(const Geo& G, const BaroArgs& a, const double* deuto, const double* deute,
                   const BaroFields& f, cudaStream_t st);
void launch_troneu_rhs(const Geo& G, const BaroArgs& a, const BaroFields& f, cudaStream_t st);
void launch_sor(const Geo& G, const BaroArgs& a, const BaroFields& f, int parity, cudaStream_t st);
void launch_ocvtro(const Geo& G, const BaroArgs& a, const BaroFields& f, double* zo,
                   cudaStream_t st);
void launch_ocvtot(const Geo& G, const BaroArgs& a, const double* uso, const double* vse,
                   const double* uoo, const double* voe, const double* uko, const double* vke,
                   double* uoo_o, double* voe_o, double* uko_o, double* vke_o, double* wo_o,
                   cudaStream_t st);

// baroclinic.cu: OCTHER, OCMODMOM, OCCLIT
struct ThermoArgs {
  int eos;  // 0 ADISITJ + RHO1J, 1 linear
  double rho0, drdt, drds, t0, s0;
  double grav, relsal, reltem, rhoicwa, rhosnwa, wt, cstabeps, dv0, av0, cavocon, cdvocon;
};
struct ThermoFields {
  // 1D (device): PREFF[KE], DBACKV / ABACKV [KE+1], WTDECAY[KE] (exp(-DZW/40)
  // from the host's exp), TIESTU / TIESTW / DZ [KE+1]
  const double *preff, *dbackv, *abackv, *wtdecay, *tiestu, *tiestw, *dz;
  // 2D surface forcing (padded plane; zero where the caller gave none)
  const double *sicomo, *sictho, *sicsno, *relsao, *reltho, *giriv, *fu10;
  double *eminpo, *rivrun, *kcondep;  // 2D outputs (KCONDEP as integral doubles)
  double *po, *stabio, *rhoo;         // 3D p-points
};
// Coriolis factors of OCMODMOM per point, formed on the host with its own
// cos/sqrt exactly as the reference writes them (ocmodmom.f90:103-164):
//   u: dtfu = DT FTWOU, cu = DT FTWOU1, dlonu, distu
//   v: dtfv = DT FTWOV, cv = DT FTWOV1, dlonv, distv
//   w: aw = FTWOW1 dlon / dist, bw = FTWOW1 dlat / dist
struct CorFields {
  const double *dtfu, *cu, *dlonu, *distu, *dtfv, *cv, *dlonv, *distv, *aw, *bw;
};
void launch_octher_surface(const Geo& G, const ThermoArgs& a, const ThermoFields& f, double* tho,
                           double* sao, double* zo, cudaStream_t st);
void launch_octher_column(const Geo& G, const ThermoArgs& a, const ThermoFields& f, double* tho,
                          double* sao, const double* zo, const double* uko, const double* vke,
                          double* avo, double* dvo, cudaStream_t st);
// STABIO *= (1000 / DZ): orctm.f90:1443-1449, after OCVTOT
void launch_stabio_rescale(const Geo& G, const ThermoFields& f, cudaStream_t st);
void launch_ocmodmom(const Geo& G, const BaroArgs& b, const ThermoFields& f, const CorFields& c,
                     const BaroFields& bf, const double* zo, const double* uoo, const double* voe,
                     double* uko, double* vke, double* uk1o, double* vk1e, double* wno,
                     double* ub, double* vb, double* wb, double* dw, cudaStream_t st);
// OCCLIT; scratch: wpo, t1o (3D), bruva, contrij (2D); *contra receives the
// sum of CONTRIJ (device scalar)
void launch_occlit(const Geo& G, const BaroArgs& b, const ThermoFields& f, const BaroFields& bf,
                   double* uko, double* vke, double* uk1o, double* vk1e, double* wo, double* wpo,
                   double* t1o, double* bruva, double* contrij, double* contra, cudaStream_t st);

// advect.cu
void launch_ocadpo(const Geo& G, const double* T, const double* uko, const double* vke,
                   const double* wo, const double* zo, double* out, double* tA, double* vA,
                   double* vB, cudaStream_t st);
// OCADPO for ntr tracers at once (shared transports and volumes); equals
// ntr launch_ocadpo calls bit for bit
void launch_ocadpo_all(const Geo& G, int ntr, const double* const* T, double* const* out,
                       double* const* mid, const double* uko, const double* vke,
                       const double* wo, const double* zo, double* vA, double* vB,
                       cudaStream_t st);
int adpo_max_fused();
void launch_ocuad(const Geo& G, const double* T, const double* uko, const double* vke,
                  const double* wo, double* out, double* tA, double* vA, double* vB,
                  cudaStream_t st);
void launch_ocvad(const Geo& G, const double* T, const double* uko, const double* vke,
                  const double* wo, double* out, double* tA, double* vA, double* vB,
                  cudaStream_t st);
void launch_ocwad(const Geo& G, const double* T, const double* uko, const double* vke,
                  const double* wo, const double* zo, double* out, double* tA, double* vA,
                  double* vB, cudaStream_t st);

// diffuse.cu
void launch_octdiff_vert(const Geo& G, int ntr, const double* const* in, double* const* out,
                         const double* dvo, const double* zo, cudaStream_t st);
// Laplacian + biharmonic of OCTDIFF_TS for every tracer, fused (no scratch field)
void launch_octdiff_hbih(const Geo& G, int ntr, const double* const* in, double* const* out,
                         const double* zo, cudaStream_t st);
void launch_ocvisc(const Geo& G, const double* uoo, const double* voe, const double* wno,
                   const double* uko, const double* vke, const double* avo, double* spu,
                   double* spv, double* ukv, double* vkv, double* wnv, double* u1, double* v1,
                   double* w1, double* uo, double* vo, double* wo, cudaStream_t st);

// obc.cu: FORC_OBCS_ETA + SPONGE_OBCS_ETA on ZO, and FORC_OBCS_UV +
// UPGRADE_OBCS_UV + SPONGE_OBCS_UV on UOO / VOE, in place
void launch_obc_eta(const Geo& G, const ObcArgs& a, double* zo, cudaStream_t st);
void launch_obc_uv(const Geo& G, const ObcArgs& au, const ObcArgs& av, double* uoo, double* voe,
                   cudaStream_t st);
// FORC_OBCS_TS + SPONGE_OBCS_TS on one tracer: a.side[s].amp holds side s's
// climatology record (n, KE)
void launch_obc_ts(const Geo& G, const ObcArgs& a, double* tracer, cudaStream_t st);

// nh.cu
void launch_nh_rhs(const Geo& G, const double* uoo, const double* uoo1, const double* voe,
                   const double* voe1, const double* wno, const double* wno1, const double* zo,
                   double* b, cudaStream_t st);
// poisson.cu
void launch_factor(const Geo& G, const PoissonGeo& P, double* dinv64, float* dinv32,
                   cudaStream_t st);
size_t solver_max_blocks(const Geo& G);
template <typename T, typename TX>
void launch_pcg_col(const Geo& G, const PoissonGeo& P, SolverState* S, int mode, const T* b, TX* x,
                    T* r, const T* p, const T* q, T* z, int variant, cudaStream_t st);
template <typename T>
cudaError_t launch_pcg_spmv(const Geo& G, const PoissonGeo& P, SolverState* S, const T* z,
                            const T* pold, T* pnew, T* q, int first, int variant,
                            cudaStream_t st);
// kernel variants the autotuner chooses between (a variant a grid cannot use
// falls back to variant 0)
int pcg_col_variants();
// raises the shared-memory opt-in of the column-kernel variants on the
// current device (called once per handle at creation)
cudaError_t pcg_prepare_device();
template <typename T>
bool pcg_col_variant_ok(const Geo& G, int variant);
int pcg_spmv_variants();
bool pcg_spmv_variant_ok(int variant);
// r = b - A x in double-double, and x := 0 on land rows (their solution)
void launch_resid(const Geo& G, const PoissonGeo& P, SolverState* S, const double* b, double* x,
                  double* r, cudaStream_t st);
void launch_axpy_f64(const Geo& G, const double* d, double* x, cudaStream_t st);
void launch_scale_to_f32(const Geo& G, const double* r, const SolverState* S, float* r32,
                         cudaStream_t st);
void launch_axpy_f32(const Geo& G, const float* d, const SolverState* S, double* x,
                     cudaStream_t st);
void launch_solver_reset(SolverState* S, double tol, int keep_bb, cudaStream_t st);
// device-side PCG loop: the limit of iterations, and the kernel that ends a
// while-node body (keep looping while not converged and a further chunk of
// `chunk` iterations stays within the limit)
void launch_set_limit(SolverState* S, int limit, cudaStream_t st);
void launch_pcg_continue(cudaGraphConditionalHandle hc, const SolverState* S, int chunk,
                         cudaStream_t st);
void launch_nh_post(const Geo& G, const double* x, const double* pold, double* pnh,
                    const double* uoo, const double* voe, double* uo, double* vo, double* wno,
                    cudaStream_t st);

int cuda_status(cudaError_t e);
// message of the calling thread's last failed call made without a handle,
// returned by orctm_last_error(NULL); cleared at the start of such calls
void set_unbound_error(const char* msg);
void clear_unbound_errors();

// number of kernels launched by this library (all handles, this process)
void count_launch();
void add_launches(long long n);  // kernels run by a replayed graph (negative: undo a capture's count)
unsigned long long launch_count();

}  // namespace orctm
