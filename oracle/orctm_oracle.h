/*
 * CPU restatement (oracle) of ORCTM's nonhydrostatic hot path.
 *
 * TEST INFRASTRUCTURE ONLY: this library is the checker that the CUDA path is
 * compared against, and the CPU baseline that bench.py times.  Nothing in the
 * product (orctm_b200/, include/) links or calls it.
 *
 * PARITY PINNED ONLY IN PART: the reference (Fortran 90 + PETSc 3.10.2 +
 * MPI) cannot be compiled here and ships no golden outputs or tests.  The
 * values the reference does hold pin it: the equation of state's check
 * values (adisitj.f90:48-51 and the UNESCO 1981 values of RHO1J) and the
 * reference's own input files (the Sect. 3.3 tank's grid, T/S and forcing,
 * the Sect. 3.5 boundary constants and climatology), which tests run through
 * this restatement.  Beyond those it is checked against itself (golden
 * fixtures it generated, an independent numpy restatement of every routine,
 * and property tests).
 *
 * Arrays use the reference's Fortran layout (column-major, i fastest) with its
 * halos and index origins on a single-rank domain (I_start = J_start = 0):
 *   p-points  X(1:IE, 1:JE, 1:KE)      u-points X(0:IE, 1:JE, 1:KE)
 *   v-points  X(1:IE, 0:JE, 1:KE)      w-points X(1:IE, 1:JE, 1:KE+1)
 *   2D arrays analogous (p: IE*JE, u: (IE+1)*JE, v: IE*(JE+1)).
 * All arithmetic is IEEE binary64, evaluated in the textual (left-to-right)
 * order of the Fortran source; compile with -ffp-contract=off.
 */
#ifndef ORCTM_ORACLE_H
#define ORCTM_ORACLE_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct og_grid {
  int ie, je, ke;              /* IE, JE, KE including the 1-cell halo */
  int ob_west, ob_east, ob_north, ob_south; /* open-boundary switches (mo_obcs.f90:9-20) */
  double dt, almzer, aulapts, aulapuv, ah00;
  /* 1D vertical grid, 1-based in the comments: DZW(KE), DI(KEP), DZ(KEP), TIESTU(KEP), TIESTW(KEP) */
  const double *dzw, *di, *dz, *tiestu, *tiestw;
  /* 2D metrics */
  const double *dlxp, *dlyp, *dtdxpo, *dtdyo;        /* p: IE*JE */
  const double *dlxu, *dlyu, *dtdxuo, *dpyo;         /* u: (IE+1)*JE */
  const double *dlxv, *dlyv, *dtdxue, *dpye;         /* v: IE*(JE+1) */
  /* 3D geometry (BODEN) */
  const double *ddpo, *weto;                         /* p: IE*JE*KE */
  const double *dduo, *amsuo;                        /* u: (IE+1)*JE*KE */
  const double *ddue, *amsue;                        /* v: IE*(JE+1)*KE */
} og_grid;

/* BELEG (beleg.f90:48-139) + BODEN (boden.f90:38-286) restated.  depto is
 * modified in place exactly as BODEN does (ISTART == 0 branch).  Outputs are
 * caller-allocated in the layouts above; tiestu/tiestw/dz/di have KE+1
 * entries, dwi KE. */
void og_build_grid(int ie, int je, int ke, double dt, const double *dzw,
                   double *depto,
                   const double *dlxp, const double *dlyp,
                   const double *dlxu, const double *dlyu,
                   const double *dlxv, const double *dlyv,
                   double *tiestu, double *tiestw, double *dz, double *di,
                   double *dtdxpo, double *dtdyo, double *dtdxuo, double *dpyo,
                   double *dtdxue, double *dpye,
                   double *ddpo, double *weto, double *dduo, double *amsuo,
                   double *ddue, double *amsue);

/* Hot-path routines (in/out arrays in reference layout). */
void og_ocadpo(const og_grid *g, double *trf, const double *uko, const double *vke,
               const double *wo, const double *zo);
void og_ocuad(const og_grid *g, double *uoo, const double *uko, const double *vke,
              const double *wo);
void og_ocvad(const og_grid *g, double *voe, const double *uko, const double *vke,
              const double *wo);
void og_ocwad(const og_grid *g, double *wno, const double *uko, const double *vke,
              const double *wo, const double *zo);
void og_octdiff(const og_grid *g, int ntr, double *const *tr, const double *dvo,
                const double *zo);
void og_ocvisc(const og_grid *g, double *uoo, double *voe, double *wno,
               double *uko, double *vke, const double *avo);

/* OCVTOT_NH, split around the solve.  b has (IE-2)*(JE-2)*KE entries in PETSc
 * DMDA natural order (x fastest). */
void og_nh_rhs(const og_grid *g, const double *uoo, const double *uoo1,
               const double *voe, const double *voe1, const double *wno,
               const double *wno1, const double *zo, double *b);
/* Number of stored entries of the compute_matrix operator. */
size_t og_matrix_nnz(const og_grid *g);
/* compute_matrix (mo_petsc.f90:543-782) as CSR over the DMDA natural order. */
void og_matrix_csr(const og_grid *g, int *rowptr, int *colind, double *val);
/* Writes the solve's x into PNH interior, fills the open-boundary halo,
 * corrects u/v, re-diagnoses WNO and rotates the _1 copies (ocvtot_nh.f90:150-255). */
void og_nh_post(const og_grid *g, const double *x, double *pnh, double *uoo,
                double *voe, double *wno, double *uoo1, double *voe1,
                double *wno1, double *wo);

/* CPU Krylov solve of the assembled operator: right-preconditioned restarted
 * FGMRES with the column (line) tridiagonal preconditioner.  x holds the
 * initial guess on entry.  Returns the iteration count (negative if not
 * converged); *relres = ||b - A x||_2 / ||b||_2 on exit. */
int og_solve(const og_grid *g, const int *rowptr, const int *colind,
             const double *val, const double *b, double *x, double rtol,
             int maxit, double *relres);

/* Open-boundary tide forcing and 1/x sponge relaxation (mo_obcs.f90 as built
 * with OBC_TIDE on and OBC_SPONGE_EXP off, Makefile:49-50).  Boundaries b:
 * 0 west, 1 east, 2 north, 3 south; variables v: 0 z (p-points), 1 u, 2 v.
 * amp[b][v] / pha[b][v] are OB{W,E,N,S}{Z,U,V}am / ...ph (mo_obcs.f90:40-46)
 * as (n, ntide) arrays, column-major, n the points along the boundary:
 * west/east z JE (j = 1..JE), u JE (j = 1..JE), v JE+1 (j = 0..JE);
 * north/south z IE (i = 1..IE), u IE+1 (i = 0..IE), v IE (i = 1..IE).
 * The open-boundary switches are og_grid's ob_*. */
typedef struct og_obc {
  int ntide;                        /* tidalnumber */
  const double *period;             /* tidalPeriod(ntide), s */
  int sponge[4];                    /* SpongeWest, SpongeEast, SpongeNorth, SpongeSouth */
  int width[4];                     /* spongew, spongee, spongen, sponges */
  double relax_inner, relax_bound;  /* Urelaxinner, Urelaxbound, s */
  const double *amp[4][3], *pha[4][3];
  /* OBC_SPONGE_EXP: TAO (s) of the exponential sponge (SPONGE_OBCS_ETA_EXP,
   * _UV_EXP, _TS_EXP, mo_obcs.f90:2588-3222); 0 for the 1/x sponge */
  double tao;
  /* og_obc_ts in the exponential form: the tracer is SAO, whose south band
   * reads the rate T's loop left behind (mo_obcs.f90:2976) */
  int salinity;
} og_obc;

/* FORC_OBCS_ETA + SPONGE_OBCS_ETA(ZO) at time step `step` (orctm.f90:1347-1351). */
void og_obc_eta(const og_grid *g, const og_obc *o, int step, double *zo);
/* FORC_OBCS_UV (with UPGRADE_OBCS_UV) + SPONGE_OBCS_UV(UOO, VOE) at time step
 * `step` (orctm.f90:1358-1362). */
void og_obc_uv(const og_grid *g, const og_obc *o, int step, double *uoo, double *voe);

/* FORC_OBCS_TS's boundary values (obc_t? = CLI_T?G * WETO of the boundary
 * cell, level by level, mo_obcs.f90:964-1012) and SPONGE_OBCS_TS
 * (mo_obcs.f90:1019-1272) on one tracer (octher.f90:114-119).  cli[b] is the
 * climatology record of side b as (n, KE), column-major, n = JE west/east,
 * IE north/south; NULL where the side is not open and sponged. */
void og_obc_ts(const og_grid *g, const og_obc *o, const double *const cli[4], double *trf);

/* Applies OCTIMF (octimf.f90:1-22): uko <- uoo, vke <- voe. */
void og_octimf(const og_grid *g, const double *uoo, const double *voe,
               double *uko, double *vke);

/* ---- Barotropic (free-surface) solve and total velocities ------------------
 * Constants of the reference's driver (orctm.f90:352-353, 657-661, 680):
 * G = 9.806, STABN = 0.6, CONN = 0.5, CONO = 1 - CONN, RLSA1 = 1 - 0.085.
 * 2D layouts: p (IE, JE), u (IE+1, JE) from I = 0, v (IE, JE+1) from J = 0. */
typedef struct og_baro {
  double grav, stabn, conn, rlsa1, sorpar;
  int niter;      /* SOR sweeps (250, troneu.f90:104) */
  int eta_forc;   /* OBC_ETA_FORC set: the boundary Z1O stays 0 (troneu.f90:67-102) */
} og_baro;

/* DEUTO / DEUTE and their inverses DEUTIO / DEUTIE from the BODEN-adjusted
 * DEPTO (boden.f90:117-128, 264-274); minvalue is the reference's small
 * threshold. */
void og_deut(const og_grid *g, const double *depto, double minvalue, double *deuto,
             double *deute, double *deutio, double *deutie);
/* ITPREP (itprep.f90:15-40): XX, FF (p), UF (u), VF (v). */
void og_itprep(const og_grid *g, const og_baro *b, const double *deuto, const double *deute,
               double *xx, double *uf, double *vf, double *ff);
/* TRONEU (troneu.f90:48-134): B1O and the red-black SOR for Z1O. */
void og_troneu(const og_grid *g, const og_baro *b, const double *xx, const double *uf,
               const double *vf, const double *ff, const double *u1o, const double *v1e,
               const double *uzo, const double *vze, double *b1o, double *z1o);
/* TROTEST (trotest.f90:1-118) with SQRTRND (sqrtrnd.f90:1-8): SORPAR from
 * 1.751 to 1.950 in steps of 0.001 (accumulated), each tried for `niter`
 * SOR sweeps from Z1O = 0 on a pseudo-random right-hand side; returns the
 * SORPAR of the smallest ratio of the squared changes of the last sweep to
 * those of the first.  ntry and niter are 200 in the reference. */
double og_trotest(const og_grid *g, const og_baro *b, const double *xx, const double *uf,
                  const double *vf, const double *ff, int ntry, int niter);
/* OCVTRO (ocvtro.f90:1-62): UZO, VZE scaled by the inverse depths, the
 * barotropic velocities USO, VSE, and ZO += Z1O. */
void og_ocvtro(const og_grid *g, const og_baro *b, const double *deutio, const double *deutie,
               const double *z1o, double *uzo, double *vze, double *uso, double *vse, double *zo);
/* OCBARP (ocbarp.f90:1-48): UZO = USO, VZE = VSE, then all four times the
 * surface masks AMSUO(.,.,1) / AMSUE(.,.,1). */
void og_ocbarp(const og_grid *g, double *uso, double *vse, double *uzo, double *vze);
/* OCWIND (ocwind.f90:1-42): the surface stress on UOO(.,.,1), VOE(.,.,1).
 * txo u-points, tye v-points; sicomu, sicomv, tauwatu, tauwatv (IE, JE). */
void og_ocwind(const og_grid *g, const double *txo, const double *tye, const double *sicomu,
               const double *sicomv, const double *tauwatu, const double *tauwatv, double *uoo,
               double *voe);
/* OCVTOT (ocvtot.f90:13-96): UKO, VKE with the barotropic part, the time
 * filter UKO <- CONN UKO + CONO UOO with UOO <- the unfiltered value, and WO
 * from the divergence, bottom up. */
void og_ocvtot(const og_grid *g, const og_baro *b, const double *uso, const double *vse,
               double *uoo, double *voe, double *uko, double *vke, double *wo);

/* ---- Thermodynamics, baroclinic pressure and mixing (OCTHER) ---------------
 * As built by the reference's Makefile:42-51: EISREST (REISCON = 1 - SICOMO),
 * REDWMICE (wind mixing (1 - SICOMO)**2), NURDIF (the convective switch
 * counts KCONDEP but mixes no tracer), no PLUME, no UMKLAP.  eos 0 is the
 * reference's ADISITJ + RHO1J (adisitj.f90, rho1j.f90); eos 1 is a linear
 * equation of state, RHO = rho0 + drdt (T - t0) + drds (S - s0), which the
 * reference lacks. */
typedef struct og_thermo {
  int eos;
  double rho0, drdt, drds, t0, s0;    /* linear EOS */
  double grav;                        /* G */
  double relsal, reltem;              /* RELSAL, RELTEM (orctm.f90:561, 569) */
  double rhoicwa, rhosnwa;            /* RHOICE/RHOWAT, RHOSNO/RHOWAT (orctm.f90:742-743) */
  double wt;                          /* WT = CWT / 6**3 (orctm.f90:503) */
  double cstabeps, dv0, av0, cavocon, cdvocon; /* orctm.f90:311-318 */
  const double *preff;                /* PREFF(KE) = 0.1026 TIESTU (beleg.f90:127) */
  const double *dbackv, *abackv;      /* DBACKV, ABACKV (KE+1) */
  /* 2D (IE, JE); NULL reads as 0 */
  const double *sicomo, *sictho, *sicsno, *relsao, *reltho, *giriv, *fu10;
} og_thermo;
/* ADISITJ on one value: potential to in-situ temperature at pressure pa. */
double og_adisit(double th, double sh, double pa);
/* RHO1J on one value (in-situ temperature t). */
double og_rho1(double t, double s, double p);
/* OCTHER part A (octher.f90:37-107): salinity / temperature restoring at the
 * surface, the fresh-water flux EMINPO into ZO, river input.  rivrun (IE, JE)
 * receives RIVRUN; PRECO / PRECH (flux diagnostics) are not kept. */
void og_octher_surface(const og_grid *g, const og_thermo *t, double *tho, double *sao,
                       double *zo, double *eminpo, double *rivrun);
/* OCTHER parts C and D (octher.f90:123-451): density, baroclinic pressure PO,
 * stability STABIO, the convection counter KCONDEP, the Richardson-number
 * mixing coefficients AVO / DVO (w-points, KE+1 levels), the tracers copied
 * down into land, and RHOO.  Part B, the T/S boundary forcing, runs between
 * og_octher_surface and this (og_obc_ts). */
void og_octher_column(const og_grid *g, const og_thermo *t, double *tho, double *sao,
                      const double *zo, const double *uko, const double *vke, double *po,
                      double *stabio, double *rhoo, double *avo, double *dvo, int *kcondep);

/* ---- Barotropic / baroclinic decomposition (OCMODMOM) ----------------------
 * Coriolis inputs: ftwou u-points, ftwov v-points (the grid file's FTWOU,
 * FTWOV), gila / giph (2 IE, 2 JE) the double-resolution longitudes and
 * latitudes (coriol.f90:46-47), omega (orctm.f90:678). */
typedef struct og_coriolis {
  const double *ftwou, *ftwov, *gila, *giph;
  double omega;
} og_coriolis;
/* OCMODMOM (ocmodmom.f90:1-243), NON_HYDROSTATIC: 12 Coriolis iterations on
 * UK1O, VK1E and WN1O (WNO follows WN1O), PO shifted by G ZO RLSA1 meanwhile,
 * STABIO scaled to a density step, the vertical sums U1O, USO (u) and V1E,
 * VSE (v), and UKO, VKE, UK1O, VK1E made baroclinic. */
void og_ocmodmom(const og_grid *g, const og_baro *b, const og_coriolis *c,
                 const double *deutio, const double *deutie, const double *zo,
                 const double *uoo, const double *voe, double *uko, double *vke, double *uk1o,
                 double *vk1e, double *wno, double *wn1o, double *po, double *stabio,
                 double *u1o, double *uso, double *v1e, double *vse);
/* OCCLIT (occlit.f90:1-332): 8 iterations of the baroclinic system in UKO,
 * VKE with the vertical velocity WO; returns CONTRA, the sum of the squared
 * WPO changes of the last completed update (the reference aborts above
 * 1e-3). */
double og_occlit(const og_grid *g, const og_baro *b, const double *deutio,
                 const double *deutie, double *uko, double *vke, double *uk1o, double *vk1e,
                 double *wo, double *stabio);

#ifdef __cplusplus
}
#endif
#endif
