/*
 * orctm_gpu.h -- C ABI of the B200 (sm_100a) implementation of ORCTM's
 * nonhydrostatic time-step hot path.
 *
 * The entry points replace the bodies of the reference's Fortran subroutines
 * (paths relative to the reference project, ORCTM/src_orctm/):
 *
 *   orctm_create        petsc_start          mo_petsc.f90:41-128 (operator set up
 *                                            once, like KSPSetComputeOperators)
 *   orctm_destroy       petsc_end            mo_petsc.f90:131-143
 *   orctm_ocuad         SUBROUTINE OCUAD     ocuad.f90:1-271
 *   orctm_ocvad         SUBROUTINE OCVAD     ocvad.f90:1-271
 *   orctm_ocwad         SUBROUTINE OCWAD     ocwad.f90:1-238
 *   orctm_ocadpo        SUBROUTINE OCADPO    ocadpo.f90:1-368
 *   orctm_octdiff       OCTDIFF_BASE + OCTDIFF_TS  octdiff_base.f90:1-229,
 *                                            octdiff_ts.f90:1-430
 *   orctm_octimf        SUBROUTINE OCTIMF    octimf.f90:1-22
 *   orctm_ocvisc        SUBROUTINE OCVISC    ocvisc.f90:1-772 (FREESLIP)
 *   orctm_ocvtot_nh     SUBROUTINE OCVTOT_NH ocvtot_nh.f90:1-259, including
 *                       petsc_solve_3D / ComputeRHS / compute_matrix
 *                                            mo_petsc.f90:211-397, 543-782
 *   orctm_step_hotpath  the driver's call sequence orctm.f90:1454-1562
 *   orctm_set_obc       INI_OBCS (tidal constants, 1/x sponge parameters)
 *                                            mo_obcs.f90:263-506
 *   orctm_obc_eta       FORC_OBCS_ETA + SPONGE_OBCS_ETA(ZO)  orctm.f90:1347-1351,
 *                                            mo_obcs.f90:569-642, 1561-1720
 *   orctm_obc_uv        FORC_OBCS_UV + SPONGE_OBCS_UV(UOO,VOE) orctm.f90:1358-1362,
 *                                            mo_obcs.f90:1881-2032, 2295-2582
 *   orctm_set_obc_ts / orctm_obc_ts  FORC_OBCS_TS + SPONGE_OBCS_TS(THO,SAO)
 *                       octher.f90:114-119, mo_obcs.f90:932-1272
 *   orctm_set_obc_sponge_exp  OBC_SPONGE_EXP: SPONGE_OBCS_ETA_EXP, _UV_EXP,
 *                       _TS_EXP instead of the 1/x sponge  orctm.f90:1348-1362,
 *                       octher.f90:116-120, mo_obcs.f90:507-522, 2588-3222
 *   orctm_set_barotropic  SUBROUTINE ITPREP  itprep.f90:15-40 (with BODEN's
 *                       inverse u/v depths, boden.f90:264-274)
 *   orctm_trotest       SUBROUTINE TROTEST   trotest.f90:1-118
 *   orctm_troneu        SUBROUTINE TRONEU    troneu.f90:48-134
 *   orctm_ocvtro        SUBROUTINE OCVTRO    ocvtro.f90:1-62
 *   orctm_ocvtot        SUBROUTINE OCVTOT    ocvtot.f90:13-96
 *   orctm_ocbarp        SUBROUTINE OCBARP    ocbarp.f90:1-48
 *   orctm_ocwind        SUBROUTINE OCWIND    ocwind.f90:1-42
 *   orctm_upload / orctm_download   the module arrays of MO_COMMO1
 *                                   (mo_commo1.f90:32-146) that the path reads
 *                                   and writes, moved between host and device
 *   orctm_write_gridinfo  SUBROUTINE WRTE_GRIDINFO  wrte_gridinfo.f90:1-175
 *   orctm_build_grid    BELEG + BODEN geometry (beleg.f90:48-139,
 *                       boden.f90:38-286), a set-up helper for callers that
 *                       have no Fortran host
 *
 * Conventions
 *  - Every function returns an int status: ORCTM_OK (0) or a negative error
 *    class.  The library never aborts; a Fortran caller maps a nonzero status
 *    to ABSTURZ (absturz.f90:10-11) as the reference's fatal path does.
 *  - Host arrays are the reference's Fortran arrays on a single-rank domain
 *    (I_start = J_start = 0), column-major, halos included:
 *        p-points  X(1:IE, 1:JE, 1:KE)     IE*JE*KE values
 *        u-points  X(0:IE, 1:JE, 1:KE)     (IE+1)*JE*KE
 *        v-points  X(1:IE, 0:JE, 1:KE)     IE*(JE+1)*KE
 *        w-points  X(1:IE, 1:JE, 1:KE+1)   IE*JE*(KE+1)
 *        2D arrays analogous (IE*JE, (IE+1)*JE, IE*(JE+1)).
 *  - All arithmetic of the default path is IEEE binary64.
 *  - A handle is used by one host thread at a time.  The model state lives
 *    on the device between calls (resident mode); only orctm_upload and
 *    orctm_download move it.  Both return after the copy has completed.
 *  - All entry points are asynchronous with respect to the host except the
 *    copies, orctm_synchronize and the solve statistics of orctm_ocvtot_nh.
 */
#ifndef ORCTM_GPU_H
#define ORCTM_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORCTM_ABI_VERSION 1

/* status codes */
#define ORCTM_OK 0
#define ORCTM_E_ARG (-1)           /* bad argument or size */
#define ORCTM_E_CUDA (-2)          /* CUDA runtime error */
#define ORCTM_E_NOMEM (-3)         /* device allocation failed */
#define ORCTM_E_NOT_CONVERGED (-4) /* Poisson solve hit maxit (state still updated) */
#define ORCTM_E_GEOMETRY (-5)      /* masks/thicknesses not of the BODEN form */
#define ORCTM_E_UNSUPPORTED (-6)   /* option outside the restated path */
#define ORCTM_E_NODEVICE (-7)      /* no usable CUDA device */
#define ORCTM_E_TOO_LARGE (-8)     /* size beyond orctm_octdiff_noalloc's fixed scratch */
#define ORCTM_E_UNSTABLE (-9)      /* OCCLIT's CONTRA above 1e-3, where the reference aborts
                                      (occlit.f90:321-326); the state is still updated */

/* field ids for orctm_upload / orctm_download (MO_COMMO1 array names) */
enum {
  ORCTM_F_UOO = 0,   /* u-points */
  ORCTM_F_VOE = 1,   /* v-points */
  ORCTM_F_WNO = 2,   /* w-points */
  ORCTM_F_UKO = 3,   /* u-points */
  ORCTM_F_VKE = 4,   /* v-points */
  ORCTM_F_WO = 5,    /* w-points */
  ORCTM_F_UOO_1 = 6, /* u-points */
  ORCTM_F_VOE_1 = 7, /* v-points */
  ORCTM_F_WNO_1 = 8, /* w-points */
  ORCTM_F_PNH = 9,   /* p-points */
  ORCTM_F_ZO = 10,   /* 2D p-points */
  ORCTM_F_DVO = 11,  /* w-points (IE,JE,KEP) */
  ORCTM_F_AVO = 12,  /* w-points (IE,JE,KEP) */
  ORCTM_F_THO = 13,  /* tracer 0; tracer n is ORCTM_F_THO + n (SAO = tracer 1) */
  ORCTM_F_SAO = 14
};

/* solver modes (orctm_set_solver) */
#define ORCTM_SOLVER_FP64 0        /* FP64 PCG, column-tridiagonal preconditioner */
#define ORCTM_SOLVER_FP32_REFINED 1 /* FP32 inner PCG inside FP64 iterative refinement */

typedef struct orctm_desc {
  int ie, je, ke;          /* IE, JE, KE including the 1-cell halo */
  int i_start, j_start;    /* must be 0: single-rank domain (mo_parallel.f90:197-206) */
  int ntracers;            /* >= 2: THO, SAO, then passive tracers (max 8) */
  int ob_west, ob_east, ob_north, ob_south; /* open-boundary switches (mo_obcs.f90:9-20) */
  double dt;               /* DT */
  double almzer;           /* ALMZER (orctm.f90:240) */
  double aulapts, aulapuv; /* biharmonic coefficients (orctm.f90:500-501) */
  double ah00;             /* harmonic tracer diffusion; must be <= almzer */
  const double* dzw;       /* DZW(KE) */
  const double* di;        /* DI(KE+1) */
  const double *dlxp, *dlyp, *dtdxpo, *dtdyo; /* 2D p-points */
  const double *dlxu, *dlyu, *dtdxuo;         /* 2D u-points */
  const double *dlxv, *dlyv, *dpye;           /* 2D v-points */
  const double *ddpo, *weto;                  /* 3D p-points */
  const double *dduo, *amsuo;                 /* 3D u-points */
  const double *ddue, *amsue;                 /* 3D v-points */
  int device;              /* CUDA device ordinal */
} orctm_desc;

typedef struct orctm_solve_stats {
  int iterations;       /* Krylov iterations (inner iterations for the refined solver) */
  int outer_iterations; /* refinement sweeps (1 for the FP64 solver) */
  int converged;        /* 1 if ||b - A x||_2 <= rtol ||b||_2 */
  double relres;        /* final ||b - A x||_2 / ||b||_2, computed in FP64 */
  double relres_initial;/* the same for the warm start */
  double solve_ms;      /* device time of the solve */
} orctm_solve_stats;

typedef struct orctm_handle orctm_handle;

int orctm_abi_version(void);
const char* orctm_status_string(int status);
/* last error message of a handle (or of the thread's last failed create) */
const char* orctm_last_error(const orctm_handle* h);

int orctm_create(const orctm_desc* desc, orctm_handle** out);
int orctm_destroy(orctm_handle* h);

/* number of doubles of a field in the host layout */
int orctm_field_size(const orctm_handle* h, int field, size_t* n);
int orctm_upload(orctm_handle* h, int field, const double* host, size_t n);
int orctm_download(orctm_handle* h, int field, double* host, size_t n);
/* Asynchronous copies on the handle's copy stream, overlapping the kernels.
 * An upload is ordered after the work already issued on the handle and
 * before the first routine that reads the field; routines that read other
 * fields do not wait for it (the tracers can upload while the momentum
 * advection runs).  A download is ordered after the work issued so far.  For
 * the copies to be asynchronous the host arrays must be page-locked
 * (cudaHostAlloc / cudaHostRegister); they must stay valid until
 * orctm_wait_copies returns, which waits for every copy of the handle.
 * orctm_set_step_outputs registers fields that orctm_step_hotpath downloads
 * as soon as they are final in the step (the tracers after OCTDIFF, while
 * OCVISC and the Poisson solve run; the rest at its end); n = 0 clears the
 * list.  These are extensions with no counterpart in the reference (its
 * model arrays live on the host). */
int orctm_upload_async(orctm_handle* h, int field, const double* host, size_t n);
int orctm_download_async(orctm_handle* h, int field, double* host, size_t n);
int orctm_set_step_outputs(orctm_handle* h, int n, const int* fields, double* const* host,
                           const size_t* sizes);
int orctm_wait_copies(orctm_handle* h);

/* EXTRA-format output, the reference's restart and output format (aufw.f90,
 * write_slice in mo_parallel.f90:733-779): per level a header record
 * (IDATE, ICODE, KCODE, IEDIM) of 4-byte integers and a record of the values
 * as 4-byte reals, Fortran sequential unformatted records, big-endian
 * (Makefile:75 builds with -convert big_endian), so the files read with the
 * same cdo scripts.  orctm_write_extra writes the given fields of a handle
 * (codes from ORCTM/code_output.txt: THO 2, SAO 5, UKO 3, VKE 4, ZO 1, WO and
 * WNO 7, DVO 111, AVO 110), with KCODE = INT(TIESTU(K)) for p, u and v
 * levels, INT(TIESTW(K)) for w levels and -100 for 2D fields, and IEDIM the
 * values of a level in the host layout; the first field truncates the file
 * unless append is set.  orctm_write_extra_host writes nlev levels of one
 * field from a host array (levels consecutive, iedim values each). */
int orctm_write_extra(orctm_handle* h, const char* path, int append, int idate, int nfield,
                      const int* fields, const int* codes);
int orctm_write_extra_host(const char* path, int append, int idate, int code, int nlev,
                           const int* kcodes, int iedim, const double* data);
/* GRID_INFO.ext, the grid file of WRTE_GRIDINFO (wrte_gridinfo.f90:19-172),
 * in the same records (IDATE 0): LONP/LATP 110/120, LONU/LATU 111/121,
 * LONV/LATV 112/122 (degrees), DEPTO/DEUTO/DEUTE 200-202, DLXP/DLXU/DLXV
 * 410-412 and DLYP/DLYU/DLYV 420-422 as 2D records (KCODE -100), then per
 * level (KCODE = K) WETO/AMSUO/AMSUE 300-302 and DDPO/DDUO/DDUE 430-432.
 * Spacings, masks and thicknesses come from the descriptor; the
 * coordinates and depths, which the hot path does not use, from g.  The
 * coordinates are GILA_G/GIPH_G at the points divided by PI/180, as
 * wrte_gridinfo.f90:26-44 forms them.  Host only; truncates the file. */
typedef struct orctm_gridinfo {
  const double *lonp, *latp;   /* IE*JE */
  const double *lonu, *latu;   /* (IE+1)*JE */
  const double *lonv, *latv;   /* IE*(JE+1) */
  const double *depto;         /* IE*JE, DEPTO after BODEN */
  const double *deuto;         /* (IE+1)*JE */
  const double *deute;         /* IE*(JE+1) */
} orctm_gridinfo;
int orctm_write_gridinfo(const char* path, const orctm_desc* desc, const orctm_gridinfo* g);

/* Restart reading (the role of AUFR, aufr.f90:103-167, which reads the same
 * records in a fixed order): for each field the first records of its code
 * and level size, in file order, are read as 4-byte reals, converted to
 * double exactly and uploaded.  orctm_read_extra_host reads nlev such records
 * of one code into a host array (kcodes may be NULL). */
int orctm_read_extra(orctm_handle* h, const char* path, int nfield, const int* fields,
                     const int* codes);
int orctm_read_extra_host(const char* path, int code, int nlev, int iedim, double* out,
                          int* kcodes);

int orctm_ocuad(orctm_handle* h);
int orctm_ocvad(orctm_handle* h);
int orctm_ocwad(orctm_handle* h);
int orctm_ocadpo(orctm_handle* h, int tracer);
/* OCADPO for every tracer of the handle in one call: the driver calls OCADPO
 * once per tracer with unchanged velocities (orctm.f90:1459-1460), so the
 * transports and volumes are formed once and shared; the results equal one
 * orctm_ocadpo call per tracer, bit for bit.  orctm_step_hotpath uses it. */
int orctm_ocadpo_all(orctm_handle* h);
int orctm_octdiff(orctm_handle* h);
int orctm_octimf(orctm_handle* h);
int orctm_ocvisc(orctm_handle* h);
int orctm_ocvtot_nh(orctm_handle* h, orctm_solve_stats* stats);
int orctm_step_hotpath(orctm_handle* h, orctm_solve_stats* stats);

/* ---- Open-boundary tide forcing and sponge (mo_obcs.f90) -------------------
 * The reference's build forces the open boundaries with tidal harmonics and
 * relaxes a sponge band towards them with the 1/x weights (OBC_TIDE on,
 * OBC_SPONGE_EXP off, Makefile:49-50); the driver calls the pair before
 * OCTIMF (orctm.f90:1347-1362).  Sides s: 0 west, 1 east, 2 north, 3 south
 * (open when the descriptor's ob_* switch is set); variables v: 0 z
 * (p-points), 1 u, 2 v.  amp[s][v] / pha[s][v] are OB{W,E,N,S}{Z,U,V}am /
 * ...ph as read by INI_OBCS (amplitude; phase as a time in s), each an
 * (n, ntide) array, column-major, n the points along the side:
 *     west/east   z JE (j = 1..JE)   u JE (j = 1..JE)     v JE+1 (j = 0..JE)
 *     north/south z IE (i = 1..IE)   u IE+1 (i = 0..IE)   v IE (i = 1..IE)
 * They are needed for the open, sponged sides only (others may be NULL).
 * The boundary value of a point is
 *     sum_td AM(q,td) * MASK * COS(2 PI (LDTRUN * DT - PH(q,td)) / T(td))
 * with MASK the level-1 mask of the boundary cell; in a band of width w the
 * cell at distance d = 1..w from the boundary cell relaxes towards it with
 * rate DT / ((s1 Urelaxbound + s2 Urelaxinner) / w), s1 = w - d + 1,
 * s2 = d - 1, and the nearer band wins where two bands cross. */
#define ORCTM_OBC_MAX_TIDES 8
typedef struct orctm_obc {
  int ntide;                 /* tidalnumber (mo_obcs.f90:19), 1..ORCTM_OBC_MAX_TIDES */
  const double* period;      /* tidalPeriod(ntide), s, nonzero */
  int sponge[4];             /* SpongeWest, SpongeEast, SpongeNorth, SpongeSouth */
  int width[4];              /* spongew, spongee, spongen, sponges: 1..IE (w/e), 1..JE (n/s) */
  double relax_inner;        /* Urelaxinner, s */
  double relax_bound;        /* Urelaxbound, s */
  const double* amp[4][3];
  const double* pha[4][3];
} orctm_obc;
/* Copies the constants to the device (INI_OBCS); may be called again, which
 * discards the T/S records of orctm_set_obc_ts. */
int orctm_set_obc(orctm_handle* h, const orctm_obc* obc);
/* ZO relaxed towards the tidal elevation at time step ldtrun, in place. */
int orctm_obc_eta(orctm_handle* h, int ldtrun);
/* UOO and VOE relaxed towards the tidal velocities at time step ldtrun. */
int orctm_obc_uv(orctm_handle* h, int ldtrun);
/* T/S boundary forcing, which the reference calls from OCTHER
 * (octher.f90:114-119).  orctm_set_obc_ts is FORC_OBCS_TS for one tracer
 * (0 THO, 1 SAO; mo_obcs.f90:932-1012): cli[s] is the climatology record of
 * side s that FORC_OBCS_TS reads every CLI_STEP / DT steps from
 * OB_<Side>_T.bin / OB_<Side>_S.bin, an (n, KE) array, column-major, n = JE
 * west/east and IE north/south (NULL for sides that are not open and
 * sponged); the boundary value at level K is the record times the boundary
 * cell's WETO.  orctm_obc_ts is SPONGE_OBCS_TS (mo_obcs.f90:1019-1272): the
 * tracers with a record relax in the bands of orctm_set_obc, in place. */
int orctm_set_obc_ts(orctm_handle* h, int tracer, const double* const* cli);
int orctm_obc_ts(orctm_handle* h);
/* The exponential sponge of a build with OBC_SPONGE_EXP (Makefile:50 has it
 * off): orctm_obc_eta, orctm_obc_uv, orctm_obc_ts and orctm_step_full then
 * run SPONGE_OBCS_ETA_EXP, SPONGE_OBCS_UV_EXP and SPONGE_OBCS_TS_EXP
 * (mo_obcs.f90:2588-3222).  Same bands and corner rule as the 1/x form; the
 * cell at distance d from the boundary cell changes by
 *     MASK_b * MASK * DT * EXP(-4 L/Lsp) / TAO * (boundary value - X),
 * L the summed DLX* (west, east) or DLY* (north, south) of the staggering
 * from the boundary cell to the cell, Lsp that of the whole band
 * (mo_obcs.f90:507-522); SAO's south band uses its innermost rate in every
 * row, as the reference's loop does (mo_obcs.f90:2976).  tao is the namelist
 * TAO (OCEOBC, orctm.f90:164-166), in s; 0 returns to the 1/x form, as does
 * orctm_set_obc.  Needs orctm_set_obc first. */
int orctm_set_obc_sponge_exp(orctm_handle* h, double tao);

/* ---- Barotropic (free-surface) solve and total velocities --------------
 * The part of the reference step that runs just before the hot path
 * (orctm.f90:1411-1431): TRONEU, OCVTRO, OCVTOT.  2D host arrays use the
 * layouts above: p (IE, JE), u (IE+1, JE) from I = 0, v (IE, JE+1) from J = 0.
 *
 * orctm_set_barotropic replaces ITPREP (itprep.f90:15-40, called once at
 * start-up, orctm.f90:872) and BODEN's inverse u/v depths
 * (boden.f90:264-274): XX, UF, VF, FF and DEUTIO, DEUTIE on the device, from
 * DEUTO / DEUTE (boden.f90:117-128) and the run's constants. */
typedef struct orctm_barotropic {
  const double* deuto;  /* host, u-points: MIN of the neighbouring DEPTO */
  const double* deute;  /* host, v-points */
  double minvalue;      /* BODEN's threshold MIN(1, DZW(1)/10): DEUTIO = 0 at or below it */
  double grav;          /* G (9.806, orctm.f90:680) */
  double stabn;         /* STABN (0.6, orctm.f90:657) */
  double conn;          /* CONN (0.5, orctm.f90:660); CONO = 1 - CONN */
  double rlsa1;         /* 1 - rlsa (0.915, orctm.f90:352-353) */
  double sorpar;        /* SORPAR (TROTEST's choice, trotest.f90) */
  int niter;            /* SOR sweeps (250, troneu.f90:104) */
  int eta_forc;         /* OBC_ETA_FORC: the boundary Z1O stays 0 (troneu.f90:67) */
} orctm_barotropic;
int orctm_set_barotropic(orctm_handle* h, const orctm_barotropic* b);
/* TRONEU (troneu.f90:48-134): uploads U1O, UZO (u-points) and V1E, VZE
 * (v-points), forms B1O and runs the red-black SOR for Z1O on the device.
 * With all four NULL it uses the device's U1O, V1E (orctm_ocmodmom) and UZO,
 * VZE (orctm_ocbarp). */
int orctm_troneu(orctm_handle* h, const double* u1o, const double* v1e, const double* uzo,
                 const double* vze);
/* TROTEST (trotest.f90:1-118, called once at start-up, orctm.f90:873): tries
 * SORPAR = 1.751, 1.752, ... (ntry values; 200 in the reference) for niter
 * SOR sweeps each (200) on SQRTRND's pseudo-random right-hand side and keeps
 * the one whose squared changes shrink most from the first sweep to the last;
 * TRONEU uses it from then on and *sorpar receives it.  Needs
 * orctm_set_barotropic. */
int orctm_trotest(orctm_handle* h, int ntry, int niter, double* sorpar);
/* OCVTRO (ocvtro.f90:1-62): UZO, VZE scaled by the inverse depths, the
 * barotropic velocities USO, VSE, and ZO += Z1O (device, in place). */
int orctm_ocvtro(orctm_handle* h);
/* OCBARP (ocbarp.f90:1-48): UZO = USO, VZE = VSE, all four times the
 * surface masks (device, in place; USO / VSE as OCVTRO left them). */
int orctm_ocbarp(orctm_handle* h);
/* OCWIND (ocwind.f90:1-42): the surface stress added to UOO and VOE at level
 * 1, in place.  Host arrays: TXO u-points (IE+1)*JE, TYE v-points IE*(JE+1),
 * SICOMU, SICOMV, TAUWATU, TAUWATV IE*JE (as mo_commo1.f90:160-167 declares
 * them); all six NULL reuses the forcing of the previous call. */
int orctm_ocwind(orctm_handle* h, const double* txo, const double* tye, const double* sicomu,
                 const double* sicomv, const double* tauwatu, const double* tauwatv);
/* OCVTOT (ocvtot.f90:13-96): UKO, VKE with USO, VSE added and the time filter
 * UKO <- CONN UKO + CONO UOO, UOO <- the unfiltered value (the same for v),
 * and WO from the divergence of the filtered velocities, bottom up. */
int orctm_ocvtot(orctm_handle* h);
/* 2D barotropic fields to the host: which = ORCTM_B_* below. */
enum {
  ORCTM_B_Z1O = 0,  /* p-points */
  ORCTM_B_B1O = 1,  /* p-points */
  ORCTM_B_USO = 2,  /* u-points */
  ORCTM_B_VSE = 3,  /* v-points */
  ORCTM_B_UZO = 4,  /* u-points */
  ORCTM_B_VZE = 5,  /* v-points */
  ORCTM_B_U1O = 6,  /* u-points: OCMODMOM's sum of DDUO UOO, TRONEU's input */
  ORCTM_B_V1E = 7   /* v-points */
};
int orctm_download_barotropic(orctm_handle* h, int which, double* host, size_t n);

/* ---- OCTHER, OCMODMOM, OCCLIT and the whole step -------------------------
 * The rest of the reference step before the hot path, on the device, as the
 * reference is built (Makefile:42-51: EISREST, REDWMICE, NURDIF,
 * NON_HYDROSTATIC; no PLUME, UMKLAP).  Host 2D arrays are (IE, JE)
 * p-points; NULL reads as zero. */
#define ORCTM_EOS_UNESCO 0 /* ADISITJ + RHO1J (adisitj.f90, rho1j.f90) */
#define ORCTM_EOS_LINEAR 1 /* RHO = rho0 + drdt (T - t0) + drds (S - s0); not in the reference */
typedef struct orctm_thermo {
  int eos;                      /* ORCTM_EOS_* */
  double rho0, drdt, drds, t0, s0; /* linear EOS */
  double grav;                  /* G (9.806) */
  double relsal, reltem;        /* RELSAL = CRELSAL 20/DZW(1), RELTEM (orctm.f90:561, 569), 1/s */
  double rhoicwa, rhosnwa;      /* RHOICE/RHOWAT, RHOSNO/RHOWAT (orctm.f90:739-743) */
  double wt;                    /* WT = CWT / 6**3 (orctm.f90:503) */
  double cstabeps, dv0, av0, cavocon, cdvocon; /* orctm.f90:311-318 */
  const double* preff;          /* KE reference pressures; NULL = 0.1026 TIESTU (beleg.f90:127) */
  const double* dbackv;         /* KE+1 background diffusivity DBACKV */
  const double* abackv;         /* KE+1 background viscosity ABACKV */
  const double *sicomo, *sictho, *sicsno; /* sea-ice fraction, thickness, snow */
  const double *relsao, *reltho;          /* surface restoring targets */
  const double *giriv;                    /* river inflow (m/s) */
  const double *fu10;                     /* 10 m wind speed */
} orctm_thermo;
/* Sets OCTHER's constants and forcing; may be called again (daily forcing).
 * The first call sets KCONDEP as BODEN does (boden.f90:261). */
int orctm_set_thermo(orctm_handle* h, const orctm_thermo* t);
/* OCMODMOM's Coriolis inputs: FTWOU (IE+1)*JE, FTWOV IE*(JE+1) (the grid
 * file's, orctm.f90:811), GILA / GIPH (2 IE)*(2 JE) (coriol.f90:46-47),
 * OMEGA (7.292e-5, orctm.f90:678).  The grid-angle factors are formed here
 * on the host. */
typedef struct orctm_coriolis {
  const double *ftwou, *ftwov, *gila, *giph;
  double omega;
} orctm_coriolis;
int orctm_set_coriolis(orctm_handle* h, const orctm_coriolis* c);
/* OCTHER (octher.f90:1-455): restoring, fresh water and rivers into THO,
 * SAO, ZO; the T/S boundary forcing when orctm_set_obc_ts was called; PO,
 * STABIO, KCONDEP, AVO, DVO, RHOO; tracers copied down into land. */
int orctm_octher(orctm_handle* h);
/* OCMODMOM (ocmodmom.f90:1-243): 12 Coriolis iterations on UK1O, VK1E,
 * WNO; U1O, USO, V1E, VSE; baroclinic UKO, VKE, UK1O, VK1E.  Needs
 * orctm_set_thermo, orctm_set_coriolis and orctm_set_barotropic. */
int orctm_ocmodmom(orctm_handle* h);
/* OCCLIT (occlit.f90:1-332): the baroclinic iteration with WO; *contra
 * (may be NULL) receives CONTRA, summed in a fixed order of its own;
 * ORCTM_E_UNSTABLE above 1e-3. */
int orctm_occlit(orctm_handle* h, double* contra);
/* Baroclinic arrays to and from the host: which = ORCTM_C_* below. */
enum {
  ORCTM_C_PO = 0,      /* p-points (IE, JE, KE) */
  ORCTM_C_STABIO = 1,  /* p-points */
  ORCTM_C_RHOO = 2,    /* p-points */
  ORCTM_C_UK1O = 3,    /* u-points (IE+1, JE, KE) */
  ORCTM_C_VK1E = 4,    /* v-points (IE, JE+1, KE) */
  ORCTM_C_EMINPO = 5,  /* 2D p-points */
  ORCTM_C_RIVRUN = 6,  /* 2D p-points */
  ORCTM_C_KCONDEP = 7  /* 2D p-points, integral values */
};
int orctm_upload_baroclinic(orctm_handle* h, int which, const double* host, size_t n);
int orctm_download_baroclinic(orctm_handle* h, int which, double* host, size_t n);
/* One whole time step in the driver's order (orctm.f90:1327-1562): OCTHER,
 * OCWIND (with the forcing of the last orctm_ocwind call, if any), the open-
 * boundary forcing (when orctm_set_obc was called; the elevation only with
 * eta_forc), OCTIMF, OCMODMOM, OCBARP, OCCLIT, TRONEU, OCVTRO, OCVTOT, STABIO
 * times 1000/DZ, and orctm_step_hotpath.  ldtrun is the step number the
 * tides are evaluated at.  Returns the hot path's status, else OCCLIT's. */
int orctm_step_full(orctm_handle* h, int ldtrun, orctm_solve_stats* s, double* contra);

/* solver mode and relative-residual target (default FP64, 1e-10, 5000) */
int orctm_set_solver(orctm_handle* h, int mode, double rtol, int maxit);
int orctm_synchronize(orctm_handle* h);

/* Device-time measurement on the handle's stream (CUDA events). */
int orctm_timer_start(orctm_handle* h);
int orctm_timer_stop(orctm_handle* h, double* ms);

/* Optional per-launcher device timing: when on, every launcher group of the
 * kinds below is bracketed by CUDA events; orctm_profile_get returns the
 * number of bracketed launches and their summed device time since the last
 * orctm_set_profiling call. */
enum {
  ORCTM_PROF_OCUAD = 0, ORCTM_PROF_OCVAD, ORCTM_PROF_OCWAD, ORCTM_PROF_OCADPO,
  ORCTM_PROF_OCTDIFF, ORCTM_PROF_OCVISC, ORCTM_PROF_NH_RHS, ORCTM_PROF_PCG_SPMV,
  ORCTM_PROF_PCG_COL, ORCTM_PROF_RESID, ORCTM_PROF_NH_POST, ORCTM_PROF_KINDS
};
int orctm_set_profiling(orctm_handle* h, int on);
int orctm_profile_get(orctm_handle* h, int kind, long long* launches, double* total_ms);

/* Number of CUDA kernels this library has launched in the calling process. */
unsigned long long orctm_kernel_launches(void);

/* Numerical self-check: q[k] = a[k] / b[k] computed on the device by the
 * division the stencil kernels use (Newton-Raphson refinement of a reciprocal
 * estimate, within 1 ulp of IEEE division).  Test support; allocates. */
int orctm_check_division(int device, const double* a, const double* b, double* q, size_t n);

/* Kernel variants of the Poisson solver: 6 column-kernel variants (forward
 * values in global or shared memory, 4 or 8 levels per load batch, 32x4,
 * 32x2 or 128x1 blocks) and 9 stencil variants (0-5: shared-memory ring,
 * L1 form or warp-row form, 32x8 or 32x4 blocks; 6-8: TMA-staged tiles).
 * All variants give bit-identical results.  A variant of -1 (the default)
 * lets the handle time the variants on its own grid before its first solve
 * in each precision and keep the fastest (the choice is cached per grid size
 * in the process).  orctm_get_tuning returns the variants in use for a
 * precision (0 FP64, 1 FP32), -1 before the first solve.  A shared-memory
 * column variant that does not fit the grid's KE falls back to variant 0. */
int orctm_set_tuning(orctm_handle* h, int col_variant, int spmv_variant);
int orctm_get_tuning(const orctm_handle* h, int precision, int* col_variant, int* spmv_variant);

/* Device memory.  A handle allocates from a stream-ordered pool that the
 * library keeps per device; destroying a handle returns its blocks to the
 * pool without a device-wide synchronisation.  orctm_device_bytes gives the
 * bytes a handle holds now (it grows on the first step and the first solve
 * of each solver mode); orctm_trim_device_memory hands the pool's unused
 * blocks of a device back to the driver. */
int orctm_device_bytes(const orctm_handle* h, unsigned long long* bytes);
int orctm_trim_device_memory(int device);

/* ---- Batched and served execution of independent instances ----------------
 * A server runs independent regional instances on one device (the serving
 * loop of an ensemble; the reference runs one domain per MPI job, so these
 * entry points have no counterpart in it).  A request carries a descriptor,
 * the fields to upload, a number of hot-path steps and the fields to
 * download afterwards.  The server admits requests in submission order when a
 * slot is free and the request's estimated device memory fits the budget
 * (memory_fraction of the device memory free when the server was created; a
 * request is always admitted when nothing else is in flight).  Each slot is a
 * host thread with its own handle and stream, so the device work of the
 * requests in flight overlaps; every instance's state stays on the device
 * from upload to download.  A request's results do not depend on what else
 * is in flight (each instance's kernels and reductions are deterministic).
 * Host buffers named by a request must stay valid until orctm_serve_wait or
 * orctm_serve_poll reports it done; input sizes are those of
 * orctm_field_size.  The server is internally synchronised: any thread may
 * submit, poll or wait. */
typedef struct orctm_server orctm_server;

typedef struct orctm_serve_opts {
  int device;             /* CUDA device ordinal */
  int slots;              /* requests in flight at once, >= 1 */
  double memory_fraction; /* share of the free device memory admitted requests may use, (0, 1] */
  int solver;             /* ORCTM_SOLVER_FP64 or ORCTM_SOLVER_FP32_REFINED */
  double rtol;            /* Poisson relative-residual target */
  int maxit;              /* Krylov iteration limit per solve */
} orctm_serve_opts;

typedef struct orctm_request {
  const orctm_desc* desc;      /* geometry and parameters (desc->device is ignored) */
  int nsteps;                  /* orctm_step_hotpath calls, >= 0 */
  int nin;                     /* fields uploaded before the first step */
  const int* in_fields;
  const double* const* in_data;
  int nout;                    /* fields downloaded after the last step */
  const int* out_fields;
  double* const* out_data;
} orctm_request;

typedef struct orctm_request_stats {
  int status;                  /* ORCTM_OK or the first error of the request */
  int steps_done;
  int iterations;              /* Krylov iterations summed over the steps */
  double relres_max;           /* largest final relative residual of its solves */
  double queued_ms;            /* submission to admission */
  double run_ms;               /* admission to results written */
  double step_ms_p50, step_ms_p99, step_ms_max; /* per-step latency (host clock, step + sync) */
  unsigned long long device_bytes;             /* device memory the instance held */
  unsigned long long estimated_bytes;          /* what admission reserved for it */
} orctm_request_stats;

typedef struct orctm_serve_stats {
  long long submitted, completed, failed;
  long long steps;             /* steps completed over all requests */
  double cell_steps;           /* interior cells x steps, summed over completed steps */
  double elapsed_ms;           /* first submission to last completion */
  double step_ms_p50, step_ms_p99; /* per-step latency over all steps */
  int peak_in_flight;
  unsigned long long peak_reserved_bytes;
  unsigned long long budget_bytes;
} orctm_serve_stats;

int orctm_serve_create(const orctm_serve_opts* opts, orctm_server** out);
int orctm_serve_submit(orctm_server* s, const orctm_request* req, unsigned long long* id);
/* blocks until request id is done; its record is released */
int orctm_serve_wait(orctm_server* s, unsigned long long id, orctm_request_stats* stats);
/* *done = 1 (and stats filled, record released) when request id is done */
int orctm_serve_poll(orctm_server* s, unsigned long long id, int* done, orctm_request_stats* stats);
/* blocks until every submitted request is done */
int orctm_serve_drain(orctm_server* s);
int orctm_serve_get_stats(orctm_server* s, orctm_serve_stats* stats);
/* drains, then stops the slots */
int orctm_serve_destroy(orctm_server* s);

/* Runs n requests submitted together (an ensemble batch) and waits for all;
 * per_request may be NULL.  With opts->slots == 1 the requests run one at a
 * time. */
int orctm_batch_run(const orctm_serve_opts* opts, int n, const orctm_request* reqs,
                    orctm_request_stats* per_request, orctm_serve_stats* total);

/* Upper bound of the device bytes one instance needs (fields, geometry
 * tables and the solver vectors of the given solver mode). */
int orctm_estimate_device_bytes(const orctm_desc* desc, int solver, unsigned long long* bytes);

/* BELEG + BODEN restated on the host.  depto (IE*JE) is adjusted in place as
 * BODEN does (ISTART == 0).  Output arrays are caller-allocated in the host
 * layouts above; tiestu, tiestw, dz and di hold KE+1 values. */
int orctm_build_grid(int ie, int je, int ke, double dt, const double* dzw, double* depto,
                     const double* dlxp, const double* dlyp, const double* dlxu,
                     const double* dlyu, const double* dlxv, const double* dlyv,
                     double* tiestu, double* tiestw, double* dz, double* di, double* dtdxpo,
                     double* dtdyo, double* dtdxuo, double* dpyo, double* dtdxue, double* dpye,
                     double* ddpo, double* weto, double* dduo, double* amsuo, double* ddue,
                     double* amsue);

/* ---- Scratch-free tracer diffusion -------------------------------------
 * No counterpart in the reference: an extra entry point for callers that
 * cannot allocate device memory -- code that runs while a CUDA graph is being
 * captured, hosts whose device memory belongs to another runtime or pool (an
 * OpenACC / OpenMP-offload Fortran model, a framework allocator), loops that
 * must not block on the driver's allocator.  It computes OCTDIFF_BASE +
 * OCTDIFF_TS (implicit vertical diffusion, then the biharmonic operator) for
 * ONE tracer on caller-owned device arrays in the reference's Fortran
 * layouts, without a handle and without allocating anything.
 *
 * Its two scratch fields live in a fixed array compiled into the library
 * (32 MiB, held on every GPU that loads the library until the process
 * exits), which limits IE*JE*KE to 2,097,152 cells; larger grids return
 * ORCTM_E_TOO_LARGE.  The first call on each device looks up that array's
 * device address (cudaGetSymbolAddress) with the device current: make that
 * first call before any stream capture (a first call on a capturing stream
 * returns ORCTM_E_ARG).  Calls on a stream that is not capturing look the
 * address up again, so after a cudaDeviceReset one such call must precede
 * the next capture.  A refused call's message is orctm_last_error(NULL).
 * All calls share the array and it
 * keeps the last call's contents; every value a call reads is written earlier
 * in the same call.  Calls that overlap on the GPU race on the array: order
 * them on one stream.  The kernels are enqueued on args->stream and the call
 * returns without waiting for them. */
typedef struct orctm_octdiff_noalloc_args {
  int ie, je, ke;                 /* IE, JE, KE including halos */
  double dt, almzer, aulapts, ah00; /* as in orctm_desc; ah00 must be <= almzer */
  const double* tracer_in;        /* device, p-points IE*JE*KE */
  double* tracer_out;             /* device, p-points, a different buffer */
  const double* dvo;              /* device, w-points IE*JE*(KE+1) */
  const double *ddpo, *weto;      /* device, p-points IE*JE*KE */
  const double *di, *dzw;         /* device, DI(KE+1), DZW(KE) */
  const double *dlxp, *dlyp;      /* device, 2D p-points IE*JE */
  const double *dlxu, *dlyu;      /* device, 2D u-points (IE+1)*JE */
  const double *dlxv, *dlyv;      /* device, 2D v-points IE*(JE+1) */
  const double* zo;               /* device, 2D p-points IE*JE */
  void* stream;                   /* cudaStream_t; NULL = legacy default stream */
} orctm_octdiff_noalloc_args;
int orctm_octdiff_noalloc(const orctm_octdiff_noalloc_args* args);

#ifdef __cplusplus
}
#endif
#endif /* ORCTM_GPU_H */
