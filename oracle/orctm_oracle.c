/*
 * CPU restatement (oracle) of ORCTM's nonhydrostatic hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load this library, and
 * only as the checker or the timed CPU baseline; the CUDA product never calls
 * it.  PARITY PINNED ONLY IN PART: the reference (Fortran 90 + PETSc 3.10.2)
 * cannot be built here and ships no golden outputs; its check values and
 * input files pin what they cover (see orctm_oracle.h).
 *
 * Every routine follows the reference loop by loop; the file:line cited in
 * front of each block is the reference code it restates
 * (ORCTM/src_orctm/...).  Build flags: -O2 -ffp-contract=off -fopenmp.
 * OpenMP only splits loops whose iterations are independent, so results do
 * not depend on the thread count (the Krylov solve's dot products excepted).
 */
#include "orctm_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Fortran-layout accessors (see orctm_oracle.h). */
#define P3(a, i, j, k) (a)[((size_t)((k)-1) * JE + (size_t)((j)-1)) * IE + (size_t)((i)-1)]
#define U3(a, i, j, k) (a)[((size_t)((k)-1) * JE + (size_t)((j)-1)) * (IE + 1) + (size_t)(i)]
#define V3(a, i, j, k) (a)[((size_t)((k)-1) * (JE + 1) + (size_t)(j)) * IE + (size_t)((i)-1)]
/* levels 0..KE (TRM/WTM in the reference are dimensioned 0:KE) */
#define M3(a, i, j, k) (a)[((size_t)(k) * JE + (size_t)((j)-1)) * IE + (size_t)((i)-1)]
#define MU3(a, i, j, k) (a)[((size_t)(k) * JE + (size_t)((j)-1)) * (IE + 1) + (size_t)(i)]
#define MV3(a, i, j, k) (a)[((size_t)(k) * (JE + 1) + (size_t)(j)) * IE + (size_t)((i)-1)]
#define P2(a, i, j) (a)[(size_t)((j)-1) * IE + (size_t)((i)-1)]
#define U2(a, i, j) (a)[(size_t)((j)-1) * (IE + 1) + (size_t)(i)]
#define V2(a, i, j) (a)[(size_t)(j) * IE + (size_t)((i)-1)]
#define K1(a, k) (a)[(k)-1]

#define DIMS                      \
  const int IE = g->ie;           \
  const int JE = g->je;           \
  const int KE = g->ke;           \
  const int KEP = KE + 1;         \
  const int IE1 = IE - 1;         \
  const int JE1 = JE - 1;         \
  (void)KEP; (void)IE1; (void)JE1

/* Fortran MAX(a,b) / MIN(a,b) for non-NaN operands. */
static inline double fmx(double a, double b) { return a > b ? a : b; }
static inline double fmn(double a, double b) { return b < a ? b : a; }

static double *zalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

/* ------------------------------------------------------------------------ */
/* BELEG (beleg.f90:48-139) + BODEN (boden.f90:38-213)                      */
/* ------------------------------------------------------------------------ */
void og_build_grid(int ie, int je, int ke, double dt, const double *dzw,
                   double *depto, const double *dlxp, const double *dlyp,
                   const double *dlxu, const double *dlyu, const double *dlxv,
                   const double *dlyv, double *tiestu, double *tiestw,
                   double *dz, double *di, double *dtdxpo, double *dtdyo,
                   double *dtdxuo, double *dpyo, double *dtdxue, double *dpye,
                   double *ddpo, double *weto, double *dduo, double *amsuo,
                   double *ddue, double *amsue) {
  const int IE = ie, JE = je, KE = ke, KEP = ke + 1, IE1 = ie - 1, JE1 = je - 1;
  /* beleg.f90:42-76 */
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      P2(dtdxpo, i, j) = dt / P2(dlxp, i, j);
      P2(dtdyo, i, j) = dt / P2(dlyp, i, j);
    }
  for (int j = 1; j <= JE; ++j)
    for (int i = 0; i <= IE; ++i) {
      U2(dtdxuo, i, j) = dt / U2(dlxu, i, j);
      U2(dpyo, i, j) = dt / U2(dlyu, i, j);
    }
  for (int j = 0; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      V2(dtdxue, i, j) = dt / V2(dlxv, i, j);
      V2(dpye, i, j) = dt / V2(dlyv, i, j);
    }
  /* beleg.f90:87-105, 125-139 */
  K1(tiestu, 1) = 0.5 * K1(dzw, 1);
  K1(tiestw, 1) = 0.0;
  for (int k = 1; k <= KE; ++k) K1(tiestw, k + 1) = K1(tiestw, k) + K1(dzw, k);
  for (int k = 2; k <= KE; ++k) K1(tiestu, k) = 0.5 * (K1(tiestw, k + 1) + K1(tiestw, k));
  K1(tiestu, KEP) = 9000.;
  K1(dz, 1) = K1(tiestu, 1);
  for (int k = 2; k <= KEP; ++k) K1(dz, k) = K1(tiestu, k) - K1(tiestu, k - 1);
  for (int k = 1; k <= KE; ++k) K1(di, k) = 1. / K1(dz, k);
  K1(di, KEP) = 1. / K1(dz, KE);

  /* boden.f90:38-62 (ISTART == 0) */
  const double minvalue = fmn(1.0, K1(dzw, 1) / 10.0);
  const double depmin = K1(dzw, 1) + K1(dzw, 2) + minvalue;
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      if (P2(depto, i, j) <= minvalue) P2(depto, i, j) = 0.;
      if (P2(depto, i, j) > minvalue && P2(depto, i, j) < depmin) P2(depto, i, j) = depmin;
    }
  /* boden.f90:101-107 */
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i)
      for (int k = 1; k <= KE; ++k)
        if (fabs(P2(depto, i, j) - K1(tiestu, k)) < minvalue / 2)
          P2(depto, i, j) = K1(tiestu, k) + minvalue;
  /* boden.f90:116-130: DEUTO (u-points, 0:IE) and DEUTE (v-points, 0:JE) */
  double *deuto = zalloc((size_t)(IE + 1) * JE);
  double *deute = zalloc((size_t)IE * (JE + 1));
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE1; ++i) U2(deuto, i, j) = fmn(P2(depto, i, j), P2(depto, i + 1, j));
  for (int j = 1; j <= JE; ++j) {
    U2(deuto, 0, j) = U2(deuto, 1, j);
    U2(deuto, IE, j) = U2(deuto, IE1, j);
  }
  for (int j = 1; j <= JE1; ++j)
    for (int i = 1; i <= IE; ++i) V2(deute, i, j) = fmn(P2(depto, i, j), P2(depto, i, j + 1));
  for (int i = 1; i <= IE; ++i) {
    V2(deute, i, 0) = V2(deute, i, 1);
    V2(deute, i, JE) = V2(deute, i, JE1);
  }
  /* boden.f90:182-213 (arrays start at zero, BELEG_ZERO) */
  memset(ddpo, 0, sizeof(double) * (size_t)IE * JE * KE);
  memset(weto, 0, sizeof(double) * (size_t)IE * JE * KE);
  memset(dduo, 0, sizeof(double) * (size_t)(IE + 1) * JE * KE);
  memset(amsuo, 0, sizeof(double) * (size_t)(IE + 1) * JE * KE);
  memset(ddue, 0, sizeof(double) * (size_t)IE * (JE + 1) * KE);
  memset(amsue, 0, sizeof(double) * (size_t)IE * (JE + 1) * KE);
  for (int k = 1; k <= KE; ++k) {
    const double tu = K1(tiestu, k), tu1 = K1(tiestu, k + 1), tw = K1(tiestw, k);
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        const double d = P2(depto, i, j);
        if (tu < d) P3(weto, i, j, k) = 1.;
        if (tu1 < d) P3(ddpo, i, j, k) = K1(dzw, k);
        if (tu < d && tu1 >= d) P3(ddpo, i, j, k) = d - tw;
      }
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i) {
        const double d = U2(deuto, i, j);
        if (tu1 < d) U3(dduo, i, j, k) = K1(dzw, k);
        if (tu < d && tu1 >= d) U3(dduo, i, j, k) = d - tw;
        if (U3(dduo, i, j, k) > 0.) U3(amsuo, i, j, k) = 1.;
      }
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        const double d = V2(deute, i, j);
        if (tu1 < d) V3(ddue, i, j, k) = K1(dzw, k);
        if (tu < d && tu1 >= d) V3(ddue, i, j, k) = d - tw;
        if (V3(ddue, i, j, k) > 0.) V3(amsue, i, j, k) = 1.;
      }
  }
  free(deuto);
  free(deute);
}

/* ------------------------------------------------------------------------ */
/* OCADPO (ocadpo.f90:94-348), options ADPO on, SMOADV/SMOADH and           */
/* SLOPECON_ADPO off (Makefile:42-51).  Sea-ice terms SICTHO/SICSNO are     */
/* zero: the ice model is not called (octher.f90:51).                      */
/* ------------------------------------------------------------------------ */
void og_ocadpo(const og_grid *g, double *trf, const double *uko, const double *vke,
               const double *wo, const double *zo) {
  DIMS;
  const double DT = g->dt;
  const size_t n3 = (size_t)IE * JE * KE, n0 = (size_t)IE * JE * (KE + 1);
  double *s1o = zalloc(n3), *t1o = zalloc(n3);
  double *trp = zalloc(n0), *wtp = zalloc(n0); /* 1..KEP */
  double *trm = zalloc(n0), *wtm = zalloc(n0); /* 0..KE  */
  /* ocadpo.f90:94-116 */
  for (int k = 1; k <= KE; ++k)
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        P3(s1o, i, j, k) = P3(g->weto, i, j, k) * P2(g->dlxp, i, j) * P2(g->dlyp, i, j) *
                           P3(g->ddpo, i, j, k);
        P3(t1o, i, j, k) = P3(trf, i, j, k);
      }
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i)
      P3(s1o, i, j, 1) = P3(s1o, i, j, 1) + P2(g->dlxp, i, j) * P2(g->dlyp, i, j) *
                                                P3(g->weto, i, j, 1) *
                                                (P2(zo, i, j) - P3(wo, i, j, 1) * DT);
  /* vertical transports, ocadpo.f90:120-143 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    const int klo = k + 1 < KE ? k + 1 : KE;
    const int kup = k - 1 > 1 ? k - 1 : 1;
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        const double t = P3(trf, i, j, k), tu = P3(trf, i, j, kup), tl = P3(trf, i, j, klo);
        const double abl = fabs(tu - tl);
        const double zwabl = fabs(tu + tl - 2. * t);
        const double w0 = P3(wo, i, j, k), w1 = P3(wo, i, j, k + 1);
        const double up = 0.5 * DT * P2(g->dlyp, i, j) * P2(g->dlxp, i, j) * (w0 + fabs(w0));
        const double um = 0.5 * DT * P2(g->dlyp, i, j) * P2(g->dlxp, i, j) * (fabs(w1) - w1);
        const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20));
        double sch = fmn(P3(g->weto, i, j, klo), scha * P3(s1o, i, j, k) / (up + um + 1.E-20));
        if (k == 1 || k == KE) sch = 0.;
        const double schi = 1. - sch;
        P3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + tu));
        M3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + tl));
        P3(wtp, i, j, k) = up;
        M3(wtm, i, j, k) = um;
      }
  }
  /* ocadpo.f90:158-173 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        if (P3(g->weto, i, j, k) > 0.5) {
          const double rn = P3(s1o, i, j, k) + P3(wtp, i, j, k + 1) - P3(wtp, i, j, k) -
                            M3(wtm, i, j, k) + M3(wtm, i, j, k - 1);
          P3(t1o, i, j, k) = (P3(trf, i, j, k) * P3(s1o, i, j, k) + P3(trp, i, j, k + 1) -
                              P3(trp, i, j, k) - M3(trm, i, j, k) + M3(trm, i, j, k - 1)) /
                             rn;
          P3(s1o, i, j, k) = rn;
        }
  for (int k = 1; k <= KE; ++k)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) P3(trf, i, j, k) = P3(t1o, i, j, k);

  /* x-direction, ocadpo.f90:181-258 */
  memset(trp, 0, sizeof(double) * n0);
  memset(trm, 0, sizeof(double) * n0);
  memset(wtp, 0, sizeof(double) * n0);
  memset(wtm, 0, sizeof(double) * n0);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        const double t = P3(trf, i, j, k), te = P3(trf, i + 1, j, k), tw = P3(trf, i - 1, j, k);
        const double abl = fabs(te - tw);
        const double zwabl = fabs(te + tw - 2. * t);
        const double u0 = U3(uko, i, j, k), um1 = U3(uko, i - 1, j, k);
        const double up = 0.5 * DT * U3(g->dduo, i, j, k) * U2(g->dlyu, i, j) * (u0 + fabs(u0));
        const double um = 0.5 * DT * U3(g->dduo, i - 1, j, k) * (fabs(um1) - um1) *
                          U2(g->dlyu, i - 1, j);
        const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20)) * P3(g->weto, i, j, k) *
                            P3(g->weto, i + 1, j, k) * P3(g->weto, i - 1, j, k);
        const double sch = fmn(1., scha * P3(s1o, i, j, k) / (up + um + 1.E-20));
        const double schi = 1. - sch;
        P3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + te));
        M3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + tw));
        P3(wtp, i, j, k) = up;
        M3(wtm, i, j, k) = um;
      }
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        if (P3(g->weto, i, j, k) > 0.5) {
          const double rn = P3(s1o, i, j, k) + P3(wtp, i - 1, j, k) - P3(wtp, i, j, k) -
                            M3(wtm, i, j, k) + M3(wtm, i + 1, j, k);
          P3(t1o, i, j, k) = (P3(trf, i, j, k) * P3(s1o, i, j, k) + P3(trp, i - 1, j, k) -
                              P3(trp, i, j, k) - M3(trm, i, j, k) + M3(trm, i + 1, j, k)) /
                             rn;
          P3(s1o, i, j, k) = rn;
        }
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) P3(trf, i, j, k) = P3(t1o, i, j, k);
  }

  /* y-direction, ocadpo.f90:266-345 */
  memset(trp, 0, sizeof(double) * n0);
  memset(trm, 0, sizeof(double) * n0);
  memset(wtp, 0, sizeof(double) * n0);
  memset(wtm, 0, sizeof(double) * n0);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        const double t = P3(trf, i, j, k), tn = P3(trf, i, j - 1, k), ts = P3(trf, i, j + 1, k);
        const double abl = fabs(tn - ts);
        const double zwabl = fabs(tn + ts - 2. * t);
        const double vn = V3(vke, i, j - 1, k), vs = V3(vke, i, j, k);
        const double up = 0.5 * DT * V3(g->ddue, i, j - 1, k) * V2(g->dlxv, i, j - 1) * (vn + fabs(vn));
        const double um = 0.5 * DT * V3(g->ddue, i, j, k) * V2(g->dlxv, i, j) * (fabs(vs) - vs);
        const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20)) * P3(g->weto, i, j, k) *
                            P3(g->weto, i, j - 1, k) * P3(g->weto, i, j + 1, k);
        const double sch = fmn(1., scha * P3(s1o, i, j, k) / (up + um + 1.E-20));
        const double schi = 1. - sch;
        P3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + tn));
        M3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + ts));
        P3(wtp, i, j, k) = up;
        M3(wtm, i, j, k) = um;
      }
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        if (P3(g->weto, i, j, k) > 0.5) {
          const double rn = P3(s1o, i, j, k) + P3(wtp, i, j + 1, k) - P3(wtp, i, j, k) -
                            M3(wtm, i, j, k) + M3(wtm, i, j - 1, k);
          P3(t1o, i, j, k) = (P3(trf, i, j, k) * P3(s1o, i, j, k) + P3(trp, i, j + 1, k) -
                              P3(trp, i, j, k) - M3(trm, i, j, k) + M3(trm, i, j - 1, k)) /
                             rn;
          P3(s1o, i, j, k) = rn;
        }
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) P3(trf, i, j, k) = P3(t1o, i, j, k);
  }
  free(s1o); free(t1o); free(trp); free(wtp); free(trm); free(wtm);
}

/* ------------------------------------------------------------------------ */
/* OCUAD (ocuad.f90:1-271): u-points, TRF(I_start:IE,JE,KE), I_start = 0.   */
/* ------------------------------------------------------------------------ */
void og_ocuad(const og_grid *g, double *trf, const double *uko, const double *vke,
              const double *wo) {
  DIMS;
  const double DT = g->dt;
  const size_t n3 = (size_t)(IE + 1) * JE * KE, n0 = (size_t)(IE + 1) * JE * (KE + 1);
  double *trvol = zalloc(n3), *tr1 = zalloc(n3);
  double *trp = zalloc(n0), *wtp = zalloc(n0), *trm = zalloc(n0), *wtm = zalloc(n0);
  /* ocuad.f90:20-32 */
  for (int k = 1; k <= KE; ++k)
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i) {
        U3(trvol, i, j, k) = U3(g->amsuo, i, j, k) * U2(g->dlxu, i, j) * U2(g->dlyu, i, j) *
                             U3(g->dduo, i, j, k);
        U3(tr1, i, j, k) = U3(trf, i, j, k);
      }
  /* vertical, ocuad.f90:35-55 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    const int klo = k + 1 < KE ? k + 1 : KE;
    const int kup = k - 1 > 1 ? k - 1 : 1;
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i) {
        const double t = U3(trf, i, j, k), tu = U3(trf, i, j, kup), tl = U3(trf, i, j, klo);
        const double abl = fabs(tu - tl);
        const double zwabl = fabs(tu + tl - 2. * t);
        const double wup = 0.5 * (P3(wo, i, j, k) + P3(wo, i + 1, j, k));
        const double wlo = 0.5 * (P3(wo, i, j, k + 1) + P3(wo, i + 1, j, k + 1));
        const double up = 0.5 * DT * P2(g->dlyp, i, j) * P2(g->dlxp, i, j) * (wup + fabs(wup));
        const double um = 0.5 * DT * P2(g->dlyp, i, j) * P2(g->dlxp, i, j) * (fabs(wlo) - wlo);
        const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20));
        const double sch = fmn(1., scha * U3(trvol, i, j, k) / (up + um + 1.E-20));
        const double schi = 1. - sch;
        U3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + tu));
        MU3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + tl));
        U3(wtp, i, j, k) = up;
        MU3(wtm, i, j, k) = um;
      }
  }
  /* ocuad.f90:71-86 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i)
        if (U3(g->amsuo, i, j, k) > 0.5) {
          const double rn = U3(trvol, i, j, k) + U3(wtp, i, j, k + 1) - U3(wtp, i, j, k) -
                            MU3(wtm, i, j, k) + MU3(wtm, i, j, k - 1);
          U3(tr1, i, j, k) = (U3(trf, i, j, k) * U3(trvol, i, j, k) + U3(trp, i, j, k + 1) -
                              U3(trp, i, j, k) - MU3(trm, i, j, k) + MU3(trm, i, j, k - 1)) /
                             rn;
          U3(trvol, i, j, k) = rn;
        }
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i) U3(trf, i, j, k) = U3(tr1, i, j, k);
  }
  memset(trp, 0, sizeof(double) * n0); memset(trm, 0, sizeof(double) * n0);
  memset(wtp, 0, sizeof(double) * n0); memset(wtm, 0, sizeof(double) * n0);
  /* x-direction, ocuad.f90:99-148 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i) {
        const double t = U3(trf, i, j, k), te = U3(trf, i + 1, j, k), tw = U3(trf, i - 1, j, k);
        const double abl = fabs(te - tw);
        const double zwabl = fabs(te + tw - 2. * t);
        const double uos = 0.5 * (U3(uko, i, j, k) * U3(g->dduo, i, j, k) +
                                  U3(uko, i + 1, j, k) * U3(g->dduo, i + 1, j, k));
        const double uwe = 0.5 * (U3(uko, i - 1, j, k) * U3(g->dduo, i - 1, j, k) +
                                  U3(uko, i, j, k) * U3(g->dduo, i, j, k));
        const double up = 0.5 * DT * P2(g->dlyp, i + 1, j) * (uos + fabs(uos));
        const double um = 0.5 * DT * (fabs(uwe) - uwe) * P2(g->dlyp, i, j);
        const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20));
        const double sch = fmn(1., scha * U3(trvol, i, j, k) / (up + um + 1.E-20));
        const double schi = 1. - sch;
        U3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + te));
        MU3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + tw));
        U3(wtp, i, j, k) = up;
        MU3(wtm, i, j, k) = um;
      }
    for (int j = 2; j <= JE1; ++j) { /* have_g_is, I = 0 */
      const int i = 0;
      const double uos = 0.5 * (U3(uko, i, j, k) * U3(g->dduo, i, j, k) +
                                U3(uko, i + 1, j, k) * U3(g->dduo, i + 1, j, k));
      const double uwe = U3(uko, i, j, k) * U3(g->dduo, i, j, k);
      const double up = 0.5 * DT * P2(g->dlyp, i + 1, j) * (uos + fabs(uos));
      const double um = 0.5 * DT * (fabs(uwe) - uwe) * U2(g->dlyu, i, j);
      U3(trp, i, j, k) = up * U3(trf, i, j, k);
      MU3(trm, i, j, k) = um * U3(trf, i, j, k);
      U3(wtp, i, j, k) = up;
      MU3(wtm, i, j, k) = um;
    }
    for (int j = 2; j <= JE1; ++j) { /* have_g_ie, I = IE */
      const int i = IE;
      const double uos = U3(uko, i, j, k) * U3(g->dduo, i, j, k);
      const double uwe = 0.5 * (U3(uko, i - 1, j, k) * U3(g->dduo, i - 1, j, k) +
                                U3(uko, i, j, k) * U3(g->dduo, i, j, k));
      const double up = 0.5 * DT * P2(g->dlyp, i, j) * (uos + fabs(uos));
      const double um = 0.5 * DT * (fabs(uwe) - uwe) * U2(g->dlyu, i, j);
      U3(trp, i, j, k) = up * U3(trf, i, j, k);
      MU3(trm, i, j, k) = um * U3(trf, i, j, k);
      U3(wtp, i, j, k) = up;
      MU3(wtm, i, j, k) = um;
    }
  }
  /* ocuad.f90:157-172 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i)
        if (U3(g->amsuo, i, j, k) > 0.5) {
          const double rn = U3(trvol, i, j, k) + U3(wtp, i - 1, j, k) - U3(wtp, i, j, k) -
                            MU3(wtm, i, j, k) + MU3(wtm, i + 1, j, k);
          U3(tr1, i, j, k) = (U3(trf, i, j, k) * U3(trvol, i, j, k) + U3(trp, i - 1, j, k) -
                              U3(trp, i, j, k) - MU3(trm, i, j, k) + MU3(trm, i + 1, j, k)) /
                             rn;
          U3(trvol, i, j, k) = rn;
        }
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i) U3(trf, i, j, k) = U3(tr1, i, j, k);
  }
  memset(trp, 0, sizeof(double) * n0); memset(trm, 0, sizeof(double) * n0);
  memset(wtp, 0, sizeof(double) * n0); memset(wtm, 0, sizeof(double) * n0);
  /* y-direction, ocuad.f90:184-233 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i) {
        const double t = U3(trf, i, j, k), tn = U3(trf, i, j - 1, k), ts = U3(trf, i, j + 1, k);
        const double abl = fabs(tn - ts);
        const double zwabl = fabs(tn + ts - 2. * t);
        const double vsu = 0.5 * (V3(vke, i, j, k) * V3(g->ddue, i, j, k) +
                                  V3(vke, i + 1, j, k) * V3(g->ddue, i + 1, j, k));
        const double vno = 0.5 * (V3(vke, i, j - 1, k) * V3(g->ddue, i, j - 1, k) +
                                  V3(vke, i + 1, j - 1, k) * V3(g->ddue, i + 1, j - 1, k));
        const double up = 0.5 * DT * (0.5 * (V2(g->dlxv, i, j - 1) + V2(g->dlxv, i + 1, j - 1))) *
                          (vno + fabs(vno));
        const double um = 0.5 * DT * (0.5 * (V2(g->dlxv, i, j) + V2(g->dlxv, i + 1, j))) *
                          (fabs(vsu) - vsu);
        const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20));
        const double sch = fmn(1., scha * U3(trvol, i, j, k) / (up + um + 1.E-20));
        const double schi = 1. - sch;
        U3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + tn));
        MU3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + ts));
        U3(wtp, i, j, k) = up;
        MU3(wtm, i, j, k) = um;
      }
    for (int e = 0; e < 2; ++e) { /* have_g_js (J = 1) and have_g_je (J = JE) */
      const int j = e == 0 ? 1 : JE;
      for (int i = 1; i <= IE1; ++i) {
        const double vsu = 0.5 * (V3(vke, i, j, k) * V3(g->ddue, i, j, k) +
                                  V3(vke, i + 1, j, k) * V3(g->ddue, i + 1, j, k));
        const double vno = 0.5 * (V3(vke, i, j - 1, k) * V3(g->ddue, i, j - 1, k) +
                                  V3(vke, i + 1, j - 1, k) * V3(g->ddue, i + 1, j - 1, k));
        const double up = 0.5 * DT * (0.5 * (V2(g->dlxv, i, j - 1) + V2(g->dlxv, i + 1, j - 1))) *
                          (vno + fabs(vno));
        const double um = 0.5 * DT * (0.5 * (V2(g->dlxv, i, j) + V2(g->dlxv, i + 1, j))) *
                          (fabs(vsu) - vsu);
        U3(trp, i, j, k) = up * U3(trf, i, j, k);
        MU3(trm, i, j, k) = um * U3(trf, i, j, k);
        U3(wtp, i, j, k) = up;
        MU3(wtm, i, j, k) = um;
      }
    }
  }
  /* ocuad.f90:242-257 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i)
        if (U3(g->amsuo, i, j, k) > 0.5) {
          const double rn = U3(trvol, i, j, k) + U3(wtp, i, j + 1, k) - U3(wtp, i, j, k) -
                            MU3(wtm, i, j, k) + MU3(wtm, i, j - 1, k);
          U3(tr1, i, j, k) = (U3(trf, i, j, k) * U3(trvol, i, j, k) + U3(trp, i, j + 1, k) -
                              U3(trp, i, j, k) - MU3(trm, i, j, k) + MU3(trm, i, j - 1, k)) /
                             rn;
          U3(trvol, i, j, k) = rn;
        }
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i) U3(trf, i, j, k) = U3(tr1, i, j, k);
  }
  free(trvol); free(tr1); free(trp); free(wtp); free(trm); free(wtm);
}

/* ------------------------------------------------------------------------ */
/* OCVAD (ocvad.f90:1-271): v-points, TRF(IE,J_start:JE,KE), J_start = 0.   */
/* The J = 0 edge flux reads DLXU(I,0) (ocvad.f90:211), an element outside  */
/* DLXU's bounds (J from 1): the restatement reads DLXV(I,0), the zonal     */
/* width at that v-point, in its place.                                    */
/* ------------------------------------------------------------------------ */
void og_ocvad(const og_grid *g, double *trf, const double *uko, const double *vke,
              const double *wo) {
  DIMS;
  const double DT = g->dt;
  const size_t n3 = (size_t)IE * (JE + 1) * KE, n0 = (size_t)IE * (JE + 1) * (KE + 1);
  double *trvol = zalloc(n3), *tr1 = zalloc(n3);
  double *trp = zalloc(n0), *wtp = zalloc(n0), *trm = zalloc(n0), *wtm = zalloc(n0);
  for (int k = 1; k <= KE; ++k)
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        V3(trvol, i, j, k) = V3(g->amsue, i, j, k) * V2(g->dlxv, i, j) * V2(g->dlyv, i, j) *
                             V3(g->ddue, i, j, k);
        V3(tr1, i, j, k) = V3(trf, i, j, k);
      }
  /* vertical, ocvad.f90:35-55 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    const int klo = k + 1 < KE ? k + 1 : KE;
    const int kup = k - 1 > 1 ? k - 1 : 1;
    for (int j = 1; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        const double t = V3(trf, i, j, k), tu = V3(trf, i, j, kup), tl = V3(trf, i, j, klo);
        const double abl = fabs(tu - tl);
        const double zwabl = fabs(tu + tl - 2. * t);
        const double wup = 0.5 * (P3(wo, i, j, k) + P3(wo, i, j + 1, k));
        const double wlo = 0.5 * (P3(wo, i, j, k + 1) + P3(wo, i, j + 1, k + 1));
        const double up = 0.5 * DT * P2(g->dlyp, i, j) * P2(g->dlxp, i, j) * (wup + fabs(wup));
        const double um = 0.5 * DT * P2(g->dlyp, i, j) * P2(g->dlxp, i, j) * (fabs(wlo) - wlo);
        const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20));
        const double sch = fmn(1., scha * V3(trvol, i, j, k) / (up + um + 1.E-20));
        const double schi = 1. - sch;
        V3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + tu));
        MV3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + tl));
        V3(wtp, i, j, k) = up;
        MV3(wtm, i, j, k) = um;
      }
  }
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        if (V3(g->amsue, i, j, k) > 0.5) {
          const double rn = V3(trvol, i, j, k) + V3(wtp, i, j, k + 1) - V3(wtp, i, j, k) -
                            MV3(wtm, i, j, k) + MV3(wtm, i, j, k - 1);
          V3(tr1, i, j, k) = (V3(trf, i, j, k) * V3(trvol, i, j, k) + V3(trp, i, j, k + 1) -
                              V3(trp, i, j, k) - MV3(trm, i, j, k) + MV3(trm, i, j, k - 1)) /
                             rn;
          V3(trvol, i, j, k) = rn;
        }
    for (int j = 1; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) V3(trf, i, j, k) = V3(tr1, i, j, k);
  }
  memset(trp, 0, sizeof(double) * n0); memset(trm, 0, sizeof(double) * n0);
  memset(wtp, 0, sizeof(double) * n0); memset(wtm, 0, sizeof(double) * n0);
  /* x-direction, ocvad.f90:99-148 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE1; ++j)
      for (int i = 1; i <= IE; ++i) {
        const int edge = (i == 1 || i == IE);
        const double t = V3(trf, i, j, k);
        const double uos = 0.5 * (U3(uko, i, j, k) * U3(g->dduo, i, j, k) +
                                  U3(uko, i, j + 1, k) * U3(g->dduo, i, j + 1, k));
        const double uwe = 0.5 * (U3(uko, i - 1, j, k) * U3(g->dduo, i - 1, j, k) +
                                  U3(uko, i - 1, j + 1, k) * U3(g->dduo, i - 1, j + 1, k));
        const double up = 0.5 * DT * (0.5 * (U2(g->dlyu, i, j) + U2(g->dlyu, i, j + 1))) *
                          (uos + fabs(uos));
        const double um = 0.5 * DT * (fabs(uwe) - uwe) *
                          (0.5 * (U2(g->dlyu, i - 1, j) + U2(g->dlyu, i - 1, j + 1)));
        if (edge) { /* have_g_is / have_g_ie rows, ocvad.f90:120-148 */
          V3(trp, i, j, k) = up * t;
          MV3(trm, i, j, k) = um * t;
        } else {
          const double te = V3(trf, i + 1, j, k), tw = V3(trf, i - 1, j, k);
          const double abl = fabs(te - tw);
          const double zwabl = fabs(te + tw - 2. * t);
          const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20));
          const double sch = fmn(1., scha * V3(trvol, i, j, k) / (up + um + 1.E-20));
          const double schi = 1. - sch;
          V3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + te));
          MV3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + tw));
        }
        V3(wtp, i, j, k) = up;
        MV3(wtm, i, j, k) = um;
      }
  }
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        if (V3(g->amsue, i, j, k) > 0.5) {
          const double rn = V3(trvol, i, j, k) + V3(wtp, i - 1, j, k) - V3(wtp, i, j, k) -
                            MV3(wtm, i, j, k) + MV3(wtm, i + 1, j, k);
          V3(tr1, i, j, k) = (V3(trf, i, j, k) * V3(trvol, i, j, k) + V3(trp, i - 1, j, k) -
                              V3(trp, i, j, k) - MV3(trm, i, j, k) + MV3(trm, i + 1, j, k)) /
                             rn;
          V3(trvol, i, j, k) = rn;
        }
    for (int j = 1; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) V3(trf, i, j, k) = V3(tr1, i, j, k);
  }
  memset(trp, 0, sizeof(double) * n0); memset(trm, 0, sizeof(double) * n0);
  memset(wtp, 0, sizeof(double) * n0); memset(wtm, 0, sizeof(double) * n0);
  /* y-direction, ocvad.f90:184-233 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        const double t = V3(trf, i, j, k), tn = V3(trf, i, j - 1, k), ts = V3(trf, i, j + 1, k);
        const double abl = fabs(tn - ts);
        const double zwabl = fabs(tn + ts - 2. * t);
        const double vno = 0.5 * (V3(vke, i, j, k) * V3(g->ddue, i, j, k) +
                                  V3(vke, i, j - 1, k) * V3(g->ddue, i, j - 1, k));
        const double vsu = 0.5 * (V3(vke, i, j, k) * V3(g->ddue, i, j, k) +
                                  V3(vke, i, j + 1, k) * V3(g->ddue, i, j + 1, k));
        const double up = 0.5 * DT * P2(g->dlxp, i, j) * (vno + fabs(vno));
        const double um = 0.5 * DT * P2(g->dlxp, i, j + 1) * (fabs(vsu) - vsu);
        const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20));
        const double sch = fmn(1., scha * V3(trvol, i, j, k) / (up + um + 1.E-20));
        const double schi = 1. - sch;
        V3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + tn));
        MV3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + ts));
        V3(wtp, i, j, k) = up;
        MV3(wtm, i, j, k) = um;
      }
    for (int i = 2; i <= IE1; ++i) { /* have_g_js, J = 0 */
      const int j = 0;
      const double vno = V3(vke, i, j, k) * V3(g->ddue, i, j, k);
      const double vsu = 0.5 * (V3(vke, i, j, k) * V3(g->ddue, i, j, k) +
                                V3(vke, i, j + 1, k) * V3(g->ddue, i, j + 1, k));
      const double up = 0.5 * DT * V2(g->dlxv, i, j) * (vno + fabs(vno)); /* DLXU(I,0) in ref */
      const double um = 0.5 * DT * P2(g->dlxp, i, j + 1) * (fabs(vsu) - vsu);
      V3(trp, i, j, k) = up * V3(trf, i, j, k);
      MV3(trm, i, j, k) = um * V3(trf, i, j, k);
      V3(wtp, i, j, k) = up;
      MV3(wtm, i, j, k) = um;
    }
    for (int i = 2; i <= IE1; ++i) { /* have_g_je, J = JE */
      const int j = JE;
      const double vno = 0.5 * (V3(vke, i, j, k) * V3(g->ddue, i, j, k) +
                                V3(vke, i, j - 1, k) * V3(g->ddue, i, j - 1, k));
      const double vsu = V3(vke, i, j, k) * V3(g->ddue, i, j, k);
      const double up = 0.5 * DT * P2(g->dlxp, i, j) * (vno + fabs(vno));
      const double um = 0.5 * DT * U2(g->dlxu, i, j) * (fabs(vsu) - vsu);
      V3(trp, i, j, k) = up * V3(trf, i, j, k);
      MV3(trm, i, j, k) = um * V3(trf, i, j, k);
      V3(wtp, i, j, k) = up;
      MV3(wtm, i, j, k) = um;
    }
  }
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        if (V3(g->amsue, i, j, k) > 0.5) {
          const double rn = V3(trvol, i, j, k) + V3(wtp, i, j + 1, k) - V3(wtp, i, j, k) -
                            MV3(wtm, i, j, k) + MV3(wtm, i, j - 1, k);
          V3(tr1, i, j, k) = (V3(trf, i, j, k) * V3(trvol, i, j, k) + V3(trp, i, j + 1, k) -
                              V3(trp, i, j, k) - MV3(trm, i, j, k) + MV3(trm, i, j - 1, k)) /
                             rn;
          V3(trvol, i, j, k) = rn;
        }
    for (int j = 1; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) V3(trf, i, j, k) = V3(tr1, i, j, k);
  }
  free(trvol); free(tr1); free(trp); free(wtp); free(trm); free(wtm);
}

/* ------------------------------------------------------------------------ */
/* OCWAD (ocwad.f90:1-238): w-points, TRF(IE,JE,KEP).  At K = KE the        */
/* vertical limiter reads WETO(I,J,KEP) (ocwad.f90:63), one level past      */
/* WETO's last level: the restatement takes it as 0 (no water below the    */
/* deepest level), which makes that interface first-order upwind.          */
/* ------------------------------------------------------------------------ */
void og_ocwad(const og_grid *g, double *trf, const double *uko, const double *vke,
              const double *wo, const double *zo) {
  DIMS;
  const double DT = g->dt;
  const size_t n3 = (size_t)IE * JE * KE, n0 = (size_t)IE * JE * (KE + 1);
  double *s1o = zalloc(n3), *t1o = zalloc(n3);
  double *trp = zalloc(n0), *wtp = zalloc(n0), *trm = zalloc(n0), *wtm = zalloc(n0);
  /* ocwad.f90:14-37 */
  for (int k = 1; k <= KE; ++k)
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        P3(t1o, i, j, k) = P3(trf, i, j, k);
        const double a = P3(g->weto, i, j, k) * P2(g->dlxp, i, j) * P2(g->dlyp, i, j);
        if (k == 1)
          P3(s1o, i, j, k) = a * (P3(g->ddpo, i, j, k) + P2(zo, i, j)) / 2.0;
        else if (k == 2)
          P3(s1o, i, j, k) = a * (P3(g->ddpo, i, j, k - 1) + P3(g->ddpo, i, j, k) + P2(zo, i, j)) / 2.0;
        else
          P3(s1o, i, j, k) = a * (P3(g->ddpo, i, j, k - 1) + P3(g->ddpo, i, j, k)) / 2.0;
      }
  /* vertical, ocwad.f90:50-69 */
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= KE; ++k) {
    const int klo = k + 1, kup = k - 1;
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        const double t = P3(trf, i, j, k), tu = P3(trf, i, j, kup), tl = P3(trf, i, j, klo);
        const double abl = fabs(tu - tl);
        const double zwabl = fabs(tu + tl - 2. * t);
        const double wup = 0.5 * (P3(wo, i, j, k) + P3(wo, i, j, kup));
        const double wum = 0.5 * (P3(wo, i, j, k) + P3(wo, i, j, klo));
        const double up = 0.5 * DT * P2(g->dlyp, i, j) * P2(g->dlxp, i, j) * (wup + fabs(wup));
        const double um = 0.5 * DT * P2(g->dlyp, i, j) * P2(g->dlxp, i, j) * (fabs(wum) - wum);
        const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20));
        const double wklo = klo <= KE ? P3(g->weto, i, j, klo) : 0.0;
        const double sch = fmn(wklo, scha * P3(s1o, i, j, k) / (up + um + 1.E-20));
        const double schi = 1. - sch;
        P3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + tu));
        M3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + tl));
        P3(wtp, i, j, k) = up;
        M3(wtm, i, j, k) = um;
      }
  }
  /* ocwad.f90:72-83 */
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      const double wup = 0.5 * (P3(wo, i, j, KEP) + P3(wo, i, j, KE));
      const double up = 0.5 * DT * P2(g->dlyp, i, j) * P2(g->dlxp, i, j) * (wup + fabs(wup));
      P3(trp, i, j, KEP) = up * (0.5 * (P3(trf, i, j, KE) + P3(trf, i, j, KEP)));
      P3(wtp, i, j, KEP) = up;
      const double wum = 0.5 * (P3(wo, i, j, 1) + P3(wo, i, j, 2));
      const double um = 0.5 * DT * P2(g->dlyp, i, j) * P2(g->dlxp, i, j) * (fabs(wum) - wum);
      M3(trm, i, j, 1) = um * (0.5 * (P3(trf, i, j, 1) + P3(trf, i, j, 2)));
      M3(wtm, i, j, 1) = um;
    }
  /* ocwad.f90:88-102 */
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        if (P3(g->weto, i, j, k) > 0.5) {
          const double rn = P3(s1o, i, j, k) + P3(wtp, i, j, k + 1) - P3(wtp, i, j, k) -
                            M3(wtm, i, j, k) + M3(wtm, i, j, k - 1);
          P3(t1o, i, j, k) = (P3(trf, i, j, k) * P3(s1o, i, j, k) + P3(trp, i, j, k + 1) -
                              P3(trp, i, j, k) - M3(trm, i, j, k) + M3(trm, i, j, k - 1)) /
                             rn;
          P3(s1o, i, j, k) = rn;
        }
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) P3(trf, i, j, k) = P3(t1o, i, j, k);
  }
  /* x-direction, ocwad.f90:110-165 (TRP etc. keep their vertical values
   * elsewhere; only zero entries at the halo columns are read) */
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        const double t = P3(trf, i, j, k), te = P3(trf, i + 1, j, k), tw = P3(trf, i - 1, j, k);
        const double abl = fabs(te - tw);
        const double zwabl = fabs(te + tw - 2. * t);
        const double uos = 0.5 * (U3(uko, i, j, k) * U3(g->dduo, i, j, k) +
                                  U3(uko, i, j, k - 1) * U3(g->dduo, i, j, k - 1));
        const double uwe = 0.5 * (U3(uko, i - 1, j, k) * U3(g->dduo, i - 1, j, k) +
                                  U3(uko, i - 1, j, k - 1) * U3(g->dduo, i - 1, j, k - 1));
        const double up = 0.5 * DT * U2(g->dlyu, i, j) * (uos + fabs(uos));
        const double um = 0.5 * DT * U2(g->dlyu, i - 1, j) * (fabs(uwe) - uwe);
        const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20)) * P3(g->weto, i, j, k) *
                            P3(g->weto, i + 1, j, k) * P3(g->weto, i - 1, j, k);
        const double sch = fmn(1., scha * P3(s1o, i, j, k) / (up + um + 1.E-20));
        const double schi = 1. - sch;
        P3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + te));
        M3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + tw));
        P3(wtp, i, j, k) = up;
        M3(wtm, i, j, k) = um;
      }
  }
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        if (P3(g->weto, i, j, k) > 0.5) {
          const double rn = P3(s1o, i, j, k) + P3(wtp, i - 1, j, k) - P3(wtp, i, j, k) -
                            M3(wtm, i, j, k) + M3(wtm, i + 1, j, k);
          P3(t1o, i, j, k) = (P3(trf, i, j, k) * P3(s1o, i, j, k) + P3(trp, i - 1, j, k) -
                              P3(trp, i, j, k) - M3(trm, i, j, k) + M3(trm, i + 1, j, k)) /
                             rn;
          P3(s1o, i, j, k) = rn;
        }
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) P3(trf, i, j, k) = P3(t1o, i, j, k);
  }
  /* y-direction, ocwad.f90:173-228 */
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        const double t = P3(trf, i, j, k), tn = P3(trf, i, j - 1, k), ts = P3(trf, i, j + 1, k);
        const double abl = fabs(tn - ts);
        const double zwabl = fabs(tn + ts - 2. * t);
        const double vsu = 0.5 * (V3(vke, i, j, k) * V3(g->ddue, i, j, k) +
                                  V3(vke, i, j, k - 1) * V3(g->ddue, i, j, k - 1));
        const double vno = 0.5 * (V3(vke, i, j - 1, k) * V3(g->ddue, i, j - 1, k) +
                                  V3(vke, i, j - 1, k - 1) * V3(g->ddue, i, j - 1, k - 1));
        const double up = 0.5 * DT * V2(g->dlxv, i, j - 1) * (vno + fabs(vno));
        const double um = 0.5 * DT * V2(g->dlxv, i, j) * (fabs(vsu) - vsu);
        const double scha = fmx(0., (abl - zwabl) / (abl + 1.E-20)) * P3(g->weto, i, j, k) *
                            P3(g->weto, i, j - 1, k) * P3(g->weto, i, j + 1, k);
        const double sch = fmn(1., scha * P3(s1o, i, j, k) / (up + um + 1.E-20));
        const double schi = 1. - sch;
        P3(trp, i, j, k) = up * (schi * t + sch * 0.5 * (t + tn));
        M3(trm, i, j, k) = um * (schi * t + sch * 0.5 * (t + ts));
        P3(wtp, i, j, k) = up;
        M3(wtm, i, j, k) = um;
      }
  }
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        if (P3(g->weto, i, j, k) > 0.5) {
          const double rn = P3(s1o, i, j, k) + P3(wtp, i, j + 1, k) - P3(wtp, i, j, k) -
                            M3(wtm, i, j, k) + M3(wtm, i, j - 1, k);
          P3(t1o, i, j, k) = (P3(trf, i, j, k) * P3(s1o, i, j, k) + P3(trp, i, j + 1, k) -
                              P3(trp, i, j, k) - M3(trm, i, j, k) + M3(trm, i, j - 1, k)) /
                             rn;
          P3(s1o, i, j, k) = rn;
        }
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) P3(trf, i, j, k) = P3(t1o, i, j, k);
  }
  free(s1o); free(t1o); free(trp); free(wtp); free(trm); free(wtm);
}

/* ------------------------------------------------------------------------ */
/* OCTDIFF_BASE (octdiff_base.f90:182-221) + OCTDIFF_TS                     */
/* (octdiff_ts.f90:51-59, 282-407) generalised from (THO,SAO) to ntr        */
/* tracers, each treated exactly as THO.  Harmonic/isopycnal diffusion      */
/* (AH00 > ALMZER) is not restated: the caller must pass AH00 = 0, as all   */
/* verification runs do (OCECTL CAH00 = 0).  VOL_TERM is only assigned      */
/* under AH00 > ALMZER, so it is taken as 0 here and T1O at the halo cells, */
/* which the biharmonic second pass reads, is 0.  I3DREST = 0.             */
/* ------------------------------------------------------------------------ */
void og_octdiff(const og_grid *g, int ntr, double *const *tr, const double *dvo,
                const double *zo) {
  DIMS;
  const double DT = g->dt, ALMZER = g->almzer;
  const size_t n3 = (size_t)IE * JE * KE;
  double *t1o = zalloc(n3);
  /* vertical implicit diffusion, octdiff_base.f90:182-204 + octdiff_ts.f90:294-324 */
#pragma omp parallel
  {
    double *t1 = (double *)malloc(sizeof(double) * (size_t)KE * 3 + 8);
    double *t2 = t1 + KE, *t3 = t2 + KE;
    double *col = (double *)malloc(sizeof(double) * (size_t)KE + 8);
#pragma omp for schedule(static)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        for (int k = 1; k <= KE; ++k) {
          const double zzsurf = k == 1 ? 1. : 0.;
          const double den = P3(g->ddpo, i, j, k) + zzsurf * (P2(zo, i, j)) + ALMZER;
          t1[k - 1] = -DT * P3(dvo, i, j, k) * P3(g->weto, i, j, k) * K1(g->di, k) / den;
          t3[k - 1] = -DT * P3(dvo, i, j, k + 1) * K1(g->di, k + 1) / den;
          t2[k - 1] = 1. - t1[k - 1] - t3[k - 1];
        }
        for (int k = 2; k <= KE; ++k) {
          const double a = t1[k - 1];
          t1[k - 2] = a / t2[k - 2];
          t2[k - 1] = t2[k - 1] - t3[k - 2] * a / t2[k - 2];
        }
        for (int n = 0; n < ntr; ++n) {
          double *T = tr[n];
          for (int k = 1; k <= KE; ++k) col[k - 1] = P3(T, i, j, k);
          for (int k = 2; k <= KE; ++k) col[k - 1] = col[k - 1] - t1[k - 2] * col[k - 2];
          P3(T, i, j, KE) = col[KE - 1] / t2[KE - 1];
          for (int k = 1; k <= KE - 1; ++k) {
            const int l = KE - k;
            P3(T, i, j, l) = (col[l - 1] - t3[l - 1] * P3(T, i, j, l + 1)) / t2[l - 1];
          }
        }
      }
    free(t1);
    free(col);
  }
  /* biharmonic, octdiff_base.f90:208-221 + octdiff_ts.f90:344-407 */
  if (g->aulapts > ALMZER) {
    double *aulx = zalloc((size_t)IE * JE), *auly = zalloc((size_t)IE * JE);
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        const double x = U2(g->dlxu, i, j), y = V2(g->dlyv, i, j);
        P2(aulx, i, j) = g->aulapts * ((x * x) * (x * x));
        P2(auly, i, j) = g->aulapts * ((y * y) * (y * y));
      }
    for (int n = 0; n < ntr; ++n) {
      double *T = tr[n];
      memset(t1o, 0, sizeof(double) * n3);
#pragma omp parallel for schedule(static)
      for (int k = 1; k <= KE; ++k)
        for (int j = 2; j <= JE1; ++j)
          for (int i = 2; i <= IE1; ++i) {
            const double c = P3(T, i, j, k);
            P3(t1o, i, j, k) =
                P3(g->weto, i, j, k) *
                ((P3(g->weto, i - 1, j, k) * (P3(T, i - 1, j, k) - c) / U2(g->dlxu, i - 1, j) +
                  P3(g->weto, i + 1, j, k) * (P3(T, i + 1, j, k) - c) / U2(g->dlxu, i, j)) /
                     P2(g->dlxp, i, j) +
                 (P3(g->weto, i, j - 1, k) * (P3(T, i, j - 1, k) - c) / V2(g->dlyv, i, j - 1) +
                  P3(g->weto, i, j + 1, k) * (P3(T, i, j + 1, k) - c) / V2(g->dlyv, i, j)) /
                     P2(g->dlyp, i, j));
          }
#pragma omp parallel for schedule(static)
      for (int k = 1; k <= KE; ++k) {
        const double zzsurf = k == 1 ? 1. : 0.;
        for (int j = 2; j <= JE1; ++j)
          for (int i = 2; i <= IE1; ++i) {
            const double c = P3(t1o, i, j, k);
            const double den = (P3(g->ddpo, i, j, k) + ALMZER + zzsurf * (P2(zo, i, j))) *
                               P2(g->dlxp, i, j) * P2(g->dlyp, i, j);
            P3(T, i, j, k) =
                P3(T, i, j, k) -
                (P3(g->weto, i, j, k) / den) * K1(g->dzw, k) *
                    (P3(g->weto, i - 1, j, k) * P2(aulx, i - 1, j) * U2(g->dlyu, i - 1, j) *
                         (P3(t1o, i - 1, j, k) - c) / U2(g->dlxu, i - 1, j) +
                     P3(g->weto, i + 1, j, k) * P2(aulx, i, j) * U2(g->dlyu, i, j) *
                         (P3(t1o, i + 1, j, k) - c) / U2(g->dlxu, i, j) +
                     P3(g->weto, i, j - 1, k) * P2(auly, i, j - 1) * V2(g->dlxv, i, j - 1) *
                         (P3(t1o, i, j - 1, k) - c) / V2(g->dlyv, i, j - 1) +
                     P3(g->weto, i, j + 1, k) * P2(auly, i, j) * V2(g->dlxv, i, j) *
                         (P3(t1o, i, j + 1, k) - c) / V2(g->dlyv, i, j));
          }
      }
    }
    free(aulx);
    free(auly);
  }
  free(t1o);
}

/* ------------------------------------------------------------------------ */
/* OCVISC (ocvisc.f90:37-478, 615-688), FREESLIP branch (Makefile:47),      */
/* AULREDUV off; x**4 is evaluated as (x*x)*(x*x).  Ends with OCTIMF.       */
/* ------------------------------------------------------------------------ */
void og_ocvisc(const og_grid *g, double *uoo, double *voe, double *wno,
               double *uko, double *vke, const double *avo) {
  DIMS;
  const double DT = g->dt, ALMZER = g->almzer, AULAPUV = g->aulapuv;
  const double minvalue = fmn(1.0, K1(g->dzw, 1) / 10.0);
  const double BOFRIC = 3.E-3, RAYFRIC = 3.E-3;
  double *speedu = zalloc((size_t)IE * JE), *speedv = zalloc((size_t)IE * JE);
  /* ocvisc.f90:53-104 */
  for (int j = 2; j <= JE1; ++j) {
    for (int k = 1; k <= KE - 1; ++k)
      for (int i = 1; i <= IE1; ++i)
        if (U3(g->amsuo, i, j, k) - U3(g->amsuo, i, j, k + 1) > 0.5) {
          const double a = 0.25 * (V3(voe, i, j, k) + V3(voe, i + 1, j, k) + V3(voe, i, j - 1, k) +
                                   V3(voe, i + 1, j - 1, k));
          const double u = U3(uoo, i, j, k);
          P2(speedu, i, j) = fmx(sqrt(u * u + a * a), 1.E-3);
        }
    for (int i = 1; i <= IE1; ++i)
      if (U3(g->amsuo, i, j, KE) > 0.5) {
        const int k = KE;
        const double a = 0.25 * (V3(voe, i, j, k) + V3(voe, i + 1, j, k) + V3(voe, i, j - 1, k) +
                                 V3(voe, i + 1, j - 1, k));
        const double u = U3(uoo, i, j, k);
        P2(speedu, i, j) = fmx(sqrt(u * u + a * a), 1.E-3);
      }
  }
  for (int j = 1; j <= JE1; ++j) {
    for (int k = 1; k <= KE - 1; ++k)
      for (int i = 2; i <= IE1; ++i)
        if (V3(g->amsue, i, j, k) - V3(g->amsue, i, j, k + 1) > 0.5) {
          const double a = 0.25 * (U3(uoo, i, j, k) + U3(uoo, i - 1, j, k) + U3(uoo, i, j + 1, k) +
                                   U3(uoo, i - 1, j + 1, k));
          const double v = V3(voe, i, j, k);
          P2(speedv, i, j) = fmx(sqrt(v * v + a * a), 1.E-3);
        }
    for (int i = 2; i <= IE1; ++i)
      if (V3(g->amsue, i, j, KE) > 0.5) {
        const int k = KE;
        const double a = 0.25 * (U3(uoo, i, j, k) + U3(uoo, i - 1, j, k) + U3(uoo, i, j + 1, k) +
                                 U3(uoo, i - 1, j + 1, k));
        const double v = V3(voe, i, j, k);
        P2(speedv, i, j) = fmx(sqrt(v * v + a * a), 1.E-3);
      }
  }
  /* vertical diffusion of v, ocvisc.f90:114-165 */
#pragma omp parallel
  {
    double *t1 = (double *)malloc(sizeof(double) * (size_t)(KE + 1) * 3 + 8);
    double *t2 = t1 + (KE + 1), *t3 = t2 + (KE + 1);
    double *x1 = (double *)malloc(sizeof(double) * (size_t)(KE + 1) + 8);
#define TR1(k) t1[(k)-1]
#define TR2(k) t2[(k)-1]
#define TR3(k) t3[(k)-1]
#pragma omp for schedule(static)
    for (int i = 2; i <= IE1; ++i)
      for (int j = 1; j <= JE1; ++j) {
        for (int k = 1; k <= KE - 1; ++k) {
          const double avup = 0.5 * (P3(avo, i, j, k) + P3(avo, i, j + 1, k)) * V3(g->amsue, i, j, k);
          const double avlo = 0.5 * (P3(avo, i, j, k + 1) + P3(avo, i, j + 1, k + 1)) *
                                  V3(g->amsue, i, j, k + 1) +
                              (BOFRIC + RAYFRIC * V3(g->ddue, i, j, k) * P2(speedv, i, j)) *
                                  (V3(g->amsue, i, j, k) - V3(g->amsue, i, j, k + 1));
          TR1(k) = -DT * avup * V3(g->amsue, i, j, k) * K1(g->di, k) / (ALMZER + V3(g->ddue, i, j, k));
          TR3(k) = -DT * avlo * V3(g->amsue, i, j, k) * K1(g->di, k + 1) / (ALMZER + V3(g->ddue, i, j, k));
          TR2(k) = 1. - TR1(k) - TR3(k);
          TR3(k) = TR3(k) * V3(g->amsue, i, j, k + 1);
        }
        {
          const int k = KE;
          const double avup = 0.5 * (P3(avo, i, j, k) + P3(avo, i, j + 1, k)) * V3(g->amsue, i, j, k);
          const double avlo = (BOFRIC + RAYFRIC * V3(g->ddue, i, j, k) * P2(speedv, i, j)) *
                              V3(g->amsue, i, j, k);
          TR1(k) = -DT * avup * V3(g->amsue, i, j, k) * K1(g->di, k) / (ALMZER + V3(g->ddue, i, j, k));
          TR3(k) = -DT * avlo * V3(g->amsue, i, j, k) * K1(g->di, k + 1) / (ALMZER + V3(g->ddue, i, j, k));
          TR2(k) = 1. - TR1(k) - TR3(k);
          TR3(k) = 0.;
        }
        for (int k = 2; k <= KE; ++k) {
          const double a = TR1(k);
          TR1(k - 1) = a / TR2(k - 1);
          TR2(k) = TR2(k) - TR3(k - 1) * a / TR2(k - 1);
        }
        for (int k = 1; k <= KE; ++k) x1[k] = V3(voe, i, j, k);
        for (int k = 2; k <= KE; ++k) x1[k] = x1[k] - TR1(k - 1) * x1[k - 1];
        V3(vke, i, j, KE) = V3(g->amsue, i, j, KE) * x1[KE] / TR2(KE);
        for (int k = 1; k <= KE - 1; ++k) {
          const int l = KE - k;
          V3(vke, i, j, l) = (x1[l] - TR3(l) * V3(vke, i, j, l + 1)) * V3(g->amsue, i, j, l) / TR2(l);
        }
      }
    /* vertical diffusion of u, ocvisc.f90:168-218 */
#pragma omp for schedule(static)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i) {
        for (int k = 1; k <= KE - 1; ++k) {
          const double avup = 0.5 * (P3(avo, i, j, k) + P3(avo, i + 1, j, k)) * U3(g->amsuo, i, j, k);
          const double avlo = 0.5 * (P3(avo, i, j, k + 1) + P3(avo, i + 1, j, k + 1)) *
                                  U3(g->amsuo, i, j, k + 1) +
                              (BOFRIC + RAYFRIC * U3(g->dduo, i, j, k) * P2(speedu, i, j)) *
                                  (U3(g->amsuo, i, j, k) - U3(g->amsuo, i, j, k + 1));
          TR1(k) = -DT * avup * U3(g->amsuo, i, j, k) * K1(g->di, k) / (ALMZER + U3(g->dduo, i, j, k));
          TR3(k) = -DT * avlo * U3(g->amsuo, i, j, k) * K1(g->di, k + 1) / (ALMZER + U3(g->dduo, i, j, k));
          TR2(k) = 1. - TR1(k) - TR3(k);
          TR3(k) = TR3(k) * U3(g->amsuo, i, j, k + 1);
        }
        {
          const int k = KE;
          const double avup = 0.5 * (P3(avo, i, j, k) + P3(avo, i + 1, j, k)) * U3(g->amsuo, i, j, k);
          const double avlo = (BOFRIC + RAYFRIC * U3(g->dduo, i, j, k) * P2(speedu, i, j)) *
                              U3(g->amsuo, i, j, k);
          TR1(k) = -DT * avup * U3(g->amsuo, i, j, k) * K1(g->di, k) / (ALMZER + U3(g->dduo, i, j, k));
          TR3(k) = -DT * avlo * U3(g->amsuo, i, j, k) * K1(g->di, k + 1) / (ALMZER + U3(g->dduo, i, j, k));
          TR2(k) = 1. - TR1(k) - TR3(k);
          TR3(k) = 0.;
        }
        for (int k = 2; k <= KE; ++k) {
          const double a = TR1(k);
          TR1(k - 1) = a / TR2(k - 1);
          TR2(k) = TR2(k) - TR3(k - 1) * a / TR2(k - 1);
        }
        for (int k = 1; k <= KE; ++k) x1[k] = U3(uoo, i, j, k);
        for (int k = 2; k <= KE; ++k) x1[k] = x1[k] - TR1(k - 1) * x1[k - 1];
        U3(uko, i, j, KE) = U3(g->amsuo, i, j, KE) * x1[KE] / TR2(KE);
        for (int k = 1; k <= KE - 1; ++k) {
          const int l = KE - k;
          U3(uko, i, j, l) = (x1[l] - TR3(l) * U3(uko, i, j, l + 1)) * U3(g->amsuo, i, j, l) / TR2(l);
        }
      }
    /* vertical diffusion of w, ocvisc.f90:225-270 */
#pragma omp for schedule(static)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        for (int k = 2; k <= KE - 1; ++k) {
          const double avup = 0.5 * (P3(avo, i, j, k - 1) + P3(avo, i, j, k)) * P3(g->weto, i, j, k - 1);
          const double avlo = 0.5 * (P3(avo, i, j, k + 1) + P3(avo, i, j, k)) * P3(g->weto, i, j, k);
          const double den = 2.0 * ALMZER + P3(g->ddpo, i, j, k - 1) + P3(g->ddpo, i, j, k);
          TR1(k) = -2.0 * DT * avup * P3(g->weto, i, j, k) * K1(g->di, k - 1) / den;
          TR3(k) = -2.0 * DT * avlo * P3(g->weto, i, j, k) * K1(g->di, k) / den;
          TR2(k) = 1. - TR1(k) - TR3(k);
        }
        {
          const int k = KE;
          const double avup = 0.5 * (P3(avo, i, j, k - 1) + P3(avo, i, j, k)) * P3(g->weto, i, j, k - 1);
          const double avlo = 0.0;
          const double den = 2.0 * ALMZER + P3(g->ddpo, i, j, k - 1) + P3(g->ddpo, i, j, k);
          TR1(k) = -2.0 * DT * avup * P3(g->weto, i, j, k) * K1(g->di, k - 1) / den;
          TR3(k) = -2.0 * DT * avlo * P3(g->weto, i, j, k) * K1(g->di, k) / den;
          TR2(k) = 1. - TR1(k) - TR3(k);
          TR3(k) = 0.;
        }
        for (int k = 3; k <= KE; ++k) {
          const double a = TR1(k);
          TR1(k - 1) = a / TR2(k - 1);
          TR2(k) = TR2(k) - TR3(k - 1) * a / TR2(k - 1);
        }
        for (int k = 2; k <= KE; ++k) x1[k] = P3(wno, i, j, k);
        for (int k = 3; k <= KE; ++k) x1[k] = x1[k] - TR1(k - 1) * x1[k - 1];
        P3(wno, i, j, KE) = P3(g->weto, i, j, KE) * x1[KE] / TR2(KE);
        for (int k = KE - 1; k >= 2; --k)
          P3(wno, i, j, k) = (x1[k] - TR3(k) * P3(wno, i, j, k + 1)) * P3(g->weto, i, j, k) / TR2(k);
      }
#undef TR1
#undef TR2
#undef TR3
    free(t1);
    free(x1);
  }
  /* biharmonic coefficients, ocvisc.f90:286-340 */
  double *dlypsi = zalloc((size_t)(IE + 1) * JE); /* U2 layout (I_start:IE, JE) */
  double *dlxpsi = zalloc((size_t)IE * (JE + 1)); /* V2 layout (IE, J_start:JE) */
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE1; ++i) U2(dlypsi, i, j) = 0.5 * (V2(g->dlyv, i, j) + V2(g->dlyv, i + 1, j));
  for (int j = 1; j <= JE; ++j) {
    U2(dlypsi, 0, j) = V2(g->dlyv, 1, j);
    U2(dlypsi, IE, j) = V2(g->dlyv, IE, j);
  }
  for (int i = 1; i <= IE; ++i)
    for (int j = 1; j <= JE1; ++j) V2(dlxpsi, i, j) = 0.5 * (U2(g->dlxu, i, j) + U2(g->dlxu, i, j + 1));
  for (int i = 1; i <= IE; ++i) {
    V2(dlxpsi, i, 0) = U2(g->dlxu, i, 1);
    V2(dlxpsi, i, JE) = U2(g->dlxu, i, JE);
  }
  const size_t n2 = (size_t)IE * JE;
  double *aulux = zalloc(n2), *auluy = zalloc(n2), *aulvx = zalloc(n2), *aulvy = zalloc(n2);
  double *aulwx = zalloc(n2), *aulwy = zalloc(n2);
#define POW4(x) (((x) * (x)) * ((x) * (x)))
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      double m;
      m = fmx(P2(g->dlxp, i, j), minvalue); P2(aulux, i, j) = AULAPUV * POW4(m);
      m = fmx(minvalue, U2(dlypsi, i, j)); P2(auluy, i, j) = AULAPUV * POW4(m);
      m = fmx(minvalue, P2(g->dlyp, i, j)); P2(aulvy, i, j) = AULAPUV * POW4(m);
      m = fmx(V2(dlxpsi, i, j), minvalue); P2(aulvx, i, j) = AULAPUV * POW4(m);
      m = fmx(U2(g->dlxu, i, j), minvalue); P2(aulwx, i, j) = AULAPUV * POW4(m);
      m = fmx(V2(g->dlyv, i, j), minvalue); P2(aulwy, i, j) = AULAPUV * POW4(m);
    }
#undef POW4
  const size_t nu = (size_t)(IE + 1) * JE * KE, nv = (size_t)IE * (JE + 1) * KE, np = (size_t)IE * JE * KE;
  double *uk1o = zalloc(nu), *vk1e = zalloc(nv), *wn1o = zalloc(np);
  /* first Laplacian, ocvisc.f90:350-438 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
#define AO(i, j) U3(g->amsuo, i, j, k)
#define UK(i, j) U3(uko, i, j, k)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i)
        U3(uk1o, i, j, k) = AO(i, j) *
            ((AO(i + 1, j) * (UK(i + 1, j) - UK(i, j)) / P2(g->dlxp, i + 1, j) -
              AO(i - 1, j) * (UK(i, j) - UK(i - 1, j)) / P2(g->dlxp, i, j)) / U2(g->dlxu, i, j) +
             (AO(i, j - 1) * (UK(i, j - 1) - UK(i, j)) / U2(dlypsi, i, j - 1) -
              AO(i, j + 1) * (UK(i, j) - UK(i, j + 1)) / U2(dlypsi, i, j)) / U2(g->dlyu, i, j));
#define AE(i, j) V3(g->amsue, i, j, k)
#define VK(i, j) V3(vke, i, j, k)
    for (int j = 1; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        V3(vk1e, i, j, k) = AE(i, j) *
            ((AE(i + 1, j) * (VK(i + 1, j) - VK(i, j)) / V2(dlxpsi, i, j) -
              AE(i - 1, j) * (VK(i, j) - VK(i - 1, j)) / V2(dlxpsi, i - 1, j)) / V2(g->dlxv, i, j) +
             (AE(i, j - 1) * (VK(i, j - 1) - VK(i, j)) / P2(g->dlyp, i, j) -
              AE(i, j + 1) * (VK(i, j) - VK(i, j + 1)) / P2(g->dlyp, i, j + 1)) / V2(g->dlyv, i, j));
    /* have_g_is */
    for (int j = 2; j <= JE1; ++j) {
      const int i = 0;
      U3(uk1o, i, j, k) = AO(i, j) *
          ((AO(i + 1, j) * (UK(i + 1, j) - UK(i, j)) / P2(g->dlxp, i + 1, j)) / U2(g->dlxu, i, j) +
           (AO(i, j - 1) * (UK(i, j - 1) - UK(i, j)) / U2(dlypsi, i, j - 1) -
            AO(i, j + 1) * (UK(i, j) - UK(i, j + 1)) / U2(dlypsi, i, j)) / U2(g->dlyu, i, j));
    }
    for (int j = 1; j <= JE1; ++j) {
      const int i = 1;
      V3(vk1e, i, j, k) = AE(i, j) *
          ((AE(i + 1, j) * (VK(i + 1, j) - VK(i, j)) / V2(dlxpsi, i, j)) / V2(g->dlxv, i, j) +
           (AE(i, j - 1) * (VK(i, j - 1) - VK(i, j)) / P2(g->dlyp, i, j) -
            AE(i, j + 1) * (VK(i, j) - VK(i, j + 1)) / P2(g->dlyp, i, j + 1)) / V2(g->dlyv, i, j));
    }
    /* have_g_ie */
    for (int j = 2; j <= JE1; ++j) {
      const int i = IE;
      U3(uk1o, i, j, k) = AO(i, j) *
          ((-AO(i - 1, j) * (UK(i, j) - UK(i - 1, j)) / P2(g->dlxp, i, j)) / U2(g->dlxu, i, j) +
           (AO(i, j - 1) * (UK(i, j - 1) - UK(i, j)) / U2(dlypsi, i, j - 1) -
            AO(i, j + 1) * (UK(i, j) - UK(i, j + 1)) / U2(dlypsi, i, j)) / U2(g->dlyu, i, j));
    }
    for (int j = 1; j <= JE1; ++j) {
      const int i = IE;
      V3(vk1e, i, j, k) = AE(i, j) *
          ((-AE(i - 1, j) * (VK(i, j) - VK(i - 1, j)) / V2(dlxpsi, i - 1, j)) / V2(g->dlxv, i, j) +
           (AE(i, j - 1) * (VK(i, j - 1) - VK(i, j)) / P2(g->dlyp, i, j) -
            AE(i, j + 1) * (VK(i, j) - VK(i, j + 1)) / P2(g->dlyp, i, j + 1)) / V2(g->dlyv, i, j));
    }
    /* have_g_js */
    for (int i = 1; i <= IE1; ++i) {
      const int j = 1;
      U3(uk1o, i, j, k) = AO(i, j) *
          ((AO(i + 1, j) * (UK(i + 1, j) - UK(i, j)) / P2(g->dlxp, i + 1, j) -
            AO(i - 1, j) * (UK(i, j) - UK(i - 1, j)) / P2(g->dlxp, i, j)) / U2(g->dlxu, i, j) +
           (-AO(i, j + 1) * (UK(i, j) - UK(i, j + 1)) / U2(dlypsi, i, j)) / U2(g->dlyu, i, j));
    }
    for (int i = 2; i <= IE1; ++i) {
      const int j = 0;
      V3(vk1e, i, j, k) = AE(i, j) *
          ((AE(i + 1, j) * (VK(i + 1, j) - VK(i, j)) / V2(dlxpsi, i, j) -
            AE(i - 1, j) * (VK(i, j) - VK(i - 1, j)) / V2(dlxpsi, i - 1, j)) / V2(g->dlxv, i, j) +
           (-AE(i, j + 1) * (VK(i, j) - VK(i, j + 1)) / P2(g->dlyp, i, j + 1)) / V2(g->dlyv, i, j));
    }
    /* have_g_je */
    for (int i = 1; i <= IE1; ++i) {
      const int j = JE;
      U3(uk1o, i, j, k) = AO(i, j) *
          ((AO(i + 1, j) * (UK(i + 1, j) - UK(i, j)) / P2(g->dlxp, i + 1, j) -
            AO(i - 1, j) * (UK(i, j) - UK(i - 1, j)) / P2(g->dlxp, i, j)) / U2(g->dlxu, i, j) +
           (AO(i, j - 1) * (UK(i, j - 1) - UK(i, j)) / U2(dlypsi, i, j - 1)) / U2(g->dlyu, i, j));
    }
    for (int i = 2; i <= IE1; ++i) {
      const int j = JE;
      V3(vk1e, i, j, k) = AE(i, j) *
          ((AE(i + 1, j) * (VK(i + 1, j) - VK(i, j)) / V2(dlxpsi, i, j) -
            AE(i - 1, j) * (VK(i, j) - VK(i - 1, j)) / V2(dlxpsi, i - 1, j)) / V2(g->dlxv, i, j) +
           (AE(i, j - 1) * (VK(i, j - 1) - VK(i, j)) / P2(g->dlyp, i, j)) / V2(g->dlyv, i, j));
    }
  }
  /* second pass, ocvisc.f90:445-477 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
#define U1(i, j) U3(uk1o, i, j, k)
#define V1(i, j) V3(vk1e, i, j, k)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i) {
        const double a = U2(g->dlxu, i, j) * U2(g->dlyu, i, j);
        U3(uoo, i, j, k) = (AO(i, j) / (U2(g->dlxu, i, j) * U2(g->dlyu, i, j))) *
            (U2(g->dlxu, i, j) * U2(g->dlyu, i, j) * UK(i, j) -
             (P2(aulux, i + 1, j) * P2(g->dlyp, i + 1, j) * AO(i + 1, j) * (U1(i + 1, j) - U1(i, j)) / P2(g->dlxp, i + 1, j) -
              P2(aulux, i, j) * P2(g->dlyp, i, j) * AO(i - 1, j) * (U1(i, j) - U1(i - 1, j)) / P2(g->dlxp, i, j) +
              P2(auluy, i, j - 1) * V2(dlxpsi, i, j - 1) * AO(i, j - 1) * (U1(i, j - 1) - U1(i, j)) / U2(dlypsi, i, j - 1) -
              P2(auluy, i, j) * V2(dlxpsi, i, j) * AO(i, j + 1) * (U1(i, j) - U1(i, j + 1)) / U2(dlypsi, i, j)));
        (void)a;
      }
    for (int j = 1; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        V3(voe, i, j, k) = (AE(i, j) / (V2(g->dlxv, i, j) * V2(g->dlyv, i, j))) *
            (V2(g->dlxv, i, j) * V2(g->dlyv, i, j) * VK(i, j) -
             (P2(aulvx, i, j) * U2(dlypsi, i, j) * AE(i + 1, j) * (V1(i + 1, j) - V1(i, j)) / V2(dlxpsi, i, j) -
              P2(aulvx, i - 1, j) * U2(dlypsi, i - 1, j) * AE(i - 1, j) * (V1(i, j) - V1(i - 1, j)) / V2(dlxpsi, i - 1, j) +
              P2(aulvy, i, j) * P2(g->dlxp, i, j) * AE(i, j - 1) * (V1(i, j - 1) - V1(i, j)) / P2(g->dlyp, i, j) -
              P2(aulvy, i, j + 1) * P2(g->dlxp, i, j + 1) * AE(i, j + 1) * (V1(i, j) - V1(i, j + 1)) / P2(g->dlyp, i, j + 1)));
#undef U1
#undef V1
  }
#undef AO
#undef UK
#undef AE
#undef VK
  /* w biharmonic, ocvisc.f90:617-688 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
#define WE(i, j) P3(g->weto, i, j, k)
#define WN(i, j) P3(wno, i, j, k)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        P3(wn1o, i, j, k) = WE(i, j) *
            ((WE(i + 1, j) * (WN(i + 1, j) - WN(i, j)) / U2(g->dlxu, i, j) -
              WE(i - 1, j) * (WN(i, j) - WN(i - 1, j)) / U2(g->dlxu, i - 1, j)) / P2(g->dlxp, i, j) +
             (WE(i, j - 1) * (WN(i, j - 1) - WN(i, j)) / V2(g->dlyv, i, j - 1) -
              WE(i, j + 1) * (WN(i, j) - WN(i, j + 1)) / V2(g->dlyv, i, j)) / P2(g->dlyp, i, j));
    for (int j = 2; j <= JE1; ++j) {
      const int i = 1;
      P3(wn1o, i, j, k) = WE(i, j) *
          ((WE(i + 1, j) * (WN(i + 1, j) - WN(i, j)) / U2(g->dlxu, i, j)) / P2(g->dlxp, i, j) +
           (WE(i, j - 1) * (WN(i, j - 1) - WN(i, j)) / V2(g->dlyv, i, j - 1) -
            WE(i, j + 1) * (WN(i, j) - WN(i, j + 1)) / V2(g->dlyv, i, j)) / P2(g->dlyp, i, j));
    }
    for (int j = 2; j <= JE1; ++j) {
      const int i = IE;
      P3(wn1o, i, j, k) = WE(i, j) *
          ((-WE(i - 1, j) * (WN(i, j) - WN(i - 1, j)) / U2(g->dlxu, i - 1, j)) / P2(g->dlxp, i, j) +
           (WE(i, j - 1) * (WN(i, j - 1) - WN(i, j)) / V2(g->dlyv, i, j - 1) -
            WE(i, j + 1) * (WN(i, j) - WN(i, j + 1)) / V2(g->dlyv, i, j)) / P2(g->dlyp, i, j));
    }
    for (int i = 2; i <= IE1; ++i) {
      const int j = 1;
      P3(wn1o, i, j, k) = WE(i, j) *
          ((WE(i + 1, j) * (WN(i + 1, j) - WN(i, j)) / U2(g->dlxu, i, j) -
            WE(i - 1, j) * (WN(i, j) - WN(i - 1, j)) / U2(g->dlxu, i - 1, j)) / P2(g->dlxp, i, j) +
           (-WE(i, j + 1) * (WN(i, j) - WN(i, j + 1)) / V2(g->dlyv, i, j)) / P2(g->dlyp, i, j));
    }
    for (int i = 2; i <= IE1; ++i) {
      const int j = JE;
      P3(wn1o, i, j, k) = WE(i, j) *
          ((WE(i + 1, j) * (WN(i + 1, j) - WN(i, j)) / U2(g->dlxu, i, j) -
            WE(i - 1, j) * (WN(i, j) - WN(i - 1, j)) / U2(g->dlxu, i - 1, j)) / P2(g->dlxp, i, j) +
           (WE(i, j - 1) * (WN(i, j - 1) - WN(i, j)) / V2(g->dlyv, i, j - 1)) / P2(g->dlyp, i, j));
    }
  }
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
#define W1(i, j) P3(wn1o, i, j, k)
#define DZU(i, j) fmx(U3(g->dduo, i, j, k), minvalue)
#define DZV(i, j) fmx(V3(g->ddue, i, j, k), minvalue)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        const double dzp = fmx(P3(g->ddpo, i, j, k), minvalue);
        P3(wno, i, j, k) = (WE(i, j) / (P2(g->dlxp, i, j) * P2(g->dlyp, i, j) * dzp)) *
            (P2(g->dlxp, i, j) * P2(g->dlyp, i, j) * dzp * WN(i, j) -
             (+P2(aulwx, i, j) * U2(g->dlyu, i, j) * DZU(i, j) * WE(i + 1, j) * (W1(i + 1, j) - W1(i, j)) / U2(g->dlxu, i, j) -
              P2(aulwx, i - 1, j) * U2(g->dlyu, i - 1, j) * DZU(i - 1, j) * WE(i - 1, j) * (W1(i, j) - W1(i - 1, j)) / U2(g->dlxu, i - 1, j) +
              P2(aulwy, i, j - 1) * V2(g->dlxv, i, j - 1) * DZV(i, j - 1) * WE(i, j - 1) * (W1(i, j - 1) - W1(i, j)) / V2(g->dlyv, i, j - 1) -
              P2(aulwy, i, j) * V2(g->dlxv, i, j) * DZV(i, j) * WE(i, j + 1) * (W1(i, j) - W1(i, j + 1)) / V2(g->dlyv, i, j)));
      }
#undef W1
#undef DZU
#undef DZV
#undef WE
#undef WN
  }
  og_octimf(g, uoo, voe, uko, vke);
  free(speedu); free(speedv); free(dlypsi); free(dlxpsi);
  free(aulux); free(auluy); free(aulvx); free(aulvy); free(aulwx); free(aulwy);
  free(uk1o); free(vk1e); free(wn1o);
}

void og_octimf(const og_grid *g, const double *uoo, const double *voe, double *uko,
               double *vke) {
  DIMS;
  memcpy(uko, uoo, sizeof(double) * (size_t)(IE + 1) * JE * KE);
  memcpy(vke, voe, sizeof(double) * (size_t)IE * (JE + 1) * KE);
}

/* ------------------------------------------------------------------------ */
/* OCVTOT_NH right-hand side: ocvtot_nh.f90:11-62 and ComputeRHS            */
/* (mo_petsc.f90:298-376, CG2D4NONHY off: rhs = DIVG*WETO).                 */
/* ------------------------------------------------------------------------ */
void og_nh_rhs(const og_grid *g, const double *uoo, const double *uoo1,
               const double *voe, const double *voe1, const double *wno,
               const double *wno1, const double *zo, double *b) {
  DIMS;
  const double DT = g->dt;
  const int nx = IE - 2, ny = JE - 2;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        const double gu0 = (U3(uoo, i, j, k) - U3(uoo1, i, j, k)) / DT;
        const double gum = (U3(uoo, i - 1, j, k) - U3(uoo1, i - 1, j, k)) / DT;
        const double divgu = (gu0 - gum) / P2(g->dlxp, i, j);
        const double gvm = (V3(voe, i, j - 1, k) - V3(voe1, i, j - 1, k)) / DT;
        const double gv0 = (V3(voe, i, j, k) - V3(voe1, i, j, k)) / DT;
        const double divgv = (gvm - gv0) / P2(g->dlyp, i, j);
        const double gw0 = (P3(wno, i, j, k) - P3(wno1, i, j, k)) / DT;
        const double gw1 = (P3(wno, i, j, k + 1) - P3(wno1, i, j, k + 1)) / DT;
        double divgw;
        if (k >= 2)
          divgw = (gw0 - gw1) / fmx(P3(g->ddpo, i, j, k), 1.E-3);
        else
          divgw = (gw0 - gw1) / (fmx(P3(g->ddpo, i, j, 1), 1.E-3) + P2(zo, i, j));
        const double divg = divgu + divgv + divgw;
        b[(size_t)(i - 2) + (size_t)nx * ((size_t)(j - 2) + (size_t)ny * (size_t)(k - 1))] =
            divg * P3(g->weto, i, j, k);
      }
}

/* ------------------------------------------------------------------------ */
/* compute_matrix (mo_petsc.f90:543-782), single rank (xs = ys = zs = 0),   */
/* CYCLICWE/CYCLICNS off, Neumann = .FALSE.                                */
/* ------------------------------------------------------------------------ */
typedef struct { double zw[2]; double zp; } og_zz;

/* ZW(K) for the matrix copy, mo_petsc.f90:557-583 */
static double og_zw(const og_grid *g, int i, int j, int k) {
  DIMS;
  double dd;
  if (k == 1) {
    dd = P3(g->ddpo, i, j, 1) == 0 ? K1(g->dzw, 1) / 2.0 : P3(g->ddpo, i, j, 1) / 2.0;
  } else if (k == KEP) {
    dd = P3(g->ddpo, i, j, KE) == 0 ? K1(g->dzw, KE) : P3(g->ddpo, i, j, KE);
  } else {
    if (P3(g->ddpo, i, j, k - 1) == 0)
      dd = (K1(g->dzw, k) + K1(g->dzw, k - 1)) / 2.0;
    else if (P3(g->ddpo, i, j, k) == 0)
      dd = P3(g->ddpo, i, j, k - 1);
    else
      dd = (P3(g->ddpo, i, j, k - 1) + P3(g->ddpo, i, j, k)) / 2.0;
  }
  return 1.0 / dd;
}

typedef struct { int col[7]; double val[7]; int n; } og_row;

static void og_matrix_row(const og_grid *g, int i, int j, int k, og_row *r) {
  DIMS;
  const int nx = IE - 2, ny = JE - 2;
  const long row = (long)(i - 2) + (long)nx * ((long)(j - 2) + (long)ny * (long)(k - 1));
  const double xu_w = 1.0 / U2(g->dlxu, i - 1, j), xu_e = 1.0 / U2(g->dlxu, i, j);
  const double xp = 1.0 / P2(g->dlxp, i, j);
  const double yv_n = 1.0 / V2(g->dlyv, i, j - 1), yv_s = 1.0 / V2(g->dlyv, i, j);
  const double yp = 1.0 / P2(g->dlyp, i, j);
  const double zw0 = og_zw(g, i, j, k), zw1 = og_zw(g, i, j, k + 1);
  const double zp = 1.0 / ((1.0 / zw0 + 1.0 / zw1) / 2.0);
  double X_W = xu_w * xp, X_C = (xu_w + xu_e) * xp, X_E = xu_e * xp;
  double Y_N = yv_n * yp, Y_C = (yv_n + yv_s) * yp, Y_S = yv_s * yp;
  double Z_U = zw0 * zp, Z_C = (zw0 + zw1) * zp, Z_D = zw1 * zp;
  r->n = 0;
#define WET(ii, jj, kk) P3(g->weto, ii, jj, kk)
  if (WET(i, j, k) == 0) {
    r->col[0] = (int)row;
    r->val[0] = -(X_C + Y_C + Z_C);
    r->n = 1;
    return;
  }
  if (WET(i - 1, j, k) == 0 && WET(i + 1, j, k) == 1) {
    X_W = 0.0; X_C = xu_e * xp;
  } else if (WET(i - 1, j, k) == 1 && WET(i + 1, j, k) == 0) {
    X_E = 0.0; X_C = xu_w * xp;
  } else if (WET(i - 1, j, k) == 0 && WET(i + 1, j, k) == 0) {
    X_W = 0.0; X_E = 0.0; X_C = 0.0;
  }
  if (WET(i, j - 1, k) == 0 && WET(i, j + 1, k) == 1) {
    Y_N = 0.0; Y_C = yv_s * yp;
  } else if (WET(i, j - 1, k) == 1 && WET(i, j + 1, k) == 0) {
    Y_S = 0.0; Y_C = yv_n * yp;
  } else if (WET(i, j - 1, k) == 0 && WET(i, j + 1, k) == 0) {
    Y_N = 0.0; Y_S = 0.0; Y_C = 0.0;
  }
  if (k == 1) {
    Z_U = 0.0;
  } else if (k == KE) {
    Z_D = 0.0; Z_C = zw0 * zp;
  } else if (WET(i, j, k + 1) == 0) {
    Z_D = 0.0; Z_C = zw0 * zp;
  }
  if (g->ob_west && i == 2) X_W = 0.0;
  if (g->ob_east && i == IE1) X_E = 0.0;
  if (g->ob_north && j == 2) Y_N = 0.0;
  if (g->ob_south && j == JE1) Y_S = 0.0;
  /* entries in increasing column order: up, north, west, centre, east, south, down */
  if (k != 1) { r->col[r->n] = (int)(row - (long)nx * ny); r->val[r->n++] = Z_U; }
  if (WET(i, j - 1, k) == 1 && j - 2 != 0) { r->col[r->n] = (int)(row - nx); r->val[r->n++] = Y_N; }
  if (WET(i - 1, j, k) == 1 && i - 2 != 0) { r->col[r->n] = (int)(row - 1); r->val[r->n++] = X_W; }
  r->col[r->n] = (int)row; r->val[r->n++] = -(X_C + Y_C + Z_C);
  if (WET(i + 1, j, k) == 1 && i - 2 != nx - 1) { r->col[r->n] = (int)(row + 1); r->val[r->n++] = X_E; }
  if (WET(i, j + 1, k) == 1 && j - 2 != ny - 1) { r->col[r->n] = (int)(row + nx); r->val[r->n++] = Y_S; }
  if (k != KE && WET(i, j, k + 1) == 1) { r->col[r->n] = (int)(row + (long)nx * ny); r->val[r->n++] = Z_D; }
#undef WET
}

size_t og_matrix_nnz(const og_grid *g) {
  DIMS;
  size_t nnz = 0;
  og_row r;
  for (int k = 1; k <= KE; ++k)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        og_matrix_row(g, i, j, k, &r);
        nnz += (size_t)r.n;
      }
  return nnz;
}

void og_matrix_csr(const og_grid *g, int *rowptr, int *colind, double *val) {
  DIMS;
  size_t p = 0, row = 0;
  og_row r;
  rowptr[0] = 0;
  for (int k = 1; k <= KE; ++k)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i) {
        og_matrix_row(g, i, j, k, &r);
        for (int e = 0; e < r.n; ++e) { colind[p] = r.col[e]; val[p] = r.val[e]; ++p; }
        rowptr[++row] = (int)p;
      }
}

/* ------------------------------------------------------------------------ */
/* OCVTOT_NH after the solve: ocvtot_nh.f90:150-255, petsc_solve_3D         */
/* (mo_petsc.f90:222-229).                                                  */
/* ------------------------------------------------------------------------ */
void og_nh_post(const og_grid *g, const double *x, double *pnh, double *uoo,
                double *voe, double *wno, double *uoo1, double *voe1,
                double *wno1, double *wo) {
  DIMS;
  const double DT = g->dt, DTI = 1. / DT;
  const int nx = IE - 2, ny = JE - 2;
  for (int k = 1; k <= KE; ++k)
    for (int j = 2; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        P3(pnh, i, j, k) = x[(size_t)(i - 2) + (size_t)nx * ((size_t)(j - 2) + (size_t)ny * (size_t)(k - 1))];
  if (g->ob_west)
    for (int j = 2; j <= JE1; ++j)
      for (int k = 1; k <= KE; ++k) P3(pnh, 1, j, k) = P3(pnh, 2, j, k);
  if (g->ob_east)
    for (int j = 2; j <= JE1; ++j)
      for (int k = 1; k <= KE; ++k) P3(pnh, IE, j, k) = P3(pnh, IE1, j, k);
  if (g->ob_north)
    for (int i = 1; i <= IE; ++i)
      for (int k = 1; k <= KE; ++k) P3(pnh, i, 1, k) = P3(pnh, i, 2, k);
  if (g->ob_south)
    for (int i = 1; i <= IE; ++i)
      for (int k = 1; k <= KE; ++k) P3(pnh, i, JE, k) = P3(pnh, i, JE1, k);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 2; j <= JE1; ++j)
      for (int i = 1; i <= IE1; ++i)
        U3(uoo, i, j, k) = U3(uoo, i, j, k) + U3(g->amsuo, i, j, k) * U2(g->dtdxuo, i, j) *
                                                  (P3(pnh, i, j, k) - P3(pnh, i + 1, j, k));
    for (int j = 1; j <= JE1; ++j)
      for (int i = 2; i <= IE1; ++i)
        V3(voe, i, j, k) = V3(voe, i, j, k) + V3(g->amsue, i, j, k) * V2(g->dpye, i, j) *
                                                  (P3(pnh, i, j + 1, k) - P3(pnh, i, j, k));
  }
  memset(wno, 0, sizeof(double) * (size_t)IE * JE * KEP);
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= JE; ++j)
    for (int k = KE; k >= 1; --k)
      for (int i = 1; i <= IE; ++i)
        P3(wno, i, j, k) =
            P3(wno, i, j, k + 1) +
            DTI * P3(g->weto, i, j, k) *
                (P2(g->dtdxpo, i, j) *
                 (U3(uoo, i - 1, j, k) * U3(g->dduo, i - 1, j, k) * U2(g->dlyu, i - 1, j) -
                  U3(uoo, i, j, k) * U3(g->dduo, i, j, k) * U2(g->dlyu, i, j)) /
                 P2(g->dlyp, i, j)) +
            DTI * P3(g->weto, i, j, k) *
                (+P2(g->dtdyo, i, j) *
                 (V3(voe, i, j, k) * V3(g->ddue, i, j, k) * V2(g->dlxv, i, j) -
                  V3(voe, i, j - 1, k) * V3(g->ddue, i, j - 1, k) * V2(g->dlxv, i, j - 1)) /
                 P2(g->dlxp, i, j));
  memcpy(uoo1, uoo, sizeof(double) * (size_t)(IE + 1) * JE * KE);
  memcpy(voe1, voe, sizeof(double) * (size_t)IE * (JE + 1) * KE);
  memcpy(wno1, wno, sizeof(double) * (size_t)IE * JE * KEP);
  memcpy(wo, wno, sizeof(double) * (size_t)IE * JE * KEP);
}

/* ------------------------------------------------------------------------ */
/* CPU Krylov solve: right-preconditioned FGMRES(30) with a column          */
/* tridiagonal (line Jacobi in z) preconditioner.  Stands in for PETSc's    */
/* -ksp_type fgmres -pc_type mg -pc_mg_levels 1 (whose single level is a    */
/* direct solve); the operator and right-hand side are the reference's.     */
/* ------------------------------------------------------------------------ */
typedef struct { int nx, ny, nz; double *a, *d, *c; } og_linepc;

static void og_pc_setup(const og_grid *g, const int *rp, const int *ci, const double *v,
                        og_linepc *pc) {
  DIMS;
  pc->nx = IE - 2; pc->ny = JE - 2; pc->nz = KE;
  const size_t n = (size_t)pc->nx * pc->ny * pc->nz, plane = (size_t)pc->nx * pc->ny;
  pc->a = zalloc(n); pc->d = zalloc(n); pc->c = zalloc(n);
#pragma omp parallel for schedule(static)
  for (long r = 0; r < (long)n; ++r)
    for (int e = rp[r]; e < rp[r + 1]; ++e) {
      const long cc = ci[e];
      if (cc == r) pc->d[r] = v[e];
      else if (cc == r - (long)plane) pc->a[r] = v[e];
      else if (cc == r + (long)plane) pc->c[r] = v[e];
    }
}

static void og_pc_apply(const og_linepc *pc, const double *r, double *z) {
  const size_t plane = (size_t)pc->nx * pc->ny;
#pragma omp parallel
  {
    double *cp = (double *)malloc(sizeof(double) * (size_t)pc->nz + 8);
#pragma omp for schedule(static)
    for (long q = 0; q < (long)plane; ++q) {
      /* Thomas algorithm down the column */
      double den = pc->d[q];
      cp[0] = pc->c[q] / den;
      z[q] = r[q] / den;
      for (int k = 1; k < pc->nz; ++k) {
        const size_t ix = (size_t)q + plane * (size_t)k;
        den = pc->d[ix] - pc->a[ix] * cp[k - 1];
        cp[k] = pc->c[ix] / den;
        z[ix] = (r[ix] - pc->a[ix] * z[ix - plane]) / den;
      }
      for (int k = pc->nz - 2; k >= 0; --k) {
        const size_t ix = (size_t)q + plane * (size_t)k;
        z[ix] = z[ix] - cp[k] * z[ix + plane];
      }
    }
    free(cp);
  }
}

static void og_spmv(long n, const int *rp, const int *ci, const double *v, const double *x,
                    double *y) {
#pragma omp parallel for schedule(static)
  for (long r = 0; r < n; ++r) {
    double s = 0.0;
    for (int e = rp[r]; e < rp[r + 1]; ++e) s += v[e] * x[ci[e]];
    y[r] = s;
  }
}

static double og_dot(long n, const double *a, const double *b) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

int og_solve(const og_grid *g, const int *rp, const int *ci, const double *val,
             const double *b, double *x, double rtol, int maxit, double *relres) {
  DIMS;
  const long n = (long)(IE - 2) * (JE - 2) * KE;
  const int m = 30;
  og_linepc pc;
  og_pc_setup(g, rp, ci, val, &pc);
  double *V = zalloc((size_t)n * (m + 1)), *Z = zalloc((size_t)n * m);
  double *H = zalloc((size_t)(m + 1) * m), *cs = zalloc(m), *sn = zalloc(m), *s = zalloc(m + 1);
  double *r = zalloc(n), *w = zalloc(n);
  const double bnorm = sqrt(og_dot(n, b, b));
  int it = 0, converged = 0;
  double rel = 0.0;
  if (bnorm == 0.0) {
    memset(x, 0, sizeof(double) * (size_t)n);
    converged = 1;
  }
  while (!converged && it < maxit) {
    og_spmv(n, rp, ci, val, x, r);
    for (long i = 0; i < n; ++i) r[i] = b[i] - r[i];
    double beta = sqrt(og_dot(n, r, r));
    rel = beta / bnorm;
    if (rel <= rtol) { converged = 1; break; }
    for (long i = 0; i < n; ++i) V[i] = r[i] / beta;
    memset(s, 0, sizeof(double) * (m + 1));
    s[0] = beta;
    int j;
    for (j = 0; j < m && it < maxit; ++j, ++it) {
      og_pc_apply(&pc, V + (size_t)n * j, Z + (size_t)n * j);
      og_spmv(n, rp, ci, val, Z + (size_t)n * j, w);
      for (int q = 0; q <= j; ++q) { /* modified Gram-Schmidt */
        const double h = og_dot(n, w, V + (size_t)n * q);
        H[q * m + j] = h;
        const double *vq = V + (size_t)n * q;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) w[i] -= h * vq[i];
      }
      const double hn = sqrt(og_dot(n, w, w));
      H[(j + 1) * m + j] = hn;
      if (hn != 0.0)
        for (long i = 0; i < n; ++i) V[(size_t)n * (j + 1) + i] = w[i] / hn;
      for (int q = 0; q < j; ++q) {
        const double t = cs[q] * H[q * m + j] + sn[q] * H[(q + 1) * m + j];
        H[(q + 1) * m + j] = -sn[q] * H[q * m + j] + cs[q] * H[(q + 1) * m + j];
        H[q * m + j] = t;
      }
      const double den = sqrt(H[j * m + j] * H[j * m + j] + hn * hn);
      cs[j] = H[j * m + j] / den;
      sn[j] = hn / den;
      H[j * m + j] = den;
      H[(j + 1) * m + j] = 0.0;
      s[j + 1] = -sn[j] * s[j];
      s[j] = cs[j] * s[j];
      if (fabs(s[j + 1]) / bnorm <= rtol * 0.5) { ++j; ++it; break; }
    }
    /* back substitution and x += Z y */
    double *y = zalloc(m);
    for (int q = j - 1; q >= 0; --q) {
      double t = s[q];
      for (int p = q + 1; p < j; ++p) t -= H[q * m + p] * y[p];
      y[q] = t / H[q * m + q];
    }
    for (int q = 0; q < j; ++q) {
      const double *zq = Z + (size_t)n * q;
      const double yq = y[q];
#pragma omp parallel for schedule(static)
      for (long i = 0; i < n; ++i) x[i] += yq * zq[i];
    }
    free(y);
  }
  if (!converged) {
    og_spmv(n, rp, ci, val, x, r);
    for (long i = 0; i < n; ++i) r[i] = b[i] - r[i];
    rel = bnorm == 0.0 ? 0.0 : sqrt(og_dot(n, r, r)) / bnorm;
    converged = rel <= rtol;
  }
  if (relres) *relres = rel;
  free(V); free(Z); free(H); free(cs); free(sn); free(s); free(r); free(w);
  free(pc.a); free(pc.d); free(pc.c);
  return converged ? it : -it - 1;
}

/* ------------------------------------------------------------------------ */
/* Open-boundary tides and sponge (mo_obcs.f90, OBC_TIDE on; the 1/x sponge,  */
/* or the exponential one of OBC_SPONGE_EXP where og_obc.tao is nonzero).   */
/* ------------------------------------------------------------------------ */
/* One boundary value of the tidal sum (mo_obcs.f90:578-584 and the like):
 * sum over td of AM(idx,td) * MASK * COS(2 PI (t - PH(idx,td)) / T(td)). */
static double og_tide(const og_obc *o, const double *am, const double *ph, int n, int idx,
                      double mask, double t, double pi) {
  double s = 0.0;
  for (int td = 0; td < o->ntide; ++td) {
    const size_t q = (size_t)idx + (size_t)n * (size_t)td;
    s = s + am[q] * mask * cos(2.0 * pi * (t - ph[q]) / o->period[td]);
  }
  return s;
}

/* lambda of one sponge row (mo_obcs.f90:1578-1583): DT / the interpolated
 * relaxation time, 0 where that time is 0 */
static double og_lambda(double s1, double s2, double relb, double reli, int w, double dt) {
  double lambda = (s1 * relb + s2 * reli) / (double)w;
  return lambda != 0.0 ? dt / lambda : 0.0;
}

/* OBC_SPONGE_EXP (mo_obcs.f90:2588-3222): the rate EXP(-4*L/Lsp)/TAO of the
 * band cell with normal index x (i west/east, j north/south) in row `row`
 * (the other index) of side b, staggering `kind` (0 p, 1 u, 2 v).  L is the
 * SUM of DLX* (west, east) or DLY* (north, south) from the boundary cell to
 * the cell, Lsp that of the whole band as INI_OBCS forms it
 * (mo_obcs.f90:508-522): u west from I_START = 0, v north from J_START = 0.
 * sal: SAO's south band, whose loop reads Lt_s, the L T's loop ended with
 * (x = JE - w + 1), mo_obcs.f90:2974-2978. */
static double og_met(const og_grid *g, const double *a, int kind, int i, int j) {
  DIMS;
  (void)KE;
  if (kind == 1) return U2(a, i, j);
  if (kind == 2) return V2(a, i, j);
  return P2(a, i, j);
}
static double og_sum_x(const og_grid *g, const double *a, int kind, int lo, int hi, int j) {
  double s = 0.0;
  for (int i = lo; i <= hi; ++i) s = s + og_met(g, a, kind, i, j);
  return s;
}
static double og_sum_y(const og_grid *g, const double *a, int kind, int i, int lo, int hi) {
  double s = 0.0;
  for (int j = lo; j <= hi; ++j) s = s + og_met(g, a, kind, i, j);
  return s;
}
static double og_rate(const og_grid *g, double tao, int kind, int b, int x, int row, int w, int sal) {
  const int IE = g->ie, JE = g->je;
  const double *dx = kind == 0 ? g->dlxp : kind == 1 ? g->dlxu : g->dlxv;
  const double *dy = kind == 0 ? g->dlyp : kind == 1 ? g->dlyu : g->dlyv;
  double l, lsp;
  if (b == 0) {
    const int lo = kind == 1 ? 0 : 1;
    l = og_sum_x(g, dx, kind, lo, x, row);
    lsp = og_sum_x(g, dx, kind, lo, lo + w - 1, row);
  } else if (b == 1) {
    l = og_sum_x(g, dx, kind, x, IE, row);
    lsp = og_sum_x(g, dx, kind, IE - w + 1, IE, row);
  } else if (b == 2) {
    const int lo = kind == 2 ? 0 : 1;
    l = og_sum_y(g, dy, kind, row, lo, x);
    lsp = og_sum_y(g, dy, kind, row, lo, lo + w - 1);
  } else {
    l = og_sum_y(g, dy, kind, row, sal ? JE - w + 1 : x, JE);
    lsp = og_sum_y(g, dy, kind, row, JE - w + 1, JE);
  }
  return exp(-(4.0 * l / lsp)) / tao;
}

void og_obc_eta(const og_grid *g, const og_obc *o, int step, double *zo) {
  DIMS;
  const double pi = 4.0 * atan(1.0);     /* orctm.f90:525 */
  const double t = (double)step * g->dt; /* mytime = i_step * DT, mo_obcs.f90:574 */
  const int W = g->ob_west, E = g->ob_east, N = g->ob_north, S = g->ob_south;
  const double relb = o->relax_bound, reli = o->relax_inner; /* rel_eta*, mo_obcs.f90:499-506 */
  const double dt = g->dt;
  /* FORC_OBCS_ETA, mo_obcs.f90:569-642 */
  double *zw = zalloc(JE), *ze = zalloc(JE), *zn = zalloc(IE), *zs = zalloc(IE);
  for (int j = 1; j <= JE; ++j) {
    if (W) zw[j - 1] = og_tide(o, o->amp[0][0], o->pha[0][0], JE, j - 1, P3(g->weto, 1, j, 1), t, pi);
    if (E) ze[j - 1] = og_tide(o, o->amp[1][0], o->pha[1][0], JE, j - 1, P3(g->weto, IE, j, 1), t, pi);
  }
  for (int i = 1; i <= IE; ++i) {
    if (N) zn[i - 1] = og_tide(o, o->amp[2][0], o->pha[2][0], IE, i - 1, P3(g->weto, i, 1, 1), t, pi);
    if (S) zs[i - 1] = og_tide(o, o->amp[3][0], o->pha[3][0], IE, i - 1, P3(g->weto, i, JE, 1), t, pi);
  }
  /* SPONGE_OBCS_ETA, mo_obcs.f90:1561-1720 */
  const size_t n2 = (size_t)IE * JE;
  double *zz = zalloc(n2), *fo = zalloc(n2), *fw = zalloc(n2), *fe = zalloc(n2), *fn = zalloc(n2),
         *fs = zalloc(n2);
  memcpy(zz, zo, sizeof(double) * n2);
  const int sw = o->width[0], se = o->width[1], sn = o->width[2], ss = o->width[3];
  const int SW_ = W && o->sponge[0], SE_ = E && o->sponge[1], SN_ = N && o->sponge[2],
            SS_ = S && o->sponge[3];
  if (SW_)
    for (int i = 1; i <= sw; ++i) {
      const double s1 = (double)(sw - i + 1), s2 = (double)(i - 1);
      const double lambda = og_lambda(s1, s2, relb, reli, sw, dt);
      for (int j = 1; j <= JE; ++j) {
        if (o->tao != 0.0) {
          P2(fw, i, j) =
              P3(g->weto, 1, j, 1) * P3(g->weto, i, j, 1) * dt *
              og_rate(g, o->tao, 0, 0, i, j, sw, 0) * (zw[j - 1] - P2(zz, i, j));
          continue;
        }
        const double zr = (s1 * zw[j - 1] + s2 * P2(zz, i, j)) / (double)sw;
        P2(fw, i, j) = P3(g->weto, 1, j, 1) * P3(g->weto, i, j, 1) * lambda * (zr - P2(zz, i, j));
      }
    }
  if (SE_)
    for (int i = IE; i >= IE - se + 1; --i) {
      const double s1 = (double)(i - IE + se), s2 = (double)(IE - i);
      const double lambda = og_lambda(s1, s2, relb, reli, se, dt);
      for (int j = 1; j <= JE; ++j) {
        if (o->tao != 0.0) {
          P2(fe, i, j) =
              P3(g->weto, IE, j, 1) * P3(g->weto, i, j, 1) * dt *
              og_rate(g, o->tao, 0, 1, i, j, se, 0) * (ze[j - 1] - P2(zz, i, j));
          continue;
        }
        const double zr = (s1 * ze[j - 1] + s2 * P2(zz, i, j)) / (double)se;
        P2(fe, i, j) = P3(g->weto, IE, j, 1) * P3(g->weto, i, j, 1) * lambda * (zr - P2(zz, i, j));
      }
    }
  if (SN_)
    for (int j = 1; j <= sn; ++j) {
      const double s1 = (double)(sn - j + 1), s2 = (double)(j - 1);
      const double lambda = og_lambda(s1, s2, relb, reli, sn, dt);
      for (int i = 1; i <= IE; ++i) {
        if (o->tao != 0.0) {
          P2(fn, i, j) =
              P3(g->weto, i, 1, 1) * P3(g->weto, i, j, 1) * dt *
              og_rate(g, o->tao, 0, 2, j, i, sn, 0) * (zn[i - 1] - P2(zz, i, j));
          continue;
        }
        const double zr = (s1 * zn[i - 1] + s2 * P2(zz, i, j)) / (double)sn;
        P2(fn, i, j) = P3(g->weto, i, 1, 1) * P3(g->weto, i, j, 1) * lambda * (zr - P2(zz, i, j));
      }
    }
  if (SS_)
    for (int j = JE; j >= JE - ss + 1; --j) {
      const double s1 = (double)(j - JE + ss), s2 = (double)(JE - j);
      const double lambda = og_lambda(s1, s2, relb, reli, ss, dt);
      for (int i = 1; i <= IE; ++i) {
        if (o->tao != 0.0) {
          P2(fs, i, j) =
              P3(g->weto, i, JE, 1) * P3(g->weto, i, j, 1) * dt *
              og_rate(g, o->tao, 0, 3, j, i, ss, 0) * (zs[i - 1] - P2(zz, i, j));
          continue;
        }
        const double zr = (s1 * zs[i - 1] + s2 * P2(zz, i, j)) / (double)ss;
        P2(fs, i, j) = P3(g->weto, i, JE, 1) * P3(g->weto, i, j, 1) * lambda * (zr - P2(zz, i, j));
      }
    }
  for (size_t q = 0; q < n2; ++q) fo[q] = fw[q] + fe[q] + fn[q] + fs[q];
  /* corners: the band nearer to the cell wins (mo_obcs.f90:1646-1714) */
  if (SN_ && SW_)
    for (int i = 1; i <= sw; ++i)
      for (int j = 1; j <= sn; ++j) P2(fo, i, j) = i < j ? P2(fw, i, j) : P2(fn, i, j);
  if (SS_ && SW_)
    for (int i = 1; i <= sw; ++i)
      for (int j = JE; j >= JE - ss + 1; --j)
        P2(fo, i, j) = i < (JE - j + 1) ? P2(fw, i, j) : P2(fs, i, j);
  if (SN_ && SE_)
    for (int i = IE; i >= IE - se + 1; --i)
      for (int j = 1; j <= sn; ++j) P2(fo, i, j) = (IE - i + 1) < j ? P2(fe, i, j) : P2(fn, i, j);
  if (SS_ && SE_)
    for (int i = IE; i >= IE - se + 1; --i)
      for (int j = JE; j >= JE - ss + 1; --j)
        P2(fo, i, j) = (IE - i + 1) < (JE - j + 1) ? P2(fe, i, j) : P2(fs, i, j);
  for (size_t q = 0; q < n2; ++q) zo[q] = zz[q] + fo[q];
  free(zw); free(ze); free(zn); free(zs);
  free(zz); free(fo); free(fw); free(fe); free(fn); free(fs);
}

void og_obc_uv(const og_grid *g, const og_obc *o, int step, double *uoo, double *voe) {
  DIMS;
  const double pi = 4.0 * atan(1.0);     /* orctm.f90:525 */
  const double t = (double)step * g->dt; /* mytime = i_step * DT, mo_obcs.f90:1886 */
  const int W = g->ob_west, E = g->ob_east, N = g->ob_north, S = g->ob_south;
  const double relb = o->relax_bound, reli = o->relax_inner; /* rel_uv*, mo_obcs.f90:499-500 */
  const double dt = g->dt;
  /* FORC_OBCS_UV, mo_obcs.f90:1881-1994 (add_tide is .FALSE., line 18) */
  double *uzw = zalloc(JE), *uze = zalloc(JE), *vzw = zalloc(JE + 1), *vze = zalloc(JE + 1);
  double *uzn = zalloc(IE + 1), *uzs = zalloc(IE + 1), *vzn = zalloc(IE), *vzs = zalloc(IE);
  for (int j = 1; j <= JE; ++j) {
    if (W) uzw[j - 1] = og_tide(o, o->amp[0][1], o->pha[0][1], JE, j - 1, U3(g->amsuo, 0, j, 1), t, pi);
    if (E) uze[j - 1] = og_tide(o, o->amp[1][1], o->pha[1][1], JE, j - 1, U3(g->amsuo, IE, j, 1), t, pi);
  }
  for (int j = 0; j <= JE; ++j) {
    if (W) vzw[j] = og_tide(o, o->amp[0][2], o->pha[0][2], JE + 1, j, V3(g->amsue, 1, j, 1), t, pi);
    if (E) vze[j] = og_tide(o, o->amp[1][2], o->pha[1][2], JE + 1, j, V3(g->amsue, IE, j, 1), t, pi);
  }
  for (int i = 0; i <= IE; ++i) {
    if (N) uzn[i] = og_tide(o, o->amp[2][1], o->pha[2][1], IE + 1, i, U3(g->amsuo, i, 1, 1), t, pi);
    if (S) uzs[i] = og_tide(o, o->amp[3][1], o->pha[3][1], IE + 1, i, U3(g->amsuo, i, JE, 1), t, pi);
  }
  for (int i = 1; i <= IE; ++i) {
    if (N) vzn[i - 1] = og_tide(o, o->amp[2][2], o->pha[2][2], IE, i - 1, V3(g->amsue, i, 0, 1), t, pi);
    if (S) vzs[i - 1] = og_tide(o, o->amp[3][2], o->pha[3][2], IE, i - 1, V3(g->amsue, i, JE, 1), t, pi);
  }
  /* SPONGE_OBCS_UV, mo_obcs.f90:2295-2582, with the level values of
   * UPGRADE_OBCS_UV (mo_obcs.f90:1997-2032) formed in place:
   * obc_uw(j,k) = obc_uzw(j) * AMSUO(0,j,k) and so on */
  const size_t nu = (size_t)(IE + 1) * JE * KE, nv = (size_t)IE * (JE + 1) * KE;
  double *uu = zalloc(nu), *uf = zalloc(nu), *uw = zalloc(nu), *ue = zalloc(nu), *un = zalloc(nu),
         *us = zalloc(nu);
  double *vv = zalloc(nv), *vf = zalloc(nv), *vw = zalloc(nv), *ve = zalloc(nv), *vn = zalloc(nv),
         *vs = zalloc(nv);
  memcpy(uu, uoo, sizeof(double) * nu);
  memcpy(vv, voe, sizeof(double) * nv);
  const int sw = o->width[0], se = o->width[1], sn = o->width[2], ss = o->width[3];
  const int SW_ = W && o->sponge[0], SE_ = E && o->sponge[1], SN_ = N && o->sponge[2],
            SS_ = S && o->sponge[3];
  for (int k = 1; k <= KE; ++k) {
    if (SW_) {
      for (int i = 0; i <= sw - 1; ++i) {
        const double s1 = (double)(sw - i), s2 = (double)i;
        const double lambda = og_lambda(s1, s2, relb, reli, sw, dt);
        for (int j = 1; j <= JE; ++j) {
          const double ob = uzw[j - 1] * U3(g->amsuo, 0, j, k);
          if (o->tao != 0.0) {
            U3(uw, i, j, k) =
                U3(g->amsuo, 0, j, k) * U3(g->amsuo, i, j, k) * dt *
                og_rate(g, o->tao, 1, 0, i, j, sw, 0) * (ob - U3(uu, i, j, k));
            continue;
          }
          const double ur = (s1 * ob + s2 * U3(uu, i, j, k)) / (double)sw;
          U3(uw, i, j, k) = U3(g->amsuo, 0, j, k) * U3(g->amsuo, i, j, k) * lambda * (ur - U3(uu, i, j, k));
        }
      }
      for (int i = 1; i <= sw; ++i) {
        const double s1 = (double)(sw - i + 1), s2 = (double)(i - 1);
        const double lambda = og_lambda(s1, s2, relb, reli, sw, dt);
        for (int j = 0; j <= JE; ++j) {
          const double ob = vzw[j] * V3(g->amsue, 1, j, k);
          if (o->tao != 0.0) {
            V3(vw, i, j, k) =
                V3(g->amsue, 1, j, k) * V3(g->amsue, i, j, k) * dt *
                og_rate(g, o->tao, 2, 0, i, j, sw, 0) * (ob - V3(vv, i, j, k));
            continue;
          }
          const double vr = (s1 * ob + s2 * V3(vv, i, j, k)) / (double)sw;
          V3(vw, i, j, k) = V3(g->amsue, 1, j, k) * V3(g->amsue, i, j, k) * lambda * (vr - V3(vv, i, j, k));
        }
      }
    }
    if (SE_) {
      for (int i = IE; i >= IE - se + 1; --i) {
        const double s1 = (double)(i - IE + se), s2 = (double)(IE - i);
        const double lambda = og_lambda(s1, s2, relb, reli, se, dt);
        for (int j = 1; j <= JE; ++j) {
          const double ob = uze[j - 1] * U3(g->amsuo, IE, j, k);
          if (o->tao != 0.0) {
            U3(ue, i, j, k) =
                U3(g->amsuo, IE, j, k) * U3(g->amsuo, i, j, k) * dt *
                og_rate(g, o->tao, 1, 1, i, j, se, 0) * (ob - U3(uu, i, j, k));
            continue;
          }
          const double ur = (s1 * ob + s2 * U3(uu, i, j, k)) / (double)se;
          U3(ue, i, j, k) = U3(g->amsuo, IE, j, k) * U3(g->amsuo, i, j, k) * lambda * (ur - U3(uu, i, j, k));
        }
        for (int j = 0; j <= JE; ++j) {
          const double ob = vze[j] * V3(g->amsue, IE, j, k);
          if (o->tao != 0.0) {
            V3(ve, i, j, k) =
                V3(g->amsue, IE, j, k) * V3(g->amsue, i, j, k) * dt *
                og_rate(g, o->tao, 2, 1, i, j, se, 0) * (ob - V3(vv, i, j, k));
            continue;
          }
          const double vr = (s1 * ob + s2 * V3(vv, i, j, k)) / (double)se;
          V3(ve, i, j, k) = V3(g->amsue, IE, j, k) * V3(g->amsue, i, j, k) * lambda * (vr - V3(vv, i, j, k));
        }
      }
    }
    if (SN_) {
      for (int j = 1; j <= sn; ++j) {
        const double s1 = (double)(sn - j + 1), s2 = (double)(j - 1);
        const double lambda = og_lambda(s1, s2, relb, reli, sn, dt);
        for (int i = 0; i <= IE; ++i) {
          const double ob = uzn[i] * U3(g->amsuo, i, 1, k);
          if (o->tao != 0.0) {
            U3(un, i, j, k) =
                U3(g->amsuo, i, 1, k) * U3(g->amsuo, i, j, k) * dt *
                og_rate(g, o->tao, 1, 2, j, i, sn, 0) * (ob - U3(uu, i, j, k));
            continue;
          }
          const double ur = (s1 * ob + s2 * U3(uu, i, j, k)) / (double)sn;
          U3(un, i, j, k) = U3(g->amsuo, i, 1, k) * U3(g->amsuo, i, j, k) * lambda * (ur - U3(uu, i, j, k));
        }
      }
      for (int j = 0; j <= sn - 1; ++j) {
        const double s1 = (double)(sn - j), s2 = (double)j;
        const double lambda = og_lambda(s1, s2, relb, reli, sn, dt);
        for (int i = 1; i <= IE; ++i) {
          const double ob = vzn[i - 1] * V3(g->amsue, i, 0, k);
          if (o->tao != 0.0) {
            V3(vn, i, j, k) =
                V3(g->amsue, i, 0, k) * V3(g->amsue, i, j, k) * dt *
                og_rate(g, o->tao, 2, 2, j, i, sn, 0) * (ob - V3(vv, i, j, k));
            continue;
          }
          const double vr = (s1 * ob + s2 * V3(vv, i, j, k)) / (double)sn;
          V3(vn, i, j, k) = V3(g->amsue, i, 0, k) * V3(g->amsue, i, j, k) * lambda * (vr - V3(vv, i, j, k));
        }
      }
    }
    if (SS_) {
      for (int j = JE; j >= JE - ss + 1; --j) {
        const double s1 = (double)(j - JE + ss), s2 = (double)(JE - j);
        const double lambda = og_lambda(s1, s2, relb, reli, ss, dt);
        for (int i = 0; i <= IE; ++i) {
          const double ob = uzs[i] * U3(g->amsuo, i, JE, k);
          if (o->tao != 0.0) {
            U3(us, i, j, k) =
                U3(g->amsuo, i, JE, k) * U3(g->amsuo, i, j, k) * dt *
                og_rate(g, o->tao, 1, 3, j, i, ss, 0) * (ob - U3(uu, i, j, k));
            continue;
          }
          const double ur = (s1 * ob + s2 * U3(uu, i, j, k)) / (double)ss;
          U3(us, i, j, k) = U3(g->amsuo, i, JE, k) * U3(g->amsuo, i, j, k) * lambda * (ur - U3(uu, i, j, k));
        }
        for (int i = 1; i <= IE; ++i) {
          const double ob = vzs[i - 1] * V3(g->amsue, i, JE, k);
          if (o->tao != 0.0) {
            V3(vs, i, j, k) =
                V3(g->amsue, i, JE, k) * V3(g->amsue, i, j, k) * dt *
                og_rate(g, o->tao, 2, 3, j, i, ss, 0) * (ob - V3(vv, i, j, k));
            continue;
          }
          const double vr = (s1 * ob + s2 * V3(vv, i, j, k)) / (double)ss;
          V3(vs, i, j, k) = V3(g->amsue, i, JE, k) * V3(g->amsue, i, j, k) * lambda * (vr - V3(vv, i, j, k));
        }
      }
    }
  }
  for (size_t q = 0; q < nu; ++q) uf[q] = uw[q] + ue[q] + un[q] + us[q];
  for (size_t q = 0; q < nv; ++q) vf[q] = vw[q] + ve[q] + vn[q] + vs[q];
  /* corners, mo_obcs.f90:2453-2566 */
  for (int k = 1; k <= KE; ++k) {
    if (SN_ && SW_) {
      for (int i = 0; i <= sw - 1; ++i)
        for (int j = 1; j <= sn; ++j)
          U3(uf, i, j, k) = (i + 1) < j ? U3(uw, i, j, k) : U3(un, i, j, k);
      for (int i = 1; i <= sw; ++i)
        for (int j = 0; j <= sn - 1; ++j)
          V3(vf, i, j, k) = i < (j + 1) ? V3(vw, i, j, k) : V3(vn, i, j, k);
    }
    if (SS_ && SW_) {
      for (int i = 0; i <= sw - 1; ++i)
        for (int j = JE; j >= JE - ss + 1; --j)
          U3(uf, i, j, k) = (i + 1) < (JE - j + 1) ? U3(uw, i, j, k) : U3(us, i, j, k);
      for (int i = 1; i <= sw; ++i)
        for (int j = JE; j >= JE - ss + 1; --j)
          V3(vf, i, j, k) = i < (JE - j + 1) ? V3(vw, i, j, k) : V3(vs, i, j, k);
    }
    if (SN_ && SE_) {
      for (int i = IE; i >= IE - se + 1; --i)
        for (int j = 1; j <= sn; ++j)
          U3(uf, i, j, k) = (IE - i + 1) < j ? U3(ue, i, j, k) : U3(un, i, j, k);
      for (int i = IE; i >= IE - se + 1; --i)
        for (int j = 0; j <= sn - 1; ++j)
          V3(vf, i, j, k) = (IE - i + 1) < (j + 1) ? V3(ve, i, j, k) : V3(vn, i, j, k);
    }
    if (SS_ && SE_) {
      for (int i = IE; i >= IE - se + 1; --i)
        for (int j = JE; j >= JE - ss + 1; --j)
          U3(uf, i, j, k) = (IE - i + 1) < (JE - j + 1) ? U3(ue, i, j, k) : U3(us, i, j, k);
      for (int i = IE; i >= IE - se + 1; --i)
        for (int j = JE; j >= JE - ss + 1; --j)
          V3(vf, i, j, k) = (IE - i + 1) < (JE - j + 1) ? V3(ve, i, j, k) : V3(vs, i, j, k);
    }
  }
  for (size_t q = 0; q < nu; ++q) uoo[q] = uu[q] + uf[q];
  for (size_t q = 0; q < nv; ++q) voe[q] = vv[q] + vf[q];
  free(uzw); free(uze); free(vzw); free(vze); free(uzn); free(uzs); free(vzn); free(vzs);
  free(uu); free(uf); free(uw); free(ue); free(un); free(us);
  free(vv); free(vf); free(vw); free(ve); free(vn); free(vs);
}

void og_obc_ts(const og_grid *g, const og_obc *o, const double *const cli[4], double *trf) {
  DIMS;
  const int W = g->ob_west, E = g->ob_east, N = g->ob_north, S = g->ob_south;
  const double relb = o->relax_bound, reli = o->relax_inner; /* rel_ts*, mo_obcs.f90:502-503 */
  const double dt = g->dt;
  const int sw = o->width[0], se = o->width[1], sn = o->width[2], ss = o->width[3];
  const int SW_ = W && o->sponge[0], SE_ = E && o->sponge[1], SN_ = N && o->sponge[2],
            SS_ = S && o->sponge[3];
  /* FORC_OBCS_TS: obc_tw(j,k) = cli_twg(j,k) * WETO(1,j,k) and so on */
  double *bw = zalloc((size_t)JE * KE), *be = zalloc((size_t)JE * KE);
  double *bn = zalloc((size_t)IE * KE), *bs = zalloc((size_t)IE * KE);
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE; ++j) {
      const size_t q = (size_t)(j - 1) + (size_t)JE * (k - 1);
      if (SW_) bw[q] = cli[0][q] * P3(g->weto, 1, j, k);
      if (SE_) be[q] = cli[1][q] * P3(g->weto, IE, j, k);
    }
    for (int i = 1; i <= IE; ++i) {
      const size_t q = (size_t)(i - 1) + (size_t)IE * (k - 1);
      if (SN_) bn[q] = cli[2][q] * P3(g->weto, i, 1, k);
      if (SS_) bs[q] = cli[3][q] * P3(g->weto, i, JE, k);
    }
  }
  const size_t n3 = (size_t)IE * JE * KE;
  double *tt = zalloc(n3), *fo = zalloc(n3), *fw = zalloc(n3), *fe = zalloc(n3), *fn = zalloc(n3),
         *fs = zalloc(n3);
  memcpy(tt, trf, sizeof(double) * n3);
  for (int k = 1; k <= KE; ++k) {
    if (SW_)
      for (int i = 1; i <= sw; ++i) {
        const double s1 = (double)(sw - i + 1), s2 = (double)(i - 1);
        const double lambda = og_lambda(s1, s2, relb, reli, sw, dt);
        for (int j = 1; j <= JE; ++j) {
          if (o->tao != 0.0) {
            P3(fw, i, j, k) =
                P3(g->weto, 1, j, k) * P3(g->weto, i, j, k) * dt *
                og_rate(g, o->tao, 0, 0, i, j, sw, 0) * (bw[(j - 1) + (size_t)JE * (k - 1)] - P3(tt, i, j, k));
            continue;
          }
          const double tr = (s1 * bw[(j - 1) + (size_t)JE * (k - 1)] + s2 * P3(tt, i, j, k)) / (double)sw;
          P3(fw, i, j, k) = P3(g->weto, 1, j, k) * P3(g->weto, i, j, k) * lambda * (tr - P3(tt, i, j, k));
        }
      }
    if (SE_)
      for (int i = IE; i >= IE - se + 1; --i) {
        const double s1 = (double)(i - IE + se), s2 = (double)(IE - i);
        const double lambda = og_lambda(s1, s2, relb, reli, se, dt);
        for (int j = 1; j <= JE; ++j) {
          if (o->tao != 0.0) {
            P3(fe, i, j, k) =
                P3(g->weto, IE, j, k) * P3(g->weto, i, j, k) * dt *
                og_rate(g, o->tao, 0, 1, i, j, se, 0) * (be[(j - 1) + (size_t)JE * (k - 1)] - P3(tt, i, j, k));
            continue;
          }
          const double tr = (s1 * be[(j - 1) + (size_t)JE * (k - 1)] + s2 * P3(tt, i, j, k)) / (double)se;
          P3(fe, i, j, k) = P3(g->weto, IE, j, k) * P3(g->weto, i, j, k) * lambda * (tr - P3(tt, i, j, k));
        }
      }
    if (SN_)
      for (int j = 1; j <= sn; ++j) {
        const double s1 = (double)(sn - j + 1), s2 = (double)(j - 1);
        const double lambda = og_lambda(s1, s2, relb, reli, sn, dt);
        for (int i = 1; i <= IE; ++i) {
          if (o->tao != 0.0) {
            P3(fn, i, j, k) =
                P3(g->weto, i, 1, k) * P3(g->weto, i, j, k) * dt *
                og_rate(g, o->tao, 0, 2, j, i, sn, 0) * (bn[(i - 1) + (size_t)IE * (k - 1)] - P3(tt, i, j, k));
            continue;
          }
          const double tr = (s1 * bn[(i - 1) + (size_t)IE * (k - 1)] + s2 * P3(tt, i, j, k)) / (double)sn;
          P3(fn, i, j, k) = P3(g->weto, i, 1, k) * P3(g->weto, i, j, k) * lambda * (tr - P3(tt, i, j, k));
        }
      }
    if (SS_)
      for (int j = JE; j >= JE - ss + 1; --j) {
        const double s1 = (double)(j - JE + ss), s2 = (double)(JE - j);
        const double lambda = og_lambda(s1, s2, relb, reli, ss, dt);
        for (int i = 1; i <= IE; ++i) {
          if (o->tao != 0.0) {
            P3(fs, i, j, k) =
                P3(g->weto, i, JE, k) * P3(g->weto, i, j, k) * dt *
                og_rate(g, o->tao, 0, 3, j, i, ss, o->salinity) * (bs[(i - 1) + (size_t)IE * (k - 1)] - P3(tt, i, j, k));
            continue;
          }
          const double tr = (s1 * bs[(i - 1) + (size_t)IE * (k - 1)] + s2 * P3(tt, i, j, k)) / (double)ss;
          P3(fs, i, j, k) = P3(g->weto, i, JE, k) * P3(g->weto, i, j, k) * lambda * (tr - P3(tt, i, j, k));
        }
      }
  }
  for (size_t q = 0; q < n3; ++q) fo[q] = fw[q] + fe[q] + fn[q] + fs[q];
  /* corners, mo_obcs.f90:1190-1250 */
  for (int k = 1; k <= KE; ++k) {
    if (SN_ && SW_)
      for (int i = 1; i <= sw; ++i)
        for (int j = 1; j <= sn; ++j) P3(fo, i, j, k) = i < j ? P3(fw, i, j, k) : P3(fn, i, j, k);
    if (SS_ && SW_)
      for (int i = 1; i <= sw; ++i)
        for (int j = JE; j >= JE - ss + 1; --j)
          P3(fo, i, j, k) = i < (JE - j + 1) ? P3(fw, i, j, k) : P3(fs, i, j, k);
    if (SN_ && SE_)
      for (int i = IE; i >= IE - se + 1; --i)
        for (int j = 1; j <= sn; ++j)
          P3(fo, i, j, k) = (IE - i + 1) < j ? P3(fe, i, j, k) : P3(fn, i, j, k);
    if (SS_ && SE_)
      for (int i = IE; i >= IE - se + 1; --i)
        for (int j = JE; j >= JE - ss + 1; --j)
          P3(fo, i, j, k) = (IE - i + 1) < (JE - j + 1) ? P3(fe, i, j, k) : P3(fs, i, j, k);
  }
  for (size_t q = 0; q < n3; ++q) trf[q] = tt[q] + fo[q];
  free(bw); free(be); free(bn); free(bs);
  free(tt); free(fo); free(fw); free(fe); free(fn); free(fs);
}

/* ------------------------------------------------------------------------ */
/* Barotropic solve: DEUTO/DEUTE (boden.f90), ITPREP, TRONEU, OCVTRO, OCVTOT */
/* ------------------------------------------------------------------------ */
void og_deut(const og_grid *g, const double *depto, double minvalue, double *deuto,
             double *deute, double *deutio, double *deutie) {
  DIMS;
  /* boden.f90:117-128 */
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE1; ++i) U2(deuto, i, j) = fmn(P2(depto, i, j), P2(depto, i + 1, j));
  for (int j = 1; j <= JE; ++j) {
    U2(deuto, 0, j) = U2(deuto, 1, j);
    U2(deuto, IE, j) = U2(deuto, IE1, j);
  }
  for (int j = 1; j <= JE1; ++j)
    for (int i = 1; i <= IE; ++i) V2(deute, i, j) = fmn(P2(depto, i, j), P2(depto, i, j + 1));
  for (int i = 1; i <= IE; ++i) {
    V2(deute, i, 0) = V2(deute, i, 1);
    V2(deute, i, JE) = V2(deute, i, JE1);
  }
  /* boden.f90:264-274 (zero elsewhere, beleg_zero.f90:59,69) */
  for (int j = 1; j <= JE; ++j)
    for (int i = 0; i <= IE; ++i)
      U2(deutio, i, j) = U2(deuto, i, j) > minvalue ? 1. / U2(deuto, i, j) : 0.0;
  for (int j = 0; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i)
      V2(deutie, i, j) = V2(deute, i, j) > minvalue ? 1. / V2(deute, i, j) : 0.0;
}

void og_itprep(const og_grid *g, const og_baro *b, const double *deuto, const double *deute,
               double *xx, double *uf, double *vf, double *ff) {
  DIMS;
  const double dt = g->dt;
  /* itprep.f90:17-21 */
  for (int i = 1; i <= IE; ++i)
    for (int j = 1; j <= JE; ++j) P2(xx, i, j) = P2(g->dlxp, i, j) * P2(g->dlyp, i, j);
  /* itprep.f90:23-27: DEUTO*DLYU/DLXU*G*CONN*STABN*DT**2, left to right */
  for (int i = 0; i <= IE; ++i)
    for (int j = 1; j <= JE; ++j)
      U2(uf, i, j) = U2(deuto, i, j) * U2(g->dlyu, i, j) / U2(g->dlxu, i, j) * b->grav * b->conn *
                     b->stabn * (dt * dt);
  /* itprep.f90:29-33 */
  for (int i = 1; i <= IE; ++i)
    for (int j = 0; j <= JE; ++j)
      V2(vf, i, j) = V2(deute, i, j) * V2(g->dlxv, i, j) / V2(g->dlyv, i, j) * b->grav * b->conn *
                     b->stabn * (dt * dt);
  /* itprep.f90:35-40 */
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i)
      P2(ff, i, j) = 1. / (P2(xx, i, j) + U2(uf, i, j) + U2(uf, i - 1, j) + V2(vf, i, j) +
                           V2(vf, i, j - 1));
}

/* one SOR colour of troneu.f90:108-127: J = 2..JE-1, I = IS..IE-1 step 2 */
static void sor_colour(const og_grid *g, const og_baro *b, int parity, const double *uf,
                       const double *vf, const double *ff, const double *b1o, double *z1o) {
  DIMS;
  const double sorpai = 1. - b->sorpar;
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= JE1; ++j) {
    const int is = (j + parity) % 2 + 2;  /* MOD(p_ioff+p_joff+j(+1),2)+2 on one rank */
    for (int i = is; i <= IE1; i += 2)
      P2(z1o, i, j) = b->sorpar * P2(ff, i, j) *
                          (P2(b1o, i, j) + U2(uf, i, j) * P2(z1o, i + 1, j) +
                           U2(uf, i - 1, j) * P2(z1o, i - 1, j) + V2(vf, i, j) * P2(z1o, i, j + 1) +
                           V2(vf, i, j - 1) * P2(z1o, i, j - 1)) +
                      sorpai * P2(z1o, i, j);
  }
}

void og_troneu(const og_grid *g, const og_baro *b, const double *xx, const double *uf,
               const double *vf, const double *ff, const double *u1o, const double *v1e,
               const double *uzo, const double *vze, double *b1o, double *z1o) {
  DIMS;
  const double conn = b->conn, cono = 1. - b->conn;
  /* troneu.f90:48-60 */
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      double v = P3(g->weto, i, j, 1) *
                 (P2(g->dtdxpo, i, j) *
                      ((cono * U2(u1o, i - 1, j) + U2(uzo, i - 1, j) * conn) * U2(g->dlyu, i - 1, j) -
                       (U2(u1o, i, j) * cono + U2(uzo, i, j) * conn) * U2(g->dlyu, i, j)) /
                      P2(g->dlyp, i, j) +
                  P2(g->dtdyo, i, j) *
                      ((V2(v1e, i, j) * cono + conn * V2(vze, i, j)) * V2(g->dlxv, i, j) -
                       (V2(v1e, i, j - 1) * cono + conn * V2(vze, i, j - 1)) * V2(g->dlxv, i, j - 1)) /
                      P2(g->dlxp, i, j));
      P2(b1o, i, j) = v * P2(xx, i, j);
    }
  memset(z1o, 0, sizeof(double) * (size_t)IE * JE);
  if (!b->eta_forc) {  /* troneu.f90:67-102 (one rank holds every edge) */
    for (int j = 1; j <= JE; ++j) P2(z1o, 1, j) = P2(b1o, 1, j) / P2(xx, 1, j);
    for (int j = 1; j <= JE; ++j) P2(z1o, IE, j) = P2(b1o, IE, j) / P2(xx, IE, j);
    for (int i = 1; i <= IE; ++i) P2(z1o, i, 1) = P2(b1o, i, 1) / P2(xx, i, 1);
    for (int i = 1; i <= IE; ++i) P2(z1o, i, JE) = P2(b1o, i, JE) / P2(xx, i, JE);
  }
  /* troneu.f90:104-134 */
  for (int it = 0; it < b->niter; ++it) {
    sor_colour(g, b, 0, uf, vf, ff, b1o, z1o);
    sor_colour(g, b, 1, uf, vf, ff, b1o, z1o);
  }
}

void og_ocvtro(const og_grid *g, const og_baro *b, const double *deutio, const double *deutie,
               const double *z1o, double *uzo, double *vze, double *uso, double *vse, double *zo) {
  DIMS;
  const double c = b->rlsa1 * b->grav * b->stabn;
  /* ocvtro.f90:11-23 */
  for (int j = 1; j <= JE; ++j)
    for (int i = 0; i <= IE; ++i) {
      U2(uzo, i, j) = U2(uzo, i, j) * U2(deutio, i, j);
      U2(uso, i, j) = U2(uzo, i, j);
    }
  for (int j = 0; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      V2(vze, i, j) = V2(vze, i, j) * V2(deutie, i, j);
      V2(vse, i, j) = V2(vze, i, j);
    }
  /* ocvtro.f90:34-48: rlsa1*G*STABN*DTDXUO*(Z1O(I)-Z1O(I+1))*AMSUO(I,J,1) */
  for (int j = 2; j <= JE1; ++j)
    for (int i = 1; i <= IE1; ++i)
      U2(uso, i, j) = U2(uzo, i, j) + c * U2(g->dtdxuo, i, j) * (P2(z1o, i, j) - P2(z1o, i + 1, j)) *
                                          U3(g->amsuo, i, j, 1);
  for (int j = 1; j <= JE1; ++j)
    for (int i = 2; i <= IE1; ++i)
      V2(vse, i, j) = V2(vze, i, j) + c * V2(g->dpye, i, j) * (P2(z1o, i, j + 1) - P2(z1o, i, j)) *
                                          V3(g->amsue, i, j, 1);
  /* ocvtro.f90:53-57 */
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) P2(zo, i, j) = P2(zo, i, j) + P2(z1o, i, j);
}

void og_ocvtot(const og_grid *g, const og_baro *b, const double *uso, const double *vse,
               double *uoo, double *voe, double *uko, double *vke, double *wo) {
  DIMS;
  const double conn = b->conn, cono = 1. - b->conn, dti = 1. / g->dt;
  /* ocvtot.f90:13-29 (T1O/S1O, copies of UOO/VOE, are not kept) */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i)
        U3(uko, i, j, k) = U3(g->amsuo, i, j, k) * (U2(uso, i, j) + U3(uko, i, j, k));
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i)
        V3(vke, i, j, k) = V3(g->amsue, i, j, k) * (V2(vse, i, j) + V3(vke, i, j, k));
  }
  /* ocvtot.f90:43-61 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i) {
        const double uako = U3(uko, i, j, k);
        U3(uko, i, j, k) = conn * U3(uko, i, j, k) + U3(uoo, i, j, k) * cono;
        U3(uoo, i, j, k) = uako;
      }
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        const double vake = V3(vke, i, j, k);
        V3(vke, i, j, k) = conn * V3(vke, i, j, k) + V3(voe, i, j, k) * cono;
        V3(voe, i, j, k) = vake;
      }
  }
  /* ocvtot.f90:73-93, WO(KEP) = 0 */
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      P3(wo, i, j, KE + 1) = 0.0;
      for (int k = KE; k >= 1; --k)
        P3(wo, i, j, k) =
            P3(wo, i, j, k + 1) +
            dti * P3(g->weto, i, j, k) *
                (P2(g->dtdxpo, i, j) *
                 (U3(uko, i - 1, j, k) * U3(g->dduo, i - 1, j, k) * U2(g->dlyu, i - 1, j) -
                  U3(uko, i, j, k) * U3(g->dduo, i, j, k) * U2(g->dlyu, i, j)) /
                 P2(g->dlyp, i, j)) +
            dti * P3(g->weto, i, j, k) *
                (+P2(g->dtdyo, i, j) *
                 (V3(vke, i, j, k) * V3(g->ddue, i, j, k) * V2(g->dlxv, i, j) -
                  V3(vke, i, j - 1, k) * V3(g->ddue, i, j - 1, k) * V2(g->dlxv, i, j - 1)) /
                 P2(g->dlxp, i, j));
    }
}

/* ocbarp.f90:10-45 */
void og_ocbarp(const og_grid *g, double *uso, double *vse, double *uzo, double *vze) {
  DIMS;
  for (int j = 1; j <= JE; ++j)
    for (int i = 0; i <= IE; ++i) U2(uzo, i, j) = U2(uso, i, j);
  for (int j = 0; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) V2(vze, i, j) = V2(vse, i, j);
  for (int j = 1; j <= JE; ++j)
    for (int i = 0; i <= IE; ++i) {
      U2(uso, i, j) = U2(uso, i, j) * U3(g->amsuo, i, j, 1);
      U2(uzo, i, j) = U2(uzo, i, j) * U3(g->amsuo, i, j, 1);
    }
  for (int j = 0; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      V2(vse, i, j) = V2(vse, i, j) * V3(g->amsue, i, j, 1);
      V2(vze, i, j) = V2(vze, i, j) * V3(g->amsue, i, j, 1);
    }
}

/* ocwind.f90:20-38 */
void og_ocwind(const og_grid *g, const double *txo, const double *tye, const double *sicomu,
               const double *sicomv, const double *tauwatu, const double *tauwatv, double *uoo,
               double *voe) {
  DIMS;
  const double dtdect = g->dt / K1(g->dzw, 1);
  for (int j = 2; j <= JE1; ++j)
    for (int i = 1; i <= IE1; ++i) {
      const double ur = P2(sicomu, i, j);
      U3(uoo, i, j, 1) = U3(uoo, i, j, 1) +
                         dtdect * U3(g->amsuo, i, j, 1) *
                             (U2(txo, i, j) * ur + (1. - ur) * U3(g->amsuo, i, j, 1) * P2(tauwatu, i, j));
    }
  for (int j = 1; j <= JE1; ++j)
    for (int i = 2; i <= IE1; ++i) {
      const double vr = P2(sicomv, i, j);
      V3(voe, i, j, 1) = V3(voe, i, j, 1) +
                         dtdect * V3(g->amsue, i, j, 1) *
                             (V2(tye, i, j) * vr + (1. - vr) * V3(g->amsue, i, j, 1) * P2(tauwatv, i, j));
    }
}

/* sqrtrnd.f90:1-8: C = SQRT(B*D); D = C - INT(C); the state D persists */
static double sqrtrnd(double *d) {
  const double b = 34251.;
  const double c = sqrt(b * *d);
  const int m = (int)c;
  *d = c - m;
  return *d;
}

/* trotest.f90:24-115 on one rank (p_ioff = p_joff = 0, IE_G = IE, JE_G = JE) */
double og_trotest(const og_grid *g, const og_baro *b, const double *xx, const double *uf,
                  const double *vf, const double *ff, int ntry, int niter) {
  DIMS;
  double *b1o = zalloc((size_t)IE * JE), *z = zalloc((size_t)IE * JE);
  double d = 0.34679201245;  /* DATA D of SQRTRND */
  for (int jj = 1; jj <= JE; ++jj)
    for (int ii = 1; ii <= IE; ++ii) {
      const double rnd = sqrtrnd(&d);
      P2(b1o, ii, jj) = (rnd - 0.5) * P3(g->weto, ii, jj, 1) * P2(xx, ii, jj);
    }
  double sorpar = 1.75, convmin = 9.E99, sorpmin = sorpar;
  for (int isor = 1; isor <= ntry; ++isor) {
    sorpar = sorpar + 0.001;
    memset(z, 0, sizeof(double) * (size_t)IE * JE);
    const double sorpai = 1. - sorpar;
    double chabas = 0.0, sumcha = 0.0;
    for (int kiter = 1; kiter <= niter; ++kiter) {
      sumcha = 0.;
      for (int parity = 0; parity < 2; ++parity)
        for (int j = 2; j <= JE1; ++j) {
          const int is = (j + parity) % 2 + 2;
          for (int i = is; i <= IE1; i += 2) {
            const double zalt = P2(z, i, j);
            P2(z, i, j) = sorpar * P2(ff, i, j) *
                              (P2(b1o, i, j) + U2(uf, i, j) * P2(z, i + 1, j) +
                               U2(uf, i - 1, j) * P2(z, i - 1, j) + V2(vf, i, j) * P2(z, i, j + 1) +
                               V2(vf, i, j - 1) * P2(z, i, j - 1)) +
                          sorpai * P2(z, i, j);
            const double dz = zalt - P2(z, i, j);
            sumcha = sumcha + dz * dz;
          }
        }
      if (kiter == 1) chabas = sumcha;
    }
    const double contric = sumcha / chabas;
    if (contric < convmin) {
      sorpmin = sorpar;
      convmin = contric;
    }
  }
  free(b1o);
  free(z);
  (void)b;
  return sorpmin;
}

/* ------------------------------------------------------------------------ */
/* OCTHER (octher.f90) with ADISITJ / RHO1J                                  */
/* ------------------------------------------------------------------------ */

/* adisitj.f90:46-69 with MO_PARAM3's coefficients (mo_param3.f90:11-13) */
double og_adisit(double th, double sh, double pa) {
  const double a1 = 3.6504E-4, a2 = 8.3198E-5, a3 = 5.4065E-7, a4 = 4.0274E-9;
  const double b1 = 1.7439E-5, b2 = 2.9778E-7, c1 = 8.9309E-7, c2 = 3.1628E-8;
  const double c3 = 2.1987E-10, d = 4.1057E-9, e1 = 1.6056E-10, e2 = 5.0484E-12;
  const double pr = pa;
  const double qc = pr * (a1 + pr * (c1 - e1 * pr));
  const double qv = pr * (b1 - d * pr);
  const double dc = 1. + pr * (-a2 + pr * (c2 - e2 * pr));
  const double dv = b2 * pr;
  const double qnq = -pr * (-a3 + pr * c3);
  const double qn3 = -pr * a4;
  const double qvs = qv * (sh - 35.) + qc;
  const double dvs = dv * (sh - 35.) + dc;
  const double tpo = th;
  th = (th + qvs) / dvs;
  const double t = th;
  const double fne = -qvs + t * (dvs + t * (qnq + t * qn3)) - tpo;
  const double fst = dvs + t * (2 * qnq + 3 * qn3 * t);
  return th - fne / fst;
}

/* rho1j.f90:82-115 */
double og_rho1(double t, double s, double p) {
  const double b0 = 8.24493E-1, b1 = -4.0899E-3, b2 = 7.6438E-5, b3 = -8.2467E-7, b4 = 5.3875E-9;
  const double c0 = -5.72466E-3, c1 = 1.0227E-4, c2 = -1.6546E-6, d0 = 4.8314E-4;
  const double a0 = 999.8426, a1 = 6.793952E-2, a2 = -9.095290E-3, a3 = 1.001685E-4,
               a4 = -1.120083E-6, a5 = 6.536332E-9;
  const double f0 = 54.6746, f1 = -0.603459, f2 = 1.09987E-2, f3 = -6.1670E-5;
  const double g0 = 7.944E-2, g1 = 1.6483E-2, g2 = -5.3009E-4;
  const double ai0 = 2.2838E-3, ai1 = -1.0981E-5, ai2 = -1.6078E-6, aj0 = 1.91075E-4;
  const double am0 = -9.9348E-7, am1 = 2.0816E-8, am2 = 9.1697E-10;
  const double e0 = 19652.21, e1 = 148.4206, e2 = -2.327105, e3 = 1.360477E-2, e4 = -5.155288E-5;
  const double h0 = 3.239908, h1 = 1.43713E-3, h2 = 1.16092E-4, h3 = -5.77905E-7;
  const double ak0 = 8.50935E-5, ak1 = -6.12293E-6, ak2 = 5.2787E-8;
  s = fmx(s, 28.);
  const double s3h = sqrt(s * s * s);
  const double num = a0 + t * (a1 + t * (a2 + t * (a3 + t * (a4 + t * a5)))) +
                     s * (b0 + t * (b1 + t * (b2 + t * (b3 + t * b4)))) + d0 * (s * s) +
                     s3h * (c0 + t * (c1 + c2 * t));
  const double kk = p * (h0 + t * (h1 + t * (h2 + t * h3)) + s * (ai0 + t * (ai1 + ai2 * t)) +
                         aj0 * s3h + (ak0 + t * (ak1 + t * ak2) + s * (am0 + t * (am1 + t * am2))) * p) +
                    e0 + t * (e1 + t * (e2 + t * (e3 + t * e4))) +
                    s * (f0 + t * (f1 + t * (f2 + t * f3))) + s3h * (g0 + t * (g1 + g2 * t));
  return num / (1. - p / kk);
}

/* density of potential temperature th, salinity s at reference pressure p
 * (ADISITJ then RHO1J, octher.f90:147-148), or the linear option */
static double og_density(const og_thermo *t, double th, double s, double p) {
  if (t->eos == 1) return t->rho0 + t->drdt * (th - t->t0) + t->drds * (s - t->s0);
  return og_rho1(og_adisit(th, s, p), s, p);
}

#define OPT2(a, i, j) ((a) ? P2((a), i, j) : 0.0)

/* octher.f90:43-107 */
void og_octher_surface(const og_grid *g, const og_thermo *t, double *tho, double *sao,
                       double *zo, double *eminpo, double *rivrun) {
  DIMS;
  const double dt = g->dt;
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      P2(eminpo, i, j) = 0.;
      const double reiscon = 1. - OPT2(t->sicomo, i, j); /* EISREST */
      const double oldso = P3(sao, i, j, 1);
      P3(sao, i, j, 1) = P3(sao, i, j, 1) + dt * t->relsal * reiscon *
                                                (OPT2(t->relsao, i, j) - P3(sao, i, j, 1));
      P3(tho, i, j, 1) =
          P3(tho, i, j, 1) + dt * t->reltem * (OPT2(t->reltho, i, j) - P3(tho, i, j, 1));
      P2(eminpo, i, j) = (P3(g->ddpo, i, j, 1) + P2(zo, i, j) - OPT2(t->sictho, i, j) * t->rhoicwa -
                          OPT2(t->sicsno, i, j) * t->rhosnwa) *
                         (fmx(oldso, 1.E-3) / fmx(P3(sao, i, j, 1), 1.E-3) - 1.);
    }
  const double dti = 1. / dt;
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      P2(zo, i, j) = (P2(zo, i, j) + P2(eminpo, i, j)) * P3(g->weto, i, j, 1);
      P2(eminpo, i, j) = P2(eminpo, i, j) * dti;
    }
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      const double zzzdz = fmx(g->almzer, P3(g->ddpo, i, j, 1) + P2(zo, i, j) -
                                              OPT2(t->sictho, i, j) * t->rhoicwa -
                                              OPT2(t->sicsno, i, j) * t->rhosnwa);
      const double driv = OPT2(t->giriv, i, j) * dt;
      P3(sao, i, j, 1) = P3(sao, i, j, 1) * zzzdz / (zzzdz + driv);
      P2(zo, i, j) = P2(zo, i, j) + driv;
      P2(rivrun, i, j) = driv / dt;
    }
}

/* octher.f90:139-451 */
void og_octher_column(const og_grid *g, const og_thermo *t, double *tho, double *sao,
                      const double *zo, const double *uko, const double *vke, double *po,
                      double *stabio, double *rhoo, double *avo, double *dvo, int *kcondep) {
  DIMS;
  const double G = t->grav;
  const double one = 1.;
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      /* C.1 upper layer (octher.f90:142-154) */
      const double rh1 = og_density(t, P3(tho, i, j, 1), P3(sao, i, j, 1), K1(t->preff, 1));
      P3(stabio, i, j, 1) = 0.;
      P3(po, i, j, 1) = G * K1(g->tiestu, 1) * 0.00097 * rh1;
      /* C.2 levels 2..KE (octher.f90:164-259); ZSURF(K-1) = 1 only for K = 2 */
      for (int k = 2; k <= KE; ++k) {
        const double disti = 1. / K1(g->dz, k);
        const double rh = og_density(t, P3(tho, i, j, k), P3(sao, i, j, k), K1(t->preff, k));
        const double rup = og_density(t, P3(tho, i, j, k - 1), P3(sao, i, j, k - 1), K1(t->preff, k));
        P3(stabio, i, j, k) = disti * (rh - rup);
        P3(po, i, j, k) = P3(po, i, j, k - 1) + G * K1(g->dz, k) * 0.00049 * (rh + rup);
        const double zs = k - 1 == 1 ? 1. : 0.;
        const double surf =
            zs * (P2(zo, i, j) - OPT2(t->sictho, i, j) * t->rhoicwa - OPT2(t->sicsno, i, j) * t->rhosnwa);
        const double tq = ((P3(g->ddpo, i, j, k - 1) + surf) * P3(tho, i, j, k - 1) +
                           P3(g->ddpo, i, j, k) * P3(tho, i, j, k)) /
                          (P3(g->ddpo, i, j, k) + P3(g->ddpo, i, j, k - 1) + surf +
                           (1. - P3(g->weto, i, j, k)));
        const double sq = ((P3(g->ddpo, i, j, k - 1) + surf) * P3(sao, i, j, k - 1) +
                           P3(g->ddpo, i, j, k) * P3(sao, i, j, k)) /
                          (P3(g->ddpo, i, j, k) + P3(g->ddpo, i, j, k - 1) + surf +
                           (1. - P3(g->weto, i, j, k)));
        const double st = P3(stabio, i, j, k);
        double switc = fmx(0., -st / (1.E-11 + fabs(st))) * P3(g->weto, i, j, k);
        const double helpswi = switc; /* NURDIF */
        switc = 0.;
        P3(tho, i, j, k - 1) = tq * switc + (one - switc) * P3(tho, i, j, k - 1);
        P3(tho, i, j, k) = tq * switc + (one - switc) * P3(tho, i, j, k);
        P3(sao, i, j, k - 1) = sq * switc + (one - switc) * P3(sao, i, j, k - 1);
        P3(sao, i, j, k) = sq * switc + (one - switc) * P3(sao, i, j, k);
        P3(stabio, i, j, k) = (one - switc) * P3(stabio, i, j, k);
        P3(stabio, i, j, k) = fmx(P3(stabio, i, j, k), 0.);
        switc = helpswi;
        if (P2(kcondep, i, j) == k - 1) P2(kcondep, i, j) += switc >= 0.5 ? 1 : 0; /* NINT */
      }
    }
  /* D: Richardson-number mixing (octher.f90:294-403) */
  const double relne = 0.4, relax = 1. - relne, gor = G / 1025.;
  const double cra = 5., crd = 5., wpendep = 40.;
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= JE1; ++j)
    for (int i = 1; i <= IE1; ++i) {
      const double ice = 1. - OPT2(t->sicomo, i, j);
      const double f = OPT2(t->fu10, i, j);
      double t1 = t->wt * (ice * ice) * (f * f * f); /* REDWMICE */
      double s1 = t->wt * (ice * ice) * (f * f * f);
      for (int k = 2; k <= KE; ++k) {
        const int ko = k - 1;
        const double stabeps = t->cstabeps / K1(g->dzw, ko);
        const double wtdecay = exp(-K1(g->dzw, ko) / wpendep);
        const double topnah = 0.0;
        const double zs = ko == 1 ? 1. : 0.;
        t1 = t1 * wtdecay * stabeps /
             (stabeps + 0.5 * (P3(stabio, i, j, k) + (1. - zs) * P3(stabio, i, j, ko)));
        s1 = s1 * wtdecay * stabeps /
             (stabeps + 0.5 * (P3(stabio, i, j, k) + (1. - zs) * P3(stabio, i, j, ko)));
        const double du1 = U3(uko, i - 1, j, k) - U3(uko, i - 1, j, ko);
        const double du2 = U3(uko, i, j, k) - U3(uko, i, j, ko);
        const double dv1 = V3(vke, i, j - 1, k) - V3(vke, i, j - 1, ko);
        const double dv2 = V3(vke, i, j, k) - V3(vke, i, j, ko);
        const double w = P3(g->weto, i, j, k);
        const double dik = K1(g->di, k);
        const double dudo =
            g->almzer + w * (dik * dik) * (du1 * du1 + du2 * du2 + dv1 * dv1 + dv2 * dv2) * 0.5;
        const double hho = w * (U3(g->amsuo, i, j, k) + U3(g->amsuo, i - 1, j, k) +
                                V3(g->amsue, i, j - 1, k) + V3(g->amsue, i, j, k)) *
                           0.25;
        const double rinumo = hho * fmx(gor * P3(stabio, i, j, k) / dudo, 0.);
        const double xd = 1. + crd * rinumo, xa = 1. + cra * rinumo;
        double *dv = &P3(dvo, i, j, k), *av = &P3(avo, i, j, k);
        *dv = (relax * fmn(*dv, t->dv0 + s1) +
               relne * (s1 + t->dv0 / (xd * xd * xd) + K1(t->dbackv, k) + topnah)) * w;
        *av = (relax * fmn(*av, t->av0 + K1(t->abackv, k)) +
               relne * (t1 + t->av0 / (xa * xa) + K1(t->abackv, k) + topnah)) * w;
        const double st = P3(stabio, i, j, k);
        *av = w * fmx(t->cavocon * (1.E-11 - st) / (1.E-11 + fabs(st)), *av);
        *dv = w * fmx(t->cdvocon * (1.E-11 - st) / (1.E-11 + fabs(st)), *dv);
        P3(stabio, i, j, k) = fmx(P3(stabio, i, j, k), 0.);
      }
    }
  /* octher.f90:415-451 */
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      P3(avo, i, j, KEP) = 0.;
      P3(dvo, i, j, KEP) = 0.;
      for (int k = 2; k <= KE; ++k)
        if (P3(g->weto, i, j, k) < 0.5) {
          P3(tho, i, j, k) = P3(tho, i, j, k - 1);
          P3(sao, i, j, k) = P3(sao, i, j, k - 1);
        }
      for (int k = 1; k <= KE; ++k)
        P3(rhoo, i, j, k) = og_density(t, P3(tho, i, j, k), P3(sao, i, j, k), K1(t->preff, k));
    }
}

/* ------------------------------------------------------------------------ */
/* OCMODMOM (ocmodmom.f90), NON_HYDROSTATIC                                  */
/* ------------------------------------------------------------------------ */
/* GILA / GIPH are (ITO, JTO) = (2 IE, 2 JE), 1-based */
#define GI(a, ii, jj) (a)[(size_t)((jj)-1) * (2 * IE) + (size_t)((ii)-1)]
#define W3(a, i, j, k) P3(a, i, j, k)

void og_ocmodmom(const og_grid *g, const og_baro *b, const og_coriolis *c,
                 const double *deutio, const double *deutie, const double *zo,
                 const double *uoo, const double *voe, double *uko, double *vke, double *uk1o,
                 double *vk1e, double *wno, double *wn1o, double *po, double *stabio,
                 double *u1o, double *uso, double *v1e, double *vse) {
  DIMS;
  const double G = b->grav, stabn = b->stabn, stabo = 1. - b->stabn, dt = g->dt;
  const double almzer = g->almzer, omega = c->omega;
  const size_t nu = (size_t)(IE + 1) * JE * KE, nv = (size_t)IE * (JE + 1) * KE;
  const size_t nw = (size_t)IE * JE * KEP;
  double *ucor = zalloc(nu), *vcor = zalloc(nv), *wcor = zalloc(nw);
  /* ocmodmom.f90:24-36 */
  for (int j = 1; j <= JE; ++j)
    for (int i = 0; i <= IE; ++i) U2(u1o, i, j) = U2(uso, i, j) = 0.;
  for (int j = 0; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) V2(v1e, i, j) = V2(vse, i, j) = 0.;
  /* ocmodmom.f90:39-62 */
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        P3(stabio, i, j, k) = 0.001 * K1(g->dz, k) * P3(stabio, i, j, k) * P3(g->weto, i, j, k);
        P3(po, i, j, k) = P3(po, i, j, k) + G * P2(zo, i, j) * b->rlsa1;
      }
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i) {
        U3(uko, i, j, k) = U3(uko, i, j, k) * U3(g->dduo, i, j, k);
        U3(uk1o, i, j, k) = U3(uko, i, j, k);
      }
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        V3(vke, i, j, k) = V3(vke, i, j, k) * V3(g->ddue, i, j, k);
        V3(vk1e, i, j, k) = V3(vke, i, j, k);
      }
  }
  memcpy(wn1o, wno, sizeof(double) * nw);
  for (int iter = 1; iter <= 12; ++iter) {
    /* ocmodmom.f90:76-96 */
    for (int k = 1; k <= KE; ++k) {
      for (int j = 1; j <= JE; ++j)
        for (int i = 0; i <= IE; ++i)
          U3(ucor, i, j, k) = stabn * U3(uk1o, i, j, k) + stabo * U3(uko, i, j, k);
      for (int j = 0; j <= JE; ++j)
        for (int i = 1; i <= IE; ++i)
          V3(vcor, i, j, k) = stabn * V3(vk1e, i, j, k) + stabo * V3(vke, i, j, k);
    }
    for (int k = 1; k <= KEP; ++k)
      for (int j = 1; j <= JE; ++j)
        for (int i = 1; i <= IE; ++i)
          W3(wcor, i, j, k) = stabn * W3(wn1o, i, j, k) + stabo * W3(wno, i, j, k);
    /* ocmodmom.f90:99-170 */
    for (int k = 1; k <= KE; ++k) {
      for (int j = 2; j <= JE1; ++j)
        for (int i = 1; i <= IE1; ++i) {
          const double vcor_u = 0.25 * (V3(vcor, i, j, k) + V3(vcor, i + 1, j, k) +
                                        V3(vcor, i, j - 1, k) + V3(vcor, i + 1, j - 1, k));
          U3(uk1o, i, j, k) = U3(uko, i, j, k) +
                              U2(g->dtdxuo, i, j) * (P3(po, i, j, k) - P3(po, i + 1, j, k)) *
                                  U3(g->dduo, i, j, k) +
                              dt * U2(c->ftwou, i, j) * vcor_u * U3(g->amsuo, i, j, k);
        }
      for (int j = 1; j <= JE1; ++j)
        for (int i = 2; i <= IE1; ++i) {
          const double ucor_v = 0.25 * (U3(ucor, i, j, k) + U3(ucor, i - 1, j, k) +
                                        U3(ucor, i, j + 1, k) + U3(ucor, i - 1, j + 1, k));
          V3(vk1e, i, j, k) = V3(vke, i, j, k) +
                              V2(g->dpye, i, j) * (P3(po, i, j + 1, k) - P3(po, i, j, k)) *
                                  V3(g->ddue, i, j, k) -
                              dt * V2(c->ftwov, i, j) * ucor_v * V3(g->amsue, i, j, k);
        }
      for (int j = 2; j <= JE1; ++j)
        for (int i = 1; i <= IE1; ++i) {
          const double dlon = (GI(c->gila, 2 * i + 2, 2 * j) - GI(c->gila, 2 * i + 1, 2 * j)) *
                              cos(GI(c->gila, 2 * i + 1, 2 * j));
          const double dlat = GI(c->giph, 2 * i + 2, 2 * j) - GI(c->giph, 2 * i + 1, 2 * j);
          const double dist = sqrt(dlon * dlon + dlat * dlat) + almzer;
          const double ftwou1 = 2 * omega * cos(GI(c->giph, 2 * i + 1, 2 * j));
          const double wcor_u = 0.25 *
                                ((W3(wcor, i, j, k) + W3(wcor, i, j, k + 1)) * P2(g->dlxp, i, j) +
                                 (W3(wcor, i + 1, j, k) + W3(wcor, i + 1, j, k + 1)) * P2(g->dlxp, i + 1, j)) /
                                U2(g->dlxu, i, j);
          U3(uk1o, i, j, k) =
              U3(uk1o, i, j, k) - dt * ftwou1 * wcor_u * U3(g->dduo, i, j, k) * dlon / dist;
        }
      for (int j = 1; j <= JE1; ++j)
        for (int i = 2; i <= IE1; ++i) {
          const double dlon = (GI(c->gila, 2 * i, 2 * j) - GI(c->gila, 2 * i, 2 * j + 1)) *
                              cos(GI(c->gila, 2 * i, 2 * j + 1));
          const double dlat = GI(c->giph, 2 * i, 2 * j) - GI(c->giph, 2 * i, 2 * j + 1);
          const double dist = sqrt(dlon * dlon + dlat * dlat) + almzer;
          const double ftwov1 = 2 * omega * cos(GI(c->giph, 2 * i, 2 * j + 1));
          const double wcor_v = 0.25 *
                                ((W3(wcor, i, j, k) + W3(wcor, i, j, k + 1)) * P2(g->dlyp, i, j) +
                                 (W3(wcor, i, j + 1, k) + W3(wcor, i, j + 1, k + 1)) * P2(g->dlyp, i, j + 1)) /
                                V2(g->dlyv, i, j);
          V3(vk1e, i, j, k) =
              V3(vk1e, i, j, k) - dt * ftwov1 * wcor_v * V3(g->ddue, i, j, k) * dlon / dist;
        }
      if (k > 1)
        for (int j = 2; j <= JE1; ++j)
          for (int i = 2; i <= IE1; ++i) {
            const double dlon = (GI(c->gila, 2 * i + 1, 2 * j) - GI(c->gila, 2 * i, 2 * j)) *
                                cos(GI(c->gila, 2 * i, 2 * j));
            const double dlat = GI(c->giph, 2 * i, 2 * j - 1) - GI(c->giph, 2 * i, 2 * j);
            const double dist = sqrt(dlon * dlon + dlat * dlat) + almzer;
            const double ftwow1 = 2 * omega * cos(GI(c->giph, 2 * i, 2 * j));
            const double ucor_w =
                0.25 * ((U3(uko, i, j, k) + U3(uko, i - 1, j, k)) / (P3(g->ddpo, i, j, k) + almzer) +
                        (U3(uko, i, j, k - 1) + U3(uko, i - 1, j, k - 1)) /
                            (P3(g->ddpo, i, j, k - 1) + almzer));
            const double vcor_w =
                0.25 * ((V3(vke, i, j, k) + V3(vke, i, j - 1, k)) / (P3(g->ddpo, i, j, k) + almzer) +
                        (V3(vke, i, j, k - 1) + V3(vke, i, j - 1, k - 1)) /
                            (P3(g->ddpo, i, j, k - 1) + almzer));
            W3(wn1o, i, j, k) = W3(wno, i, j, k) +
                                dt * P3(g->weto, i, j, k) *
                                    (ftwow1 * dlon / dist * ucor_w - ftwow1 * dlat / dist * vcor_w);
          }
    }
    /* ocmodmom.f90:177-183 */
    memcpy(wno, wn1o, sizeof(double) * nw);
  }
  /* ocmodmom.f90:193-215 */
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) P3(po, i, j, k) = P3(po, i, j, k) - G * P2(zo, i, j) * b->rlsa1;
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i) {
        U2(u1o, i, j) = U2(u1o, i, j) + U3(g->dduo, i, j, k) * U3(uoo, i, j, k);
        U2(uso, i, j) = U2(uso, i, j) + U3(uk1o, i, j, k);
      }
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        V2(v1e, i, j) = V2(v1e, i, j) + V3(g->ddue, i, j, k) * V3(voe, i, j, k);
        V2(vse, i, j) = V2(vse, i, j) + V3(vk1e, i, j, k);
      }
  }
  /* ocmodmom.f90:219-237 */
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i) {
        U3(uko, i, j, k) = U3(uoo, i, j, k) - U3(g->amsuo, i, j, k) * U2(deutio, i, j) * U2(u1o, i, j);
        U3(uk1o, i, j, k) = U3(uk1o, i, j, k) * (U3(g->amsuo, i, j, k) / (almzer + U3(g->dduo, i, j, k))) -
                            U3(g->amsuo, i, j, k) * U2(deutio, i, j) * U2(uso, i, j);
      }
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        V3(vke, i, j, k) = V3(voe, i, j, k) - V3(g->amsue, i, j, k) * V2(deutie, i, j) * V2(v1e, i, j);
        V3(vk1e, i, j, k) = V3(vk1e, i, j, k) * (V3(g->amsue, i, j, k) / (almzer + V3(g->ddue, i, j, k))) -
                            V3(g->amsue, i, j, k) * V2(deutie, i, j) * V2(vse, i, j);
      }
  }
  free(ucor);
  free(vcor);
  free(wcor);
}

/* ------------------------------------------------------------------------ */
/* OCCLIT (occlit.f90)                                                       */
/* ------------------------------------------------------------------------ */
/* vertical velocity from the divergence of transports uko / vke (already
 * multiplied by the thicknesses), bottom up from `bottom` (occlit.f90:108-112,
 * 250-254): out(k) = below + DTI WETO (...) */
static double og_occlit_div(const og_grid *g, const double *uko, const double *vke, int i, int j,
                            int k, double below) {
  const int IE = g->ie, JE = g->je;
  const double dti = 1. / g->dt;
  return below + dti * P3(g->weto, i, j, k) *
                     (P2(g->dtdxpo, i, j) *
                          (U3(uko, i - 1, j, k) * U2(g->dlyu, i - 1, j) - U3(uko, i, j, k) * U2(g->dlyu, i, j)) /
                          P2(g->dlyp, i, j) +
                      P2(g->dtdyo, i, j) *
                          (V3(vke, i, j, k) * V2(g->dlxv, i, j) - V3(vke, i, j - 1, k) * V2(g->dlxv, i, j - 1)) /
                          P2(g->dlxp, i, j));
}

double og_occlit(const og_grid *g, const og_baro *b, const double *deutio,
                 const double *deutie, double *uko, double *vke, double *uk1o, double *vk1e,
                 double *wo, double *stabio) {
  DIMS;
  const double G = b->grav, stabn = b->stabn, conn = b->conn, dt = g->dt, almzer = g->almzer;
  const size_t n2 = (size_t)IE * JE, n3 = n2 * KE;
  double *bruva = zalloc(n2), *slow = zalloc(n2), *tlow = zalloc(n2), *contrij = zalloc(n2);
  double *pxoin = zalloc((size_t)(IE + 1) * JE), *ucos = zalloc((size_t)(IE + 1) * JE);
  double *pyein = zalloc((size_t)IE * (JE + 1)), *vcos = zalloc((size_t)IE * (JE + 1));
  double *t1o = zalloc(n3), *wpo = zalloc(n3);
  /* occlit.f90:20-63 (PXOIN / PYEIN of this first pass are reset before use) */
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) P3(stabio, i, j, 1) = 0.;
  for (int k = 1; k <= KE; ++k)
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i)
        P2(bruva, i, j) = P2(bruva, i, j) + K1(g->tiestw, k + 1) * P3(stabio, i, j, k);
  /* occlit.f90:85-101 */
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i) {
        U3(uko, i, j, k) = U3(uko, i, j, k) * U3(g->dduo, i, j, k);
        U3(uk1o, i, j, k) = U3(uk1o, i, j, k) * U3(g->dduo, i, j, k);
      }
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        V3(vke, i, j, k) = V3(vke, i, j, k) * V3(g->ddue, i, j, k);
        V3(vk1e, i, j, k) = V3(vk1e, i, j, k) * V3(g->ddue, i, j, k);
      }
  }
  /* occlit.f90:104-127 */
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i)
      for (int k = KE; k >= 1; --k) P3(wo, i, j, k) = og_occlit_div(g, uko, vke, i, j, k, P3(wo, i, j, k + 1));
  for (int j = 1; j <= JE; ++j)
    for (int k = 1; k <= KE; ++k)
      for (int i = 1; i <= IE; ++i) {
        P3(t1o, i, j, k) = P3(wo, i, j, k);
        P2(slow, i, j) = P2(slow, i, j) + P3(stabio, i, j, k) * dt * P3(wo, i, j, k);
        P3(wpo, i, j, k) = P2(slow, i, j);
      }
  double under = 0.;
  const int itermax = 8;
  for (int iter = 1; iter <= itermax; ++iter) {
    /* occlit.f90:139-183 */
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i) U2(ucos, i, j) = U2(pxoin, i, j) = 0.;
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) V2(vcos, i, j) = V2(pyein, i, j) = 0.;
    for (int k = 1; k <= KE; ++k) {
      for (int j = 1; j <= JE; ++j)
        for (int i = 1; i <= IE1; ++i)
          U2(pxoin, i, j) = U2(pxoin, i, j) + U3(g->dduo, i, j, k) * U2(g->dtdxuo, i, j) *
                                                  (P3(wpo, i + 1, j, k) - P3(wpo, i, j, k)) *
                                                  U3(g->amsuo, i, j, k);
      for (int j = 1; j <= JE1; ++j)
        for (int i = 1; i <= IE; ++i)
          V2(pyein, i, j) = V2(pyein, i, j) + V3(g->ddue, i, j, k) * V2(g->dpye, i, j) *
                                                  (P3(wpo, i, j, k) - P3(wpo, i, j + 1, k)) *
                                                  V3(g->amsue, i, j, k);
    }
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE1; ++i) U2(pxoin, i, j) = U2(pxoin, i, j) * U2(deutio, i, j);
    for (int j = 1; j <= JE1; ++j)
      for (int i = 1; i <= IE; ++i) V2(pyein, i, j) = V2(pyein, i, j) * V2(deutie, i, j);
    /* occlit.f90:191-228 */
    for (int k = 1; k <= KE; ++k) {
      for (int j = 2; j <= JE1; ++j)
        for (int i = 1; i <= IE1; ++i) {
          U3(uko, i, j, k) = U3(uk1o, i, j, k) +
                             stabn * (U2(pxoin, i, j) - U2(g->dtdxuo, i, j) * (P3(wpo, i + 1, j, k) - P3(wpo, i, j, k))) *
                                 U3(g->dduo, i, j, k);
          U2(ucos, i, j) = U2(ucos, i, j) + U3(uko, i, j, k);
          U3(uko, i, j, k) = U3(uko, i, j, k) * U3(g->amsuo, i, j, k);
        }
      for (int j = 1; j <= JE1; ++j)
        for (int i = 2; i <= IE1; ++i) {
          V3(vke, i, j, k) = V3(vk1e, i, j, k) +
                             stabn * (V2(pyein, i, j) - V2(g->dpye, i, j) * (P3(wpo, i, j, k) - P3(wpo, i, j + 1, k))) *
                                 V3(g->ddue, i, j, k);
          V2(vcos, i, j) = V2(vcos, i, j) + V3(vke, i, j, k);
          V3(vke, i, j, k) = V3(vke, i, j, k) * V3(g->amsue, i, j, k);
        }
    }
    for (int k = 1; k <= KE; ++k) {
      for (int j = 2; j <= JE1; ++j)
        for (int i = 1; i <= IE1; ++i)
          U3(uko, i, j, k) = U3(uko, i, j, k) - U2(ucos, i, j) * U2(deutio, i, j) * U3(g->dduo, i, j, k);
      for (int j = 1; j <= JE1; ++j)
        for (int i = 2; i <= IE1; ++i)
          V3(vke, i, j, k) = V3(vke, i, j, k) - V2(vcos, i, j) * V2(deutie, i, j) * V3(g->ddue, i, j, k);
    }
    if (iter == itermax) break;
    /* occlit.f90:238-284 */
    for (size_t q = 0; q < n2; ++q) tlow[q] = slow[q] = contrij[q] = 0.;
    for (int k = KE; k >= 1; --k)
      for (int j = 1; j <= JE; ++j)
        for (int i = 1; i <= IE; ++i) {
          P3(t1o, i, j, k) = og_occlit_div(g, uko, vke, i, j, k, P2(slow, i, j));
          P2(slow, i, j) = P3(t1o, i, j, k);
        }
    for (int k = 2; k <= KE; ++k)
      for (int j = 1; j <= JE; ++j)
        for (int i = 1; i <= IE; ++i) {
          const double ove = P3(wpo, i, j, k);
          P2(tlow, i, j) = P2(tlow, i, j) + G * P3(stabio, i, j, k) * dt *
                                                (conn * P3(t1o, i, j, k) + P3(wo, i, j, k));
          const double speed = 2. * G * P2(bruva, i, j) *
                               (U2(g->dtdxuo, i, j) * U2(g->dtdxuo, i, j) + P2(g->dtdyo, i, j) * P2(g->dtdyo, i, j));
          const double brems = under * speed * conn * stabn / (1. + speed);
          const double vorw = 1. - brems;
          P3(wpo, i, j, k) = vorw * P2(tlow, i, j) + brems * P3(wpo, i, j, k);
          const double d = ove - P3(wpo, i, j, k);
          P2(contrij, i, j) = P2(contrij, i, j) + d * d;
        }
    under = 1.;
  }
  /* occlit.f90:289-305 */
  for (int k = 1; k <= KE; ++k) {
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i) {
        U3(uko, i, j, k) = U3(uko, i, j, k) * U3(g->amsuo, i, j, k) / (almzer + U3(g->dduo, i, j, k));
        U3(uk1o, i, j, k) = U3(uk1o, i, j, k) * U3(g->amsuo, i, j, k) / (almzer + U3(g->dduo, i, j, k));
      }
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        V3(vke, i, j, k) = V3(vke, i, j, k) * V3(g->amsue, i, j, k) / (almzer + V3(g->ddue, i, j, k));
        V3(vk1e, i, j, k) = V3(vk1e, i, j, k) * V3(g->amsue, i, j, k) / (almzer + V3(g->ddue, i, j, k));
      }
  }
  /* occlit.f90:309-317, global (J, I) order */
  double contra = 0.;
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) contra = contra + P2(contrij, i, j);
  free(bruva);
  free(slow);
  free(tlow);
  free(contrij);
  free(pxoin);
  free(ucos);
  free(pyein);
  free(vcos);
  free(t1o);
  free(wpo);
  return contra;
}
