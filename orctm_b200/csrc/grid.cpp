// Host-side BELEG (beleg.f90:48-139) and BODEN (boden.f90:38-213) geometry:
// vertical grid, DT-scaled metrics, wet masks and partial-cell thicknesses.
// The reference computes these once at start-up on the host; callers that
// have no Fortran host get the identical arrays from orctm_build_grid.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/orctm_gpu.h"

namespace {
struct Ix {
  int IE, JE, KE;
  size_t p2(int i, int j) const { return (size_t)(j - 1) * IE + (i - 1); }
  size_t u2(int i, int j) const { return (size_t)(j - 1) * (IE + 1) + i; }
  size_t v2(int i, int j) const { return (size_t)j * IE + (i - 1); }
  size_t p3(int i, int j, int k) const { return ((size_t)(k - 1) * JE + (j - 1)) * IE + (i - 1); }
  size_t u3(int i, int j, int k) const { return ((size_t)(k - 1) * JE + (j - 1)) * (IE + 1) + i; }
  size_t v3(int i, int j, int k) const { return ((size_t)(k - 1) * (JE + 1) + j) * IE + (i - 1); }
};
inline double fmn(double a, double b) { return b < a ? b : a; }
}  // namespace

extern "C" int orctm_build_grid(int ie, int je, int ke, double dt, const double* dzw, double* depto,
                                const double* dlxp, const double* dlyp, const double* dlxu,
                                const double* dlyu, const double* dlxv, const double* dlyv,
                                double* tiestu, double* tiestw, double* dz, double* di,
                                double* dtdxpo, double* dtdyo, double* dtdxuo, double* dpyo,
                                double* dtdxue, double* dpye, double* ddpo, double* weto,
                                double* dduo, double* amsuo, double* ddue, double* amsue) {
  if (ie < 3 || je < 3 || ke < 2 || !dzw || !depto || !dlxp || !dlyp || !dlxu || !dlyu ||
      !dlxv || !dlyv || !tiestu || !tiestw || !dz || !di || !dtdxpo || !dtdyo || !dtdxuo ||
      !dpyo || !dtdxue || !dpye || !ddpo || !weto || !dduo || !amsuo || !ddue || !amsue)
    return ORCTM_E_ARG;
  const Ix x{ie, je, ke};
  const int IE = ie, JE = je, KE = ke, IE1 = ie - 1, JE1 = je - 1;
  // DT-scaled metrics (beleg.f90:42-76)
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      dtdxpo[x.p2(i, j)] = dt / dlxp[x.p2(i, j)];
      dtdyo[x.p2(i, j)] = dt / dlyp[x.p2(i, j)];
    }
  for (int j = 1; j <= JE; ++j)
    for (int i = 0; i <= IE; ++i) {
      dtdxuo[x.u2(i, j)] = dt / dlxu[x.u2(i, j)];
      dpyo[x.u2(i, j)] = dt / dlyu[x.u2(i, j)];
    }
  for (int j = 0; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      dtdxue[x.v2(i, j)] = dt / dlxv[x.v2(i, j)];
      dpye[x.v2(i, j)] = dt / dlyv[x.v2(i, j)];
    }
  // layer depths (beleg.f90:87-105) and DI (beleg.f90:125-139)
  tiestu[0] = 0.5 * dzw[0];
  tiestw[0] = 0.0;
  for (int k = 1; k <= KE; ++k) tiestw[k] = tiestw[k - 1] + dzw[k - 1];
  for (int k = 2; k <= KE; ++k) tiestu[k - 1] = 0.5 * (tiestw[k] + tiestw[k - 1]);
  tiestu[KE] = 9000.;
  dz[0] = tiestu[0];
  for (int k = 2; k <= KE + 1; ++k) dz[k - 1] = tiestu[k - 1] - tiestu[k - 2];
  for (int k = 1; k <= KE; ++k) di[k - 1] = 1. / dz[k - 1];
  di[KE] = 1. / dz[KE - 1];
  // depth clean-up (boden.f90:38-62, 101-107)
  const double minvalue = fmn(1.0, dzw[0] / 10.0);
  const double depmin = dzw[0] + dzw[1] + minvalue;
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      double& d = depto[x.p2(i, j)];
      if (d <= minvalue) d = 0.;
      if (d > minvalue && d < depmin) d = depmin;
    }
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i)
      for (int k = 1; k <= KE; ++k) {
        double& d = depto[x.p2(i, j)];
        if (std::fabs(d - tiestu[k - 1]) < minvalue / 2) d = tiestu[k - 1] + minvalue;
      }
  // depths at u and v points (boden.f90:116-130)
  std::vector<double> deuto((size_t)(IE + 1) * JE, 0.0), deute((size_t)IE * (JE + 1), 0.0);
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE1; ++i) deuto[x.u2(i, j)] = fmn(depto[x.p2(i, j)], depto[x.p2(i + 1, j)]);
  for (int j = 1; j <= JE; ++j) {
    deuto[x.u2(0, j)] = deuto[x.u2(1, j)];
    deuto[x.u2(IE, j)] = deuto[x.u2(IE1, j)];
  }
  for (int j = 1; j <= JE1; ++j)
    for (int i = 1; i <= IE; ++i) deute[x.v2(i, j)] = fmn(depto[x.p2(i, j)], depto[x.p2(i, j + 1)]);
  for (int i = 1; i <= IE; ++i) {
    deute[x.v2(i, 0)] = deute[x.v2(i, 1)];
    deute[x.v2(i, JE)] = deute[x.v2(i, JE1)];
  }
  // masks and thicknesses (boden.f90:182-213), arrays start at zero
  std::memset(ddpo, 0, sizeof(double) * (size_t)IE * JE * KE);
  std::memset(weto, 0, sizeof(double) * (size_t)IE * JE * KE);
  std::memset(dduo, 0, sizeof(double) * (size_t)(IE + 1) * JE * KE);
  std::memset(amsuo, 0, sizeof(double) * (size_t)(IE + 1) * JE * KE);
  std::memset(ddue, 0, sizeof(double) * (size_t)IE * (JE + 1) * KE);
  std::memset(amsue, 0, sizeof(double) * (size_t)IE * (JE + 1) * KE);
  for (int k = 1; k <= KE; ++k) {
    const double tu = tiestu[k - 1], tu1 = tiestu[k], tw = tiestw[k - 1], dzk = dzw[k - 1];
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        const double d = depto[x.p2(i, j)];
        if (tu < d) weto[x.p3(i, j, k)] = 1.;
        if (tu1 < d) ddpo[x.p3(i, j, k)] = dzk;
        if (tu < d && tu1 >= d) ddpo[x.p3(i, j, k)] = d - tw;
      }
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i) {
        const double d = deuto[x.u2(i, j)];
        double& t = dduo[x.u3(i, j, k)];
        if (tu1 < d) t = dzk;
        if (tu < d && tu1 >= d) t = d - tw;
        if (t > 0.) amsuo[x.u3(i, j, k)] = 1.;
      }
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        const double d = deute[x.v2(i, j)];
        double& t = ddue[x.v3(i, j, k)];
        if (tu1 < d) t = dzk;
        if (tu < d && tu1 >= d) t = d - tw;
        if (t > 0.) amsue[x.v3(i, j, k)] = 1.;
      }
  }
  return ORCTM_OK;
}
