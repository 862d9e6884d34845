// EXTRA-format records, the reference's output and restart format: a header
// record of four 4-byte integers (IDATE, ICODE, KCODE, IEDIM) followed by a
// record of the field's values as 4-byte reals, REAL(x, sp)
// (write_slice, mo_parallel.f90:733-779, called after the header as in
// aufw.f90:54-160).  The records are Fortran sequential unformatted records
// (a 4-byte length before and after the payload), and the model is built with
// -convert big_endian (ORCTM/src_orctm/Makefile:75), so every integer, real
// and record length is written big-endian.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/orctm_gpu.h"

namespace {

uint32_t be32(uint32_t v) {
  return ((v & 0xffu) << 24) | ((v & 0xff00u) << 8) | ((v >> 8) & 0xff00u) | (v >> 24);
}

bool put_record(FILE* f, const void* payload, uint32_t bytes) {
  const uint32_t m = be32(bytes);
  return fwrite(&m, 4, 1, f) == 1 && (bytes == 0 || fwrite(payload, 1, bytes, f) == bytes) &&
         fwrite(&m, 4, 1, f) == 1;
}

}  // namespace

extern "C" int orctm_write_extra_host(const char* path, int append, int idate, int code, int nlev,
                                      const int* kcodes, int iedim, const double* data) {
  if (!path || nlev < 1 || iedim < 1 || !kcodes || !data) return ORCTM_E_ARG;
  FILE* f = fopen(path, append ? "ab" : "wb");
  if (!f) return ORCTM_E_ARG;
  std::vector<uint32_t> vals((size_t)iedim);
  bool ok = true;
  for (int l = 0; l < nlev && ok; ++l) {
    const int32_t hdr[4] = {idate, code, kcodes[l], iedim};
    uint32_t bhdr[4];
    for (int k = 0; k < 4; ++k) {
      uint32_t u;
      std::memcpy(&u, &hdr[k], 4);
      bhdr[k] = be32(u);
    }
    ok = put_record(f, bhdr, 16);
    const double* src = data + (size_t)l * iedim;
    for (int n = 0; n < iedim && ok; ++n) {
      const float x = (float)src[n];  // REAL(x, sp): round to nearest
      uint32_t u;
      std::memcpy(&u, &x, 4);
      vals[(size_t)n] = be32(u);
    }
    if (ok) ok = put_record(f, vals.data(), (uint32_t)(4 * (size_t)iedim));
  }
  if (fclose(f) != 0) ok = false;
  return ok ? ORCTM_OK : ORCTM_E_ARG;
}

namespace {

// One Fortran sequential record whose length must be `expected` bytes: the
// marker is checked before anything is allocated, so a corrupt or
// wrong-endian file cannot ask for a huge buffer.
bool get_record(FILE* f, std::vector<unsigned char>& payload, uint64_t expected) {
  uint32_t m0, m1;
  if (fread(&m0, 4, 1, f) != 1) return false;
  const uint32_t n = be32(m0);
  if (n != expected) return false;
  try {
    payload.resize(n);
  } catch (const std::bad_alloc&) {
    return false;
  }
  if (n && fread(payload.data(), 1, n, f) != n) return false;
  if (fread(&m1, 4, 1, f) != 1 || m1 != m0) return false;
  return true;
}

}  // namespace

// Reads the first nlev records of field code `code` and size iedim (in file
// order) into out (levels consecutive), converting the 4-byte reals to double
// exactly as the reference's read_slice assigns REAL(sp) to its REAL arrays
// (aufr.f90:103-167); kcodes (may be NULL) receives their KCODE.
extern "C" int orctm_read_extra_host(const char* path, int code, int nlev, int iedim,
                                     double* out, int* kcodes) {
  if (!path || nlev < 1 || iedim < 1 || !out) return ORCTM_E_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) return ORCTM_E_ARG;
  std::vector<unsigned char> hdr, vals;
  int found = 0;
  bool ok = true;
  while (found < nlev && (ok = get_record(f, hdr, 16))) {
    int32_t h[4];
    for (int k = 0; k < 4; ++k) {
      uint32_t u;
      std::memcpy(&u, hdr.data() + 4 * k, 4);
      u = be32(u);
      std::memcpy(&h[k], &u, 4);
    }
    // IEDIM of the header sizes the data record (4-byte reals; a record
    // length is a 32-bit marker)
    if (h[3] < 1 || (uint64_t)h[3] * 4 > 0xFFFFFFFFull ||
        !(ok = get_record(f, vals, (uint64_t)h[3] * 4))) {
      ok = false;
      break;
    }
    if (h[1] != code || h[3] != iedim) continue;
    double* dst = out + (size_t)found * iedim;
    for (int n = 0; n < iedim; ++n) {
      uint32_t u;
      std::memcpy(&u, vals.data() + 4 * (size_t)n, 4);
      u = be32(u);
      float x;
      std::memcpy(&x, &u, 4);
      dst[n] = (double)x;
    }
    if (kcodes) kcodes[found] = h[2];
    ++found;
  }
  fclose(f);
  return found == nlev ? ORCTM_OK : ORCTM_E_ARG;
}

// GRID_INFO.ext (WRTE_GRIDINFO, wrte_gridinfo.f90:19-172): the grid in the
// same EXTRA records, IDATE 0, codes by the ABC rule of
// ORCTM/code_output.txt (A 1 lon/lat, 2 depth, 3 mask, 4 spacing; B 0/1/2/3
// none/x/y/z; C 0/1/2 p/u/v point): longitudes and latitudes 110-122, depths
// 200-202 and spacings 410-422 as 2D records (KCODE -100), then per level
// K = 1..KE (KCODE K) the masks 300-302 and thicknesses 430-432.
extern "C" int orctm_write_gridinfo(const char* path, const orctm_desc* d,
                                    const orctm_gridinfo* g) {
  if (!path || !d || !g || d->ie < 1 || d->je < 1 || d->ke < 1) return ORCTM_E_ARG;
  const int IE = d->ie, JE = d->je, KE = d->ke;
  const int np = IE * JE, nu = (IE + 1) * JE, nv = IE * (JE + 1);
  struct Rec2 { int code; int n; const double* a; };
  const Rec2 flat[] = {
      {110, np, g->lonp}, {120, np, g->latp}, {111, nu, g->lonu}, {121, nu, g->latu},
      {112, nv, g->lonv}, {122, nv, g->latv}, {200, np, g->depto}, {201, nu, g->deuto},
      {202, nv, g->deute}, {410, np, d->dlxp}, {411, nu, d->dlxu}, {412, nv, d->dlxv},
      {420, np, d->dlyp}, {421, nu, d->dlyu}, {422, nv, d->dlyv}};
  const Rec2 levels[] = {{300, np, d->weto}, {301, nu, d->amsuo}, {302, nv, d->amsue},
                         {430, np, d->ddpo}, {431, nu, d->dduo}, {432, nv, d->ddue}};
  for (const Rec2& r : flat)
    if (!r.a) return ORCTM_E_ARG;
  for (const Rec2& r : levels)
    if (!r.a) return ORCTM_E_ARG;
  std::vector<int> kc((size_t)KE);
  for (int k = 0; k < KE; ++k) kc[(size_t)k] = k + 1;
  const int m100 = -100;
  bool first = true;
  int st;
  for (const Rec2& r : flat) {
    if ((st = orctm_write_extra_host(path, first ? 0 : 1, 0, r.code, 1, &m100, r.n, r.a))) return st;
    first = false;
  }
  for (const Rec2& r : levels)
    if ((st = orctm_write_extra_host(path, 1, 0, r.code, KE, kc.data(), r.n, r.a))) return st;
  return ORCTM_OK;
}
