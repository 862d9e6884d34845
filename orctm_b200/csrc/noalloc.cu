// orctm_octdiff_noalloc: tracer diffusion of one tracer (OCTDIFF_BASE +
// OCTDIFF_TS) for callers that cannot allocate device memory.
//
// Who needs it.  Some callers are not allowed to call cudaMalloc: code that
// runs while a CUDA graph is being captured (an allocation would break the
// capture), host programs whose device memory is owned by another runtime or
// pool (an OpenACC/OpenMP-offload Fortran model, a framework allocator) and
// must not take memory behind its back, and time-critical loops that must
// not block on the driver's allocator.  orctm_create needs device memory for
// its handle; this entry point needs none: the caller passes device pointers
// to every input and output in the reference's own Fortran layouts, and the
// two scratch fields the routine needs live in one fixed array compiled into
// the library.
//
// The scratch array.  g_noalloc_scratch below is a file-scope __device__
// array of kNoAllocMaxCells * 2 doubles (32 MiB).  Every GPU that loads the
// library holds it until the process exits.  All calls on a device share it
// and it keeps the last call's contents; every element a call reads was
// written earlier in that same call, so nothing has to be cleared between
// calls.  Calls whose kernels overlap on the GPU (different streams, or
// host threads, without ordering) race on it: order them on one stream.
//
// The device address of the array is looked up with cudaGetSymbolAddress on
// the first call made on each device, with that device current; make that
// first call before any stream capture begins.  Sizes beyond the maximum are
// rejected with ORCTM_E_TOO_LARGE before anything is launched.
#include <mutex>
#include <string>

#include "../../include/orctm_gpu.h"
#include "common.cuh"
#include "ops.h"

namespace orctm {

namespace {

constexpr long long kNoAllocMaxCells = 1LL << 21;  // IE*JE*KE limit, 2,097,152 cells
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxCells];

std::mutex g_na_mutex;
double* g_na_ptr[kNoAllocMaxDevices] = {};

struct NaArgs {
  int IE, JE, KE;
  double dt, almzer, aulapts;
  const double *dvo, *ddpo, *weto, *di, *dzw, *dlxp, *dlyp, *dlxu, *dlyu, *dlxv, *dlyv, *zo;
};

// Fortran-layout accessors (p-points 1..IE x 1..JE, u-points 0..IE, v-points 0..JE)
__device__ __forceinline__ long long p3(const NaArgs& a, int i, int j, int k) {
  return ((long long)(k - 1) * a.JE + (j - 1)) * a.IE + (i - 1);
}
__device__ __forceinline__ long long p2(const NaArgs& a, int i, int j) {
  return (long long)(j - 1) * a.IE + (i - 1);
}
__device__ __forceinline__ long long u2(const NaArgs& a, int i, int j) {
  return (long long)(j - 1) * (a.IE + 1) + i;
}
__device__ __forceinline__ long long v2(const NaArgs& a, int i, int j) {
  return (long long)j * a.IE + (i - 1);
}

// implicit vertical diffusion (octdiff_base.f90:182-204, octdiff_ts.f90:294-324);
// columns outside the interior are copied
__global__ void k_na_vert(NaArgs a, const double* __restrict__ T, double* __restrict__ O) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int IE = a.IE, JE = a.JE, KE = a.KE;
  if (i > IE || j > JE) return;
  if (!(i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1)) {
    for (int K = 1; K <= KE; ++K) O[p3(a, i, j, K)] = T[p3(a, i, j, K)];
    return;
  }
  double t1[kMaxKe], t2[kMaxKe], t3[kMaxKe];
  const double zo = a.zo[p2(a, i, j)];
  for (int K = 1; K <= KE; ++K) {
    const double zzsurf = K == 1 ? 1. : 0.;
    const double den = a.ddpo[p3(a, i, j, K)] + zzsurf * (zo) + a.almzer;
    t1[K - 1] = -a.dt * a.dvo[p3(a, i, j, K)] * a.weto[p3(a, i, j, K)] * a.di[K - 1] / den;
    t3[K - 1] = -a.dt * a.dvo[p3(a, i, j, K + 1)] * a.di[K] / den;
    t2[K - 1] = 1. - t1[K - 1] - t3[K - 1];
  }
  for (int K = 2; K <= KE; ++K) {
    const double m = t1[K - 1];
    t1[K - 2] = m / t2[K - 2];
    t2[K - 1] = t2[K - 1] - t3[K - 2] * m / t2[K - 2];
  }
  double prev = T[p3(a, i, j, 1)];
  O[p3(a, i, j, 1)] = prev;
  for (int K = 2; K <= KE; ++K) {
    prev = T[p3(a, i, j, K)] - t1[K - 2] * prev;
    O[p3(a, i, j, K)] = prev;
  }
  double nxt = O[p3(a, i, j, KE)] / t2[KE - 1];
  O[p3(a, i, j, KE)] = nxt;
  for (int l = KE - 1; l >= 1; --l) {
    nxt = (O[p3(a, i, j, l)] - t3[l - 1] * nxt) / t2[l - 1];
    O[p3(a, i, j, l)] = nxt;
  }
}

// masked Laplacian (octdiff_ts.f90:346-362); halo cells are written as 0
__global__ void k_na_lap(NaArgs a, const double* __restrict__ T, double* __restrict__ L1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int K = blockIdx.z + 1;
  const int IE = a.IE, JE = a.JE;
  if (i > IE || j > JE) return;
  double r = 0.0;
  if (i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1) {
    const double c = T[p3(a, i, j, K)];
    auto w = [&](int ii, int jj) { return a.weto[p3(a, ii, jj, K)]; };
    r = w(i, j) *
        ((w(i - 1, j) * (T[p3(a, i - 1, j, K)] - c) / a.dlxu[u2(a, i - 1, j)] +
          w(i + 1, j) * (T[p3(a, i + 1, j, K)] - c) / a.dlxu[u2(a, i, j)]) /
             a.dlxp[p2(a, i, j)] +
         (w(i, j - 1) * (T[p3(a, i, j - 1, K)] - c) / a.dlyv[v2(a, i, j - 1)] +
          w(i, j + 1) * (T[p3(a, i, j + 1, K)] - c) / a.dlyv[v2(a, i, j)]) /
             a.dlyp[p2(a, i, j)]);
  }
  L1[p3(a, i, j, K)] = r;
}

// biharmonic update (octdiff_ts.f90:369-399)
__global__ void k_na_bih(NaArgs a, const double* __restrict__ T, const double* __restrict__ L1,
                         double* __restrict__ O) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int K = blockIdx.z + 1;
  const int IE = a.IE, JE = a.JE;
  if (i > IE || j > JE) return;
  const double t = T[p3(a, i, j, K)];
  double r = t;
  if (i >= 2 && i <= IE - 1 && j >= 2 && j <= JE - 1) {
    auto w = [&](int ii, int jj) { return a.weto[p3(a, ii, jj, K)]; };
    auto aulx = [&](int ii, int jj) {
      const double x = a.dlxu[u2(a, ii, jj)];
      return a.aulapts * ((x * x) * (x * x));
    };
    auto auly = [&](int ii, int jj) {
      const double y = a.dlyv[v2(a, ii, jj)];
      return a.aulapts * ((y * y) * (y * y));
    };
    const double zzsurf = K == 1 ? 1. : 0.;
    const double c = L1[p3(a, i, j, K)];
    const double den = (a.ddpo[p3(a, i, j, K)] + a.almzer + zzsurf * (a.zo[p2(a, i, j)])) *
                       a.dlxp[p2(a, i, j)] * a.dlyp[p2(a, i, j)];
    r = t - (w(i, j) / den) * a.dzw[K - 1] *
                (w(i - 1, j) * aulx(i - 1, j) * a.dlyu[u2(a, i - 1, j)] *
                     (L1[p3(a, i - 1, j, K)] - c) / a.dlxu[u2(a, i - 1, j)] +
                 w(i + 1, j) * aulx(i, j) * a.dlyu[u2(a, i, j)] * (L1[p3(a, i + 1, j, K)] - c) /
                     a.dlxu[u2(a, i, j)] +
                 w(i, j - 1) * auly(i, j - 1) * a.dlxv[v2(a, i, j - 1)] *
                     (L1[p3(a, i, j - 1, K)] - c) / a.dlyv[v2(a, i, j - 1)] +
                 w(i, j + 1) * auly(i, j) * a.dlxv[v2(a, i, j)] * (L1[p3(a, i, j + 1, K)] - c) /
                     a.dlyv[v2(a, i, j)]);
  }
  O[p3(a, i, j, K)] = r;
}

// Device address of the scratch array on the current device.  The first call
// on a device looks it up (cudaGetSymbolAddress, with that device current).
// Later calls look it up again when their stream is not being captured, so
// an address cached before a cudaDeviceReset (which unloads the module and
// may place the array elsewhere) is not reused; a call on a capturing stream
// uses the cached address, so the first call on a device must come before
// any capture, and a device reset must be followed by one call outside a
// capture before the next capture.
int scratch_for_current_device(cudaStream_t s, double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e);
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_unbound_error("device ordinal beyond the no-allocation table");
    return ORCTM_E_ARG;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const bool capturing = cudaStreamIsCapturing(s, &cs) != cudaSuccess ||
                         cs != cudaStreamCaptureStatusNone;
  std::lock_guard<std::mutex> lk(g_na_mutex);
  if (!g_na_ptr[dev] || !capturing) {
    if (capturing) {
      set_unbound_error("the first call on a device must not be made under stream capture");
      return ORCTM_E_ARG;
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      const int st = cuda_status(e);
      set_unbound_error((std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e)).c_str());
      return st;
    }
    g_na_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_na_ptr[dev];
  return ORCTM_OK;
}

}  // namespace
}  // namespace orctm

using namespace orctm;

extern "C" int orctm_octdiff_noalloc(const orctm_octdiff_noalloc_args* in) {
  clear_unbound_errors();
  if (!in) {
    set_unbound_error("null argument block");
    return ORCTM_E_ARG;
  }
  const long long cells = (long long)in->ie * in->je * in->ke;
  if (in->ie < 3 || in->je < 3 || in->ke < 2 || in->ke > kMaxKe) {
    set_unbound_error("grid size out of range");
    return ORCTM_E_ARG;
  }
  if (cells > kNoAllocMaxCells) {
    set_unbound_error("IE*JE*KE exceeds the no-allocation limit of 2097152 cells");
    return ORCTM_E_TOO_LARGE;
  }
  const void* req[] = {in->tracer_in, in->tracer_out, in->dvo, in->ddpo, in->weto, in->di,
                       in->dzw, in->dlxp, in->dlyp, in->dlxu, in->dlyu, in->dlxv, in->dlyv,
                       in->zo};
  for (const void* p : req)
    if (!p) {
      set_unbound_error("missing device pointer");
      return ORCTM_E_ARG;
    }
  if (in->tracer_in == in->tracer_out) {
    set_unbound_error("tracer_in and tracer_out must be different buffers");
    return ORCTM_E_ARG;
  }
  if (in->ah00 > in->almzer) {
    set_unbound_error("harmonic tracer diffusion (AH00 > ALMZER) is not implemented");
    return ORCTM_E_UNSUPPORTED;
  }
  cudaStream_t s = static_cast<cudaStream_t>(in->stream);
  double* scratch = nullptr;
  int st = scratch_for_current_device(s, &scratch);
  if (st != ORCTM_OK) return st;
  double* vdiff = scratch;                     // vertically diffused tracer
  double* lap = scratch + kNoAllocMaxCells;    // first Laplacian T1O
  NaArgs a{in->ie, in->je, in->ke, in->dt, in->almzer, in->aulapts, in->dvo, in->ddpo, in->weto,
           in->di, in->dzw, in->dlxp, in->dlyp, in->dlxu, in->dlyu, in->dlxv, in->dlyv, in->zo};
  const dim3 bc(32, 2), b3(32, 4);
  const dim3 gc((in->ie + 31) / 32, (in->je + 1) / 2, 1);
  const dim3 g3((in->ie + 31) / 32, (in->je + 3) / 4, in->ke);
  const bool bih = in->aulapts > in->almzer;
  k_na_vert<<<gc, bc, 0, s>>>(a, in->tracer_in, bih ? vdiff : in->tracer_out);
  count_launch();
  if (bih) {
    k_na_lap<<<g3, b3, 0, s>>>(a, vdiff, lap);
    count_launch();
    k_na_bih<<<g3, b3, 0, s>>>(a, vdiff, lap, in->tracer_out);
    count_launch();
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e);
  return ORCTM_OK;
}
