// Handle, device memory, geometry compression, routine sequencing, Poisson
// solver driver and the extern "C" entry points of include/orctm_gpu.h.
//
// Device memory.  All 3D fields share one padded layout (common.cuh) and
// hence one buffer size, so buffers come from a single pool.  A field slot
// points at a reference-counted buffer; routines never update a field in
// place but write a fresh buffer and rebind the slot, which lets OCTIMF and
// the state rotation of OCVTOT_NH (UOO_1 <- UOO, WO <- WNO, ...) alias buffers
// instead of copying them.  The one exception, the open-boundary sponge,
// touches a few bands of UOO / VOE: it updates them in place when no other
// slot or pending copy holds the buffer, and copies the buffer first
// otherwise.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/orctm_gpu.h"
#include "common.cuh"
#include "ops.h"

namespace orctm {

static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void add_launches(long long n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

// text of the calling thread's last CUDA failure (orctm_last_error)
thread_local std::string g_cuda_error;

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return ORCTM_OK;
  g_cuda_error = std::string("CUDA error ") + std::to_string((int)e) + " (" + cudaGetErrorName(e) +
                 "): " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return ORCTM_E_NOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return ORCTM_E_NODEVICE;
  return ORCTM_E_CUDA;
}

namespace {

// text of the calling thread's last failure of a call made without a handle
// (orctm_create, orctm_octdiff_noalloc), returned by orctm_last_error(NULL)
thread_local std::string g_create_error;

// One stream-ordered memory pool per device, owned by the library.  Freed
// blocks stay reserved in the pool (release threshold: unlimited), so a
// handle created after another was destroyed reuses its memory without
// mapping new pages; orctm_trim_device_memory returns them to the driver.
std::mutex g_pool_mu;
cudaMemPool_t g_pools[256] = {};

int device_pool(int dev, cudaMemPool_t* out) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (dev < 0 || dev >= 256) return ORCTM_E_ARG;
  if (!g_pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t mp = nullptr;
    ORCTM_CUDA_OK(cudaMemPoolCreate(&mp, &props));
    unsigned long long thr = ~0ULL;
    ORCTM_CUDA_OK(cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr));
    g_pools[dev] = mp;
  }
  *out = g_pools[dev];
  return ORCTM_OK;
}

// Pinned host mirrors of the solver scalars come from slabs that are never
// freed: cudaFreeHost would wait for the whole device.
std::mutex g_pin_mu;
std::vector<SolverState*> g_pin_free;

SolverState* pinned_state_get() {
  std::lock_guard<std::mutex> lk(g_pin_mu);
  if (g_pin_free.empty()) {
    constexpr int kSlab = 64;
    SolverState* slab = nullptr;
    if (cudaMallocHost((void**)&slab, sizeof(SolverState) * kSlab) != cudaSuccess) return nullptr;
    for (int k = kSlab - 1; k >= 0; --k) g_pin_free.push_back(slab + k);
  }
  SolverState* s = g_pin_free.back();
  g_pin_free.pop_back();
  return s;
}

void pinned_state_put(SolverState* s) {
  std::lock_guard<std::mutex> lk(g_pin_mu);
  g_pin_free.push_back(s);
}

enum Kind { KP = 0, KU = 1, KV = 2, KW = 3, K2P = 4 };

constexpr int kNumFixed = ORCTM_F_THO;  // fields before the tracers
constexpr int kMaxTracers = 8;

Kind field_kind(int f) {
  switch (f) {
    case ORCTM_F_UOO: case ORCTM_F_UKO: case ORCTM_F_UOO_1: return KU;
    case ORCTM_F_VOE: case ORCTM_F_VKE: case ORCTM_F_VOE_1: return KV;
    case ORCTM_F_WNO: case ORCTM_F_WO: case ORCTM_F_WNO_1: case ORCTM_F_DVO: case ORCTM_F_AVO:
      return KW;
    case ORCTM_F_ZO: return K2P;
    default: return KP;
  }
}

}  // namespace

void set_unbound_error(const char* msg) { g_create_error = msg ? msg : ""; }
void clear_unbound_errors() {
  g_create_error.clear();
  g_cuda_error.clear();
}

}  // namespace orctm

using namespace orctm;

struct orctm_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaMemPool_t mempool = nullptr;  // the library's stream-ordered pool of this device
  size_t bytes = 0;                 // device bytes allocated by this handle
  Layout L{};
  Geo G{};
  PoissonGeo P{};
  int ntr = 2;
  std::string err;
  std::vector<double> tiestu, tiestw;  // level depths (BELEG), the EXTRA level codes
  std::vector<double> dzw;             // layer thicknesses DZW

  // geometry / tables (device)
  std::vector<void*> owned;  // freed at destroy
  // pool of 3D buffers (double, L.n3() elements)
  std::vector<double*> free_;
  std::unordered_map<double*, int> refs;
  std::vector<double*> slot;  // per field id
  double* zo = nullptr;       // 2D

  // solver
  int solver_mode = ORCTM_SOLVER_FP64;
  double rtol = 1e-10;
  int maxit = 5000;
  double* b = nullptr;
  double *xs = nullptr, *r = nullptr, *z = nullptr, *p0 = nullptr, *p1 = nullptr, *q = nullptr;
  double *d = nullptr, *rw = nullptr;
  float *r32b = nullptr, *r32 = nullptr, *z32 = nullptr, *p32a = nullptr, *p32b = nullptr,
        *q32 = nullptr, *d32 = nullptr;
  SolverState* S = nullptr;
  SolverState* S_tune = nullptr;  // scratch scalars for the autotuner
  SolverState* S_tune0 = nullptr; // their initial value
  double* partials = nullptr;
  // kernel variants per precision (0 FP64, 1 FP32); -1 = not chosen yet
  int col_var[2] = {-1, -1}, spmv_var[2] = {-1, -1};
  int force_col = -1, force_spmv = -1;  // orctm_set_tuning
  // asynchronous copies (orctm_upload_async / orctm_download_async): a copy
  // stream, per-field "upload landed" events the compute stream waits for
  // before a routine reads the field, buffers held until their download ends,
  // and the outputs orctm_step_hotpath downloads as soon as they are final
  cudaStream_t cstream = nullptr;
  cudaEvent_t field_ready[64] = {};
  bool pending[64] = {};
  std::vector<double*> held;
  std::vector<cudaEvent_t> copy_events;
  struct StepOut { int field; double* host; size_t n; };
  std::vector<StepOut> step_out;
  // open-boundary tides and sponge (orctm_set_obc): launch arguments per
  // variable (z, u, v), the constants in one device buffer
  bool obc_ready = false;
  ObcArgs obc[3] = {};
  double* obc_buf = nullptr;
  size_t obc_cap = 0;
  // T/S boundary climatology records (orctm_set_obc_ts) of tracers 0 and 1
  bool obc_ts_ready[2] = {false, false};
  ObcArgs obc_ts[2] = {};
  double* obc_ts_buf[2] = {nullptr, nullptr};
  size_t obc_ts_cap[2] = {0, 0};
  // the exponential sponge's rate tables (orctm_set_obc_sponge_exp); SAO's
  // south band has its own (mo_obcs.f90:2976)
  double* obc_exp_buf = nullptr;
  size_t obc_exp_cap = 0;
  const double* obc_exp_sao_south = nullptr;
  // barotropic solve (orctm_set_barotropic): its constants, its 2D device
  // fields and TRONEU's SOR sweeps captured once as a graph
  bool baro_ready = false;
  BaroArgs baro{};
  BaroFields bf{};
  cudaGraphExec_t sor_graph = nullptr;
  WindFields wind{};  // OCWIND's forcing (orctm_ocwind), allocated on first use
  bool wind_ready = false;
  // OCTHER (orctm_set_thermo), OCMODMOM's Coriolis factors
  // (orctm_set_coriolis), UK1O / VK1E and the scratch of OCMODMOM and OCCLIT
  bool thermo_ready = false, cor_ready = false;
  ThermoArgs th{};
  ThermoFields tf{};
  CorFields cf{};
  double *uk1o = nullptr, *vk1e = nullptr;
  double *occ_wpo = nullptr, *occ_t1o = nullptr, *occ_bruva = nullptr, *occ_contrij = nullptr;
  double* occ_contra = nullptr;  // device scalar
  double* h_contra = nullptr;    // its page-locked mirror
  double* trotest_buf = nullptr;  // orctm_trotest's scratch, allocated on first use
  // replayed chunk of PCG iterations per precision and the variants it holds
  cudaGraphExec_t pcg_graph[2] = {nullptr, nullptr};
  int pcg_graph_key[2][2] = {{-1, -1}, {-1, -1}};
  SolverState* hS = nullptr;  // pinned mirror
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t tm0 = nullptr, tm1 = nullptr;  // orctm_timer_start / _stop

  // optional per-launcher device timing (orctm_set_profiling)
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_pairs[ORCTM_PROF_KINDS];
  double prof_ms[ORCTM_PROF_KINDS] = {};
  long long prof_n[ORCTM_PROF_KINDS] = {};
  cudaEvent_t get_event() {
    if (!ev_pool.empty()) {
      cudaEvent_t e = ev_pool.back();
      ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  void prof_begin(cudaEvent_t* e0) {
    *e0 = nullptr;
    if (!prof) return;
    *e0 = get_event();
    cudaEventRecord(*e0, stream);
  }
  void prof_end(int kind, cudaEvent_t e0) {
    if (!prof || !e0) return;
    cudaEvent_t e1 = get_event();
    cudaEventRecord(e1, stream);
    prof_pairs[kind].push_back({e0, e1});
    if (prof_pairs[kind].size() > 4096) prof_flush();
  }
  void prof_flush() {
    cudaStreamSynchronize(stream);
    for (int k = 0; k < ORCTM_PROF_KINDS; ++k) {
      for (auto& pr : prof_pairs[k]) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, pr.first, pr.second);
        prof_ms[k] += ms;
        prof_n[k] += 1;
        ev_pool.push_back(pr.first);
        ev_pool.push_back(pr.second);
      }
      prof_pairs[k].clear();
    }
  }

  // Every device array is allocated with a zero-filled guard zone of one
  // plane plus two rows of elements on each side.  Stencils that evaluate a
  // neighbour outside an array's index range (a value a zero mask or
  // coefficient then discards) read the guard, never memory of another
  // allocation, so results never depend on other instances' data.
  std::unordered_map<void*, void*> base_of;  // user pointer -> allocation
  size_t guard_elems() const { return (size_t)L.plane + 2 * (size_t)L.P + 64; }
  int guarded_alloc(void** out, size_t elem, size_t n) {
    const size_t g = guard_elems() * elem;
    const size_t total = n * elem + 2 * g;
    char* base = nullptr;
    ORCTM_CUDA_OK(cudaMallocFromPoolAsync((void**)&base, total, mempool, stream));
#ifdef ORCTM_GUARD_NAN
    // diagnostic build: guards hold NaN (bytes 0xFF), so any read of a guard
    // that reaches a result shows up as NaN
    ORCTM_CUDA_OK(cudaMemsetAsync(base, 0xFF, total, stream));
    ORCTM_CUDA_OK(cudaMemsetAsync(base + g, 0, n * elem, stream));
#else
    ORCTM_CUDA_OK(cudaMemsetAsync(base, 0, total, stream));
#endif
    bytes += total;
    *out = base + g;
    base_of[*out] = base;
    return ORCTM_OK;
  }
  void* base(void* p) const {
    auto it = base_of.find(p);
    return it == base_of.end() ? p : it->second;
  }

  // ---------------------------------------------------------------- pool
  int alloc(double** out) {
    if (!free_.empty()) {
      *out = free_.back();
      free_.pop_back();
      refs[*out] = 1;
      return ORCTM_OK;
    }
    double* p = nullptr;
    int st;
    if ((st = guarded_alloc((void**)&p, sizeof(double), (size_t)L.n3()))) return st;
    refs[p] = 1;
    *out = p;
    return ORCTM_OK;
  }
  void unref(double* p) {
    if (!p) return;
    auto it = refs.find(p);
    if (it == refs.end()) return;
    if (--it->second == 0) {
      refs.erase(it);
      free_.push_back(p);
    }
  }
  void bind(int f, double* p) {  // slot takes ownership of one reference
    unref(slot[f]);
    slot[f] = p;
  }
  void alias(int dst, int src) {
    double* p = slot[src];
    refs[p]++;
    unref(slot[dst]);
    slot[dst] = p;
  }
  int fail(int st, const char* msg) {
    err = msg;
    return st;
  }
  template <typename T>
  int dev_alloc(T** p, size_t n) {
    int st;
    if ((st = guarded_alloc((void**)p, sizeof(T), std::max<size_t>(n, 1)))) return st;
    owned.push_back(*p);
    return ORCTM_OK;
  }
};

namespace {

// wraps one launcher call in device events when profiling is on
#define PROF(h, kind, call)        \
  do {                             \
    cudaEvent_t e0_;               \
    (h)->prof_begin(&e0_);         \
    call;                          \
    (h)->prof_end((kind), e0_);    \
  } while (0)

// field extent in the reference's host layout
void extent(const orctm_handle* h, int f, int& i0, int& ni, int& j0, int& nj, int& nk) {
  const int IE = h->L.ie, JE = h->L.je, KE = h->L.ke;
  i0 = 1; ni = IE; j0 = 1; nj = JE; nk = KE;
  switch (field_kind(f)) {
    case KU: i0 = 0; ni = IE + 1; break;
    case KV: j0 = 0; nj = JE + 1; break;
    case KW: nk = KE + 1; break;
    case K2P: nk = 1; break;
    default: break;
  }
}

// Geometry checks and compression -------------------------------------------
struct Ix {
  int IE, JE, KE;
  size_t p3(int i, int j, int k) const { return ((size_t)(k - 1) * JE + (j - 1)) * IE + (i - 1); }
  size_t u3(int i, int j, int k) const { return ((size_t)(k - 1) * JE + (j - 1)) * (IE + 1) + i; }
  size_t v3(int i, int j, int k) const { return ((size_t)(k - 1) * (JE + 1) + j) * IE + (i - 1); }
  size_t p2(int i, int j) const { return (size_t)(j - 1) * IE + (i - 1); }
  size_t u2(int i, int j) const { return (size_t)(j - 1) * (IE + 1) + i; }
  size_t v2(int i, int j) const { return (size_t)j * IE + (i - 1); }
};

// Finds kb (wet levels) and the bottom thickness of one column and checks the
// column has the BODEN form: thickness DZW(K) above kb, bot at kb, 0 below,
// mask 1 down to kb and 0 below.
bool compress_column(const double* dd, const double* mk, size_t stride, const double* dzw, int KE,
                     int& kb, double& bot) {
  kb = 0;
  while (kb < KE && dd[stride * kb] > 0.) ++kb;
  bot = kb > 0 ? dd[stride * (kb - 1)] : 0.0;
  for (int K = 1; K <= KE; ++K) {
    const double want = K < kb ? dzw[K - 1] : (K == kb ? bot : 0.0);
    if (dd[stride * (K - 1)] != want) return false;
    if (mk[stride * (K - 1)] != (K <= kb ? 1.0 : 0.0)) return false;
  }
  return true;
}

// ZW(K) of compute_matrix (mo_petsc.f90:557-583) for one column
double zw_ref(const double* ddcol, const double* dzw, int KE, int K) {
  double dd;
  if (K == 1) {
    dd = ddcol[0] == 0 ? dzw[0] / 2.0 : ddcol[0] / 2.0;
  } else if (K == KE + 1) {
    dd = ddcol[KE - 1] == 0 ? dzw[KE - 1] : ddcol[KE - 1];
  } else {
    if (ddcol[K - 2] == 0)
      dd = (dzw[K - 1] + dzw[K - 2]) / 2.0;
    else if (ddcol[K - 1] == 0)
      dd = ddcol[K - 2];
    else
      dd = (ddcol[K - 2] + ddcol[K - 1]) / 2.0;
  }
  return 1.0 / dd;
}

int upload_2d(orctm_handle* h, double* dst, const double* src, int i0, int ni, int j0, int nj) {
  ORCTM_CUDA_OK(cudaMemcpy2DAsync(dst + h->L.at2(i0, j0), sizeof(double) * h->L.P, src,
                                  sizeof(double) * ni, sizeof(double) * ni, nj,
                                  cudaMemcpyHostToDevice, h->stream));
  return ORCTM_OK;
}

int setup(orctm_handle* h, const orctm_desc* d) {
  const int IE = d->ie, JE = d->je, KE = d->ke;
  const Ix x{IE, JE, KE};
  Layout& L = h->L;
  L.ie = IE; L.je = JE; L.ke = KE;
  L.P = ((IE + 1) + 31) / 32 * 32;
  L.JN = JE + 1;
  L.plane = L.P * L.JN;  // below 2^31: checked by orctm_create
  h->ntr = d->ntracers;
  // TIESTW / TIESTU of BELEG (beleg.f90:87-139): interface and layer-centre depths
  h->tiestw.assign(KE + 1, 0.0);
  h->tiestu.assign(KE + 1, 0.0);
  for (int k = 1; k <= KE; ++k) h->tiestw[k] = h->tiestw[k - 1] + d->dzw[k - 1];
  h->tiestu[0] = 0.5 * d->dzw[0];
  for (int k = 2; k <= KE; ++k) h->tiestu[k - 1] = 0.5 * (h->tiestw[k] + h->tiestw[k - 1]);
  h->tiestu[KE] = 9000.;
  h->dzw.assign(d->dzw, d->dzw + KE);
  Geo& G = h->G;
  G.L = L;
  G.dt = d->dt;
  G.dti = 1. / d->dt;
  G.almzer = d->almzer;
  G.aulapts = d->aulapts;
  G.aulapuv = d->aulapuv;
  G.minvalue = d->dzw[0] / 10.0 < 1.0 ? d->dzw[0] / 10.0 : 1.0;  // MIN(1.0, DZW(1)/10.0)
  G.ob_w = d->ob_west; G.ob_e = d->ob_east; G.ob_n = d->ob_north; G.ob_s = d->ob_south;

  // compressed columns
  const size_t n2 = (size_t)L.plane;
  std::vector<int> kbp(n2, 0), kbu(n2, 0), kbv(n2, 0);
  std::vector<double> botp(n2, 0.), botu(n2, 0.), botv(n2, 0.);
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      const size_t s = L.at2(i, j);
      if (!compress_column(d->ddpo + x.p3(i, j, 1), d->weto + x.p3(i, j, 1), (size_t)IE * JE, d->dzw,
                           KE, kbp[s], botp[s]))
        return h->fail(ORCTM_E_GEOMETRY, "DDPO/WETO column is not of the BODEN form");
    }
  for (int j = 1; j <= JE; ++j)
    for (int i = 0; i <= IE; ++i) {
      const size_t s = L.at2(i, j);
      if (!compress_column(d->dduo + x.u3(i, j, 1), d->amsuo + x.u3(i, j, 1), (size_t)(IE + 1) * JE,
                           d->dzw, KE, kbu[s], botu[s]))
        return h->fail(ORCTM_E_GEOMETRY, "DDUO/AMSUO column is not of the BODEN form");
    }
  for (int j = 0; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      const size_t s = L.at2(i, j);
      if (!compress_column(d->ddue + x.v3(i, j, 1), d->amsue + x.v3(i, j, 1), (size_t)IE * (JE + 1),
                           d->dzw, KE, kbv[s], botv[s]))
        return h->fail(ORCTM_E_GEOMETRY, "DDUE/AMSUE column is not of the BODEN form");
    }
  int* dk = nullptr;
  double* db = nullptr;
  int st;
  auto up_col = [&](ColGeo& cg, const std::vector<int>& kb, const std::vector<double>& bot) -> int {
    int s2;
    if ((s2 = h->dev_alloc(&dk, n2))) return s2;
    if ((s2 = h->dev_alloc(&db, n2))) return s2;
    ORCTM_CUDA_OK(cudaMemcpyAsync(dk, kb.data(), sizeof(int) * n2, cudaMemcpyHostToDevice, h->stream));
    ORCTM_CUDA_OK(cudaMemcpyAsync(db, bot.data(), sizeof(double) * n2, cudaMemcpyHostToDevice, h->stream));
    cg.kb = dk;
    cg.bot = db;
    return ORCTM_OK;
  };
  if ((st = up_col(G.gp, kbp, botp))) return st;
  if ((st = up_col(G.gu, kbu, botu))) return st;
  if ((st = up_col(G.gv, kbv, botv))) return st;

  // 1D tables
  double *ddzw, *ddi;
  if ((st = h->dev_alloc(&ddzw, KE))) return st;
  if ((st = h->dev_alloc(&ddi, KE + 1))) return st;
  ORCTM_CUDA_OK(cudaMemcpyAsync(ddzw, d->dzw, sizeof(double) * KE, cudaMemcpyHostToDevice, h->stream));
  ORCTM_CUDA_OK(cudaMemcpyAsync(ddi, d->di, sizeof(double) * (KE + 1), cudaMemcpyHostToDevice, h->stream));
  G.dzw = ddzw;
  G.di = ddi;

  // 2D metrics into the padded plane
  auto up2 = [&](const double*& dst, const double* src, Kind k) -> int {
    double* p;
    int s2;
    if ((s2 = h->dev_alloc(&p, n2))) return s2;
    const int i0 = k == KU ? 0 : 1, ni = k == KU ? IE + 1 : IE;
    const int j0 = k == KV ? 0 : 1, nj = k == KV ? JE + 1 : JE;
    if ((s2 = upload_2d(h, p, src, i0, ni, j0, nj))) return s2;
    dst = p;
    return ORCTM_OK;
  };
  if ((st = up2(G.dlxp, d->dlxp, KP)) || (st = up2(G.dlyp, d->dlyp, KP)) ||
      (st = up2(G.dtdxpo, d->dtdxpo, KP)) || (st = up2(G.dtdyo, d->dtdyo, KP)) ||
      (st = up2(G.dlxu, d->dlxu, KU)) || (st = up2(G.dlyu, d->dlyu, KU)) ||
      (st = up2(G.dtdxuo, d->dtdxuo, KU)) || (st = up2(G.dlxv, d->dlxv, KV)) ||
      (st = up2(G.dlyv, d->dlyv, KV)) || (st = up2(G.dpye, d->dpye, KV)))
    return st;

  // biharmonic coefficients (octdiff_base.f90:210-219, ocvisc.f90:286-327)
  {
    auto pow4 = [](double x) { return (x * x) * (x * x); };
    auto fmx = [](double a, double b) { return a > b ? a : b; };
    const double mv = G.minvalue, A = d->aulapuv, At = d->aulapts;
    std::vector<double> aulx(n2, 0.), auly(n2, 0.), aulux(n2, 0.), auluy(n2, 0.), aulvx(n2, 0.),
        aulvy(n2, 0.), aulwx(n2, 0.), aulwy(n2, 0.), dlypsi(n2, 0.), dlxpsi(n2, 0.);
    for (int j = 1; j <= JE; ++j) {
      for (int i = 1; i <= IE - 1; ++i)
        dlypsi[L.at2(i, j)] = 0.5 * (d->dlyv[x.v2(i, j)] + d->dlyv[x.v2(i + 1, j)]);
      dlypsi[L.at2(0, j)] = d->dlyv[x.v2(1, j)];
      dlypsi[L.at2(IE, j)] = d->dlyv[x.v2(IE, j)];
    }
    for (int i = 1; i <= IE; ++i) {
      for (int j = 1; j <= JE - 1; ++j)
        dlxpsi[L.at2(i, j)] = 0.5 * (d->dlxu[x.u2(i, j)] + d->dlxu[x.u2(i, j + 1)]);
      dlxpsi[L.at2(i, 0)] = d->dlxu[x.u2(i, 1)];
      dlxpsi[L.at2(i, JE)] = d->dlxu[x.u2(i, JE)];
    }
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {
        const size_t s = L.at2(i, j);
        aulx[s] = At * pow4(d->dlxu[x.u2(i, j)]);
        auly[s] = At * pow4(d->dlyv[x.v2(i, j)]);
        aulux[s] = A * pow4(fmx(d->dlxp[x.p2(i, j)], mv));
        auluy[s] = A * pow4(fmx(mv, dlypsi[s]));
        aulvy[s] = A * pow4(fmx(mv, d->dlyp[x.p2(i, j)]));
        aulvx[s] = A * pow4(fmx(dlxpsi[s], mv));
        aulwx[s] = A * pow4(fmx(d->dlxu[x.u2(i, j)], mv));
        aulwy[s] = A * pow4(fmx(d->dlyv[x.v2(i, j)], mv));
      }
    auto upg = [&](const double*& dst, const std::vector<double>& v) -> int {
      double* q;
      int s2;
      if ((s2 = h->dev_alloc(&q, v.size()))) return s2;
      ORCTM_CUDA_OK(cudaMemcpyAsync(q, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, h->stream));
      dst = q;
      return ORCTM_OK;
    };
    if ((st = upg(G.aulx, aulx)) || (st = upg(G.auly, auly)) || (st = upg(G.aulux, aulux)) ||
        (st = upg(G.auluy, auluy)) || (st = upg(G.aulvx, aulvx)) || (st = upg(G.aulvy, aulvy)) ||
        (st = upg(G.aulwx, aulwx)) || (st = upg(G.aulwy, aulwy)) || (st = upg(G.dlypsi, dlypsi)) ||
        (st = upg(G.dlxpsi, dlxpsi)))
      return st;

    // reciprocal metrics over each staggering's own index range
    auto rec = [](double v) { return v != 0.0 ? 1.0 / v : 0.0; };
    std::vector<double> rdlxp(n2, 0.), rdlyp(n2, 0.), rdlxu(n2, 0.), rdlyu(n2, 0.),
        rdlxv(n2, 0.), rdlyv(n2, 0.), rdlxpsi(n2, 0.), rdlypsi(n2, 0.), tfx(n2, 0.), tfy(n2, 0.),
        ugx(n2, 0.), ugy(n2, 0.), vgx(n2, 0.), vgy(n2, 0.), wgx(n2, 0.), wgy(n2, 0.),
        rareau(n2, 0.), rareav(n2, 0.), rareap(n2, 0.);
    for (int j = 1; j <= JE; ++j)
      for (int i = 0; i <= IE; ++i) {  // u-points
        const size_t s = L.at2(i, j);
        const double xu = d->dlxu[x.u2(i, j)], yu = d->dlyu[x.u2(i, j)];
        rdlxu[s] = rec(xu);
        rdlyu[s] = rec(yu);
        rdlypsi[s] = rec(dlypsi[s]);
        rareau[s] = rec(xu * yu);
      }
    for (int j = 0; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {  // v-points
        const size_t s = L.at2(i, j);
        const double xv = d->dlxv[x.v2(i, j)], yv = d->dlyv[x.v2(i, j)];
        rdlxv[s] = rec(xv);
        rdlyv[s] = rec(yv);
        rdlxpsi[s] = rec(dlxpsi[s]);
        rareav[s] = rec(xv * yv);
      }
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i) {  // p-points and the face coefficients
        const size_t s = L.at2(i, j);
        const double xp = d->dlxp[x.p2(i, j)], yp = d->dlyp[x.p2(i, j)];
        rdlxp[s] = rec(xp);
        rdlyp[s] = rec(yp);
        rareap[s] = rec(xp * yp);
        tfx[s] = aulx[s] * d->dlyu[x.u2(i, j)] * rec(d->dlxu[x.u2(i, j)]);
        tfy[s] = auly[s] * d->dlxv[x.v2(i, j)] * rec(d->dlyv[x.v2(i, j)]);
        ugx[s] = aulux[s] * yp * rec(xp);
        ugy[s] = auluy[s] * dlxpsi[s] * rec(dlypsi[s]);
        vgx[s] = aulvx[s] * dlypsi[s] * rec(dlxpsi[s]);
        vgy[s] = aulvy[s] * xp * rec(yp);
        wgx[s] = aulwx[s] * d->dlyu[x.u2(i, j)] * rec(d->dlxu[x.u2(i, j)]);
        wgy[s] = aulwy[s] * d->dlxv[x.v2(i, j)] * rec(d->dlyv[x.v2(i, j)]);
      }
    if ((st = upg(G.rdlxp, rdlxp)) || (st = upg(G.rdlyp, rdlyp)) || (st = upg(G.rdlxu, rdlxu)) ||
        (st = upg(G.rdlyu, rdlyu)) || (st = upg(G.rdlxv, rdlxv)) || (st = upg(G.rdlyv, rdlyv)) ||
        (st = upg(G.rdlxpsi, rdlxpsi)) || (st = upg(G.rdlypsi, rdlypsi)) ||
        (st = upg(G.tfx, tfx)) || (st = upg(G.tfy, tfy)) || (st = upg(G.ugx, ugx)) ||
        (st = upg(G.ugy, ugy)) || (st = upg(G.vgx, vgx)) || (st = upg(G.vgy, vgy)) ||
        (st = upg(G.wgx, wgx)) || (st = upg(G.wgy, wgy)) || (st = upg(G.rareau, rareau)) ||
        (st = upg(G.rareav, rareav)) || (st = upg(G.rareap, rareap)))
      return st;
  }

  // Poisson tables (mo_petsc.f90:557-599)
  std::vector<double> xu(n2, 0.), xp(n2, 0.), yv(n2, 0.), yp(n2, 0.);
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      const size_t s = L.at2(i, j);
      xu[s] = 1.0 / d->dlxu[x.u2(i, j)];
      xp[s] = 1.0 / d->dlxp[x.p2(i, j)];
      yv[s] = 1.0 / d->dlyv[x.v2(i, j)];
      yp[s] = 1.0 / d->dlyp[x.p2(i, j)];
    }
  std::vector<double> zwn(KE + 1), zpn(KE);
  {
    std::vector<double> zero(KE, 0.0);
    for (int K = 1; K <= KE + 1; ++K) zwn[K - 1] = zw_ref(zero.data(), d->dzw, KE, K);
    // nominal wet column: DDPO(K) = DZW(K) everywhere except the last level
    std::vector<double> full(d->dzw, d->dzw + KE);
    for (int K = 2; K <= KE; ++K) zwn[K - 1] = zw_ref(full.data(), d->dzw, KE, K);
    zwn[0] = zw_ref(full.data(), d->dzw, KE, 1);
    for (int K = 1; K <= KE; ++K) zpn[K - 1] = 1.0 / ((1.0 / zwn[K - 1] + 1.0 / zwn[K]) / 2.0);
  }
  std::vector<double> izn(KE);
  for (int K = 1; K <= KE; ++K) izn[K - 1] = (1.0 / zwn[K - 1] + 1.0 / zwn[K]) / 2.0;
  std::vector<double> zwa(n2, 0.), zwb(n2, 0.), zpa(n2, 0.), zpb(n2, 0.), zpc(n2, 0.);
  std::vector<double> iza(n2, 0.), izb(n2, 0.), izc(n2, 0.);
  std::vector<double> col(KE), zw(KE + 1), zp(KE), iz(KE);
  for (int j = 1; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      const size_t s = L.at2(i, j);
      for (int K = 1; K <= KE; ++K) col[K - 1] = d->ddpo[x.p3(i, j, K)];
      for (int K = 1; K <= KE + 1; ++K) zw[K - 1] = zw_ref(col.data(), d->dzw, KE, K);
      for (int K = 1; K <= KE; ++K) {
        iz[K - 1] = (1.0 / zw[K - 1] + 1.0 / zw[K]) / 2.0;  // dddpo, mo_petsc.f90:588
        zp[K - 1] = 1.0 / iz[K - 1];
      }
      const int kb = kbp[s];
      if (kb >= 1) {
        zwa[s] = zw[kb - 1];
        zwb[s] = zw[kb];
        if (kb >= 2) { zpa[s] = zp[kb - 2]; iza[s] = iz[kb - 2]; }
        zpb[s] = zp[kb - 1];
        izb[s] = iz[kb - 1];
        if (kb + 1 <= KE) { zpc[s] = zp[kb]; izc[s] = iz[kb]; }
      }
      // the selection used on the device must reproduce every level exactly
      for (int K = 1; K <= KE + 1; ++K) {
        double sel = zwn[K - 1];
        if (kb >= 1 && K == kb) sel = zwa[s];
        if (kb >= 1 && K == kb + 1) sel = zwb[s];
        if (sel != zw[K - 1]) return h->fail(ORCTM_E_GEOMETRY, "ZW table selection mismatch");
      }
      for (int K = 1; K <= KE; ++K) {
        double sel = zpn[K - 1];
        if (kb >= 1 && K == kb - 1) sel = zpa[s];
        if (kb >= 1 && K == kb) sel = zpb[s];
        if (kb >= 1 && K == kb + 1) sel = zpc[s];
        if (sel != zp[K - 1]) return h->fail(ORCTM_E_GEOMETRY, "ZP table selection mismatch");
        double isel = izn[K - 1];
        if (kb >= 1 && K == kb - 1) isel = iza[s];
        if (kb >= 1 && K == kb) isel = izb[s];
        if (kb >= 1 && K == kb + 1) isel = izc[s];
        if (isel != iz[K - 1]) return h->fail(ORCTM_E_GEOMETRY, "1/ZP table selection mismatch");
      }
    }
  auto upv = [&](const double*& dst, const std::vector<double>& v) -> int {
    double* p;
    int s2;
    if ((s2 = h->dev_alloc(&p, v.size()))) return s2;
    ORCTM_CUDA_OK(cudaMemcpyAsync(p, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, h->stream));
    dst = p;
    return ORCTM_OK;
  };
  PoissonGeo& P = h->P;
  if ((st = upv(P.xu, xu)) || (st = upv(P.xp, xp)) || (st = upv(P.yv, yv)) ||
      (st = upv(P.yp, yp)) || (st = upv(P.zwa, zwa)) || (st = upv(P.zwb, zwb)) ||
      (st = upv(P.zpa, zpa)) || (st = upv(P.zpb, zpb)) || (st = upv(P.zpc, zpc)) ||
      (st = upv(P.zwn, zwn)) || (st = upv(P.zpn, zpn)) || (st = upv(P.iza, iza)) ||
      (st = upv(P.izb, izb)) || (st = upv(P.izc, izc)) || (st = upv(P.izn, izn)))
    return st;

  // state slots
  h->slot.assign(kNumFixed + h->ntr, nullptr);
  for (int f = 0; f < kNumFixed + h->ntr; ++f) {
    if (f == ORCTM_F_ZO) continue;
    double* p;
    if ((st = h->alloc(&p))) return st;
    h->slot[f] = p;
  }
  if ((st = h->dev_alloc(&h->zo, n2))) return st;

  // pivots of the preconditioner (the operator is constant: factorise once)
  {
    double* d64;
    float* d32;
    if ((st = h->dev_alloc(&d64, (size_t)L.n3())) || (st = h->dev_alloc(&d32, (size_t)L.n3())))
      return st;
    P.dinv64 = d64;
    P.dinv32 = d32;
    ORCTM_CUDA_OK(pcg_prepare_device());
    launch_factor(G, P, d64, d32, h->stream);
    ORCTM_CUDA_OK(cudaGetLastError());
  }
  // solver scalars
  const int maxb = (int)solver_max_blocks(G);
  if ((st = h->dev_alloc(&h->S, 1))) return st;
  if ((st = h->dev_alloc(&h->partials, (size_t)4 * maxb))) return st;
  if (!(h->hS = pinned_state_get())) return h->fail(ORCTM_E_NOMEM, "pinned host memory exhausted");
  std::memset(h->hS, 0, sizeof(SolverState));
  h->hS->max_blocks = maxb;
  h->hS->rows = G.L.je - 2;
  h->hS->partials = h->partials;
  ORCTM_CUDA_OK(cudaMemcpyAsync(h->S, h->hS, sizeof(SolverState), cudaMemcpyHostToDevice, h->stream));
  ORCTM_CUDA_OK(cudaEventCreate(&h->ev0));
  ORCTM_CUDA_OK(cudaEventCreate(&h->ev1));
  ORCTM_CUDA_OK(cudaEventCreate(&h->tm0));
  ORCTM_CUDA_OK(cudaEventCreate(&h->tm1));
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  return ORCTM_OK;
}

int ensure_solver_buffers(orctm_handle* h) {
  int st;
  const size_t n = (size_t)h->L.n3();
  if (!h->b) {
    if ((st = h->dev_alloc(&h->b, n)) || (st = h->dev_alloc(&h->xs, n)) ||
        (st = h->dev_alloc(&h->r, n)) || (st = h->dev_alloc(&h->z, n)) ||
        (st = h->dev_alloc(&h->p0, n)) || (st = h->dev_alloc(&h->p1, n)) ||
        (st = h->dev_alloc(&h->q, n)) || (st = h->dev_alloc(&h->d, n)) ||
        (st = h->dev_alloc(&h->rw, n)))
      return st;
  }
  if (h->solver_mode == ORCTM_SOLVER_FP32_REFINED && !h->r32) {
    if ((st = h->dev_alloc(&h->r32b, n)) || (st = h->dev_alloc(&h->r32, n)) ||
        (st = h->dev_alloc(&h->z32, n)) || (st = h->dev_alloc(&h->p32a, n)) ||
        (st = h->dev_alloc(&h->p32b, n)) || (st = h->dev_alloc(&h->q32, n)) ||
        (st = h->dev_alloc(&h->d32, n)))
      return st;
  }
  return ORCTM_OK;
}

int read_state(orctm_handle* h) {
  ORCTM_CUDA_OK(cudaMemcpyAsync(h->hS, h->S, sizeof(SolverState), cudaMemcpyDeviceToHost, h->stream));
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  return ORCTM_OK;
}

// Eight PCG iterations (stencil + column kernel each) are captured once per
// precision into a CUDA graph and replayed between convergence checks: the
// vectors, the solver scalars and the kernel variants of a handle are fixed,
// and after an even number of iterations the two p buffers are back in their
// starting roles, so every chunk from iteration 8 on issues the same launches.
// The graph is rebuilt when the variants change; with profiling on, the
// launches go one by one (they are bracketed by events).
constexpr int kPcgChunk = 8;

template <typename T, typename TX>
int pcg_loop_graph(orctm_handle* h, const T* b, TX* x, T* r, T* z, T* pa, T* pb, T* q,
                   cudaGraphExec_t* out) {
  const int pr = sizeof(T) == 4;
  const int cv = h->col_var[pr], sv = h->spmv_var[pr];
  if (h->pcg_graph[pr] && h->pcg_graph_key[pr][0] == cv && h->pcg_graph_key[pr][1] == sv) {
    *out = h->pcg_graph[pr];
    return ORCTM_OK;
  }
  if (h->pcg_graph[pr]) {
    cudaGraphExecDestroy(h->pcg_graph[pr]);
    h->pcg_graph[pr] = nullptr;
  }
  // a graph holding one conditional while node; its body is a chunk of
  // kPcgChunk iterations ended by the kernel that sets the loop condition
  cudaGraph_t g = nullptr;
  ORCTM_CUDA_OK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle hc;
  cudaError_t e = cudaGraphConditionalHandleCreate(&hc, g, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = hc;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return cuda_status(e);
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  const unsigned long long before = launch_count();
  e = cudaStreamBeginCaptureToGraph(h->stream, body, nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return cuda_status(e);
  }
  cudaError_t e0 = cudaSuccess;
  T *pc = pa, *pn = pb;
  for (int k = 0; k < kPcgChunk; ++k) {
    if (e0 == cudaSuccess) e0 = launch_pcg_spmv<T>(h->G, h->P, h->S, z, pc, pn, q, 0, sv, h->stream);
    launch_pcg_col<T, TX>(h->G, h->P, h->S, 2, b, x, r, pn, q, z, cv, h->stream);
    std::swap(pc, pn);
  }
  launch_pcg_continue(hc, h->S, kPcgChunk, h->stream);
  const cudaError_t e1 = cudaStreamEndCapture(h->stream, &body);
  // launches are counted from the iterations the solve reports, not here
  add_launches(-(long long)(launch_count() - before));
  if (e0 != cudaSuccess || e1 != cudaSuccess) {
    cudaGraphDestroy(g);
    return cuda_status(e0 != cudaSuccess ? e0 : e1);
  }
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e2 = cudaGraphInstantiate(&ex, g, 0ULL);
  cudaGraphDestroy(g);
  ORCTM_CUDA_OK(e2);
  h->pcg_graph[pr] = ex;
  h->pcg_graph_key[pr][0] = cv;
  h->pcg_graph_key[pr][1] = sv;
  *out = ex;
  return ORCTM_OK;
}

template <typename T, typename TX>
int pcg_loop(orctm_handle* h, int init_mode, const T* b, TX* x, T* r, T* z, T* pa, T* pb, T* q,
             int maxit, int* iters, int* conv) {
  const Geo& G = h->G;
  const int pr = sizeof(T) == 4;
  const int cv = h->col_var[pr], sv = h->spmv_var[pr];
  launch_pcg_col<T, TX>(G, h->P, h->S, init_mode, b, x, r, nullptr, nullptr, z, cv, h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  int it = 0;
  T *pc = pa, *pn = pb;
  // the first chunk one by one (its first stencil launch forms p = z), then,
  // unless profiling, the device-side loop: chunks of kPcgChunk iterations
  // replayed by a conditional while node until the solve converges or another
  // chunk would pass maxit; no host round trip in between.  The p buffers are
  // back in their roles after every (even) chunk.
  while (it < maxit) {
    if (it > 0 && it % kPcgChunk == 0 && it + kPcgChunk <= maxit && !h->prof) {
      cudaGraphExec_t ex;
      int st;
      if ((st = pcg_loop_graph<T, TX>(h, b, x, r, z, pa, pb, q, &ex))) return st;
      launch_set_limit(h->S, maxit, h->stream);
      ORCTM_CUDA_OK(cudaGraphLaunch(ex, h->stream));
      ORCTM_CUDA_OK(cudaGetLastError());
      if ((st = read_state(h))) return st;
      // every body run launches the whole chunk and the condition kernel;
      // after convergence the chunk's remaining kernels return at once
      const int done = h->hS->iter;
      add_launches((long long)((done - it + kPcgChunk - 1) / kPcgChunk) * (2 * kPcgChunk + 1));
      if (h->hS->converged) break;
      // not converged: the loop stopped because one more chunk would pass
      // maxit, after whole chunks, so the p buffers are in their roles
      it = done;
      continue;
    } else {
      PROF(h, ORCTM_PROF_PCG_SPMV,
           ORCTM_CUDA_OK(launch_pcg_spmv<T>(G, h->P, h->S, z, pc, pn, q, it == 0, sv, h->stream)));
      PROF(h, ORCTM_PROF_PCG_COL, (launch_pcg_col<T, TX>(G, h->P, h->S, 2, b, x, r, pn, q, z, cv, h->stream)));
      ORCTM_CUDA_OK(cudaGetLastError());  // a rejected launch is reported at once
      std::swap(pc, pn);
      ++it;
    }
    if (it % kPcgChunk == 0 || it == maxit) {
      int st;
      ORCTM_CUDA_OK(cudaGetLastError());
      if ((st = read_state(h))) return st;
      if (h->hS->converged) break;
    }
  }
  int st;
  if ((st = read_state(h))) return st;
  *iters = h->hS->iter;
  *conv = h->hS->converged;
  return ORCTM_OK;
}

// Autotuner.  Times every usable variant of the column kernel and of the
// stencil kernel on this handle's grid in precision T and keeps the fastest
// (two untimed launches, then three timed with CUDA events).  It runs before
// the first solve of the precision, on solver vectors that the solve writes
// before it reads them (x is zeroed before every inner solve), with scratch
// solver scalars.  The variants compute bit-identical results (the dot
// products are summed in a fixed order), so the choice changes only speed.
// Choices are cached per grid size and precision for later handles.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, std::pair<int, int>> g_tune_cache;

template <typename T>
int autotune(orctm_handle* h, T* x, T* r, T* z, T* pa, T* pb, T* q) {
  const Geo& G = h->G;
  const int pr = sizeof(T) == 4;
  const auto key = std::make_tuple(G.L.ie, G.L.je, G.L.ke, pr);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      h->col_var[pr] = h->force_col >= 0 ? h->force_col : it->second.first;
      h->spmv_var[pr] = h->force_spmv >= 0 ? h->force_spmv : it->second.second;
      return ORCTM_OK;
    }
  }
  if (!h->S_tune) {
    int st;
    if ((st = h->dev_alloc(&h->S_tune, 1)) || (st = h->dev_alloc(&h->S_tune0, 1))) return st;
    SolverState s0 = *h->hS;
    s0.converged = 0;
    s0.alpha = 0.0;
    s0.beta = 0.0;
    s0.rho = 1.0;
    s0.bb = 1.0;
    s0.tol = 0.0;
    s0.ticket = 0;
    ORCTM_CUDA_OK(cudaMemcpyAsync(h->S_tune0, &s0, sizeof(SolverState), cudaMemcpyHostToDevice,
                                  h->stream));
  }
  auto timed = [&](auto launch, float* best_ms) -> int {
    float tot = 0.f;
    for (int rep = 0; rep < 5; ++rep) {
      ORCTM_CUDA_OK(cudaMemcpyAsync(h->S_tune, h->S_tune0, sizeof(SolverState),
                                    cudaMemcpyDeviceToDevice, h->stream));
      if (rep >= 2) ORCTM_CUDA_OK(cudaEventRecord(h->ev0, h->stream));
      launch();
      ORCTM_CUDA_OK(cudaGetLastError());
      if (rep >= 2) {
        ORCTM_CUDA_OK(cudaEventRecord(h->ev1, h->stream));
        ORCTM_CUDA_OK(cudaEventSynchronize(h->ev1));
        float ms = 0.f;
        ORCTM_CUDA_OK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
        tot += ms;
      }
    }
    *best_ms = tot;
    return ORCTM_OK;
  };
  int st, best_c = 0, best_s = 0;
  float bc = 1e30f, bs = 1e30f;
  for (int v = 0; v < pcg_col_variants(); ++v) {
    if (!pcg_col_variant_ok<T>(G, v)) continue;
    float ms;
    if ((st = timed([&] { launch_pcg_col<T, T>(G, h->P, h->S_tune, 2, nullptr, x, r, pa, q, z, v,
                                               h->stream); }, &ms)))
      return st;
    if (ms < bc) { bc = ms; best_c = v; }
  }
  for (int v = 0; v < pcg_spmv_variants(); ++v) {
    if (!pcg_spmv_variant_ok(v)) continue;
    float ms;
    cudaError_t le = cudaSuccess;
    if ((st = timed([&] { le = launch_pcg_spmv<T>(G, h->P, h->S_tune, z, pa, pb, q, 0, v, h->stream); },
                    &ms)))
      return st;
    if (le != cudaSuccess) continue;
    if (ms < bs) { bs = ms; best_s = v; }
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = {best_c, best_s};
  }
  h->col_var[pr] = h->force_col >= 0 ? h->force_col : best_c;
  h->spmv_var[pr] = h->force_spmv >= 0 ? h->force_spmv : best_s;
  return ORCTM_OK;
}

int ensure_tuned(orctm_handle* h, bool f32) {
  const int pr = f32 ? 1 : 0;
  if (h->col_var[pr] >= 0 && h->spmv_var[pr] >= 0) return ORCTM_OK;
  if (h->force_col >= 0 && h->force_spmv >= 0) {
    h->col_var[pr] = h->force_col;
    h->spmv_var[pr] = h->force_spmv;
    return ORCTM_OK;
  }
  if (f32) return autotune<float>(h, h->d32, h->r32, h->z32, h->p32a, h->p32b, h->q32);
  return autotune<double>(h, h->d, h->rw, h->z, h->p0, h->p1, h->q);
}

// converged = 4: a bounded wait inside a kernel (a TMA stage that never
// arrived) gave up; the solve stops and reports it as a device error.
int check_device_wait(orctm_handle* h, int conv) {
  if (conv != 4) return ORCTM_OK;
  h->err = "a device-side wait for a staged copy timed out in the Poisson stencil kernel";
  return ORCTM_E_CUDA;
}

// Solves A x = b (b in h->b, x in h->xs holding the warm start) by iterative
// refinement: r = b - A x in double-double against the exact operator, then
// a PCG correction on the row-scaled operator (FP64, or FP32 for the refined
// form), until ||r||_2 <= rtol ||b||_2.
int poisson_solve(orctm_handle* h, orctm_solve_stats* stats) {
  const Geo& G = h->G;
  int st;
  orctm_solve_stats s{};
  const bool f32 = h->solver_mode == ORCTM_SOLVER_FP32_REFINED;
  const size_t n3 = (size_t)h->L.n3();
  if ((st = ensure_tuned(h, f32))) return st;
  ORCTM_CUDA_OK(cudaEventRecord(h->ev0, h->stream));
  int total = 0, outer = 0;
  double prev = 1e300, rel = 0.0;
  for (;; ++outer) {
    launch_solver_reset(h->S, h->rtol, 0, h->stream);
    PROF(h, ORCTM_PROF_RESID, launch_resid(G, h->P, h->S, h->b, h->xs, h->r, h->stream));
    ORCTM_CUDA_OK(cudaGetLastError());
    if ((st = read_state(h))) return st;
    const double bnorm = std::sqrt(h->hS->res_bb);
    if (bnorm == 0.0) {  // zero right-hand side: the solution is zero
      ORCTM_CUDA_OK(cudaMemsetAsync(h->xs, 0, sizeof(double) * n3, h->stream));
      rel = 0.0;
      if (outer == 0) s.relres_initial = 0.0;
      break;
    }
    rel = std::sqrt(h->hS->res_rr) / bnorm;
    if (outer == 0) s.relres_initial = rel;
    if (rel <= h->rtol || total >= h->maxit || outer >= 40 || !(rel < 0.5 * prev)) break;
    prev = rel;
    double inner = 0.3 * h->rtol / rel;
    inner = std::min(0.5, std::max(inner, f32 ? 2e-5 : 1e-13));
    int its = 0, conv = 0;
    if (f32) {
      launch_scale_to_f32(G, h->r, h->S, h->r32b, h->stream);
      ORCTM_CUDA_OK(cudaMemsetAsync(h->d32, 0, sizeof(float) * n3, h->stream));
      launch_solver_reset(h->S, inner, 0, h->stream);
      if ((st = pcg_loop<float, float>(h, 1, h->r32b, h->d32, h->r32, h->z32, h->p32a, h->p32b,
                                       h->q32, h->maxit - total, &its, &conv)))
        return st;
      if ((st = check_device_wait(h, conv))) return st;
      launch_axpy_f32(G, h->d32, h->S, h->xs, h->stream);
    } else {
      ORCTM_CUDA_OK(cudaMemsetAsync(h->d, 0, sizeof(double) * n3, h->stream));
      launch_solver_reset(h->S, inner, 0, h->stream);
      if ((st = pcg_loop<double, double>(h, 1, h->r, h->d, h->rw, h->z, h->p0, h->p1, h->q,
                                         h->maxit - total, &its, &conv)))
        return st;
      if ((st = check_device_wait(h, conv))) return st;
      launch_axpy_f64(G, h->d, h->xs, h->stream);
    }
    ORCTM_CUDA_OK(cudaGetLastError());
    total += its;
  }
  ORCTM_CUDA_OK(cudaEventRecord(h->ev1, h->stream));
  ORCTM_CUDA_OK(cudaEventSynchronize(h->ev1));
  s.relres = rel;
  s.iterations = total;
  s.outer_iterations = outer;
  s.converged = rel <= h->rtol;
  float ms = 0.f;
  ORCTM_CUDA_OK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  s.solve_ms = ms;
  if (stats) *stats = s;
  return s.converged ? ORCTM_OK : ORCTM_E_NOT_CONVERGED;
}

// ------------------------------------------------------------- routines
// ------------------------------------------------------ asynchronous copies
// The compute stream waits for the uploads in flight of the listed fields
// (a negative id ends the list) or of every field.
int wait_uploads(orctm_handle* h, std::initializer_list<int> fields) {
  for (int f : fields) {
    if (f < 0 || f >= 64 || !h->pending[f]) continue;
    ORCTM_CUDA_OK(cudaStreamWaitEvent(h->stream, h->field_ready[f], 0));
    h->pending[f] = false;
  }
  return ORCTM_OK;
}

int wait_all_uploads(orctm_handle* h) {
  for (int f = 0; f < 64; ++f)
    if (h->pending[f]) {
      ORCTM_CUDA_OK(cudaStreamWaitEvent(h->stream, h->field_ready[f], 0));
      h->pending[f] = false;
    }
  return ORCTM_OK;
}

// copy stream after everything queued so far on the compute stream
int copy_after_compute(orctm_handle* h) {
  cudaEvent_t e = h->get_event();
  h->copy_events.push_back(e);
  ORCTM_CUDA_OK(cudaEventRecord(e, h->stream));
  ORCTM_CUDA_OK(cudaStreamWaitEvent(h->cstream, e, 0));
  return ORCTM_OK;
}

int download_async(orctm_handle* h, int f, double* host) {
  int st;
  if ((st = wait_uploads(h, {f}))) return st;
  int i0, ni, j0, nj, nk;
  extent(h, f, i0, ni, j0, nj, nk);
  double* src = f == ORCTM_F_ZO ? h->zo : h->slot[f];
  if ((st = copy_after_compute(h))) return st;
  for (int k = 0; k < nk; ++k)
    ORCTM_CUDA_OK(cudaMemcpy2DAsync(host + (size_t)k * ni * nj, sizeof(double) * ni,
                                    src + h->L.at(i0, j0, k), sizeof(double) * h->L.P,
                                    sizeof(double) * ni, nj, cudaMemcpyDeviceToHost, h->cstream));
  // routines never write a buffer in place, and a referenced buffer is never
  // handed out again: holding a reference keeps the source intact until the
  // copy has ended
  if (f != ORCTM_F_ZO) {
    h->refs[src]++;
    h->held.push_back(src);
  }
  return ORCTM_OK;
}

// the registered step outputs that are final at this point of the step
int step_outputs(orctm_handle* h, bool tracers) {
  int st;
  for (const auto& o : h->step_out) {
    const bool is_tracer = o.field >= ORCTM_F_THO;
    if (is_tracer == tracers && (st = download_async(h, o.field, o.host))) return st;
  }
  return ORCTM_OK;
}

int r_ocadpo(orctm_handle* h, int n) {
  int st;
  if ((st = wait_uploads(h, {ORCTM_F_THO + n, ORCTM_F_UKO, ORCTM_F_VKE, ORCTM_F_WO, ORCTM_F_ZO})))
    return st;
  double *out, *tA, *vA, *vB;
  if ((st = h->alloc(&out)) || (st = h->alloc(&tA)) || (st = h->alloc(&vA)) || (st = h->alloc(&vB)))
    return st;
  const int f = ORCTM_F_THO + n;
  PROF(h, ORCTM_PROF_OCADPO,
       launch_ocadpo(h->G, h->slot[f], h->slot[ORCTM_F_UKO], h->slot[ORCTM_F_VKE],
                     h->slot[ORCTM_F_WO], h->zo, out, tA, vA, vB, h->stream));
  ORCTM_CUDA_OK(cudaGetLastError());
  h->bind(f, out);
  h->unref(tA); h->unref(vA); h->unref(vB);
  return ORCTM_OK;
}

// OCADPO for every tracer: one set of sweeps per group of tracers shares the
// transports and volumes (launch_ocadpo_all); the same results as r_ocadpo
// tracer by tracer.  uko / vke / wo, when given, are the transports to use
// (the step's initial ones, held while the momentum path ran first)
int r_ocadpo_all(orctm_handle* h, const double* uko = nullptr, const double* vke = nullptr,
                 const double* wo = nullptr) {
  int st;
  const int ntr = h->ntr;
  for (int n = 0; n < ntr; ++n)
    if ((st = wait_uploads(h, {ORCTM_F_THO + n}))) return st;
  if ((st = wait_uploads(h, {ORCTM_F_UKO, ORCTM_F_VKE, ORCTM_F_WO, ORCTM_F_ZO}))) return st;
  if (!uko) {
    uko = h->slot[ORCTM_F_UKO];
    vke = h->slot[ORCTM_F_VKE];
    wo = h->slot[ORCTM_F_WO];
  }
  double *out[kMaxTracers] = {}, *mid[kMaxTracers] = {}, *vA = nullptr, *vB = nullptr;
  const double* in[kMaxTracers] = {};
  for (int n = 0; n < ntr; ++n) {
    if ((st = h->alloc(&out[n])) || (st = h->alloc(&mid[n]))) return st;
    in[n] = h->slot[ORCTM_F_THO + n];
  }
  if ((st = h->alloc(&vA)) || (st = h->alloc(&vB))) return st;
  PROF(h, ORCTM_PROF_OCADPO,
       launch_ocadpo_all(h->G, ntr, in, out, mid, uko, vke, wo, h->zo, vA, vB, h->stream));
  ORCTM_CUDA_OK(cudaGetLastError());
  for (int n = 0; n < ntr; ++n) {
    h->bind(ORCTM_F_THO + n, out[n]);
    h->unref(mid[n]);
  }
  h->unref(vA);
  h->unref(vB);
  return ORCTM_OK;
}

template <int WHICH>
int r_momadv(orctm_handle* h) {
  {
    const int own = WHICH == 0 ? ORCTM_F_UOO : WHICH == 1 ? ORCTM_F_VOE : ORCTM_F_WNO;
    const int st0 = wait_uploads(h, {own, ORCTM_F_UKO, ORCTM_F_VKE, ORCTM_F_WO, ORCTM_F_ZO});
    if (st0) return st0;
  }
  int st;
  double *out, *tA, *vA, *vB;
  if ((st = h->alloc(&out)) || (st = h->alloc(&tA)) || (st = h->alloc(&vA)) || (st = h->alloc(&vB)))
    return st;
  const double *uko = h->slot[ORCTM_F_UKO], *vke = h->slot[ORCTM_F_VKE], *wo = h->slot[ORCTM_F_WO];
  int f;
  if (WHICH == 0) {
    f = ORCTM_F_UOO;
    PROF(h, ORCTM_PROF_OCUAD, launch_ocuad(h->G, h->slot[f], uko, vke, wo, out, tA, vA, vB, h->stream));
  } else if (WHICH == 1) {
    f = ORCTM_F_VOE;
    PROF(h, ORCTM_PROF_OCVAD, launch_ocvad(h->G, h->slot[f], uko, vke, wo, out, tA, vA, vB, h->stream));
  } else {
    f = ORCTM_F_WNO;
    PROF(h, ORCTM_PROF_OCWAD, launch_ocwad(h->G, h->slot[f], uko, vke, wo, h->zo, out, tA, vA, vB, h->stream));
  }
  ORCTM_CUDA_OK(cudaGetLastError());
  h->bind(f, out);
  h->unref(tA); h->unref(vA); h->unref(vB);
  return ORCTM_OK;
}

int r_octdiff(orctm_handle* h) {
  int st;
  const int ntr = h->ntr;
  // what it reads and the slots it rebinds
  for (int n = 0; n < ntr; ++n)
    if ((st = wait_uploads(h, {ORCTM_F_THO + n}))) return st;
  if ((st = wait_uploads(h, {ORCTM_F_DVO, ORCTM_F_ZO}))) return st;
  const double* in[kMaxTracers];
  double* outv[kMaxTracers];
  for (int n = 0; n < ntr; ++n) {
    in[n] = h->slot[ORCTM_F_THO + n];
    if ((st = h->alloc(&outv[n]))) return st;
  }
  PROF(h, ORCTM_PROF_OCTDIFF, launch_octdiff_vert(h->G, ntr, in, outv, h->slot[ORCTM_F_DVO], h->zo, h->stream));
  ORCTM_CUDA_OK(cudaGetLastError());
  for (int n = 0; n < ntr; ++n) h->bind(ORCTM_F_THO + n, outv[n]);
  if (h->G.aulapts > h->G.almzer) {
    // Laplacian and biharmonic update of every tracer in one fused launch
    const double* vin[kMaxTracers];
    double* bout[kMaxTracers];
    for (int n = 0; n < ntr; ++n) {
      vin[n] = h->slot[ORCTM_F_THO + n];
      if ((st = h->alloc(&bout[n]))) return st;
    }
    PROF(h, ORCTM_PROF_OCTDIFF, launch_octdiff_hbih(h->G, ntr, vin, bout, h->zo, h->stream));
    ORCTM_CUDA_OK(cudaGetLastError());
    for (int n = 0; n < ntr; ++n) h->bind(ORCTM_F_THO + n, bout[n]);
  }
  return ORCTM_OK;
}

int r_octimf(orctm_handle* h) {
  {
    // the slots it rebinds: their uploads land first
    const int st0 = wait_uploads(h, {ORCTM_F_UKO, ORCTM_F_VKE, ORCTM_F_UOO, ORCTM_F_VOE});
    if (st0) return st0;
  }
  h->alias(ORCTM_F_UKO, ORCTM_F_UOO);
  h->alias(ORCTM_F_VKE, ORCTM_F_VOE);
  return ORCTM_OK;
}

int r_ocvisc(orctm_handle* h) {
  {
    // what it reads and the slots it rebinds
    const int st0 = wait_uploads(h, {ORCTM_F_UOO, ORCTM_F_VOE, ORCTM_F_WNO, ORCTM_F_UKO,
                                     ORCTM_F_VKE, ORCTM_F_AVO});
    if (st0) return st0;
  }
  int st;
  double *sp, *ukv, *vkv, *wnv, *u1, *v1, *w1, *uo, *vo, *wo;
  if ((st = h->alloc(&sp)) || (st = h->alloc(&ukv)) || (st = h->alloc(&vkv)) ||
      (st = h->alloc(&wnv)) || (st = h->alloc(&u1)) || (st = h->alloc(&v1)) ||
      (st = h->alloc(&w1)) || (st = h->alloc(&uo)) || (st = h->alloc(&vo)) || (st = h->alloc(&wo)))
    return st;
  // the two 2D speed fields live in the first two planes of one scratch buffer
  PROF(h, ORCTM_PROF_OCVISC,
       launch_ocvisc(h->G, h->slot[ORCTM_F_UOO], h->slot[ORCTM_F_VOE], h->slot[ORCTM_F_WNO],
                     h->slot[ORCTM_F_UKO], h->slot[ORCTM_F_VKE], h->slot[ORCTM_F_AVO], sp,
                     sp + h->L.plane, ukv, vkv, wnv, u1, v1, w1, uo, vo, wo, h->stream));
  ORCTM_CUDA_OK(cudaGetLastError());
  h->bind(ORCTM_F_UOO, uo);
  h->bind(ORCTM_F_VOE, vo);
  h->bind(ORCTM_F_WNO, wo);
  h->unref(sp); h->unref(ukv); h->unref(vkv); h->unref(wnv);
  h->unref(u1); h->unref(v1); h->unref(w1);
  return r_octimf(h);  // ocvisc.f90:767
}

int r_ocvtot_nh(orctm_handle* h, orctm_solve_stats* stats) {
  {
    // what it reads and the slots it rebinds
    const int st0 = wait_uploads(h, {ORCTM_F_UOO, ORCTM_F_VOE, ORCTM_F_WNO, ORCTM_F_UOO_1,
                                     ORCTM_F_VOE_1, ORCTM_F_WNO_1, ORCTM_F_PNH, ORCTM_F_WO,
                                     ORCTM_F_ZO});
    if (st0) return st0;
  }
  int st;
  if ((st = ensure_solver_buffers(h))) return st;
  PROF(h, ORCTM_PROF_NH_RHS,
       launch_nh_rhs(h->G, h->slot[ORCTM_F_UOO], h->slot[ORCTM_F_UOO_1], h->slot[ORCTM_F_VOE],
                     h->slot[ORCTM_F_VOE_1], h->slot[ORCTM_F_WNO], h->slot[ORCTM_F_WNO_1], h->zo,
                     h->b, h->stream));
  // warm start from the previous PNH (KSPSetInitialGuessNonzero, mo_petsc.f90:232)
  ORCTM_CUDA_OK(cudaMemcpyAsync(h->xs, h->slot[ORCTM_F_PNH], sizeof(double) * h->L.n3(),
                                cudaMemcpyDeviceToDevice, h->stream));
  ORCTM_CUDA_OK(cudaGetLastError());
  const int solve_status = poisson_solve(h, stats);
  if (solve_status != ORCTM_OK && solve_status != ORCTM_E_NOT_CONVERGED) return solve_status;
  double *pnh, *uo, *vo, *wn;
  if ((st = h->alloc(&pnh)) || (st = h->alloc(&uo)) || (st = h->alloc(&vo)) || (st = h->alloc(&wn)))
    return st;
  PROF(h, ORCTM_PROF_NH_POST,
       launch_nh_post(h->G, h->xs, h->slot[ORCTM_F_PNH], pnh, h->slot[ORCTM_F_UOO],
                      h->slot[ORCTM_F_VOE], uo, vo, wn, h->stream));
  ORCTM_CUDA_OK(cudaGetLastError());
  h->bind(ORCTM_F_PNH, pnh);
  h->bind(ORCTM_F_UOO, uo);
  h->bind(ORCTM_F_VOE, vo);
  h->bind(ORCTM_F_WNO, wn);
  // UOO_1 <- UOO, VOE_1 <- VOE, WNO_1 <- WNO, WO <- WNO (ocvtot_nh.f90:238-255)
  h->alias(ORCTM_F_UOO_1, ORCTM_F_UOO);
  h->alias(ORCTM_F_VOE_1, ORCTM_F_VOE);
  h->alias(ORCTM_F_WNO_1, ORCTM_F_WNO);
  h->alias(ORCTM_F_WO, ORCTM_F_WNO);
  return solve_status;
}

}  // namespace

__global__ void k_div_nr(const double* __restrict__ a, const double* __restrict__ b,
                         double* __restrict__ q, size_t n) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) q[k] = div_nr(a[k], b[k]);
}

// ====================================================================== C ABI
extern "C" {

int orctm_check_division(int device, const double* a, const double* b, double* q, size_t n) {
  if (!a || !b || !q) return ORCTM_E_ARG;
  if (n == 0) return ORCTM_OK;
  ORCTM_CUDA_OK(cudaSetDevice(device));
  double* d = nullptr;
  ORCTM_CUDA_OK(cudaMalloc(&d, 3 * n * sizeof(double)));
  int st = cuda_status(cudaMemcpy(d, a, n * sizeof(double), cudaMemcpyHostToDevice));
  if (!st) st = cuda_status(cudaMemcpy(d + n, b, n * sizeof(double), cudaMemcpyHostToDevice));
  if (!st) {
    k_div_nr<<<(unsigned)((n + 255) / 256), 256>>>(d, d + n, d + 2 * n, n);
    count_launch();
    st = cuda_status(cudaGetLastError());
  }
  if (!st) st = cuda_status(cudaMemcpy(q, d + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost));
  cudaFree(d);
  return st;
}

int orctm_abi_version(void) { return ORCTM_ABI_VERSION; }

const char* orctm_status_string(int s) {
  switch (s) {
    case ORCTM_OK: return "ok";
    case ORCTM_E_ARG: return "invalid argument";
    case ORCTM_E_CUDA: return "CUDA runtime error";
    case ORCTM_E_NOMEM: return "device memory exhausted";
    case ORCTM_E_NOT_CONVERGED: return "Poisson solve did not reach the residual target";
    case ORCTM_E_GEOMETRY: return "geometry is not of the BODEN form";
    case ORCTM_E_UNSUPPORTED: return "option outside the implemented path";
    case ORCTM_E_NODEVICE: return "no usable CUDA device";
    case ORCTM_E_TOO_LARGE: return "grid too large (2^31 elements per padded field, or the scratch-free entry point's limit)";
    case ORCTM_E_UNSTABLE: return "OCCLIT's baroclinic iteration did not settle (CONTRA above 1e-3)";
    default: return "unknown status";
  }
}

const char* orctm_last_error(const orctm_handle* h) {
  if (h && !h->err.empty()) return h->err.c_str();
  if (!g_cuda_error.empty()) return g_cuda_error.c_str();
  return h ? h->err.c_str() : g_create_error.c_str();
}

int orctm_destroy(orctm_handle* h) {
  if (!h) return ORCTM_E_ARG;
  cudaSetDevice(h->device);
  if (h->cstream) cudaStreamSynchronize(h->cstream);
  for (double* p : h->held) h->unref(p);
  h->held.clear();
  if (h->stream) cudaStreamSynchronize(h->stream);
  std::vector<double*> all(h->free_.begin(), h->free_.end());
  for (auto& kv : h->refs) all.push_back(kv.first);
  std::sort(all.begin(), all.end());
  all.erase(std::unique(all.begin(), all.end()), all.end());
  // stream-ordered frees: no device-wide synchronisation, so other handles'
  // work in flight on the device is not stalled
  if (h->stream) {
    for (double* p : all) cudaFreeAsync(h->base(p), h->stream);
    for (void* p : h->owned) cudaFreeAsync(h->base(p), h->stream);
    cudaStreamSynchronize(h->stream);
  }
  for (int pr = 0; pr < 2; ++pr)
    if (h->pcg_graph[pr]) cudaGraphExecDestroy(h->pcg_graph[pr]);
  if (h->sor_graph) cudaGraphExecDestroy(h->sor_graph);
  if (h->hS) pinned_state_put(h->hS);
  if (h->h_contra) cudaFreeHost(h->h_contra);
  for (int k = 0; k < ORCTM_PROF_KINDS; ++k)
    for (auto& pr : h->prof_pairs[k]) {
      h->ev_pool.push_back(pr.first);
      h->ev_pool.push_back(pr.second);
    }
  for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
  if (h->tm0) cudaEventDestroy(h->tm0);
  if (h->tm1) cudaEventDestroy(h->tm1);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  for (cudaEvent_t e : h->copy_events) cudaEventDestroy(e);
  for (int f = 0; f < 64; ++f)
    if (h->field_ready[f]) cudaEventDestroy(h->field_ready[f]);
  if (h->cstream) cudaStreamDestroy(h->cstream);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return ORCTM_OK;
}

int orctm_create(const orctm_desc* d, orctm_handle** out) {
  g_create_error.clear();
  g_cuda_error.clear();
  if (!d || !out) return ORCTM_E_ARG;
  *out = nullptr;
  auto bad = [&](int st, const char* m) {
    g_create_error = m;
    return st;
  };
  if (d->ie < 4 || d->je < 3 || d->ke < 2 || d->ke > kMaxKe) return bad(ORCTM_E_ARG, "grid size out of range");
  {
    // the kernels index a padded field with 32-bit offsets
    const long long pitch = ((long long)d->ie + 1 + 31) / 32 * 32;
    if (pitch * ((long long)d->je + 1) * ((long long)d->ke + 1) >= (1LL << 31))
      return bad(ORCTM_E_TOO_LARGE, "padded field exceeds 2^31 elements");
  }
  if (d->i_start != 0 || d->j_start != 0) return bad(ORCTM_E_UNSUPPORTED, "only single-rank domains (I_start = J_start = 0)");
  if (d->ntracers < 2 || d->ntracers > kMaxTracers) return bad(ORCTM_E_ARG, "ntracers must be in [2, 8]");
  if (!(d->dt > 0)) return bad(ORCTM_E_ARG, "dt must be positive");
  if (d->ah00 > d->almzer) return bad(ORCTM_E_UNSUPPORTED, "harmonic tracer diffusion (AH00 > ALMZER) is not implemented");
  const void* req[] = {d->dzw, d->di, d->dlxp, d->dlyp, d->dtdxpo, d->dtdyo, d->dlxu, d->dlyu,
                       d->dtdxuo, d->dlxv, d->dlyv, d->dpye, d->ddpo, d->weto, d->dduo,
                       d->amsuo, d->ddue, d->amsue};
  for (const void* p : req)
    if (!p) return bad(ORCTM_E_ARG, "missing geometry array");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return bad(ORCTM_E_NODEVICE, "no CUDA device");
  if (d->device < 0 || d->device >= ndev) return bad(ORCTM_E_ARG, "device ordinal out of range");
  orctm_handle* h = new orctm_handle();
  h->device = d->device;
  int st = cuda_status(cudaSetDevice(h->device));
  if (!st) st = cuda_status(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  if (!st) st = cuda_status(cudaStreamCreateWithFlags(&h->cstream, cudaStreamNonBlocking));
  if (!st) st = device_pool(h->device, &h->mempool);
  if (!st) st = setup(h, d);
  if (st) {
    g_create_error = h->err.empty() ? orctm_status_string(st) : h->err;
    orctm_destroy(h);
    return st;
  }
  *out = h;
  return ORCTM_OK;
}

int orctm_field_size(const orctm_handle* h, int f, size_t* n) {
  if (!h || !n || f < 0 || f >= kNumFixed + h->ntr) return ORCTM_E_ARG;
  int i0, ni, j0, nj, nk;
  extent(h, f, i0, ni, j0, nj, nk);
  *n = (size_t)ni * nj * nk;
  return ORCTM_OK;
}

int orctm_upload(orctm_handle* h, int f, const double* host, size_t n) {
  size_t want;
  if (!host || orctm_field_size(h, f, &want) != ORCTM_OK || n != want) return ORCTM_E_ARG;
  cudaSetDevice(h->device);
  {
    const int st0 = wait_all_uploads(h);
    if (st0) return st0;
  }
  int i0, ni, j0, nj, nk;
  extent(h, f, i0, ni, j0, nj, nk);
  double* dst;
  if (f == ORCTM_F_ZO) {
    dst = h->zo;
  } else {
    int st;
    if (h->refs[h->slot[f]] > 1) {  // shared with another field: copy on write
      double* p;
      if ((st = h->alloc(&p))) return st;
      h->bind(f, p);
    }
    dst = h->slot[f];
  }
  for (int k = 0; k < nk; ++k)
    ORCTM_CUDA_OK(cudaMemcpy2DAsync(dst + h->L.at(i0, j0, k), sizeof(double) * h->L.P,
                                    host + (size_t)k * ni * nj, sizeof(double) * ni,
                                    sizeof(double) * ni, nj, cudaMemcpyHostToDevice, h->stream));
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  return ORCTM_OK;
}

int orctm_download(orctm_handle* h, int f, double* host, size_t n) {
  size_t want;
  if (!host || orctm_field_size(h, f, &want) != ORCTM_OK || n != want) return ORCTM_E_ARG;
  cudaSetDevice(h->device);
  {
    const int st0 = wait_all_uploads(h);
    if (st0) return st0;
  }
  int i0, ni, j0, nj, nk;
  extent(h, f, i0, ni, j0, nj, nk);
  const double* src = f == ORCTM_F_ZO ? h->zo : h->slot[f];
  for (int k = 0; k < nk; ++k)
    ORCTM_CUDA_OK(cudaMemcpy2DAsync(host + (size_t)k * ni * nj, sizeof(double) * ni,
                                    src + h->L.at(i0, j0, k), sizeof(double) * h->L.P,
                                    sizeof(double) * ni, nj, cudaMemcpyDeviceToHost, h->stream));
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  return ORCTM_OK;
}

int orctm_upload_async(orctm_handle* h, int f, const double* host, size_t n) {
  size_t want;
  if (!host || orctm_field_size(h, f, &want) != ORCTM_OK || n != want) return ORCTM_E_ARG;
  cudaSetDevice(h->device);
  int st, i0, ni, j0, nj, nk;
  extent(h, f, i0, ni, j0, nj, nk);
  double* dst;
  if (f == ORCTM_F_ZO) {
    dst = h->zo;
  } else {
    if (h->refs[h->slot[f]] > 1) {  // shared with another field: copy on write
      double* p;
      if ((st = h->alloc(&p))) return st;
      h->bind(f, p);
    }
    dst = h->slot[f];
  }
  // after the kernels queued so far (which may still read the old contents)
  // and after the allocation above, which is ordered on the compute stream
  if ((st = copy_after_compute(h))) return st;
  for (int k = 0; k < nk; ++k)
    ORCTM_CUDA_OK(cudaMemcpy2DAsync(dst + h->L.at(i0, j0, k), sizeof(double) * h->L.P,
                                    host + (size_t)k * ni * nj, sizeof(double) * ni,
                                    sizeof(double) * ni, nj, cudaMemcpyHostToDevice, h->cstream));
  if (!h->field_ready[f]) ORCTM_CUDA_OK(cudaEventCreateWithFlags(&h->field_ready[f], cudaEventDisableTiming));
  ORCTM_CUDA_OK(cudaEventRecord(h->field_ready[f], h->cstream));
  h->pending[f] = true;
  return ORCTM_OK;
}

int orctm_download_async(orctm_handle* h, int f, double* host, size_t n) {
  size_t want;
  if (!host || orctm_field_size(h, f, &want) != ORCTM_OK || n != want) return ORCTM_E_ARG;
  cudaSetDevice(h->device);
  return download_async(h, f, host);
}

int orctm_set_step_outputs(orctm_handle* h, int n, const int* fields, double* const* host,
                           const size_t* sizes) {
  if (!h || n < 0 || (n > 0 && (!fields || !host || !sizes))) return ORCTM_E_ARG;
  std::vector<orctm_handle::StepOut> v;
  for (int k = 0; k < n; ++k) {
    size_t want;
    if (!host[k] || orctm_field_size(h, fields[k], &want) != ORCTM_OK || sizes[k] != want)
      return ORCTM_E_ARG;
    v.push_back({fields[k], host[k], sizes[k]});
  }
  h->step_out = v;
  return ORCTM_OK;
}

int orctm_wait_copies(orctm_handle* h) {
  if (!h) return ORCTM_E_ARG;
  cudaSetDevice(h->device);
  // later work on the compute stream (a timer's stop event, say) comes after
  // the copies
  cudaEvent_t e = h->get_event();
  ORCTM_CUDA_OK(cudaEventRecord(e, h->cstream));
  ORCTM_CUDA_OK(cudaStreamWaitEvent(h->stream, e, 0));
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->cstream));
  h->ev_pool.push_back(e);
  for (cudaEvent_t x : h->copy_events) h->ev_pool.push_back(x);
  h->copy_events.clear();
  for (double* p : h->held) h->unref(p);
  h->held.clear();
  return ORCTM_OK;
}

int orctm_write_extra(orctm_handle* h, const char* path, int append, int idate, int nfield,
                      const int* fields, const int* codes) {
  if (!h || !path || nfield < 1 || !fields || !codes) return ORCTM_E_ARG;
  int st;
  for (int k = 0; k < nfield; ++k) {
    size_t n;
    if ((st = orctm_field_size(h, fields[k], &n))) return st;
    std::vector<double> buf(n);
    if ((st = orctm_download(h, fields[k], buf.data(), n))) return st;
    int i0, ni, j0, nj, nk;
    extent(h, fields[k], i0, ni, j0, nj, nk);
    // KCODE: INT(TIESTU(K)) for p/u/v levels, INT(TIESTW(K)) for w levels,
    // -100 for 2D fields (aufw.f90:63-160)
    std::vector<int> kc((size_t)nk);
    const Kind kind = field_kind(fields[k]);
    for (int l = 0; l < nk; ++l)
      kc[(size_t)l] = kind == K2P ? -100 : (int)(kind == KW ? h->tiestw[l] : h->tiestu[l]);
    if ((st = orctm_write_extra_host(path, append || k > 0, idate, codes[k], nk, kc.data(),
                                     ni * nj, buf.data())))
      return st;
  }
  return ORCTM_OK;
}

int orctm_read_extra(orctm_handle* h, const char* path, int nfield, const int* fields,
                     const int* codes) {
  if (!h || !path || nfield < 1 || !fields || !codes) return ORCTM_E_ARG;
  int st;
  for (int k = 0; k < nfield; ++k) {
    size_t n;
    if ((st = orctm_field_size(h, fields[k], &n))) return st;
    int i0, ni, j0, nj, nk;
    extent(h, fields[k], i0, ni, j0, nj, nk);
    std::vector<double> buf(n);
    if ((st = orctm_read_extra_host(path, codes[k], nk, ni * nj, buf.data(), nullptr))) {
      h->err = "EXTRA file lacks the levels of a requested field";
      return st;
    }
    if ((st = orctm_upload(h, fields[k], buf.data(), n))) return st;
  }
  return ORCTM_OK;
}

#define ORCTM_ENTER(h)             \
  if (!(h)) return ORCTM_E_ARG;    \
  cudaSetDevice((h)->device)

int orctm_ocuad(orctm_handle* h) { ORCTM_ENTER(h); return r_momadv<0>(h); }
int orctm_ocvad(orctm_handle* h) { ORCTM_ENTER(h); return r_momadv<1>(h); }
int orctm_ocwad(orctm_handle* h) { ORCTM_ENTER(h); return r_momadv<2>(h); }
int orctm_ocadpo(orctm_handle* h, int tracer) {
  ORCTM_ENTER(h);
  if (tracer < 0 || tracer >= h->ntr) return ORCTM_E_ARG;
  return r_ocadpo(h, tracer);
}

int orctm_ocadpo_all(orctm_handle* h) {
  ORCTM_ENTER(h);
  return r_ocadpo_all(h);
}
int orctm_octdiff(orctm_handle* h) { ORCTM_ENTER(h); return r_octdiff(h); }
int orctm_octimf(orctm_handle* h) { ORCTM_ENTER(h); return r_octimf(h); }
int orctm_ocvisc(orctm_handle* h) { ORCTM_ENTER(h); return r_ocvisc(h); }
int orctm_ocvtot_nh(orctm_handle* h, orctm_solve_stats* s) { ORCTM_ENTER(h); return r_ocvtot_nh(h, s); }

// ---------------------------------------------------------------------------
// Open-boundary tides and sponge (mo_obcs.f90)
namespace {
// points along side b (0 W, 1 E, 2 N, 3 S) of variable v (0 z, 1 u, 2 v),
// the dimensions of OB{W,E,N,S}{Z,U,V}am (mo_obcs.f90:124-138)
int obc_points(const orctm_handle* h, int b, int v) {
  const int IE = h->L.ie, JE = h->L.je;
  if (b < 2) return v == 2 ? JE + 1 : JE;
  return v == 1 ? IE + 1 : IE;
}
bool obc_open(const orctm_handle* h, int b) {
  const int sw[4] = {h->G.ob_w, h->G.ob_e, h->G.ob_n, h->G.ob_s};
  return sw[b] != 0;
}
// the compute stream waits for every copy queued so far (a routine about to
// overwrite a buffer that a pending download reads)
int compute_after_copies(orctm_handle* h) {
  cudaEvent_t e = h->get_event();
  h->copy_events.push_back(e);
  ORCTM_CUDA_OK(cudaEventRecord(e, h->cstream));
  ORCTM_CUDA_OK(cudaStreamWaitEvent(h->stream, e, 0));
  return ORCTM_OK;
}
// field f's buffer, made private to the slot (copied when shared)
int own_buffer(orctm_handle* h, int f) {
  if (h->refs[h->slot[f]] <= 1) return ORCTM_OK;
  double* p;
  int st;
  if ((st = h->alloc(&p))) return st;
  ORCTM_CUDA_OK(cudaMemcpyAsync(h->base(p), h->base(h->slot[f]),
                                sizeof(double) * ((size_t)h->L.n3() + 2 * h->guard_elems()),
                                cudaMemcpyDeviceToDevice, h->stream));
  h->bind(f, p);
  return ORCTM_OK;
}
}  // namespace

int orctm_set_obc(orctm_handle* h, const orctm_obc* o) {
  ORCTM_ENTER(h);
  if (!o || o->ntide < 1 || o->ntide > ORCTM_OBC_MAX_TIDES || !o->period)
    return h->fail(ORCTM_E_ARG, "orctm_set_obc: ntide out of range or no periods");
  for (int td = 0; td < o->ntide; ++td)
    if (!std::isfinite(o->period[td]) || o->period[td] == 0.0)
      return h->fail(ORCTM_E_ARG, "orctm_set_obc: tidal periods must be finite and nonzero");
  if (!std::isfinite(o->relax_inner) || !std::isfinite(o->relax_bound))
    return h->fail(ORCTM_E_ARG, "orctm_set_obc: relaxation times must be finite");
  const int IE = h->L.ie, JE = h->L.je;
  size_t total = 0;
  bool on[4];
  for (int b = 0; b < 4; ++b) {
    on[b] = obc_open(h, b) && o->sponge[b];
    if (!on[b]) continue;
    const int wmax = b < 2 ? IE : JE;
    if (o->width[b] < 1 || o->width[b] > wmax)
      return h->fail(ORCTM_E_ARG, "orctm_set_obc: sponge width out of range");
    for (int v = 0; v < 3; ++v) {
      if (!o->amp[b][v] || !o->pha[b][v])
        return h->fail(ORCTM_E_ARG, "orctm_set_obc: missing constants of an open, sponged side");
      total += 2 * (size_t)obc_points(h, b, v) * (size_t)o->ntide;
    }
  }
  {
    const int st0 = wait_all_uploads(h);
    if (st0) return st0;
  }
  if (total > h->obc_cap) {
    int st;
    double* p;
    if ((st = h->dev_alloc(&p, total))) return st;
    h->obc_buf = p;
    h->obc_cap = total;
  }
  // the previous constants may still be read by queued launches
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  size_t off = 0;
  for (int v = 0; v < 3; ++v) {
    ObcArgs& a = h->obc[v];
    a = ObcArgs{};
    a.ntide = o->ntide;
    for (int td = 0; td < o->ntide; ++td) a.period[td] = o->period[td];
    a.pi = 4.0 * std::atan(1.0);  // PI = 4.*ATAN(1.), orctm.f90:525
    a.dt = h->G.dt;
    // rel_uv* = rel_ts* = rel_eta* = Urelax* (mo_obcs.f90:499-506)
    a.relb = o->relax_bound;
    a.reli = o->relax_inner;
    for (int b = 0; b < 4; ++b) {
      a.on[b] = on[b] ? 1 : 0;
      a.width[b] = on[b] ? o->width[b] : 1;
      if (!on[b]) continue;
      const size_t n = (size_t)obc_points(h, b, v) * (size_t)o->ntide;
      double* amp = h->obc_buf + off;
      double* pha = amp + n;
      off += 2 * n;
      ORCTM_CUDA_OK(cudaMemcpy(amp, o->amp[b][v], sizeof(double) * n, cudaMemcpyHostToDevice));
      ORCTM_CUDA_OK(cudaMemcpy(pha, o->pha[b][v], sizeof(double) * n, cudaMemcpyHostToDevice));
      a.side[b] = ObcSide{amp, pha, obc_points(h, b, v), nullptr};
    }
  }
  h->obc_ready = true;
  // the T/S records follow the sides and widths set here: set them again;
  // the sponge is the 1/x form until orctm_set_obc_sponge_exp
  h->obc_ts_ready[0] = h->obc_ts_ready[1] = false;
  h->obc_exp_sao_south = nullptr;
  return ORCTM_OK;
}

namespace {
// the exponential sponge's rates of a tracer's side: the p-point table,
// except SAO's south band, whose loop reads the rate T's loop left behind
// (Ms_s from Lt_s, mo_obcs.f90:2974-2978); null in the 1/x form
const double* ts_rates(const orctm_handle* h, int tracer, int b) {
  if (!h->obc[0].expo) return nullptr;
  return tracer == 1 && b == 3 ? h->obc_exp_sao_south : h->obc[0].side[b].wexp;
}
}  // namespace

int orctm_set_obc_ts(orctm_handle* h, int tracer, const double* const* cli) {
  ORCTM_ENTER(h);
  if (!h->obc_ready) return h->fail(ORCTM_E_ARG, "orctm_set_obc_ts: orctm_set_obc not called");
  if (tracer < 0 || tracer > 1 || tracer >= h->ntr || !cli)
    return h->fail(ORCTM_E_ARG, "orctm_set_obc_ts: tracer must be 0 (THO) or 1 (SAO)");
  const int IE = h->L.ie, JE = h->L.je, KE = h->L.ke;
  const ObcArgs& base = h->obc[0];
  size_t total = 0;
  for (int b = 0; b < 4; ++b) {
    if (!base.on[b]) continue;
    if (!cli[b]) return h->fail(ORCTM_E_ARG, "orctm_set_obc_ts: missing record of an open, sponged side");
    total += (size_t)(b < 2 ? JE : IE) * (size_t)KE;
  }
  {
    const int st0 = wait_all_uploads(h);
    if (st0) return st0;
  }
  if (total > h->obc_ts_cap[tracer]) {
    int st;
    double* p;
    if ((st = h->dev_alloc(&p, total))) return st;
    h->obc_ts_buf[tracer] = p;
    h->obc_ts_cap[tracer] = total;
  }
  // the previous record may still be read by queued launches
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  ObcArgs a = base;
  size_t off = 0;
  for (int b = 0; b < 4; ++b) {
    a.side[b] = ObcSide{nullptr, nullptr, 0, nullptr};
    if (!base.on[b]) continue;
    const int n = b < 2 ? JE : IE;
    const size_t cnt = (size_t)n * (size_t)KE;
    double* d = h->obc_ts_buf[tracer] + off;
    off += cnt;
    ORCTM_CUDA_OK(cudaMemcpy(d, cli[b], sizeof(double) * cnt, cudaMemcpyHostToDevice));
    a.side[b] = ObcSide{d, nullptr, n, ts_rates(h, tracer, b)};
  }
  h->obc_ts[tracer] = a;
  h->obc_ts_ready[tracer] = true;
  return ORCTM_OK;
}

int orctm_obc_ts(orctm_handle* h) {
  ORCTM_ENTER(h);
  if (!h->obc_ts_ready[0] && !h->obc_ts_ready[1])
    return h->fail(ORCTM_E_ARG, "orctm_obc_ts: orctm_set_obc_ts not called");
  int st;
  for (int n = 0; n < 2; ++n) {
    if (!h->obc_ts_ready[n]) continue;
    const int f = ORCTM_F_THO + n;
    if ((st = wait_uploads(h, {f})) || (st = own_buffer(h, f))) return st;
    launch_obc_ts(h->G, h->obc_ts[n], h->slot[f], h->stream);
    ORCTM_CUDA_OK(cudaGetLastError());
  }
  return ORCTM_OK;
}

int orctm_obc_eta(orctm_handle* h, int ldtrun) {
  ORCTM_ENTER(h);
  if (!h->obc_ready) return h->fail(ORCTM_E_ARG, "orctm_obc_eta: orctm_set_obc not called");
  int st;
  if ((st = wait_uploads(h, {ORCTM_F_ZO})) || (st = compute_after_copies(h))) return st;
  ObcArgs a = h->obc[0];
  a.t = (double)ldtrun * h->G.dt;  // mytime = i_step * DT
  launch_obc_eta(h->G, a, h->zo, h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  return ORCTM_OK;
}

int orctm_obc_uv(orctm_handle* h, int ldtrun) {
  ORCTM_ENTER(h);
  if (!h->obc_ready) return h->fail(ORCTM_E_ARG, "orctm_obc_uv: orctm_set_obc not called");
  int st;
  if ((st = wait_uploads(h, {ORCTM_F_UOO, ORCTM_F_VOE})) || (st = own_buffer(h, ORCTM_F_UOO)) ||
      (st = own_buffer(h, ORCTM_F_VOE)))
    return st;
  ObcArgs au = h->obc[1], av = h->obc[2];
  au.t = av.t = (double)ldtrun * h->G.dt;
  launch_obc_uv(h->G, au, av, h->slot[ORCTM_F_UOO], h->slot[ORCTM_F_VOE], h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  return ORCTM_OK;
}

// OBC_SPONGE_EXP: the band rates EXP(-4 L/Lsp)/TAO of SPONGE_OBCS_ETA_EXP,
// _UV_EXP and _TS_EXP (mo_obcs.f90:2588-3222), formed here once from the
// metrics: L is the length from the boundary cell to the band cell and Lsp
// the band's (INI_OBCS, mo_obcs.f90:508-522), both SUMs of DLX* (west, east)
// or DLY* (north, south) of the staggering in ascending index order, as the
// reference's SUM over its index ranges.
int orctm_set_obc_sponge_exp(orctm_handle* h, double tao) {
  ORCTM_ENTER(h);
  if (!h->obc_ready)
    return h->fail(ORCTM_E_ARG, "orctm_set_obc_sponge_exp: orctm_set_obc not called");
  if (!std::isfinite(tao)) return h->fail(ORCTM_E_ARG, "orctm_set_obc_sponge_exp: TAO must be finite");
  {
    const int st0 = wait_all_uploads(h);
    if (st0) return st0;
  }
  // the previous tables may still be read by queued launches
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  const int IE = h->L.ie, JE = h->L.je;
  auto apply = [&]() {
    for (int t = 0; t < 2; ++t) {
      h->obc_ts[t].expo = h->obc[0].expo;
      for (int b = 0; b < 4; ++b)
        if (h->obc_ts[t].on[b]) h->obc_ts[t].side[b].wexp = ts_rates(h, t, b);
    }
  };
  if (tao == 0.0) {  // back to the 1/x form
    for (ObcArgs& a : h->obc) {
      a.expo = 0;
      for (ObcSide& sd : a.side) sd.wexp = nullptr;
    }
    h->obc_exp_sao_south = nullptr;
    apply();
    return ORCTM_OK;
  }
  // DLXP, DLYP, DLXU, DLYU, DLXV, DLYV from their device copies (padded plane)
  const size_t n2 = (size_t)h->L.plane;
  std::vector<double> met[6];
  const double* dev[6] = {h->G.dlxp, h->G.dlyp, h->G.dlxu, h->G.dlyu, h->G.dlxv, h->G.dlyv};
  for (int m = 0; m < 6; ++m) {
    met[m].resize(n2);
    ORCTM_CUDA_OK(cudaMemcpy(met[m].data(), dev[m], sizeof(double) * n2, cudaMemcpyDeviceToHost));
  }
  const bool south = h->obc[0].on[3] != 0;
  size_t total = south ? (size_t)IE * (size_t)h->obc[0].width[3] : 0;
  for (int v = 0; v < 3; ++v)
    for (int b = 0; b < 4; ++b)
      if (h->obc[v].on[b]) total += (size_t)obc_points(h, b, v) * (size_t)h->obc[v].width[b];
  std::vector<double> tab(std::max<size_t>(total, 1));
  // the band length from the boundary cell to distance d of row q
  auto length = [&](int v, int b, int q, int d) {
    const int ilo = v == 1 ? 0 : 1, jlo = v == 2 ? 0 : 1;
    const std::vector<double>& dl = met[2 * v + (b < 2 ? 0 : 1)];
    int lo, hi;
    if (b == 0) lo = ilo, hi = ilo + d - 1;
    else if (b == 1) lo = IE - d + 1, hi = IE;
    else if (b == 2) lo = jlo, hi = jlo + d - 1;
    else lo = JE - d + 1, hi = JE;
    double L = 0.0;
    for (int x = lo; x <= hi; ++x)
      L = L + dl[b < 2 ? h->L.at2(x, q + jlo) : h->L.at2(q + ilo, x)];
    return L;
  };
  size_t off = 0;
  double* base = nullptr;
  if (total > h->obc_exp_cap) {
    int st;
    double* p;
    if ((st = h->dev_alloc(&p, total))) return st;
    h->obc_exp_buf = p;
    h->obc_exp_cap = total;
  }
  base = h->obc_exp_buf;
  const double* wptr[3][4] = {};
  for (int v = 0; v < 3; ++v)
    for (int b = 0; b < 4; ++b) {
      if (!h->obc[v].on[b]) continue;
      const int n = obc_points(h, b, v), w = h->obc[v].width[b];
      for (int q = 0; q < n; ++q) {
        const double lsp = length(v, b, q, w);
        if (!(lsp > 0.0)) return h->fail(ORCTM_E_ARG, "orctm_set_obc_sponge_exp: a sponge band's length is not positive");
        for (int d = 1; d <= w; ++d)
          tab[off + q + (size_t)n * (d - 1)] = std::exp(-(4.0 * length(v, b, q, d) / lsp)) / tao;
      }
      wptr[v][b] = base + off;
      off += (size_t)n * w;
    }
  const double* sao_south = nullptr;
  if (south) {
    // every row of SAO's band takes the rate of the band's innermost T cell
    const int w = h->obc[0].width[3];
    for (int q = 0; q < IE; ++q) {
      const double lsp = length(0, 3, q, w);
      const double r = std::exp(-(4.0 * length(0, 3, q, w) / lsp)) / tao;
      for (int d = 1; d <= w; ++d) tab[off + q + (size_t)IE * (d - 1)] = r;
    }
    sao_south = base + off;
    off += (size_t)IE * w;
  }
  if (total) ORCTM_CUDA_OK(cudaMemcpy(base, tab.data(), sizeof(double) * total, cudaMemcpyHostToDevice));
  for (int v = 0; v < 3; ++v) {
    h->obc[v].expo = 1;
    for (int b = 0; b < 4; ++b) h->obc[v].side[b].wexp = wptr[v][b];
  }
  h->obc_exp_sao_south = sao_south;
  apply();
  return ORCTM_OK;
}

// ------------------------------------------------------------ barotropic
int orctm_set_barotropic(orctm_handle* h, const orctm_barotropic* b) {
  ORCTM_ENTER(h);
  if (!b || !b->deuto || !b->deute)
    return h->fail(ORCTM_E_ARG, "orctm_set_barotropic: missing DEUTO or DEUTE");
  if (b->niter < 0 || !(b->sorpar > 0.0 && b->sorpar < 2.0) || !(b->grav > 0.0))
    return h->fail(ORCTM_E_ARG, "orctm_set_barotropic: niter >= 0, 0 < SORPAR < 2 and G > 0");
  const int IE = h->L.ie, JE = h->L.je;
  const size_t n2 = (size_t)h->L.plane;
  int st;
  {
    const int st0 = wait_all_uploads(h);
    if (st0) return st0;
  }
  if (!h->bf.xx) {
    double** all[] = {&h->bf.xx,  &h->bf.ff,     &h->bf.b1o, &h->bf.z1o, &h->bf.uf,
                      &h->bf.deutio, &h->bf.u1o, &h->bf.uzo, &h->bf.uso, &h->bf.vf,
                      &h->bf.deutie, &h->bf.v1e, &h->bf.vze, &h->bf.vse};
    for (double** p : all)
      if ((st = h->dev_alloc(p, n2))) return st;
  }
  // the depths pass through the two scratch slots of the transports
  if ((st = upload_2d(h, h->bf.u1o, b->deuto, 0, IE + 1, 1, JE)) ||
      (st = upload_2d(h, h->bf.v1e, b->deute, 1, IE, 0, JE + 1)))
    return st;
  BaroArgs a{b->grav, b->stabn, b->conn, b->rlsa1, b->sorpar, b->minvalue, b->niter, b->eta_forc ? 1 : 0};
  launch_itprep(h->G, a, h->bf.u1o, h->bf.v1e, h->bf, h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  // the new constants change the SOR launches: capture them again
  if (h->sor_graph) {
    ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
    cudaGraphExecDestroy(h->sor_graph);
    h->sor_graph = nullptr;
  }
  h->baro = a;
  h->baro_ready = true;
  return ORCTM_OK;
}

namespace {
int sor_graph(orctm_handle* h, cudaGraphExec_t* out) {
  if (h->sor_graph) {
    *out = h->sor_graph;
    return ORCTM_OK;
  }
  const unsigned long long before = launch_count();
  ORCTM_CUDA_OK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  for (int it = 0; it < h->baro.niter; ++it) {
    launch_sor(h->G, h->baro, h->bf, 0, h->stream);
    launch_sor(h->G, h->baro, h->bf, 1, h->stream);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e1 = cudaStreamEndCapture(h->stream, &g);
  add_launches(-(long long)(launch_count() - before));  // counted when the graph runs
  ORCTM_CUDA_OK(e1);
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e2 = cudaGraphInstantiate(&ex, g, 0ULL);
  cudaGraphDestroy(g);
  ORCTM_CUDA_OK(e2);
  h->sor_graph = *out = ex;
  return ORCTM_OK;
}
}  // namespace

int orctm_troneu(orctm_handle* h, const double* u1o, const double* v1e, const double* uzo,
                 const double* vze) {
  ORCTM_ENTER(h);
  if (!h->baro_ready) return h->fail(ORCTM_E_ARG, "orctm_troneu: orctm_set_barotropic not called");
  const bool host = u1o || v1e || uzo || vze;
  if (host && !(u1o && v1e && uzo && vze))
    return h->fail(ORCTM_E_ARG, "orctm_troneu: give all four arrays or none");
  const int IE = h->L.ie, JE = h->L.je;
  int st;
  if ((st = compute_after_copies(h))) return st;
  if (host && ((st = upload_2d(h, h->bf.u1o, u1o, 0, IE + 1, 1, JE)) ||
               (st = upload_2d(h, h->bf.uzo, uzo, 0, IE + 1, 1, JE)) ||
               (st = upload_2d(h, h->bf.v1e, v1e, 1, IE, 0, JE + 1)) ||
               (st = upload_2d(h, h->bf.vze, vze, 1, IE, 0, JE + 1))))
    return st;
  ORCTM_CUDA_OK(cudaMemsetAsync(h->bf.z1o, 0, sizeof(double) * (size_t)h->L.plane, h->stream));
  launch_troneu_rhs(h->G, h->baro, h->bf, h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  if (h->baro.niter > 0) {
    cudaGraphExec_t ex;
    if ((st = sor_graph(h, &ex))) return st;
    ORCTM_CUDA_OK(cudaGraphLaunch(ex, h->stream));
    add_launches(2LL * h->baro.niter);
  }
  return ORCTM_OK;
}

int orctm_ocvtro(orctm_handle* h) {
  ORCTM_ENTER(h);
  if (!h->baro_ready) return h->fail(ORCTM_E_ARG, "orctm_ocvtro: orctm_set_barotropic not called");
  int st;
  // ZO is updated in place: after its uploads, and after downloads queued before
  if ((st = wait_uploads(h, {ORCTM_F_ZO})) || (st = compute_after_copies(h))) return st;
  launch_ocvtro(h->G, h->baro, h->bf, h->zo, h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  return ORCTM_OK;
}

// TROTEST: the device runs the SOR trials; the host draws SQRTRND's
// sequence and sums the squared changes of the first and the last sweep of
// each trial in the reference's loop order, so SORPAR is the reference's
// choice bit for bit.
int orctm_trotest(orctm_handle* h, int ntry, int niter, double* sorpar_out) {
  ORCTM_ENTER(h);
  if (!h->baro_ready) return h->fail(ORCTM_E_ARG, "orctm_trotest: orctm_set_barotropic not called");
  if (ntry < 1 || niter < 1 || !sorpar_out) return h->fail(ORCTM_E_ARG, "orctm_trotest: arguments");
  const int IE = h->L.ie, JE = h->L.je;
  const size_t n2 = (size_t)h->L.plane;
  int st;
  if ((st = compute_after_copies(h))) return st;
  if (!h->trotest_buf && (st = h->dev_alloc(&h->trotest_buf, 4 * n2 + 1))) return st;
  double* d2 = h->trotest_buf;  // squared changes: first sweep, last sweep (2 colours each)
  double* sp = h->trotest_buf + 4 * n2;  // SORPAR of the trial
  // sqrtrnd.f90:1-8 in trotest.f90:43-55's order (II fastest)
  std::vector<double> rnd((size_t)IE * JE);
  double d = 0.34679201245;
  for (size_t k = 0; k < rnd.size(); ++k) {
    const double c = std::sqrt(34251. * d);
    d = c - (int)c;
    rnd[k] = d;
  }
  if ((st = upload_2d(h, h->bf.b1o, rnd.data(), 1, IE, 1, JE))) return st;
  launch_trotest_rhs(h->G, h->bf, h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  // one trial as a graph: niter sweeps, the first and last recording their changes
  const unsigned long long before = launch_count();
  ORCTM_CUDA_OK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  for (int k = 1; k <= niter; ++k)
    for (int c = 0; c < 2; ++c) {
      double* out = k == niter ? d2 + (2 + c) * n2 : (k == 1 ? d2 + c * n2 : nullptr);
      launch_sor_trial(h->G, h->bf, sp, out, c, h->stream);
    }
  cudaGraph_t g = nullptr;
  const cudaError_t e1 = cudaStreamEndCapture(h->stream, &g);
  const long long per_trial = (long long)(launch_count() - before);
  add_launches(-per_trial);
  ORCTM_CUDA_OK(e1);
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e2 = cudaGraphInstantiate(&ex, g, 0ULL);
  cudaGraphDestroy(g);
  ORCTM_CUDA_OK(e2);
  std::vector<double> first(2 * n2), last(2 * n2);
  auto serial = [&](const std::vector<double>& a) {  // trotest.f90:69-91 order
    double s = 0.;
    for (int c = 0; c < 2; ++c)
      for (int j = 2; j <= JE - 1; ++j)
        for (int i = (j + c) % 2 + 2; i <= IE - 1; i += 2) s = s + a[c * n2 + h->L.at2(i, j)];
    return s;
  };
  double sorpar = 1.75, convmin = 9.E99, sorpmin = sorpar;
  int rc = ORCTM_OK;
  for (int isor = 1; isor <= ntry && rc == ORCTM_OK; ++isor) {
    sorpar = sorpar + 0.001;
    cudaError_t e = cudaMemcpyAsync(sp, &sorpar, sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->bf.z1o, 0, sizeof(double) * n2, h->stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(ex, h->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(first.data(), d2, sizeof(double) * 2 * n2, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(last.data(), d2 + 2 * n2, sizeof(double) * 2 * n2, cudaMemcpyDeviceToHost,
                          h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
      rc = cuda_status(e);
      break;
    }
    add_launches(per_trial);
    const double chabas = serial(first), sumcha = niter == 1 ? chabas : serial(last);
    const double contric = sumcha / chabas;
    if (contric < convmin) {
      sorpmin = sorpar;
      convmin = contric;
    }
  }
  cudaGraphExecDestroy(ex);
  if (rc != ORCTM_OK) return rc;
  *sorpar_out = sorpmin;
  // TRONEU uses the chosen value from now on
  if (h->sor_graph) {
    cudaGraphExecDestroy(h->sor_graph);
    h->sor_graph = nullptr;
  }
  h->baro.sorpar = sorpmin;
  return ORCTM_OK;
}

int orctm_ocbarp(orctm_handle* h) {
  ORCTM_ENTER(h);
  if (!h->baro_ready) return h->fail(ORCTM_E_ARG, "orctm_ocbarp: orctm_set_barotropic not called");
  launch_ocbarp(h->G, h->bf, h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  return ORCTM_OK;
}

int orctm_ocwind(orctm_handle* h, const double* txo, const double* tye, const double* sicomu,
                 const double* sicomv, const double* tauwatu, const double* tauwatv) {
  ORCTM_ENTER(h);
  const bool host = txo || tye || sicomu || sicomv || tauwatu || tauwatv;
  if (host && !(txo && tye && sicomu && sicomv && tauwatu && tauwatv))
    return h->fail(ORCTM_E_ARG, "orctm_ocwind: give all six arrays or none");
  if (!host && !h->wind_ready)
    return h->fail(ORCTM_E_ARG, "orctm_ocwind: no forcing given yet");
  const int IE = h->L.ie, JE = h->L.je;
  int st;
  if (!h->wind.txo) {
    double** all[] = {&h->wind.txo, &h->wind.tye, &h->wind.sicomu, &h->wind.sicomv,
                      &h->wind.tauwatu, &h->wind.tauwatv};
    for (double** p : all)
      if ((st = h->dev_alloc(p, (size_t)h->L.plane))) return st;
  }
  if (host) {
    // the forcing of the previous call may still be read by queued launches
    ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
    if ((st = upload_2d(h, h->wind.txo, txo, 0, IE + 1, 1, JE)) ||
        (st = upload_2d(h, h->wind.tye, tye, 1, IE, 0, JE + 1)) ||
        (st = upload_2d(h, h->wind.sicomu, sicomu, 1, IE, 1, JE)) ||
        (st = upload_2d(h, h->wind.sicomv, sicomv, 1, IE, 1, JE)) ||
        (st = upload_2d(h, h->wind.tauwatu, tauwatu, 1, IE, 1, JE)) ||
        (st = upload_2d(h, h->wind.tauwatv, tauwatv, 1, IE, 1, JE)))
      return st;
    h->wind_ready = true;
  }
  // UOO and VOE are updated in place (level 1)
  if ((st = wait_uploads(h, {ORCTM_F_UOO, ORCTM_F_VOE})) || (st = own_buffer(h, ORCTM_F_UOO)) ||
      (st = own_buffer(h, ORCTM_F_VOE)))
    return st;
  launch_ocwind(h->G, h->wind, h->slot[ORCTM_F_UOO], h->slot[ORCTM_F_VOE], h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  return ORCTM_OK;
}

int orctm_ocvtot(orctm_handle* h) {
  ORCTM_ENTER(h);
  if (!h->baro_ready) return h->fail(ORCTM_E_ARG, "orctm_ocvtot: orctm_set_barotropic not called");
  {
    const int st0 = wait_all_uploads(h);  // rebinds slots
    if (st0) return st0;
  }
  int st;
  double *uo, *vo, *uk, *vk, *wo;
  if ((st = h->alloc(&uo)) || (st = h->alloc(&vo)) || (st = h->alloc(&uk)) ||
      (st = h->alloc(&vk)) || (st = h->alloc(&wo)))
    return st;
  launch_ocvtot(h->G, h->baro, h->bf.uso, h->bf.vse, h->slot[ORCTM_F_UOO], h->slot[ORCTM_F_VOE],
                h->slot[ORCTM_F_UKO], h->slot[ORCTM_F_VKE], uo, vo, uk, vk, wo, h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  h->bind(ORCTM_F_UOO, uo);
  h->bind(ORCTM_F_VOE, vo);
  h->bind(ORCTM_F_UKO, uk);
  h->bind(ORCTM_F_VKE, vk);
  h->bind(ORCTM_F_WO, wo);
  return ORCTM_OK;
}

int orctm_download_barotropic(orctm_handle* h, int which, double* host, size_t n) {
  ORCTM_ENTER(h);
  if (!h->baro_ready) return h->fail(ORCTM_E_ARG, "orctm_download_barotropic: not set up");
  const int IE = h->L.ie, JE = h->L.je;
  const double* src;
  int i0 = 1, ni = IE, j0 = 1, nj = JE;
  switch (which) {
    case ORCTM_B_Z1O: src = h->bf.z1o; break;
    case ORCTM_B_B1O: src = h->bf.b1o; break;
    case ORCTM_B_USO: src = h->bf.uso; i0 = 0; ni = IE + 1; break;
    case ORCTM_B_UZO: src = h->bf.uzo; i0 = 0; ni = IE + 1; break;
    case ORCTM_B_VSE: src = h->bf.vse; j0 = 0; nj = JE + 1; break;
    case ORCTM_B_VZE: src = h->bf.vze; j0 = 0; nj = JE + 1; break;
    case ORCTM_B_U1O: src = h->bf.u1o; i0 = 0; ni = IE + 1; break;
    case ORCTM_B_V1E: src = h->bf.v1e; j0 = 0; nj = JE + 1; break;
    default: return h->fail(ORCTM_E_ARG, "orctm_download_barotropic: unknown field");
  }
  if (!host || n != (size_t)ni * nj) return h->fail(ORCTM_E_ARG, "orctm_download_barotropic: size");
  ORCTM_CUDA_OK(cudaMemcpy2DAsync(host, sizeof(double) * ni, src + h->L.at2(i0, j0),
                                  sizeof(double) * h->L.P, sizeof(double) * ni, nj,
                                  cudaMemcpyDeviceToHost, h->stream));
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  return ORCTM_OK;
}

// ------------------------------------------- OCTHER, OCMODMOM, OCCLIT
int orctm_set_thermo(orctm_handle* h, const orctm_thermo* t) {
  ORCTM_ENTER(h);
  if (!t || !t->dbackv || !t->abackv)
    return h->fail(ORCTM_E_ARG, "orctm_set_thermo: missing DBACKV or ABACKV");
  if (t->eos != ORCTM_EOS_UNESCO && t->eos != ORCTM_EOS_LINEAR)
    return h->fail(ORCTM_E_ARG, "orctm_set_thermo: unknown equation of state");
  if (!(t->grav > 0.0)) return h->fail(ORCTM_E_ARG, "orctm_set_thermo: G must be positive");
  const int IE = h->L.ie, JE = h->L.je, KE = h->L.ke;
  const size_t n2 = (size_t)h->L.plane;
  int st;
  {
    const int st0 = wait_all_uploads(h);
    if (st0) return st0;
  }
  ThermoFields& f = h->tf;
  if (!f.po) {
    double *preff, *dbackv, *abackv, *wtd, *tiu, *tiw, *dz;
    if ((st = h->dev_alloc(&preff, KE)) || (st = h->dev_alloc(&dbackv, KE + 1)) ||
        (st = h->dev_alloc(&abackv, KE + 1)) || (st = h->dev_alloc(&wtd, KE)) ||
        (st = h->dev_alloc(&tiu, KE + 1)) || (st = h->dev_alloc(&tiw, KE + 1)) ||
        (st = h->dev_alloc(&dz, KE + 1)))
      return st;
    f.preff = preff; f.dbackv = dbackv; f.abackv = abackv; f.wtdecay = wtd;
    f.tiestu = tiu; f.tiestw = tiw; f.dz = dz;
    double* d2[10];
    for (double*& p : d2)
      if ((st = h->dev_alloc(&p, n2))) return st;
    f.sicomo = d2[0]; f.sictho = d2[1]; f.sicsno = d2[2]; f.relsao = d2[3]; f.reltho = d2[4];
    f.giriv = d2[5]; f.fu10 = d2[6]; f.eminpo = d2[7]; f.rivrun = d2[8]; f.kcondep = d2[9];
    const size_t n3 = (size_t)h->L.n3();
    if ((st = h->dev_alloc(&f.po, n3)) || (st = h->dev_alloc(&f.stabio, n3)) ||
        (st = h->dev_alloc(&f.rhoo, n3)) || (st = h->dev_alloc(&h->uk1o, n3)) ||
        (st = h->dev_alloc(&h->vk1e, n3)))
      return st;
    ORCTM_CUDA_OK(cudaHostAlloc((void**)&h->h_contra, sizeof(double), cudaHostAllocDefault));
  } else {
    // the tables of the previous call may still be read by queued launches
    ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  }
  // vertical tables: PREFF (0.1026 TIESTU unless given), DBACKV, ABACKV, the
  // wind-mixing decay EXP(-DZW(K)/WPENDEP) with WPENDEP = 40 (octher.f90:321,
  // 349), TIESTU, TIESTW and DZ (beleg.f90:87-105)
  std::vector<double> preff(KE), wtd(KE), dz(KE + 1);
  for (int k = 0; k < KE; ++k) preff[k] = t->preff ? t->preff[k] : 0.1026 * h->tiestu[k];
  for (int k = 0; k < KE; ++k) wtd[k] = std::exp(-h->dzw[k] / 40.);
  dz[0] = h->tiestu[0];
  for (int k = 1; k <= KE; ++k) dz[k] = h->tiestu[k] - h->tiestu[k - 1];
  auto up1 = [&](const double* dst, const double* src, int n) {
    return cudaMemcpyAsync((void*)dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream);
  };
  ORCTM_CUDA_OK(up1(f.preff, preff.data(), KE));
  ORCTM_CUDA_OK(up1(f.dbackv, t->dbackv, KE + 1));
  ORCTM_CUDA_OK(up1(f.abackv, t->abackv, KE + 1));
  ORCTM_CUDA_OK(up1(f.wtdecay, wtd.data(), KE));
  ORCTM_CUDA_OK(up1(f.tiestu, h->tiestu.data(), KE + 1));
  ORCTM_CUDA_OK(up1(f.tiestw, h->tiestw.data(), KE + 1));
  ORCTM_CUDA_OK(up1(f.dz, dz.data(), KE + 1));
  const double* src2[7] = {t->sicomo, t->sictho, t->sicsno, t->relsao, t->reltho, t->giriv, t->fu10};
  const double* dst2[7] = {f.sicomo, f.sictho, f.sicsno, f.relsao, f.reltho, f.giriv, f.fu10};
  for (int q = 0; q < 7; ++q) {
    if (src2[q]) {
      if ((st = upload_2d(h, (double*)dst2[q], src2[q], 1, IE, 1, JE))) return st;
    } else {
      ORCTM_CUDA_OK(cudaMemsetAsync((void*)dst2[q], 0, sizeof(double) * n2, h->stream));
    }
  }
  if (!h->thermo_ready) {  // KCONDEP as BODEN sets it (boden.f90:261): 1 wet, -99 land
    std::vector<double> kc((size_t)IE * JE);
    std::vector<int> kb((size_t)n2);
    ORCTM_CUDA_OK(cudaMemcpyAsync(kb.data(), h->G.gp.kb, sizeof(int) * n2, cudaMemcpyDeviceToHost,
                                  h->stream));
    ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
    for (int j = 1; j <= JE; ++j)
      for (int i = 1; i <= IE; ++i)
        kc[(size_t)(j - 1) * IE + (i - 1)] = kb[(size_t)h->L.at2(i, j)] >= 1 ? 1.0 : -99.0;
    if ((st = upload_2d(h, f.kcondep, kc.data(), 1, IE, 1, JE))) return st;
  }
  h->th = ThermoArgs{t->eos, t->rho0, t->drdt, t->drds, t->t0, t->s0, t->grav, t->relsal, t->reltem,
                     t->rhoicwa, t->rhosnwa, t->wt, t->cstabeps, t->dv0, t->av0, t->cavocon,
                     t->cdvocon};
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));  // the host vectors go out of scope
  h->thermo_ready = true;
  return ORCTM_OK;
}

int orctm_set_coriolis(orctm_handle* h, const orctm_coriolis* c) {
  ORCTM_ENTER(h);
  if (!c || !c->ftwou || !c->ftwov || !c->gila || !c->giph)
    return h->fail(ORCTM_E_ARG, "orctm_set_coriolis: missing array");
  const int IE = h->L.ie, JE = h->L.je;
  const size_t n2 = (size_t)h->L.plane;
  int st;
  if (!h->cf.dtfu) {
    double* p[10];
    for (double*& q : p)
      if ((st = h->dev_alloc(&q, n2))) return st;
    h->cf = CorFields{p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], p[9]};
  } else {
    ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  }
  // ocmodmom.f90:103-164 on the host (COS and SQRT of the host's library)
  const double dt = h->G.dt, almzer = h->G.almzer, omega = c->omega;
  auto gi = [&](const double* a, int ii, int jj) { return a[(size_t)(jj - 1) * (2 * IE) + (ii - 1)]; };
  std::vector<std::vector<double>> t(10, std::vector<double>(n2, 0.0));
  for (int j = 1; j <= JE; ++j)
    for (int i = 0; i <= IE; ++i) {
      const size_t ij = (size_t)h->L.at2(i, j);
      t[0][ij] = dt * c->ftwou[(size_t)(j - 1) * (IE + 1) + i];
      if (j >= 2 && j <= JE - 1 && i >= 1 && i <= IE - 1) {
        const double dlon = (gi(c->gila, 2 * i + 2, 2 * j) - gi(c->gila, 2 * i + 1, 2 * j)) *
                            std::cos(gi(c->gila, 2 * i + 1, 2 * j));
        const double dlat = gi(c->giph, 2 * i + 2, 2 * j) - gi(c->giph, 2 * i + 1, 2 * j);
        t[1][ij] = dt * (2 * omega * std::cos(gi(c->giph, 2 * i + 1, 2 * j)));
        t[2][ij] = dlon;
        t[3][ij] = std::sqrt(dlon * dlon + dlat * dlat) + almzer;
      }
    }
  for (int j = 0; j <= JE; ++j)
    for (int i = 1; i <= IE; ++i) {
      const size_t ij = (size_t)h->L.at2(i, j);
      t[4][ij] = dt * c->ftwov[(size_t)j * IE + (i - 1)];
      if (j >= 1 && j <= JE - 1 && i >= 2 && i <= IE - 1) {
        const double dlon = (gi(c->gila, 2 * i, 2 * j) - gi(c->gila, 2 * i, 2 * j + 1)) *
                            std::cos(gi(c->gila, 2 * i, 2 * j + 1));
        const double dlat = gi(c->giph, 2 * i, 2 * j) - gi(c->giph, 2 * i, 2 * j + 1);
        t[5][ij] = dt * (2 * omega * std::cos(gi(c->giph, 2 * i, 2 * j + 1)));
        t[6][ij] = dlon;
        t[7][ij] = std::sqrt(dlon * dlon + dlat * dlat) + almzer;
      }
    }
  for (int j = 2; j <= JE - 1; ++j)
    for (int i = 2; i <= IE - 1; ++i) {
      const size_t ij = (size_t)h->L.at2(i, j);
      const double dlon = (gi(c->gila, 2 * i + 1, 2 * j) - gi(c->gila, 2 * i, 2 * j)) *
                          std::cos(gi(c->gila, 2 * i, 2 * j));
      const double dlat = gi(c->giph, 2 * i, 2 * j - 1) - gi(c->giph, 2 * i, 2 * j);
      const double dist = std::sqrt(dlon * dlon + dlat * dlat) + almzer;
      const double ftwow1 = 2 * omega * std::cos(gi(c->giph, 2 * i, 2 * j));
      t[8][ij] = ftwow1 * dlon / dist;
      t[9][ij] = ftwow1 * dlat / dist;
    }
  const double* dst[10] = {h->cf.dtfu, h->cf.cu, h->cf.dlonu, h->cf.distu, h->cf.dtfv,
                           h->cf.cv,   h->cf.dlonv, h->cf.distv, h->cf.aw, h->cf.bw};
  for (int q = 0; q < 10; ++q)
    ORCTM_CUDA_OK(cudaMemcpyAsync((void*)dst[q], t[q].data(), sizeof(double) * n2,
                                  cudaMemcpyHostToDevice, h->stream));
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  h->cor_ready = true;
  return ORCTM_OK;
}

namespace {
int r_octher(orctm_handle* h) {
  int st;
  const int ft = ORCTM_F_THO, fs = ORCTM_F_THO + 1;
  if ((st = wait_uploads(h, {ft, fs, ORCTM_F_ZO, ORCTM_F_UKO, ORCTM_F_VKE, ORCTM_F_AVO, ORCTM_F_DVO})) ||
      (st = compute_after_copies(h)) || (st = own_buffer(h, ft)) || (st = own_buffer(h, fs)) ||
      (st = own_buffer(h, ORCTM_F_AVO)) || (st = own_buffer(h, ORCTM_F_DVO)))
    return st;
  launch_octher_surface(h->G, h->th, h->tf, h->slot[ft], h->slot[fs], h->zo, h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  // B: the T/S boundary forcing (octher.f90:113-121)
  for (int n = 0; n < 2; ++n) {
    if (!h->obc_ts_ready[n]) continue;
    launch_obc_ts(h->G, h->obc_ts[n], h->slot[ORCTM_F_THO + n], h->stream);
    ORCTM_CUDA_OK(cudaGetLastError());
  }
  launch_octher_column(h->G, h->th, h->tf, h->slot[ft], h->slot[fs], h->zo, h->slot[ORCTM_F_UKO],
                       h->slot[ORCTM_F_VKE], h->slot[ORCTM_F_AVO], h->slot[ORCTM_F_DVO], h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  return ORCTM_OK;
}

int r_ocmodmom(orctm_handle* h) {
  int st;
  {
    const int st0 = wait_all_uploads(h);
    if (st0) return st0;
  }
  if ((st = compute_after_copies(h)) || (st = own_buffer(h, ORCTM_F_UKO)) ||
      (st = own_buffer(h, ORCTM_F_VKE)) || (st = own_buffer(h, ORCTM_F_WNO)))
    return st;
  double *ub, *vb, *wb, *dw;
  if ((st = h->alloc(&ub)) || (st = h->alloc(&vb)) || (st = h->alloc(&wb)) || (st = h->alloc(&dw)))
    return st;
  launch_ocmodmom(h->G, h->baro, h->tf, h->cf, h->bf, h->zo, h->slot[ORCTM_F_UOO],
                  h->slot[ORCTM_F_VOE], h->slot[ORCTM_F_UKO], h->slot[ORCTM_F_VKE], h->uk1o,
                  h->vk1e, h->slot[ORCTM_F_WNO], ub, vb, wb, dw, h->stream);
  const cudaError_t e = cudaGetLastError();
  h->unref(ub);  // stream-ordered: a later user of the buffer runs after these launches
  h->unref(vb);
  h->unref(wb);
  h->unref(dw);
  ORCTM_CUDA_OK(e);
  return ORCTM_OK;
}

int r_occlit(orctm_handle* h) {
  int st;
  {
    const int st0 = wait_all_uploads(h);
    if (st0) return st0;
  }
  if ((st = compute_after_copies(h)) || (st = own_buffer(h, ORCTM_F_UKO)) ||
      (st = own_buffer(h, ORCTM_F_VKE)) || (st = own_buffer(h, ORCTM_F_WO)))
    return st;
  if (!h->occ_wpo) {
    const size_t n3 = (size_t)h->L.n3(), n2 = (size_t)h->L.plane;
    if ((st = h->dev_alloc(&h->occ_wpo, n3)) || (st = h->dev_alloc(&h->occ_t1o, n3)) ||
        (st = h->dev_alloc(&h->occ_bruva, n2)) || (st = h->dev_alloc(&h->occ_contrij, n2)) ||
        (st = h->dev_alloc(&h->occ_contra, 1)))
      return st;
  }
  launch_occlit(h->G, h->baro, h->tf, h->bf, h->slot[ORCTM_F_UKO], h->slot[ORCTM_F_VKE], h->uk1o,
                h->vk1e, h->slot[ORCTM_F_WO], h->occ_wpo, h->occ_t1o, h->occ_bruva,
                h->occ_contrij, h->occ_contra, h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  ORCTM_CUDA_OK(cudaMemcpyAsync(h->h_contra, h->occ_contra, sizeof(double), cudaMemcpyDeviceToHost,
                                h->stream));
  return ORCTM_OK;
}

// OCCLIT's check (occlit.f90:321-326), once the copy of CONTRA has landed
int contra_status(orctm_handle* h, double* contra) {
  const double c = *h->h_contra;
  if (contra) *contra = c;
  if (!(c <= 1.E-3)) return h->fail(ORCTM_E_UNSTABLE, "OCCLIT: CONTRA above 1e-3 (the reference aborts)");
  return ORCTM_OK;
}
}  // namespace

int orctm_octher(orctm_handle* h) {
  ORCTM_ENTER(h);
  if (!h->thermo_ready) return h->fail(ORCTM_E_ARG, "orctm_octher: orctm_set_thermo not called");
  return r_octher(h);
}

int orctm_ocmodmom(orctm_handle* h) {
  ORCTM_ENTER(h);
  if (!h->thermo_ready || !h->cor_ready || !h->baro_ready)
    return h->fail(ORCTM_E_ARG,
                   "orctm_ocmodmom: needs orctm_set_thermo, orctm_set_coriolis and orctm_set_barotropic");
  return r_ocmodmom(h);
}

int orctm_occlit(orctm_handle* h, double* contra) {
  ORCTM_ENTER(h);
  if (!h->thermo_ready || !h->baro_ready)
    return h->fail(ORCTM_E_ARG, "orctm_occlit: needs orctm_set_thermo and orctm_set_barotropic");
  int st;
  if ((st = r_occlit(h))) return st;
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  return contra_status(h, contra);
}

namespace {
// the baroclinic state arrays: device buffer, staggering and levels
int baroclinic_array(orctm_handle* h, int which, double** p, int* i0, int* ni, int* j0, int* nj,
                     int* nk) {
  const int IE = h->L.ie, JE = h->L.je, KE = h->L.ke;
  *i0 = 1; *ni = IE; *j0 = 1; *nj = JE; *nk = KE;
  switch (which) {
    case ORCTM_C_PO: *p = h->tf.po; break;
    case ORCTM_C_STABIO: *p = h->tf.stabio; break;
    case ORCTM_C_RHOO: *p = h->tf.rhoo; break;
    case ORCTM_C_UK1O: *p = h->uk1o; *i0 = 0; *ni = IE + 1; break;
    case ORCTM_C_VK1E: *p = h->vk1e; *j0 = 0; *nj = JE + 1; break;
    case ORCTM_C_EMINPO: *p = h->tf.eminpo; *nk = 1; break;
    case ORCTM_C_RIVRUN: *p = h->tf.rivrun; *nk = 1; break;
    case ORCTM_C_KCONDEP: *p = h->tf.kcondep; *nk = 1; break;
    default: return h->fail(ORCTM_E_ARG, "unknown baroclinic array");
  }
  return ORCTM_OK;
}
}  // namespace

int orctm_upload_baroclinic(orctm_handle* h, int which, const double* host, size_t n) {
  ORCTM_ENTER(h);
  if (!h->thermo_ready) return h->fail(ORCTM_E_ARG, "orctm_upload_baroclinic: orctm_set_thermo not called");
  double* p;
  int i0, ni, j0, nj, nk, st;
  if ((st = baroclinic_array(h, which, &p, &i0, &ni, &j0, &nj, &nk))) return st;
  if (!host || n != (size_t)ni * nj * nk) return h->fail(ORCTM_E_ARG, "orctm_upload_baroclinic: size");
  if ((st = compute_after_copies(h))) return st;
  for (int k = 0; k < nk; ++k)
    ORCTM_CUDA_OK(cudaMemcpy2DAsync(p + h->L.at(i0, j0, k), sizeof(double) * h->L.P,
                                    host + (size_t)k * ni * nj, sizeof(double) * ni,
                                    sizeof(double) * ni, nj, cudaMemcpyHostToDevice, h->stream));
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  return ORCTM_OK;
}

int orctm_download_baroclinic(orctm_handle* h, int which, double* host, size_t n) {
  ORCTM_ENTER(h);
  if (!h->thermo_ready) return h->fail(ORCTM_E_ARG, "orctm_download_baroclinic: orctm_set_thermo not called");
  double* p;
  int i0, ni, j0, nj, nk, st;
  if ((st = baroclinic_array(h, which, &p, &i0, &ni, &j0, &nj, &nk))) return st;
  if (!host || n != (size_t)ni * nj * nk) return h->fail(ORCTM_E_ARG, "orctm_download_baroclinic: size");
  for (int k = 0; k < nk; ++k)
    ORCTM_CUDA_OK(cudaMemcpy2DAsync(host + (size_t)k * ni * nj, sizeof(double) * ni,
                                    p + h->L.at(i0, j0, k), sizeof(double) * h->L.P,
                                    sizeof(double) * ni, nj, cudaMemcpyDeviceToHost, h->stream));
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  return ORCTM_OK;
}

// The routines of the step in the driver's order (orctm.f90:1454-1562)
// depend on one another through the velocities only: OCADPO and OCTDIFF
// read the transports UKO, VKE, WO the step starts with (and ZO, DVO), and
// nothing of the momentum path reads the tracers.  So the momentum path
// (OCUAD, OCVAD, OCWAD, OCTIMF, OCVISC, OCVTOT_NH, OCTIMF) runs first, on
// the momentum fields alone, and the tracer path after it on the held
// initial transports: the results are those of the driver's order bit for
// bit, while the tracers' uploads land during the momentum path and the
// momentum outputs download during the tracer path.
int orctm_step_hotpath(orctm_handle* h, orctm_solve_stats* s) {
  ORCTM_ENTER(h);
  int st;
  if ((st = r_momadv<0>(h)) || (st = r_momadv<1>(h)) || (st = r_momadv<2>(h))) return st;
  double* held[3] = {h->slot[ORCTM_F_UKO], h->slot[ORCTM_F_VKE], h->slot[ORCTM_F_WO]};
  for (double* p : held) h->refs[p]++;
  auto release = [&]() {
    for (double* p : held) h->unref(p);
  };
  if ((st = r_octimf(h)) || (st = r_ocvisc(h))) {
    release();
    return st;
  }
  const int ns = r_ocvtot_nh(h, s);
  if (ns != ORCTM_OK && ns != ORCTM_E_NOT_CONVERGED) {
    release();
    return ns;
  }
  r_octimf(h);
  // the momentum outputs are final: registered ones start downloading
  // while the tracers are advected and diffused
  if ((st = step_outputs(h, false))) {
    release();
    return st;
  }
  st = r_ocadpo_all(h, held[0], held[1], held[2]);  // OCADPO(THO), OCADPO(SAO), passive tracers
  release();  // stream-ordered: a later user of these buffers runs after OCADPO
  if (st || (st = r_octdiff(h)) || (st = step_outputs(h, true))) return st;
  return ns;
}

// One whole time step in the reference driver's order (orctm.f90:1327-1562):
// OCTHER, OCWIND, the open-boundary forcing, OCTIMF, OCMODMOM, OCBARP,
// OCCLIT, TRONEU, OCVTRO, OCVTOT, the STABIO rescaling, then the hot path.
// Nothing crosses to the host but the solve's scalars and OCCLIT's CONTRA.
int orctm_step_full(orctm_handle* h, int ldtrun, orctm_solve_stats* s, double* contra) {
  ORCTM_ENTER(h);
  if (!h->thermo_ready || !h->cor_ready || !h->baro_ready)
    return h->fail(ORCTM_E_ARG,
                   "orctm_step_full: needs orctm_set_thermo, orctm_set_coriolis and orctm_set_barotropic");
  int st;
  if ((st = r_octher(h))) return st;
  if (h->wind_ready && (st = orctm_ocwind(h, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr)))
    return st;
  if (h->obc_ready) {
    if (h->baro.eta_forc && (st = orctm_obc_eta(h, ldtrun))) return st;
    if ((st = orctm_obc_uv(h, ldtrun))) return st;
  }
  if ((st = r_octimf(h)) || (st = r_ocmodmom(h)) || (st = orctm_ocbarp(h)) || (st = r_occlit(h)))
    return st;
  cudaEvent_t contra_done = h->get_event();
  ORCTM_CUDA_OK(cudaEventRecord(contra_done, h->stream));
  if ((st = orctm_troneu(h, nullptr, nullptr, nullptr, nullptr)) || (st = orctm_ocvtro(h)) ||
      (st = orctm_ocvtot(h)))
    return st;
  launch_stabio_rescale(h->G, h->tf, h->stream);
  ORCTM_CUDA_OK(cudaGetLastError());
  const int ns = orctm_step_hotpath(h, s);
  if (ns != ORCTM_OK && ns != ORCTM_E_NOT_CONVERGED) return ns;
  ORCTM_CUDA_OK(cudaEventSynchronize(contra_done));  // long done: the solve waited on the host
  h->ev_pool.push_back(contra_done);
  const int cs = contra_status(h, contra);
  return ns != ORCTM_OK ? ns : cs;
}

int orctm_set_solver(orctm_handle* h, int mode, double rtol, int maxit) {
  if (!h || (mode != ORCTM_SOLVER_FP64 && mode != ORCTM_SOLVER_FP32_REFINED) || !(rtol > 0) ||
      maxit < 1)
    return ORCTM_E_ARG;
  h->solver_mode = mode;
  h->rtol = rtol;
  h->maxit = maxit;
  return ORCTM_OK;
}

int orctm_synchronize(orctm_handle* h) {
  ORCTM_ENTER(h);
  ORCTM_CUDA_OK(cudaStreamSynchronize(h->stream));
  ORCTM_CUDA_OK(cudaGetLastError());
  return ORCTM_OK;
}

int orctm_timer_start(orctm_handle* h) {
  ORCTM_ENTER(h);
  ORCTM_CUDA_OK(cudaEventRecord(h->tm0, h->stream));
  return ORCTM_OK;
}

int orctm_timer_stop(orctm_handle* h, double* ms) {
  ORCTM_ENTER(h);
  if (!ms) return ORCTM_E_ARG;
  ORCTM_CUDA_OK(cudaEventRecord(h->tm1, h->stream));
  ORCTM_CUDA_OK(cudaEventSynchronize(h->tm1));
  float f = 0.f;
  ORCTM_CUDA_OK(cudaEventElapsedTime(&f, h->tm0, h->tm1));
  *ms = f;
  return ORCTM_OK;
}

int orctm_set_profiling(orctm_handle* h, int on) {
  ORCTM_ENTER(h);
  h->prof_flush();
  for (int k = 0; k < ORCTM_PROF_KINDS; ++k) {
    h->prof_ms[k] = 0.0;
    h->prof_n[k] = 0;
  }
  h->prof = on != 0;
  return ORCTM_OK;
}

int orctm_profile_get(orctm_handle* h, int kind, long long* launches, double* total_ms) {
  ORCTM_ENTER(h);
  if (kind < 0 || kind >= ORCTM_PROF_KINDS || !launches || !total_ms) return ORCTM_E_ARG;
  h->prof_flush();
  *launches = h->prof_n[kind];
  *total_ms = h->prof_ms[kind];
  return ORCTM_OK;
}

unsigned long long orctm_kernel_launches(void) { return launch_count(); }

int orctm_set_tuning(orctm_handle* h, int col_variant, int spmv_variant) {
  if (!h || col_variant < -1 || col_variant >= pcg_col_variants() || spmv_variant < -1 ||
      spmv_variant >= pcg_spmv_variants())
    return ORCTM_E_ARG;
  h->force_col = col_variant;
  h->force_spmv = spmv_variant;
  for (int pr = 0; pr < 2; ++pr) h->col_var[pr] = h->spmv_var[pr] = -1;
  return ORCTM_OK;
}

int orctm_get_tuning(const orctm_handle* h, int precision, int* col_variant, int* spmv_variant) {
  if (!h || precision < 0 || precision > 1 || !col_variant || !spmv_variant) return ORCTM_E_ARG;
  *col_variant = h->col_var[precision];
  *spmv_variant = h->spmv_var[precision];
  return ORCTM_OK;
}

int orctm_device_bytes(const orctm_handle* h, unsigned long long* bytes) {
  if (!h || !bytes) return ORCTM_E_ARG;
  *bytes = h->bytes;
  return ORCTM_OK;
}

int orctm_estimate_device_bytes(const orctm_desc* d, int solver, unsigned long long* bytes) {
  if (!d || !bytes || d->ie < 4 || d->je < 3 || d->ke < 2 || d->ntracers < 2) return ORCTM_E_ARG;
  const double P = (double)(((long long)d->ie + 1 + 31) / 32 * 32);
  const double plane = P * (d->je + 1), n3 = plane * (d->ke + 1);
  // 3D buffers: 12 state fields and the tracers, the routine temporaries of
  // the field pool (at most max(8, 2 ntracers + 2), the advection of all
  // tracers at once, plus the step's initial transports held for it), 9
  // FP64 solver vectors, the FP64 + FP32 pivots, and 7
  // FP32 vectors for the refined solver
  const double tmp = std::max(8.0, 2.0 * d->ntracers + 2.0) + 3.0;  // + the held transports
  const double f3 = 12.0 + d->ntracers + tmp + 9.0 + 1.5 +
                    (solver == ORCTM_SOLVER_FP32_REFINED ? 3.5 : 0.0);
  // 2D tables (compressed columns, metrics, biharmonic and Poisson factors)
  const double f2 = 96.0;
  // every array carries two guard zones of about one plane
  const double guard = 2.0 * (plane + 2.0 * P + 64.0);
  *bytes = (unsigned long long)((f3 * (n3 + guard) + f2 * (plane + guard) + 16.0 * guard) * 8.0) +
           (1ULL << 20);
  return ORCTM_OK;
}

int orctm_trim_device_memory(int device) {
  cudaMemPool_t mp = nullptr;
  int st = device_pool(device, &mp);
  if (st) return st;
  ORCTM_CUDA_OK(cudaMemPoolTrimTo(mp, 0));
  return ORCTM_OK;
}

}  // extern "C"
