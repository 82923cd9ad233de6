// solar_gpu.cu -- context management and the C-ABI of include/solar_gpu.h.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <sched.h>

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/solar_gpu.h"
#include "kernels.cuh"
#include "tables.h"

namespace solar {

static_assert(SOLAR_KERNEL_EDGE == kInjEdge && SOLAR_KERNEL_STAGE == kInjStage && SOLAR_KERNEL_FILTER == kInjFilter &&
                  SOLAR_KERNEL_ADJ_STAGE == kInjAdjStage,
              "C-ABI kernel bits and device injection bits agree");

thread_local std::string g_last_error;

// Host threads of one context for the FP32 state uploads: run(f) calls f(t) for t = 0 ..
// size()-1, t = 0 on the calling thread, and returns when every call has returned.
class HostPool {
 public:
  explicit HostPool(int n) : n_(std::max(1, n)) {
    for (int t = 1; t < n_; ++t) th_.emplace_back([this, t] { loop(t); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> l(m_);
      quit_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  int size() const { return n_; }
  void run(const std::function<void(int)>& f) {
    {
      std::lock_guard<std::mutex> l(m_);
      f_ = &f;
      left_ = n_ - 1;
      ++gen_;
    }
    cv_.notify_all();
    f(0);
    std::unique_lock<std::mutex> l(m_);
    done_.wait(l, [this] { return left_ == 0; });
  }

 private:
  void loop(int t) {
    int seen = 0;
    for (;;) {
      const std::function<void(int)>* f;
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return gen_ != seen; });
        seen = gen_;
        if (quit_) return;
        f = f_;
      }
      (*f)(t);
      std::lock_guard<std::mutex> l(m_);
      if (--left_ == 0) done_.notify_one();
    }
  }
  int n_;
  std::vector<std::thread> th_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* f_ = nullptr;
  int gen_ = 0, left_ = 0;
  bool quit_ = false;
};

// Host cores this process may run on (its affinity mask), at most 16.
static int host_threads() {
  cpu_set_t set;
  int n = 1;
  if (sched_getaffinity(0, sizeof(set), &set) == 0) n = CPU_COUNT(&set);
  return std::min(16, std::max(1, n));
}

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

// Shared with the other translation units of the library.
int report_error(int code, const char* msg) { return fail(code, "%s", msg); }

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(SOLAR_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,              \
                  cudaGetErrorString(e_));                                                \
  } while (0)

struct DevTables {
  void* rad = nullptr;     // T [kNumRadial][nr]
  void* met = nullptr;     // T [kNumMetric][n][n]
  void* radT = nullptr;    // T [nr][16]   radial rows of one plane together (zero padded)
  void* conv = nullptr;    // T [3][4][n][n]
  void* ew = nullptr;      // T [6][4][3][9][n]     folded edge weights (scalar)
  void* eg = nullptr;      // T [6][4][3][9][2][n]  folded edge weights (vector)
  int* s0t = nullptr;      // [6][4][3][n]          first tap of every ghost point
  int* ewin = nullptr;     // [24][nseg] int2       edge-kernel staging window per edge segment
  int ewin_sp = 0, ewin_ts = 0, ewin_nseg = 0;
  void* egc = nullptr;     // T [6][4][3][9][2][2][n] curl halo weights (both components), on first use
  void* c2 = nullptr;      // T [6][nr][n][n] optional
  double* rad64 = nullptr; // FP64 copies for diagnostics
  double* vol2 = nullptr;  // [n][n]
  double* drw = nullptr;   // [nr]
  double* c2_64 = nullptr; // optional
  double* tanx = nullptr;  // [n]
  double* gr = nullptr;    // [nr]
};

// Device arrays of the discrete adjoint, allocated on first use (nruns == 1 only).
struct AdjBuffers {
  void* L = nullptr;        // lambda_q (padded state layout; frames hold ghost adjoints)
  void* LW = nullptr;       // lambda_w
  void* T1 = nullptr;       // filter-transpose scratch
  void* T2 = nullptr;
  void* rb = nullptr;       // R1, R2 of the one-sided radial rows (planes 1, 2, nr-3, nr-2)
  int* tspan = nullptr;     // ghost-point range of every source position (transposed exchange)
  void* wt = nullptr;       // T [3][72][wt_span][n] edge weights in the gather's order
  int wt_span = 0;
  double* grad = nullptr;   // dJ/dc, compact [face][k][j][i]
  void* ckpt = nullptr;     // state checkpoints (padded copies of the state buffer)
  size_t ckpt_bytes = 0;
  void* ckpt2 = nullptr;    // inner checkpoints of one outer segment (nested sweep)
  size_t ckpt2_bytes = 0;
  void* div = nullptr;      // stage-input divergences of one checkpoint segment
  size_t div_bytes = 0;
  void* clk = nullptr;      // source-term clocks of the checkpoints
  size_t clk_bytes = 0;
  double* traces = nullptr; // receiver traces and residuals
  size_t traces_bytes = 0;
  long long* rec_off = nullptr;
  double* rec_w = nullptr;
  int nrec = 0;
};

}  // namespace solar

using namespace solar;

struct solar_ctx {
  solar_desc desc;
  HostTables ht;
  Geom g;
  int fp32 = 0;
  size_t esize = 8;
  int device = 0;
  int nsm = 148;           // streaming multiprocessors of the device
  cudaStream_t stream = nullptr;
  void* A = nullptr;       // state
  void* B = nullptr;       // stage ping-pong
  void* W = nullptr;       // RK register qw
  double* stage64 = nullptr;   // one (face, field) compact FP64 volume
  double* part = nullptr;      // reduction partials
  double* red_out = nullptr;   // reduction result (device)
  int* run_order = nullptr;    // batched runs: stored runs, most steps first
  int run_count = 0;           // runs in the launched grids while a run map is in use
  int* err = nullptr;          // device words: [0] error code of a bounded wait that gave up,
                               // [1] step at which the watchdog first saw a non-finite value
  int inject_mask = 0;         // failure-injection tests: kernels that issue no loads ...
  uint32_t inject_polls = 0;   // ... and their wait bound
  int watch_every = 0;         // NaN/Inf watchdog: check the state every N steps (0 = off)
  long long steps_done = 0;    // steps taken by this context (watchdog step numbers)
  double* norm_ring = nullptr; // per-step sums of squares (solar_gpu_rk4_norms)
  int norm_ring_len = 0;
  DevTables dt;
  int tile_x = 32, tile_y = 8, kchunk = 0, edge_kchunk = 16;
  cudaGraphExec_t step_graph = nullptr;
  std::vector<cudaGraphExec_t> batch_graphs;   // batched step graph per number of live runs
  cudaEvent_t ev[8] = {};
  // FP32 contexts upload the state across PCIe as float: two pinned blocks of one compact
  // volume each, the events of their last copies, and the host threads that round the
  // caller's FP64 values into them (allocated on first use).
  float* pin32 = nullptr;
  cudaEvent_t xev[2] = {};
  std::unique_ptr<HostPool> pool;
  AdjBuffers adj;
  int forcing = 0;             // SOLAR_FORCING_*
  int force_nstep = 0, force_nt = 0;
  double force_cad = 0;        // forcing sample cadence, cadforcing (ic_acoustic_wave.f90:113)
  void* force_clock = nullptr;  // ForceClock (device)
  double* force_exy = nullptr;  // analytic: exp(-A^2 - B^2) [face][j][i]
  double* force_samples = nullptr;  // sampled: S_t [nt][face][j][i]
  void* force_xy = nullptr;     // this step's forcing field (kernel precision)
  void* force_r = nullptr;      // radial factor (kernel precision)
  int* split_items = nullptr;  // (zone, edge) pairs of one line pack/unpack
  int* split_slots = nullptr;  // slots exchanged per phase
};

namespace solar {

template <typename T>
static int upload(void** dst, const std::vector<double>& src) {
  std::vector<T> tmp(src.begin(), src.end());
  CK(cudaMalloc(dst, tmp.size() * sizeof(T)));
  CK(cudaMemcpy(*dst, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice));
  return SOLAR_OK;
}

template <typename T>
static int upload_tables(solar_ctx* c) {
  int rc;
  if ((rc = upload<T>(&c->dt.rad, c->ht.radial))) return rc;
  if ((rc = upload<T>(&c->dt.met, c->ht.metric))) return rc;
  {
    const int nr = c->ht.nr;
    std::vector<double> rt((size_t)nr * 16, 0.0);
    for (int k = 0; k < nr; ++k)
      for (int q = 0; q < kNumRadial; ++q) rt[(size_t)k * 16 + q] = c->ht.radial[(size_t)q * nr + k];
    if ((rc = upload<T>(&c->dt.radT, rt))) return rc;
  }
  if ((rc = upload<T>(&c->dt.ew, c->ht.ew))) return rc;
  if ((rc = upload<T>(&c->dt.eg, c->ht.eg))) return rc;
  return SOLAR_OK;
}

static int upload_constants() {
  double drp[4], bdy[3][7], filt[4], filtr[6];
  float drpf[4], bdyf[3][7], filtf[4], filtrf[6];
  for (int m = 0; m < 4; ++m) { drp[m] = kDrp[m]; drpf[m] = (float)kDrp[m]; }
  for (int r = 0; r < 3; ++r)
    for (int m = 0; m < 7; ++m) { bdy[r][m] = kBdy[r][m]; bdyf[r][m] = (float)kBdy[r][m]; }
  for (int m = 0; m < 4; ++m) { filt[m] = kFilt[m]; filtf[m] = (float)kFilt[m]; }
  for (int m = 0; m < 6; ++m) { filtr[m] = kFiltR[m]; filtrf[m] = (float)kFiltR[m]; }
  EdgeRouteDev rt[6][4];
  for (int f = 0; f < 6; ++f)
    for (int e = 0; e < 4; ++e) rt[f][e] = {kRoutes[f][e].src_face, kRoutes[f][e].src_edge, kRoutes[f][e].reversed};
  CK(cudaMemcpyToSymbol(cDrpD, drp, sizeof(drp)));
  CK(cudaMemcpyToSymbol(cBdyD, bdy, sizeof(bdy)));
  CK(cudaMemcpyToSymbol(cFiltD, filt, sizeof(filt)));
  CK(cudaMemcpyToSymbol(cFiltRD, filtr, sizeof(filtr)));
  CK(cudaMemcpyToSymbol(cDrpF, drpf, sizeof(drpf)));
  CK(cudaMemcpyToSymbol(cBdyF, bdyf, sizeof(bdyf)));
  CK(cudaMemcpyToSymbol(cFiltF, filtf, sizeof(filtf)));
  CK(cudaMemcpyToSymbol(cFiltRF, filtrf, sizeof(filtrf)));
  CK(cudaMemcpyToSymbol(cRoute, rt, sizeof(rt)));
  return SOLAR_OK;
}

// ---------------------------------------------------------------- launches
// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda needed).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Runs covered by a launch: all of them, or the first run_count entries of a run map.
static int launched_runs(const solar_ctx* c, const int* runs) { return runs ? c->run_count : c->g.nruns; }

// Wait control of one kernel kind (InjectKernel): the error word, the one-second bound,
// or the failure-injection settings when a test has switched them on for that kernel.
static WaitCtl wait_ctl(const solar_ctx* c, int kind) {
  WaitCtl w;
  w.err = c->err;
  const bool inj = (c->inject_mask & kind) != 0;
  w.polls = inj ? c->inject_polls : kWaitPolls;
  w.no_loads = inj ? 1 : 0;
  return w;
}

// Launch with programmatic stream serialization: the kernel starts as the previous kernel
// in the stream retires its last CTAs, does its constant-table prologue, and waits on the
// device (griddepcontrol.wait) before it touches anything that kernel wrote.  Used for the
// stepping kernels, which all wait before reading the state, so the completion of each
// implies that of the ones before.
template <typename Args>
static cudaError_t launch_pdl(void (*kernel)(Args), dim3 grid, dim3 block, size_t smem, cudaStream_t st, const Args& a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, a);
}

// 3-D view of a whole buffer: x = padded column, y = padded row, z = plane index
// ((run*6 + face)*nf + slot)*nr + k; box bx x by x 1.  The L2 fetches 256-byte blocks around
// each request (promotion) unless `promote` is false: boxes whose rows are only a few
// values wide (the edge kernel's column sources) would otherwise pull whole blocks of
// unused neighbours from DRAM for every row.
static bool make_map(const solar_ctx* c, const void* base, int bx, int by, CUtensorMap* m, bool promote = true) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  const Geom& g = c->g;
  cuuint64_t dims[3] = {(cuuint64_t)g.pitch, (cuuint64_t)g.rows, (cuuint64_t)g.nruns * 6 * g.nf * g.nr};
  cuuint64_t strides[2] = {(cuuint64_t)g.pitch * c->esize, (cuuint64_t)g.plane * c->esize};
  cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(m, c->fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                   const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE,
                   promote ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B : CU_TENSOR_MAP_L2_PROMOTION_NONE,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// A compact six-zone field [face][k][j][i] (c^2, stored divergences) as a 3-D array:
// x = i, y = j, z = face * nr + k; box bx x by x 1.
static bool make_compact_map(const solar_ctx* c, const void* base, int bx, int by, CUtensorMap* m) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  const Geom& g = c->g;
  cuuint64_t dims[3] = {(cuuint64_t)g.n, (cuuint64_t)g.n, (cuuint64_t)6 * g.nr};
  cuuint64_t strides[2] = {(cuuint64_t)g.n * c->esize, (cuuint64_t)g.n * g.n * c->esize};
  cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(m, c->fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                   const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Staging windows of the edge kernel: the receiving edge is cut into segments of ts
// positions (one thread per layer and position); a segment's ghost points read the source
// positions [min s0t, max s0t + 9), widened to whole 16-byte pieces.
static int edge_windows(solar_ctx* c) {
  const int n = c->g.n, w16 = c->fp32 ? 4 : 2;
  const int ts = std::min(n, 128), nseg = (n + ts - 1) / ts;
  std::vector<int> win((size_t)24 * nseg * 2);
  int sp = 0;
  for (int fe = 0; fe < 24; ++fe)
    for (int sg = 0; sg < nseg; ++sg) {
      int lo = n, hi = 0;
      for (int l = 0; l < 3; ++l)
        for (int t = sg * ts; t < std::min(n, (sg + 1) * ts); ++t) {
          const int s0 = c->ht.s0t[((size_t)fe * 3 + l) * n + t];
          lo = std::min(lo, s0);
          hi = std::max(hi, s0 + 9);
        }
      lo = lo / w16 * w16;
      hi = std::min(n, (hi + w16 - 1) / w16 * w16);
      win[((size_t)fe * nseg + sg) * 2 + 0] = lo;
      win[((size_t)fe * nseg + sg) * 2 + 1] = hi - lo;
      sp = std::max(sp, hi - lo);
    }
  c->dt.ewin_sp = (sp + 7) / 8 * 8;       // 128-byte aligned tiles in shared memory
  c->dt.ewin_ts = ts;
  c->dt.ewin_nseg = nseg;
  CK(cudaMalloc((void**)&c->dt.ewin, win.size() * sizeof(int)));
  CK(cudaMemcpy(c->dt.ewin, win.data(), win.size() * sizeof(int), cudaMemcpyHostToDevice));
  return SOLAR_OK;
}

template <typename T>
static int launch_edge(solar_ctx* c, void* buf, int mode, const int* runs) {
  EdgeArgs<T> a;
  a.q = (T*)buf;
  a.ew = (const T*)c->dt.ew;
  a.eg = (const T*)c->dt.eg;
  a.s0t = c->dt.s0t;
  a.runs = runs;
  a.win = (const int2*)c->dt.ewin;
  a.g = c->g;
  a.mode = mode;
  a.ts = c->dt.ewin_ts;
  a.nseg = c->dt.ewin_nseg;
  a.sp = c->dt.ewin_sp;
  a.ngroups = mode == 1 ? (c->g.nf + 1) / 2 : 2;
  // About one wave of resident CTAs, each marching at least 4 planes.
  const int nrl = launched_runs(c, runs);
  const long long per_chunk = 4LL * c->g.nface * a.ngroups * a.nseg * nrl;
  const long long slots = (long long)c->nsm * EdgeMinBlocks<T>::value;
  const long long nch = std::max<long long>(1, slots / per_chunk);
  const int nk = c->g.k1 - c->g.k0;
  a.kchunk = std::max<int>(4, (int)((nk + nch - 1) / nch));
  const size_t smem = (size_t)edge_smem_bytes(a.sp, a.ts, (int)sizeof(T));
  // a tile box side is at most 256 values; each thread spreads at most one row
  if (smem > 200 * 1024 || a.sp > 256 || 2 * a.sp > 3 * a.ts)
    return fail(SOLAR_ERR_ARG, "edge staging window of %d positions is too wide", a.sp);
  if (!make_map(c, buf, a.sp, 3, &a.mRow) || !make_map(c, buf, 4, a.sp, &a.mCol, false))
    return fail(SOLAR_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  a.wc = wait_ctl(c, kInjEdge);
  static bool attr_set = false;
  if (!attr_set) {
    CK(cudaFuncSetAttribute(edge_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr_set = true;
  }
  dim3 grid((nk + a.kchunk - 1) / a.kchunk, 4 * c->g.nface * a.ngroups * a.nseg, nrl);
  CK(launch_pdl(edge_kernel<T>, grid, dim3(3 * a.ts), smem, c->stream, a));
  return SOLAR_OK;
}

template <typename T, int TX, int TY, int MODE, bool HAS_RHO, bool FORCE = false>
static int launch_stage_t(solar_ctx* c, StageArgs<T>& a, const void* qin) {
  using L = StageLayout<T, TX, TY, HAS_RHO>;
  if (!make_map(c, qin, TX + 8, TY + 6, &a.mP) || !make_map(c, qin, TX + 8, TY, &a.mX) ||
      !make_map(c, qin, TX, TY + 6, &a.mY) || !make_map(c, qin, TX, TY, &a.mO) ||
      !make_map(c, c->W, TX, TY, &a.mW))
    return fail(SOLAR_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  static bool attr_set = false;
  if (!attr_set) {
    CK(cudaFuncSetAttribute(stage_kernel<T, TX, TY, MODE, HAS_RHO, FORCE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)L::TOTAL));
    attr_set = true;
  }
  const int nchunks = (c->g.k1 - c->g.k0 + a.kchunk - 1) / a.kchunk;
  const int ntiles = stage_tile_count(a.tsel, c->g.n / TX, c->g.n / TY);
  if (ntiles <= 0) return SOLAR_OK;                // no interior tiles at this size
  dim3 grid(ntiles, nchunks, launched_runs(c, a.runs) * c->g.nface);
  CK(launch_pdl(stage_kernel<T, TX, TY, MODE, HAS_RHO, FORCE>, grid, dim3(TX / Vec16<T>::V, TY), L::TOTAL, c->stream, a));
  return SOLAR_OK;
}

template <typename T, int TX, int TY>
static int launch_stage_mode(solar_ctx* c, StageArgs<T>& a, const void* qin, int mode) {
  const bool rho = c->g.slot[kRho] >= 0;
  if (a.force) {                    // forcing term (stepping and COMPUTE_RHS modes only)
    switch (mode) {
      case 0: return rho ? launch_stage_t<T, TX, TY, 0, true, true>(c, a, qin) : launch_stage_t<T, TX, TY, 0, false, true>(c, a, qin);
      case 1: return rho ? launch_stage_t<T, TX, TY, 1, true, true>(c, a, qin) : launch_stage_t<T, TX, TY, 1, false, true>(c, a, qin);
      case 2: return rho ? launch_stage_t<T, TX, TY, 2, true, true>(c, a, qin) : launch_stage_t<T, TX, TY, 2, false, true>(c, a, qin);
      case 4: return rho ? launch_stage_t<T, TX, TY, 4, true, true>(c, a, qin) : launch_stage_t<T, TX, TY, 4, false, true>(c, a, qin);
      case 5: return rho ? launch_stage_t<T, TX, TY, 5, true, true>(c, a, qin) : launch_stage_t<T, TX, TY, 5, false, true>(c, a, qin);
      default: return fail(SOLAR_ERR_ARG, "forcing is not available in stage mode %d", mode);
    }
  }
  switch (mode) {
    case 0: return rho ? launch_stage_t<T, TX, TY, 0, true>(c, a, qin) : launch_stage_t<T, TX, TY, 0, false>(c, a, qin);
    case 1: return rho ? launch_stage_t<T, TX, TY, 1, true>(c, a, qin) : launch_stage_t<T, TX, TY, 1, false>(c, a, qin);
    case 2: return rho ? launch_stage_t<T, TX, TY, 2, true>(c, a, qin) : launch_stage_t<T, TX, TY, 2, false>(c, a, qin);
    case 3: return rho ? launch_stage_t<T, TX, TY, 3, true>(c, a, qin) : launch_stage_t<T, TX, TY, 3, false>(c, a, qin);
    case 4: return rho ? launch_stage_t<T, TX, TY, 4, true>(c, a, qin) : launch_stage_t<T, TX, TY, 4, false>(c, a, qin);
    default: return rho ? launch_stage_t<T, TX, TY, 5, true>(c, a, qin) : launch_stage_t<T, TX, TY, 5, false>(c, a, qin);
  }
}

// Stage tiles (TX x TY points).  The default is 64 x 8 when nx is a multiple of 64 (the
// fastest shape measured at 64^3, 128^3 and 384^3 in both precisions), else 32 x 16 in
// float and 32 x 8 in double, and 16 x 16 when nx is not a multiple of 32.
static void default_tile(int n, bool fp32, int* tx, int* ty) {
  if (n % 32) { *tx = 16; *ty = 16; return; }
  if (n % 64 == 0) { *tx = 64; *ty = 8; return; }
  *tx = 32;
  *ty = fp32 ? 16 : 8;
}

template <typename T>
static int launch_stage(solar_ctx* c, const void* qin, void* qout, int mode, int stage,
                        const int* runs, void* divout = nullptr, int tsel = kTilesAll) {
  StageArgs<T> a;
  a.divout = (T*)divout;
  const bool forced = c->forcing && mode != 3;     // every mode but the gradient/divergence operator
  a.force = forced ? (const T*)c->force_xy : nullptr;
  a.force_r = forced ? (const T*)c->force_r : nullptr;
  a.qout = (T*)qout;
  a.qw = (T*)c->W;
  a.rad = (const T*)c->dt.rad;
  a.met = (const T*)c->dt.met;
  a.c2 = (const T*)c->dt.c2;
  a.runs = runs;
  a.wc = wait_ctl(c, kInjStage);
  a.g = c->g;
  a.dt = (T)c->desc.dt;
  a.alpha = (T)kAlpha[stage];
  a.beta = (T)kBeta[stage];
  a.inv_dxi = (T)(1.0 / c->ht.dxi);
  a.kchunk = c->kchunk;
  int tx = c->tile_x, ty = c->tile_y;
  if (mode == 2 || mode == 3) default_tile(c->g.n, c->fp32, &tx, &ty);   // operator-level calls
  // a face of fewer than 3 x 3 tiles has no interior tile: its ring is every tile
  const bool subsets = c->g.n / tx >= 3 && c->g.n / ty >= 3;
  a.tsel = subsets ? tsel : (tsel == kTilesInterior ? -1 : kTilesAll);
  if (a.tsel < 0) return SOLAR_OK;
  if (tx == 16 && ty == 16) return launch_stage_mode<T, 16, 16>(c, a, qin, mode);
  if (tx == 32 && ty == 8) return launch_stage_mode<T, 32, 8>(c, a, qin, mode);
  if (tx == 32 && ty == 16) return launch_stage_mode<T, 32, 16>(c, a, qin, mode);
  if (tx == 64 && ty == 8) return launch_stage_mode<T, 64, 8>(c, a, qin, mode);
  return fail(SOLAR_ERR_ARG, "unsupported stage tile %d x %d", tx, ty);
}

template <typename T, int TX, int TY, int R>
static int launch_filter_t(solar_ctx* c, const void* qin, void* qout, const int* runs) {
  using L = FilterLayout<T, TX, TY>;
  FilterArgs<T> a;
  if (!make_map(c, qin, TX + 8, TY + 6, &a.mP)) return fail(SOLAR_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  a.qout = (T*)qout;
  a.runs = runs;
  a.wc = wait_ctl(c, kInjFilter);
  a.g = c->g;
  static bool attr_set = false;
  static int resident = 1;
  const int threads = (TX / Vec16<T>::V) * (TY / R);
  if (!attr_set) {
    CK(cudaFuncSetAttribute(filter_kernel<T, TX, TY, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::TOTAL));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, filter_kernel<T, TX, TY, R>, threads, L::TOTAL));
    resident = std::max(resident, 1);
    attr_set = true;
  }
  // Whole-column CTAs for every full wave; the units of a last, partial wave are cut into
  // radial chunks (at least 11 planes each) so that they fill one wave.  When every unit
  // fits in one wave, SMs would hold units / nsm or one more whole column: the units past
  // an even share are cut into chunks, about one per SM, which run in the spare CTA slot
  // beside the whole columns (6 x 128^3 float: 740 columns and 140 chunks of 118 / 5
  // planes instead of 28 SMs with six columns).
  const long long units = (long long)(c->g.n / TX) * (c->g.n / TY) * c->g.nf * launched_runs(c, runs) * c->g.nface;
  const long long slots = (long long)c->nsm * resident;
  const long long nk = c->g.k1 - c->g.k0;
  a.whole = (int)units;
  a.chunks = 1;
  long long cut = 0, chunks = 1;
  if (units > slots) {
    cut = units % slots;
    if (cut > 0) chunks = std::min<long long>(nk / 11, std::max<long long>(1, (slots + cut / 2) / cut));
  } else {
    const long long per = units / c->nsm;
    cut = units % c->nsm;
    if (per >= 1 && per < resident && cut > 0) chunks = std::min<long long>(nk / 11, c->nsm / cut);
  }
  if (chunks > 1) {
    a.whole = (int)(units - cut);
    a.chunks = (int)chunks;
  }
  const long long grid = a.whole + (units - a.whole) * a.chunks;
  CK(launch_pdl(filter_kernel<T, TX, TY, R>, dim3((unsigned)grid), dim3(TX / Vec16<T>::V, TY / R), L::TOTAL, c->stream, a));
  return SOLAR_OK;
}

template <typename T>
static int launch_filter(solar_ctx* c, const void* qin, void* qout, const int* runs) {
  // Rows per thread: float keeps one row per thread (four warps of 91 registers, five CTAs
  // to an SM); double takes two, which reads 6 rows of shared memory for 2 output rows
  // (measured at 6 x 128^3: float 100 us with R = 1, 114-119 us with R = 2; double 250 us
  // with R = 2, 282 us with R = 1).
  constexpr int R = sizeof(T) == 4 ? 1 : 2;
  if (c->g.n % 32 == 0) return launch_filter_t<T, 32, 16, R>(c, qin, qout, runs);
  return launch_filter_t<T, 16, 16, R>(c, qin, qout, runs);
}

static int force_begin(solar_ctx* c);   // forcing.cuh: this step's source field
static int force_end(solar_ctx* c);     // forcing.cuh: time += dt, step += 1

// One full time step (timestep.f90:61-82) on every run.  With ev != nullptr each kernel
// is bracketed by events: ev_pairs[kind] accumulates into times[kind].
template <typename T>
static int enqueue_step(solar_ctx* c, const int* runs, std::vector<cudaEvent_t>* evs) {
  void* bufs[2] = {c->A, c->B};
  int cur = 0, rc;
  if ((rc = force_begin(c))) return rc;
  auto mark = [&]() {
    if (!evs) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, c->stream);
    evs->push_back(e);
  };
  for (int s = 0; s < 5; ++s) {
    mark();
    if ((rc = launch_edge<T>(c, bufs[cur], 0, runs))) return rc;
    mark();
    if ((rc = launch_stage<T>(c, bufs[cur], bufs[cur ^ 1], s == 0 ? 1 : 0, s, runs))) return rc;
    mark();
    cur ^= 1;
  }
  mark();
  if ((rc = launch_edge<T>(c, bufs[cur], 1, runs))) return rc;
  mark();
  if ((rc = launch_filter<T>(c, bufs[cur], bufs[cur ^ 1], runs))) return rc;
  mark();
  return force_end(c);
}

static int enqueue_step_any(solar_ctx* c, const int* runs, std::vector<cudaEvent_t>* evs) {
  return c->fp32 ? enqueue_step<float>(c, runs, evs) : enqueue_step<double>(c, runs, evs);
}

static const char* device_error_name(int code) {
  switch (code) {
    case kErrStageLead: return "stage kernel, lead ring";
    case kErrStageTile: return "stage kernel, tile ring";
    case kErrFilterRing: return "filter kernel";
    case kErrEdgeRing: return "edge kernel";
    case kErrAdjointRing: return "transposed stage kernel";
    default: return "unknown kernel";
  }
}

// Device words: [0] set by a kernel whose bounded wait gave up (or by the forcing sampler),
// [1] the step at which the watchdog first saw a non-finite value.  Both are cleared once
// read.
static int check_device_error(solar_ctx* c) {
  int h[2] = {0, 0};
  CK(cudaMemcpyAsync(h, c->err, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (h[0] || h[1]) {
    CK(cudaMemsetAsync(c->err, 0, 2 * sizeof(int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  if (h[0] == kErrForcingSample) return fail(SOLAR_ERR_ARG, "forcing: a time sample outside the loaded samples was needed");
  if (h[0]) return fail(SOLAR_ERR_TIMEOUT, "a device wait gave up (code %d: %s)", h[0], device_error_name(h[0]));
  if (h[1]) return fail(SOLAR_ERR_NAN, "watchdog: non-finite value in the state after step %d of this context", h[1]);
  return SOLAR_OK;
}

// NaN/Inf watchdog: count one step of the context and, every watch_every steps, enqueue a
// scan of the state buffer (no host wait; check_device_error reports it).
static int watch_after_step(solar_ctx* c) {
  ++c->steps_done;
  if (c->watch_every <= 0 || c->steps_done % c->watch_every) return SOLAR_OK;
  const Geom& g = c->g;
  const int V = c->fp32 ? 4 : 2;
  const long long nv = g.vs / V;
  const unsigned bx = (unsigned)std::max<long long>(1, std::min<long long>(64, (nv + 2047) / 2048));
  const dim3 grid(bx, (unsigned)(g.nruns * g.nface * g.nf));
  const int step = (int)std::min<long long>(c->steps_done, 0x7fffffff);
  if (c->fp32) nonfinite_kernel<float><<<grid, 256, 0, c->stream>>>((const float*)c->A, g, step, c->err + 1);
  else nonfinite_kernel<double><<<grid, 256, 0, c->stream>>>((const double*)c->A, g, step, c->err + 1);
  CK(cudaGetLastError());
  return SOLAR_OK;
}

static int capture_step_graph(solar_ctx* c) {
  if (c->step_graph) return SOLAR_OK;
  cudaGraph_t graph;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step_any(c, nullptr, nullptr);
  cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
  if (rc) return rc;
  CK(ce);
  CK(cudaGraphInstantiate(&c->step_graph, graph, 0));
  CK(cudaGraphDestroy(graph));
  return SOLAR_OK;
}

// Step graph over the first `live` runs of run_order (the runs with the most steps left).
static int capture_batch_graph(solar_ctx* c, int live) {
  if ((int)c->batch_graphs.size() < c->g.nruns + 1) c->batch_graphs.resize(c->g.nruns + 1, nullptr);
  if (c->batch_graphs[live]) return SOLAR_OK;
  cudaGraph_t graph;
  c->run_count = live;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step_any(c, c->run_order, nullptr);
  cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
  c->run_count = 0;
  if (rc) return rc;
  CK(ce);
  CK(cudaGraphInstantiate(&c->batch_graphs[live], graph, 0));
  CK(cudaGraphDestroy(graph));
  return SOLAR_OK;
}

static void drop_batch_graphs(solar_ctx* c) {
  for (auto& gx : c->batch_graphs)
    if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
}

// ---------------------------------------------------------------- transfers
static long long vol_compact(const solar_ctx* c) { return (long long)c->g.n * c->g.n * c->g.nr; }

// FP32 transfers: the pinned blocks, their events and the host threads, on first use.
static int ensure_pin32(solar_ctx* c) {
  if (c->pin32) return SOLAR_OK;
  const size_t bytes = (size_t)2 * vol_compact(c) * sizeof(float);
  CK(cudaHostAlloc((void**)&c->pin32, bytes, cudaHostAllocDefault));
  for (auto& e : c->xev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  c->pool.reset(new HostPool(host_threads()));
  return SOLAR_OK;
}

// The slice [lo, hi) of n items that host thread t of p handles.
static void slice(long long n, int t, int p, long long* lo, long long* hi) {
  *lo = n * t / p;
  *hi = n * (t + 1) / p;
}

// FP32 context: each compact volume is rounded to float on the host (round to nearest even,
// as the device conversion does, so the stored state is the same bit for bit) into one of
// two pinned blocks while the previous block is copied, then copied (half the bytes of
// FP64) and placed in the padded layout on the device.  (Reading back as float and
// widening on the host was slower than copying FP64 at C2: 14.6 ms against 9.0 ms for
// the 403 MB state; uploading this way takes 6.2 ms against 7.9 ms.)
static int upload_fields32(solar_ctx* c, void* buf, int run, const double* host, int nh,
                           const int* fields, int nfields_h) {
  int rc;
  if ((rc = ensure_pin32(c))) return rc;
  const long long V = vol_compact(c);
  const int threads = 256;
  const int blocks = (int)((V + threads - 1) / threads);
  float* dev = reinterpret_cast<float*>(c->stage64);          // two blocks of V floats
  HostPool& pool = *c->pool;
  int q = 0;
  for (int z = 0; z < 6; ++z)
    for (int m = 0; m < nfields_h; ++m) {
      const int s = c->g.slot[fields[m]];
      if (s < 0) continue;
      const int b = q & 1;
      if (q >= 2) CK(cudaEventSynchronize(c->xev[b]));       // the copy out of block b is done
      const double* src = host + ((long long)z * nh + m) * V;
      float* pin = c->pin32 + b * V;
      pool.run([&](int t) {
        long long lo, hi;
        slice(V, t, pool.size(), &lo, &hi);
        for (long long k = lo; k < hi; ++k) pin[k] = (float)src[k];
      });
      CK(cudaMemcpyAsync(dev + b * V, pin, V * sizeof(float), cudaMemcpyHostToDevice, c->stream));
      CK(cudaEventRecord(c->xev[b], c->stream));
      unpack_f32_kernel<<<blocks, threads, 0, c->stream>>>(dev + b * V, (float*)buf + c->g.vol(run, z, s), c->g);
      CK(cudaGetLastError());
      ++q;
    }
  return SOLAR_OK;
}

// Host six-zone field(s) -> device padded slot volumes of `buf`, for run `run`.
// `fields` lists the reference fields present in the host array in order; the host array
// holds nh fields per zone (5 for a state, 1 for a single field).
static int upload_fields(solar_ctx* c, void* buf, int run, const double* host, int nh,
                         const int* fields, int nfields_h) {
  if (c->fp32) return upload_fields32(c, buf, run, host, nh, fields, nfields_h);
  const long long V = vol_compact(c);
  const int threads = 256;
  const int blocks = (int)((V + threads - 1) / threads);
  for (int z = 0; z < 6; ++z)
    for (int m = 0; m < nfields_h; ++m) {
      const int f = fields[m];
      const int s = c->g.slot[f];
      if (s < 0) continue;
      CK(cudaMemcpyAsync(c->stage64, host + ((long long)z * nh + m) * V, V * sizeof(double),
                         cudaMemcpyHostToDevice, c->stream));
      const long long off = c->g.vol(run, z, s);
      if (c->fp32) unpack_kernel<float><<<blocks, threads, 0, c->stream>>>(c->stage64, (float*)buf + off, c->g);
      else unpack_kernel<double><<<blocks, threads, 0, c->stream>>>(c->stage64, (double*)buf + off, c->g);
      CK(cudaGetLastError());
    }
  return SOLAR_OK;
}

static int download_fields(solar_ctx* c, const void* buf, int run, double* host, int nh,
                           const int* fields, int nfields_h) {
  const long long V = vol_compact(c);
  const int threads = 256;
  const int blocks = (int)((V + threads - 1) / threads);
  for (int z = 0; z < 6; ++z)
    for (int m = 0; m < nfields_h; ++m) {
      const int f = fields[m];
      const int s = c->g.slot[f];
      double* dst = host + ((long long)z * nh + m) * V;
      if (s < 0) {                     // a field the context does not store reads back as zero
        std::memset(dst, 0, (size_t)V * sizeof(double));
        continue;
      }
      if (c->fp32) pack_kernel<float><<<blocks, threads, 0, c->stream>>>((const float*)buf + c->g.vol(run, z, s), c->stage64, c->g);
      else pack_kernel<double><<<blocks, threads, 0, c->stream>>>((const double*)buf + c->g.vol(run, z, s), c->stage64, c->g);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(dst, c->stage64, V * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
  CK(cudaStreamSynchronize(c->stream));
  return SOLAR_OK;
}

static const int kAllFields[5] = {kRho, kVxi, kVeta, kVr, kP};

static int check_ctx(solar_ctx* c) {
  if (!c) return fail(SOLAR_ERR_STATE, "null context");
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fail(SOLAR_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  return SOLAR_OK;
}

static int reduce(solar_ctx* c, int run, int sel_field, double* out5) {
  const int nblocks = c->g.nface * (c->g.k1 - c->g.k0);
  const int sel = (sel_field >= 0 && sel_field < 5) ? c->g.slot[sel_field] : -1;
  if (c->fp32)
    reduce_plane_kernel<float><<<nblocks, 256, 0, c->stream>>>((const float*)c->A, c->g, run, sel, c->dt.rad64,
                                                               c->dt.vol2, c->dt.drw, c->dt.c2_64, c->part);
  else
    reduce_plane_kernel<double><<<nblocks, 256, 0, c->stream>>>((const double*)c->A, c->g, run, sel, c->dt.rad64,
                                                                c->dt.vol2, c->dt.drw, c->dt.c2_64, c->part);
  CK(cudaGetLastError());
  reduce_final_kernel<<<1, 256, 0, c->stream>>>(c->part, nblocks, c->red_out);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out5, c->red_out, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SOLAR_OK;
}

// Sum of squares of reference field sel_field (0-based) of one run over the owned zones;
// zero for a field the context does not store.
static int sumsq(solar_ctx* c, int run, int sel_field, double* out) {
  const int s = c->g.slot[sel_field];
  if (s < 0) { *out = 0.0; return SOLAR_OK; }
  const int nblocks = c->g.nface * (c->g.k1 - c->g.k0);
  if (c->fp32) sumsq_plane_kernel<float><<<nblocks, 256, 0, c->stream>>>((const float*)c->A, c->g, run, s, c->part);
  else sumsq_plane_kernel<double><<<nblocks, 256, 0, c->stream>>>((const double*)c->A, c->g, run, s, c->part);
  CK(cudaGetLastError());
  sumsq_final_kernel<<<1, 256, 0, c->stream>>>(c->part, nblocks, c->red_out);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, c->red_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SOLAR_OK;
}

}  // namespace solar

// ===================================================================== C-ABI
extern "C" {

void solar_desc_defaults(solar_desc* d) {
  if (!d) return;
  std::memset(d, 0, sizeof(*d));
  d->precision = SOLAR_FP64;
  d->nfields = 5;
  d->nruns = 1;
  d->sponge_amp = 0.1;
  d->sponge_exp = 3.0;
  d->sponge_len = 30;
  d->sponge_lower = 1;
  d->sponge_upper = 1;
}

int solar_gpu_abi_version(void) { return SOLAR_GPU_ABI_VERSION; }

int solar_gpu_device_name(int device, char* buf, int len) {
  if (!buf || len <= 0) return fail(SOLAR_ERR_ARG, "null buffer");
  cudaDeviceProp p;
  cudaError_t e = cudaGetDeviceProperties(&p, device);
  if (e != cudaSuccess) return fail(SOLAR_ERR_CUDA, "cudaGetDeviceProperties: %s", cudaGetErrorString(e));
  std::snprintf(buf, (size_t)len, "%s", p.name);
  return SOLAR_OK;
}

int solar_gpu_last_error(char* buf, int len) {
  if (!buf || len <= 0) return SOLAR_ERR_ARG;
  std::snprintf(buf, (size_t)len, "%s", solar::g_last_error.c_str());
  return SOLAR_OK;
}

int solar_gpu_finalize(solar_ctx* c) {
  if (!c) return SOLAR_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
  drop_batch_graphs(c);
  void* ptrs[] = {c->A, c->B, c->W, c->stage64, c->part, c->red_out, c->run_order,
                  c->err, c->dt.rad, c->dt.met, c->dt.radT, c->dt.ew, c->dt.eg, c->dt.egc, c->dt.s0t, c->dt.ewin, c->dt.c2,
                  c->dt.rad64, c->dt.vol2, c->dt.drw, c->dt.c2_64, c->dt.tanx, c->dt.gr};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  void* aptrs[] = {c->adj.L, c->adj.LW, c->adj.T1, c->adj.T2, c->adj.rb, c->adj.tspan, c->adj.wt, c->adj.grad, c->adj.ckpt, c->adj.ckpt2,
                   c->adj.div, c->adj.traces, c->adj.rec_off, c->adj.rec_w, c->adj.clk, c->split_items, c->split_slots,
                   c->force_clock, c->force_exy, c->force_samples, c->force_xy, c->force_r, c->norm_ring};
  for (void* p : aptrs)
    if (p) cudaFree(p);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : c->xev)
    if (e) cudaEventDestroy(e);
  if (c->pin32) cudaFreeHost(c->pin32);
  c->pool.reset();
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return SOLAR_OK;
}

int solar_gpu_init(const solar_desc* d, solar_ctx** out) {
  if (!d || !out) return fail(SOLAR_ERR_ARG, "null descriptor or output pointer");
  *out = nullptr;
  if (d->precision != SOLAR_FP64 && d->precision != SOLAR_FP32) return fail(SOLAR_ERR_ARG, "precision must be SOLAR_FP64 or SOLAR_FP32");
  if (d->nfields != 5 && d->nfields != 4) return fail(SOLAR_ERR_ARG, "nfields must be 4 or 5");
  if (d->nruns < 1) return fail(SOLAR_ERR_ARG, "nruns must be >= 1");
  if (!(d->dt > 0.0)) return fail(SOLAR_ERR_ARG, "dt must be > 0");
  solar_ctx* c = new solar_ctx();
  c->desc = *d;
  std::string err;
  int rc = build_tables(*d, c->ht, err);
  if (rc) { delete c; return fail(rc, "%s", err.c_str()); }
  if (d->nfields == 4)
    for (int k = 0; k < d->nr; ++k)
      if (c->ht.g0[k] != 0.0) { delete c; return fail(SOLAR_ERR_ARG, "nfields = 4 drops rho, which needs g0 == 0"); }
  c->device = d->device;
  cudaError_t ce = cudaSetDevice(c->device);
  if (ce != cudaSuccess) { delete c; return fail(SOLAR_ERR_CUDA, "cudaSetDevice(%d): %s", d->device, cudaGetErrorString(ce)); }
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device);
  c->fp32 = d->precision == SOLAR_FP32;
  c->esize = c->fp32 ? 4 : 8;
  Geom& g = c->g;
  g.n = d->nx;
  g.nr = d->nr;
  g.nf = d->nfields;
  g.pitch = d->nx + 2 * IOFF;
  g.rows = d->nx + 2 * JOFF;
  g.plane = (long long)g.pitch * g.rows;
  g.vs = g.plane * g.nr;   // volumes back to back: the whole buffer is one 3-D array of planes
  g.nruns = d->nruns;
  g.face0 = 0;
  g.nface = 6;
  g.k0 = 0;
  g.k1 = g.nr;
  if (g.nf == 5) { for (int f = 0; f < 5; ++f) g.slot[f] = f; }
  else { g.slot[kRho] = -1; g.slot[kVxi] = 0; g.slot[kVeta] = 1; g.slot[kVr] = 2; g.slot[kP] = 3; }
  // tile choice (16x16, 32x8, 32x16, 64x8)
  default_tile(g.n, c->fp32, &c->tile_x, &c->tile_y);
  if (d->tile_x) c->tile_x = d->tile_x;
  if (d->tile_y) c->tile_y = d->tile_y;
  {
    const int tx = c->tile_x, ty = c->tile_y;
    const bool known = (tx == 16 && ty == 16) || (tx == 32 && (ty == 8 || ty == 16)) || (tx == 64 && ty == 8);
    if (!known || g.n % tx || g.n % ty) {
      const int nx = g.n;          // g refers into c
      delete c;
      return fail(SOLAR_ERR_ARG, "unsupported stage tile %d x %d for nx %d", tx, ty, nx);
    }
  }
  if (d->kchunk > 0) c->kchunk = d->kchunk;
  else {
    // Radial planes per stage CTA.  Measured best on B200: about nr/3 in float and nr/6 in
    // double, between 16 and 64 (43 / 22 at 128^3, 64 at 384^3, ~21 at 64 runs of 64^3).
    // Grids too small to fill one wave of two CTAs per SM that way get about four waves.
    const long long blocks = 6LL * g.nruns * (g.n / c->tile_x) * (g.n / c->tile_y);
    int kc = std::min(64, std::max(16, c->fp32 ? g.nr / 3 : g.nr / 6));
    int nch = (g.nr + kc - 1) / kc;
    if (blocks * nch < 148LL * 2) {
      const long long want = 148LL * 2 * 4;
      nch = (int)std::max<long long>(1, (want + blocks - 1) / blocks);
      c->kchunk = std::max(8, (g.nr + nch - 1) / nch);
    } else {
      c->kchunk = (g.nr + nch - 1) / nch;
    }
  }
#define TRY(x) do { int rc_ = (x); if (rc_) { solar_gpu_finalize(c); return rc_; } } while (0)
#define TRYC(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { std::string m_ = cudaGetErrorString(e_); solar_gpu_finalize(c); return fail(e_ == cudaErrorMemoryAllocation ? SOLAR_ERR_NOMEM : SOLAR_ERR_CUDA, "%s: %s", #call, m_.c_str()); } } while (0)
  TRYC(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  const size_t bytes = (size_t)g.nruns * 6 * g.nf * g.vs * c->esize;
  TRYC(cudaMalloc(&c->A, bytes));
  TRYC(cudaMalloc(&c->B, bytes));
  TRYC(cudaMalloc(&c->W, bytes));
  TRYC(cudaMemset(c->A, 0, bytes));
  TRYC(cudaMemset(c->B, 0, bytes));
  TRYC(cudaMemset(c->W, 0, bytes));

  TRYC(cudaMalloc((void**)&c->stage64, (size_t)vol_compact(c) * sizeof(double)));
  TRYC(cudaMalloc((void**)&c->part, (size_t)6 * g.nr * 5 * sizeof(double)));
  TRYC(cudaMalloc((void**)&c->red_out, 5 * sizeof(double)));
  TRYC(cudaMalloc((void**)&c->run_order, g.nruns * sizeof(int)));
  TRY(upload_constants());
  if (c->fp32) TRY(upload_tables<float>(c));
  else TRY(upload_tables<double>(c));
  TRYC(cudaMalloc((void**)&c->dt.s0t, c->ht.s0t.size() * sizeof(int)));
  TRYC(cudaMemcpy(c->dt.s0t, c->ht.s0t.data(), c->ht.s0t.size() * sizeof(int), cudaMemcpyHostToDevice));
  TRY(edge_windows(c));
  TRYC(cudaMalloc((void**)&c->err, 2 * sizeof(int)));
  TRYC(cudaMemset(c->err, 0, 2 * sizeof(int)));
  if (!tensor_map_encoder()) { solar_gpu_finalize(c); return fail(SOLAR_ERR_CUDA, "cuTensorMapEncodeTiled entry point unavailable"); }
  TRY(upload<double>((void**)&c->dt.rad64, c->ht.radial));
  {
    std::vector<double> vol2(c->ht.metric.begin() + (size_t)kMVol * g.n * g.n,
                             c->ht.metric.begin() + (size_t)(kMVol + 1) * g.n * g.n);
    TRY(upload<double>((void**)&c->dt.vol2, vol2));
  }
  TRY(upload<double>((void**)&c->dt.drw, c->ht.dr_weight));
  TRY(upload<double>((void**)&c->dt.tanx, c->ht.tanx));
  TRY(upload<double>((void**)&c->dt.gr, c->ht.gr));
  if (d->c2_3d) {
    std::vector<double> c2(d->c2_3d, d->c2_3d + (size_t)6 * vol_compact(c));
    TRY(upload<double>((void**)&c->dt.c2_64, c2));
    if (c->fp32) TRY(upload<float>(&c->dt.c2, c2));
    else TRY(upload<double>(&c->dt.c2, c2));
  }
  for (auto& e : c->ev) TRYC(cudaEventCreate(&e));
  TRYC(cudaStreamSynchronize(c->stream));
#undef TRY
#undef TRYC
  *out = c;
  return SOLAR_OK;
}

int solar_gpu_set_state(solar_ctx* c, int run, const double* q) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!q || run < 0 || run >= c->g.nruns) return fail(SOLAR_ERR_ARG, "bad run or null state");
  if ((rc = upload_fields(c, c->A, run, q, 5, kAllFields, 5))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return SOLAR_OK;
}

int solar_gpu_get_state(solar_ctx* c, int run, double* q) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!q || run < 0 || run >= c->g.nruns) return fail(SOLAR_ERR_ARG, "bad run or null state");
  return download_fields(c, c->A, run, q, 5, kAllFields, 5);
}

int solar_gpu_add_gaussian(solar_ctx* c, int run, double x0, double y0, double z0, double width,
                           double amp) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (run < 0 || run >= c->g.nruns || !(width > 0.0)) return fail(SOLAR_ERR_ARG, "bad run or width");
  // face by face: pressure volume -> compact FP64 scratch, add the pulse, write back
  const long long V = vol_compact(c);
  const int threads = 256, blocks = (int)((V + threads - 1) / threads);
  const int s = c->g.slot[kP];
  for (int z = 0; z < 6; ++z) {
    const long long off = c->g.vol(run, z, s);
    if (c->fp32) pack_kernel<float><<<blocks, threads, 0, c->stream>>>((const float*)c->A + off, c->stage64, c->g);
    else pack_kernel<double><<<blocks, threads, 0, c->stream>>>((const double*)c->A + off, c->stage64, c->g);
    gaussian_kernel<<<blocks, threads, 0, c->stream>>>(c->stage64, c->g, z, c->dt.tanx, c->dt.gr, x0, y0, z0,
                                                       width, amp);
    if (c->fp32) unpack_kernel<float><<<blocks, threads, 0, c->stream>>>(c->stage64, (float*)c->A + off, c->g);
    else unpack_kernel<double><<<blocks, threads, 0, c->stream>>>(c->stage64, (double*)c->A + off, c->g);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(c->stream));
  return SOLAR_OK;
}

int solar_gpu_rk4(solar_ctx* c, int nsteps) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nsteps < 0) return fail(SOLAR_ERR_ARG, "nsteps < 0");
  if ((rc = capture_step_graph(c))) return rc;
  for (int s = 0; s < nsteps; ++s) {
    CK(cudaGraphLaunch(c->step_graph, c->stream));
    if ((rc = watch_after_step(c))) return rc;
  }
  CK(cudaStreamSynchronize(c->stream));
  return check_device_error(c);
}

static int rk4_runs_impl(solar_ctx* c, const int* nsteps_per_run, double* ms);

int solar_gpu_rk4_runs(solar_ctx* c, const int* nsteps_per_run) { return rk4_runs_impl(c, nsteps_per_run, nullptr); }

int solar_gpu_time_rk4_runs(solar_ctx* c, const int* nsteps_per_run, double* ms) {
  if (!ms) return fail(SOLAR_ERR_ARG, "null output");
  return rk4_runs_impl(c, nsteps_per_run, ms);
}

static int rk4_runs_impl(solar_ctx* c, const int* nsteps_per_run, double* ms) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!nsteps_per_run) return fail(SOLAR_ERR_ARG, "null step counts");
  const int R = c->g.nruns;
  for (int r = 0; r < R; ++r)
    if (nsteps_per_run[r] < 0) return fail(SOLAR_ERR_ARG, "negative step count");
  // Runs ordered by step count, most first: while s steps are done, the live runs are the
  // first (count of runs with more than s steps) entries, so each stretch of steps with the
  // same live count replays one graph whose grids cover exactly those runs.
  std::vector<int> order(R);
  for (int r = 0; r < R; ++r) order[r] = r;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return nsteps_per_run[x] > nsteps_per_run[y]; });
  CK(cudaMemcpyAsync(c->run_order, order.data(), R * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));   // the host copy of `order` goes out of scope below
  std::vector<std::pair<int, int>> stretches;   // (live runs, steps)
  int done = 0;
  for (int live = R; live > 0; --live) {
    const int until = nsteps_per_run[order[live - 1]];
    if (until > done) { stretches.push_back({live, until - done}); done = until; }
  }
  for (const auto& st : stretches)
    if ((rc = capture_batch_graph(c, st.first))) return rc;
  CK(cudaEventRecord(c->ev[0], c->stream));
  for (const auto& st : stretches)
    for (int s = 0; s < st.second; ++s) {
      CK(cudaGraphLaunch(c->batch_graphs[st.first], c->stream));
      if ((rc = watch_after_step(c))) return rc;
    }
  CK(cudaEventRecord(c->ev[1], c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (ms) {
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, c->ev[0], c->ev[1]));
    *ms = f;
  }
  return check_device_error(c);
}

// Operator-level drop-ins: inputs go to buffer B (run 0), results come from buffer W.
// The state buffer A is left untouched.
static int op_prepare_state(solar_ctx* c, const double* q) {
  return upload_fields(c, c->B, 0, q, 5, kAllFields, 5);
}

int solar_gpu_compute_rhs(solar_ctx* c, const double* q, double* rhs) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!q || !rhs) return fail(SOLAR_ERR_ARG, "null array");
  if ((rc = op_prepare_state(c, q))) return rc;
  if ((rc = force_begin(c))) return rc;
  if (c->fp32) { launch_edge<float>(c, c->B, 0, nullptr); rc = launch_stage<float>(c, c->B, c->W, 2, 0, nullptr); }
  else { launch_edge<double>(c, c->B, 0, nullptr); rc = launch_stage<double>(c, c->B, c->W, 2, 0, nullptr); }
  if (rc) return rc;
  CK(cudaGetLastError());
  if ((rc = check_device_error(c))) return rc;
  return download_fields(c, c->W, 0, rhs, 5, kAllFields, 5);
}

static int bc_sponge_op(solar_ctx* c, const double* q, double* rhs, int do_bc, int do_sponge) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!rhs || (do_sponge && !q)) return fail(SOLAR_ERR_ARG, "null array");
  if ((rc = upload_fields(c, c->W, 0, rhs, 5, kAllFields, 5))) return rc;
  if (q && (rc = upload_fields(c, c->B, 0, q, 5, kAllFields, 5))) return rc;
  const long long n6 = 6 * vol_compact(c);
  const int threads = 256, blocks = (int)((n6 + threads - 1) / threads);
  if (c->fp32) bc_sponge_kernel<float><<<blocks, threads, 0, c->stream>>>((float*)c->W, (const float*)c->B, (const float*)c->dt.rad, c->g, 0, do_bc, do_sponge);
  else bc_sponge_kernel<double><<<blocks, threads, 0, c->stream>>>((double*)c->W, (const double*)c->B, (const double*)c->dt.rad, c->g, 0, do_bc, do_sponge);
  CK(cudaGetLastError());
  return download_fields(c, c->W, 0, rhs, 5, kAllFields, 5);
}

int solar_gpu_bc_rhs(solar_ctx* c, double* rhs) { return bc_sponge_op(c, nullptr, rhs, 1, 0); }
int solar_gpu_sponge(solar_ctx* c, const double* q, double* rhs) { return bc_sponge_op(c, q, rhs, 0, 1); }

int solar_gpu_filter_exp(solar_ctx* c, const double* q, double* qf) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!q || !qf) return fail(SOLAR_ERR_ARG, "null array");
  if ((rc = op_prepare_state(c, q))) return rc;
  if (c->fp32) { launch_edge<float>(c, c->B, 1, nullptr); rc = launch_filter<float>(c, c->B, c->W, nullptr); }
  else { launch_edge<double>(c, c->B, 1, nullptr); rc = launch_filter<double>(c, c->B, c->W, nullptr); }
  if (rc) return rc;
  CK(cudaGetLastError());
  if ((rc = check_device_error(c))) return rc;
  return download_fields(c, c->W, 0, qf, 5, kAllFields, 5);
}

static int grad_div_op(solar_ctx* c, const double* fields[4], double* outs[4]) {
  // fields: v_xi, v_eta, v_r, p (any may be null -> zero); outs: grad_xi, grad_eta, grad_r, div
  int rc = check_ctx(c);
  if (rc) return rc;
  const long long n6 = 6 * vol_compact(c);
  std::vector<double> q((size_t)5 * n6, 0.0);
  const long long V = vol_compact(c);
  const int ref[4] = {kVxi, kVeta, kVr, kP};
  for (int m = 0; m < 4; ++m)
    if (fields[m])
      for (int z = 0; z < 6; ++z)
        std::memcpy(&q[((size_t)z * 5 + ref[m]) * V], fields[m] + (size_t)z * V, V * sizeof(double));
  if ((rc = op_prepare_state(c, q.data()))) return rc;
  if (c->fp32) { launch_edge<float>(c, c->B, 0, nullptr); rc = launch_stage<float>(c, c->B, c->W, 3, 0, nullptr); }
  else { launch_edge<double>(c, c->B, 0, nullptr); rc = launch_stage<double>(c, c->B, c->W, 3, 0, nullptr); }
  if (rc) return rc;
  CK(cudaGetLastError());
  if ((rc = check_device_error(c))) return rc;
  for (int m = 0; m < 4; ++m) {
    if (!outs[m]) continue;
    const int f = ref[m];
    if ((rc = download_fields(c, c->W, 0, outs[m], 1, &f, 1))) return rc;
  }
  return SOLAR_OK;
}

int solar_gpu_gradient(solar_ctx* c, const double* p, double* gxi, double* geta, double* gr) {
  if (!p) return fail(SOLAR_ERR_ARG, "null array");
  const double* f[4] = {nullptr, nullptr, nullptr, p};
  double* o[4] = {gxi, geta, gr, nullptr};
  return grad_div_op(c, f, o);
}

int solar_gpu_divergence(solar_ctx* c, const double* vxi, const double* veta, const double* vr, double* div) {
  if (!vxi || !veta || !vr || !div) return fail(SOLAR_ERR_ARG, "null array");
  const double* f[4] = {vxi, veta, vr, nullptr};
  double* o[4] = {nullptr, nullptr, nullptr, div};
  return grad_div_op(c, f, o);
}

int solar_gpu_norm(solar_ctx* c, int run, int field, double* out) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!out || field < 1 || field > 5 || run < 0 || run >= c->g.nruns) return fail(SOLAR_ERR_ARG, "bad field/run");
  double ss = 0.0;
  if ((rc = sumsq(c, run, field - 1, &ss))) return rc;
  // auxiliary.f90:122
  *out = std::pow(ss / ((double)c->g.n * c->g.n * c->g.nr) * 6.0, 0.5);
  return SOLAR_OK;
}

int solar_gpu_diag(solar_ctx* c, int run, double* out4) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!out4 || run < 0 || run >= c->g.nruns) return fail(SOLAR_ERR_ARG, "bad run");
  double r[5];
  if ((rc = reduce(c, run, -1, r))) return rc;
  out4[0] = r[1];
  out4[1] = r[2];
  out4[2] = r[3];
  out4[3] = r[4] > 0 ? 1.0 : 0.0;
  return SOLAR_OK;
}

int solar_gpu_time_rk4(solar_ctx* c, int nsteps, int per_kernel, double* out7) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!out7 || nsteps < 1) return fail(SOLAR_ERR_ARG, "bad arguments");
  for (int m = 0; m < 7; ++m) out7[m] = 0.0;
  if (!per_kernel) {
    if ((rc = capture_step_graph(c))) return rc;
    CK(cudaEventRecord(c->ev[0], c->stream));
    for (int s = 0; s < nsteps; ++s) {
      CK(cudaGraphLaunch(c->step_graph, c->stream));
      if ((rc = watch_after_step(c))) return rc;
    }
    CK(cudaEventRecord(c->ev[1], c->stream));
    CK(cudaEventSynchronize(c->ev[1]));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    out7[0] = ms;
    return check_device_error(c);
  }
  std::vector<cudaEvent_t> evs;
  CK(cudaEventRecord(c->ev[0], c->stream));
  for (int s = 0; s < nsteps; ++s) {
    if ((rc = enqueue_step_any(c, nullptr, &evs))) return rc;
    if ((rc = watch_after_step(c))) return rc;
  }
  CK(cudaEventRecord(c->ev[1], c->stream));
  CK(cudaEventSynchronize(c->ev[1]));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
  out7[0] = ms;
  // event layout per step: [e, edge, e, stage, e] x5 then [e, edge, e, filter, e]
  // marks are recorded around every launch: pairs (0,1)=edge, (1,2)=stage, ... per stage
  const size_t per_step = 18;
  for (size_t s = 0; s + per_step <= evs.size(); s += per_step) {
    for (int st = 0; st < 5; ++st) {
      float a = 0, b = 0;
      cudaEventElapsedTime(&a, evs[s + st * 3 + 0], evs[s + st * 3 + 1]);
      cudaEventElapsedTime(&b, evs[s + st * 3 + 1], evs[s + st * 3 + 2]);
      out7[3] += a;
      out7[1] += b;
      out7[6] += 1;
      out7[4] += 1;
    }
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, evs[s + 15], evs[s + 16]);
    cudaEventElapsedTime(&b, evs[s + 16], evs[s + 17]);
    out7[3] += a;
    out7[2] += b;
    out7[6] += 1;
    out7[5] += 1;
  }
  for (auto e : evs) cudaEventDestroy(e);
  if (out7[4] > 0) out7[1] /= out7[4];
  if (out7[5] > 0) out7[2] /= out7[5];
  if (out7[6] > 0) out7[3] /= out7[6];
  return check_device_error(c);
}

int solar_gpu_rk4_norms(solar_ctx* c, int run, int field, int nsteps, double* norms) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!norms || nsteps < 0 || field < 1 || field > 5 || run < 0 || run >= c->g.nruns)
    return fail(SOLAR_ERR_ARG, "bad run, field, step count or null output");
  if (nsteps == 0) return SOLAR_OK;
  if (c->norm_ring_len < nsteps) {
    CK(cudaStreamSynchronize(c->stream));
    if (c->norm_ring) cudaFree(c->norm_ring);
    c->norm_ring = nullptr;
    c->norm_ring_len = 0;
    cudaError_t e = cudaMalloc((void**)&c->norm_ring, (size_t)nsteps * sizeof(double));
    if (e != cudaSuccess) return fail(SOLAR_ERR_NOMEM, "per-step norms: %s", cudaGetErrorString(e));
    c->norm_ring_len = nsteps;
  }
  if ((rc = capture_step_graph(c))) return rc;
  const int slot = c->g.slot[field - 1];
  const int nblocks = c->g.nface * (c->g.k1 - c->g.k0);
  if (slot < 0) CK(cudaMemsetAsync(c->norm_ring, 0, (size_t)nsteps * sizeof(double), c->stream));
  for (int s = 0; s < nsteps; ++s) {
    CK(cudaGraphLaunch(c->step_graph, c->stream));
    if ((rc = watch_after_step(c))) return rc;
    if (slot < 0) continue;
    if (c->fp32) sumsq_plane_kernel<float><<<nblocks, 256, 0, c->stream>>>((const float*)c->A, c->g, run, slot, c->part);
    else sumsq_plane_kernel<double><<<nblocks, 256, 0, c->stream>>>((const double*)c->A, c->g, run, slot, c->part);
    sumsq_final_kernel<<<1, 256, 0, c->stream>>>(c->part, nblocks, c->norm_ring + s);
    CK(cudaGetLastError());
  }
  CK(cudaMemcpyAsync(norms, c->norm_ring, (size_t)nsteps * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // auxiliary.f90:122, as solar_gpu_norm
  const double npts = (double)c->g.n * c->g.n * c->g.nr;
  for (int s = 0; s < nsteps; ++s) norms[s] = std::pow(norms[s] / npts * 6.0, 0.5);
  return check_device_error(c);
}

int solar_gpu_set_watchdog(solar_ctx* c, int every) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (every < 0) return fail(SOLAR_ERR_ARG, "watchdog interval must be >= 0");
  c->watch_every = every;
  return SOLAR_OK;
}

int solar_gpu_inject_wait_timeout(solar_ctx* c, int kernels, int polls) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (kernels & ~(SOLAR_KERNEL_EDGE | SOLAR_KERNEL_STAGE | SOLAR_KERNEL_FILTER | SOLAR_KERNEL_ADJ_STAGE))
    return fail(SOLAR_ERR_ARG, "unknown kernel bits 0x%x", kernels);
  if (kernels && (polls < 1 || polls > (int)kWaitPolls)) return fail(SOLAR_ERR_ARG, "polls must be in 1..%u", kWaitPolls);
  CK(cudaStreamSynchronize(c->stream));
  c->inject_mask = kernels;
  c->inject_polls = kernels ? (uint32_t)polls : 0u;
  // the captured step graphs hold the old launch arguments
  if (c->step_graph) { cudaGraphExecDestroy(c->step_graph); c->step_graph = nullptr; }
  drop_batch_graphs(c);
  return SOLAR_OK;
}

int solar_gpu_synchronize(solar_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  return check_device_error(c);
}

}  // extern "C"

#include "split_host.cuh"
#include "io_host.cuh"
#include "forcing.cuh"
#include "adjoint_host.cuh"
#include "curl.cuh"
