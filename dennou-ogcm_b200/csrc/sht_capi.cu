// sht_capi.cu -- the extern "C" boundary (include/dogcm_sht.h).
//
// Each SpmlUtil_mod operator is composed from three device stages:
//   analysis:  longitude FFT (row scale) -> Legendre contraction -> pack (+ recurrence)
//   synthesis: unpack (+ recurrence) -> Legendre contraction -> longitude FFT (row scale)
// Two-input operators (w_AlphaOptr_xy, calc_UVCosLat2VorDiv, xy_AlphaOptr_w,
// calc_VorDiv2UV) run both inputs as one batch of 2 nb columns through a
// single pass. The reference instead calls SPMODEL once per input and per
// derivative (SpmlUtil_mod.f90:308-312, 335-338, 410, 426).
#include "sht_internal.h"

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

namespace sht {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

void set_error(const std::string &msg) { g_last_error = msg; }
int cuda_fail(cudaError_t e, const char *what)
{
  char buf[512];
  snprintf(buf, sizeof(buf), "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
  g_last_error = buf;
  if (e == cudaErrorMemoryAllocation) return SHT_ERR_ALLOC;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return SHT_ERR_NO_DEVICE;
  return SHT_ERR_CUDA;
}
// this thread's launches, for the kernel count of a graph it captures
static thread_local long long t_launches = 0;

void count_launch(int n)
{
  g_launches.fetch_add(n, std::memory_order_relaxed);
  t_launches += n;
}

cudaError_t kernel_setup(const void *kern, size_t smem, int threads, int *per_sm)
{
  struct Opt { int dev; const void *k; size_t max_smem; };
  struct Occ { int dev; const void *k; size_t smem; int threads, blocks; };
  static std::mutex mu;
  static std::vector<Opt> opts;
  static std::vector<Occ> occs;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (smem > 48 * 1024) {
    Opt *o = nullptr;
    for (Opt &c : opts)
      if (c.dev == dev && c.k == kern) o = &c;
    if (!o || o->max_smem < smem) {
      // raised under the lock, so a concurrent smaller request cannot lower it
      if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
        return e;
      if (o) o->max_smem = smem;
      else opts.push_back({dev, kern, smem});
    }
  }
  if (!per_sm) return cudaSuccess;
  for (const Occ &c : occs)
    if (c.dev == dev && c.k == kern && c.smem == smem && c.threads == threads) {
      *per_sm = c.blocks;
      return cudaSuccess;
    }
  int blocks = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, threads, smem)) != cudaSuccess) return e;
  occs.push_back({dev, kern, smem, threads, blocks});
  *per_sm = blocks;
  return cudaSuccess;
}

// The bounded device-side waits are those of the split-precision kernel; its
// error word is read only once its tables exist.
int device_error_status(sht_plan *p) { return split_error_status(p); }

namespace {

struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev)
  {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) ok = (cudaSetDevice(dev) == cudaSuccess);
  }
  ~DeviceGuard()
  {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

bool live(const sht_plan *p) { return p && p->magic == kPlanMagic; }

int check_plan(const sht_plan *p)
{
  if (!live(p)) {
    set_error("plan is not initialised");
    return SHT_ERR_NOT_INITIALIZED;
  }
  return SHT_OK;
}

// Device workspace: Fourier array F, internal spectral S, spectral temp W.
struct Workspace {
  double2 *F;
  double2 *S;
  double *W;
};

int ensure_ws(sht_plan *p, int ncol, int nb_temp, Workspace *ws)
{
  const size_t fbytes = sizeof(double2) * (size_t)(p->N + 1) * ncol * p->J;
  const size_t sbytes = sizeof(double2) * (size_t)p->R * ncol;
  const size_t wbytes = sizeof(double) * (size_t)p->L * nb_temp;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t need = al(fbytes) + al(sbytes) + al(wbytes);
  if (need > p->ws_bytes) {
    if (p->d_ws) {
      cudaStreamSynchronize(p->stream);
      cudaFree(p->d_ws);
      p->d_ws = nullptr;
      p->ws_bytes = 0;
    }
    ++p->buf_gen;
    cudaError_t e = cudaMalloc(&p->d_ws, need);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(workspace)");
    p->ws_bytes = need;
  }
  char *base = static_cast<char *>(p->d_ws);
  ws->F = reinterpret_cast<double2 *>(base);
  ws->S = reinterpret_cast<double2 *>(base + al(fbytes));
  ws->W = reinterpret_cast<double *>(base + al(fbytes) + al(sbytes));
  return SHT_OK;
}

// The device staging of the host-pointer calls, grown on demand (a growth
// invalidates the plan's host-call graphs, which name the old array).
int ensure_io(sht_plan *p, size_t need)
{
  if (need <= p->io_bytes) return SHT_OK;
  ++p->buf_gen;
  if (p->d_io) {
    cudaStreamSynchronize(p->stream);
    cudaFree(p->d_io);
    p->d_io = nullptr;
    p->io_bytes = 0;
  }
  cudaError_t e = cudaMalloc(&p->d_io, need);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(io staging)");
  p->io_bytes = need;
  return SHT_OK;
}

void mark(sht_plan *p, int k, cudaStream_t s)
{
  if (p->timing.on) cudaEventRecord(p->timing.ev[k], s);
}

int leg_fwd(sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s)
{
  if (use_split(p, true)) return launch_leg_fwd_split(p, F, ncol, S, s);
  return launch_leg_fwd_fp64(p, F, ncol, S, s);
}
int leg_inv(sht_plan *p, const double2 *S, int ncol, double2 *F, cudaStream_t s)
{
  if (use_split(p, false)) return launch_leg_inv_split(p, S, ncol, F, s);
  return launch_leg_inv_fp64(p, S, ncol, F, s);
}

// timing convention: ev[0] start, ev[1] after stage A, ev[2] after stage B, ev[3] end
void finish_timing(sht_plan *p, bool analysis)
{
  if (!p->timing.on) return;
  cudaEventSynchronize(p->timing.ev[3]);
  float a = 0, b = 0, c = 0;
  cudaEventElapsedTime(&a, p->timing.ev[0], p->timing.ev[1]);
  cudaEventElapsedTime(&b, p->timing.ev[1], p->timing.ev[2]);
  cudaEventElapsedTime(&c, p->timing.ev[2], p->timing.ev[3]);
  if (analysis) { p->timing.ms_fft = a; p->timing.ms_leg = b; p->timing.ms_spec = c; }
  else { p->timing.ms_spec = a; p->timing.ms_leg = b; p->timing.ms_fft = c; }
}

// grid inputs g0 (and g1) -> spectral outputs w0 (and w1)
// (with `mul`, every input field-level k is first multiplied point by point by
// the grid mul + k I J)
int run_analysis(sht_plan *p, int pack_op, int rs, const double *g0, const double *g1, int nb,
                 double *w0, double *w1, const double *mul = nullptr, const double *add0 = nullptr,
                 const double *add1 = nullptr)
{
  const int nin = g1 ? 2 : 1, ncol = nin * nb;
  cudaStream_t s = p->stream;
  int rc;
  if (pack_op == PACK_PLAIN && rs == RS_FWD_PLAIN && !g1 && !mul && use_small(p, true)) {
    // one kernel: the stage marks all fall around it (timed as the longitude stage)
    mark(p, 0, s);
    if ((rc = launch_small_fwd(p, g0, nullptr, nb, w0, nullptr, s))) return rc;
    mark(p, 1, s); mark(p, 2, s); mark(p, 3, s);
    return SHT_OK;
  }
  Workspace ws{};
  if ((rc = ensure_ws(p, ncol, 0, &ws))) return rc;
  mark(p, 0, s);
  if ((rc = launch_fft_fwd(p, g0, g1, nb, ncol, ws.F, ncol, 0, rs, s, nullptr, mul, nb, add0, add1))) return rc;
  mark(p, 1, s);
  if ((rc = leg_fwd(p, ws.F, ncol, ws.S, s))) return rc;
  mark(p, 2, s);
  if ((rc = launch_pack(p, pack_op, ws.S, ncol, nb, w0, w1, s))) return rc;
  mark(p, 3, s);
  return SHT_OK;
}

// spectral inputs w0 (and w1) -> grid outputs g0 (and g1, for two-output ops)
int run_synthesis(sht_plan *p, int unpack_op, int rs, const double *w0, const double *w1, int nb,
                  double *g0, double *g1)
{
  const int nout = g1 ? 2 : 1, ncol = nout * nb;
  cudaStream_t s = p->stream;
  int rc;
  if (unpack_op == UNPACK_PLAIN && rs == RS_INV_PLAIN && !w1 && !g1 && use_small(p, false)) {
    // one kernel: the stage marks all fall around it (timed as the longitude stage)
    mark(p, 0, s); mark(p, 1, s); mark(p, 2, s);
    if ((rc = launch_small_inv(p, w0, nullptr, nb, g0, nullptr, s))) return rc;
    mark(p, 3, s);
    return SHT_OK;
  }
  Workspace ws{};
  if ((rc = ensure_ws(p, ncol, 0, &ws))) return rc;
  mark(p, 0, s);
  if ((rc = launch_unpack(p, unpack_op, w0, w1, nb, ws.S, ncol, s))) return rc;
  mark(p, 1, s);
  if ((rc = leg_inv(p, ws.S, ncol, ws.F, s))) return rc;
  mark(p, 2, s);
  if ((rc = launch_fft_inv(p, ws.F, ncol, 0, ncol, g0, g1, nb, rs, s))) return rc;
  mark(p, 3, s);
  return SHT_OK;
}

enum Op : int {
  OP_W_XY, OP_XY_W, OP_DIVLAMBDA, OP_DIVMU, OP_GRADLAMBDA, OP_GRADMU, OP_GRADLON, OP_GRADLAT,
  OP_W_ALPHA, OP_XY_ALPHA, OP_UV2VORDIV, OP_VORDIV2UV, OP_LAPLA, OP_LAPLAINV,
  OP_AVRLONLAT, OP_INTLONLAT, OP_YA_AVRLON, OP_YA_INTLON,
  OP_W_ALPHA_PROD,  // w_AlphaOptr_xy(A Q, B Q): third input Q
  OP_HGRAD,         // xy_GradLon_w and xy_GradLat_w of one spectrum
  OP_HGRAD_G,       // the same of w_xy(grid)
  OP_FLUXDIV_G,     // xy_w(w_AlphaOptr_xy(A, B)), grid to grid
};

struct OpShape {
  int nin, nout;
  bool in_grid, out_grid;  // else spectral (reductions: out sized separately)
};

OpShape shape_of(int op)
{
  switch (op) {
  case OP_W_XY: case OP_DIVLAMBDA: case OP_DIVMU: return {1, 1, true, false};
  case OP_XY_W: case OP_GRADLAMBDA: case OP_GRADMU: case OP_GRADLON: case OP_GRADLAT: return {1, 1, false, true};
  case OP_W_ALPHA: return {2, 1, true, false};
  case OP_W_ALPHA_PROD: return {3, 1, true, false};
  case OP_HGRAD: return {1, 2, false, true};
  case OP_HGRAD_G: return {1, 2, true, true};
  case OP_FLUXDIV_G: return {2, 1, true, true};
  case OP_XY_ALPHA: return {2, 1, false, true};
  case OP_UV2VORDIV: return {2, 2, true, false};
  case OP_VORDIV2UV: return {2, 2, false, true};
  case OP_LAPLA: case OP_LAPLAINV: return {1, 1, false, false};
  default: return {1, 1, true, false};
  }
}

// run an operator on device pointers (plan mutex held by the caller)
int run_dev(sht_plan *p, int op, const double *i0, const double *i1, int nb, double *o0, double *o1,
            const double *i2 = nullptr)
{
  if (nb == 0) return SHT_OK;
  switch (op) {
  case OP_W_ALPHA_PROD: return run_analysis(p, PACK_ALPHA, RS_FWD_INV1MMU2, i0, i1, nb, o0, nullptr, i2);
  case OP_HGRAD: return run_synthesis(p, UNPACK_HGRAD, RS_INV_INVCOS, i0, nullptr, nb, o0, o1);
  case OP_HGRAD_G: {
    // the spectra stay in the workspace temp, sized for both steps up front
    // so that neither step reallocates under it
    Workspace ws{};
    int rc = ensure_ws(p, 2 * nb, nb, &ws);
    if (rc) return rc;
    if ((rc = run_analysis(p, PACK_PLAIN, RS_FWD_PLAIN, i0, nullptr, nb, ws.W, nullptr))) return rc;
    return run_synthesis(p, UNPACK_HGRAD, RS_INV_INVCOS, ws.W, nullptr, nb, o0, o1);
  }
  case OP_FLUXDIV_G: {
    Workspace ws{};
    int rc = ensure_ws(p, 2 * nb, nb, &ws);
    if (rc) return rc;
    if ((rc = run_analysis(p, PACK_ALPHA, RS_FWD_INV1MMU2, i0, i1, nb, ws.W, nullptr))) return rc;
    return run_synthesis(p, UNPACK_PLAIN, RS_INV_PLAIN, ws.W, nullptr, nb, o0, nullptr);
  }
  case OP_W_XY: return run_analysis(p, PACK_PLAIN, RS_FWD_PLAIN, i0, nullptr, nb, o0, nullptr);
  case OP_DIVLAMBDA: return run_analysis(p, PACK_DIVLAMBDA, RS_FWD_INV1MMU2, i0, nullptr, nb, o0, nullptr);
  case OP_DIVMU: return run_analysis(p, PACK_DIVMU, RS_FWD_INV1MMU2, i0, nullptr, nb, o0, nullptr);
  case OP_W_ALPHA: return run_analysis(p, PACK_ALPHA, RS_FWD_INV1MMU2, i0, i1, nb, o0, nullptr);
  case OP_UV2VORDIV: return run_analysis(p, PACK_VORDIV, RS_FWD_INV1MMU2, i0, i1, nb, o0, o1);
  case OP_XY_W: return run_synthesis(p, UNPACK_PLAIN, RS_INV_PLAIN, i0, nullptr, nb, o0, nullptr);
  case OP_GRADLAMBDA: return run_synthesis(p, UNPACK_GRADLAMBDA, RS_INV_PLAIN, i0, nullptr, nb, o0, nullptr);
  case OP_GRADMU: return run_synthesis(p, UNPACK_GRADMU, RS_INV_PLAIN, i0, nullptr, nb, o0, nullptr);
  case OP_GRADLON: return run_synthesis(p, UNPACK_GRADLAMBDA, RS_INV_INVCOS, i0, nullptr, nb, o0, nullptr);
  case OP_GRADLAT: return run_synthesis(p, UNPACK_GRADMU, RS_INV_INVCOS, i0, nullptr, nb, o0, nullptr);
  case OP_XY_ALPHA: return run_synthesis(p, UNPACK_ALPHA, RS_INV_INVA1MMU2, i0, i1, nb, o0, nullptr);
  case OP_VORDIV2UV: return run_synthesis(p, UNPACK_VORDIV2UV, RS_INV_INVACOS, i0, i1, nb, o0, o1);
  case OP_LAPLA: return launch_lapla(p, i0, nb, o0, false, p->stream);
  case OP_LAPLAINV: return launch_lapla(p, i0, nb, o0, true, p->stream);
  case OP_INTLONLAT: return launch_lonlat_reduce(p, i0, nb, o0, 0, p->stream);
  case OP_AVRLONLAT: return launch_lonlat_reduce(p, i0, nb, o0, 1, p->stream);
  case OP_YA_INTLON: return launch_lonlat_reduce(p, i0, nb, o0, 2, p->stream);
  case OP_YA_AVRLON: return launch_lonlat_reduce(p, i0, nb, o0, 3, p->stream);
  default: set_error("unknown operator"); return SHT_ERR_INVALID_ARG;
  }
}

size_t out_count(const sht_plan *p, int op, int nb)
{
  switch (op) {
  case OP_AVRLONLAT: case OP_INTLONLAT: return (size_t)nb;
  case OP_YA_AVRLON: case OP_YA_INTLON: return (size_t)nb * p->J;
  default: return shape_of(op).out_grid ? (size_t)nb * p->I * p->J : (size_t)nb * p->L;
  }
}

int check_args(const sht_plan *p, int op, const double *i0, const double *i1, int nb, const double *o0, const double *o1,
               const double *i2 = nullptr)
{
  int rc = check_plan(p);
  if (rc) return rc;
  const OpShape sh = shape_of(op);
  if (nb < 0) { set_error("nb must be >= 0"); return SHT_ERR_INVALID_ARG; }
  if (nb == 0) return SHT_OK;
  if (!i0 || (sh.nin >= 2 && !i1) || (sh.nin == 3 && !i2) || !o0 || (sh.nout == 2 && !o1)) {
    set_error("null array argument");
    return SHT_ERR_INVALID_ARG;
  }
  return SHT_OK;
}

// Device grid arrays are read and written as 16-byte pairs of doubles.
int check_dev_alignment(int op, const double *i0, const double *i1, const double *o0, const double *o1,
                        const double *i2 = nullptr)
{
  const OpShape sh = shape_of(op);
  auto mis = [](const double *x) { return x && (reinterpret_cast<uintptr_t>(x) & 15u) != 0; };
  if ((sh.in_grid && (mis(i0) || mis(i1) || mis(i2))) || (sh.out_grid && (mis(o0) || mis(o1)))) {
    set_error("device grid arrays must be 16-byte aligned");
    return SHT_ERR_INVALID_ARG;
  }
  return SHT_OK;
}

int api_dev(sht_plan *p, int op, const double *i0, const double *i1, int nb, double *o0, double *o1,
            const double *i2 = nullptr)
{
  int rc = check_args(p, op, i0, i1, nb, o0, o1, i2);
  if (rc || nb == 0) return rc;
  if ((rc = check_dev_alignment(op, i0, i1, o0, o1, i2))) return rc;
  std::lock_guard<std::mutex> lk(p->mtx);
  DeviceGuard g(p->device);
  if (!g.ok) { set_error("cudaSetDevice failed"); return SHT_ERR_CUDA; }
  rc = run_dev(p, op, i0, i1, nb, o0, o1, i2);
  if (!rc) finish_timing(p, !shape_of(op).out_grid);
  return rc;
}

int host_call(sht_plan *p, int op, const double *i0, const double *i1, int nb, double *o0, double *o1,
              const double *i2);

// Calls whose host arrays total at most this many bytes and are pageable are
// staged through page-locked host memory (per-level calls up to T341).
constexpr size_t kPinnedStageMax = 8u << 20;
constexpr size_t kMaxHostGraphs = 32;

// Runs the device half of a staged host call (enqueue) as a CUDA graph.  The
// first call of an (operator, size, precision, kernel choice) runs directly
// and allocates whatever the operator needs; the second is captured on the
// plan's capture stream and instantiated; later ones replay it, one graph
// launch instead of two copies and three to six kernel launches.  Graphs
// made before a plan buffer was reallocated are dropped.  A capture that the
// runtime refuses leaves that key on the direct path.
template <typename Enqueue>
int host_graph_call(sht_plan *p, int op, int nb, Enqueue &&enqueue)
{
  cudaStream_t s = p->stream;
  auto &gs = p->graphs;
  for (size_t i = 0; i < gs.size();) {
    if (gs[i].gen != p->buf_gen) {
      if (gs[i].exec) cudaGraphExecDestroy(gs[i].exec);
      gs.erase(gs.begin() + (long)i);
    } else {
      ++i;
    }
  }
  HostGraph *g = nullptr;
  for (HostGraph &c : gs)
    if (c.op == op && c.nb == nb && c.precision == p->precision && c.leg_kernel == p->leg_kernel &&
        c.leg_tile == p->leg_tile)
      g = &c;
  cudaError_t e;
  if (g && g->exec) {
    if ((e = cudaGraphLaunch(g->exec, s)) != cudaSuccess) return cuda_fail(e, "graph launch");
    count_launch(g->launches);
    return SHT_OK;
  }
  if (!g || g->failed) {
    if (!g) {
      if (gs.size() >= kMaxHostGraphs) {
        if (gs.front().exec) cudaGraphExecDestroy(gs.front().exec);
        gs.erase(gs.begin());
      }
      HostGraph n;
      n.op = op; n.nb = nb; n.precision = p->precision; n.leg_kernel = p->leg_kernel; n.leg_tile = p->leg_tile;
      n.gen = p->buf_gen;
      gs.push_back(n);
    }
    return enqueue(s);
  }
  if (!p->cap_stream && cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    p->cap_stream = nullptr;
    g->failed = true;
    return enqueue(s);
  }
  const unsigned long long gen0 = p->buf_gen;
  const long long n0 = t_launches;
  if ((e = cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
    cudaGetLastError();
    g->failed = true;
    return enqueue(s);
  }
  p->stream = p->cap_stream;
  int rc = enqueue(p->cap_stream);
  p->stream = s;
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(p->cap_stream, &graph);
  const int captured = (int)(t_launches - n0);  // recorded into the graph, not run
  g_launches.fetch_sub(captured, std::memory_order_relaxed);
  t_launches = n0;
  cudaGraphExec_t exec = nullptr;
  if (rc == SHT_OK && e == cudaSuccess && graph && p->buf_gen == gen0) e = cudaGraphInstantiate(&exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  // g may have moved if the list changed; find the entry again
  g = nullptr;
  for (HostGraph &c : gs)
    if (c.op == op && c.nb == nb && c.precision == p->precision && c.leg_kernel == p->leg_kernel &&
        c.leg_tile == p->leg_tile)
      g = &c;
  if (rc != SHT_OK || e != cudaSuccess || !exec) {
    cudaGetLastError();
    if (exec) cudaGraphExecDestroy(exec);
    if (g) g->failed = true;
    return enqueue(s);  // nothing captured has run
  }
  if (!g) {
    cudaGraphExecDestroy(exec);
    return enqueue(s);
  }
  g->exec = exec;
  g->launches = captured;
  if ((e = cudaGraphLaunch(exec, s)) != cudaSuccess) return cuda_fail(e, "graph launch");
  count_launch(g->launches);
  return SHT_OK;
}

int api_host(sht_plan *p, int op, const double *i0, const double *i1, int nb, double *o0, double *o1,
             const double *i2 = nullptr)
{
  int rc = check_args(p, op, i0, i1, nb, o0, o1, i2);
  if (rc || nb == 0) return rc;
  std::lock_guard<std::mutex> lk(p->mtx);
  DeviceGuard g(p->device);
  if (!g.ok) { set_error("cudaSetDevice failed"); return SHT_ERR_CUDA; }
  return host_call(p, op, i0, i1, nb, o0, o1, i2);
}

// the body of a host-pointer call (arguments checked, plan mutex held, device set)
int host_call(sht_plan *p, int op, const double *i0, const double *i1, int nb, double *o0, double *o1,
              const double *i2)
{
  int rc;
  const OpShape sh = shape_of(op);
  const size_t nin_each = sh.in_grid ? (size_t)nb * p->I * p->J : (size_t)nb * p->L;
  const size_t nout_each = out_count(p, op, nb);
  // each staging buffer starts on a 256-byte boundary (the longitude transform
  // moves grid rows as 16-byte pairs; lm = (nm+1)^2 may be odd)
  auto al = [](size_t n) { return (n + 31) & ~(size_t)31; };  // in doubles
  const size_t need = sizeof(double) * (al(nin_each) * sh.nin + al(nout_each) * sh.nout) + 1024;
  cudaError_t e;
  if ((rc = ensure_io(p, need))) return rc;
  double *d = static_cast<double *>(p->d_io);
  // staging: the operator's inputs, then its outputs
  const double *hin[3] = {i0, i1, i2};
  double *din[3] = {nullptr, nullptr, nullptr};
  for (int k = 0; k < sh.nin; ++k) din[k] = d + k * al(nin_each);
  double *const di0 = din[0];
  double *do0 = d + al(nin_each) * sh.nin, *do1 = sh.nout == 2 ? do0 + al(nout_each) : nullptr;
  // device input k (or null past the operator's inputs), offset by `off` doubles
  auto dev_in = [&](int k, size_t off) -> const double * { return k < sh.nin ? din[k] + off : nullptr; };
  cudaStream_t s = p->stream;
  // Large transform batches run as a pipeline of chunks: the upload of chunk
  // c+1 (copy_in), the kernels of chunk c (plan stream) and the download of
  // chunk c-1 (copy_out) overlap, and PCIe carries both directions at once.
  const bool per_level = op != OP_AVRLONLAT && op != OP_INTLONLAT && op != OP_YA_AVRLON && op != OP_YA_INTLON;
  int nchunk = per_level ? nb / 48 : 1;
  nchunk = nchunk < 1 ? 1 : (nchunk > 8 ? 8 : nchunk);
  if (nchunk > 1 && !p->copy_in) {
    if ((e = cudaStreamCreateWithFlags(&p->copy_in, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&p->copy_out, cudaStreamNonBlocking)) != cudaSuccess)
      return cuda_fail(e, "copy streams");
    for (auto &ev : p->chunk_ev)
      if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return cuda_fail(e, "chunk events");
  }
  // Small calls on pageable host arrays (one level at a time, as the
  // reference's loops call) go through the plan's pinned staging buffer: a
  // host memcpy plus an asynchronous copy costs less than the driver's
  // pageable path.  Page-locked arrays are copied directly.
  double *hs = nullptr;
  if (nchunk == 1) {
    const size_t stage_bytes = sizeof(double) * (nin_each * sh.nin + nout_each * sh.nout);
    bool pageable = false;
    auto is_pageable = [](const void *ptr) {
      cudaPointerAttributes at;
      if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) { cudaGetLastError(); return true; }
      return at.type == cudaMemoryTypeUnregistered;
    };
    for (int k = 0; k < sh.nin; ++k) pageable = pageable || is_pageable(hin[k]);
    pageable = pageable || is_pageable(o0) || (sh.nout == 2 && is_pageable(o1));
    if (pageable && stage_bytes <= kPinnedStageMax) {
      if (stage_bytes > p->h_stage_bytes) {
        ++p->buf_gen;
        if (p->h_stage) { cudaStreamSynchronize(s); cudaFreeHost(p->h_stage); p->h_stage = nullptr; p->h_stage_bytes = 0; }
        if ((e = cudaMallocHost(&p->h_stage, stage_bytes)) != cudaSuccess) return cuda_fail(e, "cudaMallocHost(staging)");
        p->h_stage_bytes = stage_bytes;
      }
      hs = static_cast<double *>(p->h_stage);
    }
  }
  if (nchunk == 1) {
    double *hso = hs ? hs + nin_each * sh.nin : nullptr;  // staged outputs
    if (hs)
      for (int k = 0; k < sh.nin; ++k) std::memcpy(hs + k * nin_each, hin[k], sizeof(double) * nin_each);
    // the device half of the call on stream q (the plan's stream during it)
    auto enqueue = [&](cudaStream_t q) -> int {
      cudaError_t ee;
      for (int k = 0; k < sh.nin; ++k)
        if ((ee = cudaMemcpyAsync(din[k], hs ? hs + k * nin_each : hin[k], sizeof(double) * nin_each,
                                  cudaMemcpyHostToDevice, q)) != cudaSuccess)
          return cuda_fail(ee, "H2D");
      int r = run_dev(p, op, di0, dev_in(1, 0), nb, do0, sh.nout == 2 ? do1 : nullptr, dev_in(2, 0));
      if (r) return r;
      if ((ee = cudaMemcpyAsync(hs ? hso : o0, do0, sizeof(double) * nout_each, cudaMemcpyDeviceToHost, q)) != cudaSuccess)
        return cuda_fail(ee, "D2H");
      if (sh.nout == 2 && (ee = cudaMemcpyAsync(hs ? hso + nout_each : o1, do1, sizeof(double) * nout_each,
                                                cudaMemcpyDeviceToHost, q)) != cudaSuccess)
        return cuda_fail(ee, "D2H");
      return SHT_OK;
    };
    // staged calls name only plan buffers, so they can replay as graphs
    rc = (hs && p->host_graphs && !p->timing.on) ? host_graph_call(p, op, nb, enqueue) : enqueue(s);
    if (rc) return rc;
  } else {
    const size_t pin = nin_each / nb, pout = nout_each / nb;  // doubles per field-level
    // Chunk sizes ramp up and down (weights 1, 2, 3, ..., 3, 2, 1): only the
    // first chunk's upload and kernels and the last chunk's kernels and
    // download overlap nothing, so those chunks are the small ones.
    int wsum = 0, wpre[9] = {0};
    for (int c = 0; c < nchunk; ++c) {
      const int w = std::min(std::min(c + 1, nchunk - c), 3);
      wpre[c + 1] = wpre[c] + w;
      wsum += w;
    }
    // the plan stream and the copy streams start after any earlier work on the plan stream
    if ((e = cudaEventRecord(p->chunk_ev[0], s)) != cudaSuccess) return cuda_fail(e, "chunk event");
    if ((e = cudaStreamWaitEvent(p->copy_in, p->chunk_ev[0], 0)) != cudaSuccess) return cuda_fail(e, "chunk wait");
    for (int c = 0; c < nchunk; ++c) {
      const int b0 = (int)((long long)nb * wpre[c] / wsum), b1 = (int)((long long)nb * wpre[c + 1] / wsum), n = b1 - b0;
      cudaEvent_t ein = p->chunk_ev[2 * c], eout = p->chunk_ev[2 * c + 1];
      for (int k = 0; k < sh.nin; ++k)
        if ((e = cudaMemcpyAsync(din[k] + b0 * pin, hin[k] + b0 * pin, sizeof(double) * n * pin,
                                 cudaMemcpyHostToDevice, p->copy_in)) != cudaSuccess)
          return cuda_fail(e, "H2D");
      if ((e = cudaEventRecord(ein, p->copy_in)) != cudaSuccess || (e = cudaStreamWaitEvent(s, ein, 0)) != cudaSuccess)
        return cuda_fail(e, "chunk event");
      rc = run_dev(p, op, di0 + b0 * pin, dev_in(1, b0 * pin), n, do0 + b0 * pout,
                   sh.nout == 2 ? do1 + b0 * pout : nullptr, dev_in(2, b0 * pin));
      if (rc) return rc;
      if ((e = cudaEventRecord(eout, s)) != cudaSuccess || (e = cudaStreamWaitEvent(p->copy_out, eout, 0)) != cudaSuccess)
        return cuda_fail(e, "chunk event");
      if ((e = cudaMemcpyAsync(o0 + b0 * pout, do0 + b0 * pout, sizeof(double) * n * pout, cudaMemcpyDeviceToHost,
                               p->copy_out)) != cudaSuccess ||
          (sh.nout == 2 && (e = cudaMemcpyAsync(o1 + b0 * pout, do1 + b0 * pout, sizeof(double) * n * pout,
                                                 cudaMemcpyDeviceToHost, p->copy_out)) != cudaSuccess))
        return cuda_fail(e, "D2H");
    }
    if ((e = cudaStreamSynchronize(p->copy_out)) != cudaSuccess) return cuda_fail(e, "D2H");
  }
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "transform");
  if (hs) {
    const double *hso = hs + nin_each * sh.nin;
    std::memcpy(o0, hso, sizeof(double) * nout_each);
    if (sh.nout == 2) std::memcpy(o1, hso + nout_each, sizeof(double) * nout_each);
  }
  if ((rc = device_error_status(p))) return rc;
  finish_timing(p, !sh.out_grid);
  return SHT_OK;
}

void free_plan(sht_plan *p)
{
  cudaFree(p->d_mu); cudaFree(p->d_wgt); cudaFree(p->d_rowscale); cudaFree(p->d_P);
  cudaFree(p->d_poff); cudaFree(p->d_rowoff); cudaFree(p->d_eps); cudaFree(p->d_tw);
  cudaFree(p->d_twI); cudaFree(p->d_rn); cudaFree(p->d_spec_tiles); cudaFree(p->d_pairs);
  cudaFree(p->d_ws); cudaFree(p->d_io);
  if (p->h_stage) cudaFreeHost(p->h_stage);
  free_split_tables(p);
  for (auto &g : p->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  p->graphs.clear();
  if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
  for (auto &ev : p->timing.ev)
    if (ev) cudaEventDestroy(ev);
  if (p->own_stream) cudaStreamDestroy(p->own_stream);
  if (p->copy_in) cudaStreamDestroy(p->copy_in);
  if (p->copy_out) cudaStreamDestroy(p->copy_out);
  for (auto &ev : p->chunk_ev)
    if (ev) cudaEventDestroy(ev);
}

}  // namespace

// Plain analysis / synthesis over per-column pointer tables with caller-owned
// Fourier (F) and internal spectral (S) buffers: the multi-instance batches.
int run_analysis_cols(sht_plan *p, const double *const *gcol, int ncol, double *const *wcol, double2 *F,
                      double2 *S, cudaStream_t s)
{
  int rc;
  if (use_small(p, true)) return launch_small_fwd(p, nullptr, gcol, ncol, nullptr, wcol, s);
  if ((rc = launch_fft_fwd(p, nullptr, nullptr, ncol, ncol, F, ncol, 0, RS_FWD_PLAIN, s, gcol))) return rc;
  if ((rc = leg_fwd(p, F, ncol, S, s))) return rc;
  return launch_pack(p, PACK_PLAIN, S, ncol, ncol, nullptr, nullptr, s, wcol);
}

int run_synthesis_cols(sht_plan *p, const double *const *wcol, int ncol, double *const *gcol, double2 *F,
                       double2 *S, cudaStream_t s)
{
  int rc;
  if (use_small(p, false)) return launch_small_inv(p, nullptr, wcol, ncol, nullptr, gcol, s);
  if ((rc = launch_unpack(p, UNPACK_PLAIN, nullptr, nullptr, ncol, S, ncol, s, wcol))) return rc;
  if ((rc = leg_inv(p, S, ncol, F, s))) return rc;
  return launch_fft_inv(p, F, ncol, 0, ncol, nullptr, nullptr, ncol, RS_INV_PLAIN, s, gcol);
}

namespace {

int check_strided(const sht_plan *p, const void *g, int ldi, int ldj, int nb, const void *w, int ldw, int mode)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (nb < 0) { set_error("nb must be >= 0"); return SHT_ERR_INVALID_ARG; }
  if (mode != -1 && mode != SHT_PREC_FP64 && mode != SHT_PREC_SPLIT && mode != SHT_PREC_AUTO) {
    set_error("unknown precision mode");
    return SHT_ERR_INVALID_ARG;
  }
  if (nb == 0) return SHT_OK;
  if (!g || !w) { set_error("null array argument"); return SHT_ERR_INVALID_ARG; }
  if (ldi < p->I || ldj < p->J || ldw < p->L) {
    set_error("leading dimensions must be at least im, jm and lm");
    return SHT_ERR_INVALID_ARG;
  }
  return SHT_OK;
}

// copies nb levels of an im x jm section (row pitch ldi, ldj rows per level)
// to or from a contiguous im x jm x nb array
cudaError_t copy_grid(const sht_plan *p, void *dst, int dst_ldi, int dst_ldj, const void *src, int src_ldi,
                      int src_ldj, int nb, cudaMemcpyKind kind, cudaStream_t s)
{
  cudaMemcpy3DParms c = {};
  c.srcPtr = make_cudaPitchedPtr(const_cast<void *>(src), sizeof(double) * src_ldi, sizeof(double) * p->I, src_ldj);
  c.dstPtr = make_cudaPitchedPtr(dst, sizeof(double) * dst_ldi, sizeof(double) * p->I, dst_ldj);
  c.extent = make_cudaExtent(sizeof(double) * p->I, p->J, nb);
  c.kind = kind;
  return cudaMemcpy3DAsync(&c, s);
}

// staging: grid (im jm nb) then spectra (lm nb), each on a 256-byte boundary
int strided_staging(sht_plan *p, int nb, double **dg, double **dw)
{
  auto al = [](size_t n) { return (n + 31) & ~(size_t)31; };
  const size_t ng = (size_t)nb * p->I * p->J, nw = (size_t)nb * p->L;
  const int rc = ensure_io(p, sizeof(double) * (al(ng) + al(nw)) + 1024);
  if (rc) return rc;
  *dg = static_cast<double *>(p->d_io);
  *dw = *dg + al(ng);
  return SHT_OK;
}

// The plan's precision for one call (mode -1 keeps it), restored on scope exit.
struct PrecisionScope {
  sht_plan *p;
  int saved;
  PrecisionScope(sht_plan *plan, int mode) : p(plan), saved(plan->precision)
  {
    if (mode >= 0) p->precision = mode;
  }
  ~PrecisionScope() { p->precision = saved; }
};

int strided_call(sht_plan *p, bool analysis, const double *g_in, double *g_out, int ldi, int ldj, int nb,
                 const double *w_in, double *w_out, int ldw, int mode, bool host)
{
  std::lock_guard<std::mutex> lk(p->mtx);
  DeviceGuard guard(p->device);
  if (!guard.ok) { set_error("cudaSetDevice failed"); return SHT_ERR_CUDA; }
  PrecisionScope ps(p, mode);
  int rc;
  if (ldi == p->I && ldj == p->J && ldw == p->L) {  // contiguous: the ordinary call
    const int op = analysis ? OP_W_XY : OP_XY_W;
    const double *in = analysis ? g_in : w_in;
    double *out = analysis ? w_out : g_out;
    if (host) return host_call(p, op, in, nullptr, nb, out, nullptr, nullptr);
    if ((rc = check_dev_alignment(op, in, nullptr, out, nullptr))) return rc;
    if ((rc = run_dev(p, op, in, nullptr, nb, out, nullptr))) return rc;
    finish_timing(p, analysis);
    return SHT_OK;
  }
  cudaStream_t s = p->stream;
  const cudaMemcpyKind to_dev = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  const cudaMemcpyKind from_dev = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  double *dg = nullptr, *dw = nullptr;
  rc = strided_staging(p, nb, &dg, &dw);
  if (rc) return rc;
  cudaError_t e;
  if (analysis) {
    if ((e = copy_grid(p, dg, p->I, p->J, g_in, ldi, ldj, nb, to_dev, s)) != cudaSuccess) return cuda_fail(e, "grid copy in");
    if ((rc = run_dev(p, OP_W_XY, dg, nullptr, nb, dw, nullptr))) return rc;
    if ((e = cudaMemcpy2DAsync(w_out, sizeof(double) * ldw, dw, sizeof(double) * p->L, sizeof(double) * p->L, nb,
                               from_dev, s)) != cudaSuccess)
      return cuda_fail(e, "spectral copy out");
  } else {
    if ((e = cudaMemcpy2DAsync(dw, sizeof(double) * p->L, w_in, sizeof(double) * ldw, sizeof(double) * p->L, nb,
                               to_dev, s)) != cudaSuccess)
      return cuda_fail(e, "spectral copy in");
    if ((rc = run_dev(p, OP_XY_W, dw, nullptr, nb, dg, nullptr))) return rc;
    if ((e = copy_grid(p, g_out, ldi, ldj, dg, p->I, p->J, nb, from_dev, s)) != cudaSuccess) return cuda_fail(e, "grid copy out");
  }
  if (host) {
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "transform");
    if ((rc = device_error_status(p))) return rc;
  }
  finish_timing(p, analysis);
  return SHT_OK;
}

}  // namespace

}  // namespace sht

using namespace sht;

extern "C" {

const char *sht_status_string(int status)
{
  switch (status) {
  case SHT_OK: return "ok";
  case SHT_ERR_INVALID_ARG: return "invalid argument";
  case SHT_ERR_UNSUPPORTED_SIZE: return "unsupported grid size";
  case SHT_ERR_NOT_INITIALIZED: return "plan not initialised";
  case SHT_ERR_CUDA: return "CUDA error";
  case SHT_ERR_NO_DEVICE: return "no CUDA device";
  case SHT_ERR_ALLOC: return "allocation failed";
  case SHT_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
  case SHT_ERR_TOO_LARGE: return "request exceeds capacity";
  default: return "unknown status";
  }
}

const char *sht_last_error(void) { return g_last_error.c_str(); }

int sht_l_nm(int n, int m) { return n * (n + 1) + m + 1; }

int sht_nm_l(int l, int *n, int *m)
{
  if (l < 1 || !n || !m) { set_error("nm_l: bad argument"); return SHT_ERR_INVALID_ARG; }
  int nn = (int)std::floor(std::sqrt((double)(l - 1)));
  while ((nn + 1) * (nn + 1) <= l - 1) ++nn;
  while (nn * nn > l - 1) --nn;
  *n = nn;
  *m = (l - 1) - nn * (nn + 1);
  return SHT_OK;
}

int sht_plan_l_nm(const sht_plan *p, int n, int m)
{
  if (!live(p)) { set_error("plan is not initialised"); return 0; }
  if (n < 0 || n > p->N || m < -n || m > n || (p->zonal && m != 0)) return 0;
  return p->zonal ? n + 1 : n * (n + 1) + m + 1;
}

int sht_plan_nm_l(const sht_plan *p, int l, int *n, int *m)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (!n || !m || l < 1 || l > p->L) { set_error("nm_l: index out of range"); return SHT_ERR_INVALID_ARG; }
  if (p->zonal) { *n = l - 1; *m = 0; return SHT_OK; }
  return sht_nm_l(l, n, m);
}

int sht_init(int im, int jm, int km, int nm, double radius, sht_plan **out)
{
  if (!out) { set_error("init: plan pointer is NULL"); return SHT_ERR_INVALID_ARG; }
  *out = nullptr;
  const bool zonal = (im == 1);  // DOGCM_MODE_AXISYM: wa_zonal_module, lm = nm + 1
  // default truncations of util/grid/DOGCM_GaussSpmVFvmGrid_mod.f90:206-209
  if (nm == -1) nm = zonal ? (2 * jm - 1) / 3 : (im - 1) / 3;
  int lg = 0;
  while ((1 << lg) < im) ++lg;
  const bool pow2 = (1 << lg) == im;
  // powers of two take the four-step FFT; other even counts (factors 3 and 5,
  // e.g. 96, 192, 320, 640) the direct transform
  if (!zonal && (im < 16 || im > 2048 || (!pow2 && (im & 1)))) {
    set_error("init: im must be 1 (axisymmetric) or even in [16, 2048]");
    return SHT_ERR_UNSUPPORTED_SIZE;
  }
  if (jm < 2 || (jm & 1)) { set_error("init: jm must be even and >= 2"); return SHT_ERR_UNSUPPORTED_SIZE; }
  if (nm < 0 || (!zonal && im < 2 * nm + 2) || jm <= nm) {
    set_error("init: need 0 <= nm, im >= 2 nm + 2 (unless im = 1) and jm > nm");
    return SHT_ERR_UNSUPPORTED_SIZE;
  }
  if (nm > 1023 || !(radius > 0.0) || km < 0) { set_error("init: bad nm/radius/km"); return SHT_ERR_INVALID_ARG; }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    set_error(std::string("init: no CUDA device: ") + cudaGetErrorString(e));
    return SHT_ERR_NO_DEVICE;
  }
  sht_plan *p = new (std::nothrow) sht_plan();
  if (!p) { set_error("init: host allocation failed"); return SHT_ERR_ALLOC; }
  p->I = im; p->J = jm; p->N = nm; p->K = km; p->JH = jm / 2; p->NC = im / 2; p->radius = radius;
  p->zonal = zonal;
  p->direct_dft = !zonal && !pow2;
  cudaGetDevice(&p->device);
  int rc = SHT_OK;
  if ((e = cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking)) != cudaSuccess) rc = cuda_fail(e, "stream create");
  p->stream = p->own_stream;
  for (int k = 0; k < 8 && !rc; ++k)
    if ((e = cudaEventCreate(&p->timing.ev[k])) != cudaSuccess) rc = cuda_fail(e, "event create");
  if (!rc) rc = build_tables(p);
  if (rc) {
    free_plan(p);
    delete p;
    return rc;
  }
  p->magic = kPlanMagic;
  *out = p;
  return SHT_OK;
}

int sht_final(sht_plan *p)
{
  int rc = check_plan(p);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lk(p->mtx);
    DeviceGuard g(p->device);
    cudaStreamSynchronize(p->stream);
    p->magic = 0;
    free_plan(p);
  }
  delete p;
  return SHT_OK;
}

int sht_is_initialized(const sht_plan *p) { return live(p) ? 1 : 0; }

int sht_dims(const sht_plan *p, int *im, int *jm, int *nm, int *lm)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (im) *im = p->I;
  if (jm) *jm = p->J;
  if (nm) *nm = p->N;
  if (lm) *lm = p->L;
  return SHT_OK;
}

int sht_grid_info(const sht_plan *p, double *x_lon, double *y_lat, double *x_lon_weight, double *y_lat_weight)
{
  int rc = check_plan(p);
  if (rc) return rc;
  for (int i = 0; i < p->I; ++i) {
    if (x_lon) x_lon[i] = 2.0 * M_PI * i / p->I;
    if (x_lon_weight) x_lon_weight[i] = 2.0 * M_PI / p->I;
  }
  for (int j = 0; j < p->J; ++j) {
    if (y_lat) y_lat[j] = std::asin(p->h_mu[j]);
    if (y_lat_weight) y_lat_weight[j] = 2.0 * p->h_wgt[j];
  }
  return SHT_OK;
}

int sht_rn(const sht_plan *p, double *rn)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (!rn) { set_error("rn: NULL output"); return SHT_ERR_INVALID_ARG; }
  // p->L entries in the plan's layout: l = n(n+1)+m, or l = n for a zonal plan
  for (int n = 0; n <= p->N; ++n)
    for (int m = -n; m <= n; ++m) {
      if (p->zonal && m != 0) continue;
      rn[p->zonal ? n : n * (n + 1) + m] = -(double)n * (n + 1);
    }
  return SHT_OK;
}

int sht_set_precision(sht_plan *p, int mode)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (mode != SHT_PREC_FP64 && mode != SHT_PREC_SPLIT && mode != SHT_PREC_AUTO) {
    set_error("unknown precision mode");
    return SHT_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lk(p->mtx);
  p->precision = mode;
  return SHT_OK;
}

int sht_get_precision(const sht_plan *p, int *mode)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (!mode) { set_error("NULL output"); return SHT_ERR_INVALID_ARG; }
  *mode = p->precision;
  return SHT_OK;
}

int sht_set_option(sht_plan *p, int option, int value)
{
  int rc = check_plan(p);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(p->mtx);
  switch (option) {
  case SHT_OPT_LEGENDRE_KERNEL:
    if (value < 0 || value > 4) { set_error("legendre kernel option must be 0, 1, 2, 3 or 4"); return SHT_ERR_INVALID_ARG; }
    p->leg_kernel = value;
    return SHT_OK;
  case SHT_OPT_LEGENDRE_TILE:
    if (value != 0 && value != 8 && value != 16 && value != 32) {
      set_error("legendre tile option must be 0, 8, 16 or 32");
      return SHT_ERR_INVALID_ARG;
    }
    p->leg_tile = value;
    return SHT_OK;
  case SHT_OPT_HOST_GRAPHS:
    if (value != 0 && value != 1) { set_error("host graphs option must be 0 or 1"); return SHT_ERR_INVALID_ARG; }
    p->host_graphs = value == 1;
    return SHT_OK;
  default: set_error("unknown option"); return SHT_ERR_INVALID_ARG;
  }
}

int sht_get_option(const sht_plan *p, int option, int *value)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (!value) { set_error("NULL output"); return SHT_ERR_INVALID_ARG; }
  switch (option) {
  case SHT_OPT_LEGENDRE_KERNEL: *value = p->leg_kernel; return SHT_OK;
  case SHT_OPT_LEGENDRE_TILE: *value = p->leg_tile; return SHT_OK;
  case SHT_OPT_HOST_GRAPHS: *value = p->host_graphs ? 1 : 0; return SHT_OK;
  case SHT_OPT_HOST_GRAPH_COUNT: {
    std::lock_guard<std::mutex> lk(const_cast<sht_plan *>(p)->mtx);
    int n = 0;
    for (const HostGraph &g : p->graphs) n += g.exec != nullptr;
    *value = n;
    return SHT_OK;
  }
  default: set_error("unknown option"); return SHT_ERR_INVALID_ARG;
  }
}

int sht_selftest_device_timeout(sht_plan *p, int limit_ms)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (limit_ms < 1 || limit_ms > 1000) { set_error("limit_ms must be in 1..1000"); return SHT_ERR_INVALID_ARG; }
  std::lock_guard<std::mutex> lk(p->mtx);
  DeviceGuard g(p->device);
  if (!g.ok) { set_error("cudaSetDevice failed"); return SHT_ERR_CUDA; }
  if ((rc = wait_selftest(p, (unsigned long long)limit_ms * 1000000ull))) return rc;
  return device_error_status(p);
}

int sht_set_stream(sht_plan *p, void *stream)
{
  int rc = check_plan(p);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(p->mtx);
  p->stream = static_cast<cudaStream_t>(stream);
  return SHT_OK;
}

int sht_synchronize(sht_plan *p)
{
  int rc = check_plan(p);
  if (rc) return rc;
  DeviceGuard g(p->device);
  if (!g.ok) { set_error("cudaSetDevice failed"); return SHT_ERR_CUDA; }
  cudaError_t e = cudaStreamSynchronize(p->stream);
  if (e != cudaSuccess) return cuda_fail(e, "synchronize");
  return device_error_status(p);
}

int sht_set_timing(sht_plan *p, int on)
{
  int rc = check_plan(p);
  if (rc) return rc;
  p->timing.on = on != 0;
  return SHT_OK;
}

int sht_last_timing(const sht_plan *p, float *ms_fft, float *ms_legendre, float *ms_spectral)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (ms_fft) *ms_fft = p->timing.ms_fft;
  if (ms_legendre) *ms_legendre = p->timing.ms_leg;
  if (ms_spectral) *ms_spectral = p->timing.ms_spec;
  return SHT_OK;
}

long long sht_launch_count(void) { return g_launches.load(); }

#define SHT_G2S(name, op)                                                                  \
  int name(sht_plan *p, const double *x, int nb, double *w) { return api_host(p, op, x, nullptr, nb, w, nullptr); } \
  int name##_dev(sht_plan *p, const double *x, int nb, double *w) { return api_dev(p, op, x, nullptr, nb, w, nullptr); }

SHT_G2S(sht_wa_xya, OP_W_XY)
SHT_G2S(sht_xya_wa, OP_XY_W)
SHT_G2S(sht_wa_divlambda_xya, OP_DIVLAMBDA)
SHT_G2S(sht_wa_divmu_xya, OP_DIVMU)
SHT_G2S(sht_xya_gradlambda_wa, OP_GRADLAMBDA)
SHT_G2S(sht_xya_gradmu_wa, OP_GRADMU)
SHT_G2S(sht_xya_gradlon_wa, OP_GRADLON)
SHT_G2S(sht_xya_gradlat_wa, OP_GRADLAT)
SHT_G2S(sht_wa_lapla_wa, OP_LAPLA)
SHT_G2S(sht_wa_laplainv_wa, OP_LAPLAINV)
SHT_G2S(sht_avrlonlat_xya, OP_AVRLONLAT)
SHT_G2S(sht_intlonlat_xya, OP_INTLONLAT)
SHT_G2S(sht_ya_avrlon_xya, OP_YA_AVRLON)
SHT_G2S(sht_ya_intlon_xya, OP_YA_INTLON)

int sht_wa_alphaoptr_xya(sht_plan *p, const double *a, const double *b, int nb, double *w)
{ return api_host(p, OP_W_ALPHA, a, b, nb, w, nullptr); }
int sht_wa_alphaoptr_xya_dev(sht_plan *p, const double *a, const double *b, int nb, double *w)
{ return api_dev(p, OP_W_ALPHA, a, b, nb, w, nullptr); }
int sht_xya_alphaoptr_wa(sht_plan *p, const double *a, const double *b, int nb, double *x)
{ return api_host(p, OP_XY_ALPHA, a, b, nb, x, nullptr); }
int sht_xya_alphaoptr_wa_dev(sht_plan *p, const double *a, const double *b, int nb, double *x)
{ return api_dev(p, OP_XY_ALPHA, a, b, nb, x, nullptr); }
int sht_wa_alphaoptr_prod_xya(sht_plan *p, const double *a, const double *b, const double *q, int nb, double *w)
{ return api_host(p, OP_W_ALPHA_PROD, a, b, nb, w, nullptr, q); }
int sht_wa_alphaoptr_prod_xya_dev(sht_plan *p, const double *a, const double *b, const double *q, int nb, double *w)
{ return api_dev(p, OP_W_ALPHA_PROD, a, b, nb, w, nullptr, q); }
int sht_xya_hgrad_wa(sht_plan *p, const double *w, int nb, double *lon, double *lat)
{ return api_host(p, OP_HGRAD, w, nullptr, nb, lon, lat); }
int sht_xya_hgrad_wa_dev(sht_plan *p, const double *w, int nb, double *lon, double *lat)
{ return api_dev(p, OP_HGRAD, w, nullptr, nb, lon, lat); }
int sht_xya_hgrad_xya(sht_plan *p, const double *x, int nb, double *lon, double *lat)
{ return api_host(p, OP_HGRAD_G, x, nullptr, nb, lon, lat); }
int sht_xya_hgrad_xya_dev(sht_plan *p, const double *x, int nb, double *lon, double *lat)
{ return api_dev(p, OP_HGRAD_G, x, nullptr, nb, lon, lat); }
int sht_xya_fluxdiv_xya(sht_plan *p, const double *a, const double *b, int nb, double *x)
{ return api_host(p, OP_FLUXDIV_G, a, b, nb, x, nullptr); }
int sht_xya_fluxdiv_xya_dev(sht_plan *p, const double *a, const double *b, int nb, double *x)
{ return api_dev(p, OP_FLUXDIV_G, a, b, nb, x, nullptr); }
int sht_uvcoslat2vordiv(sht_plan *p, const double *u, const double *v, int nb, double *vor, double *div)
{ return api_host(p, OP_UV2VORDIV, u, v, nb, vor, div); }
int sht_uvcoslat2vordiv_dev(sht_plan *p, const double *u, const double *v, int nb, double *vor, double *div)
{ return api_dev(p, OP_UV2VORDIV, u, v, nb, vor, div); }
int sht_vordiv2uv(sht_plan *p, const double *vor, const double *div, int nb, double *u, double *v)
{ return api_host(p, OP_VORDIV2UV, vor, div, nb, u, v); }
int sht_vordiv2uv_dev(sht_plan *p, const double *vor, const double *div, int nb, double *u, double *v)
{ return api_dev(p, OP_VORDIV2UV, vor, div, nb, u, v); }

// calc_UVCosLat2VorDiv(cos(phi) (x1 q + z1), cos(phi) (x2 q + z2)): the
// momentum products of the vorticity-divergence tendency, formed while the
// grids load into the longitude transform.  The two products share q; the
// cos(phi) factor and the 1 / (1 - mu^2) of the analysis meet in one row scale
// w_j / (I cos(phi_j)).  z1 and z2 are both given or both null (no sums).
static int uv_fma_impl(sht_plan *p, const double *x1, const double *x2, const double *q, const double *z1,
                       const double *z2, int nb, double *vor, double *div, bool host)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (nb < 0) { set_error("nb must be >= 0"); return SHT_ERR_INVALID_ARG; }
  if (nb == 0) return SHT_OK;
  if (!x1 || !x2 || !q || !vor || !div || (!z1) != (!z2)) {
    set_error("null array argument (z1 and z2 must be both given or both null)");
    return SHT_ERR_INVALID_ARG;
  }
  auto mis = [](const double *x) { return x && (reinterpret_cast<uintptr_t>(x) & 15u) != 0; };
  if (!host && (mis(x1) || mis(x2) || mis(q) || mis(z1) || mis(z2))) {
    set_error("device grid arrays must be 16-byte aligned");
    return SHT_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lk(p->mtx);
  DeviceGuard g(p->device);
  if (!g.ok) { set_error("cudaSetDevice failed"); return SHT_ERR_CUDA; }
  if (!host) {
    rc = run_analysis(p, PACK_VORDIV, RS_FWD_INVCOS, x1, x2, nb, vor, div, q, z1, z2);
    if (!rc) finish_timing(p, true);
    return rc;
  }
  // host arrays: stage every grid, run, copy both spectra back
  const size_t ng = (size_t)nb * p->I * p->J, nw = (size_t)nb * p->L;
  auto al = [](size_t n) { return (n + 31) & ~(size_t)31; };  // whole 256-byte blocks
  const int nin = z1 ? 5 : 3;
  if ((rc = ensure_io(p, sizeof(double) * (nin * al(ng) + 2 * al(nw))))) return rc;
  double *d = static_cast<double *>(p->d_io);
  const double *hin[5] = {x1, x2, q, z1, z2};
  cudaStream_t s = p->stream;
  cudaError_t e;
  for (int k = 0; k < nin; ++k)
    if ((e = cudaMemcpyAsync(d + k * al(ng), hin[k], sizeof(double) * ng, cudaMemcpyHostToDevice, s)) != cudaSuccess)
      return cuda_fail(e, "H2D");
  double *dv = d + nin * al(ng), *dd = dv + al(nw);
  rc = run_analysis(p, PACK_VORDIV, RS_FWD_INVCOS, d, d + al(ng), nb, dv, dd, d + 2 * al(ng),
                    z1 ? d + 3 * al(ng) : nullptr, z1 ? d + 4 * al(ng) : nullptr);
  if (rc) return rc;
  if ((e = cudaMemcpyAsync(vor, dv, sizeof(double) * nw, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(div, dd, sizeof(double) * nw, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_fail(e, "D2H");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "transform");
  if ((rc = device_error_status(p))) return rc;
  finish_timing(p, true);
  return SHT_OK;
}

int sht_uvcoslat2vordiv_fma(sht_plan *p, const double *x1, const double *x2, const double *q, const double *z1,
                            const double *z2, int nb, double *vor, double *div)
{ return uv_fma_impl(p, x1, x2, q, z1, z2, nb, vor, div, true); }
int sht_uvcoslat2vordiv_fma_dev(sht_plan *p, const double *x1, const double *x2, const double *q, const double *z1,
                                const double *z2, int nb, double *vor, double *div)
{ return uv_fma_impl(p, x1, x2, q, z1, z2, nb, vor, div, false); }

// ---------------------------------------------------------------- strided
// Analysis and synthesis of arrays with leading dimensions: the model keeps
// its fields with halos, xyz(IA, JA, KA) with the transform's points at
// (IS:IE, JS:JE) of every level, and copies each section in and out around
// every SpmlUtil call (explicit-shape dummies).  These entry points take the
// whole array instead: grid point (i, j) of level k at
// xya[i + ldi (j + ldj k)], spectral entry l of level k at wa[l + ldw k].
// The section moves between the caller's array and the contiguous staging by
// pitched copies (cudaMemcpy3DAsync / cudaMemcpy2DAsync, one per array);
// the transform itself is the ordinary batched one.

int sht_analysis(sht_plan *p, const double *xya, int ldi, int ldj, int nb, double *wa, int ldw, int mode)
{
  int rc = check_strided(p, xya, ldi, ldj, nb, wa, ldw, mode);
  if (rc || nb == 0) return rc;
  return strided_call(p, true, xya, nullptr, ldi, ldj, nb, nullptr, wa, ldw, mode, true);
}
int sht_analysis_dev(sht_plan *p, const double *xya, int ldi, int ldj, int nb, double *wa, int ldw, int mode)
{
  int rc = check_strided(p, xya, ldi, ldj, nb, wa, ldw, mode);
  if (rc || nb == 0) return rc;
  return strided_call(p, true, xya, nullptr, ldi, ldj, nb, nullptr, wa, ldw, mode, false);
}
int sht_synthesis(sht_plan *p, const double *wa, int ldw, int nb, double *xya, int ldi, int ldj, int mode)
{
  int rc = check_strided(p, xya, ldi, ldj, nb, wa, ldw, mode);
  if (rc || nb == 0) return rc;
  return strided_call(p, false, nullptr, xya, ldi, ldj, nb, wa, nullptr, ldw, mode, true);
}
int sht_synthesis_dev(sht_plan *p, const double *wa, int ldw, int nb, double *xya, int ldi, int ldj, int mode)
{
  int rc = check_strided(p, xya, ldi, ldj, nb, wa, ldw, mode);
  if (rc || nb == 0) return rc;
  return strided_call(p, false, nullptr, xya, ldi, ldj, nb, wa, nullptr, ldw, mode, false);
}

static int diffuse_impl(sht_plan *p, double *w, int nb, const double *coef, double dt, const double *filter, bool host)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (nb < 0 || (nb > 0 && (!w || !coef))) { set_error("diffuse: bad argument"); return SHT_ERR_INVALID_ARG; }
  if (nb == 0) return SHT_OK;
  std::lock_guard<std::mutex> lk(p->mtx);
  DeviceGuard g(p->device);
  if (!g.ok) { set_error("cudaSetDevice failed"); return SHT_ERR_CUDA; }
  cudaStream_t s = p->stream;
  cudaError_t e;
  if (!host) return launch_diffuse(p, w, nb, coef, dt, filter, s);
  const size_t nw = (size_t)nb * p->L;
  if ((rc = ensure_io(p, sizeof(double) * (nw + 2 * p->L) + 1024))) return rc;
  double *dw = static_cast<double *>(p->d_io), *dc = dw + nw, *df = dc + p->L;
  if ((e = cudaMemcpyAsync(dw, w, sizeof(double) * nw, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(dc, coef, sizeof(double) * p->L, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (filter && (e = cudaMemcpyAsync(df, filter, sizeof(double) * p->L, cudaMemcpyHostToDevice, s)) != cudaSuccess))
    return cuda_fail(e, "H2D");
  if ((rc = launch_diffuse(p, dw, nb, dc, dt, filter ? df : nullptr, s))) return rc;
  if ((e = cudaMemcpyAsync(w, dw, sizeof(double) * nw, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return cuda_fail(e, "D2H");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "diffuse");
  return SHT_OK;
}

int sht_wa_diffuse(sht_plan *p, double *w, int nb, const double *coef, double dt, const double *filter)
{ return diffuse_impl(p, w, nb, coef, dt, filter, true); }
int sht_wa_diffuse_dev(sht_plan *p, double *w, int nb, const double *coef, double dt, const double *filter)
{ return diffuse_impl(p, w, nb, coef, dt, filter, false); }

int sht_roundtrip_diffuse_dev(sht_plan *p, double *xya, int nb, const double *coef, double dt, const double *filter)
{
  int rc = check_plan(p);
  if (rc) return rc;
  if (nb < 0 || (nb > 0 && !xya)) { set_error("roundtrip: bad argument"); return SHT_ERR_INVALID_ARG; }
  if ((reinterpret_cast<uintptr_t>(xya) & 15u) != 0) { set_error("device grid arrays must be 16-byte aligned"); return SHT_ERR_INVALID_ARG; }
  if (nb == 0) return SHT_OK;
  std::lock_guard<std::mutex> lk(p->mtx);
  DeviceGuard g(p->device);
  if (!g.ok) { set_error("cudaSetDevice failed"); return SHT_ERR_CUDA; }
  Workspace ws{};
  if ((rc = ensure_ws(p, nb, nb, &ws))) return rc;
  if ((rc = run_analysis(p, PACK_PLAIN, RS_FWD_PLAIN, xya, nullptr, nb, ws.W, nullptr))) return rc;
  if (coef && (rc = launch_diffuse(p, ws.W, nb, coef, dt, filter, p->stream))) return rc;
  return run_synthesis(p, UNPACK_PLAIN, RS_INV_PLAIN, ws.W, nullptr, nb, xya, nullptr);
}

}  // extern "C"
