// sht_multi.cu -- many independent transform instances as one step.
//
// Instances that share a plan (one grid and truncation) are concatenated into
// one column range: per-column pointer tables tell the longitude transforms
// where each field-level's grid lives and the spectral conversions where its
// SPML vector lives, so the instances of a plan cost one launch per stage, the
// same as one batched call.  Plans run side by side on their own streams,
// forked from and joined into the batch's stream.  Each step kind is captured
// once as a CUDA graph (fork, per-plan stages, join) and replayed.
//
// The tuner times, per plan, every Legendre variant that covers the grid
// (paired persistent, latitude-chunked persistent and per-band FP64, and split
// precision on the tensor cores when allowed) on the plan's own columns and
// keeps the fastest.
//
// Workspaces belong to the batch, not to the plans, so single-plan calls made
// between runs cannot move memory that a captured graph refers to.
#include "sht_internal.h"

#include <algorithm>

namespace {

constexpr uint32_t kMultiMagic = 0x4D554C54u;  // "MULT"

struct Inst {
  sht_plan *plan;
  int nb;
  double *wa, *xya;
};

struct Group {
  sht_plan *plan = nullptr;
  std::vector<int> members;     // instance indices, in registration order
  int ncol = 0;                 // total field-levels
  const double **d_gcol = nullptr;  // ncol grid column pointers (device)
  double **d_wcol = nullptr;        // ncol spectral column pointers (device)
  double2 *F = nullptr, *S = nullptr;
  int precision = SHT_PREC_FP64, leg_kernel = 0, leg_tile = 0;
  int sm_cap = 0;               // SMs its persistent kernels size their grids for (0: all)
  float tuned_ms = 0.f;
  cudaEvent_t join = nullptr;
};

}  // namespace

struct sht_multi_s {
  uint32_t magic = kMultiMagic;
  int device = 0;
  cudaStream_t stream = nullptr;      // own stream: warm-up, tuning and capture
  cudaStream_t run_stream = nullptr;  // stream the runs are ordered on (default: own)
  cudaEvent_t fork = nullptr;
  std::vector<Inst> inst;
  std::vector<Group> groups;
  bool built = false, use_graph = true;
  cudaGraphExec_t exec[4] = {};
  int kernels[4] = {};
  std::mutex mtx;
};

namespace sht {
namespace {

struct DevGuard {
  int prev = -1;
  bool ok = true;
  explicit DevGuard(int dev)
  {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) ok = (cudaSetDevice(dev) == cudaSuccess);
  }
  ~DevGuard()
  {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

bool live(const sht_multi *m) { return m && m->magic == kMultiMagic; }

// Holds the plan mutexes of all groups (in group order, which is plan-address
// order) and points each plan at its own stream with the group's Legendre
// configuration; everything is restored on release.
struct PlanLease {
  struct Saved { sht_plan *p; cudaStream_t stream; int precision, leg_kernel, leg_tile, sm_cap; bool timing; };
  std::vector<Saved> saved;
  explicit PlanLease(sht_multi *m)
  {
    for (Group &g : m->groups) {
      g.plan->mtx.lock();
      saved.push_back({g.plan, g.plan->stream, g.plan->precision, g.plan->leg_kernel, g.plan->leg_tile,
                       g.plan->sm_cap, g.plan->timing.on});
      g.plan->stream = g.plan->own_stream;
      g.plan->timing.on = false;
      apply(g);
    }
  }
  static void apply(const Group &g)
  {
    g.plan->precision = g.precision;
    g.plan->leg_kernel = g.leg_kernel;
    g.plan->leg_tile = g.leg_tile;
    g.plan->sm_cap = g.sm_cap;
  }
  ~PlanLease()
  {
    for (auto it = saved.rbegin(); it != saved.rend(); ++it) {
      it->p->stream = it->stream;
      it->p->precision = it->precision;
      it->p->leg_kernel = it->leg_kernel;
      it->p->leg_tile = it->leg_tile;
      it->p->sm_cap = it->sm_cap;
      it->p->timing.on = it->timing;
      it->p->mtx.unlock();
    }
  }
};

int group_step(Group &g, int what)
{
  sht_plan *p = g.plan;
  int rc = SHT_OK;
  if (what & SHT_MULTI_SYNTHESIS)
    rc = run_synthesis_cols(p, g.d_wcol, g.ncol, const_cast<double *const *>(g.d_gcol), g.F, g.S, p->stream);
  if (!rc && (what & SHT_MULTI_ANALYSIS))
    rc = run_analysis_cols(p, g.d_gcol, g.ncol, g.d_wcol, g.F, g.S, p->stream);
  return rc;
}

// fork from `origin`, run every group on its plan's stream, join back
int enqueue_step(sht_multi *m, int what, cudaStream_t origin)
{
  cudaError_t e;
  if ((e = cudaEventRecord(m->fork, origin)) != cudaSuccess) return cuda_fail(e, "multi fork");
  for (Group &g : m->groups) {
    if ((e = cudaStreamWaitEvent(g.plan->stream, m->fork, 0)) != cudaSuccess) return cuda_fail(e, "multi fork wait");
    int rc = group_step(g, what);
    if (rc) return rc;
    if ((e = cudaEventRecord(g.join, g.plan->stream)) != cudaSuccess) return cuda_fail(e, "multi join");
    if ((e = cudaStreamWaitEvent(origin, g.join, 0)) != cudaSuccess) return cuda_fail(e, "multi join wait");
  }
  return SHT_OK;
}

int check_device_errors(sht_multi *m)
{
  for (Group &g : m->groups) {
    int rc = device_error_status(g.plan);
    if (rc) return rc;
  }
  return SHT_OK;
}

// Mean time of one round trip of group g in the current configuration.
int time_group(Group &g, int reps, float *ms)
{
  sht_plan *p = g.plan;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e;
  int rc = SHT_OK;
  if ((e = cudaEventCreate(&a)) != cudaSuccess || (e = cudaEventCreate(&b)) != cudaSuccess) {
    rc = cuda_fail(e, "tuner events");
  } else {
    rc = group_step(g, SHT_MULTI_ROUND_TRIP);  // warm-up (builds lazy tables)
    if (!rc && (e = cudaStreamSynchronize(p->stream)) != cudaSuccess) rc = cuda_fail(e, "tuner warm-up");
    if (!rc) rc = device_error_status(p);
    if (!rc) cudaEventRecord(a, p->stream);
    for (int r = 0; r < reps && !rc; ++r) rc = group_step(g, SHT_MULTI_ROUND_TRIP);
    if (!rc) {
      cudaEventRecord(b, p->stream);
      if ((e = cudaEventSynchronize(b)) != cudaSuccess) rc = cuda_fail(e, "tuner timing");
    }
    if (!rc) {
      float t = 0.f;
      cudaEventElapsedTime(&t, a, b);
      *ms = t / reps;
    }
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  return rc;
}

int tune_group(Group &g, bool allow_split)
{
  // kernel families and their tiles: analysis columns per item of the paired
  // kernels, latitudes per chunk of the chunked kernels (a tile a kernel
  // cannot take falls back to its automatic one and is timed again
  // harmlessly), and the single-kernel transform of small grids
  struct Cand { int precision, leg_kernel, leg_tile; };
  std::vector<Cand> cands;
  if (leg_pair_supported(g.plan)) {
    cands.push_back({SHT_PREC_FP64, 2, 8});
    cands.push_back({SHT_PREC_FP64, 2, 16});
  }
  if (leg_chunk_supported(g.plan)) {
    cands.push_back({SHT_PREC_FP64, 3, 16});
    cands.push_back({SHT_PREC_FP64, 3, 32});
  }
  cands.push_back({SHT_PREC_FP64, 1, 0});
  if (small_supported(g.plan)) cands.push_back({SHT_PREC_FP64, 4, 0});  // one kernel per direction
  if (allow_split && split_supported(g.plan)) {
    cands.push_back({SHT_PREC_SPLIT, 0, 0});
    cands.push_back({SHT_PREC_AUTO, 0, 0});  // split where the contraction is long, FP64 elsewhere
  }
  float best = 0.f;
  Cand win = cands.front();
  for (const Cand &c : cands) {
    g.precision = c.precision;
    g.leg_kernel = c.leg_kernel;
    g.leg_tile = c.leg_tile;
    PlanLease::apply(g);
    float ms = 0.f;
    int rc = time_group(g, 3, &ms);
    if (rc) return rc;
    if (best == 0.f || ms < best) { best = ms; win = c; }
  }
  g.precision = win.precision;
  g.leg_kernel = win.leg_kernel;
  g.leg_tile = win.leg_tile;
  g.tuned_ms = best;
  PlanLease::apply(g);
  return SHT_OK;
}

// Mean time of `reps` eager round-trip steps of the whole batch.
int time_step(sht_multi *m, int reps, float *ms)
{
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e;
  int rc = SHT_OK;
  if ((e = cudaEventCreate(&a)) != cudaSuccess || (e = cudaEventCreate(&b)) != cudaSuccess) {
    rc = cuda_fail(e, "tuner events");
  } else {
    rc = enqueue_step(m, SHT_MULTI_ROUND_TRIP, m->stream);  // warm-up
    if (!rc) cudaEventRecord(a, m->stream);
    for (int r = 0; r < reps && !rc; ++r) rc = enqueue_step(m, SHT_MULTI_ROUND_TRIP, m->stream);
    if (!rc) {
      cudaEventRecord(b, m->stream);
      if ((e = cudaEventSynchronize(b)) != cudaSuccess) rc = cuda_fail(e, "tuner timing");
    }
    if (!rc) {
      float t = 0.f;
      cudaEventElapsedTime(&t, a, b);
      *ms = t / reps;
    }
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  return rc ? rc : check_device_errors(m);
}

// The groups run on their own streams, but each persistent kernel sizes its
// grid for the whole GPU, so a kernel of one group waits for the SMs another
// holds.  Alternatively every group's persistent kernels are sized for a
// share of the SMs in proportion to its tuned time (its columns when not
// tuned), so that the groups run side by side.
void share_sms(sht_multi *m)
{
  float sum = 0.f;
  for (const Group &g : m->groups) sum += g.tuned_ms > 0.f ? g.tuned_ms : (float)g.ncol;
  const int nsm = m->groups.front().plan->num_sms;
  for (Group &g : m->groups) {
    const float w = g.tuned_ms > 0.f ? g.tuned_ms : (float)g.ncol;
    const int share = (int)(nsm * (w / sum) + 0.5f);
    g.sm_cap = share < 4 ? 4 : share;
    PlanLease::apply(g);
  }
}

// the tuner keeps whichever of whole-GPU grids and shared SMs measures faster
int tune_partition(sht_multi *m)
{
  float whole = 0.f, split = 0.f;
  int rc = time_step(m, 3, &whole);
  if (rc) return rc;
  share_sms(m);
  if ((rc = time_step(m, 3, &split))) return rc;
  if (!(split < whole)) {
    for (Group &g : m->groups) {
      g.sm_cap = 0;
      PlanLease::apply(g);
    }
  }
  return SHT_OK;
}

void free_groups(sht_multi *m)
{
  for (auto &x : m->exec)
    if (x) { cudaGraphExecDestroy(x); x = nullptr; }
  for (Group &g : m->groups) {
    cudaFree(g.d_gcol); cudaFree(g.d_wcol); cudaFree(g.F);
    if (g.join) cudaEventDestroy(g.join);
  }
  m->groups.clear();
  m->built = false;
}

int build(sht_multi *m, int flags)
{
  free_groups(m);
  // group by plan, in plan-address order (a fixed lock order across batches)
  std::vector<sht_plan *> plans;
  for (const Inst &x : m->inst) plans.push_back(x.plan);
  std::sort(plans.begin(), plans.end());
  plans.erase(std::unique(plans.begin(), plans.end()), plans.end());
  cudaError_t e;
  for (sht_plan *p : plans) {
    Group g;
    g.plan = p;
    for (int i = 0; i < (int)m->inst.size(); ++i)
      if (m->inst[i].plan == p) { g.members.push_back(i); g.ncol += m->inst[i].nb; }
    std::vector<const double *> gc;
    std::vector<double *> wc;
    const long long IJ = (long long)p->I * p->J;
    for (int i : g.members)
      for (int k = 0; k < m->inst[i].nb; ++k) {
        gc.push_back(m->inst[i].xya + k * IJ);
        wc.push_back(m->inst[i].wa + (long long)k * p->L);
      }
    const size_t fbytes = sizeof(double2) * (size_t)(p->N + 1) * g.ncol * p->J;
    const size_t sbytes = sizeof(double2) * (size_t)p->R * g.ncol;
    m->groups.push_back(g);
    Group &G = m->groups.back();
    if ((e = cudaMalloc(&G.d_gcol, sizeof(double *) * gc.size())) != cudaSuccess ||
        (e = cudaMalloc(&G.d_wcol, sizeof(double *) * wc.size())) != cudaSuccess ||
        (e = cudaMalloc(&G.F, ((fbytes + 255) & ~(size_t)255) + sbytes)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&G.join, cudaEventDisableTiming)) != cudaSuccess)
      return cuda_fail(e, "multi group allocation");
    G.S = reinterpret_cast<double2 *>(reinterpret_cast<char *>(G.F) + ((fbytes + 255) & ~(size_t)255));
    if ((e = cudaMemcpy(G.d_gcol, gc.data(), sizeof(double *) * gc.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(G.d_wcol, wc.data(), sizeof(double *) * wc.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
      return cuda_fail(e, "multi column tables");
    G.precision = p->precision;
    G.leg_kernel = p->leg_kernel;
    G.leg_tile = p->leg_tile;
  }

  PlanLease lease(m);
  int rc = SHT_OK;
  if (flags & SHT_MULTI_AUTOTUNE)
    for (Group &g : m->groups)
      if ((rc = tune_group(g, (flags & SHT_MULTI_ALLOW_SPLIT) != 0))) return rc;
  // one eager step: builds every lazily created table before capture
  if ((rc = enqueue_step(m, SHT_MULTI_ROUND_TRIP, m->stream))) return rc;
  if ((e = cudaStreamSynchronize(m->stream)) != cudaSuccess) return cuda_fail(e, "multi warm-up");
  if ((rc = check_device_errors(m))) return rc;
  if (flags & SHT_MULTI_SIDE_BY_SIDE) {
    share_sms(m);
    if ((rc = enqueue_step(m, SHT_MULTI_ROUND_TRIP, m->stream))) return rc;
    if ((e = cudaStreamSynchronize(m->stream)) != cudaSuccess) return cuda_fail(e, "multi warm-up");
    if ((rc = check_device_errors(m))) return rc;
  } else if ((flags & SHT_MULTI_AUTOTUNE) && m->groups.size() > 1 && (rc = tune_partition(m))) {
    return rc;
  }

  // Capture each step kind: the graph is kept for replay unless the batch
  // runs stage by stage, and the capture counts the kernels of one step.
  m->use_graph = !(flags & SHT_MULTI_NO_GRAPH);
  for (int what = 1; what <= 3; ++what) {
    const long long before = sht_launch_count();
    cudaGraph_t graph = nullptr;
    if ((e = cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return cuda_fail(e, "multi capture begin");
    rc = enqueue_step(m, what, m->stream);
    e = cudaStreamEndCapture(m->stream, &graph);
    m->kernels[what] = (int)(sht_launch_count() - before);
    count_launch(-m->kernels[what]);  // captured launches have not run
    if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
    if (e != cudaSuccess) return cuda_fail(e, "multi capture end");
    if (m->use_graph) e = cudaGraphInstantiate(&m->exec[what], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "multi graph instantiate");
  }
  m->built = true;
  return SHT_OK;
}

}  // namespace
}  // namespace sht

using namespace sht;

extern "C" {

int sht_multi_create(sht_multi **multi)
{
  if (!multi) { set_error("multi: null output"); return SHT_ERR_INVALID_ARG; }
  *multi = nullptr;
  int dev = 0, n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_error("multi: no CUDA device");
    return SHT_ERR_NO_DEVICE;
  }
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e, "multi device");
  auto *m = new sht_multi_s();
  m->device = dev;
  if ((e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&m->fork, cudaEventDisableTiming)) != cudaSuccess) {
    int rc = cuda_fail(e, "multi stream");
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return rc;
  }
  m->run_stream = m->stream;
  *multi = m;
  return SHT_OK;
}

int sht_multi_add(sht_multi *m, sht_plan *plan, int nb, double *wa, double *xya, int *instance)
{
  if (!live(m)) { set_error("multi: not a batch"); return SHT_ERR_INVALID_ARG; }
  if (!plan || plan->magic != kPlanMagic) { set_error("multi: plan is not initialised"); return SHT_ERR_NOT_INITIALIZED; }
  if (nb <= 0 || !wa || !xya) { set_error("multi: instance needs nb > 0 and both arrays"); return SHT_ERR_INVALID_ARG; }
  if (plan->device != m->device) { set_error("multi: plan lives on another device"); return SHT_ERR_INVALID_ARG; }
  if ((reinterpret_cast<uintptr_t>(xya) & 15u) || (reinterpret_cast<uintptr_t>(wa) & 7u)) {
    set_error("multi: grid arrays must be 16-byte aligned, spectral arrays 8-byte aligned");
    return SHT_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lk(m->mtx);
  m->inst.push_back({plan, nb, wa, xya});
  m->built = false;
  if (instance) *instance = (int)m->inst.size() - 1;
  return SHT_OK;
}

int sht_multi_build(sht_multi *m, int flags)
{
  if (!live(m)) { set_error("multi: not a batch"); return SHT_ERR_INVALID_ARG; }
  std::lock_guard<std::mutex> lk(m->mtx);
  if (m->inst.empty()) { set_error("multi: no instances"); return SHT_ERR_INVALID_ARG; }
  DevGuard g(m->device);
  if (!g.ok) { set_error("cudaSetDevice failed"); return SHT_ERR_CUDA; }
  int rc = build(m, flags);
  if (rc) free_groups(m);
  return rc;
}

int sht_multi_run(sht_multi *m, int what)
{
  if (!live(m)) { set_error("multi: not a batch"); return SHT_ERR_INVALID_ARG; }
  if (what < SHT_MULTI_SYNTHESIS || what > SHT_MULTI_ROUND_TRIP) { set_error("multi: unknown step"); return SHT_ERR_INVALID_ARG; }
  std::lock_guard<std::mutex> lk(m->mtx);
  if (!m->built) { set_error("multi: call sht_multi_build first"); return SHT_ERR_NOT_INITIALIZED; }
  DevGuard g(m->device);
  if (!g.ok) { set_error("cudaSetDevice failed"); return SHT_ERR_CUDA; }
  if (m->use_graph) {
    cudaError_t e = cudaGraphLaunch(m->exec[what], m->run_stream);
    if (e != cudaSuccess) return cuda_fail(e, "multi graph launch");
    count_launch(m->kernels[what]);
    return SHT_OK;
  }
  PlanLease lease(m);
  return enqueue_step(m, what, m->run_stream);
}

int sht_multi_set_stream(sht_multi *m, void *stream)
{
  if (!live(m)) { set_error("multi: not a batch"); return SHT_ERR_INVALID_ARG; }
  std::lock_guard<std::mutex> lk(m->mtx);
  m->run_stream = static_cast<cudaStream_t>(stream);
  return SHT_OK;
}

int sht_multi_synchronize(sht_multi *m)
{
  if (!live(m)) { set_error("multi: not a batch"); return SHT_ERR_INVALID_ARG; }
  std::lock_guard<std::mutex> lk(m->mtx);
  DevGuard g(m->device);
  cudaError_t e = cudaStreamSynchronize(m->run_stream);
  if (e != cudaSuccess) return cuda_fail(e, "multi synchronize");
  return check_device_errors(m);
}

int sht_multi_groups(const sht_multi *m, int *ngroups)
{
  if (!live(m) || !ngroups) { set_error("multi: bad argument"); return SHT_ERR_INVALID_ARG; }
  *ngroups = (int)m->groups.size();
  return SHT_OK;
}

int sht_multi_group_info(const sht_multi *m, int group, int *ncol, int *precision, int *legendre_kernel, float *tuned_ms)
{
  if (!live(m) || group < 0 || group >= (int)m->groups.size()) { set_error("multi: bad group"); return SHT_ERR_INVALID_ARG; }
  const Group &g = m->groups[group];
  if (ncol) *ncol = g.ncol;
  if (precision) *precision = g.precision;
  if (legendre_kernel) *legendre_kernel = g.leg_kernel;
  if (tuned_ms) *tuned_ms = g.tuned_ms;
  return SHT_OK;
}

int sht_multi_group_sms(const sht_multi *m, int group, int *sms)
{
  if (!live(m) || !sms || group < 0 || group >= (int)m->groups.size()) {
    set_error("multi: bad group");
    return SHT_ERR_INVALID_ARG;
  }
  *sms = m->groups[group].sm_cap;
  return SHT_OK;
}

int sht_multi_group_tile(const sht_multi *m, int group, int *legendre_tile)
{
  if (!live(m) || !legendre_tile || group < 0 || group >= (int)m->groups.size()) {
    set_error("multi: bad group");
    return SHT_ERR_INVALID_ARG;
  }
  *legendre_tile = m->groups[group].leg_tile;
  return SHT_OK;
}

int sht_multi_kernels(const sht_multi *m, int what, int *nkernels)
{
  if (!live(m) || !nkernels || what < SHT_MULTI_SYNTHESIS || what > SHT_MULTI_ROUND_TRIP) {
    set_error("multi: bad argument");
    return SHT_ERR_INVALID_ARG;
  }
  *nkernels = m->kernels[what];
  return SHT_OK;
}

int sht_multi_destroy(sht_multi *m)
{
  if (!live(m)) { set_error("multi: not a batch"); return SHT_ERR_INVALID_ARG; }
  {
    std::lock_guard<std::mutex> lk(m->mtx);
    DevGuard g(m->device);
    cudaStreamSynchronize(m->run_stream);
    cudaStreamSynchronize(m->stream);
    free_groups(m);
    cudaEventDestroy(m->fork);
    cudaStreamDestroy(m->stream);
    m->magic = 0;
  }
  delete m;
  return SHT_OK;
}

}  // extern "C"
