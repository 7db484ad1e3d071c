// fa_server.cu -- the serving loop behind fa_server_* (include/fa_b200.h): continuous batching of
// frames from several acquisitions on one device.
//
// One worker thread owns all device work. Per acquisition (one FrameWarpAligner each,
// FrameWarpAligner.cpp:77-251): the reference, gradient, Hessian blocks, phase correlator and the
// last solution stay resident; submitted frames wait in a FIFO until a frame slot is free and the
// slot memory fits the server's budget, then upload, convert (+1 offset) and phase-correlate on the
// acquisition's own stream. Per class of frames that can share a kernel (dimensionality, slot
// storage, reference precision, row width a multiple of 4): a job table of max_in_flight entries, a
// CUDA graph of iterations_per_launch x (compact, fused pass, trust-region step) + compact, and a
// stream. Between graph launches newly correlated frames are activated (device-side zero start),
// finished frames are read from host-mapped reports and their slots reused; host callbacks on the
// streams wake the worker, so uploads and correlations of new frames overlap the solves of others.
//
// Determinism: a frame's fused passes and steps use only its own tiles, partial sums and state, so
// its result is the same whichever frames share its launches. With a warm-start lag d, frame k of an
// acquisition evaluates its cold starting points (zero, rigid) as soon as it is correlated, then waits
// on the device (out of the passes) until frame k-d has written its solution to the warm-start ring
// entry stamped with k-d's sequence number, and continues from that fourth starting point; results
// therefore do not depend on arrival timing either.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <unordered_map>
#include <unordered_set>

#include "fa_runtime.h"

using fa::Job;
using namespace fa_rt;

namespace {

constexpr int kAdmitMax = 32;  // frames admitted per acquisition per intake (one correlator call)

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct SrvRequest {
  unsigned long long ticket = 0;
  int acq = -1;
  const void* data = nullptr;
  bool on_device = false;
  double t_submit = 0;
};

struct SrvResult {
  fa_status status = FA_OK;
  std::string error;
  std::vector<double> D;
  fa_align_stats stats{};
  double latency_ms = 0;
};

struct SrvClass;
struct SrvAcq;

// fa_server_reserve's request to the worker.
struct SrvReserve {
  int acq = -1;
  int n = 0;
  bool done = false;
  fa_status status = FA_OK;
  std::string error;
};

struct SrvSlot {
  SrvAcq* acq = nullptr;
  fa_frame* F = nullptr;      // zero-halo frame storage + solve buffers
  int index = -1;             // entry in the class job table
  void* raw = nullptr;        // dense raw frame uploaded from the host
  float* vol = nullptr;       // downsampled frame for the correlator (spatial_binning > 1)
  char* report = nullptr;     // host-mapped FrameState + P doubles (written by the solve kernel)
  size_t bytes = 0;           // device bytes charged to the server budget
  std::vector<Alloc> allocs;  // raw / vol
  SrvRequest req;
  long long seq = 0;          // admission order within the acquisition
  double rigid[3] = {0, 0, 0};
};

struct SrvAcq {
  int id = -1;
  fa_aligner* A = nullptr;
  fa_dtype dtype = FA_F32;   // frame dtype
  int kind = 0;              // slot FrameKind
  SrvClass* cls = nullptr;
  size_t raw_bytes = 0;
  std::deque<SrvRequest> pending;
  std::vector<SrvSlot*> idle;
  int n_busy = 0;            // admitted, not finished
  int n_slots = 0;           // slots that exist (busy or idle)
  long long next_seq = 0;
  std::map<long long, SrvSlot*> ready;      // correlated, waiting to start (by sequence number)
  bool corr_busy = false;
  std::vector<SrvSlot*> corr_slots;
  cudaEvent_t corr_ev = nullptr;
  long long* h_idx = nullptr;  // pinned: peak indices of the last correlator call
  double* warm = nullptr;        // device, lag x P doubles: frame k reads and writes entry k % lag
  long long* warm_seq = nullptr; // device, lag: sequence number of the frame whose solution each entry holds
  std::vector<Alloc> allocs;
};

struct SrvClass {
  int n_dim = 0, kind = 0;
  bool bf16 = false, vec4 = false;
  int cap = 0;
  Job* jobs_dev = nullptr;
  Job* h_jobs = nullptr;              // pinned shadow of the table (entry uploads)
  int* list = nullptr;                // active list
  int* prefix = nullptr;              // cap + 1
  int* busy = nullptr;
  int* counts = nullptr;              // [n_active, n_done, done list (cap)]
  int* h_counts = nullptr;            // pinned copy, written by the graph's last node
  fa::Activation* d_act = nullptr;
  fa::Activation* h_act = nullptr;    // pinned
  fa::FrameState* dummy = nullptr;    // phase Done, for unused entries
  std::vector<SrvSlot*> owner;
  std::vector<int> free_idx;
  std::vector<SrvAcq*> acqs;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool dirty = true;
  cudaEvent_t ev = nullptr;
  bool running = false;
  int in_solve = 0;
  int max_nD = 0, max_tiles = 0, mb = 2, grid_mult = 2;
  long long tuned_for = -1;  // N of the acquisition whose tuning the class uses
  std::vector<Alloc> allocs;
};

}  // namespace

struct fa_server {
  fa_context* ctx = nullptr;
  fa_server_config cfg{};
  int sms = 148;
  // shared with submitting threads (mu)
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool wake = false;
  bool stop = false;
  std::deque<SrvRequest> inbox;
  std::deque<SrvReserve*> reserves;
  std::vector<std::unique_ptr<SrvAcq>> acqs;
  std::unordered_map<unsigned long long, SrvResult> results;
  std::unordered_set<unsigned long long> outstanding;
  unsigned long long next_ticket = 1;
  fa_status fatal = FA_OK;
  std::string fatal_msg;
  std::vector<double> latencies_ms;
  double t_first_submit = -1, t_last_done = -1;
  long long submitted = 0, completed = 0, failed = 0;
  long long peak_in_flight = 0;
  size_t peak_slot_bytes = 0;
  std::atomic<size_t> slot_bytes{0};
  std::atomic<long long> in_flight{0};
  std::atomic<long long> graph_launches{0};
  // worker only
  std::vector<SrvAcq*> wacqs;
  std::vector<std::unique_ptr<SrvClass>> classes;
  std::vector<std::unique_ptr<SrvSlot>> slots;
  size_t rr = 0;  // round-robin start of admission
  std::thread worker;
};

namespace {

void CUDART_CB wake_worker(void* p) {
  fa_server* S = static_cast<fa_server*>(p);
  std::lock_guard<std::mutex> lk(S->mu);
  S->wake = true;
  S->cv_work.notify_one();
}

size_t slot_estimate(const SrvAcq* q) {
  const fa_reference* R = q->A->ref;
  const int hz = R->nz > 1 ? fa::kHaloZ : 0;
  const size_t esz = q->kind == fa::kFrameF32 ? 4 : 2;
  size_t b = (size_t)(R->nx + 2 * fa::kHaloX) * (R->ny + 2 * fa::kHaloY) * (R->nz + 2 * hz) * esz;
  b += (size_t)R->nD * fa::kDParamF4 * sizeof(float4) + (size_t)R->G.n_tiles * fa::kPartialDoubles * sizeof(double);
  b += sizeof(fa::FrameState) + sizeof(Job) + (size_t)R->P * sizeof(double) * (5 + 2 * R->n_dim + 3) + 64;
  b += q->raw_bytes;
  const fa_aligner* A = q->A;
  if (A->prm.spatial_binning > 1) b += (size_t)A->dz * A->dy * A->dx * sizeof(float);
  return b;
}

// ------------------------------------------------------------------ classes -----------------------

void class_release(fa_server* S, SrvClass* C);

fa_status class_create_impl(fa_server* S, SrvClass* C);

fa_status class_create(fa_server* S, int n_dim, int kind, bool bf16, bool vec4, SrvClass** out) {
  auto C = std::make_unique<SrvClass>();
  C->n_dim = n_dim;
  C->kind = kind;
  C->bf16 = bf16;
  C->vec4 = vec4;
  C->cap = S->cfg.max_in_flight;
  fa_status st = class_create_impl(S, C.get());
  if (st != FA_OK) {
    std::string keep = g_err;
    class_release(S, C.get());
    g_err = keep;
    return st;
  }
  *out = C.get();
  S->classes.push_back(std::move(C));
  return FA_OK;
}

// Device table, pinned staging, stream and event of a class.
fa_status class_create_impl(fa_server* S, SrvClass* C) {
  fa_context* ctx = S->ctx;
  const int cap = C->cap;
  FA_TRY(dalloc_t(ctx, (size_t)cap, &C->jobs_dev, C->allocs));
  FA_TRY(dalloc_t(ctx, (size_t)cap, &C->list, C->allocs));
  FA_TRY(dalloc_t(ctx, (size_t)cap + 1, &C->prefix, C->allocs));
  FA_TRY(dalloc_t(ctx, (size_t)cap, &C->busy, C->allocs));
  FA_TRY(dalloc_t(ctx, (size_t)cap + 2, &C->counts, C->allocs));
  FA_TRY(dalloc_t(ctx, (size_t)cap, &C->d_act, C->allocs));
  FA_TRY(dalloc_t(ctx, 1, &C->dummy, C->allocs));
  if (cudaMallocHost(&C->h_jobs, (size_t)cap * sizeof(Job)) != cudaSuccess ||
      cudaMallocHost(&C->h_counts, (size_t)(cap + 2) * sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&C->h_act, (size_t)cap * sizeof(fa::Activation)) != cudaSuccess)
    return fail(FA_ERR_OOM, "cudaMallocHost failed");
  FA_CU(cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking));
  FA_CU(cudaEventCreateWithFlags(&C->ev, cudaEventDisableTiming));
  fa::FrameState done{};
  done.phase = fa::kPhaseDone;
  Job empty{};
  empty.state = C->dummy;
  for (int i = 0; i < cap; i++) C->h_jobs[i] = empty;
  C->owner.assign(cap, nullptr);
  for (int i = cap - 1; i >= 0; i--) C->free_idx.push_back(i);
  FA_CU(cudaMemcpyAsync(C->dummy, &done, sizeof(done), cudaMemcpyHostToDevice, C->stream));
  FA_CU(cudaMemcpyAsync(C->jobs_dev, C->h_jobs, (size_t)cap * sizeof(Job), cudaMemcpyHostToDevice, C->stream));
  FA_CU(cudaMemsetAsync(C->busy, 0, (size_t)cap * sizeof(int), C->stream));
  FA_CU(cudaMemsetAsync(C->counts, 0, (size_t)(cap + 2) * sizeof(int), C->stream));
  FA_CU(cudaStreamSynchronize(C->stream));
  return FA_OK;
}

void class_release(fa_server* S, SrvClass* C) {
  if (C->stream) cudaStreamSynchronize(C->stream);
  if (C->exec) cudaGraphExecDestroy(C->exec);
  if (C->graph) cudaGraphDestroy(C->graph);
  if (C->ev) cudaEventDestroy(C->ev);
  if (C->stream) cudaStreamDestroy(C->stream);
  if (C->h_jobs) cudaFreeHost(C->h_jobs);
  if (C->h_counts) cudaFreeHost(C->h_counts);
  if (C->h_act) cudaFreeHost(C->h_act);
  dfree_all(S->ctx, C->allocs);
}

// Attaches an acquisition to the class its frames run in (created on first use).
fa_status attach(fa_server* S, SrvAcq* q) {
  const fa_reference* R = q->A->ref;
  const bool bf16 = R->prec == FA_PREC_MIXED;
  const bool vec4 = R->nx % 4 == 0;
  SrvClass* C = nullptr;
  for (auto& c : S->classes)
    if (c->n_dim == R->n_dim && c->kind == q->kind && c->bf16 == bf16 && c->vec4 == vec4) C = c.get();
  if (!S->cfg.shared_launches) C = nullptr;  // one launch group per acquisition
  if (!C) FA_TRY(class_create(S, R->n_dim, q->kind, bf16, vec4, &C));
  q->cls = C;
  C->acqs.push_back(q);
  C->max_nD = std::max(C->max_nD, R->nD);
  C->max_tiles = std::max(C->max_tiles, R->G.n_tiles);
  if (R->N > C->tuned_for) {  // the largest volume's register budget tuned for launches of a few frames
    C->tuned_for = R->N;
    C->mb = R->host.tune_mb_small;
    C->grid_mult = R->host.tune_mb_small;
  }
  C->dirty = true;
  return FA_OK;
}

// Graph of one launch: iterations_per_launch x (compact, fused pass, step), a final compact, and
// the copy of the counts and done list to pinned host memory.
fa_status class_capture(fa_server* S, SrvClass* C) {
  if (C->exec) cudaGraphExecDestroy(C->exec);
  if (C->graph) cudaGraphDestroy(C->graph);
  C->exec = nullptr;
  C->graph = nullptr;
  cudaStream_t s = C->stream;
  int* n_active = C->counts;
  int* n_done = C->counts + 1;
  int* done_list = C->counts + 2;
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    e = cudaMemsetAsync(n_done, 0, sizeof(int), s);
    for (int it = 0; it < S->cfg.iterations_per_launch && e == cudaSuccess; it++) {
      e = fa::launch_compact(C->jobs_dev, C->cap, C->list, n_active, C->prefix, C->busy, done_list, n_done, s);
      if (e == cudaSuccess) {
        if (C->vec4)
          e = fa::launch_eval4_active(C->jobs_dev, C->list, n_active, C->prefix, 2LL * C->cap * C->max_tiles,
                                      C->n_dim, C->kind, C->bf16, C->mb, C->grid_mult * S->sms, s);
        else
          e = fa::launch_eval(C->jobs_dev, C->cap, C->max_tiles, C->n_dim, C->kind, C->bf16, s, false);
      }
      if (e == cudaSuccess) e = fa::launch_solve(C->jobs_dev, C->cap, C->max_nD, C->n_dim, s, C->list, n_active);
    }
    if (e == cudaSuccess)
      e = fa::launch_compact(C->jobs_dev, C->cap, C->list, n_active, C->prefix, C->busy, done_list, n_done, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(C->h_counts, C->counts, (size_t)(C->cap + 2) * sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaError_t e2 = cudaStreamEndCapture(s, &C->graph);
    if (e == cudaSuccess) e = e2;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&C->exec, C->graph, 0);
  if (e != cudaSuccess) return fail(FA_ERR_CUDA, std::string("server graph: ") + cudaGetErrorString(e));
  C->dirty = false;
  return FA_OK;
}

// ------------------------------------------------------------------ slots -------------------------

// Releases a slot; always completes (after a device error the frees are best effort) and reports
// the first CUDA failure.
fa_status slot_destroy(fa_server* S, SrvSlot* sl) {
  SrvClass* C = sl->acq->cls;
  cudaError_t e = cudaSuccess;
  if (sl->index >= 0) {  // the table entry goes back to the dummy before its memory is freed
    Job empty{};
    empty.state = C->dummy;
    C->h_jobs[sl->index] = empty;
    e = cudaMemcpyAsync(C->jobs_dev + sl->index, C->h_jobs + sl->index, sizeof(Job), cudaMemcpyHostToDevice,
                        C->stream);
    cudaError_t e2 = cudaStreamSynchronize(C->stream);
    if (e == cudaSuccess) e = e2;
    C->owner[sl->index] = nullptr;
    C->free_idx.push_back(sl->index);
  }
  if (sl->F) fa_deregister_frame(sl->F);
  dfree_all(S->ctx, sl->allocs);
  if (sl->report) cudaFreeHost(sl->report);
  S->slot_bytes -= sl->bytes;
  if (sl->bytes) sl->acq->n_slots--;
  for (auto it = S->slots.begin(); it != S->slots.end(); ++it)
    if (it->get() == sl) {
      S->slots.erase(it);
      break;
    }
  if (e != cudaSuccess) return fail(FA_ERR_CUDA, std::string("slot release: ") + cudaGetErrorString(e));
  return FA_OK;
}

fa_status slot_create(fa_server* S, SrvAcq* q, SrvSlot** out) {
  SrvClass* C = q->cls;
  fa_aligner* A = q->A;
  fa_reference* R = A->ref;
  auto owned = std::make_unique<SrvSlot>();
  SrvSlot* sl = owned.get();
  sl->acq = q;
  S->slots.push_back(std::move(owned));
  auto undo = [&](fa_status st) {
    std::string keep = g_err;
    slot_destroy(S, sl);
    g_err = keep;
    return st;
  };
  fa_status st = frame_alloc(R, q->kind, &sl->F);
  if (st != FA_OK) return undo(st);
  if (cudaStreamSynchronize(sl->F->stream) != cudaSuccess) return undo(fail(FA_ERR_CUDA, "slot set-up"));
  if ((st = dalloc(S->ctx, q->raw_bytes, &sl->raw, sl->allocs)) != FA_OK) return undo(st);
  if (A->prm.spatial_binning > 1 &&
      (st = dalloc_t(S->ctx, (size_t)A->dz * A->dy * A->dx, &sl->vol, sl->allocs)) != FA_OK)
    return undo(st);
  const size_t rep = fa::kReportHeaderBytes + (size_t)R->P * sizeof(double);
  void* hp = nullptr;
  if (cudaHostAlloc(&hp, rep, cudaHostAllocMapped) != cudaSuccess) return undo(fail(FA_ERR_OOM, "cudaHostAlloc failed"));
  sl->report = static_cast<char*>(hp);
  void* rep_dev = nullptr;
  if (cudaHostGetDevicePointer(&rep_dev, hp, 0) != cudaSuccess)
    return undo(fail(FA_ERR_CUDA, "cudaHostGetDevicePointer failed"));
  size_t bytes = 0;
  for (const Alloc& a : sl->F->allocs) bytes += a.n;
  for (const Alloc& a : sl->allocs) bytes += a.n;
  sl->bytes = bytes;
  S->slot_bytes += bytes;
  q->n_slots++;
  sl->index = C->free_idx.back();
  C->free_idx.pop_back();
  C->owner[sl->index] = sl;
  // The entry is visible to every launch of the class from now on: its state starts as done, so the
  // frame stays out of the active list until it is activated.
  FA_CU(cudaMemcpyAsync(sl->F->state, C->dummy, sizeof(fa::FrameState), cudaMemcpyDeviceToDevice, C->stream));
  Job j = sl->F->job;
  j.state = sl->F->state;
  j.report = rep_dev;
  C->h_jobs[sl->index] = j;
  FA_CU(cudaMemcpyAsync(C->jobs_dev + sl->index, C->h_jobs + sl->index, sizeof(Job), cudaMemcpyHostToDevice,
                        C->stream));
  *out = sl;
  return FA_OK;
}

// An idle slot of the acquisition, or a new one if the class table and the memory budget allow
// (idle slots of other acquisitions are released to make room); null when neither.
fa_status slot_take(fa_server* S, SrvAcq* q, SrvSlot** out) {
  *out = nullptr;
  if (!q->idle.empty()) {
    *out = q->idle.back();
    q->idle.pop_back();
    return FA_OK;
  }
  const size_t need = slot_estimate(q);
  while (S->slot_bytes + need > S->cfg.memory_budget || q->cls->free_idx.empty()) {
    SrvAcq* victim = nullptr;
    for (SrvAcq* o : S->wacqs)
      if (o != q && !o->idle.empty() && (!victim || o->idle.size() > victim->idle.size())) victim = o;
    if (!victim) return FA_OK;
    if (q->cls->free_idx.empty() && victim->cls != q->cls) {
      bool any = false;  // the table is full: only a slot of the same class frees an entry
      for (SrvAcq* o : q->cls->acqs)
        if (o != q && !o->idle.empty()) {
          victim = o;
          any = true;
          break;
        }
      if (!any) return FA_OK;
    }
    SrvSlot* v = victim->idle.back();
    victim->idle.pop_back();
    FA_TRY(slot_destroy(S, v));
  }
  return slot_create(S, q, out);
}

// ------------------------------------------------------------------ results -----------------------

void deliver(fa_server* S, SrvSlot* sl, double t) {
  SrvAcq* q = sl->acq;
  const fa_reference* R = q->A->ref;
  const fa::FrameState st = *reinterpret_cast<const fa::FrameState*>(sl->report);
  const double* x = reinterpret_cast<const double*>(sl->report + fa::kReportHeaderBytes);
  SrvResult res;
  const int nd = R->n_dim;
  res.D.assign((size_t)R->nD * 3, 0.0);
  for (int k = 0; k < R->nD; k++)
    for (int c = 0; c < nd; c++) res.D[3 * k + c] = x[k * nd + c];
  res.stats.iterations = st.iter;
  res.stats.evaluations = st.evaluations;
  res.stats.accepted = st.accepted;
  res.stats.status = st.hit_max ? 1 : 0;
  res.stats.f_final = st.f;
  res.stats.radius_final = st.radius;
  res.latency_ms = (t - sl->req.t_submit) * 1e3;
  q->n_busy--;
  S->in_flight--;
  q->idle.push_back(sl);
  q->cls->in_solve--;
  std::lock_guard<std::mutex> lk(S->mu);
  S->latencies_ms.push_back(res.latency_ms);
  S->completed++;
  S->t_last_done = t;
  S->outstanding.erase(sl->req.ticket);
  S->results[sl->req.ticket] = std::move(res);
  S->cv_done.notify_all();
}

// Fails every request not yet delivered (the worker stops after a device error).
void fail_all(fa_server* S, fa_status st, const std::string& msg) {
  std::lock_guard<std::mutex> lk(S->mu);
  S->fatal = st;
  S->fatal_msg = msg;
  for (unsigned long long t : S->outstanding) {
    SrvResult r;
    r.status = st;
    r.error = msg;
    S->results[t] = std::move(r);
    S->failed++;
  }
  S->outstanding.clear();
  S->inbox.clear();
  S->cv_done.notify_all();
}

// ------------------------------------------------------------------ worker ------------------------

// Uploads, converts and phase-correlates the frames just admitted for one acquisition.
fa_status intake(fa_server* S, SrvAcq* q, std::vector<SrvSlot*>& batch) {
  fa_aligner* A = q->A;
  cudaStream_t s = A->corr->stream;
  const int m = (int)batch.size();
  std::vector<const void*> cin((size_t)m);
  int cin_kind = q->dtype;
  for (int i = 0; i < m; i++) {
    SrvSlot* sl = batch[i];
    fa_frame* F = sl->F;
    const void* src = sl->req.data;
    if (!sl->req.on_device) {
      FA_CU(cudaMemcpyAsync(sl->raw, src, q->raw_bytes, cudaMemcpyHostToDevice, s));
      src = sl->raw;
    }
    if (A->prm.smoothing > 0) {  // smoothStack, then + 1; the correlator keeps the raw frame
      FA_TRY(aligner_smooth(A, src, q->dtype, s));
      FA_CU(fa::launch_to_slot(A->smooth_out, FA_F32, F->data, q->kind, A->nz, A->ny, A->nx, F->job.fpitch,
                               F->job.fplane, true, s));
    } else {
      FA_CU(fa::launch_to_slot(src, q->dtype, F->data, q->kind, A->nz, A->ny, A->nx, F->job.fpitch, F->job.fplane,
                               true, s));
    }
    g_launches += 1;
    if (A->prm.spatial_binning > 1) {
      FA_CU(fa::launch_downsample(src, q->dtype, A->nz, A->ny, A->nx, A->prm.spatial_binning, sl->vol, s));
      g_launches += 1;
      cin[i] = sl->vol;
      cin_kind = FA_F32;
    } else {
      cin[i] = src;
    }
  }
  FA_TRY(correlator_enqueue(A->corr, cin.data(), cin_kind, m));
  FA_CU(cudaMemcpyAsync(q->h_idx, A->corr->d_idx, (size_t)m * sizeof(long long), cudaMemcpyDeviceToHost, s));
  FA_CU(cudaEventRecord(q->corr_ev, s));
  FA_CU(cudaLaunchHostFunc(s, wake_worker, S));
  q->corr_busy = true;
  q->corr_slots = batch;
  return FA_OK;
}

// Starts the next graph launch of a class with the frames ready to enter it.
fa_status class_launch(fa_server* S, SrvClass* C, bool* launched) {
  *launched = false;
  int n_act = 0;
  const long long lag = S->cfg.warm_start;
  for (SrvAcq* q : C->acqs) {
    for (auto it = q->ready.begin(); it != q->ready.end() && n_act < C->cap;) {
      // every correlated frame starts; one with a warm start waits on the device for frame seq - lag
      // (the first lag frames start cold)
      const long long seq = it->first;
      SrvSlot* sl = it->second;
      it = q->ready.erase(it);
      fa::Activation& a = C->h_act[n_act++];
      a.job = sl->index;
      a.use_warm = (lag > 0 && seq >= lag) ? 1 : 0;
      a.max_iter = q->A->prm.max_iterations;
      a.pair = C->vec4 ? 1 : 0;  // the persistent pass evaluates both cold starting points at once
      for (int c = 0; c < 3; c++) a.rigid[c] = sl->rigid[c];
      a.warm = lag > 0 ? q->warm + (size_t)(seq % lag) * q->A->ref->P : nullptr;
      a.warm_seq = lag > 0 ? q->warm_seq + seq % lag : nullptr;
      a.warm_need = seq - lag;
      a.seq = seq;
    }
  }
  if (n_act == 0 && C->in_solve == 0) return FA_OK;
  if (C->dirty) FA_TRY(class_capture(S, C));
  if (n_act > 0) {
    FA_CU(cudaMemcpyAsync(C->d_act, C->h_act, (size_t)n_act * sizeof(fa::Activation), cudaMemcpyHostToDevice,
                          C->stream));
    FA_CU(fa::launch_activate(C->jobs_dev, C->d_act, n_act, C->busy, C->stream));
    g_launches += 1;
  }
  FA_CU(cudaGraphLaunch(C->exec, C->stream));
  g_launches += 3 * S->cfg.iterations_per_launch + 1;
  FA_CU(cudaEventRecord(C->ev, C->stream));
  FA_CU(cudaLaunchHostFunc(C->stream, wake_worker, S));
  C->in_solve += n_act;
  C->running = true;
  S->graph_launches++;
  *launched = true;
  return FA_OK;
}

// One pass over completions, admissions and launches; *progress when anything changed.
fa_status worker_pass(fa_server* S, bool* progress) {
  *progress = false;
  // finished graph launches
  for (auto& cp : S->classes) {
    SrvClass* C = cp.get();
    if (!C->running) continue;
    cudaError_t e = cudaEventQuery(C->ev);
    if (e == cudaErrorNotReady) continue;
    if (e != cudaSuccess) return fail(FA_ERR_CUDA, std::string("server solve: ") + cudaGetErrorString(e));
    C->running = false;
    *progress = true;
    const double t = now_s();
    const int n_done = C->h_counts[1];
    for (int k = 0; k < n_done; k++) {
      const int idx = C->h_counts[2 + k];
      if (idx >= 0 && idx < C->cap && C->owner[idx]) deliver(S, C->owner[idx], t);
    }
  }
  // finished correlations
  for (SrvAcq* q : S->wacqs) {
    if (!q->corr_busy) continue;
    cudaError_t e = cudaEventQuery(q->corr_ev);
    if (e == cudaErrorNotReady) continue;
    if (e != cudaSuccess) return fail(FA_ERR_CUDA, std::string("server correlation: ") + cudaGetErrorString(e));
    q->corr_busy = false;
    *progress = true;
    const int b = q->A->prm.spatial_binning;
    for (size_t i = 0; i < q->corr_slots.size(); i++) {
      SrvSlot* sl = q->corr_slots[i];
      unravel_shift(q->A->corr, q->h_idx[i], sl->rigid);
      sl->rigid[0] *= b;  // FrameWarpAligner.cpp:186-188
      sl->rigid[1] *= b;
      q->ready[sl->seq] = sl;
    }
    q->corr_slots.clear();
  }
  // admissions, round robin over acquisitions
  const size_t na = S->wacqs.size();
  const int per_acq = std::max(2, S->cfg.max_in_flight / (int)std::max<size_t>(1, na));
  for (size_t k = 0; k < na; k++) {
    SrvAcq* q = S->wacqs[(S->rr + k) % na];
    if (q->corr_busy || q->pending.empty()) continue;
    std::vector<SrvSlot*> batch;
    while (!q->pending.empty() && (int)batch.size() < kAdmitMax && S->in_flight < S->cfg.max_in_flight &&
           q->n_busy < per_acq) {
      SrvSlot* sl = nullptr;
      FA_TRY(slot_take(S, q, &sl));
      if (!sl) break;
      sl->req = q->pending.front();
      q->pending.pop_front();
      sl->seq = q->next_seq++;
      q->n_busy++;
      S->in_flight++;
      batch.push_back(sl);
    }
    if (batch.empty()) continue;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->peak_in_flight = std::max<long long>(S->peak_in_flight, S->in_flight.load());
      S->peak_slot_bytes = std::max(S->peak_slot_bytes, S->slot_bytes.load());
    }
    FA_TRY(intake(S, q, batch));
    *progress = true;
  }
  if (na) S->rr = (S->rr + 1) % na;
  // graph launches
  for (auto& cp : S->classes) {
    if (cp->running) continue;
    bool launched = false;
    FA_TRY(class_launch(S, cp.get(), &launched));
    *progress = *progress || launched;
  }
  return FA_OK;
}

bool worker_idle(const fa_server* S) {
  for (const SrvAcq* q : S->wacqs)
    if (!q->pending.empty() || q->corr_busy || q->n_busy > 0) return false;
  for (const auto& c : S->classes)
    if (c->running) return false;
  return true;
}

// Creates the idle slots fa_server_reserve asked for (within the budget; no eviction).
fa_status serve_reserves(fa_server* S) {
  std::deque<SrvReserve*> todo;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    // requests for acquisitions this pass has not attached yet wait for the next pass
    std::deque<SrvReserve*> later;
    for (SrvReserve* r : S->reserves) {
      if (r->acq < (int)S->wacqs.size() && S->wacqs[r->acq]->cls)
        todo.push_back(r);
      else
        later.push_back(r);
    }
    S->reserves.swap(later);
    if (!S->reserves.empty()) S->wake = true;
  }
  for (SrvReserve* r : todo) {
    SrvAcq* q = S->wacqs[r->acq];
    fa_status st = FA_OK;
    std::string err;
    while (q->n_slots < r->n) {
      if (S->slot_bytes + slot_estimate(q) > S->cfg.memory_budget || q->cls->free_idx.empty()) {
        st = FA_ERR_OOM;
        err = "the server's memory budget or job table holds no more slots for this acquisition";
        break;
      }
      SrvSlot* sl = nullptr;
      st = slot_create(S, q, &sl);
      if (st != FA_OK) {
        err = g_err;
        break;
      }
      q->idle.push_back(sl);
    }
    const bool device_error = st == FA_ERR_CUDA;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      r->status = st;
      r->error = err;
      r->done = true;
      S->peak_slot_bytes = std::max(S->peak_slot_bytes, S->slot_bytes.load());
      S->cv_done.notify_all();
    }
    if (device_error) return fail(st, err);
  }
  return FA_OK;
}

// Longest a shutdown waits for submitted frames before failing the rest.
constexpr double kStopDeadlineS = 120.0;

void worker_main(fa_server* S) {
  cudaSetDevice(S->ctx->device);
  double stop_since = -1;
  for (;;) {
    std::deque<SrvRequest> incoming;
    bool stopping;
    size_t n_acq;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (!S->wake && S->inbox.empty() && !S->stop)
        S->cv_work.wait_for(lk, std::chrono::milliseconds(2),
                            [&] { return S->wake || !S->inbox.empty() || S->stop; });
      S->wake = false;
      incoming.swap(S->inbox);
      stopping = S->stop;
      n_acq = S->acqs.size();
      for (size_t i = S->wacqs.size(); i < n_acq; i++) S->wacqs.push_back(S->acqs[i].get());
    }
    fa_status st = FA_OK;
    for (SrvAcq* q : S->wacqs)
      if (!q->cls && st == FA_OK) st = attach(S, q);
    if (st == FA_OK) st = serve_reserves(S);
    for (SrvRequest& r : incoming) S->wacqs[r.acq]->pending.push_back(r);
    bool progress = true;
    while (st == FA_OK && progress) st = worker_pass(S, &progress);
    if (st != FA_OK) {
      fail_all(S, st, g_err);
      return;
    }
    if (stopping && worker_idle(S)) return;
    if (stopping) {
      if (stop_since < 0) stop_since = now_s();
      if (now_s() - stop_since > kStopDeadlineS) {
        fail_all(S, FA_ERR_TIMEOUT, "server destroyed before the frame finished");
        return;
      }
    }
  }
}

}  // namespace

// ================================================================== C ABI ==========================

extern "C" fa_status fa_server_create(fa_context* ctx, const fa_server_config* cfg, fa_server** out) {
  if (!ctx || !out) return fail(FA_ERR_BAD_ARG, "NULL argument");
  fa_server_config c{};
  if (cfg) c = *cfg;
  if (c.memory_budget == 0) c.memory_budget = (size_t)40 << 30;
  if (c.max_in_flight <= 0) c.max_in_flight = 256;
  if (c.iterations_per_launch <= 0) c.iterations_per_launch = 4;
  if (c.max_in_flight > 4096 || c.iterations_per_launch > 64 || c.warm_start < 0 || c.warm_start > 64)
    return fail(FA_ERR_BAD_ARG, "need max_in_flight <= 4096, iterations_per_launch <= 64, 0 <= warm_start <= 64");
  FA_CU(cudaSetDevice(ctx->device));
  fa_server* S = new fa_server;
  S->ctx = ctx;
  S->cfg = c;
  cudaDeviceGetAttribute(&S->sms, cudaDevAttrMultiProcessorCount, ctx->device);
  S->worker = std::thread(worker_main, S);
  *out = S;
  return FA_OK;
}

extern "C" fa_status fa_server_destroy(fa_server* S) {
  if (!S) return fail(FA_ERR_BAD_ARG, "NULL server");
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->cv_work.notify_one();
  }
  if (S->worker.joinable()) S->worker.join();
  cudaSetDevice(S->ctx->device);
  for (auto& c : S->classes) cudaStreamSynchronize(c->stream);
  for (auto& q : S->acqs)
    if (q->A && q->A->corr) cudaStreamSynchronize(q->A->corr->stream);
  while (!S->slots.empty()) slot_destroy(S, S->slots.back().get());
  for (auto& c : S->classes) class_release(S, c.get());
  for (auto& q : S->acqs) {
    if (q->corr_ev) cudaEventDestroy(q->corr_ev);
    if (q->h_idx) cudaFreeHost(q->h_idx);
    dfree_all(S->ctx, q->allocs);
    if (q->A) fa_aligner_destroy(q->A);
  }
  delete S;
  return FA_OK;
}

extern "C" fa_status fa_server_add_acquisition(fa_server* S, const fa_aligner_params* params, const void* reference,
                                               fa_dtype reference_dtype, int nz, int ny, int nx,
                                               const fa_scan_params* scan, fa_dtype frame_dtype, int* acquisition) {
  if (!S || !params || !reference || !scan || !acquisition) return fail(FA_ERR_BAD_ARG, "NULL argument");
  if (frame_dtype != FA_F32 && frame_dtype != FA_U16) return fail(FA_ERR_BAD_ARG, "frames must be FA_F32 or FA_U16");
  FA_CU(cudaSetDevice(S->ctx->device));
  auto q = std::make_unique<SrvAcq>();
  fa_aligner* A = nullptr;
  FA_TRY(fa_aligner_create(S->ctx, params, &A));
  q->A = A;
  auto undo = [&](fa_status st) {
    std::string keep = g_err;
    if (q->corr_ev) cudaEventDestroy(q->corr_ev);
    if (q->h_idx) cudaFreeHost(q->h_idx);
    dfree_all(S->ctx, q->allocs);
    fa_aligner_destroy(A);
    g_err = keep;
    return st;
  };
  fa_status st = fa_aligner_set_reference(A, reference, reference_dtype, nz, ny, nx, scan);
  if (st != FA_OK) return undo(st);
  q->dtype = frame_dtype;
  q->kind = slot_kind_for(A, frame_dtype);
  q->raw_bytes = (size_t)A->ref->N * dtype_size(frame_dtype);
  if (slot_estimate(q.get()) > S->cfg.memory_budget)
    return undo(fail(FA_ERR_OOM, "one frame slot of this acquisition (" + std::to_string(slot_estimate(q.get())) +
                                     " bytes) is larger than the server's memory budget"));
  if (cudaEventCreateWithFlags(&q->corr_ev, cudaEventDisableTiming) != cudaSuccess)
    return undo(fail(FA_ERR_CUDA, "cudaEventCreate failed"));
  if (cudaMallocHost(&q->h_idx, kAdmitMax * sizeof(long long)) != cudaSuccess)
    return undo(fail(FA_ERR_OOM, "cudaMallocHost failed"));
  if (S->cfg.warm_start > 0) {
    const size_t nw = (size_t)S->cfg.warm_start * A->ref->P;
    if ((st = dalloc_t(S->ctx, nw, &q->warm, q->allocs)) != FA_OK) return undo(st);
    if ((st = dalloc_t(S->ctx, (size_t)S->cfg.warm_start, &q->warm_seq, q->allocs)) != FA_OK) return undo(st);
    if (cudaMemset(q->warm, 0, nw * sizeof(double)) != cudaSuccess ||
        cudaMemset(q->warm_seq, 0xff, (size_t)S->cfg.warm_start * sizeof(long long)) != cudaSuccess)  // -1: empty
      return undo(fail(FA_ERR_CUDA, "cudaMemset failed"));
  }
  std::unique_lock<std::mutex> lk(S->mu);
  if (S->fatal != FA_OK) {
    const std::string msg = S->fatal_msg;
    lk.unlock();  // no CUDA call under the mutex: stream callbacks take it
    return undo(fail(FA_ERR_STATE, "server stopped after an error: " + msg));
  }
  q->id = (int)S->acqs.size();
  *acquisition = q->id;
  S->acqs.push_back(std::move(q));
  S->cv_work.notify_one();
  return FA_OK;
}

extern "C" fa_status fa_server_reserve(fa_server* S, int acquisition, int n_slots) {
  if (!S) return fail(FA_ERR_BAD_ARG, "NULL server");
  if (n_slots < 0 || n_slots > S->cfg.max_in_flight)
    return fail(FA_ERR_BAD_ARG, "n_slots must be in 0..max_in_flight");
  SrvReserve r;
  r.acq = acquisition;
  r.n = n_slots;
  std::unique_lock<std::mutex> lk(S->mu);
  if (acquisition < 0 || acquisition >= (int)S->acqs.size()) return fail(FA_ERR_NOT_FOUND, "unknown acquisition");
  if (S->fatal != FA_OK) return fail(S->fatal, "server stopped after an error: " + S->fatal_msg);
  if (S->stop) return fail(FA_ERR_STATE, "server is shutting down");
  S->reserves.push_back(&r);
  S->cv_work.notify_one();
  S->cv_done.wait(lk, [&] { return r.done || S->fatal != FA_OK; });
  if (!r.done) {  // the worker stopped: withdraw the request
    for (auto it = S->reserves.begin(); it != S->reserves.end(); ++it)
      if (*it == &r) {
        S->reserves.erase(it);
        break;
      }
    return fail(S->fatal, "server stopped after an error: " + S->fatal_msg);
  }
  if (r.status != FA_OK) return fail(r.status, r.error);
  return FA_OK;
}

extern "C" fa_status fa_server_acquisition_info(fa_server* S, int acquisition, int* nD, int* n_dim) {
  if (!S) return fail(FA_ERR_BAD_ARG, "NULL server");
  std::lock_guard<std::mutex> lk(S->mu);
  if (acquisition < 0 || acquisition >= (int)S->acqs.size()) return fail(FA_ERR_NOT_FOUND, "unknown acquisition");
  const fa_reference* R = S->acqs[acquisition]->A->ref;
  if (nD) *nD = R->nD;
  if (n_dim) *n_dim = R->n_dim;
  return FA_OK;
}

extern "C" fa_status fa_server_submit(fa_server* S, int acquisition, const void* frame, int frame_on_device,
                                      unsigned long long* ticket) {
  if (!S || !frame || !ticket) return fail(FA_ERR_BAD_ARG, "NULL argument");
  const double t = now_s();
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->fatal != FA_OK) return fail(S->fatal, "server stopped after an error: " + S->fatal_msg);
  if (S->stop) return fail(FA_ERR_STATE, "server is shutting down");
  if (acquisition < 0 || acquisition >= (int)S->acqs.size()) return fail(FA_ERR_NOT_FOUND, "unknown acquisition");
  SrvRequest r;
  r.ticket = S->next_ticket++;
  r.acq = acquisition;
  r.data = frame;
  r.on_device = frame_on_device != 0;
  r.t_submit = t;
  if (S->t_first_submit < 0) S->t_first_submit = t;
  S->submitted++;
  S->outstanding.insert(r.ticket);
  S->inbox.push_back(r);
  S->cv_work.notify_one();
  *ticket = r.ticket;
  return FA_OK;
}

extern "C" fa_status fa_server_wait(fa_server* S, unsigned long long ticket, double timeout_s, double* D_out,
                                    fa_align_stats* stats, double* latency_ms) {
  if (!S) return fail(FA_ERR_BAD_ARG, "NULL server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto ready = [&] { return S->results.count(ticket) != 0 || !S->outstanding.count(ticket); };
  if (timeout_s < 0)
    S->cv_done.wait(lk, ready);
  else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
    return fail(FA_ERR_TIMEOUT, "result not ready");
  auto it = S->results.find(ticket);
  if (it == S->results.end()) return fail(FA_ERR_NOT_FOUND, "unknown or already collected ticket");
  SrvResult r = std::move(it->second);
  S->results.erase(it);
  lk.unlock();
  if (r.status != FA_OK) return fail(r.status, r.error);
  if (D_out) std::memcpy(D_out, r.D.data(), r.D.size() * sizeof(double));
  if (stats) *stats = r.stats;
  if (latency_ms) *latency_ms = r.latency_ms;
  return FA_OK;
}

extern "C" fa_status fa_server_get_stats(fa_server* S, fa_server_stats* out) {
  if (!S || !out) return fail(FA_ERR_BAD_ARG, "NULL argument");
  std::vector<double> lat;
  fa_server_stats r{};
  {
    std::lock_guard<std::mutex> lk(S->mu);
    lat = S->latencies_ms;
    r.submitted = S->submitted;
    r.completed = S->completed;
    r.failed = S->failed;
    r.peak_in_flight = S->peak_in_flight;
    r.peak_slot_bytes = S->peak_slot_bytes;
    if (S->completed > 0 && S->t_last_done > S->t_first_submit)
      r.frames_per_s = S->completed / (S->t_last_done - S->t_first_submit);
  }
  r.in_flight = S->in_flight.load();
  r.slot_bytes = S->slot_bytes.load();
  r.graph_launches = S->graph_launches.load();
  if (!lat.empty()) {
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double p) {  // nearest rank
      size_t k = (size_t)std::ceil(p / 100.0 * lat.size());
      return lat[std::min(lat.size(), std::max<size_t>(k, 1)) - 1];
    };
    double sum = 0;
    for (double v : lat) sum += v;
    r.p50_ms = pct(50);
    r.p99_ms = pct(99);
    r.mean_ms = sum / lat.size();
    r.max_ms = lat.back();
  }
  *out = r;
  return FA_OK;
}

extern "C" fa_status fa_server_reset_stats(fa_server* S) {
  if (!S) return fail(FA_ERR_BAD_ARG, "NULL server");
  std::lock_guard<std::mutex> lk(S->mu);
  S->latencies_ms.clear();
  S->t_first_submit = -1;
  S->t_last_done = -1;
  S->submitted = S->completed = S->failed = 0;
  S->peak_in_flight = 0;
  S->peak_slot_bytes = 0;
  S->graph_launches = 0;
  return FA_OK;
}
