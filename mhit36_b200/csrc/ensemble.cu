// Served ensemble: many independent MHIT36 simulations on one GPU.
//
// Requests (grid size, parameters, initial fields, step count) are queued
// and admitted as slots and HBM free up (continuous batching).  Simulations
// of the same class -- grid size, precision form, phase field, k^2 and grid
// conventions -- advance together: one CUDA graph per class holds the
// batched kernels of one step for all of the class's slots, and each kernel
// reads its per-slot arguments from a device slot table, so admitting or
// retiring a request only rewrites that table (no re-capture).  Classes run on
// their own streams, so their work overlaps on the device.  Each slot runs
// exactly the arithmetic of a single simulation (own control block, own
// deterministic reductions), so a result does not depend on the mix.
//
// Host side.  The scheduling round (mhit_ens_progress) never waits on the
// device: it polls events, keeps a few milliseconds of rounds queued on every
// busy class, and hands every host<->device transfer of request fields to
// transfer threads (two for uploads, four for downloads).  Each moves fields
// through two pinned staging chunks (double-buffered, with the FP32 rounding
// done while staging) on its own stream, so transfers overlap the rounds of
// every class.
// Slot-table entries are written by one-thread kernels that take the entry
// by value, in stream order with the class's rounds.
//
// The stencil kernels' tile shape of a class comes from an online autotuner:
// the first rounds of a class time the candidates on live data with CUDA
// events (polled, not waited on), then the class graph is re-captured once
// with the fastest.
//
// There is no counterpart in the reference, which runs one simulation per job.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"
#include "mhit.h"

using mhit::Ctrl;
using mhit::SlotArgs;
using mhit::StepConst;

namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

enum { RQ_QUEUED = 0, RQ_RUNNING = 1, RQ_DONE = 2, RQ_FAILED = 3, RQ_CANCELLED = 4 };
// progress of a request's job on a transfer thread
enum { IO_NONE = 0, IO_QUEUED = 1, IO_DONE = 2, IO_FAILED = 3 };

struct Request {
  int64_t id = 0;
  int n = 0, pf = 0, precision = 0, nsteps = 0, keep = 1, borrow = 0;
  mhit_params prm;
  std::vector<double> in[4];          // owned copies of the inputs (not borrowed), dropped after upload
  const double* src[4] = {nullptr, nullptr, nullptr, nullptr};  // what the upload reads
  std::vector<double> out[4];         // final fields when keep = 1
  Ctrl fin;                           // final control block (downloaded)
  int state = RQ_QUEUED;
  int cls = -1, slot = -1;
  int steps_issued = 0;
  int status = MHIT_OK;
  double t_submit = 0, t_admit = 0, t_done = 0;
  mhit_diag diag;
  bool loading = false;               // admitted, upload not yet complete
  bool finishing = false;             // retirement enqueued, download pending
  cudaEvent_t done_ev = nullptr;      // class stream: after the retirement kernels
  std::atomic<int> up{IO_NONE}, down{IO_NONE};
  std::string io_error;
};

// Device buffers of one slot (either precision; unused pointers stay null).
struct SlotBuf {
  bool allocated = false;
  size_t bytes = 0;
  std::vector<void*> ptrs;
  void* f[16] = {nullptr};  // u v w us vs ws ru rv rw phi0 phi1 p/p0 dp spec partials fsin|fcos
  double* fsin = nullptr;
  double* fcos = nullptr;
  Ctrl* ctrl = nullptr;      // into the class's contiguous ctrl array
  int64_t req = -1;          // request holding the slot (loading, running or finishing), or -1
};

struct Class {
  int n = 0, pf = 0, precision = 0, k2_mode = 0, grid_mode = 0;
  int nslots = 0;
  int kz = 32, mty = 16;
  cudaStream_t st = nullptr;
  void* d_slots = nullptr;   // SlotArgs<T>[nslots]
  Ctrl* d_ctrl = nullptr;    // [nslots]
  void* tw = nullptr;        // twiddles (double2 or float2)
  double* k2tab = nullptr;
  std::vector<SlotBuf> slots;
  std::vector<SlotArgs<double>> hd;  // host copies of the slot tables
  std::vector<SlotArgs<float>> hf;
  std::vector<int64_t> running;      // requests whose steps are still being issued
  cudaGraphExec_t graph = nullptr;
  // autotuner: candidate (kz, mty) tile shapes, timed one trial round at a time
  std::vector<std::pair<int, int>> cand;
  std::vector<double> cand_ms;
  std::vector<int> cand_runs;
  int tune_idx = 0;
  bool tuned = false, trial_pending = false;
  double round_ms = 0;               // the chosen shape's round time
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::deque<cudaEvent_t> inflight;  // one event per queued round
  long long rounds = 0;
};

// ---------------------------------------------------------------- transfer threads
// Move request fields between pageable host memory and slot buffers through
// two pinned staging chunks on a stream of their own.  Jobs are queued by
// the scheduling round; completion is reported through the request's atomics.
struct Job {
  int kind;  // 0 upload, 1 download
  Request* r;
  Class* c;
  SlotBuf* b;
};

class Transfer {
 public:
  static constexpr size_t kChunk = (size_t)32 << 20;  // bytes per staging chunk
  static constexpr size_t kSmall = (size_t)64 << 10;  // tables and control block

  cudaError_t start(int device) {
    device_ = device;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking))) return e;
    for (int k = 0; k < 2; ++k) {
      if ((e = cudaMallocHost(&stage_[k], kChunk))) return e;
      // blocking-sync events: a transfer thread waiting for a copy sleeps
      // instead of spinning on a core the other transfer threads and the
      // scheduling thread need
      if ((e = cudaEventCreateWithFlags(&sev_[k], cudaEventDisableTiming | cudaEventBlockingSync))) return e;
      if ((e = cudaEventRecord(sev_[k], st_))) return e;
    }
    if ((e = cudaMallocHost(&small_, kSmall))) return e;
    if ((e = cudaEventCreateWithFlags(&jev_, cudaEventDisableTiming | cudaEventBlockingSync))) return e;
    th_ = std::thread([this] { loop(); });
    return cudaSuccess;
  }

  void push(const Job& j) {
    {
      std::lock_guard<std::mutex> g(mu_);
      q_.push_back(j);
    }
    cv_.notify_one();
  }

  // Finishes the queued jobs, then releases the thread, stream and buffers.
  void stop() {
    if (th_.joinable()) {
      {
        std::lock_guard<std::mutex> g(mu_);
        stop_ = true;
      }
      cv_.notify_one();
      th_.join();
    }
    for (int k = 0; k < 2; ++k) {
      if (sev_[k]) cudaEventDestroy(sev_[k]);
      if (k == 0 && jev_) cudaEventDestroy(jev_);
      if (stage_[k]) cudaFreeHost(stage_[k]);
      sev_[k] = nullptr;
      if (k == 0) jev_ = nullptr;
      stage_[k] = nullptr;
    }
    if (small_) cudaFreeHost(small_);
    small_ = nullptr;
    if (st_) cudaStreamDestroy(st_);
    st_ = nullptr;
  }

 private:
  void loop() {
    cudaSetDevice(device_);
    for (;;) {
      Job j;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [this] { return stop_ || !q_.empty(); });
        if (q_.empty()) return;  // stop requested and nothing left
        j = q_.front();
        q_.pop_front();
      }
      std::string err;
      const cudaError_t e = (j.kind == 0) ? upload(j, &err) : download(j, &err);
      if (e != cudaSuccess) {
        j.r->io_error = err + ": " + cudaGetErrorString(e);
        cudaGetLastError();
      }
      (j.kind == 0 ? j.r->up : j.r->down).store(e == cudaSuccess ? IO_DONE : IO_FAILED);
      if (notify_) notify_();
    }
  }

 public:
  // called after every finished job (wakes mhit_ens_wait)
  std::function<void()> notify_;

  // wait for every copy issued on the transfer stream so far (sleeping)
  cudaError_t sync() {
    cudaError_t e = cudaEventRecord(jev_, st_);
    return e ? e : cudaEventSynchronize(jev_);
  }

 private:

  // host float64 -> device field of `el` bytes per value, chunk by chunk
  cudaError_t put(void* dst, const double* src, size_t count, size_t el) {
    const size_t per = kChunk / sizeof(double);
    cudaError_t e;
    for (size_t done = 0; done < count;) {
      const size_t cnt = std::min(per, count - done);
      if ((e = cudaEventSynchronize(sev_[k_]))) return e;  // the chunk's previous copy has finished
      if (el == sizeof(double)) {
        memcpy(stage_[k_], src + done, cnt * sizeof(double));
      } else {
        float* s = static_cast<float*>(stage_[k_]);
        for (size_t q = 0; q < cnt; ++q) s[q] = (float)src[done + q];
      }
      if ((e = cudaMemcpyAsync(static_cast<char*>(dst) + done * el, stage_[k_], cnt * el, cudaMemcpyHostToDevice,
                               st_)))
        return e;
      if ((e = cudaEventRecord(sev_[k_], st_))) return e;
      k_ ^= 1;
      done += cnt;
    }
    return cudaSuccess;
  }

  // device field of `el` bytes per value -> host float64, chunk by chunk: the
  // copy of chunk i+1 is in flight while chunk i is unpacked
  cudaError_t get(double* dst, const void* src, size_t count, size_t el) {
    const size_t per = kChunk / sizeof(double);
    cudaError_t e;
    size_t prev_off = 0, prev_cnt = 0;
    int prev_k = -1;
    auto drain = [&](int k, size_t off, size_t cnt) -> cudaError_t {
      cudaError_t q = cudaEventSynchronize(sev_[k]);
      if (q) return q;
      if (el == sizeof(double)) {
        memcpy(dst + off, stage_[k], cnt * sizeof(double));
      } else {
        const float* s = static_cast<const float*>(stage_[k]);
        for (size_t i = 0; i < cnt; ++i) dst[off + i] = (double)s[i];
      }
      return cudaSuccess;
    };
    for (size_t done = 0; done < count;) {
      const size_t cnt = std::min(per, count - done);
      if ((e = cudaEventSynchronize(sev_[k_]))) return e;
      if ((e = cudaMemcpyAsync(stage_[k_], static_cast<const char*>(src) + done * el, cnt * el,
                               cudaMemcpyDeviceToHost, st_)))
        return e;
      if ((e = cudaEventRecord(sev_[k_], st_))) return e;
      if (prev_k >= 0 && (e = drain(prev_k, prev_off, prev_cnt))) return e;
      prev_k = k_;
      prev_off = done;
      prev_cnt = cnt;
      k_ ^= 1;
      done += cnt;
    }
    if (prev_k >= 0 && (e = drain(prev_k, prev_off, prev_cnt))) return e;
    return cudaSuccess;
  }

  cudaError_t upload(const Job& j, std::string* where);
  cudaError_t download(const Job& j, std::string* where);

  int device_ = 0;
  cudaStream_t st_ = nullptr;
  void* stage_[2] = {nullptr, nullptr};
  cudaEvent_t sev_[2] = {nullptr, nullptr};
  cudaEvent_t jev_ = nullptr;  // end of a job's copies (blocking sync)
  void* small_ = nullptr;
  int k_ = 0;
  std::thread th_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<Job> q_;
  bool stop_ = false;
};

}  // namespace

struct mhit_ensemble {
  int device = 0;
  size_t budget = 0, used = 0;
  int slots_per_class = 8;
  int64_t next_id = 1;
  double t0 = 0;
  std::map<int64_t, std::unique_ptr<Request>> reqs;
  std::deque<int64_t> queue;
  std::vector<std::unique_ptr<Class>> classes;
  std::vector<cudaEvent_t> free_events;
  // Transfer threads: kUp for uploads, then kDown for downloads (a download
  // ends in page-faulting copies into fresh host vectors, the slower side).
  // Jobs go round-robin, so neither direction waits behind the other.
  static constexpr int kUp = 2, kDown = 4;
  Transfer xfer[kUp + kDown];
  unsigned next_up = 0, next_down = 0;
  bool xfer_started = false;
  std::string last_error;
  long long rounds = 0, launches = 0;
  // mhit_ens_wait sleeps on this until a transfer thread finishes a job (or
  // a short interval passes, after which it looks at the class streams)
  std::mutex wait_mu;
  std::condition_variable wait_cv;
  unsigned long long io_done = 0;
};

namespace {

bool built_size(int n) {
  bool ok = false;
#define MHIT_CASE(NN) ok |= (n == NN);
  MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
  return ok && mhit::stencil_size_ok(n);
}

size_t elem(int precision) { return precision == MHIT_FP64 ? sizeof(double) : sizeof(float); }

// Device bytes of one slot of a class.
size_t slot_bytes(int n, int pf, int precision) {
  const size_t N3 = (size_t)n * n * n, e = elem(precision);
  size_t fields = 9 + 1 + (pf ? 2 : 0) + (precision == MHIT_FP64 ? 0 : 1);  // + p / (p0, dp)
  const size_t spec = (size_t)n * n * mhit::spectrum_pitch(n, precision != MHIT_FP64) * 2 * e;
  return fields * N3 * e + spec + (size_t)mhit::partials_capacity(n) * 7 * sizeof(double) + 2 * n * sizeof(double);
}

StepConst make_const(const mhit_params* p, int n) {
  StepConst c;
  memset(&c, 0, sizeof(c));
  const double twopi = 8.0 * atan(1.0);
  const double dx = (p->grid_mode == MHIT_GRID_CONSISTENT) ? twopi / n : twopi / (n - 1);
  c.n = n;
  c.dt = p->dt; c.mu = p->mu; c.rho = p->rho;
  c.rhoi = 1.0 / p->rho;
  c.dxi = 1.0 / dx;
  c.ddxi = 1.0 / dx / dx;
  c.eps = p->epsr * dx;
  c.epsi = 1.0 / c.eps;
  c.enumv = (double)(float)1.e-16;
  c.tiny = (double)(float)1.0E-16;
  c.sigma = p->sigma;
  c.lin_force = p->lin_force;
  c.f1 = p->f1; c.f2 = p->f2; c.f3 = p->f3;
  c.abc = (p->f1 != 0.0 || p->f2 != 0.0 || p->f3 != 0.0) ? 1 : 0;
  c.tanh_identity = p->tanh_identity ? 1 : 0;
  c.phi_floor = p->phi_floor ? 1 : 0;
  c.cdiv = p->rho * c.dxi / p->dt;
  c.dtr = p->dt / p->rho;
  return c;
}

int fail(mhit_ensemble* e, cudaError_t err, const char* where) {
  e->last_error = std::string(where) + ": " + cudaGetErrorString(err);
  return err == cudaErrorMemoryAllocation ? MHIT_ERR_NOMEM : MHIT_ERR_CUDA;
}

#define ECK(e, call)                                        \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return fail(e, e_, #call);       \
  } while (0)

// Slot-table writes in stream order: the entry travels as a kernel argument,
// so no host buffer has to outlive the call.  The entry holds the slot's
// tensor maps, so the writes are released to the tensor-map proxy.
template <class T>
__global__ void slot_write_kernel(SlotArgs<T>* __restrict__ dst, const __grid_constant__ SlotArgs<T> val) {
  const int* s = reinterpret_cast<const int*>(&val);
  int* d = reinterpret_cast<int*>(dst);
  for (int q = threadIdx.x; q < (int)(sizeof(SlotArgs<T>) / sizeof(int)); q += blockDim.x) d[q] = s[q];
  mhit::tensormap_release();
}

template <class T>
__global__ void slot_active_kernel(SlotArgs<T>* __restrict__ dst, int active) {
  dst->active = active;
}

// dst = phi[nstep & 1]: the phi of the slot's last completed step, chosen on
// the device (a request that stopped early on an error has an odd or even
// step count the host does not know).
template <class T>
__global__ void select_phi_kernel(T* __restrict__ dst, const T* __restrict__ a, const T* __restrict__ b,
                                  const Ctrl* __restrict__ ctrl, size_t count) {
  const T* src = (ctrl->nstep & 1) ? b : a;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < count; g += (size_t)gridDim.x * blockDim.x)
    dst[g] = src[g];
}

cudaError_t get_event(mhit_ensemble* e, cudaEvent_t* ev) {
  if (!e->free_events.empty()) {
    *ev = e->free_events.back();
    e->free_events.pop_back();
    return cudaSuccess;
  }
  return cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
}

void put_event(mhit_ensemble* e, cudaEvent_t ev) {
  if (ev) e->free_events.push_back(ev);
}

void free_slot_buffers(mhit_ensemble* e, SlotBuf& b) {
  for (void* q : b.ptrs) cudaFree(q);
  b.ptrs.clear();
  for (auto& f : b.f) f = nullptr;
  b.fsin = b.fcos = nullptr;
  e->used -= b.bytes;
  b.bytes = 0;
  b.allocated = false;
}

cudaError_t alloc_slot_buffers(mhit_ensemble* e, Class* c, SlotBuf& b) {
  const int n = c->n;
  const size_t N3 = (size_t)n * n * n, el = elem(c->precision);
  auto get = [&](size_t bytes, void** out) {
    cudaError_t r = cudaMalloc(out, bytes);
    if (r == cudaSuccess) {
      b.ptrs.push_back(*out);
      b.bytes += bytes;
      e->used += bytes;
    }
    return r;
  };
  cudaError_t r;
  const int nf = 9 + 1 + (c->precision == MHIT_FP64 ? 0 : 1);  // + p (or p0, dp)
  for (int q = 0; q < 9; ++q)
    if ((r = get(N3 * el, &b.f[q]))) return r;
  if (c->pf) {
    if ((r = get(N3 * el, &b.f[9])) || (r = get(N3 * el, &b.f[10]))) return r;
  }
  for (int q = 9; q < nf; ++q)
    if ((r = get(N3 * el, &b.f[11 + (q - 9)]))) return r;
  const size_t spec = (size_t)n * n * mhit::spectrum_pitch(n, c->precision != MHIT_FP64) * 2 * el;
  if ((r = get(spec, &b.f[13]))) return r;
  if ((r = cudaMemsetAsync(b.f[13], 0, spec, c->st))) return r;
  if ((r = get((size_t)mhit::partials_capacity(n) * 7 * sizeof(double), &b.f[14]))) return r;
  void* t = nullptr;
  if ((r = get(2 * n * sizeof(double), &t))) return r;
  b.fsin = static_cast<double*>(t);
  b.fcos = b.fsin + n;
  b.allocated = true;
  return cudaSuccess;
}

template <class T> SlotArgs<T> build_args(Class* c, SlotBuf& b, const StepConst& k, int active) {
  SlotArgs<T> a;
  memset((void*)&a, 0, sizeof(a));
  T* f[16];
  for (int q = 0; q < 16; ++q) f[q] = static_cast<T*>(b.f[q]);
  a.st.u = f[0]; a.st.v = f[1]; a.st.w = f[2];
  a.st.us = f[3]; a.st.vs = f[4]; a.st.ws = f[5];
  a.st.ru = f[6]; a.st.rv = f[7]; a.st.rw = f[8];
  a.st.p = f[11];
  a.st.uo = f[0]; a.st.vo = f[1]; a.st.wo = f[2];
  a.st.partials = static_cast<double*>(b.f[14]);
  a.st.fsin = b.fsin;
  a.st.fcos = b.fcos;
  a.st.ctrl = b.ctrl;
  a.st.c = k;
  typedef typename mhit::C2<T>::t CT;
  a.po.us = f[3]; a.po.vs = f[4]; a.po.ws = f[5];
  a.po.spec = static_cast<CT*>(b.f[13]);
  a.po.p = f[11];
  a.po.tw = static_cast<const CT*>(c->tw);
  a.po.k2tab = c->k2tab;
  a.po.ctrl = b.ctrl;
  a.po.cdiv = k.cdiv;
  a.po.ddxi = k.ddxi;
  a.pr = a.po;
  a.pr.pres = f[11];
  a.pr.p = f[12];
  a.phi[0] = f[9];
  a.phi[1] = f[10];
  a.dp = static_cast<float*>(b.f[12]);
  a.active = active;
  return a;
}

// Write slot s's table entry (the request's buffers, constants and tensor
// maps) on the class stream.
cudaError_t write_entry(Class* c, int s, const StepConst& k, int active) {
  cudaError_t e;
  if (c->precision == MHIT_FP64) {
    c->hd[s] = build_args<double>(c, c->slots[s], k, active);
    if ((e = mhit::encode_slot_maps<double>(&c->hd[s], c->n, c->pf != 0))) return e;
    slot_write_kernel<double><<<1, 64, 0, c->st>>>(static_cast<SlotArgs<double>*>(c->d_slots) + s, c->hd[s]);
  } else {
    c->hf[s] = build_args<float>(c, c->slots[s], k, active);
    if ((e = mhit::encode_slot_maps<float>(&c->hf[s], c->n, c->pf != 0))) return e;
    slot_write_kernel<float><<<1, 64, 0, c->st>>>(static_cast<SlotArgs<float>*>(c->d_slots) + s, c->hf[s]);
  }
  return cudaGetLastError();
}

cudaError_t set_active(Class* c, int s, int active) {
  if (c->precision == MHIT_FP64) {
    c->hd[s].active = active;
    slot_active_kernel<double><<<1, 1, 0, c->st>>>(static_cast<SlotArgs<double>*>(c->d_slots) + s, active);
  } else {
    c->hf[s].active = active;
    slot_active_kernel<float><<<1, 1, 0, c->st>>>(static_cast<SlotArgs<float>*>(c->d_slots) + s, active);
  }
  return cudaGetLastError();
}

// Enqueue one batched step of every slot of class c (inactive slots return at once).
cudaError_t enqueue_class_step(Class* c, int kz, int mty) {
  const int n = c->n, S = c->nslots;
  cudaError_t err;
  if (c->precision == MHIT_FP64) {
    const SlotArgs<double>* t = static_cast<const SlotArgs<double>*>(c->d_slots);
    if (c->pf && (err = mhit::launch_phase_batched<double>(t, S, n, kz, c->st))) return err;
    if ((err = mhit::launch_momentum_batched<double>(t, S, n, kz, c->pf != 0, c->st, mty))) return err;
    const bool fused = mhit::fused_projection(n) != 0;  // x inverse fused into the projection
    for (int k = 0; k < (fused ? 4 : 5); ++k)
      if ((err = mhit::launch_poisson_stage_batched<double>(t, S, n, k, 0, c->st))) return err;
    if (fused) {
      if ((err = mhit::launch_xinv_project_batched<double>(t, S, n, c->st))) return err;
    } else if ((err = mhit::launch_project_batched<double>(t, S, n, c->st))) {
      return err;
    }
    return mhit::launch_finalize_batched(t, S, n, c->st);
  }
  const SlotArgs<float>* t = static_cast<const SlotArgs<float>*>(c->d_slots);
  if (c->pf && (err = mhit::launch_phase_batched<float>(t, S, n, kz, c->st))) return err;
  if ((err = mhit::launch_momentum_batched<float>(t, S, n, kz, c->pf != 0, c->st, mty))) return err;
  // first solve -> p0; correction solve of the FP64 residual, whose x inverse
  // is fused into the projection where the size allows
  const bool fused = mhit::fused_projection(n) != 0;
  for (int w = 0; w < 2; ++w)
    for (int k = 0; k < ((w && fused) ? 4 : 5); ++k)
      if ((err = mhit::launch_poisson_stage_batched<float>(t, S, n, k, w, c->st))) return err;
  if (fused) {
    if ((err = mhit::launch_xinv_project_batched<float>(t, S, n, c->st))) return err;
  } else if ((err = mhit::launch_project_batched<float>(t, S, n, c->st))) {
    return err;
  }
  return mhit::launch_finalize_batched_f32(t, S, n, c->st);
}

cudaError_t capture_class(Class* c, int kz, int mty) {
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  cudaGraph_t g = nullptr;
  cudaError_t err = cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal);
  if (err) return err;
  cudaError_t e2 = enqueue_class_step(c, kz, mty);
  err = cudaStreamEndCapture(c->st, &g);
  if (e2) {
    if (g) cudaGraphDestroy(g);
    return e2;
  }
  if (err) return err;
  err = cudaGraphInstantiate(&c->graph, g, 0);
  cudaGraphDestroy(g);
  return err;
}

int class_for(mhit_ensemble* e, const Request* r) {
  for (size_t i = 0; i < e->classes.size(); ++i) {
    Class* c = e->classes[i].get();
    if (c->n == r->n && c->pf == r->pf && c->precision == r->precision && c->k2_mode == r->prm.k2_mode &&
        c->grid_mode == r->prm.grid_mode)
      return (int)i;
  }
  return -1;
}

// Create a class (stream, tables, empty slot table, graph).
int make_class(mhit_ensemble* e, const Request* r, int* out) {
  std::unique_ptr<Class> c(new Class());
  c->n = r->n; c->pf = r->pf; c->precision = r->precision;
  c->k2_mode = r->prm.k2_mode; c->grid_mode = r->prm.grid_mode;
  const int n = c->n;
  // slots: as many as the grid dimension limit allows, capped by the setting
  c->nslots = std::max(1, std::min(e->slots_per_class, 65535 / n));
  ECK(e, mhit::prepare_stencils());
  ECK(e, mhit::prepare_poisson(n));
  ECK(e, cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  ECK(e, cudaEventCreate(&c->ev0));
  ECK(e, cudaEventCreate(&c->ev1));
  const size_t tsz = (c->precision == MHIT_FP64) ? sizeof(SlotArgs<double>) : sizeof(SlotArgs<float>);
  ECK(e, cudaMalloc(&c->d_slots, tsz * c->nslots));
  ECK(e, cudaMalloc(&c->d_ctrl, sizeof(Ctrl) * c->nslots));
  // tables (same values as mhit_create builds)
  const double twopi = 8.0 * atan(1.0), lx = twopi;
  const double dx = (c->grid_mode == MHIT_GRID_CONSISTENT) ? lx / n : lx / (n - 1);
  const double ddxi = 1.0 / dx / dx, pi = 4.0 * atan(1.0);
  std::vector<double> k2(n);
  std::vector<double2> twd(n);
  std::vector<float2> twf(n);
  for (int m = 0; m < n; ++m) {
    long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)n;
    twd[m].x = (double)cosl(a); twd[m].y = -(double)sinl(a);
    twf[m].x = (float)cosl(a); twf[m].y = -(float)sinl(a);
    if (c->k2_mode == MHIT_K2_FD) {
      const double s = sin(pi * m / n);
      k2[m] = (4.0 * ddxi) * (s * s);
    } else {
      const double kk = (m < n / 2 ? (double)m : (double)(m - n)) * (twopi / lx);
      k2[m] = kk * kk;
    }
  }
  ECK(e, cudaMalloc(&c->k2tab, n * sizeof(double)));
  ECK(e, cudaMemcpy(c->k2tab, k2.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  if (c->precision == MHIT_FP64) {
    ECK(e, cudaMalloc(&c->tw, n * sizeof(double2)));
    ECK(e, cudaMemcpy(c->tw, twd.data(), n * sizeof(double2), cudaMemcpyHostToDevice));
    c->hd.assign(c->nslots, SlotArgs<double>());
    memset((void*)c->hd.data(), 0, sizeof(SlotArgs<double>) * c->nslots);
    ECK(e, cudaMemcpy(c->d_slots, c->hd.data(), tsz * c->nslots, cudaMemcpyHostToDevice));
  } else {
    ECK(e, cudaMalloc(&c->tw, n * sizeof(float2)));
    ECK(e, cudaMemcpy(c->tw, twf.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    c->hf.assign(c->nslots, SlotArgs<float>());
    memset((void*)c->hf.data(), 0, sizeof(SlotArgs<float>) * c->nslots);
    ECK(e, cudaMemcpy(c->d_slots, c->hf.data(), tsz * c->nslots, cudaMemcpyHostToDevice));
  }
  c->slots.assign(c->nslots, SlotBuf());
  for (int s = 0; s < c->nslots; ++s) c->slots[s].ctrl = c->d_ctrl + s;
  // autotuner candidates for the stencil kernels' z chunk
  for (int kz : {8, 16, 32})
    for (int mty : {8, 16})
      if (mhit::stencil_kz_ok(n, kz)) c->cand.push_back(std::make_pair(kz, mty));
  c->cand_ms.assign(c->cand.size(), 0.0);
  c->cand_runs.assign(c->cand.size(), 0);
  c->kz = c->cand.empty() ? 32 : c->cand[0].first;
  c->mty = c->cand.empty() ? 16 : c->cand[0].second;
  ECK(e, capture_class(c.get(), c->kz, c->mty));
  e->classes.push_back(std::move(c));
  *out = (int)e->classes.size() - 1;
  return MHIT_OK;
}

}  // namespace

// ---------------------------------------------------------------- transfer jobs
#define TCK(call)      \
  if ((e = (call))) {  \
    *where = #call;    \
    return e;          \
  }

// Initial state of an admitted request into its (inactive) slot: u, v, w,
// phi, zeroed rhs_o and pressure, the ABC forcing tables and the control
// block (gumax = 1, Euler first step: multi/main.f90:323-325).
cudaError_t Transfer::upload(const Job& j, std::string* where) {
  Request* r = j.r;
  Class* c = j.c;
  SlotBuf& b = *j.b;
  const int n = c->n;
  const size_t N3 = (size_t)n * n * n, el = elem(c->precision);
  cudaError_t e;
  TCK(put(b.f[0], r->src[0], N3, el));
  TCK(put(b.f[1], r->src[1], N3, el));
  TCK(put(b.f[2], r->src[2], N3, el));
  if (c->pf) TCK(put(b.f[9], r->src[3], N3, el));
  for (int f = 6; f < 9; ++f) TCK(cudaMemsetAsync(b.f[f], 0, N3 * el, st_));
  TCK(cudaMemsetAsync(b.f[11], 0, N3 * el, st_));
  if (c->precision != MHIT_FP64) TCK(cudaMemsetAsync(b.f[12], 0, N3 * sizeof(float), st_));
  // ABC forcing tables of this request (multi/main.f90:150-153, 591-593)
  double* tab = static_cast<double*>(small_);
  const double twopi = 8.0 * atan(1.0);
  const double dx = (r->prm.grid_mode == MHIT_GRID_CONSISTENT) ? twopi / n : twopi / (n - 1);
  double x = 0.0;
  for (int m = 0; m < n; ++m) {
    if (m) x += dx;  // x(i+1) = x(i) + dx, as the reference accumulates it
    tab[m] = sin(r->prm.k0 * x);
    tab[n + m] = cos(r->prm.k0 * x);
  }
  TCK(cudaMemcpyAsync(b.fsin, tab, 2 * n * sizeof(double), cudaMemcpyHostToDevice, st_));
  Ctrl* ctl = reinterpret_cast<Ctrl*>(static_cast<char*>(small_) + kSmall / 2);
  memset(ctl, 0, sizeof(Ctrl));
  ctl->gumax = 1.0;
  ctl->alpha = 1.0;
  ctl->beta = 0.0;
  ctl->cfl_limit = r->prm.cfl_limit > 0 ? r->prm.cfl_limit : 7.0;
  TCK(cudaMemcpyAsync(b.ctrl, ctl, sizeof(Ctrl), cudaMemcpyHostToDevice, st_));
  TCK(sync());  // the small area and the caller's input are free again
  return cudaSuccess;
}

// Final control block, and the fields when the request keeps them (phi was
// staged into the spectrum buffer by the retirement kernels).
cudaError_t Transfer::download(const Job& j, std::string* where) {
  Request* r = j.r;
  Class* c = j.c;
  SlotBuf& b = *j.b;
  const size_t N3 = (size_t)c->n * c->n * c->n, el = elem(c->precision);
  cudaError_t e;
  Ctrl* ctl = reinterpret_cast<Ctrl*>(small_);
  TCK(cudaMemcpyAsync(ctl, b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st_));
  TCK(sync());
  r->fin = *ctl;
  if (r->keep) {
    const void* src[4] = {b.f[0], b.f[1], b.f[2], b.f[13]};
    const int nf = c->pf ? 4 : 3;
    for (int f = 0; f < nf; ++f) {
      r->out[f].resize(N3);
      TCK(get(r->out[f].data(), src[f], N3, el));
    }
  }
  return cudaSuccess;
}
#undef TCK

namespace {

// Try to start request r: class, slot and buffers, then queue its upload.
// Returns 1 when admitted, 0 when it has to wait (or failed: *err set).
int admit(mhit_ensemble* e, Request* r, int* err) {
  *err = MHIT_OK;
  int ci = class_for(e, r);
  if (ci < 0) {
    int rc = make_class(e, r, &ci);
    if (rc) {
      *err = rc;
      return 0;
    }
  }
  Class* c = e->classes[ci].get();
  int s = -1;
  for (int q = 0; q < c->nslots && s < 0; ++q)
    if (c->slots[q].req == -1 && c->slots[q].allocated) s = q;
  for (int q = 0; q < c->nslots && s < 0; ++q)
    if (c->slots[q].req == -1) s = q;
  if (s < 0) return 0;  // class full
  SlotBuf& b = c->slots[s];
  if (!b.allocated) {
    const size_t need = slot_bytes(c->n, c->pf, c->precision);
    // admission by HBM footprint: reclaim idle pooled slots of other classes
    for (auto& oc : e->classes) {
      if (e->used + need <= e->budget) break;
      if (oc.get() == c) continue;
      for (auto& ob : oc->slots)
        if (ob.allocated && ob.req == -1 && e->used + need > e->budget) {
          cudaStreamSynchronize(oc->st);
          free_slot_buffers(e, ob);
        }
    }
    if (e->used + need > e->budget) return 0;
    cudaError_t a = alloc_slot_buffers(e, c, b);
    if (a) {
      free_slot_buffers(e, b);
      cudaGetLastError();
      return 0;  // device memory tighter than the budget says: wait
    }
  }
  b.req = r->id;
  r->cls = ci;
  r->slot = s;
  r->state = RQ_RUNNING;
  r->loading = true;
  r->t_admit = now_s();
  r->up.store(IO_QUEUED);
  Job j;
  j.kind = 0;
  j.r = r;
  j.c = c;
  j.b = &b;
  e->xfer[e->next_up++ % mhit_ensemble::kUp].push(j);
  return 1;
}

// After the request's last step is enqueued: materialise the mean removal,
// stage phi, take the slot out of the batch and mark the point in the class
// stream after which a transfer thread may read the slot -- all in stream
// order, without waiting.
cudaError_t retire_enqueue(mhit_ensemble* e, Class* c, Request* r) {
  SlotBuf& b = c->slots[r->slot];
  const size_t N3 = (size_t)c->n * c->n * c->n;
  cudaError_t q;
  if (c->precision == MHIT_FP64)
    q = mhit::launch_materialize<double>(static_cast<double*>(b.f[0]), static_cast<double*>(b.f[1]),
                                         static_cast<double*>(b.f[2]), c->n, b.ctrl, c->st);
  else
    q = mhit::launch_materialize<float>(static_cast<float*>(b.f[0]), static_cast<float*>(b.f[1]),
                                        static_cast<float*>(b.f[2]), c->n, b.ctrl, c->st);
  if (q) return q;
  // phi of the last completed step, staged through the (now idle) spectrum buffer
  if (c->pf && r->keep) {
    if (c->precision == MHIT_FP64)
      select_phi_kernel<double><<<1184, 256, 0, c->st>>>(static_cast<double*>(b.f[13]), static_cast<double*>(b.f[9]),
                                                        static_cast<double*>(b.f[10]), b.ctrl, N3);
    else
      select_phi_kernel<float><<<1184, 256, 0, c->st>>>(static_cast<float*>(b.f[13]), static_cast<float*>(b.f[9]),
                                                       static_cast<float*>(b.f[10]), b.ctrl, N3);
    if ((q = cudaGetLastError())) return q;
  }
  if ((q = set_active(c, r->slot, 0))) return q;
  if ((q = get_event(e, &r->done_ev))) return q;
  if ((q = cudaEventRecord(r->done_ev, c->st))) return q;
  r->finishing = true;
  return cudaSuccess;
}

// The download finished: publish the request's final state and free its slot.
void complete(mhit_ensemble* e, Request* r) {
  Class* c = e->classes[r->cls].get();
  put_event(e, r->done_ev);
  r->done_ev = nullptr;
  if (r->down.load() == IO_FAILED) {
    r->state = RQ_FAILED;
    r->status = MHIT_ERR_CUDA;
    e->last_error = r->io_error;
  } else {
    const Ctrl& ctl = r->fin;
    r->diag.umax = ctl.gumax;
    r->diag.cfl = ctl.cfl;
    r->diag.umean = ctl.last_mean[0];
    r->diag.vmean = ctl.last_mean[1];
    r->diag.wmean = ctl.last_mean[2];
    r->diag.gamma = ctl.gumax;
    r->diag.max_div = ctl.max_div;
    r->diag.step = ctl.nstep;
    r->diag.status = ctl.status;
    r->status = ctl.status;
    r->state = ctl.status ? RQ_FAILED : RQ_DONE;
  }
  r->t_done = now_s();
  r->finishing = false;
  c->slots[r->slot].req = -1;  // slot free, buffers pooled
}

// Count one issued round for every running request of the class; a request
// whose last step was just issued is retired behind it.
int account_round(mhit_ensemble* e, Class* c) {
  ++c->rounds;
  ++e->launches;
  for (size_t q = 0; q < c->running.size();) {
    Request* r = e->reqs[c->running[q]].get();
    if (++r->steps_issued >= r->nsteps) {
      ECK(e, retire_enqueue(e, c, r));
      c->running.erase(c->running.begin() + q);
    } else {
      ++q;
    }
  }
  return MHIT_OK;
}

// Rounds of device work kept queued per class: about 4 ms, at least 2.
int queue_depth(const Class* c) {
  const double ms = std::max(c->round_ms, 0.02);
  return std::max(2, std::min(64, (int)ceil(4.0 / ms)));
}

// Block until a transfer thread is done with a job of the request (cancel).
void wait_io(const std::atomic<int>& s) {
  for (int it = 0; s.load() == IO_QUEUED && it < 1200000; ++it) std::this_thread::sleep_for(std::chrono::microseconds(100));
}

// Whether a scheduling round now has something to do: a transfer job of a
// request finished, a retiring request's class stream passed its retirement,
// an autotuner trial finished (or can start), or a busy class has room in its
// queue of rounds.
bool work_ready(mhit_ensemble* e) {
  for (auto& kv : e->reqs) {
    Request* r = kv.second.get();
    if (r->loading && r->up.load() != IO_QUEUED) return true;
    if (r->finishing) {
      const int d = r->down.load();
      if (d == IO_DONE || d == IO_FAILED) return true;
      if (d == IO_NONE && cudaEventQuery(r->done_ev) != cudaErrorNotReady) return true;
    }
  }
  for (auto& cp : e->classes) {
    Class* c = cp.get();
    if (!c->tuned) {
      if (c->trial_pending ? cudaEventQuery(c->ev1) != cudaErrorNotReady : !c->running.empty()) return true;
      continue;
    }
    if (c->running.empty()) continue;
    if ((int)c->inflight.size() < queue_depth(c)) return true;
    if (cudaEventQuery(c->inflight.front()) != cudaErrorNotReady) return true;
  }
  return false;
}

}  // namespace

extern "C" {

int mhit_ens_create(size_t hbm_budget_bytes, int slots_per_class, mhit_ensemble** out) {
  if (!out || slots_per_class < 1) return MHIT_ERR_INVALID;
  std::unique_ptr<mhit_ensemble> e(new mhit_ensemble());
  cudaGetDevice(&e->device);
  size_t freeb = 0, total = 0;
  if (cudaMemGetInfo(&freeb, &total) != cudaSuccess) return MHIT_ERR_CUDA;
  // default budget: 85% of the free memory
  e->budget = hbm_budget_bytes ? hbm_budget_bytes : (size_t)(0.85 * (double)freeb);
  e->slots_per_class = slots_per_class;
  e->t0 = now_s();
  mhit_ensemble* ep = e.get();
  for (auto& x : e->xfer)
    x.notify_ = [ep] {
      {
        std::lock_guard<std::mutex> g(ep->wait_mu);
        ++ep->io_done;
      }
      ep->wait_cv.notify_all();
    };
  bool ok = true;
  for (auto& x : e->xfer) ok = ok && x.start(e->device) == cudaSuccess;
  if (!ok) {
    for (auto& x : e->xfer) x.stop();
    cudaGetLastError();
    return MHIT_ERR_CUDA;
  }
  e->xfer_started = true;
  *out = e.release();
  return MHIT_OK;
}

int mhit_ens_submit(mhit_ensemble* e, const mhit_params* p, int n, int precision, int phase_field, int nsteps,
                    const double* u, const double* v, const double* w, const double* phi, int flags,
                    int64_t* id) {
  if (!e || !p || !u || !v || !w || !id || nsteps < 1) return MHIT_ERR_INVALID;
  if (phase_field && !phi) return MHIT_ERR_INVALID;
  if (!built_size(n)) return MHIT_ERR_UNSUPPORTED;
  if (precision != MHIT_FP64 && precision != MHIT_FP32_REFINE) return MHIT_ERR_UNSUPPORTED;
  if (precision == MHIT_FP32_REFINE && p->k2_mode != MHIT_K2_FD) return MHIT_ERR_UNSUPPORTED;
  if (slot_bytes(n, phase_field, precision) > e->budget) return MHIT_ERR_NOMEM;
  std::unique_ptr<Request> r(new Request());
  r->id = e->next_id++;
  r->n = n;
  r->pf = phase_field ? 1 : 0;
  r->precision = precision;
  r->nsteps = nsteps;
  r->keep = (flags & MHIT_ENS_KEEP_RESULT) ? 1 : 0;
  r->borrow = (flags & MHIT_ENS_BORROW_INPUT) ? 1 : 0;
  r->prm = *p;
  memset(&r->diag, 0, sizeof(r->diag));
  const double* in[4] = {u, v, w, r->pf ? phi : nullptr};
  const size_t N3 = (size_t)n * n * n;
  for (int f = 0; f < 4; ++f) {
    if (!in[f]) continue;
    if (r->borrow) {
      r->src[f] = in[f];
    } else {
      r->in[f].assign(in[f], in[f] + N3);
      r->src[f] = r->in[f].data();
    }
  }
  r->t_submit = now_s();
  *id = r->id;
  e->queue.push_back(r->id);
  e->reqs[r->id] = std::move(r);
  return MHIT_OK;
}

// One scheduling round; never waits on the device:
//   1. retirements: queue the download of a request once the class stream has
//      passed its retirement kernels; publish it once downloaded;
//   2. activations: a slot whose upload finished joins the batch;
//   3. admission, FIFO, of every queued request that fits (class slot + HBM);
//   4. every class with running requests gets rounds queued up to its depth
//      (one timed trial round at a time while its autotuner runs).
// *pending = requests queued or running after the round.
int mhit_ens_progress(mhit_ensemble* e, int* pending) {
  if (!e) return MHIT_ERR_INVALID;
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != e->device) cudaSetDevice(e->device);
  // 1. retirements
  for (auto& kv : e->reqs) {
    Request* r = kv.second.get();
    if (!r->finishing) continue;
    const int d = r->down.load();
    if (d == IO_NONE) {
      const cudaError_t q = cudaEventQuery(r->done_ev);
      if (q == cudaSuccess) {
        Class* c = e->classes[r->cls].get();
        r->down.store(IO_QUEUED);
        Job j;
        j.kind = 1;
        j.r = r;
        j.c = c;
        j.b = &c->slots[r->slot];
        e->xfer[mhit_ensemble::kUp + e->next_down++ % mhit_ensemble::kDown].push(j);
      } else if (q != cudaErrorNotReady) {
        return fail(e, q, "cudaEventQuery(done_ev)");
      }
    } else if (d == IO_DONE || d == IO_FAILED) {
      complete(e, r);
    }
  }
  // 2. activations
  for (auto& cp : e->classes) {
    Class* c = cp.get();
    for (int s = 0; s < c->nslots; ++s) {
      SlotBuf& b = c->slots[s];
      if (b.req < 0) continue;
      Request* r = e->reqs[b.req].get();
      if (!r->loading) continue;
      const int u = r->up.load();
      if (u == IO_QUEUED) continue;
      r->loading = false;
      for (auto& v : r->in) std::vector<double>().swap(v);
      if (u == IO_FAILED) {
        r->state = RQ_FAILED;
        r->status = MHIT_ERR_CUDA;
        r->t_done = now_s();
        e->last_error = r->io_error;
        b.req = -1;
        continue;
      }
      ECK(e, write_entry(c, s, make_const(&r->prm, c->n), 1));
      c->running.push_back(r->id);
    }
  }
  // 3. admission, in arrival order, of everything that fits now
  for (auto it = e->queue.begin(); it != e->queue.end();) {
    Request* r = e->reqs[*it].get();
    int err = MHIT_OK;
    if (admit(e, r, &err)) {
      it = e->queue.erase(it);
    } else if (err) {
      r->state = RQ_FAILED;
      r->status = err;
      r->t_done = now_s();
      it = e->queue.erase(it);
    } else {
      ++it;
    }
  }
  // 4. rounds
  for (auto& cp : e->classes) {
    Class* c = cp.get();
    while (!c->inflight.empty()) {
      const cudaError_t q = cudaEventQuery(c->inflight.front());
      if (q == cudaErrorNotReady) break;
      if (q != cudaSuccess) return fail(e, q, "cudaEventQuery(round)");
      put_event(e, c->inflight.front());
      c->inflight.pop_front();
    }
    if (!c->tuned) {
      const int nc = (int)c->cand.size();
      if (c->trial_pending) {
        const cudaError_t q = cudaEventQuery(c->ev1);
        if (q == cudaErrorNotReady) continue;
        if (q != cudaSuccess) return fail(e, q, "cudaEventQuery(trial)");
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        const int ci = c->tune_idx % nc;
        if (c->tune_idx >= nc) {  // the first pass over the candidates is warm-up
          c->cand_ms[ci] += ms;
          c->cand_runs[ci] += 1;
        }
        ++c->tune_idx;
        c->trial_pending = false;
        if (c->tune_idx >= 3 * nc) {
          int best = 0;
          for (int q2 = 1; q2 < nc; ++q2)
            if (c->cand_ms[q2] / c->cand_runs[q2] < c->cand_ms[best] / c->cand_runs[best]) best = q2;
          c->kz = c->cand[best].first;
          c->mty = c->cand[best].second;
          c->round_ms = c->cand_ms[best] / c->cand_runs[best];
          ECK(e, capture_class(c, c->kz, c->mty));
          c->tuned = true;
        }
      }
      if (!c->tuned) {
        if (c->running.empty()) continue;
        const int ci = c->tune_idx % nc;
        ECK(e, cudaEventRecord(c->ev0, c->st));
        ECK(e, enqueue_class_step(c, c->cand[ci].first, c->cand[ci].second));
        ECK(e, cudaEventRecord(c->ev1, c->st));
        c->trial_pending = true;
        const int rc = account_round(e, c);
        if (rc) return rc;
        continue;
      }
    }
    const int depth = queue_depth(c);
    while (!c->running.empty() && (int)c->inflight.size() < depth) {
      ECK(e, cudaGraphLaunch(c->graph, c->st));
      cudaEvent_t ev = nullptr;
      ECK(e, get_event(e, &ev));
      c->inflight.push_back(ev);
      ECK(e, cudaEventRecord(ev, c->st));
      const int rc = account_round(e, c);
      if (rc) return rc;
    }
  }
  ++e->rounds;
  int pend = 0;
  for (auto& kv : e->reqs)
    if (kv.second->state == RQ_QUEUED || kv.second->state == RQ_RUNNING) ++pend;
  if (pending) *pending = pend;
  if (dev >= 0 && dev != e->device) cudaSetDevice(dev);
  return MHIT_OK;
}

// Sleep until a scheduling round has something to do, or `timeout_s`
// passes: *ready = 1 or 0.  Transfer threads wake it when a job finishes;
// the class streams are looked at every 200 us (their queues hold a few
// milliseconds of rounds, so nothing idles meanwhile).
int mhit_ens_wait(mhit_ensemble* e, double timeout_s, int* ready) {
  if (!e || !(timeout_s >= 0)) return MHIT_ERR_INVALID;
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != e->device) cudaSetDevice(e->device);
  const double deadline = now_s() + timeout_s;
  int rdy = 0;
  for (;;) {
    unsigned long long seen;
    {
      std::lock_guard<std::mutex> g(e->wait_mu);
      seen = e->io_done;
    }
    if (work_ready(e)) {
      rdy = 1;
      break;
    }
    const double left = deadline - now_s();
    if (left <= 0) break;
    std::unique_lock<std::mutex> g(e->wait_mu);
    e->wait_cv.wait_for(g, std::chrono::microseconds((long long)std::min(left * 1e6, 200.0) + 1),
                        [&] { return e->io_done != seen; });
  }
  if (ready) *ready = rdy;
  if (dev >= 0 && dev != e->device) cudaSetDevice(dev);
  return MHIT_OK;
}

int mhit_ens_query(mhit_ensemble* e, int64_t id, mhit_ens_info* out) {
  if (!e || !out) return MHIT_ERR_INVALID;
  auto it = e->reqs.find(id);
  if (it == e->reqs.end()) return MHIT_ERR_INVALID;
  const Request* r = it->second.get();
  memset(out, 0, sizeof(*out));
  out->state = r->state;
  out->status = r->status;
  out->n = r->n;
  out->steps_issued = r->steps_issued;
  out->t_submit = r->t_submit - e->t0;
  out->t_admit = r->t_admit > 0 ? r->t_admit - e->t0 : -1.0;
  out->t_done = r->t_done > 0 ? r->t_done - e->t0 : -1.0;
  out->diag = r->diag;
  if (r->cls >= 0) {
    out->kz = e->classes[r->cls]->kz;
    out->mty = e->classes[r->cls]->mty;
  }
  return MHIT_OK;
}

int mhit_ens_result(mhit_ensemble* e, int64_t id, double* u, double* v, double* w, double* phi) {
  if (!e) return MHIT_ERR_INVALID;
  auto it = e->reqs.find(id);
  if (it == e->reqs.end()) return MHIT_ERR_INVALID;
  Request* r = it->second.get();
  if (r->state != RQ_DONE && r->state != RQ_FAILED) return MHIT_ERR_STATE;
  if (!r->keep || r->out[0].empty()) return MHIT_ERR_STATE;
  double* dst[4] = {u, v, w, phi};
  for (int f = 0; f < 4; ++f)
    if (dst[f] && !r->out[f].empty()) memcpy(dst[f], r->out[f].data(), r->out[f].size() * sizeof(double));
  return MHIT_OK;
}

// Drop a finished request's record (and its kept fields).
int mhit_ens_release(mhit_ensemble* e, int64_t id) {
  if (!e) return MHIT_ERR_INVALID;
  auto it = e->reqs.find(id);
  if (it == e->reqs.end()) return MHIT_ERR_INVALID;
  if (it->second->state == RQ_QUEUED || it->second->state == RQ_RUNNING) return MHIT_ERR_STATE;
  e->reqs.erase(it);
  return MHIT_OK;
}

// Cancel a queued or running request.  A running one is taken out of its
// batch at once: this call waits for the class stream to pass that point and
// for the transfer threads to finish any job of the request.
int mhit_ens_cancel(mhit_ensemble* e, int64_t id) {
  if (!e) return MHIT_ERR_INVALID;
  auto it = e->reqs.find(id);
  if (it == e->reqs.end()) return MHIT_ERR_INVALID;
  Request* r = it->second.get();
  if (r->state == RQ_QUEUED) {
    e->queue.erase(std::remove(e->queue.begin(), e->queue.end(), id), e->queue.end());
  } else if (r->state == RQ_RUNNING) {
    Class* c = e->classes[r->cls].get();
    if (r->loading) {
      wait_io(r->up);
      r->loading = false;
    } else if (r->finishing) {
      ECK(e, cudaEventSynchronize(r->done_ev));
      if (r->down.load() == IO_QUEUED) wait_io(r->down);
      put_event(e, r->done_ev);
      r->done_ev = nullptr;
      r->finishing = false;
    } else {
      c->running.erase(std::remove(c->running.begin(), c->running.end(), id), c->running.end());
      ECK(e, set_active(c, r->slot, 0));
      cudaEvent_t ev = nullptr;
      ECK(e, get_event(e, &ev));
      ECK(e, cudaEventRecord(ev, c->st));
      ECK(e, cudaEventSynchronize(ev));
      put_event(e, ev);
    }
    for (auto& v : r->in) std::vector<double>().swap(v);
    c->slots[r->slot].req = -1;
  } else {
    return MHIT_OK;
  }
  r->state = RQ_CANCELLED;
  r->t_done = now_s();
  return MHIT_OK;
}

int mhit_ens_stats(mhit_ensemble* e, mhit_ens_stats_t* out) {
  if (!e || !out) return MHIT_ERR_INVALID;
  memset(out, 0, sizeof(*out));
  out->rounds = e->rounds;
  out->graph_launches = e->launches;
  out->bytes_used = e->used;
  out->bytes_budget = e->budget;
  out->classes = (int)e->classes.size();
  for (auto& c : e->classes) out->slots += c->nslots;
  return MHIT_OK;
}

const char* mhit_ens_last_error(mhit_ensemble* e) { return e ? e->last_error.c_str() : ""; }

int mhit_ens_destroy(mhit_ensemble* e) {
  if (!e) return MHIT_ERR_INVALID;
  if (e->xfer_started)  // finishes the queued jobs first
    for (auto& x : e->xfer) x.stop();
  for (auto& c : e->classes) cudaStreamSynchronize(c->st);
  for (auto& kv : e->reqs)
    if (kv.second->done_ev) cudaEventDestroy(kv.second->done_ev);
  for (auto& c : e->classes) {
    for (auto& b : c->slots) free_slot_buffers(e, b);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    for (auto ev : c->inflight) cudaEventDestroy(ev);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    cudaFree(c->d_slots);
    cudaFree(c->d_ctrl);
    cudaFree(c->tw);
    cudaFree(c->k2tab);
    cudaStreamDestroy(c->st);
  }
  for (auto ev : e->free_events) cudaEventDestroy(ev);
  delete e;
  return MHIT_OK;
}

}  // extern "C"
