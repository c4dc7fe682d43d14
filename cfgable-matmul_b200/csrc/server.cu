// server.cu -- the density-serving loop: continuous batching of AO-DM-AO
// requests from many molecules on one GPU under an HBM budget.
//
// A molecule is opened once (its phi and mask from host arrays, from the
// caller's device arrays, or evaluated on the device from Gaussian shells)
// and then receives requests: "contract these density matrices with my phi".
// One worker thread owns the GPU side:
//   * admission: pending requests are taken in arrival order; a request
//     starts when a slot (a CUDA stream) is free, its molecule has no request
//     on the GPU (requests of one molecule run in order), and its molecule is
//     resident or fits in the budget -- idle molecules are evicted, least
//     recently used first, to make room.  Later requests of resident molecules
//     may start ahead of an earlier one that waits for memory;
//   * residency: the molecule's phi, mask, density-matrix and rho buffers and
//     its batched plan (active lists, graph-captured persistent contraction;
//     in split precision also the phi digit tiles) stay on the device across
//     its requests, so a request moves only D in and rho out;
//   * completion: every request ends with a host callback on its stream that
//     copies rho to the caller's buffer and wakes the worker and waiters.
// Requests of different molecules overlap on the device (copies of one with
// the contraction of another, and kernels where resources allow).  Results
// do not depend on what else runs: every reduction has a fixed order.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/cfgmm.h"
#include "ao_eval.cuh"
#include "aodmao2rho_fp64.cuh"
#include "aodmao2rho_split.cuh"
#include "server.cuh"

namespace cfgmm {
void set_last_error(const std::string& msg);
int aodm_plan_release_idle(cfgmm_aodm_plan* plan, cudaStream_t stream);
double aodm_plan_flops(const cfgmm_aodm_plan* plan);
}  // namespace cfgmm

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kLoaders = 4;  // molecules put on the device at once

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

size_t a256(size_t v) { return (v + 255) / 256 * 256; }

// ---- pinned host staging, reused by size class ----------------------------
// One pool for the process (portable pinned memory, usable from every
// device): a buffer outlives the server that pinned it, so a later server, or
// a later request of the same size class, gets it without pinning host memory
// while other requests run.  cfgmm_release_workspace frees the idle ones.
class PinnedPool {
 public:
  void* get(size_t bytes) {
    const size_t cls = size_class(bytes);
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto it = free_.find(cls);
      if (it != free_.end() && !it->second.empty()) {
        void* p = it->second.back();
        it->second.pop_back();
        return p;
      }
    }
    void* p = nullptr;
    if (cudaHostAlloc(&p, cls, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    std::lock_guard<std::mutex> lk(mu_);
    size_of_[p] = cls;
    return p;
  }
  void put(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu_);
    free_[size_of_[p]].push_back(p);
  }
  // Frees the buffers no request holds.
  void trim() {
    std::lock_guard<std::mutex> lk(mu_);
    for (auto& kv : free_)
      for (void* p : kv.second) {
        cudaFreeHost(p);
        size_of_.erase(p);
      }
    free_.clear();
  }

 private:
  static size_t size_class(size_t b) {
    size_t c = 4096;
    while (c < b) c <<= 1;
    return c;
  }
  std::mutex mu_;
  std::map<size_t, std::vector<void*>> free_;
  std::unordered_map<void*, size_t> size_of_;
};

// Never destroyed: freeing pinned memory from a static destructor would race
// the CUDA runtime's own teardown at exit.
PinnedPool& pinned_pool() {
  static PinnedPool* pool = new PinnedPool();
  return *pool;
}

enum Kind { kHost = 0, kDevice = 1, kShells = 2 };

struct Molecule {
  uint64_t id = 0;
  Kind kind = kHost;
  size_t nao = 0, ngrid = 0, ldtab = 0, nset_max = 0;
  // sources
  const double* src_lhs = nullptr;  // host (kHost) or caller device (kDevice)
  const double* src_rhs = nullptr;
  const uint8_t* src_tab = nullptr;
  std::vector<double> pts, sxyz, salpha, snorm;  // kShells
  std::vector<int> sl, srow;
  double density = 0.0;
  // resident state
  bool resident = false;
  void* mem = nullptr;
  const double* d_lhs = nullptr;
  const double* d_rhs = nullptr;
  const uint8_t* d_tab = nullptr;
  double* d_dms = nullptr;
  double* d_rho = nullptr;
  std::map<size_t, cfgmm_aodm_plan*> plans;  // by nset
  size_t cost = 0;                            // bytes counted against the budget
  bool busy = false, closed = false;
  bool loading = false;  // being put on the device by the loader thread
  int pending = 0;  // requests queued or on the GPU
  uint64_t last_use = 0;
  // recorded after the device work that puts the molecule and its plans on
  // the device; every request's slot stream waits for it (no host wait)
  cudaEvent_t ready = nullptr;
  Molecule() = default;
  Molecule(const Molecule&) = delete;
  Molecule& operator=(const Molecule&) = delete;
  ~Molecule() {
    if (ready) cudaEventDestroy(ready);
  }
};

struct Request {
  uint64_t ticket = 0;
  uint64_t mol = 0;
  size_t nset = 0;
  double* user_rho = nullptr;
  void* pin_d = nullptr;
  void* pin_rho = nullptr;
  // device-resident request: the caller's D and rho on the device, D read
  // after `ready` (recorded on the caller's stream at submit)
  bool on_device = false;
  const double* dev_d = nullptr;
  cudaEvent_t ready = nullptr;
  size_t d_bytes = 0, rho_bytes = 0;
  Clock::time_point t_submit, t_launch, t_done;
  float device_ms = 0.f;
  double flops = 0.0;
  int slot = -1;
  bool cold = false;         // its molecule was put on the device for it
  // set by the host callback, which takes no lock: a host function must not
  // wait on a thread that may itself be inside a CUDA call
  std::atomic<bool> device_done{false};
  bool finished = false;     // set by the worker
  int status = CFGMM_OK;
  std::string error;
  struct cfgmm_server* srv = nullptr;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  Request* req = nullptr;
};

}  // namespace

namespace cfgmm {
void release_pinned_staging() { pinned_pool().trim(); }
}  // namespace cfgmm

struct cfgmm_server {
  int dev = 0;
  size_t budget = 0;
  int precision = CFGMM_PREC_FP64;
  size_t blksize = 64;
  std::vector<Slot> slots;
  cudaStream_t admin = nullptr;

  std::mutex mu;
  std::condition_variable cv_work;  // worker: new requests, completions, stop
  std::condition_variable cv_done;  // waiters
  std::condition_variable cv_load;  // loader: molecules to put on the device
  bool stop = false, stop_loader = false;  // the loaders stop after the worker
  std::thread worker;
  // molecules are put on the device by several loader threads at once, each on
  // its own high-priority stream (the eval / mask / plan work of one molecule
  // is serial, of different molecules independent)
  std::vector<std::thread> loaders;
  std::vector<cudaStream_t> load_streams;
  size_t inflight = 0, max_inflight = 0;  // requests on the slots, and their maximum
  std::deque<uint64_t> to_load;  // tickets whose molecule is being loaded
  int loading = 0;

  uint64_t next_mol = 1, next_ticket = 1, tick = 0;
  std::unordered_map<uint64_t, std::unique_ptr<Molecule>> mols;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  std::deque<uint64_t> pending;  // tickets in arrival order

  size_t used = 0, peak = 0;
  uint64_t admitted_molecules = 0, evictions = 0, completed = 0, failed = 0;
  double flops_done = 0.0;
  std::vector<double> lat_total, lat_queue, lat_device, lat_warm, lat_load, lat_plan;
  std::string stats_json;
};

namespace {

int fail(int status, const std::string& msg) {
  cfgmm::set_last_error(msg);
  return status;
}

std::string cuda_msg(cudaError_t e, const char* where) {
  return std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
}

// Offsets of a molecule's server-owned device buffers.
struct MolLayout {
  size_t lhs, rhs, tab, dms, rho, pts, xyz, alpha, norm, l, row, bmax, bytes;
};

MolLayout mol_layout(const Molecule& m, size_t blksize) {
  const size_t phi = m.nao * m.ngrid * sizeof(double);
  const size_t nsh = m.sl.size(), nblk = (m.ngrid + blksize - 1) / blksize;
  const bool owned = m.kind != kDevice;
  MolLayout L{};
  size_t off = 0;
  L.lhs = off;
  if (owned) off += a256(phi);
  L.rhs = off;
  if (m.kind == kHost && m.src_rhs != m.src_lhs) off += a256(phi);
  L.tab = off;
  if (owned) off += a256(m.nao * m.ldtab);
  L.dms = off;
  off += a256(m.nset_max * m.nao * m.nao * sizeof(double));
  L.rho = off;
  off += a256(m.nset_max * m.ngrid * sizeof(double));
  L.pts = L.xyz = L.alpha = L.norm = L.l = L.row = L.bmax = off;
  if (m.kind == kShells) {
    L.pts = off;
    off += a256(m.ngrid * 3 * sizeof(double));
    L.xyz = off;
    off += a256(nsh * 3 * sizeof(double));
    L.alpha = off;
    off += a256(nsh * sizeof(double));
    L.norm = off;
    off += a256(nsh * sizeof(double));
    L.l = off;
    off += a256(nsh * sizeof(int));
    L.row = off;
    off += a256(nsh * sizeof(int));
    L.bmax = off;
    off += a256(nsh * nblk * sizeof(double));
  }
  L.bytes = off;
  return L;
}

// Device bytes a molecule holds while resident: its own buffers, the caller's
// phi and mask for a device molecule, and an upper bound of its plan (the
// single-call workspace bounds the plan's lists, work list, digits and
// partial sums).
size_t molecule_cost(const Molecule& m, int precision, size_t blksize) {
  size_t cost = mol_layout(m, blksize).bytes;
  if (m.kind == kDevice)
    cost += m.nao * m.ngrid * sizeof(double) * (m.src_rhs != m.src_lhs ? 2 : 1) + m.nao * m.ldtab;
  const size_t plan = precision == CFGMM_PREC_OZAKI_INT8
                          ? cfgmm::aodmao2rho_split_workspace(m.nao, m.ngrid, m.nset_max, blksize)
                          : cfgmm::aodmao2rho_fp64_workspace(m.nao, m.ngrid, m.nset_max, blksize);
  return cost + plan + (1u << 20);
}

// Frees a resident, idle molecule's device state (lock held).
void release(cfgmm_server* s, Molecule& m) {
  // the frees on the admin stream come after the molecule's load and plan work
  if (m.ready) cudaStreamWaitEvent(s->admin, m.ready, 0);
  for (auto& kv : m.plans) cfgmm::aodm_plan_release_idle(kv.second, s->admin);
  m.plans.clear();
  if (m.mem) cudaFreeAsync(m.mem, s->admin);
  m.mem = nullptr;
  m.resident = false;
  s->used -= m.cost;
}

// Puts the molecule's phi, mask and buffers on the device (a loader thread,
// without the lock: the molecule is reserved; the GPU work is enqueued on the
// loader's stream `st`).
int materialize(cfgmm_server* s, Molecule& m, cudaStream_t st, std::string* err) {
  const size_t phi = m.nao * m.ngrid * sizeof(double);
  const size_t nblk = (m.ngrid + s->blksize - 1) / s->blksize;
  const size_t nsh = m.sl.size();
  const MolLayout L = mol_layout(m, s->blksize);
  cudaError_t e = cudaMallocAsync(&m.mem, L.bytes, st);
  if (e != cudaSuccess) {
    m.mem = nullptr;
    *err = cuda_msg(e, "molecule memory");
    return e == cudaErrorMemoryAllocation ? CFGMM_ERR_OUT_OF_MEMORY : CFGMM_ERR_CUDA;
  }
  char* base = static_cast<char*>(m.mem);
  m.d_dms = reinterpret_cast<double*>(base + L.dms);
  m.d_rho = reinterpret_cast<double*>(base + L.rho);
  if (m.kind == kDevice) {
    m.d_lhs = m.src_lhs;
    m.d_rhs = m.src_rhs;
    m.d_tab = m.src_tab;
  } else {
    m.d_lhs = reinterpret_cast<double*>(base + L.lhs);
    m.d_rhs = (m.kind == kHost && m.src_rhs != m.src_lhs) ? reinterpret_cast<double*>(base + L.rhs)
                                                          : m.d_lhs;
    m.d_tab = reinterpret_cast<uint8_t*>(base + L.tab);
  }
  if (m.kind == kHost) {
    e = cudaMemcpyAsync(const_cast<double*>(m.d_lhs), m.src_lhs, phi, cudaMemcpyHostToDevice,
                        st);
    if (e == cudaSuccess && m.d_rhs != m.d_lhs)
      e = cudaMemcpyAsync(const_cast<double*>(m.d_rhs), m.src_rhs, phi, cudaMemcpyHostToDevice,
                          st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(const_cast<uint8_t*>(m.d_tab), m.src_tab, m.nao * m.ldtab,
                          cudaMemcpyHostToDevice, st);
  } else if (m.kind == kShells) {
    double* d_pts = reinterpret_cast<double*>(base + L.pts);
    double* d_xyz = reinterpret_cast<double*>(base + L.xyz);
    double* d_alpha = reinterpret_cast<double*>(base + L.alpha);
    double* d_norm = reinterpret_cast<double*>(base + L.norm);
    int* d_l = reinterpret_cast<int*>(base + L.l);
    int* d_row = reinterpret_cast<int*>(base + L.row);
    double* d_bmax = reinterpret_cast<double*>(base + L.bmax);
    e = cudaMemcpyAsync(d_pts, m.pts.data(), m.ngrid * 3 * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_xyz, m.sxyz.data(), nsh * 3 * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_alpha, m.salpha.data(), nsh * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_norm, m.snorm.data(), nsh * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_l, m.sl.data(), nsh * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_row, m.srow.data(), nsh * 4, cudaMemcpyHostToDevice, st);
    double* ao = const_cast<double*>(m.d_lhs);
    if (e == cudaSuccess)
      e = cfgmm::eval_ao(ao, m.ngrid, d_pts, int(m.ngrid), d_xyz, d_l, d_alpha, d_norm, d_row,
                         int(nsh), d_bmax, int(s->blksize), st);
    // threshold: the (1 - density) quantile of the (shell, block) maxima
    double thr = -1.0;
    if (e == cudaSuccess && m.density < 1.0) {
      std::vector<double> h(nsh * nblk);
      e = cudaMemcpyAsync(h.data(), d_bmax, h.size() * 8, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e == cudaSuccess) {
        const size_t k = std::min(h.size() - 1, size_t((1.0 - m.density) * double(h.size() - 1)));
        std::nth_element(h.begin(), h.begin() + k, h.end());
        thr = h[k];
      }
    }
    if (e == cudaSuccess)
      e = cfgmm::mask_ao(ao, m.ngrid, int(m.ngrid), d_l, d_row, int(nsh), d_bmax, thr,
                         const_cast<uint8_t*>(m.d_tab), m.ldtab, int(s->blksize), st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    *err = cuda_msg(e, "molecule upload");
    cudaFreeAsync(m.mem, st);
    m.mem = nullptr;
    return CFGMM_ERR_CUDA;
  }
  return CFGMM_OK;
}

cfgmm_aodm_plan* plan_for(cfgmm_server* s, Molecule& m, size_t nset, cudaStream_t st, int* rc) {
  auto it = m.plans.find(nset);
  if (it != m.plans.end()) return it->second;
  cfgmm_aodm_batch b;
  b.rhos = m.d_rho;
  b.ao_lhs = m.d_lhs;
  b.ao_rhs = m.d_rhs;
  b.tab = m.d_tab;
  b.stride_grid = m.ngrid;
  b.ngrid = m.ngrid;
  b.ldtab = m.ldtab;
  b.nset = nset;
  cfgmm_aodm_plan* plan = nullptr;
  *rc = cfgmm_aodm_plan_create(&plan, &b, 1, m.d_dms, m.nao, m.nao, nset, s->blksize, s->precision,
                               0, st);
  if (*rc != CFGMM_OK) return nullptr;
  m.plans[nset] = plan;
  return plan;
}

void CUDART_CB on_device_done(void* arg) {
  Request* r = static_cast<Request*>(arg);
  if (!r->on_device) std::memcpy(r->user_rho, r->pin_rho, r->rho_bytes);
  cfgmm_server* s = r->srv;
  // r may be gone once the flag is up; the server outlives its slot streams'
  // callbacks (destroy synchronises them).  A wakeup lost to the unlocked
  // notify costs the worker at most its 5 ms poll.
  r->device_done.store(true, std::memory_order_release);
  s->cv_work.notify_one();
}

void finish(cfgmm_server* s, Request& r, int status, const std::string& err) {
  r.status = status;
  r.error = err;
  r.finished = true;
  r.t_done = Clock::now();
  pinned_pool().put(r.pin_d);
  pinned_pool().put(r.pin_rho);
  r.pin_d = r.pin_rho = nullptr;
  if (r.ready) cudaEventDestroy(r.ready);
  r.ready = nullptr;
  auto it = s->mols.find(r.mol);
  if (it != s->mols.end()) {
    Molecule& m = *it->second;
    m.busy = false;
    --m.pending;
    m.last_use = ++s->tick;
  }
  if (status == CFGMM_OK) {
    ++s->completed;
    s->lat_total.push_back(ms_between(r.t_submit, r.t_done));
    s->lat_queue.push_back(ms_between(r.t_submit, r.t_launch));
    s->lat_device.push_back(r.device_ms);
    if (!r.cold) s->lat_warm.push_back(ms_between(r.t_submit, r.t_done));
    s->flops_done += r.flops;
  } else {
    ++s->failed;
  }
  s->cv_done.notify_all();
}

// Frees closed molecules that have no work left.
void reap(cfgmm_server* s) {
  for (auto it = s->mols.begin(); it != s->mols.end();) {
    Molecule& m = *it->second;
    if (m.closed && m.pending == 0) {
      if (m.resident) release(s, m);
      it = s->mols.erase(it);
    } else {
      ++it;
    }
  }
}

// Makes room for `need` bytes by evicting idle resident molecules, least
// recently used first, closed ones and those without queued requests before
// the others.  Returns whether the room is there.
bool make_room(cfgmm_server* s, size_t need, uint64_t keep) {
  if (s->used + need <= s->budget) return true;
  std::vector<Molecule*> idle;
  for (auto& kv : s->mols) {
    Molecule& m = *kv.second;
    if (m.resident && !m.busy && m.id != keep) idle.push_back(&m);
  }
  std::sort(idle.begin(), idle.end(), [](const Molecule* a, const Molecule* b) {
    const int pa = a->pending > 0, pb = b->pending > 0;
    return pa != pb ? pa < pb : a->last_use < b->last_use;
  });
  for (Molecule* m : idle) {
    if (s->used + need <= s->budget) break;
    release(s, *m);
    ++s->evictions;
  }
  return s->used + need <= s->budget;
}

// Enqueues one request on its slot (worker thread, without the lock: the
// molecule and the slot are reserved).  Returns a status and message.
int launch(cfgmm_server* s, Request& r, Molecule& m, Slot& sl, std::string* err) {
  int rc = CFGMM_OK;
  const bool built = m.plans.count(r.nset) == 0;
  cfgmm_aodm_plan* plan = plan_for(s, m, r.nset, s->admin, &rc);
  if (!plan) {
    *err = std::string("plan: ") + cfgmm_last_error();
    return rc;
  }
  // a plan built here (a request with another nset): its device work on the
  // admin stream, after what the event stood for, comes before the request's
  if (built) {
    cudaError_t e = cudaSuccess;
    if (m.ready) e = cudaStreamWaitEvent(s->admin, m.ready, 0);
    else e = cudaEventCreateWithFlags(&m.ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(m.ready, s->admin);
    if (e != cudaSuccess) {
      *err = cuda_msg(e, "plan");
      return CFGMM_ERR_CUDA;
    }
  }
  r.flops = cfgmm::aodm_plan_flops(plan);
  r.t_launch = Clock::now();
  cudaError_t e = m.ready ? cudaStreamWaitEvent(sl.stream, m.ready, 0) : cudaSuccess;
  if (e == cudaSuccess && r.on_device) {
    e = cudaStreamWaitEvent(sl.stream, r.ready, 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(m.d_dms, r.dev_d, r.d_bytes, cudaMemcpyDeviceToDevice, sl.stream);
  } else if (e == cudaSuccess) {
    e = cudaMemcpyAsync(m.d_dms, r.pin_d, r.d_bytes, cudaMemcpyHostToDevice, sl.stream);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(m.d_rho, 0, r.rho_bytes, sl.stream);
  if (e == cudaSuccess) e = cudaEventRecord(sl.e0, sl.stream);
  if (e == cudaSuccess && (rc = cfgmm_aodm_plan_run(plan, sl.stream)) != CFGMM_OK) {
    *err = cfgmm_last_error();
    return rc;
  }
  if (e == cudaSuccess) e = cudaEventRecord(sl.e1, sl.stream);
  if (e == cudaSuccess)
    e = r.on_device ? cudaMemcpyAsync(r.user_rho, m.d_rho, r.rho_bytes, cudaMemcpyDeviceToDevice,
                                      sl.stream)
                    : cudaMemcpyAsync(r.pin_rho, m.d_rho, r.rho_bytes, cudaMemcpyDeviceToHost,
                                      sl.stream);
  if (e == cudaSuccess) e = cudaLaunchHostFunc(sl.stream, on_device_done, &r);
  if (e != cudaSuccess) {
    *err = cuda_msg(e, "request launch");
    return CFGMM_ERR_CUDA;
  }
  return CFGMM_OK;
}

// The next request that can start now, with its slot reserved, or null.
// A request whose molecule is not on the device goes to the loader instead
// (its memory reserved) and comes back to the front of the queue when the
// molecule is resident, so warm requests keep flowing meanwhile.  Lock held.
Request* pick(cfgmm_server* s, int* slot_out) {
  int free_slot = -1;
  for (size_t i = 0; i < s->slots.size(); ++i)
    if (!s->slots[i].req) {
      free_slot = int(i);
      break;
    }
  for (auto it = s->pending.begin(); it != s->pending.end();) {
    Request& r = *s->reqs.find(*it)->second;
    Molecule& m = *s->mols.find(r.mol)->second;
    if (m.busy) {  // one request of a molecule at a time, in order
      ++it;
      continue;
    }
    if (!m.resident) {
      if (!make_room(s, m.cost, m.id)) {  // waits for memory
        ++it;
        continue;
      }
      s->used += m.cost;  // reserved; the loader puts it on the device
      s->peak = std::max(s->peak, s->used);
      m.resident = true;
      m.loading = true;
      m.busy = true;
      m.mem = nullptr;
      r.cold = true;
      s->to_load.push_back(*it);
      it = s->pending.erase(it);
      s->cv_load.notify_one();
      continue;
    }
    if (free_slot < 0) return nullptr;
    s->pending.erase(it);
    m.busy = true;
    m.last_use = ++s->tick;
    s->slots[free_slot].req = &r;
    r.slot = free_slot;
    *slot_out = free_slot;
    return &r;
  }
  return nullptr;
}

// Puts molecules on the device (phi, mask, buffers, plan) one at a time on
// the admin stream, beside the requests running on the slots.
void loader_loop(cfgmm_server* s, cudaStream_t st) {
  cudaSetDevice(s->dev);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    s->cv_load.wait(lk, [&] { return s->stop_loader || !s->to_load.empty(); });
    if (s->to_load.empty()) {
      if (s->stop_loader) break;
      continue;
    }
    const uint64_t ticket = s->to_load.front();
    s->to_load.pop_front();
    ++s->loading;
    Request& r = *s->reqs.find(ticket)->second;
    Molecule& m = *s->mols.find(r.mol)->second;
    lk.unlock();
    std::string err;
    const Clock::time_point t0 = Clock::now();
    int rc = materialize(s, m, st, &err);
    if (rc == CFGMM_OK) {  // the load's device work (copies, AO evaluation) counts as the load
      const cudaError_t e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) {
        rc = CFGMM_ERR_CUDA;
        err = cuda_msg(e, "molecule load");
      }
    }
    const Clock::time_point t1 = Clock::now();
    if (rc == CFGMM_OK && !plan_for(s, m, r.nset, st, &rc))
      err = std::string("plan: ") + cfgmm_last_error();
    if (rc == CFGMM_OK) {  // the requests' slot streams wait for this point of st
      cudaError_t e = m.ready ? cudaSuccess
                              : cudaEventCreateWithFlags(&m.ready, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventRecord(m.ready, st);
      if (e != cudaSuccess) {
        rc = CFGMM_ERR_CUDA;
        err = cuda_msg(e, "molecule load");
      }
    }
    const Clock::time_point t2 = Clock::now();
    lk.lock();
    s->lat_load.push_back(ms_between(t0, t1));
    s->lat_plan.push_back(ms_between(t1, t2));
    --s->loading;
    m.loading = false;
    if (rc == CFGMM_OK) {
      ++s->admitted_molecules;
      m.busy = false;
      s->pending.push_front(ticket);
    } else {
      for (auto& kv : m.plans) cfgmm::aodm_plan_release_idle(kv.second, s->admin);
      m.plans.clear();
      if (m.mem) cudaFreeAsync(m.mem, s->admin);
      m.mem = nullptr;
      m.resident = false;
      s->used -= m.cost;
      finish(s, r, rc, err);
    }
    s->cv_work.notify_one();
  }
}

void worker_loop(cfgmm_server* s) {
  cudaSetDevice(s->dev);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    // completions
    for (Slot& sl : s->slots) {
      if (sl.req && sl.req->device_done.load(std::memory_order_acquire)) {
        Request& r = *sl.req;
        cudaEventElapsedTime(&r.device_ms, sl.e0, sl.e1);
        sl.req = nullptr;
        --s->inflight;
        finish(s, r, CFGMM_OK, "");
      }
    }
    reap(s);
    // admission: one request at a time, the GPU work enqueued without the lock
    int slot = -1;
    if (Request* r = pick(s, &slot)) {
      Molecule& m = *s->mols.find(r->mol)->second;
      s->max_inflight = std::max(s->max_inflight, ++s->inflight);
      lk.unlock();
      std::string err;
      const int rc = launch(s, *r, m, s->slots[slot], &err);
      lk.lock();
      if (rc != CFGMM_OK) {
        s->slots[slot].req = nullptr;
        --s->inflight;
        finish(s, *r, rc, err);
      }
      continue;  // look for more work before sleeping
    }
    bool inflight = false;
    for (Slot& sl : s->slots) inflight |= sl.req != nullptr;
    if (s->stop && !inflight && s->pending.empty() && s->to_load.empty() && s->loading == 0)
      break;
    s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
  }
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * double(v.size() - 1);
  const size_t i = size_t(pos);
  const double f = pos - double(i);
  return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

int check_server(cfgmm_server* s) {
  cfgmm::set_last_error("");
  if (!s) return fail(CFGMM_ERR_INVALID_ARGUMENT, "null server");
  return CFGMM_OK;
}

int open_common(cfgmm_server* s, std::unique_ptr<Molecule> m, uint64_t* id) {
  m->cost = molecule_cost(*m, s->precision, s->blksize);
  if (m->cost > s->budget)
    return fail(CFGMM_ERR_OUT_OF_MEMORY, "molecule needs " + std::to_string(m->cost) +
                                             " bytes, above the server's budget of " +
                                             std::to_string(s->budget));
  std::lock_guard<std::mutex> lk(s->mu);
  m->id = s->next_mol++;
  *id = m->id;
  s->mols[m->id] = std::move(m);
  return CFGMM_OK;
}

int check_sizes(size_t nao, size_t ngrid, size_t ldtab, size_t nset_max, size_t blksize,
                int precision) {
  if (nao == 0 || ngrid == 0 || nset_max == 0)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "empty molecule");
  if (nao > 1000000 || ngrid > 0x7fff0000u || nset_max > 64)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "molecule dimensions out of range");
  if (ldtab < (ngrid + blksize - 1) / blksize)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "ldtab below the number of grid blocks");
  if (precision == CFGMM_PREC_OZAKI_INT8 && nao > 16384)
    return fail(CFGMM_ERR_UNIMPLEMENTED, "split-precision AO-DM-AO supports nao <= 16384");
  return CFGMM_OK;
}

}  // namespace

extern "C" {

int cfgmm_server_create(cfgmm_server** out, size_t hbm_budget, int nslots, int precision,
                        size_t blksize) {
  cfgmm::set_last_error("");
  if (!out) return fail(CFGMM_ERR_INVALID_ARGUMENT, "null server pointer");
  *out = nullptr;
  if (precision != CFGMM_PREC_FP64 && precision != CFGMM_PREC_OZAKI_INT8)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "unknown precision " + std::to_string(precision));
  if (nslots < 1 || nslots > 64 || blksize == 0 || blksize > 65536 || hbm_budget == 0)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "invalid server configuration");
  int ndev = 0, dev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return fail(CFGMM_ERR_NO_DEVICE, "no CUDA device");
  }
  // the stream-ordered pool keeps freed molecule memory for the next one
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  auto s = std::make_unique<cfgmm_server>();
  s->dev = dev;
  s->budget = hbm_budget;
  s->precision = precision;
  s->blksize = blksize;
  s->slots.resize(nslots);
  // molecule loading runs at the highest stream priority: its kernels are
  // scheduled ahead of queued request kernels as SMs free up
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  cudaError_t e = cudaStreamCreateWithPriority(&s->admin, cudaStreamNonBlocking, prio_hi);
  s->load_streams.assign(kLoaders, nullptr);
  for (cudaStream_t& ls : s->load_streams)
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&ls, cudaStreamNonBlocking, prio_hi);
  for (Slot& sl : s->slots) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&sl.e0);
    if (e == cudaSuccess) e = cudaEventCreate(&sl.e1);
  }
  if (e != cudaSuccess) return fail(CFGMM_ERR_CUDA, cuda_msg(e, "server streams"));
  cfgmm_server* raw = s.release();
  raw->worker = std::thread(worker_loop, raw);
  for (cudaStream_t ls : raw->load_streams) raw->loaders.emplace_back(loader_loop, raw, ls);
  *out = raw;
  return CFGMM_OK;
}

int cfgmm_server_destroy(cfgmm_server* s) {
  if (!s) return CFGMM_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_one();
  if (s->worker.joinable()) s->worker.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop_loader = true;
  }
  s->cv_load.notify_all();
  for (std::thread& t : s->loaders)
    if (t.joinable()) t.join();
  for (auto& kv : s->mols)
    if (kv.second->resident) release(s, *kv.second);
  cudaStreamSynchronize(s->admin);
  for (Slot& sl : s->slots) {
    cudaStreamSynchronize(sl.stream);  // the last host callbacks have returned
    cudaStreamDestroy(sl.stream);
    cudaEventDestroy(sl.e0);
    cudaEventDestroy(sl.e1);
  }
  for (cudaStream_t ls : s->load_streams) {
    cudaStreamSynchronize(ls);
    cudaStreamDestroy(ls);
  }
  cudaStreamDestroy(s->admin);
  delete s;
  return CFGMM_OK;
}

int cfgmm_server_open(cfgmm_server* s, const double* ao_lhs, const double* ao_rhs,
                      const uint8_t* tab, size_t nao, size_t ngrid, size_t ldtab, size_t nset_max,
                      int on_device, uint64_t* molecule) {
  int rc = check_server(s);
  if (rc != CFGMM_OK) return rc;
  if (!ao_lhs || !tab || !molecule) return fail(CFGMM_ERR_INVALID_ARGUMENT, "null pointer");
  if ((rc = check_sizes(nao, ngrid, ldtab, nset_max, s->blksize, s->precision)) != CFGMM_OK)
    return rc;
  auto m = std::make_unique<Molecule>();
  m->kind = on_device ? kDevice : kHost;
  m->src_lhs = ao_lhs;
  m->src_rhs = ao_rhs ? ao_rhs : ao_lhs;
  m->src_tab = tab;
  m->nao = nao;
  m->ngrid = ngrid;
  m->ldtab = ldtab;
  m->nset_max = nset_max;
  return open_common(s, std::move(m), molecule);
}

int cfgmm_server_open_shells(cfgmm_server* s, const double* points, size_t ngrid,
                             const double* shell_xyz, const int* shell_l,
                             const double* shell_alpha, const double* shell_norm, size_t nshell,
                             double density, size_t nset_max, uint64_t* molecule) {
  int rc = check_server(s);
  if (rc != CFGMM_OK) return rc;
  if (!points || !shell_xyz || !shell_l || !shell_alpha || !shell_norm || !molecule)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "null pointer");
  if (nshell == 0 || nshell > 65535 || !(density > 0.0 && density <= 1.0))
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "need 1..65535 shells and 0 < density <= 1");
  auto m = std::make_unique<Molecule>();
  m->kind = kShells;
  size_t nao = 0;
  m->srow.resize(nshell);
  for (size_t i = 0; i < nshell; ++i) {
    if (shell_l[i] < 0 || shell_l[i] > 3)
      return fail(CFGMM_ERR_INVALID_ARGUMENT, "shell angular momentum must be 0..3");
    m->srow[i] = int(nao);
    nao += size_t(2 * shell_l[i] + 1);
  }
  const size_t ldtab = (ngrid + s->blksize - 1) / s->blksize;
  if ((rc = check_sizes(nao, ngrid, ldtab, nset_max, s->blksize, s->precision)) != CFGMM_OK)
    return rc;
  m->pts.assign(points, points + 3 * ngrid);
  m->sxyz.assign(shell_xyz, shell_xyz + 3 * nshell);
  m->sl.assign(shell_l, shell_l + nshell);
  m->salpha.assign(shell_alpha, shell_alpha + nshell);
  m->snorm.assign(shell_norm, shell_norm + nshell);
  m->density = density;
  m->nao = nao;
  m->ngrid = ngrid;
  m->ldtab = ldtab;
  m->nset_max = nset_max;
  m->src_lhs = m->src_rhs = nullptr;
  return open_common(s, std::move(m), molecule);
}

int cfgmm_server_close(cfgmm_server* s, uint64_t molecule) {
  int rc = check_server(s);
  if (rc != CFGMM_OK) return rc;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->mols.find(molecule);
    if (it == s->mols.end() || it->second->closed)
      return fail(CFGMM_ERR_INVALID_ARGUMENT, "unknown molecule");
    it->second->closed = true;
  }
  s->cv_work.notify_one();
  return CFGMM_OK;
}

}  // extern "C"

namespace {

// Queues a request: host D copied to pinned staging now, or (on_device) the
// caller's device D read once the work enqueued on `stream` so far is done.
int submit_common(cfgmm_server* s, uint64_t molecule, const double* dms, size_t nset,
                  double* rhos, bool on_device, cudaStream_t stream, uint64_t* ticket) {
  int rc = check_server(s);
  if (rc != CFGMM_OK) return rc;
  if (!dms || !rhos || !ticket) return fail(CFGMM_ERR_INVALID_ARGUMENT, "null pointer");
  size_t nao, ngrid;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->mols.find(molecule);
    if (it == s->mols.end() || it->second->closed)
      return fail(CFGMM_ERR_INVALID_ARGUMENT, "unknown or closed molecule");
    if (nset == 0 || nset > it->second->nset_max)
      return fail(CFGMM_ERR_INVALID_ARGUMENT, "nset must be 1..nset_max of the molecule");
    nao = it->second->nao;
    ngrid = it->second->ngrid;
  }
  auto r = std::make_unique<Request>();
  r->mol = molecule;
  r->nset = nset;
  r->user_rho = rhos;
  r->d_bytes = nset * nao * nao * sizeof(double);
  r->rho_bytes = nset * ngrid * sizeof(double);
  r->on_device = on_device;
  if (on_device) {
    r->dev_d = dms;
    cudaError_t e = cudaSetDevice(s->dev);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(r->ready, stream);
    if (e != cudaSuccess) {
      if (r->ready) cudaEventDestroy(r->ready);
      return fail(CFGMM_ERR_CUDA, cuda_msg(e, "submit"));
    }
  } else {
    r->pin_d = pinned_pool().get(r->d_bytes);
    r->pin_rho = pinned_pool().get(r->rho_bytes);
    if (!r->pin_d || !r->pin_rho) {
      pinned_pool().put(r->pin_d);
      pinned_pool().put(r->pin_rho);
      return fail(CFGMM_ERR_OUT_OF_MEMORY, "pinned staging");
    }
    std::memcpy(r->pin_d, dms, r->d_bytes);
  }
  r->srv = s;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->mols.find(molecule);
    if (it == s->mols.end() || it->second->closed) {
      pinned_pool().put(r->pin_d);
      pinned_pool().put(r->pin_rho);
      if (r->ready) cudaEventDestroy(r->ready);
      return fail(CFGMM_ERR_INVALID_ARGUMENT, "molecule closed during submit");
    }
    ++it->second->pending;
    r->ticket = s->next_ticket++;
    *ticket = r->ticket;
    s->pending.push_back(r->ticket);
    s->reqs[r->ticket] = std::move(r);
  }
  s->cv_work.notify_one();
  return CFGMM_OK;
}

}  // namespace

extern "C" {

int cfgmm_server_submit(cfgmm_server* s, uint64_t molecule, const double* dms, size_t nset,
                        double* rhos, uint64_t* ticket) {
  return submit_common(s, molecule, dms, nset, rhos, false, nullptr, ticket);
}

int cfgmm_server_submit_dev(cfgmm_server* s, uint64_t molecule, const double* dms, size_t nset,
                            double* rhos, void* stream, uint64_t* ticket) {
  return submit_common(s, molecule, dms, nset, rhos, true, static_cast<cudaStream_t>(stream),
                       ticket);
}

int cfgmm_server_wait(cfgmm_server* s, uint64_t ticket, double timeout_s,
                      cfgmm_request_stats* stats) {
  int rc = check_server(s);
  if (rc != CFGMM_OK) return rc;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return fail(CFGMM_ERR_INVALID_ARGUMENT, "unknown ticket");
  Request* r = it->second.get();
  auto done = [&] { return r->finished; };
  if (timeout_s < 0) {
    s->cv_done.wait(lk, done);
  } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
    return fail(CFGMM_ERR_TIMEOUT, "request still running");
  }
  if (stats) {
    stats->queue_ms = ms_between(r->t_submit, r->t_launch);
    stats->device_ms = r->device_ms;
    stats->total_ms = ms_between(r->t_submit, r->t_done);
    stats->flops = r->flops;
  }
  const int status = r->status;
  const std::string err = r->error;
  s->reqs.erase(it);
  if (status != CFGMM_OK) return fail(status, err);
  return CFGMM_OK;
}

const char* cfgmm_server_stats(cfgmm_server* s) {
  if (!s) return "";
  std::lock_guard<std::mutex> lk(s->mu);
  size_t resident = 0;
  for (auto& kv : s->mols) resident += kv.second->resident;
  double device_total = 0.0;  // sum of the requests' device spans
  for (double d : s->lat_device) device_total += d;
  char buf[1536];
  std::snprintf(
      buf, sizeof(buf),
      "{\"completed\":%llu,\"failed\":%llu,\"pending\":%zu,\"molecules\":%zu,\"resident\":%zu,"
      "\"admitted_molecules\":%llu,\"evictions\":%llu,\"budget_bytes\":%zu,\"used_bytes\":%zu,"
      "\"peak_bytes\":%zu,\"flops_completed\":%.6e,\"latency_ms\":{\"p50\":%.4f,\"p99\":%.4f,\"max\":%.4f},"
      "\"warm_latency_ms\":{\"p50\":%.4f,\"p99\":%.4f,\"count\":%zu},"
      "\"load_ms\":{\"p50\":%.4f,\"max\":%.4f},\"plan_ms\":{\"p50\":%.4f,\"max\":%.4f},"
      "\"queue_ms\":{\"p50\":%.4f,\"p99\":%.4f},\"device_ms\":{\"p50\":%.4f,\"p99\":%.4f},"
      "\"device_ms_total\":%.4f,\"max_inflight\":%zu,\"loaders\":%d}",
      (unsigned long long)s->completed, (unsigned long long)s->failed, s->pending.size(),
      s->mols.size(), resident, (unsigned long long)s->admitted_molecules,
      (unsigned long long)s->evictions, s->budget, s->used, s->peak, s->flops_done,
      percentile(s->lat_total, 0.5), percentile(s->lat_total, 0.99),
      percentile(s->lat_total, 1.0), percentile(s->lat_warm, 0.5), percentile(s->lat_warm, 0.99),
      s->lat_warm.size(), percentile(s->lat_load, 0.5), percentile(s->lat_load, 1.0),
      percentile(s->lat_plan, 0.5), percentile(s->lat_plan, 1.0), percentile(s->lat_queue, 0.5),
      percentile(s->lat_queue, 0.99), percentile(s->lat_device, 0.5),
      percentile(s->lat_device, 0.99), device_total, s->max_inflight, kLoaders);
  s->stats_json = buf;
  return s->stats_json.c_str();
}

}  // extern "C"
