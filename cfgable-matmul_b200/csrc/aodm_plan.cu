// aodm_plan.cu -- many grid batches of one molecule in one persistent,
// graph-captured launch, with tile shapes chosen by an autotuner.
//
// A plan is built once for a set of grid batches whose phi tables and masks
// stay resident and unchanged (the density matrices may change between runs,
// as in an SCF loop).  Building it:
//   1. active AO lists of every block of every batch (one kernel per batch);
//   2. one global work list (batch, 64-point tile, 64-row tile of I(b)),
//      heaviest items first, so the persistent kernel's atomic counter hands
//      out work largest-first and the tail stays short;
//   3. autotuning: every tile configuration of the main kernel (density
//      matrices per ao_rhs tile x compacted AOs per stage) is timed on this
//      very problem and the fastest kept; results are cached on disk
//      (CFGMM_AUTOTUNE_CACHE, default $HOME/.cache/cfgmm/autotune.txt) under a
//      key made of the problem's size classes;
//   4. the run -- counter reset, persistent kernel, reduction -- is captured
//      in a CUDA graph, so a run is one graph launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/cfgmm.h"
#include "aodmao2rho_fp64.cuh"
#include "aodmao2rho_split.cuh"

namespace cfgmm {
void set_last_error(const std::string& msg);
}

struct cfgmm_aodm_plan {
  int dev = 0;
  bool split = false;
  cfgmm::AodmArgs args{};
  cfgmm::AodmConfig cfg{1, 32};
  // split precision: D digits are rebuilt every run, phi digits once here
  cfgmm::SplitArgs sargs{};
  // the pair form of split precision (two alike block tiles per item)
  bool pair = false;
  int nsl = 7;
  cfgmm::PairArgs pargs{};
  int* d_npairs = nullptr;  // device: the plan's pair count (the reduction's grid bound)
  const double* dms = nullptr;
  size_t stride_ao = 0;
  int nao = 0, nset_max = 0, stages = 0;
  int npairs = 0, nitems = 0;
  double flops = 0.0;   // sum_batches sum_s sum_b (2|I_b|^2 + 2|I_b|)|b| per run
  void* mem = nullptr;  // one device allocation for lists, descriptors, work list, partials
  void* mem2 = nullptr;  // split precision: digits, scales, its work list and partials
  void* mem3 = nullptr;  // pair form: the partial sums
  int2* rpairs = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::string info;
};

namespace {

int fail(int status, const std::string& msg) {
  cfgmm::set_last_error(msg);
  return status;
}

int cuda_fail(cudaError_t err, const char* where) {
  return fail(err == cudaErrorMemoryAllocation ? CFGMM_ERR_OUT_OF_MEMORY : CFGMM_ERR_CUDA,
              std::string(where) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) +
                  ")");
}

#define PLAN_CUDA(call)                                  \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

size_t a256(size_t v) { return (v + 255) / 256 * 256; }

// ---- autotune cache: one "key ns tk ms" line per entry -------------------
std::mutex g_cache_mu;

std::string cache_path() {
  if (const char* p = std::getenv("CFGMM_AUTOTUNE_CACHE")) return p;
  const char* home = std::getenv("HOME");
  return std::string(home ? home : "/tmp") + "/.cache/cfgmm/autotune.txt";
}

bool cache_lookup(const std::string& key, cfgmm::AodmConfig* cfg) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  FILE* f = std::fopen(cache_path().c_str(), "r");
  if (!f) return false;
  char k[256];
  int ns, tk;
  double ms;
  bool found = false;
  while (std::fscanf(f, "%255s %d %d %lf", k, &ns, &tk, &ms) == 4)
    if (key == k) {
      *cfg = cfgmm::AodmConfig{ns, tk};
      found = true;
    }
  std::fclose(f);
  return found;
}

void cache_store(const std::string& key, const cfgmm::AodmConfig& cfg, double ms) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  const std::string path = cache_path();
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos) {  // mkdir -p of the parent
    std::string dir;
    for (size_t i = 0; i <= slash; ++i) {
      dir += path[i];
      if (path[i] == '/' && i > 0) mkdir(dir.c_str(), 0755);
    }
  }
  if (FILE* f = std::fopen(path.c_str(), "a")) {
    std::fprintf(f, "%s %d %d %.6f\n", key.c_str(), cfg.ns, cfg.tk, ms);
    std::fclose(f);
  }
}

int bucket(double v) { return v <= 0 ? 0 : int(std::floor(std::log2(v) * 2)); }  // half-octaves


// D digits of a split-precision run, after the device-side symmetry check
// that selects the symmetric mode (sargs.asym, null when it is switched off).
cudaError_t split_prepare_run(cfgmm_aodm_plan* plan, cudaStream_t s) {
  const cfgmm::SplitArgs& a = plan->sargs;
  int* asym = const_cast<int*>(a.asym);
  cudaError_t err = cudaSuccess;
  if (asym) {
    err = cudaMemsetAsync(asym, 0, sizeof(int), s);
    if (err == cudaSuccess)
      err = cfgmm::aodm_launch_sym_check(plan->dms, plan->stride_ao, plan->nao, plan->nset_max,
                                         asym, s);
  }
  if (err == cudaSuccess)
    err = cfgmm::split_prepare_d(plan->dms, plan->stride_ao, plan->nao, plan->nset_max,
                                 const_cast<uint2*>(a.dsl), const_cast<int*>(a.tau), s, asym);
  return err;
}

// D digits of a pair-form run, after the symmetry check.
cudaError_t pair_prepare_run(cfgmm_aodm_plan* plan, cudaStream_t s) {
  const cfgmm::PairArgs& a = plan->pargs;
  int* asym = const_cast<int*>(a.asym);
  cudaError_t err = cudaSuccess;
  if (asym) err = cudaMemsetAsync(asym, 0, sizeof(int), s);
  if (err == cudaSuccess)
    err = cfgmm::split_pair_prepare_d(plan->dms, plan->stride_ao, plan->nao, plan->nset_max,
                                      plan->nsl, const_cast<uint2*>(a.dsl),
                                      const_cast<int*>(a.tau), const_cast<uint2*>(a.dhalf),
                                      asym, s);
  return err;
}

cudaError_t pair_run_on(cfgmm_aodm_plan* plan, cudaStream_t s) {
  cudaError_t err = cudaMemsetAsync(plan->pargs.counter, 0, sizeof(int), s);
  if (err == cudaSuccess) err = pair_prepare_run(plan, s);
  if (err == cudaSuccess)
    err = cfgmm::split_pair_launch_main(plan->pargs, plan->nsl, s, false, plan->stages);
  if (err == cudaSuccess)
    err = cfgmm::split_pair_launch_reduce(plan->pargs, plan->nsl, plan->d_npairs, 0, plan->npairs,
                                          s);
  return err;
}

// One split-precision run: D digits, the persistent kernel, the reduction.
int split_run(cfgmm_aodm_plan* plan, cudaStream_t s) {
  if (plan->pair) {
    const cudaError_t err = pair_run_on(plan, s);
    return err == cudaSuccess ? CFGMM_OK : cuda_fail(err, "split plan run");
  }
  cudaError_t err = split_prepare_run(plan, s);
  if (err == cudaSuccess) err = cfgmm::split_launch_main(plan->sargs, s, plan->stages);
  if (err == cudaSuccess)
    err = cfgmm::split_launch_reduce(plan->sargs, plan->rpairs, plan->npairs, s);
  return err == cudaSuccess ? CFGMM_OK : cuda_fail(err, "split plan run");
}

// Captures `body` (launches on the given stream) into plan->exec.
template <class F>
cudaError_t capture(cfgmm_aodm_plan* plan, F body) {
  cudaStream_t cs;
  cudaError_t err = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (err != cudaSuccess) return err;
  cudaGraph_t graph = nullptr;
  err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (err == cudaSuccess) {
    const cudaError_t e1 = body(cs);
    err = cudaStreamEndCapture(cs, &graph);
    if (err == cudaSuccess) err = e1;
  }
  if (err == cudaSuccess) err = cudaGraphInstantiate(&plan->exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  cudaStreamDestroy(cs);
  return err;
}

// The split-precision half of cfgmm_aodm_plan_create: phi digit tiles of
// every batch are built here once; items are (tile, row tile, matrix, batch),
// matrix-major (one D in L2 at a time), heaviest first within a matrix.
// Whether every batch passes one phi array for both sides of the contraction.
bool same_phi(const cfgmm_aodm_batch* batches, size_t nbatch) {
  for (size_t i = 0; i < nbatch; ++i)
    if (batches[i].ao_lhs != batches[i].ao_rhs) return false;
  return true;
}

int build_split(cfgmm_aodm_plan* plan, const cfgmm_aodm_batch* batches, size_t nbatch,
                const double* dms, size_t stride_ao, size_t nao, size_t nset_max, size_t blksize,
                int flags, int* d_lists, int* d_counts, const std::vector<size_t>& list_off,
                const std::vector<size_t>& cnt_off, const std::vector<size_t>& nblk,
                const std::vector<int>& counts, cudaStream_t s) {
  const int TU = cfgmm::split_row_tile(), TG = cfgmm::split_point_tile(), TK = cfgmm::split_chunk();
  const int gsub = int((blksize + TG - 1) / TG);
  const int max_ut = int((nao + TU - 1) / TU);
  const int parts = cfgmm::split_epi_parts();
  std::vector<int> cbase;
  std::vector<size_t> cb_off(nbatch), sg_off(nbatch);
  std::vector<cfgmm::SplitBatch> hb(nbatch);
  std::vector<int4> items;
  std::vector<int2> pairs;
  size_t ngrid_max = 0, sg_n = 0;
  long long groups = 0;
  int chunks = 0;
  for (size_t i = 0; i < nbatch; ++i) {
    const cfgmm_aodm_batch& b = batches[i];
    ngrid_max = std::max(ngrid_max, size_t(b.ngrid));
    cb_off[i] = cbase.size();
    sg_off[i] = sg_n;
    sg_n += (b.ngrid + 63) / 64 * 64;
    for (size_t blk = 0; blk < nblk[i]; ++blk) {
      const int nb = counts[cnt_off[i] + blk];
      for (int gt = 0; gt < gsub; ++gt) {
        cbase.push_back(chunks);
        chunks += (nb + TK - 1) / TK;
        if (nb > 0) pairs.push_back(make_int2(int(i), int(blk) * gsub + gt));
      }
    }
    hb[i].partial_off = groups;
    groups += (long long)(nblk[i] * gsub) * max_ut * (long long)b.nset * parts;
  }
  for (size_t sidx = 0; sidx < nset_max; ++sidx) {
    const size_t first = items.size();
    for (size_t i = 0; i < nbatch; ++i) {
      if (batches[i].nset <= sidx) continue;
      for (size_t blk = 0; blk < nblk[i]; ++blk) {
        const int nb = counts[cnt_off[i] + blk];
        for (int gt = 0; gt < gsub; ++gt)
          for (int u = 0; u * TU < nb; ++u)
            items.push_back(make_int4(int(blk) * gsub + gt, u, int(sidx), int(i)));
      }
    }
    // heaviest first: chunks of the tile's block
    std::stable_sort(items.begin() + first, items.end(), [&](const int4& x, const int4& y) {
      return counts[cnt_off[x.w] + x.x / gsub] > counts[cnt_off[y.w] + y.x / gsub];
    });
  }
  plan->nitems = int(items.size());
  plan->npairs = int(pairs.size());

  // ---- device memory ----
  const size_t o_cbase = 0;
  const size_t o_sigma = o_cbase + a256(std::max<size_t>(cbase.size(), 1) * sizeof(int));
  const size_t o_pmax = o_sigma + a256(std::max<size_t>(sg_n, 1) * sizeof(int));
  const size_t o_dsl = o_pmax + a256(ngrid_max * sizeof(unsigned long long));
  const size_t o_tau = o_dsl + a256(nset_max * nao * nao * 8);
  const size_t o_batch = o_tau + a256(nset_max * nao * sizeof(int));
  const size_t o_items = o_batch + a256(nbatch * sizeof(cfgmm::SplitBatch));
  const size_t o_total = o_items + a256(std::max<size_t>(items.size(), 1) * sizeof(int4));
  const size_t o_pairs = o_total + 256;
  const size_t o_phisl = o_pairs + a256(std::max<size_t>(pairs.size(), 1) * sizeof(int2));
  const size_t o_part = o_phisl + a256(size_t(chunks) * cfgmm::split_chunk_bytes());
  const size_t bytes = o_part + size_t(groups) * TG * sizeof(double);
  cudaError_t err = cudaMallocAsync(&plan->mem2, bytes, s);
  if (err != cudaSuccess) return cuda_fail(err, "cudaMalloc(split plan)");
  char* base = static_cast<char*>(plan->mem2);
  int* d_cbase = reinterpret_cast<int*>(base + o_cbase);
  int* d_sigma = reinterpret_cast<int*>(base + o_sigma);
  auto* d_pmax = reinterpret_cast<unsigned long long*>(base + o_pmax);
  uint8_t* d_phisl = reinterpret_cast<uint8_t*>(base + o_phisl);
  for (size_t i = 0; i < nbatch; ++i) {
    const cfgmm_aodm_batch& b = batches[i];
    hb[i].ao_lhs = b.ao_lhs;
    hb[i].rhos = b.rhos;
    hb[i].lists = d_lists + list_off[i];
    hb[i].counts = d_counts + cnt_off[i];
    hb[i].cbase = d_cbase + cb_off[i];
    hb[i].sigma = d_sigma + sg_off[i];
    hb[i].stride_grid = b.stride_grid;
    hb[i].ngrid = int(b.ngrid);
    hb[i].nset = int(b.nset);
  }
  const int total[2] = {int(items.size()), int(items.size())};
  err = cudaMemcpyAsync(d_cbase, cbase.data(), cbase.size() * sizeof(int), cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(base + o_batch, hb.data(), nbatch * sizeof(cfgmm::SplitBatch),
                          cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess && !items.empty())
    err = cudaMemcpyAsync(base + o_items, items.data(), items.size() * sizeof(int4),
                          cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(base + o_total, total, sizeof(total), cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess && !pairs.empty())
    err = cudaMemcpyAsync(base + o_pairs, pairs.data(), pairs.size() * sizeof(int2),
                          cudaMemcpyHostToDevice, s);
  // phi digit tiles of every batch, once
  for (size_t i = 0; i < nbatch && err == cudaSuccess; ++i)
    err = cfgmm::split_prepare_phi(batches[i].ao_rhs, batches[i].stride_grid, hb[i].lists,
                                   hb[i].counts, hb[i].cbase, int(nao), int(batches[i].ngrid),
                                   int(blksize), d_pmax, const_cast<int*>(hb[i].sigma), d_phisl, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);  // host vectors die on return
  if (err != cudaSuccess) return cuda_fail(err, "split plan setup");

  plan->split = true;
  plan->dms = dms;
  plan->stride_ao = stride_ao;
  plan->nao = int(nao);
  plan->nset_max = int(nset_max);
  plan->rpairs = reinterpret_cast<int2*>(base + o_pairs);
  cfgmm::SplitArgs& a = plan->sargs;
  a.dsl = reinterpret_cast<const uint2*>(base + o_dsl);
  a.tau = reinterpret_cast<const int*>(base + o_tau);
  a.phisl = d_phisl;
  a.batches = reinterpret_cast<const cfgmm::SplitBatch*>(base + o_batch);
  a.items = reinterpret_cast<const int4*>(base + o_items);
  a.total = reinterpret_cast<const int*>(base + o_total);
  a.partial = reinterpret_cast<double*>(base + o_part);
  a.nao = int(nao);
  a.blk = int(blksize);
  a.gsub = gsub;
  a.max_ut = max_ut;
  // total[2]: the asymmetry flag of the symmetric mode, which also needs every
  // batch to use one phi array for both sides
  a.asym = cfgmm::aodm_sym_enabled() && same_phi(batches, nbatch)
               ? reinterpret_cast<const int*>(base + o_total) + 2
               : nullptr;

  // ---- autotuning: pipeline depth of the persistent kernel ----
  std::string tune = "default";
  char key[256];
  double work = 0.0;
  for (size_t i = 0; i < nbatch; ++i)
    for (size_t blk = 0; blk < nblk[i]; ++blk) {
      const double nb = counts[cnt_off[i] + blk];
      work += double(batches[i].nset) * nb * nb;
    }
  std::snprintf(key, sizeof(key), "aodm_split:nao%d:work%d:items%d:nset%zu:blk%zu",
                bucket(double(nao)), bucket(work), bucket(double(plan->nitems)), nset_max, blksize);
  if (!(flags & CFGMM_PLAN_NO_TUNE) && plan->nitems > 0) {
    cfgmm::AodmConfig c{};
    if (cache_lookup(key, &c)) {
      plan->stages = c.ns;
      tune = "cache";
    } else {
      if ((err = split_prepare_run(plan, s)) != cudaSuccess) return cuda_fail(err, "autotune");
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      double best_ms = 1e30;
      std::string trials;
      const int st0 = cfgmm::split_min_stages();
      for (int st : {st0, st0 + 1, st0 + 2}) {
        float best = 1e30f;
        for (int rep = 0; rep < 3 && err == cudaSuccess; ++rep) {
          err = cudaEventRecord(e0, s);
          if (err == cudaSuccess) err = cfgmm::split_launch_main(a, s, st);
          if (err == cudaSuccess) err = cudaEventRecord(e1, s);
          if (err == cudaSuccess) err = cudaEventSynchronize(e1);
          float t = 0.f;
          if (err == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
          if (rep > 0) best = std::min(best, t);
        }
        if (err != cudaSuccess) break;
        char buf[96];
        std::snprintf(buf, sizeof(buf), "%s{\"stages\":%d,\"ms\":%.4f}", trials.empty() ? "" : ",",
                      st, best);
        trials += buf;
        if (best < best_ms) {
          best_ms = best;
          plan->stages = st;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      if (err != cudaSuccess) return cuda_fail(err, "autotune");
      cache_store(key, cfgmm::AodmConfig{plan->stages, 0}, best_ms);
      tune = "[" + trials + "]";
    }
  }

  // ---- capture the run ----
  if (!(flags & CFGMM_PLAN_NO_GRAPH)) {
    // kernel attributes are set outside the capture
    err = cfgmm::split_launch_main(a, s, plan->stages, true);
    if (err == cudaSuccess)
      err = capture(plan, [&](cudaStream_t cs) {
        cudaError_t e = split_prepare_run(plan, cs);
        if (e == cudaSuccess) e = cfgmm::split_launch_main(a, cs, plan->stages);
        if (e == cudaSuccess) e = cfgmm::split_launch_reduce(a, plan->rpairs, plan->npairs, cs);
        return e;
      });
    if (err != cudaSuccess) return cuda_fail(err, "graph capture");
  }
  char buf[512];
  std::snprintf(buf, sizeof(buf),
                "{\"precision\":\"split\",\"batches\":%zu,\"items\":%d,\"block_tiles\":%d,"
                "\"phi_chunks\":%d,\"flops\":%.6e,\"config\":{\"stages\":%d},\"graph\":%s,"
                "\"tuning\":",
                nbatch, plan->nitems, plan->npairs, chunks, plan->flops, plan->stages,
                plan->exec ? "true" : "false");
  plan->info = std::string(buf) + (tune[0] == '[' ? tune : "\"" + tune + "\"") + ",\"key\":\"" +
               key + "\"}";
  return CFGMM_OK;
}

// The pair form of the split-precision plan: every batch's pairing, unions,
// work list and phi digit tiles are built once here on the device (batch by
// batch, the host reading each batch's pair and chunk counts to place the
// next), then the work list is ordered matrix by matrix, heaviest first, and
// the run (D digits, persistent kernel, reduction) is captured in a graph.
// Per batch the result equals the single call's bit for bit: the same pairs,
// unions, tiles and fixed-order sums.
int build_split_pair(cfgmm_aodm_plan* plan, const cfgmm_aodm_batch* batches, size_t nbatch,
                     const double* dms, size_t stride_ao, size_t nao, size_t nset_max,
                     size_t blksize, int flags, int* d_lists, int* d_counts,
                     const std::vector<size_t>& list_off, const std::vector<size_t>& cnt_off,
                     const std::vector<size_t>& nblk, const std::vector<int>& counts,
                     cudaStream_t s) {
  const int nsl = cfgmm::split_pair_digits();
  const int tn = cfgmm::split_pair_row_tile(nsl);
  constexpr int HT = 64, TK = 32, PT = 128, WIN2 = 64;
  const int gsub = int((blksize + HT - 1) / HT);
  const size_t nwords = (nao + 31) / 32;
  const size_t a_stage = size_t(nsl) * PT * TK;
  size_t nbg_tot = 0, nbg_max = 0, ngrid_max = 0, sg_n = 0, chunk_bound = 0, item_bound = 0;
  size_t row_bound = 0;  // partial row tiles of all pairs, at most
  double work = 0.0;     // the autotune key's work: sum over the block tiles of |I|^2
  std::vector<size_t> sg_off(nbatch);
  for (size_t i = 0; i < nbatch; ++i) {
    const size_t nbg = nblk[i] * gsub;
    nbg_tot += nbg;
    nbg_max = std::max(nbg_max, nbg);
    ngrid_max = std::max(ngrid_max, size_t(batches[i].ngrid));
    sg_off[i] = sg_n;
    sg_n += (batches[i].ngrid + 63) / 64 * 64;
    for (size_t b = 0; b < nblk[i]; ++b) {
      const size_t nb = size_t(counts[cnt_off[i] + b]);
      // |U| <= |I_a| + |I_b|: a pair's chunks and row tiles are bounded by its tiles'
      chunk_bound += gsub * ((nb + TK - 1) / TK);
      item_bound += gsub * ((nb + tn - 1) / tn) * batches[i].nset;
      row_bound += gsub * ((nb + tn - 1) / tn);
      work += double(gsub) * double(nb) * double(nb);
    }
  }
  // ---- device memory (the partial sums follow once the pairs are known) ----
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t off = o;
    o += a256(std::max<size_t>(bytes, 1));
    return off;
  };
  const size_t o_bits = take(nbg_max * nwords * 4), o_cnt = take(nbg_max * 4),
               o_key = take(nbg_max * 8), o_order = take(nbg_max * 4),
               o_cand = take(nbg_max * WIN2 * 4), o_ncand = take(nbg_max * 4),
               o_partner = take(nbg_max * 4), o_pos = take(nbg_max * 4),
               o_choice = take(nbg_max * 4), o_pmax = take(ngrid_max * 8),
               o_cpair = take(nbg_max * ((nao + 31) / 32) * 4),
               o_pairs = take(nbg_tot * sizeof(int4)), o_np = take(8),
               o_ulist = take(nbg_tot * nao * 4), o_uflag = take(nbg_tot * nao),
               o_ucount = take(nbg_tot * 4), o_cbase = take((nbg_tot + 1) * 4),
               o_poff = take((nbg_tot + 1) * 4), o_items = take(item_bound * sizeof(int4)),
               o_total = take(16), o_sigma = take(sg_n * 4),
               o_dsl = take(nset_max * nao * nao * 8), o_tau = take(nset_max * nao * 4),
               o_dhalf = take(nset_max * nao * 8),
               o_batch = take(nbatch * sizeof(cfgmm::PairBatch)),
               o_phisl = take(chunk_bound * a_stage);
  cudaError_t err = cudaMallocAsync(&plan->mem2, o, s);
  if (err != cudaSuccess) return cuda_fail(err, "cudaMalloc(split plan)");
  char* base = static_cast<char*>(plan->mem2);
  auto at = [&](size_t off) { return static_cast<void*>(base + off); };
  int* d_np = static_cast<int*>(at(o_np));
  int* d_total = static_cast<int*>(at(o_total));
  err = cudaMemsetAsync(d_total, 0, 16, s);

  std::vector<cfgmm::PairBatch> hb(nbatch);
  int pair0 = 0, chunk0 = 0;
  for (size_t i = 0; i < nbatch && err == cudaSuccess; ++i) {
    const cfgmm_aodm_batch& b = batches[i];
    cfgmm::PairPrep q{};
    q.tab = b.tab;
    q.ldtab = b.ldtab;
    q.ao_rhs = b.ao_rhs;
    q.stride_grid = b.stride_grid;
    q.nao = int(nao);
    q.ngrid = int(b.ngrid);
    q.blk = int(blksize);
    q.nset = int(b.nset);
    q.nsl = nsl;
    q.batch = int(i);
    q.pair0 = pair0;
    q.chunk0 = chunk0;
    q.lists = d_lists + list_off[i];
    q.counts = d_counts + cnt_off[i];
    q.bits = static_cast<uint32_t*>(at(o_bits));
    q.cnt = static_cast<int*>(at(o_cnt));
    q.key = static_cast<unsigned long long*>(at(o_key));
    q.order = static_cast<int*>(at(o_order));
    q.cand = static_cast<int*>(at(o_cand));
    q.ncand = static_cast<int*>(at(o_ncand));
    q.partner = static_cast<int*>(at(o_partner));
    q.pos = static_cast<int*>(at(o_pos));
    q.choice = static_cast<int*>(at(o_choice));
    q.pairs = static_cast<int4*>(at(o_pairs));
    q.npairs = d_np + 1;  // this batch's count, read back below
    q.ulist = static_cast<int*>(at(o_ulist));
    q.uflag = static_cast<uint8_t*>(at(o_uflag));
    q.ucount = static_cast<int*>(at(o_ucount));
    q.cbase = static_cast<int*>(at(o_cbase));
    q.cpair = static_cast<int*>(at(o_cpair));
    q.items = static_cast<int4*>(at(o_items));
    q.total = d_total;
    q.chunks_end = d_total + 2;
    q.sigma = static_cast<int*>(at(o_sigma)) + sg_off[i];
    q.pmax = static_cast<unsigned long long*>(at(o_pmax));
    q.phisl = static_cast<uint8_t*>(at(o_phisl));
    err = cfgmm::split_pair_prepare_batch(q, s);
    if (nbatch > 1) {  // the next batch's pairs and chunks follow this one's
      int got[2] = {0, 0};
      if (err == cudaSuccess)
        err = cudaMemcpyAsync(&got[0], d_np + 1, 4, cudaMemcpyDeviceToHost, s);
      if (err == cudaSuccess)
        err = cudaMemcpyAsync(&got[1], d_total + 2, 4, cudaMemcpyDeviceToHost, s);
      if (err == cudaSuccess) err = cudaStreamSynchronize(s);
      pair0 += got[0];
      chunk0 = got[1];
    }
    hb[i] = cfgmm::PairBatch{b.ao_lhs, b.rhos, q.sigma, b.stride_grid, int(b.ngrid), int(b.nset)};
  }
  if (err != cudaSuccess) return cuda_fail(err, "split plan setup");
  int P = pair0, nitems = 0;
  if (nbatch == 1) {
    // One batch (a server molecule): the work list stays in the device's
    // order (pair-major, heaviest pairs first by chunk count), the partial
    // offsets come from a device scan and the partial sums from the host
    // bound -- no host round trip, so a plan builds without waiting for the
    // device.  Counts reported below are bounds.
    P = int(nbg_tot);
    nitems = int(item_bound);
    const size_t part_bytes =
        row_bound * nset_max * cfgmm::split_pair_partial_points() * sizeof(double);
    err = cudaMallocAsync(&plan->mem3, std::max<size_t>(part_bytes, 256), s);
    if (err != cudaSuccess) return cuda_fail(err, "cudaMalloc(split plan partials)");
    err = cudaMemcpyAsync(d_np, d_np + 1, 4, cudaMemcpyDeviceToDevice, s);
    if (err == cudaSuccess)
      err = cfgmm::split_pair_partial_offsets(static_cast<const int*>(at(o_ucount)), d_np, tn,
                                              static_cast<int*>(at(o_poff)), s);
    if (err != cudaSuccess) return cuda_fail(err, "split plan work list");
  } else {
    if (size_t(chunk0) > chunk_bound) return fail(CFGMM_ERR_CUDA, "split plan: chunk bound exceeded");
    // ---- work list: pair-major (a pair's phi tiles and D rows shared in L2 by
    // the CTAs running at one time), heaviest pairs first ----
    err = cudaMemcpyAsync(&nitems, d_total, 4, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_fail(err, "split plan work list");
    if (size_t(nitems) > item_bound) return fail(CFGMM_ERR_CUDA, "split plan: item bound exceeded");
    std::vector<int4> items(size_t(std::max(nitems, 0)));
    std::vector<int> ucount(size_t(std::max(P, 1)));
    if (err == cudaSuccess && nitems > 0)
      err = cudaMemcpyAsync(items.data(), at(o_items), size_t(nitems) * sizeof(int4),
                            cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess && P > 0)
      err = cudaMemcpyAsync(ucount.data(), at(o_ucount), size_t(P) * 4, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_fail(err, "split plan work list");
    std::stable_sort(items.begin(), items.end(), [&](const int4& x, const int4& y) {
      const int kx = (ucount[x.x] + TK - 1) / TK, ky = (ucount[y.x] + TK - 1) / TK;
      if (kx != ky) return kx > ky;
      if (x.x != y.x) return x.x < y.x;
      if (x.y != y.y) return x.y < y.y;
      return x.z < y.z;
    });
    // partial row tiles: exact, from the unions
    std::vector<int> poff(size_t(P) + 1, 0);
    for (int q = 0; q < P; ++q) poff[q + 1] = poff[q] + (ucount[q] + tn - 1) / tn;
    const size_t part_bytes =
        size_t(poff[P]) * nset_max * cfgmm::split_pair_partial_points() * sizeof(double);
    err = cudaMallocAsync(&plan->mem3, std::max<size_t>(part_bytes, 256), s);
    if (err != cudaSuccess) return cuda_fail(err, "cudaMalloc(split plan partials)");
    const int np_all = P;
    if (nitems > 0)
      err = cudaMemcpyAsync(at(o_items), items.data(), size_t(nitems) * sizeof(int4),
                            cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(at(o_poff), poff.data(), poff.size() * 4, cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess) err = cudaMemcpyAsync(d_np, &np_all, 4, cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(at(o_batch), hb.data(), nbatch * sizeof(cfgmm::PairBatch),
                            cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);  // host vectors die on return
    if (err != cudaSuccess) return cuda_fail(err, "split plan upload");
  }

  plan->split = true;
  plan->pair = true;
  plan->nsl = nsl;
  plan->dms = dms;
  plan->stride_ao = stride_ao;
  plan->nao = int(nao);
  plan->nset_max = int(nset_max);
  plan->nitems = nitems;
  plan->npairs = P;
  plan->d_npairs = d_np;
  cfgmm::PairArgs& a = plan->pargs;
  a.dsl = static_cast<const uint2*>(at(o_dsl));
  a.tau = static_cast<const int*>(at(o_tau));
  a.dhalf = static_cast<const uint2*>(at(o_dhalf));
  a.phisl = static_cast<const uint8_t*>(at(o_phisl));
  a.items = static_cast<const int4*>(at(o_items));
  a.total = d_total;
  a.pairs = static_cast<const int4*>(at(o_pairs));
  a.ucount = static_cast<const int*>(at(o_ucount));
  a.ulist = static_cast<const int*>(at(o_ulist));
  a.uflag = static_cast<const uint8_t*>(at(o_uflag));
  a.cbase = static_cast<const int*>(at(o_cbase));
  a.batches = nbatch == 1 ? nullptr : static_cast<const cfgmm::PairBatch*>(at(o_batch));
  a.one = hb[0];
  a.partial = static_cast<double*>(plan->mem3);
  a.poff = static_cast<const int*>(at(o_poff));
  a.nao = int(nao);
  a.blk = int(blksize);
  a.gsub = gsub;
  a.max_t = int((nao + tn - 1) / tn);
  a.nset_max = int(nset_max);
  a.counter = d_total + 3;
  a.wait_ns = 0;  // the default bound
  a.inject = 0;
  // total[1]: the asymmetry flag (the half contraction also needs one phi array per batch)
  a.asym = cfgmm::aodm_sym_enabled() && same_phi(batches, nbatch) ? d_total + 1 : nullptr;

  // ---- autotuning: pipeline depth of the persistent kernel ----
  std::string tune = "default";
  char key[256];
  std::snprintf(key, sizeof(key), "aodm_split_pair%d:nao%d:work%d:items%d:nset%zu:blk%zu", nsl,
                bucket(double(nao)), bucket(work), bucket(double(nitems)), nset_max, blksize);
  plan->stages = 0;
  if (!(flags & CFGMM_PLAN_NO_TUNE) && nitems > 0) {
    cfgmm::AodmConfig c{};
    if (cache_lookup(key, &c)) {
      plan->stages = c.ns;
      tune = "cache";
    } else {
      if ((err = pair_prepare_run(plan, s)) != cudaSuccess) return cuda_fail(err, "autotune");
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      double best_ms = 1e30;
      std::string trials;
      for (int st : {cfgmm::split_pair_stages()}) {
        float best = 1e30f;
        for (int rep = 0; rep < 3 && err == cudaSuccess; ++rep) {
          err = cudaMemsetAsync(a.counter, 0, sizeof(int), s);
          if (err == cudaSuccess) err = cudaEventRecord(e0, s);
          if (err == cudaSuccess) err = cfgmm::split_pair_launch_main(a, nsl, s, false, st);
          if (err == cudaSuccess) err = cudaEventRecord(e1, s);
          if (err == cudaSuccess) err = cudaEventSynchronize(e1);
          float t = 0.f;
          if (err == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
          if (rep > 0) best = std::min(best, t);
        }
        if (err != cudaSuccess) break;
        char tb[96];
        std::snprintf(tb, sizeof(tb), "%s{\"stages\":%d,\"ms\":%.4f}", trials.empty() ? "" : ",",
                      st, best);
        trials += tb;
        if (best < best_ms) {
          best_ms = best;
          plan->stages = st;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      if (err != cudaSuccess) return cuda_fail(err, "autotune");
      cache_store(key, cfgmm::AodmConfig{plan->stages, 0}, best_ms);
      tune = "[" + trials + "]";
    }
  }

  // ---- capture the run ----
  if (!(flags & CFGMM_PLAN_NO_GRAPH)) {
    // attributes outside the capture
    err = cfgmm::split_pair_launch_main(a, nsl, s, true, plan->stages);
    if (err == cudaSuccess)
      err = capture(plan, [&](cudaStream_t cs) { return pair_run_on(plan, cs); });
    if (err != cudaSuccess) return cuda_fail(err, "graph capture");
  }
  char buf[512];
  std::snprintf(buf, sizeof(buf),
                "{\"precision\":\"split\",\"form\":\"pair\",\"digits\":%d,\"batches\":%zu,"
                "\"items\":%d,\"block_tiles\":%zu,\"pairs\":%d,\"phi_chunks\":%d,"
                "\"counts\":\"%s\",\"flops\":%.6e,\"config\":{\"row_tile\":%d,\"stages\":%d},"
                "\"graph\":%s,\"tuning\":",
                nsl, nbatch, nitems, nbg_tot, P, nbatch == 1 ? int(chunk_bound) : chunk0,
                nbatch == 1 ? "bounds" : "exact", plan->flops, tn, plan->stages,
                plan->exec ? "true" : "false");
  plan->info = std::string(buf) + (tune[0] == '[' ? tune : "\"" + tune + "\"") + ",\"key\":\"" +
               key + "\"}";
  return CFGMM_OK;
}

}  // namespace

extern "C" {

int cfgmm_aodm_plan_create(cfgmm_aodm_plan** out, const cfgmm_aodm_batch* batches, size_t nbatch,
                           const double* dms, size_t stride_ao, size_t nao, size_t nset_max,
                           size_t blksize, int precision, int flags, void* stream) {
  cfgmm::set_last_error("");
  if (!out) return fail(CFGMM_ERR_INVALID_ARGUMENT, "null plan pointer");
  *out = nullptr;
  if (precision != CFGMM_PREC_FP64 && precision != CFGMM_PREC_OZAKI_INT8)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "unknown precision " + std::to_string(precision));
  if (precision == CFGMM_PREC_OZAKI_INT8 && nao > 16384)
    return fail(CFGMM_ERR_UNIMPLEMENTED, "split-precision AO-DM-AO supports nao <= 16384");
  if (!batches || nbatch == 0 || !dms || nao == 0 || nset_max == 0 || blksize == 0)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "empty plan or null pointer");
  if (nao > 1000000 || nset_max > 1024 || blksize > 1000000 || nbatch > 1000000)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "plan dimensions out of range");
  for (size_t i = 0; i < nbatch; ++i) {
    const cfgmm_aodm_batch& b = batches[i];
    if (!b.rhos || !b.ao_lhs || !b.ao_rhs || !b.tab || b.nset == 0 || b.nset > nset_max ||
        b.stride_grid < b.ngrid || b.ngrid == 0 || b.ngrid > 0x7fff0000u ||
        b.ldtab < (b.ngrid + blksize - 1) / blksize)
      return fail(CFGMM_ERR_INVALID_ARGUMENT, "invalid batch " + std::to_string(i));
  }
  int dev = 0, ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return fail(CFGMM_ERR_NO_DEVICE, "no CUDA device");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cfgmm_aodm_plan* plan = new cfgmm_aodm_plan;
  plan->dev = dev;
  auto cleanup = [&](int rc) {
    if (plan->mem) cudaFree(plan->mem);
    if (plan->mem2) cudaFree(plan->mem2);
    if (plan->mem3) cudaFree(plan->mem3);
    delete plan;
    return rc;
  };
  const int TU = cfgmm::aodm_row_tile(), TG = cfgmm::aodm_point_tile();
  const int gsub = int((blksize + TG - 1) / TG);
  const int max_ut = int((nao + TU - 1) / TU);

  // ---- layout of the plan's device memory ----
  std::vector<size_t> nblk(nbatch), list_off(nbatch), cnt_off(nbatch);
  size_t lists_n = 0, cnt_n = 0;
  for (size_t i = 0; i < nbatch; ++i) {
    nblk[i] = (batches[i].ngrid + blksize - 1) / blksize;
    list_off[i] = lists_n;
    cnt_off[i] = cnt_n;
    lists_n += nblk[i] * nao;
    cnt_n += nblk[i];
  }
  const size_t slots = cnt_n * gsub * max_ut;
  const size_t o_lists = 0;
  const size_t o_counts = o_lists + a256(lists_n * sizeof(int));
  const size_t o_batch = o_counts + a256(cnt_n * sizeof(int));
  const size_t o_items = o_batch + a256(nbatch * sizeof(cfgmm::AodmBatch));
  const size_t o_pairs = o_items + a256(slots * sizeof(int4));
  const size_t o_ctr = o_pairs + a256(cnt_n * gsub * sizeof(int2));
  const size_t o_part = o_ctr + a256((nset_max + 2) * sizeof(int));  // + total, asymmetry flag
  const size_t o_maps = o_part + a256(slots * nset_max * TG * sizeof(double));
  // split precision keeps only the active lists here (its own layout follows)
  const size_t bytes = precision == CFGMM_PREC_OZAKI_INT8
                           ? o_batch
                           : o_maps + nbatch * sizeof(CUtensorMap);
  cudaError_t err = cudaMallocAsync(&plan->mem, bytes, s);
  if (err != cudaSuccess) return cleanup(cuda_fail(err, "cudaMalloc(plan)"));
  char* base = static_cast<char*>(plan->mem);
  int* d_lists = reinterpret_cast<int*>(base + o_lists);
  int* d_counts = reinterpret_cast<int*>(base + o_counts);

  // ---- 1. active lists of every batch ----
  for (size_t i = 0; i < nbatch; ++i) {
    err = cfgmm::aodm_block_lists_launch(batches[i].tab, batches[i].ldtab, int(nao), int(nblk[i]),
                                         d_lists + list_off[i], d_counts + cnt_off[i], s);
    if (err != cudaSuccess) return cleanup(cuda_fail(err, "active lists"));
  }
  std::vector<int> counts(cnt_n);
  err = cudaMemcpyAsync(counts.data(), d_counts, cnt_n * sizeof(int), cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return cleanup(cuda_fail(err, "active list counts"));

  for (size_t i = 0; i < nbatch; ++i)
    for (size_t blk = 0; blk < nblk[i]; ++blk) {
      const double nb = counts[cnt_off[i] + blk];
      const double w = double(std::min(blksize, batches[i].ngrid - blk * blksize));
      plan->flops += double(batches[i].nset) * (2.0 * nb * nb + 2.0 * nb) * w;
    }
  if (precision == CFGMM_PREC_OZAKI_INT8) {
    size_t points = 0;
    for (size_t i = 0; i < nbatch; ++i) points += batches[i].ngrid;
    const int rc =
        cfgmm::split_pair_form(nao, points)
            ? build_split_pair(plan, batches, nbatch, dms, stride_ao, nao, nset_max, blksize,
                               flags, d_lists, d_counts, list_off, cnt_off, nblk, counts, s)
            : build_split(plan, batches, nbatch, dms, stride_ao, nao, nset_max, blksize, flags,
                          d_lists, d_counts, list_off, cnt_off, nblk, counts, s);
    if (rc != CFGMM_OK) return cleanup(rc);
    *out = plan;
    return CFGMM_OK;
  }

  // ---- 2. descriptors and the global work list, heaviest first ----
  std::vector<cfgmm::AodmBatch> hb(nbatch);
  std::vector<int4> items;
  std::vector<int2> pairs;
  long long slot = 0;
  double work = 0.0;
  for (size_t i = 0; i < nbatch; ++i) {
    const cfgmm_aodm_batch& b = batches[i];
    hb[i] = cfgmm::AodmBatch{b.ao_lhs, b.ao_rhs, b.rhos, d_lists + list_off[i],
                             d_counts + cnt_off[i], b.stride_grid, int(b.ngrid), int(b.nset), slot};
    for (size_t blk = 0; blk < nblk[i]; ++blk) {
      const int nb = counts[cnt_off[i] + blk];
      const int nt = (nb + TU - 1) / TU;
      for (int gt = 0; gt < gsub; ++gt) {
        const int bg = int(blk) * gsub + gt;
        if (nt > 0) pairs.push_back(make_int2(int(i), bg));
        for (int u = 0; u < nt; ++u) items.push_back(make_int4(int(i), bg, u, nb));
      }
      work += double(b.nset) * nb * nb;
    }
    slot += (long long)(nblk[i] * gsub * max_ut);
  }
  std::stable_sort(items.begin(), items.end(),
                   [](const int4& x, const int4& y) { return x.w > y.w; });
  // ao_rhs gather maps of the pipelined form (batches whose rows TMA cannot
  // address are gathered by cp.async)
  const bool pipe_ok = cfgmm::aodm_pipe_enabled();
  std::vector<CUtensorMap> maps(nbatch);
  std::memset(maps.data(), 0, nbatch * sizeof(CUtensorMap));
  for (size_t i = 0; i < nbatch && pipe_ok; ++i)
    hb[i].rhs_tma = cfgmm::aodm_rhs_map(&maps[i], batches[i].ao_rhs, batches[i].stride_grid,
                                        int(nao), int(batches[i].ngrid), int(blksize))
                        ? 1
                        : 0;
  plan->nitems = int(items.size());
  plan->npairs = int(pairs.size());
  plan->rpairs = reinterpret_cast<int2*>(base + o_pairs);
  err = cudaMemcpyAsync(base + o_batch, hb.data(), nbatch * sizeof(cfgmm::AodmBatch),
                        cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess && !items.empty())
    err = cudaMemcpyAsync(base + o_items, items.data(), items.size() * sizeof(int4),
                          cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess && !pairs.empty())
    err = cudaMemcpyAsync(plan->rpairs, pairs.data(), pairs.size() * sizeof(int2),
                          cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess && pipe_ok)
    err = cudaMemcpyAsync(base + o_maps, maps.data(), nbatch * sizeof(CUtensorMap),
                          cudaMemcpyHostToDevice, s);
  if (err != cudaSuccess) return cleanup(cuda_fail(err, "plan upload"));

  cfgmm::AodmArgs& a = plan->args;
  a.dms = dms;
  a.stride_ao = stride_ao;
  a.dm_stride = stride_ao * stride_ao;
  a.nao = int(nao);
  a.blk = int(blksize);
  a.gsub = gsub;
  a.max_utiles = max_ut;
  a.nset_max = int(nset_max);
  a.batches = reinterpret_cast<const cfgmm::AodmBatch*>(base + o_batch);
  a.rhs_maps = pipe_ok ? reinterpret_cast<const CUtensorMap*>(base + o_maps) : nullptr;
  a.items = reinterpret_cast<const int4*>(base + o_items);
  a.counters = reinterpret_cast<int*>(base + o_ctr);
  // the half contraction needs D = D^T and, in every batch, phi_lhs = phi_rhs
  const bool sym = pipe_ok && cfgmm::aodm_sym_enabled() && same_phi(batches, nbatch);
  // reset, symmetry check of D, main kernel (the reduction follows in a run)
  auto launch = [&](const cfgmm::AodmConfig& c, cudaStream_t st) -> cudaError_t {
    a.asym = sym && c.tk == 0 ? a.counters + a.ngroups + 1 : nullptr;
    cudaError_t e = cfgmm::aodm_launch_reset(a.counters, a.ngroups, st);
    if (e == cudaSuccess && a.asym)
      e = cfgmm::aodm_launch_sym_check(dms, stride_ao, int(nao), int(nset_max),
                                       a.counters + a.ngroups + 1, st);
    if (e == cudaSuccess) e = cfgmm::aodm_launch_main(a, c, st);
    return e;
  };
  a.partial = reinterpret_cast<double*>(base + o_part);

  // ---- 3. autotuning ----
  auto set_cfg = [&](const cfgmm::AodmConfig& c) -> cudaError_t {
    a.ngroups = cfgmm::aodm_groups(c, int(nset_max));
    std::vector<int> ctr(a.ngroups + 1, 0);
    ctr[a.ngroups] = plan->nitems;
    cudaError_t e = cudaMemcpyAsync(a.counters, ctr.data(), ctr.size() * sizeof(int),
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
  };
  auto time_cfg = [&](const cfgmm::AodmConfig& c, double* ms) -> cudaError_t {
    cudaError_t e = set_cfg(c);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
      e = cudaEventRecord(e0, s);
      if (e == cudaSuccess) e = launch(c, s);
      if (e == cudaSuccess) e = cudaEventRecord(e1, s);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float t = 0.f;
      if (e == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0) best = std::min(best, t);  // the first run warms up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = best;
    return e;
  };
  char key[256];
  std::snprintf(key, sizeof(key), "aodm_fp64%s:nao%d:work%d:items%d:nset%zu:blk%zu",
                pipe_ok ? "_pipe" : "", bucket(double(nao)), bucket(work),
                bucket(double(plan->nitems)), nset_max, blksize);
  std::string tune = "default";
  plan->cfg = cfgmm::aodm_default_config(int(nset_max));
  if (pipe_ok) plan->cfg.tk = 0;  // the pipelined form
  const std::vector<int> tks = pipe_ok ? std::vector<int>{0, 32, 16} : std::vector<int>{32, 16};
  if (!(flags & CFGMM_PLAN_NO_TUNE) && plan->nitems > 0) {
    if (cache_lookup(key, &plan->cfg)) {
      tune = "cache";
    } else {
      double best_ms = 1e30;
      std::string trials;
      for (int tk : tks)
        for (int ns = 1; ns <= 3 && ns <= int(nset_max); ++ns) {
          const cfgmm::AodmConfig c{ns, tk};
          double ms = 0;
          err = time_cfg(c, &ms);
          if (err != cudaSuccess) return cleanup(cuda_fail(err, "autotune"));
          char buf[96];
          std::snprintf(buf, sizeof(buf), "%s{\"ns\":%d,\"tk\":%d,\"ms\":%.4f}",
                        trials.empty() ? "" : ",", ns, tk, ms);
          trials += buf;
          if (ms < best_ms) {
            best_ms = ms;
            plan->cfg = c;
          }
        }
      cache_store(key, plan->cfg, best_ms);
      tune = "[" + trials + "]";
    }
  }
  if ((err = set_cfg(plan->cfg)) != cudaSuccess) return cleanup(cuda_fail(err, "plan config"));
  a.asym = sym && plan->cfg.tk == 0 ? a.counters + a.ngroups + 1 : nullptr;

  // ---- 4. capture the run ----
  if (!(flags & CFGMM_PLAN_NO_GRAPH)) {
    cudaStream_t cs;
    if ((err = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess)
      return cleanup(cuda_fail(err, "capture stream"));
    // kernel attributes are set outside the capture
    err = cfgmm::aodm_launch_main(a, plan->cfg, cs, true);
    cudaGraph_t graph = nullptr;
    if (err == cudaSuccess) err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
      cudaError_t e1 = launch(plan->cfg, cs);
      if (e1 == cudaSuccess) e1 = cfgmm::aodm_launch_reduce(a, plan->rpairs, plan->npairs, cs);
      err = cudaStreamEndCapture(cs, &graph);
      if (err == cudaSuccess) err = e1;
    }
    if (err == cudaSuccess) err = cudaGraphInstantiate(&plan->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    if (err != cudaSuccess) return cleanup(cuda_fail(err, "graph capture"));
  }
  char buf[512];
  std::snprintf(buf, sizeof(buf),
                "{\"precision\":\"fp64\",\"batches\":%zu,\"items\":%d,\"block_tiles\":%d,"
                "\"flops\":%.6e,\"config\":{\"ns\":%d,\"tk\":%d},\"graph\":%s,\"tuning\":",
                nbatch, plan->nitems, plan->npairs, plan->flops, plan->cfg.ns, plan->cfg.tk,
                plan->exec ? "true" : "false");
  plan->info = std::string(buf) + (tune[0] == '[' ? tune : "\"" + tune + "\"") + ",\"key\":\"" +
               key + "\"}";
  *out = plan;
  return CFGMM_OK;
}

int cfgmm_aodm_plan_run(cfgmm_aodm_plan* plan, void* stream) {
  cfgmm::set_last_error("");
  if (!plan) return fail(CFGMM_ERR_INVALID_ARGUMENT, "null plan");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (plan->exec) {
    PLAN_CUDA(cudaGraphLaunch(plan->exec, s));
    return CFGMM_OK;
  }
  if (plan->split) {
    const int rc = split_run(plan, s);
    return rc;
  }
  const cfgmm::AodmArgs& a = plan->args;
  PLAN_CUDA(cfgmm::aodm_launch_reset(a.counters, a.ngroups, s));
  if (a.asym)
    PLAN_CUDA(cfgmm::aodm_launch_sym_check(a.dms, a.stride_ao, a.nao, a.nset_max,
                                           a.counters + a.ngroups + 1, s));
  PLAN_CUDA(cfgmm::aodm_launch_main(plan->args, plan->cfg, s));
  PLAN_CUDA(cfgmm::aodm_launch_reduce(plan->args, plan->rpairs, plan->npairs, s));
  return CFGMM_OK;
}

const char* cfgmm_aodm_plan_info(const cfgmm_aodm_plan* plan) {
  return plan ? plan->info.c_str() : "";
}

int cfgmm_aodm_plan_destroy(cfgmm_aodm_plan* plan) {
  if (!plan) return CFGMM_OK;
  if (plan->exec) cudaGraphExecDestroy(plan->exec);
  // cudaFree waits for work still using the memory
  if (plan->mem) cudaFree(plan->mem);
  if (plan->mem2) cudaFree(plan->mem2);
  if (plan->mem3) cudaFree(plan->mem3);
  delete plan;
  return CFGMM_OK;
}

}  // extern "C"

namespace cfgmm {

// For owners that know the plan is idle (no run in flight): the memory goes
// back to the stream-ordered pool on `stream` without a device-wide wait.
int aodm_plan_release_idle(cfgmm_aodm_plan* plan, cudaStream_t stream) {
  if (!plan) return CFGMM_OK;
  if (plan->exec) cudaGraphExecDestroy(plan->exec);
  if (plan->mem) cudaFreeAsync(plan->mem, stream);
  if (plan->mem2) cudaFreeAsync(plan->mem2, stream);
  if (plan->mem3) cudaFreeAsync(plan->mem3, stream);
  delete plan;
  return CFGMM_OK;
}

double aodm_plan_flops(const cfgmm_aodm_plan* plan) { return plan ? plan->flops : 0.0; }

}  // namespace cfgmm
