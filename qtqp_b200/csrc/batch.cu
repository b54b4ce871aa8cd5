// Batched device-resident dense IPM: persistent launches (one per size class)
// in which one thread block runs one QP at a time, QPs taken from a
// cost-sorted work list.
#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "batch_kernel.cuh"

namespace qtqp {

static int launch_nt(int nt, int lean, const BatchParams& p, int smem_total, cudaStream_t st) {
  switch (nt) {
    case 32: return lean ? launch_group_32_lean(p, smem_total, st)
                         : launch_group_32(p, smem_total, st);
    case 64: return lean ? launch_group_64_lean(p, smem_total, st)
                         : launch_group_64(p, smem_total, st);
    case 128: return lean ? launch_group_128_lean(p, smem_total, st)
                          : launch_group_128(p, smem_total, st);
    case 256: return lean ? launch_group_256_lean(p, smem_total, st)
                          : launch_group_256(p, smem_total, st);
    default: return fail(QTQP_ERR_BAD_ARG, "block_threads must be 32, 64, 128 or 256");
  }
}

// Side streams/events used to run the groups concurrently (created once per
// device, never destroyed).
struct ForkStreams {
  cudaStream_t s[QTQP_MAX_GROUPS] = {};
  cudaEvent_t join[QTQP_MAX_GROUPS] = {};
  cudaEvent_t fork = nullptr;
  bool ready = false;
};
static std::mutex g_fork_mu[64];
static ForkStreams g_fork[64];

// The side streams of the current device.  The caller holds `lk`, the
// device's fork lock, from the fork record until the last join has been
// enqueued: the fork/join events are shared by every call on the device, and
// a second host thread re-recording them in between would make this call's
// groups wait on the other call's stream instead of this one's.
static int fork_streams(ForkStreams** out, std::unique_lock<std::mutex>& lk) {
  int dev = 0;
  int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= 64) return fail(QTQP_ERR_BAD_ARG, "device index out of range");
  lk = std::unique_lock<std::mutex>(g_fork_mu[dev]);
  ForkStreams& f = g_fork[dev];
  if (!f.ready) {
    // Group 0 holds the costliest instances (the plan sorts by cost), the
    // batch's critical path: its stream gets the highest priority, so that
    // its blocks are placed first and the other groups fill the SMs around
    // them (measured: 24.1 -> 23.3 ms per 4096-QP batch).
    int least = 0, greatest = 0;
    rc = cuda_check(cudaDeviceGetStreamPriorityRange(&least, &greatest),
                    "cudaDeviceGetStreamPriorityRange");
    if (rc) return rc;
    for (int g = 0; g < QTQP_MAX_GROUPS; ++g) {
      rc = cuda_check(cudaStreamCreateWithPriority(&f.s[g], cudaStreamNonBlocking,
                                                   g == 0 ? greatest : least),
                      "cudaStreamCreateWithPriority");
      if (rc) return rc;
      rc = cuda_check(cudaEventCreateWithFlags(&f.join[g], cudaEventDisableTiming),
                      "cudaEventCreateWithFlags");
      if (rc) return rc;
    }
    rc = cuda_check(cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming),
                    "cudaEventCreateWithFlags");
    if (rc) return rc;
    f.ready = true;
  }
  *out = &f;
  return QTQP_OK;
}

}  // namespace qtqp

using namespace qtqp;

static int dense_batch_plan(qtqp_dense_instance* h_inst, int32_t count,
                            const qtqp_options* opt, int32_t* h_order, int32_t block_threads,
                            int32_t smem_bytes, const qtqp_batch_tuning* table,
                            int32_t entries, qtqp_batch_plan* plan) {
  if (h_inst == nullptr || h_order == nullptr || opt == nullptr || plan == nullptr ||
      count < 0)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_plan: null argument or negative count");
  if (block_threads != 0 && block_threads != 32 && block_threads != 64 &&
      block_threads != 128 && block_threads != 256)
    return fail(QTQP_ERR_BAD_ARG, "block_threads must be 0, 32, 64, 128 or 256");
  for (int i = 0; i < count; ++i) {
    const qtqp_dense_instance& d = h_inst[i];
    if (d.n < 1 || d.m < 1 || d.z < 0 || d.z >= d.m)
      return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_plan: instance " + std::to_string(i) +
                                        " needs n >= 1, m >= 1 and 0 <= z < m");
  }
  std::vector<int32_t> ord(count);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
    return inst_cost(h_inst[a].n, h_inst[a].m) > inst_cost(h_inst[b].n, h_inst[b].m);
  });
  std::copy(ord.begin(), ord.end(), h_order);

  // Size class of an instance: blocks per SM when all its data is on chip
  // (0 = too large for one block's shared memory).
  auto threads_for = [&](int N) {
    if (block_threads) return int(block_threads);
    return N <= 64 ? 64 : (N <= 192 ? 128 : 256);
  };
  auto onchip = [&](int i) {
    const InstLayout L = plan_layout(h_inst[i].n, h_inst[i].m, size_t(1) << 40);
    return L.smem_bytes;
  };
  auto klass = [&](int i) {
    const size_t f = onchip(i) + red_bytes_rt(threads_for(h_inst[i].n + h_inst[i].m));
    if (smem_bytes) return 1;
    if (f > kSmemBlockMax) return 0;
    return int(std::min<size_t>(8, kSmemPerSm / (f + kSmemReserved)));
  };
  struct Run { int begin, count, cls; };
  std::vector<Run> runs;
  for (int k = 0; k < count; ++k) {
    const int c = klass(ord[k]);
    if (!runs.empty() && runs.back().cls == c) {
      ++runs.back().count;
    } else {
      runs.push_back({k, 1, c});
    }
  }
  // Merge the smallest adjacent runs until the groups fit the plan.
  while (int(runs.size()) > QTQP_MAX_GROUPS) {
    size_t best = 0;
    for (size_t r = 1; r + 1 < runs.size(); ++r)
      if (runs[r].count + runs[r + 1].count < runs[best].count + runs[best + 1].count) best = r;
    runs[best].count += runs[best + 1].count;
    runs[best].cls = std::min(runs[best].cls, runs[best + 1].cls);
    runs.erase(runs.begin() + best + 1);
  }
  *plan = qtqp_batch_plan{};
  plan->num_groups = int32_t(runs.size());
  size_t off = kWsHeader;
  for (size_t g = 0; g < runs.size(); ++g) {
    const Run& r = runs[g];
    int max_N = 0, max_n = 0;
    size_t max_all = 0, max_gv = 0;
    for (int k = r.begin; k < r.begin + r.count; ++k) {
      const qtqp_dense_instance& d = h_inst[ord[k]];
      max_N = std::max(max_N, d.n + d.m);
      max_n = std::max(max_n, d.n);
      const InstLayout L = plan_layout(d.n, d.m, 0);
      max_gv = std::max(max_gv, L.g_bytes + L.v_bytes);
      max_all = std::max(max_all, L.g_bytes + L.v_bytes + L.a_bytes + L.p_bytes);
    }
    int nt = threads_for(max_N);
    if (!block_threads && r.cls == 1 && max_N > 128) nt = 256;
    // A tuning entry (first match on the group's largest n) replaces the
    // default launch shape unless a shape is forced.
    const qtqp_batch_tuning* tu = nullptr;
    for (int e = 0; e < entries && !block_threads && !smem_bytes; ++e)
      if (table[e].n_lo <= max_n && max_n <= table[e].n_hi) {
        tu = &table[e];
        break;
      }
    int lean = 0;
    if (tu) {
      nt = tu->block_threads;
      lean = tu->lean != 0;
    }
    const size_t red = red_bytes_rt(nt);
    size_t cap;
    if (tu) {
      if (tu->onchip && max_all + red <= kSmemBlockMax) {
        cap = max_all;
      } else if (max_gv + red <= kSmemBlockMax) {
        cap = max_gv;
      } else {
        cap = 0;
      }
    } else if (smem_bytes) {
      if (size_t(smem_bytes) < red || size_t(smem_bytes) > kSmemBlockMax)
        return fail(QTQP_ERR_BAD_ARG, "smem_bytes outside [reduction scratch, 227 KiB]");
      cap = size_t(smem_bytes) - red;
    } else if (max_all + red <= kSmemBlockMax &&
               (r.cls > 1 || 2 * (max_gv + red + kSmemReserved) > kSmemPerSm)) {
      cap = max_all;  // everything on chip
    } else if (max_all + red <= kSmemBlockMax) {
      // One block per SM if A and P stay on chip: keeping only G and the
      // vectors there (A and P through L2) fits two or more QPs per SM,
      // which is faster for these latency-bound solves (measured: n 49..64,
      // m = 2n: 16.8 -> 14.7 ms per 1172 QPs).
      cap = max_gv;
    } else if (max_gv + red <= kSmemBlockMax) {
      cap = max_gv;   // G + vectors on chip, A and P through L2
    } else {
      cap = 0;        // large instances: everything in the global workspace
    }
    for (int k = r.begin; k < r.begin + r.count; ++k) {
      qtqp_dense_instance& d = h_inst[ord[k]];
      const InstLayout L = plan_layout(d.n, d.m, cap);
      d.ws_off = int64_t(off);
      off += (L.global_bytes + 255) & ~size_t(255);
    }
    plan->groups[g] = qtqp_launch_group{r.begin, r.count, nt, int32_t(cap + red), 0, lean};
  }
  plan->workspace_bytes = off;
  return QTQP_OK;
}

extern "C" int qtqp_dense_batch_plan(qtqp_dense_instance* h_inst, int32_t count,
                                     const qtqp_options* opt, int32_t* h_order,
                                     int32_t block_threads, int32_t smem_bytes,
                                     qtqp_batch_plan* plan) {
  return dense_batch_plan(h_inst, count, opt, h_order, block_threads, smem_bytes, nullptr, 0,
                          plan);
}

extern "C" int qtqp_dense_batch_plan_tuned(qtqp_dense_instance* h_inst, int32_t count,
                                           const qtqp_options* opt, int32_t* h_order,
                                           const qtqp_batch_tuning* table, int32_t entries,
                                           qtqp_batch_plan* plan) {
  if (entries < 0 || (entries > 0 && table == nullptr))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_plan_tuned: bad tuning table");
  for (int e = 0; e < entries; ++e) {
    const int nt = table[e].block_threads;
    if (nt != 32 && nt != 64 && nt != 128 && nt != 256)
      return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_plan_tuned: entry " + std::to_string(e) +
                                        ": block_threads must be 32, 64, 128 or 256");
  }
  return dense_batch_plan(h_inst, count, opt, h_order, 0, 0, table, entries, plan);
}

static int dense_batch_solve(const qtqp_dense_instance* d_inst, const int32_t* d_order,
                             const qtqp_batch_plan* plan, const double* d_a_pool,
                             const double* d_p_pool, const double* d_b_pool,
                             const double* d_c_pool, double* d_x_pool, double* d_y_pool,
                             double* d_s_pool, qtqp_result* d_results, qtqp_iter_stats* d_stats,
                             void* d_workspace, size_t workspace_bytes, const qtqp_options* opt,
                             const double* d_x0_pool, const double* d_y0_pool,
                             const double* d_s0_pool, void* stream, int only = -1) {
  if (plan == nullptr || opt == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve: null plan/options");
  if (plan->num_groups == 0) return QTQP_OK;
  if (plan->num_groups < 0 || plan->num_groups > QTQP_MAX_GROUPS)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve: bad group count");
  if (d_inst == nullptr || d_order == nullptr || d_a_pool == nullptr || d_b_pool == nullptr ||
      d_c_pool == nullptr || d_x_pool == nullptr || d_y_pool == nullptr || d_s_pool == nullptr ||
      d_results == nullptr || d_workspace == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve: null argument");
  if (workspace_bytes < plan->workspace_bytes)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve: workspace smaller than the plan's");
  if (opt->max_iter < 1 || opt->max_iterative_refinement_steps < 1 ||
      !(opt->step_size_scale > 0.0 && opt->step_size_scale < 1.0))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve: invalid options");
  if (only >= plan->num_groups)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve_group: group index out of range");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The work counters must start at zero: every group's, or the one group's
  // (the others may belong to launches still running on other streams).
  int rc = only < 0 ? cuda_check(cudaMemsetAsync(d_workspace, 0, kWsHeader, st), "cudaMemsetAsync")
                    : cuda_check(cudaMemsetAsync(static_cast<int*>(d_workspace) + only, 0,
                                                 sizeof(int), st),
                                 "cudaMemsetAsync");
  if (rc) return rc;
  BatchParams base;
  base.inst = d_inst;
  base.a_pool = d_a_pool;
  base.p_pool = d_p_pool != nullptr ? d_p_pool : d_a_pool;
  base.b_pool = d_b_pool;
  base.c_pool = d_c_pool;
  base.x_pool = d_x_pool;
  base.y_pool = d_y_pool;
  base.s_pool = d_s_pool;
  base.results = d_results;
  base.stats = d_stats;
  base.ws = static_cast<char*>(d_workspace);
  base.opt = *opt;
  base.x0_pool = d_x0_pool;
  base.y0_pool = d_y0_pool;
  base.s0_pool = d_s0_pool;
  const int ng = plan->num_groups;
  ForkStreams* fk = nullptr;
  std::unique_lock<std::mutex> fork_lock;  // held until every join is enqueued
  if (ng > 1 && only < 0) {
    rc = fork_streams(&fk, fork_lock);
    if (rc) return rc;
    rc = cuda_check(cudaEventRecord(fk->fork, st), "cudaEventRecord");
    if (rc) return rc;
  }
  for (int g = 0; g < ng; ++g) {
    const qtqp_launch_group& G = plan->groups[g];
    if (G.count <= 0 || (only >= 0 && g != only)) continue;
    const size_t red = red_bytes_rt(G.block_threads);
    if (size_t(G.smem_bytes) < red)
      return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve: group smem below scratch");
    BatchParams p = base;
    p.order = d_order + G.begin;
    p.count = G.count;
    p.counter = static_cast<int*>(d_workspace) + g;
    p.smem_cap = size_t(G.smem_bytes) - red;
    cudaStream_t gs = st;
    if (fk) {
      gs = fk->s[g];
      rc = cuda_check(cudaStreamWaitEvent(gs, fk->fork, 0), "cudaStreamWaitEvent");
      if (rc) return rc;
    }
    rc = launch_nt(G.block_threads, G.lean, p, G.smem_bytes, gs);
    if (rc) return rc;
    if (fk) {
      rc = cuda_check(cudaEventRecord(fk->join[g], gs), "cudaEventRecord");
      if (rc) return rc;
      rc = cuda_check(cudaStreamWaitEvent(st, fk->join[g], 0), "cudaStreamWaitEvent");
      if (rc) return rc;
    }
  }
  return QTQP_OK;
}

extern "C" int qtqp_dense_batch_solve(const qtqp_dense_instance* d_inst, const int32_t* d_order,
                                      const qtqp_batch_plan* plan, const double* d_a_pool,
                                      const double* d_p_pool, const double* d_b_pool,
                                      const double* d_c_pool, double* d_x_pool, double* d_y_pool,
                                      double* d_s_pool, qtqp_result* d_results,
                                      qtqp_iter_stats* d_stats, void* d_workspace,
                                      size_t workspace_bytes, const qtqp_options* opt,
                                      void* stream) {
  return dense_batch_solve(d_inst, d_order, plan, d_a_pool, d_p_pool, d_b_pool, d_c_pool,
                           d_x_pool, d_y_pool, d_s_pool, d_results, d_stats, d_workspace,
                           workspace_bytes, opt, nullptr, nullptr, nullptr, stream);
}

extern "C" int qtqp_dense_batch_solve_group(
    const qtqp_dense_instance* d_inst, const int32_t* d_order, const qtqp_batch_plan* plan,
    int32_t group, const double* d_a_pool, const double* d_p_pool, const double* d_b_pool,
    const double* d_c_pool, double* d_x_pool, double* d_y_pool, double* d_s_pool,
    qtqp_result* d_results, qtqp_iter_stats* d_stats, void* d_workspace,
    size_t workspace_bytes, const qtqp_options* opt, void* stream) {
  if (group < 0)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve_group: negative group index");
  return dense_batch_solve(d_inst, d_order, plan, d_a_pool, d_p_pool, d_b_pool, d_c_pool,
                           d_x_pool, d_y_pool, d_s_pool, d_results, d_stats, d_workspace,
                           workspace_bytes, opt, nullptr, nullptr, nullptr, stream, group);
}

extern "C" int qtqp_dense_batch_solve_from(
    const qtqp_dense_instance* d_inst, const int32_t* d_order, const qtqp_batch_plan* plan,
    const double* d_a_pool, const double* d_p_pool, const double* d_b_pool,
    const double* d_c_pool, double* d_x_pool, double* d_y_pool, double* d_s_pool,
    qtqp_result* d_results, qtqp_iter_stats* d_stats, void* d_workspace,
    size_t workspace_bytes, const qtqp_options* opt, const double* d_x0_pool,
    const double* d_y0_pool, const double* d_s0_pool, void* stream) {
  if (d_x0_pool == nullptr || d_y0_pool == nullptr || d_s0_pool == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve_from: null starting point pool");
  return dense_batch_solve(d_inst, d_order, plan, d_a_pool, d_p_pool, d_b_pool, d_c_pool,
                           d_x_pool, d_y_pool, d_s_pool, d_results, d_stats, d_workspace,
                           workspace_bytes, opt, d_x0_pool, d_y0_pool, d_s0_pool, stream);
}

// ---------------------------------------------------------------------------
// Allocation-free batch solve.
//
// Some callers cannot allocate device memory when they solve: code running
// inside another framework's memory pool, a real-time control loop that must
// not touch the allocator after start-up, or a process whose allocator is
// locked.  For them the scratch of the batch solve lives in a fixed array
// that is part of this library's device image; it is reserved on every GPU
// that loads the library, for the lifetime of the process.
// ---------------------------------------------------------------------------
namespace qtqp {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

static std::mutex g_static_mu;
static void* g_static_ptr[64];
static unsigned long long g_static_ctx[64];  // context the cached address belongs to

// Unique id of the calling thread's current CUDA context (the driver's
// cuCtxGetCurrent + cuCtxGetId, reached through the runtime so that the
// library needs no link against the driver library); 0 if unavailable.
static unsigned long long current_context_id() {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(p);
  });
  if (get_current == nullptr || get_id == nullptr) return 0;
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != 0 || ctx == nullptr || get_id(ctx, &id) != 0) return 0;
  return id;
}

// Device address of g_static_scratch on the current device.  The symbol's
// name is only a host-side handle, so the address is looked up with that
// device current and cached per device.  The cache remembers the context it
// was taken in: after a cudaDeviceReset the device's next context gets a new
// id and the address is looked up again instead of pointing into the
// destroyed context.
static int static_scratch(void** out) {
  int dev = 0;
  int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= 64) return fail(QTQP_ERR_BAD_ARG, "device index out of range");
  // Before the runtime's first call on this device there is no current
  // context (id 0): the lookup then runs, initialises the context, and the
  // id is read afterwards.
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (g_static_ptr[dev] == nullptr || ctx == 0 || g_static_ctx[dev] != ctx) {
    void* p = nullptr;
    rc = cuda_check(cudaGetSymbolAddress(&p, g_static_scratch), "cudaGetSymbolAddress");
    if (rc) return rc;
    g_static_ptr[dev] = p;
    g_static_ctx[dev] = current_context_id();
  }
  *out = g_static_ptr[dev];
  return QTQP_OK;
}

}  // namespace qtqp

extern "C" size_t qtqp_dense_batch_noalloc_max_workspace(void) { return kStaticScratchBytes; }

extern "C" int qtqp_dense_batch_solve_noalloc(
    const qtqp_dense_instance* d_inst, const int32_t* d_order, const qtqp_batch_plan* plan,
    const double* d_a_pool, const double* d_p_pool, const double* d_b_pool,
    const double* d_c_pool, double* d_x_pool, double* d_y_pool, double* d_s_pool,
    qtqp_result* d_results, qtqp_iter_stats* d_stats, const qtqp_options* opt, void* stream) {
  if (plan == nullptr || opt == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve_noalloc: null plan/options");
  if (plan->num_groups == 0) return QTQP_OK;
  if (plan->num_groups < 0 || plan->num_groups > QTQP_MAX_GROUPS)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve_noalloc: bad group count");
  if (plan->workspace_bytes > kStaticScratchBytes)
    return fail(QTQP_ERR_BAD_ARG,
                "qtqp_dense_batch_solve_noalloc: the plan needs " +
                    std::to_string(plan->workspace_bytes) +
                    " bytes of scratch, more than the library's fixed 16 MiB; use "
                    "qtqp_dense_batch_solve with a caller-provided workspace");
  if (d_inst == nullptr || d_order == nullptr || d_a_pool == nullptr || d_b_pool == nullptr ||
      d_c_pool == nullptr || d_x_pool == nullptr || d_y_pool == nullptr || d_s_pool == nullptr ||
      d_results == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve_noalloc: null argument");
  if (opt->max_iter < 1 || opt->max_iterative_refinement_steps < 1 ||
      !(opt->step_size_scale > 0.0 && opt->step_size_scale < 1.0))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve_noalloc: invalid options");
  void* ws = nullptr;
  int rc = static_scratch(&ws);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The work counters must start at zero; everything else in the scratch is
  // written by the kernel before it is read.
  rc = cuda_check(cudaMemsetAsync(ws, 0, kWsHeader, st), "cudaMemsetAsync");
  if (rc) return rc;
  BatchParams base;
  base.inst = d_inst;
  base.a_pool = d_a_pool;
  base.p_pool = d_p_pool != nullptr ? d_p_pool : d_a_pool;
  base.b_pool = d_b_pool;
  base.c_pool = d_c_pool;
  base.x_pool = d_x_pool;
  base.y_pool = d_y_pool;
  base.s_pool = d_s_pool;
  base.results = d_results;
  base.stats = d_stats;
  base.ws = static_cast<char*>(ws);
  base.opt = *opt;
  base.x0_pool = base.y0_pool = base.s0_pool = nullptr;
  // Groups run one after another on the caller's stream (no side streams).
  for (int g = 0; g < plan->num_groups; ++g) {
    const qtqp_launch_group& G = plan->groups[g];
    if (G.count <= 0) continue;
    const size_t red = red_bytes_rt(G.block_threads);
    if (size_t(G.smem_bytes) < red)
      return fail(QTQP_ERR_BAD_ARG, "qtqp_dense_batch_solve_noalloc: group smem below scratch");
    BatchParams p = base;
    p.order = d_order + G.begin;
    p.count = G.count;
    p.counter = static_cast<int*>(ws) + g;
    p.smem_cap = size_t(G.smem_bytes) - red;
    rc = launch_nt(G.block_threads, G.lean, p, G.smem_bytes, st);
    if (rc) return rc;
  }
  return QTQP_OK;
}
