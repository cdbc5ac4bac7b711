// Host side of libccb: device graphs, kernel planning, the PBILS and Neighborhood drivers, and the C ABI
// declared in include/ccb.h.
//
// The drivers enqueue whole iterations on one stream and never wait on the device inside the loop: the
// record, stall counter, early stop and GWW ranking run on the device (k_record), so the host only
// polls a stop flag once per chunk of iterations, one chunk behind the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "ccb.h"
#include "ccb_error.h"
#include "ccb_kernels.cuh"
#include "ccb_plans.h"

namespace ccb {

namespace {
thread_local char g_last_error[1024];
}  // namespace

void SetLastError(const char* message) {
  std::strncpy(g_last_error, message, sizeof(g_last_error) - 1);
  g_last_error[sizeof(g_last_error) - 1] = '\0';
}

const char* LastError() { return g_last_error; }

namespace {

struct Failure {
  int status;
  std::string message;
};

#define CCB_CUDA(call)                                                                                     \
  do {                                                                                                     \
    const cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess) {                                                                               \
      throw ::ccb::Failure{CCB_ERR_CUDA, std::string("cuda error at ") + __FILE__ + ":" +                  \
                                             std::to_string(__LINE__) + ": " + cudaGetErrorString(e_)};    \
    }                                                                                                      \
  } while (0)

[[noreturn]] void Fail(int status, const std::string& message) { throw Failure{status, message}; }

template <typename F>
int Guard(F&& body) {
  try {
    body();
    g_last_error[0] = '\0';
    return CCB_OK;
  } catch (const Failure& e) {
    SetLastError(e.message);
    return e.status;
  } catch (const std::bad_alloc&) {
    SetLastError("host memory exhausted");
    return CCB_ERR_DEVICE_MEMORY;
  } catch (const std::exception& e) {
    SetLastError(e.what());
    return CCB_ERR_INVALID;
  }
}

constexpr int kAuxThreads = 256;
constexpr int kRebuildThreads = 512;
constexpr int kRecordThreads = 1024;
constexpr int kPollChunk = 4;  // iterations enqueued between stop-flag polls

int BitWidth(unsigned x) { return x == 0 ? 0 : 32 - __builtin_clz(x); }
size_t Round16(size_t b) { return (b + 15) / 16 * 16; }
long long CeilDiv(long long a, long long b) { return (a + b - 1) / b; }
std::string Mebibytes(size_t bytes) { return std::to_string(CeilDiv((long long)bytes, 1 << 20)) + " MiB"; }

struct Device {
  int id = 0;
  int sms = 0;
  int l2_bytes = 0;
  int smem_optin = 0;

  static Device Current() {
    Device d;
    CCB_CUDA(cudaGetDevice(&d.id));
    CCB_CUDA(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, d.id));
    CCB_CUDA(cudaDeviceGetAttribute(&d.l2_bytes, cudaDevAttrL2CacheSize, d.id));
    CCB_CUDA(cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d.id));
    return d;
  }
};

// Parameter checks shared with the CPU backend (CheckParams, src/cc_pbils_cpu.cpp:177-181), in the
// same order and with the same messages.
void CheckParams(const ccb_params& p) {
  if (p.k < 1) Fail(CCB_ERR_INVALID, "k must be >= 1");
  if (p.population < 1) Fail(CCB_ERR_INVALID, "population must be >= 1");
  if (p.gww < 0.0 || p.gww > 0.5) Fail(CCB_ERR_INVALID, "gww must be in [0, 0.5]");
}

// SolveGpu's extra limits (cuda/cc_pbils_gpu.cu:443-450).
void CheckGpuLimits(const ccb_params& p, uint32_t n) {
  if (p.k > CCB_MAX_CLUSTERS) {
    Fail(CCB_ERR_INVALID, "k exceeds kMaxClusters (" + std::to_string(CCB_MAX_CLUSTERS) +
                              "); raise it in cc_gpu.hpp and rebuild");
  }
  if (n > (uint32_t)CCB_MAX_VERTICES_WIDE) {
    Fail(CCB_ERR_INVALID,
         "n exceeds " + std::to_string(CCB_MAX_VERTICES_WIDE) + ", the range of the packed move");
  }
}

// Neighborhood's checks (cuda/cc_pbils_gpu.cu:427-432).
void CheckNeighborhood(const ccb_params& p, uint32_t n) {
  if (p.k != 2) Fail(CCB_ERR_INVALID, "Neighborhood algorithms require k = 2");
  if (p.population < 1) Fail(CCB_ERR_INVALID, "population must be >= 1");
  if (n == 0 || n > (uint32_t)CCB_MAX_VERTICES_WIDE) {
    Fail(CCB_ERR_INVALID, "Neighborhood requires 1 <= n <= " + std::to_string(CCB_MAX_VERTICES_WIDE));
  }
}

int CountClustersUsed(const int32_t* labels, uint32_t n, int k) {
  std::vector<char> seen(std::max(k, 1), 0);
  int used = 0;
  for (uint32_t v = 0; v < n; ++v) {
    const int l = labels[v];
    if (l >= 0 && l < k && !seen[l]) {
      seen[l] = 1;
      ++used;
    }
  }
  return used;
}

}  // namespace
}  // namespace ccb

using namespace ccb;

// ------------------------------------------------------------------------------------------------
// Device graph
// ------------------------------------------------------------------------------------------------
struct ccb_graph {
  int device = 0;
  int n = 0;
  int words = 0;  // ceil(n / 32)
  int pitch = 0;  // words per row in memory (multiple of 4)
  int64_t edges = 0;
  uint32_t* bits = nullptr;
  int32_t* degrees = nullptr;

  GraphView View() const { return GraphView{bits, degrees, n, words, pitch, edges}; }
  ~ccb_graph() {
    if (bits) cudaFree(bits);
    if (degrees) cudaFree(degrees);
  }
};

namespace {

ccb_graph* MakeGraph(const uint32_t* src, bool src_on_device, uint32_t n, uint32_t words_per_row, uint64_t edges,
                     cudaStream_t stream) {
  if (n > (uint32_t)CCB_MAX_VERTICES_WIDE) {
    Fail(CCB_ERR_INVALID, "n exceeds " + std::to_string(CCB_MAX_VERTICES_WIDE) + ", the range of the packed move");
  }
  const int words = (int)((n + 31) / 32);
  if (n > 0 && words_per_row < (uint32_t)words) Fail(CCB_ERR_INVALID, "words_per_row < ceil(n / 32)");
  if (n > 0 && src == nullptr) Fail(CCB_ERR_INVALID, "null bitset");
  std::unique_ptr<ccb_graph> g(new ccb_graph());
  CCB_CUDA(cudaGetDevice(&g->device));
  g->n = (int)n;
  g->words = words;
  g->pitch = std::max(4, (words + 3) / 4 * 4);
  g->edges = (int64_t)edges;
  const size_t rows = std::max<uint32_t>(n, 1);
  const size_t bytes = rows * g->pitch * sizeof(uint32_t);
  size_t free_b = 0, total_b = 0;
  CCB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (bytes + rows * 4 > free_b) {
    Fail(CCB_ERR_DEVICE_MEMORY, "graph needs " + Mebibytes(bytes) + " of device memory, " + Mebibytes(free_b) + " free");
  }
  CCB_CUDA(cudaMalloc(&g->bits, bytes));
  CCB_CUDA(cudaMalloc(&g->degrees, rows * sizeof(int32_t)));
  CCB_CUDA(cudaMemsetAsync(g->bits, 0, bytes, stream));
  CCB_CUDA(cudaMemsetAsync(g->degrees, 0, rows * sizeof(int32_t), stream));
  if (n > 0) {
    CCB_CUDA(cudaMemcpy2DAsync(g->bits, g->pitch * sizeof(uint32_t), src, words_per_row * sizeof(uint32_t),
                               words * sizeof(uint32_t), n,
                               src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream));
    k_degrees<<<(int)CeilDiv(n, kAuxThreads), kAuxThreads, 0, stream>>>(g->bits, (int)n, words, g->pitch,
                                                                         g->degrees);
    CCB_CUDA(cudaGetLastError());
  }
  CCB_CUDA(cudaStreamSynchronize(stream));
  return g.release();
}

// ------------------------------------------------------------------------------------------------
// Kernel plan
// ------------------------------------------------------------------------------------------------
struct Plan {
  bool wide = false;        // int32 G, 64-bit keys, state in global memory
  bool smem_state = false;  // labels + G of the slot in shared memory
  bool smem_rows = false;   // whole bitset in shared memory
  int threads = 512;
  size_t smem_bytes = 0;
  int key_bits = 0;
  bool small_k = false;     // the packed K <= 8 descents (registers / streamed)
  bool incremental = false; // the incremental 9 <= k <= 64 descent
  SmallKPlan sk;
};

// Threads and vertices per thread of the register descent: the smallest block that covers n with 4
// vertices per thread (measured on the plain configuration, n = 1000, k = 5: 256 x 4 beats 128 x 8 by 10%
// and 512 x 4 by 50%); CCB_REG_SHAPE=T,V overrides it for tuning sweeps.
void RegisterShape(int n, int* threads, int* vpt) {
  *vpt = 4;
  *threads = 128;
  while (*threads * *vpt < n) *threads *= 2;
  if (const char* env = std::getenv("CCB_REG_SHAPE")) {
    int t = 0, v = 0;
    if (std::sscanf(env, "%d,%d", &t, &v) == 2 && RegistersShapeBuilt(t, v) && t * v >= n) {
      *threads = t;
      *vpt = v;
    }
  }
}


int DescentThreads(int n, bool wide) {
  if (wide) return 1024;
  if (n <= 256) return 128;
  if (n <= 512) return 256;
  if (n <= 2048) return 512;
  return 1024;
}

size_t DescentSmem(const Plan& p, int n, int pitch, int k, int ld, int kpad) {
  const int warps = p.threads / kWarp;
  const size_t gain = p.wide ? 4 : 2;
  const size_t rec = p.wide ? sizeof(MoveRecord<unsigned long long>) : sizeof(MoveRecord<uint32_t>);
  size_t b = 0;
  if (p.smem_rows) b += Round16((size_t)n * pitch * 4);
  if (p.smem_state) b += Round16((size_t)k * ld * gain) + Round16(ld);
  b += (size_t)warps * kpad * 4 + 15 + 2 * warps * rec;
  return b;
}

Plan MakePlan(int n, int pitch, int k, int ld, int kpad, int ls_kernel, const Device& dev) {
  Plan p;
  p.wide = n > CCB_MAX_VERTICES_NARROW || ls_kernel == CCB_LS_WIDE;
  p.threads = DescentThreads(n, p.wide);
  p.key_bits = BitWidth((unsigned)std::max(n, 1));
  const size_t limit = (size_t)dev.smem_optin - 1024;  // static shared memory and margin
  if (!p.wide) {
    Plan with_state = p;
    with_state.smem_state = true;
    const size_t state_bytes = DescentSmem(with_state, n, pitch, k, ld, kpad);
    const bool fits = state_bytes <= limit;
    if (ls_kernel == CCB_LS_SHARED && !fits) {
      Fail(CCB_ERR_DEVICE_MEMORY, "state needs " + std::to_string((size_t)k * ld * 2 + ld) +
                                      " bytes of shared memory, device allows " + std::to_string(dev.smem_optin));
    }
    p.smem_state = ls_kernel != CCB_LS_GLOBAL && fits;
    Plan with_rows = p;
    with_rows.smem_rows = true;
    p.smem_rows = DescentSmem(with_rows, n, pitch, k, ld, kpad) <= limit;
  }
  p.smem_bytes = DescentSmem(p, n, pitch, k, ld, kpad);
  if (!p.wide && k >= 2 && k <= 8 && ls_kernel == CCB_LS_AUTO) {
    SmallKPlan& sk = p.sk;
    sk.k = k;
    if (n <= 4096) {
      sk.registers = true;
      sk.smem_state = true;  // nothing of the state lives in global memory
      RegisterShape(n, &sk.threads, &sk.vpt);
      sk.smem_rows = RegistersSmem(n, pitch, true) <= limit;
      sk.smem_bytes = RegistersSmem(n, pitch, sk.smem_rows);
    } else {
      sk.threads = 1024;
      sk.smem_state = SmallKSmem(k, n, pitch, ld, sk.threads, true, false) <= limit;
      sk.smem_rows = false;
      sk.smem_bytes = SmallKSmem(k, n, pitch, ld, sk.threads, sk.smem_state, false);
    }
    p.small_k = true;
    p.smem_state = sk.smem_state;
    p.smem_rows = sk.smem_rows;
    p.threads = sk.threads;
    p.smem_bytes = sk.smem_bytes;
  }
  if (!p.wide && k > 8 && ls_kernel == CCB_LS_AUTO) {
    SmallKPlan& sk = p.sk;
    sk.k = k;
    sk.threads = n <= 2048 ? 256 : (n <= 8192 ? 512 : 1024);
    sk.smem_state = IncrementalBytes(k, ld) + 10 * 1024 <= limit;  // the kernel's static shared memory
    sk.smem_bytes = sk.smem_state ? IncrementalBytes(k, ld) : 0;
    p.incremental = true;
    p.smem_state = sk.smem_state;
    p.smem_rows = false;
    p.threads = sk.threads;
    p.smem_bytes = sk.smem_bytes;
  }
  return p;
}

template <typename GainT, typename Key, bool S, bool R, int T>
void LaunchDescentT(const DescentArgs<GainT>& a, int grid, size_t smem, cudaStream_t st, bool configure) {
  auto kernel = k_descent<GainT, Key, S, R, T>;
  if (configure) {
    CCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return;
  }
  kernel<<<grid, T, smem, st>>>(a);
}

template <typename GainT, typename Key, bool S, bool R>
void LaunchDescentThreads(const DescentArgs<GainT>& a, int threads, int grid, size_t smem, cudaStream_t st,
                          bool configure) {
  switch (threads) {
    case 128: return LaunchDescentT<GainT, Key, S, R, 128>(a, grid, smem, st, configure);
    case 256: return LaunchDescentT<GainT, Key, S, R, 256>(a, grid, smem, st, configure);
    case 512: return LaunchDescentT<GainT, Key, S, R, 512>(a, grid, smem, st, configure);
    default: return LaunchDescentT<GainT, Key, S, R, 1024>(a, grid, smem, st, configure);
  }
}

template <typename GainT>
void LaunchDescent(const Plan& p, const DescentArgs<GainT>& a, int grid, cudaStream_t st, bool configure) {
  if constexpr (std::is_same_v<GainT, int32_t>) {
    LaunchDescentThreads<int32_t, unsigned long long, false, false>(a, p.threads, grid, p.smem_bytes, st, configure);
  } else {
    if (p.smem_state && p.smem_rows) {
      LaunchDescentThreads<int16_t, uint32_t, true, true>(a, p.threads, grid, p.smem_bytes, st, configure);
    } else if (p.smem_state) {
      LaunchDescentThreads<int16_t, uint32_t, true, false>(a, p.threads, grid, p.smem_bytes, st, configure);
    } else if (p.smem_rows) {
      LaunchDescentThreads<int16_t, uint32_t, false, true>(a, p.threads, grid, p.smem_bytes, st, configure);
    } else {
      LaunchDescentThreads<int16_t, uint32_t, false, false>(a, p.threads, grid, p.smem_bytes, st, configure);
    }
  }
}

const char* KernelName(const Plan& p) {
  if (p.incremental) return p.smem_state ? "incremental 9 <= k <= 64, shared memory" : "incremental 9 <= k <= 64, L2";
  if (p.small_k) {
    if (p.sk.registers) return p.smem_rows ? "packed k <= 8, registers, bitset in shared memory"
                                           : "packed k <= 8, registers";
    return p.smem_state ? "packed k <= 8, streamed from shared memory" : "packed k <= 8, streamed from L2";
  }
  if (p.wide) return "generic wide (int32 G), global memory";
  if (p.smem_state) return p.smem_rows ? "generic, shared memory, bitset in shared memory" : "generic, shared memory";
  return p.smem_rows ? "generic, global memory, bitset in shared memory" : "generic, global memory";
}

// Per-category CUDA-event timing of kernel launches (profiling only).
struct LaunchTimer {
  bool enabled = false;
  struct Span {
    cudaEvent_t start, stop;
    int category;
  };
  std::vector<Span> spans;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;

  cudaEvent_t Take() {
    if (used == pool.size()) {
      cudaEvent_t e;
      CCB_CUDA(cudaEventCreate(&e));
      pool.push_back(e);
    }
    return pool[used++];
  }
  template <typename F>
  void Time(int category, cudaStream_t st, F&& launch) {
    if (!enabled) {
      launch();
      return;
    }
    Span s{Take(), Take(), category};
    CCB_CUDA(cudaEventRecord(s.start, st));
    launch();
    CCB_CUDA(cudaEventRecord(s.stop, st));
    spans.push_back(s);
  }
  void Reset() {
    spans.clear();
    used = 0;
  }
  void Collect(ccb_kernel_stats* out) {
    std::memset(out, 0, sizeof(*out));
    for (const Span& s : spans) {
      float ms = 0.f;
      CCB_CUDA(cudaEventElapsedTime(&ms, s.start, s.stop));
      switch (s.category) {
        case 0: out->descent_ms += ms; out->descent_launches++; break;
        case 1: out->rebuild_ms += ms; out->rebuild_launches++; break;
        case 2: out->record_ms += ms; out->record_launches++; break;
        default: out->other_ms += ms; out->other_launches++; break;
      }
    }
  }
  ~LaunchTimer() {
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
  }
};

enum { kCatDescent = 0, kCatRebuild = 1, kCatRecord = 2, kCatOther = 3 };

}  // namespace

// ------------------------------------------------------------------------------------------------
// Solver: buffers for one (graph, k, population, kernel choice)
// ------------------------------------------------------------------------------------------------
struct ccb_solver {
  const ccb_graph* graph = nullptr;
  Device device;
  int n = 0, k = 0, kpad = 0, pop = 0, ld = 0;
  int ls_kernel = 0;
  Plan plan;
  std::vector<void*> allocations;
  void* cur_g = nullptr;
  void* next_g = nullptr;
  uint8_t* cur_lab = nullptr;
  uint8_t* next_lab = nullptr;
  int32_t* cur_sizes = nullptr;
  int64_t* cur_f = nullptr;
  int64_t* next_f = nullptr;
  uint32_t* masks = nullptr;
  int32_t* src_map = nullptr;
  int32_t* order = nullptr;
  uint8_t* record_lab = nullptr;
  Control* ctl = nullptr;
  TraceEntry* trace = nullptr;
  int trace_cap = 0;
  Control* host_ctl = nullptr;      // pinned, kPollSlots entries
  uint8_t* host_labels = nullptr;   // pinned, n entries
  TraceEntry* host_trace = nullptr; // pinned, trace_cap entries
  cudaEvent_t poll_event[2] = {nullptr, nullptr};
  size_t device_bytes = 0;
  std::string description;
  LaunchTimer timer;
  ccb_kernel_stats stats{};

  template <typename T>
  void Alloc(T*& ptr, size_t count) {
    void* p = nullptr;
    CCB_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    allocations.push_back(p);
    ptr = static_cast<T*>(p);
  }
  size_t GainBytes() const { return plan.wide ? 4 : 2; }

  ~ccb_solver() {
    for (void* p : allocations) cudaFree(p);
    if (host_ctl) cudaFreeHost(host_ctl);
    if (host_labels) cudaFreeHost(host_labels);
    if (host_trace) cudaFreeHost(host_trace);
    for (cudaEvent_t e : poll_event)
      if (e) cudaEventDestroy(e);
  }

  template <typename GainT>
  PopView<GainT> Cur() const {
    return PopView<GainT>{cur_lab, static_cast<GainT*>(cur_g), cur_sizes, cur_f};
  }
  template <typename GainT>
  PopView<GainT> Next() const {
    return PopView<GainT>{next_lab, static_cast<GainT*>(next_g), nullptr, next_f};
  }
};

namespace {

ccb_solver* MakeSolver(const ccb_graph* g, int k, int pop, int ls_kernel) {
  std::unique_ptr<ccb_solver> s(new ccb_solver());
  s->graph = g;
  s->device = Device::Current();
  if (s->device.id != g->device) Fail(CCB_ERR_STATE, "graph lives on another device");
  s->n = g->n;
  s->k = k;
  s->kpad = (k + 3) / 4 * 4;
  s->pop = pop;
  s->ld = std::max(32, (g->n + 31) / 32 * 32);
  s->ls_kernel = ls_kernel;
  s->plan = MakePlan(g->n, g->pitch, k, s->ld, s->kpad, ls_kernel, s->device);

  const size_t labels = (size_t)pop * s->ld;
  const size_t gains = labels * k;
  const size_t gb = s->GainBytes();
  const size_t next_bytes =
      s->plan.smem_state ? 0
                         : (s->plan.incremental ? (size_t)pop * IncrementalBytes(k, s->ld)
                                                : labels * (s->plan.small_k ? std::max(k, SmallKLanes(k)) : k) * gb);
  size_t bytes = 2 * labels + gains * gb + next_bytes + (size_t)pop * s->kpad * 4 + 2 * pop * 8 +
                 (size_t)pop * k * g->pitch * 4 + 2 * (size_t)pop * 4 + s->ld + sizeof(Control);
  size_t free_b = 0, total_b = 0;
  CCB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (bytes > free_b) {
    Fail(CCB_ERR_DEVICE_MEMORY, "run needs " + Mebibytes(bytes) + " of device memory, " + Mebibytes(free_b) + " free");
  }
  s->device_bytes = bytes;
  s->Alloc(s->cur_lab, labels);
  s->Alloc(s->next_lab, labels);
  uint8_t* cg = nullptr;
  s->Alloc(cg, gains * gb);
  s->cur_g = cg;
  if (!s->plan.smem_state) {
    // the global-state descents work in the slot's rows of next: cluster-major G, or packed vectors
    const size_t bytes_next = s->plan.incremental ? (size_t)pop * IncrementalBytes(k, s->ld)
                                                  : labels * (s->plan.small_k ? std::max(k, SmallKLanes(k)) : k) * gb;
    uint8_t* ng = nullptr;
    s->Alloc(ng, bytes_next);
    s->next_g = ng;
  }
  s->Alloc(s->cur_sizes, (size_t)pop * s->kpad);
  s->Alloc(s->cur_f, pop);
  s->Alloc(s->next_f, pop);
  s->Alloc(s->masks, (size_t)pop * k * g->pitch);
  s->Alloc(s->src_map, pop);
  s->Alloc(s->order, pop);
  s->Alloc(s->record_lab, s->ld);
  s->Alloc(s->ctl, 1);
  CCB_CUDA(cudaMemset(s->cur_lab, 0, labels));
  CCB_CUDA(cudaMemset(s->next_lab, 0, labels));
  CCB_CUDA(cudaMallocHost(&s->host_ctl, 2 * sizeof(Control)));
  CCB_CUDA(cudaMallocHost(&s->host_labels, std::max<size_t>(s->ld, 1)));
  CCB_CUDA(cudaEventCreateWithFlags(&s->poll_event[0], cudaEventDisableTiming));
  CCB_CUDA(cudaEventCreateWithFlags(&s->poll_event[1], cudaEventDisableTiming));

  // Shared-memory opt-in for the descent instance of this plan.
  if (s->plan.incremental) {
    CCB_CUDA(LaunchDescentIncremental(s->plan.sk, DescentArgs<int16_t>{}, 0, nullptr, true));
  } else if (s->plan.small_k) {
    CCB_CUDA(LaunchDescentSmallK(s->plan.sk, DescentArgs<int16_t>{}, 0, nullptr, true));
  } else if (s->plan.wide) {
    LaunchDescent<int32_t>(s->plan, DescentArgs<int32_t>{}, 0, nullptr, true);
  } else {
    LaunchDescent<int16_t>(s->plan, DescentArgs<int16_t>{}, 0, nullptr, true);
  }
  char text[256];
  std::snprintf(text, sizeof(text), "%s, %d threads per block, %d blocks, %zu bytes of shared memory",
                KernelName(s->plan), s->plan.threads, pop, s->plan.smem_bytes);
  s->description = text;
  return s.release();
}

void EnsureTrace(ccb_solver& s, int iterations) {
  if (iterations <= s.trace_cap) return;
  void* p = nullptr;
  CCB_CUDA(cudaMalloc(&p, (size_t)iterations * sizeof(TraceEntry)));
  s.allocations.push_back(p);
  s.trace = static_cast<TraceEntry*>(p);
  if (s.host_trace) cudaFreeHost(s.host_trace);
  CCB_CUDA(cudaMallocHost(&s.host_trace, (size_t)iterations * sizeof(TraceEntry)));
  s.trace_cap = iterations;
}

template <typename GainT>
void LaunchRebuild(ccb_solver& s, int grid, int mode, const int32_t* src_map, uint64_t stream, int iteration,
                   float prob, int first, bool check_stop, cudaStream_t st) {
  if (grid <= 0) return;
  s.timer.Time(kCatRebuild, st, [&] {
    k_rebuild<GainT, kRebuildThreads><<<grid, kRebuildThreads, 0, st>>>(
        s.graph->View(), s.Cur<GainT>(), s.next_lab, src_map, s.masks, s.k, s.kpad, s.ld, mode, stream, iteration,
        prob, first, check_stop ? s.ctl : nullptr);
  });
  CCB_CUDA(cudaGetLastError());
}

template <typename GainT>
void LaunchDescentStep(ccb_solver& s, int grid, int population, int tournament, int iteration, uint64_t stream,
                       cudaStream_t st) {
  DescentArgs<GainT> a;
  a.gr = s.graph->View();
  a.cur = s.Cur<GainT>();
  a.next = s.Next<GainT>();
  a.ctl = s.ctl;
  a.k = s.k;
  a.kpad = s.kpad;
  a.ld = s.ld;
  a.key_bits = s.plan.key_bits;
  a.population = population;
  a.tournament = tournament;
  a.iteration = iteration;
  a.select_stream = stream;
  if constexpr (std::is_same_v<GainT, int16_t>) {
    if (s.plan.small_k || s.plan.incremental) {
      cudaError_t e = cudaSuccess;
      s.timer.Time(kCatDescent, st, [&] {
        e = s.plan.incremental ? LaunchDescentIncremental(s.plan.sk, a, grid, st, false)
                               : LaunchDescentSmallK(s.plan.sk, a, grid, st, false);
      });
      CCB_CUDA(e);
      return;
    }
  }
  s.timer.Time(kCatDescent, st, [&] { LaunchDescent<GainT>(s.plan, a, grid, st, false); });
  CCB_CUDA(cudaGetLastError());
}

void LaunchRecord(ccb_solver& s, const RecordArgs& a, cudaStream_t st) {
  s.timer.Time(kCatRecord, st, [&] { k_record<kRecordThreads><<<1, kRecordThreads, 0, st>>>(a); });
  CCB_CUDA(cudaGetLastError());
}

void CopyOutLabels(ccb_solver& s, int32_t* labels_out, cudaStream_t st) {
  if (s.n > 0) CCB_CUDA(cudaMemcpyAsync(s.host_labels, s.record_lab, s.n, cudaMemcpyDeviceToHost, st));
  CCB_CUDA(cudaMemcpyAsync(s.host_ctl, s.ctl, sizeof(Control), cudaMemcpyDeviceToHost, st));
  CCB_CUDA(cudaStreamSynchronize(st));
  if (labels_out) {
    for (int v = 0; v < s.n; ++v) labels_out[v] = s.host_labels[v];
  }
}

void PrintPlan(const ccb_solver& s, size_t free_hint) {
  std::printf("  local search: %s\n  device memory: %s of %s free\n", s.description.c_str(),
              Mebibytes(s.device_bytes).c_str(), Mebibytes(free_hint).c_str());
}

template <typename GainT>
void RunPbils(ccb_solver& s, const ccb_params& p, cudaStream_t st, int32_t* labels_out, ccb_result* res) {
  const auto started = std::chrono::steady_clock::now();
  const int n = s.n, k = s.k, pop = s.pop;
  const uint64_t init_stream = StreamSeed(p.seed, kInitTag, 0);
  const uint64_t select_stream = StreamSeed(p.seed, kSelectTag, 0);
  const uint64_t perturb_stream = StreamSeed(p.seed, kPerturbTag, 0);
  const int copies = (int)(p.gww * pop);
  const bool perturb = k >= 2 && p.perturbation > 0.0;
  const float prob = (float)p.perturbation;
  const bool verbose = p.verbose != 0;
  if (verbose) {
    size_t free_b = 0, total_b = 0;
    CCB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    PrintPlan(s, free_b);
    EnsureTrace(s, std::max(p.iterations, 1));
  }
  s.timer.Reset();

  CCB_CUDA(cudaMemsetAsync(s.ctl, 0, sizeof(Control), st));
  s.timer.Time(kCatOther, st, [&] { k_mark_start<<<1, 1, 0, st>>>(s.ctl); });
  const long long total = (long long)pop * n;
  const int init_grid = (int)std::max<long long>(1, std::min<long long>(CeilDiv(total, kAuxThreads), 4096));
  s.timer.Time(kCatOther, st, [&] {
    k_init_labels<<<init_grid, kAuxThreads, 0, st>>>(s.cur_lab, pop, n, s.ld, k, init_stream);
  });
  CCB_CUDA(cudaGetLastError());
  LaunchRebuild<GainT>(s, pop, kRebuildInPlace, nullptr, 0, 0, 0.f, 0, false, st);

  RecordArgs r{};
  r.ld = s.ld;
  r.n = n;
  r.count = pop;
  r.ctl = s.ctl;
  r.record_labels = s.record_lab;
  r.early_stop = p.early_stop;
  r.copies = copies;
  r.src_map = s.src_map;
  r.order = s.order;
  r.trace = verbose ? s.trace : nullptr;
  r.time_limit_ns = p.time_limit_sec > 0 ? (unsigned long long)(p.time_limit_sec * 1e9) : 0ull;
  r.f = s.cur_f;
  r.labels = s.cur_lab;
  r.mode = kRecordInitial;
  LaunchRecord(s, r, st);
  r.f = s.next_f;
  r.labels = s.next_lab;
  r.mode = kRecordIteration;

  int chunk = 0;
  for (int it = 0; it < p.iterations; ++it) {
    LaunchDescentStep<GainT>(s, pop, pop, p.tournament, it, select_stream, st);
    r.iteration = it;
    LaunchRecord(s, r, st);
    LaunchRebuild<GainT>(s, pop, perturb ? kRebuildPerturb : kRebuildCopy, copies > 0 ? s.src_map : nullptr,
                         perturb_stream, it, prob, 0, true, st);
    if ((it + 1) % kPollChunk == 0 && it + 1 < p.iterations) {
      // Poll the stop flag one chunk behind the device: the device always has a chunk queued.
      const int slot = chunk % 2;
      if (chunk >= 1) {
        CCB_CUDA(cudaEventSynchronize(s.poll_event[1 - slot]));
        if (s.host_ctl[1 - slot].stop) break;
      }
      CCB_CUDA(cudaMemcpyAsync(&s.host_ctl[slot], s.ctl, sizeof(Control), cudaMemcpyDeviceToHost, st));
      CCB_CUDA(cudaEventRecord(s.poll_event[slot], st));
      ++chunk;
    }
  }
  CopyOutLabels(s, labels_out, st);
  const Control& c = s.host_ctl[0];
  if (c.error) Fail(CCB_ERR_STATE, "descent exceeded its move bound: inconsistent device state");
  res->objective = c.record_f;
  res->iterations_done = c.iterations_done;
  res->local_searches = (int64_t)c.iterations_done * pop;
  res->accepted_moves = (int64_t)c.moves;
  res->clusters_used = labels_out ? CountClustersUsed(labels_out, (uint32_t)n, k) : 0;
  if (!labels_out) {
    std::vector<int32_t> tmp(n);
    for (int v = 0; v < n; ++v) tmp[v] = s.host_labels[v];
    res->clusters_used = CountClustersUsed(tmp.data(), (uint32_t)n, k);
  }
  res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
  if (s.timer.enabled) s.timer.Collect(&s.stats);
  if (verbose && c.iterations_done > 0) {
    CCB_CUDA(cudaMemcpy(s.host_trace, s.trace, (size_t)c.iterations_done * sizeof(TraceEntry),
                        cudaMemcpyDeviceToHost));
    for (int i = 0; i < c.iterations_done; ++i) {
      std::printf("  iter %3d  record %lld  stall %d  %.3fs\n", i + 1, (long long)s.host_trace[i].record,
                  s.host_trace[i].stall, s.host_trace[i].t_ns * 1e-9);
    }
  }
}

template <typename GainT>
void RunNeighborhood(ccb_solver& s, const ccb_params& p, bool local_search, cudaStream_t st, int32_t* labels_out,
                     ccb_result* res) {
  const auto started = std::chrono::steady_clock::now();
  const int n = s.n;
  const int capacity = std::min(s.pop, n);
  s.timer.Reset();
  if (p.verbose) {
    size_t free_b = 0, total_b = 0;
    CCB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    PrintPlan(s, free_b);
  }
  CCB_CUDA(cudaMemsetAsync(s.ctl, 0, sizeof(Control), st));
  RecordArgs r{};
  r.ld = s.ld;
  r.n = n;
  r.ctl = s.ctl;
  r.record_labels = s.record_lab;
  r.mode = kRecordNeighborhood;
  r.f = local_search ? s.next_f : s.cur_f;
  r.labels = local_search ? s.next_lab : s.cur_lab;
  for (int first = 0; first < n; first += capacity) {
    const int count = std::min(capacity, n - first);
    LaunchRebuild<GainT>(s, count, kRebuildNeighborhood, nullptr, 0, 0, 0.f, first, false, st);
    if (local_search) LaunchDescentStep<GainT>(s, count, count, 0, 0, 0, st);
    r.count = count;
    LaunchRecord(s, r, st);
  }
  CopyOutLabels(s, labels_out, st);
  const Control& c = s.host_ctl[0];
  if (c.error) Fail(CCB_ERR_STATE, "descent exceeded its move bound: inconsistent device state");
  res->objective = c.record_f;
  res->iterations_done = 0;
  res->local_searches = local_search ? n : 0;
  res->accepted_moves = (int64_t)c.moves;
  std::vector<int32_t> tmp(n);
  for (int v = 0; v < n; ++v) tmp[v] = s.host_labels[v];
  res->clusters_used = CountClustersUsed(tmp.data(), (uint32_t)n, 2);
  res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
  if (s.timer.enabled) s.timer.Collect(&s.stats);
  if (p.verbose) std::printf("  neighborhoods %d/%d  record %lld  %.3fs\n", n, n, (long long)c.record_f, res->seconds);
}

// PBILS on an empty graph: nothing to place, every offer takes (the reference tests an empty label
// vector, cc_pbils_cpu.cpp:210), so only the iteration count moves.
void EmptyPbils(const ccb_params& p, ccb_result* res) {
  std::memset(res, 0, sizeof(*res));
  int done = 0;
  for (int it = 0; it < p.iterations; ++it) {
    ++done;
    if (0 >= p.early_stop) break;
  }
  res->iterations_done = done;
  res->local_searches = (int64_t)done * p.population;
}

void CheckSolverMatches(const ccb_solver* s, const ccb_params& p) {
  if (s == nullptr) Fail(CCB_ERR_STATE, "null solver");
  if (p.k != s->k || p.population != s->pop) {
    Fail(CCB_ERR_STATE, "solver was created for k = " + std::to_string(s->k) + ", population = " +
                            std::to_string(s->pop));
  }
}

}  // namespace

// ------------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------------
extern "C" {

const char* ccb_last_error(void) { return LastError(); }

void ccb_params_init(ccb_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->k = 2;
  p->population = 128;
  p->tournament = 5;
  p->iterations = 100;
  p->early_stop = 6;
  p->perturbation = 0.4;
  p->gww = 0.1;
  p->threads = 1;
  p->seed = 1;
  p->time_limit_sec = 0.0;
  p->verbose = 0;
  p->ls_kernel = CCB_LS_AUTO;
}

int ccb_graph_upload(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges, void* stream,
                     ccb_graph** out) {
  return Guard([&] {
    if (!out) Fail(CCB_ERR_STATE, "null output handle");
    *out = MakeGraph(bits, false, n, words_per_row, edges, static_cast<cudaStream_t>(stream));
  });
}

int ccb_graph_from_device(const uint32_t* device_bits, uint32_t n, uint32_t words_per_row, uint64_t edges,
                          void* stream, ccb_graph** out) {
  return Guard([&] {
    if (!out) Fail(CCB_ERR_STATE, "null output handle");
    *out = MakeGraph(device_bits, true, n, words_per_row, edges, static_cast<cudaStream_t>(stream));
  });
}

int ccb_graph_size(const ccb_graph* g, uint32_t* n, uint64_t* edges) {
  return Guard([&] {
    if (!g) Fail(CCB_ERR_STATE, "null graph");
    if (n) *n = (uint32_t)g->n;
    if (edges) *edges = (uint64_t)g->edges;
  });
}

void ccb_graph_destroy(ccb_graph* g) { delete g; }

int ccb_solver_create(const ccb_graph* g, const ccb_params* params, ccb_solver** out) {
  return Guard([&] {
    if (!g || !params || !out) Fail(CCB_ERR_STATE, "null argument");
    CheckParams(*params);
    CheckGpuLimits(*params, (uint32_t)g->n);
    *out = MakeSolver(g, params->k, params->population, params->ls_kernel);
  });
}

int ccb_solver_pbils(ccb_solver* s, const ccb_params* params, void* stream, int32_t* labels_out,
                     ccb_result* result) {
  return Guard([&] {
    if (!params || !result) Fail(CCB_ERR_STATE, "null argument");
    CheckParams(*params);
    CheckSolverMatches(s, *params);
    std::memset(result, 0, sizeof(*result));
    if (s->n == 0) {
      EmptyPbils(*params, result);
      return;
    }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (s->plan.wide) {
      RunPbils<int32_t>(*s, *params, st, labels_out, result);
    } else {
      RunPbils<int16_t>(*s, *params, st, labels_out, result);
    }
  });
}

int ccb_solver_neighborhood(ccb_solver* s, const ccb_params* params, int32_t local_search, void* stream,
                            int32_t* labels_out, ccb_result* result) {
  return Guard([&] {
    if (!s || !params || !result) Fail(CCB_ERR_STATE, "null argument");
    CheckNeighborhood(*params, (uint32_t)s->n);
    if (s->k != 2) Fail(CCB_ERR_STATE, "solver was created for k = " + std::to_string(s->k));
    std::memset(result, 0, sizeof(*result));
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (s->plan.wide) {
      RunNeighborhood<int32_t>(*s, *params, local_search != 0, st, labels_out, result);
    } else {
      RunNeighborhood<int16_t>(*s, *params, local_search != 0, st, labels_out, result);
    }
  });
}

const char* ccb_solver_describe(const ccb_solver* s) { return s ? s->description.c_str() : ""; }

void ccb_solver_destroy(ccb_solver* s) { delete s; }

int ccb_solver_set_profiling(ccb_solver* s, int32_t enabled) {
  return Guard([&] {
    if (!s) Fail(CCB_ERR_STATE, "null solver");
    s->timer.enabled = enabled != 0;
  });
}

int ccb_solver_stats(const ccb_solver* s, ccb_kernel_stats* stats) {
  return Guard([&] {
    if (!s || !stats) Fail(CCB_ERR_STATE, "null argument");
    *stats = s->stats;
  });
}

int ccb_pbils_solve(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges,
                    const ccb_params* params, int32_t* labels_out, ccb_result* result) {
  return Guard([&] {
    if (!params || !result) Fail(CCB_ERR_STATE, "null argument");
    const auto started = std::chrono::steady_clock::now();
    CheckParams(*params);
    CheckGpuLimits(*params, n);
    std::memset(result, 0, sizeof(*result));
    if (n == 0) {
      EmptyPbils(*params, result);
      return;
    }
    std::unique_ptr<ccb_graph> g(MakeGraph(bits, false, n, words_per_row, edges, nullptr));
    std::unique_ptr<ccb_solver> s(MakeSolver(g.get(), params->k, params->population, params->ls_kernel));
    if (s->plan.wide) {
      RunPbils<int32_t>(*s, *params, nullptr, labels_out, result);
    } else {
      RunPbils<int16_t>(*s, *params, nullptr, labels_out, result);
    }
    result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
  });
}

int ccb_neighborhood_solve(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges,
                           const ccb_params* params, int32_t local_search, int32_t* labels_out,
                           ccb_result* result) {
  return Guard([&] {
    if (!params || !result) Fail(CCB_ERR_STATE, "null argument");
    const auto started = std::chrono::steady_clock::now();
    CheckNeighborhood(*params, n);
    std::memset(result, 0, sizeof(*result));
    std::unique_ptr<ccb_graph> g(MakeGraph(bits, false, n, words_per_row, edges, nullptr));
    const int batch = std::min<int>(params->population, (int)n);
    std::unique_ptr<ccb_solver> s(MakeSolver(g.get(), 2, batch, params->ls_kernel));
    if (s->plan.wide) {
      RunNeighborhood<int32_t>(*s, *params, local_search != 0, nullptr, labels_out, result);
    } else {
      RunNeighborhood<int16_t>(*s, *params, local_search != 0, nullptr, labels_out, result);
    }
    result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
  });
}

}  // extern "C"
