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
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <tuple>
#include <new>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "ccb.h"
#include "ccb_batch.h"
#include "ccb_error.h"
#include "ccb_util.h"
#include "ccb_kernels.cuh"
#include "ccb_plans.h"
#include "ccb_rebuild_tensor.h"

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

constexpr int kAuxThreads = 256;
constexpr int kRebuildThreads = 512;
constexpr int kRebuildTileThreads = 512;  // 16 rows per tile, one per warp
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

// The device's error flag (Control::error) after a solve: kErrorMoveBound from a descent that exceeded its move
// bound, kErrorWaitTimeout from a kernel whose bounded wait on its own pipeline gave up.
void CheckDeviceError(const Control& c) {
  if (c.error == kErrorWaitTimeout) {
    Fail(CCB_ERR_TIMEOUT, "a bounded device-side wait of the tensor-core rebuild gave up");
  }
  if (c.error) Fail(CCB_ERR_STATE, "descent exceeded its move bound: inconsistent device state");
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

#include "ccb_graph.h"

namespace {

ccb_graph* MakeGraph(const uint32_t* src, bool src_on_device, uint32_t n, uint32_t words_per_row, uint64_t edges,
                     cudaStream_t stream) {
  const int words = (int)((n + 31) / 32);
  if (n > 0 && words_per_row < (uint32_t)words) Fail(CCB_ERR_INVALID, "words_per_row < ceil(n / 32)");
  if (n > 0 && src == nullptr) Fail(CCB_ERR_INVALID, "null bitset");
  std::unique_ptr<ccb_graph> g(AllocateGraph(n, stream));
  g->edges = (int64_t)edges;
  if (n > 0) {
    CCB_CUDA(cudaMemcpy2DAsync(g->bits, g->pitch * sizeof(uint32_t), src, words_per_row * sizeof(uint32_t),
                               words * sizeof(uint32_t), n,
                               src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream));
  }
  FinishGraph(*g, stream);
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
  bool packed_wide = false;  // the packed wide descent (k = 2, 3)
  bool sparse = false;       // k = 2 packed wide: the degree-proportional form (sparse graphs)
  bool smem16 = false;       // sparse k = 2 / 3: the slot's words in shared memory (int16 / 26-bit records)
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

constexpr int kMaxVerticesIncrementalWide = 65536;

// The streamed K <= 8 descent from global memory gives its state an L2 evict_last priority and the bitset rows
// evict_first when the population's state takes more than 3/8 of L2: then the rows would evict dirty state lines
// (n = 32000, k = 8, pop 128: 64 MB of state, 482 GB of DRAM write-back per launch without the hints, 37 MB with
// them, 4 % faster), while a state that fits beside the rows anyway runs 2.5 % slower with the hinted accesses
// (n = 32000, k = 3, pop 128: 32 MB).  CCB_L2_HINTS=0 / 1 forces either form (for comparisons).
bool StreamL2Hints(size_t state_bytes, const Device& dev) {
  const char* env = std::getenv("CCB_L2_HINTS");
  if (env != nullptr && (env[0] == '0' || env[0] == '1')) return env[0] == '1';
  return state_bytes * 8 > (size_t)dev.l2_bytes * 3;
}
// The streamed K <= 8 descent with its state in a thread-block cluster's shared memory when it does not fit one
// CTA, used when all the population's clusters run at once: a slot then moves ~1.8x faster than streaming its
// state from L2, but takes C SMs instead of one, so with more slots than one wave of clusters the L2 form is
// faster (n = 32000, k = 8, pop 128: 608 ms per descent launch in clusters of 4 against 322 ms streamed).
constexpr bool kClusterDescent = true;

Plan MakePlan(int n, int pitch, int k, int ld, int kpad, int ls_kernel, const Device& dev, int pop) {
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
      if (!sk.smem_state && kClusterDescent) {
        // the state spread over a cluster's shared memory instead of streaming from L2, when the population's
        // clusters fit one wave (the batched engine keeps the L2 form: its buckets are one CTA per slot)
        size_t per_cta = 0;
        const int c = StreamCluster(k, n, limit - 4096, &per_cta);
        if (c > 0 && (long long)pop * c <= dev.sms) {
          sk.cluster = c;
          sk.smem_bytes = per_cta;
        }
      }
      const size_t state_bytes = (size_t)pop * ld * 2 * SmallKLanes(k);  // packed 16-bit lanes per vertex
      sk.l2_hints = !sk.smem_state && sk.cluster == 0 && StreamL2Hints(state_bytes, dev);
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
    if (n <= 16384) {
      // kbest / kown in registers, counters in shared memory when they fit
      sk.registers = true;
      IncrementalRegsShape(n, &sk.threads, &sk.vpt);
      sk.smem_state = IncrementalRegsSmem(k, ld, sk.threads, sk.vpt, true) + 10 * 1024 <= limit;
      sk.smem_bytes = IncrementalRegsSmem(k, ld, sk.threads, sk.vpt, sk.smem_state);
    } else {
      sk.threads = 1024;
      sk.smem_state = IncrementalBytes(k, ld) + 10 * 1024 <= limit;  // the kernel's static shared memory
      sk.smem_bytes = sk.smem_state ? IncrementalBytes(k, ld) : 0;
    }
    p.incremental = true;
    p.smem_state = sk.smem_state;
    p.smem_rows = false;
    p.threads = sk.threads;
    p.smem_bytes = sk.smem_bytes;
  }
  if (p.wide && (k == 2 || k == 3) && ls_kernel == CCB_LS_AUTO) {
    // one packed word per vertex: the population's state stays in L2
    p.packed_wide = true;
    p.sk.k = k;
    p.threads = 1024;
    p.smem_state = false;
    p.smem_rows = false;
    p.smem_bytes = 0;
    return p;
  }
  if (p.wide && n <= kMaxVerticesIncrementalWide && k >= 2 && ls_kernel == CCB_LS_AUTO) {
    // cached-key descent over uint16 counters: exact while every degree < 65536
    SmallKPlan& sk = p.sk;
    sk.k = k;
    sk.threads = 1024;
    sk.smem_state = false;
    sk.smem_bytes = 0;
    p.incremental = true;
    p.smem_state = false;
    p.smem_rows = false;
    p.threads = sk.threads;
    p.smem_bytes = 0;
  }
  return p;
}

template <typename GainT, typename Key, bool S, bool R, int T>
void LaunchDescentT(const DescentArgs<GainT>& a, int grid, size_t smem, cudaStream_t st, bool configure) {
  auto kernel = k_descent<GainT, Key, S, R, T>;
  if (configure) {
    CCB_CUDA(RaiseDynamicSmem(kernel, smem));
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
  if (p.packed_wide) {
    if (p.sk.k == 3) {
      if (p.smem16) return "packed wide k = 3, degree-proportional (per-thread best of each (cluster, target) class), "
                           "26-bit records in shared memory";
      return p.sparse ? "packed wide k = 3, degree-proportional (per-thread best of each (cluster, target) class), L2"
                      : "packed wide k = 3 (three 20-bit counters and the label, 8 bytes per vertex), L2";
    }
    if (p.smem16) return "packed wide k = 2, degree-proportional (per-thread best of each cluster), int16 state in "
                         "shared memory";
    return p.sparse ? "packed wide k = 2, degree-proportional (per-thread best of each cluster), L2"
                    : "packed wide k = 2 (e = G1 - G0 and the label, 4 bytes per vertex), L2";
  }
  if (p.incremental && p.wide) return "incremental wide (n <= 65536, uint16 counters, 64-bit keys), L2";
  if (p.incremental) {
    if (p.sk.registers) {
      return p.smem_state ? "incremental 9 <= k <= 64, cached keys in registers, counters in shared memory"
                          : "incremental 9 <= k <= 64, cached keys in registers, counters in L2";
    }
    return p.smem_state ? "incremental 9 <= k <= 64, shared memory" : "incremental 9 <= k <= 64, L2";
  }
  if (p.small_k) {
    if (p.sk.registers) return p.smem_rows ? "packed k <= 8, registers, bitset in shared memory"
                                           : "packed k <= 8, registers";
    if (p.sk.cluster > 0) return "packed k <= 8, state in the distributed shared memory of a CTA cluster";
    if (p.smem_state) return "packed k <= 8, streamed from shared memory";
    return p.sk.l2_hints ? "packed k <= 8, streamed from L2 (state evict_last, rows evict_first)"
                         : "packed k <= 8, streamed from L2";
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
  int64_t* intra = nullptr;    // tiled rebuild (wide path): per-slot intra-cluster sums; null: per-slot rebuild
  int rebuild_kind = CCB_REBUILD_AUTO;
  std::unique_ptr<TensorRebuild> tensor;  // set: the wide path rebuilds G on the tensor cores
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

// The largest vertex degree of a device graph (a host copy of its degree array).
int MaxDegree(const ccb_graph& g) {
  std::vector<int32_t> d(std::max(g.n, 1));
  if (g.n > 0) CCB_CUDA(cudaMemcpy(d.data(), g.degrees, (size_t)g.n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  return g.n > 0 ? *std::max_element(d.begin(), d.end()) : 0;
}

// The sparse wide descents keep the slot's words in shared memory when they fit: k = 2 as int16 (2e + label) when
// every degree is below 16384 (|2e + 1| < 2^15), k = 3 as 26-bit records (the label and two 12-bit counter
// differences) when every degree is below 2048; else in global memory (int32 / 64-bit words).
void PlanSmem16(ccb_solver& s) {
  s.plan.smem16 = false;
  if (!(s.plan.packed_wide && s.plan.sparse && (s.k == 2 || s.k == 3))) return;
  const size_t bytes = s.k == 2 ? Wide2Smem16Bytes(s.n) : Wide3Smem26Bytes(s.n);
  // room beside the state for the kernel's static shared memory (k = 2: per-thread keys and neighbour lists, ~18 KB)
  if (bytes + (s.k == 2 ? 24 * 1024 : 4096) > (size_t)s.device.smem_optin) return;
  s.plan.smem16 = MaxDegree(*s.graph) < (s.k == 2 ? 16384 : 2048);
}

// The plan in words (ccb_solver_describe, --verbose); redone whenever the plan changes.
void Describe(ccb_solver& s) {
  char text[320];
  // the sparse wide descents size their own shared state at launch (the slot's words when they fit)
  const size_t smem = s.plan.smem16 ? (s.k == 2 ? Wide2Smem16Bytes(s.n) : Wide3Smem26Bytes(s.n)) : s.plan.smem_bytes;
  std::snprintf(text, sizeof(text), "%s, %d threads per block, %d blocks, %zu bytes of shared memory%s",
                KernelName(s.plan), s.plan.threads, s.pop * std::max(1, s.plan.sk.cluster), smem,
                s.tensor ? "; G rebuilt on the tensor cores (int8 tcgen05, TMA)" : "");
  s.description = text;
}

// CCB_REBUILD_AUTO's choice on the wide path: the tensor cores (measured at G(65536, 0.02), pop 128: the rebuild
// phase of a 50-iteration solve takes 83 ms at k = 2 and 125 ms at k = 3, against 412 / 654 ms by popcount).
constexpr bool kTensorRebuildByDefault = true;

// Whether the solver rebuilds G on the tensor cores: the tiled wide rebuild (int32 G) with n >= 128, chosen
// explicitly or by CCB_REBUILD_AUTO.
bool WantTensor(const ccb_solver& s, int kind) {
  if (s.intra == nullptr || kind == CCB_REBUILD_POPCOUNT) return false;
  if (kind == CCB_REBUILD_AUTO && !kTensorRebuildByDefault) return false;
  TensorRebuild t;
  const char* why = nullptr;
  return PlanTensorRebuild(t, s.n, s.pop * s.k, &why);
}

// Sets the rebuild kind; allocates the one-hot buffer and encodes the tensor maps when the tensor path is on.
void SetRebuild(ccb_solver& s, int kind) {
  if (kind != CCB_REBUILD_AUTO && kind != CCB_REBUILD_POPCOUNT && kind != CCB_REBUILD_TENSOR) {
    Fail(CCB_ERR_INVALID, "rebuild kind must be CCB_REBUILD_AUTO, CCB_REBUILD_POPCOUNT or CCB_REBUILD_TENSOR");
  }
  if (kind == CCB_REBUILD_TENSOR && !WantTensor(s, kind)) {
    Fail(CCB_ERR_INVALID, "the tensor-core rebuild runs on the wide path (int32 G: n > 32767 or --ls-kernel wide) "
                          "with n >= 128");
  }
  s.rebuild_kind = kind;
  if (!WantTensor(s, kind)) {
    s.tensor.reset();
    return;
  }
  if (s.tensor) return;
  std::unique_ptr<TensorRebuild> t(new TensorRebuild());
  const char* why = nullptr;
  PlanTensorRebuild(*t, s.n, s.pop * s.k, &why);
  uint8_t* z = nullptr;
  s.Alloc(z, (size_t)t->z_rows * t->kz);
  CCB_CUDA(cudaMemset(z, 0, (size_t)t->z_rows * t->kz));
  CCB_CUDA(EncodeTensorRebuild(*t, s.graph->bits, s.graph->pitch, z));
  s.device_bytes += (size_t)t->z_rows * t->kz;
  s.tensor = std::move(t);
}

ccb_solver* MakeSolver(const ccb_graph* g, int k, int pop, int ls_kernel) {
  TraceRange trace_range("ccb.solver.create");
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
  s->plan = MakePlan(g->n, g->pitch, k, s->ld, s->kpad, ls_kernel, s->device, pop);
  // k = 2, 3 wide on a sparse graph (average degree <= n / 8): work per move follows the degree, not n
  s->plan.sparse = s->plan.packed_wide && 2.0 * (double)g->edges <= (double)g->n * g->n / 8.0;
  PlanSmem16(*s);

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
  // Wide graphs do not fit L2: rebuild G with each row read once for all slots (a tile of 16 rows per block in
  // shared memory) instead of once per slot.
  if (s->plan.wide && (size_t)kRebuildTileThreads / kWarp * g->pitch * 4 + 2048 <= (size_t)s->device.smem_optin) {
    s->Alloc(s->intra, pop);
    CCB_CUDA(RaiseDynamicSmem(k_rebuild_tiles<kRebuildTileThreads>,
                              (size_t)kRebuildTileThreads / kWarp * g->pitch * 4));
  }
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
  if ((s->plan.incremental && s->plan.wide) || s->plan.packed_wide) {
    // no dynamic shared memory
  } else if (s->plan.incremental) {
    CCB_CUDA(LaunchDescentIncremental(s->plan.sk, DescentArgs<int16_t>{}, 0, nullptr, true));
  } else if (s->plan.small_k) {
    CCB_CUDA(LaunchDescentSmallK(s->plan.sk, DescentArgs<int16_t>{}, 0, nullptr, true));
  } else if (s->plan.wide) {
    LaunchDescent<int32_t>(s->plan, DescentArgs<int32_t>{}, 0, nullptr, true);
  } else {
    LaunchDescent<int16_t>(s->plan, DescentArgs<int16_t>{}, 0, nullptr, true);
  }
  SetRebuild(*s, CCB_REBUILD_AUTO);
  Describe(*s);
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
  const Control* ctl = check_stop ? s.ctl : nullptr;
  RebuildArgs<GainT> a{s.graph->View(), s.Cur<GainT>(), s.next_lab, src_map, s.masks, s.k, s.kpad, s.ld,
                       mode, stream, iteration, prob, first, ctl};
  if constexpr (std::is_same_v<GainT, int32_t>) {
    if (s.intra != nullptr) {
      a.intra = s.intra;
      const ccb_graph& g = *s.graph;
      const RebuildTilesArgs t{g.View(), s.cur_lab, s.masks, s.Cur<int32_t>().g, s.intra, grid, s.k, s.ld, mode, ctl};
      const int tiles = (g.n + kRebuildTileThreads / kWarp - 1) / (kRebuildTileThreads / kWarp);
      const size_t smem = (size_t)kRebuildTileThreads / kWarp * g.pitch * 4;
      if (s.tensor) {
        // labels, masks and sizes as above; then Z, the tensor-core contraction and f
        const Control* stop = (mode == kRebuildPerturb || mode == kRebuildCopy) ? ctl : nullptr;
        int32_t* error = reinterpret_cast<int32_t*>(reinterpret_cast<char*>(s.ctl) + offsetof(Control, error));
        cudaError_t e = cudaSuccess;
        s.timer.Time(kCatRebuild, st, [&] {
          k_rebuild<GainT, kRebuildThreads><<<grid, kRebuildThreads, 0, st>>>(a);
          e = LaunchBuildZ<uint8_t>(*s.tensor, s.cur_lab, s.ld, grid, s.k, nullptr, 0, nullptr, nullptr, stop, st);
          if (e == cudaSuccess) {
            e = LaunchTensorRebuild<uint8_t>(*s.tensor, s.Cur<int32_t>().g, s.ld, g.n, grid, s.k, s.cur_lab, s.ld,
                                             s.intra, error, stop, st);
          }
          if (e == cudaSuccess) {
            k_rebuild_finish<GainT><<<(grid + 127) / 128, 128, 0, st>>>(s.Cur<GainT>(), s.intra, grid, s.k, s.kpad,
                                                                        (int64_t)g.edges, mode, ctl);
          }
        });
        CCB_CUDA(e);
        CCB_CUDA(cudaGetLastError());
        return;
      }
      s.timer.Time(kCatRebuild, st, [&] {
        k_rebuild<GainT, kRebuildThreads><<<grid, kRebuildThreads, 0, st>>>(a);
        k_rebuild_tiles<kRebuildTileThreads><<<tiles, kRebuildTileThreads, smem, st>>>(t);
        k_rebuild_finish<GainT><<<(grid + 127) / 128, 128, 0, st>>>(s.Cur<GainT>(), s.intra, grid, s.k, s.kpad,
                                                                    (int64_t)g.edges, mode, ctl);
      });
      CCB_CUDA(cudaGetLastError());
      return;
    }
  }
  s.timer.Time(kCatRebuild, st, [&] { k_rebuild<GainT, kRebuildThreads><<<grid, kRebuildThreads, 0, st>>>(a); });
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
  } else {
    if (s.plan.packed_wide) {
      cudaError_t e = cudaSuccess;
      s.timer.Time(kCatDescent, st, [&] { e = LaunchDescentWidePacked(a, grid, s.plan.sparse, s.plan.smem16, st); });
      CCB_CUDA(e);
      return;
    }
    if (s.plan.incremental) {
      cudaError_t e = cudaSuccess;
      s.timer.Time(kCatDescent, st, [&] { e = LaunchDescentIncrementalWide(a, grid, st); });
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

// The record arguments of the iterations of a solve (Progress::Next's stall / early-stop / time rules and the GWW
// ranking; cc_pbils.hpp:69-78, cc_pbils_gpu.cu:325-345).
RecordArgs IterationRecord(const ccb_solver& s, const ccb_params& p, TraceEntry* trace) {
  RecordArgs r{};
  r.ld = s.ld;
  r.n = s.n;
  r.count = s.pop;
  r.ctl = s.ctl;
  r.record_labels = s.record_lab;
  r.early_stop = p.early_stop;
  r.copies = (int)(p.gww * s.pop);
  r.src_map = s.src_map;
  r.order = s.order;
  r.trace = trace;
  r.time_limit_ns = p.time_limit_sec > 0 ? (unsigned long long)(p.time_limit_sec * 1e9) : 0ull;
  r.f = s.next_f;
  r.labels = s.next_lab;
  r.mode = kRecordIteration;
  return r;
}

// One PBILS iteration of the plain path on `st`: select + descent, record, GWW + perturbation + rebuild
// (cc_pbils_gpu.cu:347-387).  Once the record has set the stop flag every later kernel returns at once.
template <typename GainT>
void LaunchPlainIteration(ccb_solver& s, const ccb_params& p, RecordArgs r, int it, cudaStream_t st) {
  const int copies = (int)(p.gww * s.pop);
  const bool perturb = s.k >= 2 && p.perturbation > 0.0;
  LaunchDescentStep<GainT>(s, s.pop, s.pop, p.tournament, it, StreamSeed(p.seed, kSelectTag, 0), st);
  r.iteration = it;
  LaunchRecord(s, r, st);
  LaunchRebuild<GainT>(s, s.pop, perturb ? kRebuildPerturb : kRebuildCopy, copies > 0 ? s.src_map : nullptr,
                       StreamSeed(p.seed, kPerturbTag, 0), it, (float)p.perturbation, 0, true, st);
}

template <typename GainT>
void RunPbils(ccb_solver& s, const ccb_params& p, cudaStream_t st, int32_t* labels_out, ccb_result* res) {
  TraceRange trace_range("ccb.pbils");
  const auto started = std::chrono::steady_clock::now();
  const int n = s.n, k = s.k, pop = s.pop;
  const uint64_t init_stream = StreamSeed(p.seed, kInitTag, 0);
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

  RecordArgs r = IterationRecord(s, p, verbose ? s.trace : nullptr);
  r.f = s.cur_f;
  r.labels = s.cur_lab;
  r.mode = kRecordInitial;
  LaunchRecord(s, r, st);
  r = IterationRecord(s, p, verbose ? s.trace : nullptr);

  int chunk = 0;
  for (int it = 0; it < p.iterations; ++it) {
    LaunchPlainIteration<GainT>(s, p, r, it, st);
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
  CheckDeviceError(c);
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
  TraceRange trace_range("ccb.neighborhood");
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
  CheckDeviceError(c);
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
// Batched engine: many instances, one CUDA graph per PBILS iteration, persistent bucket kernels
// ------------------------------------------------------------------------------------------------
// Device work lists of a set of instances (the batch or the server's active set): one descent bucket per
// persistent kernel instance, plus the rebuild queue over all instances.
struct WorkLists {
  struct Bucket {
    BatchShape shape;
    std::vector<int> members;  // entry indices, heaviest first
    int total = 0;
    size_t offset = 0;         // of the member list in d_lists (int32 units)
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
  };
  std::vector<Bucket> buckets;
  BatchQueue rebuild{};
  int rebuild_grid = 0;
  int32_t* d_lists = nullptr;
  size_t lists_cap = 0;
  int32_t* d_heads = nullptr;  // one queue head per bucket + one for the rebuild queue
  size_t heads_cap = 0;
  cudaEvent_t fork = nullptr;
  std::string description;

  void ReleaseBuckets() {
    for (Bucket& b : buckets) {
      if (b.stream) cudaStreamDestroy(b.stream);
      if (b.done) cudaEventDestroy(b.done);
    }
    buckets.clear();
  }
  ~WorkLists() {
    ReleaseBuckets();
    if (d_lists) cudaFree(d_lists);
    if (d_heads) cudaFree(d_heads);
    if (fork) cudaEventDestroy(fork);
  }
};

struct ccb_batch {
  struct Instance {
    const ccb_graph* graph = nullptr;
    ccb_params params{};
    std::unique_ptr<ccb_solver> solver;
    bool batched = false;  // false: solved on the plain path (k = 1, n = 0, n > 32767)
    ccb_result result{};
    std::vector<int32_t> labels;
  };
  Device device;
  std::vector<Instance> inst;
  std::vector<int> entry_of;   // instance -> entry (-1 if not batched)
  std::vector<int> batched;    // entry -> instance
  WorkLists work;
  BatchEntry* d_entries = nullptr;
  int32_t* d_active = nullptr;
  int32_t* h_active = nullptr;  // pinned, two slots
  cudaStream_t stream = nullptr;
  cudaEvent_t poll[2] = {nullptr, nullptr};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool prepared = false;
  int max_iterations = 0;
  long long replays = 0;
  double l2_share = 0.0;  // 0: persistent grids fill every SM (see BuildWorkLists)
  int engine = CCB_BATCH_LOCKSTEP;
  double wait_limit_sec = 30.0;        // flow engine: a block's idle wait gives up after this long
  std::vector<int32_t> withheld;       // per instance: its flow work is never published (fault injection)
  FlowState* d_flow = nullptr;         // per entry
  int32_t* d_flow_counters = nullptr;  // remaining per bucket, then the error flag
  int32_t* d_withheld = nullptr;       // per entry
  unsigned long long* d_t0 = nullptr;  // %globaltimer at the start of a flow run

  ~ccb_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (cudaEvent_t e : poll)
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
    if (d_entries) cudaFree(d_entries);
    if (d_active) cudaFree(d_active);
    if (h_active) cudaFreeHost(h_active);
    if (d_flow) cudaFree(d_flow);
    if (d_flow_counters) cudaFree(d_flow_counters);
    if (d_withheld) cudaFree(d_withheld);
    if (d_t0) cudaFree(d_t0);
  }
};

namespace {

// Work estimate of one slot's descent, for ordering a queue heaviest first.
double SlotWork(const ccb_solver& s) { return (double)s.n * s.n * std::max(2, std::min(s.k, 8)); }

BatchEntry MakeEntry(const ccb_solver& s, const ccb_params& p) {
  BatchEntry e{};
  DescentArgs<int16_t>& d = e.descent;
  d.gr = s.graph->View();
  d.cur = s.Cur<int16_t>();
  d.next = s.Next<int16_t>();
  d.ctl = s.ctl;
  d.k = s.k;
  d.kpad = s.kpad;
  d.ld = s.ld;
  d.key_bits = s.plan.key_bits;
  d.population = s.pop;
  d.tournament = p.tournament;
  d.iteration = 0;
  d.select_stream = StreamSeed(p.seed, kSelectTag, 0);
  const int copies = (int)(p.gww * s.pop);
  const bool perturb = s.k >= 2 && p.perturbation > 0.0;
  e.rebuild = RebuildArgs<int16_t>{s.graph->View(), s.Cur<int16_t>(), s.next_lab, copies > 0 ? s.src_map : nullptr,
                                   s.masks, s.k, s.kpad, s.ld, perturb ? kRebuildPerturb : kRebuildCopy,
                                   StreamSeed(p.seed, kPerturbTag, 0), 0, (float)p.perturbation, 0, s.ctl};
  RecordArgs& r = e.record;
  r.f = s.next_f;
  r.labels = s.next_lab;
  r.ld = s.ld;
  r.n = s.n;
  r.count = s.pop;
  r.ctl = s.ctl;
  r.record_labels = s.record_lab;
  r.mode = kRecordIteration;
  r.early_stop = p.early_stop;
  r.copies = copies;
  r.src_map = s.src_map;
  r.order = s.order;
  r.trace = nullptr;
  r.time_limit_ns = p.time_limit_sec > 0 ? (unsigned long long)(p.time_limit_sec * 1e9) : 0ull;
  e.iterations = p.iterations;
  return e;
}

std::mutex g_tuning_mutex;
std::vector<ccb_tuning_entry> g_tuning;

// The plan's batched kernel, then the first matching tuning entry applied to it.
BatchShape ShapeOfPlan(const ccb_solver& s);

BatchShape ShapeOf(const ccb_solver& s) {
  BatchShape sh = ShapeOfPlan(s);
  std::lock_guard<std::mutex> lock(g_tuning_mutex);
  for (const ccb_tuning_entry& t : g_tuning) {
    if ((t.kind >= 0 && t.kind != sh.kind) || s.n < t.n_min || s.n > t.n_max || s.k < t.k_min || s.k > t.k_max) {
      continue;
    }
    if (t.use_kind == kBatchIncremental && !s.plan.smem_state &&
        (sh.kind == kBatchIncrementalRegs || sh.kind == kBatchIncremental) &&
        (t.threads == 256 || t.threads == 512 || t.threads == 1024)) {
      sh.kind = kBatchIncremental;  // the slot's rows of `next` hold IncrementalBytes: the global-state form fits
      sh.threads = t.threads;
      sh.vpt = 4;
      sh.smem = false;
      sh.smem_bytes = 0;
    }
    sh.blocks_per_sm = std::max(0, t.blocks_per_sm);
    sh.max_slots = std::max(0, t.max_slots);
    break;
  }
  return sh;
}

BatchShape ShapeOfPlan(const ccb_solver& s) {
  BatchShape sh;
  const SmallKPlan& sk = s.plan.sk;
  sh.k = s.k;
  sh.threads = sk.threads;
  sh.vpt = sk.vpt;
  if (s.plan.incremental) {
    sh.kind = sk.registers ? kBatchIncrementalRegs : kBatchIncremental;
    sh.k = 0;
    sh.smem = sk.smem_state;
  } else if (sk.registers) {
    sh.kind = kBatchRegisters;
    sh.smem = sk.smem_rows;
  } else {
    sh.kind = kBatchStream;
    sh.smem = sk.smem_state;
  }
  sh.smem_bytes = sk.cluster > 0 ? 0 : sk.smem_bytes;  // a cluster plan's batched form streams from L2
  return sh;
}

// Global-memory state bytes per running slot of an L2-streamed bucket (0 when the state is in shared memory).
size_t L2StateBytes(const ccb_solver& s) {
  if (s.plan.incremental) return s.plan.smem_state ? 0 : (s.plan.sk.registers ? (size_t)s.k * s.ld * 2
                                                                                : IncrementalBytes(s.k, s.ld));
  if (!s.plan.sk.registers && !s.plan.smem_state) return (size_t)s.ld * SmallKLanes(s.k) * 2;
  return 0;
}

// Buckets, queues and persistent grids for the entries whose solvers are `solvers` (entry e = solvers[e]).
// Persistent grids take the resident blocks per SM at the bucket's shared memory on every SM; with l2_share > 0
// an L2-streamed bucket runs no more slots than keep their states within that share of L2 (the reference's
// ResidentBlocks rule, cc_pbils_gpu.cu:61-67) -- off by default: on B200 the batched mix measured faster with
// every SM busy.
void BuildWorkLists(WorkLists& w, const std::vector<const ccb_solver*>& solvers, const Device& dev,
                    double l2_share) {
  w.ReleaseBuckets();
  const int count = (int)solvers.size();
  std::map<std::tuple<int, int, int, int, int, int, int>, int> index;
  for (int e = 0; e < count; ++e) {
    const BatchShape sh = ShapeOf(*solvers[e]);
    const auto key = std::make_tuple(sh.kind, sh.k, sh.threads, sh.vpt, (int)sh.smem, sh.blocks_per_sm, sh.max_slots);
    auto it = index.find(key);
    if (it == index.end()) {
      it = index.emplace(key, (int)w.buckets.size()).first;
      w.buckets.emplace_back();
      w.buckets.back().shape = sh;
    }
    WorkLists::Bucket& bk = w.buckets[it->second];
    bk.shape.smem_bytes = std::max(bk.shape.smem_bytes, sh.smem_bytes);
    bk.members.push_back(e);
  }
  std::vector<int32_t> lists;
  auto add_queue = [&](std::vector<int>& members, BatchQueue& q) {
    std::sort(members.begin(), members.end(),
              [&](int x, int y) { return SlotWork(*solvers[x]) > SlotWork(*solvers[y]); });
    const size_t at = lists.size();
    for (int m : members) lists.push_back(m);
    int total = 0;
    for (int m : members) {
      lists.push_back(total);
      total += solvers[m]->pop;
    }
    lists.push_back(total);
    q = BatchQueue{};
    q.count = (int)members.size();
    q.total = total;
    return at;
  };
  std::vector<BatchQueue> queues(w.buckets.size());
  for (size_t i = 0; i < w.buckets.size(); ++i) {
    w.buckets[i].offset = add_queue(w.buckets[i].members, queues[i]);
    w.buckets[i].total = queues[i].total;
  }
  std::vector<int> all(count);
  for (int e = 0; e < count; ++e) all[e] = e;
  BatchQueue rq{};
  const size_t rebuild_at = add_queue(all, rq);
  if (lists.size() > w.lists_cap) {
    if (w.d_lists) cudaFree(w.d_lists);
    w.lists_cap = std::max<size_t>(lists.size(), 2 * w.lists_cap);
    CCB_CUDA(cudaMalloc(&w.d_lists, w.lists_cap * sizeof(int32_t)));
  }
  if (w.buckets.size() + 1 > w.heads_cap) {
    if (w.d_heads) cudaFree(w.d_heads);
    w.heads_cap = std::max<size_t>(w.buckets.size() + 1, 2 * w.heads_cap);
    CCB_CUDA(cudaMalloc(&w.d_heads, w.heads_cap * sizeof(int32_t)));
  }
  if (!lists.empty()) {
    CCB_CUDA(cudaMemcpy(w.d_lists, lists.data(), lists.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  if (w.fork == nullptr) CCB_CUDA(cudaEventCreateWithFlags(&w.fork, cudaEventDisableTiming));
  std::string desc;
  for (size_t i = 0; i < w.buckets.size(); ++i) {
    WorkLists::Bucket& bk = w.buckets[i];
    size_t state = 0;
    for (int m : bk.members) state = std::max(state, L2StateBytes(*solvers[m]));
    int per_sm = BatchDescentBlocksPerSm(bk.shape);
    if (bk.shape.blocks_per_sm > 0) per_sm = std::min(per_sm, bk.shape.blocks_per_sm);
    long long grid = (long long)per_sm * dev.sms;
    if (state > 0 && l2_share > 0.0) {
      grid = std::min<long long>(grid, std::max<long long>(1, (long long)(l2_share * dev.l2_bytes / state)));
    }
    if (bk.shape.max_slots > 0) grid = std::min<long long>(grid, bk.shape.max_slots);
    bk.shape.grid = (int)std::max<long long>(1, std::min<long long>(grid, bk.total));
    CCB_CUDA(LaunchBatchDescent(bk.shape, nullptr, BatchQueue{}, nullptr, true));
    CCB_CUDA(LaunchBatchFlow(bk.shape, nullptr, nullptr, FlowBucket{}, nullptr, true));
    CCB_CUDA(cudaStreamCreateWithFlags(&bk.stream, cudaStreamNonBlocking));
    CCB_CUDA(cudaEventCreateWithFlags(&bk.done, cudaEventDisableTiming));
    char line[200];
    std::snprintf(line, sizeof(line), "%s k=%d threads=%d vpt=%d smem=%d: %zu instances, %d slots, grid %d; ",
                  bk.shape.kind == kBatchRegisters          ? "registers"
                  : bk.shape.kind == kBatchStream           ? "stream"
                  : bk.shape.kind == kBatchIncrementalRegs  ? "incremental-registers"
                                                            : "incremental",
                  bk.shape.k, bk.shape.threads, bk.shape.vpt, (int)bk.shape.smem, bk.members.size(), bk.total,
                  bk.shape.grid);
    desc += line;
    queues[i].instances = w.d_lists + bk.offset;
    queues[i].prefix = w.d_lists + bk.offset + queues[i].count;
    queues[i].head = w.d_heads + i;
  }
  rq.instances = w.d_lists + rebuild_at;
  rq.prefix = w.d_lists + rebuild_at + rq.count;
  rq.head = w.d_heads + w.buckets.size();
  w.rebuild = rq;
  w.rebuild_grid = std::max(1, std::min(2 * dev.sms, rq.total));
  // bucket queue views are rebuilt from offsets at enqueue time
  w.description = desc;
}

// One PBILS iteration of every entry: descents (bucket kernels on parallel streams), record, rebuild with
// perturbation and GWW, advance.  `stops` (may be null) receives every entry's stop flag after the advance.
void EnqueueIteration(WorkLists& w, const BatchEntry* d_entries, int count, int32_t* d_active, int32_t* d_stops,
                      cudaStream_t st) {
  if (count == 0) return;
  CCB_CUDA(cudaMemsetAsync(w.d_heads, 0, (w.buckets.size() + 1) * sizeof(int32_t), st));
  CCB_CUDA(cudaEventRecord(w.fork, st));
  for (size_t i = 0; i < w.buckets.size(); ++i) {
    WorkLists::Bucket& bk = w.buckets[i];
    BatchQueue q{};
    q.count = (int32_t)bk.members.size();
    q.total = bk.total;
    q.instances = w.d_lists + bk.offset;
    q.prefix = w.d_lists + bk.offset + q.count;
    q.head = w.d_heads + i;
    CCB_CUDA(cudaStreamWaitEvent(bk.stream, w.fork, 0));
    CCB_CUDA(LaunchBatchDescent(bk.shape, d_entries, q, bk.stream, false));
    CCB_CUDA(cudaEventRecord(bk.done, bk.stream));
    CCB_CUDA(cudaStreamWaitEvent(st, bk.done, 0));
  }
  CCB_CUDA(LaunchBatchRecord(d_entries, count, st));
  CCB_CUDA(LaunchBatchRebuild(d_entries, w.rebuild, w.rebuild_grid, st));
  CCB_CUDA(cudaMemsetAsync(d_active, 0, sizeof(int32_t), st));
  CCB_CUDA(LaunchBatchAdvance(d_entries, count, d_active, d_stops, st));
}

void PrepareBatch(ccb_batch& b) {
  if (b.prepared) return;
  if (b.stream == nullptr) CCB_CUDA(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking));
  b.entry_of.assign(b.inst.size(), -1);
  b.batched.clear();
  std::vector<BatchEntry> entries;
  std::vector<const ccb_solver*> solvers;
  for (size_t i = 0; i < b.inst.size(); ++i) {
    ccb_batch::Instance& in = b.inst[i];
    if (in.graph->n == 0) continue;
    in.solver.reset(MakeSolver(in.graph, in.params.k, in.params.population, CCB_LS_AUTO));
    const Plan& pl = in.solver->plan;
    in.batched = !pl.wide && (pl.small_k || pl.incremental);
    if (!in.batched) continue;
    b.entry_of[i] = (int)entries.size();
    b.batched.push_back((int)i);
    entries.push_back(MakeEntry(*in.solver, in.params));
    solvers.push_back(in.solver.get());
    b.max_iterations = std::max(b.max_iterations, in.params.iterations);
  }
  const int count = (int)entries.size();
  BuildWorkLists(b.work, solvers, b.device, b.l2_share);
  CCB_CUDA(cudaMalloc(&b.d_entries, std::max<size_t>(1, entries.size()) * sizeof(BatchEntry)));
  CCB_CUDA(cudaMalloc(&b.d_active, sizeof(int32_t)));
  CCB_CUDA(cudaMallocHost(&b.h_active, 2 * sizeof(int32_t)));
  if (!entries.empty()) {
    CCB_CUDA(cudaMemcpy(b.d_entries, entries.data(), entries.size() * sizeof(BatchEntry), cudaMemcpyHostToDevice));
  }
  for (cudaEvent_t& e : b.poll) CCB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  if (b.engine == CCB_BATCH_FLOW) {
    CCB_CUDA(cudaMalloc(&b.d_flow, std::max(1, count) * sizeof(FlowState)));
    CCB_CUDA(cudaMalloc(&b.d_flow_counters, (3 * b.work.buckets.size() + 1) * sizeof(int32_t)));
    CCB_CUDA(cudaMalloc(&b.d_t0, sizeof(unsigned long long)));
    std::vector<int32_t> held(std::max(1, count), 0);
    for (int e = 0; e < count; ++e) held[e] = b.withheld[b.batched[e]];
    CCB_CUDA(cudaMalloc(&b.d_withheld, held.size() * sizeof(int32_t)));
    CCB_CUDA(cudaMemcpy(b.d_withheld, held.data(), held.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    b.prepared = true;
    return;
  }
  // One PBILS iteration of every instance, captured once as a graph and replayed.
  if (count > 0) {
    CCB_CUDA(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal));
    EnqueueIteration(b.work, b.d_entries, count, b.d_active, nullptr, b.stream);
    CCB_CUDA(cudaStreamEndCapture(b.stream, &b.graph));
    CCB_CUDA(cudaGraphInstantiate(&b.exec, b.graph, 0));
  }
  b.prepared = true;
}

// Initial population, rebuild and record of one instance (as RunPbils does before its loop).
template <typename GainT>
void EnqueueInit(ccb_solver& s, const ccb_params& p, cudaStream_t st) {
  CCB_CUDA(cudaMemsetAsync(s.ctl, 0, sizeof(Control), st));
  k_mark_start<<<1, 1, 0, st>>>(s.ctl);
  const long long total = (long long)s.pop * s.n;
  const int init_grid = (int)std::max<long long>(1, std::min<long long>(CeilDiv(total, kAuxThreads), 4096));
  k_init_labels<<<init_grid, kAuxThreads, 0, st>>>(s.cur_lab, s.pop, s.n, s.ld, s.k, StreamSeed(p.seed, kInitTag, 0));
  CCB_CUDA(cudaGetLastError());
  LaunchRebuild<GainT>(s, s.pop, kRebuildInPlace, nullptr, 0, 0, 0.f, 0, false, st);
  RecordArgs r{};
  r.f = s.cur_f;
  r.labels = s.cur_lab;
  r.ld = s.ld;
  r.n = s.n;
  r.count = s.pop;
  r.ctl = s.ctl;
  r.record_labels = s.record_lab;
  r.mode = kRecordInitial;
  LaunchRecord(s, r, st);
  if (p.iterations <= 0) {
    // nothing to iterate: mark the instance stopped before the first graph replay
    const int one = 1;
    CCB_CUDA(cudaMemcpyAsync(&s.ctl->stop, &one, sizeof(one), cudaMemcpyHostToDevice, st));
  }
}

// The flow engine's run: one persistent kernel per bucket, each on its stream, carrying its instances through
// all their iterations; returns the device clock at the start (for per-instance completion times).
unsigned long long RunFlow(ccb_batch& b, std::vector<FlowState>& states) {
  const cudaStream_t st = b.stream;
  const int count = (int)b.batched.size();
  WorkLists& w = b.work;
  const int nb = (int)w.buckets.size();
  CCB_CUDA(cudaMemsetAsync(b.d_flow_counters, 0, (3 * nb + 1) * sizeof(int32_t), st));
  std::vector<FlowBucket> fb(nb);
  for (int i = 0; i < nb; ++i) {
    fb[i].members = w.d_lists + w.buckets[i].offset;
    fb[i].count = (int32_t)w.buckets[i].members.size();
    fb[i].remaining = b.d_flow_counters + 3 * i;
    fb[i].error = b.d_flow_counters + 3 * nb;
    fb[i].idle_limit_ns = (unsigned long long)(std::max(1e-3, b.wait_limit_sec) * 1e9);
    CCB_CUDA(LaunchFlowInit(b.d_entries, b.d_flow, fb[i], b.d_withheld, st));
  }
  k_clock<<<1, 1, 0, st>>>(b.d_t0);
  CCB_CUDA(cudaGetLastError());
  CCB_CUDA(cudaEventRecord(w.fork, st));
  for (int i = 0; i < nb; ++i) {
    WorkLists::Bucket& bk = w.buckets[i];
    CCB_CUDA(cudaStreamWaitEvent(bk.stream, w.fork, 0));
    CCB_CUDA(LaunchBatchFlow(bk.shape, b.d_entries, b.d_flow, fb[i], bk.stream, false));
    CCB_CUDA(cudaEventRecord(bk.done, bk.stream));
    CCB_CUDA(cudaStreamWaitEvent(st, bk.done, 0));
  }
  int32_t error = 0;
  unsigned long long t0 = 0;
  states.resize(std::max(1, count));
  CCB_CUDA(cudaMemcpyAsync(&error, b.d_flow_counters + 3 * nb, sizeof(error), cudaMemcpyDeviceToHost, st));
  CCB_CUDA(cudaMemcpyAsync(&t0, b.d_t0, sizeof(t0), cudaMemcpyDeviceToHost, st));
  CCB_CUDA(cudaMemcpyAsync(states.data(), b.d_flow, count * sizeof(FlowState), cudaMemcpyDeviceToHost, st));
  CCB_CUDA(cudaStreamSynchronize(st));
  if (error == kErrorWaitTimeout) {
    Fail(CCB_ERR_TIMEOUT, "batched flow engine: a block found no work to claim for the wait limit (" +
                              std::to_string(b.wait_limit_sec) + " s) while instances were unfinished");
  }
  for (int e = 0; e < count; ++e) {
    if (!states[e].finished) Fail(CCB_ERR_STATE, "batched flow engine: the run ended with an unfinished instance");
  }
  return t0;
}

void RunBatch(ccb_batch& b) {
  TraceRange trace_range("ccb.batch.run");
  const auto started = std::chrono::steady_clock::now();
  PrepareBatch(b);
  const cudaStream_t st = b.stream;
  for (int e = 0; e < (int)b.batched.size(); ++e) {
    ccb_batch::Instance& in = b.inst[b.batched[e]];
    EnqueueInit<int16_t>(*in.solver, in.params, st);
  }
  std::vector<FlowState> states;
  unsigned long long flow_t0 = 0;
  if (b.engine == CCB_BATCH_FLOW && !b.batched.empty()) flow_t0 = RunFlow(b, states);
  if (b.engine == CCB_BATCH_LOCKSTEP && b.exec != nullptr) {
    int chunk = 0;
    for (int r = 0; r < b.max_iterations; ++r) {
      CCB_CUDA(cudaGraphLaunch(b.exec, st));
      ++b.replays;
      if ((r + 1) % kPollChunk == 0 && r + 1 < b.max_iterations) {
        const int slot = chunk % 2;
        if (chunk >= 1) {
          CCB_CUDA(cudaEventSynchronize(b.poll[1 - slot]));
          if (b.h_active[1 - slot] == 0) break;
        }
        CCB_CUDA(cudaMemcpyAsync(&b.h_active[slot], b.d_active, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        CCB_CUDA(cudaEventRecord(b.poll[slot], st));
        ++chunk;
      }
    }
  }
  CCB_CUDA(cudaStreamSynchronize(st));
  const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
  for (size_t i = 0; i < b.inst.size(); ++i) {
    ccb_batch::Instance& in = b.inst[i];
    std::memset(&in.result, 0, sizeof(in.result));
    in.labels.assign(in.graph->n, 0);
    if (in.graph->n == 0) {
      EmptyPbils(in.params, &in.result);
      continue;
    }
    if (!in.batched) {
      RunPbils<int16_t>(*in.solver, in.params, st, in.labels.data(), &in.result);
      continue;
    }
    ccb_solver& s = *in.solver;
    CopyOutLabels(s, in.labels.data(), st);
    const Control& c = s.host_ctl[0];
    CheckDeviceError(c);
    in.result.objective = c.record_f;
    in.result.iterations_done = c.iterations_done;
    in.result.local_searches = (int64_t)c.iterations_done * s.pop;
    in.result.accepted_moves = (int64_t)c.moves;
    in.result.clusters_used = CountClustersUsed(in.labels.data(), (uint32_t)s.n, s.k);
    in.result.seconds = seconds;
    if (b.engine == CCB_BATCH_FLOW) {  // this instance's own completion, from the start of the run
      const FlowState& f = states[b.entry_of[i]];
      in.result.seconds = f.t_done_ns > flow_t0 ? (double)(f.t_done_ns - flow_t0) * 1e-9 : 0.0;
    }
  }
}

}  // namespace

// ------------------------------------------------------------------------------------------------
// Serving engine: continuous batching at iteration granularity
// ------------------------------------------------------------------------------------------------
struct ccb_server {
  struct Request {
    int id = 0;
    int source = 0;  // 0: host bitset, 1: Erdős–Rényi generated on the device, 2: planted generated on the device
    std::vector<uint32_t> bits;
    uint32_t n = 0, words = 0;
    uint64_t edges = 0;
    double density = 0, p_in = 0, p_out = 0, flip = 0;
    int parts = 2;
    uint64_t graph_seed = 0;
    ccb_params params{};
    size_t bytes = 0;  // device-memory estimate used for admission
  };
  struct Active {
    Request req;
    std::unique_ptr<ccb_graph> graph;
    std::unique_ptr<ccb_solver> solver;
    std::chrono::steady_clock::time_point admitted;
    bool cancel = false;  // stop it before its lane's next iteration; report CCB_ERR_CANCELLED
  };
  struct Done {
    int status = CCB_OK;
    std::string error;
    ccb_result result{};
    std::vector<int32_t> labels;
  };
  // A request the batched kernels do not take (wide: n > 32767; k = 1), solved by the plain path's kernels on a
  // stream of its own that the server loop steps a chunk of iterations at a time, between the lanes' iterations.
  struct Wide {
    Active a;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    Control* h_ctl = nullptr;  // pinned: the control block after the last chunk
    int next = 0;              // first iteration not yet enqueued
    bool in_flight = false;
    ~Wide() {
      if (stream) cudaStreamSynchronize(stream);
      if (h_ctl) cudaFreeHost(h_ctl);
      if (done) cudaEventDestroy(done);
      if (stream) cudaStreamDestroy(stream);
    }
  };
  static constexpr int kWideChunk = 4;
  Device device;
  size_t budget = 0;
  int max_active = 0;
  size_t in_use = 0;
  int next_id = 0;
  std::deque<Request> queue;
  // Requests in the batched iterations run in lanes by size (n <= 1024, 2048, 4096, 8192, larger).  Each lane steps
  // on a stream of its own, so while a lane of large requests runs one iteration, a lane of small ones runs
  // many, and small requests finish in the time their own work takes.
  struct Lane {
    std::vector<Active> active;  // entry order of the lane's device table
    WorkLists work;
    BatchEntry* d_entries = nullptr;
    size_t entries_cap = 0;
    int32_t* d_active = nullptr;
    int32_t* d_stops = nullptr;
    int32_t* h_stops = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    bool dirty = true;
    bool in_flight = false;
    int launched = 0;  // entries of the iteration in flight (later admissions are appended behind them)
    ~Lane() {
      if (stream) cudaStreamSynchronize(stream);
      active.clear();
      if (d_entries) cudaFree(d_entries);
      if (d_active) cudaFree(d_active);
      if (d_stops) cudaFree(d_stops);
      if (h_stops) cudaFreeHost(h_stops);
      if (done) cudaEventDestroy(done);
      if (stream) cudaStreamDestroy(stream);
    }
  };
  static constexpr int kLanes = 5;
  Lane lanes[kLanes];
  std::unordered_map<int, Done> done;
  cudaStream_t stream = nullptr;  // admission: graph upload or generation, solver initialisation
  long long steps = 0;
  std::vector<std::unique_ptr<Wide>> wides;
  int max_wides = 4;

  static int LaneOf(uint32_t n) { return n <= 1024 ? 0 : n <= 2048 ? 1 : n <= 4096 ? 2 : n <= 8192 ? 3 : 4; }
  int ActiveCount() const {
    size_t c = wides.size();
    for (const Lane& l : lanes) c += l.active.size();
    return (int)c;
  }

  ~ccb_server() {
    wides.clear();
    for (Lane& L : lanes) {
      if (L.stream) cudaStreamSynchronize(L.stream);
    }
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// Device bytes of a request: its graph rows and degrees plus the solver's population buffers.
size_t RequestBytes(const ccb_server& sv, uint32_t n, const ccb_params& p) {
  const int words = (int)((n + 31) / 32);
  const int pitch = std::max(4, (words + 3) / 4 * 4);
  const size_t graph = (size_t)std::max<uint32_t>(n, 1) * pitch * 4 + (size_t)std::max<uint32_t>(n, 1) * 4;
  const int ld = std::max(32, ((int)n + 31) / 32 * 32);
  const int kpad = (p.k + 3) / 4 * 4;
  const Plan plan = MakePlan((int)n, pitch, p.k, ld, kpad, CCB_LS_AUTO, sv.device, p.population);
  const size_t labels = (size_t)p.population * ld;
  const size_t gb = plan.wide ? 4 : 2;
  const size_t next = plan.smem_state ? 0
                      : plan.incremental ? (size_t)p.population * IncrementalBytes(p.k, ld)
                                         : labels * (plan.small_k ? std::max(p.k, SmallKLanes(p.k)) : p.k) * gb;
  return graph + 2 * labels + labels * p.k * gb + next + (size_t)p.population * kpad * 4 + 2 * (size_t)p.population * 8 +
         (size_t)p.population * p.k * pitch * 4 + 2 * (size_t)p.population * 4 + ld + sizeof(Control);
}

// Sets up the plain solve of an admitted request on a stream of its own (its memory stays charged to the budget
// until it is retired); the server loop then enqueues its iterations a chunk at a time.
void StartWide(ccb_server& sv, ccb_server::Active&& a) {
  std::unique_ptr<ccb_server::Wide> w(new ccb_server::Wide());
  w->a = std::move(a);
  CCB_CUDA(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
  CCB_CUDA(cudaEventCreateWithFlags(&w->done, cudaEventDisableTiming));
  CCB_CUDA(cudaMallocHost(&w->h_ctl, sizeof(Control)));
  std::memset(w->h_ctl, 0, sizeof(Control));  // read before the first chunk's copy lands: not stopped
  ccb_solver& s = *w->a.solver;
  if (s.plan.wide) {
    EnqueueInit<int32_t>(s, w->a.req.params, w->stream);
  } else {
    EnqueueInit<int16_t>(s, w->a.req.params, w->stream);
  }
  sv.in_use += w->a.req.bytes;
  sv.wides.push_back(std::move(w));
}

// The next chunk of iterations of every idle wide request, each followed by a copy of its control block.
void LaunchWides(ccb_server& sv) {
  for (auto& wp : sv.wides) {
    ccb_server::Wide& w = *wp;
    if (w.in_flight || w.a.cancel) continue;
    ccb_solver& s = *w.a.solver;
    const ccb_params& p = w.a.req.params;
    const int last = std::min(p.iterations, w.next + ccb_server::kWideChunk);
    const RecordArgs r = IterationRecord(s, p, nullptr);
    for (int it = w.next; it < last; ++it) {
      if (s.plan.wide) {
        LaunchPlainIteration<int32_t>(s, p, r, it, w.stream);
      } else {
        LaunchPlainIteration<int16_t>(s, p, r, it, w.stream);
      }
    }
    w.next = last;
    CCB_CUDA(cudaMemcpyAsync(w.h_ctl, s.ctl, sizeof(Control), cudaMemcpyDeviceToHost, w.stream));
    CCB_CUDA(cudaEventRecord(w.done, w.stream));
    w.in_flight = true;
  }
}

// Retires the wide requests whose chunk completed and that stopped (or were cancelled); returns whether any chunk
// completed.
bool RetireWides(ccb_server& sv, std::vector<int>& finished) {
  bool any = false;
  for (size_t i = 0; i < sv.wides.size();) {
    ccb_server::Wide& w = *sv.wides[i];
    if (w.in_flight) {
      const cudaError_t q = cudaEventQuery(w.done);
      if (q == cudaErrorNotReady) {
        ++i;
        continue;
      }
      CCB_CUDA(q);
      w.in_flight = false;
      any = true;
    }
    const ccb_params& p = w.a.req.params;
    if (!w.a.cancel && !w.h_ctl->stop && w.next < p.iterations) {
      ++i;
      continue;
    }
    if (w.a.cancel) {
      CCB_CUDA(cudaStreamSynchronize(w.stream));
      ccb_server::Done d;
      d.status = CCB_ERR_CANCELLED;
      d.error = "request cancelled";
      sv.done[w.a.req.id] = std::move(d);
    } else {
      ccb_solver& s = *w.a.solver;
      std::vector<int32_t> labels(s.n);
      CopyOutLabels(s, labels.data(), w.stream);
      const Control& c = s.host_ctl[0];
      ccb_server::Done d;
      try {
        CheckDeviceError(c);
        d.result.objective = c.record_f;
        d.result.iterations_done = c.iterations_done;
        d.result.local_searches = (int64_t)c.iterations_done * s.pop;
        d.result.accepted_moves = (int64_t)c.moves;
        d.result.clusters_used = CountClustersUsed(labels.data(), (uint32_t)s.n, s.k);
        d.result.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - w.a.admitted).count();
        d.labels = std::move(labels);
      } catch (const Failure& f) {
        d.status = f.status;
        d.error = f.message;
      }
      sv.done[w.a.req.id] = std::move(d);
    }
    finished.push_back(w.a.req.id);
    sv.in_use -= w.a.req.bytes;
    sv.wides.erase(sv.wides.begin() + i);
    any = true;
  }
  return any;
}

void Finish(ccb_server& sv, ccb_server::Active& a, const ccb_result& r, std::vector<int32_t> labels) {
  ccb_server::Done d;
  d.result = r;
  d.result.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - a.admitted).count();
  d.labels = std::move(labels);
  sv.done[a.req.id] = std::move(d);
}

// Whether a request runs in the batched iterations (else stepped alone on its stream): the plan's narrow small-k or
// incremental descents.
bool BatchedKernelsTake(const ccb_server& sv, const ccb_server::Request& r) {
  const int words = (int)((r.n + 31) / 32);
  const int pitch = std::max(4, (words + 3) / 4 * 4);
  const int ld = std::max(32, ((int)r.n + 31) / 32 * 32);
  const Plan pl = MakePlan((int)r.n, pitch, r.params.k, ld, (r.params.k + 3) / 4 * 4, CCB_LS_AUTO, sv.device,
                           r.params.population);
  return !pl.wide && (pl.small_k || pl.incremental);
}

// Admits queued requests (FIFO) while the device-memory budget and the active-slot cap allow; a request
// larger than the whole budget is admitted alone.  Requests the batched kernels do not take (n = 0, k = 1,
// n > 32767) are solved on admission on the plain path.
void Admit(ccb_server& sv) {
  bool admitted = false;
  while (!sv.queue.empty() && sv.ActiveCount() < sv.max_active) {
    ccb_server::Request& r = sv.queue.front();
    if (sv.in_use + r.bytes > sv.budget && sv.ActiveCount() > 0) break;
    if ((int)sv.wides.size() >= sv.max_wides && r.n > 0 && !BatchedKernelsTake(sv, r)) break;
    ccb_server::Active a;
    a.admitted = std::chrono::steady_clock::now();
    a.req = std::move(r);
    sv.queue.pop_front();
    const ccb_server::Request& q = a.req;
    try {
      if (q.source == 0) {
        a.graph.reset(MakeGraph(q.bits.data(), false, q.n, q.words, q.edges, sv.stream));
        a.req.bits.clear();
        a.req.bits.shrink_to_fit();
      } else {
        ccb_graph* g = nullptr;
        const int status =
            q.source == 1 ? ccb_graph_generate_erdos_renyi(q.n, q.density, q.graph_seed, sv.stream, &g)
                          : ccb_graph_generate_planted(q.n, q.parts, 0, q.p_in, q.p_out, q.flip, q.graph_seed, sv.stream,
                                                       &g, nullptr);
        if (status != CCB_OK) Fail(status, LastError());
        a.graph.reset(g);
      }
      if (q.n == 0) {
        ccb_result r0{};
        EmptyPbils(q.params, &r0);
        Finish(sv, a, r0, {});
        continue;
      }
      a.solver.reset(MakeSolver(a.graph.get(), q.params.k, q.params.population, CCB_LS_AUTO));
      const Plan& pl = a.solver->plan;
      if (pl.wide || !(pl.small_k || pl.incremental)) {
        CCB_CUDA(cudaStreamSynchronize(sv.stream));  // the graph is complete before another stream reads it
        StartWide(sv, std::move(a));
        continue;
      }
      EnqueueInit<int16_t>(*a.solver, q.params, sv.stream);
    } catch (const Failure& f) {
      // the request fails alone (its graph or buffers could not be made): ccb_server_result reports the error
      ccb_server::Done d;
      d.status = f.status;
      d.error = f.message;
      sv.done[q.id] = std::move(d);
      continue;
    }
    sv.in_use += q.bytes;
    ccb_server::Lane& lane = sv.lanes[ccb_server::LaneOf(q.n)];
    lane.active.push_back(std::move(a));
    lane.dirty = true;
    admitted = true;
  }
  // the lanes' streams read what admission wrote on its stream
  if (admitted) CCB_CUDA(cudaStreamSynchronize(sv.stream));
}

// One iteration of every request of the lane, enqueued on the lane's stream (its device table and work lists
// rebuilt first if its set of requests changed); the stop flags come back to pinned memory behind it.
void LaunchLane(ccb_server::Lane& L, const Device& device) {
  const int count = (int)L.active.size();
  if (L.dirty) {
    std::vector<BatchEntry> entries;
    std::vector<const ccb_solver*> solvers;
    for (ccb_server::Active& a : L.active) {
      entries.push_back(MakeEntry(*a.solver, a.req.params));
      solvers.push_back(a.solver.get());
    }
    if ((size_t)count > L.entries_cap) {
      if (L.d_entries) cudaFree(L.d_entries);
      if (L.d_stops) cudaFree(L.d_stops);
      if (L.h_stops) cudaFreeHost(L.h_stops);
      L.entries_cap = std::max<size_t>(count, 2 * L.entries_cap);
      CCB_CUDA(cudaMalloc(&L.d_entries, L.entries_cap * sizeof(BatchEntry)));
      CCB_CUDA(cudaMalloc(&L.d_stops, L.entries_cap * sizeof(int32_t)));
      CCB_CUDA(cudaMallocHost(&L.h_stops, L.entries_cap * sizeof(int32_t)));
    }
    CCB_CUDA(cudaMemcpyAsync(L.d_entries, entries.data(), count * sizeof(BatchEntry), cudaMemcpyHostToDevice,
                             L.stream));
    CCB_CUDA(cudaStreamSynchronize(L.stream));
    BuildWorkLists(L.work, solvers, device, 0.0);
    L.dirty = false;
  }
  static const int32_t kStop = 1;
  for (ccb_server::Active& a : L.active) {
    if (a.cancel) {  // every kernel of the iteration skips it; the advance reports it stopped
      CCB_CUDA(cudaMemcpyAsync(&a.solver->ctl->stop, &kStop, sizeof(int32_t), cudaMemcpyHostToDevice, L.stream));
    }
  }
  EnqueueIteration(L.work, L.d_entries, count, L.d_active, L.d_stops, L.stream);
  CCB_CUDA(cudaMemcpyAsync(L.h_stops, L.d_stops, count * sizeof(int32_t), cudaMemcpyDeviceToHost, L.stream));
  CCB_CUDA(cudaEventRecord(L.done, L.stream));
  L.in_flight = true;
  L.launched = count;
}

// After the lane's iteration completed: results of the requests that stopped, their memory back to the budget.
void RetireLane(ccb_server& sv, ccb_server::Lane& L, std::vector<int>& finished) {
  L.in_flight = false;
  for (int e = L.launched - 1; e >= 0; --e) {
    if (!L.h_stops[e]) continue;
    ccb_server::Active& a = L.active[e];
    if (a.cancel) {
      ccb_server::Done d;
      d.status = CCB_ERR_CANCELLED;
      d.error = "request cancelled";
      sv.done[a.req.id] = std::move(d);
      finished.push_back(a.req.id);
      sv.in_use -= a.req.bytes;
      L.active.erase(L.active.begin() + e);
      L.dirty = true;
      continue;
    }
    ccb_solver& s = *a.solver;
    std::vector<int32_t> labels(s.n);
    CopyOutLabels(s, labels.data(), L.stream);
    const Control& c = s.host_ctl[0];
    CheckDeviceError(c);
    ccb_result r{};
    r.objective = c.record_f;
    r.iterations_done = c.iterations_done;
    r.local_searches = (int64_t)c.iterations_done * s.pop;
    r.accepted_moves = (int64_t)c.moves;
    r.clusters_used = CountClustersUsed(labels.data(), (uint32_t)s.n, s.k);
    Finish(sv, a, r, std::move(labels));
    finished.push_back(a.req.id);
    sv.in_use -= a.req.bytes;
    L.active.erase(L.active.begin() + e);
    L.dirty = true;
  }
}

void ServerStep(ccb_server& sv, int32_t* finished_ids, int32_t capacity, int32_t* finished_count) {
  TraceRange trace_range("ccb.server.step");
  const size_t done_before = sv.done.size();
  std::vector<int> newly;
  // ids finished on the plain path during admission
  std::vector<int> before_ids;
  before_ids.reserve(sv.done.size());
  for (const auto& kv : sv.done) before_ids.push_back(kv.first);
  RetireWides(sv, newly);
  Admit(sv);
  if (sv.done.size() != done_before + newly.size()) {
    std::sort(before_ids.begin(), before_ids.end());
    for (const auto& kv : sv.done)
      if (!std::binary_search(before_ids.begin(), before_ids.end(), kv.first) &&
          std::find(newly.begin(), newly.end(), kv.first) == newly.end())
        newly.push_back(kv.first);
  }
  bool any = false;
  for (ccb_server::Lane& L : sv.lanes) {
    if (!L.in_flight && !L.active.empty()) LaunchLane(L, sv.device);
    any |= L.in_flight;
  }
  LaunchWides(sv);
  for (const auto& w : sv.wides) any |= w->in_flight;
  if (any) {
    // wait until at least one lane finished its iteration or one wide request its chunk (bounded: every kernel
    // of an iteration ends)
    for (bool got = false; !got;) {
      for (ccb_server::Lane& L : sv.lanes) {
        if (!L.in_flight) continue;
        const cudaError_t q = cudaEventQuery(L.done);
        if (q == cudaErrorNotReady) continue;
        CCB_CUDA(q);
        RetireLane(sv, L, newly);
        got = true;
      }
      got |= RetireWides(sv, newly);
      if (!got) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    ++sv.steps;
  }
  if (finished_count) *finished_count = (int32_t)newly.size();
  if (finished_ids) {
    for (int i = 0; i < (int)newly.size() && i < capacity; ++i) finished_ids[i] = newly[i];
  }
}

int Submit(ccb_server* sv, ccb_server::Request&& r, int32_t* id_out) {
  return Guard([&] {
    if (!sv) Fail(CCB_ERR_STATE, "null server");
    CheckParams(r.params);
    CheckGpuLimits(r.params, r.n);
    r.id = sv->next_id++;
    r.bytes = RequestBytes(*sv, r.n, r.params);
    if (id_out) *id_out = r.id;
    sv->queue.push_back(std::move(r));
  });
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

int ccb_solver_set_rebuild(ccb_solver* s, int32_t kind) {
  return Guard([&] {
    if (!s) Fail(CCB_ERR_STATE, "null solver");
    SetRebuild(*s, kind);
    Describe(*s);
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

int ccb_batch_create(ccb_batch** out) {
  return Guard([&] {
    if (!out) Fail(CCB_ERR_STATE, "null output handle");
    std::unique_ptr<ccb_batch> b(new ccb_batch());
    b->device = Device::Current();
    *out = b.release();
  });
}

int ccb_batch_add(ccb_batch* b, const ccb_graph* g, const ccb_params* params, int32_t* id_out) {
  return Guard([&] {
    if (!b || !g || !params) Fail(CCB_ERR_STATE, "null argument");
    if (b->prepared) Fail(CCB_ERR_STATE, "batch already prepared: create a new batch to add instances");
    CheckParams(*params);
    CheckGpuLimits(*params, (uint32_t)g->n);
    ccb_batch::Instance in;
    in.graph = g;
    in.params = *params;
    b->inst.push_back(std::move(in));
    b->withheld.push_back(0);
    if (id_out) *id_out = (int32_t)b->inst.size() - 1;
  });
}

int ccb_batch_run(ccb_batch* b) {
  return Guard([&] {
    if (!b) Fail(CCB_ERR_STATE, "null batch");
    RunBatch(*b);
  });
}

int ccb_batch_result(const ccb_batch* b, int32_t id, int32_t* labels_out, ccb_result* result) {
  return Guard([&] {
    if (!b || !result) Fail(CCB_ERR_STATE, "null argument");
    if (id < 0 || id >= (int32_t)b->inst.size()) Fail(CCB_ERR_STATE, "no such instance");
    const ccb_batch::Instance& in = b->inst[id];
    *result = in.result;
    if (labels_out && !in.labels.empty()) std::memcpy(labels_out, in.labels.data(), in.labels.size() * 4);
  });
}

int ccb_batch_set_engine(ccb_batch* b, int32_t engine, double wait_limit_sec) {
  return Guard([&] {
    if (!b) Fail(CCB_ERR_STATE, "null batch");
    if (b->prepared) Fail(CCB_ERR_STATE, "batch already prepared: set the engine before the first run");
    if (engine != CCB_BATCH_FLOW && engine != CCB_BATCH_LOCKSTEP) Fail(CCB_ERR_INVALID, "unknown batch engine");
    if (wait_limit_sec < 0) Fail(CCB_ERR_INVALID, "wait limit must be >= 0");
    b->engine = engine;
    b->wait_limit_sec = wait_limit_sec > 0 ? wait_limit_sec : 30.0;
  });
}

int ccb_batch_withhold(ccb_batch* b, int32_t id) {
  return Guard([&] {
    if (!b) Fail(CCB_ERR_STATE, "null batch");
    if (b->prepared) Fail(CCB_ERR_STATE, "batch already prepared");
    if (id < 0 || id >= (int32_t)b->inst.size()) Fail(CCB_ERR_STATE, "no such instance");
    b->withheld[id] = 1;
  });
}

const char* ccb_batch_describe(const ccb_batch* b) { return b ? b->work.description.c_str() : ""; }

void ccb_batch_destroy(ccb_batch* b) { delete b; }

int ccb_tuning_set(const ccb_tuning_entry* entries, int32_t count) {
  return Guard([&] {
    if (count < 0 || (count > 0 && !entries)) Fail(CCB_ERR_INVALID, "bad tuning table");
    std::lock_guard<std::mutex> lock(g_tuning_mutex);
    g_tuning.assign(entries, entries + count);
  });
}

int ccb_tuning_get(ccb_tuning_entry* entries, int32_t capacity, int32_t* count) {
  return Guard([&] {
    std::lock_guard<std::mutex> lock(g_tuning_mutex);
    if (count) *count = (int32_t)g_tuning.size();
    for (int32_t i = 0; entries && i < capacity && i < (int32_t)g_tuning.size(); ++i) entries[i] = g_tuning[i];
  });
}

int ccb_server_create(uint64_t hbm_budget_bytes, int32_t max_active, ccb_server** out) {
  return Guard([&] {
    if (!out) Fail(CCB_ERR_STATE, "null output handle");
    std::unique_ptr<ccb_server> sv(new ccb_server());
    sv->device = Device::Current();
    size_t free_b = 0, total_b = 0;
    CCB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    sv->budget = hbm_budget_bytes > 0 ? (size_t)hbm_budget_bytes : free_b * 8 / 10;
    sv->max_active = max_active > 0 ? max_active : 1024;
    CCB_CUDA(cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking));
    for (ccb_server::Lane& L : sv->lanes) {
      CCB_CUDA(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
      CCB_CUDA(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming));
      CCB_CUDA(cudaMalloc(&L.d_active, sizeof(int32_t)));
    }
    *out = sv.release();
  });
}

int ccb_server_submit(ccb_server* sv, const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges,
                      const ccb_params* params, int32_t* id_out) {
  if (!params) return Guard([] { Fail(CCB_ERR_STATE, "null argument"); });
  ccb_server::Request r;
  r.source = 0;
  r.n = n;
  r.words = words_per_row;
  r.edges = edges;
  r.params = *params;
  if (n > 0) {
    if (!bits || words_per_row < (n + 31) / 32) return Guard([] { Fail(CCB_ERR_INVALID, "bad bitset"); });
    r.bits.assign(bits, bits + (size_t)n * words_per_row);
  }
  return Submit(sv, std::move(r), id_out);
}

int ccb_server_submit_generated(ccb_server* sv, int32_t planted, uint32_t n, double density_or_p_in, double p_out,
                                double flip, int32_t parts, uint64_t graph_seed, const ccb_params* params,
                                int32_t* id_out) {
  if (!params) return Guard([] { Fail(CCB_ERR_STATE, "null argument"); });
  ccb_server::Request r;
  r.source = planted ? 2 : 1;
  r.n = n;
  r.density = density_or_p_in;
  r.p_in = density_or_p_in;
  r.p_out = p_out;
  r.flip = flip;
  r.parts = parts;
  r.graph_seed = graph_seed;
  r.params = *params;
  return Submit(sv, std::move(r), id_out);
}

int ccb_server_step(ccb_server* sv, int32_t* finished_ids, int32_t capacity, int32_t* finished_count) {
  return Guard([&] {
    if (!sv) Fail(CCB_ERR_STATE, "null server");
    ServerStep(*sv, finished_ids, capacity, finished_count);
  });
}

int ccb_server_status(const ccb_server* sv, int32_t* queued, int32_t* active, uint64_t* bytes_in_use) {
  return Guard([&] {
    if (!sv) Fail(CCB_ERR_STATE, "null server");
    if (queued) *queued = (int32_t)sv->queue.size();
    if (active) *active = (int32_t)sv->ActiveCount();
    if (bytes_in_use) *bytes_in_use = (uint64_t)sv->in_use;
  });
}

int ccb_server_result(ccb_server* sv, int32_t id, int32_t* done, int32_t* labels_out, ccb_result* result) {
  return Guard([&] {
    if (!sv || !done) Fail(CCB_ERR_STATE, "null argument");
    auto it = sv->done.find(id);
    *done = it != sv->done.end();
    if (it == sv->done.end()) return;
    if (it->second.status != CCB_OK) {
      const int status = it->second.status;
      const std::string error = it->second.error;
      sv->done.erase(it);
      Fail(status, error);
    }
    if (result) *result = it->second.result;
    if (labels_out && !it->second.labels.empty()) {
      std::memcpy(labels_out, it->second.labels.data(), it->second.labels.size() * 4);
    }
    sv->done.erase(it);
  });
}

int ccb_server_cancel(ccb_server* sv, int32_t id, int32_t* found) {
  return Guard([&] {
    if (!sv) Fail(CCB_ERR_STATE, "null server");
    bool hit = false;
    for (auto it = sv->queue.begin(); it != sv->queue.end() && !hit; ++it) {
      if (it->id != id) continue;
      sv->queue.erase(it);
      ccb_server::Done d;
      d.status = CCB_ERR_CANCELLED;
      d.error = "request cancelled";
      sv->done[id] = std::move(d);
      hit = true;
      break;
    }
    for (ccb_server::Lane& L : sv->lanes) {
      for (ccb_server::Active& a : L.active) {
        if (!hit && a.req.id == id && !a.cancel) a.cancel = hit = true;
      }
    }
    for (auto& w : sv->wides) {
      if (!hit && w->a.req.id == id && !w->a.cancel) w->a.cancel = hit = true;
    }
    if (found) *found = hit;
  });
}

void ccb_server_destroy(ccb_server* sv) { delete sv; }

namespace {

// The one-call entry points keep, per host thread, the device graph and solver buffers of their last call and
// reuse them when the next call has the same device, n, k, population and kernel choice: such a call pays
// the bitset upload and the degree count, not the allocations (ccb_release_cache frees them).
struct OneCallCache {
  std::unique_ptr<ccb_solver> solver;
  std::unique_ptr<ccb_graph> graph;
  int device = -1;
  uint32_t n = 0;
  int k = 0, pop = 0, ls = 0;
  void Release() {
    solver.reset();  // the solver refers to the graph: it goes first
    graph.reset();
    device = -1;
  }
  ~OneCallCache() { Release(); }
};
thread_local OneCallCache t_cache;

ccb_solver& CachedSolver(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges, int k, int pop,
                         int ls_kernel) {
  int device = 0;
  CCB_CUDA(cudaGetDevice(&device));
  OneCallCache& c = t_cache;
  if (c.solver && c.device == device && c.n == n && c.k == k && c.pop == pop && c.ls == ls_kernel) {
    const int words = (int)((n + 31) / 32);
    if (words_per_row < (uint32_t)words) Fail(CCB_ERR_INVALID, "words_per_row < ceil(n / 32)");
    if (bits == nullptr) Fail(CCB_ERR_INVALID, "null bitset");
    ccb_graph& g = *c.graph;
    g.edges = (int64_t)edges;
    CCB_CUDA(cudaMemcpy2DAsync(g.bits, g.pitch * sizeof(uint32_t), bits, words_per_row * sizeof(uint32_t),
                               words * sizeof(uint32_t), n, cudaMemcpyHostToDevice, nullptr));
    FinishGraph(g, nullptr);
    // the plan's k = 2 / 3 wide form depends on the density
    ccb_solver& s = *c.solver;
    s.plan.sparse = s.plan.packed_wide && 2.0 * (double)edges <= (double)n * n / 8.0;
    PlanSmem16(s);
    Describe(s);
    return s;
  }
  c.Release();
  std::unique_ptr<ccb_graph> g(MakeGraph(bits, false, n, words_per_row, edges, nullptr));
  std::unique_ptr<ccb_solver> s(MakeSolver(g.get(), k, pop, ls_kernel));
  c.graph = std::move(g);
  c.solver = std::move(s);
  c.device = device;
  c.n = n;
  c.k = k;
  c.pop = pop;
  c.ls = ls_kernel;
  return *c.solver;
}

}  // namespace

void ccb_release_cache(void) { t_cache.Release(); }

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
    ccb_solver& s = CachedSolver(bits, n, words_per_row, edges, params->k, params->population, params->ls_kernel);
    if (s.plan.wide) {
      RunPbils<int32_t>(s, *params, nullptr, labels_out, result);
    } else {
      RunPbils<int16_t>(s, *params, nullptr, labels_out, result);
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
    const int batch = std::min<int>(params->population, (int)n);
    ccb_solver& s = CachedSolver(bits, n, words_per_row, edges, 2, batch, params->ls_kernel);
    if (s.plan.wide) {
      RunNeighborhood<int32_t>(s, *params, local_search != 0, nullptr, labels_out, result);
    } else {
      RunNeighborhood<int16_t>(s, *params, local_search != 0, nullptr, labels_out, result);
    }
    result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
  });
}

}  // extern "C"
