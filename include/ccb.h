/*
 * ccb.h — C ABI of the B200 PBILS k-correlation-clustering library (libccb.so).
 *
 * Plain pointers, sizes and status codes only: no C++ or framework types cross this boundary, so a
 * C, C++ (cc::SolveGpu adapter), ctypes or cgo caller binds it directly.  Each entry point names the
 * reference interface of oQaris/cuda_graph_clustering it replaces.
 *
 * Graph format (the reference's cc::Graph, include/cc_graph.hpp:15-59): n rows of `words_per_row`
 * uint32 words, row-major; bit u of row v is set iff {u, v} is an edge; no self loops; the matrix is
 * symmetric; bits past column n-1 are zero.  words_per_row >= ceil(n / 32) (the reference stores
 * max(1, ceil(n / 32))).
 *
 * Errors: every function returns CCB_OK or a nonzero status; ccb_last_error() then gives the message
 * (the text of the std::runtime_error the reference would throw, thread-local).  All work runs on the
 * calling thread's current CUDA device.
 */
#ifndef CCB_H_
#define CCB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum ccb_status {
  CCB_OK = 0,
  CCB_ERR_INVALID = 1,       /* parameters rejected (bad k, population, gww, n, ...) */
  CCB_ERR_DEVICE_MEMORY = 2, /* the run does not fit the free device memory / shared memory */
  CCB_ERR_CUDA = 3,          /* a CUDA runtime call failed */
  CCB_ERR_TIMEOUT = 4,       /* a bounded device-side wait gave up (the tensor-core rebuild's pipeline) */
  CCB_ERR_STATE = 5,         /* handle misuse (null handle, queue full, ...) */
  CCB_ERR_CANCELLED = 6      /* a served request was cancelled (ccb_server_cancel) */
};

/* PbilsParams::LocalSearchKernel (include/cc_pbils.hpp:27-36). */
enum ccb_ls_kernel { CCB_LS_AUTO = 0, CCB_LS_GLOBAL = 1, CCB_LS_SHARED = 2, CCB_LS_WIDE = 3 };

/* cc::kMaxClusters (include/cc_gpu.hpp:10) and the packed-move vertex limit (cuda/cc_gpu_common.cuh:31-32). */
#define CCB_MAX_CLUSTERS 64
#define CCB_MAX_VERTICES_NARROW 32767
#define CCB_MAX_VERTICES_WIDE (1 << 20)

/* cc::PbilsParams (include/cc_pbils.hpp:26-49), field for field. */
typedef struct ccb_params {
  int32_t k;
  int32_t population;
  int32_t tournament;
  int32_t iterations;
  int32_t early_stop;
  double perturbation;
  double gww;
  int32_t threads; /* CPU-only knob of the reference; accepted and ignored */
  uint64_t seed;
  double time_limit_sec; /* 0 = no limit */
  int32_t verbose;
  int32_t ls_kernel; /* enum ccb_ls_kernel */
} ccb_params;

/* cc::PbilsResult (include/cc_pbils.hpp:51-59) without the label vector, which the caller passes. */
typedef struct ccb_result {
  int64_t objective;
  int32_t iterations_done;
  int32_t clusters_used;
  double seconds;
  int64_t local_searches;
  int64_t accepted_moves;
} ccb_result;

/* Message of the last failed call on this thread ("" after success). */
const char* ccb_last_error(void);

/* Fills the reference defaults: k 2, population 128, tournament 5, iterations 100, early_stop 6,
 * perturbation 0.4, gww 0.1, threads 1, seed 1, no time limit, auto kernel (cc_pbils.hpp:32-43). */
void ccb_params_init(ccb_params* params);

/* ---- one-call solvers (host buffers in, host buffers out) ------------------------------------ */

/* cc::SolveGpu (cuda/cc_pbils_gpu.cu:441-454).  labels_out: n int32 labels in [0, k). */
int ccb_pbils_solve(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges,
                    const ccb_params* params, int32_t* labels_out, ccb_result* result);

/* cc::SolveNeighborhoodGpu (local_search = 0) and cc::SolveNeighborhoodWithManyLocalSearchesGpu
 * (local_search = 1) (cuda/cc_pbils_gpu.cu:456-462).  Uses params->k (must be 2), population (batch)
 * and ls_kernel. */
int ccb_neighborhood_solve(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges,
                           const ccb_params* params, int32_t local_search, int32_t* labels_out,
                           ccb_result* result);

/* The two one-call entry points above keep, per calling host thread, the device buffers of their last call
 * (graph rows, population, scratch) and reuse them when the next call on the same device has the same n, k,
 * population and ls_kernel: a repeated solve then pays the bitset upload, not the allocations.  No
 * counterpart in the reference, whose calls allocate and free everything (cuda/cc_pbils_gpu.cu:105-122).
 * ccb_release_cache frees the calling thread's buffers; they are also freed when the thread exits. */
void ccb_release_cache(void);

/* ---- device-resident graphs and reusable solvers ----------------------------------------------
 * The reference uploads the graph and allocates the population inside every solve
 * (cuda/cc_pbils_gpu.cu:186-226).  These split that constructor so that a caller can keep the graph
 * and buffers on the device across solves.  `stream` is a cudaStream_t (NULL = legacy default). */
typedef struct ccb_graph ccb_graph;
typedef struct ccb_solver ccb_solver;

/* Copies a host bitset to the device (rows re-pitched to 16-byte multiples) and counts degrees. */
int ccb_graph_upload(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges, void* stream,
                     ccb_graph** out);
/* Same from a device bitset (e.g. a framework tensor); the library keeps its own copy. */
int ccb_graph_from_device(const uint32_t* device_bits, uint32_t n, uint32_t words_per_row, uint64_t edges,
                          void* stream, ccb_graph** out);
/* Graph::ErdosRenyi (src/cc_graph.cpp:168-177) generated on the device: the same bits as
 * ccb_generate_erdos_renyi on the host, by closed-form jump-ahead of the splitmix64 stream. */
int ccb_graph_generate_erdos_renyi(uint32_t n, double density, uint64_t seed, void* stream, ccb_graph** out);
/* The planted partition of ccb_generate_planted, generated on the device (communities on the host).
 * community_out (host, n entries) may be NULL.  No counterpart in the reference. */
int ccb_graph_generate_planted(uint32_t n, int32_t parts, int32_t shuffle_split, double p_in, double p_out,
                               double flip, uint64_t seed, void* stream, ccb_graph** out, int32_t* community_out);
/* Graph::LoadTags (src/cc_graph.cpp:311-371) built on the device: the objects of a tags JSON file ({"key":
 * ["tag", ...], ...}), n of them sampled by the seeded partial Fisher-Yates shuffle of SampleWithoutReplacement
 * (all when n is 0 or at least their count), joined when the similarity of their tag sets ("jaccard", "cosine",
 * "dice" or "overlap") is at least the threshold.  The same bits and edge count as the reference's loader;
 * parse errors carry its messages. */
int ccb_graph_load_tags(const char* path, const char* similarity, double threshold, uint32_t n, uint64_t seed,
                        void* stream, ccb_graph** out);
/* Copies a device graph back into the reference's host layout (n rows of words_per_row words). */
int ccb_graph_download(const ccb_graph* graph, uint32_t* bits, uint32_t words_per_row);
int ccb_graph_size(const ccb_graph* graph, uint32_t* n, uint64_t* edges);
void ccb_graph_destroy(ccb_graph* graph);

/* Plans kernels and allocates buffers for (graph, k, population, ls_kernel); the solver can then run
 * any number of solves with other seeds / iteration counts / gww / perturbation / tournament. */
int ccb_solver_create(const ccb_graph* graph, const ccb_params* params, ccb_solver** out);
/* Runs PBILS on the solver's graph.  Host labels_out (n int32) may be NULL.  Inputs already resident:
 * no host-to-device copies happen inside. */
int ccb_solver_pbils(ccb_solver* solver, const ccb_params* params, void* stream, int32_t* labels_out,
                     ccb_result* result);
/* Neighborhood enumerators on the solver's graph (k must be 2). */
int ccb_solver_neighborhood(ccb_solver* solver, const ccb_params* params, int32_t local_search, void* stream,
                            int32_t* labels_out, ccb_result* result);
/* How a solver rebuilds G = A*Z after each perturbation.  No counterpart in the reference, whose rebuild is the
 * popcount of cuda/cc_population_kernels.cuh:44-136 (KernelRebuild / KernelRebuild2).  CCB_REBUILD_TENSOR runs
 * the whole population's rebuild as one int8 contraction on the tensor cores (tcgen05 kind::i8, int32
 * accumulators in TMEM, operands fed by TMA): G[slot][c][v] = sum_u A[v][u] Z[slot*k + c][u] with Z the one-hot
 * labels.  The counts are the same integers either way, so every trajectory is unchanged.  It applies to the
 * wide path (int32 G: n > 32767, or ls_kernel CCB_LS_WIDE) with n >= 128; CCB_REBUILD_AUTO takes it there. */
enum ccb_rebuild_kind { CCB_REBUILD_AUTO = 0, CCB_REBUILD_POPCOUNT = 1, CCB_REBUILD_TENSOR = 2 };
int ccb_solver_set_rebuild(ccb_solver* solver, int32_t kind);
/* Text description of the plan ("generic, shared memory, 512 threads, ..."). */
const char* ccb_solver_describe(const ccb_solver* solver);
void ccb_solver_destroy(ccb_solver* solver);

/* Per-kernel timing of the last solve (CUDA events around each launch; enabled by
 * ccb_solver_set_profiling).  Times in milliseconds, launches counted. */
typedef struct ccb_kernel_stats {
  double descent_ms;
  double rebuild_ms;
  double record_ms;
  double other_ms;
  int64_t descent_launches;
  int64_t rebuild_launches;
  int64_t record_launches;
  int64_t other_launches;
} ccb_kernel_stats;
int ccb_solver_set_profiling(ccb_solver* solver, int32_t enabled);
int ccb_solver_stats(const ccb_solver* solver, ccb_kernel_stats* stats);

/* ---- batched solves ----------------------------------------------------------------------------
 * No counterpart in the reference (which solves one instance per call).  Many independent PBILS instances
 * (each its own graph, k, population, seed, ...) run together in persistent kernels, one per shape bucket,
 * that pull (instance, slot) work items from device queues (see ccb_batch_set_engine).  Results are the
 * same as ccb_solver_pbils / ccb_pbils_solve would give each instance alone, bit for bit.
 * Graphs are device-resident (ccb_graph_upload) and must outlive the batch.  Instances with k = 1 or
 * n > 32767 are solved one by one on the plain path after the batched ones. */
typedef struct ccb_batch ccb_batch;
int ccb_batch_create(ccb_batch** out);
int ccb_batch_add(ccb_batch* batch, const ccb_graph* graph, const ccb_params* params, int32_t* id_out);
/* Solves every instance (again on each call: same inputs, same results).  Synchronous.  Each result's `seconds`
 * is the instance's own completion time from the start of the run under the flow engine, the run's time under
 * the lock-step engine. */
int ccb_batch_run(ccb_batch* batch);
/* The engine, chosen before the first run.  CCB_BATCH_LOCKSTEP (default): one CUDA graph replay per iteration
 * of all instances (bucket descents, then record, rebuild and advance of every instance).  CCB_BATCH_FLOW: one
 * persistent kernel per shape bucket carries every instance through all its iterations; a block claims the next
 * (instance, slot) item of the heaviest instance that has one, and the block that completes an instance's last
 * descent (rebuild) slot runs its record and stop rule (advances its iteration) and publishes its next phase,
 * so no instance waits for another: small instances finish early (per-instance completion far sooner) at some
 * cost in whole-batch throughput.  A flow block that finds nothing to claim while instances are unfinished
 * sleeps, leaves when its bucket has more blocks than unfinished slots, and gives up after wait_limit_sec
 * (0: 30 s) with CCB_ERR_TIMEOUT. */
enum ccb_batch_engine { CCB_BATCH_FLOW = 0, CCB_BATCH_LOCKSTEP = 1 };
int ccb_batch_set_engine(ccb_batch* batch, int32_t engine, double wait_limit_sec);
/* Host-side fault injection for tests of the bounded wait: instance `id`'s work is never published to the flow
 * engine's blocks, so the run ends in CCB_ERR_TIMEOUT after the wait limit instead of waiting forever. */
int ccb_batch_withhold(ccb_batch* batch, int32_t id);
int ccb_batch_result(const ccb_batch* batch, int32_t id, int32_t* labels_out, ccb_result* result);
/* Text description of the buckets (kernel, shape, instances, slots, persistent grid). */
const char* ccb_batch_describe(const ccb_batch* batch);
void ccb_batch_destroy(ccb_batch* batch);

/* ---- batched-engine tuning ------------------------------------------------------------------------
 * No counterpart in the reference.  A process-wide table, written by the project's autotuner
 * (cuda_graph_clustering_b200/autotune.py, table committed as tuning.json), that picks per shape bucket of
 * the batched engine the descent kernel, its threads per slot and its resident block count.  Batches and
 * servers built after ccb_tuning_set use it; an instance matches the first entry whose kind and n, k
 * ranges contain it.  Tuning never changes a result: every choice runs the same trajectory. */
typedef struct ccb_tuning_entry {
  int32_t kind;          /* the plan's batched kernel: 0 registers, 1 streamed, 2 incremental with its state in
                            global memory, 3 incremental with cached keys in registers / shared memory; -1 any */
  int32_t n_min, n_max;  /* inclusive */
  int32_t k_min, k_max;
  int32_t use_kind;      /* -1: the plan's kernel; 2: the incremental kernel with its state in global memory
                            (taken by kind-2 and kind-3 instances whose state is not in shared memory) */
  int32_t threads;       /* threads per slot for use_kind 2: 256, 512 or 1024 */
  int32_t blocks_per_sm; /* resident slots per SM of the persistent grid; 0: the occupancy limit */
  int32_t max_slots;     /* cap on the slots running at once (the L2-resident block count); 0: none */
} ccb_tuning_entry;
/* Replaces the table (count 0 clears it). */
int ccb_tuning_set(const ccb_tuning_entry* entries, int32_t count);
/* Copies up to capacity entries; count receives the table size. */
int ccb_tuning_get(ccb_tuning_entry* entries, int32_t capacity, int32_t* count);

/* ---- serving ------------------------------------------------------------------------------------
 * No counterpart in the reference.  A request loop with continuous batching: submitted requests wait in a
 * FIFO queue; every ccb_server_step admits queued requests while their estimated device memory (graph rows
 * + population buffers) fits the budget, and advances the admitted ones with the batched bucket kernels.
 * Admitted requests run in five lanes by size (n <= 1024, 2048, 4096, 8192, larger), each stepping one PBILS
 * iteration of all its requests at a time on a stream of its own, so the lanes overlap on the device and a
 * small request is not held to the pace of a large one; requests admitted later join their lane at its next
 * iteration.  Requests the batched kernels do not take (k = 1, n > 32767) are stepped by the same loop on a stream
 * of their own each, four iterations of the plain path's kernels at a time, so their kernels overlap the lanes'
 * on the device.  A step launches every idle lane and wide request, waits until at least one of them finished
 * its iteration (chunk), and retires the requests that stopped, freeing their memory for the queue.  Each
 * result equals the request's plain solve.  Not thread-safe: one host thread drives a server. */
typedef struct ccb_server ccb_server;
/* hbm_budget_bytes 0: 80% of the free device memory; max_active 0: 1024. */
int ccb_server_create(uint64_t hbm_budget_bytes, int32_t max_active, ccb_server** out);
/* A request with a host bitset (copied at submission, uploaded at admission). */
int ccb_server_submit(ccb_server* server, const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges,
                      const ccb_params* params, int32_t* id_out);
/* A request whose graph the server generates on the device at admission: Erdős–Rényi (planted = 0,
 * density_or_p_in = density) or the planted partition (planted = 1, `parts` communities, p_in, p_out, flip). */
int ccb_server_submit_generated(ccb_server* server, int32_t planted, uint32_t n, double density_or_p_in,
                                double p_out, double flip, int32_t parts, uint64_t graph_seed,
                                const ccb_params* params, int32_t* id_out);
/* Admission, an iteration of every idle lane, retirement (see above).  Writes the ids finished in this step
 * (up to capacity) and their count.  Returns after at least one lane finished an iteration. */
int ccb_server_step(ccb_server* server, int32_t* finished_ids, int32_t capacity, int32_t* finished_count);
int ccb_server_status(const ccb_server* server, int32_t* queued, int32_t* active, uint64_t* bytes_in_use);
/* done = 1 and the result (labels: n int32) once request `id` finished; the result is then released. */
int ccb_server_result(ccb_server* server, int32_t id, int32_t* done, int32_t* labels_out, ccb_result* result);
/* Cancels request `id` (found = 0 if it is unknown or already finished): a queued request leaves the queue, an
 * admitted one stops before its next iteration (chunk) and frees its memory when the one in flight completes.
 * Its result reports CCB_ERR_CANCELLED. */
int ccb_server_cancel(ccb_server* server, int32_t id, int32_t* found);
void ccb_server_destroy(ccb_server* server);

/* ---- device recount -----------------------------------------------------------------------------
 * Objective f, cluster sizes and G = A*Z of `count` labelings of one graph, computed on the device:
 * the GPU form of the reference's post-solve recount ObjectiveBitwise (src/cc_pbils_cpu.cpp:25-53,
 * called from include/cc_cli.hpp:337-343) and of State::Rebuild (src/cc_pbils_cpu.cpp:74-95).
 * Device pointers: bits (n rows of words_per_row words), labels [count][n] int32, f_out [count];
 * sizes_out [count][k] and g_out [count][k][n] (int32, cluster-major) may be NULL.  A labeling with a
 * label outside [0, k) gets f = -1.  Scratch (count * k * ceil(n/32) mask words) is taken from the
 * stream-ordered allocator for the call.  Asynchronous on `stream`. */
int ccb_evaluate_labelings(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges, int32_t k,
                           int32_t count, const int32_t* labels, int64_t* f_out, int32_t* sizes_out,
                           int32_t* g_out, void* stream);

/* No counterpart in the reference.  ccb_evaluate_labelings for callers that cannot allocate device
 * memory when they call in (their device memory is already reserved by their own pool allocator, or
 * their loop must not pay cudaMalloc/cudaFree and the device-wide synchronisation cudaFree can cause).
 * Allocates nothing: the mask scratch is a fixed 4 MiB array in device memory that every GPU holds
 * until exit once libccb.so's module is loaded on it.  Limit: count * k * ceil(n / 32) <= 1048576 mask
 * words, else CCB_ERR_INVALID.  The first call on a device is its set-up: it looks the array's device
 * address up and, under CUDA's default lazy module loading, is when the 4 MiB are taken.  Make it before
 * any stream capture and before a pool of the caller's reserves the free memory; a call with count = 0
 * does only this set-up.  The address is kept for the process: do not use this entry point across a
 * cudaDeviceReset.  All calls share the array, so calls whose kernels overlap on the GPU race and must
 * be ordered by the caller.  Same arguments, outputs and asynchrony as ccb_evaluate_labelings. */
int ccb_evaluate_labelings_noalloc(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges,
                                   int32_t k, int32_t count, const int32_t* labels, int64_t* f_out,
                                   int32_t* sizes_out, int32_t* g_out, void* stream);

/* No counterpart in the reference.  ccb_evaluate_labelings with G = A*Z computed on the tensor cores (the
 * contraction of ccb_solver_set_rebuild's CCB_REBUILD_TENSOR): the same outputs, exactly.  Needs n >= 128,
 * words_per_row a multiple of 4 and a 16-byte aligned bitset (its rows are read by TMA).  Scratch (the one-hot
 * Z, count * k rows of ceil(ceil(n/32)/4) * 128 bytes) comes from the stream-ordered allocator.  A labeling's
 * f is -2 if the kernel's bounded pipeline wait gave up.  Asynchronous on `stream`. */
int ccb_evaluate_labelings_tensor(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges,
                                  int32_t k, int32_t count, const int32_t* labels, int64_t* f_out,
                                  int32_t* sizes_out, int32_t* g_out, void* stream);

/* ---- host instance generators (the instances of the reference's CLI and of the benchmarks) ----- */

/* Graph::ErdosRenyi (src/cc_graph.cpp:168-177): bits holds n * words_per_row words. Returns edges. */
uint64_t ccb_generate_erdos_renyi(uint32_t n, double density, uint64_t seed, uint32_t* bits,
                                  uint32_t words_per_row);
/* Seeded planted partition (no counterpart in the reference): `parts` communities, or with
 * shuffle_split a seeded permutation split into halves; edge probability p_in inside a community,
 * p_out across, then every pair flipped with probability `flip`.  community_out may be NULL. */
uint64_t ccb_generate_planted(uint32_t n, int32_t parts, int32_t shuffle_split, double p_in, double p_out,
                              double flip, uint64_t seed, uint32_t* bits, uint32_t words_per_row,
                              int32_t* community_out);

#ifdef __cplusplus
}
#endif

#endif /* CCB_H_ */
