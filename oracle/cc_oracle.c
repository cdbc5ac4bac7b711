/*
 * CPU ORACLE — test infrastructure only.
 *
 * A plain-C restatement of the reference CPU solver of oQaris/cuda_graph_clustering
 * (src/cc_pbils_cpu.cpp, include/cc_math.hpp, src/cc_graph.cpp) and of the sequential
 * Neighborhood brute force of cuda/cc_verify_gpu.cu.  Its only callers are the tests,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py, where it is the checker.
 * The product (cuda_graph_clustering_b200) never links, loads or calls it.
 *
 * Parity of this restatement is pinned two ways (see tests/test_oracle_golden.py):
 *   - against the reference's published golden rows (docs/data/gpu.csv, gww_stop.csv,
 *     cpu.csv), extracted into tests/golden/ by tests/golden/make_golden.py;
 *   - against the reference's own CPU code, compiled from its sources by oracle/Makefile
 *     into oracle/_ref/ and compared case by case (tests/test_oracle_vs_ref.py).
 *
 * Every exported function names the reference file:line it restates.  Arithmetic is
 * integer except the 24-bit RandFloat compare, which is exact in IEEE float.
 */
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------------------------
 * splitmix64 streams: include/cc_math.hpp:84-145
 * ---------------------------------------------------------------------------------------- */
#define GOLDEN_GAMMA 0x9E3779B97F4A7C15ull

static inline uint64_t sm64(uint64_t *state) { /* cc_math.hpp:84-90 */
  *state += GOLDEN_GAMMA;
  uint64_t z = *state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static inline uint32_t next_u32(uint64_t *state) { return (uint32_t)(sm64(state) >> 32); } /* :92 */

static inline uint32_t rand_below(uint64_t *state, uint32_t bound) { /* :95-98 */
  if (bound == 0) return 0;
  return (uint32_t)(((uint64_t)next_u32(state) * bound) >> 32);
}

static inline float rand_float(uint64_t *state) { /* :101-104, 24-bit mantissa */
  return (float)(next_u32(state) >> 8) * (1.0f / 16777216.0f);
}

ORC_EXPORT uint64_t orc_stream_seed(uint64_t seed, uint64_t stream, uint64_t step) { /* :107-111 */
  uint64_t s = seed ^ (stream * 0xD1B54A32D192ED03ull) ^ (step * 0xA0761D6478BD642Full);
  sm64(&s);
  return s;
}

/* Stream tags: cc_math.hpp:118-121 (solver), cc_graph.cpp:20-21 (generator). */
#define INIT_STREAM 0xA11CEull
#define SELECT_STREAM 0x5E1EC7ull
#define PERTURB_STREAM 0xBEEFull
#define PERTURB_FIRST_STEP 0x5000000ull
#define ER_STREAM 0xE4D05Full

ORC_EXPORT int orc_initial_label(uint64_t base, uint64_t index, int k) { /* cc_math.hpp:123-126 */
  uint64_t rng = orc_stream_seed(base, index, 0);
  return (int)rand_below(&rng, (uint32_t)k);
}

/* cc_math.hpp:129-138: best of `tournament` uniform draws, strict < keeps the earlier draw. */
ORC_EXPORT int orc_tournament(uint64_t base, int slot, int iteration, const int64_t *f, int population,
                              int tournament) {
  uint64_t rng = orc_stream_seed(base, (uint64_t)slot, (uint64_t)(iteration + 1));
  int chosen = (int)rand_below(&rng, (uint32_t)population);
  for (int t = 1; t < tournament; ++t) {
    int candidate = (int)rand_below(&rng, (uint32_t)population);
    if (f[candidate] < f[chosen]) chosen = candidate;
  }
  return chosen;
}

/* cc_math.hpp:141-145 */
ORC_EXPORT int orc_perturbed_label(uint64_t base, uint64_t index, int iteration, int label, int k,
                                   float probability) {
  uint64_t rng = orc_stream_seed(base, index, (uint64_t)iteration + PERTURB_FIRST_STEP);
  if (rand_float(&rng) >= probability) return label;
  return (label + 1 + (int)rand_below(&rng, (uint32_t)(k - 1))) % k;
}

/* ------------------------------------------------------------------------------------------
 * Bitset graph: include/cc_graph.hpp:15-59, src/cc_graph.cpp:149-161.
 * Row v holds words = max(1, ceil(n/32)) uint32 words; bit u of row v set iff edge {u, v}.
 * ---------------------------------------------------------------------------------------- */
ORC_EXPORT uint32_t orc_words_per_row(uint32_t n) { return n == 0 ? 1u : (n + 31u) / 32u; }

static inline int joined(const uint32_t *bits, uint32_t words, uint32_t i, uint32_t j) {
  return (int)((bits[(size_t)i * words + j / 32u] >> (j % 32u)) & 1u);
}

static inline void set_pair(uint32_t *bits, uint32_t words, uint32_t i, uint32_t j) {
  bits[(size_t)i * words + j / 32u] |= 1u << (j % 32u);
  bits[(size_t)j * words + i / 32u] |= 1u << (i % 32u);
}

/* Graph::ErdosRenyi, cc_graph.cpp:168-177: one sequential stream, pairs (i asc, j < i asc). */
ORC_EXPORT uint64_t orc_erdos_renyi(uint32_t n, double density, uint64_t seed, uint32_t *bits) {
  const uint32_t words = orc_words_per_row(n);
  memset(bits, 0, (size_t)n * words * sizeof(uint32_t));
  uint64_t state = orc_stream_seed(seed, ER_STREAM, 0);
  uint64_t edges = 0;
  for (uint32_t i = 0; i < n; ++i) {
    for (uint32_t j = 0; j < i; ++j) {
      if ((double)rand_float(&state) < density) {
        set_pair(bits, words, i, j);
        ++edges;
      }
    }
  }
  return edges;
}

/*
 * Planted-partition generator.  The reference has none; this is the project's own seeded
 * definition, restated independently of the product's generator so that tests can check
 * both emit the same bits:
 *   communities: if `shuffle_split` the vertices are a Fisher-Yates shuffle (stream 0x9A27ED, step 1:
 *     for i = n-1 .. 1: j = RandBelow(i + 1), swap) and position < n/2 -> community 0, else 1;
 *     otherwise community[v] = RandBelow(parts) for v ascending (stream 0x9A27ED, step 2).
 *   edges: one stream (0x9A27ED, step 3), pairs (i asc, j < i asc), two draws per pair:
 *     edge = (RandFloat < (same community ? p_in : p_out)) XOR (RandFloat < flip).
 */
#define PLANTED_STREAM 0x9A27EDull
ORC_EXPORT uint64_t orc_planted(uint32_t n, int parts, int shuffle_split, double p_in, double p_out, double flip,
                                uint64_t seed, uint32_t *bits, int32_t *community) {
  const uint32_t words = orc_words_per_row(n);
  memset(bits, 0, (size_t)n * words * sizeof(uint32_t));
  if (shuffle_split) {
    uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    uint64_t rng = orc_stream_seed(seed, PLANTED_STREAM, 1);
    for (uint32_t i = n; i-- > 1;) {
      uint32_t j = rand_below(&rng, i + 1);
      uint32_t t = perm[i];
      perm[i] = perm[j];
      perm[j] = t;
    }
    for (uint32_t i = 0; i < n; ++i) community[perm[i]] = i < n / 2 ? 0 : 1;
    free(perm);
  } else {
    uint64_t rng = orc_stream_seed(seed, PLANTED_STREAM, 2);
    for (uint32_t v = 0; v < n; ++v) community[v] = (int32_t)rand_below(&rng, (uint32_t)parts);
  }
  uint64_t state = orc_stream_seed(seed, PLANTED_STREAM, 3);
  uint64_t edges = 0;
  for (uint32_t i = 0; i < n; ++i) {
    for (uint32_t j = 0; j < i; ++j) {
      const double p = community[i] == community[j] ? p_in : p_out;
      const int e = (double)rand_float(&state) < p;
      const int x = (double)rand_float(&state) < flip;
      if (e ^ x) {
        set_pair(bits, words, i, j);
        ++edges;
      }
    }
  }
  return edges;
}

/* ------------------------------------------------------------------------------------------
 * Objective and solution state: cc_math.hpp:56-77, src/cc_pbils_cpu.cpp:12-139.
 * ---------------------------------------------------------------------------------------- */
static int64_t same_pairs(const int32_t *sizes, int k) { /* cc_math.hpp:56-64 */
  int64_t acc = 0;
  for (int c = 0; c < k; ++c) acc += (int64_t)sizes[c] * (sizes[c] - 1) / 2;
  return acc;
}

/* ObjectiveDirect, cc_pbils_cpu.cpp:12-23: disagreements over pairs i < j. */
ORC_EXPORT int64_t orc_objective_direct(const uint32_t *bits, uint32_t n, uint32_t words, const int32_t *labels) {
  int64_t d = 0;
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t j = i + 1; j < n; ++j) d += (labels[i] == labels[j]) != joined(bits, words, i, j);
  return d;
}

/* ObjectiveBitwise, cc_pbils_cpu.cpp:25-53: popcount(row XOR own-cluster mask) - 1 per vertex, halved. */
ORC_EXPORT int64_t orc_objective_bitwise(const uint32_t *bits, uint32_t n, uint32_t words, const int32_t *labels) {
  int k = 0;
  for (uint32_t v = 0; v < n; ++v) k = labels[v] + 1 > k ? labels[v] + 1 : k;
  uint32_t *masks = (uint32_t *)calloc((size_t)(k ? k : 1) * words, sizeof(uint32_t));
  for (uint32_t v = 0; v < n; ++v) masks[(size_t)labels[v] * words + v / 32] |= 1u << (v % 32);
  int64_t acc = 0;
  for (uint32_t v = 0; v < n; ++v) {
    const uint32_t *row = bits + (size_t)v * words;
    const uint32_t *mask = masks + (size_t)labels[v] * words;
    for (uint32_t w = 0; w < words; ++w) acc += __builtin_popcount(row[w] ^ mask[w]);
    acc -= 1;
  }
  free(masks);
  return acc / 2;
}

typedef struct {
  int n, k;
  int32_t *labels; /* n */
  int32_t *g;      /* k * n, g[c * n + v] */
  int32_t *sizes;  /* k */
  int64_t f;
} state_t;

static void state_alloc(state_t *s, int n, int k) {
  s->n = n;
  s->k = k;
  s->labels = (int32_t *)calloc((size_t)(n ? n : 1), sizeof(int32_t));
  s->g = (int32_t *)calloc((size_t)k * (n ? n : 1), sizeof(int32_t));
  s->sizes = (int32_t *)calloc((size_t)k, sizeof(int32_t));
  s->f = 0;
}

static void state_free(state_t *s) {
  free(s->labels);
  free(s->g);
  free(s->sizes);
}

static void state_copy(state_t *dst, const state_t *src) {
  memcpy(dst->labels, src->labels, sizeof(int32_t) * src->n);
  memcpy(dst->g, src->g, sizeof(int32_t) * (size_t)src->k * src->n);
  memcpy(dst->sizes, src->sizes, sizeof(int32_t) * src->k);
  dst->f = src->f;
}

/* State::Rebuild, cc_pbils_cpu.cpp:74-95: G[c][v] = popcount(row_v & mask_c); f = m + sum C(n_c,2) - W. */
static void rebuild(state_t *s, const uint32_t *bits, uint32_t words, uint64_t edges, uint32_t *masks) {
  const int n = s->n, k = s->k;
  memset(s->sizes, 0, sizeof(int32_t) * k);
  memset(masks, 0, sizeof(uint32_t) * (size_t)k * words);
  for (int v = 0; v < n; ++v) {
    ++s->sizes[s->labels[v]];
    masks[(size_t)s->labels[v] * words + v / 32] |= 1u << (v % 32);
  }
  int64_t intra_twice = 0;
  for (int v = 0; v < n; ++v) {
    const uint32_t *row = bits + (size_t)v * words;
    for (int c = 0; c < k; ++c) {
      const uint32_t *mask = masks + (size_t)c * words;
      int acc = 0;
      for (uint32_t w = 0; w < words; ++w) acc += __builtin_popcount(row[w] & mask[w]);
      s->g[(size_t)c * n + v] = acc;
    }
    intra_twice += s->g[(size_t)s->labels[v] * n + v];
  }
  s->f = (int64_t)edges + same_pairs(s->sizes, k) - intra_twice;
}

/* State::BestMove, cc_pbils_cpu.cpp:99-118: v ascending, target ascending, strictly smaller delta wins. */
static int best_move(const state_t *s, int *out_v, int *out_to) {
  int best = 0;
  *out_v = -1;
  *out_to = -1;
  const int n = s->n, k = s->k;
  for (int v = 0; v < n; ++v) {
    const int a = s->labels[v];
    const int ga = s->g[(size_t)a * n + v];
    const int sa = s->sizes[a];
    for (int c = 0; c < k; ++c) {
      if (c == a) continue;
      const int delta = (s->sizes[c] - sa + 1) - 2 * (s->g[(size_t)c * n + v] - ga); /* MoveDelta, cc_math.hpp:75-77 */
      if (delta < best) {
        best = delta;
        *out_v = v;
        *out_to = c;
      }
    }
  }
  return best;
}

/* State::ApplyMove, cc_pbils_cpu.cpp:120-139 */
static void apply_move(state_t *s, const uint32_t *bits, uint32_t words, int v, int to) {
  const int n = s->n;
  const int from = s->labels[v];
  if (from == to) return;
  const int delta = (s->sizes[to] - s->sizes[from] + 1) - 2 * (s->g[(size_t)to * n + v] - s->g[(size_t)from * n + v]);
  int32_t *gf = s->g + (size_t)from * n;
  int32_t *gt = s->g + (size_t)to * n;
  const uint32_t *row = bits + (size_t)v * words;
  for (uint32_t w = 0; w < words; ++w) {
    for (uint32_t b = row[w]; b; b &= b - 1) {
      const uint32_t u = w * 32 + (uint32_t)__builtin_ctz(b);
      --gf[u];
      ++gt[u];
    }
  }
  --s->sizes[from];
  ++s->sizes[to];
  s->labels[v] = to;
  s->f += delta;
}

/* LocalSearch, cc_pbils_cpu.cpp:141-149 */
static int64_t local_search(state_t *s, const uint32_t *bits, uint32_t words, int64_t *moves) {
  int v, to;
  while (best_move(s, &v, &to) < 0) {
    apply_move(s, bits, words, v, to);
    ++*moves;
  }
  return s->f;
}

/* ------------------------------------------------------------------------------------------
 * Exported single-state helpers (unit parity of the GPU kernels).
 * ---------------------------------------------------------------------------------------- */
ORC_EXPORT int64_t orc_rebuild(const uint32_t *bits, uint32_t n, uint32_t words, uint64_t edges, int k,
                               const int32_t *labels, int32_t *g_out, int32_t *sizes_out) {
  state_t s;
  state_alloc(&s, (int)n, k);
  memcpy(s.labels, labels, sizeof(int32_t) * n);
  uint32_t *masks = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)k * words);
  rebuild(&s, bits, words, edges, masks);
  free(masks);
  if (g_out) memcpy(g_out, s.g, sizeof(int32_t) * (size_t)k * n);
  if (sizes_out) memcpy(sizes_out, s.sizes, sizeof(int32_t) * k);
  const int64_t f = s.f;
  state_free(&s);
  return f;
}

/* Runs LocalSearch from `labels` (rebuilt first); returns f, writes final labels, move count. */
ORC_EXPORT int64_t orc_local_search(const uint32_t *bits, uint32_t n, uint32_t words, uint64_t edges, int k,
                                    int32_t *labels, int64_t *moves) {
  state_t s;
  state_alloc(&s, (int)n, k);
  memcpy(s.labels, labels, sizeof(int32_t) * n);
  uint32_t *masks = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)k * words);
  rebuild(&s, bits, words, edges, masks);
  free(masks);
  int64_t m = 0;
  local_search(&s, bits, words, &m);
  memcpy(labels, s.labels, sizeof(int32_t) * n);
  if (moves) *moves = m;
  const int64_t f = s.f;
  state_free(&s);
  return f;
}

/* WinnerCopies, cc_pbils_cpu.cpp:168 */
ORC_EXPORT int orc_winner_copies(double gww, int population) { return (int)(gww * population); }

/* RankSlots, cc_pbils_cpu.cpp:170-175: by f, ties by slot (a stable order). */
ORC_EXPORT void orc_rank_slots(const int64_t *f, int population, int32_t *order) {
  for (int i = 0; i < population; ++i) order[i] = i;
  /* insertion sort keeps equal keys in slot order */
  for (int i = 1; i < population; ++i) {
    const int32_t x = order[i];
    int j = i - 1;
    while (j >= 0 && f[order[j]] > f[x]) {
      order[j + 1] = order[j];
      --j;
    }
    order[j + 1] = x;
  }
}

/* ------------------------------------------------------------------------------------------
 * Parallel-for over slots (the reference's WorkerPool, include/cc_parallel.hpp:20-95: an
 * atomic counter hands out items).  Results never depend on the thread count.
 * ---------------------------------------------------------------------------------------- */
typedef void (*item_fn)(void *ctx, int item, int worker);
typedef struct {
  item_fn fn;
  void *ctx;
  int count;
  atomic_int next;
} pool_job;
typedef struct {
  pool_job *job;
  int worker;
} pool_arg;

static void *pool_main(void *p) {
  pool_arg *a = (pool_arg *)p;
  for (int i = atomic_fetch_add(&a->job->next, 1); i < a->job->count; i = atomic_fetch_add(&a->job->next, 1))
    a->job->fn(a->job->ctx, i, a->worker);
  return NULL;
}

static void parallel_for(int threads, int count, item_fn fn, void *ctx) {
  if (threads > count) threads = count;
  if (threads <= 1) {
    for (int i = 0; i < count; ++i) fn(ctx, i, 0);
    return;
  }
  pool_job job = {fn, ctx, count, 0};
  pthread_t tid[256];
  pool_arg args[256];
  if (threads > 256) threads = 256;
  for (int t = 1; t < threads; ++t) {
    args[t].job = &job;
    args[t].worker = t;
    pthread_create(&tid[t], NULL, pool_main, &args[t]);
  }
  args[0].job = &job;
  args[0].worker = 0;
  pool_main(&args[0]);
  for (int t = 1; t < threads; ++t) pthread_join(tid[t], NULL);
}

/* ------------------------------------------------------------------------------------------
 * PBILS: SolveCpu, src/cc_pbils_cpu.cpp:183-252 (with Progress::Next, include/cc_pbils.hpp:69-78).
 * ---------------------------------------------------------------------------------------- */
typedef struct {
  int32_t k, population, tournament, iterations, early_stop;
  double perturbation, gww;
  uint64_t seed;
} orc_params;

typedef struct {
  int64_t objective;
  int32_t iterations_done, clusters_used;
  int64_t local_searches, accepted_moves;
} orc_result;

typedef struct {
  const uint32_t *bits;
  uint32_t n, words;
  uint64_t edges;
  const orc_params *p;
  state_t *pop, *next;
  int64_t *fitness, *moves;
  uint32_t **masks; /* per worker */
  uint64_t init_stream, select_stream, perturb_stream;
  int iteration;
  const int32_t *order;
  int copies;
} solve_ctx;

static void init_item(void *vc, int slot, int worker) { /* cc_pbils_cpu.cpp:198-205 */
  solve_ctx *c = (solve_ctx *)vc;
  state_t *s = &c->pop[slot];
  for (uint32_t v = 0; v < c->n; ++v)
    s->labels[v] = orc_initial_label(c->init_stream, (uint64_t)slot * c->n + v, c->p->k);
  rebuild(s, c->bits, c->words, c->edges, c->masks[worker]);
}

static void descend_item(void *vc, int slot, int worker) { /* cc_pbils_cpu.cpp:220-226 */
  (void)worker;
  solve_ctx *c = (solve_ctx *)vc;
  const int chosen =
      orc_tournament(c->select_stream, slot, c->iteration, c->fitness, c->p->population, c->p->tournament);
  state_copy(&c->next[slot], &c->pop[chosen]);
  int64_t m = 0;
  local_search(&c->next[slot], c->bits, c->words, &m);
  c->moves[slot] = m;
}

static void gww_item(void *vc, int i, int worker) { /* cc_pbils_cpu.cpp:237-238 */
  (void)worker;
  solve_ctx *c = (solve_ctx *)vc;
  state_copy(&c->next[c->order[c->p->population - 1 - i]], &c->next[c->order[i]]);
}

static void perturb_item(void *vc, int slot, int worker) { /* Perturb, cc_pbils_cpu.cpp:151-161 */
  solve_ctx *c = (solve_ctx *)vc;
  state_t *s = &c->next[slot];
  if (s->k < 2) return;
  int touched = 0;
  for (int v = 0; v < s->n; ++v) {
    const uint64_t index = (uint64_t)slot * s->n + v;
    const int label = orc_perturbed_label(c->perturb_stream, index, c->iteration, s->labels[v], s->k,
                                          (float)c->p->perturbation);
    touched |= label != s->labels[v];
    s->labels[v] = label;
  }
  if (touched) rebuild(s, c->bits, c->words, c->edges, c->masks[worker]);
}

static int count_clusters(const int32_t *labels, uint32_t n, int k) { /* CountClustersUsed, :55-63 */
  char seen[64] = {0};
  int used = 0;
  for (uint32_t v = 0; v < n; ++v)
    if (labels[v] >= 0 && labels[v] < k && labels[v] < 64 && !seen[labels[v]]) {
      seen[labels[v]] = 1;
      ++used;
    }
  return used;
}

/*
 * record_trace (optional, `iterations` entries): record objective after each finished iteration.
 * Returns 0, or -1 on bad parameters (CheckParams, cc_pbils_cpu.cpp:177-181).
 */
ORC_EXPORT int orc_pbils(const uint32_t *bits, uint32_t n, uint32_t words, uint64_t edges, const orc_params *p,
                         int threads, int32_t *labels_out, orc_result *res, int64_t *record_trace) {
  if (p->k < 1 || p->population < 1 || p->gww < 0.0 || p->gww > 0.5) return -1;
  const int size = p->population;
  solve_ctx c;
  memset(&c, 0, sizeof(c));
  c.bits = bits;
  c.n = n;
  c.words = words;
  c.edges = edges;
  c.p = p;
  c.init_stream = orc_stream_seed(p->seed, INIT_STREAM, 0);
  c.select_stream = orc_stream_seed(p->seed, SELECT_STREAM, 0);
  c.perturb_stream = orc_stream_seed(p->seed, PERTURB_STREAM, 0);
  c.pop = (state_t *)calloc(size, sizeof(state_t));
  c.next = (state_t *)calloc(size, sizeof(state_t));
  for (int s = 0; s < size; ++s) {
    state_alloc(&c.pop[s], (int)n, p->k);
    state_alloc(&c.next[s], (int)n, p->k);
  }
  c.fitness = (int64_t *)calloc(size, sizeof(int64_t));
  c.moves = (int64_t *)calloc(size, sizeof(int64_t));
  if (threads < 1) threads = 1;
  if (threads > size) threads = size;
  c.masks = (uint32_t **)calloc(threads, sizeof(uint32_t *));
  for (int t = 0; t < threads; ++t) c.masks[t] = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)p->k * words);
  int32_t *order = (int32_t *)calloc(size, sizeof(int32_t));

  parallel_for(threads, size, init_item, &c);

  memset(res, 0, sizeof(*res));
  int have = 0;
  int64_t record = 0;
  /* offer_record, cc_pbils_cpu.cpp:208-215: first minimum, strict improvement */
#define OFFER(states)                                                              \
  ({                                                                               \
    int b = 0;                                                                     \
    for (int s = 1; s < size; ++s)                                                 \
      if ((states)[s].f < (states)[b].f) b = s;                                    \
    int took = 0;                                                                  \
    if (!have || (states)[b].f < record) {                                         \
      record = (states)[b].f;                                                      \
      memcpy(labels_out, (states)[b].labels, sizeof(int32_t) * n);                 \
      have = 1;                                                                    \
      took = 1;                                                                    \
    }                                                                              \
    took;                                                                          \
  })
  OFFER(c.pop);
  int stall = 0;
  for (int it = 0; it < p->iterations; ++it) {
    c.iteration = it;
    for (int s = 0; s < size; ++s) c.fitness[s] = c.pop[s].f;
    parallel_for(threads, size, descend_item, &c);
    const int improved = OFFER(c.next);
    for (int s = 0; s < size; ++s) res->accepted_moves += c.moves[s];
    /* Progress::Next, cc_pbils.hpp:69-78 */
    res->iterations_done++;
    res->local_searches += size;
    stall = improved ? 0 : stall + 1;
    if (record_trace) record_trace[it] = record;
    if (stall >= p->early_stop) break;

    const int copies = orc_winner_copies(p->gww, size);
    if (copies > 0) {
      for (int s = 0; s < size; ++s) c.fitness[s] = c.next[s].f;
      orc_rank_slots(c.fitness, size, order);
      c.order = order;
      parallel_for(threads, copies, gww_item, &c);
    }
    if (p->k >= 2 && p->perturbation > 0.0) parallel_for(threads, size, perturb_item, &c);
    state_t *t = c.pop;
    c.pop = c.next;
    c.next = t;
  }
#undef OFFER
  res->objective = record;
  res->clusters_used = count_clusters(labels_out, n, p->k);

  for (int s = 0; s < size; ++s) {
    state_free(&c.pop[s]);
    state_free(&c.next[s]);
  }
  for (int t = 0; t < threads; ++t) free(c.masks[t]);
  free(c.masks);
  free(c.pop);
  free(c.next);
  free(c.fitness);
  free(c.moves);
  free(order);
  return 0;
}

/* ------------------------------------------------------------------------------------------
 * Neighborhood brute force: cuda/cc_verify_gpu.cu:21-35 (the reference's sequential check of
 * NeighborhoodCuda / NeighborhoodWithManyLocalSearchesCuda).  For v ascending: cluster 0 =
 * {v} + N(v), cluster 1 = the rest; optional LocalSearch; strict < keeps the smaller v.
 * Parallel over v with a per-v result, then reduced in v order (same answer as sequential).
 * ---------------------------------------------------------------------------------------- */
typedef struct {
  const uint32_t *bits;
  uint32_t n, words;
  uint64_t edges;
  int local_search;
  int64_t *f, *moves;
  uint32_t **masks;
  state_t *work;
} nb_ctx;

static void nb_item(void *vc, int v, int worker) {
  nb_ctx *c = (nb_ctx *)vc;
  state_t *s = &c->work[worker];
  for (uint32_t u = 0; u < c->n; ++u) s->labels[u] = (u == (uint32_t)v || joined(c->bits, c->words, v, u)) ? 0 : 1;
  rebuild(s, c->bits, c->words, c->edges, c->masks[worker]);
  int64_t m = 0;
  if (c->local_search) local_search(s, c->bits, c->words, &m);
  c->f[v] = s->f;
  c->moves[v] = m;
}

ORC_EXPORT int orc_neighborhood(const uint32_t *bits, uint32_t n, uint32_t words, uint64_t edges, int with_ls,
                                int threads, int32_t *labels_out, orc_result *res) {
  if (n == 0) return -1;
  if (threads < 1) threads = 1;
  if ((uint32_t)threads > n) threads = (int)n;
  nb_ctx c = {bits, n, words, edges, with_ls, NULL, NULL, NULL, NULL};
  c.f = (int64_t *)calloc(n, sizeof(int64_t));
  c.moves = (int64_t *)calloc(n, sizeof(int64_t));
  c.masks = (uint32_t **)calloc(threads, sizeof(uint32_t *));
  c.work = (state_t *)calloc(threads, sizeof(state_t));
  for (int t = 0; t < threads; ++t) {
    c.masks[t] = (uint32_t *)malloc(sizeof(uint32_t) * 2 * words);
    state_alloc(&c.work[t], (int)n, 2);
  }
  parallel_for(threads, (int)n, nb_item, &c);
  memset(res, 0, sizeof(*res));
  int best = 0;
  for (uint32_t v = 0; v < n; ++v) {
    if (c.f[v] < c.f[best]) best = (int)v;
    res->accepted_moves += c.moves[v];
  }
  res->objective = c.f[best];
  /* labels of the winning partition, after its local search when asked */
  state_t s;
  state_alloc(&s, (int)n, 2);
  for (uint32_t u = 0; u < n; ++u) s.labels[u] = (u == (uint32_t)best || joined(bits, words, best, u)) ? 0 : 1;
  rebuild(&s, bits, words, edges, c.masks[0]);
  int64_t m = 0;
  if (with_ls) local_search(&s, bits, words, &m);
  memcpy(labels_out, s.labels, sizeof(int32_t) * n);
  state_free(&s);
  res->local_searches = with_ls ? n : 0;
  res->clusters_used = count_clusters(labels_out, n, 2);
  for (int t = 0; t < threads; ++t) {
    free(c.masks[t]);
    state_free(&c.work[t]);
  }
  free(c.masks);
  free(c.work);
  free(c.f);
  free(c.moves);
  return 0;
}
