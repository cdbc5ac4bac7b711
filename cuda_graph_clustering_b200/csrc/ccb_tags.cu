// Graph::LoadTags (src/cc_graph.cpp:311-371) built on the device: objects with tag sets, an edge between two
// objects when the similarity of their tag sets (jaccard, cosine, dice, overlap) is at least the threshold.
//
// Objects with the same tag set have the same adjacency row apart from their own diagonal bit, so the host
// groups the sampled objects into classes (distinct tag sets, in order of first appearance) and the device
// builds one row per class: k_tags_rows gives each block a class c, evaluates its join row J[c][c'] =
// [similarity(c, c') >= threshold] over all classes into shared memory (one bit per class), then forms each
// word of the class's row from the classes of its 32 vertices and writes it to every member's row with the
// member's own bit cleared.  The similarity is computed in IEEE double with the reference's formulas and order
// of operations, so the comparison with the threshold, NaN for two empty sets included, is the same.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "ccb.h"
#include "ccb_graph.h"
#include "ccb_streams.cuh"
#include "ccb_util.h"

namespace ccb {
namespace {

// The reference's sampling stream (src/cc_graph.cpp:22).
constexpr uint64_t kSampleTag = 0x7A65;

enum TagSimilarity : int { kJaccard = 0, kCosine = 1, kDice = 2, kOverlap = 3 };

int ParseSimilarity(const std::string& name) {
  if (name == "jaccard") return kJaccard;
  if (name == "cosine") return kCosine;
  if (name == "dice") return kDice;
  if (name == "overlap") return kOverlap;
  Fail(CCB_ERR_INVALID, "unknown similarity '" + name + "', expected jaccard, cosine, dice or overlap");
}

// {"key": ["tag", ...], ...}: one tag set per object in file order, tags numbered by first appearance over the
// file, each set sorted without repeats (the format src/cc_graph.cpp:35-96 reads; an escaped character is
// taken as it is).
std::vector<std::vector<int>> ReadTagSets(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) Fail(CCB_ERR_INVALID, "cannot open file: " + path);
  std::stringstream buffer;
  buffer << in.rdbuf();
  const std::string text = buffer.str();
  size_t pos = 0;
  auto fail = [&](const char* what) {
    Fail(CCB_ERR_INVALID,
         std::string("malformed tags json (") + what + ") at byte " + std::to_string(pos) + " of " + path);
  };
  auto skip = [&] {
    while (pos < text.size() && std::isspace(static_cast<unsigned char>(text[pos]))) ++pos;
  };
  auto at = [&](char ch) {
    skip();
    return pos < text.size() && text[pos] == ch;
  };
  auto take = [&](char ch) {
    if (!at(ch)) fail("unexpected character");
    ++pos;
  };
  std::string token;
  auto string_token = [&] {
    take('"');
    token.clear();
    while (pos < text.size() && text[pos] != '"') {
      if (text[pos] == '\\') ++pos;
      if (pos < text.size()) token += text[pos++];
    }
    if (pos >= text.size()) fail("unterminated string");
    ++pos;
  };
  std::unordered_map<std::string, int> ids;
  std::vector<std::vector<int>> sets;
  take('{');
  if (at('}')) return sets;
  for (;;) {
    string_token();  // the object's key: a vertex is its position in the file
    take(':');
    take('[');
    std::vector<int> tags;
    if (!at(']')) {
      for (;;) {
        string_token();
        tags.push_back(ids.emplace(token, (int)ids.size()).first->second);
        if (at(']')) break;
        take(',');
      }
    }
    take(']');
    std::sort(tags.begin(), tags.end());
    tags.erase(std::unique(tags.begin(), tags.end()), tags.end());
    sets.push_back(std::move(tags));
    if (at('}')) break;
    take(',');
  }
  return sets;
}

// n objects of `total` by a partial Fisher-Yates shuffle on the sampling stream (src/cc_graph.cpp:373-381); all
// of them in file order when n is 0 or at least total.
std::vector<uint32_t> Sample(uint32_t total, uint32_t n, uint64_t seed) {
  std::vector<uint32_t> items(total);
  for (uint32_t i = 0; i < total; ++i) items[i] = i;
  if (n == 0 || n >= total) return items;
  uint64_t state = StreamSeed(seed, kSampleTag, 0);
  for (uint32_t i = 0; i < n; ++i) std::swap(items[i], items[i + DrawBelow(state, total - i)]);
  items.resize(n);
  return items;
}

__device__ __forceinline__ bool Joined(int kind, int common, int size_a, int size_b, double threshold) {
  const double inter = static_cast<double>(common);
  const double a = static_cast<double>(size_a);
  const double b = static_cast<double>(size_b);
  double s;
  switch (kind) {
    case kJaccard: s = inter / static_cast<double>(size_a + size_b - common); break;
    case kCosine: s = inter / sqrt(a * b); break;
    case kDice: s = 2.0 * inter / (a + b); break;
    default: s = inter / fmin(a, b); break;
  }
  return s >= threshold;  // false for NaN (two empty sets)
}

struct TagsArgs {
  const int32_t* class_off;   // [classes + 1] into class_tags
  const int32_t* class_tags;  // sorted tag ids of each class
  int classes;
  const int32_t* vertex_class;  // [n]
  const int32_t* member_off;    // [classes + 1] into members
  const int32_t* members;       // vertices grouped by class
  int n, words, pitch;
  int kind;
  double threshold;
  uint32_t* bits;
  unsigned long long* degree_sum;
};

constexpr int kTagsThreads = 256;

__global__ void __launch_bounds__(kTagsThreads) k_tags_rows(TagsArgs a) {
  extern __shared__ uint32_t s_join[];  // ceil(classes / 32) words
  __shared__ unsigned long long s_ones[kTagsThreads / 32];
  const int jwords = (a.classes + 31) / 32;
  for (int c = blockIdx.x; c < a.classes; c += gridDim.x) {
    const int32_t* ta = a.class_tags + a.class_off[c];
    const int na = a.class_off[c + 1] - a.class_off[c];
    for (int w = threadIdx.x; w < jwords; w += blockDim.x) {
      uint32_t word = 0;
      for (int bit = 0; bit < 32; ++bit) {
        const int o = w * 32 + bit;
        if (o >= a.classes) break;
        const int32_t* tb = a.class_tags + a.class_off[o];
        const int nb = a.class_off[o + 1] - a.class_off[o];
        int common = 0;
        for (int i = 0, j = 0; i < na && j < nb;) {  // both lists sorted ascending
          const int x = ta[i], y = tb[j];
          common += x == y;
          i += x <= y;
          j += y <= x;
        }
        if (Joined(a.kind, common, na, nb, a.threshold)) word |= 1u << bit;
      }
      s_join[w] = word;
    }
    __syncthreads();
    const int m0 = a.member_off[c], m1 = a.member_off[c + 1];
    unsigned long long ones = 0;
    for (int w = threadIdx.x; w < a.words; w += blockDim.x) {
      uint32_t word = 0;
      for (int bit = 0; bit < 32; ++bit) {
        const int u = w * 32 + bit;
        if (u >= a.n) break;
        const int cu = a.vertex_class[u];
        word |= ((s_join[cu >> 5] >> (cu & 31)) & 1u) << bit;
      }
      ones += __popc(word);
      for (int i = m0; i < m1; ++i) {
        const int v = a.members[i];
        a.bits[static_cast<size_t>(v) * a.pitch + w] = (v >> 5) == w ? word & ~(1u << (v & 31)) : word;
      }
    }
    for (int o = 16; o > 0; o /= 2) ones += __shfl_xor_sync(0xffffffffu, ones, o);
    if (threadIdx.x % 32 == 0) s_ones[threadIdx.x / 32] = ones;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long row = 0;
      for (int i = 0; i < kTagsThreads / 32; ++i) row += s_ones[i];
      // the class row holds each member's own bit when the class is joined with itself (every non-empty set
      // is); a vertex has no loop, so a member's degree is the row's ones minus that bit
      const unsigned long long self = (s_join[c >> 5] >> (c & 31)) & 1u;
      atomicAdd(a.degree_sum, (row - self) * static_cast<unsigned long long>(m1 - m0));
    }
    __syncthreads();
  }
}

template <typename T>
T* Upload(const std::vector<T>& v, cudaStream_t st, std::vector<void*>& owned) {
  void* p = nullptr;
  CCB_CUDA(cudaMalloc(&p, std::max<size_t>(1, v.size()) * sizeof(T)));
  owned.push_back(p);
  if (!v.empty()) CCB_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return static_cast<T*>(p);
}

ccb_graph* LoadTags(const char* path, const char* similarity, double threshold, uint32_t n, uint64_t seed,
                    cudaStream_t st) {
  if (path == nullptr || similarity == nullptr) Fail(CCB_ERR_INVALID, "null path or similarity");
  const int kind = ParseSimilarity(similarity);
  const std::vector<std::vector<int>> sets = ReadTagSets(path);
  if (sets.empty()) Fail(CCB_ERR_INVALID, std::string("no objects in ") + path);
  const std::vector<uint32_t> objects = Sample((uint32_t)sets.size(), n, seed);
  const uint32_t size = (uint32_t)objects.size();

  // classes: distinct tag sets in order of first appearance; members of each class contiguous
  std::map<std::vector<int>, int> class_of;
  std::vector<const std::vector<int>*> class_set;
  std::vector<int32_t> vertex_class(size);
  for (uint32_t v = 0; v < size; ++v) {
    const auto it = class_of.emplace(sets[objects[v]], (int)class_set.size());
    if (it.second) class_set.push_back(&it.first->first);
    vertex_class[v] = it.first->second;
  }
  const int classes = (int)class_set.size();
  std::vector<int32_t> class_off(classes + 1, 0), class_tags;
  for (int c = 0; c < classes; ++c) {
    class_tags.insert(class_tags.end(), class_set[c]->begin(), class_set[c]->end());
    class_off[c + 1] = (int32_t)class_tags.size();
  }
  std::vector<int32_t> member_off(classes + 1, 0), members(size);
  for (uint32_t v = 0; v < size; ++v) ++member_off[vertex_class[v] + 1];
  for (int c = 0; c < classes; ++c) member_off[c + 1] += member_off[c];
  std::vector<int32_t> cursor(member_off.begin(), member_off.end() - 1);
  for (uint32_t v = 0; v < size; ++v) members[cursor[vertex_class[v]]++] = (int32_t)v;

  const size_t smem = (size_t)(classes + 31) / 32 * sizeof(uint32_t);
  int optin = 0, device = 0, sms = 0;
  CCB_CUDA(cudaGetDevice(&device));
  CCB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  CCB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  if (smem + 1024 > (size_t)optin) {
    Fail(CCB_ERR_DEVICE_MEMORY, "too many distinct tag sets (" + std::to_string(classes) +
                                    ") for one join row in shared memory");
  }
  std::unique_ptr<ccb_graph> g(AllocateGraph(size, st));
  std::vector<void*> owned;
  struct Free {
    std::vector<void*>& p;
    ~Free() {
      for (void* x : p) cudaFree(x);
    }
  } free_on_exit{owned};
  TagsArgs a{};
  a.class_off = Upload(class_off, st, owned);
  a.class_tags = Upload(class_tags, st, owned);
  a.classes = classes;
  a.vertex_class = Upload(vertex_class, st, owned);
  a.member_off = Upload(member_off, st, owned);
  a.members = Upload(members, st, owned);
  a.n = (int)size;
  a.words = g->words;
  a.pitch = g->pitch;
  a.kind = kind;
  a.threshold = threshold;
  a.bits = g->bits;
  a.degree_sum = Upload(std::vector<unsigned long long>(1, 0ull), st, owned);
  CCB_CUDA(cudaFuncSetAttribute(k_tags_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = std::max(1, std::min(classes, 8 * sms));
  k_tags_rows<<<grid, kTagsThreads, smem, st>>>(a);
  CCB_CUDA(cudaGetLastError());
  unsigned long long degree_sum = 0;
  CCB_CUDA(cudaMemcpyAsync(&degree_sum, a.degree_sum, sizeof(degree_sum), cudaMemcpyDeviceToHost, st));
  CCB_CUDA(cudaStreamSynchronize(st));
  g->edges = (int64_t)(degree_sum / 2);
  FinishGraph(*g, st);
  return g.release();
}

}  // namespace
}  // namespace ccb

using namespace ccb;

extern "C" int ccb_graph_load_tags(const char* path, const char* similarity, double threshold, uint32_t n,
                                   uint64_t seed, void* stream, ccb_graph** out) {
  return Guard([&] {
    if (!out) Fail(CCB_ERR_STATE, "null output handle");
    *out = LoadTags(path, similarity, threshold, n, seed, static_cast<cudaStream_t>(stream));
  });
}
