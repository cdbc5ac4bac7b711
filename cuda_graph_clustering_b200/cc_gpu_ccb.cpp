// The reference's GPU backend entry points (include/cc_gpu.hpp:10-20) implemented over libccb's C ABI:
// linked in place of cuda/cc_pbils_gpu.cu, the reference's own cc_gpu command line (cli::Main,
// include/cc_cli.hpp:284-377) runs on this project's sm_100a kernels with no other change.  Parameters map
// field for field (include/cc_pbils.hpp:26-59); a nonzero status is rethrown as the std::runtime_error the
// reference would have thrown, with the same message.
//
// With CCB_CC_GPU_MAIN defined the file also provides main(), so that it plus the reference's host sources
// (src/cc_graph.cpp, src/cc_pbils_cpu.cpp for the recount) and libccb.so make the drop-in cc_gpu binary.
#include <stdexcept>

#include "cc_gpu.hpp"
#include "ccb.h"
#ifdef CCB_CC_GPU_MAIN
#include "cc_cli.hpp"
#endif

namespace cc {
namespace {

ccb_params ToC(const PbilsParams& p) {
  ccb_params c;
  ccb_params_init(&c);
  c.k = p.k;
  c.population = p.population;
  c.tournament = p.tournament;
  c.iterations = p.iterations;
  c.early_stop = p.early_stop;
  c.perturbation = p.perturbation;
  c.gww = p.gww;
  c.threads = p.threads;
  c.seed = p.seed;
  c.time_limit_sec = p.time_limit_sec;
  c.verbose = p.verbose;
  c.ls_kernel = p.ls_kernel;
  return c;
}

// algorithm: 0 PBILS, 1 Neighborhood, 2 Neighborhood with a local search per partition
PbilsResult Run(const Graph& g, const PbilsParams& p, int algorithm) {
  const ccb_params c = ToC(p);
  PbilsResult r;
  r.labels.resize(g.Size());
  ccb_result out{};
  const int status =
      algorithm == 0
          ? ccb_pbils_solve(g.Bits().data(), g.Size(), g.WordsPerRow(), g.EdgeCount(), &c, r.labels.data(), &out)
          : ccb_neighborhood_solve(g.Bits().data(), g.Size(), g.WordsPerRow(), g.EdgeCount(), &c, algorithm == 2,
                                   r.labels.data(), &out);
  if (status != CCB_OK) throw std::runtime_error(ccb_last_error());
  r.objective = out.objective;
  r.iterations_done = out.iterations_done;
  r.clusters_used = out.clusters_used;
  r.seconds = out.seconds;
  r.local_searches = out.local_searches;
  r.accepted_moves = out.accepted_moves;
  return r;
}

}  // namespace

PbilsResult SolveGpu(const Graph& g, const PbilsParams& p) { return Run(g, p, 0); }
PbilsResult SolveNeighborhoodGpu(const Graph& g, const PbilsParams& p) { return Run(g, p, 1); }
PbilsResult SolveNeighborhoodWithManyLocalSearchesGpu(const Graph& g, const PbilsParams& p) { return Run(g, p, 2); }

}  // namespace cc

#ifdef CCB_CC_GPU_MAIN
int main(int argc, char** argv) {
  return cc::cli::Main(argc, argv, "gpu", &cc::SolveGpu, &cc::SolveNeighborhoodGpu,
                       &cc::SolveNeighborhoodWithManyLocalSearchesGpu);
}
#endif
