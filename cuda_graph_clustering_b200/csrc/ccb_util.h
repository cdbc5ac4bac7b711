// Error plumbing shared by the C-ABI translation units: a failure carries a status and the message the
// reference's std::runtime_error would carry; Guard turns it into a status plus ccb_last_error().
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <new>
#include <stdexcept>
#include <string>

#include "ccb.h"
#include "ccb_error.h"

namespace ccb {

// NVTX range over a host-side phase (solve, batch run, server step, solver set-up): visible in Nsight
// timelines, a no-op when no tool is attached.
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

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

[[noreturn]] inline void Fail(int status, const std::string& message) { throw Failure{status, message}; }

template <typename F>
inline int Guard(F&& body) {
  try {
    body();
    SetLastError("");
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

}  // namespace ccb
