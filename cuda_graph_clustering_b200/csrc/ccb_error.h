// Thread-local message of the last failed C-ABI call, shared by every translation unit of libccb
// (returned by ccb_last_error()).
#pragma once

#include <string>

namespace ccb {
// Copies the message (truncated to the buffer) into thread-local storage; never allocates.
void SetLastError(const char* message);
inline void SetLastError(const std::string& message) { SetLastError(message.c_str()); }
const char* LastError();
}  // namespace ccb
