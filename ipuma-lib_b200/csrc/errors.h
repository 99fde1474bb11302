// errors.h -- the per-thread last-error message behind ipuma_last_error(),
// shared by the .cu files of the library.
#pragma once

namespace ipuma_internal {
// Records a printf-style message for the calling thread and returns `code`.
int fail(int code, const char* fmt, ...);
}  // namespace ipuma_internal
