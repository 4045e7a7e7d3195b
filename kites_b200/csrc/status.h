// status.h -- per-host-thread error text behind kites_last_error_string().
#pragma once
#include <stdarg.h>
#include <stdio.h>

namespace kites_internal {

char *error_buffer();  // thread-local, 512 bytes (defined in capi.cu)

inline void clear_error() { error_buffer()[0] = '\0'; }

inline int fail(int status, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(error_buffer(), 512, fmt, ap);
  va_end(ap);
  return status;
}

}  // namespace kites_internal
