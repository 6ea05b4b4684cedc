// Error state and version of libnectb.
#include "common.cuh"

namespace nectb {

namespace {
thread_local char g_last_error[512] = {0};
}

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

void clear_error() { g_last_error[0] = 0; }

}  // namespace nectb

extern "C" const char* nectb_version(void) { return "nectb 0.1 sm_100a"; }
extern "C" const char* nectb_last_error(void) { return nectb::g_last_error; }
