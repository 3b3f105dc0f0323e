// Status strings, version and the thread-local error message.
#include "mbc_internal.h"

namespace mbc {
const char *last_error_cstr();
}

extern "C" const char *mbc_status_string(mbc_status s)
{
  switch (s) {
    case MBC_OK: return "ok";
    case MBC_NOT_CONVERGED: return "not converged";
    case MBC_BREAKDOWN: return "pcg breakdown";
    case MBC_NONSPD_PIVOT: return "non-positive pivot";
    case MBC_BAD_ARG: return "bad argument";
    case MBC_CUDA_ERROR: return "cuda error";
    case MBC_TIMEOUT: return "device wait timed out";
    case MBC_NO_MEMORY: return "out of memory";
    case MBC_COVERAGE: return "aggregation coverage";
    case MBC_UNSUPPORTED: return "unsupported";
  }
  return "unknown status";
}

extern "C" const char *mbc_last_error(void) { return mbc::last_error_cstr(); }

extern "C" int32_t mbc_version(void) { return 100; }
