// Status codes and the thread-local last-error message of the C ABI.
#include "ubolt_internal.h"

#include <cstdio>

namespace {
thread_local char g_last_error[1024] = "";
}

namespace ubolt {

int SetError(int status, const char *fmt, ...)
{
   va_list ap;
   va_start(ap, fmt);
   vsnprintf(g_last_error, sizeof g_last_error, fmt, ap);
   va_end(ap);
   return status;
}

void ClearError() { g_last_error[0] = '\0'; }

}  // namespace ubolt

extern "C" const char *ubolt_last_error(void) { return g_last_error; }

extern "C" const char *ubolt_version(void) { return "ubolt_b200 0.1 (sm_100a)"; }
