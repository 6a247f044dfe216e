// Thread-local last-error message behind btd_last_error (no exception crosses the C ABI).
#include <cstring>
#include <string>

#include "btd.h"

namespace btd {
namespace {
thread_local std::string g_lastError;
}
void setError(const std::string& msg) { g_lastError = msg; }
}  // namespace btd

extern "C" int btd_last_error(char* buf, size_t n) {
  if (!buf || n == 0) return BTD_E_INVALID;
  size_t k = btd::g_lastError.size() < n - 1 ? btd::g_lastError.size() : n - 1;
  std::memcpy(buf, btd::g_lastError.data(), k);
  buf[k] = '\0';
  return BTD_OK;
}
