// Checks shb::guarded, the wrapper every status-returning C ABI entry point
// runs its body in: statuses pass through, a failed host allocation becomes
// SHB_ERR_OOM and any other exception SHB_ERR_INTERNAL, each with a message,
// and no exception leaves it.  Host code only.
#include <cstdio>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "shb_internal.h"

namespace shb {
static std::string g_last;
void set_error(const std::string& m) { g_last = m; }
shb_status cuda_fail(cudaError_t, const char*) { return SHB_ERR_CUDA; }
}  // namespace shb

int main() {
  int failures = 0;
  auto expect = [&](bool ok, const char* what) {
    if (!ok) {
      std::printf("FAIL %s (last error: %s)\n", what, shb::g_last.c_str());
      ++failures;
    }
  };
  expect(shb::guarded("shb_x", []() -> shb_status { return SHB_ERR_TIMEOUT; }) == SHB_ERR_TIMEOUT,
         "a status passes through");
  expect(shb::guarded("shb_x", []() -> shb_status { throw std::bad_alloc(); }) == SHB_ERR_OOM &&
             shb::g_last == "shb_x: host allocation failed",
         "bad_alloc becomes SHB_ERR_OOM");
  expect(shb::guarded("shb_x", []() -> shb_status {
           std::vector<char> v;
           v.reserve(v.max_size() + 1);  // throws std::length_error
           return SHB_OK;
         }) == SHB_ERR_INTERNAL && shb::g_last.rfind("shb_x: ", 0) == 0,
         "length_error becomes SHB_ERR_INTERNAL");
  expect(shb::guarded("shb_x", []() -> shb_status { throw 7; }) == SHB_ERR_INTERNAL &&
             shb::g_last == "shb_x: unknown exception",
         "a non-standard exception becomes SHB_ERR_INTERNAL");
  std::printf(failures ? "guard test failed\n" : "guard test passed\n");
  return failures ? 1 : 0;
}
