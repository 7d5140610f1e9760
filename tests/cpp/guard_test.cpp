// Checks shb::guarded, the wrapper every status-returning C ABI entry point
// runs its body in: statuses pass through, a failed host allocation becomes
// SHB_ERR_OOM and any other exception SHB_ERR_INTERNAL, each with a message,
// and no exception leaves it.  And shb::run_host_threads, the library's
// host thread pool: every item is done, and an exception thrown on a worker
// thread reaches guarded instead of terminating the process.  Host code only.
#include <atomic>
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
  std::atomic<int> next{0}, done{0};
  auto items = [&] {
    for (int k; (k = next.fetch_add(1)) < 1000;) done.fetch_add(1);
  };
  shb::run_host_threads(8, items);
  expect(done.load() == 1000, "the pool does every item");
  std::atomic<int> claimed{0};
  const std::thread::id caller = std::this_thread::get_id();
  const shb_status st = shb::guarded("shb_pool", [&]() -> shb_status {
    shb::run_host_threads(4, [&] {
      for (int k; (k = claimed.fetch_add(1)) < 64;)
        if (k == 40 && std::this_thread::get_id() != caller) throw std::bad_alloc();
        else if (k == 40) throw std::runtime_error("caller thread");
    });
    return SHB_OK;
  });
  expect(st == SHB_ERR_OOM || (st == SHB_ERR_INTERNAL && shb::g_last == "shb_pool: caller thread"),
         "an exception on a pool thread comes back as a status");
  std::printf(failures ? "guard test failed\n" : "guard test passed\n");
  return failures ? 1 : 0;
}
