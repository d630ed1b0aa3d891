// libdivsufsort's C ABI on the sufgpu engine (include/sufgpu/divsufsort_cuda.h):
// one process-wide context, created on the first call, serves divsufsort and
// divsufsort64 through sufgpu_divsufsort / sufgpu_divsufsort64.
#include "sufgpu/divsufsort_cuda.h"

#include <mutex>

#include "sufgpu/sufgpu.h"

namespace {

std::mutex g_mutex;
sufgpu_ctx* g_ctx = nullptr;
bool g_failed = false;

sufgpu_ctx* context_locked() {
  if (!g_ctx && !g_failed) {
    if (sufgpu_create(&g_ctx, 0) != SUFGPU_OK) {
      g_ctx = nullptr;
      g_failed = true;  // no device: every later call returns -2 at once
    }
  }
  return g_ctx;
}

struct Release {
  ~Release() {
    if (g_ctx) sufgpu_destroy(g_ctx);
  }
} g_release;

}  // namespace

extern "C" __attribute__((visibility("default"))) saint_t divsufsort(const sauchar_t* T,
                                                                     saidx_t* SA, saidx_t n) {
  if (!T || !SA || n < 0) return -1;
  std::lock_guard<std::mutex> lock(g_mutex);
  sufgpu_ctx* ctx = context_locked();
  if (!ctx) return -2;
  return sufgpu_divsufsort(ctx, T, SA, n);
}

extern "C" __attribute__((visibility("default"))) saint_t divsufsort64(const sauchar_t* T,
                                                                       saidx64_t* SA,
                                                                       saidx64_t n) {
  if (!T || !SA || n < 0) return -1;
  std::lock_guard<std::mutex> lock(g_mutex);
  sufgpu_ctx* ctx = context_locked();
  if (!ctx) return -2;
  return sufgpu_divsufsort64(ctx, T, SA, n);
}
