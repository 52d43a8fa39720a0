// Host-side copies of the read-back path: pinned staging buffer -> the
// caller's result array, split over host threads.  The destinations are large
// arrays that nothing reads soon after, so on x86-64 hosts with AVX the copies
// write with streaming (non-temporal) stores: no read-for-ownership of the
// destination lines and no eviction of the cache, which roughly halves the
// host memory traffic of a read-back.  Elsewhere they are plain loops.
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include "xfb_internal.h"

namespace xfb {
namespace {

#if defined(__x86_64__)
bool have_avx() {
  static const bool ok = __builtin_cpu_supports("avx");
  return ok;
}

// dst[q] = double(src[q]), q < n: scalar until dst is 32-byte aligned, then
// eight elements per iteration with streaming stores.
__attribute__((target("avx"))) void widen_f32_nt(const float* src, double* dst, long long n) {
  long long q = 0;
  for (; q < n && (reinterpret_cast<uintptr_t>(dst + q) & 31u); ++q) dst[q] = static_cast<double>(src[q]);
  for (; q + 8 <= n; q += 8) {
    const __m256 v = _mm256_loadu_ps(src + q);
    _mm256_stream_pd(dst + q, _mm256_cvtps_pd(_mm256_castps256_ps128(v)));
    _mm256_stream_pd(dst + q + 4, _mm256_cvtps_pd(_mm256_extractf128_ps(v, 1)));
  }
  for (; q < n; ++q) dst[q] = static_cast<double>(src[q]);
  _mm_sfence();
}

__attribute__((target("avx"))) void copy_f64_nt(const double* src, double* dst, long long n) {
  long long q = 0;
  for (; q < n && (reinterpret_cast<uintptr_t>(dst + q) & 31u); ++q) dst[q] = src[q];
  for (; q + 8 <= n; q += 8) {
    _mm256_stream_pd(dst + q, _mm256_loadu_pd(src + q));
    _mm256_stream_pd(dst + q + 4, _mm256_loadu_pd(src + q + 4));
  }
  for (; q < n; ++q) dst[q] = src[q];
  _mm_sfence();
}

// Bytes: scalar head to a 32-byte destination boundary, 64 bytes per
// iteration with streaming stores, scalar tail.
__attribute__((target("avx"))) void copy_bytes_nt(const char* src, char* dst, size_t n) {
  size_t q = 0;
  for (; q < n && (reinterpret_cast<uintptr_t>(dst + q) & 31u); ++q) dst[q] = src[q];
  for (; q + 64 <= n; q += 64) {
    const __m256i a = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + q));
    const __m256i b = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + q + 32));
    _mm256_stream_si256(reinterpret_cast<__m256i*>(dst + q), a);
    _mm256_stream_si256(reinterpret_cast<__m256i*>(dst + q + 32), b);
  }
  if (q < n) std::memcpy(dst + q, src + q, n - q);
  _mm_sfence();
}
#endif

int copy_threads() { return std::max(1, std::min(16, omp_get_max_threads())); }

// Thread t's part [a, b) of n elements: parts of whole 64-element groups.
inline void part(long long n, int threads, int t, long long& a, long long& b) {
  const long long per = ((n + threads - 1) / threads + 63) / 64 * 64;
  a = std::min(n, t * per);
  b = std::min(n, a + per);
}

}  // namespace

void host_widen(const float* src, double* dst, long long n) {
  const int threads = copy_threads();
#pragma omp parallel for schedule(static) num_threads(threads)
  for (int t = 0; t < threads; ++t) {
    long long a, b;
    part(n, threads, t, a, b);
    if (a >= b) continue;
#if defined(__x86_64__)
    if (have_avx()) {
      widen_f32_nt(src + a, dst + a, b - a);
      continue;
    }
#endif
    for (long long q = a; q < b; ++q) dst[q] = static_cast<double>(src[q]);
  }
}

void host_widen(const double* src, double* dst, long long n) {
  const int threads = copy_threads();
#pragma omp parallel for schedule(static) num_threads(threads)
  for (int t = 0; t < threads; ++t) {
    long long a, b;
    part(n, threads, t, a, b);
    if (a >= b) continue;
#if defined(__x86_64__)
    if (have_avx()) {
      copy_f64_nt(src + a, dst + a, b - a);
      continue;
    }
#endif
    std::memcpy(dst + a, src + a, static_cast<size_t>(b - a) * sizeof(double));
  }
}

void host_copy(const void* src, void* dst, size_t bytes) {
  const int threads = copy_threads();
  const char* s = static_cast<const char*>(src);
  char* d = static_cast<char*>(dst);
#pragma omp parallel for schedule(static) num_threads(threads)
  for (int t = 0; t < threads; ++t) {
    long long a, b;
    part(static_cast<long long>(bytes), threads, t, a, b);
    if (a >= b) continue;
#if defined(__x86_64__)
    if (have_avx()) {
      copy_bytes_nt(s + a, d + a, static_cast<size_t>(b - a));
      continue;
    }
#endif
    std::memcpy(d + a, s + a, static_cast<size_t>(b - a));
  }
}

}  // namespace xfb
