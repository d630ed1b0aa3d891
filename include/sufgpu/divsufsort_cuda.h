/* libdivsufsort's C entry points, built on the GPU.
 *
 * sufkit_b200/libdivsufsort_cuda.so exports divsufsort and divsufsort64 with
 * the exact signatures, types and return codes of libdivsufsort 2.0.2 as
 * vendored by sufkit (third_party/libdivsufsort/include/divsufsort.h and
 * divsufsort64.h; lib/divsufsort.c:331-358), so a program linked with
 * -ldivsufsort / -ldivsufsort64 relinks against it unchanged.  The suffix
 * array is sufgpu's (include/sufgpu/sufgpu.h), equal to divsufsort's word for
 * word.  One device context per process (device 0) serves every call; calls
 * are serialised.  Returns 0 on success, -1 for invalid arguments (T or SA
 * NULL, n < 0) and -2 when the device build fails (no device, allocation
 * failure, n above 2^32 - 1 symbols), as divsufsort returns -2 when it
 * cannot allocate.  It is a separate library because these names are
 * libdivsufsort's own: keeping them out of libsufgpu.so lets both be loaded
 * in one process. */
#ifndef SUFGPU_DIVSUFSORT_CUDA_H
#define SUFGPU_DIVSUFSORT_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint8_t sauchar_t;
typedef int32_t saint_t;
typedef int32_t saidx_t;
typedef int64_t saidx64_t;

saint_t divsufsort(const sauchar_t *T, saidx_t *SA, saidx_t n);
saint_t divsufsort64(const sauchar_t *T, saidx64_t *SA, saidx64_t n);

#ifdef __cplusplus
}
#endif

#endif /* SUFGPU_DIVSUFSORT_CUDA_H */
