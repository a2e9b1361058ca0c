/*
 * gwb200: B200-native (sm_100a) kernels for the matched-filter hot path of gw-gpu-search.
 *
 * Plain C ABI. Every entry point takes device pointers, element counts and strides (in elements), a cudaStream_t
 * passed as void*, and returns an int status (GWB_OK = 0). Nothing here allocates device memory across calls: the
 * caller owns inputs, outputs and any workspace; a handle (gwb_handle_t) owns only cached cuFFT plans. Work is queued
 * on the caller's stream; no entry point synchronises the device unless its comment says so.
 *
 * Each entry point names the reference interface it replaces, as path:line within gw-gpu-search.
 */
#ifndef GWB200_H
#define GWB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define GWB_API __attribute__((visibility("default")))
#else
#define GWB_API
#endif

#define GWB_VERSION 1

/* status codes */
#define GWB_OK 0
#define GWB_ERR_SHAPE 1           /* inconsistent sizes */
#define GWB_ERR_NOT_POW2 2        /* a time length that must be a power of two is not */
#define GWB_ERR_EDGE_ORDER 3      /* chi-squared bin edges decreasing or outside [kmin, flen] */
#define GWB_ERR_ALLOC 4           /* device allocation (plan workspace) failed */
#define GWB_ERR_CUFFT 5           /* cuFFT returned an error */
#define GWB_ERR_TIMEOUT 6         /* a device-side wait gave up (kernel returned early) */
#define GWB_ERR_CUDA 7            /* CUDA runtime error on launch */
#define GWB_ERR_ARG 8             /* bad argument (null pointer, bad mode) */
#define GWB_ERR_NOT_IMPLEMENTED 9 /* a reference stage this library does not provide */
#define GWB_ERR_ALIGN 10          /* pointer or row stride misaligned for TMA (16 bytes) */
#define GWB_ERR_CAPACITY 11       /* a bounded output list overflowed (count still reported) */

/* ---- library ---------------------------------------------------------------------------------------------- */
GWB_API int gwb_version(void);
GWB_API const char* gwb_status_string(int status);
/* Message for the last non-zero status returned on this host thread. */
GWB_API const char* gwb_last_error(void);
/* Reads (and optionally clears) the current device's error word, set by kernels whose own checks or bounded waits
 * failed. Synchronous (one 16-byte copy). */
GWB_API int gwb_device_error(int* code, int* where, int* info0, int* info1, int clear);
GWB_API int gwb_num_sms(void);

/* ---- per-window peak picking ------------------------------------------------------------------------------ */
/* Replaces peak_kernel.window_peaks (pipeline/peak_kernel.py:41-47, kernel win_peak :10-36).
 * z: complex64 (rows, ldz) as interleaved float pairs. For each (row, w < nwin): max |z|^2 over samples
 * a0 + w*cw .. a0 + (w+1)*cw - 1 and its offset inside the window (first index on ties).
 * pmax, pidx: (rows, nwin), row stride nwin. */
GWB_API int gwb_window_peaks(const float* z, long long ldz, int rows, long long a0, int cw, int nwin, float* pmax,
                     int32_t* pidx, void* stream);

/* ---- reconstruction GEMM with |z|^2 and blocked argmax ---------------------------------------------------- */
/* Replaces fp_gemm.fused_peaks / gemm_absmax (pipeline/fp_gemm.py:14-44).
 * z_re = Are @ Z, z_im = Aim @ Z with Are, Aim (M, K) row-major (row stride lda) and Z (K, Tn) row-major (row
 * stride ldz). For each row and each output group of `group` consecutive 128-sample blocks (group = 1 reproduces the
 * reference's per-block output; group = cw/128 gives the per-window maximum directly) the maximum of
 * z_re^2 + z_im^2 and its sample index (first index on ties; samples >= Tn are ignored). V, I: (M, nout) with row
 * stride ldv, nout = ceil(ceil(Tn/128) / group).
 *
 * gwb_fused_peaks_f16: fp16 operands, fp32 accumulation, tcgen05 tensor cores (TMA-fed). K a multiple of 64,
 *   lda and ldz multiples of 8, base pointers 16-byte aligned.
 * gwb_fused_peaks_bf16x3: split-bf16 form. Each operand is given as a hi and lo bf16 pair (x ~ hi + lo); the
 *   accumulator receives hi*hi + hi*lo + lo*hi. Same alignment rules as f16.
 * gwb_fused_peaks_f32: plain fp32 operands on the fp32 pipe (no tensor cores), same output. K a multiple of 8. */
GWB_API int gwb_fused_peaks_f16(const uint16_t* Are, const uint16_t* Aim, long long lda, const uint16_t* Z, long long ldz,
                        int M, int K, long long Tn, int group, float* V, int32_t* I, long long ldv, void* stream);
GWB_API int gwb_fused_peaks_bf16x3(const uint16_t* Are_hi, const uint16_t* Are_lo, const uint16_t* Aim_hi,
                           const uint16_t* Aim_lo, long long lda, const uint16_t* Z_hi, const uint16_t* Z_lo,
                           long long ldz, int M, int K, long long Tn, int group, float* V, int32_t* I,
                           long long ldv, void* stream);
GWB_API int gwb_fused_peaks_f32(const float* Are, const float* Aim, long long lda, const float* Z, long long ldz, int M,
                        int K, long long Tn, int group, float* V, int32_t* I, long long ldv, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GWB200_H */
