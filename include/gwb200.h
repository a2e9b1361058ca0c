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

/* ---- shared record types (device arrays of these are exchanged between entry points) ---------------------- */
/* A window candidate: global template row (row of the caller's template array), segment, sample index within the
 * segment's time series, window index, rebuilt SNR sqrt(max |z|^2), the rebuilt complex SNR (zr, zi) and the index
 * of its unit. */
typedef struct {
    int32_t row, seg, sample, window;
    float approx, zr, zi;
    int32_t unit;
} GwbCand;
/* One exact-stage work unit: up to 8 candidates of one unit (consecutive in the candidate array). */
typedef struct {
    int32_t unit, first, count, pad;
} GwbGroup;
/* A (template row, segment) pair that has candidates: its chi-squared bin edges are computed once. */
typedef struct {
    int32_t row, seg, first, count;
} GwbUnit;
/* Exact-stage result for one candidate. */
typedef struct {
    float zr, zi;      /* exact complex SNR numerator z = sum_j Z_j */
    float pw;          /* sum_j |Z_j|^2 */
    float snr;         /* |z| norm */
    float chisq;       /* (nb pw - |z|^2) norm^2 */
    float newsnr;      /* pycbc newsnr of snr and chisq / dof */
    float fpeak;       /* (2 e[nb-1] - e[nb-2]) df */
    int32_t dof;       /* 2 nb - 2 */
} GwbPeak;

typedef struct gwb_handle_s* gwb_handle_t;

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
 * gwb_fused_peaks_f32: plain fp32 operands on the fp32 pipe (no tensor cores), same output, any K. */
GWB_API int gwb_fused_peaks_f16(const uint16_t* Are, const uint16_t* Aim, long long lda, const uint16_t* Z, long long ldz,
                        int M, int K, long long Tn, int group, float* V, int32_t* I, long long ldv, void* stream);
GWB_API int gwb_fused_peaks_bf16x3(const uint16_t* Are_hi, const uint16_t* Are_lo, const uint16_t* Aim_hi,
                           const uint16_t* Aim_lo, long long lda, const uint16_t* Z_hi, const uint16_t* Z_lo,
                           long long ldz, int M, int K, long long Tn, int group, float* V, int32_t* I,
                           long long ldv, void* stream);
GWB_API int gwb_fused_peaks_f32(const float* Are, const float* Aim, long long lda, const float* Z, long long ldz, int M,
                        int K, long long Tn, int group, float* V, int32_t* I, long long ldv, void* stream);
/* The fp32 form's kernel: 1 (default) copies the operand tiles by cp.async through a three-stage ring (needs K, lda,
 * ldz multiples of 4 and 16-byte aligned operands, else the synchronous kernel runs), 0 the synchronous kernel. Both
 * give the same V and I up to the order of the fp32 sums (identical K order: the same bits). */
GWB_API int gwb_f32_set_async(int on);

/* Compact complex form (same outputs): A = [Re As | Im As] (M, 2 Kh), Z = [Re zb ; Im zb] (2 Kh, Tn), each half Kh
 * wide (Kh a multiple of 16, halves zero-padded past r). z_re = ReA.ReZ - ImA.ImZ and z_im = ImA.ReZ + ReA.ImZ are
 * issued as four products per K step (the minus by the MMA's A negation), so A takes half the space of the
 * reference's stacked Are/Aim (pipeline/fp_filter.py:615-621) and stays in shared memory. form 0: fp16 A_hi, Z_hi;
 * 1: bf16; 2: split bf16 with A_lo, Z_lo (hi.hi + hi.lo + lo.hi); 3: fp8 e4m3 (the screening form, no reference
 * counterpart; Kh a multiple of 32), V = rowscale[i]^2 max |z|^2 with rowscale the per-row scale of A
 * (gwb_stacked_a8); rowscale is ignored by the other forms (may be NULL); 6: fp16 Z with A split into fp16 hi + lo
 * (A_lo; Z_lo unused), two products hi.Z + lo.Z (no reference counterpart: the rounding of A is removed, that of Z
 * kept). Kh <= 192 (forms 0, 1, 3); forms 2 and 6 keep A hi and lo in shared memory where they fit beside the Z
 * stages (one CTA: Kh <= 128; CTA pairs: Kh <= 160) and beyond that keep A hi there and stream A lo with the Z
 * chunks (Kh <= 320). lda, ldz in elements, multiples of 16 bytes. work (gwb_fused_peaks_cplx_work_bytes(M) bytes,
 * 16-byte aligned, may
 * be NULL): with it the CTAs take tile-granular ranges of the time axis (balanced to one 128-sample tile) and windows
 * cut by a range boundary are merged by a second kernel, bit for bit the same V and I; without it every CTA takes
 * whole windows (up to one window of imbalance between CTAs). With work, forms 0, 1 and 2 run on CTA pairs (clusters
 * of two CTAs, tcgen05.mma.cta_group::2 with M = 256 over two SMs, each SM loading half of every Z tile; the split
 * form's A lo resident or streamed per CTA) unless the launch table says otherwise (gwb_gemm_set_config); form 6 runs
 * one CTA per M block unless the table asks for pairs. */
GWB_API long long gwb_fused_peaks_cplx_work_bytes(int M);
/* Launch table of gwb_fused_peaks_cplx, per (form, Kh), filled by the autotuner (no reference counterpart; the
 * reference's own tuner is fp_gemm.pick_cfg, pipeline/fp_gemm.py:47-64): pair 1 = CTA pairs (forms 0, 1, 2, 6 with a
 * work buffer), 0 = one CTA per M block; stages = depth of the Z ring (0 = the most that fit, else at most that);
 * order = the CTA-pair kernel's MMA order (0: per K step re+=ReA.ReZ, re-=ImA.ImZ, im+=ImA.ReZ, im+=ReA.ImZ; 1: per K
 * step grouped by A half; 2: per Z chunk all real-part MMAs, then all imaginary-part ones; 3: per Z chunk one product
 * at a time; for the split forms 2 and 6 on pairs, order 1 takes K chunks of 64: A hi and lo resident beside two
 * stages where they fit, else A lo streamed in chunks of 64 where two such stages fit, else the chunks of 32 as order
 * 0). Forms 4 and 5 are the stacked drop-in kernels (gwb_fused_peaks_f16, gwb_fused_peaks_bf16x3; kh = K;
 * only stages applies). Process-wide, guarded by a mutex; a shape without an entry uses pair 1 (0 for form 6), stages 0, order 0 (1 for form 2).
 * Every entry computes the same products; the MMA order only changes the order of the fp32 accumulation. */
GWB_API int gwb_gemm_set_config(int form, int kh, int pair, int stages, int order);
GWB_API int gwb_gemm_clear_configs(void);
GWB_API int gwb_fused_peaks_cplx(int form, const void* A_hi, const void* A_lo, long long lda, const void* Z_hi,
                                 const void* Z_lo, long long ldz, int M, int Kh, long long Tn, int group, float* V,
                                 int32_t* I, long long ldv, const float* rowscale, void* work, long long work_bytes,
                                 void* stream);

/* ---- handle and transforms (cuFFT) ----------------------------------------------------------------------------- */
/* The handle caches cuFFT plans per (kind, n, batch, strides); plans are made on first use of a shape. Transforms are
 * unnormalised (cuFFT convention), as the reference's norm='forward' inverse transforms and its explicit dt / df
 * scale factors expect (pipeline/gpu_prep.py:109,148,156,197-199,421; pipeline/fp_filter.py:608). A complex-to-real
 * transform may overwrite its input. */
GWB_API int gwb_create(gwb_handle_t* out);
GWB_API int gwb_destroy(gwb_handle_t h);
GWB_API int gwb_fft_c2c(gwb_handle_t h, const float* in, float* out, long long n, int batch, long long idist,
                        long long odist, int inverse, void* stream);
GWB_API int gwb_fft_r2c(gwb_handle_t h, const float* in, float* out, long long n, int batch, long long idist,
                        long long odist, void* stream);
GWB_API int gwb_fft_c2r(gwb_handle_t h, const float* in, float* out, long long n, int batch, long long idist,
                        long long odist, void* stream);

/* ---- strain conditioning (pipeline/gpu_prep.py) -------------------------------------------------------------- */
/* Welch / segment frames: out[(r * nfr + f) * ldo + j] = x[r * ldx + s_f + j] * w[j] (w may be NULL), with
 * s_f = starts[f] if starts is given, else start + f * stride. Replaces the gathers of gpu_prep.py:104-108 and :420. */
GWB_API int gwb_frames(const float* x, long long ldx, int rows, long long start, long long stride,
                       const long long* starts, int nfr, int L, const float* w, float* out, long long ldo, void* stream);
/* Welch average over nfr frames of each row's rFFT X (complex, row stride ldx): p = |X dt|^2 in float32, bins 0 and
 * nbin-1 halved, then the median (mean of the two middle values for an even count) divided by bias, or the mean;
 * times fac. Replaces welch's per-row loop (gpu_prep.py:107-124). nfr <= 256 (mean), <= 8192 (median). */
GWB_API int gwb_welch_avg(const float* X, long long ldx, int rows, int nfr, int nbin, float dt, int median,
                          double bias, float fac, float* psd, long long ldp, void* stream);
/* np.interp of each PSD row (float64) from k df_old onto k df_new, k < nnew; replaces gpu_prep.interpolate
 * (gpu_prep.py:128-135). */
GWB_API int gwb_interp(const float* psd, long long ldp, int rows, int nold, double df_old, double df_new, int nnew,
                       float* out, long long ldo, void* stream);
/* Inverse spectrum truncation around two real transforms (gpu_prep.inverse_spectrum_truncation, :138-158):
 * pre: out (complex) = sqrt(1/P) for kmin <= k < N/2, else 0;  [C2R of length N = 2 (flen - 1)]
 * mid: q *= df, Hann taper of max_filter_len/2 samples at each end when taper != NULL, zero q[ts:te];  [R2C]
 * post: out = 1 / |X scale|^2. */
GWB_API int gwb_ist_pre(const float* P, long long ldp, int rows, int flen, int kmin, float* out, long long ldo,
                        void* stream);
GWB_API int gwb_ist_mid(float* q, long long ldq, int rows, int N, float df, int max_filter_len, const float* taper,
                        void* stream);
GWB_API int gwb_ist_post(const float* X, long long ldx, int rows, int flen, float scale, float* out, long long ldo,
                         void* stream);
/* D = stilde * IP and IP = 1/P (float64, 0 where P <= 0 or k < kmin), P = psd row pick[s] (gpu_stage2,
 * gpu_prep.py:447-451); stilde = X * scale with X the segment rFFT (scale = 1/sample rate). */
GWB_API int gwb_d_ip(const float* stilde, long long ldst, int nseg, const float* psd, long long ldp,
                     const int32_t* pick, int flen, int kmin, float scale, float* D, long long ldd, float* IP,
                     long long ldip, void* stream);
/* SVD metric sw = sqrt(mean over segments of IP) (float64 mean) and isw = 1/sw or 0 (fp_filter.py:363-364). */
GWB_API int gwb_sw(const float* IP, long long ldip, int nseg, int flen, float* sw, float* isw, void* stream);
/* detect_loud_glitches pieces (gpu_prep.py:175-209): taper_pad ramps the first and last cl samples and centres the
 * series in a zeroed buffer of length L; whiten scales a spectrum by dt (psd norm)^(-1/2) (0 where psd is inf);
 * above appends (index, value) for |x df| > thr over samples cl .. n-cl-1 of the centred series, at most cap, with
 * the true count in *count (zero it first). */
GWB_API int gwb_taper_pad(const float* s, long long n, int cl, long long L, long long pad_start, float* tapered,
                          float* sp, void* stream);
GWB_API int gwb_whiten(float* st, int nbin, const float* psd, float dt, float norm, void* stream);
GWB_API int gwb_above(const float* wt, long long pad_start, long long n, int cl, float df, float thr, int32_t* idx,
                      float* val, int cap, int32_t* count, void* stream);
/* Inverted-Tukey gates in place (gpu_prep.gate_taper, :212-231). gates: ngates x (offset, window samples, taper
 * samples, i1, i2) as computed on the host from GPS arithmetic; the product is taken in float64. */
GWB_API int gwb_apply_gates(float* x, long long n, const long long* gates, int ngates, void* stream);
/* The lal IIR highpass (gpu_prep.py:56-64) and the ldas FIR resampler (:67-84) are not provided: both return
 * GWB_ERR_NOT_IMPLEMENTED. */
GWB_API int gwb_highpass(void);
GWB_API int gwb_resample(void);

/* ---- template bank: templates, norms, tile SVD ------------------------------------------------------------------ */
/* TaylorF2 templates (the synthetic bank; the reference evaluates IMR waveforms, pipeline/imr_interp.py:56-85):
 * H[i, k] = f^(-7/6) exp(-i (Psi(f) - pi/4)) for kmin <= k < kmax[i], f = k df, else 0. */
GWB_API int gwb_taylorf2(const double* m1, const double* m2, const double* chi1, const double* chi2, const double* e0,
                         const int32_t* kmax, int n, double df, int kmin, int flen, double f_ecc, float* H,
                         long long ldh, void* stream);
/* Template norms (fp_filter.py:710-714) in float64: sig[i * ldsig + s] = 4 df sum_{k >= kmin} |H_ik|^2 IP_sk.
 * part: workspace of part_elems doubles (>= n * nseg; more allows more k-splits). */
GWB_API int gwb_sigma2(const float* H, long long ldh, int n, const float* IP, long long ldip, int nseg, int kmin,
                       int flen, double df, double* part, long long part_elems, double* sig, long long ldsig,
                       void* stream);
/* Template norms as gwb_sigma2, for callers that must not allocate device memory: no counterpart in the reference.
 * Some callers cannot let a library call cudaMalloc: a host program (for example a Go or Java service over the C ABI)
 * whose own pool owns every byte of device memory, code that runs between stream-capture begin and end, where an
 * allocation would break the capture, or a latency-bound loop where cudaMalloc / cudaFree synchronise the device.
 * This variant takes no workspace and allocates nothing: its split-k scratch is a static device array of 2^19
 * doubles (4 MiB) inside the library, held by every GPU that loads the library until the process exits, so
 * n * nseg must not exceed 524,288 (else GWB_ERR_CAPACITY, nothing queued). The first call on each device looks up
 * the array's device address (once, with that device current); make that first call before any stream capture.
 * All calls on a device share the one array: calls that overlap on the GPU (different streams, no ordering between
 * them) race and must not be issued. Each call overwrites every scratch element it later reads, so nothing carries
 * over from the previous call. */
GWB_API int gwb_sigma2_noalloc(const float* H, long long ldh, int n, const float* IP, long long ldip, int nseg,
                               int kmin, int flen, double df, double* sig, long long ldsig, void* stream);
/* Tile Gram matrix (svd_tile, fp_filter.py:578-581) in float64: G (n x n complex128, interleaved) =
 * sum_{k >= kmin} (H_k sw_k)(H_k sw_k)^H. part: workspace of part_elems doubles (>= 2 n^2). */
GWB_API int gwb_gram(const float* H, long long ldh, int n, const float* sw, int kmin, int flen, double* part,
                     long long part_elems, double* G, void* stream);
/* Hermitian eigendecomposition of the normalised Gram matrices (the eigh of svd_tile, fp_filter.py:583), float64, by
 * one-sided Jacobi on the device: nmat matrices of n[m] <= ld <= 256 rows, stored column-major complex128 in U
 * (U[(m ld + j) ld + i] = G_m[i, j]); one call runs one sweep (every column pair rotated once, n - 1 rounds of n/2
 * disjoint pairs) over U and V (V set to the identity when init != 0); *rotated counts the pairs rotated (cosine
 * above tol, both column norms above floor: columns below it, about 1e-12 of the largest, are numerically null), 0 when
 * the sweep found U's columns orthogonal. Then G_m V_m = U_m: the eigenvectors are V's columns and gwb_eigh_values
 * gives the eigenvalues, lam[m ld + j] = ||U_m[:, j]|| (unsorted). */
GWB_API int gwb_eigh_jacobi_sweep(double* U, double* V, const int* n, int nmat, int ld, int init, double tol,
                                  double floor, int* rotated, void* stream);
GWB_API int gwb_eigh_values(const double* U, const int* n, int nmat, int ld, double* lam, void* stream);
/* Basis filters (svd_tile, fp_filter.py:589-591): Vh[j, k] = sum_i Bm[j, i] H[i, k] sw[k] for k >= kmin, else 0;
 * Bm (r x n complex64). */
GWB_API int gwb_basis_vh(const float* Bm, long long ldb, int r, int n, const float* H, long long ldh, const float* sw,
                         int kmin, int flen, float* Vh, long long ldv, void* stream);

/* ---- basis series and stacked A (fp_filter.basis_series / stacked_A, pipeline/fp_filter.py:597-621) ----------- */
/* q[(s * rows + j) * ldq + k] = conj(Vh[j, k]) (D_s[k] isw[k]) for k < flen, for nseg consecutive segments D_s at
 * stride ldd. The caller keeps q[.., flen:ldq) zero; q is the input of a C2C inverse transform of length ldq. */
GWB_API int gwb_basis_premul(const float* Vh, long long ldvh, int rows, const float* D, long long ldd, int nseg,
                             const float* isw, long long flen, float* q, long long ldq, void* stream);
/* scale_out = sqrt(mean over rows x [a0, a0+Tn) of |zb|^2 / 2), float64 partial sums in a fixed order. partials:
 * npartials doubles; ticket: one uint32, zero on entry (left zero). */
GWB_API int gwb_basis_scale(const float* zb, long long ldz, int rows, long long a0, long long Tn, double* partials,
                            int npartials, uint32_t* ticket, float* scale_out, void* stream);
/* Z rows row0+j (real) and im_off+row0+j (imaginary) = zb[j, a0 + t] / scale for t < Tn; im_off = r gives the
 * reference's layout, im_off = Kh the compact one. form 0 fp16, 1 fp32, 2 bf16 hi in Z and lo in Zlo, 3 bf16. */
GWB_API int gwb_basis_pack(const float* zb, long long ldzb, int rows, int im_off, int row0, long long a0, long long Tn,
                           const float* scale, int form, void* Z, void* Zlo, long long ldz, void* stream);
/* As = A (norm_i scale); Are = [Re As, -Im As, 0...], Aim = [Im As, Re As, 0...] padded to Kp columns, or with
 * kh > 0 the compact single operand Are = [Re As (kh) | Im As (kh)] (Kp = 2 kh; Aim unused). nrm is read at
 * nrm[i * nrm_stride] (float64): the norm itself when df4 <= 0, else sigma^2 with norm = df4 / sqrt(sigma^2)
 * (df4 = 4 df). form as gwb_basis_pack, plus 5 = compact fp16 hi in Are and lo in Are_lo (for the GEMM's form 6). */
GWB_API int gwb_stacked_a(const float* A, long long lda, int n, int r, const double* nrm, long long nrm_stride,
                          double df4, const float* scale, int Kp, int kh, int form, void* Are, void* Aim,
                          void* Are_lo, void* Aim_lo, long long ldo, void* stream);
/* fp8 screening form of stacked A (no reference counterpart): compact row i = [Re As' | Im As'] with As'_ij = A_ij
 * norm_i zscale[j] (norm as gwb_stacked_a from nrm and df4; zscale the basis-row scales of Z from gwb_basis_fused
 * form 4), in e4m3 divided by the row's scale sa[i] = max_j |As'_ij| / 448 (out, n floats; the GEMM's and the
 * selection's rowscale). kh a multiple of 32, >= r; columns r..kh-1 of each half are zero. */
GWB_API int gwb_stacked_a8(const float* A, long long lda, int n, int r, const double* nrm, long long nrm_stride,
                           double df4, const float* zscale, int kh, void* A8, long long ldo, float* sa, void* stream);

/* Fused basis series in two passes over HBM (replaces premul + C2C inverse transform + pack, fp_filter.py:597-613).
 * N = N1 N2 (N1 = 2^ceil(log2(N) / 2)), k = N2 k1 + k2; only k <= N/2 enters (the reference zero-pads the half
 * spectrum). Inputs in four-step order (gwb_fourstep_order): Vp (rows x ldvp, the basis filters) and Dp (D isw of one
 * segment, the product the reference passes at fp_filter.py:741). Pass 1 forms q = conj(Vp) Dp and transforms over k1;
 * pass 2 transforms over k2 and packs z[a0 .. a0+Tn) / scale into Z (rows row0+j and im_off+row0+j; form as
 * gwb_basis_pack). tw: e^{2 pi i m / N}, m < N (gwb_fft_twiddles). W: workspace of wrows x N complex; rows are
 * transformed in batches of wrows through it. The scale is computed from the inputs of the first min(nfirst, wrows)
 * rows by Parseval (rms over the whole series; the reference takes the rms of the outputs over the analysed span of
 * its first batch; the scale cancels between Z and A). partials: >= that many rows x N2 / 8 doubles; ticket: one
 * uint32, zero on entry. N a power of two in [2^12, 2^20]; for N1 = 1024 (N = 2^19, 2^20) Vp and ldvp must be
 * 16-byte aligned (an even ldvp; fourstep_order pads its rows to N/2 + 2). */
GWB_API int gwb_fft_twiddles(long long N, float* tw, void* stream);
/* Four-step order of rows of a half spectrum: P[j][k2 (N1/2) + k1] = X[j][N2 k1 + k2] isw[k] for k1 < N1/2, k2 < N2,
 * P[j][N/2] = X[j][N/2] isw[N/2], zero where k >= flen (isw NULL: no weight). ldp >= N/2 + 1. */
GWB_API int gwb_fourstep_order(const float* X, long long ldx, int rows, const float* isw, long long flen, long long N,
                               float* P, long long ldp, void* stream);
/* form 4 (fp8 e4m3, the screening form; no reference counterpart): each basis row j gets its own scale,
 * rowscale[j] = (rms of one component of its series) / 16 from the row's |q|^2 sums (Parseval), and Z rows hold
 * z_j / rowscale[j] in e4m3 (saturating). rowscale: rows floats (out); rowpart: workspace of min(rows, wrows) x P
 * floats, P = N2 for N1 = 1024 else N2 / 8. Other forms ignore both (may be NULL). */
GWB_API int gwb_basis_fused(const float* Vp, long long ldvp, int rows, const float* Dp, long long N, const float* tw,
                            float* W, int wrows, long long a0, long long Tn, int form, void* Z, void* Zlo, long long ldz,
                            int im_off, int row0, int nfirst, double* partials, long long npartials, uint32_t* ticket,
                            float* scale, float* rowscale, float* rowpart, long long rowpart_elems, void* stream);
/* Columns of the transform per pass-2 CTA of gwb_basis_fused at N = 2^20, process-wide per Z form (0-4 as
 * gwb_basis_fused's `form`; -1 sets every form): 16 (default; a CTA writes runs of 16 consecutive Z samples: whole
 * 32-byte sectors for 16-bit Z, one 512-thread CTA per SM) or 8 (runs of 8, twice the L2 write requests).
 * Bit-identical results either way; the autotuner times both. gwb_basis_pass2_columns returns a form's setting. */
GWB_API int gwb_basis_set_pass2_columns(int form, int cols);
GWB_API int gwb_basis_pass2_columns(int form);
/* Z stores of the 16-column pass 2: 1 (default) pairs the samples (t, t + 1), t even, into one 32-bit word per plane
 * (64-bit for fp32) through a lane shuffle, wherever a0, Tn and ldz are even and the planes word-aligned (fp8 and
 * other shapes store per sample); 0 stores every sample separately. Bit-identical results either way. */
GWB_API int gwb_basis_set_pass2_pairs(int on);
/* The same basis series for N = 2^20 in one persistent launch that keeps W in L2 (same reference call,
 * fp_filter.py:597-613): rows go in chunks of pc through a ring of nslot slots of W (pc x nslot rows of N complex,
 * 128-byte aligned; wrows = the rows W holds), pass 1 running `look` chunks ahead of pass 2; each W tile's L2 lines
 * are dropped after pass 2 has read it, so per row HBM carries the basis filters in and Z out. Work items are taken in
 * order from a ticket; an item waits (bounded, one second, then GWB_ERR_TIMEOUT in the device error word) only for
 * items earlier in that order. The scale is the Parseval rms of the first chunk's rows (min(pc, rows) rows) instead
 * of min(nfirst, wrows) rows. partials: >= 1024 doubles; sync: gwb_basis_ring_sync_ints(rows) int32, cleared by the
 * call on the stream; fp8: rowpart >= rows x 1024 floats, rowscale rows floats. Other arguments as gwb_basis_fused.
 * gwb_basis_ring_set_config sets (pc in 1..4, nslot > look, look >= 0; 0 splits the grid into pass-1 and pass-2
 * CTAs) process-wide (default 2, 3, 1; the autotuner times the choices); gwb_basis_ring_rows and gwb_basis_ring_sync_ints size W and sync for the current one. */
GWB_API int gwb_basis_ring_set_config(int pc, int nslot, int look);
GWB_API int gwb_basis_ring_rows(void);
GWB_API int gwb_basis_ring_sync_ints(int rows);
GWB_API int gwb_basis_fused_ring(const float* Vp, long long ldvp, int rows, const float* Dp, long long N,
                                 const float* tw, float* W, int wrows, long long a0, long long Tn, int form, void* Z,
                                 void* Zlo, long long ldz, int im_off, int row0, double* partials, long long npartials,
                                 float* scale, float* rowscale, float* rowpart, long long rowpart_elems,
                                 int32_t* sync, long long sync_ints, void* stream);

/* ---- differentiation (the adjoint form; no reference counterpart: the reference has no gradients) ------------- */
/* Per trigger i, parameters params[i * 7 + (0..6)] = (Mc [M_sun], q = m2/m1 <= 1, chi1z, chi2z, e0 at f_ecc, t_c [s],
 * phi_c), the library's TaylorF2 template (gwb_taylorf2's phase) h = f^-7/6 exp(-i (Psi - pi/4 + 2 pi f t_c - phi_c))
 * on kmin <= k < kmax (the ISCO bin) against the trigger's over-whitened data D (row i, ldd) and inverse PSD IP (row i,
 * ldip; 0 shares one row): z = 4 df sum conj(h) D, sigma^2 = 4 df sum |h|^2 IP, snr = |z| / sigma, chisq over nbins
 * equal-power bins (the pipeline's edges, held fixed; dof 2 nbins - 2), newsnr (coinc_rank.py:39-46), and their
 * derivatives with respect to the 7 parameters (forward-mode dual numbers through the phase in float64; sums in
 * float32 (fp64 = 0) or float64). out row (ldout >= 28 doubles): snr, newsnr, chisq, sigma^2, z re, z im, kmax,
 * dsnr[7], dnewsnr[7], dchisq[7]. */
GWB_API int gwb_snr_grad(const double* params, int n, const float* D, long long ldd, const float* IP, long long ldip,
                         int flen, double df, int kmin, double f_ecc, int nbins, int fp64, double* out,
                         long long ldout, void* stream);
/* Phase metric per bank point (n x 7 x 7 doubles): g_ij = Cov_w(dPhi/dtheta_i, dPhi/dtheta_j) with w = |h|^2 IP, the
 * quadratic form of the phase-maximised match (1 - match ~ dtheta^T g dtheta / 2); the phi_c row and column are 0. */
GWB_API int gwb_phase_metric(const double* params, int n, const float* IP, long long ldip, int flen, double df,
                             int kmin, double f_ecc, double* g, void* stream);
/* One Levenberg-Marquardt step of the SNR ascent per trigger over the 6 parameters other than phi_c: out = params +
 * (g + lam[i] diag g)^-1 (dsnr / snr), from gwb_snr_grad's rows (res) and gwb_phase_metric (g), clamped to Mc > 0,
 * q in [0.05, 1], |chi| <= 0.99, e0 in [0, 0.5]; the caller adapts lam[i] per trigger. */
GWB_API int gwb_refine_step(const double* params, const double* res, long long ldres, const double* g,
                            const double* lam, int n, double* out, void* stream);

/* ---- candidate selection and the exact stage ---------------------------------------------------------------- */
/* Window candidates of one (tile, segment) (fp_filter.py:745-764): rows i < n whose windowed maximum vw (the fused
 * GEMM output with group = cw/128) exceeds thr2 become GwbCand records (row0 + i, seg, a0 + iw, window, sqrt(vw),
 * rebuilt z), appended per row in window order; each row with candidates becomes one GwbUnit and groups of <= 8
 * candidates become GwbGroup records. With ecut > 0, the reference's exact/rebuilt split (fp_filter.py:769-770,
 * --exact-snr: ecut = exact_snr (1 - margin), rthr = the SNR threshold, both compared in float32 with sqrt(vw)):
 * only windows with sqrt(vw) >= ecut are exact-stage candidates as above; those below ecut with sqrt(vw) > rthr are
 * appended to `rebuilt` (unit -1) and keep their rebuilt SNR and z. ecut <= 0: every window above thr2 is a
 * candidate (rebuilt may be NULL). counters[0..4]: candidates, groups, units, overflow flag (1 when a capacity was
 * exceeded; the row's list is then dropped), rebuilt peaks. Operands in the layout the GEMM used: stacked Are/Aim
 * (kh = 0, K = Kp) or compact A = [ReA | ImA] with Z = [ReZ ; ImZ] (kh > 0, Kp = 2 kh); form as gwb_basis_pack,
 * plus 4 = fp8 e4m3 (compact only), whose rebuilt z is multiplied by rowscale[i] (gwb_stacked_a8's sa; NULL for the
 * other forms), and 5 = fp16 Z with A as fp16 hi + lo (compact only). */
GWB_API int gwb_select_windows(const float* vw, const int32_t* iw, long long ldv, int n, int nw, float thr2,
                               float ecut, float rthr, long long a0, int row0, int seg, const void* Are,
                               const void* Aim, const void* Are_lo, const void* Aim_lo, long long lda, const void* Z,
                               const void* Zlo, long long ldz, int Kp, int kh, int form, const float* rowscale,
                               GwbCand* cands, int cand_cap, GwbGroup* groups, int group_cap, GwbUnit* units,
                               int unit_cap, GwbCand* rebuilt, int rebuilt_cap, int32_t* counters, void* stream);
/* Exact-stage selection by rank (the rank form of the reference's exact/rebuilt split, fp_filter.py:769-781): from
 * the lists gwb_select_windows wrote for a whole step with ecut <= 0 (cands, units, counters; every candidate
 * carries its rebuilt z), per segment only the candidates whose rebuilt SNR is at least the k-th largest of their
 * segment (ties kept) become exact-stage candidates in cands_out / groups_out / units_out / counters_out (same
 * record layout, candidate order kept within each unit); the others with rebuilt SNR > rthr are appended to
 * `rebuilt` (unit -1, counting on from counters[4]) and keep their rebuilt SNR and z. k = top_n (> 0), else
 * ceil(top_frac * count of the segment's candidates) with top_frac in (0, 1]. Segments are 0..nseg-1; the output
 * lists have cand_cap entries each. work: gwb_select_top_work_bytes(nseg, cand_cap) bytes, 256-byte aligned. No host
 * synchronisation: every count is read on the device. */
GWB_API long long gwb_select_top_work_bytes(int nseg, int cand_cap);
GWB_API int gwb_select_top(const GwbCand* cands, const GwbGroup* groups, const GwbUnit* units, const int32_t* counters,
                           int cand_cap, int nseg, int top_n, float top_frac, float rthr, GwbCand* cands_out,
                           GwbGroup* groups_out, GwbUnit* units_out, int32_t* counters_out, GwbCand* rebuilt,
                           int rebuilt_cap, void* work, long long work_bytes, void* stream);
/* Local search of a screening form (no reference counterpart; the fp8 screen's argmax is only near the window's
 * peak): every candidate of the selection's lists (cands, units, counters as gwb_select_windows writes them) becomes
 * 2 radius + 1 consecutive exact-stage candidates in cands_out / groups_out / units_out / counters_out at the samples
 * s - radius .. s + radius, clamped into its cluster window [a0 + window cw, a0 + (window + 1) cw); counters[4]
 * (rebuilt peaks) passes through. After gwb_exact_finalize on those lists, gwb_search_best keeps in each run of
 * 2 radius + 1 peaks the one with the largest snr (first on ties) and sets the others' snr to -1. radius 1..8. */
GWB_API int gwb_search_expand(const GwbCand* cands, const GwbUnit* units, const int32_t* counters, int radius,
                              long long a0, int cw, GwbCand* cands_out, int cand_cap, GwbGroup* groups_out,
                              GwbUnit* units_out, int32_t* counters_out, void* stream);
GWB_API int gwb_search_best(const int32_t* ccount, int cmax, int radius, GwbPeak* peaks, void* stream);
/* Chi-squared bin edges per unit (multi_filter.edges_per_template, pipeline/multi_filter.py:264-282; the fused
 * kernel of chisq_edges.py:92-143): E[u, 0..B] int32, B >= max nbins. Unit count = min(*ucount, umax) when ucount is
 * not NULL, else umax. nbins and kmax are indexed by the unit's row. offset_mode 1 reproduces the reference's
 * row-offset comparison (cs/tot + u > u + j/nb). */
GWB_API int gwb_edges(const GwbUnit* units, const int32_t* ucount, int umax, const float* H, long long ldh,
                      const float* IP, long long ldip, const int32_t* nbins, const int32_t* kmax, int kmin, int B,
                      int offset_mode, int32_t* E, void* stream);
/* Binned sums at peaks (chisq_kernel.bin_power_sums, pipeline/chisq_kernel.py:17-121): for every group and every
 * chunk of the band, Z_j partial sums into slots[(cand * nchunk + chunk) * B + j] (float2; zero slots first).
 * q_k = conj(H_k) D_k when D is given (fused mode), else q_k = H_k. tlen: the time length N (a power of two). */
GWB_API int gwb_bin_sums(const GwbGroup* groups, const int32_t* gcount, int gmax, const GwbUnit* units,
                         const GwbCand* cands, const int32_t* E, int B, const int32_t* nbins, const float* H,
                         long long ldh, const float* D, long long ldd, int kmin, int flen, long long tlen, float* slots,
                         void* stream);
/* The same binned sums (fused mode: D given) with the work in template-row order: the groups are counting-sorted
 * by their unit's row (nrows rows; a row outside [0, nrows) sets status[0] = 1) and the items run chunk by chunk, so
 * the groups in flight share a few template chunks and every segment's data chunk in L2 and each template band is
 * read from HBM about once per call instead of once per segment. Same slots as gwb_bin_sums, bit for bit. work:
 * gwb_bin_sums_work_bytes(gmax, nrows) bytes; status: one device int32 (cleared here). */
GWB_API long long gwb_bin_sums_work_bytes(int gmax, int nrows);
GWB_API int gwb_bin_sums_ordered(const GwbGroup* groups, const int32_t* gcount, int gmax, const GwbUnit* units,
                                 const GwbCand* cands, const int32_t* E, int B, const int32_t* nbins, int nrows,
                                 const float* H, long long ldh, const float* D, long long ldd, int kmin, int flen,
                                 long long tlen, void* work, long long work_bytes, int32_t* status, float* slots,
                                 void* stream);
/* Number of band chunks the slots are laid out for. */
GWB_API int gwb_exact_chunks(int flen, int kmin);
/* Appends one step's exact-stage results to a run-wide list on the device (no reference counterpart: the reference
 * copies peaks to the host per (tile, segment), fp_filter.py:752-753): n = min(counters[0], cap) candidates and their
 * peaks go to out_cands / out_peaks at the next free place of out_count (at most out_cap in all), each tagged `tag` in
 * out_tag; meta[tag * 8 + 0..7] records the step's five counters, the first place, the number appended and 1 when the
 * run list overflowed. work: 2 int32 of scratch. Sizes are read on the device: many steps can be queued (or captured
 * in one graph) and copied to the host once. */
GWB_API int gwb_append_results(const GwbCand* cands, const GwbPeak* peaks, const int32_t* counters, int cap, int tag,
                               GwbCand* out_cands, GwbPeak* out_peaks, int32_t* out_tag, int32_t* out_count,
                               int out_cap, int32_t* work, int32_t* meta, void* stream);
/* Process-wide choice of gwb_bin_sums_ordered's loads (the TMA-staged chi-squared tiles; no reference counterpart):
 * bulk 1 (the default) stages every tile of 2048 bins of the template and data bands in shared memory with
 * cp.async.bulk copies (double-buffered, bounded waits), 0 loads them straight from L2; the slots are bit for bit the
 * same. */
GWB_API int gwb_exact_set_staging(int bulk);
/* Per candidate: z, pw from the slots (float64 sums), and with sig given (float64, sig[row * ldsig + seg]) snr,
 * chisq, dof, newsnr (fp_filter.py:837-853, coinc_rank.py:39-46); fpeak (exact_stage.py:236-238). */
GWB_API int gwb_exact_finalize(const GwbCand* cands, const int32_t* ccount, int cmax, const GwbUnit* units,
                               const int32_t* E, int B, const int32_t* nbins, int kmin, int flen, const float* slots,
                               const double* sig, long long ldsig, double df, GwbPeak* out, void* stream);

/* ---- the whole filter step ---------------------------------------------------------------------------------- */
/* One tile of the bank as the step reads it (made once per bank: the SVD, fp_filter.py:576-593, and
 * gwb_fourstep_order of its basis filters). */
typedef struct {
    const float* Vp;     /* (r, ldvp) complex: basis filters in four-step order (ldvp even, rows 16-byte aligned) */
    long long ldvp;
    const float* A;      /* (n, r) complex64 mixing matrix, row stride lda (complex elements) */
    long long lda;
    int r, n, row0;      /* rank, templates, first row of the tile in the bank arrays */
} GwbTile;
typedef struct {
    int form;            /* GEMM precision: 0 fp16, 1 bf16, 2 split bf16, 6 fp16 with A split into hi + lo */
    int cw;              /* cluster window in samples, a multiple of 128 */
    long long a0, Tn;    /* analysed span of each segment: samples [a0, a0 + Tn) (Tn cut to whole windows) */
    float snr_threshold; /* exact-stage threshold; windows above (thr (1 - margin))^2 are candidates */
    float margin;
    int nbins_max;       /* B: the largest chi-squared bin count of the bank */
    int cand_cap;        /* capacity of the candidate, group and unit lists */
} GwbStepConfig;
/* One step of the compressed filter over a batch of conditioned segments (the loop of fp_filter.py:700-888, run_group
 * :741-836, with every candidate sent to the exact stage): template norms sig (M x nseg, float64, out), D isw in
 * four-step order, then for every tile and segment the fused basis series (two passes, gwb_basis_fused), stacked A,
 * the fused GEMM with |z|^2 and windowed argmax, the window selection; then edges, binned sums in template-row order
 * and the finalisation into cands / peaks (cand_cap each) with counters[0..4] as gwb_select_windows (counters[3] = 1:
 * a list overflowed). H (M x ldh complex), kmax and nbins per bank row; D, IP (nseg rows); isw = 1 / sw of the SVD
 * metric. work: gwb_filter_step_work_bytes(...) bytes; nothing is allocated and nothing is copied to the host. */
GWB_API long long gwb_filter_step_work_bytes(const GwbTile* tiles, int ntiles, int M, int nseg, long long tlen,
                                             int flen, int kmin, const GwbStepConfig* cfg);
GWB_API int gwb_filter_step(const GwbTile* tiles, int ntiles, const float* H, long long ldh, int M,
                            const int32_t* kmax, const int32_t* nbins, int kmin, double df, const float* D,
                            const float* IP, long long ldd, long long ldip, int nseg, const float* isw, long long tlen,
                            int flen, const GwbStepConfig* cfg, void* work, long long work_bytes, GwbCand* cands,
                            GwbPeak* peaks, int32_t* counters, double* sig, void* stream);

/* The conditioning of a batch of raw chunks, each one dataset holding one analysis segment and one PSD span
 * (gpu_stage2, gpu_prep.py:405-454, as gwb200.gpu_prep.BatchConditioner runs it). */
typedef struct {
    double sr;           /* sample rate (Hz); df = sr / tlen */
    double f_low;        /* low-frequency cutoff (Hz); kmin = (int)(f_low / df) */
    int psd_len;         /* Welch frame length (samples), Hann window; the frames must tile the chunk */
    int psd_stride;      /* Welch frame stride (samples) */
    int median;          /* 1: median average with PyCBC's bias (the reference's default); 0: mean */
    int inv_len;         /* inverse spectrum truncation length (samples); 0: none */
    int inv_taper;       /* 1: Hann taper in the truncation; 0: none (the reference's default) */
} GwbCondConfig;
/* A batch of nseg raw float32 chunks x (DYN_RANGE_FAC units, row stride ldx, tlen samples each) through the whole
 * path in one call (the batched entry behind the batched form, the per-dataset loop of fp_filter.py:700-888):
 * median-Welch PSD, interpolation, inverse spectrum truncation, segment rFFT, D and IP into the caller's D (nseg x
 * flen complex) and IP (nseg x flen), then gwb_filter_step (kmin and df from cond). h: a handle (cuFFT plans).
 * work: gwb_filter_batch_work_bytes(...) bytes; nothing is allocated except the handle's plans on first use, and
 * nothing is copied to the host. */
GWB_API long long gwb_filter_batch_work_bytes(const GwbTile* tiles, int ntiles, int M, int nseg, long long tlen,
                                              const GwbCondConfig* cond, const GwbStepConfig* cfg);
GWB_API int gwb_filter_batch(gwb_handle_t h, const float* x, long long ldx, int nseg, long long tlen,
                             const GwbCondConfig* cond, const GwbTile* tiles, int ntiles, const float* H,
                             long long ldh, int M, const int32_t* kmax, const int32_t* nbins, const float* isw,
                             const GwbStepConfig* cfg, void* work, long long work_bytes, float* D, float* IP,
                             GwbCand* cands, GwbPeak* peaks, int32_t* counters, double* sig, void* stream);

/* ---- consolidation (downstream of the exact stage) -------------------------------------------------------- */
/* Workspace bytes of gwb_consolidate for n items and nwin keep-loudest windows. */
GWB_API long long gwb_consolidate_work_bytes(int n, int nwin);
/* Keep mask of one dataset's items (device arrays), in one of two modes:
 *   mode 0, consolidate (pipeline/fp_filter.py:629-661, pycbc's EventManager.consolidate_events over the whole
 *     bank): stat = PyCBC's newsnr of snr and chisq / max(dof, 1) in float64 (fp_filter.py:250), or snr when
 *     use_chisq == 0; kept: stat >= newsnr_thr or exempt (has_exempt and snr >= exempt_snr, float32);
 *   mode 1, pre_keep (fp_filter.py:663-695): items with snr >= exact_cut (float32) are kept; of the rest, those with
 *     snr > thr pass the same cut with stat = snr, and with floor_in given (nfloor windows) those at or below the
 *     floor of their window are dropped.
 * Both: t = gps_start + ti / sr (ti int64 samples since the dataset's start, float64), and the gate veto drops
 * |t - g| <= w + taper + 0.5 for each of ng gates (device (ng, 3) float64: g, w, taper). With keep_interval > 0 the
 * non-exempt kept items are ranked in windows trunc(rint((t - gps_start) sr) / (keep_interval sr)) by stat
 * descending, ties to the smaller order key (position when order is NULL; keys must be distinct), and only the
 * keep_num first stay. floor_out (nwin doubles, may be NULL): the keep_num-th stat of every window that has at least
 * keep_num ranked items, -inf elsewhere (the reference's --pre-consolidate floor). keep: n bytes, 1 = kept.
 * status[0] (device int32, cleared here) becomes 1 when an item's window lies outside [0, nwin): the mask is then not
 * valid. work: gwb_consolidate_work_bytes(n, nwin) bytes. */
GWB_API int gwb_consolidate(int mode, int n, const float* snr, const float* chisq, const int32_t* dof,
                            const long long* ti, const long long* order, int use_chisq, double gps_start, double sr,
                            float exact_cut, float thr, double newsnr_thr, int has_exempt, float exempt_snr,
                            const double* gates, int ng, double keep_interval, int keep_num, const double* floor_in,
                            int nfloor, double* floor_out, int nwin, void* work, long long work_bytes, uint8_t* keep,
                            int32_t* status, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GWB200_H */
