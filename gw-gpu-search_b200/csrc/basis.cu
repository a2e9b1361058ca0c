// Basis series (fp_filter.basis_series, pipeline/fp_filter.py:597-613), stacked A (stacked_A :615-621) and the window
// candidate selection with the rebuilt complex SNR (fp_filter.py:745-764).
//
// basis series for one segment and a batch of basis rows:
//   premul: q[j, k] = conj(Vh[j, k]) * (D[k] * isw[k]) for k < flen (the caller keeps q's upper half zero), the input
//           of a batched C2C inverse FFT (cuFFT, no 1/N: norm='forward' in the reference);
//   scale:  rms of the first batch over the analysed span, sqrt(mean(re^2 + im^2) / 2), reduced in float64 in a fixed
//           order (per-block partials, the last block to finish sums them);
//   pack:   Z rows 0..r-1 = Re / scale, rows r..2r-1 = Im / scale, over samples a0..a0+Tn-1, written as fp16 (the
//           reference's form), fp32, or a bf16 hi/lo pair (split form).
#include "common.cuh"
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

namespace gwb {
namespace {

constexpr int kThreads = 256;

__global__ void premul_kernel(const float2* __restrict__ Vh, long long ldvh, int rows, const float2* __restrict__ D,
                              long long ldd, const float* __restrict__ isw, long long flen, float2* __restrict__ q,
                              long long ldq) {
    const int j = blockIdx.y % rows, s = blockIdx.y / rows;
    const float2* v = Vh + (long long)j * ldvh;
    const float2* d = D + (long long)s * ldd;
    float2* o = q + ((long long)s * rows + j) * ldq;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < flen; k += (long long)gridDim.x * blockDim.x) {
        const float2 a = v[k], dk = d[k];
        const float w = isw[k];
        const float dr = dk.x * w, di = dk.y * w;             // D * isw, rounded as the reference's product
        o[k] = make_float2(fmaf(a.x, dr, a.y * di), fmaf(a.x, di, -(a.y * dr)));   // conj(v) * (D isw)
    }
}

// Partial sums of |zb|^2 over the first `rows` rows, samples a0..a0+Tn-1; the last block sums the partials in order
// and writes scale. ticket must be zero on entry; the last block resets it.
__global__ void scale_kernel(const float2* __restrict__ zb, long long ldz, int rows, long long a0, long long Tn,
                             double* __restrict__ partials, unsigned int* __restrict__ ticket,
                             float* __restrict__ scale_out) {
    double acc = 0.0;
    const long long total = (long long)rows * Tn;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const long long j = e / Tn, t = e - j * Tn;
        const float2 v = zb[j * ldz + a0 + t];
        acc += (double)v.x * v.x + (double)v.y * v.y;
    }
    __shared__ double red[kThreads / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) s += red[w];
        partials[blockIdx.x] = s;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double s = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) s += ((volatile double*)partials)[b];
        *scale_out = (float)sqrt(s / (double)total / 2.0);
        *ticket = 0;
    }
}

template <int FORM>   // 0 fp16, 1 fp32, 2 bf16 hi/lo, 3 bf16
__global__ void pack_kernel(const float2* __restrict__ zb, long long ldzb, int rows, int im_off, int row0, long long a0,
                            long long Tn, const float* __restrict__ scale, void* __restrict__ Z, void* __restrict__ Zlo,
                            long long ldz) {
    const int j = blockIdx.y;
    const float inv = 1.0f / *scale;
    const float2* src = zb + (long long)j * ldzb + a0;
    const long long re_row = row0 + j, im_row = im_off + row0 + j;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < Tn; t += (long long)gridDim.x * blockDim.x) {
        const float2 v = src[t];
        const float xr = v.x * inv, xi = v.y * inv;
        if (FORM == 0) {
            __half* z = static_cast<__half*>(Z);
            z[re_row * ldz + t] = __float2half_rn(xr);
            z[im_row * ldz + t] = __float2half_rn(xi);
        } else if (FORM == 1) {
            float* z = static_cast<float*>(Z);
            z[re_row * ldz + t] = xr;
            z[im_row * ldz + t] = xi;
        } else if (FORM == 3) {
            __nv_bfloat16* z = static_cast<__nv_bfloat16*>(Z);
            z[re_row * ldz + t] = __float2bfloat16_rn(xr);
            z[im_row * ldz + t] = __float2bfloat16_rn(xi);
        } else {
            __nv_bfloat16* hi = static_cast<__nv_bfloat16*>(Z);
            __nv_bfloat16* lo = static_cast<__nv_bfloat16*>(Zlo);
            const __nv_bfloat16 hr = __float2bfloat16_rn(xr), hm = __float2bfloat16_rn(xi);
            hi[re_row * ldz + t] = hr;
            hi[im_row * ldz + t] = hm;
            lo[re_row * ldz + t] = __float2bfloat16_rn(xr - __bfloat162float(hr));
            lo[im_row * ldz + t] = __float2bfloat16_rn(xi - __bfloat162float(hm));
        }
    }
}

template <int FORM>
__global__ void stacked_a_kernel(const float2* __restrict__ A, long long lda, int n, int r, const double* __restrict__ nrm,
                                 long long nrm_stride, double df4, const float* __restrict__ scale, int Kp, int kh,
                                 void* __restrict__ Are,
                                 void* __restrict__ Aim, void* __restrict__ Are_lo, void* __restrict__ Aim_lo,
                                 long long ldo) {
    const int i = blockIdx.x;
    if (i >= n) return;
    // nrm holds the norm itself, or sigma^2 when df4 = 4 df > 0 (norm = 4 df / sqrt(sigma^2), fp_filter.py:714)
    const double v = nrm[(long long)i * nrm_stride];
    const float f = (float)(df4 > 0.0 ? df4 / sqrt(v) : v) * *scale;
    for (int c = threadIdx.x; c < Kp; c += blockDim.x) {
        float re = 0.f, im = 0.f;
        if (kh > 0) {
            // compact: one row [Re As (Kh) | Im As (Kh)] in Are; Aim is not written
            const int cc = c < kh ? c : c - kh;
            if (cc < r) {
                const float2 a = A[(long long)i * lda + cc];
                re = c < kh ? a.x * f : a.y * f;
            }
        } else if (c < r) {
            const float2 a = A[(long long)i * lda + c];
            re = a.x * f;
            im = a.y * f;
        } else if (c < 2 * r) {
            const float2 a = A[(long long)i * lda + c - r];
            re = -(a.y * f);
            im = a.x * f;
        }
        const long long o = (long long)i * ldo + c;
        if (kh > 0) {
            if (FORM == 0) static_cast<__half*>(Are)[o] = __float2half_rn(re);
            else if (FORM == 1) static_cast<float*>(Are)[o] = re;
            else if (FORM == 5) {       // fp16 hi + lo (the fp16 form with split A)
                const __half hr = __float2half_rn(re);
                static_cast<__half*>(Are)[o] = hr;
                static_cast<__half*>(Are_lo)[o] = __float2half_rn(re - __half2float(hr));
            }
            else {
                const __nv_bfloat16 hr = __float2bfloat16_rn(re);
                static_cast<__nv_bfloat16*>(Are)[o] = hr;
                if (FORM == 2) static_cast<__nv_bfloat16*>(Are_lo)[o] = __float2bfloat16_rn(re - __bfloat162float(hr));
            }
            continue;
        }
        if (FORM == 3) {
            static_cast<__nv_bfloat16*>(Are)[o] = __float2bfloat16_rn(re);
            static_cast<__nv_bfloat16*>(Aim)[o] = __float2bfloat16_rn(im);
        } else if (FORM == 0) {
            static_cast<__half*>(Are)[o] = __float2half_rn(re);
            static_cast<__half*>(Aim)[o] = __float2half_rn(im);
        } else if (FORM == 1) {
            static_cast<float*>(Are)[o] = re;
            static_cast<float*>(Aim)[o] = im;
        } else {
            const __nv_bfloat16 hr = __float2bfloat16_rn(re), hm = __float2bfloat16_rn(im);
            static_cast<__nv_bfloat16*>(Are)[o] = hr;
            static_cast<__nv_bfloat16*>(Aim)[o] = hm;
            static_cast<__nv_bfloat16*>(Are_lo)[o] = __float2bfloat16_rn(re - __bfloat162float(hr));
            static_cast<__nv_bfloat16*>(Aim_lo)[o] = __float2bfloat16_rn(im - __bfloat162float(hm));
        }
    }
}

// fp8 screening form, compact A: row i of [Re As' | Im As'] with As'_ij = A_ij norm_i rowscale_z[j] (the basis-row
// scales of Z folded in), quantised to e4m3 with the row's own scale sa_i = max_j |As'_ij| / 448 (written to sa).
__global__ void stacked_a8_kernel(const float2* __restrict__ A, long long lda, int n, int r,
                                  const double* __restrict__ nrm, long long nrm_stride, double df4,
                                  const float* __restrict__ zscale, int kh, __nv_fp8_storage_t* __restrict__ A8,
                                  long long ldo, float* __restrict__ sa) {
    const int i = blockIdx.x;
    if (i >= n) return;
    const double v = nrm[(long long)i * nrm_stride];
    const float f = (float)(df4 > 0.0 ? df4 / sqrt(v) : v);
    auto value = [&](int c) {
        const int cc = c < kh ? c : c - kh;
        if (cc >= r) return 0.f;
        const float2 a = A[(long long)i * lda + cc];
        return (c < kh ? a.x : a.y) * f * zscale[cc];
    };
    float m = 0.f;
    for (int c = threadIdx.x; c < 2 * kh; c += blockDim.x) m = fmaxf(m, fabsf(value(c)));
    __shared__ float red[32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    float mx = 0.f;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) mx = fmaxf(mx, red[w]);
    const float s = mx > 0.f ? mx / 448.f : 1.f;
    if (threadIdx.x == 0) sa[i] = s;
    const float inv = 1.f / s;
    for (int c = threadIdx.x; c < 2 * kh; c += blockDim.x)
        A8[(long long)i * ldo + c] = __nv_cvt_float_to_fp8(value(c) * inv, __NV_SATFINITE, __NV_E4M3);
}

__device__ __forceinline__ float ld_as_float(const void* p, long long i, int form) {
    if (form == 0 || form == 5) return __half2float(static_cast<const __half*>(p)[i]);
    if (form == 1) return static_cast<const float*>(p)[i];
    if (form == 4)
        return __half2float(__half(__nv_cvt_fp8_to_halfraw(static_cast<const __nv_fp8_storage_t*>(p)[i], __NV_E4M3)));
    return __bfloat162float(static_cast<const __nv_bfloat16*>(p)[i]);    // forms 2 (hi or lo) and 3
}

// Window candidates of one (tile, segment). One block per template row: windows whose maximum |z|^2 (the fused GEMM's
// windowed output) exceeds thr2 become candidates, written contiguously in window order at an offset taken with one
// atomic per row; the row's candidates are cut into groups of at most 8 (one group = one exact-stage work unit) and
// the row is registered once as an edges unit. The rebuilt complex SNR Are[row].Z[:, col] + i Aim[row].Z[:, col]
// (fp_filter.py:760-764) is computed for each candidate; for the split form the hi and lo parts are summed. With
// ecut > 0 the reference's split (fp_filter.py:769-770) divides the windows: rebuilt SNR >= ecut go to the exact
// stage as above, the others above rthr become rebuilt peaks (their own list, counters[4], unit -1), which keep the
// rebuilt SNR and phase.
__global__ void select_kernel(const float* __restrict__ vw, const int32_t* __restrict__ iw, long long ldv, int n,
                              int nw, float thr2, float ecut, float rthr, long long a0, int row0, int seg,
                              const void* __restrict__ Are, const void* __restrict__ Aim,
                              const void* __restrict__ Are_lo, const void* __restrict__ Aim_lo, long long lda,
                              const void* __restrict__ Z, const void* __restrict__ Zlo, long long ldz, int Kp, int kh,
                              int form, const float* __restrict__ rowscale, GwbCand* __restrict__ cands,
                              int cand_cap, GwbGroup* __restrict__ groups, int group_cap, GwbUnit* __restrict__ units,
                              int unit_cap, GwbCand* __restrict__ rebuilt, int rebuilt_cap,
                              int32_t* __restrict__ counters) {
    const int row = blockIdx.x;
    if (row >= n) return;
    const float* v = vw + (long long)row * ldv;
    // class of a window: 1 = exact-stage candidate (rebuilt SNR >= ecut), 2 = rebuilt peak (below ecut, above rthr)
    auto cls = [&](int w) -> int {
        const float x = v[w];
        if (!(x > thr2)) return 0;
        const float a = sqrtf(x);
        return a >= ecut ? 1 : (a > rthr ? 2 : 0);
    };
    __shared__ int s_cnt[2], s_base, s_unit, s_gbase, s_rbase, s_ok;
    __shared__ int s_warp[kThreads / 32];
    if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    int ce = 0, cr = 0;
    for (int w = threadIdx.x; w < nw; w += blockDim.x) {
        const int c = cls(w);
        ce += c == 1;
        cr += c == 2;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        ce += __shfl_down_sync(0xffffffffu, ce, off);
        cr += __shfl_down_sync(0xffffffffu, cr, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&s_cnt[0], ce);
        atomicAdd(&s_cnt[1], cr);
    }
    __syncthreads();
    const int total = s_cnt[0], rtotal = s_cnt[1];
    if (total == 0 && rtotal == 0) return;
    const int ng = (total + 7) / 8;
    if (threadIdx.x == 0) {
        int ok = 0;
        if (total > 0) {
            s_base = atomicAdd(&counters[0], total);
            s_gbase = atomicAdd(&counters[1], ng);
            s_unit = atomicAdd(&counters[2], 1);
            if (s_base + total > cand_cap || s_gbase + ng > group_cap || s_unit >= unit_cap) atomicOr(&counters[3], 1);
            else {
                units[s_unit] = GwbUnit{row0 + row, seg, s_base, total};
                ok |= 1;
            }
        }
        if (rtotal > 0) {
            s_rbase = atomicAdd(&counters[4], rtotal);
            if (rebuilt == nullptr || s_rbase + rtotal > rebuilt_cap) atomicOr(&counters[3], 1);
            else ok |= 2;
        }
        s_ok = ok;
    }
    __syncthreads();
    const int okf = s_ok;
    if (okf & 1)
        for (int g = threadIdx.x; g < ng; g += blockDim.x)
            groups[s_gbase + g] = GwbGroup{s_unit, s_base + 8 * g, min(8, total - 8 * g), 0};
    // ordered writes (window order within the row): chunks of blockDim windows, prefix over warps
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int want = 1; want <= 2; ++want) {
        if (!(okf & want)) continue;
        GwbCand* out = want == 1 ? cands + s_base : rebuilt + s_rbase;
        const int unit = want == 1 ? s_unit : -1;
        int written = 0;
        for (int w0 = 0; w0 < nw; w0 += blockDim.x) {
            const int w = w0 + threadIdx.x;
            const bool hit = w < nw && cls(w) == want;
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) s_warp[warp] = __popc(m);
            __syncthreads();
            int before = 0;
            for (int k = 0; k < warp; ++k) before += s_warp[k];
            int chunk_total = 0;
            for (int k = 0; k < kThreads / 32; ++k) chunk_total += s_warp[k];
            if (hit) {
                const int pos = written + before + __popc(m & ((1u << lane) - 1));
                const int col = iw[(long long)row * ldv + w];
                GwbCand cd;
                cd.row = row0 + row;
                cd.seg = seg;
                cd.sample = (int)(a0 + col);
                cd.window = w;
                cd.approx = sqrtf(v[w]);
                cd.zr = 0.f;
                cd.zi = 0.f;
                cd.unit = unit;
                out[pos] = cd;
            }
            written += chunk_total;
            __syncthreads();
        }
    }
    // rebuilt complex SNR of each candidate of this row: one warp per candidate, lanes over K
    auto ldz_ = [&](long long c, int col) {
        return ld_as_float(Z, c * ldz + col, form) + (form == 2 ? ld_as_float(Zlo, c * ldz + col, 2) : 0.f);
    };
    auto lda_ = [&](const void* hi, const void* lo, long long c) {
        return ld_as_float(hi, (long long)row * lda + c, form) +
               (form == 2 || form == 5 ? ld_as_float(lo, (long long)row * lda + c, form) : 0.f);
    };
    const int ne = (okf & 1) ? total : 0, nr = (okf & 2) ? rtotal : 0;
    for (int i = warp; i < ne + nr; i += kThreads / 32) {
        GwbCand* cd = i < ne ? cands + s_base + i : rebuilt + s_rbase + (i - ne);
        const int col = cd->sample - (int)a0;
        float zr = 0.f, zi = 0.f;
        if (kh > 0) {       // compact operands: A = [ReA | ImA], Z = [ReZ ; ImZ]
            for (int c = lane; c < kh; c += 32) {
                const float ar = lda_(Are, Are_lo, c), ai = lda_(Are, Are_lo, kh + c);
                const float zc = ldz_(c, col), zs = ldz_(kh + c, col);
                zr = fmaf(ar, zc, fmaf(-ai, zs, zr));
                zi = fmaf(ai, zc, fmaf(ar, zs, zi));
            }
        } else {
            for (int c = lane; c < Kp; c += 32) {
                const float zc = ldz_(c, col);
                zr = fmaf(lda_(Are, Are_lo, c), zc, zr);
                zi = fmaf(lda_(Aim, Aim_lo, c), zc, zi);
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            zr += __shfl_down_sync(0xffffffffu, zr, off);
            zi += __shfl_down_sync(0xffffffffu, zi, off);
        }
        if (lane == 0) {
            const float rs = rowscale ? rowscale[row] : 1.f;     // fp8: the row scale of A
            cd->zr = zr * rs;
            cd->zi = zi * rs;
        }
    }
}

}  // namespace
}  // namespace gwb

extern "C" {

int gwb_basis_premul(const float* Vh, long long ldvh, int rows, const float* D, long long ldd, int nseg,
                     const float* isw, long long flen, float* q, long long ldq, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(Vh && D && isw && q, GWB_ERR_ARG, "basis_premul: null pointer");
    GWB_CHECK_ARG(rows > 0 && nseg > 0 && flen > 0 && ldvh >= flen && ldd >= flen && ldq >= flen, GWB_ERR_SHAPE,
                  "basis_premul: rows=%d nseg=%d flen=%lld", rows, nseg, flen);
    GWB_CHECK_ARG((long long)rows * nseg < 65536, GWB_ERR_SHAPE, "basis_premul: too many rows");
    const int gx = (int)std::min<long long>(cdiv(flen, kThreads), 512);
    dim3 grid(gx, rows * nseg);
    premul_kernel<<<grid, kThreads, 0, (cudaStream_t)stream>>>(reinterpret_cast<const float2*>(Vh), ldvh, rows,
                                                                reinterpret_cast<const float2*>(D), ldd, isw, flen,
                                                                reinterpret_cast<float2*>(q), ldq);
    GWB_LAUNCH_CHECK("premul_kernel");
    return GWB_OK;
}

int gwb_basis_scale(const float* zb, long long ldz, int rows, long long a0, long long Tn, double* partials,
                    int npartials, uint32_t* ticket, float* scale_out, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(zb && partials && ticket && scale_out, GWB_ERR_ARG, "basis_scale: null pointer");
    GWB_CHECK_ARG(rows > 0 && Tn > 0 && a0 >= 0 && a0 + Tn <= ldz && npartials > 0, GWB_ERR_SHAPE,
                  "basis_scale: rows=%d a0=%lld Tn=%lld ldz=%lld", rows, a0, Tn, ldz);
    const int nb = (int)std::min<long long>((long long)npartials, cdiv((long long)rows * Tn, kThreads * 8));
    scale_kernel<<<nb, kThreads, 0, (cudaStream_t)stream>>>(reinterpret_cast<const float2*>(zb), ldz, rows, a0, Tn,
                                                             partials, ticket, scale_out);
    GWB_LAUNCH_CHECK("scale_kernel");
    return GWB_OK;
}

int gwb_basis_pack(const float* zb, long long ldzb, int rows, int im_off, int row0, long long a0, long long Tn,
                   const float* scale, int form, void* Z, void* Zlo, long long ldz, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(zb && scale && Z && (form != 2 || Zlo), GWB_ERR_ARG, "basis_pack: null pointer");
    GWB_CHECK_ARG(form >= 0 && form <= 3, GWB_ERR_ARG, "basis_pack: form %d", form);
    GWB_CHECK_ARG(rows > 0 && row0 >= 0 && row0 + rows <= im_off && Tn > 0 && a0 >= 0 && a0 + Tn <= ldzb && ldz >= Tn,
                  GWB_ERR_SHAPE, "basis_pack: rows=%d row0=%d im_off=%d a0=%lld Tn=%lld", rows, row0, im_off, a0, Tn);
    const int gx = (int)std::min<long long>(cdiv(Tn, kThreads), 1024);
    dim3 grid(gx, rows);
    const float2* src = reinterpret_cast<const float2*>(zb);
    cudaStream_t s = (cudaStream_t)stream;
    if (form == 0) pack_kernel<0><<<grid, kThreads, 0, s>>>(src, ldzb, rows, im_off, row0, a0, Tn, scale, Z, Zlo, ldz);
    else if (form == 1) pack_kernel<1><<<grid, kThreads, 0, s>>>(src, ldzb, rows, im_off, row0, a0, Tn, scale, Z, Zlo, ldz);
    else if (form == 2) pack_kernel<2><<<grid, kThreads, 0, s>>>(src, ldzb, rows, im_off, row0, a0, Tn, scale, Z, Zlo, ldz);
    else pack_kernel<3><<<grid, kThreads, 0, s>>>(src, ldzb, rows, im_off, row0, a0, Tn, scale, Z, Zlo, ldz);
    GWB_LAUNCH_CHECK("pack_kernel");
    return GWB_OK;
}

int gwb_stacked_a(const float* A, long long lda, int n, int r, const double* nrm, long long nrm_stride, double df4,
                  const float* scale, int Kp, int kh, int form, void* Are, void* Aim, void* Are_lo, void* Aim_lo,
                  long long ldo, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(A && nrm && scale && Are && (kh > 0 || Aim) &&
                  (form != 2 || (Are_lo && (kh > 0 || Aim_lo))) && (form != 5 || Are_lo), GWB_ERR_ARG,
                  "stacked_a: null pointer");
    GWB_CHECK_ARG(form >= 0 && form <= 5 && form != 4 && (form != 5 || kh > 0), GWB_ERR_ARG,
                  "stacked_a: form %d (0 fp16, 1 fp32, 2 split bf16, 3 bf16, 5 fp16 with split A, compact)", form);
    GWB_CHECK_ARG(n > 0 && r > 0 && lda >= r && ldo >= Kp && (kh > 0 ? (kh >= r && Kp == 2 * kh) : Kp >= 2 * r),
                  GWB_ERR_SHAPE, "stacked_a: n=%d r=%d Kp=%d kh=%d", n, r, Kp, kh);
    cudaStream_t s = (cudaStream_t)stream;
    const float2* a = reinterpret_cast<const float2*>(A);
    if (form == 0) stacked_a_kernel<0><<<n, 128, 0, s>>>(a, lda, n, r, nrm, nrm_stride, df4, scale, Kp, kh, Are, Aim, Are_lo, Aim_lo, ldo);
    else if (form == 1) stacked_a_kernel<1><<<n, 128, 0, s>>>(a, lda, n, r, nrm, nrm_stride, df4, scale, Kp, kh, Are, Aim, Are_lo, Aim_lo, ldo);
    else if (form == 2) stacked_a_kernel<2><<<n, 128, 0, s>>>(a, lda, n, r, nrm, nrm_stride, df4, scale, Kp, kh, Are, Aim, Are_lo, Aim_lo, ldo);
    else if (form == 5) stacked_a_kernel<5><<<n, 128, 0, s>>>(a, lda, n, r, nrm, nrm_stride, df4, scale, Kp, kh, Are, Aim, Are_lo, Aim_lo, ldo);
    else stacked_a_kernel<3><<<n, 128, 0, s>>>(a, lda, n, r, nrm, nrm_stride, df4, scale, Kp, kh, Are, Aim, Are_lo, Aim_lo, ldo);
    GWB_LAUNCH_CHECK("stacked_a_kernel");
    return GWB_OK;
}

int gwb_stacked_a8(const float* A, long long lda, int n, int r, const double* nrm, long long nrm_stride, double df4,
                   const float* zscale, int kh, void* A8, long long ldo, float* sa, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(A && nrm && zscale && A8 && sa, GWB_ERR_ARG, "stacked_a8: null pointer");
    GWB_CHECK_ARG(n > 0 && r > 0 && kh >= r && kh % 32 == 0 && lda >= r && ldo >= 2 * kh, GWB_ERR_SHAPE,
                  "stacked_a8: n=%d r=%d kh=%d (a multiple of 32, >= r) ldo=%lld", n, r, kh, ldo);
    stacked_a8_kernel<<<n, 128, 0, (cudaStream_t)stream>>>(reinterpret_cast<const float2*>(A), lda, n, r, nrm,
                                                            nrm_stride, df4, zscale, kh,
                                                            static_cast<__nv_fp8_storage_t*>(A8), ldo, sa);
    GWB_LAUNCH_CHECK("stacked_a8_kernel");
    return GWB_OK;
}

int gwb_select_windows(const float* vw, const int32_t* iw, long long ldv, int n, int nw, float thr2, float ecut,
                       float rthr, long long a0, int row0, int seg, const void* Are, const void* Aim,
                       const void* Are_lo, const void* Aim_lo, long long lda, const void* Z, const void* Zlo,
                       long long ldz, int Kp, int kh, int form, const float* rowscale, GwbCand* cands, int cand_cap,
                       GwbGroup* groups, int group_cap, GwbUnit* units, int unit_cap, GwbCand* rebuilt,
                       int rebuilt_cap, int32_t* counters, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(vw && iw && Are && (kh > 0 || Aim) && Z && cands && groups && units && counters, GWB_ERR_ARG,
                  "select_windows: null pointer");
    GWB_CHECK_ARG(form >= 0 && form <= 5 && (form != 2 || (Are_lo && (kh > 0 || Aim_lo) && Zlo)) &&
                      (form != 4 || (kh > 0 && rowscale)) && (form != 5 || (Are_lo && kh > 0)), GWB_ERR_ARG,
                  "select_windows: form %d", form);
    GWB_CHECK_ARG(kh == 0 || Kp == 2 * kh, GWB_ERR_SHAPE, "select_windows: Kp=%d with kh=%d", Kp, kh);
    GWB_CHECK_ARG(n > 0 && nw >= 0 && ldv >= nw && Kp > 0 && lda >= Kp, GWB_ERR_SHAPE, "select_windows: n=%d nw=%d", n,
                  nw);
    if (nw == 0) return GWB_OK;
    GWB_CHECK_ARG(ecut <= 0.f || (rebuilt && rebuilt_cap > 0), GWB_ERR_ARG, "select_windows: no rebuilt-peak list");
    select_kernel<<<n, kThreads, 0, (cudaStream_t)stream>>>(vw, iw, ldv, n, nw, thr2, ecut, rthr, a0, row0, seg, Are,
                                                            Aim, Are_lo, Aim_lo, lda, Z, Zlo, ldz, Kp, kh, form,
                                                            form == 4 ? rowscale : nullptr, cands, cand_cap, groups,
                                                            group_cap, units, unit_cap, rebuilt, rebuilt_cap,
                                                            counters);
    GWB_LAUNCH_CHECK("select_kernel");
    return GWB_OK;
}

}  // extern "C"
