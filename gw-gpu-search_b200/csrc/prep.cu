// Strain conditioning kernels: the streaming steps of pipeline/gpu_prep.py around cuFFT's transforms.
//
//   frames        Welch / segment frames: out[r, s, j] = x[r, start + s * stride + j] (* w[j])      (gpu_prep.py:104-108,420)
//   welch_avg     |X dt|^2 per frame (float32), DC and Nyquist halved, median (mean of the two middle values for an
//                 even count, as numpy) or mean over frames, / median bias, * PyCBC's scale            (:109-124)
//   interp        np.interp in float64 onto k df_new, cast to float32                                  (:128-135)
//   ist_pre/mid/post   1/sqrt(psd) band; irfft * df, Hann-tapered truncation; rfft / (df N), 1/|.|^2   (:138-158)
//   d_ip          IP = 1/P (float64, zero below kmin), D = stilde IP rounded to complex64              (:447-451)
//   sw            sqrt(mean over segments of IP) in float64, and 1/sw                                 (fp_filter.py:363-364)
//   taper_pad     corrupt-time ramps and centring in a power-of-two buffer                           (:179-189)
//   whiten        st *= (psd norm)^(-1/2)                                                             (:196-198)
//   above         indices and values of |x| above a threshold, appended with an atomic counter         (:200-206)
//   gates         inverted-Tukey gates, the product taken in float64 and rounded to float32           (:212-231)
// Each kernel uses the same operation order and rounding points as the numpy/cupy code it replaces, so results
// match it to float32 rounding (transforms excepted: cuFFT and pocketfft round differently).
#include "common.cuh"

namespace gwb {
namespace {

constexpr int kT = 256;

__global__ void frames_kernel(const float* __restrict__ x, long long ldx, int rows, long long start, long long stride,
                              const long long* __restrict__ starts, int nfr, int L, const float* __restrict__ w,
                              float* __restrict__ out, long long ldo) {
    const int f = blockIdx.y % nfr, r = blockIdx.y / nfr;
    const long long s0 = starts ? starts[f] : start + (long long)f * stride;
    const float* src = x + (long long)r * ldx + s0;
    float* dst = out + (long long)blockIdx.y * ldo;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < L; j += gridDim.x * blockDim.x)
        dst[j] = w ? src[j] * w[j] : src[j];
}

template <int MAXN>
__global__ void welch_avg_kernel(const float2* __restrict__ X, long long ldx, int rows, int nfr, int nbin, float dt,
                                 int median, float bias32, double bias64, int wide, float fac, float* __restrict__ psd,
                                 long long ldp) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)rows * nbin) return;
    const int r = (int)(e / nbin), k = (int)(e % nbin);
    float v[MAXN];
    for (int s = 0; s < nfr; ++s) {
        const float2 c = X[((long long)r * nfr + s) * ldx + k];
        const float a = c.x * dt, b = c.y * dt;
        float p = __fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b));
        if (k == 0 || k == nbin - 1) p = p / 2.f;
        v[s] = p;
    }
    float q;
    if (median) {
        for (int i = 1; i < nfr; ++i) {   // insertion sort, nfr is small
            const float t = v[i];
            int j = i - 1;
            while (j >= 0 && v[j] > t) {
                v[j + 1] = v[j];
                --j;
            }
            v[j + 1] = t;
        }
        q = (nfr & 1) ? v[nfr / 2] : __fdiv_rn(__fadd_rn(v[nfr / 2 - 1], v[nfr / 2]), 2.f);
        if (wide) {
            psd[(long long)r * ldp + k] = (float)(((double)q / bias64) * (double)fac);
            return;
        }
        q = __fdiv_rn(q, bias32);
    } else {
        float s = 0.f;
        for (int i = 0; i < nfr; ++i) s = __fadd_rn(s, v[i]);
        q = __fdiv_rn(s, (float)nfr);
    }
    psd[(long long)r * ldp + k] = __fmul_rn(q, fac);
}

// Median Welch average for many frames (more than 256, e.g. the 4 s estimate over a long segment in the autogating):
// one CTA per (row, bin), the frames' powers sorted in shared memory (bitonic, padded to a power of two with +inf),
// then the same median, bias and scale arithmetic as welch_avg_kernel.
__global__ void welch_median_big_kernel(const float2* __restrict__ X, long long ldx, int rows, int nfr, int nbin,
                                        float dt, float bias32, double bias64, int wide, float fac, int p2,
                                        float* __restrict__ psd, long long ldp) {
    extern __shared__ float v[];
    const int r = blockIdx.x / nbin, k = blockIdx.x % nbin;
    for (int s = threadIdx.x; s < p2; s += blockDim.x) {
        float p = __int_as_float(0x7f800000);      // +inf pads past nfr
        if (s < nfr) {
            const float2 c = X[((long long)r * nfr + s) * ldx + k];
            const float a = c.x * dt, b = c.y * dt;
            p = __fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b));
            if (k == 0 || k == nbin - 1) p = p / 2.f;
        }
        v[s] = p;
    }
    __syncthreads();
    for (int size = 2; size <= p2; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < p2; i += blockDim.x) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const float a = v[i], b = v[j];
                    if ((a > b) == up) {
                        v[i] = b;
                        v[j] = a;
                    }
                }
            }
            __syncthreads();
        }
    if (threadIdx.x == 0) {
        float q = (nfr & 1) ? v[nfr / 2] : __fdiv_rn(__fadd_rn(v[nfr / 2 - 1], v[nfr / 2]), 2.f);
        if (wide) {
            psd[(long long)r * ldp + k] = (float)(((double)q / bias64) * (double)fac);
            return;
        }
        q = __fdiv_rn(q, bias32);
        psd[(long long)r * ldp + k] = __fmul_rn(q, fac);
    }
}

__global__ void interp_kernel(const float* __restrict__ psd, long long ldp, int rows, int nold, double df_old,
                              double df_new, int nnew, float* __restrict__ out, long long ldo) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)rows * nnew) return;
    const int r = (int)(e / nnew), k = (int)(e % nnew);
    const float* p = psd + (long long)r * ldp;
    const double x = (double)k * df_new;
    double y;
    const double xl = (double)(nold - 1) * df_old;
    if (x >= xl) {
        y = (double)p[nold - 1];
    } else if (x <= 0.0) {
        y = (double)p[0];
    } else {
        int j = (int)floor(x / df_old);
        if (j > nold - 2) j = nold - 2;
        while (j > 0 && (double)j * df_old > x) --j;
        while (j < nold - 2 && (double)(j + 1) * df_old <= x) ++j;
        const double x0 = (double)j * df_old, x1 = (double)(j + 1) * df_old;
        const double y0 = p[j], y1 = p[j + 1];
        const double slope = __ddiv_rn(__dsub_rn(y1, y0), __dsub_rn(x1, x0));
        y = __dadd_rn(__dmul_rn(slope, __dsub_rn(x, x0)), y0);
    }
    out[(long long)r * ldo + k] = (float)y;
}

__global__ void ist_pre_kernel(const float* __restrict__ P, long long ldp, int rows, int flen, int kmin, int half,
                               float2* __restrict__ out, long long ldo) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)rows * flen) return;
    const int r = (int)(e / flen), k = (int)(e % flen);
    float v = 0.f;
    if (k >= kmin && k < half) v = __fsqrt_rn(__fdiv_rn(1.0f, P[(long long)r * ldp + k]));
    out[(long long)r * ldo + k] = make_float2(v, 0.f);
}

__global__ void ist_mid_kernel(float* __restrict__ q, long long ldq, int rows, int N, float df, int ts, int te,
                               const float* __restrict__ tw, int mfl) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)rows * N) return;
    const int r = (int)(e / N), i = (int)(e % N);
    float v = q[(long long)r * ldq + i] * df;
    if (tw) {
        if (i < ts) v = v * tw[mfl - ts + i];
        else if (i >= te) v = v * tw[i - te];
    }
    if (ts < te && i >= ts && i < te) v = 0.f;
    q[(long long)r * ldq + i] = v;
}

__global__ void ist_post_kernel(const float2* __restrict__ X, long long ldx, int rows, int flen, float s,
                                float* __restrict__ out, long long ldo) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)rows * flen) return;
    const int r = (int)(e / flen), k = (int)(e % flen);
    const float2 c = X[(long long)r * ldx + k];
    const float a = c.x * s, b = c.y * s;
    out[(long long)r * ldo + k] = __fdiv_rn(1.0f, __fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)));
}

__global__ void d_ip_kernel(const float2* __restrict__ st, long long ldst, int nseg, const float* __restrict__ psd,
                            long long ldp, const int32_t* __restrict__ pick, int flen, int kmin, float scale,
                            float2* __restrict__ D, long long ldd, float* __restrict__ IP, long long ldip) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)nseg * flen) return;
    const int s = (int)(e / flen), k = (int)(e % flen);
    const double P = (double)psd[(long long)pick[s] * ldp + k];
    double ip = P > 0.0 ? 1.0 / P : 0.0;
    if (k < kmin) ip = 0.0;
    const float2 c = st[(long long)s * ldst + k];
    const float cr = c.x * scale, ci = c.y * scale;   // stilde = rfft(x) * (1/sr), complex64
    D[(long long)s * ldd + k] = make_float2((float)((double)cr * ip), (float)((double)ci * ip));
    IP[(long long)s * ldip + k] = (float)ip;
}

__global__ void sw_kernel(const float* __restrict__ IP, long long ldip, int nseg, int flen, float* __restrict__ sw,
                          float* __restrict__ isw) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= flen) return;
    double s = 0.0;
    for (int i = 0; i < nseg; ++i) s += (double)IP[(long long)i * ldip + k];
    const float v = (float)sqrt(s / (double)nseg);
    sw[k] = v;
    isw[k] = v > 0.f ? 1.0f / fmaxf(v, 1e-30f) : 0.f;
}

__global__ void taper_pad_kernel(const float* __restrict__ s, long long n, int cl, long long L, long long pad_start,
                                 float* __restrict__ tapered, float* __restrict__ sp) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L; i += (long long)gridDim.x * blockDim.x) {
        const long long j = i - pad_start;
        if (j >= 0 && j < n) {
            float v = s[j];
            if (j < cl) v = v * (float)((double)j / (double)cl);
            else if (j >= n - cl) v = v * (float)((double)(n - 1 - j) / (double)cl);
            tapered[j] = v;
            sp[i] = v;
        } else {
            sp[i] = 0.f;
        }
    }
}

__global__ void whiten_kernel(float2* __restrict__ st, int nbin, const float* __restrict__ psd, float dt, float norm) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nbin) return;
    const float2 c = st[k];
    const float p = psd[k];
    const float w = isinf(p) ? 0.f : powf(p * norm, -0.5f);
    st[k] = make_float2((c.x * dt) * w, (c.y * dt) * w);
}

__global__ void above_kernel(const float* __restrict__ wt, long long pad_start, long long n, int cl, float df,
                             float thr, int32_t* __restrict__ idx, float* __restrict__ val, int cap,
                             int32_t* __restrict__ count) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        if (j < cl || j >= n - cl) continue;
        const float m = fabsf(wt[pad_start + j] * df);
        if (m > thr) {
            const int p = atomicAdd(count, 1);
            if (p < cap) {
                idx[p] = (int32_t)j;
                val[p] = m;
            }
        }
    }
}

__global__ void gates_kernel(float* __restrict__ x, long long n, const long long* __restrict__ g, int ngates) {
    // g: per gate (offset, win_samples, pad_samples, i1, i2)
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float v = x[i];
        bool touched = false;
        for (int q = 0; q < ngates; ++q) {
            const long long off = g[5 * q], win = g[5 * q + 1], pad = g[5 * q + 2], i1 = g[5 * q + 3], i2 = g[5 * q + 4];
            const long long m = i - off;
            if (m < i1 || m >= i2) continue;
            double wv;
            if (m < pad) wv = 0.5 * (1.0 + cos(3.141592653589793 * (double)m / (double)pad));
            else if (m >= win - pad) wv = 0.5 * (1.0 + cos(3.141592653589793 * (double)(win - 1 - m) / (double)pad));
            else wv = 0.0;
            v = (float)((double)v * wv);
            touched = true;
        }
        if (touched) x[i] = v;
    }
}

inline unsigned blocks_for(long long n) { return (unsigned)std::max(1ll, std::min<long long>(cdiv(n, kT), 1ll << 20)); }

}  // namespace
}  // namespace gwb

extern "C" {

int gwb_frames(const float* x, long long ldx, int rows, long long start, long long stride, const long long* starts,
               int nfr, int L, const float* w, float* out, long long ldo, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(x && out, GWB_ERR_ARG, "frames: null pointer");
    GWB_CHECK_ARG(rows > 0 && nfr > 0 && L > 0 && ldo >= L && (long long)rows * nfr < 65536, GWB_ERR_SHAPE,
                  "frames: rows=%d nfr=%d L=%d", rows, nfr, L);
    GWB_CHECK_ARG(starts || start + (long long)(nfr - 1) * stride + L <= ldx, GWB_ERR_SHAPE,
                  "frames: frames end beyond the row");
    dim3 grid((unsigned)std::min<long long>(cdiv(L, kT), 256), rows * nfr);
    frames_kernel<<<grid, kT, 0, (cudaStream_t)stream>>>(x, ldx, rows, start, stride, starts, nfr, L, w, out, ldo);
    GWB_LAUNCH_CHECK("frames_kernel");
    return GWB_OK;
}

int gwb_welch_avg(const float* X, long long ldx, int rows, int nfr, int nbin, float dt, int median, double bias,
                  float fac, float* psd, long long ldp, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(X && psd, GWB_ERR_ARG, "welch_avg: null pointer");
    GWB_CHECK_ARG(rows > 0 && nfr > 0 && nbin > 0 && ldx >= nbin && ldp >= nbin && (nfr <= 256 || (median &&
                  nfr <= 8192)), GWB_ERR_SHAPE, "welch_avg: rows=%d frames=%d (at most 256, or 8192 for the median) "
                  "nbin=%d", rows, nfr, nbin);
    const long long n = (long long)rows * nbin;
    const int wide = nfr >= 1000;
    cudaStream_t s = (cudaStream_t)stream;
    const float2* x2 = reinterpret_cast<const float2*>(X);
    if (nfr > 256) {
        int p2 = 1;
        while (p2 < nfr) p2 <<= 1;
        GWB_CHECK_ARG(n < (1ll << 31), GWB_ERR_SHAPE, "welch_avg: rows x nbin = %lld", n);
        welch_median_big_kernel<<<(unsigned)n, kT, (size_t)p2 * sizeof(float), s>>>(
            x2, ldx, rows, nfr, nbin, dt, (float)bias, bias, wide, fac, p2, psd, ldp);
        GWB_LAUNCH_CHECK("welch_median_big_kernel");
        return GWB_OK;
    }
    if (nfr <= 64)
        welch_avg_kernel<64><<<blocks_for(n), kT, 0, s>>>(x2, ldx, rows, nfr, nbin, dt, median, (float)bias, bias, wide,
                                                          fac, psd, ldp);
    else
        welch_avg_kernel<256><<<blocks_for(n), kT, 0, s>>>(x2, ldx, rows, nfr, nbin, dt, median, (float)bias, bias, wide,
                                                           fac, psd, ldp);
    GWB_LAUNCH_CHECK("welch_avg_kernel");
    return GWB_OK;
}

int gwb_interp(const float* psd, long long ldp, int rows, int nold, double df_old, double df_new, int nnew, float* out,
               long long ldo, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(psd && out, GWB_ERR_ARG, "interp: null pointer");
    GWB_CHECK_ARG(rows > 0 && nold >= 2 && nnew > 0 && ldo >= nnew && df_old > 0 && df_new > 0, GWB_ERR_SHAPE,
                  "interp: rows=%d nold=%d nnew=%d", rows, nold, nnew);
    const long long n = (long long)rows * nnew;
    interp_kernel<<<blocks_for(n), kT, 0, (cudaStream_t)stream>>>(psd, ldp, rows, nold, df_old, df_new, nnew, out, ldo);
    GWB_LAUNCH_CHECK("interp_kernel");
    return GWB_OK;
}

int gwb_ist_pre(const float* P, long long ldp, int rows, int flen, int kmin, float* out, long long ldo, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(P && out, GWB_ERR_ARG, "ist_pre: null pointer");
    GWB_CHECK_ARG(rows > 0 && flen > 1 && ldo >= flen, GWB_ERR_SHAPE, "ist_pre: rows=%d flen=%d", rows, flen);
    const int N = (flen - 1) * 2;
    ist_pre_kernel<<<blocks_for((long long)rows * flen), kT, 0, (cudaStream_t)stream>>>(
        P, ldp, rows, flen, kmin, N / 2, reinterpret_cast<float2*>(out), ldo);
    GWB_LAUNCH_CHECK("ist_pre_kernel");
    return GWB_OK;
}

int gwb_ist_mid(float* q, long long ldq, int rows, int N, float df, int max_filter_len, const float* taper,
                void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(q, GWB_ERR_ARG, "ist_mid: null pointer");
    GWB_CHECK_ARG(rows > 0 && N > 0 && max_filter_len > 0, GWB_ERR_SHAPE, "ist_mid: rows=%d N=%d", rows, N);
    const int ts = max_filter_len / 2, te = N - max_filter_len / 2;
    ist_mid_kernel<<<blocks_for((long long)rows * N), kT, 0, (cudaStream_t)stream>>>(q, ldq, rows, N, df, ts, te, taper,
                                                                                     max_filter_len);
    GWB_LAUNCH_CHECK("ist_mid_kernel");
    return GWB_OK;
}

int gwb_ist_post(const float* X, long long ldx, int rows, int flen, float scale, float* out, long long ldo,
                 void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(X && out, GWB_ERR_ARG, "ist_post: null pointer");
    GWB_CHECK_ARG(rows > 0 && flen > 0 && ldo >= flen, GWB_ERR_SHAPE, "ist_post: rows=%d flen=%d", rows, flen);
    ist_post_kernel<<<blocks_for((long long)rows * flen), kT, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const float2*>(X), ldx, rows, flen, scale, out, ldo);
    GWB_LAUNCH_CHECK("ist_post_kernel");
    return GWB_OK;
}

int gwb_d_ip(const float* stilde, long long ldst, int nseg, const float* psd, long long ldp, const int32_t* pick,
             int flen, int kmin, float scale, float* D, long long ldd, float* IP, long long ldip, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(stilde && psd && pick && D && IP, GWB_ERR_ARG, "d_ip: null pointer");
    GWB_CHECK_ARG(nseg > 0 && flen > 0 && ldd >= flen && ldip >= flen, GWB_ERR_SHAPE, "d_ip: nseg=%d flen=%d", nseg, flen);
    d_ip_kernel<<<blocks_for((long long)nseg * flen), kT, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const float2*>(stilde), ldst, nseg, psd, ldp, pick, flen, kmin, scale,
        reinterpret_cast<float2*>(D), ldd, IP, ldip);
    GWB_LAUNCH_CHECK("d_ip_kernel");
    return GWB_OK;
}

int gwb_sw(const float* IP, long long ldip, int nseg, int flen, float* sw, float* isw, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(IP && sw && isw, GWB_ERR_ARG, "sw: null pointer");
    GWB_CHECK_ARG(nseg > 0 && flen > 0, GWB_ERR_SHAPE, "sw: nseg=%d flen=%d", nseg, flen);
    sw_kernel<<<(unsigned)cdiv(flen, kT), kT, 0, (cudaStream_t)stream>>>(IP, ldip, nseg, flen, sw, isw);
    GWB_LAUNCH_CHECK("sw_kernel");
    return GWB_OK;
}

int gwb_taper_pad(const float* s, long long n, int cl, long long L, long long pad_start, float* tapered, float* sp,
                  void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(s && tapered && sp, GWB_ERR_ARG, "taper_pad: null pointer");
    GWB_CHECK_ARG(n > 0 && L >= n && pad_start >= 0 && pad_start + n <= L && cl >= 0 && 2ll * cl <= n, GWB_ERR_SHAPE,
                  "taper_pad: n=%lld L=%lld", n, L);
    taper_pad_kernel<<<blocks_for(L), kT, 0, (cudaStream_t)stream>>>(s, n, cl, L, pad_start, tapered, sp);
    GWB_LAUNCH_CHECK("taper_pad_kernel");
    return GWB_OK;
}

int gwb_whiten(float* st, int nbin, const float* psd, float dt, float norm, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(st && psd, GWB_ERR_ARG, "whiten: null pointer");
    GWB_CHECK_ARG(nbin > 0, GWB_ERR_SHAPE, "whiten: nbin=%d", nbin);
    whiten_kernel<<<(unsigned)cdiv(nbin, kT), kT, 0, (cudaStream_t)stream>>>(reinterpret_cast<float2*>(st), nbin, psd,
                                                                             dt, norm);
    GWB_LAUNCH_CHECK("whiten_kernel");
    return GWB_OK;
}

int gwb_above(const float* wt, long long pad_start, long long n, int cl, float df, float thr, int32_t* idx, float* val,
              int cap, int32_t* count, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(wt && idx && val && count, GWB_ERR_ARG, "above: null pointer");
    GWB_CHECK_ARG(n > 0 && cap > 0, GWB_ERR_SHAPE, "above: n=%lld cap=%d", n, cap);
    above_kernel<<<blocks_for(n), kT, 0, (cudaStream_t)stream>>>(wt, pad_start, n, cl, df, thr, idx, val, cap, count);
    GWB_LAUNCH_CHECK("above_kernel");
    return GWB_OK;
}

int gwb_apply_gates(float* x, long long n, const long long* gates, int ngates, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(x && (gates || ngates == 0), GWB_ERR_ARG, "apply_gates: null pointer");
    GWB_CHECK_ARG(n > 0 && ngates >= 0, GWB_ERR_SHAPE, "apply_gates: n=%lld ngates=%d", n, ngates);
    if (ngates == 0) return GWB_OK;
    gates_kernel<<<blocks_for(n), kT, 0, (cudaStream_t)stream>>>(x, n, gates, ngates);
    GWB_LAUNCH_CHECK("gates_kernel");
    return GWB_OK;
}

int gwb_highpass(void) {
    gwb::set_error("the lal IIR highpass (pipeline/gpu_prep.py:56-64) stays outside this library");
    return GWB_ERR_NOT_IMPLEMENTED;
}

int gwb_resample(void) {
    gwb::set_error("the ldas FIR resampler (pipeline/gpu_prep.py:67-84) stays outside this library");
    return GWB_ERR_NOT_IMPLEMENTED;
}

}  // extern "C"
