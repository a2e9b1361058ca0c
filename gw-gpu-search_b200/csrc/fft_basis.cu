// Fused basis series: conj(Vh) D isw -> inverse DFT of length N -> Re / scale, Im / scale packed into Z, in two
// passes over HBM instead of premul + cuFFT (two passes) + pack (fp_filter.basis_series, fp_filter.py:597-613).
//
// N = N1 N2 with k = N2 k1 + k2 and t = t1 + N1 t2 (Cooley-Tukey, four-step):
//   z[t1 + N1 t2] = sum_k2 e^{2 pi i k2 t2 / N2} e^{2 pi i k2 t1 / N} [ sum_k1 q[N2 k1 + k2] e^{2 pi i k1 t1 / N1} ]
// pass 1, CTA = (8 consecutive k2, one basis row): forms q = conj(Vh) D isw on load (zero above N/2, where the
//   reference zero-pads), DFT of length N1 over k1 in shared memory, multiplies by e^{2 pi i k2 t1 / N} and writes
//   W[row][k2][t1] (t1 contiguous). For the first rows it also sums |q|^2 for the scale.
// pass 2, CTA = (8 consecutive t1, one basis row): DFT of length N2 over k2, then z at t in [a0, a0 + Tn) is divided
//   by the scale and written to Z as fp16, fp32, bf16 or bf16 hi + lo.
// The in-CTA DFT is a Stockham radix-4 (plus one radix-2 when log2 L is odd) over 8 interleaved columns, each stage
// staged through registers so one shared buffer suffices. Twiddles come from one table e^{2 pi i m / N} (float from
// double), also used with stride N / L for the in-CTA stages.
// Scale: the reference divides by the rms of the first batch's outputs over the analysed span; here the rms over the
// whole series is taken from the inputs by Parseval (sum_t |z_t|^2 = N sum_k |q_k|^2), so no pass re-reads the
// outputs. The scale only normalises Z for its 16-bit range: A is multiplied by the same scale, so the SNR is
// unchanged (fp_filter.py:617).
#include "common.cuh"
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <utility>
#include <type_traits>

namespace gwb {
namespace {

constexpr int TB = 8;   // interleaved columns per CTA

__global__ void twiddle_kernel(float2* tw, long long N) {
    const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= N) return;
    double s, c;
    sincospi(2.0 * (double)m / (double)N, &s, &c);
    tw[m] = make_float2((float)c, (float)s);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -(a.y * b.y)), fmaf(a.x, b.y, a.y * b.x));
}

// One Stockham stage of an in-place inverse DFT of length L over TB interleaved columns (X[p * TB + c] holds element
// p of column c); NS = product of the radices already applied, all compile-time so index arithmetic is shifts and
// masks. Each thread stages its butterflies' inputs in registers, the block syncs, then outputs are stored.
// tw_s: e^{2 pi i m / L}, m < L.
template <int L, int NT, int NS>
__device__ __forceinline__ void radix4_stage(float2* X, const float2* tw_s) {
    constexpr int Q = (L / 4) * TB / NT;
    constexpr int STEP = L / (NS * 4);
    const int tid = threadIdx.x;
    float2 v[Q][4];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int b = tid + NT * q;
        const int c = b % TB, j = b / TB;
#pragma unroll
        for (int r = 0; r < 4; ++r) v[q][r] = X[(j + r * (L / 4)) * TB + c];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int b = tid + NT * q;
        const int c = b % TB, j = b / TB;
        const int k = j % NS;
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < 4; ++r) v[q][r] = cmul(v[q][r], tw_s[k * r * STEP]);
        }
        const float2 a = make_float2(v[q][0].x + v[q][2].x, v[q][0].y + v[q][2].y);
        const float2 bb = make_float2(v[q][0].x - v[q][2].x, v[q][0].y - v[q][2].y);
        const float2 cc = make_float2(v[q][1].x + v[q][3].x, v[q][1].y + v[q][3].y);
        const float2 d = make_float2(v[q][1].x - v[q][3].x, v[q][1].y - v[q][3].y);
        const int idx = (j / NS) * NS * 4 + k;
        X[(idx + 0 * NS) * TB + c] = make_float2(a.x + cc.x, a.y + cc.y);
        X[(idx + 1 * NS) * TB + c] = make_float2(bb.x - d.y, bb.y + d.x);      // b + i d
        X[(idx + 2 * NS) * TB + c] = make_float2(a.x - cc.x, a.y - cc.y);
        X[(idx + 3 * NS) * TB + c] = make_float2(bb.x + d.y, bb.y - d.x);      // b - i d
    }
    __syncthreads();
}

template <int L, int NT, int NS>
__device__ __forceinline__ void radix2_stage(float2* X, const float2* tw_s) {
    constexpr int Q = (L / 2) * TB / NT;
    constexpr int STEP = L / (NS * 2);
    const int tid = threadIdx.x;
    float2 v[Q][2];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int b = tid + NT * q;
        const int c = b % TB, j = b / TB;
        v[q][0] = X[j * TB + c];
        v[q][1] = X[(j + L / 2) * TB + c];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int b = tid + NT * q;
        const int c = b % TB, j = b / TB;
        const int k = j % NS;
        const float2 w = NS > 1 ? cmul(v[q][1], tw_s[k * STEP]) : v[q][1];
        const int idx = (j / NS) * NS * 2 + k;
        X[idx * TB + c] = make_float2(v[q][0].x + w.x, v[q][0].y + w.y);
        X[(idx + NS) * TB + c] = make_float2(v[q][0].x - w.x, v[q][0].y - w.y);
    }
    __syncthreads();
}

template <int L, int NT, int NS = 1>
__device__ __forceinline__ void fft_smem(float2* X, const float2* tw_s) {
    if constexpr (NS * 4 <= L) {
        radix4_stage<L, NT, NS>(X, tw_s);
        fft_smem<L, NT, NS * 4>(X, tw_s);
    } else if constexpr (NS * 2 == L) {
        radix2_stage<L, NT, NS>(X, tw_s);
    }
}

// ---- register two-level DFT (L <= 1024): L = R1 R2, k = R2 a + b, t = u + R1 v ----
//   X[u + R1 v] = sum_b e^{2 pi i b v / R2} e^{2 pi i b u / L} [ sum_a x[R2 a + b] e^{2 pi i a u / R1} ]
// step 1: one thread per (b, column) holds x[R2 a + b] for all a in registers, R1-point DFT, twiddle, store to shared
// step 2: one thread per (u, column) reads the R2 values, R2-point DFT in registers.
// Shared memory is crossed once per pass (one store, one load per element) instead of once per radix-4 stage.

// sin / cos of 2 pi k / n in double at compile time (argument reduced to [-pi, pi], Taylor series to 30 terms)
__host__ __device__ constexpr double sin_taylor(double x) {
    double term = x, sum = x;
    for (int i = 1; i < 30; ++i) {
        term *= -x * x / ((2.0 * i) * (2.0 * i + 1.0));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double cos_taylor(double x) {
    double term = 1.0, sum = 1.0;
    for (int i = 1; i < 30; ++i) {
        term *= -x * x / ((2.0 * i - 1.0) * (2.0 * i));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double turn_angle(int k, int n) {
    const int m = ((k % n) + n) % n;
    const int r = 2 * m > n ? m - n : m;
    return 6.283185307179586476925286766559 * (double)r / (double)n;
}

template <int I>
using ic = std::integral_constant<int, I>;

template <typename F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
    (f(ic<I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }
constexpr int brev(int x, int bits) { return bits == 0 ? 0 : ((x & 1) << (bits - 1)) | brev(x >> 1, bits - 1); }

// v * e^{2 pi i J / M}, trivial angles without multiplies
template <int J, int M>
__device__ __forceinline__ float2 rot(float2 v) {
    constexpr int j = ((J % M) + M) % M;
    if constexpr (j == 0) {
        return v;
    } else if constexpr (4 * j == M) {
        return make_float2(-v.y, v.x);
    } else if constexpr (2 * j == M) {
        return make_float2(-v.x, -v.y);
    } else if constexpr (4 * j == 3 * M) {
        return make_float2(v.y, -v.x);
    } else {
        constexpr float c = (float)cos_taylor(turn_angle(J, M)), s = (float)sin_taylor(turn_angle(J, M));
        return make_float2(fmaf(v.x, c, -(v.y * s)), fmaf(v.x, s, v.y * c));
    }
}

// in-register inverse DFT (e^{+2 pi i}) of size R, decimation in frequency: natural input order, output X[u] in
// x[brev(u)]
template <int R>
__device__ __forceinline__ void dft_reg(float2 (&x)[R]) {
    static_for<ilog2(R)>([&](auto S) {
        constexpr int h = R >> (decltype(S)::value + 1);
        static_for<R / (2 * h)>([&](auto B) {
            constexpr int base = decltype(B)::value * 2 * h;
            static_for<h>([&](auto J) {
                constexpr int j = decltype(J)::value;
                const float2 a = x[base + j], b = x[base + j + h];
                x[base + j] = make_float2(a.x + b.x, a.y + b.y);
                x[base + j + h] = rot<j, 2 * h>(make_float2(a.x - b.x, a.y - b.y));
            });
        });
    });
}

template <int L>
struct Split {
    static constexpr int R1 = 1 << ((ilog2(L) + 1) / 2);
    static constexpr int R2 = L / R1;
    static constexpr int NT = TB * R2;                 // step 1: one R1-point DFT per thread
    static constexpr int P2 = R1 / R2;                 // step 2: R2-point DFTs per thread
    static constexpr int SB = ((R1 + 15) / 16) * 16 + 1;           // = 1 mod 16 (8-byte words)
    static constexpr int SC = R2 * SB + ((4 - (R2 * SB) % 16) + 16) % 16;   // = 4 mod 16
    static_assert(R1 >= R2 && R1 % R2 == 0, "split");
};

template <int L>
constexpr int threads_for() {
    return (L * TB / 16) < 64 ? 64 : (L * TB / 16);
}

// pass 1: rows of the batch in blockIdx.y, 8 consecutive k2 in blockIdx.x
template <int N1>
__global__ void __launch_bounds__(threads_for<N1>()) basis_pass1(
    const float2* __restrict__ Vh, long long ldvh, const float2* __restrict__ D, const float* __restrict__ isw,
    long long flen, long long N, int N2, const float2* __restrict__ tw, float2* __restrict__ W, int nfirst,
    double* __restrict__ partials, unsigned int* __restrict__ ticket, float* __restrict__ scale_out) {
    constexpr int NT = threads_for<N1>();
    extern __shared__ float2 sm[];
    float2* X = sm;                  // N1 x TB
    float2* tw_s = sm + N1 * TB;     // N1
    const int row = blockIdx.y, k20 = blockIdx.x * TB, tid = threadIdx.x;
    const long long stride = N / N1;
    for (int m = tid; m < N1; m += NT) tw_s[m] = tw[(long long)m * stride];
    // e^{2 pi i k2 t1 / N} = TH[c][t1 / 32] TL[c][t1 % 32] for this CTA's 8 columns k2 = k20 + c
    // rows padded by one entry so the 8 columns of a warp fall in different banks
    constexpr int NH = (N1 + 31) / 32, NHP = NH + 1, NLP = 33;
    float2* TH = tw_s + N1;             // TB x NHP
    float2* TL = TH + TB * NHP;         // TB x NLP
    const unsigned long long mask = (unsigned long long)N - 1;
    for (int e = tid; e < TB * NH; e += NT) {
        const int c = e / NH, a = e % NH;
        TH[c * NHP + a] = tw[((unsigned long long)(k20 + c) * (unsigned long long)(32 * a)) & mask];
    }
    for (int e = tid; e < TB * 32; e += NT) {
        const int c = e / 32, b = e % 32;
        TL[c * NLP + b] = tw[((unsigned long long)(k20 + c) * (unsigned long long)b) & mask];
    }
    const float2* v = Vh + (long long)row * ldvh;
    double acc = 0.0;
    const long long lim = min(N / 2 + 1, flen);     // q is zero from N/2 + 1 on (the reference's zero padding)
    // all loads of a batch issued before any use, so each thread keeps several requests in flight
    constexpr int PER = N1 * TB / NT, BATCH = 8;
    static_assert(PER % BATCH == 0, "loads per thread");
#pragma unroll
    for (int i0 = 0; i0 < PER; i0 += BATCH) {
        float2 av[BATCH], dv[BATCH];
        float wv[BATCH];
#pragma unroll
        for (int i = 0; i < BATCH; ++i) {
            const int e = tid + NT * (i0 + i);
            const long long k = (long long)N2 * (e / TB) + k20 + (e % TB);
            const bool ok = k < lim;
            av[i] = ok ? v[k] : make_float2(0.f, 0.f);
            dv[i] = ok ? D[k] : make_float2(0.f, 0.f);
            wv[i] = ok ? isw[k] : 0.f;
        }
#pragma unroll
        for (int i = 0; i < BATCH; ++i) {
            const int e = tid + NT * (i0 + i);
            const float dr = dv[i].x * wv[i], di = dv[i].y * wv[i];
            const float2 q = make_float2(fmaf(av[i].x, dr, av[i].y * di), fmaf(av[i].x, di, -(av[i].y * dr)));
            acc += (double)q.x * q.x + (double)q.y * q.y;
            X[e] = q;              // e = k1 * TB + c
        }
    }
    if (row >= nfirst) acc = 0.0;
    __syncthreads();
    fft_smem<N1, NT>(X, tw_s);
    // twiddle e^{2 pi i k2 t1 / N} and write W[row][k2][t1], t1 contiguous
    float2* Wr = W + (long long)row * N;
    for (int e = tid; e < N1 * TB; e += NT) {
        const int c = e % TB, t1 = e / TB;     // shared reads conflict-free; global writes in 32-byte runs
        const float2 w = cmul(TH[c * NHP + (t1 >> 5)], TL[c * NLP + (t1 & 31)]);
        Wr[(long long)(k20 + c) * N1 + t1] = cmul(X[t1 * TB + c], w);
    }
    // scale partials: one per CTA of the first rows, summed in a fixed order by the last CTA to finish
    if (nfirst > 0) {
        __shared__ double red[32];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        if ((tid & 31) == 0) red[tid >> 5] = acc;
        __syncthreads();
        __shared__ bool last;
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < NT / 32; ++w) s += red[w];
            const unsigned nb = gridDim.x * (unsigned)min(nfirst, (int)gridDim.y);
            if (row < nfirst) partials[(long long)row * gridDim.x + blockIdx.x] = s;
            __threadfence();
            last = false;
            if (row < nfirst) last = atomicAdd(ticket, 1u) == nb - 1;
        }
        __syncthreads();
        if (last && tid == 0) {
            __threadfence();
            const int nr = min(nfirst, (int)gridDim.y);
            double s = 0.0;
            for (long long b = 0; b < (long long)nr * gridDim.x; ++b) s += ((volatile double*)partials)[b];
            // mean over t of |z|^2 = sum_k |q|^2 (Parseval); scale = sqrt(mean / 2)
            *scale_out = (float)sqrt(s / (double)nr / 2.0);
            *ticket = 0;
        }
    }
}

template <int N2, int FORM>
__global__ void __launch_bounds__(threads_for<N2>()) basis_pass2(
    const float2* __restrict__ W, long long N, int N1, const float2* __restrict__ tw, long long a0, long long Tn,
    const float* __restrict__ scale, void* __restrict__ Z, void* __restrict__ Zlo, long long ldz, int im_off,
    int row0) {
    constexpr int NT = threads_for<N2>();
    extern __shared__ float2 sm[];
    float2* X = sm;
    float2* tw_s = sm + N2 * TB;
    const int row = blockIdx.y, t10 = blockIdx.x * TB, tid = threadIdx.x;
    const long long stride = N / N2;
    for (int m = tid; m < N2; m += NT) tw_s[m] = tw[(long long)m * stride];
    const float2* Wr = W + (long long)row * N;
    constexpr int PER = N2 * TB / NT, BATCH = 8;
    static_assert(PER % BATCH == 0, "loads per thread");
#pragma unroll
    for (int i0 = 0; i0 < PER; i0 += BATCH) {
        float2 wv[BATCH];
#pragma unroll
        for (int i = 0; i < BATCH; ++i) {
            const int e = tid + NT * (i0 + i);
            wv[i] = Wr[(long long)(e / TB) * N1 + t10 + (e % TB)];
        }
#pragma unroll
        for (int i = 0; i < BATCH; ++i) X[tid + NT * (i0 + i)] = wv[i];
    }
    __syncthreads();
    fft_smem<N2, NT>(X, tw_s);
    const float inv = 1.0f / *scale;
    const long long re_row = row0 + row, im_row = im_off + row0 + row;
    for (int e = tid; e < N2 * TB; e += NT) {
        const int c = e % TB, t2 = e / TB;
        const long long t = (long long)t10 + c + (long long)N1 * t2 - a0;
        if (t < 0 || t >= Tn) continue;
        const float2 v = X[t2 * TB + c];
        const float xr = v.x * inv, xi = v.y * inv;
        if (FORM == 0) {
            static_cast<__half*>(Z)[re_row * ldz + t] = __float2half_rn(xr);
            static_cast<__half*>(Z)[im_row * ldz + t] = __float2half_rn(xi);
        } else if (FORM == 1) {
            static_cast<float*>(Z)[re_row * ldz + t] = xr;
            static_cast<float*>(Z)[im_row * ldz + t] = xi;
        } else {
            const __nv_bfloat16 hr = __float2bfloat16_rn(xr), hm = __float2bfloat16_rn(xi);
            static_cast<__nv_bfloat16*>(Z)[re_row * ldz + t] = hr;
            static_cast<__nv_bfloat16*>(Z)[im_row * ldz + t] = hm;
            if (FORM == 2) {
                static_cast<__nv_bfloat16*>(Zlo)[re_row * ldz + t] = __float2bfloat16_rn(xr - __bfloat162float(hr));
                static_cast<__nv_bfloat16*>(Zlo)[im_row * ldz + t] = __float2bfloat16_rn(xi - __bfloat162float(hm));
            }
        }
    }
}

// pass 1, register form: rows in blockIdx.y, 8 consecutive k2 in blockIdx.x
template <int N1>
__global__ void __launch_bounds__(Split<N1>::NT) basis_pass1_reg(
    const float2* __restrict__ Vh, long long ldvh, const float2* __restrict__ D, const float* __restrict__ isw,
    long long flen, long long N, int N2, const float2* __restrict__ tw, float2* __restrict__ W, int nfirst,
    double* __restrict__ partials, unsigned int* __restrict__ ticket, float* __restrict__ scale_out) {
    using S = Split<N1>;
    constexpr int R1 = S::R1, R2 = S::R2, NT = S::NT, SB = S::SB, SC = S::SC;
    extern __shared__ float2 sm[];
    float2* Y = sm;                       // TB x SC
    float2* twL = Y + TB * SC;            // e^{2 pi i m / N1}, m < N1
    float2* TL = twL + N1;                // TB x (R1 + 1): e^{2 pi i k2 u / N}
    float2* TH = TL + TB * (R1 + 1);      // TB x (R2 + 1): e^{2 pi i k2 R1 v / N}
    const int row = blockIdx.y, k20 = blockIdx.x * TB, tid = threadIdx.x;
    const unsigned long long mask = (unsigned long long)N - 1;
    const long long stride = N / N1;
    for (int m = tid; m < N1; m += NT) twL[m] = tw[(long long)m * stride];
    for (int e = tid; e < TB * R1; e += NT) {
        const int c = e / R1, u = e % R1;
        TL[c * (R1 + 1) + u] = tw[((unsigned long long)(k20 + c) * (unsigned long long)u) & mask];
    }
    for (int e = tid; e < TB * R2; e += NT) {
        const int c = e / R2, v = e % R2;
        TH[c * (R2 + 1) + v] = tw[((unsigned long long)(k20 + c) * (unsigned long long)(R1 * v)) & mask];
    }
    // step 1: thread (b, c) loads q at k1 = R2 a + b, k2 = k20 + c; q is zero from N/2 + 1 on (the reference's zero
    // padding)
    const int c = tid % TB, b = tid / TB;
    const float2* v = Vh + (long long)row * ldvh;
    const long long lim = min(N / 2 + 1, flen);
    float2 x[R1];
    float part = 0.f;
#pragma unroll
    for (int a = 0; a < R1; ++a) {
        const long long k = (long long)N2 * (R2 * a + b) + k20 + c;
        const bool ok = k < lim;
        const float2 av = ok ? v[k] : make_float2(0.f, 0.f);
        const float2 dk = ok ? D[k] : make_float2(0.f, 0.f);
        const float w = ok ? isw[k] : 0.f;
        const float dr = dk.x * w, di = dk.y * w;
        x[a] = make_float2(fmaf(av.x, dr, av.y * di), fmaf(av.x, di, -(av.y * dr)));
        part = fmaf(x[a].x, x[a].x, fmaf(x[a].y, x[a].y, part));
    }
    dft_reg<R1>(x);
    __syncthreads();                      // tables
    static_for<R1>([&](auto U) {
        constexpr int u = decltype(U)::value;
        Y[c * SC + b * SB + u] = cmul(x[brev(u, ilog2(R1))], twL[b * u]);
    });
    __syncthreads();
    // step 2: thread (u, c), u fastest so the W stores run along t1
    float2* Wr = W + (long long)row * N;
#pragma unroll
    for (int p = 0; p < S::P2; ++p) {
        const int d = tid + NT * p;
        const int u = d % R1, c2 = d / R1;
        float2 y[R2];
#pragma unroll
        for (int bb = 0; bb < R2; ++bb) y[bb] = Y[c2 * SC + bb * SB + u];
        dft_reg<R2>(y);
        const float2 tl = TL[c2 * (R1 + 1) + u];
        float2* wc = Wr + (long long)(k20 + c2) * N1 + u;
        static_for<R2>([&](auto V) {
            constexpr int vv = decltype(V)::value;
            wc[R1 * vv] = cmul(y[brev(vv, ilog2(R2))], cmul(tl, TH[c2 * (R2 + 1) + vv]));
        });
    }
    // scale partials: one per CTA of the first rows, summed in a fixed order by the last CTA to finish
    if (nfirst > 0) {
        __shared__ double red[32];
        double acc = row < nfirst ? (double)part : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        if ((tid & 31) == 0) red[tid >> 5] = acc;
        __syncthreads();
        __shared__ bool last;
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < NT / 32; ++w) s += red[w];
            const unsigned nb = gridDim.x * (unsigned)min(nfirst, (int)gridDim.y);
            if (row < nfirst) partials[(long long)row * gridDim.x + blockIdx.x] = s;
            __threadfence();
            last = false;
            if (row < nfirst) last = atomicAdd(ticket, 1u) == nb - 1;
        }
        __syncthreads();
        if (last && tid == 0) {
            __threadfence();
            const int nr = min(nfirst, (int)gridDim.y);
            double s = 0.0;
            for (long long i = 0; i < (long long)nr * gridDim.x; ++i) s += ((volatile double*)partials)[i];
            *scale_out = (float)sqrt(s / (double)nr / 2.0);
            *ticket = 0;
        }
    }
}

template <int FORM>
__device__ __forceinline__ void store_z(void* Z, void* Zlo, long long re, long long im, float xr, float xi) {
    if constexpr (FORM == 0) {
        static_cast<__half*>(Z)[re] = __float2half_rn(xr);
        static_cast<__half*>(Z)[im] = __float2half_rn(xi);
    } else if constexpr (FORM == 1) {
        static_cast<float*>(Z)[re] = xr;
        static_cast<float*>(Z)[im] = xi;
    } else {
        const __nv_bfloat16 hr = __float2bfloat16_rn(xr), hm = __float2bfloat16_rn(xi);
        static_cast<__nv_bfloat16*>(Z)[re] = hr;
        static_cast<__nv_bfloat16*>(Z)[im] = hm;
        if constexpr (FORM == 2) {
            static_cast<__nv_bfloat16*>(Zlo)[re] = __float2bfloat16_rn(xr - __bfloat162float(hr));
            static_cast<__nv_bfloat16*>(Zlo)[im] = __float2bfloat16_rn(xi - __bfloat162float(hm));
        }
    }
}

// pass 2, register form: rows in blockIdx.y, 8 consecutive t1 in blockIdx.x
template <int N2, int FORM>
__global__ void __launch_bounds__(Split<N2>::NT) basis_pass2_reg(
    const float2* __restrict__ W, long long N, int N1, const float2* __restrict__ tw, long long a0, long long Tn,
    const float* __restrict__ scale, void* __restrict__ Z, void* __restrict__ Zlo, long long ldz, int im_off,
    int row0) {
    using S = Split<N2>;
    constexpr int R1 = S::R1, R2 = S::R2, NT = S::NT, SB = S::SB, SC = S::SC;
    extern __shared__ float2 sm[];
    float2* Y = sm;
    float2* twL = Y + TB * SC;
    const int row = blockIdx.y, t10 = blockIdx.x * TB, tid = threadIdx.x;
    const long long stride = N / N2;
    for (int m = tid; m < N2; m += NT) twL[m] = tw[(long long)m * stride];
    const int c = tid % TB, b = tid / TB;
    const float2* wc = W + (long long)row * N + t10 + c;
    float2 x[R1];
#pragma unroll
    for (int a = 0; a < R1; ++a) x[a] = wc[(long long)(R2 * a + b) * N1];
    dft_reg<R1>(x);
    __syncthreads();
    static_for<R1>([&](auto U) {
        constexpr int u = decltype(U)::value;
        Y[c * SC + b * SB + u] = cmul(x[brev(u, ilog2(R1))], twL[b * u]);
    });
    __syncthreads();
    // step 2: thread (c, u), c fastest so the Z stores run along t
    const float inv = 1.0f / *scale;
    const long long re_base = (long long)(row0 + row) * ldz, im_base = (long long)(im_off + row0 + row) * ldz;
#pragma unroll
    for (int p = 0; p < S::P2; ++p) {
        const int d = tid + NT * p;
        const int c2 = d % TB, u = d / TB;
        float2 y[R2];
#pragma unroll
        for (int bb = 0; bb < R2; ++bb) y[bb] = Y[c2 * SC + bb * SB + u];
        dft_reg<R2>(y);
        const long long t0 = (long long)t10 + c2 + (long long)N1 * u - a0;
        static_for<R2>([&](auto V) {
            constexpr int vv = decltype(V)::value;
            const long long t = t0 + (long long)N1 * (R1 * vv);
            if (t >= 0 && t < Tn) {
                const float2 z = y[brev(vv, ilog2(R2))];
                store_z<FORM>(Z, Zlo, re_base + t, im_base + t, z.x * inv, z.y * inv);
            }
        });
    }
}

int log2i(long long n) {
    int l = 0;
    while ((1ll << l) < n) ++l;
    return l;
}

template <int N1>
int launch_pass1_reg(const float2* Vh, long long ldvh, int rows, const float2* D, const float* isw, long long flen,
                     long long N, int N2, const float2* tw, float2* W, int nfirst, double* partials, unsigned* ticket,
                     float* scale_out, cudaStream_t s) {
    using S = Split<N1>;
    const size_t smem = (size_t)(TB * S::SC + N1 + TB * (S::R1 + 1) + TB * (S::R2 + 1)) * sizeof(float2);
    auto k = basis_pass1_reg<N1>;
    GWB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<dim3(N2 / TB, rows), S::NT, smem, s>>>(Vh, ldvh, D, isw, flen, N, N2, tw, W, nfirst, partials, ticket,
                                              scale_out);
    GWB_LAUNCH_CHECK("basis_pass1_reg");
    return GWB_OK;
}

template <int N2, int FORM>
int launch_pass2_reg(const float2* W, long long N, int N1, int rows, const float2* tw, long long a0, long long Tn,
                     const float* scale, void* Z, void* Zlo, long long ldz, int im_off, int row0, cudaStream_t s) {
    using S = Split<N2>;
    const size_t smem = (size_t)(TB * S::SC + N2) * sizeof(float2);
    auto k = basis_pass2_reg<N2, FORM>;
    GWB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<dim3(N1 / TB, rows), S::NT, smem, s>>>(W, N, N1, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0);
    GWB_LAUNCH_CHECK("basis_pass2_reg");
    return GWB_OK;
}

template <int N1>
int launch_pass1(const float2* Vh, long long ldvh, int rows, const float2* D, const float* isw, long long flen,
                 long long N, int N2, const float2* tw, float2* W, int nfirst, double* partials, unsigned* ticket,
                 float* scale_out, cudaStream_t s) {
    constexpr int NT = threads_for<N1>();
    const size_t smem = (size_t)(N1 * TB + N1 + TB * ((N1 + 31) / 32 + 1) + TB * 33) * sizeof(float2);
    auto k = basis_pass1<N1>;
    GWB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<dim3(N2 / TB, rows), NT, smem, s>>>(Vh, ldvh, D, isw, flen, N, N2, tw, W, nfirst, partials, ticket, scale_out);
    GWB_LAUNCH_CHECK("basis_pass1");
    return GWB_OK;
}

template <int N2, int FORM>
int launch_pass2_f(const float2* W, long long N, int N1, int rows, const float2* tw, long long a0, long long Tn,
                   const float* scale, void* Z, void* Zlo, long long ldz, int im_off, int row0, cudaStream_t s) {
    constexpr int NT = threads_for<N2>();
    const size_t smem = (size_t)(N2 * TB + N2) * sizeof(float2);
    auto k = basis_pass2<N2, FORM>;
    GWB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<dim3(N1 / TB, rows), NT, smem, s>>>(W, N, N1, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0);
    GWB_LAUNCH_CHECK("basis_pass2");
    return GWB_OK;
}

template <int N2>
int launch_pass2(int form, const float2* W, long long N, int N1, int rows, const float2* tw, long long a0,
                 long long Tn, const float* scale, void* Z, void* Zlo, long long ldz, int im_off, int row0,
                 cudaStream_t s) {
    if constexpr (N2 <= 1024) {
        switch (form) {
            case 0: return launch_pass2_reg<N2, 0>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
            case 1: return launch_pass2_reg<N2, 1>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
            case 2: return launch_pass2_reg<N2, 2>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
            default: return launch_pass2_reg<N2, 3>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
        }
    } else {
        switch (form) {
            case 0: return launch_pass2_f<N2, 0>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
            case 1: return launch_pass2_f<N2, 1>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
            case 2: return launch_pass2_f<N2, 2>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
            default: return launch_pass2_f<N2, 3>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
        }
    }
}

}  // namespace
}  // namespace gwb

extern "C" {

int gwb_fft_twiddles(long long N, float* tw, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(tw, GWB_ERR_ARG, "fft_twiddles: null pointer");
    GWB_CHECK_ARG(is_pow2(N) && N >= 64, GWB_ERR_NOT_POW2, "fft_twiddles: N=%lld must be a power of two >= 64", N);
    twiddle_kernel<<<(unsigned)cdiv(N, 256), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<float2*>(tw), N);
    GWB_LAUNCH_CHECK("twiddle_kernel");
    return GWB_OK;
}

int gwb_basis_fused(const float* Vh, long long ldvh, int rows, const float* D, const float* isw, long long flen,
                    long long N, const float* tw, float* W, long long a0, long long Tn, int form, void* Z, void* Zlo,
                    long long ldz, int im_off, int row0, int nfirst, double* partials, long long npartials,
                    uint32_t* ticket, float* scale, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(Vh && D && isw && tw && W && Z && scale && (form != 2 || Zlo), GWB_ERR_ARG,
                  "basis_fused: null pointer");
    GWB_CHECK_ARG(form >= 0 && form <= 3, GWB_ERR_ARG, "basis_fused: form %d", form);
    GWB_CHECK_ARG(is_pow2(N) && N >= (1 << 12) && N <= (1 << 22), GWB_ERR_NOT_POW2,
                  "basis_fused: N=%lld must be a power of two in [2^12, 2^22]", N);
    GWB_CHECK_ARG(rows > 0 && rows < 65536 && flen <= N / 2 + 1 && ldvh >= flen && a0 >= 0 && Tn > 0 &&
                  a0 + Tn <= N && ldz >= Tn && row0 >= 0 && row0 + rows <= im_off, GWB_ERR_SHAPE,
                  "basis_fused: rows=%d flen=%lld N=%lld a0=%lld Tn=%lld", rows, flen, N, a0, Tn);
    const int p = log2i(N);
    const int N1 = 1 << ((p + 1) / 2), N2 = (int)(N / N1);
    GWB_CHECK_ARG(nfirst <= 0 || (partials && ticket && (long long)std::min(nfirst, rows) * (N2 / TB) <= npartials),
                  GWB_ERR_SHAPE, "basis_fused: scale partials need %lld entries",
                  (long long)std::min(nfirst, rows) * (N2 / TB));
    cudaStream_t s = (cudaStream_t)stream;
    const float2* v = reinterpret_cast<const float2*>(Vh);
    const float2* d = reinterpret_cast<const float2*>(D);
    const float2* t = reinterpret_cast<const float2*>(tw);
    float2* w = reinterpret_cast<float2*>(W);
    unsigned* tk = reinterpret_cast<unsigned*>(ticket);
    int st;
    switch (N1) {
        case 64: st = launch_pass1_reg<64>(v, ldvh, rows, d, isw, flen, N, N2, t, w, nfirst, partials, tk, scale, s); break;
        case 128: st = launch_pass1_reg<128>(v, ldvh, rows, d, isw, flen, N, N2, t, w, nfirst, partials, tk, scale, s); break;
        case 256: st = launch_pass1_reg<256>(v, ldvh, rows, d, isw, flen, N, N2, t, w, nfirst, partials, tk, scale, s); break;
        case 512: st = launch_pass1_reg<512>(v, ldvh, rows, d, isw, flen, N, N2, t, w, nfirst, partials, tk, scale, s); break;
        case 1024: st = launch_pass1_reg<1024>(v, ldvh, rows, d, isw, flen, N, N2, t, w, nfirst, partials, tk, scale, s); break;
        default: st = launch_pass1<2048>(v, ldvh, rows, d, isw, flen, N, N2, t, w, nfirst, partials, tk, scale, s); break;
    }
    if (st) return st;
    switch (N2) {
        case 64: return launch_pass2<64>(form, w, N, N1, rows, t, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
        case 128: return launch_pass2<128>(form, w, N, N1, rows, t, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
        case 256: return launch_pass2<256>(form, w, N, N1, rows, t, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
        case 512: return launch_pass2<512>(form, w, N, N1, rows, t, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
        case 1024: return launch_pass2<1024>(form, w, N, N1, rows, t, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
        default: return launch_pass2<2048>(form, w, N, N1, rows, t, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
    }
}

}  // extern "C"
