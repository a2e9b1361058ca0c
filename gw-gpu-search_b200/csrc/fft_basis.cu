// Fused basis series: conj(Vh) D isw -> inverse DFT of length N -> Re / scale, Im / scale packed into Z, in two
// passes over HBM instead of premul + cuFFT (two passes) + pack (fp_filter.basis_series, fp_filter.py:597-613).
//
// N = N1 N2 with k = N2 k1 + k2 and t = t1 + N1 t2 (Cooley-Tukey, four-step):
//   z[t1 + N1 t2] = sum_k2 e^{2 pi i k2 t2 / N2} e^{2 pi i k2 t1 / N} [ sum_k1 q[N2 k1 + k2] e^{2 pi i k1 t1 / N1} ]
// q is zero from N/2 + 1 on (the reference zero-pads the half spectrum), so only k1 < N1/2 and the single bin N/2
// enter. The inputs are stored in four-step order, P[k2 (N1/2) + k1] = X[N2 k1 + k2] and P[N/2] = X[N/2]
// (gwb_fourstep_order: once per tile for the basis filters, once per segment for D isw), so every pass reads and
// writes contiguous runs:
// pass 1, CTA = (8 consecutive k2, one basis row): q = conj(Vp) Dp (contiguous), DFT of length N1 over k1,
//   multiply by e^{2 pi i k2 t1 / N}, write W in blocks of 8 t1: W[t1 / 8][k2][t1 % 8]. For the first rows it also
//   sums |q|^2 for the scale.
// pass 2, CTA = (8 consecutive t1, one basis row): reads its W block (contiguous), DFT of length N2 over k2, writes z
//   at t in [a0, a0 + Tn) divided by the scale to Z as fp16, fp32, bf16 or bf16 hi + lo.
// Each in-CTA DFT is two-level (L = R1 R2): an R1-point DFT in registers per thread, one exchange through shared
// memory, an R2-point DFT in registers. Twiddles: one table e^{2 pi i m / N} (float from double); the in-register
// stages use compile-time constants.
// Scale: the reference divides by the rms of the first batch's outputs over the analysed span; here the rms over the
// whole series is taken from the inputs by Parseval (sum_t |z_t|^2 = N sum_k |q_k|^2), so no pass re-reads the
// outputs. The scale only normalises Z for its 16-bit range: A is multiplied by the same scale, so the SNR is
// unchanged (fp_filter.py:617).
#include "common.cuh"
#include <atomic>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <type_traits>
#include <utility>

namespace gwb {
namespace {

constexpr int TB = 8;   // columns per CTA (k2 in pass 1, t1 in pass 2); also the W block width

__global__ void twiddle_kernel(float2* tw, long long N) {
    const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= N) return;
    double s, c;
    sincospi(2.0 * (double)m / (double)N, &s, &c);
    tw[m] = make_float2((float)c, (float)s);
}

// P[j][k2 H + k1] = X[j][N2 k1 + k2] (times isw) for k1 < H = N1 / 2, k2 < N2, and P[j][N / 2] = X[j][N / 2]; zero
// where k >= flen. 32 x 32 tiles through shared memory.
__global__ void fourstep_order_kernel(const float2* __restrict__ X, long long ldx, const float* __restrict__ isw,
                                      long long flen, int N2, int H, float2* __restrict__ P, long long ldp) {
    __shared__ float2 tile[32][33];
    const int j = blockIdx.z;
    const int k20 = blockIdx.x * 32, k10 = blockIdx.y * 32;
    const float2* x = X + (long long)j * ldx;
    float2* p = P + (long long)j * ldp;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const long long k = (long long)N2 * (k10 + i) + k20 + threadIdx.x;
        float2 v = make_float2(0.f, 0.f);
        if (k < flen) {
            v = x[k];
            if (isw) {
                const float w = isw[k];
                v = make_float2(v.x * w, v.y * w);
            }
        }
        tile[i][threadIdx.x] = v;
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y)
        p[(long long)(k20 + i) * H + k10 + threadIdx.x] = tile[threadIdx.x][i];
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
        const long long k = (long long)N2 * H;     // N / 2
        float2 v = make_float2(0.f, 0.f);
        if (k < flen) {
            v = x[k];
            if (isw) v = make_float2(v.x * isw[k], v.y * isw[k]);
        }
        p[k] = v;
    }
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -(a.y * b.y)), fmaf(a.x, b.y, a.y * b.x));
}

// ---- two-level DFT of length L <= 1024 inside a CTA: L = R1 R2, k = R2 a + b, t = u + R1 v ----
//   X[u + R1 v] = sum_b e^{2 pi i b v / R2} e^{2 pi i b u / L} [ sum_a x[R2 a + b] e^{2 pi i a u / R1} ]
// step 1: one thread per (b, column) holds x[R2 a + b] for all a in registers, R1-point DFT, twiddle, store to shared
// step 2: one thread per (u, column) reads the R2 values, R2-point DFT in registers.
// Shared memory is crossed once per pass (one store and one load per element).

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

// dft_reg for inputs whose upper half past R/2 is zero (x[R/2] may not be): the first stage's butterflies (j, j + R/2)
// reduce to a copy and a rotation for j >= 1, so its additions are skipped. Same output as dft_reg on those inputs
// (up to the sign of exact zeros).
template <int R>
__device__ __forceinline__ void dft_reg_upper_zero(float2 (&x)[R]) {
    constexpr int h0 = R / 2;
    {
        const float2 a = x[0], b = x[h0];
        x[0] = make_float2(a.x + b.x, a.y + b.y);
        x[h0] = make_float2(a.x - b.x, a.y - b.y);
    }
    static_for<h0 - 1>([&](auto J) {
        constexpr int j = decltype(J)::value + 1;
        x[j + h0] = rot<j, R>(x[j]);
    });
    static_for<ilog2(R) - 1>([&](auto S) {
        constexpr int h = R >> (decltype(S)::value + 2);
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

// Two-level split of a DFT of length L over TB columns. Shared buffer Y[c][b][u] at c * SC + b * SB + u (float2):
// SB = 1 (mod 16 eight-byte words) and SC = SCM (mod 16), chosen per pass so that each half-warp of a 64-bit access
// hits 16 distinct bank pairs.
template <int L, int SCM>
struct Split {
    static constexpr int R1 = 1 << ((ilog2(L) + 1) / 2);
    static constexpr int R2 = L / R1;
    static constexpr int NT = TB * R2;                 // step 1: one R1-point DFT per thread
    static constexpr int P2 = R1 / R2;                 // step 2: R2-point DFTs per thread
    static constexpr int SB = ((R1 + 15) / 16) * 16 + 1;
    static constexpr int SC = R2 * SB + ((SCM - (R2 * SB) % 16) + 16) % 16;
    static_assert(R1 >= R2 && R1 % R2 == 0 && R1 % 8 == 0, "split");
};

// Scale partials of a pass-1 CTA: sum of |q|^2 over the CTA (one double per CTA of the first nfirst rows), summed in
// a fixed order by the last CTA to finish, which writes scale = sqrt(mean / 2) and resets the ticket.
template <int NT>
__device__ __forceinline__ void scale_partials(float part, int row, int nfirst, double* __restrict__ partials,
                                               unsigned int* __restrict__ ticket, float* __restrict__ scale_out) {
    __shared__ double red[32];
    __shared__ bool last;
    const int tid = threadIdx.x;
    double acc = row < nfirst ? (double)part : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((tid & 31) == 0) red[tid >> 5] = acc;
    __syncthreads();
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
        // mean over t of |z|^2 = sum_k |q|^2 (Parseval); scale = sqrt(mean / 2)
        *scale_out = (float)sqrt(s / (double)nr / 2.0);
        *ticket = 0;
    }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

constexpr int RC = 8;   // rows per pass-1 CTA of the warp-per-column form

// pass 1 for N1 = 1024: one warp per column k2 (8 columns per CTA), RC consecutive rows per CTA. 32 x 32 split: lane
// b holds q at k1 = 32 a + b (a < 16), 32-point DFT, twiddle, exchange through the warp's own shared tile, lane u
// then holds the 32 values of t1 = u + 32 v. Per column, D isw and the twiddles stay in registers / shared memory
// across the rows, and the next row's basis-filter segment (4 KB, contiguous in four-step order) is copied into
// shared memory (cp.async) while the current row is transformed. No CTA barrier after the set-up, so the warps of a
// CTA drift apart and one warp's copies overlap another's arithmetic. Scale partials: one per (row chunk, column),
// summed in a fixed order by the last warp to finish.
__global__ void __launch_bounds__(256, 2) basis_pass1_w(
    const float2* __restrict__ Vp, long long ldvp, int rows, const float2* __restrict__ Dp, int N, int N2,
    const float2* __restrict__ tw, float2* __restrict__ W, int nfirst, double* __restrict__ partials,
    unsigned int* __restrict__ ticket, float* __restrict__ scale_out, float* __restrict__ rowpart) {
    constexpr int N1 = 1024, R = 32, H = N1 / 2, NW = 8, YS = R * (R + 1);
    constexpr int WS = YS + R + H;                          // per warp: Y tile, TH, basis-filter segment
    extern __shared__ float2 sm[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float2* tw2 = sm;                                       // tw2[u 32 + b] = e^{2 pi i b u / N1}
    float2* Yw = sm + N1 + warp * WS;                       // this warp's 32 x 33 tile
    float2* THw = Yw + YS;                                  // e^{2 pi i k2 32 v / N}, v < 32
    float2* Vs = THw + R;                                   // Vp[row][k2 H .. k2 H + H)
    const int k2 = blockIdx.x * NW + warp;
    const int j0 = blockIdx.y * RC, j1 = min(j0 + RC, rows);
    const int mask = N - 1;
    auto fetch = [&](int j) {                               // 4 KB: 8 x 16 bytes per lane
        const char* g = reinterpret_cast<const char*>(Vp + (long long)j * ldvp + k2 * H);
        char* d = reinterpret_cast<char*>(Vs);
#pragma unroll
        for (int i = 0; i < 8; ++i) cp_async16(d + i * 512 + lane * 16, g + i * 512 + lane * 16);
        cp_async_commit();
    };
    fetch(j0);
    float2 dk[R / 2];
#pragma unroll
    for (int a = 0; a < R / 2; ++a) dk[a] = __ldg(Dp + k2 * H + R * a + lane);
    const float2 dN = Dp[N / 2];
    for (int e = threadIdx.x; e < N1; e += NW * 32) tw2[e] = tw[(e % R) * (e / R) * (N / N1)];
    THw[lane] = tw[(k2 * (R * lane)) & mask];
    const float2 tl = tw[(k2 * lane) & mask];               // e^{2 pi i k2 u / N}, u = lane
    __syncthreads();
    const int nf = min(nfirst, rows);
    double acc = 0.0;
    for (int j = j0; j < j1; ++j) {
        cp_async_wait_all();
        __syncwarp();
        float2 x[R];
#pragma unroll
        for (int a = 0; a < R / 2; ++a) x[a] = Vs[R * a + lane];
        __syncwarp();
        if (j + 1 < j1) fetch(j + 1);
#pragma unroll
        for (int a = 0; a < R / 2; ++a) {
            const float2 av = x[a];
            x[a] = make_float2(fmaf(av.x, dk[a].x, av.y * dk[a].y), fmaf(av.x, dk[a].y, -(av.y * dk[a].x)));
        }
        x[R / 2] = make_float2(0.f, 0.f);
        if (k2 == 0 && lane == 0) {                         // the bin N / 2
            const float2 av = Vp[(long long)j * ldvp + N / 2];
            x[R / 2] = make_float2(fmaf(av.x, dN.x, av.y * dN.y), fmaf(av.x, dN.y, -(av.y * dN.x)));
        }
        // sums of |q|^2 only where they are used: the scale's first rows, the fp8 form's per-row sums (warp-uniform)
        if (j < nf || rowpart) {
            float part = 0.f;
#pragma unroll
            for (int a = 0; a <= R / 2; ++a) part = fmaf(x[a].x, x[a].x, fmaf(x[a].y, x[a].y, part));
            if (j < nf) acc += (double)part;
            if (rowpart) {                                  // per-row sums of |q|^2: rowpart[j][k2]
                float ps = part;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) ps += __shfl_xor_sync(0xffffffffu, ps, off);
                if (lane == 0) rowpart[(long long)j * N2 + k2] = ps;
            }
        }
        dft_reg_upper_zero<R>(x);                           // q is zero for k1 > N1 / 2
        static_for<R>([&](auto U) {
            constexpr int u = decltype(U)::value;
            Yw[lane * (R + 1) + u] = cmul(x[brev(u, ilog2(R))], tw2[u * R + lane]);
        });
        __syncwarp();
#pragma unroll
        for (int bb = 0; bb < R; ++bb) x[bb] = Yw[bb * (R + 1) + lane];
        __syncwarp();
        dft_reg<R>(x);
        // t1 = lane + 32 v: W block t1 / 8 = 4 v + lane / 8, position lane % 8
        float2* wc = W + (long long)j * N + (lane >> 3) * (N2 * 8) + k2 * 8 + (lane & 7);
        static_for<R>([&](auto V) {
            constexpr int vv = decltype(V)::value;
            wc[4 * vv * (N2 * 8)] = cmul(x[brev(vv, ilog2(R))], cmul(tl, THw[vv]));
        });
    }
    if (nf <= 0 || j0 >= nf) return;
    // scale: partials[chunk * N2 + k2]; the last of the ceil(nf / RC) * N2 warps sums them in a fixed order
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    const unsigned total = (unsigned)(((nf + RC - 1) / RC) * N2);
    unsigned last = 0;
    if (lane == 0) {
        partials[(long long)blockIdx.y * N2 + k2] = acc;
        __threadfence();
        last = atomicAdd(ticket, 1u) == total - 1;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return;
    __threadfence();
    double s = 0.0;
    for (unsigned i = lane; i < total; i += 32) s += ((volatile double*)partials)[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) {
        // mean over t of |z|^2 = sum_k |q|^2 (Parseval); scale = sqrt(mean / 2)
        *scale_out = (float)sqrt(s / (double)nf / 2.0);
        *ticket = 0;
    }
}

// pass 1: rows in blockIdx.y, TB consecutive k2 in blockIdx.x. Vp, Dp in four-step order (Dp already D isw).
template <int N1>
__global__ void __launch_bounds__(Split<N1, 8>::NT) basis_pass1(
    const float2* __restrict__ Vp, long long ldvp, const float2* __restrict__ Dp, int N, int N2,
    const float2* __restrict__ tw, float2* __restrict__ W, int nfirst, double* __restrict__ partials,
    unsigned int* __restrict__ ticket, float* __restrict__ scale_out, float* __restrict__ rowpart) {
    using S = Split<N1, 8>;
    constexpr int R1 = S::R1, R2 = S::R2, NT = S::NT, SB = S::SB, SC = S::SC, H = N1 / 2;
    extern __shared__ float2 sm[];
    float2* Y = sm;                       // TB x SC
    float2* twL = Y + TB * SC;            // e^{2 pi i m / N1} at m + m / 16 (skewed: a warp reads 32 b u)
    float2* TL = twL + N1 + N1 / 16;      // TB x (R1 + 1): e^{2 pi i k2 u / N}
    float2* TH = TL + TB * (R1 + 1);      // TB x (R2 + 1): e^{2 pi i k2 R1 v / N}
    const int row = blockIdx.y, k20 = blockIdx.x * TB, tid = threadIdx.x;
    const int mask = N - 1, stride = N / N1;
    for (int m = tid; m < N1; m += NT) twL[m + (m >> 4)] = tw[m * stride];
    for (int e = tid; e < TB * R1; e += NT) {
        const int c = e / R1, u = e % R1;
        TL[c * (R1 + 1) + u] = tw[((k20 + c) * u) & mask];
    }
    for (int e = tid; e < TB * R2; e += NT) {
        const int c = e / R2, v = e % R2;
        TH[c * (R2 + 1) + v] = tw[((k20 + c) * (R1 * v)) & mask];
    }
    // step 1: thread (b, c), b fastest: q at k1 = R2 a + b of column k2 = k20 + c, a < R1 / 2 (k1 < N1 / 2); the bin
    // N / 2 is a = R1 / 2, b = 0, k2 = 0; q is zero for the other a >= R1 / 2
    const int b = tid % R2, c = tid / R2;
    const float2* v = Vp + (long long)row * ldvp;
    const int o = (k20 + c) * H + b;
    float2 x[R1];
    float part = 0.f;
#pragma unroll
    for (int a = 0; a < R1 / 2; ++a) {
        const float2 av = __ldcs(v + o + R2 * a), dk = __ldg(Dp + o + R2 * a);
        x[a] = make_float2(fmaf(av.x, dk.x, av.y * dk.y), fmaf(av.x, dk.y, -(av.y * dk.x)));   // conj(v) d
        part = fmaf(x[a].x, x[a].x, fmaf(x[a].y, x[a].y, part));
    }
    x[R1 / 2] = make_float2(0.f, 0.f);
    if (o == 0) {
        const float2 av = v[N / 2], dk = Dp[N / 2];
        x[R1 / 2] = make_float2(fmaf(av.x, dk.x, av.y * dk.y), fmaf(av.x, dk.y, -(av.y * dk.x)));
        part = fmaf(x[R1 / 2].x, x[R1 / 2].x, fmaf(x[R1 / 2].y, x[R1 / 2].y, part));
    }
#pragma unroll
    for (int a = R1 / 2 + 1; a < R1; ++a) x[a] = make_float2(0.f, 0.f);
    dft_reg<R1>(x);
    __syncthreads();                      // tables
    static_for<R1>([&](auto U) {
        constexpr int u = decltype(U)::value;
        const int m = b * u;
        Y[c * SC + b * SB + u] = cmul(x[brev(u, ilog2(R1))], twL[m + (m >> 4)]);
    });
    __syncthreads();
    // step 2: thread (u % 8, c2, u / 8), so that a warp stores 4 columns x 8 t1 of one W block: 256 contiguous bytes
    float2* Wr = W + (long long)row * N;
#pragma unroll
    for (int p = 0; p < S::P2; ++p) {
        const int d = tid + NT * p;
        const int ul = d % 8, c2 = (d / 8) % TB, uh = d / (8 * TB);
        const int u = uh * 8 + ul;
        float2 y[R2];
#pragma unroll
        for (int bb = 0; bb < R2; ++bb) y[bb] = Y[c2 * SC + bb * SB + u];
        dft_reg<R2>(y);
        const float2 tl = TL[c2 * (R1 + 1) + u];
        float2* wc = Wr + uh * (N2 * 8) + (k20 + c2) * 8 + ul;
        static_for<R2>([&](auto V) {
            constexpr int vv = decltype(V)::value;           // t1 = u + R1 vv: block uh + (R1 / 8) vv, lane ul
            wc[(R1 / 8) * vv * (N2 * 8)] = cmul(y[brev(vv, ilog2(R2))], cmul(tl, TH[c2 * (R2 + 1) + vv]));
        });
    }
    if (rowpart) {                                          // per-row sums of |q|^2: rowpart[row][blockIdx.x]
        __shared__ float rred[NT / 32];
        float ps = part;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) ps += __shfl_xor_sync(0xffffffffu, ps, off);
        if ((tid & 31) == 0) rred[tid >> 5] = ps;
        __syncthreads();
        if (tid == 0) {
            float sum = 0.f;
            for (int w = 0; w < NT / 32; ++w) sum += rred[w];
            rowpart[(long long)row * gridDim.x + blockIdx.x] = sum;
        }
    }
    if (nfirst > 0) scale_partials<NT>(part, row, nfirst, partials, ticket, scale_out);
}

// Per-row scale of the fp8 form: rowscale[j] = (rms of one component of basis series j) / 16, from the row's |q|^2
// sums (Parseval: mean_t |z_t|^2 = sum_k |q_k|^2), summed in a fixed order in float64. Z_j / rowscale[j] then has a
// per-component rms of 16: far inside e4m3's range (448) for the peaks, above its subnormals for the bulk.
__global__ void rowscale_kernel(const float* __restrict__ rowpart, int P, float* __restrict__ rowscale) {
    __shared__ double red[256 / 32];
    const int j = blockIdx.x, tid = threadIdx.x;
    double s = 0.0;
    for (int i = tid; i < P; i += 256) s += (double)rowpart[(long long)j * P + i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((tid & 31) == 0) red[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[w];
        rowscale[j] = t > 0.0 ? (float)(sqrt(t / 2.0) / 16.0) : 1.f;
    }
}

template <int FORM>
__device__ __forceinline__ void store_z(void* Zr, void* Zi, void* Zlr, void* Zli, int t, float xr, float xi) {
    if constexpr (FORM == 0) {
        __stcs(static_cast<__half*>(Zr) + t, __float2half_rn(xr));
        __stcs(static_cast<__half*>(Zi) + t, __float2half_rn(xi));
    } else if constexpr (FORM == 1) {
        __stcs(static_cast<float*>(Zr) + t, xr);
        __stcs(static_cast<float*>(Zi) + t, xi);
    } else if constexpr (FORM == 4) {
        static_cast<__nv_fp8_storage_t*>(Zr)[t] = __nv_cvt_float_to_fp8(xr, __NV_SATFINITE, __NV_E4M3);
        static_cast<__nv_fp8_storage_t*>(Zi)[t] = __nv_cvt_float_to_fp8(xi, __NV_SATFINITE, __NV_E4M3);
    } else {
        const __nv_bfloat16 hr = __float2bfloat16_rn(xr), hm = __float2bfloat16_rn(xi);
        __stcs(static_cast<__nv_bfloat16*>(Zr) + t, hr);
        __stcs(static_cast<__nv_bfloat16*>(Zi) + t, hm);
        if constexpr (FORM == 2) {
            __stcs(static_cast<__nv_bfloat16*>(Zlr) + t, __float2bfloat16_rn(xr - __bfloat162float(hr)));
            __stcs(static_cast<__nv_bfloat16*>(Zli) + t, __float2bfloat16_rn(xi - __bfloat162float(hm)));
        }
    }
}

// pass 2: rows in blockIdx.y, W block (TB consecutive t1) in blockIdx.x
template <int N2, int FORM>
__global__ void __launch_bounds__(Split<N2, 2>::NT) basis_pass2(
    const float2* __restrict__ W, int N, int N1, const float2* __restrict__ tw, int a0, int Tn,
    const float* __restrict__ scale, void* __restrict__ Z, void* __restrict__ Zlo, long long ldz, int im_off,
    int row0) {
    using S = Split<N2, 2>;
    constexpr int R1 = S::R1, R2 = S::R2, NT = S::NT, SB = S::SB, SC = S::SC;
    constexpr int ES = FORM == 1 ? 4 : (FORM == 4 ? 1 : 2);   // bytes per Z element
    extern __shared__ float2 sm[];
    float2* Y = sm;
    float2* twL = Y + TB * SC;
    const int row = blockIdx.y, t10 = blockIdx.x * TB, tid = threadIdx.x;
    const int stride = N / N2;
    // 1 / scale: folded into the step-1 twiddles (one rms per call), applied per row at the store for fp8
    const float inv = 1.0f / (FORM == 4 ? scale[row] : *scale);
    const float tsc = FORM == 4 ? 1.f : inv, zsc = FORM == 4 ? inv : 1.f;
    for (int m = tid; m < N2; m += NT) {
        const float2 w = tw[m * stride];
        twL[m] = make_float2(w.x * tsc, w.y * tsc);
    }
    // step 1: thread (c, b), c fastest: the block's W[k2][c] at k2 = R2 a + b, 256 contiguous bytes per warp
    const int c = tid % TB, b = tid / TB;
    const float2* wc = W + (long long)row * N + (long long)blockIdx.x * (N2 * TB) + b * TB + c;
    float2 x[R1];
#pragma unroll
    for (int a = 0; a < R1; ++a) x[a] = __ldcs(wc + R2 * TB * a);
    dft_reg<R1>(x);
    __syncthreads();
    static_for<R1>([&](auto U) {
        constexpr int u = decltype(U)::value;
        Y[c * SC + b * SB + u] = cmul(x[brev(u, ilog2(R1))], twL[b * u]);
    });
    __syncthreads();
    // step 2: thread (c, u), c fastest so the Z stores run along t. fp8: scale holds one scale per row
    char* zb = static_cast<char*>(Z);
    char* zl = static_cast<char*>(Zlo);
    const long long re_off = (long long)(row0 + row) * ldz * ES, im_off_b = (long long)(im_off + row0 + row) * ldz * ES;
    void* Zr = zb + re_off;
    void* Zi = zb + im_off_b;
    void* Zlr = FORM == 2 ? (void*)(zl + re_off) : nullptr;
    void* Zli = FORM == 2 ? (void*)(zl + im_off_b) : nullptr;
#pragma unroll
    for (int p = 0; p < S::P2; ++p) {
        const int d = tid + NT * p;
        const int c2 = d % TB, u = d / TB;
        float2 y[R2];
#pragma unroll
        for (int bb = 0; bb < R2; ++bb) y[bb] = Y[c2 * SC + bb * SB + u];
        dft_reg<R2>(y);
        const int t0 = t10 + c2 + N1 * u - a0;
        static_for<R2>([&](auto V) {
            constexpr int vv = decltype(V)::value;
            const int t = t0 + N1 * (R1 * vv);
            if (t >= 0 && t < Tn) {
                const float2 z = y[brev(vv, ilog2(R2))];
                if constexpr (FORM == 4) store_z<FORM>(Zr, Zi, Zlr, Zli, t, z.x * zsc, z.y * zsc);
                else store_z<FORM>(Zr, Zi, Zlr, Zli, t, z.x, z.y);
            }
        });
    }
}

// pass 2 over row chunks: CTA = (TB consecutive t1, RC consecutive rows). One shared buffer holds the W tile of a row
// (TB x N2, contiguous in the blocked layout, copied with cp.async) and then, once every thread has its inputs in
// registers, the exchange tile; the next row's copy is issued as soon as the exchange tile has been read, and runs
// under the second DFT and the Z stores (and under the other CTA on the SM).
template <int N2, int FORM>
__global__ void __launch_bounds__(Split<N2, 2>::NT, 2) basis_pass2_p(
    const float2* __restrict__ W, int rows, int N, int N1, const float2* __restrict__ tw, int a0, int Tn,
    const float* __restrict__ scale, void* __restrict__ Z, void* __restrict__ Zlo, long long ldz, int im_off,
    int row0) {
    using S = Split<N2, 2>;
    constexpr int R1 = S::R1, R2 = S::R2, NT = S::NT, SB = S::SB, SC = S::SC, P2 = S::P2;
    constexpr int ES = FORM == 1 ? 4 : (FORM == 4 ? 1 : 2);   // bytes per Z element
    constexpr int CP = TB * N2 * 8 / 16 / NT;    // 16-byte copies per thread per tile
    static_assert(SC >= N2, "the exchange tile covers the W tile");
    extern __shared__ float2 sm[];
    float2* Bt = sm;                              // W tile Bt[k2 TB + c], then the exchange tile Bt[c SC + b SB + u]
    float2* tw2 = Bt + TB * SC;                   // tw2[u R2 + b] = e^{2 pi i b u / N2}
    const int tid = threadIdx.x, t10 = blockIdx.x * TB;
    const int j0 = blockIdx.y * RC, j1 = min(j0 + RC, rows);
    auto fetch = [&](int j) {
        const char* g = reinterpret_cast<const char*>(W + (long long)j * N + (long long)blockIdx.x * (N2 * TB));
        char* d = reinterpret_cast<char*>(Bt);
#pragma unroll
        for (int i = 0; i < CP; ++i) cp_async16(d + (i * NT + tid) * 16, g + (i * NT + tid) * 16);
        cp_async_commit();
    };
    fetch(j0);
    // 1 / scale folded into the step-1 twiddles; fp8: scale holds one scale per row, applied at the store
    const float inv0 = FORM == 4 ? 1.f : 1.0f / *scale;
    for (int e = tid; e < N2; e += NT) {
        const float2 w = tw[(e % R2) * (e / R2) * (N / N2)];
        tw2[e] = make_float2(w.x * inv0, w.y * inv0);
    }
    const int c = tid % TB, b = tid / TB;
    char* zb = static_cast<char*>(Z);
    char* zl = static_cast<char*>(Zlo);
    for (int j = j0; j < j1; ++j) {
        const float inv = FORM == 4 ? 1.0f / scale[j] : 1.f;
        cp_async_wait_all();
        __syncthreads();
        float2 x[R1];
#pragma unroll
        for (int a = 0; a < R1; ++a) x[a] = Bt[(R2 * a + b) * TB + c];
        __syncthreads();
        dft_reg<R1>(x);
        static_for<R1>([&](auto U) {
            constexpr int u = decltype(U)::value;
            Bt[c * SC + b * SB + u] = cmul(x[brev(u, ilog2(R1))], tw2[u * R2 + b]);
        });
        __syncthreads();
        float2 y[P2][R2];
#pragma unroll
        for (int p = 0; p < P2; ++p) {
            const int d = tid + NT * p;
            const int c2 = d % TB, u = d / TB;
#pragma unroll
            for (int bb = 0; bb < R2; ++bb) y[p][bb] = Bt[c2 * SC + bb * SB + u];
        }
        __syncthreads();
        if (j + 1 < j1) fetch(j + 1);
        const long long re_off = (long long)(row0 + j) * ldz * ES, im_off_b = (long long)(im_off + row0 + j) * ldz * ES;
        void* Zr = zb + re_off;
        void* Zi = zb + im_off_b;
        void* Zlr = FORM == 2 ? (void*)(zl + re_off) : nullptr;
        void* Zli = FORM == 2 ? (void*)(zl + im_off_b) : nullptr;
#pragma unroll
        for (int p = 0; p < P2; ++p) {
            const int d = tid + NT * p;
            const int c2 = d % TB, u = d / TB;
            dft_reg<R2>(y[p]);
            const int t0 = t10 + c2 + N1 * u - a0;
            static_for<R2>([&](auto V) {
                constexpr int vv = decltype(V)::value;
                const int t = t0 + N1 * (R1 * vv);
                if (t >= 0 && t < Tn) {
                    const float2 z = y[p][brev(vv, ilog2(R2))];
                    if constexpr (FORM == 4) store_z<FORM>(Zr, Zi, Zlr, Zli, t, z.x * inv, z.y * inv);
                    else store_z<FORM>(Zr, Zi, Zlr, Zli, t, z.x, z.y);
                }
            });
        }
    }
}

// Pass 2 over row chunks with TBW = 16 columns per CTA (two adjacent W blocks, 128 KB contiguous). Each Z store
// instruction of a warp covers two runs of 16 consecutive samples (32 bytes for 16-bit Z: whole L2 sectors) instead
// of four runs of 8, halving the write requests of the pass, which bound it with four 16-bit planes. One CTA of
// 16 R2 threads per SM (the tile and exchange buffer take 135 KB). Thread index bits: step 1 (c, b) with
// c = (t & 7) + 8 ((t >> 4) & 1), b = ((t >> 3) & 1) + 2 (t >> 5), so a half-warp reads 16 consecutive tile words;
// step 2 (c2, u) with the same c and u = ((t >> 3) & 1) + 2 (t >> 5); SC = 2 (mod 16) keeps both exchange accesses
// free of bank conflicts.
constexpr int TBW = 16;

template <int N2>
struct SplitW {
    using S = Split<N2, 2>;
    static constexpr int R1 = S::R1, R2 = S::R2, SB = S::SB;
    static constexpr int NT = TBW * R2;
    static constexpr int SC = R2 * SB + ((2 - (R2 * SB) % 16) + 16) % 16;
    static_assert(R1 == R2, "the 16-column pass 2 is for square splits (N2 = 1024, 256, 64)");
    static_assert(SC >= N2, "the exchange buffer holds the W tile");
};

// Paired Z stores (PAIR): the lanes c and c + 1 (c even, lane ^ 1) hold the samples t and t + 1 of every vv. Each
// lane packs its (re, im), the two swap one 32-bit word by a shuffle, and the even lane stores the two real parts,
// the odd lane the two imaginary parts, one word per plane (two 16-bit samples, or 64 bits of fp32): half the store
// instructions of one 16-bit store per plane and sample. Needs an even a0, Tn and ldz and word-aligned planes.
// Split bf16: hi = bf16(x), lo = bf16(x - hi), as store_z.
template <int FORM>
struct PairStore {
    unsigned hsel, lsel, ssel;
    bool odd;
    __device__ __forceinline__ explicit PairStore(bool o) : odd(o) {
        // __byte_perm(x, y, s): bytes 0-3 of x, 4-7 of y
        hsel = o ? 0x3276u : 0x5410u;                      // 16-bit forms: own re | partner re, partner im | own im
        if constexpr (FORM == 2) {
            ssel = o ? 0x5410u : 0x7632u;                  // send: odd (re hi, re lo), even (im hi, im lo)
            hsel = o ? 0x3254u : 0x5410u;
            lsel = o ? 0x3276u : 0x7610u;
        }
    }
    // one sample (scaled); writes through the lane's plane pointers ph, pl (element pairs) at pair index k
    template <int K>
    __device__ __forceinline__ void store(float xr, float xi, unsigned* ph, unsigned* pl, bool ok) const {
        if constexpr (FORM == 1) {
            const float snd = odd ? xr : xi;
            const float rcv = __shfl_xor_sync(0xffffffffu, snd, 1);
            const float2 w = odd ? make_float2(rcv, xi) : make_float2(xr, rcv);
            if (ok) __stcs(reinterpret_cast<float2*>(ph) + K, w);
        } else if constexpr (FORM == 2) {
            const __nv_bfloat162 h2 = __floats2bfloat162_rn(xr, xi);
            const unsigned H = *reinterpret_cast<const unsigned*>(&h2);
            const float hr = __uint_as_float(H << 16), hm = __uint_as_float(H & 0xffff0000u);
            const __nv_bfloat162 l2 = __floats2bfloat162_rn(xr - hr, xi - hm);
            const unsigned L = *reinterpret_cast<const unsigned*>(&l2);
            const unsigned R = __shfl_xor_sync(0xffffffffu, __byte_perm(H, L, ssel), 1);
            if (ok) {
                __stcs(ph + K, __byte_perm(H, R, hsel));
                __stcs(pl + K, __byte_perm(L, R, lsel));
            }
        } else {
            unsigned H;
            if constexpr (FORM == 0) {
                const __half2 h2 = __floats2half2_rn(xr, xi);
                H = *reinterpret_cast<const unsigned*>(&h2);
            } else {
                const __nv_bfloat162 h2 = __floats2bfloat162_rn(xr, xi);
                H = *reinterpret_cast<const unsigned*>(&h2);
            }
            const unsigned R = __shfl_xor_sync(0xffffffffu, H, 1);
            if (ok) __stcs(ph + K, __byte_perm(H, R, hsel));
        }
    }
};

template <int N2, int FORM, bool PAIR>
__global__ void __launch_bounds__(SplitW<N2>::NT, 1) basis_pass2_w(
    const float2* __restrict__ W, int rows, int N, const float2* __restrict__ tw, int a0, int Tn,
    const float* __restrict__ scale, void* __restrict__ Z, void* __restrict__ Zlo, long long ldz, int im_off,
    int row0) {
    using S = SplitW<N2>;
    constexpr int R1 = S::R1, R2 = S::R2, NT = S::NT, SB = S::SB, SC = S::SC;
    constexpr int N1 = N2;                        // square split: t = t1 + N1 (u + R1 v)
    constexpr int ES = FORM == 1 ? 4 : (FORM == 4 ? 1 : 2);   // bytes per Z element
    constexpr int CP = TBW * N2 * 8 / 16 / NT;   // 16-byte copies per thread per tile
    static_assert(!PAIR || FORM != 4, "fp8 Z is stored per sample");
    extern __shared__ float2 sm[];
    float2* Bt = sm;                              // W tile (two blocks of TB columns), then the exchange tile
    float2* tw2 = Bt + TBW * SC;                  // tw2[u R2 + b] = e^{2 pi i b u / N2} / scale
    const int tid = threadIdx.x, t10 = blockIdx.x * TBW;
    const int j0 = blockIdx.y * RC, j1 = min(j0 + RC, rows);
    auto fetch = [&](int j) {
        const char* g = reinterpret_cast<const char*>(W + (long long)j * N + (long long)blockIdx.x * (N2 * TBW));
        char* d = reinterpret_cast<char*>(Bt);
#pragma unroll
        for (int i = 0; i < CP; ++i) cp_async16(d + (i * NT + tid) * 16, g + (i * NT + tid) * 16);
        cp_async_commit();
    };
    fetch(j0);
    // 1 / scale folded into the step-1 twiddles; fp8: scale holds one scale per row, applied at the store
    const float inv0 = FORM == 4 ? 1.f : 1.0f / *scale;
    for (int e = tid; e < N2; e += NT) {
        const float2 w = tw[(e % R2) * (e / R2) * (N / N2)];
        tw2[e] = make_float2(w.x * inv0, w.y * inv0);
    }
    const int c = (tid & 7) + 8 * ((tid >> 4) & 1);
    const int lo = (tid >> 3) & 1, hi = tid >> 5;
    const int b = lo + 2 * hi;                    // step 1: b < R2
    const int u2 = lo + 2 * hi;                   // step 2: u < R1 (= R2)
    const int cblk = (c >> 3) * (N2 * TB) + (c & 7);
    const int t0 = t10 + c + N1 * u2 - a0;        // sample of vv = 0; vv steps by N1 R1
    const bool odd = c & 1;
    const int te = t0 - (PAIR && odd ? 1 : 0);    // the pair's even sample
    unsigned vmask = 0;                           // bit vv: the sample (pair) lies in [0, Tn)
#pragma unroll
    for (int v = 0; v < R2; ++v) {
        const int t = te + N1 * R1 * v;
        if (t >= 0 && t < Tn) vmask |= 1u << v;
    }
    const PairStore<PAIR ? FORM : 0> ps(odd);
    const int prow = row0 + (PAIR && odd ? im_off : 0);    // paired: the odd lane writes the imaginary planes
    char* zb = static_cast<char*>(Z);
    char* zl = static_cast<char*>(Zlo);
    for (int j = j0; j < j1; ++j) {
        const float inv = FORM == 4 ? 1.0f / scale[j] : 1.f;
        cp_async_wait_all();
        __syncthreads();
        float2 x[R1];
#pragma unroll
        for (int a = 0; a < R1; ++a) x[a] = Bt[cblk + (R2 * a + b) * TB];
        __syncthreads();
        dft_reg<R1>(x);
        static_for<R1>([&](auto U) {
            constexpr int u = decltype(U)::value;
            Bt[c * SC + b * SB + u] = cmul(x[brev(u, ilog2(R1))], tw2[u * R2 + b]);
        });
        __syncthreads();
        float2 y[R2];
#pragma unroll
        for (int bb = 0; bb < R2; ++bb) y[bb] = Bt[c * SC + bb * SB + u2];
        __syncthreads();
        if (j + 1 < j1) fetch(j + 1);
        dft_reg<R2>(y);
        if constexpr (PAIR) {
            const long long off = ((long long)(prow + j) * ldz + te) * ES;
            unsigned* ph = reinterpret_cast<unsigned*>(zb + off);
            unsigned* pl = FORM == 2 ? reinterpret_cast<unsigned*>(zl + off) : nullptr;
            static_for<R2>([&](auto V) {
                constexpr int vv = decltype(V)::value;
                constexpr int K = N1 * R1 * vv / 2;    // pair index of vv (64-bit pairs for fp32: same count)
                const float2 z = y[brev(vv, ilog2(R2))];
                ps.template store<K>(z.x, z.y, ph, pl, (vmask >> vv) & 1u);
            });
        } else {
            const long long re_off = (long long)(row0 + j) * ldz * ES, im_off_b = (long long)(im_off + row0 + j) * ldz * ES;
            void* Zr = zb + re_off;
            void* Zi = zb + im_off_b;
            void* Zlr = FORM == 2 ? (void*)(zl + re_off) : nullptr;
            void* Zli = FORM == 2 ? (void*)(zl + im_off_b) : nullptr;
            static_for<R2>([&](auto V) {
                constexpr int vv = decltype(V)::value;
                if ((vmask >> vv) & 1u) {
                    const float2 z = y[brev(vv, ilog2(R2))];
                    store_z<FORM>(Zr, Zi, Zlr, Zli, t0 + N1 * R1 * vv, z.x * inv, z.y * inv);
                }
            });
        }
    }
}

// ---------------------------------------------------------------------------------------------------------------------
// Persistent form of the two passes for N = 2^20 (N1 = N2 = 1024): W stays in L2.
// Rows go in chunks of pc rows through a ring of nslot slots of W (pc rows of N each). Work items, taken in order from
// a global ticket by a grid of resident CTAs:
//   P1(c, g): pass 1 of chunk c for the 8 columns k2 = 8 g .. 8 g + 7 (one basis_pass1_w CTA's work);
//   P2(c, b): pass 2 of chunk c for the 8 columns t1 = 8 b .. 8 b + 7 (one basis_pass2_p CTA's work).
// Ticket order with lookahead L: P1(0 .. L-1, *), then for c = 0, 1, ...: P1(c + L, *), P2(c, *). P2(c, *) starts when
// the 128 items P1(c, *) (and P1(0, *), for the scale) are done; P1(c, *) starts when the 128 items P2(c - nslot, *)
// are done (its slot is free; nslot > L, so those come earlier). Every item waits only on items earlier in the ticket order, all held by running CTAs, so the earliest
// unfinished item always progresses. Every wait is bounded (kWaitLimitNs): a timeout records GWB_ERR_TIMEOUT, raises
// the abort word, and every CTA returns at its next ticket with no copy in flight.
// After pass 2 has copied a W tile into shared memory its L2 lines are dropped without write-back (discard.global.L2),
// so W never reaches HBM: per row only the basis filters are read and Z is written.
// Scale: the Parseval rms of the first chunk's rows (the basis rows have unit norm under the SVD metric, so their
// series have comparable rms; the scale cancels between Z and A); each P2 item sums the first chunk's per-column
// partials in a fixed order. fp8: each P2 item sums its rows' per-column |q|^2 in a fixed order for the row scales.
// ---------------------------------------------------------------------------------------------------------------------
constexpr int PG = 128;                       // items per chunk and pass (1024 / 8)
constexpr int PC_MAX = 4;                     // rows per chunk at most (the fp8 row scales take one warp per row)

struct PersistArgs {
    const float2* Vp;
    long long ldvp;
    int rows;
    const float2* Dp;
    const float2* tw;
    float2* W;                // nslot * pc rows of N
    int pc, nslot, look;      // rows per chunk, W slots, lookahead (chunks of pass 1 ahead of pass 2)
    int a0, Tn;
    void* Z;
    void* Zlo;
    long long ldz;
    int im_off, row0;
    double* partials;         // N2 doubles: the first chunk's sum of |q|^2 per column
    float* rowpart;           // fp8: rows x N2 sums of |q|^2 per (row, column)
    float* rowscale;          // fp8: the row scales (written by the items with b = 0)
    float* scale_out;         // the scale (written by item P2(0, 0))
    int* sync;                // ticket, abort, p1done[nch], p2done[nch] (zero at launch)
    DeviceError* err;
};

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// thread 0: wait until *p >= target, bounded; false on timeout or when another CTA aborted
__device__ bool wait_count(const int* p, int target, const int* abort_word) {
    if (ld_acquire(p) >= target) return true;
    const uint64_t t0 = globaltimer_ns();
    while (true) {
        for (int i = 0; i < 16; ++i) {
            __nanosleep(64);
            if (ld_acquire(p) >= target) return true;
        }
        if (*(volatile const int*)abort_word) return false;
        if (globaltimer_ns() - t0 > kWaitLimitNs) return false;
    }
}

// item t of the ticket order: type 1 = P1, 2 = P2; false past the end
__device__ __forceinline__ bool persist_item(int t, int nch, int look, int& type, int& c, int& g) {
    const int pre = min(look, nch);                      // P1 of the first chunks
    if (t < pre * PG) {
        type = 1;
        c = t / PG;
        g = t % PG;
        return true;
    }
    t -= pre * PG;
    const int full = max(0, nch - look);                 // blocks P1(c + look, *), P2(c, *)
    if (t < full * 2 * PG) {
        const int j = t / (2 * PG), o = t % (2 * PG);
        type = o < PG ? 1 : 2;
        c = o < PG ? j + look : j;
        g = o < PG ? o : o - PG;
        return true;
    }
    t -= full * 2 * PG;
    const int j = full + t / PG;                         // the last chunks: P2 only
    if (j >= nch) return false;
    type = 2;
    c = j;
    g = t % PG;
    return true;
}

// pass 1 of chunk c, columns k2 = 8 g + warp (the body of basis_pass1_w over the chunk's rows)
__device__ __forceinline__ void persist_p1(float2* sm, const PersistArgs& a, int c, int g) {
    constexpr int N = 1 << 20, N1 = 1024, N2 = 1024, R = 32, H = N1 / 2, NW = 8, YS = R * (R + 1);
    constexpr int WS = YS + R + H;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float2* tw2 = sm;
    float2* Yw = sm + N1 + warp * WS;
    float2* THw = Yw + YS;
    float2* Vs = THw + R;
    const int k2 = g * NW + warp;
    const int j0 = c * a.pc, j1 = min(j0 + a.pc, a.rows);
    constexpr int mask = N - 1;
    float2* Wslot = a.W + (long long)(c % a.nslot) * a.pc * N;
    auto fetch = [&](int j) {
        const char* gp = reinterpret_cast<const char*>(a.Vp + (long long)j * a.ldvp + k2 * H);
        char* d = reinterpret_cast<char*>(Vs);
#pragma unroll
        for (int i = 0; i < 8; ++i) cp_async16(d + i * 512 + lane * 16, gp + i * 512 + lane * 16);
        cp_async_commit();
    };
    fetch(j0);
    float2 dk[R / 2];
#pragma unroll
    for (int q = 0; q < R / 2; ++q) dk[q] = __ldg(a.Dp + k2 * H + R * q + lane);
    const float2 dN = a.Dp[N / 2];
    THw[lane] = a.tw[(k2 * (R * lane)) & mask];
    const float2 tl = a.tw[(k2 * lane) & mask];
    __syncwarp();
    double acc = 0.0;
    for (int j = j0; j < j1; ++j) {
        cp_async_wait_all();
        __syncwarp();
        float2 x[R];
#pragma unroll
        for (int q = 0; q < R / 2; ++q) x[q] = Vs[R * q + lane];
        __syncwarp();
        if (j + 1 < j1) fetch(j + 1);
        float part = 0.f;
#pragma unroll
        for (int q = 0; q < R / 2; ++q) {
            const float2 av = x[q];
            x[q] = make_float2(fmaf(av.x, dk[q].x, av.y * dk[q].y), fmaf(av.x, dk[q].y, -(av.y * dk[q].x)));
            part = fmaf(x[q].x, x[q].x, fmaf(x[q].y, x[q].y, part));
        }
        x[R / 2] = make_float2(0.f, 0.f);
        if (k2 == 0 && lane == 0) {                         // the bin N / 2
            const float2 av = a.Vp[(long long)j * a.ldvp + N / 2];
            x[R / 2] = make_float2(fmaf(av.x, dN.x, av.y * dN.y), fmaf(av.x, dN.y, -(av.y * dN.x)));
            part = fmaf(x[R / 2].x, x[R / 2].x, fmaf(x[R / 2].y, x[R / 2].y, part));
        }
#pragma unroll
        for (int q = R / 2 + 1; q < R; ++q) x[q] = make_float2(0.f, 0.f);
        acc += (double)part;
        if (a.rowpart) {
            float ps = part;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) ps += __shfl_xor_sync(0xffffffffu, ps, off);
            if (lane == 0) a.rowpart[(long long)j * N2 + k2] = ps;
        }
        dft_reg<R>(x);
        static_for<R>([&](auto U) {
            constexpr int u = decltype(U)::value;
            Yw[lane * (R + 1) + u] = cmul(x[brev(u, ilog2(R))], tw2[u * R + lane]);
        });
        __syncwarp();
#pragma unroll
        for (int bb = 0; bb < R; ++bb) x[bb] = Yw[bb * (R + 1) + lane];
        __syncwarp();
        dft_reg<R>(x);
        float2* wc = Wslot + (long long)(j - j0) * N + (lane >> 3) * (N2 * 8) + k2 * 8 + (lane & 7);
        static_for<R>([&](auto V) {
            constexpr int vv = decltype(V)::value;
            wc[4 * vv * (N2 * 8)] = cmul(x[brev(vv, ilog2(R))], cmul(tl, THw[vv]));
        });
    }
    if (c == 0) {                                           // the scale's partials: the first chunk, per column
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0) a.partials[k2] = acc;
    }
    __threadfence();                                        // W (and the partials) before the item's done count
}

// sum of n doubles (or floats as doubles) by one warp in a fixed order: lane l adds l, l + 32, ... then a fixed tree
template <typename T>
__device__ __forceinline__ double warp_fixed_sum(const T* v, int n) {
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += (double)v[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    return s;
}

// pass 2 of chunk c, t1 = 8 b .. 8 b + 7 (the body of basis_pass2_p over the chunk's rows)
template <int FORM>
__device__ __forceinline__ void persist_p2(float2* sm, const PersistArgs& a, int c, int b, float* s_inv) {
    constexpr int N = 1 << 20, N1 = 1024, N2 = 1024;
    using S = Split<N2, 2>;
    constexpr int R1 = S::R1, R2 = S::R2, NT = S::NT, SB = S::SB, SC = S::SC, P2 = S::P2;
    constexpr int ES = FORM == 1 ? 4 : (FORM == 4 ? 1 : 2);
    constexpr int CP = TB * N2 * 8 / 16 / NT;
    static_assert(NT == 256 && SC >= N2, "persistent pass 2 layout");
    const float2* tw2 = sm;                                 // e^{2 pi i b u / N2}: the same table as pass 1's
    float2* Bt = sm + N1;
    const int tid = threadIdx.x, t10 = b * TB;
    const int j0 = c * a.pc, j1 = min(j0 + a.pc, a.rows);
    const float2* Wslot = a.W + (long long)(c % a.nslot) * a.pc * N;
    auto tile = [&](int j) { return Wslot + (long long)(j - j0) * N + (long long)b * (N2 * TB); };
    auto fetch = [&](int j) {
        const char* gp = reinterpret_cast<const char*>(tile(j));
        char* d = reinterpret_cast<char*>(Bt);
#pragma unroll
        for (int i = 0; i < CP; ++i) cp_async16(d + (i * NT + tid) * 16, gp + (i * NT + tid) * 16);
        cp_async_commit();
    };
    fetch(j0);
    // scales: the first chunk's Parseval rms (all forms; written once for the caller), and the fp8 row scales
    const int warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        const double s = warp_fixed_sum(a.partials, N2);
        const int nf = min(a.pc, a.rows);
        const float sc = (float)sqrt(s / (double)nf / 2.0);
        if (lane == 0) {
            s_inv[0] = 1.0f / sc;
            if (c == 0 && b == 0) *a.scale_out = sc;
        }
    }
    if (FORM == 4 && warp >= 1 && warp <= a.pc && j0 + warp - 1 < j1) {
        const int j = j0 + warp - 1;
        const double t = warp_fixed_sum(a.rowpart + (long long)j * N2, N2);
        const float rs = t > 0.0 ? (float)(sqrt(t / 2.0) / 16.0) : 1.f;
        if (lane == 0) {
            s_inv[warp] = 1.0f / rs;
            if (b == 0) a.rowscale[j] = rs;
        }
    }
    __syncthreads();
    const int cc = tid % TB, bb = tid / TB;
    char* zb = static_cast<char*>(a.Z);
    char* zl = static_cast<char*>(a.Zlo);
    for (int j = j0; j < j1; ++j) {
        const float inv = FORM == 4 ? s_inv[1 + j - j0] : s_inv[0];
        cp_async_wait_all();
        __syncthreads();
        {   // the W tile is in shared memory: drop its L2 lines without write-back (512 lines of 128 bytes)
            const char* gp = reinterpret_cast<const char*>(tile(j));
            asm volatile("discard.global.L2 [%0], 128;" ::"l"(gp + tid * 128) : "memory");
            asm volatile("discard.global.L2 [%0], 128;" ::"l"(gp + (tid + NT) * 128) : "memory");
        }
        float2 x[R1];
#pragma unroll
        for (int q = 0; q < R1; ++q) x[q] = Bt[(R2 * q + bb) * TB + cc];
        __syncthreads();
        dft_reg<R1>(x);
        static_for<R1>([&](auto U) {
            constexpr int u = decltype(U)::value;
            Bt[cc * SC + bb * SB + u] = cmul(x[brev(u, ilog2(R1))], tw2[u * R2 + bb]);
        });
        __syncthreads();
        float2 y[P2][R2];
#pragma unroll
        for (int p = 0; p < P2; ++p) {
            const int d = tid + NT * p;
            const int c2 = d % TB, u = d / TB;
#pragma unroll
            for (int q = 0; q < R2; ++q) y[p][q] = Bt[c2 * SC + q * SB + u];
        }
        __syncthreads();
        if (j + 1 < j1) fetch(j + 1);
        const long long re_off = (long long)(a.row0 + j) * a.ldz * ES;
        const long long im_off_b = (long long)(a.im_off + a.row0 + j) * a.ldz * ES;
        void* Zr = zb + re_off;
        void* Zi = zb + im_off_b;
        void* Zlr = FORM == 2 ? (void*)(zl + re_off) : nullptr;
        void* Zli = FORM == 2 ? (void*)(zl + im_off_b) : nullptr;
#pragma unroll
        for (int p = 0; p < P2; ++p) {
            const int d = tid + NT * p;
            const int c2 = d % TB, u = d / TB;
            dft_reg<R2>(y[p]);
            const int t0 = t10 + c2 + N1 * u - a.a0;
            static_for<R2>([&](auto V) {
                constexpr int vv = decltype(V)::value;
                const int t = t0 + N1 * (R1 * vv);
                if (t >= 0 && t < a.Tn) {
                    const float2 z = y[p][brev(vv, ilog2(R2))];
                    store_z<FORM>(Zr, Zi, Zlr, Zli, t, z.x * inv, z.y * inv);
                }
            });
        }
    }
}

template <int FORM>
__global__ void __launch_bounds__(256, 2) basis_persist(const __grid_constant__ PersistArgs a) {
    constexpr int N1 = 1024, N = 1 << 20;
    extern __shared__ float2 sm[];
    __shared__ int s_t, s_ok;
    __shared__ float s_inv[1 + PC_MAX];
    for (int e = threadIdx.x; e < N1; e += blockDim.x) sm[e] = a.tw[(e % 32) * (e / 32) * (N / N1)];
    __syncthreads();
    const int nch = (a.rows + a.pc - 1) / a.pc;
    int* ticket = a.sync;
    int* abort_word = a.sync + 1;
    int* p1done = a.sync + 2;
    int* p2done = p1done + nch;
    // look = 0: split roles, the first half of the grid takes only pass-1 items (ticket), the second half only pass-2
    // items (ticket2), each in chunk order; pass 1 then runs ahead of pass 2 as far as the ring's free slots allow
    const bool split = a.look == 0;
    const bool p1role = (int)blockIdx.x < (int)gridDim.x / 2;
    int* ticket2 = p2done + nch;
    while (true) {
        if (threadIdx.x == 0)
            s_t = *(volatile int*)abort_word ? 0x7fffffff : atomicAdd(split && !p1role ? ticket2 : ticket, 1);
        __syncthreads();
        int type = 0, c = 0, g = 0;
        if (split) {
            if (s_t >= nch * PG) break;                           // uniform over the CTA
            type = p1role ? 1 : 2;
            c = s_t / PG;
            g = s_t % PG;
        } else if (!persist_item(s_t, nch, a.look, type, c, g)) {
            break;
        }
        if (threadIdx.x == 0) {
            bool ok = true;
            if (type == 1 && c >= a.nslot) ok = wait_count(&p2done[c - a.nslot], PG, abort_word);
            if (type == 2) ok = wait_count(&p1done[0], PG, abort_word) && wait_count(&p1done[c], PG, abort_word);
            if (!ok) {
                record_error(a.err, GWB_ERR_TIMEOUT, 301, type, c);
                atomicExch(abort_word, 1);
            }
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) break;
        if (type == 1) persist_p1(sm, a, c, g);
        else persist_p2<FORM>(sm, a, c, g, s_inv);
        __syncthreads();
        if (threadIdx.x == 0) atomicAdd(type == 1 ? &p1done[c] : &p2done[c], 1);
    }
}

int log2i(long long n) {
    int l = 0;
    while ((1ll << l) < n) ++l;
    return l;
}

size_t persist_smem() { return (size_t)(1024 + 8 * (32 * 33 + 32 + 512)) * sizeof(float2); }

template <int FORM>
int launch_persist(const PersistArgs& a, cudaStream_t s) {
    auto k = basis_persist<FORM>;
    const size_t smem = persist_smem();
    GWB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    GWB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, smem));
    GWB_CHECK_ARG(per_sm >= 1, GWB_ERR_CUDA, "basis_persist: no CTA fits on an SM");
    const int nch = (a.rows + a.pc - 1) / a.pc;
    int grid = per_sm * num_sms();
    if (a.look > 0) grid = std::min(grid, 2 * PG * nch);
    else grid = std::max(2, grid & ~1);                // split roles: two equal halves
    k<<<grid, 256, smem, s>>>(a);
    GWB_LAUNCH_CHECK("basis_persist");
    return GWB_OK;
}

int launch_pass1_w(const float2* Vp, long long ldvp, int rows, const float2* Dp, int N, int N2, const float2* tw,
                   float2* W, int nfirst, double* partials, unsigned* ticket, float* scale_out, float* rowpart,
                   cudaStream_t s) {
    const size_t smem = (size_t)(1024 + 8 * (32 * 33 + 32 + 512)) * sizeof(float2);
    GWB_CUDA(cudaFuncSetAttribute(basis_pass1_w, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    basis_pass1_w<<<dim3(N2 / 8, (rows + RC - 1) / RC), 256, smem, s>>>(Vp, ldvp, rows, Dp, N, N2, tw, W, nfirst,
                                                                         partials, ticket, scale_out, rowpart);
    GWB_LAUNCH_CHECK("basis_pass1_w");
    return GWB_OK;
}

template <int N1>
int launch_pass1(const float2* Vp, long long ldvp, int rows, const float2* Dp, int N, int N2, const float2* tw,
                 float2* W, int nfirst, double* partials, unsigned* ticket, float* scale_out, float* rowpart,
                 cudaStream_t s) {
    using S = Split<N1, 8>;
    const size_t smem = (size_t)(TB * S::SC + N1 + N1 / 16 + TB * (S::R1 + 1) + TB * (S::R2 + 1)) * sizeof(float2);
    auto k = basis_pass1<N1>;
    GWB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<dim3(N2 / TB, rows), S::NT, smem, s>>>(Vp, ldvp, Dp, N, N2, tw, W, nfirst, partials, ticket, scale_out,
                                              rowpart);
    GWB_LAUNCH_CHECK("basis_pass1");
    return GWB_OK;
}

template <int N2, int FORM>
int launch_pass2_f(const float2* W, int N, int N1, int rows, const float2* tw, int a0, int Tn, const float* scale,
                   void* Z, void* Zlo, long long ldz, int im_off, int row0, cudaStream_t s) {
    using S = Split<N2, 2>;
    const size_t smem = (size_t)(TB * S::SC + N2) * sizeof(float2);
    auto k = basis_pass2<N2, FORM>;
    GWB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<dim3(N1 / TB, rows), S::NT, smem, s>>>(W, N, N1, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0);
    GWB_LAUNCH_CHECK("basis_pass2");
    return GWB_OK;
}

template <int N2, int FORM>
int launch_pass2_p(const float2* W, int N, int N1, int rows, const float2* tw, int a0, int Tn, const float* scale,
                   void* Z, void* Zlo, long long ldz, int im_off, int row0, cudaStream_t s) {
    using S = Split<N2, 2>;
    const size_t smem = (size_t)(TB * S::SC + N2) * sizeof(float2);
    auto k = basis_pass2_p<N2, FORM>;
    GWB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<dim3(N1 / TB, (rows + RC - 1) / RC), S::NT, smem, s>>>(W, rows, N, N1, tw, a0, Tn, scale, Z, Zlo, ldz,
                                                               im_off, row0);
    GWB_LAUNCH_CHECK("basis_pass2_p");
    return GWB_OK;
}

// paired Z stores when every pair of samples (t, t + 1), t even, is one aligned word of each plane
bool pair_ok(int form, int a0, int Tn, long long ldz, const void* Z, const void* Zlo) {
    const int es = form == 1 ? 4 : (form == 4 ? 1 : 2);
    const auto al = [&](const void* p) { return p == nullptr || reinterpret_cast<uintptr_t>(p) % (2 * es) == 0; };
    return form != 4 && a0 % 2 == 0 && Tn % 2 == 0 && ldz % 2 == 0 && al(Z) && (form != 2 || al(Zlo));
}
std::atomic<int> g_pass2_pair{1};            // 0: per-sample stores only (gwb_basis_set_pass2_pairs)

template <int N2, int FORM, bool PAIR>
int launch_pass2_wp(const float2* W, int N, int N1, int rows, const float2* tw, int a0, int Tn, const float* scale,
                    void* Z, void* Zlo, long long ldz, int im_off, int row0, cudaStream_t s) {
    using S = SplitW<N2>;
    GWB_CHECK_ARG(N1 == N2, GWB_ERR_SHAPE, "basis_pass2_w: N1=%d must equal N2=%d", N1, N2);
    const size_t smem = (size_t)(TBW * S::SC + N2) * sizeof(float2);
    auto k = basis_pass2_w<N2, FORM, PAIR>;
    GWB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<dim3(N1 / TBW, (rows + RC - 1) / RC), S::NT, smem, s>>>(W, rows, N, tw, a0, Tn, scale, Z, Zlo, ldz, im_off,
                                                                 row0);
    GWB_LAUNCH_CHECK("basis_pass2_w");
    return GWB_OK;
}

template <int N2, int FORM>
int launch_pass2_w(const float2* W, int N, int N1, int rows, const float2* tw, int a0, int Tn, const float* scale,
                   void* Z, void* Zlo, long long ldz, int im_off, int row0, cudaStream_t s) {
    if constexpr (FORM != 4) {
        if (g_pass2_pair.load() && pair_ok(FORM, a0, Tn, ldz, Z, Zlo))
            return launch_pass2_wp<N2, FORM, true>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
    }
    return launch_pass2_wp<N2, FORM, false>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
}

// columns per pass-2 CTA at N2 = 1024, per Z encoding (gwb_basis_set_pass2_columns): 16 (basis_pass2_w, the default:
// measured at r = 128, 5.3 against 6.0 us per row for fp16 Z and 6.1 against 8.6 for split bf16) or 8
// (basis_pass2_p, or the per-row kernel for the split form)
std::atomic<int> g_pass2_cols[5] = {{16}, {16}, {16}, {16}, {16}};

template <int N2>
int launch_pass2(int form, const float2* W, int N, int N1, int rows, const float2* tw, int a0, int Tn,
                 const float* scale, void* Z, void* Zlo, long long ldz, int im_off, int row0, cudaStream_t s) {
    if constexpr (N2 == 1024) {
        if (form >= 0 && form <= 4 && g_pass2_cols[form].load() == 16) {
            switch (form) {
                case 0: return launch_pass2_w<N2, 0>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
                case 1: return launch_pass2_w<N2, 1>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
                case 2: return launch_pass2_w<N2, 2>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
                case 3: return launch_pass2_w<N2, 3>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
                default: return launch_pass2_w<N2, 4>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
            }
        }
    }
    // row-chunk form for the long transforms; the split bf16 form (four Z planes) runs faster on the per-row kernel
    // (measured at N = 2^20, r = 128: 8.3 against 10.6 us per row)
    if constexpr (N2 >= 512) {
        switch (form) {
            case 0: return launch_pass2_p<N2, 0>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
            case 1: return launch_pass2_p<N2, 1>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
            case 3: return launch_pass2_p<N2, 3>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
            case 4: return launch_pass2_p<N2, 4>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
            default: break;
        }
    }
    switch (form) {
        case 0: return launch_pass2_f<N2, 0>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
        case 1: return launch_pass2_f<N2, 1>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
        case 2: return launch_pass2_f<N2, 2>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
        case 4: return launch_pass2_f<N2, 4>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
        default: return launch_pass2_f<N2, 3>(W, N, N1, rows, tw, a0, Tn, scale, Z, Zlo, ldz, im_off, row0, s);
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

int gwb_fourstep_order(const float* X, long long ldx, int rows, const float* isw, long long flen, long long N,
                       float* P, long long ldp, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(X && P, GWB_ERR_ARG, "fourstep_order: null pointer");
    GWB_CHECK_ARG(is_pow2(N) && N >= (1 << 12) && N <= (1 << 20), GWB_ERR_NOT_POW2,
                  "fourstep_order: N=%lld must be a power of two in [2^12, 2^20]", N);
    GWB_CHECK_ARG(rows > 0 && rows < 65536 && flen > 0 && flen <= N / 2 + 1 && ldx >= flen && ldp >= N / 2 + 1,
                  GWB_ERR_SHAPE, "fourstep_order: rows=%d flen=%lld N=%lld ldx=%lld ldp=%lld", rows, flen, N, ldx, ldp);
    const int p = log2i(N);
    const int N1 = 1 << ((p + 1) / 2), N2 = (int)(N / N1);
    fourstep_order_kernel<<<dim3(N2 / 32, N1 / 64, rows), dim3(32, 8), 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const float2*>(X), ldx, isw, flen, N2, N1 / 2, reinterpret_cast<float2*>(P), ldp);
    GWB_LAUNCH_CHECK("fourstep_order_kernel");
    return GWB_OK;
}

namespace gwb {
namespace {
// the ring's configuration (gwb_basis_ring_set_config), process-wide: rows per chunk, W slots, lookahead
std::atomic<int> g_ring_pc{2}, g_ring_nslot{3}, g_ring_look{1};
}  // namespace
}  // namespace gwb

int gwb_basis_ring_set_config(int pc, int nslot, int look) {
    using namespace gwb;
    GWB_CHECK_ARG(pc >= 1 && pc <= PC_MAX && look >= 0 && nslot > look && nslot >= 2 && nslot <= 16, GWB_ERR_ARG,
                  "basis_ring_set_config: pc=%d (1..%d) nslot=%d (> look, 2..16) look=%d (>= 0; 0: split roles)", pc,
                  PC_MAX, nslot, look);
    g_ring_pc.store(pc);
    g_ring_nslot.store(nslot);
    g_ring_look.store(look);
    return GWB_OK;
}

int gwb_basis_set_pass2_columns(int form, int cols) {
    using namespace gwb;
    GWB_CHECK_ARG(cols == 8 || cols == 16, GWB_ERR_ARG, "basis_set_pass2_columns: cols=%d (8 or 16)", cols);
    GWB_CHECK_ARG(form >= -1 && form <= 4, GWB_ERR_ARG, "basis_set_pass2_columns: form=%d (0-4, -1: all)", form);
    for (int f = 0; f < 5; ++f)
        if (form < 0 || f == form) g_pass2_cols[f].store(cols);
    return GWB_OK;
}

int gwb_basis_pass2_columns(int form) { return form >= 0 && form <= 4 ? gwb::g_pass2_cols[form].load() : -1; }

int gwb_basis_set_pass2_pairs(int on) {
    using namespace gwb;
    GWB_CHECK_ARG(on == 0 || on == 1, GWB_ERR_ARG, "basis_set_pass2_pairs: on=%d (0 or 1)", on);
    g_pass2_pair.store(on);
    return GWB_OK;
}

int gwb_basis_ring_rows(void) { return gwb::g_ring_pc.load() * gwb::g_ring_nslot.load(); }

int gwb_basis_ring_sync_ints(int rows) {
    const int pc = gwb::g_ring_pc.load();
    return 3 + 2 * ((rows + pc - 1) / pc);
}

int gwb_basis_fused_ring(const float* Vp, long long ldvp, int rows, const float* Dp, long long N, const float* tw,
                         float* W, int wrows, long long a0, long long Tn, int form, void* Z, void* Zlo, long long ldz, int im_off,
                         int row0, double* partials, long long npartials, float* scale, float* rowscale,
                         float* rowpart, long long rowpart_elems, int32_t* sync, long long sync_ints, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(Vp && Dp && tw && W && Z && scale && partials && sync && (form != 2 || Zlo), GWB_ERR_ARG,
                  "basis_fused_ring: null pointer");
    GWB_CHECK_ARG(form >= 0 && form <= 4, GWB_ERR_ARG, "basis_fused_ring: form %d", form);
    GWB_CHECK_ARG(N == (1 << 20), GWB_ERR_NOT_POW2, "basis_fused_ring: N=%lld (the ring form is for N = 2^20)", N);
    GWB_CHECK_ARG(rows > 0 && rows < 65536 && ldvp >= N / 2 + 1 && ldvp % 2 == 0 && (uintptr_t)Vp % 16 == 0 &&
                      a0 >= 0 && Tn > 0 && a0 + Tn <= N && ldz >= Tn && row0 >= 0 && row0 + rows <= im_off,
                  GWB_ERR_SHAPE, "basis_fused_ring: rows=%d ldvp=%lld a0=%lld Tn=%lld", rows, ldvp, a0, Tn);
    GWB_CHECK_ARG(npartials >= 1024 && sync_ints >= gwb_basis_ring_sync_ints(rows) && aligned(W, 128),
                  GWB_ERR_SHAPE, "basis_fused_ring: partials %lld (1024 needed), sync %lld ints (%d needed), W "
                  "128-byte aligned", npartials, sync_ints, gwb_basis_ring_sync_ints(rows));
    GWB_CHECK_ARG(form != 4 || (rowscale && rowpart && rowpart_elems >= (long long)rows * 1024), GWB_ERR_SHAPE,
                  "basis_fused_ring: the fp8 form needs rowscale (rows floats) and rowpart (rows x 1024 floats)");
    const int pc = g_ring_pc.load(), nslot = g_ring_nslot.load(), look = g_ring_look.load();
    GWB_CHECK_ARG(wrows >= pc * nslot, GWB_ERR_SHAPE, "basis_fused_ring: W holds %d rows, the ring needs %d", wrows,
                  pc * nslot);
    cudaStream_t s = (cudaStream_t)stream;
    GWB_CUDA(cudaMemsetAsync(sync, 0, sizeof(int32_t) * gwb_basis_ring_sync_ints(rows), s));
    PersistArgs a;
    a.pc = pc;
    a.nslot = nslot;
    a.look = look;
    a.Vp = reinterpret_cast<const float2*>(Vp);
    a.ldvp = ldvp;
    a.rows = rows;
    a.Dp = reinterpret_cast<const float2*>(Dp);
    a.tw = reinterpret_cast<const float2*>(tw);
    a.W = reinterpret_cast<float2*>(W);
    a.a0 = (int)a0;
    a.Tn = (int)Tn;
    a.Z = Z;
    a.Zlo = Zlo;
    a.ldz = ldz;
    a.im_off = im_off;
    a.row0 = row0;
    a.partials = partials;
    a.rowpart = form == 4 ? rowpart : nullptr;
    a.rowscale = form == 4 ? rowscale : nullptr;
    a.scale_out = scale;
    a.sync = sync;
    a.err = device_error_ptr();
    switch (form) {
        case 0: return launch_persist<0>(a, s);
        case 1: return launch_persist<1>(a, s);
        case 2: return launch_persist<2>(a, s);
        case 3: return launch_persist<3>(a, s);
        default: return launch_persist<4>(a, s);
    }
}

int gwb_basis_fused(const float* Vp, long long ldvp, int rows, const float* Dp, long long N, const float* tw, float* W,
                    int wrows, long long a0, long long Tn, int form, void* Z, void* Zlo, long long ldz, int im_off,
                    int row0, int nfirst, double* partials, long long npartials, uint32_t* ticket, float* scale,
                    float* rowscale, float* rowpart, long long rowpart_elems, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(Vp && Dp && tw && W && Z && scale && (form != 2 || Zlo), GWB_ERR_ARG, "basis_fused: null pointer");
    GWB_CHECK_ARG(form >= 0 && form <= 4, GWB_ERR_ARG, "basis_fused: form %d", form);
    GWB_CHECK_ARG(is_pow2(N) && N >= (1 << 12) && N <= (1 << 20), GWB_ERR_NOT_POW2,
                  "basis_fused: N=%lld must be a power of two in [2^12, 2^20]", N);
    GWB_CHECK_ARG(rows > 0 && rows < 65536 && wrows > 0 && ldvp >= N / 2 + 1 && a0 >= 0 && Tn > 0 && a0 + Tn <= N &&
                  ldz >= Tn && row0 >= 0 && row0 + rows <= im_off, GWB_ERR_SHAPE,
                  "basis_fused: rows=%d wrows=%d ldvp=%lld N=%lld a0=%lld Tn=%lld", rows, wrows, ldvp, N, a0, Tn);
    const int p = log2i(N);
    const int N1 = 1 << ((p + 1) / 2), N2 = (int)(N / N1);
    const int nf = std::min(nfirst, std::min(rows, wrows));
    const long long need = N1 == 1024 ? (long long)(nf + RC - 1) / RC * N2 : (long long)nf * (N2 / TB);
    GWB_CHECK_ARG(nf <= 0 || (partials && ticket && need <= npartials), GWB_ERR_SHAPE,
                  "basis_fused: scale partials need %lld entries", need);
    GWB_CHECK_ARG(N1 != 1024 || ((uintptr_t)Vp % 16 == 0 && ldvp % 2 == 0), GWB_ERR_ALIGN,
                  "basis_fused: Vp and its row stride must be 16-byte aligned");
    // fp8: per-row partial sums of |q|^2 (P per row) and one scale per row
    const int P = N1 == 1024 ? N2 : N2 / TB;
    const long long pneed = (long long)std::min(rows, wrows) * P;
    GWB_CHECK_ARG(form != 4 || (rowscale && rowpart && rowpart_elems >= pneed), GWB_ERR_SHAPE,
                  "basis_fused: the fp8 form needs rowscale (rows floats) and rowpart (%lld floats)", pneed);
    cudaStream_t s = (cudaStream_t)stream;
    const float2* d = reinterpret_cast<const float2*>(Dp);
    const float2* t = reinterpret_cast<const float2*>(tw);
    float2* w = reinterpret_cast<float2*>(W);
    unsigned* tk = reinterpret_cast<unsigned*>(ticket);
    float* rp = form == 4 ? rowpart : nullptr;
    const int n = (int)N, ia0 = (int)a0, iTn = (int)Tn;
    // batches of wrows rows through the same W (W can then stay in L2 between the passes); the scale comes from the
    // first batch and every batch's pass 2 reads it (fp8: each batch's rows get their own scales between the passes)
    for (int j0 = 0; j0 < rows; j0 += wrows) {
        const int nr = std::min(wrows, rows - j0);
        const int nfb = j0 == 0 ? nf : 0;
        const float2* v = reinterpret_cast<const float2*>(Vp) + (long long)j0 * ldvp;
        int st;
        switch (N1) {
            case 64: st = launch_pass1<64>(v, ldvp, nr, d, n, N2, t, w, nfb, partials, tk, scale, rp, s); break;
            case 128: st = launch_pass1<128>(v, ldvp, nr, d, n, N2, t, w, nfb, partials, tk, scale, rp, s); break;
            case 256: st = launch_pass1<256>(v, ldvp, nr, d, n, N2, t, w, nfb, partials, tk, scale, rp, s); break;
            case 512: st = launch_pass1<512>(v, ldvp, nr, d, n, N2, t, w, nfb, partials, tk, scale, rp, s); break;
            default: st = launch_pass1_w(v, ldvp, nr, d, n, N2, t, w, nfb, partials, tk, scale, rp, s); break;
        }
        if (st) return st;
        const float* sc = scale;
        if (form == 4) {
            rowscale_kernel<<<nr, 256, 0, s>>>(rowpart, P, rowscale + j0);
            GWB_LAUNCH_CHECK("rowscale_kernel");
            sc = rowscale + j0;
        }
        const int r0 = row0 + j0;
        switch (N2) {
            case 64: st = launch_pass2<64>(form, w, n, N1, nr, t, ia0, iTn, sc, Z, Zlo, ldz, im_off, r0, s); break;
            case 128: st = launch_pass2<128>(form, w, n, N1, nr, t, ia0, iTn, sc, Z, Zlo, ldz, im_off, r0, s); break;
            case 256: st = launch_pass2<256>(form, w, n, N1, nr, t, ia0, iTn, sc, Z, Zlo, ldz, im_off, r0, s); break;
            case 512: st = launch_pass2<512>(form, w, n, N1, nr, t, ia0, iTn, sc, Z, Zlo, ldz, im_off, r0, s); break;
            default: st = launch_pass2<1024>(form, w, n, N1, nr, t, ia0, iTn, sc, Z, Zlo, ldz, im_off, r0, s); break;
        }
        if (st) return st;
    }
    return GWB_OK;
}

}  // extern "C"
