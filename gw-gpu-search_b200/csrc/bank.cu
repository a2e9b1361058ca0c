// Template-bank kernels: TaylorF2 templates, template norms sigma^2 (float64), the tile Gram matrix (float64) and the
// basis filters Vh of the tile SVD.
//
// sigma^2 (fp_filter.py:710-714): sig[i, s] = 4 df sum_k |H_ik|^2 IP_sk, here accumulated in float64 (the reference
//   uses a float32 GEMM). Split over k into partial sums reduced in a fixed order, so results do not depend on timing.
// Gram (fp_filter.py:578-581): G = sum_{k >= kmin} (H_k sw_k)(H_k sw_k)^H, complex, accumulated in float64 (the
//   reference accumulates in complex64). Only the upper block triangle is computed; the lower is its conjugate.
// Vh (fp_filter.py:589-591): Vh[j, k] = sum_i Bm[j, i] H[i, k] sw[k] for k >= kmin, zero below, fp32 accumulation.
// TaylorF2 (the synthetic bank's template family): h(f) = f^(-7/6) exp(-i (Psi(f) - pi/4)) on k df for k in
//   [kmin, kmax_i), phase in float64 to 3.5PN with aligned-spin spin-orbit (1.5PN) and spin-spin (2PN) terms and the
//   leading eccentric term, reduced to [-pi, pi] in float64 before a float32 sincos.
#include "common.cuh"
#include <mutex>

namespace gwb {
namespace {

constexpr int kK = 32;

// Scratch of gwb_sigma2_noalloc: the split-k partial sums of the template norms, at most kNoAllocPart doubles
// (4 MiB). It lives in the library's own device image, so every GPU that loads the library holds it until exit.
constexpr long long kNoAllocPart = 1ll << 19;
static __device__ __align__(256) double g_sigma2_scratch[kNoAllocPart];
std::mutex g_scratch_mu;
double* g_scratch_ptr[64] = {nullptr};

// Split-k partial sums of sig for a 64-row x 64-segment block: 256 threads, each a 4 x 4 register tile of float64
// accumulators; per 32-bin step the block's |H|^2 (float64, exact from complex64) and IP tiles go through shared
// memory (row stride 65 doubles: the transposing stores of 16 consecutive bins hit 16 distinct bank pairs), and the
// next step's H and IP are loaded into registers while the current one is multiplied.
constexpr int kSR = 64, kSS = 64, kSK = 32, kSP = kSK * kSR / 256;    // elements of each tile per thread
__global__ void __launch_bounds__(256) sigma2_partial_kernel(const float2* __restrict__ H, long long ldh, int n,
                                                             const float* __restrict__ IP, long long ldip, int nseg,
                                                             int kmin, int flen, int kper,
                                                             double* __restrict__ part) {
    __shared__ double Ps[kSK][kSR + 1];
    __shared__ double Is[kSK][kSS + 1];
    const int tid = threadIdx.x;
    const int tr = tid >> 4, ts = tid & 15;         // rows 4 tr .. 4 tr + 3, segments 4 ts .. 4 ts + 3
    const int r0 = blockIdx.x * kSR, s0 = blockIdx.y * kSS;
    const int ka = kmin + blockIdx.z * kper, kb = min(flen, ka + kper);
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    // thread's load slots: element e = tid + 256 i, (row or segment) = e / kSK, bin = e % kSK (32 consecutive bins
    // of one row per warp: coalesced)
    float2 hv[kSP];
    float iv[kSP];
    auto load = [&](int k0) {
#pragma unroll
        for (int i = 0; i < kSP; ++i) {
            const int e = tid + 256 * i, rr = e / kSK, kk = e % kSK;
            const int row = r0 + rr, sg = s0 + rr, k = k0 + kk;
            hv[i] = (row < n && k < kb) ? H[(long long)row * ldh + k] : make_float2(0.f, 0.f);
            iv[i] = (sg < nseg && k < kb) ? IP[(long long)sg * ldip + k] : 0.f;
        }
    };
    load(ka);
    for (int k0 = ka; k0 < kb; k0 += kSK) {
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kSP; ++i) {
            const int e = tid + 256 * i, rr = e / kSK, kk = e % kSK;
            Ps[kk][rr] = (double)hv[i].x * hv[i].x + (double)hv[i].y * hv[i].y;
            Is[kk][rr] = (double)iv[i];
        }
        __syncthreads();
        if (k0 + kSK < kb) load(k0 + kSK);
#pragma unroll 4
        for (int kk = 0; kk < kSK; ++kk) {
            double p[4], w[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) p[a] = Ps[kk][4 * tr + a];
#pragma unroll
            for (int b = 0; b < 4; ++b) w[b] = Is[kk][4 * ts + b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = fma(p[a], w[b], acc[a][b]);
        }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int row = r0 + 4 * tr + a, sg = s0 + 4 * ts + b;
            if (row < n && sg < nseg) part[((long long)blockIdx.z * n + row) * nseg + sg] = acc[a][b];
        }
}

__global__ void sigma2_reduce_kernel(const double* __restrict__ part, int nsplit, int n, int nseg, double scale,
                                     double* __restrict__ sig, long long ldsig) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n * nseg) return;
    double s = 0.0;
    for (int z = 0; z < nsplit; ++z) s += part[(long long)z * n * nseg + e];
    const long long row = e / nseg, sg = e % nseg;
    sig[row * ldsig + sg] = scale * s;
}

constexpr int kG = 32;   // Gram block: 32 x 32 outputs

__global__ void __launch_bounds__(256) gram_partial_kernel(const float2* __restrict__ H, long long ldh, int n,
                                                           const float* __restrict__ sw, int kmin, int flen, int kper,
                                                           double2* __restrict__ part) {
    const int bi = blockIdx.x, bj = blockIdx.y;
    if (bi > bj) return;   // upper block triangle only
    __shared__ double2 Ha[kK][kG];
    __shared__ double2 Hb[kK][kG];
    const int tid = threadIdx.x, ta = tid >> 4, tb = tid & 15;   // 16 x 16 threads, 2 x 2 outputs each
    const int a0 = bi * kG, b0 = bj * kG;
    const int ka = kmin + blockIdx.z * kper, kb = min(flen, ka + kper);
    double2 acc[2][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) acc[a][b] = make_double2(0.0, 0.0);
    for (int k0 = ka; k0 < kb; k0 += kK) {
        for (int e = tid; e < kK * kG; e += 256) {
            const int rr = e / kK, kk = e % kK, k = k0 + kk;
            double2 va = make_double2(0.0, 0.0), vb = make_double2(0.0, 0.0);
            if (k < kb) {
                const double w = (double)sw[k];
                if (a0 + rr < n) {
                    const float2 v = H[(long long)(a0 + rr) * ldh + k];
                    va = make_double2(v.x * w, v.y * w);
                }
                if (b0 + rr < n) {
                    const float2 v = H[(long long)(b0 + rr) * ldh + k];
                    vb = make_double2(v.x * w, v.y * w);
                }
            }
            Ha[kk][rr] = va;
            Hb[kk][rr] = vb;
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < kK; ++kk) {
            const double2 x0 = Ha[kk][2 * ta], x1 = Ha[kk][2 * ta + 1];
            const double2 y0 = Hb[kk][2 * tb], y1 = Hb[kk][2 * tb + 1];
            // x conj(y)
            acc[0][0].x = fma(x0.x, y0.x, fma(x0.y, y0.y, acc[0][0].x));
            acc[0][0].y = fma(x0.y, y0.x, fma(-x0.x, y0.y, acc[0][0].y));
            acc[0][1].x = fma(x0.x, y1.x, fma(x0.y, y1.y, acc[0][1].x));
            acc[0][1].y = fma(x0.y, y1.x, fma(-x0.x, y1.y, acc[0][1].y));
            acc[1][0].x = fma(x1.x, y0.x, fma(x1.y, y0.y, acc[1][0].x));
            acc[1][0].y = fma(x1.y, y0.x, fma(-x1.x, y0.y, acc[1][0].y));
            acc[1][1].x = fma(x1.x, y1.x, fma(x1.y, y1.y, acc[1][1].x));
            acc[1][1].y = fma(x1.y, y1.x, fma(-x1.x, y1.y, acc[1][1].y));
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int i = a0 + 2 * ta + a, j = b0 + 2 * tb + b;
            if (i < n && j < n) part[((long long)blockIdx.z * n + i) * n + j] = acc[a][b];
        }
}

__global__ void gram_reduce_kernel(const double2* __restrict__ part, int nsplit, int n, double2* __restrict__ G) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n * n) return;
    const int i = (int)(e / n), j = (int)(e % n);
    const int bi = i / kG, bj = j / kG;
    // blocks below the diagonal were not computed: take the conjugate of the mirrored element
    const long long src = (bi <= bj) ? e : ((long long)j * n + i);
    double x = 0.0, y = 0.0;
    for (int z = 0; z < nsplit; ++z) {
        const double2 v = part[(long long)z * n * n + src];
        x += v.x;
        y += v.y;
    }
    G[e] = (bi <= bj) ? make_double2(x, y) : make_double2(x, -y);
}

template <int RMAX>
__global__ void __launch_bounds__(256) vh_kernel(const float2* __restrict__ Bm, long long ldb, int r, int n,
                                                 const float2* __restrict__ H, long long ldh,
                                                 const float* __restrict__ sw, int kmin, int flen,
                                                 float2* __restrict__ Vh, long long ldv) {
    __shared__ float2 sB[RMAX][64];
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float2 acc[RMAX];
#pragma unroll
    for (int j = 0; j < RMAX; ++j) acc[j] = make_float2(0.f, 0.f);
    const bool live = k >= kmin && k < flen;
    const float w = live ? sw[k] : 0.f;
    for (int i0 = 0; i0 < n; i0 += 64) {
        for (int e = threadIdx.x; e < RMAX * 64; e += blockDim.x) {
            const int j = e / 64, i = e % 64;
            sB[j][i] = (j < r && i0 + i < n) ? Bm[(long long)j * ldb + i0 + i] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        if (live) {
            const int iend = min(64, n - i0);
            for (int i = 0; i < iend; ++i) {
                const float2 hv = H[(long long)(i0 + i) * ldh + k];
                const float hx = hv.x * w, hy = hv.y * w;     // H sw, rounded as the reference's complex64 product
#pragma unroll
                for (int j = 0; j < RMAX; ++j) {
                    const float2 b = sB[j][i];
                    acc[j].x = fmaf(b.x, hx, fmaf(-b.y, hy, acc[j].x));
                    acc[j].y = fmaf(b.x, hy, fmaf(b.y, hx, acc[j].y));
                }
            }
        }
        __syncthreads();
    }
    if (k < flen) {
#pragma unroll
        for (int j = 0; j < RMAX; ++j)
            if (j < r) Vh[(long long)j * ldv + k] = live ? acc[j] : make_float2(0.f, 0.f);
    }
}

__global__ void taylorf2_kernel(const double* __restrict__ m1, const double* __restrict__ m2,
                                const double* __restrict__ chi1, const double* __restrict__ chi2,
                                const double* __restrict__ e0, const int32_t* __restrict__ kmax, int n, double df,
                                int kmin, int flen, double f_ecc, float2* __restrict__ H, long long ldh) {
    const int i = blockIdx.y;
    if (i >= n) return;
    const double pi = 3.141592653589793;
    const double M = m1[i] + m2[i];
    const double eta = m1[i] * m2[i] / (M * M);
    const double Ms = M * 4.925490947641267e-06;
    const double d1 = m1[i] / M, d2 = m2[i] / M;
    const double c1 = chi1[i], c2 = chi2[i], ec = e0[i];
    const double beta = (113.0 / 12.0) * (d1 * d1 * c1 + d2 * d2 * c2) + 6.25 * eta * (c1 + c2);
    const double sigma = eta * (474.0 / 48.0) * c1 * c2;
    const double p2 = 20.0 / 9.0 * (743.0 / 336.0 + 11.0 / 4.0 * eta);
    const double p3 = -16.0 * pi + 4.0 * beta;
    const double p4 = 10.0 * (3058673.0 / 7257600.0 + 5429.0 / 1008.0 * eta + 617.0 / 144.0 * eta * eta) - 10.0 * sigma;
    const double p5c = pi * (38645.0 / 756.0 - 65.0 / 9.0 * eta);
    const double p6c = 11583231236531.0 / 4694215680.0 - 640.0 / 3.0 * pi * pi - 6848.0 / 21.0 * 0.5772156649015329 +
                       eta * (-15737765635.0 / 3048192.0 + 2255.0 / 12.0 * pi * pi) + 76055.0 / 1728.0 * eta * eta -
                       127825.0 / 1296.0 * eta * eta * eta;
    const double p7 = pi * (77096675.0 / 254016.0 + 378515.0 / 1512.0 * eta - 74045.0 / 756.0 * eta * eta);
    const double v_isco = 0.4082482904638631;   // 1 / sqrt(6)
    const double v0 = cbrt(pi * Ms * f_ecc);
    const double pre = 3.0 / (128.0 * eta);
    const int k1 = kmax[i];
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < flen; k += (long long)gridDim.x * blockDim.x) {
        float2 out = make_float2(0.f, 0.f);
        if (k >= kmin && k < k1) {
            const double f = (double)k * df;
            const double v = cbrt(pi * Ms * f);
            const double lv = log(v);
            const double p5 = p5c * (1.0 + 3.0 * (lv - log(v_isco)));
            const double p6 = p6c - 6848.0 / 21.0 * (lv + log(4.0));
            double series = 1.0 + v * v * (p2 + v * (p3 + v * (p4 + v * (p5 + v * (p6 + v * p7)))));
            if (ec != 0.0) series -= 2355.0 / 1462.0 * ec * ec * pow(v0 / v, 19.0 / 3.0);
            const double v5 = v * v * v * v * v;
            double psi = pre / v5 * series - 0.25 * pi;
            psi -= 2.0 * pi * rint(psi * (0.5 / pi));
            const float amp = (float)pow(f, -7.0 / 6.0);
            float sn, cs;
            sincosf((float)psi, &sn, &cs);
            out = make_float2(amp * cs, -amp * sn);   // exp(-i psi)
        }
        H[(long long)i * ldh + k] = out;
    }
}

}  // namespace
}  // namespace gwb

extern "C" {

int gwb_sigma2(const float* H, long long ldh, int n, const float* IP, long long ldip, int nseg, int kmin, int flen,
               double df, double* part, long long part_elems, double* sig, long long ldsig, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(H && IP && part && sig, GWB_ERR_ARG, "sigma2: null pointer");
    GWB_CHECK_ARG(n > 0 && nseg > 0 && flen > kmin && kmin >= 0 && ldsig >= nseg, GWB_ERR_SHAPE,
                  "sigma2: n=%d nseg=%d flen=%d kmin=%d", n, nseg, flen, kmin);
    const int gx = (int)cdiv(n, kSR), gy = (int)cdiv(nseg, kSS);
    int nsplit = (int)std::max(1ll, std::min<long long>(64, (4ll * num_sms()) / std::max(1, gx * gy)));
    nsplit = (int)std::min<long long>(nsplit, part_elems / ((long long)n * nseg));
    GWB_CHECK_ARG(nsplit >= 1, GWB_ERR_SHAPE, "sigma2: workspace of %lld doubles is smaller than n*nseg", part_elems);
    const int kper = (int)(cdiv(cdiv(flen - kmin, nsplit), kSK) * kSK);
    nsplit = (int)cdiv(flen - kmin, kper);
    cudaStream_t s = (cudaStream_t)stream;
    sigma2_partial_kernel<<<dim3(gx, gy, nsplit), 256, 0, s>>>(reinterpret_cast<const float2*>(H), ldh, n, IP, ldip, nseg,
                                                                kmin, flen, kper, part);
    GWB_LAUNCH_CHECK("sigma2_partial_kernel");
    const long long ne = (long long)n * nseg;
    sigma2_reduce_kernel<<<(unsigned)cdiv(ne, 256), 256, 0, s>>>(part, nsplit, n, nseg, 4.0 * df, sig, ldsig);
    GWB_LAUNCH_CHECK("sigma2_reduce_kernel");
    return GWB_OK;
}

int gwb_sigma2_noalloc(const float* H, long long ldh, int n, const float* IP, long long ldip, int nseg, int kmin,
                       int flen, double df, double* sig, long long ldsig, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(n > 0 && nseg > 0, GWB_ERR_SHAPE, "sigma2_noalloc: n=%d nseg=%d", n, nseg);
    GWB_CHECK_ARG((long long)n * nseg <= kNoAllocPart, GWB_ERR_CAPACITY,
                  "sigma2_noalloc: n * nseg = %lld exceeds the static scratch of %lld partial sums; call gwb_sigma2 "
                  "with a workspace, or split the rows", (long long)n * nseg, kNoAllocPart);
    int dev = 0;
    GWB_CUDA(cudaGetDevice(&dev));
    GWB_CHECK_ARG(dev >= 0 && dev < 64, GWB_ERR_ARG, "sigma2_noalloc: device %d", dev);
    double* part = nullptr;
    {
        // once per device, with that device current: the device address of the static array (the host-side
        // symbol is only a stand-in and must never be handed to a kernel)
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        if (g_scratch_ptr[dev] == nullptr) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_sigma2_scratch);
            if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_sigma2_scratch)");
            g_scratch_ptr[dev] = static_cast<double*>(p);
        }
        part = g_scratch_ptr[dev];
    }
    // every partial the reduction reads is written by the partial kernel first: nothing needs clearing
    return gwb_sigma2(H, ldh, n, IP, ldip, nseg, kmin, flen, df, part, kNoAllocPart, sig, ldsig, stream);
}

int gwb_gram(const float* H, long long ldh, int n, const float* sw, int kmin, int flen, double* part,
             long long part_elems, double* G, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(H && sw && part && G, GWB_ERR_ARG, "gram: null pointer");
    GWB_CHECK_ARG(n > 0 && flen > kmin && kmin >= 0, GWB_ERR_SHAPE, "gram: n=%d flen=%d kmin=%d", n, flen, kmin);
    const int nb = (int)cdiv(n, kG);
    int nsplit = (int)std::max(1ll, std::min<long long>(128, (4ll * num_sms()) / std::max(1, nb * (nb + 1) / 2)));
    nsplit = (int)std::min<long long>(nsplit, part_elems / (2ll * n * n));
    GWB_CHECK_ARG(nsplit >= 1, GWB_ERR_SHAPE, "gram: workspace of %lld doubles is smaller than 2 n^2", part_elems);
    const int kper = (int)(cdiv(cdiv(flen - kmin, nsplit), kK) * kK);
    nsplit = (int)cdiv(flen - kmin, kper);
    cudaStream_t s = (cudaStream_t)stream;
    gram_partial_kernel<<<dim3(nb, nb, nsplit), 256, 0, s>>>(reinterpret_cast<const float2*>(H), ldh, n, sw, kmin, flen,
                                                             kper, reinterpret_cast<double2*>(part));
    GWB_LAUNCH_CHECK("gram_partial_kernel");
    gram_reduce_kernel<<<(unsigned)cdiv((long long)n * n, 256), 256, 0, s>>>(reinterpret_cast<const double2*>(part),
                                                                             nsplit, n, reinterpret_cast<double2*>(G));
    GWB_LAUNCH_CHECK("gram_reduce_kernel");
    return GWB_OK;
}

int gwb_basis_vh(const float* Bm, long long ldb, int r, int n, const float* H, long long ldh, const float* sw, int kmin,
                 int flen, float* Vh, long long ldv, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(Bm && H && sw && Vh, GWB_ERR_ARG, "basis_vh: null pointer");
    GWB_CHECK_ARG(r > 0 && n > 0 && flen > kmin && ldb >= n && ldv >= flen, GWB_ERR_SHAPE, "basis_vh: r=%d n=%d", r, n);
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned gx = (unsigned)cdiv(flen, 256);
    for (int j0 = 0; j0 < r; j0 += 32) {
        const int rr = std::min(32, r - j0);
        const float2* b = reinterpret_cast<const float2*>(Bm) + (long long)j0 * ldb;
        float2* v = reinterpret_cast<float2*>(Vh) + (long long)j0 * ldv;
        if (rr <= 16)
            vh_kernel<16><<<gx, 256, 0, s>>>(b, ldb, rr, n, reinterpret_cast<const float2*>(H), ldh, sw, kmin, flen, v, ldv);
        else
            vh_kernel<32><<<gx, 256, 0, s>>>(b, ldb, rr, n, reinterpret_cast<const float2*>(H), ldh, sw, kmin, flen, v, ldv);
        GWB_LAUNCH_CHECK("vh_kernel");
    }
    return GWB_OK;
}

int gwb_taylorf2(const double* m1, const double* m2, const double* chi1, const double* chi2, const double* e0,
                 const int32_t* kmax, int n, double df, int kmin, int flen, double f_ecc, float* H, long long ldh,
                 void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(m1 && m2 && chi1 && chi2 && e0 && kmax && H, GWB_ERR_ARG, "taylorf2: null pointer");
    GWB_CHECK_ARG(n > 0 && n < 65536 && flen > kmin && kmin > 0 && ldh >= flen && df > 0, GWB_ERR_SHAPE,
                  "taylorf2: n=%d flen=%d kmin=%d", n, flen, kmin);
    dim3 grid((unsigned)std::min<long long>(cdiv(flen, 256), 256), n);
    taylorf2_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(m1, m2, chi1, chi2, e0, kmax, n, df, kmin, flen, f_ecc,
                                                            reinterpret_cast<float2*>(H), ldh);
    GWB_LAUNCH_CHECK("taylorf2_kernel");
    return GWB_OK;
}

}  // extern "C"
