// Differentiation of the matched filter with respect to the template parameters (the north star's adjoint form; the
// reference has no gradients: its template placement maximises the match numerically, ecc_bank_place.py:79-89).
//
// Parameters per trigger, theta = (Mc [M_sun], q = m2/m1 <= 1, chi1z, chi2z, e0 at f_ecc, t_c [s], phi_c). The
// template is the library's TaylorF2 (the phase of taylorf2_kernel: 3.5PN non-spinning, 1.5PN spin-orbit, 2PN
// spin-spin, leading eccentric term), h_k = f^-7/6 exp(-i Phi_k) on kmin <= k < kmax (kmax = the ISCO bin, as the
// bank's templates), Phi = Psi(f) - pi/4 + 2 pi f t_c - phi_c.
//   z = 4 df sum_k conj(h_k) D_k,  sigma^2 = 4 df sum_k |h_k|^2 IP_k,  snr = |z| / sigma
//   chisq = (nb sum_j |z_j|^2 - |z|^2) / sigma^2 over nb equal-power bins (z_j the bin's part of z, edges from the
//   cumulative |h|^2 IP as the pipeline's, held fixed), dof = 2 nb - 2, newsnr (coinc_rank.py:39-46).
// |h_k| does not depend on theta (inside [kmin, kmax)), so d sigma = 0 and dz/dtheta_i = 4 df sum_k i dPhi_k/dtheta_i
// conj(h_k) D_k. dPsi/d(Mc, q, chi1, chi2, e0) comes from forward-mode dual numbers through the phase formula in
// float64; dPhi/dt_c = 2 pi f, dPhi/dphi_c = -1. The edges are found in the kernel (block scan of |h|^2 IP).
// One CTA per trigger; each thread takes a contiguous range of bins, so a thread's bin changes a few times only and
// its per-bin partial sums go to shared memory once per change.
//
// The phase metric (the quadratic form of the phase-maximised match, 1 - m ~ dtheta^T g dtheta / 2): with |h|
// independent of theta, g_ij = Cov_w(dPhi/dtheta_i, dPhi/dtheta_j), w_k = |h_k|^2 IP_k; the phi_c row is zero.
#include "common.cuh"

namespace gwb {
namespace {

constexpr int kNP = 7;          // parameters
constexpr int kNI = 5;          // intrinsic ones (through the phase formula)
constexpr int kThreads = 256;
constexpr int kMaxBins = 32;
constexpr double kPi = 3.141592653589793;
constexpr double kMsun = 4.925490947641267e-06;    // G M_sun / c^3 in seconds
constexpr double kEuler = 0.5772156649015329;

// forward-mode dual number: value and its derivatives with respect to the kNI intrinsic parameters
struct Dual {
    double v, d[kNI];
};
__device__ __forceinline__ Dual dc(double a) {
    Dual r;
    r.v = a;
#pragma unroll
    for (int i = 0; i < kNI; ++i) r.d[i] = 0.0;
    return r;
}
__device__ __forceinline__ Dual operator+(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < kNI; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
__device__ __forceinline__ Dual operator-(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < kNI; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
__device__ __forceinline__ Dual operator*(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < kNI; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
__device__ __forceinline__ Dual operator*(double s, const Dual& a) {
    Dual r;
    r.v = s * a.v;
#pragma unroll
    for (int i = 0; i < kNI; ++i) r.d[i] = s * a.d[i];
    return r;
}
__device__ __forceinline__ Dual operator+(double s, const Dual& a) {
    Dual r = a;
    r.v += s;
    return r;
}
__device__ __forceinline__ Dual operator/(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int i = 0; i < kNI; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
// a^p for a constant exponent p (a > 0)
__device__ __forceinline__ Dual dpow(const Dual& a, double p) {
    Dual r;
    r.v = pow(a.v, p);
    const double g = p * r.v / a.v;
#pragma unroll
    for (int i = 0; i < kNI; ++i) r.d[i] = g * a.d[i];
    return r;
}
__device__ __forceinline__ Dual dlog(const Dual& a) {
    Dual r;
    r.v = log(a.v);
    const double g = 1.0 / a.v;
#pragma unroll
    for (int i = 0; i < kNI; ++i) r.d[i] = g * a.d[i];
    return r;
}

// per-trigger quantities of the phase, as functions of (Mc, q, chi1, chi2, e0)
struct PhaseCoef {
    Dual lms;        // log(pi Ms) (v = exp((log(pi Ms) + log f) / 3))
    Dual pre, p2, p3, p4, p5c, p6c, p7, ecc;   // ecc = -2355/1462 e0^2 v0^(19/3)
    double Ms;
};

__device__ PhaseCoef phase_coef(const double* th, double f_ecc) {
    Dual Mc = dc(th[0]), q = dc(th[1]), c1 = dc(th[2]), c2 = dc(th[3]), e0 = dc(th[4]);
    Mc.d[0] = 1.0;
    q.d[1] = 1.0;
    c1.d[2] = 1.0;
    c2.d[3] = 1.0;
    e0.d[4] = 1.0;
    const Dual one_q = 1.0 + q;
    const Dual eta = q / (one_q * one_q);
    const Dual M = Mc * dpow(eta, -0.6);
    const Dual d1 = dc(1.0) / one_q, d2 = q / one_q;
    const Dual beta = (113.0 / 12.0) * (d1 * d1 * c1 + d2 * d2 * c2) + 6.25 * (eta * (c1 + c2));
    const Dual sigma = (474.0 / 48.0) * (eta * c1 * c2);
    PhaseCoef P;
    const Dual Ms = kMsun * M;
    P.Ms = Ms.v;
    P.lms = dlog(kPi * Ms);
    P.pre = dc(3.0 / 128.0) / eta;
    P.p2 = (20.0 / 9.0) * (743.0 / 336.0 + (11.0 / 4.0) * eta);
    P.p3 = -16.0 * kPi + 4.0 * beta;
    P.p4 = 10.0 * (3058673.0 / 7257600.0 + ((5429.0 / 1008.0) * eta + (617.0 / 144.0) * (eta * eta))) - 10.0 * sigma;
    P.p5c = kPi * (38645.0 / 756.0 + (-65.0 / 9.0) * eta);
    P.p6c = (11583231236531.0 / 4694215680.0 - 640.0 / 3.0 * kPi * kPi - 6848.0 / 21.0 * kEuler) +
            ((-15737765635.0 / 3048192.0 + 2255.0 / 12.0 * kPi * kPi) * eta + (76055.0 / 1728.0) * (eta * eta) +
             (-127825.0 / 1296.0) * (eta * eta * eta));
    P.p7 = kPi * (77096675.0 / 254016.0 + ((378515.0 / 1512.0) * eta + (-74045.0 / 756.0) * (eta * eta)));
    const Dual v0 = dpow(kPi * f_ecc * Ms, 1.0 / 3.0);
    P.ecc = (-2355.0 / 1462.0) * (e0 * e0 * dpow(v0, 19.0 / 3.0));
    return P;
}

// Psi(f) and its derivatives with respect to the intrinsic parameters
__device__ __forceinline__ Dual psi_at(const PhaseCoef& P, double f) {
    const double lf = log(f);
    Dual lv = (1.0 / 3.0) * (P.lms + dc(lf));
    Dual v;
    v.v = exp(lv.v);
#pragma unroll
    for (int i = 0; i < kNI; ++i) v.d[i] = v.v * lv.d[i];
    const Dual p5 = P.p5c * (1.0 + 3.0 * (lv - dc(log(0.4082482904638631))));
    const Dual p6 = P.p6c - (6848.0 / 21.0) * (lv + dc(log(4.0)));
    // Horner: 1 + v^2 (p2 + v (p3 + v (p4 + v (p5 + v (p6 + v p7)))))
    Dual series = p6 + v * P.p7;
    series = p5 + v * series;
    series = P.p4 + v * series;
    series = P.p3 + v * series;
    series = P.p2 + v * series;
    series = 1.0 + (v * v) * series;
    // eccentric term: ecc v^(-19/3)
    Dual vm193;
    vm193.v = exp((-19.0 / 3.0) * lv.v);
#pragma unroll
    for (int i = 0; i < kNI; ++i) vm193.d[i] = vm193.v * (-19.0 / 3.0) * lv.d[i];
    series = series + P.ecc * vm193;
    Dual vm5;
    vm5.v = exp(-5.0 * lv.v);
#pragma unroll
    for (int i = 0; i < kNI; ++i) vm5.d[i] = vm5.v * (-5.0) * lv.d[i];
    return P.pre * vm5 * series;
}

__device__ __forceinline__ int kmax_of(double Ms, double df, int flen) {
    const double fisco = 1.0 / (14.696938456699067 * kPi * Ms);     // 6^1.5 pi Ms
    return (int)min((long long)floor(fisco / df) + 1, (long long)flen - 1);
}

// Equal-power edges of w_k = f^-7/3 IP_k over [kmin, k1): edge j = first k whose inclusive cumulative sum exceeds
// (j / nb) total (the pipeline's edges, offset mode 0). Threads take contiguous ranges; float64 sums, block scan.
__device__ void block_edges(const float* __restrict__ ip, double df, int kmin, int k1, int nb, int* e, double* tot_out,
                            double* scan) {
    const int tid = threadIdx.x;
    const int len = k1 - kmin, chunk = (len + kThreads - 1) / kThreads;
    const int a = kmin + tid * chunk, b = min(a + chunk, k1);
    double s = 0.0;
    for (int k = a; k < b; ++k) s += pow((double)k * df, -7.0 / 3.0) * (double)ip[k];
    scan[tid] = s;
    __syncthreads();
    if (tid == 0) {
        double acc = 0.0;
        for (int t = 0; t < kThreads; ++t) {
            const double x = scan[t];
            scan[t] = acc;          // exclusive prefix
            acc += x;
        }
        scan[kThreads] = acc;
        e[0] = kmin;
        e[nb] = k1;
    }
    __syncthreads();
    const double tot = scan[kThreads], ex = scan[tid];
    for (int j = 1; j < nb; ++j) {
        const double target = (double)j / (double)nb * tot;
        if (ex <= target && target < ex + s) {
            double c = ex;
            for (int k = a; k < b; ++k) {
                c += pow((double)k * df, -7.0 / 3.0) * (double)ip[k];
                if (c > target) {
                    e[j] = k;
                    break;
                }
            }
        }
    }
    if (tid == 0) *tot_out = tot;
    __syncthreads();
}

// out row layout (doubles): snr, newsnr, chisq, sigma2, z_re, z_im, kmax, dsnr[7], dnewsnr[7], dchisq[7]
constexpr int kOut = 7 + 3 * kNP;

template <typename T>
__global__ void __launch_bounds__(kThreads) snr_grad_kernel(const double* __restrict__ params, int n,
                                                          const float2* __restrict__ D, long long ldd,
                                                          const float* __restrict__ IP, long long ldip, int flen,
                                                          double df, int kmin, double f_ecc, int nb,
                                                          double* __restrict__ out, long long ldout) {
    const int i = blockIdx.x;
    if (i >= n) return;
    __shared__ double scan[kThreads + 1];
    __shared__ int e[kMaxBins + 1];
    __shared__ double tot;
    __shared__ double acc[kMaxBins][2 + 2 * kNP];      // per bin: z_j (re, im), dz_j (re, im) x 7
    __shared__ double red[kThreads / 32][2 + 2 * kNP];
    const double* th = params + (long long)i * kNP;
    const PhaseCoef P = phase_coef(th, f_ecc);
    const double tc = th[5], phic = th[6];
    const int k1 = kmax_of(P.Ms, df, flen);
    if (k1 <= kmin + kThreads) {           // no band above kmin (f_ISCO below the low cut): nothing to filter
        if (threadIdx.x < kOut) out[(long long)i * ldout + threadIdx.x] = 0.0;
        return;
    }
    const float* ip = IP + (long long)i * ldip;
    const float2* d = D + (long long)i * ldd;
    block_edges(ip, df, kmin, k1, nb, e, &tot, scan);
    // main pass, bin by bin: threads stride over the bin's range (coalesced D and IP), then a fixed-order block
    // reduction (warp shuffles, then the warps in order) gives the bin's sums: the result does not depend on timing
    constexpr int kNS = 2 + 2 * kNP;
    for (int j = 0; j < nb; ++j) {
        T s[kNS];
#pragma unroll
        for (int x = 0; x < kNS; ++x) s[x] = T(0);
        for (int k = e[j] + threadIdx.x; k < e[j + 1]; k += kThreads) {
            const double f = (double)k * df;
            const Dual ps = psi_at(P, f);
            double ph = ps.v - 0.25 * kPi + 2.0 * kPi * f * tc - phic;
            ph -= 2.0 * kPi * rint(ph * (0.5 / kPi));
            T sn, cs;
            if constexpr (sizeof(T) == 8) {
                sincos(ph, &sn, &cs);
            } else {
                sincosf((float)ph, &sn, &cs);
            }
            const T amp = (T)pow(f, -7.0 / 6.0);
            const float2 dk = d[k];
            // q = conj(h) D = amp e^{+i ph} D
            const T hr = amp * cs, hi = amp * sn;
            const T qr = hr * (T)dk.x - hi * (T)dk.y, qi = hr * (T)dk.y + hi * (T)dk.x;
            s[0] += qr;
            s[1] += qi;
            // d q / d theta_p = i dPhi_p q
            T dph[kNP];
#pragma unroll
            for (int p = 0; p < kNI; ++p) dph[p] = (T)ps.d[p];
            dph[5] = (T)(2.0 * kPi * f);
            dph[6] = T(-1);
#pragma unroll
            for (int p = 0; p < kNP; ++p) {
                s[2 + 2 * p] -= dph[p] * qi;
                s[3 + 2 * p] += dph[p] * qr;
            }
        }
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int x = 0; x < kNS; ++x) {
            double v = (double)s[x];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0) red[warp][x] = v;
        }
        __syncthreads();
        if (threadIdx.x < kNS) {
            double v = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) v += red[w][threadIdx.x];
            acc[j][threadIdx.x] = v;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double c4 = 4.0 * df;
        const double sig2 = c4 * tot;
        double zr = 0.0, zi = 0.0, dzr[kNP] = {0}, dzi[kNP] = {0}, pw = 0.0, dpw[kNP] = {0};
        for (int j = 0; j < nb; ++j) {
            const double ar = c4 * acc[j][0], ai = c4 * acc[j][1];
            zr += ar;
            zi += ai;
            pw += ar * ar + ai * ai;
            for (int p = 0; p < kNP; ++p) {
                const double br = c4 * acc[j][2 + 2 * p], bi = c4 * acc[j][3 + 2 * p];
                dzr[p] += br;
                dzi[p] += bi;
                dpw[p] += 2.0 * (ar * br + ai * bi);
            }
        }
        const double az = sqrt(zr * zr + zi * zi), sg = sqrt(sig2);
        const double snr = az / sg;
        const double chisq = ((double)nb * pw - az * az) / sig2;
        const int dof = 2 * nb - 2;
        const double rc = chisq / (double)dof;
        double ns = snr, g = 1.0, gp = 0.0;
        if (rc > 1.0) {
            const double base = (1.0 + rc * rc * rc) / 2.0;
            g = pow(base, -1.0 / 6.0);
            gp = -1.0 / 6.0 * pow(base, -7.0 / 6.0) * 1.5 * rc * rc;   // d g / d rc
            ns = snr * g;
        }
        double* o = out + (long long)i * ldout;
        o[0] = snr;
        o[1] = ns;
        o[2] = chisq;
        o[3] = sig2;
        o[4] = zr;
        o[5] = zi;
        o[6] = (double)k1;
        for (int p = 0; p < kNP; ++p) {
            const double dabs = az > 0.0 ? (zr * dzr[p] + zi * dzi[p]) / az : 0.0;
            const double dsnr = dabs / sg;
            const double dchi = ((double)nb * dpw[p] - 2.0 * az * dabs) / sig2;
            o[7 + p] = dsnr;
            o[7 + kNP + p] = dsnr * g + snr * gp * dchi / (double)dof;
            o[7 + 2 * kNP + p] = dchi;
        }
    }
}

// phase metric g (n x 7 x 7): weighted covariance of dPhi/dtheta with weights |h|^2 IP over [kmin, kmax)
__global__ void __launch_bounds__(kThreads) phase_metric_kernel(const double* __restrict__ params, int n,
                                                              const float* __restrict__ IP, long long ldip, int flen,
                                                              double df, int kmin, double f_ecc,
                                                              double* __restrict__ g) {
    const int i = blockIdx.x;
    if (i >= n) return;
    constexpr int NS = 1 + kNP + kNP * (kNP + 1) / 2;
    __shared__ double red[kThreads / 32][NS];
    const double* th = params + (long long)i * kNP;
    const PhaseCoef P = phase_coef(th, f_ecc);
    const int k1 = kmax_of(P.Ms, df, flen);
    if (k1 <= kmin + kThreads) {
        if (threadIdx.x < kNP * kNP) g[(long long)i * kNP * kNP + threadIdx.x] = 0.0;
        return;
    }
    const float* ip = IP + (long long)i * ldip;
    double s[NS];
#pragma unroll
    for (int x = 0; x < NS; ++x) s[x] = 0.0;
    for (int k = kmin + threadIdx.x; k < k1; k += kThreads) {
        const double f = (double)k * df;
        const double w = pow(f, -7.0 / 3.0) * (double)ip[k];
        const Dual ps = psi_at(P, f);
        double dph[kNP];
#pragma unroll
        for (int p = 0; p < kNI; ++p) dph[p] = ps.d[p];
        dph[5] = 2.0 * kPi * f;
        dph[6] = -1.0;
        s[0] += w;
        int c = 1 + kNP;
#pragma unroll
        for (int p = 0; p < kNP; ++p) {
            s[1 + p] += w * dph[p];
#pragma unroll
            for (int q = p; q < kNP; ++q) s[c++] += w * dph[p] * dph[q];
        }
    }
    // fixed-order reduction: warps by shuffles, then warps in order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int x = 0; x < NS; ++x) {
        double v = s[x];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[warp][x] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[NS];
        for (int x = 0; x < NS; ++x) {
            t[x] = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) t[x] += red[w][x];
        }
        double* gi = g + (long long)i * kNP * kNP;
        int c = 1 + kNP;
        for (int p = 0; p < kNP; ++p)
            for (int q = p; q < kNP; ++q) {
                const double v = t[c++] / t[0] - (t[1 + p] / t[0]) * (t[1 + q] / t[0]);
                gi[p * kNP + q] = v;
                gi[q * kNP + p] = v;
            }
    }
}

// One Levenberg-Marquardt step of the SNR ascent per trigger, in the 6 parameters other than phi_c (|z| does not
// depend on it): near the maximum snr(theta + d) ~ snr(theta) (1 - d^T g d / 2) + grad . d, so the Newton step is
// g^-1 grad / snr; g's eigenvalues span many decades (the Mc - q - chi degeneracy) and the quadratic model fails far
// along the flat directions, so the step is d = (g + lam_i diag g)^-1 grad / snr with the caller adapting lam_i per
// trigger (down after a step that raised the SNR, up after one that did not). Then clamped to the physical ranges
// (Mc > 0, q in [0.05, 1], |chi| <= 0.99, e0 in [0, 0.5]). Cholesky in float64.
__global__ void refine_step_kernel(const double* __restrict__ params, const double* __restrict__ res, long long ldres,
                                   const double* __restrict__ g, const double* __restrict__ lam, int n,
                                   double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    constexpr int m = 6;
    const double* gi = g + (long long)i * kNP * kNP;
    const double* ri = res + (long long)i * ldres;
    double A[m][m], b[m];
    const double snr = ri[0];
    double dmax = 0.0;
    for (int p = 0; p < m; ++p) dmax = fmax(dmax, gi[p * kNP + p]);
    for (int p = 0; p < m; ++p) {
        for (int q = 0; q < m; ++q) A[p][q] = gi[p * kNP + q];
        A[p][p] *= 1.0 + lam[i];
        b[p] = snr > 0.0 ? ri[7 + p] / snr : 0.0;      // dsnr / snr
    }
    // a parameter the phase does not depend on here (e0 at 0: the phase goes with e0^2) has a zero row: it takes no
    // step (its gradient is zero too) and leaves the others' system positive definite
    for (int p = 0; p < m; ++p)
        if (!(gi[p * kNP + p] > 1e-24 * dmax)) {
            for (int q = 0; q < m; ++q) A[p][q] = A[q][p] = 0.0;
            A[p][p] = dmax > 0.0 ? dmax : 1.0;
            b[p] = 0.0;
        }
    bool ok = snr > 0.0;
    for (int p = 0; p < m && ok; ++p) {                 // A = L L^T in place (lower)
        for (int q = 0; q <= p; ++q) {
            double s = A[p][q];
            for (int r = 0; r < q; ++r) s -= A[p][r] * A[q][r];
            if (p == q) {
                if (s <= 0.0) {
                    ok = false;
                    break;
                }
                A[p][p] = sqrt(s);
            } else {
                A[p][q] = s / A[q][q];
            }
        }
    }
    double d[m] = {0, 0, 0, 0, 0, 0};
    if (ok) {
        double y[m];
        for (int p = 0; p < m; ++p) {
            double s = b[p];
            for (int r = 0; r < p; ++r) s -= A[p][r] * y[r];
            y[p] = s / A[p][p];
        }
        for (int p = m - 1; p >= 0; --p) {
            double s = y[p];
            for (int r = p + 1; r < m; ++r) s -= A[r][p] * d[r];
            d[p] = s / A[p][p];
        }
    }
    const double* th = params + (long long)i * kNP;
    double* o = out + (long long)i * kNP;
    for (int p = 0; p < kNP; ++p) o[p] = th[p] + (p < m ? d[p] : 0.0);
    o[0] = fmax(o[0], 0.05 * th[0]);
    o[1] = fmin(fmax(o[1], 0.05), 1.0);
    o[2] = fmin(fmax(o[2], -0.99), 0.99);
    o[3] = fmin(fmax(o[3], -0.99), 0.99);
    o[4] = fmin(fmax(o[4], 0.0), 0.5);
}

}  // namespace
}  // namespace gwb

extern "C" {

int gwb_snr_grad(const double* params, int n, const float* D, long long ldd, const float* IP, long long ldip, int flen,
                 double df, int kmin, double f_ecc, int nbins, int fp64, double* out, long long ldout, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(params && D && IP && out, GWB_ERR_ARG, "snr_grad: null pointer");
    GWB_CHECK_ARG(n > 0 && n < (1 << 30) && flen > kmin && kmin > 0 && ldd >= flen && ldip >= 0 && df > 0 &&
                      nbins >= 1 && nbins <= kMaxBins && ldout >= kOut,
                  GWB_ERR_SHAPE, "snr_grad: n=%d flen=%d kmin=%d nbins=%d ldout=%lld", n, flen, kmin, nbins, ldout);
    cudaStream_t s = (cudaStream_t)stream;
    const float2* d = reinterpret_cast<const float2*>(D);
    if (fp64)
        snr_grad_kernel<double><<<n, kThreads, 0, s>>>(params, n, d, ldd, IP, ldip, flen, df, kmin, f_ecc, nbins,
                                                        out, ldout);
    else
        snr_grad_kernel<float><<<n, kThreads, 0, s>>>(params, n, d, ldd, IP, ldip, flen, df, kmin, f_ecc, nbins, out,
                                                       ldout);
    GWB_LAUNCH_CHECK("snr_grad_kernel");
    return GWB_OK;
}

int gwb_phase_metric(const double* params, int n, const float* IP, long long ldip, int flen, double df, int kmin,
                     double f_ecc, double* g, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(params && IP && g, GWB_ERR_ARG, "phase_metric: null pointer");
    GWB_CHECK_ARG(n > 0 && n < (1 << 30) && flen > kmin && kmin > 0 && ldip >= 0 && df > 0, GWB_ERR_SHAPE,
                  "phase_metric: n=%d flen=%d kmin=%d", n, flen, kmin);
    phase_metric_kernel<<<n, kThreads, 0, (cudaStream_t)stream>>>(params, n, IP, ldip, flen, df, kmin, f_ecc, g);
    GWB_LAUNCH_CHECK("phase_metric_kernel");
    return GWB_OK;
}

int gwb_refine_step(const double* params, const double* res, long long ldres, const double* g, const double* lam,
                    int n, double* out, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(params && res && g && lam && out, GWB_ERR_ARG, "refine_step: null pointer");
    GWB_CHECK_ARG(n > 0 && ldres >= kOut, GWB_ERR_SHAPE, "refine_step: n=%d ldres=%lld", n, ldres);
    refine_step_kernel<<<(unsigned)cdiv(n, 128), 128, 0, (cudaStream_t)stream>>>(params, res, ldres, g, lam, n, out);
    GWB_LAUNCH_CHECK("refine_step_kernel");
    return GWB_OK;
}

}  // extern "C"
