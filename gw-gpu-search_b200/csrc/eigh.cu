// Hermitian eigendecomposition of the tiles' normalised Gram matrices on the device, in float64: one-sided (Hestenes)
// Jacobi. It replaces the eigh of svd_tile (pipeline/fp_filter.py:583, torch.linalg.eigh in complex128).
//
// For a Hermitian positive semi-definite G, the column rotations that make the columns of U = G V mutually orthogonal
// (V unitary, starting from U = G, V = I) give G V = U = [sigma_j u_j]: the singular values sigma_j = ||U_j|| are
// the eigenvalues of G and the columns of V its eigenvectors. A sweep visits every column pair once, in n - 1 rounds
// of n / 2 disjoint pairs (the circle schedule: with m = n - 1, round r pairs (r + j) mod m with (r - j) mod m for
// j = 1 .. n/2 - 1, and r with n - 1), so the pairs of a round are rotated in parallel: one CTA per (pair, matrix),
// one thread per row. For a pair (p, q): alpha = ||u_p||^2, beta = ||u_q||^2, gamma = u_p^H u_q (fixed-order float64
// block sums); when |gamma| > tol sqrt(alpha beta), zeta = (beta - alpha) / (2 |gamma|), t = sign(zeta) / (|zeta| +
// sqrt(1 + zeta^2)), c = 1 / sqrt(1 + t^2), s = c t gamma / |gamma|, and u_p <- c u_p - conj(s) u_q, u_q <- s u_p +
// c u_q (the same for v), which makes u_p^H u_q zero. The caller repeats sweeps until a sweep rotates nothing.
// Columns whose norm is below `floor` (an absolute norm, about 1e-12 of the largest column of G) are numerically null:
// U = G V holds only to rounding error eps ||G||, so their directions are noise and no rotation can make them
// orthogonal to a relative 1e-13; pairs with such a column are not rotated (V stays unitary, their eigenvalues are the
// noise-level column norms).
#include "common.cuh"

namespace gwb {
namespace {

constexpr int kEigThreads = 256;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

__global__ void __launch_bounds__(kEigThreads) jacobi_round_kernel(double2* __restrict__ U, double2* __restrict__ V,
                                                                    const int* __restrict__ nv, int ld, long long mstride,
                                                                    int round, double tol, double floor2,
                                                                    int* __restrict__ rotated) {
    __shared__ double red[3][kEigThreads / 32];
    __shared__ double coef[4];
    const int mat = blockIdx.y, j = blockIdx.x;
    const int n = nv[mat];
    const int ne = n + (n & 1);                 // an odd n gets a virtual zero column ne - 1
    if (2 * j >= ne) return;
    const int m = ne - 1;
    int p, q;
    if (j == 0) {
        p = round % m;
        q = m;
    } else {
        p = (round + j) % m;
        q = ((round - j) % m + m) % m;
    }
    if (p >= n || q >= n) return;               // the virtual column: nothing to rotate
    if (p > q) {
        const int x = p;
        p = q;
        q = x;
    }
    double2* u = U + mat * mstride;
    double2* v = V + mat * mstride;
    const int i = threadIdx.x;
    double2 up = make_double2(0.0, 0.0), uq = up;
    if (i < n) {
        up = u[(long long)p * ld + i];
        uq = u[(long long)q * ld + i];
    }
    double a = up.x * up.x + up.y * up.y, b = uq.x * uq.x + uq.y * uq.y;
    double gr = up.x * uq.x + up.y * uq.y, gi = up.x * uq.y - up.y * uq.x;        // conj(up) uq
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, off);
        b += __shfl_xor_sync(0xffffffffu, b, off);
        gr += __shfl_xor_sync(0xffffffffu, gr, off);
        gi += __shfl_xor_sync(0xffffffffu, gi, off);
    }
    __shared__ double redi[kEigThreads / 32];
    if ((i & 31) == 0) {
        red[0][i >> 5] = a;
        red[1][i >> 5] = b;
        red[2][i >> 5] = gr;
        redi[i >> 5] = gi;
    }
    __syncthreads();
    if (i == 0) {
        double A = 0.0, Bv = 0.0, Gr = 0.0, Gi = 0.0;
        for (int w = 0; w < kEigThreads / 32; ++w) {
            A += red[0][w];
            Bv += red[1][w];
            Gr += red[2][w];
            Gi += redi[w];
        }
        const double g = sqrt(Gr * Gr + Gi * Gi);
        if (g > tol * sqrt(A * Bv) && g > 0.0 && A > floor2 && Bv > floor2) {
            const double zeta = (Bv - A) / (2.0 * g);
            const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            const double c = 1.0 / sqrt(1.0 + t * t);
            coef[0] = c;
            coef[1] = c * t * Gr / g;          // s = c t gamma / |gamma|
            coef[2] = c * t * Gi / g;
            coef[3] = 1.0;
            atomicAdd(rotated, 1);
        } else {
            coef[3] = 0.0;
        }
    }
    __syncthreads();
    if (coef[3] == 0.0 || i >= n) return;
    const double c = coef[0], sr = coef[1], si = coef[2];
    // u_p <- c u_p - conj(s) u_q ; u_q <- s u_p + c u_q
    auto rot = [&](double2 xp, double2 xq, double2& op, double2& oq) {
        op = make_double2(c * xp.x - (sr * xq.x + si * xq.y), c * xp.y - (sr * xq.y - si * xq.x));
        oq = make_double2(sr * xp.x - si * xp.y + c * xq.x, sr * xp.y + si * xp.x + c * xq.y);
    };
    double2 np_, nq_;
    rot(up, uq, np_, nq_);
    u[(long long)p * ld + i] = np_;
    u[(long long)q * ld + i] = nq_;
    const double2 vp = v[(long long)p * ld + i], vq = v[(long long)q * ld + i];
    rot(vp, vq, np_, nq_);
    v[(long long)p * ld + i] = np_;
    v[(long long)q * ld + i] = nq_;
}

// column norms: lam[mat][j] = ||U_j|| (fixed-order float64 sums), the eigenvalues
__global__ void __launch_bounds__(kEigThreads) column_norm_kernel(const double2* __restrict__ U,
                                                                   const int* __restrict__ nv, int ld,
                                                                   long long mstride, double* __restrict__ lam) {
    __shared__ double red[kEigThreads / 32];
    const int mat = blockIdx.y, j = blockIdx.x, i = threadIdx.x;
    const int n = nv[mat];
    if (j >= n) return;
    double s = 0.0;
    if (i < n) {
        const double2 x = U[mat * mstride + (long long)j * ld + i];
        s = x.x * x.x + x.y * x.y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((i & 31) == 0) red[i >> 5] = s;
    __syncthreads();
    if (i == 0) {
        double t = 0.0;
        for (int w = 0; w < kEigThreads / 32; ++w) t += red[w];
        lam[(long long)mat * ld + j] = sqrt(t);
    }
}

__global__ void identity_kernel(double2* __restrict__ V, const int* __restrict__ nv, int ld, long long mstride) {
    const int mat = blockIdx.y, j = blockIdx.x, i = threadIdx.x;
    if (i < ld) V[mat * mstride + (long long)j * ld + i] = make_double2(i == j && j < nv[mat] ? 1.0 : 0.0, 0.0);
}

}  // namespace
}  // namespace gwb

extern "C" {

int gwb_eigh_jacobi_sweep(double* U, double* V, const int* n, int nmat, int ld, int init, double tol, double floor,
                          int* rotated, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(U && V && n && rotated, GWB_ERR_ARG, "eigh_jacobi_sweep: null pointer");
    GWB_CHECK_ARG(nmat > 0 && nmat < 65536 && ld >= 2 && ld <= kEigThreads && tol > 0.0 && floor >= 0.0,
                  GWB_ERR_SHAPE, "eigh_jacobi_sweep: nmat=%d ld=%d (2..%d) tol=%g floor=%g", nmat, ld, kEigThreads, tol,
                  floor);
    cudaStream_t s = (cudaStream_t)stream;
    const long long ms = (long long)ld * ld;
    double2* u = reinterpret_cast<double2*>(U);
    double2* v = reinterpret_cast<double2*>(V);
    if (init) {
        identity_kernel<<<dim3(ld, nmat), ld, 0, s>>>(v, n, ld, ms);
        GWB_LAUNCH_CHECK("identity_kernel");
    }
    GWB_CUDA(cudaMemsetAsync(rotated, 0, sizeof(int), s));
    const int ne = ld + (ld & 1);
    for (int r = 0; r < ne - 1; ++r) {
        jacobi_round_kernel<<<dim3(ne / 2, nmat), kEigThreads, 0, s>>>(u, v, n, ld, ms, r, tol, floor * floor,
                                                                        rotated);
        GWB_LAUNCH_CHECK("jacobi_round_kernel");
    }
    return GWB_OK;
}

int gwb_eigh_values(const double* U, const int* n, int nmat, int ld, double* lam, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(U && n && lam, GWB_ERR_ARG, "eigh_values: null pointer");
    GWB_CHECK_ARG(nmat > 0 && nmat < 65536 && ld >= 2 && ld <= kEigThreads, GWB_ERR_SHAPE, "eigh_values: ld=%d", ld);
    column_norm_kernel<<<dim3(ld, nmat), kEigThreads, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const double2*>(U), n, ld, (long long)ld * ld, lam);
    GWB_LAUNCH_CHECK("column_norm_kernel");
    return GWB_OK;
}

}  // extern "C"
