// Plain-fp32 form of the reconstruction GEMM with fused |z|^2 and blocked argmax, on the fp32 pipe.
//
// Same contract as gwb_fused_peaks_f16 (pipeline/fp_gemm.py:14-44 semantics) with fp32 operands: the reference only
// has an fp16 GEMM, so this is the full-precision form that the mixed forms are compared against. CTA = 128 template
// rows x one output group of `group` 128-sample blocks, walked block by block; 256 threads as 16 x 16, each thread
// owning 8 rows x 8 samples for re and im (128 accumulators). K is staged through shared memory 16 at a time.
#include "common.cuh"

namespace gwb {
namespace {

constexpr int BM = 128, BN = 128, BK = 16;

__device__ __forceinline__ void better(float ov, int oi, float& v, int& i) {
    if (ov > v || (ov == v && oi < i)) {
        v = ov;
        i = oi;
    }
}

__global__ void __launch_bounds__(256) simt_absmax_kernel(const float* __restrict__ Are, const float* __restrict__ Aim,
                                                          long long lda, const float* __restrict__ Z, long long ldz,
                                                          int M, int K, long long Tn, int ntiles, int group,
                                                          float* __restrict__ V, int32_t* __restrict__ I,
                                                          long long ldv) {
    __shared__ __align__(16) float sAr[BK][BM];
    __shared__ __align__(16) float sAi[BK][BM];
    __shared__ __align__(16) float sZ[BK][BN];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.y * BM;
    const int o = blockIdx.x;
    const int t0 = o * group, t1 = min(t0 + group, ntiles);
    float wb[8];
    int wi[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        wb[i] = -1.f;
        wi[i] = 0;
    }
    for (int t = t0; t < t1; ++t) {
        const long long c0 = (long long)t * BN;
        float ar[8][8], ai[8][8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) ar[i][j] = ai[i][j] = 0.f;
        for (int k0 = 0; k0 < K; k0 += BK) {
            // A tiles: 128 rows x 16 k, stored k-major; each thread moves 8 values of each
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int e = tid + 256 * r;       // 0..2047
                const int row = e >> 4, kk = e & 15;
                const int gr = m0 + row, gk = k0 + kk;
                const bool ok = gr < M && gk < K;
                sAr[kk][row] = ok ? Are[(long long)gr * lda + gk] : 0.f;
                sAi[kk][row] = ok ? Aim[(long long)gr * lda + gk] : 0.f;
            }
            // Z tile: 16 k x 128 samples
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int e = tid + 256 * r;
                const int kk = e >> 7, cc = e & 127;
                const long long gc = c0 + cc;
                const int gk = k0 + kk;
                sZ[kk][cc] = (gk < K && gc < Tn) ? Z[(long long)gk * ldz + gc] : 0.f;
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < BK; ++kk) {
                float a_r[8], a_i[8], z[8];
                const float4* pr = reinterpret_cast<const float4*>(&sAr[kk][ty * 8]);
                const float4* pi = reinterpret_cast<const float4*>(&sAi[kk][ty * 8]);
                const float4* pz = reinterpret_cast<const float4*>(&sZ[kk][tx * 8]);
                float4 v;
                v = pr[0]; a_r[0] = v.x; a_r[1] = v.y; a_r[2] = v.z; a_r[3] = v.w;
                v = pr[1]; a_r[4] = v.x; a_r[5] = v.y; a_r[6] = v.z; a_r[7] = v.w;
                v = pi[0]; a_i[0] = v.x; a_i[1] = v.y; a_i[2] = v.z; a_i[3] = v.w;
                v = pi[1]; a_i[4] = v.x; a_i[5] = v.y; a_i[6] = v.z; a_i[7] = v.w;
                v = pz[0]; z[0] = v.x; z[1] = v.y; z[2] = v.z; z[3] = v.w;
                v = pz[1]; z[4] = v.x; z[5] = v.y; z[6] = v.z; z[7] = v.w;
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        ar[i][j] = fmaf(a_r[i], z[j], ar[i][j]);
                        ai[i][j] = fmaf(a_i[i], z[j], ai[i][j]);
                    }
            }
            __syncthreads();
        }
        // |z|^2, max and first index per row over this thread's 8 samples, then over the 16 threads of the row
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            float best = -1.f;
            int bi = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int cc = tx * 8 + j;
                const float p = (c0 + cc < Tn) ? fmaf(ar[i][j], ar[i][j], ai[i][j] * ai[i][j]) : -1.f;
                if (p > best) {
                    best = p;
                    bi = cc;
                }
            }
#pragma unroll
            for (int off = 8; off > 0; off >>= 1) {
                const float ob = __shfl_xor_sync(0xffffffffu, best, off, 16);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, off, 16);
                better(ob, oi, best, bi);
            }
            const int gi = (int)(c0 + bi);
            if (t == t0 || best > wb[i]) {
                wb[i] = best;
                wi[i] = gi;
            }
        }
    }
    if (tx == 0) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int row = m0 + ty * 8 + i;
            if (row < M) {
                V[(long long)row * ldv + o] = wb[i];
                I[(long long)row * ldv + o] = wi[i];
            }
        }
    }
}

}  // namespace
}  // namespace gwb

extern "C" int gwb_fused_peaks_f32(const float* Are, const float* Aim, long long lda, const float* Z, long long ldz,
                                   int M, int K, long long Tn, int group, float* V, int32_t* I, long long ldv,
                                   void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(M > 0 && K > 0 && Tn > 0 && group > 0, GWB_ERR_SHAPE, "fused_peaks_f32: M=%d K=%d Tn=%lld group=%d",
                  M, K, Tn, group);
    GWB_CHECK_ARG(lda >= K && ldz >= Tn, GWB_ERR_SHAPE, "fused_peaks_f32: lda or ldz too small");
    GWB_CHECK_ARG(Are && Aim && Z && V && I, GWB_ERR_ARG, "fused_peaks_f32: null pointer");
    const long long ntiles = cdiv(Tn, BN);
    GWB_CHECK_ARG(ntiles * BN < (1ll << 31), GWB_ERR_SHAPE, "fused_peaks_f32: Tn too large for int32 indices");
    const long long nout = cdiv(ntiles, group);
    GWB_CHECK_ARG(ldv >= nout, GWB_ERR_SHAPE, "fused_peaks_f32: ldv=%lld < outputs per row %lld", ldv, nout);
    GWB_CHECK_ARG(nout < (1ll << 31), GWB_ERR_SHAPE, "fused_peaks_f32: too many outputs");
    dim3 grid((unsigned)nout, (unsigned)cdiv(M, BM));
    simt_absmax_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(Are, Aim, lda, Z, ldz, M, K, Tn, (int)ntiles, group, V,
                                                                I, ldv);
    GWB_LAUNCH_CHECK("simt_absmax_kernel");
    return GWB_OK;
}
