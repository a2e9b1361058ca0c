// Plain-fp32 form of the reconstruction GEMM with fused |z|^2 and blocked argmax, on the fp32 pipe.
//
// Same contract as gwb_fused_peaks_f16 (pipeline/fp_gemm.py:14-44 semantics) with fp32 operands: the reference only
// has an fp16 GEMM, so this is the full-precision form that the mixed forms are compared against. CTA = 128 template
// rows x one output group of `group` 128-sample blocks, walked block by block; 256 threads as 16 x 16, each thread
// owning 8 rows x 8 samples for re and im (128 accumulators). K is staged through shared memory 16 at a time.
#include <atomic>

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

// The same product with the operand tiles copied by cp.async through a ring of AS_ST stages, so the loads of the
// next K tiles overlap the FMAs of this one (the kernel above loads and computes in turn). 16-byte copies: needs K,
// lda and ldz multiples of 4 and 16-byte aligned operands (the launcher falls back to the kernel above otherwise).
// Thread (tx, ty) owns rows ty + 16 i (i < 8) and samples 4 tx + j, 64 + 4 tx + j (j < 4): the A reads of a warp
// (two rows, one float4 each) fall in distinct banks, the Z reads are two runs of 256 contiguous bytes.
constexpr int AS_ST = 3;
constexpr int AS_STAGE = 3 * BM * BK;            // floats per stage: A re, A im (BM x BK, row-major), Z (BK x BN)

__device__ __forceinline__ void cp_async16_zfill(float* smem, const float* gmem, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem), "r"(src_bytes)
                 : "memory");
}

__global__ void __launch_bounds__(256, 1) simt_absmax_async_kernel(
    const float* __restrict__ Are, const float* __restrict__ Aim, long long lda, const float* __restrict__ Z,
    long long ldz, int M, int K, long long Tn, int ntiles, int group, float* __restrict__ V, int32_t* __restrict__ I,
    long long ldv) {
    static_assert(BM == 128 && BN == 128 && BK == 16, "tile shape");
    extern __shared__ __align__(16) float smf[];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.y * BM;
    const int o = blockIdx.x;
    const int t0 = o * group, t1 = min(t0 + group, ntiles);
    const int nk = (K + BK - 1) / BK;
    const int nsteps = (t1 - t0) * nk;
    auto load = [&](int step) {
        float* sAr = smf + (step % AS_ST) * AS_STAGE;
        float* sAi = sAr + BM * BK;
        float* sZ = sAi + BM * BK;
        const int t = t0 + step / nk, k0 = (step % nk) * BK;
#pragma unroll
        for (int r = 0; r < 2; ++r) {            // A: 128 rows x 16 k, four k per copy
            const int e = tid + 256 * r;
            const int row = e >> 2, kq = (e & 3) * 4;
            const int gr = m0 + row, gk = k0 + kq;
            const bool ok = gr < M && gk < K;
            const long long off = ok ? (long long)gr * lda + gk : 0;
            cp_async16_zfill(sAr + row * BK + kq, Are + off, ok ? 16 : 0);
            cp_async16_zfill(sAi + row * BK + kq, Aim + off, ok ? 16 : 0);
        }
#pragma unroll
        for (int r = 0; r < 2; ++r) {            // Z: 16 k x 128 samples, four samples per copy
            const int e = tid + 256 * r;
            const int kk = e >> 5, cq = (e & 31) * 4;
            const int gk = k0 + kk;
            const long long gc = (long long)t * BN + cq;
            const int nb = (gk < K && gc < Tn) ? (int)min(16ll, (Tn - gc) * 4) : 0;
            cp_async16_zfill(sZ + kk * BN + cq, Z + (nb ? (long long)gk * ldz + gc : 0), nb);
        }
    };
    float wb[8];
    int wi[8];
    float ar[8][8], ai[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        wb[i] = -1.f;
        wi[i] = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) ar[i][j] = ai[i][j] = 0.f;
    }
#pragma unroll
    for (int s = 0; s < AS_ST - 1; ++s) {
        if (s < nsteps) load(s);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int step = 0; step < nsteps; ++step) {
        asm volatile("cp.async.wait_group %0;" ::"n"(AS_ST - 2) : "memory");
        __syncthreads();                         // this step's tiles are in; every thread is done with step - 1's
        if (step + AS_ST - 1 < nsteps) load(step + AS_ST - 1);
        asm volatile("cp.async.commit_group;" ::: "memory");
        const float* sAr = smf + (step % AS_ST) * AS_STAGE;
        const float* sAi = sAr + BM * BK;
        const float* sZ = sAi + BM * BK;
#pragma unroll
        for (int kq = 0; kq < BK; kq += 4) {
            float4 a4r[8], a4i[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                a4r[i] = *reinterpret_cast<const float4*>(sAr + (ty + 16 * i) * BK + kq);
                a4i[i] = *reinterpret_cast<const float4*>(sAi + (ty + 16 * i) * BK + kq);
            }
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const float4 z0 = *reinterpret_cast<const float4*>(sZ + (kq + kk) * BN + 4 * tx);
                const float4 z1 = *reinterpret_cast<const float4*>(sZ + (kq + kk) * BN + 64 + 4 * tx);
                const float z[8] = {z0.x, z0.y, z0.z, z0.w, z1.x, z1.y, z1.z, z1.w};
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float a_r = kk == 0 ? a4r[i].x : kk == 1 ? a4r[i].y : kk == 2 ? a4r[i].z : a4r[i].w;
                    const float a_i = kk == 0 ? a4i[i].x : kk == 1 ? a4i[i].y : kk == 2 ? a4i[i].z : a4i[i].w;
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        ar[i][j] = fmaf(a_r, z[j], ar[i][j]);
                        ai[i][j] = fmaf(a_i, z[j], ai[i][j]);
                    }
                }
            }
        }
        if (step % nk == nk - 1) {
            // |z|^2, max and first index per row over this thread's 8 samples (increasing order), then over the 16
            // threads of the row; then the running window maximum
            const int t = t0 + step / nk;
            const long long c0 = (long long)t * BN;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                float best = -1.f;
                int bi = 0;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int cc = (j < 4 ? 4 * tx + j : 64 + 4 * tx + (j - 4));
                    const float p = (c0 + cc < Tn) ? fmaf(ar[i][j], ar[i][j], ai[i][j] * ai[i][j]) : -1.f;
                    if (p > best) {
                        best = p;
                        bi = cc;
                    }
                    ar[i][j] = ai[i][j] = 0.f;
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
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    if (tx == 0) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int row = m0 + ty + 16 * i;
            if (row < M) {
                V[(long long)row * ldv + o] = wb[i];
                I[(long long)row * ldv + o] = wi[i];
            }
        }
    }
}

std::atomic<int> g_f32_async{1};   // 0: the synchronous kernel only (gwb_f32_set_async)

}  // namespace
}  // namespace gwb

extern "C" int gwb_f32_set_async(int on) {
    using namespace gwb;
    GWB_CHECK_ARG(on == 0 || on == 1, GWB_ERR_ARG, "f32_set_async: on=%d (0 or 1)", on);
    g_f32_async.store(on);
    return GWB_OK;
}

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
    const bool async = g_f32_async.load() && K % 4 == 0 && lda % 4 == 0 && ldz % 4 == 0 && aligned(Are, 16) &&
                       aligned(Aim, 16) && aligned(Z, 16);
    if (async) {
        const int smem = AS_ST * AS_STAGE * (int)sizeof(float);
        GWB_CUDA(cudaFuncSetAttribute(simt_absmax_async_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        simt_absmax_async_kernel<<<grid, 256, smem, (cudaStream_t)stream>>>(Are, Aim, lda, Z, ldz, M, K, Tn,
                                                                            (int)ntiles, group, V, I, ldv);
        GWB_LAUNCH_CHECK("simt_absmax_async_kernel");
        return GWB_OK;
    }
    simt_absmax_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(Are, Aim, lda, Z, ldz, M, K, Tn, (int)ntiles, group, V,
                                                                I, ldv);
    GWB_LAUNCH_CHECK("simt_absmax_kernel");
    return GWB_OK;
}
