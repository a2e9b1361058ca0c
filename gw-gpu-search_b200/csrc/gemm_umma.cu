// Reconstruction GEMM with fused |z|^2 and blocked argmax on the tcgen05 tensor cores (sm_100a).
//
// Replaces fp_gemm.gemm_absmax / fused_peaks (pipeline/fp_gemm.py:14-44): z_re = Are @ Z, z_im = Aim @ Z; per
// template row and per 128-sample block the maximum of z_re^2 + z_im^2 and its first sample index. The reference
// writes one (max, index) per block; here a row can also be reduced over `group` consecutive blocks (a 1 s cluster
// window is 16 blocks at 2048 Hz), which fuses the window reduction of fp_filter.py:745-746 into the epilogue.
//
// Design (one persistent CTA per SM, 10 warps):
//   warp 0      TMA producer: loads the whole A operand once (Are/Aim rows of up to two 128-row M blocks, kept
//               resident in shared memory), then streams Z tiles of 128 samples x K through a ring of stages.
//   warp 1      MMA issuer: one elected thread issues tcgen05.mma (M=128, N=128, K=16 steps) into TMEM. Work item =
//               (time tile, M block); accumulators for re and im sit in 256 TMEM columns, double buffered (512).
//   warps 2-9   epilogue: tcgen05.ld of re and im, |z|^2 and running max/argmax in registers. Warps w and w+4 read
//               the same TMEM lane quarter (rows) and split the 128 columns in halves, then combine through shared
//               memory. Only (max, index) per row and output group reaches global memory.
// Operands: A is K-major (row = template, K contiguous), Z is MN-major (K rows, samples contiguous); both are staged
// by TMA with the 128-byte swizzle. No multicast. Every wait is bounded (one second) and records GWB_ERR_TIMEOUT.
#include "common.cuh"

namespace gwb {
namespace {

constexpr int kTile = 128;                      // samples per block (the reference's BN)
constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;   // 320
constexpr int kATileBytes = 128 * 128;          // 128 rows x 64 two-byte elements
constexpr int kTmemCols = 512;

enum Form { kF16 = 0, kBF16x3 = 1 };

struct __align__(64) UmmaArgs {
    CUtensorMap tA[4];   // re (hi), im (hi), re lo, im lo
    CUtensorMap tZ[2];   // Z (hi), Z lo
    float* V;
    int32_t* I;
    long long ldv;
    long long Tn;
    int M, K, ntiles, group, nout, stages;
    DeviceError* err;
};

template <int FORM>
struct FormCfg {
    static constexpr int NA = FORM == kF16 ? 2 : 4;      // A tiles per (M block, K chunk)
    static constexpr int NZ = FORM == kF16 ? 1 : 2;      // Z operands per stage
    static constexpr int NPROD = FORM == kF16 ? 1 : 3;   // products accumulated per (re|im)
    static constexpr uint32_t FMT = FORM == kF16 ? 0u : 1u;
};

struct SmemLayout {
    uint32_t a_off, z_off, stage_bytes, x_off, bar_off, total;
};

__host__ __device__ inline SmemLayout smem_layout(int na, int nz, int nkc, int K, int stages) {
    SmemLayout L;
    L.a_off = 0;
    L.z_off = 2u * na * nkc * kATileBytes;
    L.stage_bytes = (uint32_t)nz * 2u * (uint32_t)K * 128u;
    L.x_off = L.z_off + (uint32_t)stages * L.stage_bytes;
    L.bar_off = L.x_off + 2u * 128u * 8u;
    L.total = L.bar_off + (uint32_t)(2 * stages + 6) * 8u + 16u;
    return L;
}

__device__ __forceinline__ void keep_best(float p, int j, float& best, int& bi) {
    if (p > best) {
        best = p;
        bi = j;
    }
}

template <int FORM>
__global__ void __launch_bounds__(kThreads, 1) umma_absmax_kernel(const __grid_constant__ UmmaArgs args) {
    using C = FormCfg<FORM>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);

    const int K = args.K, nkc = K / 64, S = args.stages;
    const SmemLayout L = smem_layout(C::NA, C::NZ, nkc, K, S);
    uint8_t* sA = smem + L.a_off;
    uint8_t* sZ = smem + L.z_off;
    float* xv = reinterpret_cast<float*>(smem + L.x_off);           // [2][128]
    int* xi = reinterpret_cast<int*>(smem + L.x_off + 1024);        // [2][128]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.bar_off);
    uint64_t* full = bars;
    uint64_t* empty = bars + S;
    uint64_t* tfull = bars + 2 * S;
    uint64_t* tempty = tfull + 2;
    uint64_t* barA = tempty + 2;
    uint64_t* done = barA + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * 256;
    const int MBe = min(2, (args.M - m0 + 127) / 128);
    const long long o0 = (long long)blockIdx.x * args.nout / gridDim.x;
    const long long o1 = (long long)(blockIdx.x + 1) * args.nout / gridDim.x;
    const int t_begin = (int)(o0 * args.group);
    const int t_end = (int)min(o1 * (long long)args.group, (long long)args.ntiles);
    const int ntl = t_end - t_begin;
    if (ntl <= 0 || MBe <= 0) return;   // uniform across the CTA

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], kEpiWarps);
        }
        mbar_init(barA, 1);
        mbar_init(done, 1);
        *abort_flag = 0;
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, kTmemCols);
        tmem_relinquish();
        tc_fence_before();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            for (int a = 0; a < C::NA; ++a) prefetch_tmap(&args.tA[a]);
            for (int z = 0; z < C::NZ; ++z) prefetch_tmap(&args.tZ[z]);
            mbar_arrive_expect_tx(barA, (uint32_t)(MBe * C::NA * nkc * kATileBytes));
            for (int mb = 0; mb < MBe; ++mb)
                for (int a = 0; a < C::NA; ++a)
                    for (int kc = 0; kc < nkc; ++kc)
                        tma_load_2d(sA + ((mb * C::NA + a) * nkc + kc) * kATileBytes, &args.tA[a], barA, kc * 64,
                                    m0 + mb * 128);
            for (int i = 0; i < ntl; ++i) {
                const int s = i % S;
                const uint32_t n = (uint32_t)(i / S);
                if (*abort_flag) break;
                if (!mbar_wait_bounded(&empty[s], (n & 1) ^ 1)) {
                    record_error(args.err, GWB_ERR_TIMEOUT, 101, blockIdx.x, i);
                    *abort_flag = 1;
                    break;
                }
                mbar_arrive_expect_tx(&full[s], L.stage_bytes);
                const int x = (t_begin + i) * kTile;
                for (int z = 0; z < C::NZ; ++z)
                    for (int h = 0; h < 2; ++h)
                        tma_load_2d(sZ + s * L.stage_bytes + (z * 2 + h) * K * 128, &args.tZ[z], &full[s],
                                    x + 64 * h, 0);
            }
            // make sure no copy is still landing in shared memory when the CTA exits
            mbar_wait_bounded(barA, 0);
            for (int s = 0; s < S && s < ntl; ++s) {
                const int nfill = (ntl - s + S - 1) / S;
                mbar_wait_bounded(&full[s], (uint32_t)((nfill - 1) & 1));
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            const uint32_t idesc = instr_desc(128, 128, C::FMT, C::FMT, 0, 1);
            const uint32_t a_base = smem_u32(sA), z_base = smem_u32(sZ);
            bool ok = mbar_wait_bounded(barA, 0);
            if (!ok) {
                record_error(args.err, GWB_ERR_TIMEOUT, 102, blockIdx.x, 0);
                *abort_flag = 1;
            }
            tc_fence_after();
            for (int i = 0; i < ntl && ok; ++i) {
                const int s = i % S;
                if (*abort_flag || !mbar_wait_bounded(&full[s], (uint32_t)((i / S) & 1))) {
                    record_error(args.err, GWB_ERR_TIMEOUT, 103, blockIdx.x, i);
                    *abort_flag = 1;
                    break;
                }
                tc_fence_after();
                for (int mb = 0; mb < MBe; ++mb) {
                    const int j = i * MBe + mb, b = j & 1;
                    const uint32_t u = (uint32_t)(j >> 1);
                    if (!mbar_wait_bounded(&tempty[b], (u & 1) ^ 1)) {
                        record_error(args.err, GWB_ERR_TIMEOUT, 104, blockIdx.x, i);
                        *abort_flag = 1;
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    for (int ri = 0; ri < 2; ++ri) {
                        const uint32_t d = tmem + (uint32_t)(b * 256 + ri * 128);
                        uint32_t acc = 0;
                        for (int pr = 0; pr < C::NPROD; ++pr) {
                            // products: (A hi, Z hi), (A hi, Z lo), (A lo, Z hi)
                            const int a = (pr == 2 ? 2 : 0) + ri;
                            const int z = (pr == 1) ? 1 : 0;
                            for (int k16 = 0; k16 < K / 16; ++k16) {
                                const uint32_t aaddr =
                                    a_base + ((mb * C::NA + a) * nkc + (k16 >> 2)) * kATileBytes + (k16 & 3) * 32;
                                const uint32_t baddr = z_base + s * L.stage_bytes + (z * 2) * K * 128 + k16 * 2048;
                                const uint64_t adesc = smem_desc(aaddr, 16, 1024, 2);
                                const uint64_t bdesc = smem_desc(baddr, (uint32_t)K * 128u, 1024, 2);
                                umma_f16(d, adesc, bdesc, idesc, acc);
                                acc = 1;
                            }
                        }
                    }
                    umma_commit(&tfull[b]);
                }
                umma_commit(&empty[s]);
            }
            umma_commit(done);
            mbar_wait_bounded(done, 0);
        }
        __syncwarp();
    } else {
        // ---------------- epilogue ----------------
        const int ew = warp - 2, q = warp & 3, hh = ew >> 2;
        const int rl = 32 * q + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(32 * q) << 16);
        float wb0 = -1.f, wb1 = -1.f;
        int wi0 = 0, wi1 = 0;
        for (int i = 0; i < ntl; ++i) {
            const int t = t_begin + i;
            const long long col0 = (long long)t * kTile;
            const bool full_tile = col0 + kTile <= args.Tn;
#pragma unroll
            for (int mb = 0; mb < 2; ++mb) {
                if (mb >= MBe) break;
                const int j = i * MBe + mb, b = j & 1;
                const uint32_t u = (uint32_t)(j >> 1);
                float best = -1.f;
                int bi = 0;
                if (*abort_flag || !mbar_wait_bounded(&tfull[b], u & 1)) {
                    record_error(args.err, GWB_ERR_TIMEOUT, 105, blockIdx.x, i);
                    *abort_flag = 1;
                } else {
                    tc_fence_after();
#pragma unroll
                    for (int c = 0; c < 64; c += 32) {
                        uint32_t re[32], im[32];
                        tmem_ld_32x32b_x32(lane_base + (uint32_t)(b * 256 + hh * 64 + c), re);
                        tmem_ld_32x32b_x32(lane_base + (uint32_t)(b * 256 + 128 + hh * 64 + c), im);
                        tmem_ld_wait();
                        // tie every value to the wait so no use is scheduled above it
#pragma unroll
                        for (int jj = 0; jj < 32; ++jj) asm volatile("" : "+r"(re[jj]), "+r"(im[jj]));
                        const int cb = hh * 64 + c;
                        float lb = -1.f;
                        int lj = 0;
                        if (full_tile) {
#pragma unroll
                            for (int jj = 0; jj < 32; ++jj) {
                                const float xr = __uint_as_float(re[jj]), xi_ = __uint_as_float(im[jj]);
                                keep_best(fmaf(xr, xr, xi_ * xi_), jj, lb, lj);
                            }
                        } else {
                            const int valid = (int)min((long long)32, max(0ll, args.Tn - (col0 + cb)));
#pragma unroll
                            for (int jj = 0; jj < 32; ++jj) {
                                const float xr = __uint_as_float(re[jj]), xi_ = __uint_as_float(im[jj]);
                                keep_best(jj < valid ? fmaf(xr, xr, xi_ * xi_) : -1.f, jj, lb, lj);
                            }
                        }
                        if (lb > best) {
                            best = lb;
                            bi = cb + lj;
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[b]);
                if (hh == 1) {
                    xv[(j & 1) * 128 + rl] = best;
                    xi[(j & 1) * 128 + rl] = bi;
                }
                named_bar_sync(1, 32 * kEpiWarps);
                if (hh == 0) {
                    const float ob = xv[(j & 1) * 128 + rl];
                    const int oi = xi[(j & 1) * 128 + rl];
                    if (ob > best) {
                        best = ob;
                        bi = oi;
                    }
                    const int gi = (int)(col0 + bi);
                    const bool first = (t % args.group) == 0;
                    const bool last = ((t + 1) % args.group) == 0 || t == args.ntiles - 1;
                    float& wb = (mb == 0) ? wb0 : wb1;
                    int& wi = (mb == 0) ? wi0 : wi1;
                    if (first || best > wb) {
                        wb = best;
                        wi = gi;
                    }
                    if (last) {
                        const int row = m0 + mb * 128 + rl;
                        if (row < args.M) {
                            const long long o = t / args.group;
                            args.V[(long long)row * args.ldv + o] = wb;
                            args.I[(long long)row * args.ldv + o] = wi;
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

template <int FORM>
int launch_umma(const uint16_t* const* A, const uint16_t* const* Zp, long long lda, long long ldz, int M, int K,
                long long Tn, int group, float* V, int32_t* I, long long ldv, cudaStream_t stream) {
    using C = FormCfg<FORM>;
    GWB_CHECK_ARG(M > 0 && Tn > 0 && group > 0, GWB_ERR_SHAPE, "fused_peaks: M=%d Tn=%lld group=%d", M, Tn, group);
    GWB_CHECK_ARG(K > 0 && K % 64 == 0 && K <= 256, GWB_ERR_SHAPE, "fused_peaks: K=%d must be a multiple of 64, <= 256",
                  K);
    GWB_CHECK_ARG(lda >= K && ldz >= Tn, GWB_ERR_SHAPE, "fused_peaks: lda=%lld < K or ldz=%lld < Tn", lda, ldz);
    GWB_CHECK_ARG(lda % 8 == 0 && ldz % 8 == 0, GWB_ERR_ALIGN, "fused_peaks: lda=%lld and ldz=%lld must be multiples of 8",
                  lda, ldz);
    for (int a = 0; a < C::NA; ++a)
        GWB_CHECK_ARG(A[a] != nullptr && aligned(A[a], 16), GWB_ERR_ALIGN, "fused_peaks: A operand %d misaligned", a);
    for (int z = 0; z < C::NZ; ++z)
        GWB_CHECK_ARG(Zp[z] != nullptr && aligned(Zp[z], 16), GWB_ERR_ALIGN, "fused_peaks: Z operand %d misaligned", z);
    GWB_CHECK_ARG(V != nullptr && I != nullptr, GWB_ERR_ARG, "fused_peaks: null output");
    const long long ntiles = cdiv(Tn, kTile);
    GWB_CHECK_ARG(ntiles * kTile < (1ll << 31), GWB_ERR_SHAPE, "fused_peaks: Tn too large for int32 indices");
    const long long nout = cdiv(ntiles, group);
    GWB_CHECK_ARG(ldv >= nout, GWB_ERR_SHAPE, "fused_peaks: ldv=%lld < outputs per row %lld", ldv, nout);

    UmmaArgs args;
    memset(&args, 0, sizeof(args));
    const CUtensorMapDataType dt = FORM == kF16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    for (int a = 0; a < C::NA; ++a) {
        int r = encode_tmap_2d(&args.tA[a], dt, A[a], (uint64_t)K, (uint64_t)M, (uint64_t)lda * 2, 64, 128,
                               CU_TENSOR_MAP_SWIZZLE_128B);
        if (r) return r;
    }
    for (int z = 0; z < C::NZ; ++z) {
        int r = encode_tmap_2d(&args.tZ[z], dt, Zp[z], (uint64_t)Tn, (uint64_t)K, (uint64_t)ldz * 2, 64, (uint32_t)K,
                               CU_TENSOR_MAP_SWIZZLE_128B);
        if (r) return r;
    }
    const int nkc = K / 64;
    const int mgroups = (M + 255) / 256;
    const int max_smem = 227 * 1024;
    int stages = 8;
    while (stages > 1 && smem_layout(C::NA, C::NZ, nkc, K, stages).total + 1024 > (uint32_t)max_smem) --stages;
    {   // the launch table may ask for a shallower Z ring (forms 4: stacked fp16, 5: stacked split bf16; kh = K)
        int pair = 0, st = 0, order = 0;
        if (tune_lookup(FORM == kF16 ? 4 : 5, K, &pair, &st, &order) && st >= 2) stages = std::min(stages, st);
    }
    const uint32_t smem = smem_layout(C::NA, C::NZ, nkc, K, stages).total + 1024;
    GWB_CHECK_ARG(smem <= (uint32_t)max_smem, GWB_ERR_SHAPE, "fused_peaks: K=%d needs %u bytes of shared memory", K,
                  smem);
    args.V = V;
    args.I = I;
    args.ldv = ldv;
    args.Tn = Tn;
    args.M = M;
    args.K = K;
    args.ntiles = (int)ntiles;
    args.group = group;
    args.nout = (int)nout;
    args.stages = stages;
    args.err = device_error_ptr();

    auto kern = umma_absmax_kernel<FORM>;
    GWB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int gx = (int)std::max(1ll, std::min(nout, (long long)std::max(1, num_sms() / mgroups)));
    dim3 grid(gx, mgroups);
    kern<<<grid, kThreads, smem, stream>>>(args);
    GWB_LAUNCH_CHECK("umma_absmax_kernel");
    return GWB_OK;
}

}  // namespace
}  // namespace gwb

extern "C" {

int gwb_fused_peaks_f16(const uint16_t* Are, const uint16_t* Aim, long long lda, const uint16_t* Z, long long ldz,
                        int M, int K, long long Tn, int group, float* V, int32_t* I, long long ldv, void* stream) {
    const uint16_t* A[2] = {Are, Aim};
    const uint16_t* Zs[1] = {Z};
    return gwb::launch_umma<gwb::kF16>(A, Zs, lda, ldz, M, K, Tn, group, V, I, ldv, (cudaStream_t)stream);
}

int gwb_fused_peaks_bf16x3(const uint16_t* Are_hi, const uint16_t* Are_lo, const uint16_t* Aim_hi,
                           const uint16_t* Aim_lo, long long lda, const uint16_t* Z_hi, const uint16_t* Z_lo,
                           long long ldz, int M, int K, long long Tn, int group, float* V, int32_t* I,
                           long long ldv, void* stream) {
    const uint16_t* A[4] = {Are_hi, Aim_hi, Are_lo, Aim_lo};
    const uint16_t* Zs[2] = {Z_hi, Z_lo};
    return gwb::launch_umma<gwb::kBF16x3>(A, Zs, lda, ldz, M, K, Tn, group, V, I, ldv, (cudaStream_t)stream);
}

}  // extern "C"
