// Complex reconstruction GEMM with fused |z|^2 and windowed argmax, compact operand layout, tcgen05 (sm_100a).
//
// Same result as the reference's stacked GEMM (pipeline/fp_filter.py:615-621, pipeline/fp_gemm.py:14-33) but with
// the complex structure used instead of stored: the reference stacks Are = [Re As, -Im As] and Aim = [Im As, Re As]
// against Z = [Re zb; Im zb]; here A = [Re As | Im As] (each half Kh columns, Kh a multiple of 16, zero-padded past
// r) and Z = [Re zb; Im zb] (each half Kh rows), and the four products are issued as
//     z_re = ReA . ReZ - ImA . ImZ      (the minus is the MMA's A-negate bit)
//     z_im = ImA . ReZ + ReA . ImZ
// so A takes half the shared memory of Are + Aim and stays resident for any r up to 192 (fp16 / bf16) or 128 (split
// bf16), while Z streams through a ring of K-chunks by TMA. Work item = (128-sample time tile, 128-row M block); the
// re and im accumulators of an item sit in 256 TMEM columns, double buffered. Epilogue as the stacked kernel: warps
// 2-9 read TMEM, form |z|^2 and keep max and first index per row over `group` tiles.
// Forms: 0 fp16 (one product), 1 bf16 (one product), 2 split bf16 (hi.hi + hi.lo + lo.hi, about 16 bits), 3 fp8 e4m3
// (kind::f8f6f4, K = 32 per MMA, 128-byte rows hold 128 elements; the screening form: A rows carry a per-row scale
// that the epilogue applies, V = rowscale^2 max |z|^2).
#include <stdlib.h>
#include <string.h>
#include "common.cuh"

namespace gwb {
namespace {

constexpr int kTile = 128;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr int kATile = 128 * 128;      // 128 rows x 64 two-byte columns
constexpr int kTmemCols = 512;

struct __align__(64) CplxArgs {
    CUtensorMap tA[2];   // A hi, A lo: (n, 2 Kh), K-major
    CUtensorMap tZ[2];   // Z hi, Z lo: (2 Kh, Tn), sample-major
    float* V;
    int32_t* I;
    const float* rowscale;   // form 3: per-row scale of A (V is multiplied by its square); else null
    long long ldv;
    long long Tn;
    int M, Kh, ntiles, group, nout, stages, MB, KC;
    // split bf16 with Kh > 128: A hi resident, A lo streamed with the Z ring (16 K rows per stage, 32-byte swizzle)
    int lo_stream;
    int order;   // CTA-pair kernel: order of the complex products' MMAs (0-3, see the kernel)
    // tile-granular CTA ranges (balanced to one tile): windows cut by a range boundary are written as partial
    // (max, first index) records, pv/pi[(row * gridDim.x + cta) * 2 + slot] (slot 0: the window began before the
    // CTA's range, 1: it goes on after it), and merged by window_merge_kernel; null: window-aligned ranges
    float* pv;
    int32_t* pi;
    DeviceError* err;
};

// Forms: 0 fp16, 1 bf16, 2 split bf16 (A and Z as hi + lo, products hi.hi + hi.lo + lo.hi), 3 fp8 e4m3, 6 fp16 with A
// split (A hi + lo in fp16, Z in fp16, products hi.Z + lo.Z).
template <int FORM>
struct Cfg {
    static constexpr bool SPLIT_A = FORM == 2 || FORM == 6;           // A as hi + lo
    static constexpr int NHA = SPLIT_A ? 2 : 1;                       // copies of A
    static constexpr int NHZ = FORM == 2 ? 2 : 1;                     // copies of Z
    static constexpr int NH = NHA > NHZ ? NHA : NHZ;                  // tensor maps per operand
    static constexpr int NPROD = FORM == 2 ? 3 : (FORM == 6 ? 2 : 1);
    static constexpr uint32_t FMT = FORM == 1 || FORM == 2 ? 1u : 0u;   // kind::f16: 0 f16, 1 bf16; kind::f8f6f4: 0 e4m3
    // product pr: A copy ha, Z copy hz (split bf16: (0,0), (0,1), (1,0); fp16 with split A: (0,0), (1,0))
    static constexpr int ha(int pr) { return SPLIT_A && pr == NPROD - 1 ? 1 : 0; }
    static constexpr int hz(int pr) { return FORM == 2 && pr == 1 ? 1 : 0; }
    static constexpr bool F8 = FORM == 3;
    static constexpr int ES = F8 ? 1 : 2;                 // bytes per element
    static constexpr int KSTEP = F8 ? 32 : 16;            // K per MMA
    static constexpr int ROWEL = 128 / ES;                // elements per 128-byte swizzle row
    static constexpr int HALVES = 128 / ROWEL;            // 128-sample tile = HALVES boxes of ROWEL samples
};

struct Layout {
    uint32_t a_tiles, a_bytes, z_off, stage_bytes, x_off, bar_off, total;
};

__host__ __device__ inline Layout layout_of(int nha, int nhz, int MB, int Kh, int KC, int stages, int rowel = 64) {
    Layout L;
    L.a_tiles = (uint32_t)((2 * Kh + rowel - 1) / rowel);
    L.a_bytes = (uint32_t)MB * nha * L.a_tiles * kATile;
    L.z_off = L.a_bytes;
    // (re, im) x (hi, lo) x the 128-sample tile as 128-byte rows (two 64-sample halves for 16-bit, one for 8-bit)
    L.stage_bytes = 2u * nhz * (uint32_t)(128 / rowel) * (uint32_t)KC * 128u;
    L.x_off = L.z_off + (uint32_t)stages * L.stage_bytes;
    L.bar_off = L.x_off + 2048u;
    L.total = L.bar_off + (uint32_t)(2 * stages + 6) * 8u + 16u;
    return L;
}

// The split-A forms with A lo streamed: A hi resident (128 rows x 2 Kh), stages of Z (re, im) x (its nhz copies) x
// KC rows x 128 samples followed by A lo (re, im) x 128 rows x KC columns (KC = 16: one 32-byte swizzle atom per row;
// KC = 32: 64-byte rows in the 64-byte swizzle).
__host__ __device__ inline Layout layout_split_stream(int Kh, int KC, int stages, int nhz) {
    Layout L;
    L.a_tiles = (uint32_t)((2 * Kh + 63) / 64);
    L.a_bytes = L.a_tiles * kATile;
    L.z_off = L.a_bytes;
    L.stage_bytes = 2u * (uint32_t)nhz * 2u * (uint32_t)KC * 128u + 2u * 128u * (uint32_t)KC * 2u;
    L.x_off = L.z_off + (uint32_t)stages * L.stage_bytes;
    L.bar_off = L.x_off + 2048u;
    L.total = L.bar_off + (uint32_t)(2 * stages + 6) * 8u + 16u;
    return L;
}

template <int FORM>
__global__ void __launch_bounds__(kThreads, 1) umma_cplx_kernel(const __grid_constant__ CplxArgs args) {
    using C = Cfg<FORM>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    const int Kh = args.Kh, KC = args.KC, S = args.stages, MB = args.MB;
    const bool los = C::SPLIT_A && args.lo_stream != 0;   // A lo streamed (MB = 1, KC = 16 or 32)
    const int nres = los ? 1 : C::NHA;                    // resident copies of A
    const Layout L = los ? layout_split_stream(Kh, KC, S, C::NHZ) : layout_of(C::NHA, C::NHZ, MB, Kh, KC, S, C::ROWEL);
    const uint32_t zst_bytes = 2u * C::NHZ * C::HALVES * (uint32_t)KC * 128u;   // the Z part of a stage
    const int nkc = (Kh + KC - 1) / KC;
    uint8_t* sA = smem;
    uint8_t* sZ = smem + L.z_off;
    float* xv = reinterpret_cast<float*>(smem + L.x_off);
    int* xi = reinterpret_cast<int*>(smem + L.x_off + 1024);
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
    const int m0 = blockIdx.y * 128 * MB;
    const int MBe = min(MB, (args.M - m0 + 127) / 128);
    int t_begin, t_end;
    if (args.pv) {
        t_begin = (int)((long long)blockIdx.x * args.ntiles / gridDim.x);
        t_end = (int)((long long)(blockIdx.x + 1) * args.ntiles / gridDim.x);
    } else {
        const long long o0 = (long long)blockIdx.x * args.nout / gridDim.x;
        const long long o1 = (long long)(blockIdx.x + 1) * args.nout / gridDim.x;
        t_begin = (int)(o0 * args.group);
        t_end = (int)min(o1 * (long long)args.group, (long long)args.ntiles);
    }
    const int ntl = t_end - t_begin;
    if (ntl <= 0 || MBe <= 0) return;
    const int nfill = ntl * nkc;   // Z stages consumed by this CTA

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
        if (lane == 0) {
            for (int h = 0; h < C::NHA; ++h) prefetch_tmap(&args.tA[h]);
            for (int h = 0; h < C::NHZ; ++h) prefetch_tmap(&args.tZ[h]);
            mbar_arrive_expect_tx(barA, (uint32_t)(MBe * nres * L.a_tiles * kATile));
            for (int mb = 0; mb < MBe; ++mb)
                for (int h = 0; h < nres; ++h)
                    for (int a = 0; a < (int)L.a_tiles; ++a)
                        tma_load_2d(sA + ((mb * nres + h) * L.a_tiles + a) * kATile, &args.tA[h], barA,
                                    a * C::ROWEL, m0 + mb * 128);
            for (int f = 0; f < nfill; ++f) {
                const int s = f % S;
                const uint32_t n = (uint32_t)(f / S);
                const int i = f / nkc, kc = f % nkc;
                if (*abort_flag) break;
                if (!mbar_wait_bounded(&empty[s], (n & 1) ^ 1)) {
                    record_error(args.err, GWB_ERR_TIMEOUT, 201, blockIdx.x, f);
                    *abort_flag = 1;
                    break;
                }
                mbar_arrive_expect_tx(&full[s], L.stage_bytes);
                const int x = (t_begin + i) * kTile;
                uint8_t* st = sZ + s * L.stage_bytes;
                for (int ri = 0; ri < 2; ++ri)
                    for (int h = 0; h < C::NHZ; ++h)
                        for (int half = 0; half < C::HALVES; ++half)
                            tma_load_2d(st + ((ri * C::NHZ + h) * C::HALVES + half) * KC * 128, &args.tZ[h],
                                        &full[s], x + C::ROWEL * half, ri * Kh + kc * KC);
                if (los)            // A lo, re then im columns of this K chunk (x a multiple of 16 elements)
                    for (int ri = 0; ri < 2; ++ri)
                        tma_load_2d(st + zst_bytes + ri * 128 * KC * 2, &args.tA[1], &full[s], ri * Kh + kc * KC, m0);
            }
            mbar_wait_bounded(barA, 0);
            for (int s = 0; s < S && s < nfill; ++s) {
                const int nf = (nfill - s + S - 1) / S;
                mbar_wait_bounded(&full[s], (uint32_t)((nf - 1) & 1));
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = instr_desc(128, 128, C::FMT, C::FMT, 0, 1);
            const uint32_t idesc_neg = idesc | (1u << 13);     // negate A
            const uint32_t a_base = smem_u32(sA), z_base = smem_u32(sZ);
            bool ok = mbar_wait_bounded(barA, 0);
            if (!ok) {
                record_error(args.err, GWB_ERR_TIMEOUT, 202, blockIdx.x, 0);
                *abort_flag = 1;
            }
            tc_fence_after();
            // the MMAs of one item (M block mb) on one Z chunk. One-product forms: every descriptor of the chunk is
            // formed first (base descriptors plus offsets), then the MMAs go out back to back in the same order (sk,
            // four real products), so the one issuing thread spends no address arithmetic between them (measured
            // 0.266 -> 0.253 ms at n = 256, r = 128, fp16). The split form keeps descriptors and MMAs interleaved (the burst measured slower there:
            // one K step per chunk when A lo is streamed).
            auto issue = [&](int kc, int mb, int b, uint32_t st) {
                if constexpr (C::NPROD == 1) {
                    constexpr int MAXS = 4;                      // K steps per chunk: KC / KSTEP (64/16, 128/32)
                    const uint32_t dre = tmem + (uint32_t)(b * 256), dim = dre + 128;
                    const int nsteps = min(KC, Kh - kc * KC) / C::KSTEP;
                    const uint32_t abase = a_base + mb * L.a_tiles * kATile;
                    // base descriptors of the chunk plus byte offsets >> 4 (the start-address field, bits 0-13;
                    // shared-memory addresses stay below 2^18, so it does not carry)
                    const uint64_t ad = smem_desc(abase, 16, 1024, 2);
                    const uint64_t zd = smem_desc(st, (uint32_t)KC * 128u, 1024, 2);
                    uint64_t dAre[MAXS], dAim[MAXS], dZre[MAXS], dZim[MAXS];
#pragma unroll
                    for (int sk = 0; sk < MAXS; ++sk) {
                        const int k = kc * KC + sk * C::KSTEP;
                        const uint32_t are = (k / C::ROWEL) * kATile + (k % C::ROWEL) * C::ES;
                        const uint32_t aim = ((Kh + k) / C::ROWEL) * kATile + ((Kh + k) % C::ROWEL) * C::ES;
                        // K step = KSTEP rows of 128 bytes (2048 bytes for 16-bit, 4096 for 8-bit)
                        dAre[sk] = ad + (uint64_t)(are >> 4);
                        dAim[sk] = ad + (uint64_t)(aim >> 4);
                        dZre[sk] = zd + (uint64_t)(sk * C::KSTEP * 8);
                        dZim[sk] = zd + (uint64_t)(((C::HALVES * KC * 128) >> 4) + sk * C::KSTEP * 8);
                    }
#pragma unroll
                    for (int sk = 0; sk < MAXS; ++sk) {
                        if (sk >= nsteps) break;
                        const uint32_t acc = (kc > 0 || sk > 0) ? 1u : 0u;
                        if constexpr (C::F8) {
                            umma_f8(dre, dAre[sk], dZre[sk], idesc, acc);
                            umma_f8(dre, dAim[sk], dZim[sk], idesc_neg, 1u);
                            umma_f8(dim, dAim[sk], dZre[sk], idesc, acc);
                            umma_f8(dim, dAre[sk], dZim[sk], idesc, 1u);
                        } else {
                            umma_f16(dre, dAre[sk], dZre[sk], idesc, acc);
                            umma_f16(dre, dAim[sk], dZim[sk], idesc_neg, 1u);
                            umma_f16(dim, dAim[sk], dZre[sk], idesc, acc);
                            umma_f16(dim, dAre[sk], dZim[sk], idesc, 1u);
                        }
                    }
                } else {
                    const uint32_t dre = tmem + (uint32_t)(b * 256), dim = dre + 128;
                    const int nsteps = min(KC, Kh - kc * KC) / C::KSTEP;
                    for (int sk = 0; sk < nsteps; ++sk) {
                        const int k = kc * KC + sk * C::KSTEP;
                        for (int pr = 0; pr < C::NPROD; ++pr) {
                            const int ha = C::ha(pr), hz = C::hz(pr);
                            const uint32_t abase = a_base + (mb * nres + ha) * L.a_tiles * kATile;
                            const uint32_t are = abase + (k / C::ROWEL) * kATile + (k % C::ROWEL) * C::ES;
                            const uint32_t aim = abase + ((Kh + k) / C::ROWEL) * kATile + ((Kh + k) % C::ROWEL) * C::ES;
                            // K step = KSTEP rows of 128 bytes (2048 bytes for 16-bit, 4096 for 8-bit)
                            const uint32_t zre = st + ((0 * C::NHZ + hz) * C::HALVES) * KC * 128 + sk * C::KSTEP * 128;
                            const uint32_t zim = st + ((1 * C::NHZ + hz) * C::HALVES) * KC * 128 + sk * C::KSTEP * 128;
                            uint64_t dAre, dAim;
                            if (los && ha == 1) {
                                // A lo of this stage: 128 rows x KC columns; KC = 16: 32-byte rows, 32-byte swizzle
                                // (8-row atoms of 256 bytes); KC = 32: 64-byte rows, 64-byte swizzle (atoms of 512
                                // bytes), K step sk 32 bytes into the row
                                const uint32_t lo_re = st + zst_bytes + sk * 32, lo_im = lo_re + 128 * KC * 2;
                                if (KC == 16) {
                                    dAre = smem_desc(lo_re, 16, 256, 6);
                                    dAim = smem_desc(lo_im, 16, 256, 6);
                                } else {
                                    dAre = smem_desc(lo_re, 16, 512, 4);
                                    dAim = smem_desc(lo_im, 16, 512, 4);
                                }
                            } else {
                                dAre = smem_desc(are, 16, 1024, 2);
                                dAim = smem_desc(aim, 16, 1024, 2);
                            }
                            const uint64_t dZre = smem_desc(zre, (uint32_t)KC * 128u, 1024, 2);
                            const uint64_t dZim = smem_desc(zim, (uint32_t)KC * 128u, 1024, 2);
                            const uint32_t acc = (kc > 0 || sk > 0 || pr > 0) ? 1u : 0u;
                            if constexpr (C::F8) {
                                umma_f8(dre, dAre, dZre, idesc, acc);
                                umma_f8(dre, dAim, dZim, idesc_neg, 1u);
                                umma_f8(dim, dAim, dZre, idesc, acc);
                                umma_f8(dim, dAre, dZim, idesc, 1u);
                            } else {
                                umma_f16(dre, dAre, dZre, idesc, acc);
                                umma_f16(dre, dAim, dZim, idesc_neg, 1u);
                                umma_f16(dim, dAim, dZre, idesc, acc);
                                umma_f16(dim, dAre, dZim, idesc, 1u);
                            }
                        }
                    }
                }
            };
            // this item's accumulators must have been read out by the epilogue
            auto wait_tempty = [&](int i, int j) {
                const uint32_t u = (uint32_t)(j >> 1);
                if (!mbar_wait_bounded(&tempty[j & 1], (u & 1) ^ 1)) {
                    record_error(args.err, GWB_ERR_TIMEOUT, 204, blockIdx.x, i);
                    *abort_flag = 1;
                    return false;
                }
                tc_fence_after();
                return true;
            };
            auto wait_full = [&](int f) {
                if (*abort_flag || !mbar_wait_bounded(&full[f % S], (uint32_t)((f / S) & 1))) {
                    record_error(args.err, GWB_ERR_TIMEOUT, 203, blockIdx.x, f);
                    *abort_flag = 1;
                    return false;
                }
                tc_fence_after();
                return true;
            };
            // Two M blocks: when the Z ring holds a whole tile, M block 0 runs through all chunks before M block 1,
            // so block 0's MMAs overlap the epilogue of the previous tile's block 1 and block 1's the epilogue of
            // this tile's block 0. Otherwise both blocks go chunk by chunk.
            const bool mb_outer = MBe == 2 && S >= nkc;
            for (int i = 0; i < ntl && ok; ++i) {
                if (mb_outer) {
                    for (int mb = 0; mb < MBe && ok; ++mb) {
                        const int j = i * MBe + mb;
                        for (int kc = 0; kc < nkc && ok; ++kc) {
                            const int f = i * nkc + kc;
                            if (mb == 0 && !(ok = wait_full(f))) break;
                            if (kc == 0 && !(ok = wait_tempty(i, j))) break;
                            issue(kc, mb, j & 1, z_base + (f % S) * L.stage_bytes);
                            if (mb == MBe - 1) umma_commit(&empty[f % S]);
                        }
                        if (ok) umma_commit(&tfull[j & 1]);
                    }
                } else {
                    for (int kc = 0; kc < nkc && ok; ++kc) {
                        const int f = i * nkc + kc;
                        if (!(ok = wait_full(f))) break;
                        for (int mb = 0; mb < MBe && ok; ++mb) {
                            const int j = i * MBe + mb;
                            if (kc == 0 && !(ok = wait_tempty(i, j))) break;
                            issue(kc, mb, j & 1, z_base + (f % S) * L.stage_bytes);
                        }
                        umma_commit(&empty[f % S]);
                    }
                    if (ok)
                        for (int mb = 0; mb < MBe; ++mb) umma_commit(&tfull[(i * MBe + mb) & 1]);
                }
            }
            umma_commit(done);
            mbar_wait_bounded(done, 0);
        }
        __syncwarp();
    } else {
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
                    record_error(args.err, GWB_ERR_TIMEOUT, 205, blockIdx.x, i);
                    *abort_flag = 1;
                } else {
                    tc_fence_after();
#pragma unroll
                    for (int c = 0; c < 64; c += 32) {
                        uint32_t re[32], im[32];
                        tmem_ld_32x32b_x32(lane_base + (uint32_t)(b * 256 + hh * 64 + c), re);
                        tmem_ld_32x32b_x32(lane_base + (uint32_t)(b * 256 + 128 + hh * 64 + c), im);
                        tmem_ld_wait();
#pragma unroll
                        for (int jj = 0; jj < 32; ++jj) asm volatile("" : "+r"(re[jj]), "+r"(im[jj]));
                        const int cb = hh * 64 + c;
                        // best of this 32-column chunk first (index as an immediate), then merged: 2 FMA-pipe and 3
                        // ALU instructions per element
                        float lb = -1.f;
                        int lj = 0;
                        if (full_tile) {
#pragma unroll
                            for (int jj = 0; jj < 32; ++jj) {
                                const float xr = __uint_as_float(re[jj]), xm = __uint_as_float(im[jj]);
                                const float p = fmaf(xr, xr, xm * xm);
                                if (p > lb) {
                                    lb = p;
                                    lj = jj;
                                }
                            }
                        } else {
                            const int valid = (int)min((long long)32, max(0ll, args.Tn - (col0 + cb)));
#pragma unroll
                            for (int jj = 0; jj < 32; ++jj) {
                                const float xr = __uint_as_float(re[jj]), xm = __uint_as_float(im[jj]);
                                const float p = jj < valid ? fmaf(xr, xr, xm * xm) : -1.f;
                                if (p > lb) {
                                    lb = p;
                                    lj = jj;
                                }
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
                    const bool first = (t % args.group) == 0 || t == t_begin;
                    const bool last = ((t + 1) % args.group) == 0 || t == args.ntiles - 1 || t == t_end - 1;
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
                            const int w0 = (int)(o * args.group);
                            const int w1 = (int)min((long long)w0 + args.group, (long long)args.ntiles);
                            if (args.pv && (t_begin > w0 || t_end < w1)) {
                                const long long pidx = ((long long)row * gridDim.x + blockIdx.x) * 2 +
                                                       (t_begin > w0 ? 0 : 1);
                                args.pv[pidx] = wb;
                                args.pi[pidx] = wi;
                            } else {
                                float vo = wb;
                                if (args.rowscale) {
                                    const float rs = args.rowscale[row];
                                    vo = wb * rs * rs;
                                }
                                args.V[(long long)row * args.ldv + o] = vo;
                                args.I[(long long)row * args.ldv + o] = wi;
                            }
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

// ---------------------------------------------------------------------------------------------------------------------
// The CTA-pair form (fp16, bf16, and the split forms 2 and 6 with their two or three products per K step; their A lo
// resident beside A hi where three stages of 32 K rows fit, else streamed per CTA beside each Z stage): a cluster of
// two CTAs along x, M blocks 2p (rank 0) and 2p + 1 (rank 1) of the
// same time range (grid y). Each CTA keeps its own 128 rows of A resident and loads its own 64-sample half of every Z tile; rank 0
// issues tcgen05.mma.cta_group::2 with M = 256 (each SM computes its 128 rows over all 128 samples, the Z halves
// shared between the SMs), so per SM the MMAs read half the Z bytes from shared memory. Barriers: the loads of both
// CTAs complete on rank 0's full / barA barriers; MMA commits arrive on the barriers at the same offset in both
// CTAs (empty, tfull, done); both CTAs' epilogue warps arrive on rank 0's tempty. Every wait is bounded; every path
// reaches the final cluster barrier.
// ---------------------------------------------------------------------------------------------------------------------
// Shared memory of one CTA of a pair: A (nres resident copies of 128 rows x 2 Kh, 128-byte rows of 64 elements),
// stages of (re, im) x (nhz copies of Z) x KC rows x 64 samples (one 128-byte row each), followed, when A lo is
// streamed (los), by A lo (re, im) x 128 rows x KC columns as in the one-CTA kernel; the epilogue's exchange, the
// barriers.
__host__ __device__ inline Layout layout_pair(int Kh, int KC, int stages, int nres = 1, int nhz = 1, bool los = false) {
    Layout L;
    L.a_tiles = (uint32_t)((2 * Kh + 63) / 64);
    L.a_bytes = (uint32_t)nres * L.a_tiles * kATile;
    L.z_off = L.a_bytes;
    L.stage_bytes = 2u * (uint32_t)nhz * (uint32_t)KC * 128u + (los ? 2u * 128u * (uint32_t)KC * 2u : 0u);
    L.x_off = L.z_off + (uint32_t)stages * L.stage_bytes;
    L.bar_off = L.x_off + 2048u;
    L.total = L.bar_off + (uint32_t)(2 * stages + 6) * 8u + 16u;
    return L;
}

template <int FORM>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    umma_cplx2_kernel(const __grid_constant__ CplxArgs args) {
    using C = Cfg<FORM>;
    static_assert(!C::F8, "the CTA-pair form takes 16-bit products");
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    const int Kh = args.Kh, KC = args.KC, S = args.stages;
    const bool los = C::SPLIT_A && args.lo_stream != 0;   // A lo streamed beside each Z stage (KC = 16 or 32)
    const int nres = los ? 1 : C::NHA;                    // resident copies of A
    const Layout L = layout_pair(Kh, KC, S, nres, C::NHZ, los);
    const uint32_t zst_bytes = 2u * C::NHZ * (uint32_t)KC * 128u;   // the Z part of a stage
    const int nkc = (Kh + KC - 1) / KC;
    uint8_t* sA = smem;
    uint8_t* sZ = smem + L.z_off;
    float* xv = reinterpret_cast<float*>(smem + L.x_off);
    int* xi = reinterpret_cast<int*>(smem + L.x_off + 1024);
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
    const uint32_t rank = cluster_ctarank();
    const bool leader = rank == 0;
    // a timeout in either CTA stops both: the flag is set here and in the peer (through its shared::cluster address)
    const uint32_t peer_abort = mapa_shared(smem_u32((const void*)abort_flag), rank ^ 1u);
    auto abort_pair = [&]() {
        *abort_flag = 1;
        asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(peer_abort), "r"(1) : "memory");
    };
    // grid: x = M block (the pair along x: ranks 0, 1 = M blocks 2p, 2p + 1), y = time range
    const int m0 = blockIdx.x * 128;
    const int tr = blockIdx.y;
    const int t_begin = (int)((long long)tr * args.ntiles / gridDim.y);
    const int t_end = (int)((long long)(tr + 1) * args.ntiles / gridDim.y);
    const int ntl = t_end - t_begin;                         // the same in both CTAs of the pair
    const int nfill = ntl * nkc;
    const uint32_t a_bytes = L.a_bytes;                      // one CTA's resident A
    const uint32_t half_stage = L.stage_bytes;               // one CTA's half of a stage

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 2 * kEpiWarps);
        }
        mbar_init(barA, 1);
        mbar_init(done, 1);
        *abort_flag = 0;
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc_pair(tmem_slot, kTmemCols);
        tmem_relinquish_pair();
        tc_fence_before();
    }
    __syncthreads();
    cluster_sync_all();                                      // the peer's barriers are initialised before any arrival
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (ntl > 0 && warp == 0) {
        if (lane == 0) {
            for (int h = 0; h < C::NHA; ++h) prefetch_tmap(&args.tA[h]);
            for (int h = 0; h < C::NHZ; ++h) prefetch_tmap(&args.tZ[h]);
            const uint32_t barA_l = mapa_shared(smem_u32(barA), 0);
            if (leader) mbar_arrive_expect_tx(barA, 2u * a_bytes);
            for (int h = 0; h < nres; ++h)
                for (int a = 0; a < (int)L.a_tiles; ++a)
                    tma_load_2d_pair(sA + (h * L.a_tiles + a) * kATile, &args.tA[h], barA_l, a * C::ROWEL, m0);
            int issued = 0;
            for (int f = 0; f < nfill; ++f) {
                const int s = f % S;
                const uint32_t n = (uint32_t)(f / S);
                const int i = f / nkc, kc = f % nkc;
                if (*abort_flag) break;
                if (!mbar_wait_bounded(&empty[s], (n & 1) ^ 1)) {
                    record_error(args.err, GWB_ERR_TIMEOUT, 211, tr, f);
                    abort_pair();
                    break;
                }
                if (leader) mbar_arrive_expect_tx(&full[s], 2u * half_stage);
                const uint32_t full_l = mapa_shared(smem_u32(&full[s]), 0);
                const int x = (t_begin + i) * kTile + 64 * (int)rank;
                uint8_t* st = sZ + s * half_stage;
                for (int ri = 0; ri < 2; ++ri)
                    for (int h = 0; h < C::NHZ; ++h)
                        tma_load_2d_pair(st + (ri * C::NHZ + h) * KC * 128, &args.tZ[h], full_l, x, ri * Kh + kc * KC);
                if (los)            // this CTA's 128 rows of A lo, re then im columns of the K chunk
                    for (int ri = 0; ri < 2; ++ri)
                        tma_load_2d_pair(st + zst_bytes + ri * 128 * KC * 2, &args.tA[1], full_l, ri * Kh + kc * KC,
                                         m0);
                issued = f + 1;
            }
            // the loads of both CTAs complete on the leader's full barriers: before the final cluster barrier (after
            // which either CTA may exit) the leader waits, bounded, for the last phase of every stage it armed, so no
            // copy still targets a CTA's shared memory on the abort path either
            if (leader) {
                mbar_wait_bounded(barA, 0);
                for (int s = 0; s < S && s < issued; ++s) {
                    const int nf = (issued - s + S - 1) / S;
                    mbar_wait_bounded(&full[s], (uint32_t)((nf - 1) & 1));
                }
            }
        }
    } else if (ntl > 0 && warp == 1) {
        if (lane == 0 && leader) {
            const uint32_t idesc = instr_desc(256, 128, C::FMT, C::FMT, 0, 1);
            const uint32_t idesc_neg = idesc | (1u << 13);  // negate A
            const int order = args.order;
            const uint32_t a_base = smem_u32(sA), z_base = smem_u32(sZ);
            // descriptors of the resident A copies at K column 0 (the split forms add offsets to them)
            uint64_t ad0[2];
            for (int h = 0; h < 2; ++h) ad0[h] = smem_desc(a_base + (h < nres ? h : 0) * L.a_tiles * kATile, 16, 1024, 2);
            bool ok = mbar_wait_bounded(barA, 0);
            if (!ok) {
                record_error(args.err, GWB_ERR_TIMEOUT, 212, tr, 0);
                abort_pair();
            }
            tc_fence_after();
            for (int i = 0; i < ntl && ok; ++i) {
                const int b = i & 1;
                const uint32_t u = (uint32_t)(i >> 1);
                if (!mbar_wait_bounded(&tempty[b], (u & 1) ^ 1)) {
                    record_error(args.err, GWB_ERR_TIMEOUT, 214, tr, i);
                    abort_pair();
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t dre = tmem + (uint32_t)(b * 256), dim = dre + 128;
                for (int kc = 0; kc < nkc && ok; ++kc) {
                    const int f = i * nkc + kc;
                    if (*abort_flag || !mbar_wait_bounded(&full[f % S], (uint32_t)((f / S) & 1))) {
                        record_error(args.err, GWB_ERR_TIMEOUT, 213, tr, f);
                        abort_pair();
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = z_base + (f % S) * half_stage;
                    const int nsteps = min(KC, Kh - kc * KC) / C::KSTEP;
                    if constexpr (C::NPROD == 1) {
                        // descriptors of K step sk: A re / im halves (K-major), Z re / im halves (sample-major)
                        auto dA = [&](int sk, int im) {
                            const int k = (im ? Kh : 0) + kc * KC + sk * C::KSTEP;
                            return smem_desc(a_base + (k / C::ROWEL) * kATile + (k % C::ROWEL) * C::ES, 16, 1024, 2);
                        };
                        auto dZ = [&](int sk, int im) {
                            return smem_desc(st + (im ? KC * 128 : 0) + sk * C::KSTEP * 128, (uint32_t)KC * 128u, 1024, 2);
                        };
                        // the first MMA into each accumulator of a tile overwrites it
                        auto acc0 = [&](int sk) { return (kc > 0 || sk > 0) ? 1u : 0u; };
                        if (order == 1) {            // per K step, grouped by A half
                            for (int sk = 0; sk < nsteps; ++sk) {
                                umma_f16_pair(dre, dA(sk, 0), dZ(sk, 0), idesc, acc0(sk));
                                umma_f16_pair(dim, dA(sk, 0), dZ(sk, 1), idesc, acc0(sk));
                                umma_f16_pair(dre, dA(sk, 1), dZ(sk, 1), idesc_neg, 1u);
                                umma_f16_pair(dim, dA(sk, 1), dZ(sk, 0), idesc, 1u);
                            }
                        } else if (order == 2) {     // the chunk's real-part MMAs, then its imaginary-part MMAs
                            for (int sk = 0; sk < nsteps; ++sk) {
                                umma_f16_pair(dre, dA(sk, 0), dZ(sk, 0), idesc, acc0(sk));
                                umma_f16_pair(dre, dA(sk, 1), dZ(sk, 1), idesc_neg, 1u);
                            }
                            for (int sk = 0; sk < nsteps; ++sk) {
                                umma_f16_pair(dim, dA(sk, 0), dZ(sk, 1), idesc, acc0(sk));
                                umma_f16_pair(dim, dA(sk, 1), dZ(sk, 0), idesc, 1u);
                            }
                        } else if (order == 3) {     // one product at a time over the chunk's K steps
                            for (int sk = 0; sk < nsteps; ++sk) umma_f16_pair(dre, dA(sk, 0), dZ(sk, 0), idesc, acc0(sk));
                            for (int sk = 0; sk < nsteps; ++sk) umma_f16_pair(dre, dA(sk, 1), dZ(sk, 1), idesc_neg, 1u);
                            for (int sk = 0; sk < nsteps; ++sk) umma_f16_pair(dim, dA(sk, 0), dZ(sk, 1), idesc, acc0(sk));
                            for (int sk = 0; sk < nsteps; ++sk) umma_f16_pair(dim, dA(sk, 1), dZ(sk, 0), idesc, 1u);
                        } else {                     // per K step: re += ReA ReZ, re -= ImA ImZ, im += ImA ReZ, += ReA ImZ
                            for (int sk = 0; sk < nsteps; ++sk) {
                                umma_f16_pair(dre, dA(sk, 0), dZ(sk, 0), idesc, acc0(sk));
                                umma_f16_pair(dre, dA(sk, 1), dZ(sk, 1), idesc_neg, 1u);
                                umma_f16_pair(dim, dA(sk, 1), dZ(sk, 0), idesc, acc0(sk));
                                umma_f16_pair(dim, dA(sk, 0), dZ(sk, 1), idesc, 1u);
                            }
                        }
                    } else {
                        // split forms: per K step the products (ha, hz) in order, each as the four real MMAs;
                        // A hi (and A lo when resident) from the resident copies, A lo streamed from the stage. The
                        // chunk's descriptors (KC <= 32: at most two K steps) are formed first, then its MMAs go out
                        // back to back. A descriptor's start address is bits 0-13 (address >> 4), so a descriptor of
                        // the same layout at a higher address is the base descriptor plus the byte offset >> 4:
                        // one base per operand and chunk, the rest by additions (shared-memory addresses stay below
                        // 2^18, so the field does not carry)
                        // (K chunks of 64 with A resident: the chunk goes out in groups of two K steps)
                        constexpr int MAXS = 2;
                        const uint64_t zd = smem_desc(st, (uint32_t)KC * 128u, 1024, 2);
                        // A lo streamed: KC-column rows in the 32-, 64- or 128-byte swizzle (KC = 16, 32, 64)
                        const uint64_t lod = !los ? 0ull
                                             : KC == 16 ? smem_desc(st + zst_bytes, 16, 256, 6)
                                             : KC == 32 ? smem_desc(st + zst_bytes, 16, 512, 4)
                                                        : smem_desc(st + zst_bytes, 16, 1024, 2);
                        const auto koff = [](int kk) {     // byte offset of K column kk in the 64-column tiles
                            return (uint32_t)((kk / C::ROWEL) * kATile + (kk % C::ROWEL) * C::ES);
                        };
                        for (int s0 = 0; s0 < nsteps; s0 += MAXS) {
                            uint64_t dAr[MAXS][C::NPROD], dAi[MAXS][C::NPROD], dZr[MAXS][C::NPROD],
                                dZi[MAXS][C::NPROD];
#pragma unroll
                            for (int sk = 0; sk < MAXS; ++sk) {
                                const int ks = s0 + sk;             // K step within the chunk
                                const int k = kc * KC + ks * C::KSTEP;
                                const uint32_t ore = koff(k) >> 4, oim = koff(Kh + k) >> 4;
#pragma unroll
                                for (int pr = 0; pr < C::NPROD; ++pr) {
                                    const int ha = C::ha(pr), hz = C::hz(pr);
                                    if (los && ha == 1) {
                                        dAr[sk][pr] = lod + (uint64_t)(ks * 2);
                                        dAi[sk][pr] = lod + (uint64_t)(ks * 2 + ((128 * KC * 2) >> 4));
                                    } else {
                                        dAr[sk][pr] = ad0[ha] + (uint64_t)ore;
                                        dAi[sk][pr] = ad0[ha] + (uint64_t)oim;
                                    }
                                    dZr[sk][pr] = zd + (uint64_t)((((0 * C::NHZ + hz) * KC * 128) >> 4) +
                                                                  ks * C::KSTEP * 8);
                                    dZi[sk][pr] = zd + (uint64_t)((((1 * C::NHZ + hz) * KC * 128) >> 4) +
                                                                  ks * C::KSTEP * 8);
                                }
                            }
#pragma unroll
                            for (int sk = 0; sk < MAXS; ++sk) {
                                if (s0 + sk >= nsteps) break;
#pragma unroll
                                for (int pr = 0; pr < C::NPROD; ++pr) {
                                    const uint32_t acc = (kc > 0 || s0 + sk > 0 || pr > 0) ? 1u : 0u;
                                    umma_f16_pair(dre, dAr[sk][pr], dZr[sk][pr], idesc, acc);
                                    umma_f16_pair(dre, dAi[sk][pr], dZi[sk][pr], idesc_neg, 1u);
                                    umma_f16_pair(dim, dAi[sk][pr], dZr[sk][pr], idesc, acc);
                                    umma_f16_pair(dim, dAr[sk][pr], dZi[sk][pr], idesc, 1u);
                                }
                            }
                        }
                    }
                    umma_commit_pair(&empty[f % S]);
                }
                if (ok) umma_commit_pair(&tfull[b]);
            }
            umma_commit_pair(done);
        }
        __syncwarp();
        if (lane == 0 && !mbar_wait_bounded(done, 0)) {   // every MMA of the pair has completed
            record_error(args.err, GWB_ERR_TIMEOUT, 216, tr, (int)rank);
            abort_pair();
        }
        __syncwarp();
    } else if (ntl > 0) {
        const int q = warp & 3, hh = (warp - 2) >> 2;
        const int rl = 32 * q + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(32 * q) << 16);
        const uint32_t tempty_l0 = mapa_shared(smem_u32(&tempty[0]), 0);
        const uint32_t tempty_l1 = mapa_shared(smem_u32(&tempty[1]), 0);
        float wb = -1.f;
        int wi = 0;
        for (int i = 0; i < ntl; ++i) {
            const int t = t_begin + i;
            const long long col0 = (long long)t * kTile;
            const bool full_tile = col0 + kTile <= args.Tn;
            const int b = i & 1;
            const uint32_t u = (uint32_t)(i >> 1);
            float best = -1.f;
            int bi = 0;
            if (*abort_flag || !mbar_wait_bounded(&tfull[b], u & 1)) {
                record_error(args.err, GWB_ERR_TIMEOUT, 215, tr, i);
                abort_pair();
            } else {
                tc_fence_after();
#pragma unroll
                for (int c = 0; c < 64; c += 32) {
                    uint32_t re[32], im[32];
                    tmem_ld_32x32b_x32(lane_base + (uint32_t)(b * 256 + hh * 64 + c), re);
                    tmem_ld_32x32b_x32(lane_base + (uint32_t)(b * 256 + 128 + hh * 64 + c), im);
                    tmem_ld_wait();
#pragma unroll
                    for (int jj = 0; jj < 32; ++jj) asm volatile("" : "+r"(re[jj]), "+r"(im[jj]));
                    const int cb = hh * 64 + c;
                    const int valid = full_tile ? 32 : (int)min((long long)32, max(0ll, args.Tn - (col0 + cb)));
                    float lb = -1.f;
                    int lj = 0;
#pragma unroll
                    for (int jj = 0; jj < 32; ++jj) {
                        const float xr = __uint_as_float(re[jj]), xm = __uint_as_float(im[jj]);
                        const float p = jj < valid ? fmaf(xr, xr, xm * xm) : -1.f;
                        if (p > lb) {
                            lb = p;
                            lj = jj;
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
            if (lane == 0) mbar_arrive_cluster(b ? tempty_l1 : tempty_l0);
            if (hh == 1) {
                xv[b * 128 + rl] = best;
                xi[b * 128 + rl] = bi;
            }
            named_bar_sync(1, 32 * kEpiWarps);
            if (hh == 0) {
                const float ob = xv[b * 128 + rl];
                const int oi = xi[b * 128 + rl];
                if (ob > best) {
                    best = ob;
                    bi = oi;
                }
                const int gi = (int)(col0 + bi);
                const bool first = (t % args.group) == 0 || t == t_begin;
                const bool last = ((t + 1) % args.group) == 0 || t == args.ntiles - 1 || t == t_end - 1;
                if (first || best > wb) {
                    wb = best;
                    wi = gi;
                }
                const int row = m0 + rl;
                if (last && row < args.M) {
                    const long long o = t / args.group;
                    const int w0 = (int)(o * args.group);
                    const int w1 = (int)min((long long)w0 + args.group, (long long)args.ntiles);
                    if (args.pv && (t_begin > w0 || t_end < w1)) {
                        const long long pidx = ((long long)row * gridDim.y + tr) * 2 + (t_begin > w0 ? 0 : 1);
                        args.pv[pidx] = wb;
                        args.pi[pidx] = wi;
                    } else {
                        args.V[(long long)row * args.ldv + o] = wb;
                        args.I[(long long)row * args.ldv + o] = wi;
                    }
                }
            }
        }
    }
    __syncthreads();
    cluster_sync_all();                                      // no CTA leaves while its peer may still signal it
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc_pair(tmem, kTmemCols);
    }
}

// Windows cut by the tile-granular CTA ranges: per (row, window) whose first and last tiles lie in different CTAs,
// the maximum over the CTAs' partial records in CTA order (strictly greater replaces, so the first index wins ties as
// in one pass), then V (times rowscale^2 for fp8) and I.
__device__ __forceinline__ int cta_of_tile(int t, int ntiles, int g) {
    int c = (int)(((long long)t * g) / ntiles);
    while (c + 1 < g && (long long)(c + 1) * ntiles / g <= t) ++c;
    while (c > 0 && (long long)c * ntiles / g > t) --c;
    return c;
}

__global__ void window_merge_kernel(int M, int ntiles, int group, int nout, int g, const float* __restrict__ pv,
                                    const int32_t* __restrict__ pi, const float* __restrict__ rowscale,
                                    float* __restrict__ V, int32_t* __restrict__ I, long long ldv) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)M * nout) return;
    const int row = (int)(e / nout), o = (int)(e % nout);
    const int w0 = o * group, w1 = min(w0 + group, ntiles);
    const int ca = cta_of_tile(w0, ntiles, g), cb = cta_of_tile(w1 - 1, ntiles, g);
    if (ca == cb) return;
    float best = -1.f;
    int bi = 0;
    for (int c = ca; c <= cb; ++c) {
        const int tb = (int)((long long)c * ntiles / g);
        const long long pidx = ((long long)row * g + c) * 2 + (tb > w0 ? 0 : 1);
        const float v = pv[pidx];
        if (v > best) {
            best = v;
            bi = pi[pidx];
        }
    }
    if (rowscale) {
        const float rs = rowscale[row];
        best = best * rs * rs;
    }
    V[(long long)row * ldv + o] = best;
    I[(long long)row * ldv + o] = bi;
}

// Launch configuration per (form, Kh) from the autotuner's table (gwb_gemm_set_config). Defaults: CTA pairs for
// fp16 / bf16, the deepest Z ring that fits, the MMA order 0.
struct GemmTune {
    int form, kh, pair, stages, order;
};

GemmTune gemm_tune(int form, int kh) {
    // without a table entry: CTA pairs, except for fp16 with split A (one CTA per M block: measured 0.368 against
    // 0.404 ms at n = 256, Kh = 128; the pair is faster at Kh = 192, 0.569 against 0.616, where the autotuner picks
    // it); split bf16 with order 1, K chunks of 64 where A hi and lo stay resident (0.526 -> 0.488 ms at Kh = 128)
    GemmTune t{form, kh, form == 6 ? 0 : 1, 0, form == 2 ? 1 : 0};
    tune_lookup(form, kh, &t.pair, &t.stages, &t.order);
    return t;
}

// The tensor maps of the CTA-pair form: A (hi, lo) in boxes of 64 columns x 128 rows (128-byte swizzle), or A lo in
// boxes of KC columns when it is streamed; Z in boxes of 64 samples x KC rows.
template <int FORM>
int encode_pair_maps(CplxArgs& args, const void* const* A, const void* const* Zp, long long lda, long long ldz, int M,
                     long long Tn, bool los, int KC) {
    using C = Cfg<FORM>;
    const CUtensorMapDataType dt = C::FMT == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const int Kh = args.Kh;
    for (int h = 0; h < C::NHA; ++h) {
        const bool lo_box = los && h == 1;
        const int r = encode_tmap_2d(&args.tA[h], dt, A[h], (uint64_t)(2 * Kh), (uint64_t)M, (uint64_t)(lda * C::ES),
                                     lo_box ? (uint32_t)KC : (uint32_t)C::ROWEL, 128,
                                     !lo_box || KC == 64 ? CU_TENSOR_MAP_SWIZZLE_128B
                                     : KC == 32          ? CU_TENSOR_MAP_SWIZZLE_64B
                                                         : CU_TENSOR_MAP_SWIZZLE_32B);
        if (r) return r;
    }
    for (int h = 0; h < C::NHZ; ++h) {
        const int r = encode_tmap_2d(&args.tZ[h], dt, Zp[h], (uint64_t)Tn, (uint64_t)(2 * Kh), (uint64_t)(ldz * C::ES),
                                     C::ROWEL, (uint32_t)KC, CU_TENSOR_MAP_SWIZZLE_128B);
        if (r) return r;
    }
    return GWB_OK;
}

template <int FORM>
int launch_pair(CplxArgs args, const void* const* A, const void* const* Zp, long long lda, long long ldz, int M,
                long long ntiles, long long nout, int group, float* V, int32_t* I, long long ldv, void* work,
                long long work_bytes, const GemmTune& tune, cudaStream_t stream) {
    using C = Cfg<FORM>;
    const uint32_t max_smem = 227 * 1024;
    const int Kh = args.Kh;
    auto most = [&](int kc, int nres, bool ls) {
        int st = 8;
        while (st > 0 && layout_pair(Kh, kc, st, nres, C::NHZ, ls).total + 1024 > max_smem) --st;
        return st;
    };
    int KC = 64, stages = 0;
    bool los = false;
    if constexpr (C::SPLIT_A) {
        // order 1: A hi and lo resident with K chunks of 64 where two stages fit. Otherwise:
        // A hi and lo resident where three stages of 32 K rows fit beside them (or two, if the launch table asks for
        // two); else A lo streamed in K chunks of 32 (64-byte swizzle) beside each Z stage, or of 16
        KC = 32;
        const int sres = most(32, 2, false);
        if (tune.order == 1 && most(64, 2, false) >= 2) {
            // order 1: K chunks of 64 (A hi and lo resident), half the barrier round trips per MMA
            KC = 64;
            stages = most(64, 2, false);
        } else if (tune.order == 1 && most(64, 1, true) >= 2) {
            // order 1 where A hi and lo do not fit beside two stages of 64: A lo streamed in chunks of 64
            // (128-byte swizzle)
            KC = 64;
            los = true;
            stages = most(64, 1, true);
        } else if (sres >= 3 || (sres == 2 && tune.stages == 2)) {
            stages = sres;
        } else {
            los = true;
            stages = most(32, 1, true);
            if (stages < 2) {
                KC = 16;
                stages = most(16, 1, true);
            }
        }
        const int r = encode_pair_maps<FORM>(args, A, Zp, lda, ldz, M, args.Tn, los, KC);
        if (r) return r;
    } else {
        stages = most(KC, 1, false);
    }
    if (tune.stages >= 2) stages = std::min(stages, tune.stages);
    args.order = tune.order;
    args.lo_stream = los ? 1 : 0;
    GWB_CHECK_ARG(stages >= 2, GWB_ERR_SHAPE, "fused_peaks_cplx: Kh=%d does not fit the CTA-pair form", args.Kh);
    const int npair = (M + 255) / 256;
    const long long per = (long long)std::max(1, num_sms() / (2 * npair));
    const int gx = (int)std::max(1ll, std::min(ntiles, per));
    GWB_CHECK_ARG(work_bytes >= 16ll * M * gx, GWB_ERR_SHAPE, "fused_peaks_cplx: work %lld bytes, %lld needed",
                  work_bytes, 16ll * M * gx);
    args.stages = stages;
    args.KC = KC;
    args.MB = 1;
    args.pv = static_cast<float*>(work);
    args.pi = reinterpret_cast<int32_t*>(static_cast<char*>(work) + 8ll * M * gx);
    const uint32_t smem = layout_pair(args.Kh, KC, stages, los ? 1 : C::NHA, C::NHZ, los).total + 1024;
    auto kern = umma_cplx2_kernel<FORM>;
    GWB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<dim3(2 * npair, gx), kThreads, smem, stream>>>(args);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
        // what the occupancy calculator says about this cluster shape, for the message
        cudaLaunchConfig_t cfg;
        memset(&cfg, 0, sizeof(cfg));
        cfg.gridDim = dim3(2 * npair, gx);
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = smem;
        int nclusters = -1;
        cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg);
        cudaGetLastError();
        set_error("umma_cplx2_kernel launch (grid %d x %d, cluster 2 x 1, %u bytes of shared memory; max active "
                  "clusters %d): %s", 2 * npair, gx, smem, nclusters, cudaGetErrorString(le));
        return GWB_ERR_CUDA;
    }
    if (gx > 1) {
        bool any = false;
        for (int c = 1; c < gx && !any; ++c) any = ((long long)c * ntiles / gx) % group != 0;
        if (any) {
            const long long ne = (long long)M * nout;
            window_merge_kernel<<<(unsigned)cdiv(ne, 256), 256, 0, stream>>>(M, (int)ntiles, group, (int)nout, gx,
                                                                            args.pv, args.pi, nullptr, V, I, ldv);
            GWB_LAUNCH_CHECK("window_merge_kernel");
        }
    }
    return GWB_OK;
}

template <int FORM>
int launch_cplx(const void* const* A, const void* const* Zp, long long lda, long long ldz, int M, int Kh,
                long long Tn, int group, float* V, int32_t* I, long long ldv, const float* rowscale, void* work,
                long long work_bytes, cudaStream_t stream) {
    using C = Cfg<FORM>;
    GWB_CHECK_ARG(M > 0 && Tn > 0 && group > 0, GWB_ERR_SHAPE, "fused_peaks_cplx: M=%d Tn=%lld group=%d", M, Tn, group);
    GWB_CHECK_ARG(Kh > 0 && Kh % C::KSTEP == 0, GWB_ERR_SHAPE,
                  "fused_peaks_cplx: Kh=%d must be a positive multiple of %d", Kh, C::KSTEP);
    GWB_CHECK_ARG(lda >= 2 * Kh && ldz >= Tn, GWB_ERR_SHAPE, "fused_peaks_cplx: lda=%lld < 2 Kh or ldz=%lld < Tn", lda,
                  ldz);
    GWB_CHECK_ARG((lda * C::ES) % 16 == 0 && (ldz * C::ES) % 16 == 0, GWB_ERR_ALIGN,
                  "fused_peaks_cplx: lda=%lld and ldz=%lld must be multiples of 16 bytes", lda, ldz);
    GWB_CHECK_ARG(!C::F8 || rowscale, GWB_ERR_ARG, "fused_peaks_cplx: the fp8 form needs the row scales of A");
    for (int h = 0; h < C::NHA; ++h)
        GWB_CHECK_ARG(A[h] && aligned(A[h], 16), GWB_ERR_ALIGN, "fused_peaks_cplx: A operand %d misaligned", h);
    for (int h = 0; h < C::NHZ; ++h)
        GWB_CHECK_ARG(Zp[h] && aligned(Zp[h], 16), GWB_ERR_ALIGN, "fused_peaks_cplx: Z operand %d misaligned", h);
    GWB_CHECK_ARG(V && I, GWB_ERR_ARG, "fused_peaks_cplx: null output");
    const long long ntiles = cdiv(Tn, kTile);
    GWB_CHECK_ARG(ntiles * kTile < (1ll << 31), GWB_ERR_SHAPE, "fused_peaks_cplx: Tn too large for int32 indices");
    const long long nout = cdiv(ntiles, group);
    GWB_CHECK_ARG(ldv >= nout, GWB_ERR_SHAPE, "fused_peaks_cplx: ldv=%lld < outputs per row %lld", ldv, nout);
    const uint32_t max_smem = 227 * 1024;
    int KC = FORM == 2 ? 32 : (C::F8 ? 128 : 64);          // K rows per Z stage (32 KB per stage in every form)
    auto fits = [&](int mb, int st) {
        return layout_of(C::NHA, C::NHZ, mb, Kh, KC, st, C::ROWEL).total + 1024 <= max_smem;
    };
    auto most_stages = [&](int mb) {
        int st = 6;
        while (st > 0 && !fits(mb, st)) --st;
        return st;
    };
    // one M block per CTA: measured faster than two per CTA sharing each Z tile (0.285 vs 0.292 ms at n = 256, Kh =
    // 128, Tn = 917,504; the second M group's Z reads hit L2), with the TMEM double buffer spanning tiles. The kernel
    // also runs two M blocks per CTA (each Z tile read once for both) when MB = 2.
    const int MB = 1;
    const GemmTune tune = gemm_tune(FORM, Kh);
    int stages = most_stages(MB);
    if (tune.stages >= 2 && stages >= 2) stages = std::min(stages, tune.stages);
    // split A beyond Kh = 128: A hi + lo no longer fit beside the Z ring, so A lo is streamed with it
    const bool los = C::SPLIT_A && stages < 2;
    if (los) {
        // K chunks of 32 (A lo in 64-byte rows) when at least three stages fit, or two and the launch table asks for
        // two; else of 16 (32-byte rows). Measured at n = 256, r = 192, fp16 with split A: 0.64 ms with chunks of 32
        // against 0.90 with chunks of 16
        auto most_split = [&](int kc) {
            int st = 8;
            while (st > 0 && layout_split_stream(Kh, kc, st, C::NHZ).total + 1024 > max_smem) --st;
            return st;
        };
        const int s32 = most_split(32);
        KC = (s32 >= 3 || (s32 == 2 && tune.stages == 2)) ? 32 : 16;
        stages = most_split(KC);
        if (tune.stages >= 2) stages = std::min(stages, tune.stages);
    }
    GWB_CHECK_ARG(stages >= 2, GWB_ERR_SHAPE, "fused_peaks_cplx: Kh=%d does not fit in shared memory for this form",
                  Kh);
    CplxArgs args;
    memset(&args, 0, sizeof(args));
    const CUtensorMapDataType dt = C::F8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                   : C::FMT == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    for (int h = 0; h < C::NHA; ++h) {
        // A lo streamed: boxes of KC columns (32 or 64 bytes) x 128 rows, 32- or 64-byte swizzle
        const bool lo_box = los && h == 1;
        const int r = encode_tmap_2d(&args.tA[h], dt, A[h], (uint64_t)(2 * Kh), (uint64_t)M, (uint64_t)(lda * C::ES),
                                     lo_box ? (uint32_t)KC : (uint32_t)C::ROWEL, 128,
                                     !lo_box ? CU_TENSOR_MAP_SWIZZLE_128B
                                             : KC == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
        if (r) return r;
    }
    for (int h = 0; h < C::NHZ; ++h) {
        const int r = encode_tmap_2d(&args.tZ[h], dt, Zp[h], (uint64_t)Tn, (uint64_t)(2 * Kh), (uint64_t)(ldz * C::ES),
                                     C::ROWEL, (uint32_t)KC, CU_TENSOR_MAP_SWIZZLE_128B);
        if (r) return r;
    }
    args.V = V;
    args.rowscale = C::F8 ? rowscale : nullptr;
    args.I = I;
    args.ldv = ldv;
    args.Tn = Tn;
    args.M = M;
    args.Kh = Kh;
    args.ntiles = (int)ntiles;
    args.group = group;
    args.nout = (int)nout;
    args.stages = stages;
    args.MB = MB;
    args.KC = KC;
    args.lo_stream = los ? 1 : 0;
    args.err = device_error_ptr();
    const uint32_t smem = (los ? layout_split_stream(Kh, KC, stages, C::NHZ)
                               : layout_of(C::NHA, C::NHZ, MB, Kh, KC, stages, C::ROWEL)).total + 1024;
    auto kern = umma_cplx_kernel<FORM>;
    GWB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if constexpr (!C::F8) {
        if (work != nullptr && tune.pair)
            return launch_pair<FORM>(args, A, Zp, lda, ldz, M, ntiles, nout, group, V, I, ldv, work, work_bytes, tune,
                                     stream);
    }
    const int mgroups = (M + 128 * MB - 1) / (128 * MB);
    const long long per = (long long)std::max(1, num_sms() / mgroups);
    // with a workspace the CTA ranges are tile-granular (balanced to one tile; split windows merged afterwards),
    // without one they are whole windows (up to one window of imbalance)
    const bool split = work != nullptr;
    if (split) {
        GWB_CHECK_ARG(work_bytes >= 16ll * M * per, GWB_ERR_SHAPE,
                      "fused_peaks_cplx: work %lld bytes, %lld needed", work_bytes, 16ll * M * per);
        GWB_CHECK_ARG(aligned(work, 16), GWB_ERR_ALIGN, "fused_peaks_cplx: work misaligned");
    }
    const int gx = (int)std::max(1ll, std::min(split ? ntiles : nout, per));
    if (split) {
        args.pv = static_cast<float*>(work);
        args.pi = reinterpret_cast<int32_t*>(static_cast<char*>(work) + 8ll * M * gx);
    }
    kern<<<dim3(gx, mgroups), kThreads, smem, stream>>>(args);
    GWB_LAUNCH_CHECK("umma_cplx_kernel");
    if (split && gx > 1) {
        bool any = false;           // a range boundary inside a window
        for (int c = 1; c < gx && !any; ++c) any = ((long long)c * ntiles / gx) % group != 0;
        if (any) {
            const long long ne = (long long)M * nout;
            window_merge_kernel<<<(unsigned)cdiv(ne, 256), 256, 0, stream>>>(M, (int)ntiles, group, (int)nout, gx,
                                                                            args.pv, args.pi, args.rowscale, V, I,
                                                                            ldv);
            GWB_LAUNCH_CHECK("window_merge_kernel");
        }
    }
    return GWB_OK;
}

}  // namespace
}  // namespace gwb

extern "C" long long gwb_fused_peaks_cplx_work_bytes(int M) { return 16ll * M * gwb::num_sms(); }

extern "C" int gwb_fused_peaks_cplx(int form, const void* A_hi, const void* A_lo, long long lda, const void* Z_hi,
                                    const void* Z_lo, long long ldz, int M, int Kh, long long Tn, int group, float* V,
                                    int32_t* I, long long ldv, const float* rowscale, void* work,
                                    long long work_bytes, void* stream) {
    const void* A[2] = {A_hi, A_lo};
    const void* Z[2] = {Z_hi, Z_lo};
    cudaStream_t s = (cudaStream_t)stream;
    switch (form) {
        case 0:
            return gwb::launch_cplx<0>(A, Z, lda, ldz, M, Kh, Tn, group, V, I, ldv, rowscale, work, work_bytes,
                                        s);
        case 1:
            return gwb::launch_cplx<1>(A, Z, lda, ldz, M, Kh, Tn, group, V, I, ldv, rowscale, work, work_bytes,
                                        s);
        case 2:
            return gwb::launch_cplx<2>(A, Z, lda, ldz, M, Kh, Tn, group, V, I, ldv, rowscale, work, work_bytes,
                                        s);
        case 3:
            return gwb::launch_cplx<3>(A, Z, lda, ldz, M, Kh, Tn, group, V, I, ldv, rowscale, work, work_bytes,
                                        s);
        case 6:
            return gwb::launch_cplx<6>(A, Z, lda, ldz, M, Kh, Tn, group, V, I, ldv, rowscale, work, work_bytes,
                                        s);
        default:
            gwb::set_error("fused_peaks_cplx: form %d (0 fp16, 1 bf16, 2 split bf16, 3 fp8 e4m3, 6 fp16 with A "
                           "split)", form);
            return GWB_ERR_ARG;
    }
}
