// Chi-squared bin edges, binned sums at peaks and the exact-stage finalisation.
//
// edges (multi_filter.edges_per_template, pipeline/multi_filter.py:264-282; chisq_edges.edges_fused :92-143):
//   one block per unit (template row, segment): float64 sums of |h_k|^2 IP_k over contiguous per-thread chunks of
//   [kmin, k1), a block scan of the chunk sums, then every edge j < nb is the first k whose cumulative sum exceeds
//   j / nb of the total, found by walking only the chunk that holds it. Edges are clipped to [kmin, k1] and padded
//   with k1 up to B + 1 entries. The comparison is written as the reference writes it, so rounding at near-ties
//   follows it too: offset_mode 1 compares cs / tot + u > u + j / nb (the flattened searchsorted of
//   edges_per_template, u the unit's index), offset_mode 0 compares cs > (j / nb) tot (chisq_edges.py:70-82, 116-121).
// binned sums (chisq_kernel.bin_power_sums :17-121, exact_stage dense path :425-439, :734-739):
//   Z_j(t) = sum_{k in bin j} q_k exp(2 pi i ((k t) mod N) / N) with q_k = conj(h_k) D_k formed in registers (or q
//   given). Work item = (group of <= 8 peaks of one unit, chunk of kChunk bins); threads take k = base + tid + NT m
//   (coalesced) and advance each peak's phasor by a fixed rotation exp(2 pi i (NT t mod N) / N), reseeded exactly with
//   sincospif every kReseed steps (the reference's regen kernel uses the same recurrence-with-reseed, exact_stage.py
//   :548-585). Per bin the block reduces in a fixed order and writes one slot per (peak, chunk, bin).
// finalize: per peak, Z_j = sum over chunks of its slots (fp32, chunk order); z = sum_j Z_j and pw = sum_j |Z_j|^2
//   in float64; then snr = |z| norm, chisq = (nb pw - |z|^2) norm^2, dof = 2 nb - 2, newsnr, fpeak
//   (fp_filter.py:837-853, exact_stage.py:236-238, coinc_rank.py:39-46) with norm = 4 df / sqrt(sigma^2).
#include <atomic>
#include "common.cuh"

namespace gwb {
namespace {

constexpr int kEdgeThreads = 512;
constexpr int kSumThreads = 256;
constexpr int kChunk = 32768;
constexpr int kReseed = 16;
constexpr int kMaxPeaks = 8;
// the ordered binned sums stage their bands with bulk copies (gwb_exact_set_staging; the default, measured 126.6
// against 133.7 ms per C2 step with direct loads); process-wide
std::atomic<bool> g_exact_bulk{true};

__device__ __forceinline__ int count_of(const int32_t* dev, int host_max) {
    return dev ? min(*dev, host_max) : host_max;
}

__device__ __forceinline__ double wgt(const float2* h, const float* ip, long long k) {
    const float2 v = h[k];
    return ((double)v.x * (double)v.x + (double)v.y * (double)v.y) * (double)ip[k];
}

__global__ void __launch_bounds__(kEdgeThreads) edges_kernel(const GwbUnit* __restrict__ units, const int32_t* ucount,
                                                             int umax, const float2* __restrict__ H, long long ldh,
                                                             const float* __restrict__ IP, long long ldip,
                                                             const int32_t* __restrict__ nbins,
                                                             const int32_t* __restrict__ kmax, int kmin, int B,
                                                             int offset_mode, int32_t* __restrict__ E) {
    __shared__ double pre[kEdgeThreads + 1];
    const int nu = count_of(ucount, umax);
    const int t = threadIdx.x;
    for (int u = blockIdx.x; u < nu; u += gridDim.x) {
        const GwbUnit un = units[u];
        const float2* h = H + (long long)un.row * ldh;
        const float* ip = IP + (long long)un.seg * ldip;
        const int k1 = kmax[un.row];
        const int nb = max(nbins[un.row], 1);
        const int span = max(k1 - kmin, 0);
        const int chunk = (span + kEdgeThreads - 1) / kEdgeThreads;
        const int a = kmin + min(t * chunk, span), b = kmin + min((t + 1) * chunk, span);
        double s = 0.0;
        for (int k = a; k < b; ++k) s += wgt(h, ip, k);
        // inclusive scan of chunk sums (Hillis-Steele over the block, float64)
        pre[t + 1] = s;
        if (t == 0) pre[0] = 0.0;
        __syncthreads();
        for (int off = 1; off < kEdgeThreads; off <<= 1) {
            const double v = (t + 1 - off >= 1) ? pre[t + 1 - off] : 0.0;
            __syncthreads();
            pre[t + 1] += v;
            __syncthreads();
        }
        const double tot = pre[kEdgeThreads];
        const double uo = (double)u;
        int32_t* e = E + (long long)u * (B + 1);
        for (int j = t; j <= B; j += kEdgeThreads) {
            int ej = k1;
            if (j < nb) {
                // mode 1: cs / tot + u > u + j / nb (the reference's flattened searchsorted);
                // mode 0: cs > (j / nb) tot (its blocked and fused edge kernels)
                const double frac = (double)j / (double)nb;
                const double target = offset_mode ? uo + frac : frac * tot;
                auto above = [&](double cs) { return offset_mode ? (cs / tot + uo > target) : (cs > target); };
                // first chunk whose end-of-chunk sum is above the target
                int lo = 0, hi = kEdgeThreads;
                while (lo < hi) {
                    const int m = (lo + hi) >> 1;
                    if (above(pre[m + 1])) hi = m; else lo = m + 1;
                }
                ej = k1;
                for (int c = lo; c < kEdgeThreads; ++c) {
                    const int ca = kmin + min(c * chunk, span), cb = kmin + min((c + 1) * chunk, span);
                    double cs = pre[c];
                    int found = -1;
                    for (int k = ca; k < cb; ++k) {
                        cs += wgt(h, ip, k);
                        if (above(cs)) {
                            found = k;
                            break;
                        }
                    }
                    if (found >= 0) {
                        ej = found;
                        break;
                    }
                }
                ej = min(max(ej, kmin), k1);
                if (nbins[un.row] == 0 && j == 0) ej = kmin;
            }
            e[j] = ej;
        }
        __syncthreads();
    }
}

// bin index of k among edges e[0..nb]: -1 below e[0], nb at or above e[nb]
__device__ __forceinline__ int bin_of(const int32_t* e, int nb, int k) {
    int lo = 0, hi = nb + 1;
    while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (e[m] > k) hi = m; else lo = m + 1;
    }
    return lo - 1;
}

__global__ void __launch_bounds__(kSumThreads) binsum_kernel(const GwbGroup* __restrict__ groups, const int32_t* gcount,
                                                             int gmax, const GwbUnit* __restrict__ units,
                                                             const GwbCand* __restrict__ cands,
                                                             const int32_t* __restrict__ E, int B,
                                                             const int32_t* __restrict__ nbins,
                                                             const float2* __restrict__ H, long long ldh,
                                                             const float2* __restrict__ D, long long ldd, int kmin,
                                                             int nchunk, unsigned nmask, float inv_half_n,
                                                             const int32_t* __restrict__ order,
                                                             float2* __restrict__ slots) {
    __shared__ float2 red[kSumThreads / 32][kMaxPeaks];
    const int ng = count_of(gcount, gmax);
    const long long nitems = (long long)ng * nchunk;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (long long it = blockIdx.x; it < nitems; it += gridDim.x) {
        // group-major over the groups as given, or chunk-major over the groups in template-row order (order): the
        // items in flight then share a few rows' template chunks and every segment's data chunk in L2
        int g, c;
        if (order) {
            c = (int)(it / ng);
            g = order[(int)(it % ng)];
        } else {
            g = (int)(it / nchunk);
            c = (int)(it % nchunk);
        }
        const GwbGroup gr = groups[g];
        const GwbUnit un = units[gr.unit];
        const int np = gr.count;
        const int nb = max(nbins[un.row], 1);
        const int32_t* e = E + (long long)gr.unit * (B + 1);
        const int c0 = kmin + c * kChunk, c1 = c0 + kChunk;
        const int lo = max(c0, e[0]), hi = min(c1, e[nb]);
        if (lo >= hi) continue;   // uniform
        unsigned tp[kMaxPeaks];
        float2 rot[kMaxPeaks];
#pragma unroll
        for (int p = 0; p < kMaxPeaks; ++p) {
            tp[p] = p < np ? (unsigned)cands[gr.first + p].sample : 0u;
            float sn, cs;
            sincospif((float)(((unsigned)kSumThreads * tp[p]) & nmask) * inv_half_n, &sn, &cs);
            rot[p] = make_float2(cs, sn);
        }
        const float2* h = H + (long long)un.row * ldh;
        const float2* d = D ? D + (long long)un.seg * ldd : nullptr;
        int j = bin_of(e, nb, lo);
        int a = lo;
        while (a < hi) {   // uniform over the block: one bin sub-range at a time
            const int b = min(hi, e[j + 1]);
            float2 acc[kMaxPeaks];
            float2 w[kMaxPeaks];
#pragma unroll
            for (int p = 0; p < kMaxPeaks; ++p) acc[p] = make_float2(0.f, 0.f);
            int step = 0;
            for (int k = a + t; k < b; k += kSumThreads, ++step) {
                if ((step & (kReseed - 1)) == 0) {
#pragma unroll
                    for (int p = 0; p < kMaxPeaks; ++p) {
                        float sn, cs;
                        sincospif((float)(((unsigned)k * tp[p]) & nmask) * inv_half_n, &sn, &cs);
                        w[p] = make_float2(cs, sn);
                    }
                }
                float qx, qy;
                const float2 hk = h[k];
                if (d) {
                    const float2 dk = d[k];
                    qx = fmaf(hk.x, dk.x, hk.y * dk.y);      // conj(h) D
                    qy = fmaf(hk.x, dk.y, -(hk.y * dk.x));
                } else {
                    qx = hk.x;
                    qy = hk.y;
                }
#pragma unroll
                for (int p = 0; p < kMaxPeaks; ++p) {
                    if (p < np) {
                        acc[p].x = fmaf(qx, w[p].x, fmaf(-qy, w[p].y, acc[p].x));
                        acc[p].y = fmaf(qx, w[p].y, fmaf(qy, w[p].x, acc[p].y));
                        const float2 ww = w[p];
                        w[p] = make_float2(fmaf(ww.x, rot[p].x, -(ww.y * rot[p].y)), fmaf(ww.x, rot[p].y, ww.y * rot[p].x));
                    }
                }
            }
#pragma unroll
            for (int p = 0; p < kMaxPeaks; ++p) {
                float x = acc[p].x, y = acc[p].y;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    x += __shfl_down_sync(0xffffffffu, x, off);
                    y += __shfl_down_sync(0xffffffffu, y, off);
                }
                if (lane == 0) red[warp][p] = make_float2(x, y);
            }
            __syncthreads();
            if (t < np) {
                float x = 0.f, y = 0.f;
                for (int q = 0; q < kSumThreads / 32; ++q) {
                    x += red[q][t].x;
                    y += red[q][t].y;
                }
                slots[((long long)(gr.first + t) * nchunk + c) * B + j] = make_float2(x, y);
            }
            __syncthreads();
            a = b;
            ++j;
        }
    }
}

// The same binned sums with the template and data bands staged in shared memory by the bulk-copy (TMA) engine:
// every bin sub-range of an item is cut into tiles of kTile bins, and one thread issues cp.async.bulk copies of the
// tile's h and D runs (16-byte aligned: a run starts at the aligned address below its first bin and is rounded up to 16
// bytes, so it covers one bin more on either side at most, both inside the row) into one of two stages while the
// block computes the previous tile from the other. Each thread visits the same bins in the same order with the same
// recurrence and reseeds as binsum_kernel, so the slots are bit for bit the same. Every wait is bounded.
constexpr int kTile = 2048;
constexpr int kStage = kTile + 4;              // float2 per stage and operand (alignment slack)

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

__global__ void __launch_bounds__(kSumThreads) binsum_bulk_kernel(
    const GwbGroup* __restrict__ groups, const int32_t* gcount, int gmax, const GwbUnit* __restrict__ units,
    const GwbCand* __restrict__ cands, const int32_t* __restrict__ E, int B, const int32_t* __restrict__ nbins,
    const float2* __restrict__ H, long long ldh, const float2* __restrict__ D, long long ldd, int kmin, int nchunk,
    unsigned nmask, float inv_half_n, const int32_t* __restrict__ order, float2* __restrict__ slots,
    DeviceError* err) {
    __shared__ float2 red[kSumThreads / 32][kMaxPeaks];
    extern __shared__ __align__(16) float2 stg[];            // sh[2][kStage], then sd[2][kStage]
    float2 (*sh)[kStage] = reinterpret_cast<float2 (*)[kStage]>(stg);
    float2 (*sd)[kStage] = reinterpret_cast<float2 (*)[kStage]>(stg + 2 * kStage);
    __shared__ __align__(8) uint64_t full[2];
    __shared__ int s_off[2][2];                    // per stage: index of the tile's first bin in sh, sd
    __shared__ int s_abort;
    const int ng = count_of(gcount, gmax);
    const long long nitems = (long long)ng * nchunk;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        s_abort = 0;
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t issued = 0;                           // tiles issued by this CTA (stage = issued & 1)
    // thread 0: copy the h and D runs of bins [k0, k1) into the next stage
    auto issue = [&](const float2* h, const float2* d, int k0, int k1) {
        const int st = issued & 1;
        const uintptr_t ha = reinterpret_cast<uintptr_t>(h + k0) & ~(uintptr_t)15;
        const uintptr_t he = (reinterpret_cast<uintptr_t>(h + k1) + 15) & ~(uintptr_t)15;
        const uintptr_t da = reinterpret_cast<uintptr_t>(d + k0) & ~(uintptr_t)15;
        const uintptr_t de = (reinterpret_cast<uintptr_t>(d + k1) + 15) & ~(uintptr_t)15;
        s_off[st][0] = (int)((reinterpret_cast<uintptr_t>(h + k0) - ha) / sizeof(float2));
        s_off[st][1] = (int)((reinterpret_cast<uintptr_t>(d + k0) - da) / sizeof(float2));
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_expect_tx(&full[st], (uint32_t)((he - ha) + (de - da)));
        bulk_g2s(sh[st], reinterpret_cast<const void*>(ha), (uint32_t)(he - ha), &full[st]);
        bulk_g2s(sd[st], reinterpret_cast<const void*>(da), (uint32_t)(de - da), &full[st]);
        ++issued;
    };
    uint32_t consumed = 0;
    for (long long it = blockIdx.x; it < nitems; it += gridDim.x) {
        int g, c;
        if (order) {
            c = (int)(it / ng);
            g = order[(int)(it % ng)];
        } else {
            g = (int)(it / nchunk);
            c = (int)(it % nchunk);
        }
        const GwbGroup gr = groups[g];
        const GwbUnit un = units[gr.unit];
        const int np = gr.count;
        const int nb = max(nbins[un.row], 1);
        const int32_t* e = E + (long long)gr.unit * (B + 1);
        const int c0 = kmin + c * kChunk, c1 = c0 + kChunk;
        const int lo = max(c0, e[0]), hi = min(c1, e[nb]);
        if (lo >= hi) continue;   // uniform
        unsigned tp[kMaxPeaks];
        float2 rot[kMaxPeaks];
#pragma unroll
        for (int p = 0; p < kMaxPeaks; ++p) {
            tp[p] = p < np ? (unsigned)cands[gr.first + p].sample : 0u;
            float sn, cs;
            sincospif((float)(((unsigned)kSumThreads * tp[p]) & nmask) * inv_half_n, &sn, &cs);
            rot[p] = make_float2(cs, sn);
        }
        const float2* h = H + (long long)un.row * ldh;
        const float2* d = D + (long long)un.seg * ldd;
        int j = bin_of(e, nb, lo);
        int a = lo;
        // the item's tiles: bin sub-range [a, b) cut at a + kTile m; the first is issued here, each next one while
        // the current is computed
        int tb = min(min(hi, e[j + 1]), a + kTile);
        if (t == 0) issue(h, d, a, tb);
        while (a < hi) {
            const int b = min(hi, e[j + 1]);
            float2 acc[kMaxPeaks];
            float2 w[kMaxPeaks];
#pragma unroll
            for (int p = 0; p < kMaxPeaks; ++p) acc[p] = make_float2(0.f, 0.f);
            int step = 0;
            for (int ta = a; ta < b; ta += kTile) {
                const int te = min(b, ta + kTile);
                // the next tile: the rest of this sub-range, else the first bins of the next non-empty sub-range
                if (t == 0) {
                    if (te < b) {
                        issue(h, d, te, min(b, te + kTile));
                    } else if (b < hi) {
                        int jj = j + 1;
                        while (jj < nb && min(hi, e[jj + 1]) <= b) ++jj;   // empty bins hold no tile
                        issue(h, d, b, min(min(hi, e[jj + 1]), b + kTile));
                    }
                }
                const int st = consumed & 1;
                if (t == 0 && !mbar_wait_bounded(&full[st], (consumed >> 1) & 1)) {
                    record_error(err, GWB_ERR_TIMEOUT, 401, (int)blockIdx.x, (int)consumed);
                    s_abort = 1;
                    // the other stage's copy, if one was issued, must land before the block leaves
                    for (uint32_t u = consumed + 1; u < issued; ++u) mbar_wait_bounded(&full[u & 1], (u >> 1) & 1);
                }
                __syncthreads();
                if (s_abort) return;                       // uniform; the error word tells the host
                const float2* hs = sh[st] + s_off[st][0] - ta;
                const float2* ds = sd[st] + s_off[st][1] - ta;
                for (int k = ta + t; k < te; k += kSumThreads, ++step) {
                    if ((step & (kReseed - 1)) == 0) {
#pragma unroll
                        for (int p = 0; p < kMaxPeaks; ++p) {
                            float sn, cs;
                            sincospif((float)(((unsigned)k * tp[p]) & nmask) * inv_half_n, &sn, &cs);
                            w[p] = make_float2(cs, sn);
                        }
                    }
                    const float2 hk = hs[k], dk = ds[k];
                    const float qx = fmaf(hk.x, dk.x, hk.y * dk.y);      // conj(h) D
                    const float qy = fmaf(hk.x, dk.y, -(hk.y * dk.x));
#pragma unroll
                    for (int p = 0; p < kMaxPeaks; ++p) {
                        if (p < np) {
                            acc[p].x = fmaf(qx, w[p].x, fmaf(-qy, w[p].y, acc[p].x));
                            acc[p].y = fmaf(qx, w[p].y, fmaf(qy, w[p].x, acc[p].y));
                            const float2 ww = w[p];
                            w[p] = make_float2(fmaf(ww.x, rot[p].x, -(ww.y * rot[p].y)),
                                               fmaf(ww.x, rot[p].y, ww.y * rot[p].x));
                        }
                    }
                }
                ++consumed;
                __syncthreads();                           // the stage is free for the copy after next
            }
#pragma unroll
            for (int p = 0; p < kMaxPeaks; ++p) {
                float x = acc[p].x, y = acc[p].y;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    x += __shfl_down_sync(0xffffffffu, x, off);
                    y += __shfl_down_sync(0xffffffffu, y, off);
                }
                if (lane == 0) red[warp][p] = make_float2(x, y);
            }
            __syncthreads();
            if (t < np) {
                float x = 0.f, y = 0.f;
                for (int q = 0; q < kSumThreads / 32; ++q) {
                    x += red[q][t].x;
                    y += red[q][t].y;
                }
                slots[((long long)(gr.first + t) * nchunk + c) * B + j] = make_float2(x, y);
            }
            __syncthreads();
            a = b;
            ++j;
        }
    }
}

// Counting sort of the groups by template row (units[group.unit].row): counts, a one-block exclusive scan, scatter.
// The order within a row is whatever the atomics give; no result depends on it.
__global__ void group_count_kernel(const GwbGroup* __restrict__ groups, const int32_t* gcount, int gmax,
                                   const GwbUnit* __restrict__ units, int nrows, int32_t* __restrict__ cnt,
                                   int32_t* __restrict__ status) {
    const int ng = count_of(gcount, gmax);
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
        int row = units[groups[g].unit].row;
        if (row < 0 || row >= nrows) {           // flagged; sorted last so that the order stays a permutation
            atomicOr(status, 1);
            row = nrows - 1;
        }
        atomicAdd(&cnt[row], 1);
    }
}

__global__ void __launch_bounds__(1024) group_scan_kernel(const int32_t* __restrict__ cnt, int nrows,
                                                          int32_t* __restrict__ off) {
    __shared__ int part[1024];
    const int T = blockDim.x, tid = threadIdx.x;
    const int per = (nrows + T - 1) / T;
    const int b = tid * per, e = min(nrows, b + per);
    int s = 0;
    for (int k = b; k < e; ++k) s += cnt[k];
    part[tid] = s;
    __syncthreads();
    for (int d = 1; d < T; d <<= 1) {
        const int v = tid >= d ? part[tid - d] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int run = tid ? part[tid - 1] : 0;
    for (int k = b; k < e; ++k) {
        off[k] = run;
        run += cnt[k];
    }
}

__global__ void group_scatter_kernel(const GwbGroup* __restrict__ groups, const int32_t* gcount, int gmax,
                                     const GwbUnit* __restrict__ units, int nrows, const int32_t* __restrict__ off,
                                     int32_t* __restrict__ fill, int32_t* __restrict__ order) {
    const int ng = count_of(gcount, gmax);
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
        int row = units[groups[g].unit].row;
        if (row < 0 || row >= nrows) row = nrows - 1;
        order[off[row] + atomicAdd(&fill[row], 1)] = g;
    }
}

__global__ void finalize_kernel(const GwbCand* __restrict__ cands, const int32_t* ccount, int cmax,
                                const GwbUnit* __restrict__ units, const int32_t* __restrict__ E, int B,
                                const int32_t* __restrict__ nbins, int kmin, int nchunk,
                                const float2* __restrict__ slots, const double* __restrict__ sig, long long ldsig,
                                double df, GwbPeak* __restrict__ out) {
    const int n = count_of(ccount, cmax);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const GwbCand cd = cands[i];
        const GwbUnit un = units[cd.unit];
        const int nbr = nbins[un.row];
        const int nb = max(nbr, 1);
        const int32_t* e = E + (long long)cd.unit * (B + 1);
        const float2* sl = slots + (long long)i * nchunk * B;
        double zx = 0.0, zy = 0.0, pw = 0.0;
        for (int j = 0; j < nb; ++j) {
            if (e[j] >= e[j + 1]) continue;
            const int ca = (e[j] - kmin) / kChunk, cb = (e[j + 1] - 1 - kmin) / kChunk;
            float x = 0.f, y = 0.f;
            for (int c = ca; c <= cb; ++c) {
                x += sl[(long long)c * B + j].x;
                y += sl[(long long)c * B + j].y;
            }
            zx += x;
            zy += y;
            pw += (double)x * x + (double)y * y;
        }
        GwbPeak pk;
        pk.zr = (float)zx;
        pk.zi = (float)zy;
        pk.pw = (float)pw;
        const double z2 = zx * zx + zy * zy;
        double norm = 0.0;
        if (sig) norm = 4.0 * df / sqrt(sig[(long long)un.row * ldsig + un.seg]);
        const double snr = sqrt(z2) * norm;
        const double chisq = ((double)nbr * (double)pk.pw - z2) * norm * norm;
        const int dof = 2 * nbr - 2;
        double ns = snr;
        const double rchisq = chisq / (double)max(dof, 1);
        if (rchisq > 1.0) ns = snr / pow((1.0 + rchisq * rchisq * rchisq) / 2.0, 1.0 / 6.0);
        pk.snr = (float)snr;
        pk.chisq = (float)chisq;
        pk.newsnr = (float)ns;
        pk.dof = dof;
        pk.fpeak = (float)((2.0 * e[max(nbr - 1, 0)] - e[max(nbr - 2, 0)]) * df);
        out[i] = pk;
    }
}

}  // namespace
}  // namespace gwb

extern "C" {

int gwb_edges(const GwbUnit* units, const int32_t* ucount, int umax, const float* H, long long ldh, const float* IP,
              long long ldip, const int32_t* nbins, const int32_t* kmax, int kmin, int B, int offset_mode, int32_t* E,
              void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(units && H && IP && nbins && kmax && E, GWB_ERR_ARG, "edges: null pointer");
    GWB_CHECK_ARG(umax >= 0 && B >= 1 && kmin >= 0, GWB_ERR_SHAPE, "edges: umax=%d B=%d kmin=%d", umax, B, kmin);
    if (umax == 0) return GWB_OK;
    const int grid = std::min(umax, 8 * num_sms());
    edges_kernel<<<grid, kEdgeThreads, 0, (cudaStream_t)stream>>>(units, ucount, umax, reinterpret_cast<const float2*>(H),
                                                                  ldh, IP, ldip, nbins, kmax, kmin, B, offset_mode, E);
    GWB_LAUNCH_CHECK("edges_kernel");
    return GWB_OK;
}

int gwb_bin_sums(const GwbGroup* groups, const int32_t* gcount, int gmax, const GwbUnit* units, const GwbCand* cands,
                 const int32_t* E, int B, const int32_t* nbins, const float* H, long long ldh, const float* D,
                 long long ldd, int kmin, int flen, long long tlen, float* slots, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(groups && units && cands && E && nbins && H && slots, GWB_ERR_ARG, "bin_sums: null pointer");
    GWB_CHECK_ARG(is_pow2(tlen) && tlen <= (1ll << 31), GWB_ERR_NOT_POW2, "bin_sums: time length %lld is not a power of two",
                  tlen);
    GWB_CHECK_ARG(gmax >= 0 && B >= 1 && flen > kmin, GWB_ERR_SHAPE, "bin_sums: gmax=%d B=%d flen=%d kmin=%d", gmax, B,
                  flen, kmin);
    if (gmax == 0) return GWB_OK;
    const int nchunk = (int)cdiv(flen - kmin, kChunk);
    const long long items = (long long)gmax * nchunk;
    const int grid = (int)std::min<long long>(items, 16ll * num_sms());
    binsum_kernel<<<grid, kSumThreads, 0, (cudaStream_t)stream>>>(
        groups, gcount, gmax, units, cands, E, B, nbins, reinterpret_cast<const float2*>(H), ldh,
        reinterpret_cast<const float2*>(D), ldd, kmin, nchunk, (unsigned)(tlen - 1), (float)(2.0 / (double)tlen),
        nullptr, reinterpret_cast<float2*>(slots));
    GWB_LAUNCH_CHECK("binsum_kernel");
    return GWB_OK;
}

long long gwb_bin_sums_work_bytes(int gmax, int nrows) {
    if (gmax < 0 || nrows <= 0) return -1;
    return 4ll * (3ll * nrows + (long long)gmax + 4);
}

int gwb_bin_sums_ordered(const GwbGroup* groups, const int32_t* gcount, int gmax, const GwbUnit* units,
                         const GwbCand* cands, const int32_t* E, int B, const int32_t* nbins, int nrows,
                         const float* H, long long ldh, const float* D, long long ldd, int kmin, int flen,
                         long long tlen, void* work, long long work_bytes, int32_t* status, float* slots,
                         void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(groups && units && cands && E && nbins && H && D && slots && work && status, GWB_ERR_ARG,
                  "bin_sums_ordered: null pointer");
    GWB_CHECK_ARG(is_pow2(tlen) && tlen <= (1ll << 31), GWB_ERR_NOT_POW2,
                  "bin_sums_ordered: time length %lld is not a power of two", tlen);
    GWB_CHECK_ARG(gmax >= 0 && B >= 1 && flen > kmin && nrows > 0, GWB_ERR_SHAPE,
                  "bin_sums_ordered: gmax=%d B=%d flen=%d kmin=%d nrows=%d", gmax, B, flen, kmin, nrows);
    GWB_CHECK_ARG(work_bytes >= gwb_bin_sums_work_bytes(gmax, nrows), GWB_ERR_SHAPE,
                  "bin_sums_ordered: work %lld bytes, %lld needed", work_bytes, gwb_bin_sums_work_bytes(gmax, nrows));
    cudaStream_t s = (cudaStream_t)stream;
    GWB_CUDA(cudaMemsetAsync(status, 0, sizeof(int32_t), s));
    if (gmax == 0) return GWB_OK;
    int32_t* cnt = static_cast<int32_t*>(work);
    int32_t* fill = cnt + nrows;
    int32_t* off = fill + nrows;
    int32_t* order = off + nrows;
    GWB_CUDA(cudaMemsetAsync(cnt, 0, 8ll * nrows, s));    // cnt and fill
    const int gs = (int)std::min<long long>(cdiv(gmax, 256), 4ll * num_sms());
    group_count_kernel<<<gs, 256, 0, s>>>(groups, gcount, gmax, units, nrows, cnt, status);
    GWB_LAUNCH_CHECK("group_count_kernel");
    group_scan_kernel<<<1, 1024, 0, s>>>(cnt, nrows, off);
    GWB_LAUNCH_CHECK("group_scan_kernel");
    group_scatter_kernel<<<gs, 256, 0, s>>>(groups, gcount, gmax, units, nrows, off, fill, order);
    GWB_LAUNCH_CHECK("group_scatter_kernel");
    const int nchunk = (int)cdiv(flen - kmin, kChunk);
    const long long items = (long long)gmax * nchunk;
    const int grid = (int)std::min<long long>(items, 16ll * num_sms());
    if (g_exact_bulk.load()) {
        const size_t smem = 4 * kStage * sizeof(float2);
        GWB_CUDA(cudaFuncSetAttribute(binsum_bulk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        binsum_bulk_kernel<<<grid, kSumThreads, smem, s>>>(
            groups, gcount, gmax, units, cands, E, B, nbins, reinterpret_cast<const float2*>(H), ldh,
            reinterpret_cast<const float2*>(D), ldd, kmin, nchunk, (unsigned)(tlen - 1), (float)(2.0 / (double)tlen),
            order, reinterpret_cast<float2*>(slots), device_error_ptr());
        GWB_LAUNCH_CHECK("binsum_bulk_kernel");
        return GWB_OK;
    }
    binsum_kernel<<<grid, kSumThreads, 0, s>>>(
        groups, gcount, gmax, units, cands, E, B, nbins, reinterpret_cast<const float2*>(H), ldh,
        reinterpret_cast<const float2*>(D), ldd, kmin, nchunk, (unsigned)(tlen - 1), (float)(2.0 / (double)tlen),
        order, reinterpret_cast<float2*>(slots));
    GWB_LAUNCH_CHECK("binsum_kernel");
    return GWB_OK;
}

int gwb_exact_set_staging(int bulk) {
    gwb::g_exact_bulk.store(bulk != 0);
    return GWB_OK;
}

int gwb_exact_finalize(const GwbCand* cands, const int32_t* ccount, int cmax, const GwbUnit* units, const int32_t* E,
                       int B, const int32_t* nbins, int kmin, int flen, const float* slots, const double* sig,
                       long long ldsig, double df, GwbPeak* out, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(cands && units && E && nbins && slots && out, GWB_ERR_ARG, "exact_finalize: null pointer");
    GWB_CHECK_ARG(cmax >= 0 && B >= 1 && flen > kmin, GWB_ERR_SHAPE, "exact_finalize: cmax=%d", cmax);
    if (cmax == 0) return GWB_OK;
    const int nchunk = (int)cdiv(flen - kmin, kChunk);
    const int grid = (int)std::min<long long>(cdiv(cmax, 128), 4ll * num_sms());
    finalize_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(cands, ccount, cmax, units, E, B, nbins, kmin, nchunk,
                                                             reinterpret_cast<const float2*>(slots), sig, ldsig, df, out);
    GWB_LAUNCH_CHECK("finalize_kernel");
    return GWB_OK;
}

int gwb_exact_chunks(int flen, int kmin) { return (int)gwb::cdiv(flen - kmin, gwb::kChunk); }

}  // extern "C"
