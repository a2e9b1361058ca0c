// Exact-stage selection by rank: per segment, only the k loudest candidates (by rebuilt SNR) go to the exact stage,
// the rest keep their rebuilt SNR and phase (as the reference's rebuilt peaks, pipeline/fp_filter.py:772-781).
// k is a fixed count ("exact stage on the top N peaks") or a fraction of the segment's candidates ("recompute the top
// p of the peaks per chunk"). The reference itself selects by a rebuilt-SNR cut (fp_filter.py:769-770); this is the
// rank form of the same split.
//
// Input: the selection's lists of one step (candidates, units, groups, counters as gwb_select_windows writes them;
// every candidate carries its rebuilt z). Steps, all on the caller's stream, with every size read from the device
// counters (no host synchronisation):
//   1. count the candidates of each segment; 2. scan the counts; 3. scatter each candidate's rebuilt SNR (as its
//   float bits, which order like the values for non-negative floats) into its segment's range;
//   4. per segment, the k-th largest value by a four-pass radix select over the 8-bit digits (tau; all candidates of
//   a segment with k >= its count are kept, tau = 0);
//   5. per input unit, in candidate order: approx >= tau[seg] stays an exact-stage candidate (new unit, groups of <=
//   8), otherwise it becomes a rebuilt peak when approx > rthr, else it is dropped.
#include "common.cuh"

namespace gwb {
namespace {

constexpr int kT = 256;

__global__ void seg_count_kernel(const GwbCand* __restrict__ c, const int32_t* __restrict__ n_in, int nseg,
                                 int32_t* __restrict__ cnt, int32_t* __restrict__ bad) {
    const int n = *n_in;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = c[i].seg;
        if (s < 0 || s >= nseg) {
            atomicOr(bad, 1);
            continue;
        }
        atomicAdd(&cnt[s], 1);
    }
}

// exclusive scan of nseg counts by one CTA (chunks of kT with a running total)
__global__ void seg_scan_kernel(const int32_t* __restrict__ cnt, int nseg, int32_t* __restrict__ off,
                                int32_t* __restrict__ fill) {
    __shared__ int32_t part[kT];
    __shared__ int32_t base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (int s0 = 0; s0 < nseg; s0 += kT) {
        const int s = s0 + threadIdx.x;
        const int v = s < nseg ? cnt[s] : 0;
        part[threadIdx.x] = v;
        __syncthreads();
        for (int d = 1; d < kT; d <<= 1) {
            const int add = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
            __syncthreads();
            part[threadIdx.x] += add;
            __syncthreads();
        }
        if (s < nseg) {
            off[s] = base + part[threadIdx.x] - v;
            fill[s] = 0;
        }
        __syncthreads();
        if (threadIdx.x == kT - 1) base += part[kT - 1];
        __syncthreads();
    }
}

__global__ void seg_scatter_kernel(const GwbCand* __restrict__ c, const int32_t* __restrict__ n_in, int nseg,
                                   const int32_t* __restrict__ off, int32_t* __restrict__ fill,
                                   uint32_t* __restrict__ keys) {
    const int n = *n_in;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = c[i].seg;
        if (s < 0 || s >= nseg) continue;
        const float a = fmaxf(c[i].approx, 0.f);
        keys[off[s] + atomicAdd(&fill[s], 1)] = __float_as_uint(a);
    }
}

// tau[s] = the k-th largest key of segment s (k = top_n, or ceil(frac * count) when top_n <= 0)
__global__ void seg_radix_select_kernel(const uint32_t* __restrict__ keys, const int32_t* __restrict__ cnt,
                                        const int32_t* __restrict__ off, int top_n, float frac,
                                        float* __restrict__ tau) {
    __shared__ int32_t hist[256];
    __shared__ uint32_t s_prefix, s_mask;
    __shared__ int32_t s_k;
    const int s = blockIdx.x;
    const int n = cnt[s];
    const uint32_t* key = keys + off[s];
    int k = top_n > 0 ? top_n : (int)ceilf(frac * (float)n);
    if (k < 1) k = 1;
    if (n <= k) {
        if (threadIdx.x == 0) tau[s] = 0.f;
        return;
    }
    if (threadIdx.x == 0) {
        s_prefix = 0u;
        s_mask = 0u;
        s_k = k;
    }
    __syncthreads();
    for (int shift = 24; shift >= 0; shift -= 8) {
        hist[threadIdx.x] = 0;
        __syncthreads();
        const uint32_t prefix = s_prefix, mask = s_mask;
        for (int i = threadIdx.x; i < n; i += kT) {
            const uint32_t v = key[i];
            if ((v & mask) == prefix) atomicAdd(&hist[(v >> shift) & 255u], 1);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int kk = s_k, d = 255;
            for (; d > 0; --d) {               // from the largest digit down: the digit holding the kk-th largest
                if (hist[d] >= kk) break;
                kk -= hist[d];
            }
            s_k = kk;
            s_prefix = prefix | ((uint32_t)d << shift);
            s_mask = mask | (255u << shift);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) tau[s] = __uint_as_float(s_prefix);
}

// one CTA per input unit (grid-stride over the device count); ordered compaction as in the selection kernel
__global__ void top_compact_kernel(const GwbCand* __restrict__ cin, const GwbUnit* __restrict__ uin,
                                   const int32_t* __restrict__ cnt_in, const float* __restrict__ tau, float rthr,
                                   GwbCand* __restrict__ cout, int cand_cap, GwbGroup* __restrict__ gout, int group_cap,
                                   GwbUnit* __restrict__ uout, int unit_cap, GwbCand* __restrict__ rebuilt,
                                   int rebuilt_cap, int32_t* __restrict__ counters) {
    __shared__ int s_cnt[2], s_base, s_gbase, s_unit, s_rbase, s_ok;
    __shared__ int s_warp[kT / 32];
    const int nu = cnt_in[2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int u = blockIdx.x; u < nu; u += gridDim.x) {
        const GwbUnit U = uin[u];
        const float t = tau[U.seg];
        auto cls = [&](int i) -> int {
            const float a = cin[U.first + i].approx;
            return a >= t ? 1 : (a > rthr ? 2 : 0);
        };
        if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0;
        __syncthreads();
        int ce = 0, cr = 0;
        for (int i = threadIdx.x; i < U.count; i += kT) {
            const int c = cls(i);
            ce += c == 1;
            cr += c == 2;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ce += __shfl_down_sync(0xffffffffu, ce, o);
            cr += __shfl_down_sync(0xffffffffu, cr, o);
        }
        if (lane == 0) {
            atomicAdd(&s_cnt[0], ce);
            atomicAdd(&s_cnt[1], cr);
        }
        __syncthreads();
        const int total = s_cnt[0], rtotal = s_cnt[1];
        const int ng = (total + 7) / 8;
        if (threadIdx.x == 0) {
            int ok = 0;
            if (total > 0) {
                s_base = atomicAdd(&counters[0], total);
                s_gbase = atomicAdd(&counters[1], ng);
                s_unit = atomicAdd(&counters[2], 1);
                if (s_base + total > cand_cap || s_gbase + ng > group_cap || s_unit >= unit_cap)
                    atomicOr(&counters[3], 1);
                else {
                    uout[s_unit] = GwbUnit{U.row, U.seg, s_base, total};
                    ok |= 1;
                }
            }
            if (rtotal > 0) {
                s_rbase = atomicAdd(&counters[4], rtotal);
                if (rebuilt == nullptr || s_rbase + rtotal > rebuilt_cap) atomicOr(&counters[3], 1);
                else ok |= 2;
            }
            s_ok = ok;
        }
        __syncthreads();
        const int okf = s_ok;
        if (okf & 1)
            for (int g = threadIdx.x; g < ng; g += kT)
                gout[s_gbase + g] = GwbGroup{s_unit, s_base + 8 * g, min(8, total - 8 * g), 0};
        for (int want = 1; want <= 2; ++want) {
            if (!(okf & want)) continue;            // uniform over the CTA
            GwbCand* out = want == 1 ? cout + s_base : rebuilt + s_rbase;
            const int unit = want == 1 ? s_unit : -1;
            int written = 0;
            for (int i0 = 0; i0 < U.count; i0 += kT) {
                const int i = i0 + threadIdx.x;
                const bool hit = i < U.count && cls(i) == want;
                const unsigned m = __ballot_sync(0xffffffffu, hit);
                if (lane == 0) s_warp[warp] = __popc(m);
                __syncthreads();
                int before = 0, chunk_total = 0;
                for (int w = 0; w < kT / 32; ++w) {
                    before += w < warp ? s_warp[w] : 0;
                    chunk_total += s_warp[w];
                }
                if (hit) {
                    GwbCand cd = cin[U.first + i];
                    cd.unit = unit;
                    out[written + before + __popc(m & ((1u << lane) - 1))] = cd;
                }
                written += chunk_total;
                __syncthreads();
            }
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace gwb

extern "C" {

long long gwb_select_top_work_bytes(int nseg, int cand_cap) {
    // cnt, off, fill (nseg int32 each), tau (nseg float), bad flag, keys (cand_cap uint32), each 256-byte aligned
    const long long a = ((4ll * nseg + 255) / 256) * 256;
    return 4 * a + 256 + ((4ll * cand_cap + 255) / 256) * 256;
}

int gwb_select_top(const GwbCand* cands, const GwbGroup* groups, const GwbUnit* units, const int32_t* counters,
                   int cand_cap, int nseg, int top_n, float top_frac, float rthr, GwbCand* cands_out,
                   GwbGroup* groups_out, GwbUnit* units_out, int32_t* counters_out, GwbCand* rebuilt, int rebuilt_cap,
                   void* work, long long work_bytes, void* stream) {
    using namespace gwb;
    (void)groups;
    GWB_CHECK_ARG(cands && units && counters && cands_out && groups_out && units_out && counters_out && work,
                  GWB_ERR_ARG, "select_top: null pointer");
    GWB_CHECK_ARG(nseg > 0 && cand_cap > 0, GWB_ERR_SHAPE, "select_top: nseg=%d cand_cap=%d", nseg, cand_cap);
    GWB_CHECK_ARG(top_n > 0 || (top_frac > 0.f && top_frac <= 1.f), GWB_ERR_ARG,
                  "select_top: top_n=%d top_frac=%g (one of a positive count or a fraction in (0, 1])", top_n,
                  (double)top_frac);
    const long long need = gwb_select_top_work_bytes(nseg, cand_cap);
    GWB_CHECK_ARG(work_bytes >= need && aligned(work, 256), GWB_ERR_SHAPE,
                  "select_top: work %lld bytes (256-byte aligned), %lld needed", work_bytes, need);
    cudaStream_t s = (cudaStream_t)stream;
    char* w = static_cast<char*>(work);
    const long long a = ((4ll * nseg + 255) / 256) * 256;
    int32_t* cnt = reinterpret_cast<int32_t*>(w);
    int32_t* off = reinterpret_cast<int32_t*>(w + a);
    int32_t* fill = reinterpret_cast<int32_t*>(w + 2 * a);
    float* tau = reinterpret_cast<float*>(w + 3 * a);
    int32_t* bad = reinterpret_cast<int32_t*>(w + 4 * a);
    uint32_t* keys = reinterpret_cast<uint32_t*>(w + 4 * a + 256);
    GWB_CUDA(cudaMemsetAsync(cnt, 0, 4ll * nseg, s));
    GWB_CUDA(cudaMemsetAsync(counters_out, 0, 5 * sizeof(int32_t), s));
    const int grid = std::max(1, std::min(num_sms() * 4, (int)cdiv(cand_cap, kT)));
    // the rebuilt list continues after the selection's own rebuilt peaks
    GWB_CUDA(cudaMemcpyAsync(counters_out + 4, counters + 4, sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    seg_count_kernel<<<grid, kT, 0, s>>>(cands, counters, nseg, cnt, bad);
    GWB_LAUNCH_CHECK("seg_count_kernel");
    seg_scan_kernel<<<1, kT, 0, s>>>(cnt, nseg, off, fill);
    GWB_LAUNCH_CHECK("seg_scan_kernel");
    seg_scatter_kernel<<<grid, kT, 0, s>>>(cands, counters, nseg, off, fill, keys);
    GWB_LAUNCH_CHECK("seg_scatter_kernel");
    seg_radix_select_kernel<<<nseg, kT, 0, s>>>(keys, cnt, off, top_n, top_frac, tau);
    GWB_LAUNCH_CHECK("seg_radix_select_kernel");
    top_compact_kernel<<<num_sms() * 4, kT, 0, s>>>(cands, units, counters, tau, rthr, cands_out, cand_cap, groups_out,
                                                    cand_cap, units_out, cand_cap, rebuilt, rebuilt_cap, counters_out);
    GWB_LAUNCH_CHECK("top_compact_kernel");
    return GWB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------------------
// Local search of a screening form (fp8): every candidate becomes 2L + 1 exact-stage candidates at the samples s - L
// .. s + L (clamped into the candidate's own cluster window), in the same unit; after the exact stage
// gwb_search_best keeps the loudest of each run (first on ties) and marks the others with snr = -1. The screen's
// argmax then only has to fall within L samples of the window's true peak.
// ---------------------------------------------------------------------------------------------------------------------
namespace gwb {
namespace {

__global__ void search_expand_kernel(const GwbCand* __restrict__ cin, const GwbUnit* __restrict__ uin,
                                     const int32_t* __restrict__ cnt_in, int L, long long a0, int cw,
                                     GwbCand* __restrict__ cout, int cand_cap, GwbGroup* __restrict__ gout,
                                     int group_cap, GwbUnit* __restrict__ uout, int unit_cap,
                                     int32_t* __restrict__ counters) {
    __shared__ int s_base, s_gbase, s_unit, s_ok;
    const int nu = cnt_in[2];
    const int W = 2 * L + 1;
    for (int u = blockIdx.x; u < nu; u += gridDim.x) {
        const GwbUnit U = uin[u];
        const int total = U.count * W, ng = (total + 7) / 8;
        if (threadIdx.x == 0) {
            s_base = atomicAdd(&counters[0], total);
            s_gbase = atomicAdd(&counters[1], ng);
            s_unit = atomicAdd(&counters[2], 1);
            s_ok = !(s_base + total > cand_cap || s_gbase + ng > group_cap || s_unit >= unit_cap);
            if (!s_ok) atomicOr(&counters[3], 1);
            else uout[s_unit] = GwbUnit{U.row, U.seg, s_base, total};
        }
        __syncthreads();
        if (s_ok) {
            for (int g = threadIdx.x; g < ng; g += kT)
                gout[s_gbase + g] = GwbGroup{s_unit, s_base + 8 * g, min(8, total - 8 * g), 0};
            for (int o = threadIdx.x; o < total; o += kT) {
                GwbCand cd = cin[U.first + o / W];
                const long long w0 = a0 + (long long)cd.window * cw;
                const long long s = min(max((long long)cd.sample + (o % W) - L, w0), w0 + cw - 1);
                cd.sample = (int)s;
                cd.unit = s_unit;
                cout[s_base + o] = cd;
            }
        }
        __syncthreads();
    }
}

__global__ void search_best_kernel(const int32_t* __restrict__ ccount, int cmax, int W, GwbPeak* __restrict__ peaks) {
    const int n = min(*ccount, cmax) / W;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        GwbPeak* p = peaks + (long long)i * W;
        int best = 0;
        for (int d = 1; d < W; ++d)
            if (p[d].snr > p[best].snr) best = d;
        for (int d = 0; d < W; ++d)
            if (d != best) p[d].snr = -1.f;
    }
}

}  // namespace
}  // namespace gwb

extern "C" {

int gwb_search_expand(const GwbCand* cands, const GwbUnit* units, const int32_t* counters, int radius, long long a0,
                      int cw, GwbCand* cands_out, int cand_cap, GwbGroup* groups_out, GwbUnit* units_out,
                      int32_t* counters_out, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(cands && units && counters && cands_out && groups_out && units_out && counters_out, GWB_ERR_ARG,
                  "search_expand: null pointer");
    GWB_CHECK_ARG(radius >= 1 && radius <= 8 && cw > 2 * radius && a0 >= 0 && cand_cap > 0, GWB_ERR_SHAPE,
                  "search_expand: radius=%d (1..8) cw=%d a0=%lld", radius, cw, a0);
    cudaStream_t s = (cudaStream_t)stream;
    GWB_CUDA(cudaMemsetAsync(counters_out, 0, 4 * sizeof(int32_t), s));
    // the selection's rebuilt-peak count passes through
    GWB_CUDA(cudaMemcpyAsync(counters_out + 4, counters + 4, sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    search_expand_kernel<<<num_sms() * 4, kT, 0, s>>>(cands, units, counters, radius, a0, cw, cands_out, cand_cap,
                                                      groups_out, cand_cap, units_out, cand_cap, counters_out);
    GWB_LAUNCH_CHECK("search_expand_kernel");
    return GWB_OK;
}

int gwb_search_best(const int32_t* ccount, int cmax, int radius, GwbPeak* peaks, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(ccount && peaks && radius >= 1 && radius <= 8 && cmax > 0, GWB_ERR_ARG,
                  "search_best: radius=%d cmax=%d", radius, cmax);
    search_best_kernel<<<num_sms() * 4, kT, 0, (cudaStream_t)stream>>>(ccount, cmax, 2 * radius + 1, peaks);
    GWB_LAUNCH_CHECK("search_best_kernel");
    return GWB_OK;
}

}  // extern "C"
