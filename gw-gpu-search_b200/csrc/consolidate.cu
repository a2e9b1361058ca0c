// Consolidation of one dataset's peaks on the device (the step downstream of the exact stage).
//
// Replaces the reference's host-side consolidate (pipeline/fp_filter.py:629-661, pycbc's
// EventManager.consolidate_events with the whole bank as one job) and its GPU pre-filter pre_keep (:663-695) with one
// entry point. Per item: the statistic (newsnr in float64, or the SNR), the newsnr / exempt cut and the gate veto
// (mark_kernel); for the keep-loudest ranking, the items of each window are bucketed (count, scan, scatter) and every
// item's rank within its window is counted against the window's items staged in shared memory (rank_kernel); ties
// go to the smaller order key (the reference's stable sorts keep the earlier position). finish_kernel combines the
// flags into the keep mask.
//
// Arithmetic follows the reference's types: float32 SNRs compare with float32 thresholds (numpy and torch cast a
// Python-float threshold to the array's type), times and windows are float64 (t = gps_start + ti / sr, window =
// trunc(rint((t - gps_start) sr) / (interval sr))), newsnr is PyCBC's snr (0.5 (1 + r^3))^(-1/6) for r =
// chisq / max(dof, 1) > 1 in float64 (CUDA's pow: within 2 ulp of the host's, so only distinct inputs whose newsnr
// agree to 2 ulp could rank differently).
#include <math.h>
#include <algorithm>
#include "common.cuh"

namespace gwb {
namespace {

constexpr int kCT = 256;
constexpr int kTile = 2048;     // window items staged per pass: stat (8 B) + order key (8 B) = 32 KB

enum : uint8_t { F_KEEP = 1, F_EXEMPT = 2, F_RANKED = 4, F_EXACT = 8, F_TOP = 16 };

struct Params {
    int mode, n, use_chisq, has_exempt, ng, keep_num, nwin, nfloor;
    double gps_start, sr, newsnr_thr, span;     // span = keep_interval * sr; 0 = no ranking
    float exact_cut, thr, exempt_snr, newsnr_thr_f;
};

__device__ __forceinline__ double newsnr_d(float snr, float chi, int dof) {
    const double r = __ddiv_rn((double)chi, (double)max(dof, 1));
    double ns = (double)snr;
    if (r > 1.0) ns = __dmul_rn(ns, pow(__dmul_rn(0.5, __dadd_rn(1.0, pow(r, 3.0))), -1.0 / 6.0));
    return ns;
}

__global__ void __launch_bounds__(kCT) mark_kernel(Params p, const float* __restrict__ snr,
                                                   const float* __restrict__ chi, const int32_t* __restrict__ dof,
                                                   const long long* __restrict__ ti, const double* __restrict__ gates,
                                                   const double* __restrict__ floor_in, double* __restrict__ stat,
                                                   int32_t* __restrict__ wt, uint8_t* __restrict__ flags,
                                                   int32_t* __restrict__ cnt, int32_t* __restrict__ status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) {
        const float s = snr[i];
        const double t = __dadd_rn(p.gps_start, __ddiv_rn((double)ti[i], p.sr));
        bool gate_ok = true;
        for (int k = 0; k < p.ng; ++k) {
            const double reach = __dadd_rn(__dadd_rn(gates[3 * k + 1], gates[3 * k + 2]), 0.5);
            gate_ok = gate_ok && fabs(__dsub_rn(t, gates[3 * k])) > reach;
        }
        uint8_t f = 0;
        double st;
        bool keep, exempt = false;
        if (p.mode == 0) {                              // consolidate
            st = p.use_chisq ? newsnr_d(s, chi[i], dof[i]) : (double)s;
            exempt = p.has_exempt && s >= p.exempt_snr;
            keep = ((p.use_chisq ? st >= p.newsnr_thr : s >= p.newsnr_thr_f) || exempt) && gate_ok;
        } else {                                        // pre_keep: newsnr of a rebuilt peak is its SNR
            st = (double)s;
            const bool ex = s >= p.exact_cut;
            if (ex) f |= F_EXACT;
            const bool ok = !ex && s > p.thr;
            exempt = ok && p.has_exempt && s >= p.exempt_snr;
            keep = ok && (s >= p.newsnr_thr_f || exempt) && gate_ok;
        }
        int w = -1;
        if (keep && !exempt && p.span > 0.0) {
            const double q = __ddiv_rn(rint(__dmul_rn(__dsub_rn(t, p.gps_start), p.sr)), p.span);
            const long long wl = (long long)q;          // truncation, as astype(int64) / long()
            bool ranked = true;
            if (p.mode == 1 && floor_in != nullptr && wl >= 0) {
                const double bar = wl < p.nfloor ? floor_in[wl] : -INFINITY;
                if (!((double)s > bar)) {               // at or below the K-th loudest already kept: dropped
                    keep = false;
                    ranked = false;
                }
            }
            if (ranked) {
                if (wl < 0 || wl >= p.nwin) {
                    atomicOr(status, 1);
                } else {
                    w = (int)wl;
                    f |= F_RANKED;
                    atomicAdd(&cnt[w], 1);
                }
            }
        }
        if (keep) f |= F_KEEP;
        if (exempt) f |= F_EXEMPT;
        stat[i] = st;
        wt[i] = w;
        flags[i] = f;
    }
}

// Exclusive scan of the window counts (one block: contiguous runs per thread, then a block scan of the run sums).
__global__ void __launch_bounds__(1024) scan_kernel(const int32_t* __restrict__ cnt, int nwin,
                                                    int32_t* __restrict__ off) {
    __shared__ int part[1024];
    const int T = blockDim.x, tid = threadIdx.x;
    const long long per = (nwin + T - 1) / T;
    const long long b = tid * per, e = min((long long)nwin, b + per);
    int s = 0;
    for (long long k = b; k < e; ++k) s += cnt[k];
    part[tid] = s;
    __syncthreads();
    for (int d = 1; d < T; d <<= 1) {
        const int v = tid >= d ? part[tid - d] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int run = tid ? part[tid - 1] : 0;
    for (long long k = b; k < e; ++k) {
        off[k] = run;
        run += cnt[k];
    }
    if (tid == T - 1) off[nwin] = part[T - 1];
}

__global__ void __launch_bounds__(kCT) scatter_kernel(int n, const int32_t* __restrict__ wt,
                                                      const int32_t* __restrict__ off, int32_t* __restrict__ fill,
                                                      int32_t* __restrict__ bucket) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int w = wt[i];
        if (w >= 0) bucket[off[w] + atomicAdd(&fill[w], 1)] = i;
    }
}

// One block per window (grid-stride): rank = number of the window's items that come first in (stat descending,
// order ascending); the keep_num first get F_TOP, and the one of rank keep_num - 1 gives the window's floor.
__global__ void __launch_bounds__(kCT) rank_kernel(Params p, const int32_t* __restrict__ off,
                                                   const int32_t* __restrict__ bucket,
                                                   const double* __restrict__ stat,
                                                   const long long* __restrict__ order, uint8_t* __restrict__ flags,
                                                   double* __restrict__ floor_out) {
    __shared__ double s_stat[kTile];
    __shared__ long long s_ord[kTile];
    for (int w = blockIdx.x; w < p.nwin; w += gridDim.x) {
        const int b = off[w], c = off[w + 1] - b;
        if (floor_out != nullptr && threadIdx.x == 0 && c < p.keep_num) floor_out[w] = -INFINITY;
        if (c == 0) continue;
        for (int i0 = 0; i0 < c; i0 += blockDim.x) {
            const int ii = i0 + threadIdx.x;
            int item = -1;
            double si = 0.0;
            long long oi = 0;
            if (ii < c) {
                item = bucket[b + ii];
                si = stat[item];
                oi = order ? order[item] : (long long)item;
            }
            int rank = 0;
            for (int j0 = 0; j0 < c; j0 += kTile) {
                const int m = min(kTile, c - j0);
                __syncthreads();
                for (int j = threadIdx.x; j < m; j += blockDim.x) {
                    const int it = bucket[b + j0 + j];
                    s_stat[j] = stat[it];
                    s_ord[j] = order ? order[it] : (long long)it;
                }
                __syncthreads();
                if (item >= 0 && rank < p.keep_num) {
                    for (int j = 0; j < m; ++j) {
                        const double sj = s_stat[j];
                        rank += (sj > si) || (sj == si && s_ord[j] < oi);
                    }
                }
            }
            if (item >= 0 && rank < p.keep_num) {
                flags[item] |= F_TOP;
                if (floor_out != nullptr && rank == p.keep_num - 1) floor_out[w] = si;
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kCT) finish_kernel(Params p, const uint8_t* __restrict__ flags,
                                                     uint8_t* __restrict__ keep) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) {
        const uint8_t f = flags[i];
        const bool base = f & F_KEEP, exempt = f & F_EXEMPT;
        bool k = p.span > 0.0 ? ((f & F_TOP) || (base && exempt)) : base;
        if (p.mode == 1) k = k || (f & F_EXACT);
        keep[i] = k;
    }
}

inline long long up16(long long b) { return (b + 15) & ~15ll; }

}  // namespace
}  // namespace gwb

extern "C" {

long long gwb_consolidate_work_bytes(int n, int nwin) {
    using gwb::up16;
    if (n < 0 || nwin < 0) return -1;
    return up16(8ll * n) + up16(4ll * n) + up16(4ll * n) + up16(n) + up16(4ll * nwin) + up16(4ll * nwin) +
           up16(4ll * (nwin + 1));
}

int gwb_consolidate(int mode, int n, const float* snr, const float* chisq, const int32_t* dof, const long long* ti,
                    const long long* order, int use_chisq, double gps_start, double sr, float exact_cut, float thr,
                    double newsnr_thr, int has_exempt, float exempt_snr, const double* gates, int ng,
                    double keep_interval, int keep_num, const double* floor_in, int nfloor, double* floor_out,
                    int nwin, void* work, long long work_bytes, uint8_t* keep, int32_t* status, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(mode == 0 || mode == 1, GWB_ERR_ARG, "consolidate: mode %d", mode);
    GWB_CHECK_ARG(n >= 0 && ng >= 0 && nfloor >= 0 && sr > 0 && keep_interval >= 0, GWB_ERR_SHAPE,
                  "consolidate: n=%d ng=%d nfloor=%d sr=%g interval=%g", n, ng, nfloor, sr, keep_interval);
    GWB_CHECK_ARG(status && work && (n == 0 || (snr && ti && keep)) && (ng == 0 || gates) &&
                  (mode == 1 || !use_chisq || n == 0 || (chisq && dof)) && (nfloor == 0 || floor_in),
                  GWB_ERR_ARG, "consolidate: null pointer");
    GWB_CHECK_ARG(keep_interval == 0 || (keep_num >= 1 && nwin >= 1), GWB_ERR_SHAPE,
                  "consolidate: keep_num=%d nwin=%d", keep_num, nwin);
    GWB_CHECK_ARG(floor_out == nullptr || keep_interval > 0, GWB_ERR_ARG, "consolidate: a floor needs the ranking");
    if (keep_interval == 0) nwin = 0;
    GWB_CHECK_ARG(work_bytes >= gwb_consolidate_work_bytes(n, nwin), GWB_ERR_SHAPE,
                  "consolidate: work %lld bytes, %lld needed", work_bytes, gwb_consolidate_work_bytes(n, nwin));
    Params p;
    p.mode = mode;
    p.n = n;
    p.use_chisq = use_chisq;
    p.has_exempt = has_exempt;
    p.ng = ng;
    p.keep_num = keep_num;
    p.nwin = nwin;
    p.nfloor = nfloor;
    p.gps_start = gps_start;
    p.sr = sr;
    p.newsnr_thr = newsnr_thr;
    p.span = keep_interval * sr;
    p.exact_cut = exact_cut;
    p.thr = thr;
    p.exempt_snr = exempt_snr;
    p.newsnr_thr_f = (float)newsnr_thr;
    char* w = static_cast<char*>(work);
    double* stat = reinterpret_cast<double*>(w);
    w += up16(8ll * n);
    int32_t* wt = reinterpret_cast<int32_t*>(w);
    w += up16(4ll * n);
    int32_t* bucket = reinterpret_cast<int32_t*>(w);
    w += up16(4ll * n);
    uint8_t* flags = reinterpret_cast<uint8_t*>(w);
    w += up16(n);
    int32_t* cnt = reinterpret_cast<int32_t*>(w);
    w += up16(4ll * nwin);
    int32_t* fill = reinterpret_cast<int32_t*>(w);
    w += up16(4ll * nwin);
    int32_t* off = reinterpret_cast<int32_t*>(w);
    cudaStream_t s = (cudaStream_t)stream;
    GWB_CUDA(cudaMemsetAsync(status, 0, sizeof(int32_t), s));
    if (nwin > 0) GWB_CUDA(cudaMemsetAsync(cnt, 0, up16(4ll * nwin) * 2, s));   // cnt and fill
    const int g = (int)std::max(1ll, std::min(cdiv(n, kCT), (long long)num_sms() * 16));
    if (n > 0) {
        mark_kernel<<<g, kCT, 0, s>>>(p, snr, chisq, dof, ti, gates, floor_in, stat, wt, flags, cnt, status);
        GWB_LAUNCH_CHECK("mark_kernel");
    }
    if (nwin > 0) {
        scan_kernel<<<1, 1024, 0, s>>>(cnt, nwin, off);
        GWB_LAUNCH_CHECK("scan_kernel");
        if (n > 0) {
            scatter_kernel<<<g, kCT, 0, s>>>(n, wt, off, fill, bucket);
            GWB_LAUNCH_CHECK("scatter_kernel");
        }
        const int gr = (int)std::min<long long>(nwin, (long long)num_sms() * 32);
        rank_kernel<<<gr, kCT, 0, s>>>(p, off, bucket, stat, order, flags, floor_out);
        GWB_LAUNCH_CHECK("rank_kernel");
    }
    if (n > 0) {
        finish_kernel<<<g, kCT, 0, s>>>(p, flags, keep);
        GWB_LAUNCH_CHECK("finish_kernel");
    }
    return GWB_OK;
}

}  // extern "C"
