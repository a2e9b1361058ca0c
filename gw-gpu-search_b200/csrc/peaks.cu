// Per-window peak picking over a dense complex SNR series.
//
// Replaces peak_kernel.window_peaks / win_peak (pipeline/peak_kernel.py:10-47): for each (row, window) the maximum
// of |z|^2 over the window's cw samples and its offset inside the window, the first offset on ties (numpy argmax
// order). One 128-thread block per (window, row); each thread walks its samples in increasing order, then a warp
// shuffle tree and a shared-memory pass combine (value, offset) pairs with ties broken toward the smaller offset.
#include "common.cuh"

namespace gwb {
namespace {

constexpr int kWinThreads = 128;

__device__ __forceinline__ void take_better(float ov, int oi, float& v, int& i) {
    if (ov > v || (ov == v && oi < i)) {
        v = ov;
        i = oi;
    }
}

__global__ void __launch_bounds__(kWinThreads) window_peaks_kernel(const float2* __restrict__ z, long long ldz,
                                                                   long long a0, int cw, int nwin,
                                                                   float* __restrict__ pmax,
                                                                   int32_t* __restrict__ pidx) {
    const int w = blockIdx.x, row = blockIdx.y;
    const float2* zr = z + (long long)row * ldz + a0 + (long long)w * cw;
    float best = -1.f;
    int bi = 0;
    for (int i = threadIdx.x; i < cw; i += kWinThreads) {
        const float2 v = zr[i];
        const float p = __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));   // numpy's rounding, no FMA
        if (p > best) {
            best = p;
            bi = i;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float ob = __shfl_down_sync(0xffffffffu, best, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        take_better(ob, oi, best, bi);
    }
    __shared__ float sb[kWinThreads / 32];
    __shared__ int si[kWinThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sb[warp] = best;
        si[warp] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kWinThreads / 32; ++k) take_better(sb[k], si[k], best, bi);
        pmax[(long long)row * nwin + w] = best;
        pidx[(long long)row * nwin + w] = bi;
    }
}

}  // namespace
}  // namespace gwb

extern "C" int gwb_window_peaks(const float* z, long long ldz, int rows, long long a0, int cw, int nwin, float* pmax,
                                int32_t* pidx, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(z && pmax && pidx, GWB_ERR_ARG, "window_peaks: null pointer");
    GWB_CHECK_ARG(rows >= 0 && cw > 0 && nwin >= 0 && a0 >= 0, GWB_ERR_SHAPE, "window_peaks: rows=%d cw=%d nwin=%d a0=%lld",
                  rows, cw, nwin, a0);
    GWB_CHECK_ARG(a0 + (long long)nwin * cw <= ldz, GWB_ERR_SHAPE,
                  "window_peaks: windows end at %lld beyond the row length %lld", a0 + (long long)nwin * cw, ldz);
    GWB_CHECK_ARG(rows < 65536, GWB_ERR_SHAPE, "window_peaks: rows=%d above 65535", rows);
    if (rows == 0 || nwin == 0) return GWB_OK;
    dim3 grid(nwin, rows);
    window_peaks_kernel<<<grid, kWinThreads, 0, (cudaStream_t)stream>>>(reinterpret_cast<const float2*>(z), ldz, a0,
                                                                        cw, nwin, pmax, pidx);
    GWB_LAUNCH_CHECK("window_peaks_kernel");
    return GWB_OK;
}
