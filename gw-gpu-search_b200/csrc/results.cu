// Appending one step's exact-stage results to a run-wide list on the device, so that a whole batched run (many steps
// in one CUDA graph) copies its results to the host once at the end instead of once per step. No reference
// counterpart: the reference copies each (tile, segment)'s peaks to the host as it goes (pipeline/fp_filter.py:752-753,
// 837-853).
#include "common.cuh"

namespace gwb {
namespace {

// one thread: reserve n = min(counters[0], cap) entries of the run list; base[0] = the first, base[1] = n; the step's
// five counters and the reservation are recorded in meta[tag * 8 ..] (the run's per-step record)
__global__ void append_reserve_kernel(const int32_t* __restrict__ counters, int cap, int tag, int out_cap,
                                      int32_t* __restrict__ out_count, int32_t* __restrict__ base,
                                      int32_t* __restrict__ meta) {
    const int n = min(counters[0], cap);
    const int b = *out_count;
    const int m = max(0, min(n, out_cap - b));
    *out_count = b + m;
    base[0] = b;
    base[1] = m;
    int32_t* r = meta + (long long)tag * 8;
    for (int i = 0; i < 5; ++i) r[i] = counters[i];
    r[5] = b;
    r[6] = m;
    r[7] = m < n;            // the run list overflowed
}

__global__ void append_copy_kernel(const GwbCand* __restrict__ cands, const GwbPeak* __restrict__ peaks,
                                   const int32_t* __restrict__ base, int tag, GwbCand* __restrict__ out_c,
                                   GwbPeak* __restrict__ out_p, int32_t* __restrict__ out_tag) {
    const int b = base[0], m = base[1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        out_c[b + i] = cands[i];
        out_p[b + i] = peaks[i];
        out_tag[b + i] = tag;
    }
}

}  // namespace
}  // namespace gwb

extern "C" int gwb_append_results(const GwbCand* cands, const GwbPeak* peaks, const int32_t* counters, int cap,
                                  int tag, GwbCand* out_cands, GwbPeak* out_peaks, int32_t* out_tag, int32_t* out_count,
                                  int out_cap, int32_t* work, int32_t* meta, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(cands && peaks && counters && out_cands && out_peaks && out_tag && out_count && work && meta,
                  GWB_ERR_ARG, "append_results: null pointer");
    GWB_CHECK_ARG(cap >= 0 && out_cap >= 0 && tag >= 0, GWB_ERR_SHAPE, "append_results: cap=%d out_cap=%d tag=%d", cap,
                  out_cap, tag);
    cudaStream_t s = (cudaStream_t)stream;
    append_reserve_kernel<<<1, 1, 0, s>>>(counters, cap, tag, out_cap, out_count, work, meta);
    GWB_LAUNCH_CHECK("append_reserve_kernel");
    append_copy_kernel<<<num_sms() * 2, 256, 0, s>>>(cands, peaks, work, tag, out_cands, out_peaks, out_tag);
    GWB_LAUNCH_CHECK("append_copy_kernel");
    return GWB_OK;
}
