// Handle with a cache of cuFFT plans, and the batched transforms the path needs (cuFFT is the one library call the
// path uses). Plans are made on first use of a (kind, n, batch, strides) shape and reused; making them allocates
// cuFFT's work area, so a caller that captures CUDA graphs runs each shape once before capture.
#include "common.cuh"
#include <cufft.h>
#include <map>
#include <mutex>
#include <tuple>

struct gwb_handle_s {
    std::mutex mu;
    std::map<std::tuple<int, long long, int, long long, long long>, cufftHandle> plans;
    int device = 0;
};

namespace gwb {

static int get_plan(gwb_handle_t h, int kind, long long n, int batch, long long idist, long long odist,
                    cufftHandle* out) {
    std::lock_guard<std::mutex> lk(h->mu);
    auto key = std::make_tuple(kind, n, batch, idist, odist);
    auto it = h->plans.find(key);
    if (it != h->plans.end()) {
        *out = it->second;
        return GWB_OK;
    }
    cufftHandle p;
    cufftResult r = cufftCreate(&p);
    if (r != CUFFT_SUCCESS) return cufft_status(r, "cufftCreate");
    long long nn[1] = {n};
    long long inembed[1] = {kind == 1 ? n : (kind == 2 ? n / 2 + 1 : n)};
    long long onembed[1] = {kind == 1 ? n / 2 + 1 : n};
    cufftType t = kind == 0 ? CUFFT_C2C : (kind == 1 ? CUFFT_R2C : CUFFT_C2R);
    size_t ws = 0;
    r = cufftMakePlanMany64(p, 1, nn, inembed, 1, idist, onembed, 1, odist, t, batch, &ws);
    if (r != CUFFT_SUCCESS) {
        cufftDestroy(p);
        return cufft_status(r, "cufftMakePlanMany64");
    }
    h->plans[key] = p;
    *out = p;
    return GWB_OK;
}

}  // namespace gwb

extern "C" {

int gwb_create(gwb_handle_t* out) {
    GWB_CHECK_ARG(out != nullptr, GWB_ERR_ARG, "gwb_create: null output");
    gwb_handle_t h = new (std::nothrow) gwb_handle_s();
    GWB_CHECK_ARG(h != nullptr, GWB_ERR_ALLOC, "gwb_create: out of host memory");
    cudaGetDevice(&h->device);
    *out = h;
    return GWB_OK;
}

int gwb_destroy(gwb_handle_t h) {
    if (h == nullptr) return GWB_OK;
    for (auto& kv : h->plans) cufftDestroy(kv.second);
    delete h;
    return GWB_OK;
}

int gwb_fft_c2c(gwb_handle_t h, const float* in, float* out, long long n, int batch, long long idist,
                long long odist, int inverse, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(h && in && out, GWB_ERR_ARG, "fft_c2c: null argument");
    GWB_CHECK_ARG(n > 0 && batch > 0 && idist >= n && odist >= n, GWB_ERR_SHAPE, "fft_c2c: n=%lld batch=%d", n, batch);
    cufftHandle p;
    int st = get_plan(h, 0, n, batch, idist, odist, &p);
    if (st) return st;
    cufftResult r = cufftSetStream(p, (cudaStream_t)stream);
    if (r != CUFFT_SUCCESS) return cufft_status(r, "cufftSetStream");
    r = cufftExecC2C(p, (cufftComplex*)in, (cufftComplex*)out, inverse ? CUFFT_INVERSE : CUFFT_FORWARD);
    if (r != CUFFT_SUCCESS) return cufft_status(r, "cufftExecC2C");
    return GWB_OK;
}

int gwb_fft_r2c(gwb_handle_t h, const float* in, float* out, long long n, int batch, long long idist,
                long long odist, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(h && in && out, GWB_ERR_ARG, "fft_r2c: null argument");
    GWB_CHECK_ARG(n > 0 && batch > 0 && idist >= n && odist >= n / 2 + 1, GWB_ERR_SHAPE, "fft_r2c: n=%lld batch=%d", n,
                  batch);
    cufftHandle p;
    int st = get_plan(h, 1, n, batch, idist, odist, &p);
    if (st) return st;
    cufftResult r = cufftSetStream(p, (cudaStream_t)stream);
    if (r != CUFFT_SUCCESS) return cufft_status(r, "cufftSetStream");
    r = cufftExecR2C(p, (cufftReal*)in, (cufftComplex*)out);
    if (r != CUFFT_SUCCESS) return cufft_status(r, "cufftExecR2C");
    return GWB_OK;
}

int gwb_fft_c2r(gwb_handle_t h, const float* in, float* out, long long n, int batch, long long idist,
                long long odist, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(h && in && out, GWB_ERR_ARG, "fft_c2r: null argument");
    GWB_CHECK_ARG(n > 0 && batch > 0 && idist >= n / 2 + 1 && odist >= n, GWB_ERR_SHAPE, "fft_c2r: n=%lld batch=%d",
                  n, batch);
    cufftHandle p;
    int st = get_plan(h, 2, n, batch, idist, odist, &p);
    if (st) return st;
    cufftResult r = cufftSetStream(p, (cudaStream_t)stream);
    if (r != CUFFT_SUCCESS) return cufft_status(r, "cufftSetStream");
    r = cufftExecC2R(p, (cufftComplex*)in, (cufftReal*)out);
    if (r != CUFFT_SUCCESS) return cufft_status(r, "cufftExecC2R");
    return GWB_OK;
}

}  // extern "C"
