// Library runtime: status strings, the last-error message, the per-device error word, SM counts and the tensor-map
// encoder (fetched from the driver at run time, so the library does not link libcuda).
#include "common.cuh"
#include <cudaTypedefs.h>
#include <mutex>
#include <string.h>

namespace gwb {

static thread_local char g_msg[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
    va_end(ap);
}

int cuda_status(cudaError_t e, const char* what) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return GWB_ERR_CUDA;
}

int cufft_status(int r, const char* what) {
    set_error("%s: cufft error %d", what, r);
    return GWB_ERR_CUFFT;
}

static const int kMaxDev = 64;
static std::mutex g_mu;
static DeviceError* g_err[kMaxDev] = {nullptr};
static int g_sms[kMaxDev] = {0};

// The error word lives in a file-scope device variable, so reading or clearing it never allocates.
static __device__ DeviceError g_device_error;

static int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}

DeviceError* device_error_ptr() {
    int d = current_device();
    if (d < 0 || d >= kMaxDev) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_err[d] == nullptr) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_device_error) != cudaSuccess) return nullptr;
        g_err[d] = static_cast<DeviceError*>(p);
    }
    return g_err[d];
}

// The GEMM launch table (gwb_gemm_set_config), process-wide under a mutex.
namespace {
struct TuneEntry {
    int form, kh, pair, stages, order;
};
std::mutex g_tune_mu;
TuneEntry g_tune[128];
int g_ntune = 0;
}  // namespace

bool tune_lookup(int form, int kh, int* pair, int* stages, int* order) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (int i = 0; i < g_ntune; ++i)
        if (g_tune[i].form == form && g_tune[i].kh == kh) {
            *pair = g_tune[i].pair;
            *stages = g_tune[i].stages;
            *order = g_tune[i].order;
            return true;
        }
    return false;
}

int num_sms() {
    int d = current_device();
    if (d >= 0 && d < kMaxDev && g_sms[d] > 0) return g_sms[d];
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d);
    if (n <= 0) n = 148;
    if (d >= 0 && d < kMaxDev) g_sms[d] = n;
    return n;
}

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int encode_tmap_2d(CUtensorMap* map, CUtensorMapDataType dtype, const void* base, uint64_t inner, uint64_t outer,
                   uint64_t row_stride_bytes, uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle swz) {
    if (g_encode == nullptr) {
        std::lock_guard<std::mutex> lk(g_mu);
        if (g_encode == nullptr) {
            void* fn = nullptr;
            cudaDriverEntryPointQueryResult q;
            cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
            if (e != cudaSuccess || fn == nullptr || q != cudaDriverEntryPointSuccess) {
                set_error("cuTensorMapEncodeTiled not available from the driver");
                return GWB_ERR_CUDA;
            }
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        }
    }
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {row_stride_bytes};
    cuuint32_t box[2] = {box_inner, box_outer};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(map, dtype, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d): dims %llu x %llu stride %llu box %u x %u", (int)r,
                  (unsigned long long)inner, (unsigned long long)outer, (unsigned long long)row_stride_bytes,
                  box_inner, box_outer);
        return GWB_ERR_ALIGN;
    }
    return GWB_OK;
}

}  // namespace gwb

extern "C" {

int gwb_version(void) { return GWB_VERSION; }

const char* gwb_status_string(int status) {
    switch (status) {
        case GWB_OK: return "ok";
        case GWB_ERR_SHAPE: return "bad shape";
        case GWB_ERR_NOT_POW2: return "length is not a power of two";
        case GWB_ERR_EDGE_ORDER: return "chi-squared bin edges out of order or outside the band";
        case GWB_ERR_ALLOC: return "device allocation failed";
        case GWB_ERR_CUFFT: return "cuFFT error";
        case GWB_ERR_TIMEOUT: return "a device wait ran out of time";
        case GWB_ERR_CUDA: return "CUDA error";
        case GWB_ERR_ARG: return "bad argument";
        case GWB_ERR_NOT_IMPLEMENTED: return "not implemented in this library";
        case GWB_ERR_ALIGN: return "pointer or stride misaligned for TMA";
        case GWB_ERR_CAPACITY: return "output capacity exceeded";
        default: return "unknown status";
    }
}

const char* gwb_last_error(void) { return gwb::g_msg; }

int gwb_device_error(int* code, int* where, int* info0, int* info1, int clear) {
    gwb::DeviceError* p = gwb::device_error_ptr();
    if (p == nullptr) {
        gwb::set_error("device error word unavailable");
        return GWB_ERR_ALLOC;
    }
    gwb::DeviceError h;
    GWB_CUDA(cudaMemcpy(&h, p, sizeof(h), cudaMemcpyDeviceToHost));
    if (code) *code = h.code;
    if (where) *where = h.where;
    if (info0) *info0 = h.info0;
    if (info1) *info1 = h.info1;
    if (clear) GWB_CUDA(cudaMemset(p, 0, sizeof(h)));
    return GWB_OK;
}

int gwb_num_sms(void) { return gwb::num_sms(); }

}  // extern "C"

extern "C" int gwb_gemm_set_config(int form, int kh, int pair, int stages, int order) {
    using namespace gwb;
    GWB_CHECK_ARG(form >= 0 && form <= 6 && kh > 0 && (pair == 0 || pair == 1) && stages >= 0 && stages <= 8 &&
                      order >= 0 && order <= 3, GWB_ERR_ARG,
                  "gemm_set_config: form=%d kh=%d pair=%d stages=%d order=%d", form, kh, pair, stages, order);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (int i = 0; i < g_ntune; ++i)
        if (g_tune[i].form == form && g_tune[i].kh == kh) {
            g_tune[i] = TuneEntry{form, kh, pair, stages, order};
            return GWB_OK;
        }
    GWB_CHECK_ARG(g_ntune < 128, GWB_ERR_CAPACITY, "gemm_set_config: the table holds 128 shapes");
    g_tune[g_ntune++] = TuneEntry{form, kh, pair, stages, order};
    return GWB_OK;
}

extern "C" int gwb_gemm_clear_configs(void) {
    std::lock_guard<std::mutex> lk(gwb::g_tune_mu);
    gwb::g_ntune = 0;
    return GWB_OK;
}
