// A batch of raw strain chunks through the whole hot path in one C entry: the conditioning of gpu_stage2 for
// datasets that each hold one analysis segment and one PSD span (pipeline/gpu_prep.py:405-454: median-Welch PSD,
// interpolation, inverse spectrum truncation, the segment rFFT, D = stilde / psd and IP = 1 / psd), then the filter
// step of gwb_filter_step. It is the batched entry behind the batched form (the per-dataset loop of
// pipeline/fp_filter.py:700-888 driven over many segments) for a caller without Python: the caller cuts its segments
// into chunks, calls this once per batch and reads the candidate and exact-stage lists back when it wants them.
#include <math.h>
#include <string.h>
#include "common.cuh"

namespace {

struct CondShapes {
    int nfr, nb, flen, kmin;
    long long n;
    double df;
};

int cond_shapes(long long tlen, const GwbCondConfig* c, CondShapes* s) {
    using namespace gwb;
    GWB_CHECK_ARG(c, GWB_ERR_ARG, "filter_batch: null conditioning config");
    GWB_CHECK_ARG(c->sr > 0.0 && c->f_low > 0.0 && c->psd_len >= 2 && c->psd_stride > 0 && c->psd_len <= tlen &&
                      c->inv_len >= 0 && c->inv_len <= tlen && (c->median == 0 || c->median == 1) &&
                      (c->inv_taper == 0 || c->inv_taper == 1),
                  GWB_ERR_SHAPE, "filter_batch: sr=%g f_low=%g psd_len=%d stride=%d inv_len=%d", c->sr, c->f_low,
                  c->psd_len, c->psd_stride, c->inv_len);
    s->n = tlen;
    s->nfr = (int)((tlen - c->psd_len) / c->psd_stride + 1);
    GWB_CHECK_ARG((long long)(s->nfr - 1) * c->psd_stride + c->psd_len == tlen, GWB_ERR_SHAPE,
                  "filter_batch: the Welch frames (%d of %d, stride %d) must tile the chunk of %lld samples", s->nfr,
                  c->psd_len, c->psd_stride, tlen);
    s->nb = c->psd_len / 2 + 1;
    s->flen = (int)(tlen / 2 + 1);
    s->df = c->sr / (double)tlen;
    s->kmin = (int)(c->f_low / s->df);
    GWB_CHECK_ARG(s->kmin > 0 && s->kmin < s->flen, GWB_ERR_SHAPE, "filter_batch: kmin=%d", s->kmin);
    return GWB_OK;
}

struct CondWork {
    float *frames, *F, *psd_w, *psd, *inv, *q, *pt, *st, *w, *tw;
    int32_t* pick;
};

long long cond_carve(const CondShapes& s, int nseg, const GwbCondConfig* c, char* base, CondWork* w) {
    long long off = 0;
    auto take = [&](long long bytes) {
        off = (off + 255) & ~255ll;
        char* p = base ? base + off : nullptr;
        off += bytes;
        return p;
    };
    const long long rows = (long long)nseg * s.nfr;
    w->frames = reinterpret_cast<float*>(take(4ll * rows * c->psd_len));
    w->F = reinterpret_cast<float*>(take(8ll * rows * s.nb));
    w->psd_w = reinterpret_cast<float*>(take(4ll * nseg * s.nb));
    w->psd = reinterpret_cast<float*>(take(4ll * nseg * s.flen));
    w->inv = reinterpret_cast<float*>(take(8ll * nseg * s.flen));
    w->q = reinterpret_cast<float*>(take(4ll * nseg * s.n));
    w->pt = reinterpret_cast<float*>(take(8ll * nseg * s.flen));
    w->st = reinterpret_cast<float*>(take(8ll * nseg * s.flen));
    w->w = reinterpret_cast<float*>(take(4ll * c->psd_len));
    w->tw = reinterpret_cast<float*>(take(4ll * (c->inv_len > 0 ? c->inv_len : 1)));
    w->pick = reinterpret_cast<int32_t*>(take(4ll * nseg));
    return (off + 255) & ~255ll;
}

// numpy's Hann window: 0.5 - 0.5 cos(2 pi i / (m - 1)), computed in double and rounded to float
__global__ void hann_kernel(float* __restrict__ w, int m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) w[i] = m == 1 ? 1.0f : (float)(0.5 - 0.5 * cos(2.0 * 3.141592653589793 * (double)i / (double)(m - 1)));
}

__global__ void iota_kernel(int32_t* __restrict__ p, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = i;
}

// PyCBC's median bias for n frames (the reference's gpu_prep.py:47-53)
double median_bias(int n) {
    if (n >= 1000) return log(2.0);
    double ans = 1.0;
    for (int i = 1; i <= (n - 1) / 2; ++i) ans += 1.0 / (2.0 * i + 1.0) - 1.0 / (2.0 * i);
    return ans;
}

// the Welch scale 2 / (sr sum w^2) folded as numpy does for the reference's psd (with dt = 1 / sr): 2 sr / sum w^2,
// the window's float values squared and summed in double
float welch_fac(double sr, int L) {
    double s = 0.0;
    for (int i = 0; i < L; ++i) {
        const float wi = L == 1 ? 1.0f : (float)(0.5 - 0.5 * cos(2.0 * 3.141592653589793 * (double)i / (double)(L - 1)));
        s += (double)wi * (double)wi;
    }
    return (float)(2.0 * sr / s);
}

#define GWB_TRY(call)                  \
    do {                               \
        const int st_ = (call);        \
        if (st_ != GWB_OK) return st_; \
    } while (0)

}  // namespace

extern "C" {

long long gwb_filter_batch_work_bytes(const GwbTile* tiles, int ntiles, int M, int nseg, long long tlen,
                                      const GwbCondConfig* cond, const GwbStepConfig* cfg) {
    CondShapes s;
    if (cond_shapes(tlen, cond, &s) != GWB_OK || nseg <= 0) return -1;
    CondWork w;
    const long long head = cond_carve(s, nseg, cond, nullptr, &w);
    const long long step = gwb_filter_step_work_bytes(tiles, ntiles, M, nseg, tlen, s.flen, s.kmin, cfg);
    return step < 0 ? -1 : head + step + 256;
}

int gwb_filter_batch(gwb_handle_t h, const float* x, long long ldx, int nseg, long long tlen,
                     const GwbCondConfig* cond, const GwbTile* tiles, int ntiles, const float* H, long long ldh, int M,
                     const int32_t* kmax, const int32_t* nbins, const float* isw, const GwbStepConfig* cfg, void* work,
                     long long work_bytes, float* D, float* IP, GwbCand* cands, GwbPeak* peaks, int32_t* counters,
                     double* sig, void* stream) {
    using namespace gwb;
    GWB_CHECK_ARG(h && x && work && D && IP, GWB_ERR_ARG, "filter_batch: null pointer");
    CondShapes s;
    GWB_TRY(cond_shapes(tlen, cond, &s));
    GWB_CHECK_ARG(nseg > 0 && ldx >= tlen, GWB_ERR_SHAPE, "filter_batch: nseg=%d ldx=%lld tlen=%lld", nseg, ldx, tlen);
    const long long need = gwb_filter_batch_work_bytes(tiles, ntiles, M, nseg, tlen, cond, cfg);
    GWB_CHECK_ARG(need > 0 && work_bytes >= need, GWB_ERR_SHAPE, "filter_batch: work %lld bytes, %lld needed",
                  work_bytes, need);
    char* base = reinterpret_cast<char*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
    CondWork w;
    const long long head = cond_carve(s, nseg, cond, base, &w);
    cudaStream_t st = (cudaStream_t)stream;
    const int L = cond->psd_len, flen = s.flen, n = (int)tlen;
    const float dt = (float)(1.0 / cond->sr);
    hann_kernel<<<(unsigned)cdiv(L, 256), 256, 0, st>>>(w.w, L);
    GWB_LAUNCH_CHECK("hann_kernel");
    iota_kernel<<<(unsigned)cdiv(nseg, 256), 256, 0, st>>>(w.pick, nseg);
    GWB_LAUNCH_CHECK("iota_kernel");
    // median (or mean) Welch PSD of each chunk over its whole length, interpolated onto the chunk's bins
    GWB_TRY(gwb_frames(x, ldx, nseg, 0, cond->psd_stride, nullptr, s.nfr, L, w.w, w.frames, L, st));
    GWB_TRY(gwb_fft_r2c(h, w.frames, w.F, L, nseg * s.nfr, L, s.nb, st));
    GWB_TRY(gwb_welch_avg(w.F, s.nb, nseg, s.nfr, s.nb, dt, cond->median, median_bias(s.nfr),
                          welch_fac(cond->sr, L), w.psd_w, s.nb, st));
    GWB_TRY(gwb_interp(w.psd_w, s.nb, nseg, s.nb, 1.0 / (1.0 / cond->sr) / (double)L, s.df, flen, w.psd, flen, st));
    if (cond->inv_len > 0) {
        // inverse spectrum truncation to inv_len samples (optionally Hann-tapered)
        if (cond->inv_taper) {
            hann_kernel<<<(unsigned)cdiv(cond->inv_len, 256), 256, 0, st>>>(w.tw, cond->inv_len);
            GWB_LAUNCH_CHECK("hann_kernel");
        }
        GWB_TRY(gwb_ist_pre(w.psd, flen, nseg, flen, s.kmin, w.inv, flen, st));
        GWB_TRY(gwb_fft_c2r(h, w.inv, w.q, n, nseg, flen, n, st));
        GWB_TRY(gwb_ist_mid(w.q, n, nseg, n, (float)s.df, cond->inv_len, cond->inv_taper ? w.tw : nullptr, st));
        GWB_TRY(gwb_fft_r2c(h, w.q, w.pt, n, nseg, n, flen, st));
        GWB_TRY(gwb_ist_post(w.pt, flen, nseg, flen, (float)(1.0 / (s.df * (double)n)), w.psd, flen, st));
    }
    // segment rFFT, D = stilde / psd and IP = 1 / psd (gpu_stage2)
    GWB_TRY(gwb_fft_r2c(h, x, w.st, n, nseg, ldx, flen, st));
    GWB_TRY(gwb_d_ip(w.st, flen, nseg, w.psd, flen, w.pick, flen, s.kmin, dt, D, flen, IP, flen, st));
    // the filter step on the conditioned batch
    return gwb_filter_step(tiles, ntiles, H, ldh, M, kmax, nbins, s.kmin, s.df, D, IP, flen, flen, nseg, isw, tlen,
                           flen, cfg, base + head, work_bytes - (head + (base - reinterpret_cast<char*>(work))), cands,
                           peaks, counters, sig, st);
}

}  // extern "C"
