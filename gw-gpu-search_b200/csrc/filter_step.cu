// The whole filter step through the C ABI: template norms, D isw in four-step order, then for every (tile, segment)
// the basis series, stacked A, fused GEMM with |z|^2 and windowed argmax and the window selection, then the exact
// stage over every candidate (edges, binned sums in template-row order, finalisation). It is the loop of
// pipeline/fp_filter.py:700-888 over one batch of segments (the reference's run_group, :741-836), as gwb200's
// MatchedFilter.step runs it from Python, for a caller that has no Python: every array is the caller's (inputs,
// outputs and one workspace), every launch goes to the caller's stream, nothing is copied to the host.
#include <string.h>
#include "common.cuh"

namespace {

struct Carve {
    char* base;
    long long off, size;
    template <typename T>
    T* take(long long n) {
        off = (off + 255) & ~255ll;
        T* p = reinterpret_cast<T*>(base ? base + off : nullptr);
        off += n * (long long)sizeof(T);
        return p;
    }
};

struct StepShapes {
    int rmax, nmax, khmax, K, lda, nw;
    long long ldz, Tn, ldp;
};

int shapes_of(const GwbTile* tiles, int ntiles, long long tlen, const GwbStepConfig* cfg, StepShapes* s) {
    using namespace gwb;
    GWB_CHECK_ARG(tiles && ntiles > 0 && cfg, GWB_ERR_ARG, "filter_step: null tiles or config");
    GWB_CHECK_ARG((cfg->form >= 0 && cfg->form <= 2) || cfg->form == 6, GWB_ERR_ARG,
                  "filter_step: form %d (0 fp16, 1 bf16, 2 split bf16, 6 fp16 with split A)", cfg->form);
    GWB_CHECK_ARG(is_pow2(tlen) && tlen >= (1 << 12) && tlen <= (1 << 20), GWB_ERR_NOT_POW2,
                  "filter_step: tlen=%lld must be a power of two in [2^12, 2^20]", tlen);
    GWB_CHECK_ARG(cfg->cw > 0 && cfg->cw % 128 == 0 && cfg->a0 >= 0 && cfg->Tn >= cfg->cw &&
                      cfg->a0 + cfg->Tn <= tlen && cfg->cand_cap > 0 && cfg->nbins_max >= 1,
                  GWB_ERR_SHAPE, "filter_step: cw=%d a0=%lld Tn=%lld cand_cap=%d", cfg->cw, cfg->a0, cfg->Tn,
                  cfg->cand_cap);
    s->rmax = s->nmax = 0;
    for (int t = 0; t < ntiles; ++t) {
        GWB_CHECK_ARG(tiles[t].Vp && tiles[t].A && tiles[t].r > 0 && tiles[t].n > 0 && tiles[t].r <= tiles[t].n &&
                          tiles[t].row0 >= 0, GWB_ERR_SHAPE, "filter_step: tile %d (r=%d n=%d)", t, tiles[t].r,
                      tiles[t].n);
        s->rmax = std::max(s->rmax, tiles[t].r);
        s->nmax = std::max(s->nmax, tiles[t].n);
    }
    s->khmax = (s->rmax + 15) / 16 * 16;
    s->K = 2 * s->khmax;
    s->lda = (s->K + 15) / 16 * 16;
    s->nw = (int)(cfg->Tn / cfg->cw);
    s->Tn = (long long)s->nw * cfg->cw;
    s->ldz = (s->Tn + 15) / 16 * 16;
    s->ldp = tlen / 2 + 2;
    return GWB_OK;
}

// the workspace layout (base null: sizes only)
struct StepWork {
    double* part;
    float *Dp, *tw, *W, *scale;
    double* partials;
    uint32_t* ticket;
    uint16_t *Z, *Zlo, *Are, *Are_lo;
    float* V;
    int32_t* I;
    void* gemm_work;
    GwbGroup* groups;
    GwbUnit* units;
    int32_t* E;
    float* slots;
    void* sort_work;
    int32_t* sort_status;
    long long gemm_bytes, sort_bytes, npartials;
    int wrows;
};

long long carve(const StepShapes& s, int M, int nseg, long long tlen, int flen, int kmin, const GwbStepConfig* cfg,
                void* base, StepWork* w) {
    Carve c{static_cast<char*>(base), 0, 0};
    const int split = cfg->form == 2, split_a = cfg->form == 2 || cfg->form == 6;
    const long long cap = cfg->cand_cap;
    w->part = c.take<double>((long long)M * nseg * 16);
    w->Dp = c.take<float>(2ll * nseg * s.ldp);
    w->tw = c.take<float>(2ll * tlen);
    w->wrows = s.rmax;           // the two-pass basis series, W for all of a tile's rows (the ring measured slower)
    w->W = c.take<float>(2ll * tlen * w->wrows);
    w->npartials = std::max(1024ll, 64ll * std::max(1ll, tlen / 64));
    w->partials = c.take<double>(w->npartials);
    w->scale = c.take<float>(1);
    w->ticket = c.take<uint32_t>(1);
    w->Z = c.take<uint16_t>((long long)s.K * s.ldz);
    w->Zlo = split ? c.take<uint16_t>((long long)s.K * s.ldz) : nullptr;
    w->Are = c.take<uint16_t>((long long)s.nmax * s.lda);
    w->Are_lo = split_a ? c.take<uint16_t>((long long)s.nmax * s.lda) : nullptr;
    w->V = c.take<float>((long long)s.nmax * s.nw);
    w->I = c.take<int32_t>((long long)s.nmax * s.nw);
    w->gemm_bytes = gwb_fused_peaks_cplx_work_bytes(s.nmax);
    w->gemm_work = c.take<char>(w->gemm_bytes);
    w->groups = c.take<GwbGroup>(cap);
    w->units = c.take<GwbUnit>(cap);
    w->E = c.take<int32_t>(cap * (cfg->nbins_max + 1));
    w->slots = c.take<float>(2ll * cap * gwb_exact_chunks(flen, kmin) * cfg->nbins_max);
    w->sort_bytes = gwb_bin_sums_work_bytes((int)cap, M);
    w->sort_work = c.take<char>(w->sort_bytes);
    w->sort_status = c.take<int32_t>(1);
    return c.off;
}

#define GWB_TRY(call)                  \
    do {                               \
        const int st_ = (call);        \
        if (st_ != GWB_OK) return st_; \
    } while (0)

}  // namespace

extern "C" {

long long gwb_filter_step_work_bytes(const GwbTile* tiles, int ntiles, int M, int nseg, long long tlen, int flen,
                                     int kmin, const GwbStepConfig* cfg) {
    StepShapes s;
    if (shapes_of(tiles, ntiles, tlen, cfg, &s) != GWB_OK || M <= 0 || nseg <= 0) return -1;
    StepWork w;
    return carve(s, M, nseg, tlen, flen, kmin, cfg, nullptr, &w) + 256;
}

int gwb_filter_step(const GwbTile* tiles, int ntiles, const float* H, long long ldh, int M, const int32_t* kmax,
                    const int32_t* nbins, int kmin, double df, const float* D, const float* IP, long long ldd,
                    long long ldip, int nseg, const float* isw, long long tlen, int flen, const GwbStepConfig* cfg,
                    void* work, long long work_bytes, GwbCand* cands, GwbPeak* peaks, int32_t* counters, double* sig,
                    void* stream) {
    using namespace gwb;
    StepShapes s;
    GWB_TRY(shapes_of(tiles, ntiles, tlen, cfg, &s));
    GWB_CHECK_ARG(H && kmax && nbins && D && IP && isw && work && cands && peaks && counters && sig, GWB_ERR_ARG,
                  "filter_step: null pointer");
    GWB_CHECK_ARG(M > 0 && nseg > 0 && flen == tlen / 2 + 1 && ldd >= flen && ldip >= flen && ldh >= flen &&
                      kmin > 0 && kmin < flen, GWB_ERR_SHAPE, "filter_step: M=%d nseg=%d flen=%d kmin=%d", M, nseg,
                  flen, kmin);
    for (int t = 0; t < ntiles; ++t)
        GWB_CHECK_ARG(tiles[t].row0 + tiles[t].n <= M, GWB_ERR_SHAPE, "filter_step: tile %d past the bank", t);
    const long long need = gwb_filter_step_work_bytes(tiles, ntiles, M, nseg, tlen, flen, kmin, cfg);
    GWB_CHECK_ARG(work_bytes >= need, GWB_ERR_SHAPE, "filter_step: work %lld bytes, %lld needed", work_bytes, need);
    char* base = reinterpret_cast<char*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
    StepWork w;
    carve(s, M, nseg, tlen, flen, kmin, cfg, base, &w);
    cudaStream_t st = (cudaStream_t)stream;
    const int cap = cfg->cand_cap, B = cfg->nbins_max;
    // Z encoding of the basis series and operand encoding of stacked A and the selection: f16, bf16, split bf16, and
    // for the fp16 form with split A, fp16 Z with fp16 hi + lo A
    const int pack = cfg->form == 0 ? 0 : (cfg->form == 1 ? 3 : (cfg->form == 2 ? 2 : 0));
    const int apack = cfg->form == 6 ? 5 : pack;
    GWB_CUDA(cudaMemsetAsync(counters, 0, 5 * sizeof(int32_t), st));
    GWB_CUDA(cudaMemsetAsync(w.ticket, 0, sizeof(uint32_t), st));
    // the Z rows past a tile's rank (up to its 16-row K step) are read by the GEMM against zero columns of A: they must
    // hold finite values, so the planes start at zero (a smaller rank later leaves finite values there)
    GWB_CUDA(cudaMemsetAsync(w.Z, 0, 2ll * s.K * s.ldz, st));
    if (w.Zlo) GWB_CUDA(cudaMemsetAsync(w.Zlo, 0, 2ll * s.K * s.ldz, st));
    // template norms (float64) and every segment's D isw in four-step order
    GWB_TRY(gwb_sigma2(H, ldh, M, IP, ldip, nseg, kmin, flen, df, w.part, (long long)M * nseg * 16, sig, nseg, st));
    GWB_TRY(gwb_fourstep_order(D, ldd, nseg, isw, flen, tlen, w.Dp, s.ldp, st));
    GWB_TRY(gwb_fft_twiddles(tlen, w.tw, st));
    const float thr2 = (float)((double)cfg->snr_threshold * (1.0 - cfg->margin) *
                               ((double)cfg->snr_threshold * (1.0 - cfg->margin)));
    for (int t = 0; t < ntiles; ++t) {
        const GwbTile& T = tiles[t];
        const int kh = (T.r + 15) / 16 * 16;
        for (int sg = 0; sg < nseg; ++sg) {
            const float* dp = w.Dp + 2ll * sg * s.ldp;
            GWB_TRY(gwb_basis_fused(T.Vp, T.ldvp, T.r, dp, tlen, w.tw, w.W, s.rmax, cfg->a0, s.Tn, pack, w.Z, w.Zlo,
                                    s.ldz, kh, 0, std::min(64, T.r), w.partials, w.npartials, w.ticket, w.scale,
                                    nullptr, nullptr, 0, st));
            GWB_TRY(gwb_stacked_a(T.A, T.lda, T.n, T.r, sig + (long long)T.row0 * nseg + sg, nseg, 4.0 * df,
                                  w.scale, 2 * kh, kh, apack, w.Are, nullptr, w.Are_lo, nullptr, s.lda, st));
            GWB_TRY(gwb_fused_peaks_cplx(cfg->form, w.Are, w.Are_lo, s.lda, w.Z, w.Zlo, s.ldz, T.n, kh, s.Tn,
                                         cfg->cw / 128, w.V, w.I, s.nw, nullptr, w.gemm_work, w.gemm_bytes, st));
            GWB_TRY(gwb_select_windows(w.V, w.I, s.nw, T.n, s.nw, thr2, 0.f, cfg->snr_threshold, cfg->a0, T.row0, sg,
                                       w.Are, nullptr, w.Are_lo, nullptr, s.lda, w.Z, w.Zlo, s.ldz, 2 * kh, kh, apack,
                                       nullptr, cands, cap, w.groups, cap, w.units, cap, nullptr, 0, counters, st));
        }
    }
    // the exact stage over every candidate of the step
    GWB_TRY(gwb_edges(w.units, counters + 2, cap, H, ldh, IP, ldip, nbins, kmax, kmin, B, 0, w.E, st));
    GWB_TRY(gwb_bin_sums_ordered(w.groups, counters + 1, cap, w.units, cands, w.E, B, nbins, M, H, ldh, D, ldd, kmin,
                                 flen, tlen, w.sort_work, w.sort_bytes, w.sort_status, w.slots, st));
    GWB_TRY(gwb_exact_finalize(cands, counters, cap, w.units, w.E, B, nbins, kmin, flen, w.slots, sig, nseg, df, peaks,
                               st));
    return GWB_OK;
}

}  // extern "C"
