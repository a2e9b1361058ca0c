"""Autotuner of the launch shapes the filter uses, over the (K, chunk length) grid of a run: the fused GEMM's launch
table (CTA pairs or one CTA per M block, depth of the Z ring, order of the complex products' MMAs) for every basis
width Kh of the bank's tiles at the run's analysed length Tn, and the basis-series form (persistent ring with W in
L2, or two passes with W in batches) for the run's transform length.

The reference's counterpart is fp_gemm.pick_cfg (pipeline/fp_gemm.py:47-64): it times its Triton configurations
(BM, BK, warps, stages) once on one shape and keeps the fastest. Here every candidate is timed with CUDA events on
synthetic operands of the exact shape (a warm-up launch, then `reps` launches), the fastest is written into the
library's table (gwb_gemm_set_config) and kept in a cache keyed by (device, form, n, Kh, Tn), so a later bank or
MatchedFilter of the same shapes reuses it without timing. The candidates compute the same products; only the order
of the fp32 accumulation differs between MMA orders (identical V and I where the sums are exact, as in the tests;
otherwise the last bits of V and, at near-ties, I), so tuning changes speed, not precision.
"""
import torch

from . import _lib, fp_filter

FORM_CODE = {'f16': 0, 'bf16': 1, 'bf16x3': 2, 'fp8': 3, 'f16x2': 6}
# the persistent basis series' (rows per chunk, W slots, lookahead): W in L2 holds rows x slots rows of 8 MB at 2^20
# (lookahead 0: split roles, half the CTAs on each pass)
RING_CONFIGS = [(2, 3, 1), (2, 4, 2), (4, 2, 1), (2, 3, 0), (2, 2, 0), (4, 2, 0), (1, 4, 0)]
_CACHE = {}


def _events_ms(fn, reps):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def gemm_space(form):
    """The candidate launch configurations (pair, stages, order) of one form."""
    if form in ('f16', 'bf16'):
        return ([(1, st, o) for st in (0, 4) for o in (0, 1, 2, 3)] +
                [(0, st, 0) for st in (0, 3)])
    if form in ('bf16x3', 'f16x2'):        # the split forms: one CTA per M block, or CTA pairs
        return [(0, st, 0) for st in (0, 4, 3, 2)] + [(1, st, 0) for st in (0, 3, 2)] + [(1, 0, 1)]
    return [(0, st, 0) for st in (0, 4, 3, 2)]


def tune_gemm(form, n, Kh, Tn, group=16, reps=3, device='cuda'):
    """Times every candidate of gemm_space(form) for an (n x 2 Kh) by (2 Kh x Tn) launch; sets the fastest in the
    library's table and returns (best (pair, stages, order), {candidate: ms or error text})."""
    key = (torch.cuda.get_device_name(device), form, int(n), int(Kh), int(Tn))
    hit = _CACHE.get(key)
    code = FORM_CODE[form]
    if hit is not None:
        _lib.call('gwb_gemm_set_config', code, Kh, *hit[0])
        return hit
    g = torch.Generator(device=device).manual_seed(1)
    A = torch.randn((n, 2 * Kh), generator=g, device=device)
    ldz = -(-Tn // 16) * 16
    Z = torch.randn((2 * Kh, ldz), generator=g, device=device)
    if form == 'fp8':
        A, Z = A.to(torch.float8_e4m3fn).view(torch.uint8), Z.to(torch.float8_e4m3fn).view(torch.uint8)
    else:
        dt = torch.float16 if form in ('f16', 'f16x2') else torch.bfloat16
        A, Z = A.to(dt), Z.to(dt)
    lo = (A.clone(), Z.clone()) if form == 'bf16x3' else ((A.clone(), None) if form == 'f16x2' else (None, None))
    rs = torch.ones(n, device=device)
    ntiles = -(-Tn // 128)
    nout = -(-ntiles // group)
    V = torch.empty((n, nout), dtype=torch.float32, device=device)
    I = torch.empty((n, nout), dtype=torch.int32, device=device)
    work = torch.empty(_lib.load().gwb_fused_peaks_cplx_work_bytes(n), dtype=torch.uint8, device=device)

    def run():
        _lib.call('gwb_fused_peaks_cplx', code, _lib.ptr(A), _lib.ptr(lo[0]), A.stride(0), _lib.ptr(Z),
                  _lib.ptr(lo[1]), Z.stride(0), n, Kh, Tn, group, _lib.ptr(V), _lib.ptr(I), V.stride(0),
                  _lib.ptr(rs), _lib.ptr(work), work.numel(), _lib.stream_ptr())

    res, best = {}, None
    for cand in gemm_space(form):
        _lib.call('gwb_gemm_set_config', code, Kh, *cand)
        try:
            ms = _events_ms(run, reps)
        except _lib.GwbError as ex:          # a ring deeper than fits is refused before launch; reported
            res[cand] = str(ex)[:200]
            continue
        res[cand] = ms
        if best is None or ms < res[best]:
            best = cand
    if best is None:
        raise RuntimeError('no GEMM launch configuration ran: %r' % res)
    _lib.call('gwb_gemm_set_config', code, Kh, *best)
    _CACHE[key] = (best, res)
    return best, res


def tune_basis(tlen, r, form='f16', reps=2, device='cuda'):
    """Times the basis-series forms for r rows of length tlen: the ring (tlen = 2^20, RING_CONFIGS) and two passes with
    W for all rows or in batches of 32, with 8 or 16 columns per pass-2 CTA (16 at tlen = 2^20 only); sets the fastest
    and returns (best: dict(ring, wrows, ring_config, pass2_cols), {candidate: ms})."""
    key = (torch.cuda.get_device_name(device), 'basis', int(tlen), int(r), form)
    if key in _CACHE:
        out = _CACHE[key]
        _apply_basis(out[0], form)
        return out
    flen = tlen // 2 + 1
    g = torch.Generator(device=device).manual_seed(2)
    Vh = torch.randn((r, flen), generator=g, device=device, dtype=torch.complex64)
    D = torch.randn(flen, generator=g, device=device, dtype=torch.complex64)
    isw = torch.rand(flen, generator=g, device=device) + 0.5
    a0, Tn = tlen * 3 // 32, tlen * 28 // 32
    Kh = fp_filter.kh_of(r, form)
    Z = torch.zeros((2 * Kh, -(-Tn // 16) * 16), dtype=fp_filter._z_dtype(form), device=device)
    Zlo = torch.zeros_like(Z) if form == 'bf16x3' else None
    Vp = fp_filter.fourstep_order(Vh, tlen)
    Dp = fp_filter.fourstep_order(D, tlen, isw)
    cands = [(False, None, None, 16), (False, 32, None, 16)]
    if tlen == fp_filter.RING_N:
        cands = ([(True, None, rc, 16) for rc in RING_CONFIGS] + cands +
                 [(False, None, None, 8), (False, 32, None, 8)])
    res, best = {}, None
    for ring, wrows, rc, cols in cands:
        _apply_basis(dict(ring_config=rc, pass2_cols=cols), form)
        ws = fp_filter.FusedBasisWorkspace(tlen, flen, r, device=device, wrows=wrows, ring=ring)
        ms = _events_ms(lambda: fp_filter.basis_series_fused(ws, Vp, Dp, a0, Tn, Z, Zlo, form, im_off=Kh), reps)
        res[(ring, wrows, rc, cols)] = ms
        if best is None or ms < res[best]:
            best = (ring, wrows, rc, cols)
        del ws
    out = (dict(ring=best[0], wrows=best[1], ring_config=best[2], pass2_cols=best[3]), res)
    _apply_basis(out[0], form)
    _CACHE[key] = out
    return out


def _apply_basis(choice, form):
    """Sets a basis-series choice's knobs in the library: the ring configuration (process-wide) and the form's
    pass-2 columns."""
    if choice.get('ring_config') is not None:
        _lib.call('gwb_basis_ring_set_config', *choice['ring_config'])
    _lib.call('gwb_basis_set_pass2_columns', fp_filter.FORMS[form], int(choice.get('pass2_cols') or 16))


def tune_filter(bank, tlen, Tn, form, group, device='cuda'):
    """Tunes every (form, Kh) of the bank's tiles at the analysed length Tn, and the basis-series form at tlen for
    the bank's widest tile. Returns a report dict (chosen configurations and timings)."""
    rep = dict(gemm={}, basis=None)
    if form != 'f32':
        nmax = max(len(t) for t in bank.tiles)
        for kh in sorted({fp_filter.kh_of(s['r'], form) for s in bank.svd}):
            best, res = tune_gemm(form, nmax, kh, Tn, group, device=device)
            rep['gemm'][kh] = dict(best=best, ms={str(k): v for k, v in res.items()})
    if fp_filter.FUSED_MIN <= tlen <= fp_filter.FUSED_MAX:
        rmax = max(s['r'] for s in bank.svd)
        best, res = tune_basis(tlen, rmax, form, device=device)
        rep['basis'] = dict(best=best, ms={str(k): v for k, v in res.items()})
    return rep
