"""Batched matched filter over many segments: the device-resident replacement of fp_filter.py's per (tile, segment)
loop (pipeline/fp_filter.py:700-888).

Layout in HBM (all resident for a run):
  H      (M, flen) complex64   every template of the bank, tile after tile (rows sorted by chirp time); read by the
                               Gram/Vh setup and by the exact stage
  Vh_t   (r_t, flen) complex64 per tile basis filters (and Vp_t, the same in four-step order for the fused basis
                               series); A_t (n_t, r_t) complex64 mixing matrices
  Dp     (S, tlen/2 + 1)       D isw of every segment in four-step order
  D, IP  (S, flen)             over-whitened data and inverse PSD of every segment
  sig    (M, S) float64        template norms
  Z      (Kp, Tn)              basis series of the current (tile, segment), fp16 / fp32 / bf16 hi+lo
  V, I   (n, nw)               per-window max |SNR|^2 and sample straight from the GEMM epilogue (group = cw/128)
  cands, groups, units         candidate lists of the whole step, appended by the selection kernel
One step = every tile against a batch of segments: basis series -> stacked A -> fused GEMM (+|z|^2, window argmax)
-> selection, then one exact stage over all candidates (edges, binned sums, finalisation) and a single copy of the
results to the host. The step's launch sequence is fixed, so it can be captured once in a CUDA graph and replayed.
"""
from dataclasses import dataclass

import numpy as np
import torch

from . import _exact, _lib, autotune, fp_filter, templates

BN = 128


@dataclass
class FilterConfig:
    f_low: float = 20.0
    sr: float = 2048.0
    tile: int = 256
    eps: float = 1e-3
    nbins: int = 16
    cluster_window: float = 1.0
    snr_threshold: float = 5.5
    margin: float = 0.04
    screen_margin: float = 0.10   # fp8 form: candidates down to thr (1 - screen_margin); the exact stage decides
    form: str = 'bf16x3'          # GEMM operands: f16, bf16, bf16x3 (split bf16), f16x2 (fp16, A hi + lo), fp8, f32
    cand_cap: int = 1 << 21
    seg_batch: int = 16
    # the reference's --exact-snr split (fp_filter.py:769-781): windows whose rebuilt SNR is below
    # exact_snr (1 - margin) skip the exact stage and keep their rebuilt SNR and phase when above snr_threshold;
    # 0 sends every candidate to the exact stage (PyCBC-equivalent values)
    exact_snr: float = 0.0
    # rank rules instead (gwb_select_top): per segment only the exact_top loudest candidates by rebuilt SNR, or the
    # loudest fraction exact_top_frac of them, go to the exact stage; the others above snr_threshold keep their
    # rebuilt SNR and phase (rebuilt peaks). 0: off
    exact_top: int = 0
    exact_top_frac: float = 0.0
    # local search of a screening form (gwb_search_expand / gwb_search_best): the exact stage at the 2 r + 1 samples
    # around each candidate's rebuilt argmax inside its window, keeping the loudest; 0: off
    screen_search: int = 0
    rebuilt_cap: int = 0          # capacity of the rebuilt-peak list (0: cand_cap)
    exact_order: bool = True      # exact stage in template-row order, chunk by chunk (gwb_bin_sums_ordered)
    # time the GEMM launch configurations of every tile width and the basis-series forms on this run's shapes before
    # the first step, and use the fastest (gwb200.autotune)
    autotune: bool = False


class Bank:
    """Template bank on the device: templates for every row (tile order), and each tile's SVD compression."""

    def __init__(self, params, flen, df, sw, cfg: FilterConfig, device='cuda'):
        self.cfg = cfg
        self.flen, self.df = flen, df
        self.kmin = int(cfg.f_low / df)
        self.tiles = templates.tiles(params, cfg.tile, cfg.f_low)
        self.order = np.concatenate(self.tiles)                     # global row -> bank index
        M = len(self.order)
        self.M = M
        self.H = torch.empty((M, flen), dtype=torch.complex64, device=device)
        km = np.empty(M, np.int32)
        self.row0 = []
        r0 = 0
        for ids in self.tiles:
            _, k = templates.generate(params, ids, flen, df, cfg.f_low, out=self.H[r0:r0 + len(ids)], device=device)
            km[r0:r0 + len(ids)] = k
            self.row0.append(r0)
            r0 += len(ids)
        self.kmax = torch.from_numpy(km).to(device)
        self.kmax_h = km
        self.nbins = torch.full((M,), cfg.nbins, dtype=torch.int32, device=device)
        self.svd = []
        for t, ids in enumerate(self.tiles):
            Ht = self.H[self.row0[t]:self.row0[t] + len(ids)]
            r, A, Vh, worst = fp_filter.svd_tile(Ht, sw, self.kmin, cfg.eps)
            self.svd.append(dict(r=r, A=A, Vh=Vh, worst=worst, Kp=fp_filter.kp_of(r), Kh=fp_filter.kh_of(r)))

    @property
    def r_over_n(self):
        return sum(s['r'] for s in self.svd) / self.M


class MatchedFilter:
    """Runs steps of the batched filter for one bank and one segment geometry (tlen, analysed span)."""

    def __init__(self, bank: Bank, tlen, a0, Tn, cfg: FilterConfig, device='cuda'):
        self.bank, self.cfg = bank, cfg
        self.tlen, self.a0 = tlen, a0
        cw = int(cfg.cluster_window * cfg.sr)
        assert cw % BN == 0, 'cluster window must be a multiple of %d samples' % BN
        self.cw, self.group = cw, cw // BN
        self.nw = Tn // cw
        self.Tn = self.nw * cw
        self.form = cfg.form
        # fp16 / bf16 / split bf16 / fp8 use the compact complex operands on the tensor cores (A = [ReA | ImA], Z =
        # [ReZ ; ImZ], halves of Kh rows); the plain fp32 form uses the reference's stacked layout on the fp32 pipe.
        # fp8 (e4m3, per-row scales) is a screening form: its candidates go to the exact stage with a wider margin
        self.compact = self.form != 'f32'
        self.fp8 = self.form == 'fp8'
        rmax = max(s['r'] for s in bank.svd)
        # the fused two-pass basis series (premul and pack folded into the transform passes) where the length allows,
        # else premul + cuFFT + pack
        self.fused = fp_filter.FUSED_MIN <= tlen <= fp_filter.FUSED_MAX
        self.tuning = None
        if cfg.autotune:
            self.tuning = autotune.tune_filter(bank, tlen, self.Tn, self.form, self.group, device=device)
        if self.fused:
            bt = self.tuning['basis']['best'] if self.tuning and self.tuning['basis'] else {}
            self.fws = fp_filter.FusedBasisWorkspace(tlen, bank.flen, rmax, device, wrows=bt.get('wrows'),
                                                     ring=bt.get('ring'))
            # basis filters in the four-step order of the transform, once per tile; D isw per step (self.Dp)
            self.vp = [fp_filter.fourstep_order(s['Vh'], tlen) for s in bank.svd]
            self.Dp = None
        else:
            self.ws = fp_filter.BasisWorkspace(tlen, bank.flen, fp_filter.RB, device)
        assert self.fused or not self.fp8, 'the fp8 form needs the fused basis series (tlen in [2^12, 2^20])'
        self.khs = [fp_filter.kh_of(s['r'], self.form) if self.compact else 0 for s in bank.svd]
        if self.compact:
            K = 2 * max(self.khs)
        else:
            K = max(s['Kp'] for s in bank.svd)
        nmax = max(len(t) for t in bank.tiles)
        dt = fp_filter._z_dtype(self.form)
        ldz = -(-self.Tn // 16) * 16          # rows on 16-byte boundaries (TMA) for every element size
        self.Z = torch.zeros((K, ldz), dtype=dt, device=device)
        self.Zlo = torch.zeros_like(self.Z) if self.form == 'bf16x3' else None
        lda = -(-K // 16) * 16
        self.Are = torch.zeros((nmax, lda), dtype=dt, device=device)
        self.Aim = None if self.compact else torch.zeros_like(self.Are)
        self.Are_lo = torch.zeros_like(self.Are) if self.form in ('bf16x3', 'f16x2') else None
        self.Aim_lo = None
        self.sa = torch.empty(nmax, dtype=torch.float32, device=device) if self.fp8 else None   # A row scales
        self.V = torch.empty((nmax, self.nw), dtype=torch.float32, device=device)
        # partial window maxima of the GEMM's tile-granular CTA ranges
        self.gemm_work = torch.empty(_lib.load().gwb_fused_peaks_cplx_work_bytes(nmax), dtype=torch.uint8,
                                     device=device) if self.compact else None
        self.I = torch.empty((nmax, self.nw), dtype=torch.int32, device=device)
        cap = cfg.cand_cap
        # the exact stage's lists: with a local search each selected window becomes 2 r + 1 candidates
        self.search = int(cfg.screen_search)
        self.search_w = 2 * self.search + 1 if self.search else 1
        capx = cap * self.search_w
        self.cands = torch.empty(capx * _exact.CAND.itemsize, dtype=torch.uint8, device=device)
        self.groups = torch.empty(capx * _exact.GROUP.itemsize, dtype=torch.uint8, device=device)
        self.units = torch.empty(capx * _exact.UNIT.itemsize, dtype=torch.uint8, device=device)
        self.counters = torch.zeros(5, dtype=torch.int32, device=device)
        self.B = cfg.nbins
        self.E = torch.empty((capx, self.B + 1), dtype=torch.int32, device=device)
        self.nchunk = _lib.load().gwb_exact_chunks(bank.flen, bank.kmin)
        self.slot_cap = capx
        assert capx <= 1 << 24
        self.slots = None
        if cfg.exact_order:
            wb = _lib.load().gwb_bin_sums_work_bytes(capx, bank.M)
            self.sort_work = torch.empty(wb, dtype=torch.uint8, device=device)
            self.sort_status = torch.zeros(1, dtype=torch.int32, device=device)
        self.peaks = torch.empty(capx * _exact.PEAK.itemsize, dtype=torch.uint8, device=device)
        margin = max(cfg.margin, cfg.screen_margin) if self.fp8 else cfg.margin
        self.thr2 = float((cfg.snr_threshold * (1 - margin)) ** 2)
        assert not (self.fp8 and cfg.exact_snr > 0), 'the fp8 screen keeps no rebuilt values: use exact_snr = 0'
        self.ecut = float(np.float32(cfg.exact_snr * (1 - cfg.margin))) if cfg.exact_snr > 0 else 0.0
        self.rthr = float(np.float32(cfg.snr_threshold))
        self.top = cfg.exact_top > 0 or cfg.exact_top_frac > 0
        assert not (self.top and cfg.exact_snr > 0), 'one exact-stage rule at a time: exact_snr or exact_top(_frac)'
        assert not (self.search and (self.top or cfg.exact_snr > 0)), 'the local search takes every candidate'
        self.rebuilt_cap = cfg.rebuilt_cap or cap
        self.rebuilt = (torch.empty(self.rebuilt_cap * _exact.CAND.itemsize, dtype=torch.uint8, device=device)
                        if cfg.exact_snr > 0 or self.top else None)
        # the selection's own lists: with a rank rule the windows are selected into these, then gwb_select_top
        # moves the ranked subset into cands / groups / units / counters for the exact stage
        if self.top or self.search:
            self.sel = dict(cands=torch.empty(cap * _exact.CAND.itemsize, dtype=torch.uint8, device=device),
                            groups=torch.empty(cap * _exact.GROUP.itemsize, dtype=torch.uint8, device=device),
                            units=torch.empty(cap * _exact.UNIT.itemsize, dtype=torch.uint8, device=device),
                            counters=torch.zeros_like(self.counters))
            self.top_work = None
        else:
            self.sel = dict(cands=self.cands, groups=self.groups, units=self.units, counters=self.counters)
        self.kernel_launches = 0
        self.fft_launches = 0
        # set to {} to record CUDA events per (tile, segment): e0 basis series e3 stacked A e1 GEMM e2 (then the
        # selection until the next e0), and ('parts': norms, four-step order of D, exact stage) per step
        self.profile = None

    def _gemm(self, n, K, Kh):
        s = _lib.stream_ptr()
        if self.compact:
            code = {'f16': 0, 'bf16': 1, 'bf16x3': 2, 'fp8': 3, 'f16x2': 6}[self.form]
            _lib.call('gwb_fused_peaks_cplx', code, _lib.ptr(self.Are), _lib.ptr(self.Are_lo), self.Are.stride(0),
                      _lib.ptr(self.Z), _lib.ptr(self.Zlo), self.Z.stride(0), n, Kh, self.Tn, self.group,
                      _lib.ptr(self.V), _lib.ptr(self.I), self.V.stride(0), _lib.ptr(self.sa),
                      _lib.ptr(self.gemm_work), self.gemm_work.numel(), s)
        else:
            _lib.call('gwb_fused_peaks_f32', _lib.ptr(self.Are), _lib.ptr(self.Aim), self.Are.stride(0),
                      _lib.ptr(self.Z), self.Z.stride(0), n, K, self.Tn, self.group, _lib.ptr(self.V), _lib.ptr(self.I),
                      self.V.stride(0), s)

    def clear_padding(self, t):
        """Zeroes the rows of Z (and Zlo) that tile t's GEMM reads but its basis series does not write: between its r
        basis rows and its width Kh in the real and the imaginary half (compact forms), or from 2 r to Kp. The GEMM
        multiplies them by A's zero columns, so whatever another tile or step left there must not be a NaN or an
        infinity (a step on empty data leaves both)."""
        r = self.bank.svd[t]['r']
        if self.compact:
            Kh = self.khs[t]
            spans = [(r, Kh), (Kh + r, 2 * Kh)] if Kh > r else []
        else:
            Kp = self.bank.svd[t]['Kp']
            spans = [(2 * r, Kp)] if Kp > 2 * r else []
        for Zp in (self.Z, self.Zlo):
            if Zp is not None:
                for a, b in spans:
                    Zp[a:b].zero_()

    def tile_segment(self, t, D, isw, sig, seg):
        """Basis series, stacked A, fused GEMM and window selection of tile t against segment seg (row of D)."""
        b = self.bank
        sv = b.svd[t]
        n = len(b.tiles[t])
        r = sv['r']
        Kh = self.khs[t]
        K = 2 * Kh if self.compact else sv['Kp']
        prof = self.profile
        if prof is not None:
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            e[0].record()
        im_off = Kh if self.compact else r
        if self.fused:
            scale = fp_filter.basis_series_fused(self.fws, self.vp[t], self.Dp[seg], self.a0, self.Tn, self.Z,
                                                 self.Zlo, self.form, im_off=im_off)
        else:
            scale = fp_filter.basis_series_into(self.ws, sv['Vh'], D[seg], isw, self.a0, self.Tn, self.Z,
                                                self.Zlo, self.form, im_off=im_off)
        if prof is not None:
            e[3].record()
        nrm = sig[b.row0[t]:b.row0[t] + n, seg]
        if self.fp8:
            fp_filter.stacked_A8_into(sv['A'], nrm, self.fws.rowscale, Kh, self.Are, self.sa, df4=4.0 * b.df)
        else:
            fp_filter.stacked_A_into(sv['A'], nrm, scale, K, self.Are, self.Aim, self.Are_lo, self.Aim_lo, self.form,
                                     df4=4.0 * b.df, kh=Kh)
        if prof is not None:
            e[1].record()
        self._gemm(n, K, Kh)
        if prof is not None:
            e[2].record()
            prof.setdefault('launches', []).append((e, n, r, K))
        f = fp_filter.A_FORMS[self.form]
        cap = self.cfg.cand_cap
        _lib.call('gwb_select_windows', _lib.ptr(self.V), _lib.ptr(self.I), self.V.stride(0), n, self.nw, self.thr2,
                  self.ecut, self.rthr, self.a0, b.row0[t], seg, _lib.ptr(self.Are), _lib.ptr(self.Aim),
                  _lib.ptr(self.Are_lo), _lib.ptr(self.Aim_lo), self.Are.stride(0), _lib.ptr(self.Z),
                  _lib.ptr(self.Zlo), self.Z.stride(0), K, Kh, f, _lib.ptr(self.sa), _lib.ptr(self.sel['cands']), cap,
                  _lib.ptr(self.sel['groups']), cap, _lib.ptr(self.sel['units']), cap, _lib.ptr(self.rebuilt),
                  self.rebuilt_cap if self.rebuilt is not None else 0, _lib.ptr(self.sel['counters']),
                  _lib.stream_ptr())
        if self.fused and self.fws.ring:
            self.kernel_launches += 4           # the persistent basis series, stacked A, GEMM, selection
        elif self.fused:
            nb = -(-r // self.fws.wrows)
            self.kernel_launches += 2 * nb + 3  # two basis passes per row batch, stacked A, GEMM, selection
        else:
            nb = -(-r // fp_filter.RB)
            self.kernel_launches += 2 * nb + 4  # premul and pack per batch; scale, stacked A, GEMM, selection
            self.fft_launches += nb

    def norms(self, IP):
        """Template norms for every (row, segment): sig (M, S) float64 = 4 df sum |H|^2 IP (fp_filter.py:710-714)."""
        b = self.bank
        nseg = IP.shape[0]
        sig = torch.empty((b.M, nseg), dtype=torch.float64, device=IP.device)
        part_elems = b.M * nseg * 16
        part = torch.empty(part_elems, dtype=torch.float64, device=IP.device)
        _lib.call('gwb_sigma2', _lib.ptr(b.H), b.H.stride(0), b.M, _lib.ptr(IP), _lib.row_stride(IP), nseg, b.kmin, b.flen,
                  float(b.df), _lib.ptr(part), part_elems, _lib.ptr(sig), sig.stride(0), _lib.stream_ptr())
        self.kernel_launches += 2
        return sig

    def exact(self, D, IP, sig):
        """Edges, binned sums and finalisation over every candidate of the step (device counts, no host sync)."""
        b = self.bank
        cap = self.cfg.cand_cap
        s = _lib.stream_ptr()
        cnt = self.counters
        if self.top:
            nseg = D.shape[0]
            if self.top_work is None or self.top_work.numel() < _lib.load().gwb_select_top_work_bytes(nseg, cap):
                self.top_work = torch.empty(_lib.load().gwb_select_top_work_bytes(nseg, cap), dtype=torch.uint8,
                                            device=D.device)
            sc = self.sel
            _lib.call('gwb_select_top', _lib.ptr(sc['cands']), _lib.ptr(sc['groups']), _lib.ptr(sc['units']),
                      _lib.ptr(sc['counters']), cap, nseg, int(self.cfg.exact_top), float(self.cfg.exact_top_frac),
                      self.rthr, _lib.ptr(self.cands), _lib.ptr(self.groups), _lib.ptr(self.units), _lib.ptr(cnt),
                      _lib.ptr(self.rebuilt), self.rebuilt_cap, _lib.ptr(self.top_work), self.top_work.numel(), s)
            self.kernel_launches += 5
        if self.search:
            sc = self.sel
            _lib.call('gwb_search_expand', _lib.ptr(sc['cands']), _lib.ptr(sc['units']), _lib.ptr(sc['counters']),
                      self.search, self.a0, self.cw, _lib.ptr(self.cands), self.slot_cap, _lib.ptr(self.groups),
                      _lib.ptr(self.units), _lib.ptr(cnt), s)
            self.kernel_launches += 1
        cap = self.slot_cap                    # the exact stage's lists
        _lib.call('gwb_edges', _lib.ptr(self.units), _lib.ptr(cnt[2:]), cap, _lib.ptr(b.H), b.H.stride(0),
                  _lib.ptr(IP), _lib.row_stride(IP), _lib.ptr(b.nbins), _lib.ptr(b.kmax), b.kmin, self.B, 0, _lib.ptr(self.E), s)
        if self.slots is None:
            # every slot the finalisation reads is written by the binned sums: no clearing between steps
            self.slots = torch.empty((self.slot_cap, self.nchunk, self.B, 2), dtype=torch.float32, device=D.device)
        if self.cfg.exact_order:
            _lib.call('gwb_bin_sums_ordered', _lib.ptr(self.groups), _lib.ptr(cnt[1:]), cap, _lib.ptr(self.units),
                      _lib.ptr(self.cands), _lib.ptr(self.E), self.B, _lib.ptr(b.nbins), b.M, _lib.ptr(b.H),
                      b.H.stride(0), _lib.ptr(D), _lib.row_stride(D), b.kmin, b.flen, self.tlen, _lib.ptr(self.sort_work),
                      self.sort_work.numel(), _lib.ptr(self.sort_status), _lib.ptr(self.slots), s)
            self.kernel_launches += 3
        else:
            _lib.call('gwb_bin_sums', _lib.ptr(self.groups), _lib.ptr(cnt[1:]), cap, _lib.ptr(self.units),
                      _lib.ptr(self.cands), _lib.ptr(self.E), self.B, _lib.ptr(b.nbins), _lib.ptr(b.H),
                      b.H.stride(0), _lib.ptr(D), _lib.row_stride(D), b.kmin, b.flen, self.tlen, _lib.ptr(self.slots), s)
        _lib.call('gwb_exact_finalize', _lib.ptr(self.cands), _lib.ptr(cnt[0:]), cap, _lib.ptr(self.units),
                  _lib.ptr(self.E), self.B, _lib.ptr(b.nbins), b.kmin, b.flen, _lib.ptr(self.slots), _lib.ptr(sig),
                  sig.stride(0), float(b.df), _lib.ptr(self.peaks), s)
        self.kernel_launches += 3
        if self.search:
            _lib.call('gwb_search_best', _lib.ptr(cnt[0:]), cap, self.search, _lib.ptr(self.peaks), s)
            self.kernel_launches += 1

    def step(self, D, IP, isw, seg_ids=None):
        """Queue one step on the current stream: every tile against every segment in seg_ids (rows of D / IP).
        Nothing is copied back; call results() after the stream is synchronised."""
        self.counters.zero_()
        if self.top or self.search:
            self.sel['counters'].zero_()
        prof = self.profile
        ev = (lambda: torch.cuda.Event(enable_timing=True)) if prof is not None else None
        if prof is not None:
            e_n = (ev(), ev())
            e_n[0].record()
        sig = self.norms(IP)
        if prof is not None:
            e_n[1].record()
            prof.setdefault('parts', []).append(('norms', e_n))
            e_f = (ev(), ev())
            e_f[0].record()
        if self.fused:
            # every segment's D isw in four-step order, shared by all tiles
            if self.Dp is None or self.Dp.shape[0] != D.shape[0]:
                self.Dp = torch.empty((D.shape[0], self.tlen // 2 + 1), dtype=torch.complex64, device=D.device)
            fp_filter.fourstep_order(D, self.tlen, isw, out=self.Dp)
            self.kernel_launches += 1
        if prof is not None:
            e_f[1].record()
            prof.setdefault('parts', []).append(('fourstep', e_f))
        segs = range(D.shape[0]) if seg_ids is None else seg_ids
        for t in range(len(self.bank.tiles)):
            self.clear_padding(t)
            for s in segs:
                self.tile_segment(t, D, isw, sig, s)
        if prof is not None:
            e_x = (ev(), ev())
            e_x[0].record()
        self.exact(D, IP, sig)
        if prof is not None:
            e_x[1].record()
            prof.setdefault('parts', []).append(('exact', e_x))
        return sig

    def results(self, sig=None, rebuilt_on_device=False):
        """Copy the step's candidates and exact values to the host; returns a dict of numpy arrays (all candidates
        and the kept peaks with exact SNR above the threshold; with exact_snr > 0 also the rebuilt peaks, whose SNR
        and phase are the rebuilt ones: `rebuilt`, GwbCand records, or with rebuilt_on_device `rebuilt_dev`, a view
        of the device list as an (n, 8) int32 tensor of the GwbCand fields)."""
        c = self.counters.cpu().numpy()
        if c[3] or ((self.top or self.search) and int(self.sel['counters'][3].item())):
            raise _lib.GwbError('select', _lib.GWB_ERR_CAPACITY, 'candidate capacity %d exceeded' % self.cfg.cand_cap)
        if self.cfg.exact_order and int(self.sort_status.item()):
            raise _lib.GwbError('bin_sums_ordered', _lib.GWB_ERR_SHAPE, 'a unit row outside the bank')
        n = int(c[0])
        cands = _exact.from_dev(self.cands, _exact.CAND, n)
        peaks = _exact.from_dev(self.peaks, _exact.PEAK, n)
        keep = peaks['snr'] > self.cfg.snr_threshold
        nr = int(c[4])
        out = dict(n_candidates=n, n_units=int(c[2]), n_groups=int(c[1]), cands=cands, peaks=peaks, keep=keep,
                   n_rebuilt=nr)
        if rebuilt_on_device:
            out['rebuilt_dev'] = (self.rebuilt[:nr * _exact.CAND.itemsize].view(torch.int32).view(nr, 8)
                                  if self.rebuilt is not None else torch.zeros((0, 8), dtype=torch.int32,
                                                                               device=self.cands.device))
        else:
            out['rebuilt'] = (_exact.from_dev(self.rebuilt, _exact.CAND, nr) if self.rebuilt is not None
                              else np.zeros(0, _exact.CAND))
        return out
