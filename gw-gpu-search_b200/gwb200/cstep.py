"""The whole filter step through the single C entry gwb_filter_step (the batched C entry a non-Python caller binds;
the loop of pipeline/fp_filter.py:700-888 over one batch of segments). This module only builds the C records
(GwbTile per tile, GwbStepConfig) from a Bank, owns the workspace and the output lists, and reads them back; the
ctypes layout below is include/gwb200.h's."""
import ctypes

import numpy as np
import torch

from . import _exact, _lib, fp_filter

FORM_CODE = {'f16': 0, 'bf16': 1, 'bf16x3': 2, 'f16x2': 6}


class GwbTile(ctypes.Structure):
    _fields_ = [('Vp', ctypes.c_void_p), ('ldvp', ctypes.c_longlong), ('A', ctypes.c_void_p),
                ('lda', ctypes.c_longlong), ('r', ctypes.c_int), ('n', ctypes.c_int), ('row0', ctypes.c_int)]


class GwbStepConfig(ctypes.Structure):
    _fields_ = [('form', ctypes.c_int), ('cw', ctypes.c_int), ('a0', ctypes.c_longlong), ('Tn', ctypes.c_longlong),
                ('snr_threshold', ctypes.c_float), ('margin', ctypes.c_float), ('nbins_max', ctypes.c_int),
                ('cand_cap', ctypes.c_int)]


class CStep:
    """gwb_filter_step for one bank (pipeline.Bank), one transform length and analysed span, one batch size."""

    def __init__(self, bank, tlen, a0, Tn, nseg, cfg, device='cuda'):
        assert cfg.form in FORM_CODE, 'the C step runs the fp16, bf16, split-bf16 and fp16 split-A forms'
        self.bank, self.cfg, self.tlen, self.nseg = bank, cfg, tlen, nseg
        self.vp = [fp_filter.fourstep_order(s['Vh'], tlen) for s in bank.svd]
        self.A = [s['A'].contiguous() for s in bank.svd]
        self.tiles = (GwbTile * len(bank.svd))()
        for t, s in enumerate(bank.svd):
            self.tiles[t] = GwbTile(self.vp[t].data_ptr(), self.vp[t].stride(0), self.A[t].data_ptr(),
                                    self.A[t].stride(0), s['r'], len(bank.tiles[t]), bank.row0[t])
        cw = int(cfg.cluster_window * cfg.sr)
        self.c = GwbStepConfig(FORM_CODE[cfg.form], cw, int(a0), int(Tn), cfg.snr_threshold, cfg.margin,
                               int(cfg.nbins), int(cfg.cand_cap))
        flen = tlen // 2 + 1
        wb = _lib.load().gwb_filter_step_work_bytes(ctypes.addressof(self.tiles), len(bank.svd), bank.M, nseg, tlen,
                                                    flen, bank.kmin, ctypes.addressof(self.c))
        if wb < 0:
            raise _lib.GwbError('gwb_filter_step_work_bytes', _lib.GWB_ERR_SHAPE,
                                _lib.load().gwb_last_error().decode())
        self.work = torch.empty(wb, dtype=torch.uint8, device=device)
        cap = cfg.cand_cap
        self.cands = torch.empty(cap * _exact.CAND.itemsize, dtype=torch.uint8, device=device)
        self.peaks = torch.empty(cap * _exact.PEAK.itemsize, dtype=torch.uint8, device=device)
        self.counters = torch.zeros(5, dtype=torch.int32, device=device)
        self.sig = torch.empty((bank.M, nseg), dtype=torch.float64, device=device)

    def step(self, D, IP, isw):
        b = self.bank
        assert D.shape[0] == self.nseg and IP.shape[0] == self.nseg
        _lib.call('gwb_filter_step', ctypes.addressof(self.tiles), len(b.svd), _lib.ptr(b.H), b.H.stride(0), b.M,
                  _lib.ptr(b.kmax), _lib.ptr(b.nbins), b.kmin, float(b.df), _lib.ptr(D), _lib.ptr(IP),
                  _lib.row_stride(D), _lib.row_stride(IP), self.nseg, _lib.ptr(isw), self.tlen, b.flen, ctypes.addressof(self.c),
                  _lib.ptr(self.work), self.work.numel(), _lib.ptr(self.cands), _lib.ptr(self.peaks),
                  _lib.ptr(self.counters), _lib.ptr(self.sig), _lib.stream_ptr())
        return self.sig

    def results(self):
        c = self.counters.cpu().numpy()
        if c[3]:
            raise _lib.GwbError('filter_step', _lib.GWB_ERR_CAPACITY, 'candidate capacity %d exceeded' % self.cfg.cand_cap)
        n = int(c[0])
        cands = _exact.from_dev(self.cands, _exact.CAND, n)
        peaks = _exact.from_dev(self.peaks, _exact.PEAK, n)
        return dict(n_candidates=n, cands=cands, peaks=peaks, keep=peaks['snr'] > self.cfg.snr_threshold)


class GwbCondConfig(ctypes.Structure):
    _fields_ = [('sr', ctypes.c_double), ('f_low', ctypes.c_double), ('psd_len', ctypes.c_int),
                ('psd_stride', ctypes.c_int), ('median', ctypes.c_int), ('inv_len', ctypes.c_int),
                ('inv_taper', ctypes.c_int)]


class CBatch(CStep):
    """gwb_filter_batch: a batch of raw chunks (nseg x tlen float32 strain) conditioned as
    gpu_prep.BatchConditioner(nseg, tlen, sr, f_low, psd_seg_len, psd_seg_stride, ..., psd_inverse_length) conditions
    them, then filtered as CStep.step, in one C call. D and IP stay on the device (self.D, self.IP)."""

    def __init__(self, bank, tlen, a0, Tn, nseg, cfg, psd_seg_len=16.0, psd_seg_stride=8.0, psd_inverse_length=16.0,
                 median=True, taper=False, device='cuda'):
        super().__init__(bank, tlen, a0, Tn, nseg, cfg, device)
        sr = float(cfg.sr)
        self.cond = GwbCondConfig(sr, float(cfg.f_low), int(psd_seg_len * sr + 0.5), int(psd_seg_stride * sr + 0.5),
                                  int(median), int(psd_inverse_length * sr) if psd_inverse_length else 0, int(taper))
        wb = _lib.load().gwb_filter_batch_work_bytes(ctypes.addressof(self.tiles), len(bank.svd), bank.M, nseg, tlen,
                                                     ctypes.addressof(self.cond), ctypes.addressof(self.c))
        if wb < 0:
            raise _lib.GwbError('gwb_filter_batch_work_bytes', _lib.GWB_ERR_SHAPE,
                                _lib.load().gwb_last_error().decode())
        del self.work
        self.work = torch.empty(wb, dtype=torch.uint8, device=device)
        flen = tlen // 2 + 1
        self.D = torch.empty((nseg, flen), dtype=torch.complex64, device=device)
        self.IP = torch.empty((nseg, flen), dtype=torch.float32, device=device)

    def batch(self, x, isw):
        """x: (nseg, tlen) float32 CUDA strain; isw: 1 / sw of the bank's SVD metric. Returns sig."""
        b = self.bank
        assert tuple(x.shape) == (self.nseg, self.tlen) and x.dtype == torch.float32 and x.stride(1) == 1
        _lib.call('gwb_filter_batch', _lib.handle(), _lib.ptr(x), x.stride(0), self.nseg, self.tlen,
                  ctypes.addressof(self.cond), ctypes.addressof(self.tiles), len(b.svd), _lib.ptr(b.H), b.H.stride(0),
                  b.M, _lib.ptr(b.kmax), _lib.ptr(b.nbins), _lib.ptr(isw), ctypes.addressof(self.c),
                  _lib.ptr(self.work), self.work.numel(), _lib.ptr(self.D), _lib.ptr(self.IP), _lib.ptr(self.cands),
                  _lib.ptr(self.peaks), _lib.ptr(self.counters), _lib.ptr(self.sig), _lib.stream_ptr())
        return self.sig
