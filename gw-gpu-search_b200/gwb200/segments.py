"""Batched filtering of many science segments of different lengths (the batched form): the library's replacement of
the reference's per-dataset loop over segments (fp_filter.py:700-888 driven once per dataset, with gpu_prep stage 1
and stage 2 per dataset, gpu_prep.py:362-454).

Each segment is autogated over its whole length (detect_loud_glitches + gate_taper, gpu_prep.py:175-231), then cut
into chunks of seg_len seconds by the reference's StrainSegments arithmetic (segment_slices, gpu_prep.py:234-271:
chunks at a fixed stride, the last one shifted back to end at the segment's end, its analysed part starting where the
previous chunk's ended). Segments shorter than seg_len hold no chunk, as in the reference, and are reported as
skipped. Chunks go through the device in batches of `batch`: one conditioning (BatchConditioner) and one filter step
(MatchedFilter) per batch, captured once as a CUDA graph and replayed for every batch. Candidates outside a chunk's
analysed part are dropped when the results are mapped back to segments.

With a Consolidation, each segment is one dataset of the reference: its exact and rebuilt peaks (FilterConfig.
exact_snr) go to a PeakStore after every batch and are consolidated on the device (consolidate.py), with order keys
that give the reference's append order (tile, chunk, rebuilt before exact, template row, window; fp_filter.py:
700-888), and the run returns each segment's peak table (write_one's datasets).
"""
from dataclasses import dataclass

import numpy as np
import torch

from . import _exact, _lib, consolidate as cons_, gpu_prep, pipeline


@dataclass
class Gating:
    threshold: float = 8.0      # whitened |x| (the reference's argv uses 50, for glitches far louder than SNR 200)
    cluster: float = 0.5
    width: float = 0.25
    taper: float = 0.25
    pad: float = 16.0
    f_low: float = 15.0
    max_iterations: int = 1


@dataclass
class Consolidation:
    """The reference's consolidation options (pycbc_inspiral's --newsnr-threshold, --keep-loudest-interval,
    --keep-loudest-num, and fp_filter's --consolidate-exempt-snr); production uses 4, 1.072, 30 and 5."""
    newsnr_threshold: float = 4.0
    keep_loudest_interval: float = 1.072
    keep_loudest_num: int = 30
    exempt_snr: float = 5.0


def order_keys(tile, chunk, exact, row_in_tile, window):
    """int64 keys of the reference's append order within one dataset: tile, chunk, rebuilt before exact, template
    row within the tile, window."""
    return ((np.asarray(tile, np.int64) << 47) | (np.asarray(chunk, np.int64) << 33) |
            (np.asarray(exact, np.int64) << 32) | (np.asarray(row_in_tile, np.int64) << 16) |
            np.asarray(window, np.int64))


def plan_chunks(lengths, sr, start_gps, seg_len, start_pad, end_pad):
    """Chunks of segments of the given lengths (samples): list of (segment index, (s0, s1) samples, (a0, a1) analysed
    samples relative to s0), by segment_slices; and the indices of the segments shorter than seg_len (skipped)."""
    tlen = int(seg_len * sr)
    chunks, skipped = [], []
    for i, n in enumerate(lengths):
        if n < tlen:
            skipped.append(i)
            continue
        for sl, an in gpu_prep.segment_slices(int(n), sr, start_gps[i], seg_len, start_pad, end_pad, None, None):
            chunks.append((i, sl, an))
    return chunks, skipped


class SegmentFilter:
    """Filters lists of segments against one bank. segments: list of dict(x = float32 CUDA strain in DYN_RANGE_FAC
    units, start_gps, det). The bank's templates must have been generated for chunks of seg_len seconds."""

    def __init__(self, bank, cfg, seg_len=512.0, start_pad=48.0, end_pad=16.0, batch=32, gating=Gating(),
                 psd=(16.0, 8.0, 63, 16.0), isw=None, graph=True, consolidation=None, device='cuda'):
        self.bank, self.cfg, self.gating = bank, cfg, gating
        self.consolidation = consolidation
        self.sr = cfg.sr
        self.seg_len, self.start_pad, self.end_pad = seg_len, start_pad, end_pad
        self.tlen = int(seg_len * self.sr)
        assert self.tlen // 2 + 1 == bank.flen, 'the bank was generated for another chunk length'
        self.batch = batch
        self.device = device
        seg_l, seg_s, nseg, inv_len = psd
        self.cond = gpu_prep.BatchConditioner(batch, self.tlen, self.sr, cfg.f_low, seg_l, seg_s, nseg, inv_len,
                                              device=device)
        a0, a1 = int(start_pad * self.sr), int((seg_len - end_pad) * self.sr)
        self.mf = pipeline.MatchedFilter(bank, self.tlen, a0, a1 - a0, cfg, device=device)
        self.X = torch.zeros((batch, self.tlen), dtype=torch.float32, device=device)
        self.isw = isw
        self.use_graph = graph
        self.graph = None
        self.sig = None
        self.row0 = np.asarray(bank.row0, np.int64)
        self.row0_d = torch.from_numpy(self.row0).to(device)
        self.order_d = torch.from_numpy(np.asarray(bank.order, np.int64)).to(device)

    def gate(self, x, start_gps):
        """Autogating of one segment in place (gpu_prep.gpu_stage1's loop); returns the gates (gps, width, taper)."""
        g = self.gating
        gates = []
        for _ in range(g.max_iterations):
            gt = gpu_prep.detect_loud_glitches(torch, x, self.sr, start_gps, g.threshold, g.cluster, g.f_low, g.pad)
            gp = [(t, g.width, g.taper) for t in gt]
            gates += gp
            gpu_prep.gate_taper(torch, x, self.sr, start_gps, gp)
            if not gt:
                break
        return [(float(t), w, tp) for t, w, tp in gates]

    def gate_all(self, segments, cap=1 << 16):
        """gate() for every segment with one host synchronisation per gating iteration for all of them: the whitening
        and thresholding of every segment are queued first, then the counts are read once and the clustering (host,
        as the reference's) and the gates follow. Same gates as gate() per segment."""
        g = self.gating
        gates = [[] for _ in segments]
        todo = list(range(len(segments)))
        for _ in range(g.max_iterations):
            if not todo:
                break
            queued = [gpu_prep.whitened_above_queue(segments[i]['x'], self.sr, g.threshold, g.f_low, g.pad, cap=cap)
                      for i in todo]
            nxt = []
            for i, q in zip(todo, queued):
                ind, v, _ = gpu_prep.above_collect(*q)
                gt = gpu_prep.glitch_times(ind, v, self.sr, segments[i]['start_gps'], g.cluster)
                gp = [(t, g.width, g.taper) for t in gt]
                gates[i] += gp
                gpu_prep.gate_taper(torch, segments[i]['x'], self.sr, segments[i]['start_gps'], gp)
                if gt:
                    nxt.append(i)
            todo = nxt
        return [[(float(t), w, tp) for t, w, tp in gs] for gs in gates]

    def prepare(self, segments, arena_cap=1 << 23):
        """Captures the whole run over these segments as one CUDA graph: for every batch of chunks the copies of the
        chunks into the batch buffer, the conditioning and filter step, and the append of the batch's exact-stage
        results to a run-wide list on the device (gwb_append_results). The graph reads the segments' strain where it
        is, so gating them in place afterwards (run_graph) changes nothing in it. Returns the capture's seconds."""
        import time
        t0 = time.perf_counter()
        chunks, skipped = self.plan(segments)
        nb = -(-len(chunks) // self.batch)
        dev = self.device
        mf = self.mf
        cap = mf.slot_cap
        self.arena = dict(cands=torch.empty(arena_cap * 32, dtype=torch.uint8, device=dev),
                          peaks=torch.empty(arena_cap * 32, dtype=torch.uint8, device=dev),
                          tag=torch.empty(arena_cap, dtype=torch.int32, device=dev),
                          count=torch.zeros(1, dtype=torch.int32, device=dev),
                          work=torch.zeros(2, dtype=torch.int32, device=dev),
                          meta=torch.zeros((max(nb, 1), 8), dtype=torch.int32, device=dev), cap=arena_cap)
        A = self.arena
        # warm-up on the first batch's chunks: plans, workspaces and cached tables outside the capture
        for r in range(self.batch):
            i, (s0, s1), _ = chunks[min(r, len(chunks) - 1)]
            self.X[r].copy_(segments[i]['x'][s0:s1])
        self._step()
        torch.cuda.synchronize()
        self.run_graph_ = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.run_graph_):
            for b in range(nb):
                part = chunks[b * self.batch:(b + 1) * self.batch]
                for r in range(self.batch):
                    i, (s0, s1), _ = part[min(r, len(part) - 1)]   # unused rows repeat a real chunk (dropped later)
                    self.X[r].copy_(segments[i]['x'][s0:s1])
                self._step()
                _lib.call('gwb_append_results', _lib.ptr(mf.cands), _lib.ptr(mf.peaks), _lib.ptr(mf.counters), cap,
                          b, _lib.ptr(A['cands']), _lib.ptr(A['peaks']), _lib.ptr(A['tag']), _lib.ptr(A['count']),
                          arena_cap, _lib.ptr(A['work']), _lib.ptr(A['meta']), _lib.stream_ptr())
        torch.cuda.synchronize()
        self.prepared = dict(chunks=chunks, skipped=skipped, nb=nb, segments=segments)
        return time.perf_counter() - t0

    def run_graph(self, gate=True):
        """The prepared run: gating of every segment (gate_all), one replay of the run's graph, one copy of the
        run-wide result list to the host. Returns run()'s dict (without consolidation)."""
        P = self.prepared
        segments, chunks = P['segments'], P['chunks']
        gates = self.gate_all(segments) if gate else [[] for _ in segments]
        A = self.arena
        A['count'].zero_()
        self.run_graph_.replay()
        torch.cuda.synchronize()
        meta = A['meta'].cpu().numpy()
        if np.any(meta[:P['nb'], 3]) or np.any(meta[:P['nb'], 7]):
            raise _lib.GwbError('run_graph', _lib.GWB_ERR_CAPACITY, 'a candidate list or the run list overflowed')
        n = int(A['count'].item())
        c = _exact.from_dev(A['cands'], _exact.CAND, n)
        p = _exact.from_dev(A['peaks'], _exact.PEAK, n)
        tag = A['tag'][:n].cpu().numpy().astype(np.int64)
        row = tag * self.batch + c['seg'].astype(np.int64)       # the chunk of each candidate
        ok = (c['seg'] < self.batch) & (row < len(chunks))
        rowc = np.minimum(row, len(chunks) - 1)
        a_lo = np.array([an[0] for _, _, an in chunks])[rowc]
        a_hi = np.array([an[1] for _, _, an in chunks])[rowc]
        ok &= (c['sample'] >= a_lo) & (c['sample'] < a_hi)
        c, p, rowc = c[ok], p[ok], rowc[ok]
        keep = p['snr'] > self.cfg.snr_threshold
        analysed = sum(an[1] - an[0] for _, _, an in chunks) / self.sr
        skipped_s = sum(segments[i]['x'].shape[0] for i in P['skipped']) / self.sr
        return dict(cands=c, peaks=p, keep=keep, segment=np.array([chunks[r][0] for r in rowc], np.int64),
                    chunk=rowc, gates=gates, analysed_s=analysed, skipped_s=skipped_s, skipped=P['skipped'],
                    n_chunks=len(chunks), batches=P['nb'], plan=chunks, graph_launches=1)

    def plan(self, segments):
        """Chunks of every segment: list of (segment index, (s0, s1) samples, (a0, a1) analysed samples in the chunk),
        and the skipped segments (shorter than seg_len)."""
        return plan_chunks([s['x'].shape[0] for s in segments], self.sr, [s['start_gps'] for s in segments],
                           self.seg_len, self.start_pad, self.end_pad)

    def _step(self):
        D, IP = self.cond(self.X)
        self.sig = self.mf.step(D, IP, self.isw)

    def _capture(self):
        self._step()                           # warm-up: plans, workspaces and cached tables outside the capture
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._step()
        torch.cuda.synchronize()

    def _peaks(self, res, part, pos):
        """This batch's output peaks per segment, as device tensors in the PeakStore layout: the exact ones above the
        threshold (fp_filter.py:837-853) and the rebuilt ones (fp_filter.py:772-781, left on the device), inside
        each chunk's analysed part; pos[r] = the chunk's index within its segment."""
        dev = self.device
        i64 = dict(dtype=torch.int64, device=dev)
        nb = len(part)
        a_lo = torch.tensor([an[0] for _, _, an in part], **i64)
        a_hi = torch.tensor([an[1] for _, _, an in part], **i64)
        s0 = torch.tensor([sl[0] for _, sl, _ in part], **i64)
        posd = torch.tensor(pos, **i64)
        segof = torch.tensor([i for i, _, _ in part], **i64)
        thr = np.float32(self.cfg.snr_threshold)
        c, p = res['cands'], res['peaks']
        sel = p['snr'] > thr
        c, p = c[sel], p[sel]
        h = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
        ex = dict(row=h(c['row']), seg=h(c['seg']), sample=h(c['sample']), window=h(c['window']), snr=h(p['snr']),
                  zr=h(p['zr']), zi=h(p['zi']), chisq=h(p['chisq']), dof=h(p['dof']))
        R = res['rebuilt_dev']
        f32 = R.view(torch.float32)
        zf = torch.zeros(R.shape[0], dtype=torch.float32, device=dev)
        rb = dict(row=R[:, 0], seg=R[:, 1], sample=R[:, 2], window=R[:, 3], snr=f32[:, 4], zr=f32[:, 5], zi=f32[:, 6],
                  chisq=zf, dof=zf.view(torch.int32))
        parts = []
        for exact, d in ((0, rb), (1, ex)):
            r = d['seg'].long()
            samp = d['sample'].long()
            rr = r.clamp(max=nb - 1)
            ok = (r < nb) & (samp >= a_lo[rr]) & (samp < a_hi[rr])
            row, rr, samp = d['row'].long()[ok], rr[ok], samp[ok]
            tile = torch.searchsorted(self.row0_d, row, right=True) - 1
            key = ((tile << 47) | (posd[rr] << 33) | (exact << 32) | ((row - self.row0_d[tile]) << 16) |
                   d['window'].long()[ok])
            parts.append((segof[rr], dict(
                tid=self.order_d[row], ti=s0[rr] + samp, snr=d['snr'][ok].contiguous(),
                phase=torch.atan2(d['zi'][ok], d['zr'][ok]), peak_sigmasq=self.sig[row, rr],
                exact=torch.full((int(row.numel()),), bool(exact), dtype=torch.bool, device=dev),
                chisq=d['chisq'][ok].contiguous(), dof=d['dof'][ok].contiguous(), order=key)))
        out = {}
        for i in sorted({i for i, _, _ in part}):
            out[i] = {f: torch.cat([d[f][si == i] for si, d in parts]) for f in cons_.FIELDS}
        return out

    def run(self, segments, gate=True, keep_raw=False):
        """Gates, plans and filters every segment. Returns dict(cands, peaks, keep (the kept peaks after the exact
        stage), segment and chunk index of each candidate, gates per segment, analysed_s, skipped_s, batches); with a
        Consolidation also tables (segment -> write_one's datasets) and n_peaks_in / n_peaks_out, and with keep_raw
        the unconsolidated peaks per segment (raw)."""
        gates = [self.gate(s['x'], s['start_gps']) if gate else [] for s in segments]
        chunks, skipped = self.plan(segments)
        if self.isw is None:
            # the SVD metric of the run (fp_filter.py:354-370) from the first batch, as the bank was built
            raise ValueError('isw (the bank\'s 1 / sw) must be given')
        co = self.consolidation
        stores, sigmasq, raw = {}, {}, {}
        n_chunks_of = {}
        pos_of = []
        for i, _, _ in chunks:
            pos_of.append(n_chunks_of.get(i, 0))
            n_chunks_of[i] = pos_of[-1] + 1
        out_c, out_p, seg_i, chunk_i = [], [], [], []
        analysed = 0.0
        for b0 in range(0, len(chunks), self.batch):
            part = chunks[b0:b0 + self.batch]
            for r in range(self.batch):
                i, (s0, s1), _ = part[min(r, len(part) - 1)]     # unused rows repeat a real chunk (dropped below)
                self.X[r].copy_(segments[i]['x'][s0:s1])
            if self.use_graph:
                if self.graph is None:
                    self._capture()
                self.graph.replay()
            else:
                self._step()
            torch.cuda.synchronize()
            res = self.mf.results(rebuilt_on_device=co is not None)
            c, p = res['cands'], res['peaks']
            row = c['seg'].astype(np.int64)
            ok = row < len(part)
            a_lo = np.array([an[0] for _, _, an in part] + [0] * (self.batch - len(part)))
            a_hi = np.array([an[1] for _, _, an in part] + [0] * (self.batch - len(part)))
            ok &= (c['sample'] >= a_lo[row]) & (c['sample'] < a_hi[row])
            out_c.append(c[ok])
            out_p.append(p[ok])
            seg_i.append(np.array([part[r][0] for r in row[ok]], np.int64))
            chunk_i.append(b0 + row[ok])
            analysed += sum((an[1] - an[0]) for _, _, an in part) / self.sr
            if co is not None:
                sig = None
                for i, d in self._peaks(res, part, pos_of[b0:b0 + len(part)]).items():
                    if keep_raw:
                        raw.setdefault(i, []).append({f: v.cpu().numpy() for f, v in d.items()})
                    st = stores.get(i)
                    if st is None:
                        st = stores[i] = cons_.PeakStore(
                            segments[i]['start_gps'], self.sr, segments[i]['x'].shape[0], gates[i],
                            co.newsnr_threshold, co.keep_loudest_interval, co.keep_loudest_num, co.exempt_snr,
                            device=self.device)
                    st.add(**d)
                if sig is None:
                    sig = self.sig.cpu().numpy()
                for r, (i, _, _) in enumerate(part):      # template norms of every chunk (the files' sigmasq)
                    sq = sigmasq.setdefault(i, np.zeros((self.bank.M, n_chunks_of[i])))
                    sq[self.bank.order, pos_of[b0 + r]] = sig[:, r]
        cands = np.concatenate(out_c) if out_c else np.zeros(0)
        peaks = np.concatenate(out_p) if out_p else np.zeros(0)
        keep = peaks['snr'] > self.cfg.snr_threshold if len(peaks) else np.zeros(0, bool)
        skipped_s = sum(segments[i]['x'].shape[0] for i in skipped) / self.sr
        out = dict(cands=cands, peaks=peaks, keep=keep, segment=np.concatenate(seg_i) if seg_i else np.zeros(0),
                   chunk=np.concatenate(chunk_i) if chunk_i else np.zeros(0), gates=gates, analysed_s=analysed,
                   skipped_s=skipped_s, skipped=skipped, n_chunks=len(chunks), batches=-(-len(chunks) // self.batch),
                   plan=chunks)
        if co is not None:
            out['tables'] = {i: cons_.peak_table(st.host(), gates[i], segments[i]['start_gps'], self.sr,
                                                 sigmasq=sigmasq.get(i)) for i, st in stores.items()}
            out['n_peaks_in'] = sum(st.n_in for st in stores.values())
            out['n_peaks_out'] = sum(len(t['snr']) for t in out['tables'].values())
            if keep_raw:
                out['raw'] = {i: {f: np.concatenate([d[f] for d in ds]) for f in cons_.FIELDS}
                              for i, ds in raw.items()}
        return out


def filter_segments(segments, bank, cfg, isw, **kw):
    """Batched filter of a list of segments (see SegmentFilter)."""
    return SegmentFilter(bank, cfg, isw=isw, **kw).run(segments)
