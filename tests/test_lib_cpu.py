"""CPU checks of the C ABI: the library loads, exports every entry point the header declares, and rejects bad
arguments with a status before any device work."""
import ctypes
import os
import re

import pytest

from conftest import ROOT
from gwb200 import _lib

HEADER = os.path.join(ROOT, 'include', 'gwb200.h')


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r'/\*.*?\*/', '', txt, flags=re.S)
    return sorted(set(re.findall(r'\b(gwb_[a-z0-9_]+)\s*\(', txt)))


def test_library_loads_and_reports_version():
    lib = _lib.load()
    assert lib.gwb_version() == 1
    assert lib.gwb_status_string(0) == b'ok'
    assert lib.gwb_status_string(_lib.GWB_ERR_TIMEOUT).startswith(b'a device wait')


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 5
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_every_declared_symbol_has_a_binding():
    names = set(declared_symbols()) - {'gwb_version', 'gwb_status_string', 'gwb_last_error', 'gwb_num_sms'}
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def _p(v):
    return ctypes.c_void_p(v)


def test_gemm_rejects_k_not_multiple_of_64():
    lib = _lib.load()
    st = lib.gwb_fused_peaks_f16(_p(16), _p(16), 48, _p(16), 1024, 64, 48, 1024, 1, _p(16), _p(16), 8, None)
    assert st == _lib.GWB_ERR_SHAPE
    assert b'multiple of 64' in lib.gwb_last_error()


def test_gemm_rejects_misaligned_operands():
    lib = _lib.load()
    st = lib.gwb_fused_peaks_f16(_p(18), _p(16), 64, _p(16), 1024, 64, 64, 1024, 1, _p(16), _p(16), 8, None)
    assert st == _lib.GWB_ERR_ALIGN
    st = lib.gwb_fused_peaks_f16(_p(16), _p(16), 64, _p(16), 1020, 64, 64, 1020, 1, _p(16), _p(16), 8, None)
    assert st == _lib.GWB_ERR_ALIGN


def test_gemm_rejects_small_output_stride():
    lib = _lib.load()
    st = lib.gwb_fused_peaks_f32(_p(16), _p(16), 64, _p(16), 1024, 64, 64, 1024, 1, _p(16), _p(16), 7, None)
    assert st == _lib.GWB_ERR_SHAPE


def test_window_peaks_rejects_windows_past_the_row():
    lib = _lib.load()
    st = lib.gwb_window_peaks(_p(16), 4096, 2, 100, 2048, 2, _p(16), _p(16), None)
    assert st == _lib.GWB_ERR_SHAPE


def test_call_raises_with_message():
    with pytest.raises(_lib.GwbError, match='multiple of 64'):
        _lib.call('gwb_fused_peaks_f16', _p(16), _p(16), 48, _p(16), 1024, 64, 48, 1024, 1, _p(16), _p(16), 8, None)


def test_segment_chunks_cover_the_analysable_time_once():
    """Batched form: the chunks of segments of any length cover each segment's [start_pad, len - end_pad) exactly
    once (the shifted last chunk's analysed part starts where the previous one ended); shorter segments are skipped."""
    import numpy as np
    from gwb200 import segments
    sr, L, sp, ep = 2048.0, 512.0, 48.0, 16.0
    lens = [512, 700, 1023, 1536, 4096, 300, 3333]
    chunks, skipped = segments.plan_chunks([int(x * sr) for x in lens], sr, [1000000000 + 10000 * i for i in
                                                                              range(len(lens))], L, sp, ep)
    assert skipped == [5]
    for i, n_s in enumerate(lens):
        if n_s < L:
            continue
        cover = np.zeros(int(n_s * sr), np.int8)
        for j, (s0, s1), (a0, a1) in chunks:
            if j == i:
                assert s1 - s0 == int(L * sr) and 0 <= s0 and s1 <= n_s * sr
                cover[s0 + a0:s0 + a1] += 1
        assert cover[int(sp * sr):int((n_s - ep) * sr)].min() == 1 and cover.max() == 1
        assert cover[:int(sp * sr)].max() == 0 and cover[int((n_s - ep) * sr):].max() == 0


def test_order_keys_follow_the_reference_append_order():
    """Consolidation ties go to the earlier peak in the reference's append order (fp_filter.py:700-888: tile, then
    chunk, then the rebuilt peaks before the exact ones, each in template-row then window order); the int64 keys sort
    exactly that way, up to the field limits (16-bit rows and windows, 14-bit chunks)."""
    import numpy as np
    from gwb200 import segments
    rng = np.random.default_rng(2)
    n = 20000
    f = dict(tile=rng.integers(0, 1 << 12, n), chunk=rng.integers(0, 1 << 14, n), exact=rng.integers(0, 2, n),
             row=rng.integers(0, 1 << 16, n), window=rng.integers(0, 1 << 16, n))
    keys = segments.order_keys(f['tile'], f['chunk'], f['exact'], f['row'], f['window'])
    assert len(np.unique(keys)) == np.unique(np.stack(list(f.values())), axis=1).shape[1]
    by_key = np.argsort(keys, kind='stable')
    by_fields = np.lexsort((f['window'], f['row'], f['exact'], f['chunk'], f['tile']))
    assert np.array_equal(keys[by_key], keys[by_fields])
    assert (keys >= 0).all()


def test_autotune_candidates_are_valid_launch_table_entries():
    """Every launch shape the autotuner times (gwb200.autotune.gemm_space) is accepted by gwb_gemm_set_config (a
    host-only table), the split forms include CTA pairs with 64-row K chunks (order 1), and out-of-range entries are
    refused with a status."""
    from gwb200 import autotune
    lib = _lib.load()
    try:
        for form, code in autotune.FORM_CODE.items():
            space = autotune.gemm_space(form)
            assert space and len(set(space)) == len(space)
            for pair, stages, order in space:
                assert lib.gwb_gemm_set_config(code, 128, pair, stages, order) == 0
            if form in ('bf16x3', 'f16x2'):
                assert (1, 0, 1) in space and any(p == 0 for p, _, _ in space)
        assert lib.gwb_gemm_set_config(2, 128, 2, 0, 0) == _lib.GWB_ERR_ARG
        assert lib.gwb_gemm_set_config(2, 128, 1, 9, 0) == _lib.GWB_ERR_ARG
        assert lib.gwb_gemm_set_config(2, 128, 1, 0, 4) == _lib.GWB_ERR_ARG
    finally:
        lib.gwb_gemm_clear_configs()
