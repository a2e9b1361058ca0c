"""CPU checks of bench.py's contract pieces: the metric string is BASELINE.json's, every ncu summary the bench line
cites exists and carries its traffic ratio, and the synthetic C2 bank has the configured size and mass ranges."""
import json
import os

import numpy as np

from conftest import ROOT


def _bench():
    import bench
    return bench


def test_metric_and_unit_match_the_baseline_file():
    b = _bench()
    base = json.load(open(os.path.join(ROOT, 'BASELINE.json')))
    assert b.METRIC == base['metric']
    assert b.UNIT == '2-det weeks / hour'


def test_cited_profiles_exist_with_traffic_ratios():
    b = _bench()
    for form in ('bf16x3', 'f16', 'bf16', 'f16x2', 'fp8', 'f32'):
        ratios, sources = b.traffic_ratios(form)
        assert 'basis' in ratios, form
        for key, src in sources.items():
            path = os.path.join(ROOT, src)
            assert os.path.exists(path), src
            txt = open(path).read()
            assert 'Command' in txt and '--clock-control none' in txt, src
            assert 0.9 < ratios[key] < 1.2, (form, key, ratios[key])
    assert set(b.traffic_ratios('bf16x3')[0]) == {'basis', 'gemm'}


def test_synthetic_c2_bank_has_the_configured_templates():
    b = _bench()
    bank = b.make_bank()
    m1, m2 = np.asarray(bank['mass1']), np.asarray(bank['mass2'])
    assert len(m1) == b.N_TEMPLATES == 5880
    assert np.all(m1 > 0) and np.all(m2 > 0)
    assert np.all(np.maximum(m1, m2) <= 100.0 + 1e-9) and np.all(np.minimum(m1, m2) >= 3.0 - 1e-9)
