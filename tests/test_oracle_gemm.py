"""The GEMM / window oracle against the reference's own Triton kernel outputs (tests/golden/fp_gemm_*.npz)."""
import numpy as np
import pytest

from oracle import gemm


@pytest.mark.parametrize('name', ['fp_gemm_a', 'fp_gemm_ragged', 'fp_gemm_ties'])
def test_oracle_matches_reference_gemm(golden, name):
    g = golden(name)
    V, I = gemm.gemm_absmax(g['Are'], g['Aim'], g['Z'], int(g['M']), int(g['Tn']))
    np.testing.assert_allclose(V, g['V'], rtol=2e-6, atol=1e-6)
    if name == 'fp_gemm_ties':
        # exact integer arithmetic: values and first-index ties are bit-exact
        assert np.array_equal(V, g['V'])
        assert np.array_equal(I, g['I'])
    else:
        assert (I == g['I']).mean() == 1.0


def test_group_reduce_keeps_first_block_on_ties():
    V = np.array([[1., 3., 3., 2.]], np.float32)
    I = np.array([[5, 130, 260, 400]], np.int32)
    v, i = gemm.group_reduce(V, I, 4)
    assert v[0, 0] == 3 and i[0, 0] == 130


def test_window_peaks_first_offset_on_ties():
    z = np.zeros((1, 8), np.complex64)
    z[0, [2, 5]] = 1 + 1j
    p, i = gemm.window_peaks(z, 0, 8, 1)
    assert i[0, 0] == 2 and p[0, 0] == 2.0
