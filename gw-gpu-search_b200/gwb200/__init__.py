"""gwb200: B200-native (sm_100a) matched-filter hot path of gw-gpu-search behind the reference's own call signatures.

Modules mirror the reference's pipeline modules for this path: gpu_prep (PSD, whitening, gating), fp_gemm (fused
reconstruction GEMM + |z|^2 + argmax), fp_filter (SVD tile compression, basis series, stacked A, window selection),
peak_kernel (per-window peaks), chisq_edges / multi_filter (chi-squared bin edges), chisq_kernel (power chi-squared)
and exact_stage (exact SNR at the loudest peaks). All compute runs in libgwb200.so (hand-written CUDA for sm_100a plus
cuFFT); torch provides device memory and streams."""
from . import _lib  # noqa: F401

__version__ = '0.1.0'
