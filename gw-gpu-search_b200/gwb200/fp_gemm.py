"""Fused reconstruction GEMM + |z|^2 + max per BN samples: drop-in for pipeline/fp_gemm.py.

z_re = Are @ Z, z_im = Aim @ Z with Z (K x Tn) the stacked real/imag basis series. Per row the kernel keeps only the
max |z|^2 and its sample per BN = 128 samples (fp_gemm.py:14-33), so the M x Tn SNR array never reaches memory.

Forms (all return the same (V, I) layout):
  fp16      fused_peaks(Are, Aim, Z, M, Tn, cfg) with fp16 operands: the reference's own precision, on tcgen05.
  fp32      fused_peaks with float32 operands: the plain fp32 form on the fp32 pipe.
  bf16x3    fused_peaks_split(...): operands split as bf16 hi + lo, three tensor-core products (hi.hi + hi.lo +
            lo.hi), fp32 accumulation; about 16 mantissa bits per operand.
`group` > 1 reduces `group` consecutive blocks per output (the cluster window), fusing fp_filter.py:745-746."""
import time

import torch

from . import _lib

BN = 128

# A cfg is ('umma', stages) (the depth of the kernel's Z ring, 0 = the most that fit; pick_cfg times them; None =
# whatever the launch table holds) or the reference's (BM, BK, warps, stages) Triton tuple, accepted for call
# compatibility (only its BK divisibility rule is checked).
DEFAULT_CFG = ('umma', None)


def _check(Are, Aim, Z, M, Tn):
    _lib.require_cuda(Are, Aim, Z)
    assert Are.shape == Aim.shape and Are.shape[0] >= M and Are.shape[1] == Z.shape[0] and Z.shape[1] >= Tn
    assert Are.stride(1) == 1 and Aim.stride(1) == 1 and Z.stride(1) == 1 and Are.stride(0) == Aim.stride(0)


def _outputs(M, Tn, group, device):
    nblk = -(-Tn // BN)
    nout = -(-nblk // group)
    V = torch.empty((M, nout), device=device, dtype=torch.float32)
    I = torch.empty((M, nout), device=device, dtype=torch.int32)
    return V, I


def fused_peaks(Are, Aim, Z, M, Tn, cfg=DEFAULT_CFG, group=1):
    """Are, Aim (M x K) and Z (K x Tn), fp16 (tensor cores) or float32 (fp32 pipe). Returns max |z|^2 and its sample,
    (M, ceil(ceil(Tn/BN)/group)). For fp16, K must be a multiple of 64 (the reference pads K to 64, fp_filter.py:601)."""
    _check(Are, Aim, Z, M, Tn)
    K = Are.shape[1]
    if isinstance(cfg, tuple) and len(cfg) == 4 and all(isinstance(c, int) for c in cfg):
        assert K % cfg[1] == 0, 'K must be a multiple of BK'
    V, I = _outputs(M, Tn, group, Z.device)
    s = _lib.stream_ptr(Z.device)
    if isinstance(cfg, tuple) and len(cfg) == 2 and cfg[0] == 'umma' and cfg[1] is not None and \
            Z.dtype == torch.float16:
        _lib.call('gwb_gemm_set_config', 4, int(K), 0, int(cfg[1]), 0)   # ('umma', stages): the Z ring depth
    if Z.dtype == torch.float16:
        assert Are.dtype == torch.float16 and Aim.dtype == torch.float16
        _lib.call('gwb_fused_peaks_f16', _lib.ptr(Are), _lib.ptr(Aim), Are.stride(0), _lib.ptr(Z), Z.stride(0), int(M),
                  int(K), int(Tn), int(group), _lib.ptr(V), _lib.ptr(I), V.stride(0), s)
    elif Z.dtype == torch.float32:
        assert Are.dtype == torch.float32 and Aim.dtype == torch.float32
        _lib.call('gwb_fused_peaks_f32', _lib.ptr(Are), _lib.ptr(Aim), Are.stride(0), _lib.ptr(Z), Z.stride(0), int(M),
                  int(K), int(Tn), int(group), _lib.ptr(V), _lib.ptr(I), V.stride(0), s)
    else:
        raise TypeError('fused_peaks takes fp16 or float32 operands (got %s); bf16 uses fused_peaks_split' % Z.dtype)
    return V, I


def fused_peaks_split(Are_hi, Are_lo, Aim_hi, Aim_lo, Z_hi, Z_lo, M, Tn, group=1):
    """Split-bf16 form: each operand as bf16 hi and lo parts; accumulates hi.hi + hi.lo + lo.hi in fp32."""
    _check(Are_hi, Aim_hi, Z_hi, M, Tn)
    for t in (Are_hi, Are_lo, Aim_hi, Aim_lo, Z_hi, Z_lo):
        assert t.dtype == torch.bfloat16
    assert Are_lo.stride(0) == Are_hi.stride(0) and Aim_lo.stride(0) == Are_hi.stride(0)
    assert Z_lo.stride(0) == Z_hi.stride(0)
    K = Are_hi.shape[1]
    V, I = _outputs(M, Tn, group, Z_hi.device)
    _lib.call('gwb_fused_peaks_bf16x3', _lib.ptr(Are_hi), _lib.ptr(Are_lo), _lib.ptr(Aim_hi), _lib.ptr(Aim_lo),
              Are_hi.stride(0), _lib.ptr(Z_hi), _lib.ptr(Z_lo), Z_hi.stride(0), int(M), int(K), int(Tn), int(group),
              _lib.ptr(V), _lib.ptr(I), V.stride(0), _lib.stream_ptr(Z_hi.device))
    return V, I


def pick_cfg(dev='cuda', M=1024, K=128, Tn=1 << 20):
    """Times the stacked fp16 kernel's launch configurations (the depth of its Z ring: the most that fit, 4, 3, 2) on
    the shape and keeps the fastest in the library's launch table (gwb_gemm_set_config, form 4, kh = K); returns
    (fastest cfg, {cfg: seconds or error text}). Same contract as the reference's autotuner (fp_gemm.py:47-64):
    raises if nothing runs. cfg = ('umma', stages)."""
    Ar = torch.randn((M, K), device=dev).half()
    Ai = torch.randn((M, K), device=dev).half()
    Zs = torch.randn((K, Tn), device=dev).half()
    res, best = {}, None
    for c in [('umma', 0), ('umma', 4), ('umma', 3), ('umma', 2)]:
        try:
            fused_peaks(Ar, Ai, Zs, M, Tn, c)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(3):
                fused_peaks(Ar, Ai, Zs, M, Tn, c)
            torch.cuda.synchronize()
            res[str(c)] = (time.perf_counter() - t0) / 3
        except Exception as ex:  # noqa: BLE001 - reported in the results, as the reference does
            res[str(c)] = repr(ex)[:300]
            continue
        if best is None or res[str(c)] < res[str(best)]:
            best = c
    if best is None:
        raise RuntimeError('no GEMM config ran: %r' % res)
    _lib.call('gwb_gemm_set_config', 4, int(K), 0, int(best[1]), 0)
    return best, res
