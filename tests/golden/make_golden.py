"""Writes the golden fixtures in this directory by running the reference's own code on seeded inputs.

Run from the repository root in a container where the reference is mounted (it is read, never modified):

    python tests/golden/make_golden.py [--ref /root/reference] [--only NAME ...]

Each fixture holds the inputs and the reference's outputs for one call. The reference functions used:
  fp_gemm_*.npz      pipeline/fp_gemm.py fused_peaks (the Triton kernel under TRITON_INTERPRET=1, on the CPU)
The tests compare the oracle (oracle/) against these files on the CPU, and the CUDA kernels against the oracle and
the files on the GPU. Nothing at test time reads the reference."""
import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _ref_path(ref):
    p = os.path.join(ref, 'pipeline')
    if not os.path.isdir(p):
        raise SystemExit('reference pipeline not found at %s' % p)
    if p not in sys.path:
        sys.path.insert(0, p)
    sys.modules.setdefault('h5py', types.ModuleType('h5py'))   # multi_filter imports h5py at module level
    return p


def gen_fp_gemm():
    os.environ['TRITON_INTERPRET'] = '1'
    import torch
    import fp_gemm
    cases = {
        'fp_gemm_a': dict(M=64, K=64, Tn=1024, cfg=(64, 32, 4, 2), seed=1, kind='normal'),
        'fp_gemm_ragged': dict(M=150, K=128, Tn=1000, cfg=(64, 64, 4, 2), seed=2, kind='normal'),
        'fp_gemm_ties': dict(M=64, K=64, Tn=640, cfg=(64, 64, 4, 2), seed=3, kind='ints'),
    }
    for name, c in cases.items():
        rng = np.random.default_rng(c['seed'])
        if c['kind'] == 'ints':
            # small integers: every product and sum is exact in fp32, so ties are real and the first index must win
            Are = rng.integers(-2, 3, (c['M'], c['K'])).astype(np.float16)
            Aim = rng.integers(-2, 3, (c['M'], c['K'])).astype(np.float16)
            Z = rng.integers(-1, 2, (c['K'], c['Tn'])).astype(np.float16)
        else:
            Are = rng.standard_normal((c['M'], c['K'])).astype(np.float16)
            Aim = rng.standard_normal((c['M'], c['K'])).astype(np.float16)
            Z = rng.standard_normal((c['K'], c['Tn'])).astype(np.float16)
        V, I = fp_gemm.fused_peaks(torch.from_numpy(Are), torch.from_numpy(Aim), torch.from_numpy(Z), c['M'], c['Tn'],
                                   c['cfg'])
        np.savez_compressed(os.path.join(HERE, name + '.npz'), Are=Are, Aim=Aim, Z=Z, V=V.numpy(), I=I.numpy(),
                            M=c['M'], Tn=c['Tn'])
        print(name, V.shape)


GENERATORS = {'fp_gemm': gen_fp_gemm}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default='/root/reference')
    ap.add_argument('--only', nargs='*')
    a = ap.parse_args()
    _ref_path(a.ref)
    for name, fn in GENERATORS.items():
        if a.only and name not in a.only:
            continue
        fn()


if __name__ == '__main__':
    main()
