"""GPU test of the distributed four-step's local steps on this library's kernels (one rank: the
exchange is the identity; the multi-rank exchange is covered with gloo in test_multigpu_gloo.py).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_dist_fft_single_rank_on_gpu(ofb, oracle):
    import torch

    from onefft_b200.distributed import dist_fft
    n1, n2 = 2048, 4096
    n = n1 * n2
    x = oracle.gen_normal(2 * n, 0xD15).view(np.complex64)
    cols = torch.from_numpy(x.reshape(n1, n2).copy()).cuda()
    out = dist_fft(cols, n1, n2).cpu().numpy()  # (n1, n2): [k1][k2] = X[k1 + n1 k2]
    got = np.ascontiguousarray(out.T).reshape(-1)  # natural order X[k1 + n1 k2]
    want = oracle.fft64_numpy(x.view(np.float32))
    err = oracle.rel_rms(got.view(np.float32), want)
    print(f"distributed four-step on one rank, n=2^23: rel RMS {err:.3g}")
    assert err < oracle.tolerance(23)
