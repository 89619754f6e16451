"""The reference's own GPU scan kernel (bntm_compute_products,
scorer-bntm/src/gpu/kernels.cu:100-178, built from the reference source for
sm_100a into oracle/_ref) agrees with the oracle and with the product's scan,
so that the bench times it on equal terms.  Measurement infrastructure: the
product never loads it."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import ref_gpu
from bnutil import N, P, uniform_fp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m", [1, 255, 4099])
def test_reference_kernel_matches_oracle_and_product(ctx, m):
    torch = pytest.importorskip("torch")
    from bn_b200 import capi

    lib = ref_gpu.load()
    if lib is None:
        pytest.skip("oracle/_ref/libbnref_gpu.so was not built (no reference checkout at build time)")
    m_enc = uniform_fp((m, N), 31 + m)
    m_enc[0, :5] = P - 1  # extreme residues
    v = uniform_fp(N, 77)
    v[:3] = P - 1
    want = O.matvec(m_enc, m, N, v)
    dev = torch.device("cuda:0")
    d_m = torch.from_numpy(m_enc.reshape(-1).view(np.int64).copy()).to(dev)
    d_v = torch.from_numpy(v.view(np.int64).copy()).to(dev)
    d_r = torch.zeros(m, dtype=torch.int64, device=dev)
    assert lib.bnref_compute_products(d_m.data_ptr(), d_v.data_ptr(), d_r.data_ptr(), m,
                                      torch.cuda.current_stream(dev).cuda_stream) == 0
    torch.cuda.synchronize(dev)
    got = d_r.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, want)
    f = capi.Flat.build(ctx, m_enc, np.zeros(m * 128, np.uint64), np.zeros(m * 128, np.uint64), m)
    assert np.array_equal(f.compute_products(v), got)
    f.close()
