"""The far-field entry point that allocates no device memory
(mlfma_rcs_pmchwt_noalloc), for callers that cannot allocate while they run
(memory reserved up front in their own pool, real-time loops). It must give
the same field as the allocating entry point mlfma_rcs_pmchwt, on two calls
in a row with different angle sets (the shared angle scratch keeps the last
call's contents), and refuse counts above its fixed scratch size.

This file is collected last so that, if it fails, a run stopping at the first
failure has already run every other test."""
import numpy as np
import pytest

from conftest import FREQ, needs_lib

pytestmark = [pytest.mark.gpu, needs_lib]


def _field_noalloc(op, I, th, ph):
    import torch
    Id = torch.from_numpy(np.ascontiguousarray(I)).cuda()
    out = torch.empty((len(th), 3), dtype=torch.complex128, device="cuda")  # every element is written
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())  # the copy of I_dev comes first
    op.calculate_rcs_noalloc(Id.data_ptr(), th, ph, out.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    return out.cpu().numpy()


def test_noalloc_far_field_matches_allocating_entry_point():
    from mlfma_pmchwt_b200 import MLFMM
    from mlfma_pmchwt_b200 import mesh as M
    op = MLFMM(M.icosphere(3, 1.0), freq=FREQ, eps_r=4.0, leaf_coeff=0.25, device=0)
    I = M.unit_disk_vector(op.n, 4)
    # a first call with no angles does the per-device set-up and leaves the current device alone
    import torch
    dev = torch.cuda.current_device()
    Id = torch.from_numpy(I).cuda()
    out = torch.empty((1, 3), dtype=torch.complex128, device="cuda")
    op.calculate_rcs_noalloc(Id.data_ptr(), np.zeros(0), np.zeros(0), out.data_ptr())
    torch.cuda.synchronize()
    assert torch.cuda.current_device() == dev
    # first call: the 361-angle bistatic cut in phi = 0
    th1 = np.arange(0.0, 180.01, 0.5)
    f_ref1, _ = op.calculate_rcs_pmchwt(I, th1, 0.0)
    f1 = _field_noalloc(op, I, th1, np.zeros_like(th1))
    np.testing.assert_allclose(f1, f_ref1, rtol=1e-12, atol=1e-12 * np.abs(f_ref1).max())
    # second call: fewer angles in another cut; the scratch still holds the first table's tail
    th2 = np.linspace(10.0, 170.0, 37)
    ph2 = np.full_like(th2, 45.0)
    f_ref2, _ = op.calculate_rcs_pmchwt(I, th2, ph2)
    f2 = _field_noalloc(op, I, th2, ph2)
    np.testing.assert_allclose(f2, f_ref2, rtol=1e-12, atol=1e-12 * np.abs(f_ref2).max())
    op.close()


def test_noalloc_far_field_rejects_counts_above_the_scratch():
    import torch
    from mlfma_pmchwt_b200 import MLFMM, MlfmaError
    from mlfma_pmchwt_b200 import mesh as M
    op = MLFMM(M.icosphere(2, 0.5), freq=FREQ, eps_r=4.0, leaf_coeff=0.25, device=0)
    cap = op._lib.mlfma_rcs_noalloc_max_angles()
    assert cap == 8192
    Id = torch.zeros(op.n, dtype=torch.complex128, device="cuda")
    out = torch.zeros((cap + 1, 3), dtype=torch.complex128, device="cuda")
    th = np.zeros(cap + 1)
    with pytest.raises(MlfmaError) as e:
        op.calculate_rcs_noalloc(Id.data_ptr(), th, th, out.data_ptr())
    assert e.value.code == -1 and "8192" in str(e.value)
    op.close()
