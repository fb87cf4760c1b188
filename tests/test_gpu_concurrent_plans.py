"""Plans built and used from several host threads at once (one plan per
thread, the documented use of the C ABI) must give the operator a plan
built alone gives, bit for bit.

Setup copies the plan's tables to the device on the plan's own stream: a
blocking copy from pageable memory may return before its DMA lands and is
not ordered with the plan's non-blocking streams, so under load a setup
kernel could read a table before it arrived (the leaf patterns of a medium
came out different in about one run in three with six threads)."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from conftest import needs_lib

pytestmark = [pytest.mark.gpu, needs_lib]

FREQ = 3e8


def _bodies():
    from mlfma_pmchwt_b200 import mesh as M
    bodies = M.uneven_bodies(1, FREQ)
    # the 3,840- and 15,360-unknown bodies: setup kernels of one overlap
    # applies and setups of the others
    return [b for b in bodies if len(b["mesh"].face_ids) <= 5120][:8]


def _operator_rows(b, X):
    import torch
    from mlfma_pmchwt_b200 import MLFMM
    torch.cuda.set_device(0)
    op = MLFMM(b["mesh"], freq=FREQ, eps_r=b["eps_r"], leaf_coeff=0.25, device=0, precision="mixed",
               tf_complex_argument=True)
    try:
        x = X[: op.n]
        w64 = op.apply_ax(x)
        Xd = torch.from_numpy(np.stack([x, 1j * x, x[::-1].copy()])).cuda()
        Wd = torch.empty_like(Xd)
        stream = torch.cuda.Stream()
        op.apply_batch_mixed_device(3, Xd.data_ptr(), Wd.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        return w64, Wd.cpu().numpy()
    finally:
        op.close()


def test_plans_from_several_threads_match_a_plan_alone():
    from mlfma_pmchwt_b200 import mesh as M
    bodies = _bodies()
    X = M.unit_disk_vector(4 * 15360, 3)
    alone = [_operator_rows(b, X) for b in bodies]
    for _ in range(3):
        with ThreadPoolExecutor(max_workers=6) as pool:
            together = list(pool.map(lambda b: _operator_rows(b, X), bodies))
        for i, (a, t) in enumerate(zip(alone, together)):
            assert np.array_equal(a[0], t[0]), f"body {i}: FP64 apply differs"
            assert np.array_equal(a[1], t[1]), f"body {i}: batched complex64 apply differs"
