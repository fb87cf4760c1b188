"""Mixed precision: the complex64 operator against the FP64 one, and FP64
iterative refinement around complex64 FGMRES reaching FP64 tolerances that
the complex64 operator alone cannot (single and lockstep multi-RHS)."""
import numpy as np
import pytest

from conftest import FREQ, needs_lib, needs_oracle, rel

pytestmark = [pytest.mark.gpu, needs_lib]

_ops = {}


def mixed_op(case_files, name):
    from mlfma_pmchwt_b200 import MLFMM
    if name not in _ops:
        m, p, eps, leaf = case_files[name]
        _ops[name] = MLFMM(m, freq=FREQ, eps_r=eps, leaf_coeff=leaf, device=0, precision="mixed")
    return _ops[name]


@pytest.mark.parametrize("name", ["sphere_s3_lossy", "ellipsoid_s3", "sphere_s4_deep"])
def test_complex64_operator_close_to_fp64(case_files, name):
    from mlfma_pmchwt_b200 import mesh as M
    op = mixed_op(case_files, name)
    for seed in (0, 5):
        x = M.unit_disk_vector(op.n, seed)
        e = rel(op.apply_ax_mixed(x), op.apply_ax(x))
        assert 1e-9 < e < 1e-5, e  # complex64 rounding, not the FP64 operator


@needs_oracle
def test_mixed_plan_keeps_the_fp64_operator(case_files, ref_ops):
    from mlfma_pmchwt_b200 import mesh as M
    op, ref = mixed_op(case_files, "sphere_s3_lossy"), ref_ops("sphere_s3_lossy")
    x = M.unit_disk_vector(op.n, 0)
    assert rel(op.apply_ax(x), ref.apply(x)) < 1e-10


def test_refinement_reaches_fp64_tolerance(case_files):
    from mlfma_pmchwt_b200 import plane_wave
    op = mixed_op(case_files, "sphere_s3_lossy")
    V = op.compute_v_pmchwt(*plane_wave(0.0, 0.0, 0.0))
    x, st = op.solve_mixed(V, itr_max=2000, mr=50, tol_rel=1e-9, tol_abs=0.0, inner_its=8, refine_max=12)
    assert st["converged"] and st["refinements"] >= 2
    assert rel(op.apply_ax(x), V) < 1e-9          # the FP64 residual, recomputed
    assert np.all(np.diff(st["history"]) < 0)     # every refinement step gains
    xf, sf = op.matrix_solver(V, itr_max=2000, mr=50, tol_rel=1e-9, tol_abs=0.0, inner_its=8)
    assert sf["converged"] and rel(x, xf) < 1e-7


def test_lockstep_mixed_solve(case_files):
    from mlfma_pmchwt_b200 import plane_wave
    op = mixed_op(case_files, "sphere_s3_lossy")
    B = np.stack([op.compute_v_pmchwt(*plane_wave(90.0 * (j % 2), 180.0 * j / 4, 0.0)) for j in range(5)])
    X, st = op.solve_mixed_batch(B, itr_max=2000, mr=50, tol_rel=1e-8, tol_abs=0.0, inner_its=8, refine_max=12)
    assert all(s["converged"] for s in st)
    W = op.apply_batch(X)
    for j in range(5):
        assert rel(W[j], B[j]) < 1e-8


def test_fp64_plan_rejects_mixed_calls(case_files):
    from mlfma_pmchwt_b200 import MLFMM, MlfmaError
    m, p, eps, leaf = case_files["sphere_s2"]
    op = MLFMM(m, freq=FREQ, eps_r=eps, leaf_coeff=leaf, device=0)
    with pytest.raises(MlfmaError):
        op.apply_ax_mixed(np.zeros(op.n, dtype=complex))
    with pytest.raises(MlfmaError):
        op.solve_mixed(np.ones(op.n, dtype=complex))


@pytest.mark.parametrize("R", [1, 5, 16])
def test_tensor_core_batched_aggregation(case_files, R):
    """The batched complex64 apply with the leaf aggregation and far-field
    testing on the tensor cores (tcgen05, TF32 high/low split) against the
    same apply on the CUDA cores (agreement at complex64 rounding) and
    against the FP64 operator (the complex64 operator's own error)."""
    import torch
    from mlfma_pmchwt_b200 import mesh as M
    op = mixed_op(case_files, "sphere_s3_lossy")
    ptr, _ = op.leaf_rwgs()
    assert np.diff(ptr).max() <= 64  # so that the tensor-core path is the one taken
    X = torch.from_numpy(np.stack([M.unit_disk_vector(op.n, 60 + j) for j in range(R)])).cuda()
    outs = {}
    for v in (0, 1):
        op.set_tuning("batch_tc.variant", v)
        W = torch.full_like(X, float("nan"))
        torch.cuda.synchronize()
        op.apply_batch_mixed_device(R, X.data_ptr(), W.data_ptr())
        torch.cuda.synchronize()
        outs[v] = W.cpu().numpy()
    op.set_tuning("batch_tc.variant", 0)
    assert op.device_status() == 0
    ref = op.apply_batch(X.cpu().numpy())
    for j in range(R):
        assert rel(outs[1][j], outs[0][j]) < 1e-6, j
        assert rel(outs[1][j], ref[j]) < 1e-5, j


@pytest.mark.parametrize("leaf,tc_path", [(0.45, True), (0.6, False)])
def test_tensor_core_batched_apply_large_leaf_boxes(leaf, tc_path):
    """Leaf boxes of up to 44 RWGs (two 32-RWG tiles in the far-field
    testing, 48-wide contractions in the aggregation) on the tensor cores;
    boxes of more than 64 RWGs take the CUDA-core kernels instead."""
    import torch
    from mlfma_pmchwt_b200 import MLFMM
    from mlfma_pmchwt_b200 import mesh as M
    op = MLFMM(M.icosphere(3, 1.0), freq=FREQ, eps_r=complex(3.0, -0.05), leaf_coeff=leaf, device=0,
               precision="mixed")
    ptr, _ = op.leaf_rwgs()
    assert (np.diff(ptr).max() <= 64) == tc_path and np.diff(ptr).max() > 32
    R = 5
    X = torch.from_numpy(np.stack([M.unit_disk_vector(op.n, 80 + j) for j in range(R)])).cuda()
    outs = {}
    for v in (0, 1):
        op.set_tuning("batch_tc.variant", v)
        W = torch.full_like(X, float("nan"))
        torch.cuda.synchronize()
        op.apply_batch_mixed_device(R, X.data_ptr(), W.data_ptr())
        torch.cuda.synchronize()
        outs[v] = W.cpu().numpy()
    ref = op.apply_batch(X.cpu().numpy())
    for j in range(R):
        # same kernels when the tensor-core path is not taken
        assert rel(outs[1][j], outs[0][j]) < (1e-6 if tc_path else 1e-12), j
        assert rel(outs[1][j], ref[j]) < 1e-5, j
    assert op.device_status() == 0
    op.close()


@pytest.mark.parametrize("name,R", [("sphere_s3_lossy", 16), ("sphere_s4_deep", 7)])
def test_slot_batched_tree_passes(case_files, name, R):
    """The batched complex64 apply with every tree pass launched once per
    level for all slots (batch_tree.variant 1, slot-major arrays) against the
    same apply one slot after another (0): the same arithmetic per slot, so
    the rows agree to complex64 rounding of identical operations."""
    import torch
    from mlfma_pmchwt_b200 import mesh as M
    op = mixed_op(case_files, name)
    X = torch.from_numpy(np.stack([M.unit_disk_vector(op.n, 100 + j) for j in range(R)])).cuda()
    outs = {}
    for v in (0, 1):
        op.set_tuning("batch_tree.variant", v)
        W = torch.full_like(X, float("nan"))
        torch.cuda.synchronize()
        op.apply_batch_mixed_device(R, X.data_ptr(), W.data_ptr())
        torch.cuda.synchronize()
        outs[v] = W.cpu().numpy()
    op.set_tuning("batch_tree.variant", 1)
    assert op.device_status() == 0
    ref = op.apply_batch(X.cpu().numpy())
    for j in range(R):
        assert rel(outs[1][j], outs[0][j]) < 1e-12, j
        assert rel(outs[1][j], ref[j]) < 1e-5, j


