"""Batched apply (several right-hand sides per pass over the leaf tables):
every right-hand side of a batch gets the single apply's result, for batch
sizes that leave partial register groups (8 in the aggregation, 4 in the
leaf testing) and cross the 16-slot group boundary."""
import numpy as np
import pytest

from conftest import FREQ, needs_lib, rel

pytestmark = [pytest.mark.gpu, needs_lib]

_ops = {}


def gpu_op(case_files, name):
    from mlfma_pmchwt_b200 import MLFMM
    if name not in _ops:
        m, p, eps, leaf = case_files[name]
        _ops[name] = MLFMM(m, freq=FREQ, eps_r=eps, leaf_coeff=leaf, device=0)
    return _ops[name]


@pytest.mark.parametrize("name", ["sphere_s3_lossy", "sphere_s4_deep"])
@pytest.mark.parametrize("R", [1, 5, 19])
def test_batch_rows_equal_single_applies(case_files, name, R):
    from mlfma_pmchwt_b200 import mesh as M
    op = gpu_op(case_files, name)
    X = np.stack([M.unit_disk_vector(op.n, 100 + j) for j in range(R)])
    W = op.apply_batch(X)
    for j in range(R):
        assert rel(W[j], op.apply_ax(X[j])) < 1e-14, j


def test_batch_device_pointers(case_files):
    import torch
    from mlfma_pmchwt_b200 import mesh as M
    op = gpu_op(case_files, "sphere_s3_lossy")
    X = np.stack([M.unit_disk_vector(op.n, 7 + j) for j in range(6)])
    xd = torch.from_numpy(X).cuda()
    wd = torch.empty_like(xd)
    op.apply_batch_device(6, xd.data_ptr(), wd.data_ptr())
    torch.cuda.synchronize()
    np.testing.assert_allclose(wd.cpu().numpy(), op.apply_batch(X), rtol=0, atol=1e-14 * np.abs(X).max())


def test_batch_argument_errors(case_files):
    from mlfma_pmchwt_b200 import MlfmaError
    op = gpu_op(case_files, "sphere_s3_lossy")
    with pytest.raises(ValueError):
        op.apply_batch(np.zeros((2, op.n + 2), dtype=np.complex128))
    with pytest.raises(MlfmaError):
        op.apply_batch_device(0, 1, 2)


def _incidences(op, R):
    from mlfma_pmchwt_b200 import plane_wave
    rows = []
    for j in range(R):
        th = 180.0 * j / max(R - 1, 1)
        rows.append(op.compute_v_pmchwt(*plane_wave(90.0 * (j % 2), th, 0.0)))
    return np.stack(rows)


@pytest.mark.parametrize("inner", [0, 8])
def test_lockstep_solve_matches_single_solves(case_files, inner):
    """Each system of the lockstep solve takes the single solve's steps: same
    iteration count, same solution to rounding (the batched reductions sum in
    another order)."""
    op = gpu_op(case_files, "sphere_s3_lossy")
    B = _incidences(op, 4)
    B[2] = 0.0  # converged before the first step: leaves the lockstep set at once
    X, st = op.matrix_solver_batch(B, itr_max=400, mr=30, tol_rel=1e-6, inner_its=inner)
    assert st[2]["converged"] and st[2]["iterations"] == 0 and not np.any(X[2])
    for j in (0, 1, 3):
        x1, s1 = op.matrix_solver(B[j], itr_max=400, mr=30, tol_rel=1e-6, inner_its=inner)
        assert st[j]["converged"] and s1["converged"]
        assert st[j]["iterations"] == s1["iterations"], (j, st[j]["iterations"], s1["iterations"])
        assert rel(X[j], x1) < 1e-9
        assert rel(op.apply_ax(X[j]), B[j]) < 1e-6 * 1.01
    if inner:
        assert st[0]["near_products"] == inner * st[0]["iterations"]


def test_lockstep_work_arrays_kept_between_calls(case_files):
    """The lockstep solve keeps its work arrays in the plan from one call to
    the next (one block, grown when a call needs more): solves of 3, then 20,
    then 2 systems on one plan give what fresh plans give, bit for bit."""
    from mlfma_pmchwt_b200 import MLFMM
    m, p, eps, leaf = case_files["sphere_s2"]
    op = MLFMM(m, freq=FREQ, eps_r=eps, leaf_coeff=leaf, device=0)
    B = _incidences(op, 20)
    for rows in (slice(0, 3), slice(0, 20), slice(5, 7)):
        X, st = op.matrix_solver_batch(B[rows], itr_max=300, mr=30, tol_rel=1e-5, inner_its=4)
        fresh = MLFMM(m, freq=FREQ, eps_r=eps, leaf_coeff=leaf, device=0)
        Xf, sf = fresh.matrix_solver_batch(B[rows], itr_max=300, mr=30, tol_rel=1e-5, inner_its=4)
        fresh.close()
        assert np.array_equal(X, Xf), rows
        assert [s["iterations"] for s in st] == [s["iterations"] for s in sf]
    op.close()


def test_lockstep_solve_more_systems_than_slots(case_files):
    """More right-hand sides than one batched apply takes (16): the applies
    go through in groups; every system converges to its own solution."""
    op = gpu_op(case_files, "sphere_s2")
    B = _incidences(op, 19)
    X, st = op.matrix_solver_batch(B, itr_max=300, mr=30, tol_rel=1e-5, inner_its=4)
    assert all(s["converged"] for s in st)
    W = op.apply_batch(X)
    for j in range(19):
        assert rel(W[j], B[j]) < 1e-5 * 1.01


def test_graph_replay_tracks_new_inputs(case_files):
    """One captured apply per stream serves every (x, w) pair: each replay
    reads the current contents of the caller's x and writes the caller's w
    (host path: the plan's own device vectors; device path: the caller's
    pointers and stream, recurring and new ones)."""
    import torch
    from mlfma_pmchwt_b200 import mesh as M
    op = gpu_op(case_files, "sphere_s3_lossy")
    xs = [M.unit_disk_vector(op.n, 40 + j) for j in range(3)]
    op.set_tuning("apply.graph", 0)
    direct = [op.apply_ax(x) for x in xs]
    op.set_tuning("apply.graph", 1)
    for _ in range(2):
        for x, w in zip(xs, direct):
            assert rel(op.apply_ax(x), w) < 1e-14
    stream = torch.cuda.Stream()
    xd = torch.empty(op.n, dtype=torch.complex128, device="cuda")
    wd = torch.empty_like(xd)
    for x, w in zip(xs + xs, direct + direct):
        xd.copy_(torch.from_numpy(x))
        torch.cuda.synchronize()
        op.apply_device(xd.data_ptr(), wd.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        assert rel(wd.cpu().numpy(), w) < 1e-14
    # a new pair of device vectors per apply (as a Krylov basis gives)
    X = [torch.from_numpy(x).to("cuda") for x in xs]
    W = [torch.full_like(X[0], float("nan")) for _ in xs]
    torch.cuda.synchronize()
    for xj, wj in zip(X, W):
        op.apply_device(xj.data_ptr(), wj.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    for wj, w in zip(W, direct):
        assert rel(wj.cpu().numpy(), w) < 1e-14
    assert op.device_status() == 0
