"""Learned preconditioner on the GPU: the library's forward pass, loss and
parameter gradient against the CPU oracle (oracle/learned_precond.py), the
Adam kernel against the oracle's step, and the near-field preconditioner
entry against the one inside the flexible solve."""
import numpy as np
import pytest

from conftest import FREQ, needs_lib, rel
from learned_util import oracle_graph

pytestmark = [pytest.mark.gpu, needs_lib]

EPS = 4.0 - 0.2j


@pytest.fixture(scope="module")
def body():
    from mlfma_pmchwt_b200 import MLFMM
    from mlfma_pmchwt_b200 import mesh as M
    m = M.ellipsoid(3, 1.2, 0.8, 0.6)
    op = MLFMM(m, freq=FREQ, eps_r=EPS, leaf_coeff=0.25, device=0)
    yield op, oracle_graph(op, m, EPS)
    op.close()


def _params(seed):
    from oracle import learned_precond as LP
    rng = np.random.default_rng(seed)
    return (LP.init_params(seed) + 0.05 * rng.normal(size=LP.param_count())).astype(np.float32)


@pytest.mark.parametrize("seed", [0, 1])
def test_forward_loss_and_gradient_match_oracle(body, seed):
    import torch
    from oracle import learned_precond as LP
    op, g = body
    rng = np.random.default_rng(10 + seed)
    n = op.n
    c = lambda: rng.normal(size=n) + 1j * rng.normal(size=n)
    v = c()
    z = 0.6 * v + 0.3 * c()
    e = z + 0.4 * c()
    th = _params(seed)
    dev = torch.device("cuda", 0)
    V, Z, E = (torch.from_numpy(a).to(dev) for a in (v, z, e))
    Y = torch.full_like(V, float("nan"))
    Y2 = torch.full_like(V, float("nan"))
    T = torch.from_numpy(th).to(dev)
    G = torch.zeros_like(T)
    L = torch.zeros(1, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    s = 0  # the plan's stream
    op.lp_loss_grad_device(T.data_ptr(), V.data_ptr(), Z.data_ptr(), E.data_ptr(), Y.data_ptr(), G.data_ptr(),
                           L.data_ptr(), s)
    op.lp_forward_device(T.data_ptr(), V.data_ptr(), Z.data_ptr(), Y2.data_ptr(), s)
    torch.cuda.synchronize()
    L_ref, g_ref, y_ref = LP.loss_grad(th, g, v, z, e)
    y = Y.cpu().numpy()
    assert rel(y - z, y_ref - z) < 1e-4           # the correction itself, FP32 against float64
    assert np.array_equal(y, Y2.cpu().numpy())   # inference = the training forward pass
    assert abs(L.item() - L_ref) < 1e-5 * L_ref
    grad = G.cpu().numpy().astype(np.float64)
    assert rel(grad, g_ref) < 1e-4
    o = 0
    for name, shape in LP.layout():
        k = int(np.prod(shape))
        assert rel(grad[o:o + k], g_ref[o:o + k]) < 1e-3, name
        o += k


def test_adam_step_matches_oracle():
    import torch
    from mlfma_pmchwt_b200 import lp_adam_device
    from oracle import learned_precond as LP
    rng = np.random.default_rng(5)
    n = 1000
    th, gr = rng.normal(size=n).astype(np.float32), rng.normal(size=n).astype(np.float32)
    m, s = np.zeros(n, np.float32), np.zeros(n, np.float32)
    dev = torch.device("cuda", 0)
    T, G, Mm, S = (torch.from_numpy(a.copy()).to(dev) for a in (th, gr, m, s))
    for step in (1, 2, 3):
        lp_adam_device(n, T.data_ptr(), G.data_ptr(), Mm.data_ptr(), S.data_ptr(), 1e-2, step, grad_scale=0.5,
                       stream=torch.cuda.current_stream().cuda_stream)
        th, m, s = LP.adam(th, 0.5 * gr, m, s, step, lr=1e-2)
    torch.cuda.synchronize()
    assert np.allclose(T.cpu().numpy(), th, rtol=1e-5, atol=1e-6)


def test_untrained_network_returns_z(body):
    import torch
    from mlfma_pmchwt_b200 import learned
    op, _ = body
    rng = np.random.default_rng(2)
    v = rng.normal(size=op.n) + 1j * rng.normal(size=op.n)
    dev = torch.device("cuda", 0)
    V = torch.from_numpy(v).to(dev)
    Z = torch.empty_like(V)
    Y = torch.empty_like(V)
    torch.cuda.synchronize()
    op.near_precondition_device(8, V.data_ptr(), Z.data_ptr())
    T = torch.from_numpy(learned.init_params(0)).to(dev)
    op.lp_forward_device(T.data_ptr(), V.data_ptr(), Z.data_ptr(), Y.data_ptr(),
                         torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert torch.equal(Y, Z)
    # the preconditioner entry is the flexible solve's: one FGMRES step from
    # zero with restart 1 returns x = alpha z for b = v
    x, st = op.matrix_solver(v, itr_max=1, mr=1, tol_rel=1e-30, tol_abs=0.0, inner_its=8)
    zz = Z.cpu().numpy()
    alpha = np.vdot(zz, x) / np.vdot(zz, zz)
    assert rel(x, alpha * zz) < 1e-12


def test_backward_of_a_given_output_gradient_matches_oracle(body):
    """The residual-space training path: forward, then the backward pass of a
    given dL/dy (here a random vector) against the oracle."""
    import torch
    from oracle import learned_precond as LP
    op, g = body
    rng = np.random.default_rng(21)
    n = op.n
    c = lambda: rng.normal(size=n) + 1j * rng.normal(size=n)
    v = c()
    z = 0.5 * v + 0.3 * c()
    gy = c() * 1e-3
    th = _params(4)
    dev = torch.device("cuda", 0)
    V, Z, GY = (torch.from_numpy(a).to(dev) for a in (v, z, gy))
    Y = torch.empty_like(V)
    T = torch.from_numpy(th).to(dev)
    G = torch.zeros_like(T)
    torch.cuda.synchronize()
    op.lp_forward_device(T.data_ptr(), V.data_ptr(), Z.data_ptr(), Y.data_ptr())
    op.lp_backward_device(T.data_ptr(), GY.data_ptr(), G.data_ptr())
    torch.cuda.synchronize()
    g_ref, y_ref = LP.grad_from_gy(th, g, v, z, gy)
    assert rel(Y.cpu().numpy() - z, y_ref - z) < 1e-4
    assert rel(G.cpu().numpy().astype(np.float64), g_ref) < 1e-4


def test_training_and_the_solve_with_the_network():
    """Harvest (v, z) pairs on three small ellipsoids, train with the
    library's kernels, and solve a held-out body with and without the
    network: training lowers the objective |A M v - v|^2 on the held-out
    body's pairs, and FGMRES with the network attached converges to the
    tolerance. The iteration counts of both are the measured gain (not
    asserted: the correction may help or not)."""
    from mlfma_pmchwt_b200 import MLFMM, learned
    from mlfma_pmchwt_b200 import mesh as M
    bodies = []
    for k, (axes, er) in enumerate([((1.0, 0.7, 0.6), 3.0), ((0.8, 0.8, 1.1), 4.5), ((1.2, 0.6, 0.7), 2.5),
                                    ((0.9, 0.75, 0.65), 3.5)]):
        op = MLFMM(M.ellipsoid(3, *axes), freq=FREQ, eps_r=er, leaf_coeff=0.25, device=0)
        bodies.append((op, learned.random_directions(op, 24, seed=k)))
    train, (hop, hdata) = bodies[:3], bodies[3]
    params, hist, secs = learned.train(train, epochs=6, lr=1e-3, batch=8)
    assert np.all(np.isfinite(hist)) and hist[-1] < hist[0]
    before = learned.Trainer(learned.init_params(0)).evaluate([(hop, hdata)])
    after = learned.Trainer(params).evaluate([(hop, hdata)])
    assert abs(before["network"] - before["near_only"]) < 1e-5 * before["near_only"]
    assert after["network"] < before["network"]
    rhs = [hop.compute_v_pmchwt(*pw) for pw in learned.incidences(2)]
    gain = learned.solve_gain(hop, params, rhs, inner_its=8)
    assert gain["near_field"]["converged"] == 2 and gain["learned"]["converged"] == 2
    print("held-out objective", before["network"], "->", after["network"], "iterations", gain)
    for op, _ in bodies:
        op.close()


def test_attached_network_in_lockstep_and_mixed_solves():
    """With a network attached, each system of the lockstep FGMRES takes the
    single solve's steps (same iterations, same solution to rounding), the
    lockstep mixed-precision solve reaches the FP64 tolerance, and detaching
    restores the near-field-only iteration."""
    from mlfma_pmchwt_b200 import MLFMM, learned
    from mlfma_pmchwt_b200 import mesh as M
    rng = np.random.default_rng(8)
    th = learned.init_params(2)
    o = learned.lp_param_count() - 32 - 32 * 64       # the output layer Wd2, d2
    th[o:] = (0.02 * rng.normal(size=th.size - o)).astype(np.float32)
    op = MLFMM(M.ellipsoid(3, 1.0, 0.8, 0.7), freq=FREQ, eps_r=3.0 - 0.1j, leaf_coeff=0.25, device=0,
               precision="mixed")
    B = np.stack([op.compute_v_pmchwt(*pw) for pw in learned.incidences(3)])
    x0, s0 = op.matrix_solver(B[0], itr_max=300, mr=30, tol_rel=1e-6, tol_abs=0.0, inner_its=4)
    op.attach_learned(th)
    X, st = op.matrix_solver_batch(B, itr_max=300, mr=30, tol_rel=1e-6, tol_abs=0.0, inner_its=4)
    for j in range(3):
        x1, s1 = op.matrix_solver(B[j], itr_max=300, mr=30, tol_rel=1e-6, tol_abs=0.0, inner_its=4)
        assert st[j]["converged"] and s1["converged"]
        assert st[j]["iterations"] == s1["iterations"], (j, st[j]["iterations"], s1["iterations"])
        assert rel(X[j], x1) < 1e-8
    Xm, sm = op.solve_mixed_batch(B, itr_max=300, mr=30, tol_rel=1e-8, tol_abs=0.0, inner_its=4, refine_max=12)
    assert all(s["converged"] for s in sm)
    for j in range(3):
        assert rel(op.apply_ax(Xm[j]), B[j]) < 1e-8
    op.attach_learned(None)
    x2, s2 = op.matrix_solver(B[0], itr_max=300, mr=30, tol_rel=1e-6, tol_abs=0.0, inner_its=4)
    assert s2["iterations"] == s0["iterations"] and rel(x2, x0) < 1e-12
    op.close()
