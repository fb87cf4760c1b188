"""The CPU oracle of the learned preconditioner: its analytic gradient
against finite differences, exact linearity in z, symmetric leaf
neighbourhoods (which the GPU backward pass relies on), and the product's
parameter initialisation against the oracle's."""
import numpy as np
import pytest

from conftest import FREQ, needs_lib
from learned_util import oracle_graph

pytestmark = [needs_lib]


@pytest.fixture(scope="module")
def graph():
    from mlfma_pmchwt_b200 import MLFMM
    from mlfma_pmchwt_b200 import mesh as M
    m = M.icosphere(2, 0.6)
    op = MLFMM(m, freq=FREQ, eps_r=3 - 0.1j, leaf_coeff=0.25, device=-1)
    return oracle_graph(op, m, 3 - 0.1j)


def _vectors(n, seed=1):
    rng = np.random.default_rng(seed)
    c = lambda: rng.normal(size=n) + 1j * rng.normal(size=n)
    v = c()
    z = 0.7 * v + 0.2 * c()
    return v, z, z + 0.3 * c()


def test_gradient_matches_finite_differences(graph):
    from oracle import learned_precond as LP
    rng = np.random.default_rng(3)
    th = LP.init_params(0).astype(np.float64) + 0.05 * rng.normal(size=LP.param_count())
    v, z, e = _vectors(2 * graph.N)
    L, gr, _ = LP.loss_grad(th, graph, v, z, e, bf16=False)
    offs = np.cumsum([0] + [int(np.prod(s)) for _, s in LP.layout()])
    idx = np.concatenate([rng.choice(th.size, 30, replace=False), offs[:-1] + 1])
    for i in idx:
        h = 1e-6 * max(1.0, abs(th[i]))
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        fd = (LP.loss_grad(tp, graph, v, z, e, bf16=False)[0] - LP.loss_grad(tm, graph, v, z, e, bf16=False)[0]) / (2 * h)
        assert abs(fd - gr[i]) <= 1e-4 * abs(gr[i]) + 1e-7 * np.abs(gr).max(), (i, fd, gr[i])


def test_output_is_linear(graph):
    """The gains depend on the static features only: y = (I + L) z."""
    from oracle import learned_precond as LP
    rng = np.random.default_rng(4)
    th = LP.init_params(1) + np.float32(0.05) * rng.normal(size=LP.param_count()).astype(np.float32)
    v1, z1, _ = _vectors(2 * graph.N, 2)
    v2, z2, _ = _vectors(2 * graph.N, 3)
    a, b = 2.5 * np.exp(0.7j), -0.3 + 1.1j
    y = LP.forward(th, graph, a * v1 + b * v2, a * z1 + b * z2)
    ref = a * LP.forward(th, graph, v1, z1) + b * LP.forward(th, graph, v2, z2)
    assert np.linalg.norm(y - ref) < 1e-12 * np.linalg.norm(ref)


def test_untrained_network_is_the_near_preconditioner(graph):
    from oracle import learned_precond as LP
    v, z, _ = _vectors(2 * graph.N, 5)
    assert np.array_equal(LP.forward(LP.init_params(0), graph, v, z), z)


def test_leaf_neighbourhoods_are_symmetric(graph):
    for b, nb in enumerate(graph.nbr):
        assert b in nb
        for c in nb:
            assert b in graph.nbr[c]


def test_product_initialisation_matches_oracle():
    from oracle import learned_precond as LP
    from mlfma_pmchwt_b200 import learned, lp_param_count
    assert lp_param_count() == LP.param_count() == 48480
    assert [s for _, s in learned.layout()] == [s for _, s in LP.layout()]
    assert np.array_equal(learned.init_params(7), LP.init_params(7))


def test_bf16_rounding_is_nearest_even():
    from oracle import learned_precond as LP
    x = np.array([1.0, 1.00390625, 1.01171875, -3.14159265, 1e-30], dtype=np.float32)
    r = LP.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625  # ties to even, both directions
    assert abs(r[3] + 3.140625) < 1e-12
