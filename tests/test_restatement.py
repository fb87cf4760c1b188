"""The C restatement of the oracle (oracle/pmchwt_oracle.c) against the
reference compiled from its sources: the restated matvec stages composed on
the reference's own tables reproduce its matvec, and the restated GMRES
reproduces MGMRES::mgmres iterate by iterate on a dense system."""
import numpy as np
import pytest

from conftest import needs_oracle, rel


@needs_oracle
@pytest.mark.parametrize("name", ["sphere_s2", "sphere_s3_lossy"])
def test_restated_matvec_matches_reference(ref_ops, name):
    from mlfma_pmchwt_b200 import mesh as M
    from oracle.oracle import RestatedOperator
    ref = ref_ops(name)
    ro = RestatedOperator(ref)
    x = M.unit_disk_vector(ref.n, 0)
    assert rel(ro.apply(x), ref.apply(x)) < 1e-13


@needs_oracle
def test_restated_gmres_matches_reference_gmres():
    from oracle.oracle import gmres_dense, restated_gmres_dense
    rng = np.random.default_rng(7)
    n = 120
    A = np.eye(n) * 3 + (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    xr, okr, hr, tr = gmres_dense(A, b, itr_max=200, mr=15, tol_rel=1e-10)
    xo, oko, ho = restated_gmres_dense(A, b, itr_max=200, mr=15, tol_rel=1e-10)
    assert okr and oko
    assert len(hr) == len(ho)
    # the reference prints residuals with std::cout's default 6 significant digits
    np.testing.assert_allclose(ho, hr, rtol=1e-5)
    assert rel(xo, xr) < 1e-10
    assert np.linalg.norm(A @ xo - b) / np.linalg.norm(b) < 1e-8  # tol_abs
