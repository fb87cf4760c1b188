"""Pins the oracle against the committed golden fixtures (outputs of the
reference compiled from its sources, tests/golden/make_golden.py): the mesh
generator reproduces the same NAS bytes, and the oracle built on this machine
(and the C restatement) reproduce the stored matvec, excitation, GMRES
history and RCS."""
import hashlib

import numpy as np
import pytest

from conftest import ROOT, needs_oracle, rel

GOLDEN = ROOT / "tests" / "golden"
NAMES = ["sphere_s2", "sphere_s3"]


def load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def nas(name, tmp_path):
    from mlfma_pmchwt_b200 import mesh as M
    g = load(name)
    return M.write_nas(M.icosphere(int(g["sub"]), float(g["radius"])), tmp_path / f"{name}.nas"), g


@pytest.mark.parametrize("name", NAMES)
def test_mesh_bytes_reproduce(name, tmp_path):
    p, g = nas(name, tmp_path)
    assert hashlib.sha256(p.read_bytes()).hexdigest() == str(g["nas_sha256"])


@needs_oracle
@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(name, tmp_path):
    from oracle import oracle as O
    p, g = nas(name, tmp_path)
    ref = O.RefOperator(p, freq=3.0e8, eps_r=complex(g["eps_r"]), leaf_coeff=float(g["leaf"]))
    assert ref.N == int(g["N"]) and ref.max_level == int(g["max_level"])
    assert rel(ref.apply(g["x"]), g["w"]) < 1e-12
    V, vecs = ref.rhs(0.0, 0.0, 0.0)
    assert rel(V, g["V"]) < 1e-14
    np.testing.assert_array_equal(vecs, g["vecs"])
    xs, info = ref.solve(V, itr_max=60, mr=30, tol_abs=1e-8, tol_rel=1e-6)
    np.testing.assert_allclose(info["history"], g["gmres_history"], rtol=1e-5)
    assert rel(xs, g["gmres_x"]) < 1e-9
    db = np.array([ref.rcs(xs, 0.0, t, 0.0)[1] for t in g["rcs_theta"][::30]])
    np.testing.assert_allclose(db, g["rcs_db"][::30], atol=1e-9)
    # the C restatement on the same tables
    ro = O.RestatedOperator(ref)
    assert rel(ro.apply(g["x"]), g["w"]) < 1e-12
    ref.close()
