"""External check of the transfer-factor choice for a lossy medium.

The reference evaluates the transfer factors with h2_l(|k2 R|), a real
argument, even for a complex (lossy) k2 (Code/AlgoMLFMM.h:259-281), while its
near field and radiation patterns use the complex k2. The plan parameter
tf_complex_argument = 1 uses h2_l(k2 R) instead. Which of the two operators
is closer to the true PMCHWT operator is settled here against the
reference's own dense MoM matrix (Code/Zmartix.h:467-539), solved directly:
on a lossy sphere (radius 1 m, icosphere sub 3, eps_r 2.5 - 0.1j, 3,840
unknowns), MLFMA solves to 1e-8 with either transfer factor against the
dense MoM solution: the residual of the MLFMA solution in the MoM system,
the current difference and the bistatic RCS (phi = 0, 361 angles) within
20 dB of the peak."""
import os

import numpy as np
import pytest

from conftest import FREQ, needs_lib, needs_oracle, rel

pytestmark = [pytest.mark.gpu, needs_lib, needs_oracle]


def test_complex_transfer_factors_against_dense_mom(tmp_path):
    from mlfma_pmchwt_b200 import MLFMM, plane_wave
    from mlfma_pmchwt_b200 import mesh as M
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)
    eps = complex(2.5, -0.1)
    m = M.icosphere(3, 1.0)
    nas = M.write_nas(m, tmp_path / "lossy.nas")
    ref = O.RefOperator(nas, freq=FREQ, eps_r=eps, leaf_coeff=0.25)
    A = ref.mom_matrix()
    V = ref.rhs(0.0, 0.0, 0.0)[0]
    x_mom = np.linalg.solve(A, V)
    ref.close()
    th = np.arange(0.0, 180.01, 0.5)
    out = {}
    for key, cplx_tf in (("reference", False), ("complex", True)):
        op = MLFMM(m, freq=FREQ, eps_r=eps, leaf_coeff=0.25, device=0, tf_complex_argument=cplx_tf)
        assert rel(op.compute_v_pmchwt(*plane_wave(0.0, 0.0, 0.0)), V) < 1e-13
        x, st = op.matrix_solver(V, itr_max=600, mr=50, tol_abs=0.0, tol_rel=1e-8, inner_its=8)
        assert st["converged"], key
        _, db = op.calculate_rcs_pmchwt(x, th, 0.0)
        _, db_mom = op.calculate_rcs_pmchwt(x_mom, th, 0.0)
        lit = db_mom[:, 0] >= db_mom[:, 0].max() - 20.0
        out[key] = dict(current=rel(x, x_mom), rcs_max=float(np.abs(db[:, 0] - db_mom[:, 0]).max()),
                        rcs_lit=float(np.abs(db[lit, 0] - db_mom[lit, 0]).max()),
                        residual_in_mom=float(np.linalg.norm(A @ x - V) / np.linalg.norm(V)))
        op.close()
    print("transfer-factor choice vs dense MoM:", out)
    # Measured on a B200: reference argument 0.241 residual in the MoM system,
    # 37 % current difference, 5.7 dB RCS error within 20 dB of the peak;
    # complex argument 0.0139, 2.1 %, 0.24 dB (the MLFMA discretisation's own
    # error at leaf 0.25 lambda with 3-point interpolation).
    c, r = out["complex"], out["reference"]
    assert c["residual_in_mom"] < 0.2 * r["residual_in_mom"] and c["residual_in_mom"] < 0.03
    assert c["current"] < 0.05 and c["rcs_lit"] < 0.5 and c["rcs_lit"] < 0.2 * r["rcs_lit"]
