"""Host-side setup of the product against the reference, no GPU needed
(host-only plans, device=-1): RWG numbering (Code/RWGGenerator.cpp:39-113),
octree boxes and near / interaction lists (Code/OCTree.cpp:161-488),
angular grids (Code/AlgoMLFMM.h:21-138) and interpolation tables
(Code/AlgoMLFMM.h:141-189, 298-368)."""
import numpy as np
import pytest

from conftest import FREQ, needs_lib, needs_oracle

HOST_CASES = ["sphere_s2", "sphere_s3", "sphere_s3_lossy", "ellipsoid_s3", "sphere_s4_deep", "ellipsoid_s4_deep",
              "sphere_s2_flat", "sphere_s1_allnear"]


def host_plan(case_files, name):
    from mlfma_pmchwt_b200 import MLFMM
    m, p, eps, leaf = case_files[name]
    return MLFMM(m, freq=FREQ, eps_r=eps, leaf_coeff=leaf, device=-1)


@needs_lib
@needs_oracle
@pytest.mark.parametrize("name", HOST_CASES)
def test_rwg_numbering(case_files, ref_ops, name):
    op = host_plan(case_files, name)
    ref = ref_ops(name)
    assert op.N == ref.N
    a, b = ref.rwgs(), op.rwgs()
    for k in ("face_pos", "face_neg", "free_pos", "free_neg", "edge_a", "edge_b"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    np.testing.assert_allclose(b["length"], a["length"], rtol=1e-15, atol=0)
    np.testing.assert_array_equal(b["mid"], a["mid"])


@needs_lib
@needs_oracle
@pytest.mark.parametrize("name", HOST_CASES)
def test_octree_boxes_and_lists(case_files, ref_ops, name):
    op = host_plan(case_files, name)
    ref = ref_ops(name)
    assert op.max_level == ref.max_level
    for lvl in range(2, ref.max_level + 1):
        rl = ref.level(lvl)
        codes, centers = op.level(lvl)
        order = np.argsort(rl["morton"])
        np.testing.assert_array_equal(rl["morton"][order], codes)
        np.testing.assert_allclose(centers, rl["center"][order], rtol=0, atol=1e-12)
        lists = op.level_lists(lvl)
        idx = {int(c): i for i, c in enumerate(codes)}
        for bi in range(len(codes)):
            rw, near, far, vec = ref.box_lists(lvl, bi, int(rl["n_rwg"][bi]), int(rl["n_near"][bi]),
                                               int(rl["n_far"][bi]))
            mi = idx[int(rl["morton"][bi])]
            mine_far = {int(codes[j]) for j in lists["far_idx"][lists["far_ptr"][mi]:lists["far_ptr"][mi + 1]]}
            mine_near = {int(codes[j]) for j in lists["near_idx"][lists["near_ptr"][mi]:lists["near_ptr"][mi + 1]]}
            assert mine_far == {int(c) for c in far}
            assert mine_near == {int(c) for c in near}
            if lvl == ref.max_level:
                ptr, rwg = op.leaf_rwgs()
                np.testing.assert_array_equal(rwg[ptr[mi]:ptr[mi + 1]], rw)


@needs_lib
@needs_oracle
@pytest.mark.parametrize("name", HOST_CASES)
def test_grids_and_interpolation(case_files, ref_ops, name):
    op = host_plan(case_files, name)
    ref = ref_ops(name)
    for med in (1, 2):
        for lvl in range(2, ref.max_level + 1):
            g1, g2 = ref.grid(med, lvl), op.grid(med, lvl)
            assert g1["L"] == g2["L"]
            np.testing.assert_allclose(g2["theta"], g1["theta"], rtol=0, atol=1e-14)
            np.testing.assert_allclose(g2["phi"], g1["phi"], rtol=0, atol=1e-14)
            np.testing.assert_allclose(g2["wtheta"], g1["wtheta"], rtol=1e-13, atol=0)
            assert abs(g2["wphi"] - g1["wphi"]) < 1e-15
            if lvl < ref.max_level:
                i1, i2 = ref.interp(med, lvl), op.interp(med, lvl)
                nph = 2 * g1["L"]
                Kp = nph * g1["L"]
                t, p = np.arange(Kp) // nph, np.arange(Kp) % nph
                np.testing.assert_array_equal(i1["tidx"], i2["tidx"][t])
                np.testing.assert_array_equal(i1["pidx"], i2["pidx"][p])
                w = (i2["lt"][t][:, :, None] * i2["lp"][p][:, None, :]).reshape(Kp, 9)
                np.testing.assert_allclose(w, i1["w"], rtol=0, atol=1e-13)


@needs_lib
def test_multipole_orders_bench_sphere():
    """Level structure of the 245,760-unknown bench sphere (radius 5 lambda,
    sub 6, leaf 0.25 lambda): maxLevel 6, and L = ceil(kD + 6 (kD)^(1/3))."""
    from mlfma_pmchwt_b200 import MLFMM, mesh as M
    lam = M.wavelength(FREQ)
    m = M.icosphere(6, 5 * lam)
    op = MLFMM(m, freq=FREQ, eps_r=2.5 - 0.1j, leaf_coeff=0.25, device=-1)
    assert op.N == 122880 and op.max_level == 6
    k = 2 * np.pi / lam
    for i, lvl in enumerate(range(2, 7)):
        D = np.sqrt(3.0) * 0.25 * lam * 2 ** (6 - lvl)
        for kk, Ls in ((k, op.info.L_k1), (abs(k * np.sqrt(2.5 - 0.1j)), op.info.L_k2)):
            assert Ls[i] == int(np.ceil(kk * D + 6 * np.cbrt(kk * D)))
