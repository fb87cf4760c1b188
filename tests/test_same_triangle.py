"""Near-field K entries of RWG pairs that share a triangle, evaluated on the
host with the reference's own arithmetic (plan parameter same_triangle_k =
'reference'), against the reference compiled from its sources. No GPU
needed: host-only plans answer mlfma_get_near_same_triangle.

For a field point on its own source triangle the reference's height
n.(r - v_i) (Code/Operator.h:582-587) is rounding noise; where it exceeds
10 eps0 the 1/R^3 integral takes its 1/|D| branch (:637-652) and the entry
is a residue of a ~1e15-sized cancellation, set by the last bits of every
operation. The host evaluation must therefore agree bit for bit, not to a
tolerance; on the deep ellipsoid some of these entries are such residues."""
import numpy as np
import pytest

from conftest import FREQ, needs_lib, needs_oracle

CASES = ["sphere_s2", "sphere_s3", "sphere_s3_lossy", "ellipsoid_s3", "sphere_s4_deep", "ellipsoid_s4_deep",
         "sphere_s2_flat", "sphere_s1_allnear"]


def _reference_z12(ref, N, target, source):
    """The reference's z12 (row t, column N + s of Z_near, Code/Zmartix.h:616-628)
    of the given pairs."""
    ptr, ids, vals = ref.znear()
    lens = np.diff(ptr[: N + 1])
    rows = np.repeat(np.arange(N, dtype=np.int64), lens)
    ids = ids[: ptr[N]].astype(np.int64)
    vals = vals[: ptr[N]]
    k12 = ids >= N
    key = rows[k12] * N + (ids[k12] - N)
    order = np.argsort(key)
    want = target.astype(np.int64) * N + source
    at = np.searchsorted(key[order], want)
    assert np.array_equal(key[order][at], want), "pair missing from the reference's near field"
    return vals[k12][order][at]


@needs_lib
@needs_oracle
@pytest.mark.parametrize("name", CASES)
def test_same_triangle_z12_bit_for_bit(case_files, ref_ops, name):
    from mlfma_pmchwt_b200 import MLFMM
    m, p, eps, leaf = case_files[name]
    op = MLFMM(m, freq=FREQ, eps_r=eps, leaf_coeff=leaf, device=-1, same_triangle_k="reference")
    st = op.near_same_triangle()
    r = op.rwgs()
    t, s = st["target"], st["source"]
    # every listed pair shares a triangle, and every RWG is listed with itself
    fp, fn = r["face_pos"], r["face_neg"]
    assert np.all((fp[t] == fp[s]) | (fp[t] == fn[s]) | (fn[t] == fp[s]) | (fn[t] == fn[s]))
    assert np.sum(t == s) == op.N
    # per triangle, 3 RWGs (or fewer on an open edge) form ordered pairs: at most 9 per face pair
    assert len(t) <= 9 * len(m.face_ids)
    want = _reference_z12(ref_ops(name), op.N, t, s)
    np.testing.assert_array_equal(st["z12"], want)
    op.close()


@needs_lib
def test_same_triangle_option_is_checked():
    from mlfma_pmchwt_b200 import MLFMM
    from mlfma_pmchwt_b200 import mesh as M
    with pytest.raises(ValueError):
        MLFMM(M.icosphere(1, 0.2), device=-1, same_triangle_k="noisy")
