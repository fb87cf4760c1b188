"""The C-ABI library: loads without a GPU, exports every symbol that
include/mlfma_pmchwt.h declares, and maps bad input onto status codes
(no exception crosses the boundary). No compute call is made here."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import FREQ, ROOT, needs_lib

HEADER = ROOT / "include" / "mlfma_pmchwt.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"MLFMA_API\s+[\w\s\*]+?\b(mlfma_\w+)\s*\(", text)))


@needs_lib
def test_exports_every_declared_symbol():
    from mlfma_pmchwt_b200 import LIB_PATH, SIGNATURES
    lib = C.CDLL(str(LIB_PATH))
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
        assert n in SIGNATURES, f"{n} missing from the Python mirror"


@needs_lib
def test_version_and_defaults():
    from mlfma_pmchwt_b200 import Params, load_library
    lib = load_library()
    assert b"sm_100a" in lib.mlfma_version()
    p = Params()
    lib.mlfma_default_params(C.byref(p))
    assert p.freq_hz == 3.0e8 and p.leaf_coeff == 0.3 and p.gauss_points == 7 and p.eps_r_re == 1.0


@needs_lib
def test_bad_arguments_return_codes(tmp_path):
    from mlfma_pmchwt_b200 import MLFMM, MlfmaError, Params, load_library
    from mlfma_pmchwt_b200 import mesh as M
    lib = load_library()
    h = C.c_void_p()
    p = Params()
    lib.mlfma_default_params(C.byref(p))
    assert lib.mlfma_plan_create(None, C.byref(p), C.byref(h)) == -1
    assert lib.mlfma_plan_create_nas(str(tmp_path / "missing.nas").encode(), C.byref(p), C.byref(h)) == -2
    assert b"cannot open" in lib.mlfma_last_error()
    assert lib.mlfma_apply(None, 4, None, None) == -1
    m = M.icosphere(1, 0.3)
    with pytest.raises(MlfmaError) as e:
        MLFMM(m, gauss_points=5, device=-1)
    assert e.value.code == -1
    # a mesh whose faces reference a missing vertex
    bad = M.Mesh(points=m.points, faces=m.faces, point_ids=m.point_ids + 1000, face_ids=m.face_ids)
    bad.face_point_ids = lambda: m.face_point_ids()
    with pytest.raises(MlfmaError) as e:
        MLFMM(bad, device=-1)
    assert e.value.code == -2


@needs_lib
def test_host_only_plan_refuses_compute():
    from mlfma_pmchwt_b200 import MLFMM, MlfmaError
    from mlfma_pmchwt_b200 import mesh as M
    op = MLFMM(M.icosphere(2, 0.5), freq=FREQ, eps_r=4.0, leaf_coeff=0.25, device=-1)
    assert op.N == 480 and op.n == 960
    with pytest.raises(MlfmaError) as e:
        op.apply_ax(np.zeros(op.n, complex))
    assert e.value.code == -5
    with pytest.raises(ValueError):
        op.apply_ax(np.zeros(op.n + 2, complex))
    w = np.zeros(op.n + 2, dtype=np.complex128)
    assert op._lib.mlfma_apply(op._h, op.n + 2, w.ctypes.data_as(C.POINTER(C.c_double)),
                               w.ctypes.data_as(C.POINTER(C.c_double))) == -1
    with pytest.raises(MlfmaError):
        op.matrix_solver(np.zeros(op.n, complex), itr_max=1)
    op.close()


@needs_lib
def test_nas_path_and_arrays_agree(tmp_path):
    from mlfma_pmchwt_b200 import MLFMM
    from mlfma_pmchwt_b200 import mesh as M
    m = M.ellipsoid(2, 0.6, 0.4, 0.3)
    p = M.write_nas(m, tmp_path / "e.nas")
    a = MLFMM(m, device=-1, eps_r=3.0)
    b = MLFMM(nas_path=p, device=-1, eps_r=3.0)
    ra, rb = a.rwgs(), b.rwgs()
    for k in ra:
        np.testing.assert_array_equal(ra[k], rb[k])
    assert a.info.near_pairs == b.info.near_pairs
