"""B200-native PMCHWT MLFMA operator and Krylov solve.

Python host mirror of the reference's operator interface (the ``MLFMM``
object of CCCCl0uD/MLFMA_PMCHWT, Code/MLFMM.h:11-82), backed by the in-tree
shared library ``libmlfma_pmchwt.so`` (C ABI: ``include/mlfma_pmchwt.h``).
All compute runs in that library's CUDA kernels; there is no CPU fallback:
if the library is missing, importing the operator raises.

    op = MLFMM(mesh, freq=3e8, eps_r=4.0, leaf_coeff=0.25)
    w = op.apply_ax(x)                                   # MLFMM::applyAx / the `ax` closure
    x, st = op.matrix_solver(rhs, itr_max=..., mr=30, tol_rel=1e-3)   # MGMRES::mgmres
    V = op.compute_v_pmchwt(*plane_wave(0.0, 0.0, 0.0))  # RHS::computeV_PMCHWT
    field, db = op.calculate_rcs_pmchwt(x, theta, phi)   # RCSUtils::calculateRCS_PMCHWT
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

from . import mesh as mesh_mod
from .mesh import Mesh

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libmlfma_pmchwt.so"

MLFMA_OK = 0
MLFMA_ERR_NOT_CONVERGED = 1
_ERRORS = {-1: "bad argument", -2: "mesh", -3: "CUDA", -4: "out of memory", -5: "unsupported"}


class MlfmaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"mlfma error {code} ({_ERRORS.get(code, '?')}): {msg}")
        self.code = code


class _MeshStruct(C.Structure):
    _fields_ = [("num_points", C.c_int), ("point_ids", C.POINTER(C.c_int)), ("xyz", C.POINTER(C.c_double)),
                ("num_faces", C.c_int), ("face_ids", C.POINTER(C.c_int)), ("face_points", C.POINTER(C.c_int))]


class Params(C.Structure):
    _fields_ = [("freq_hz", C.c_double), ("eps_r_re", C.c_double), ("eps_r_im", C.c_double),
                ("mu_r_re", C.c_double), ("mu_r_im", C.c_double), ("leaf_coeff", C.c_double),
                ("gauss_points", C.c_int), ("precision", C.c_int), ("device", C.c_int), ("verbose", C.c_int),
                ("tf_complex_argument", C.c_int), ("same_triangle_k", C.c_int)]


class Info(C.Structure):
    _fields_ = [("num_rwg", C.c_int), ("num_unknowns", C.c_int), ("max_level", C.c_int), ("num_levels", C.c_int),
                ("boxes", C.c_int * 16), ("L_k1", C.c_int * 16), ("L_k2", C.c_int * 16),
                ("K_k1", C.c_int * 16), ("K_k2", C.c_int * 16), ("near_pairs", C.c_longlong),
                ("far_pairs", C.c_longlong * 16), ("bytes_device", C.c_double), ("setup_seconds", C.c_double),
                ("k1_re", C.c_double), ("k1_im", C.c_double), ("k2_re", C.c_double), ("k2_im", C.c_double),
                ("etai_re", C.c_double), ("etai_im", C.c_double), ("wavelength", C.c_double)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("restarts", C.c_int), ("matvecs", C.c_int), ("converged", C.c_int),
                ("rel_residual", C.c_double), ("seconds", C.c_double), ("history_len", C.c_int),
                ("near_products", C.c_int)]


# Exported symbols with their ctypes signatures (mirrors include/mlfma_pmchwt.h).
_P = C.c_void_p
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
SIGNATURES = {
    "mlfma_default_params": (None, [C.POINTER(Params)]),
    "mlfma_last_error": (C.c_char_p, []),
    "mlfma_version": (C.c_char_p, []),
    "mlfma_plan_create": (C.c_int, [C.POINTER(_MeshStruct), C.POINTER(Params), C.POINTER(_P)]),
    "mlfma_plan_create_nas": (C.c_int, [C.c_char_p, C.POINTER(Params), C.POINTER(_P)]),
    "mlfma_plan_destroy": (C.c_int, [_P]),
    "mlfma_plan_info": (C.c_int, [_P, C.POINTER(Info)]),
    "mlfma_apply": (C.c_int, [_P, C.c_int, _DP, _DP]),
    "mlfma_apply_device": (C.c_int, [_P, C.c_int, _P, _P, _P]),
    "mlfma_device_status": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "mlfma_apply_batch": (C.c_int, [_P, C.c_int, C.c_int, _DP, _DP]),
    "mlfma_apply_batch_device": (C.c_int, [_P, C.c_int, C.c_int, _P, _P, _P]),
    "mlfma_apply_batch_mixed_device": (C.c_int, [_P, C.c_int, C.c_int, _P, _P, _P]),
    "mlfma_profile": (C.c_int, [_P, C.c_int]),
    "mlfma_profile_read": (C.c_int, [_P, _DP, C.POINTER(C.c_int)]),
    "mlfma_set_tuning": (C.c_int, [_P, C.c_char_p, C.c_int]),
    "mlfma_get_tuning": (C.c_int, [_P, C.c_char_p]),
    "mlfma_autotune": (C.c_int, [_P, C.c_int, _DP]),
    "mlfma_gmres": (C.c_int, [_P, C.c_int, _DP, _DP, C.c_int, C.c_int, C.c_double, C.c_double,
                              C.POINTER(SolveStats), _DP, C.c_int]),
    "mlfma_fgmres": (C.c_int, [_P, C.c_int, _DP, _DP, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                               C.POINTER(SolveStats), _DP, C.c_int]),
    "mlfma_fgmres_batch": (C.c_int, [_P, C.c_int, C.c_int, _DP, _DP, C.c_int, C.c_int, C.c_double, C.c_double,
                                     C.c_int, C.POINTER(SolveStats)]),
    "mlfma_apply_mixed": (C.c_int, [_P, C.c_int, _DP, _DP]),
    "mlfma_apply_mixed_device": (C.c_int, [_P, C.c_int, _P, _P, _P]),
    "mlfma_solve_mixed": (C.c_int, [_P, C.c_int, _DP, _DP, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                    C.c_int, C.POINTER(SolveStats), _DP, C.c_int]),
    "mlfma_solve_mixed_batch": (C.c_int, [_P, C.c_int, C.c_int, _DP, _DP, C.c_int, C.c_int, C.c_double, C.c_double,
                                          C.c_int, C.c_int, C.POINTER(SolveStats)]),
    "mlfma_apply_near_device": (C.c_int, [_P, C.c_int, _P, _P, _P]),
    "mlfma_near_precondition_device": (C.c_int, [_P, C.c_int, C.c_int, _P, _P, _P]),
    "mlfma_lp_param_count": (C.c_int, []),
    "mlfma_lp_forward_device": (C.c_int, [_P, C.c_int, _P, _P, _P, _P, _P]),
    "mlfma_lp_backward_device": (C.c_int, [_P, C.c_int, _P, _P, _P, _P]),
    "mlfma_lp_loss_grad_device": (C.c_int, [_P, C.c_int, _P, _P, _P, _P, _P, _P, _P, _P]),
    "mlfma_lp_adam_device": (C.c_int, [C.c_int, _P, _P, _P, _P, C.c_float, C.c_float, C.c_float, C.c_float,
                                       C.c_int, C.c_float, _P]),
    "mlfma_lp_attach": (C.c_int, [_P, C.POINTER(C.c_float), C.c_int]),
    "mlfma_rhs_pmchwt": (C.c_int, [_P, _DP, _DP, _DP, _DP]),
    "mlfma_rcs_pmchwt": (C.c_int, [_P, _DP, C.c_int, _DP, _DP, _DP, _DP]),
    "mlfma_rcs_pmchwt_noalloc": (C.c_int, [_P, _P, C.c_int, _DP, _DP, _P, _P]),
    "mlfma_rhs_pmchwt_batch_device": (C.c_int, [_P, C.c_int, C.c_int, _DP, _DP, _DP, _P, _P]),
    "mlfma_rcs_pmchwt_batch_device": (C.c_int, [_P, C.c_int, C.c_int, _P, C.c_int, _DP, _DP, _P, _P]),
    "mlfma_rcs_pmchwt_mono_device": (C.c_int, [_P, C.c_int, C.c_int, _P, _DP, _DP, _P, _P]),
    "mlfma_rcs_db": (C.c_int, [C.c_int, _DP, _DP, _DP, _DP]),
    "mlfma_rcs_noalloc_max_angles": (C.c_int, []),
    "mlfma_get_rwgs": (C.c_int, [_P, _IP, _IP, _IP, _IP, _IP, _IP, _DP, _DP]),
    "mlfma_get_level": (C.c_longlong, [_P, C.c_int, C.POINTER(C.c_ulonglong), _DP]),
    "mlfma_get_level_lists": (C.c_longlong, [_P, C.c_int, _IP, _IP, _IP, _IP, _IP]),
    "mlfma_get_leaf_rwgs": (C.c_longlong, [_P, _IP, _IP]),
    "mlfma_get_grid": (C.c_int, [_P, C.c_int, C.c_int, _DP, _DP, _DP, _DP]),
    "mlfma_get_interp": (C.c_int, [_P, C.c_int, C.c_int, _IP, _DP, _IP, _DP]),
    "mlfma_get_stage": (C.c_longlong, [_P, C.c_int, C.c_int, C.c_int, _DP]),
    "mlfma_get_pattern": (C.c_longlong, [_P, C.c_int, C.c_int, _DP]),
    "mlfma_get_transfer": (C.c_longlong, [_P, C.c_int, C.c_int, _IP, _DP]),
    "mlfma_get_near": (C.c_longlong, [_P, _IP, _IP, _DP, _DP, _DP]),
    "mlfma_get_near_same_triangle": (C.c_longlong, [_P, _IP, _IP, _DP]),
}

_lib = None


def load_library(path: str | Path | None = None) -> C.CDLL:
    """Loads libmlfma_pmchwt.so; raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m mlfma_pmchwt_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_IP)


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex128)


def rcs_db(theta_deg, phi_deg, field) -> np.ndarray:
    """RCS in dBsm (total, theta-pol, phi-pol) of far fields [n_angles, 3]
    (complex), formed as the reference does (mlfma_rcs_db)."""
    lib = load_library()
    f = np.ascontiguousarray(field, dtype=np.complex128).reshape(-1, 3)
    th = np.ascontiguousarray(np.atleast_1d(theta_deg), dtype=np.float64)
    ph = np.ascontiguousarray(np.broadcast_to(np.atleast_1d(phi_deg), th.shape), dtype=np.float64)
    if len(th) != len(f):
        raise ValueError("one angle per field")
    out = np.empty((len(th), 3))
    rc = lib.mlfma_rcs_db(len(th), _dp(th), _dp(ph), _dp(f.view(np.float64)), _dp(out))
    if rc < 0:
        raise MlfmaError(rc, lib.mlfma_last_error().decode(errors="replace"))
    return out


def plane_wave(pol_deg: float, theta_deg: float, phi_deg: float):
    """Incident unit vectors (k, E, H) of EMSource::initPW (Code/EMSource.cpp:34-72):
    degrees to radians with |angle| < 1e-6 snapped to zero, components below 1e-6
    snapped to zero, E = theta-hat for pol 0 ("V") or phi-hat for pol 90 ("H"),
    H = normalised k x E."""
    snap = lambda v: 0.0 if abs(v) < 1e-6 else v
    th = snap(theta_deg * math.pi / 180.0)
    ph = snap(phi_deg * math.pi / 180.0)
    pol = snap(pol_deg * math.pi / 180.0)
    k = np.array([snap(-math.sin(th) * math.cos(ph)), snap(-math.sin(th) * math.sin(ph)), snap(-math.cos(th))])
    vt = np.array([snap(-math.cos(th) * math.cos(ph)), snap(-math.cos(th) * math.sin(ph)), snap(math.sin(th))])
    vp = np.array([snap(-math.sin(ph)), snap(math.cos(ph)), 0.0])
    if abs(pol - snap(90.0 * math.pi / 180.0)) < 1e-6:
        e = vp
    elif abs(pol) < 1e-6:
        e = vt
    else:
        raise ValueError("polarisation must be 0 (V) or 90 (H) degrees")
    h = np.cross(k, e)
    nh = math.sqrt(float(h @ h))
    if nh > 1e-15:
        h = h / nh
    return k, e, h


def lp_param_count() -> int:
    """Parameters of the learned preconditioner's network."""
    return int(load_library().mlfma_lp_param_count())


def lp_adam_device(nparams: int, params_ptr: int, grad_ptr: int, m_ptr: int, v_ptr: int, lr: float, step: int,
                   beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8, grad_scale: float = 1.0,
                   stream: int | None = None):
    """One Adam step on device float32 parameters (moments m, v; step from 1)."""
    rc = load_library().mlfma_lp_adam_device(int(nparams), C.c_void_p(params_ptr), C.c_void_p(grad_ptr),
                                             C.c_void_p(m_ptr), C.c_void_p(v_ptr), lr, beta1, beta2, eps, int(step),
                                             grad_scale, C.c_void_p(stream or 0))
    if rc < 0:
        raise MlfmaError(rc, load_library().mlfma_last_error().decode(errors="replace"))


class MLFMM:
    """PMCHWT MLFMA operator for one homogeneous dielectric body on one GPU.

    Mirrors the reference's ``MLFMM`` object for the dielectric path
    (Code/MLFMM.h:11-82, Code/MLFMM.cpp:15-113): construction builds RWGs,
    octree, angular grids, transfer factors, interpolation, patterns and the
    near field; ``apply_ax`` is the matvec; ``matrix_solver`` is the GMRES
    solve. Unknowns are ordered as the reference's: x[:N] = J, x[N:] = M.

    ``device=-1`` builds only the host tables (RWGs, tree, grids,
    interpolation) for inspection; such an object refuses to apply.
    """

    def __init__(self, mesh: Mesh | None = None, *, nas_path: str | None = None, freq: float = 3.0e8,
                 eps_r: complex = 4.0, mu_r: complex = 1.0, leaf_coeff: float = 0.3, gauss_points: int = 7,
                 device: int = 0, verbose: bool = False, tf_complex_argument: bool = False,
                 precision: str = "fp64", same_triangle_k: str = "exact"):
        self._lib = load_library()
        prm = Params()
        self._lib.mlfma_default_params(C.byref(prm))
        eps_r, mu_r = complex(eps_r), complex(mu_r)
        prm.freq_hz, prm.eps_r_re, prm.eps_r_im = freq, eps_r.real, eps_r.imag
        prm.mu_r_re, prm.mu_r_im = mu_r.real, mu_r.imag
        prm.leaf_coeff, prm.gauss_points, prm.device, prm.verbose = leaf_coeff, gauss_points, device, int(verbose)
        prm.tf_complex_argument = int(tf_complex_argument)
        if same_triangle_k not in ("exact", "reference"):
            raise ValueError("same_triangle_k must be 'exact' or 'reference'")
        prm.same_triangle_k = 1 if same_triangle_k == "reference" else 0
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        prm.precision = 1 if precision == "mixed" else 0
        self.params = prm
        h = _P()
        if nas_path is not None:
            rc = self._lib.mlfma_plan_create_nas(str(nas_path).encode(), C.byref(prm), C.byref(h))
        else:
            if mesh is None:
                raise ValueError("mesh or nas_path required")
            self._keep = (np.ascontiguousarray(mesh.point_ids, dtype=np.int32),
                          np.ascontiguousarray(mesh.points, dtype=np.float64).reshape(-1),
                          np.ascontiguousarray(mesh.face_ids, dtype=np.int32),
                          np.ascontiguousarray(mesh.face_point_ids(), dtype=np.int32).reshape(-1))
            ms = _MeshStruct(len(self._keep[0]), _ip(self._keep[0]), _dp(self._keep[1]), len(self._keep[2]),
                             _ip(self._keep[2]), _ip(self._keep[3]))
            rc = self._lib.mlfma_plan_create(C.byref(ms), C.byref(prm), C.byref(h))
        self._check(rc)
        self._h = h
        self.device = device
        self.info = Info()
        self._check(self._lib.mlfma_plan_info(self._h, C.byref(self.info)))
        self.N = self.info.num_rwg
        self.n = 2 * self.N
        self.max_level = self.info.max_level

    # ------------------------------------------------------------ basics
    def _check(self, rc: int):
        if rc < 0:
            raise MlfmaError(rc, self._lib.mlfma_last_error().decode(errors="replace"))
        return rc

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mlfma_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def k1(self) -> complex:
        return complex(self.info.k1_re, self.info.k1_im)

    @property
    def k2(self) -> complex:
        return complex(self.info.k2_re, self.info.k2_im)

    @property
    def etai(self) -> complex:
        return complex(self.info.etai_re, self.info.etai_im)

    def levels(self) -> list[int]:
        return list(range(2, self.max_level + 1))

    # ----------------------------------------------------------- operator
    def apply_ax(self, x) -> np.ndarray:
        """w = A x (host arrays, complex128 [2N])."""
        x = _c128(x)
        if x.shape != (self.n,):
            raise ValueError(f"x must have shape ({self.n},)")
        w = np.empty(self.n, dtype=np.complex128)
        self._check(self._lib.mlfma_apply(self._h, self.n, _dp(x.view(np.float64)), _dp(w.view(np.float64))))
        return w

    __call__ = apply_ax

    def apply_device(self, x_ptr: int, w_ptr: int, stream: int | None = None):
        """w = A x on device pointers (complex128 [2N]); asynchronous on `stream`."""
        self._check(self._lib.mlfma_apply_device(self._h, self.n, C.c_void_p(x_ptr), C.c_void_p(w_ptr),
                                                 C.c_void_p(stream or 0)))

    def device_status(self) -> int:
        """Synchronizes the device; 0, or the status bits a kernel recorded
        (1: a bounded wait of the staged translation ran out)."""
        st = C.c_int(0)
        self._check(self._lib.mlfma_device_status(self._h, C.byref(st)))
        return st.value

    def apply_batch(self, X) -> np.ndarray:
        """W[j] = A X[j] for the rows of X (host, complex128 [R, 2N]); patterns
        and near-field entries are read once per group of 16 right-hand sides."""
        X = np.ascontiguousarray(X, dtype=np.complex128)
        if X.ndim != 2 or X.shape[1] != self.n:
            raise ValueError(f"X must have shape (R, {self.n})")
        W = np.empty_like(X)
        self._check(self._lib.mlfma_apply_batch(self._h, self.n, X.shape[0], _dp(X.view(np.float64)),
                                                _dp(W.view(np.float64))))
        return W

    def apply_batch_device(self, R: int, x_ptr: int, w_ptr: int, stream: int | None = None):
        """Batched apply on device pointers (complex128 [R, 2N]); asynchronous on `stream`."""
        self._check(self._lib.mlfma_apply_batch_device(self._h, self.n, int(R), C.c_void_p(x_ptr),
                                                       C.c_void_p(w_ptr), C.c_void_p(stream or 0)))

    def apply_batch_mixed_device(self, R: int, x_ptr: int, w_ptr: int, stream: int | None = None):
        """Batched apply with the complex64 operator on device pointers
        (complex128 [R, 2N]; mixed-precision plans); asynchronous on `stream`."""
        self._check(self._lib.mlfma_apply_batch_mixed_device(self._h, self.n, int(R), C.c_void_p(x_ptr),
                                                             C.c_void_p(w_ptr), C.c_void_p(stream or 0)))

    def set_tuning(self, key: str, value: int):
        self._check(self._lib.mlfma_set_tuning(self._h, key.encode(), int(value)))

    def get_tuning(self, key: str) -> int:
        return self._check(self._lib.mlfma_get_tuning(self._h, key.encode()))

    TUNING_KEYS = (("m2l.variant", 9), ("m2l.pair_warps", 3), ("up.variant", 4), ("up.threads", 3), ("l2l.variant", 2), ("agg.variant", 2), ("leaf.variant", 2), ("batch_tc.variant", 2), ("batch_tree.variant", 2), ("apply.graph", 2))

    def autotune(self, applies: int = 3) -> dict:
        """Times the values of each tuning key on this plan (one key at a
        time) and keeps the fastest; returns the choice and the per-apply ms
        of every value tried."""
        ms = np.zeros(sum(c for _, c in self.TUNING_KEYS))
        self._check(self._lib.mlfma_autotune(self._h, int(applies), _dp(ms)))
        out, o = {}, 0
        for key, cnt in self.TUNING_KEYS:
            out[key] = self.get_tuning(key)
            out[key + "_ms"] = [round(float(v), 4) for v in ms[o:o + cnt]]
            o += cnt
        return out

    STAGES = ("aggregation", "interpolation_up", "translation", "anterpolation_down", "leaf_testing_near")

    def profile(self, on: bool = True):
        """Record per-stage CUDA events on every apply (see stage_times)."""
        self._check(self._lib.mlfma_profile(self._h, int(on)))

    def stage_times(self):
        """Summed stage times (ms) since the last call and the apply count."""
        ms = np.zeros(len(self.STAGES))
        n = C.c_int(0)
        self._check(self._lib.mlfma_profile_read(self._h, _dp(ms), C.byref(n)))
        return dict(zip(self.STAGES, ms)), n.value

    def matrix_solver(self, rhs, x0=None, itr_max: int | None = None, mr: int = 50, tol_abs: float = 1e-8,
                      tol_rel: float = 1e-4, inner_its: int | None = None):
        """Restarted GMRES(mr) (MGMRES::mgmres with MLFMM::matrix_solver's
        arguments, Code/RCS.h:364-375 defaults: itr_max = 2N, mr = 50,
        tol_abs 1e-8, tol_rel 1e-4). With inner_its (>= 0) the solve is
        flexible GMRES preconditioned by inner_its near-field GMRES steps
        (mlfma_fgmres). Returns (x, stats dict)."""
        b = _c128(rhs)
        x = np.zeros(self.n, dtype=np.complex128) if x0 is None else _c128(x0).copy()
        itr_max = self.n if itr_max is None else int(itr_max)
        st = SolveStats()
        hist = np.zeros(max(itr_max, 1), dtype=np.float64)
        if inner_its is None:
            rc = self._lib.mlfma_gmres(self._h, self.n, _dp(x.view(np.float64)), _dp(b.view(np.float64)), itr_max,
                                       mr, tol_abs, tol_rel, C.byref(st), _dp(hist), len(hist))
        else:
            rc = self._lib.mlfma_fgmres(self._h, self.n, _dp(x.view(np.float64)), _dp(b.view(np.float64)), itr_max,
                                        mr, tol_abs, tol_rel, int(inner_its), C.byref(st), _dp(hist), len(hist))
        self._check(rc)
        stats = dict(iterations=st.iterations, restarts=st.restarts, matvecs=st.matvecs,
                     converged=bool(st.converged), rel_residual=st.rel_residual, seconds=st.seconds,
                     near_products=st.near_products, history=hist[: st.history_len].copy())
        return x, stats

    def matrix_solver_batch(self, rhs, x0=None, itr_max: int | None = None, mr: int = 50, tol_abs: float = 1e-8,
                            tol_rel: float = 1e-4, inner_its: int = 0):
        """Lockstep (F)GMRES of the R rows of rhs (complex128 [R, 2N]):
        per system matrix_solver(..., inner_its) with every operator apply,
        near-field product and Gram-Schmidt step batched over the systems
        still iterating (mlfma_fgmres_batch). Returns (X [R, 2N], list of
        per-system stats dicts)."""
        B = np.ascontiguousarray(rhs, dtype=np.complex128)
        if B.ndim != 2 or B.shape[1] != self.n:
            raise ValueError(f"rhs must have shape (R, {self.n})")
        R = B.shape[0]
        X = np.zeros_like(B) if x0 is None else np.ascontiguousarray(x0, dtype=np.complex128).copy()
        itr_max = self.n if itr_max is None else int(itr_max)
        st = (SolveStats * R)()
        rc = self._lib.mlfma_fgmres_batch(self._h, self.n, R, _dp(X.view(np.float64)), _dp(B.view(np.float64)),
                                          itr_max, mr, tol_abs, tol_rel, int(inner_its), st)
        self._check(rc)
        stats = [dict(iterations=s.iterations, restarts=s.restarts, matvecs=s.matvecs, converged=bool(s.converged),
                      rel_residual=s.rel_residual, seconds=s.seconds, near_products=s.near_products) for s in st]
        return X, stats

    def apply_ax_mixed(self, x) -> np.ndarray:
        """w = A x with the complex64 operator (plans created with precision='mixed')."""
        x = _c128(x)
        if x.shape != (self.n,):
            raise ValueError(f"x must have shape ({self.n},)")
        w = np.empty(self.n, dtype=np.complex128)
        self._check(self._lib.mlfma_apply_mixed(self._h, self.n, _dp(x.view(np.float64)), _dp(w.view(np.float64))))
        return w

    def apply_mixed_device(self, x_ptr: int, w_ptr: int, stream: int | None = None):
        self._check(self._lib.mlfma_apply_mixed_device(self._h, self.n, C.c_void_p(x_ptr), C.c_void_p(w_ptr),
                                                       C.c_void_p(stream or 0)))

    def solve_mixed(self, rhs, x0=None, itr_max: int | None = None, mr: int = 50, tol_abs: float = 1e-8,
                    tol_rel: float = 1e-4, inner_its: int = 16, refine_max: int = 10):
        """FP64 iterative refinement around complex64 FGMRES (mlfma_solve_mixed).
        Returns (x, stats); stats["history"] holds the FP64 relative residual
        after each refinement step (entry 0: initial)."""
        b = _c128(rhs)
        x = np.zeros(self.n, dtype=np.complex128) if x0 is None else _c128(x0).copy()
        itr_max = self.n if itr_max is None else int(itr_max)
        st = SolveStats()
        hist = np.zeros(refine_max + 1, dtype=np.float64)
        rc = self._lib.mlfma_solve_mixed(self._h, self.n, _dp(x.view(np.float64)), _dp(b.view(np.float64)), itr_max,
                                         mr, tol_abs, tol_rel, int(inner_its), int(refine_max), C.byref(st),
                                         _dp(hist), len(hist))
        self._check(rc)
        return x, dict(iterations=st.iterations, refinements=st.restarts, matvecs=st.matvecs,
                       converged=bool(st.converged), rel_residual=st.rel_residual, seconds=st.seconds,
                       near_products=st.near_products, history=hist[: st.history_len].copy())

    def solve_mixed_batch(self, rhs, x0=None, itr_max: int | None = None, mr: int = 50, tol_abs: float = 1e-8,
                          tol_rel: float = 1e-4, inner_its: int = 16, refine_max: int = 10):
        """solve_mixed for the rows of rhs (complex128 [R, 2N]) in lockstep
        (mlfma_solve_mixed_batch). Returns (X, list of per-system stats)."""
        B = np.ascontiguousarray(rhs, dtype=np.complex128)
        if B.ndim != 2 or B.shape[1] != self.n:
            raise ValueError(f"rhs must have shape (R, {self.n})")
        R = B.shape[0]
        X = np.zeros_like(B) if x0 is None else np.ascontiguousarray(x0, dtype=np.complex128).copy()
        itr_max = self.n if itr_max is None else int(itr_max)
        st = (SolveStats * R)()
        rc = self._lib.mlfma_solve_mixed_batch(self._h, self.n, R, _dp(X.view(np.float64)), _dp(B.view(np.float64)),
                                               itr_max, mr, tol_abs, tol_rel, int(inner_its), int(refine_max), st)
        self._check(rc)
        return X, [dict(iterations=s.iterations, refinements=s.restarts, matvecs=s.matvecs,
                        converged=bool(s.converged), rel_residual=s.rel_residual, seconds=s.seconds,
                        near_products=s.near_products) for s in st]

    def apply_near_device(self, x_ptr: int, w_ptr: int, stream: int | None = None):
        """w = Z_near x on device pointers (the near-field rows alone)."""
        self._check(self._lib.mlfma_apply_near_device(self._h, self.n, C.c_void_p(x_ptr), C.c_void_p(w_ptr),
                                                      C.c_void_p(stream or 0)))

    def near_precondition_device(self, inner_its: int, v_ptr: int, z_ptr: int, stream: int | None = None):
        """z = the near-field preconditioner of the flexible solves applied to
        v (device complex128 [2N]); returns when z is complete."""
        self._check(self._lib.mlfma_near_precondition_device(self._h, self.n, int(inner_its), C.c_void_p(v_ptr),
                                                             C.c_void_p(z_ptr), C.c_void_p(stream or 0)))

    # ------------------------------------------------- learned preconditioner
    def lp_forward_device(self, params_ptr: int | None, v_ptr: int, z_ptr: int, y_ptr: int,
                          stream: int | None = None):
        """y = the learned correction of z = P_near v (device complex128 [2N];
        params: device float32 [lp_param_count()], None = the attached network)."""
        self._check(self._lib.mlfma_lp_forward_device(self._h, self.n, C.c_void_p(params_ptr or 0),
                                                      C.c_void_p(v_ptr), C.c_void_p(z_ptr), C.c_void_p(y_ptr),
                                                      C.c_void_p(stream or 0)))

    def lp_backward_device(self, params_ptr: int, gy_ptr: int, grad_ptr: int, stream: int | None = None):
        """After lp_forward_device: adds the parameter gradient of a loss whose
        gradient with respect to y is gy = dL/dRe(y) + j dL/dIm(y) to grad_ptr."""
        self._check(self._lib.mlfma_lp_backward_device(self._h, self.n, C.c_void_p(params_ptr), C.c_void_p(gy_ptr),
                                                       C.c_void_p(grad_ptr), C.c_void_p(stream or 0)))

    def lp_loss_grad_device(self, params_ptr: int, v_ptr: int, z_ptr: int, e_ptr: int, y_ptr: int, grad_ptr: int,
                            loss_ptr: int, stream: int | None = None):
        """Forward pass into y, then adds sum|y - e|^2 / sum|e|^2 to the float
        at loss_ptr and its parameter gradient to grad_ptr (device float32)."""
        self._check(self._lib.mlfma_lp_loss_grad_device(self._h, self.n, C.c_void_p(params_ptr), C.c_void_p(v_ptr),
                                                        C.c_void_p(z_ptr), C.c_void_p(e_ptr), C.c_void_p(y_ptr),
                                                        C.c_void_p(grad_ptr), C.c_void_p(loss_ptr),
                                                        C.c_void_p(stream or 0)))

    def attach_learned(self, params) -> None:
        """Use the network with these (host float32) parameters after the
        near-field preconditioner in every flexible solve; None detaches."""
        if params is None:
            self._check(self._lib.mlfma_lp_attach(self._h, None, 0))
            return
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != lp_param_count():
            raise ValueError(f"expected {lp_param_count()} parameters")
        self._check(self._lib.mlfma_lp_attach(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))

    def compute_v_pmchwt(self, kinc, einc, hinc) -> np.ndarray:
        V = np.empty(self.n, dtype=np.complex128)
        k, e, h = (np.ascontiguousarray(v, dtype=np.float64) for v in (kinc, einc, hinc))
        self._check(self._lib.mlfma_rhs_pmchwt(self._h, _dp(k), _dp(e), _dp(h), _dp(V.view(np.float64))))
        return V

    def calculate_rcs_pmchwt(self, I, theta_deg, phi_deg):
        """Far field (3 complex components) and RCS dBsm (total, theta-pol, phi-pol) per angle."""
        I = _c128(I)
        th = np.ascontiguousarray(np.atleast_1d(theta_deg), dtype=np.float64)
        ph = np.ascontiguousarray(np.broadcast_to(np.atleast_1d(phi_deg), th.shape), dtype=np.float64)
        field = np.empty((len(th), 3), dtype=np.complex128)
        db = np.empty((len(th), 3), dtype=np.float64)
        self._check(self._lib.mlfma_rcs_pmchwt(self._h, _dp(I.view(np.float64)), len(th), _dp(th), _dp(ph),
                                               _dp(field.view(np.float64)), _dp(db)))
        return field, db

    def compute_v_pmchwt_batch_device(self, incidences, V_ptr: int, stream: int | None = None):
        """Excitation vectors of R plane waves, incidences = [(kinc, einc, hinc), ...]
        (as plane_wave returns them), into device complex128 [R, 2N] at V_ptr.
        Asynchronous on `stream`."""
        R = len(incidences)
        k, e, h = (np.ascontiguousarray(np.array([inc[i] for inc in incidences], dtype=np.float64).reshape(R, 3))
                   for i in range(3))
        self._check(self._lib.mlfma_rhs_pmchwt_batch_device(self._h, self.n, R, _dp(k), _dp(e), _dp(h),
                                                            C.c_void_p(V_ptr), C.c_void_p(stream or 0)))

    def calculate_rcs_batch_device(self, R: int, I_ptr: int, theta_deg, phi_deg, field_ptr: int,
                                   stream: int | None = None):
        """Bistatic far field of R device current vectors (complex128 [R, 2N])
        at the given angles into device complex128 [R, n_angles, 3]."""
        th = np.ascontiguousarray(np.atleast_1d(theta_deg), dtype=np.float64)
        ph = np.ascontiguousarray(np.broadcast_to(np.atleast_1d(phi_deg), th.shape), dtype=np.float64)
        self._check(self._lib.mlfma_rcs_pmchwt_batch_device(self._h, self.n, int(R), C.c_void_p(I_ptr), len(th),
                                                            _dp(th), _dp(ph), C.c_void_p(field_ptr),
                                                            C.c_void_p(stream or 0)))

    def calculate_rcs_mono_device(self, R: int, I_ptr: int, theta_deg, phi_deg, field_ptr: int,
                                  stream: int | None = None):
        """Monostatic far field: solution r seen at (theta_deg[r], phi_deg[r]),
        into device complex128 [R, 3]."""
        th = np.ascontiguousarray(np.atleast_1d(theta_deg), dtype=np.float64)
        ph = np.ascontiguousarray(np.broadcast_to(np.atleast_1d(phi_deg), th.shape), dtype=np.float64)
        if len(th) != R:
            raise ValueError("one angle per solution")
        self._check(self._lib.mlfma_rcs_pmchwt_mono_device(self._h, self.n, int(R), C.c_void_p(I_ptr), _dp(th),
                                                           _dp(ph), C.c_void_p(field_ptr), C.c_void_p(stream or 0)))

    def calculate_rcs_noalloc(self, I_ptr: int, theta_deg, phi_deg, field_ptr: int, stream: int | None = None):
        """Far field into caller-owned device memory with no device allocation
        (see mlfma_rcs_pmchwt_noalloc): I_ptr -> complex128 [2N] on the device,
        field_ptr -> complex128 [n_angles, 3] on the device. Asynchronous."""
        th = np.ascontiguousarray(np.atleast_1d(theta_deg), dtype=np.float64)
        ph = np.ascontiguousarray(np.broadcast_to(np.atleast_1d(phi_deg), th.shape), dtype=np.float64)
        self._check(self._lib.mlfma_rcs_pmchwt_noalloc(self._h, C.c_void_p(I_ptr), len(th), _dp(th), _dp(ph),
                                                       C.c_void_p(field_ptr), C.c_void_p(stream or 0)))

    # ------------------------------------------------------------ tables
    def rwgs(self) -> dict:
        N = self.N
        out = {k: np.empty(N, dtype=np.int32) for k in ("face_pos", "face_neg", "free_pos", "free_neg",
                                                          "edge_a", "edge_b")}
        out["length"] = np.empty(N)
        out["mid"] = np.empty((N, 3))
        self._check(self._lib.mlfma_get_rwgs(self._h, *(_ip(out[k]) for k in ("face_pos", "face_neg", "free_pos",
                                                                                "free_neg", "edge_a", "edge_b")),
                                             _dp(out["length"]), _dp(out["mid"])))
        return out

    def level(self, level: int):
        nb = self._check(self._lib.mlfma_get_level(self._h, level, None, None))
        codes = np.empty(nb, dtype=np.uint64)
        centers = np.empty((nb, 3))
        self._lib.mlfma_get_level(self._h, level, codes.ctypes.data_as(C.POINTER(C.c_ulonglong)), _dp(centers))
        return codes, centers

    def level_lists(self, level: int) -> dict:
        nb = self._check(self._lib.mlfma_get_level(self._h, level, None, None))
        near_ptr = np.empty(nb + 1, dtype=np.int32)
        far_ptr = np.empty(nb + 1, dtype=np.int32)
        self._check(self._lib.mlfma_get_level_lists(self._h, level, _ip(near_ptr), None, _ip(far_ptr), None, None))
        near_idx = np.empty(max(near_ptr[-1], 1), dtype=np.int32)
        far_idx = np.empty(max(far_ptr[-1], 1), dtype=np.int32)
        far_off = np.empty(max(far_ptr[-1], 1), dtype=np.int32)
        self._check(self._lib.mlfma_get_level_lists(self._h, level, _ip(near_ptr), _ip(near_idx), _ip(far_ptr),
                                                    _ip(far_idx), _ip(far_off)))
        return dict(near_ptr=near_ptr, near_idx=near_idx[: near_ptr[-1]], far_ptr=far_ptr,
                    far_idx=far_idx[: far_ptr[-1]], far_off=far_off[: far_ptr[-1]])

    def leaf_rwgs(self):
        nb = self._check(self._lib.mlfma_get_leaf_rwgs(self._h, None, None))
        ptr = np.empty(nb + 1, dtype=np.int32)
        rwg = np.empty(self.N, dtype=np.int32)
        self._lib.mlfma_get_leaf_rwgs(self._h, _ip(ptr), _ip(rwg))
        return ptr, rwg

    def grid(self, medium: int, level: int) -> dict:
        L = self._check(self._lib.mlfma_get_grid(self._h, medium, level, None, None, None, None))
        th, ph, wt, wp = np.empty(L), np.empty(2 * L), np.empty(L), np.empty(1)
        self._lib.mlfma_get_grid(self._h, medium, level, _dp(th), _dp(ph), _dp(wt), _dp(wp))
        return dict(L=L, theta=th, phi=ph, wtheta=wt, wphi=float(wp[0]))

    def interp(self, medium: int, level: int) -> dict:
        L = self.grid(medium, level)["L"]
        tidx, pidx = np.empty((L, 3), dtype=np.int32), np.empty((2 * L, 3), dtype=np.int32)
        lt, lp = np.empty((L, 3)), np.empty((2 * L, 3))
        self._check(self._lib.mlfma_get_interp(self._h, medium, level, _ip(tidx), _dp(lt), _ip(pidx), _dp(lp)))
        return dict(tidx=tidx, lt=lt, pidx=pidx, lp=lp)

    def stage(self, which: str, medium: int, level: int) -> np.ndarray:
        """Sm ('S') or Bm ('B') after the last apply: (boxes, 6, K) complex."""
        w = {"S": 0, "B": 1}[which]
        cnt = self._check(self._lib.mlfma_get_stage(self._h, w, medium, level, None))
        out = np.empty(cnt, dtype=np.complex128)
        self._check(self._lib.mlfma_get_stage(self._h, w, medium, level, _dp(out.view(np.float64))))
        K = (self.info.K_k1 if medium == 1 else self.info.K_k2)[level - 2]
        return out.reshape(-1, 6, K)

    def pattern(self, medium: int, which: str) -> np.ndarray:
        """Leaf radiation ('s') / receive ('f') patterns: (N, K, 3) complex, RWG order."""
        w = {"s": 0, "f": 1}[which]
        cnt = self._check(self._lib.mlfma_get_pattern(self._h, medium, w, None))
        out = np.empty(cnt, dtype=np.complex128)
        self._check(self._lib.mlfma_get_pattern(self._h, medium, w, _dp(out.view(np.float64))))
        return out.reshape(self.N, -1, 3)

    def transfer(self, medium: int, level: int):
        """Transfer factors (nvec, K) complex (no quadrature weight) and offsets (nvec, 3)."""
        cnt = self._check(self._lib.mlfma_get_transfer(self._h, medium, level, None, None))
        K = (self.info.K_k1 if medium == 1 else self.info.K_k2)[level - 2]
        nvec = cnt // K
        offs = np.empty((nvec, 3), dtype=np.int32)
        tf = np.empty(cnt, dtype=np.complex128)
        self._check(self._lib.mlfma_get_transfer(self._h, medium, level, _ip(offs), _dp(tf.view(np.float64))))
        return tf.reshape(nvec, K), offs

    def near(self, values: bool = True) -> dict:
        cnt = self._check(self._lib.mlfma_get_near(self._h, None, None, None, None, None))
        t = np.empty(cnt, dtype=np.int32)
        s = np.empty(cnt, dtype=np.int32)
        if not values:
            self._check(self._lib.mlfma_get_near(self._h, _ip(t), _ip(s), None, None, None))
            return dict(target=t, source=s)
        z = [np.empty(cnt, dtype=np.complex128) for _ in range(3)]
        self._check(self._lib.mlfma_get_near(self._h, _ip(t), _ip(s), *(_dp(v.view(np.float64)) for v in z)))
        return dict(target=t, source=s, z11=z[0], z12=z[1], z22=z[2])

    def near_same_triangle(self) -> dict:
        """The near pairs whose RWGs share a triangle, in the plan's order, with
        z12 evaluated on the host with the reference's own arithmetic (works on
        host-only plans)."""
        cnt = self._check(self._lib.mlfma_get_near_same_triangle(self._h, None, None, None))
        t = np.empty(cnt, dtype=np.int32)
        s = np.empty(cnt, dtype=np.int32)
        z = np.empty(cnt, dtype=np.complex128)
        self._check(self._lib.mlfma_get_near_same_triangle(self._h, _ip(t), _ip(s), _dp(z.view(np.float64))))
        return dict(target=t, source=s, z12=z)


__all__ = ["MLFMM", "Mesh", "MlfmaError", "load_library", "plane_wave", "rcs_db", "mesh_mod", "SIGNATURES", "LIB_PATH",
           "lp_param_count", "lp_adam_device"]
