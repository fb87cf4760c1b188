"""Test infrastructure: Python bindings of the two oracles.

* ``RefOperator`` -- the reference solver compiled from its own sources
  (``oracle/_ref/libmlfma_ref.so``, built by ``oracle/Makefile``) through the
  C-ABI driver ``oracle/ref_driver.cpp``.
* ``restatement()`` -- ``oracle/_ref/libpmchwt_oracle.so``, the plain-C
  restatement of the matvec and the GMRES loop (``oracle/pmchwt_oracle.c``),
  checked against ``RefOperator`` in tests/test_oracle.py.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs use
this module, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libmlfma_ref.so"
ORACLE_LIB = HERE / "_ref" / "libpmchwt_oracle.so"

_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
_ULP = C.POINTER(C.c_ulonglong)

_ref = None


def ref_available() -> bool:
    return REF_LIB.exists()


def _lib():
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} missing: run `make -C oracle`")
        lib = C.CDLL(str(REF_LIB))
        sig = {
            "ref_last_error": (C.c_char_p, []),
            "ref_set_threads": (None, [C.c_int]),
            "ref_create": (C.c_void_p, [C.c_char_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_int, C.c_int]),
            "ref_destroy": (None, [C.c_void_p]),
            "ref_sizes": (None, [C.c_void_p, _IP]),
            "ref_wave": (None, [C.c_void_p, _DP]),
            "ref_rwgs": (None, [C.c_void_p, _IP, _IP, _IP, _IP, _IP, _IP, _DP, _DP]),
            "ref_level_boxes": (C.c_int, [C.c_void_p, C.c_int]),
            "ref_level_info": (None, [C.c_void_p, C.c_int, _ULP, _DP, _DP, _IP, _IP, _IP]),
            "ref_box_lists": (None, [C.c_void_p, C.c_int, C.c_int, _IP, _ULP, _ULP, _IP]),
            "ref_dr_vec_count": (C.c_int, [C.c_void_p, C.c_int]),
            "ref_dr_vecs": (None, [C.c_void_p, C.c_int, _DP]),
            "ref_grid": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _DP, _DP, _DP, _DP]),
            "ref_tf": (None, [C.c_void_p, C.c_int, C.c_int, _DP]),
            "ref_interp": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _IP, _IP, _DP]),
            "ref_pattern": (None, [C.c_void_p, C.c_int, C.c_int, _DP]),
            "ref_znear_lengths": (None, [C.c_void_p, _IP]),
            "ref_znear": (None, [C.c_void_p, _IP, _DP]),
            "ref_apply": (None, [C.c_void_p, _DP, _DP]),
            "ref_stage": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _DP]),
            "ref_solve": (None, [C.c_void_p, _DP, _DP, C.c_int, C.c_int, C.c_double, C.c_double, C.c_char_p,
                                 C.c_int]),
            "ref_rhs": (None, [C.c_void_p, C.c_double, C.c_double, C.c_double, _DP, _DP]),
            "ref_rcs": (None, [C.c_void_p, _DP, C.c_double, C.c_double, C.c_double, _DP]),
            "ref_mom_matrix": (None, [C.c_void_p, _DP]),
            "ref_gmres_dense": (C.c_int, [C.c_int, _DP, _DP, _DP, C.c_int, C.c_int, C.c_double, C.c_double,
                                          C.c_char_p, C.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype, f.argtypes = res, args
        _ref = lib
    return _ref


def _dp(a):
    return a.ctypes.data_as(_DP)


def _ip(a):
    return a.ctypes.data_as(_IP)


def set_threads(n: int):
    _lib().ref_set_threads(int(n))


_RES_RE = re.compile(r"Cycle (\d+)\.(\d+) Res: ([0-9eE+\-.naif]+)")
_TRUE_RE = re.compile(r"(?:exact residual|Final residual|final residual): ([0-9eE+\-.naif]+)")


def parse_gmres_log(text: str):
    """Residual history printed by MGMRES::mgmres (Code/GMRES.h:155-157, 196-206)."""
    inner = [float(m.group(3)) for m in _RES_RE.finditer(text)]
    true = [float(m.group(1)) for m in _TRUE_RE.finditer(text)]
    return inner, true


class RefOperator:
    """The reference's PMCHWT MLFMA operator built from a NAS file."""

    def __init__(self, nas_path, freq=3.0e8, eps_r=4.0, mu_r=1.0, leaf_coeff=0.3, gauss_points=7, quiet=True):
        lib = _lib()
        eps_r, mu_r = complex(eps_r), complex(mu_r)
        self._h = lib.ref_create(str(nas_path).encode(), freq, eps_r.real, eps_r.imag, mu_r.real, mu_r.imag,
                                 leaf_coeff, gauss_points, 1 if quiet else 0)
        if not self._h:
            raise RuntimeError("reference operator build failed: " + lib.ref_last_error().decode())
        s = np.zeros(5, dtype=np.int32)
        lib.ref_sizes(self._h, _ip(s))
        self.N, self.max_level, self.level_span, self.num_points, self.num_faces = map(int, s)
        self.n = 2 * self.N
        w = np.zeros(11)
        lib.ref_wave(self._h, _dp(w))
        self.k1, self.k2, self.eta1, self.eta2, self.etai = (complex(w[2 * i], w[2 * i + 1]) for i in range(5))
        self.wavelength = float(w[10])

    def close(self):
        if getattr(self, "_h", None):
            _lib().ref_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- operator
    def apply(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.complex128)
        w = np.empty(self.n, dtype=np.complex128)
        _lib().ref_apply(self._h, _dp(x.view(np.float64)), _dp(w.view(np.float64)))
        return w

    def solve(self, rhs, x0=None, itr_max=None, mr=50, tol_abs=1e-8, tol_rel=1e-4):
        b = np.ascontiguousarray(rhs, dtype=np.complex128)
        x = np.zeros(self.n, dtype=np.complex128) if x0 is None else np.ascontiguousarray(x0, dtype=np.complex128).copy()
        itr_max = self.n if itr_max is None else itr_max
        buf = C.create_string_buffer(1 << 22)
        _lib().ref_solve(self._h, _dp(b.view(np.float64)), _dp(x.view(np.float64)), itr_max, mr, tol_abs, tol_rel,
                         buf, len(buf))
        text = buf.value.decode(errors="replace")
        inner, true = parse_gmres_log(text)
        return x, dict(log=text, history=inner, true_residuals=true)

    def rhs(self, pol, theta, phi):
        V = np.empty(self.n, dtype=np.complex128)
        vecs = np.empty(9)
        _lib().ref_rhs(self._h, pol, theta, phi, _dp(V.view(np.float64)), _dp(vecs))
        return V, vecs.reshape(3, 3)

    def rcs(self, I, pol, theta, phi):
        I = np.ascontiguousarray(I, dtype=np.complex128)
        out = np.empty(9)
        _lib().ref_rcs(self._h, _dp(I.view(np.float64)), pol, theta, phi, _dp(out))
        field = out[:6].view(np.complex128)
        return field, out[6:9]

    def mom_matrix(self):
        Z = np.empty((self.n, self.n), dtype=np.complex128)
        _lib().ref_mom_matrix(self._h, _dp(Z.view(np.float64)))
        return Z

    # -- tables
    def rwgs(self):
        N = self.N
        out = {k: np.empty(N, dtype=np.int32) for k in ("face_pos", "face_neg", "free_pos", "free_neg",
                                                          "edge_a", "edge_b")}
        out["length"] = np.empty(N)
        out["mid"] = np.empty((N, 3))
        _lib().ref_rwgs(self._h, *(_ip(out[k]) for k in ("face_pos", "face_neg", "free_pos", "free_neg", "edge_a",
                                                         "edge_b")), _dp(out["length"]), _dp(out["mid"]))
        return out

    def level(self, level):
        lib = _lib()
        nb = lib.ref_level_boxes(self._h, level)
        d = dict(morton=np.empty(nb, dtype=np.uint64), center=np.empty((nb, 3)), length=np.empty(nb),
                 n_rwg=np.empty(nb, dtype=np.int32), n_near=np.empty(nb, dtype=np.int32),
                 n_far=np.empty(nb, dtype=np.int32))
        lib.ref_level_info(self._h, level, d["morton"].ctypes.data_as(_ULP), _dp(d["center"]), _dp(d["length"]),
                           _ip(d["n_rwg"]), _ip(d["n_near"]), _ip(d["n_far"]))
        return d

    def box_lists(self, level, box, n_rwg, n_near, n_far):
        rwg = np.empty(max(n_rwg, 1), dtype=np.int32)
        near = np.empty(max(n_near, 1), dtype=np.uint64)
        far = np.empty(max(n_far, 1), dtype=np.uint64)
        vec = np.empty(max(n_far, 1), dtype=np.int32)
        _lib().ref_box_lists(self._h, level, box, _ip(rwg), near.ctypes.data_as(_ULP), far.ctypes.data_as(_ULP),
                             _ip(vec))
        return rwg[:n_rwg], near[:n_near], far[:n_far], vec[:n_far]

    def dr_vecs(self, level):
        n = _lib().ref_dr_vec_count(self._h, level)
        v = np.empty((max(n, 1), 3))
        _lib().ref_dr_vecs(self._h, level, _dp(v))
        return v[:n]

    def grid(self, medium, level):
        rev = self.max_level - level
        L = _lib().ref_grid(self._h, medium, rev, None, None, None, None)
        th, ph, wt, wp = np.empty(L), np.empty(2 * L), np.empty(L), np.empty(1)
        _lib().ref_grid(self._h, medium, rev, _dp(th), _dp(ph), _dp(wt), _dp(wp))
        return dict(L=L, theta=th, phi=ph, wtheta=wt, wphi=float(wp[0]))

    def transfer(self, medium, level):
        K = 2 * self.grid(medium, level)["L"] ** 2
        n = _lib().ref_dr_vec_count(self._h, level)
        tf = np.empty((max(n, 1), K), dtype=np.complex128)
        _lib().ref_tf(self._h, medium, level - 2, _dp(tf.view(np.float64)))
        return tf[:n], self.dr_vecs(level)

    def interp(self, medium, level):
        lib = _lib()
        K = lib.ref_interp(self._h, medium, level - 2, None, None, None)
        t, p, w = np.empty((K, 3), dtype=np.int32), np.empty((K, 3), dtype=np.int32), np.empty((K, 9))
        lib.ref_interp(self._h, medium, level - 2, _ip(t), _ip(p), _dp(w))
        return dict(tidx=t, pidx=p, w=w)

    def pattern(self, medium, which):
        K = 2 * self.grid(medium, self.max_level)["L"] ** 2
        out = np.empty((self.N, K, 3), dtype=np.complex128)
        _lib().ref_pattern(self._h, medium, {"s": 0, "f": 1}[which], _dp(out.view(np.float64)))
        return out

    def znear(self):
        lens = np.empty(self.n, dtype=np.int32)
        _lib().ref_znear_lengths(self._h, _ip(lens))
        tot = int(lens.sum())
        ids = np.empty(tot, dtype=np.int32)
        vals = np.empty(tot, dtype=np.complex128)
        _lib().ref_znear(self._h, _ip(ids), _dp(vals.view(np.float64)))
        ptr = np.concatenate([[0], np.cumsum(lens)])
        return ptr, ids, vals

    def stage(self, which, medium, level, box, pass_m):
        """Sm ('S') / Bm ('B') of pass J (pass_m=0) or M (1) for one box after apply: (K, 3)."""
        w = {"S": 0, "B": 1}[which]
        p = (medium - 1) * 2 + pass_m
        K = _lib().ref_stage(self._h, w, p, level - 2, box, None)
        out = np.empty((K, 3), dtype=np.complex128)
        _lib().ref_stage(self._h, w, p, level - 2, box, _dp(out.view(np.float64)))
        return out


def gmres_dense(A, b, x0=None, itr_max=100, mr=30, tol_abs=1e-8, tol_rel=1e-4):
    """MGMRES::mgmres on a dense matrix (the reference's solver, compiled)."""
    A = np.ascontiguousarray(A, dtype=np.complex128)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    n = b.shape[0]
    x = np.zeros(n, dtype=np.complex128) if x0 is None else np.ascontiguousarray(x0, dtype=np.complex128).copy()
    buf = C.create_string_buffer(1 << 22)
    ok = _lib().ref_gmres_dense(n, _dp(A.view(np.float64)), _dp(b.view(np.float64)), _dp(x.view(np.float64)),
                                itr_max, mr, tol_abs, tol_rel, buf, len(buf))
    inner, true = parse_gmres_log(buf.value.decode(errors="replace"))
    return x, bool(ok), inner, true


# ------------------------------------------------------------- restatement
_orc = None


def restatement():
    """ctypes handle of oracle/_ref/libpmchwt_oracle.so (the C restatement)."""
    global _orc
    if _orc is None:
        if not ORACLE_LIB.exists():
            raise FileNotFoundError(f"{ORACLE_LIB} missing: run `make -C oracle restatement`")
        lib = C.CDLL(str(ORACLE_LIB))
        P, I, D, CD = C.c_void_p, C.c_int, C.c_double, _Complex
        lib.orc_mexp.argtypes = [I, P, P, I, P, P, I, P]
        lib.orc_m2m.argtypes = [I, P, P, P, I, P, P, P, CD, P, I, P]
        lib.orc_m2l.argtypes = [I, P, P, P, I, I, P, P, D, P, P]
        lib.orc_l2l.argtypes = [I, P, P, P, I, P, P, P, I, P, CD, P, I, P]
        lib.orc_farfield.argtypes = [I, P, I, I, P, P, P, P, P, P, P, P, CD, CD, CD, P]
        lib.orc_near.argtypes = [I, P, P, P, P, P]
        lib.orc_gmres_dense.argtypes = [I, P, P, P, I, I, D, D, P, I, C.POINTER(C.c_int)]
        lib.orc_gmres_dense.restype = C.c_int
        for f in ("orc_mexp", "orc_m2m", "orc_m2l", "orc_l2l", "orc_farfield", "orc_near"):
            getattr(lib, f).restype = None
        _orc = lib
    return _orc


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class _Complex(C.Structure):
    """double complex passed by value (two SSE-class doubles in the x86-64 ABI)."""
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


def _cd(z):
    return _Complex(z.real, z.imag)


def _khat(grid):
    th, ph = grid["theta"], grid["phi"]
    st, ct = np.sin(th)[:, None], np.cos(th)[:, None]
    k = np.stack([np.broadcast_to(st * np.cos(ph)[None, :], (len(th), len(ph))),
                  np.broadcast_to(st * np.sin(ph)[None, :], (len(th), len(ph))),
                  np.broadcast_to(ct, (len(th), len(ph)))], axis=-1)
    return np.ascontiguousarray(k.reshape(-1, 3))


class RestatedOperator:
    """The C restatement driven with the reference operator's own tables
    (tree, grids, transfer factors, interpolation, patterns, near field)."""

    def __init__(self, ref: RefOperator):
        self.ref = ref
        L = ref.max_level
        self.L = L
        self.lv = {l: ref.level(l) for l in range(2, L + 1)}
        self.idx = {l: {int(c): i for i, c in enumerate(self.lv[l]["morton"])} for l in self.lv}
        # leaf RWG lists and interaction lists in reference order
        self.far = {}
        leaf = self.lv[L]
        rwg_ptr, rwg_ids = [0], []
        for l in range(2, L + 1):
            d = self.lv[l]
            fptr, fidx, fvec = [0], [], []
            for b in range(len(d["morton"])):
                rw, near, far, vec = ref.box_lists(l, b, int(d["n_rwg"][b]), int(d["n_near"][b]), int(d["n_far"][b]))
                fidx += [self.idx[l][int(c)] for c in far]
                fvec += list(vec)
                fptr.append(len(fidx))
                if l == L:
                    rwg_ids += list(rw)
                    rwg_ptr.append(len(rwg_ids))
            self.far[l] = tuple(np.ascontiguousarray(a, dtype=np.int32) for a in (fptr, fidx, fvec))
        self.rwg_ptr = np.array(rwg_ptr, dtype=np.int32)
        self.rwg_ids = np.array(rwg_ids, dtype=np.int32)
        self.leaf_of = np.empty(ref.N, dtype=np.int32)
        for b in range(len(leaf["morton"])):
            self.leaf_of[self.rwg_ids[self.rwg_ptr[b]:self.rwg_ptr[b + 1]]] = b
        # children of each parent, in child-level order (realSons order)
        self.children = {}
        for l in range(2, L):
            par, ch = self.lv[l], self.lv[l + 1]
            lists = [[] for _ in range(len(par["morton"]))]
            for j, c in enumerate(ch["morton"]):
                lists[self.idx[l][int(c) >> 3]].append(j)
            ptr = np.concatenate([[0], np.cumsum([len(x) for x in lists])]).astype(np.int32)
            cidx = np.array([j for x in lists for j in x], dtype=np.int32)
            pc = np.repeat(par["center"], np.diff(ptr), axis=0)
            cc = ch["center"][cidx]
            self.children[l] = (ptr, cidx, np.ascontiguousarray(pc - cc), np.ascontiguousarray(cc - pc))
        self.med = {}
        for m in (1, 2):
            g = {l: ref.grid(m, l) for l in range(2, L + 1)}
            tf = {l: np.ascontiguousarray(ref.transfer(m, l)[0]) for l in range(2, L + 1)}
            it = {}
            for l in range(2, L):
                d = ref.interp(m, l)
                nphc = 2 * g[l + 1]["L"]
                tp = (d["tidx"][:, :, None] * nphc + d["pidx"][:, None, :]).reshape(-1, 9).astype(np.int32)
                it[l] = (np.ascontiguousarray(tp), np.ascontiguousarray(d["tidx"]), np.ascontiguousarray(d["pidx"]),
                         np.ascontiguousarray(d["w"]))
            self.med[m] = dict(grid=g, khat={l: _khat(g[l]) for l in g}, tf=tf, interp=it,
                               Vs=np.ascontiguousarray(ref.pattern(m, "s")),
                               Vf=np.ascontiguousarray(ref.pattern(m, "f")),
                               k=ref.k1 if m == 1 else ref.k2)
        self.zptr, self.zids, self.zvals = (np.ascontiguousarray(a) for a in ref.znear())
        self.zptr = self.zptr.astype(np.int32)

    def apply(self, x):
        lib = restatement()
        ref, L = self.ref, self.L
        x = np.ascontiguousarray(x, dtype=np.complex128)
        N = ref.N
        Bleaf = {}
        for m in (1, 2):
            md = self.med[m]
            K = {l: 2 * md["grid"][l]["L"] ** 2 for l in range(2, L + 1)}
            nb = {l: len(self.lv[l]["morton"]) for l in range(2, L + 1)}
            for pm, off in ((0, 0), (1, N)):
                S = {l: np.zeros((nb[l], K[l], 3), dtype=np.complex128) for l in K}
                B = {l: np.zeros((nb[l], K[l], 3), dtype=np.complex128) for l in K}
                lib.orc_mexp(nb[L], _p(self.rwg_ptr), _p(self.rwg_ids), K[L], _p(md["Vs"]), _p(x), off, _p(S[L]))
                for l in range(L - 1, 1, -1):
                    ptr, cidx, v2f, _ = self.children[l]
                    tp, _, _, w = md["interp"][l]
                    lib.orc_m2m(nb[l], _p(ptr), _p(cidx), _p(v2f), K[l], _p(tp), _p(w), _p(md["khat"][l]),
                                _cd(md["k"]), _p(S[l + 1]), K[l + 1], _p(S[l]))
                for l in range(2, L + 1):
                    fptr, fidx, fvec = self.far[l]
                    g = md["grid"][l]
                    wgl = np.ascontiguousarray(g["wtheta"])
                    lib.orc_m2l(nb[l], _p(fptr), _p(fidx), _p(fvec), K[l], 2 * g["L"], _p(md["tf"][l]), _p(wgl),
                                g["wphi"], _p(S[l]), _p(B[l]))
                for l in range(2, L):
                    ptr, cidx, _, vc = self.children[l]
                    _, tidx, pidx, w = md["interp"][l]
                    lib.orc_l2l(nb[l], _p(ptr), _p(cidx), _p(vc), K[l], _p(tidx), _p(pidx), _p(w),
                                2 * md["grid"][l + 1]["L"], _p(md["khat"][l]), _cd(md["k"]), _p(B[l]), K[l + 1],
                                _p(B[l + 1]))
                Bleaf[(m, pm)] = B[L]
        w = np.zeros(2 * N, dtype=np.complex128)
        c1 = ref.k1 * ref.k1 / (16.0 * np.pi ** 2)
        c2 = ref.k2 * ref.k2 / (16.0 * np.pi ** 2)
        K1, K2 = 2 * self.med[1]["grid"][L]["L"] ** 2, 2 * self.med[2]["grid"][L]["L"] ** 2
        lib.orc_farfield(N, _p(self.leaf_of), K1, K2, _p(self.med[1]["Vf"]), _p(self.med[2]["Vf"]),
                         _p(self.med[1]["khat"][L]), _p(self.med[2]["khat"][L]), _p(Bleaf[(1, 0)]),
                         _p(Bleaf[(1, 1)]), _p(Bleaf[(2, 0)]), _p(Bleaf[(2, 1)]), _cd(c1), _cd(c2), _cd(ref.etai),
                         _p(w))
        lib.orc_near(2 * N, _p(self.zptr), _p(self.zids), _p(self.zvals), _p(x), _p(w))
        return w


def restated_gmres_dense(A, b, x0=None, itr_max=100, mr=30, tol_abs=1e-8, tol_rel=1e-4):
    A = np.ascontiguousarray(A, dtype=np.complex128)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    n = b.shape[0]
    x = np.zeros(n, dtype=np.complex128) if x0 is None else np.ascontiguousarray(x0, dtype=np.complex128).copy()
    hist = np.zeros(max(itr_max, 1))
    nh = C.c_int(0)
    ok = restatement().orc_gmres_dense(n, _p(A), _p(x), _p(b), itr_max, mr, tol_abs, tol_rel, _p(hist), len(hist),
                                       C.byref(nh))
    return x, bool(ok), hist[: nh.value]
