"""Synthetic closed triangle meshes and the NAS dialect the reference reads.

The reference's meshes are not distributed with it, so bodies are generated
here from their parametric definitions:

* ``icosphere(sub, radius)`` -- regular icosahedron, each subdivision splits
  every triangle into four with the edge midpoints projected to the sphere
  (sub 3: 1280 triangles / 1920 RWGs; sub 5: 20,480 / 30,720; sub 6: 81,920 /
  122,880).
* ``ellipsoid(sub, a, b, c)`` -- icosphere vertices scaled per axis.
* ``superellipsoid(sub, a, b, c, p)`` -- icosphere vertices mapped onto
  |x/a|^p + |y/b|^p + |z/c|^p = 1.

Faces are oriented outward (the reference derives normals from vertex order,
Code/NASReader.cpp:39-58). ``write_nas`` writes ``GRID*`` records with a
``*`` continuation line repeating the id (Code/NASReader.cpp:72-96) and
``CTRIA3`` records (Code/NASReader.cpp:97-120), ids 1-based, coordinates
with 17 significant digits so that every reader sees the same doubles.
"""
from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np

C0 = 299792458.0  # m/s (Code/PhyConstant.h:9)


def wavelength(freq_hz: float) -> float:
    """Free-space wavelength c0 / f (Code/EMSource.cpp:8)."""
    return C0 / freq_hz


@dataclass
class Mesh:
    points: np.ndarray      # (P, 3) float64
    faces: np.ndarray       # (F, 3) int, 0-based into points
    point_ids: np.ndarray   # (P,) int32 GRID ids
    face_ids: np.ndarray    # (F,) int32 CTRIA3 ids

    @property
    def num_faces(self) -> int:
        return int(self.faces.shape[0])

    @property
    def num_edges(self) -> int:
        e = np.sort(np.concatenate([self.faces[:, [0, 1]], self.faces[:, [1, 2]], self.faces[:, [2, 0]]]), axis=1)
        return int(np.unique(e, axis=0).shape[0])

    def face_point_ids(self) -> np.ndarray:
        return self.point_ids[self.faces].astype(np.int32)


def _icosahedron():
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = []
    for s1 in (-1.0, 1.0):
        for s2 in (-1.0, 1.0):
            v.append((0.0, s1, s2 * t))
            v.append((s1, s2 * t, 0.0))
            v.append((s2 * t, 0.0, s1))
    v = np.array(v, dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    d = np.linalg.norm(v[:, None, :] - v[None, :, :], axis=2)
    edge = np.min(d[d > 1e-9])
    adj = np.abs(d - edge) < 1e-9
    faces = []
    n = len(v)
    for i in range(n):
        for j in range(i + 1, n):
            if not adj[i, j]:
                continue
            for k in range(j + 1, n):
                if adj[i, k] and adj[j, k]:
                    faces.append([i, j, k])
    return v, _orient(v, np.array(faces, dtype=np.int64))


def _orient(v: np.ndarray, f: np.ndarray) -> np.ndarray:
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    n = np.cross(b - a, c - a)
    flip = np.einsum("ij,ij->i", n, a + b + c) < 0
    f = f.copy()
    f[flip, 1], f[flip, 2] = f[flip, 2].copy(), f[flip, 1].copy()
    return f


def _unit_icosphere(sub: int):
    v, f = _icosahedron()
    verts = [tuple(p) for p in v]
    for _ in range(sub):
        cache: dict[tuple[int, int], int] = {}

        def mid(i: int, j: int) -> int:
            key = (i, j) if i < j else (j, i)
            if key not in cache:
                p = np.add(verts[i], verts[j]) * 0.5
                p /= np.linalg.norm(p)
                cache[key] = len(verts)
                verts.append(tuple(p))
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = np.array(nf, dtype=np.int64)
    return np.array(verts, dtype=np.float64), f


def _finish(p: np.ndarray, f: np.ndarray) -> Mesh:
    f = _orient(p, f)
    return Mesh(points=np.ascontiguousarray(p, dtype=np.float64), faces=np.ascontiguousarray(f, dtype=np.int64),
                point_ids=np.arange(1, len(p) + 1, dtype=np.int32),
                face_ids=np.arange(1, len(f) + 1, dtype=np.int32))


def icosphere(sub: int, radius: float = 1.0) -> Mesh:
    p, f = _unit_icosphere(sub)
    return _finish(p * radius, f)


def ellipsoid(sub: int, a: float, b: float, c: float) -> Mesh:
    p, f = _unit_icosphere(sub)
    return _finish(p * np.array([a, b, c]), f)


def superellipsoid(sub: int, a: float, b: float, c: float, power: float = 4.0) -> Mesh:
    p, f = _unit_icosphere(sub)
    scale = np.sum(np.abs(p) ** power, axis=1) ** (1.0 / power)
    q = p / scale[:, None]
    return _finish(q * np.array([a, b, c]), f)


def write_nas(mesh: Mesh, path: str | Path) -> Path:
    path = Path(path)
    lines = ["$ synthetic body", "BEGIN BULK"]
    for pid, (x, y, z) in zip(mesh.point_ids, mesh.points):
        lines.append(f"GRID*   {int(pid)} {x:.17g} {y:.17g}")
        lines.append(f"*       {int(pid)} {z:.17g}")
    fp = mesh.face_point_ids()
    for fid, (a, b, c) in zip(mesh.face_ids, fp):
        lines.append(f"CTRIA3  {int(fid)} 1 {int(a)} {int(b)} {int(c)}")
    lines.append("ENDDATA")
    path.write_text("\n".join(lines) + "\n")
    return path


def read_nas(path: str | Path) -> Mesh:
    """Reads the same dialect back (GRID* + continuation, CTRIA3)."""
    ids, pts, fids, fpts = [], [], [], []
    pending = None
    for line in Path(path).read_text().splitlines():
        if line.startswith("GRID*"):
            t = line[5:].split()
            pending = (int(t[0]), float(t[1]), float(t[2]))
        elif pending is not None and line.startswith("*"):
            t = line[1:].split()
            if int(t[0]) != pending[0]:
                raise ValueError("GRID* continuation id mismatch")
            ids.append(pending[0])
            pts.append((pending[1], pending[2], float(t[1])))
            pending = None
        elif line.startswith("CTRIA3"):
            t = line[6:].split()
            fids.append(int(t[0]))
            fpts.append((int(t[2]), int(t[3]), int(t[4])))
    index = {pid: i for i, pid in enumerate(ids)}
    faces = np.array([[index[a], index[b], index[c]] for a, b, c in fpts], dtype=np.int64)
    return Mesh(points=np.array(pts, dtype=np.float64), faces=faces, point_ids=np.array(ids, dtype=np.int32),
                face_ids=np.array(fids, dtype=np.int32))


def unit_disk_vector(n: int, seed: int = 0) -> np.ndarray:
    """Seeded complex vector uniform on the unit disk: with g = mt19937_64(seed),
    u1 = (g() >> 11) * 2^-53, u2 likewise, x = sqrt(u1) exp(j 2 pi u2)."""
    g = _MT19937_64(seed)
    out = np.empty(n, dtype=np.complex128)
    for i in range(n):
        u1 = (g.next() >> 11) * 2.0 ** -53
        u2 = (g.next() >> 11) * 2.0 ** -53
        out[i] = np.sqrt(u1) * np.exp(2j * np.pi * u2)
    return out


class _MT19937_64:
    """The 64-bit Mersenne Twister (Matsumoto & Nishimura), std::mt19937_64."""

    def __init__(self, seed: int):
        self.mt = [0] * 312
        self.mt[0] = seed & 0xFFFFFFFFFFFFFFFF
        for i in range(1, 312):
            self.mt[i] = (6364136223846793005 * (self.mt[i - 1] ^ (self.mt[i - 1] >> 62)) + i) & 0xFFFFFFFFFFFFFFFF
        self.i = 312

    def next(self) -> int:
        if self.i >= 312:
            self._twist()
        y = self.mt[self.i]
        self.i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & 0xFFFFFFFFFFFFFFFF

    def _twist(self):
        mt = self.mt
        for i in range(312):
            x = (mt[i] & 0xFFFFFFFF80000000) | (mt[(i + 1) % 312] & 0x7FFFFFFF)
            xa = x >> 1
            if x & 1:
                xa ^= 0xB5026F5AA96619E9
            mt[i] = mt[(i + 156) % 312] ^ xa
        self.i = 0


def uneven_bodies(seed: int = 1, freq_hz: float = 3.0e8) -> list[dict]:
    """24 dielectric bodies drawn from std::mt19937_64(seed), in this order and
    with these distributions (u = (g() >> 11) 2^-53 uniform on [0, 1)):
      8 icospheres:      sub = 3 + floor(3u), radius = (1 + 1.5u) lambda;
      8 ellipsoids:      semi-axes (0.5 + 2.5u) lambda each, sub = 4 + floor(2u);
      8 superellipsoids: exponent 4, semi-axes (0.5 + 1.0u) lambda each, the
                         subdivision (3..5) whose mean edge is closest to 0.1 lambda;
    then for every body eps_r' = 1.5 + 4.5u and tan(delta) = 0.05u, eps_r =
    eps_r' (1 - j tan(delta)). Returns dicts with the mesh and the material."""
    g = _MT19937_64(seed)
    u = lambda: (g.next() >> 11) * 2.0 ** -53
    lam = wavelength(freq_hz)
    bodies = []
    for _ in range(8):
        sub = 3 + int(3 * u())
        r = (1.0 + 1.5 * u()) * lam
        bodies.append(dict(kind="icosphere", mesh=icosphere(sub, r), params=dict(sub=sub, radius=r)))
    for _ in range(8):
        a, b, c = ((0.5 + 2.5 * u()) * lam for _ in range(3))
        sub = 4 + int(2 * u())
        bodies.append(dict(kind="ellipsoid", mesh=ellipsoid(sub, a, b, c), params=dict(sub=sub, axes=(a, b, c))))
    for _ in range(8):
        a, b, c = ((0.5 + 1.0 * u()) * lam for _ in range(3))
        best = None
        for sub in (3, 4, 5):
            m = superellipsoid(sub, a, b, c, 4.0)
            edge = _mean_edge(m)
            if best is None or abs(edge - 0.1 * lam) < abs(best[1] - 0.1 * lam):
                best = (m, edge, sub)
        bodies.append(dict(kind="superellipsoid", mesh=best[0], params=dict(sub=best[2], axes=(a, b, c), power=4.0,
                                                                           mean_edge=best[1])))
    for b in bodies:
        er = 1.5 + 4.5 * u()
        td = 0.05 * u()
        b["eps_r"] = complex(er, -er * td)
    return bodies


def training_ellipsoids(count: int = 200, seed: int = 2, freq_hz: float = 3.0e8) -> list[dict]:
    """Triaxial ellipsoids for training the learned preconditioner, drawn
    from std::mt19937_64(seed) (u as in uneven_bodies): per body the semi-axes
    (0.5 + 1.5u) lambda each, then eps_r = 2 + 4u (lossless); icosphere
    subdivision 4 mapped onto the ellipsoid (7,680 RWGs, 15,360 unknowns)."""
    g = _MT19937_64(seed)
    u = lambda: (g.next() >> 11) * 2.0 ** -53
    lam = wavelength(freq_hz)
    out = []
    for _ in range(count):
        a, b, c = ((0.5 + 1.5 * u()) * lam for _ in range(3))
        er = 2.0 + 4.0 * u()
        out.append(dict(kind="ellipsoid", mesh=ellipsoid(4, a, b, c), params=dict(sub=4, axes=(a, b, c)),
                        eps_r=complex(er, 0.0)))
    return out


def held_out_ellipsoid(sub: int = 6, freq_hz: float = 3.0e8) -> dict:
    """The evaluation body of the learned preconditioner: a 6 x 2 x 2 lambda
    ellipsoid (semi-axes 3, 1, 1 lambda), eps_r = 3.0 - 0.05j; subdivision 6
    gives 122,880 RWGs (245,760 unknowns)."""
    lam = wavelength(freq_hz)
    return dict(kind="ellipsoid", mesh=ellipsoid(sub, 3.0 * lam, 1.0 * lam, 1.0 * lam),
                params=dict(sub=sub, axes=(3.0 * lam, lam, lam)), eps_r=complex(3.0, -0.05))


def _mean_edge(m: Mesh) -> float:
    p = np.asarray(m.points)
    idx = {int(i): k for k, i in enumerate(m.point_ids)}
    fv = np.array([[idx[int(v)] for v in tri] for tri in m.face_point_ids()])
    e = np.concatenate([np.linalg.norm(p[fv[:, i]] - p[fv[:, (i + 1) % 3]], axis=1) for i in range(3)])
    return float(e.mean())
