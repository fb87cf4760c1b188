"""Generates the golden fixtures of tests/golden/ from the reference solver
compiled from its own sources (oracle/_ref/libmlfma_ref.so).

    make -C oracle && python tests/golden/make_golden.py

The reference ships no tests, meshes or stored results, so these fixtures are
its outputs on seeded synthetic bodies, produced here once and committed:

  sphere_s2.npz  icosphere sub 2, radius 0.5 m, eps_r 4, leaf 0.25 lambda (480 RWGs)
  sphere_s3.npz  icosphere sub 3, radius 1.0 m, eps_r 4, leaf 0.25 lambda (1920 RWGs,
                 the CPU-runnable reference configuration)

Each holds: sha256 of the NAS text; x (mt19937_64 seed 0, unit disk) and
w = A x; the plane-wave excitation V (x-polarised, incident along -z); the
GMRES(30) residual history of the first 60 inner steps and the iterate; the
bistatic RCS (361 angles, phi = 0) of that iterate.
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from mlfma_pmchwt_b200 import mesh as M  # noqa: E402
from oracle import oracle as O  # noqa: E402

FIXTURES = {
    "sphere_s2": dict(sub=2, radius=0.5, eps=4.0, leaf=0.25),
    "sphere_s3": dict(sub=3, radius=1.0, eps=4.0, leaf=0.25),
}


def nas_for(spec, path: Path) -> Path:
    return M.write_nas(M.icosphere(spec["sub"], spec["radius"]), path)


def make(name: str, spec: dict, tmp: Path):
    nas = nas_for(spec, tmp / f"{name}.nas")
    digest = hashlib.sha256(nas.read_bytes()).hexdigest()
    ref = O.RefOperator(nas, freq=3.0e8, eps_r=spec["eps"], leaf_coeff=spec["leaf"])
    x = M.unit_disk_vector(ref.n, 0)
    w = ref.apply(x)
    V, vecs = ref.rhs(0.0, 0.0, 0.0)
    xs, info = ref.solve(V, itr_max=60, mr=30, tol_abs=1e-8, tol_rel=1e-6)
    th = np.arange(0.0, 180.01, 0.5)
    rcs = np.array([ref.rcs(xs, 0.0, t, 0.0)[1] for t in th])
    np.savez_compressed(HERE / f"{name}.npz", nas_sha256=np.array(digest), N=ref.N, max_level=ref.max_level,
                        eps_r=np.array(complex(spec["eps"])), leaf=spec["leaf"], sub=spec["sub"],
                        radius=spec["radius"], x=x, w=w, V=V, vecs=vecs, gmres_history=np.array(info["history"]),
                        gmres_x=xs, rcs_theta=th, rcs_db=rcs)
    print(f"{name}: N={ref.N} maxLevel={ref.max_level} sha256={digest[:12]} |w|={np.linalg.norm(w):.6e}")
    ref.close()


def main():
    import tempfile
    O.set_threads(8)
    with tempfile.TemporaryDirectory() as d:
        for name, spec in FIXTURES.items():
            make(name, spec, Path(d))


if __name__ == "__main__":
    main()
