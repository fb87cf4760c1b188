"""Shared fixtures. GPU tests carry @pytest.mark.gpu; everything else runs on CPU.

Meshes are the synthetic bodies of mlfma_pmchwt_b200.mesh written as NAS files
into a temporary directory, so the product (arrays or NAS) and the reference
oracle (NAS) read the same doubles.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from mlfma_pmchwt_b200 import mesh as M  # noqa: E402

FREQ = 3.0e8
LAMBDA = M.wavelength(FREQ)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: longer CPU-side oracle runs")


def rel(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="session")
def mesh_dir(tmp_path_factory):
    return tmp_path_factory.mktemp("meshes")


# name -> (mesh builder, eps_r, leaf_coeff)
CASES = {
    # icosphere sub 2, radius 0.5 m: 480 RWGs (fast everywhere)
    "sphere_s2": (lambda: M.icosphere(2, 0.5), 4.0, 0.25),
    # config-1 geometry: radius 1.0 m, sub 3: 1920 RWGs, eps_r 4
    "sphere_s3": (lambda: M.icosphere(3, 1.0), 4.0, 0.25),
    # same mesh, lossy medium of the at-scale configuration, reference leaf 0.3
    "sphere_s3_lossy": (lambda: M.icosphere(3, 1.0), complex(2.5, -0.1), 0.3),
    # triaxial ellipsoid
    "ellipsoid_s3": (lambda: M.ellipsoid(3, 0.8 * LAMBDA, 0.5 * LAMBDA, 0.35 * LAMBDA), 3.0 - 0.05j, 0.25),
    # deep trees (maxLevel 5) at small cost: small leaf boxes
    "sphere_s4_deep": (lambda: M.icosphere(4, 1.5), 2.5 - 0.1j, 0.12),
    "ellipsoid_s4_deep": (lambda: M.ellipsoid(4, 2.0, 1.4, 1.0), 4.0, 0.15),
    # the smallest trees (maxLevel 2): no interpolation levels; and one whose
    # boxes are all near each other (no interaction pairs: near field only)
    "sphere_s2_flat": (lambda: M.icosphere(2, 0.3), 4.0, 0.25),
    "sphere_s1_allnear": (lambda: M.icosphere(1, 0.2), complex(2.5, -0.1), 0.3),
}


@pytest.fixture(scope="session")
def case_files(mesh_dir):
    out = {}
    for name, (mk, eps, leaf) in CASES.items():
        m = mk()
        p = M.write_nas(m, mesh_dir / f"{name}.nas")
        out[name] = (m, p, eps, leaf)
    return out


def oracle_ready() -> bool:
    from oracle import oracle as O
    return O.ref_available()


needs_oracle = pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libmlfma_ref.so").exists(),
                                  reason="oracle/_ref not built (make -C oracle)")
needs_lib = pytest.mark.skipif(not (ROOT / "mlfma_pmchwt_b200" / "libmlfma_pmchwt.so").exists(),
                               reason="libmlfma_pmchwt.so not built")

_ref_cache: dict = {}


@pytest.fixture(scope="session")
def ref_ops(case_files):
    """Lazily built reference operators, one per case (session cache)."""
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)

    def get(name):
        if name not in _ref_cache:
            m, p, eps, leaf = case_files[name]
            _ref_cache[name] = O.RefOperator(p, freq=FREQ, eps_r=eps, leaf_coeff=leaf)
        return _ref_cache[name]

    return get
