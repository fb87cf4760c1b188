"""Synthetic mesh generator, NAS round trip and the seeded vector generator."""
import numpy as np
import pytest

from mlfma_pmchwt_b200 import mesh as M


@pytest.mark.parametrize("sub,faces,edges", [(0, 20, 30), (3, 1280, 1920), (5, 20480, 30720)])
def test_icosphere_counts(sub, faces, edges):
    m = M.icosphere(sub, 1.0)
    assert m.num_faces == faces
    assert m.num_edges == edges
    assert len(m.points) == 10 * 4 ** sub + 2
    np.testing.assert_allclose(np.linalg.norm(m.points, axis=1), 1.0, atol=1e-15)


def test_outward_orientation_all_bodies():
    for m in (M.icosphere(2, 1.0), M.ellipsoid(2, 2.0, 1.0, 0.5), M.superellipsoid(2, 1.0, 1.5, 0.8, 4.0)):
        a, b, c = (m.points[m.faces[:, i]] for i in range(3))
        n = np.cross(b - a, c - a)
        assert np.all(np.einsum("ij,ij->i", n, a + b + c) > 0)


def test_superellipsoid_surface():
    m = M.superellipsoid(3, 1.0, 2.0, 0.5, 4.0)
    s = np.sum(np.abs(m.points / np.array([1.0, 2.0, 0.5])) ** 4, axis=1)
    np.testing.assert_allclose(s, 1.0, atol=1e-13)


def test_nas_round_trip(tmp_path):
    m = M.ellipsoid(2, 1.3, 0.7, 0.4)
    p = M.write_nas(m, tmp_path / "b.nas")
    r = M.read_nas(p)
    np.testing.assert_array_equal(r.points, m.points)  # 17 significant digits: exact
    np.testing.assert_array_equal(r.faces, m.faces)
    text = p.read_text().splitlines()
    assert any(t.startswith("GRID*") for t in text) and any(t.startswith("CTRIA3") for t in text)


def test_mt19937_64_known_answer():
    g = M._MT19937_64(5489)
    assert g.next() == 14514284786278117030
    for _ in range(9998):
        g.next()
    assert g.next() == 9981545732273789042  # 10000th output (C++ [rand.predef])


def test_unit_disk_vector():
    x = M.unit_disk_vector(2000, 0)
    assert np.all(np.abs(x) <= 1.0)
    assert abs(np.mean(np.abs(x) ** 2) - 0.5) < 0.03
    np.testing.assert_array_equal(x, M.unit_disk_vector(2000, 0))


def test_uneven_body_set():
    """The 24-body set: order, kinds, sizes 3,840-61,440 unknowns, lossy
    materials in range, and the first body's draws pinned."""
    bodies = M.uneven_bodies(1)
    assert [b["kind"] for b in bodies] == ["icosphere"] * 8 + ["ellipsoid"] * 8 + ["superellipsoid"] * 8
    n = [3 * len(b["mesh"].face_ids) for b in bodies]  # 2N = 3 F for a closed surface
    assert min(n) == 3840 and max(n) == 61440
    for b in bodies:
        e = b["eps_r"]
        assert 1.5 <= e.real <= 6.0 and -0.05 * e.real <= e.imag <= 0.0
    first = bodies[0]
    assert first["params"]["sub"] == 3
    assert abs(first["eps_r"] - complex(4.041, -0.0981)) < 1e-3
    again = M.uneven_bodies(1)
    for a, b in zip(bodies, again):
        assert a["eps_r"] == b["eps_r"] and np.array_equal(a["mesh"].points, b["mesh"].points)


def test_learned_preconditioner_body_sets():
    """Training ellipsoids (seeded, semi-axes 0.5-2 lambda, eps_r 2-6,
    15,360 unknowns each) and the held-out 6 x 2 x 2 lambda ellipsoid
    (245,760 unknowns)."""
    lam = M.wavelength(3.0e8)
    bodies = M.training_ellipsoids(5)
    for b in bodies:
        assert 3 * len(b["mesh"].face_ids) == 15360
        assert all(0.5 * lam <= a <= 2.0 * lam for a in b["params"]["axes"])
        assert 2.0 <= b["eps_r"].real <= 6.0 and b["eps_r"].imag == 0.0
        p = b["mesh"].points / np.asarray(b["params"]["axes"])
        np.testing.assert_allclose(np.linalg.norm(p, axis=1), 1.0, atol=1e-12)
    again = M.training_ellipsoids(5)
    assert all(a["params"]["axes"] == b["params"]["axes"] and a["eps_r"] == b["eps_r"] for a, b in zip(bodies, again))
    assert [b["params"]["axes"] for b in M.training_ellipsoids(2, seed=3)] != [b["params"]["axes"] for b in bodies[:2]]
    h = M.held_out_ellipsoid(sub=3)
    assert h["eps_r"] == complex(3.0, -0.05)
    np.testing.assert_allclose(h["params"]["axes"], (3.0 * lam, lam, lam))
    assert 3 * len(M.held_out_ellipsoid(sub=4)["mesh"].face_ids) == 15360  # 245,760 at sub 6
