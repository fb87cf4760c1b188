"""Many incidences at once: the batched excitation (mlfma_rhs_pmchwt_batch_device)
and far-field entry points (bistatic mlfma_rcs_pmchwt_batch_device, monostatic
mlfma_rcs_pmchwt_mono_device) against the one-incidence entry points, which
the parity suite checks against the reference (RHS::computeV_PMCHWT,
Code/Vm.h:150-203; RCSUtils::calculateRCS_PMCHWT, Code/RCS.h:116-192).
Counts cross the launch chunks (128 incidences, 256 angles) and the tiles
(8 incidences, 4 solutions) with ragged ends."""
import numpy as np
import pytest

from conftest import FREQ, needs_lib, needs_oracle, rel

pytestmark = [pytest.mark.gpu, needs_lib]


@pytest.fixture(scope="module")
def op():
    from mlfma_pmchwt_b200 import MLFMM
    from mlfma_pmchwt_b200 import mesh as M
    o = MLFMM(M.icosphere(3, 1.0), freq=FREQ, eps_r=complex(2.5, -0.1), leaf_coeff=0.25, device=0)
    yield o
    o.close()


def test_batched_excitation_equals_single_incidences(op):
    import torch
    from mlfma_pmchwt_b200 import plane_wave
    R = 131
    th = np.linspace(0.0, 180.0, R)
    ph = np.linspace(0.0, 90.0, R)
    inc = [plane_wave(90.0 * (i % 2), th[i], ph[i]) for i in range(R)]
    V = torch.empty((R, op.n), dtype=torch.complex128, device="cuda")
    op.compute_v_pmchwt_batch_device(inc, V.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    got = V.cpu().numpy()
    for i in range(R):
        want = op.compute_v_pmchwt(*inc[i])
        assert rel(got[i], want) < 1e-14, i


def test_batched_far_fields_equal_single_solutions(op):
    import torch
    from mlfma_pmchwt_b200 import mesh as M, rcs_db
    R = 6
    I = np.stack([M.unit_disk_vector(op.n, 20 + r) for r in range(R)])
    Id = torch.from_numpy(I).cuda()
    th = np.arange(0.0, 180.01, 0.5)  # 361 angles: two launch chunks
    ph = np.full_like(th, 30.0)
    F = torch.empty((R, len(th), 3), dtype=torch.complex128, device="cuda")
    op.calculate_rcs_batch_device(R, Id.data_ptr(), th, ph, F.data_ptr(), torch.cuda.current_stream().cuda_stream)
    # monostatic: solution r at its own angle
    tm, pm = np.linspace(5.0, 175.0, R), np.linspace(0.0, 300.0, R)
    Fm = torch.empty((R, 3), dtype=torch.complex128, device="cuda")
    op.calculate_rcs_mono_device(R, Id.data_ptr(), tm, pm, Fm.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    got, gotm = F.cpu().numpy(), Fm.cpu().numpy()
    for r in range(R):
        want, db = op.calculate_rcs_pmchwt(I[r], th, ph)
        np.testing.assert_allclose(got[r], want, rtol=0, atol=1e-12 * np.abs(want).max())
        np.testing.assert_allclose(rcs_db(th, ph, got[r]), db, rtol=0, atol=1e-9)
        wm, _ = op.calculate_rcs_pmchwt(I[r], tm[r], pm[r])
        np.testing.assert_allclose(gotm[r], wm[0], rtol=0, atol=1e-12 * np.abs(wm).max())


@needs_oracle
def test_batched_excitation_and_rcs_against_the_reference(op, tmp_path):
    """The reference's excitation and RCS (its own code, compiled) for a few
    incidences of the mono-static loop (Code/RCS.h:436-494)."""
    import torch
    from mlfma_pmchwt_b200 import mesh as M, plane_wave, rcs_db
    from oracle import oracle as O
    m = M.icosphere(3, 1.0)
    nas = M.write_nas(m, tmp_path / "s3.nas")
    ref = O.RefOperator(nas, freq=FREQ, eps_r=complex(2.5, -0.1), leaf_coeff=0.25)
    angles = [(0.0, 0.0, 0.0), (90.0, 45.0, 0.0), (0.0, 120.0, 60.0)]
    inc = [plane_wave(*a) for a in angles]
    stream = torch.cuda.current_stream().cuda_stream
    V = torch.empty((len(inc), op.n), dtype=torch.complex128, device="cuda")
    op.compute_v_pmchwt_batch_device(inc, V.data_ptr(), stream)
    torch.cuda.synchronize()
    got = V.cpu().numpy()
    I = np.stack([M.unit_disk_vector(op.n, 40 + i) for i in range(len(inc))])
    th = np.array([a[1] for a in angles])
    ph = np.array([a[2] for a in angles])
    Fm = torch.empty((len(inc), 3), dtype=torch.complex128, device="cuda")
    Id = torch.from_numpy(I).cuda()
    op.calculate_rcs_mono_device(len(inc), Id.data_ptr(), th, ph, Fm.data_ptr(), stream)
    torch.cuda.synchronize()
    fm = Fm.cpu().numpy()
    for i, a in enumerate(angles):
        vr = ref.rhs(*a)[0]
        assert rel(got[i], vr) < 1e-13
        fr, dbr = ref.rcs(I[i], a[0], th[i], ph[i])
        assert rel(fm[i], fr) < 1e-12
        assert np.max(np.abs(rcs_db(th[i], ph[i], fm[i:i + 1])[0] - dbr)) < 0.01
    ref.close()
