"""Ingest and output formats on the host side of the library: the acquisition
index and per-image gather (acqTracking.cpp:9-76, processIsmrmrd.hpp:361-471)
against the oracle's numpy restatement and a hand-built case, and the NIfTI
writer (processNIFTI.hpp:37-117) byte for byte against files written through
the reference's own nifti1.h (tests/golden/make_nifti_golden.py).  The device
gather is checked against the host gather."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def ing():
    from powergrid_b200 import build as B
    B.build()
    from powergrid_b200 import ingest
    return ingest


def _acqs(ing, rng, limits, nro=5, nc=3, skip=(), dup=(), td=4):
    """One acquisition per counter tuple (shot fastest), minus `skip`, plus
    repeated counters in `dup` (appended later: they replace the first)."""
    shots, pars, slices, reps = limits[:4]
    out = []
    for rep in range(reps):
        for sl in range(slices):
            for par in range(pars):
                for shot in range(shots):
                    if (shot, par, sl, rep) in skip:
                        continue
                    out.append((shot, par, sl, rep))
    out += list(dup)
    acqs = []
    for (shot, par, sl, rep) in out:
        data = (rng.standard_normal((nc, nro)) + 1j * rng.standard_normal((nc, nro))).astype(np.complex64)
        traj = rng.standard_normal((nro, td)).astype(np.float32)
        acqs.append(ing.Acquisition(shot, par, sl, rep, 0, 0, 0, data, traj))
    return acqs


def test_gather_matches_oracle(ing):
    import acq_oracle as AO
    rng = np.random.default_rng(1)
    limits = (3, 2, 2, 2, 1, 1, 1)
    acqs = _acqs(ing, rng, limits, skip={(1, 0, 0, 0), (2, 1, 1, 1)}, dup=[(0, 1, 1, 0), (2, 0, 0, 1)])
    T = ing.acqTracking(acqs, limits)
    table = AO.acq_table(acqs, limits)
    for shot in range(3):
        for par in range(2):
            for sl in range(2):
                for rep in range(2):
                    assert T.acqArray(shot, par, sl, rep, 0, 0, 0) == table[0, 0, 0, rep, sl, par, shot]
    for sl in range(2):
        for rep in range(2):
            got = ing.getCompleteISMRMRDAcqData(T, sl, rep, 0, 0, 0)
            want = AO.complete_acq_data(acqs, table, sl, rep, 0, 0, 0)
            for g, w in zip(got, want):
                assert g.dtype == w.dtype and np.array_equal(g, w)


def test_gather_hand_built_layout(ing):
    """Two shots of one partition, 2 coils x 3 samples: data is coil-major over
    (acquisition, sample), trajectories acquisition-major."""
    d0 = np.array([[1, 2, 3], [4, 5, 6]], np.complex64)            # [coil][sample]
    d1 = np.array([[7, 8, 9], [10, 11, 12]], np.complex64)
    t0 = np.arange(12, dtype=np.float32).reshape(3, 4)             # [sample][kx, ky, kz, t]
    t1 = 100 + np.arange(12, dtype=np.float32).reshape(3, 4)
    acqs = [ing.Acquisition(1, 0, 0, 0, 0, 0, 0, d1, t1), ing.Acquisition(0, 0, 0, 0, 0, 0, 0, d0, t0)]
    T = ing.acqTracking(acqs, (2, 1, 1, 1, 1, 1, 1))
    data, kx, ky, kz, t = ing.getCompleteISMRMRDAcqData(T, 0, 0, 0, 0, 0)
    assert np.array_equal(data, np.array([1, 2, 3, 7, 8, 9, 4, 5, 6, 10, 11, 12], np.complex64))
    assert np.array_equal(kx, [0, 4, 8, 100, 104, 108]) and np.array_equal(t, [3, 7, 11, 103, 107, 111])
    assert np.array_equal(ky, [1, 5, 9, 101, 105, 109]) and np.array_equal(kz, [2, 6, 10, 102, 106, 110])


def test_gather_invalid_inputs(ing):
    from powergrid_b200._lib import PGError
    rng = np.random.default_rng(2)
    acqs = _acqs(ing, rng, (2, 1, 1, 1, 1, 1, 1))
    with pytest.raises(PGError, match="outside the encoding limits"):
        ing.acqTracking(acqs, (1, 1, 1, 1, 1, 1, 1))
    with pytest.raises(PGError, match="limit is zero"):
        ing.acqTracking(acqs, (2, 0, 1, 1, 1, 1, 1))
    # a later acquisition with the same counters replaces the earlier one
    T = ing.acqTracking(acqs + [acqs[1]], (2, 1, 1, 1, 1, 1, 1))
    assert T.acqArray(1, 0, 0, 0, 0, 0, 0) == 2
    with pytest.raises(PGError, match="outside the encoding limits"):
        ing.getCompleteISMRMRDAcqData(T, 1, 0, 0, 0, 0)
    # an image whose acquisitions differ in sample count
    short = ing.Acquisition(0, 0, 0, 0, 0, 0, 0, acqs[0].data[:, :4], acqs[0].traj[:4])
    T2 = ing.acqTracking([short, acqs[1]], (2, 1, 1, 1, 1, 1, 1))
    with pytest.raises(PGError, match="samples x"):
        ing.getCompleteISMRMRDAcqData(T2, 0, 0, 0, 0, 0)


def test_nifti_mag_phs_matches_reference_header(ing, tmp_path):
    d = np.load(os.path.join(HERE, "golden", "nifti_magphs.npz"))
    dims = [int(v) for v in d["dims"]]
    base = str(tmp_path / "img")
    ing.writeNiftiMagPhsImage(base, d["z"], *dims)
    assert np.array_equal(np.fromfile(base + "_mag.nii", np.uint8), d["mag_file"])
    assert np.array_equal(np.fromfile(base + "_phs.nii", np.uint8), d["phs_file"])
    # the real-image writer reproduces the magnitude file from its voxels
    mag = np.frombuffer(d["mag_file"][352:].tobytes(), np.float32)
    ing.writeNiftiRealImage(str(tmp_path / "real"), mag, *dims)
    assert np.array_equal(np.fromfile(str(tmp_path / "real.nii"), np.uint8), d["mag_file"])


def test_nifti_invalid(ing, tmp_path):
    from powergrid_b200._lib import PGError
    with pytest.raises(PGError, match="dimension"):
        ing.writeNiftiRealImage(str(tmp_path / "a"), np.zeros(4, np.float32), 2, 2, 0)
    with pytest.raises(PGError, match="cannot open"):
        ing.writeNiftiRealImage(str(tmp_path / "missing" / "a"), np.zeros(4, np.float32), 2, 2, 1)
    with pytest.raises(ValueError):
        ing.writeNiftiMagPhsImage(str(tmp_path / "b"), np.zeros(3, np.complex64), 2, 2, 1)


@pytest.mark.gpu
def test_device_gather_matches_host(ing):
    """The GPU permutation equals the host gather, with acquisitions whose
    trajectories carry extra rows (the strided upload)."""
    import powergrid_b200 as pg
    pg.init(0)
    rng = np.random.default_rng(3)
    limits = (4, 3, 1, 2, 1, 1, 1)
    acqs = _acqs(ing, rng, limits, nro=257, nc=5, skip={(3, 2, 0, 1)}, dup=[(1, 1, 0, 0)])
    acqs[4] = ing.Acquisition(acqs[4].kspace_encode_step_1, acqs[4].kspace_encode_step_2, 0,
                              acqs[4].repetition, 0, 0, 0, acqs[4].data,
                              np.concatenate([acqs[4].traj, np.ones((257, 2), np.float32)], axis=1))
    T = ing.acqTracking(acqs, limits)
    for rep in range(2):
        host = ing.getCompleteISMRMRDAcqData(T, 0, rep, 0, 0, 0)
        dev = ing.getCompleteISMRMRDAcqData(T, 0, rep, 0, 0, 0, device=True)
        for h, g in zip(host, dev):
            assert np.array_equal(h, g.cpu().numpy())
