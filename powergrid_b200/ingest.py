"""Ingest and output formats: the acquisition index and per-image gather that
PowerGrid's ISMRMRD readers perform (acqTracking.cpp:9-76,
processIsmrmrd.hpp:361-471), over an in-memory acquisition list instead of an
HDF5 file, and the NIfTI magnitude/phase writer (processNIFTI.hpp:37-117).

The work is done by libpowergrid_b200 (pg_acq_*, pg_write_nifti_*).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import P, U64, check

__all__ = ["Acquisition", "acqTracking", "getCompleteISMRMRDAcqData", "writeNiftiRealImage",
           "writeNiftiMagPhsImage"]


@dataclass
class Acquisition:
    """One ISMRMRD acquisition: its encoding counters, samples as
    acq.data(sample, channel) = data[channel, sample] and trajectory as
    acq.traj(dim, sample) = traj[sample, dim] (kx, ky, kz, t first)."""
    kspace_encode_step_1: int
    kspace_encode_step_2: int
    slice: int
    repetition: int
    average: int
    contrast: int
    phase: int
    data: np.ndarray
    traj: np.ndarray

    def __post_init__(self):
        self.data = np.ascontiguousarray(self.data, dtype=np.complex64)
        self.traj = np.ascontiguousarray(self.traj, dtype=np.float32)
        if self.data.ndim != 2 or self.traj.ndim != 2 or self.traj.shape[0] != self.data.shape[1]:
            raise ValueError("Acquisition: data is (channels, samples), traj is (samples, dims)")


class acqTracking:
    """acqTracking (acqTracking.h:14): acquisition numbers by (shot, partition,
    slice, repetition, average, contrast, phase); limits are the encoding
    limits' maximum + 1 in that order."""

    def __init__(self, acquisitions, limits):
        self.acqs = list(acquisitions)
        (self.NShotMax, self.NParMax, self.NSliceMax, self.NRepMax, self.NAvgMax, self.NEchoMax,
         self.NPhaseMax) = (int(v) for v in limits)
        arr = (_lib.Acquisition * max(1, len(self.acqs)))()
        for i, a in enumerate(self.acqs):
            arr[i] = _lib.Acquisition(a.kspace_encode_step_1, a.kspace_encode_step_2, a.slice, a.repetition,
                                      a.average, a.contrast, a.phase, a.data.shape[1], a.data.shape[0],
                                      a.traj.shape[1], a.data.ctypes.data, a.traj.ctypes.data)
        self._arr = arr
        lim = _lib.EncodingLimits(*(int(v) for v in limits))
        h = P()
        check(_lib.load().pg_acq_index_create(C.byref(h), arr, len(self.acqs), C.byref(lim)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            _lib.load().pg_acq_index_destroy(self._h)
            self._h = None

    def acqArray(self, shot, par, slice_, rep, avg, echo, phase) -> int:
        out = C.c_int64()
        check(_lib.load().pg_acq_index_lookup(self._h, shot, par, slice_, rep, avg, echo, phase, C.byref(out)))
        return int(out.value)


def getCompleteISMRMRDAcqData(acqTrack: acqTracking, NSlice, NRep, NAvg, NEcho, NPhase, device=False):
    """(data, kx, ky, kz, tvec) of one image (processIsmrmrd.hpp:361-471): data
    coil-major [c][acquisition][sample]; trajectories [acquisition][sample].
    device=True returns torch CUDA tensors gathered on the GPU."""
    L = _lib.load()
    na, nro, nc = U64(), U64(), U64()
    idx = (int(NSlice), int(NRep), int(NAvg), int(NEcho), int(NPhase))
    check(L.pg_acq_gather_size(acqTrack._h, *idx, C.byref(na), C.byref(nro), C.byref(nc)))
    n = na.value * nro.value
    if device:
        import torch
        data = torch.empty(n * nc.value, dtype=torch.complex64, device="cuda")
        k = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(4)]
        check(L.pg_acq_gather_device(acqTrack._h, *idx, P(data.data_ptr()), *[P(v.data_ptr()) for v in k],
                                     P(torch.cuda.current_stream().cuda_stream)))
        return (data, *k)
    data = np.empty(n * nc.value, np.complex64)
    k = [np.empty(n, np.float32) for _ in range(4)]
    check(L.pg_acq_gather(acqTrack._h, *idx, data.ctypes.data, *[v.ctypes.data for v in k]))
    return (data, *k)


def writeNiftiRealImage(filename, imageData, Nx, Ny, Nz=1, Nslab=1, N_TR=1):
    """writeNiftiRealImage (processNIFTI.hpp:37-99): "<filename>.nii"."""
    img = np.ascontiguousarray(imageData, dtype=np.float32)
    if img.size < Nx * Ny * Nz * Nslab * N_TR:
        raise ValueError("writeNiftiRealImage: image shorter than its dimensions")
    check(_lib.load().pg_write_nifti_real(str(filename).encode(), img.ctypes.data, Nx, Ny, Nz, Nslab, N_TR))


def writeNiftiMagPhsImage(filename, imageData, Nx, Ny, Nz, Nslab=1, N_TR=1):
    """writeNiftiMagPhsImage (processNIFTI.hpp:103-117): "<filename>_mag.nii" and "_phs.nii"."""
    img = np.ascontiguousarray(imageData, dtype=np.complex64)
    if img.size < Nx * Ny * Nz * Nslab * N_TR:
        raise ValueError("writeNiftiMagPhsImage: image shorter than its dimensions")
    check(_lib.load().pg_write_nifti_mag_phs(str(filename).encode(), img.ctypes.data, Nx, Ny, Nz, Nslab, N_TR))
