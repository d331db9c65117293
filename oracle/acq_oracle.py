"""ORACLE / TEST INFRASTRUCTURE ONLY — the checker, never the product.

numpy restatement of PowerGrid's acquisition sort and per-image gather:
  acqTracking::acqTracking        acqTracking.cpp:9-76
  getCompleteISMRMRDAcqData       processIsmrmrd.hpp:361-471
The Armadillo steps are written with numpy's column-major ("F") order:
Cube(nro, nc, numAcqs) filled slice by slice (:413-416, :451), permute with
D3tuple(1,3,2) (:455) and vectorise (:458-463).

Parity unpinned against the reference's own code: it needs the ISMRMRD/HDF5
and Armadillo libraries, which are absent, and the reference has no tests or
fixtures for it; the restatement follows the cited lines.
"""
from __future__ import annotations

import numpy as np


def acq_table(acqs, limits):
    """table[phase, echo, avg, rep, slice, par, shot] = acquisition number, -1 if none
    (memset -1, :52; a later acquisition with the same counters wins, :73)."""
    shots, pars, slices, reps, avgs, echos, phases = limits
    t = np.full((phases, echos, avgs, reps, slices, pars, shots), -1, np.int64)
    for i, a in enumerate(acqs):
        t[a.phase, a.contrast, a.average, a.repetition, a.slice, a.kspace_encode_step_2, a.kspace_encode_step_1] = i
    return t


def complete_acq_data(acqs, table, slice_, rep, avg, echo, phase):
    phases, echos, avgs, reps, slices, pars, shots = table.shape
    sel = [int(table[phase, echo, avg, rep, slice_, par, shot])
           for par in range(pars) for shot in range(shots)                       # :380-381, :406-407
           if table[phase, echo, avg, rep, slice_, par, shot] != -1]
    if not sel:
        e = np.zeros(0, np.float32)
        return np.zeros(0, np.complex64), e, e.copy(), e.copy(), e.copy()
    nc, nro = acqs[sel[0]].data.shape
    data_work = np.zeros((nro, nc, len(sel)), np.complex64, order="F")         # :388
    k_work = [np.zeros((nro, len(sel)), np.float32, order="F") for _ in range(4)]
    for cur, a in enumerate(sel):
        q = acqs[a]
        acq_work = np.zeros((nro, nc), np.complex64, order="F")
        for jj in range(nc):
            for kk in range(nro):
                acq_work[kk, jj] = q.data[jj, kk]                               # acq.data(kk, jj), :413-416
        for d in range(4):
            k_work[d][:, cur] = q.traj[:, d]                                     # acq.traj(d, ii), :444-448
        data_work[:, :, cur] = acq_work                                          # :451
    data = np.transpose(data_work, (0, 2, 1))                                    # permute(1,3,2), :455
    return (data.reshape(-1, order="F"),) + tuple(k.reshape(-1, order="F") for k in k_work)
