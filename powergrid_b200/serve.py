"""Python front end of the request server (pg_server_* in the C ABI).

    srv = Server(hbm_budget_bytes=64 << 30, max_inflight=8)
    ticket = srv.submit(req)            # req: ReconRequest (host numpy arrays)
    image, stats = srv.wait(ticket)     # image: n_slices x (nx*ny*nz) complex64

    # the ISMRMRD driver's image loop over an acquisition index
    ticket = srv.submit_acquisitions(acq_track, nx, ny, nz, field_map, sense_map, niter=10, beta=...)
    images, stats = srv.wait(ticket)    # images: (slice, phase, contrast, average, repetition) x N

A request's slices (or an acquisition request's images of one trajectory)
are batched into jobs of as many as fit the HBM budget; jobs are admitted
FIFO while a worker slot is free and the summed device footprint stays within
the budget.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib
from ._lib import P, U64, Request, RequestStats, ServerConfig, check


@dataclasses.dataclass
class _Shape:
    n_slices: int
    nimg: int


@dataclasses.dataclass
class ReconRequest:
    """SENSE<TimeSegmentation<Gnufft>> + QuadPenalty reconstruction of n_slices images."""
    nx: int
    ny: int
    nz: int
    nc: int
    L: int
    niter: int
    beta: float
    kx: np.ndarray
    ky: np.ndarray
    kz: np.ndarray
    t: np.ndarray
    field_map: np.ndarray      # n_slices * N, rad/s
    sense_map: np.ndarray      # complex64, n_slices * N * nc
    data: np.ndarray           # complex64, n_slices * M * nc
    n_slices: int = 1

    @property
    def n_samples(self) -> int:
        return int(self.kx.size)

    @property
    def nimg(self) -> int:
        return self.nx * self.ny * self.nz


class Server:
    def __init__(self, hbm_budget_bytes: int, max_inflight: int = 8):
        cfg = ServerConfig(int(hbm_budget_bytes), int(max_inflight), 0)
        h = P()
        check(_lib.load().pg_server_create(C.byref(h), C.byref(cfg)))
        self._h = h
        self._live = {}

    @staticmethod
    def _struct(r: ReconRequest, keep: list) -> Request:
        def f32(a):
            a = np.ascontiguousarray(a, dtype=np.float32)
            keep.append(a)
            return a.ctypes.data_as(P)

        def c64(a):
            a = np.ascontiguousarray(a, dtype=np.complex64)
            keep.append(a)
            return a.ctypes.data_as(P)

        out = np.zeros(r.n_slices * r.nimg, dtype=np.complex64)
        keep.append(out)
        return Request(r.nx, r.ny, r.nz, r.n_slices, r.nc, r.n_samples, r.L, r.niter, r.beta, f32(r.kx), f32(r.ky),
                       f32(r.kz), f32(r.t), f32(r.field_map), c64(r.sense_map), c64(r.data),
                       out.ctypes.data_as(P)), out

    @staticmethod
    def footprint(r: ReconRequest) -> int:
        keep = []
        s, _ = Server._struct(r, keep)
        return int(_lib.load().pg_request_footprint(C.byref(s)))

    def submit(self, r: ReconRequest) -> int:
        keep = []
        s, out = self._struct(r, keep)
        t = U64()
        check(_lib.load().pg_submit(self._h, C.byref(s), C.byref(t)))
        self._live[t.value] = (keep, out, r)
        return int(t.value)

    def submit_acquisitions(self, acq_track, nx: int, ny: int, nz: int, field_map, sense_map, L: int = 0,
                            niter: int = 10, beta: float = 0.0) -> int:
        """Every image of an acqTracking index (PowerGridIsmrmrd.cpp:191-264):
        slice outermost, then phase, contrast, average, repetition; field_map
        is slices x N and sense_map slices x nc x N, as the ISMRMRD file holds
        them.  L = 0 takes the driver's default ceil((max t - min t) / 2 ms)."""
        keep = [acq_track]
        fm = np.ascontiguousarray(field_map, dtype=np.float32)
        sm = np.ascontiguousarray(sense_map, dtype=np.complex64)
        nimg = (acq_track.NSliceMax * acq_track.NPhaseMax * acq_track.NEchoMax * acq_track.NAvgMax *
                acq_track.NRepMax)
        out = np.zeros(nimg * nx * ny * nz, dtype=np.complex64)
        keep += [fm, sm, out]
        q = _lib.AcqRequest(nx, ny, nz, L, niter, beta, fm.ctypes.data_as(P), sm.ctypes.data_as(P),
                            out.ctypes.data_as(P))
        t = U64()
        check(_lib.load().pg_submit_acquisitions(self._h, acq_track._h, C.byref(q), C.byref(t)))
        shape = _Shape(nimg, nx * ny * nz)
        self._live[t.value] = (keep, out, shape)
        return int(t.value)

    def poll(self, ticket: int):
        st = RequestStats()
        rc = _lib.load().pg_poll(self._h, ticket, C.byref(st))
        if rc == _lib.PG_NOT_READY:
            return None
        check(rc)
        return self._finish(ticket, st)

    def wait(self, ticket: int):
        st = RequestStats()
        check(_lib.load().pg_wait(self._h, ticket, C.byref(st)))
        return self._finish(ticket, st)

    def cancel(self, ticket: int) -> None:
        check(_lib.load().pg_cancel(self._h, ticket))

    def _finish(self, ticket, st):
        keep, out, r = self._live[ticket]
        stats = {"t_submit_ms": st.t_submit_ms, "t_start_ms": st.t_start_ms, "t_done_ms": st.t_done_ms,
                 "iters_done": int(st.iters_done), "bytes_resident": int(st.bytes_resident),
                 "status": _lib.STATUS.get(st.status, st.status), "setup_ms": st.setup_ms, "solve_ms": st.solve_ms,
                 "jobs": int(st.jobs), "error": st.error.decode(errors="replace")}
        return out.reshape(r.n_slices, r.nimg), stats

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().pg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
