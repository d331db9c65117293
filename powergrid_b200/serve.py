"""Python front end of the request server (pg_server_* in the C ABI).

    srv = Server(hbm_budget_bytes=64 << 30, max_inflight=8)
    ticket = srv.submit(req)            # req: ReconRequest (host numpy arrays)
    image, stats = srv.wait(ticket)     # image: n_slices x (nx*ny*nz) complex64

Each slice of a request runs as its own job; jobs are admitted FIFO while a
worker slot is free and the summed device footprint stays within the budget.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib
from ._lib import P, U64, Request, RequestStats, ServerConfig, check


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
                 "error": st.error.decode(errors="replace")}
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
