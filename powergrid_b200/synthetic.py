"""Seeded synthetic inputs with the shapes of PowerGrid's reconstruction workloads.

No ISMRMRD files exist here, so trajectories, field maps, coil maps, shot
phase maps and images are generated from a counter-based RNG (splitmix64),
bit-identical on every machine.  Conventions follow the reference:

* k-space in cycles/FOV within [-N/2, N/2) (the range Gnufft checks,
  Gnufft.cpp:68-76);
* field maps in rad/s (TimeSegmentation.h:56), times in seconds;
* image vectors y-fastest: index = y + Ny*x + Nx*Ny*z (reconSolve.cpp:40-53);
* coil data coil-major [c][sample] (SENSE.cpp:66, 86); multishot data
  [c][s][sample] (pcSenseTimeSeg.cpp:136-147).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _mix(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


class Rng:
    """splitmix64 stream: value i = mix(key + (i + 1) * golden)."""

    def __init__(self, seed: int, stream: int = 0):
        k = np.array([(seed * 0x100000001B3 + stream * 0x9E37) & 0xFFFFFFFFFFFFFFFF], dtype=np.uint64)
        self.key = _mix(k)[0]
        self.counter = 0

    def bits(self, n: int) -> np.ndarray:
        i = np.arange(self.counter + 1, self.counter + 1 + n, dtype=np.uint64)
        self.counter += n
        with np.errstate(over="ignore"):
            return _mix(self.key + i * _GOLDEN)

    def uniform(self, n: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
        u = (self.bits(n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
        return lo + (hi - lo) * u

    def normal(self, n: int) -> np.ndarray:
        u1 = self.uniform(n)
        u2 = self.uniform(n)
        return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * math.pi * u2)


def image_coords(nx: int, ny: int, nz: int):
    """initImageSpaceCoords (reconSolve.cpp:30-54): (i - N/2)/N per axis, y fastest."""
    z, x, y = np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij")
    ix = ((x.astype(np.float32) - np.float32(nx) / 2.0) / np.float32(nx)).astype(np.float32).ravel()
    iy = ((y.astype(np.float32) - np.float32(ny) / 2.0) / np.float32(ny)).astype(np.float32).ravel()
    iz = ((z.astype(np.float32) - np.float32(nz) / 2.0) / np.float32(nz)).astype(np.float32).ravel()
    return ix, iy, iz


def spiral(n: int, interleaves: int, per_interleave: int, t_read: float, which=None, turns=None):
    """Variable-density Archimedean-like spiral: |k| = kmax*tau^1.5, theta = 2pi(turns*tau + s/S).

    Returns kx, ky, t (float32) for the interleaves listed in `which` (default all),
    interleave-major.
    """
    kmax = n / 2.0 * (1.0 - 1e-3)
    if turns is None:
        turns = max(1.0, n / (2.0 * interleaves))
    which = range(interleaves) if which is None else which
    tau = np.arange(per_interleave, dtype=np.float64) / per_interleave
    kx, ky, tt = [], [], []
    for s in which:
        r = kmax * tau ** 1.5
        th = 2.0 * math.pi * (turns * tau + s / interleaves)
        kx.append(r * np.cos(th))
        ky.append(r * np.sin(th))
        tt.append(tau * t_read)
    return (np.concatenate(kx).astype(np.float32), np.concatenate(ky).astype(np.float32),
            np.concatenate(tt).astype(np.float32))


def field_map(rng: Rng, nx: int, ny: int, nz: int, amp_hz: float) -> np.ndarray:
    """Sum of 3 Gaussian bumps (amplitude U[-A,A] Hz), clipped to +-A, in rad/s."""
    ix, iy, iz = image_coords(nx, ny, nz)
    f = np.zeros(ix.shape, dtype=np.float64)
    if amp_hz == 0:
        return f.astype(np.float32)
    for _ in range(3):
        a, cx, cy, cz, sg = rng.uniform(5)
        a = (2 * a - 1) * amp_hz
        cx, cy, cz = cx - 0.5, cy - 0.5, (cz - 0.5) if nz > 1 else 0.0
        sg = 0.1 + 0.2 * sg
        d2 = (ix - cx) ** 2 + (iy - cy) ** 2 + ((iz - cz) ** 2 if nz > 1 else 0.0)
        f += a * np.exp(-d2 / (2 * sg * sg))
    f = np.clip(f, -amp_hz, amp_hz)
    return (2.0 * math.pi * f).astype(np.float32)


def coil_maps(rng: Rng, nx: int, ny: int, nz: int, nc: int) -> np.ndarray:
    """Gaussian sensitivities centred on a ring of radius 0.6 FOV, constant phase per coil.

    Returns complex64 of length N*nc, coil-major (SENSE.cpp:40 reshapes it to N x nc).
    """
    ix, iy, iz = image_coords(nx, ny, nz)
    out = np.empty((nc, ix.size), dtype=np.complex64)
    ph = rng.uniform(nc, -math.pi, math.pi)
    for c in range(nc):
        ang = 2 * math.pi * c / nc
        cx, cy = 0.6 * math.cos(ang), 0.6 * math.sin(ang)
        cz = (0.25 if c % 2 else -0.25) if nz > 1 else 0.0
        d2 = (ix - cx) ** 2 + (iy - cy) ** 2 + ((iz - cz) ** 2 if nz > 1 else 0.0)
        mag = np.exp(-d2 / (2 * 0.4 * 0.4))
        out[c] = (mag * np.exp(1j * ph[c])).astype(np.complex64)
    return out.ravel()


def shot_phase_maps(rng: Rng, nx: int, ny: int, nz: int, ns: int) -> np.ndarray:
    """Per-shot linear + constant phase a_s + b_s . r (rad), a, b ~ U[-pi, pi] per FOV; shot-major."""
    ix, iy, iz = image_coords(nx, ny, nz)
    out = np.empty((ns, ix.size), dtype=np.float32)
    for s in range(ns):
        a, bx, by, bz = rng.uniform(4, -math.pi, math.pi)
        out[s] = (a + bx * ix + by * iy + (bz * iz if nz > 1 else 0.0)).astype(np.float32)
    return out.ravel()


def image(rng: Rng, n: int) -> np.ndarray:
    re = rng.normal(n)
    im = rng.normal(n)
    return (re + 1j * im).astype(np.complex64)


@dataclasses.dataclass
class Problem:
    """One reconstruction problem: geometry, trajectory, maps and a ground-truth image."""
    name: str
    nx: int
    ny: int
    nz: int
    kx: np.ndarray
    ky: np.ndarray
    kz: np.ndarray
    t: np.ndarray
    fm: np.ndarray           # rad/s, length N
    smap: np.ndarray         # complex64, N*nc, coil-major
    nc: int
    L: int
    x_true: np.ndarray
    op: str = "sense_ts_nufft"   # sense_ts_nufft | sense_nufft | sense_gdft | pcsense_ts
    shots: int = 1
    pmap: np.ndarray | None = None
    penalty: str = "quad"
    beta: float = 1e-3
    delta: float = 1.0
    dims2pen: int = 3
    niter: int = 10

    @property
    def nimg(self) -> int:
        return self.nx * self.ny * self.nz


def config1(seed: int = 1) -> Problem:
    """2-D single-coil Gnufft, 64x64, 8-interleave variable-density spiral, 4096 samples."""
    rng = Rng(seed)
    n = 64
    kx, ky, t = spiral(n, 8, 512, 5e-3)
    kz = np.zeros_like(kx)
    return Problem("cfg1", n, n, 1, kx, ky, kz, t, np.zeros(n * n, np.float32),
                   np.ones(n * n, np.complex64), 1, 1, image(rng, n * n), op="sense_nufft",
                   beta=1e-3, niter=10)


def config2(seed: int = 2, n: int = 128, interleaves: int = 16, per: int = 8192, nc: int = 4, L: int = 8) -> Problem:
    """2-D TimeSegmentation<Gnufft> SENSE: 128x128, L=8 Hanning, 4 coils, 16x8192 spiral, 20 ms."""
    rng = Rng(seed)
    kx, ky, t = spiral(n, interleaves, per, 20e-3)
    kz = np.zeros_like(kx)
    fm = field_map(rng, n, n, 1, 100.0)
    sm = coil_maps(rng, n, n, 1, nc)
    return Problem("cfg2", n, n, 1, kx, ky, kz, t, fm, sm, nc, L, image(rng, n * n), beta=1e-3, niter=20)


def stack_of_spirals(n: int, nz: int, interleaves: int, per: int, t_read: float, which=None):
    kx, ky, tt = spiral(n, interleaves, per, t_read, which=which)
    reps = kx.size
    kxs, kys, kzs, ts = [], [], [], []
    for p in range(nz):
        kxs.append(kx)
        kys.append(ky)
        kzs.append(np.full(reps, p - nz / 2.0, np.float32))
        ts.append(tt)
    return (np.concatenate(kxs), np.concatenate(kys), np.concatenate(kzs).astype(np.float32), np.concatenate(ts))


def config3(seed: int = 3, n: int = 64, nz: int = 32, per: int = 4096, nc: int = 8) -> Problem:
    """3-D exact Gdft SENSE: 64x64x32, 8 coils, 32-partition stack of spirals (131072 samples), 0-25 ms."""
    rng = Rng(seed)
    kx, ky, kz, t = stack_of_spirals(n, nz, 1, per, 25e-3)
    fm = field_map(rng, n, n, nz, 150.0)
    sm = coil_maps(rng, n, n, nz, nc)
    return Problem("cfg3", n, n, nz, kx, ky, kz, t, fm, sm, nc, 1, image(rng, n * n * nz), op="sense_gdft",
                   niter=10)


def config5(seed: int = 5, n: int = 128, nz: int = 64, shots: int = 16, per: int = 2048, nc: int = 32,
            L: int = 12, t_read: float = 10e-3) -> Problem:
    """3-D multishot pcSenseTimeSeg: 128x128x64, 16 shots (one interleave of a 16-interleave
    stack of spirals over 64 partitions each), 32 coils, L=12, TV penalty."""
    rng = Rng(seed)
    kxs, kys, kzs, ts = [], [], [], []
    for s in range(shots):
        kx, ky, kz, t = stack_of_spirals(n, nz, shots, per, t_read, which=[s])
        kxs.append(kx); kys.append(ky); kzs.append(kz); ts.append(t)
    fm = field_map(rng, n, n, nz, 200.0)
    sm = coil_maps(rng, n, n, nz, nc)
    pm = shot_phase_maps(rng, n, n, nz, shots)
    return Problem("cfg5", n, n, nz, np.concatenate(kxs), np.concatenate(kys), np.concatenate(kzs),
                   np.concatenate(ts), fm, sm, nc, L, image(rng, n * n * nz), op="pcsense_ts", shots=shots,
                   pmap=pm, penalty="tv", beta=1e-3, delta=0.1, niter=30)


@dataclasses.dataclass
class StreamItem:
    """One request of a serving stream (config 4) before its data are formed."""
    arrival_s: float
    nx: int
    ny: int
    nz: int
    n_slices: int
    nc: int
    L: int
    niter: int
    beta: float
    kx: np.ndarray
    ky: np.ndarray
    kz: np.ndarray
    t: np.ndarray
    fm: np.ndarray        # N, rad/s (shared by the request's slices)
    smap: np.ndarray      # complex64 N*nc (shared by the request's slices)
    x_true: np.ndarray    # complex64 N

    @property
    def nimg(self) -> int:
        return self.nx * self.ny * self.nz


def serving_stream(seed: int = 4, n_requests: int = 16, rate_hz: float = 4.0, small: bool = False,
                   niter: int = 10):
    """Seeded config-4 stream: Poisson arrivals at rate_hz; per request an
    in-plane matrix 64-256 (square), 1-32 slices (2-D) or a 3-D volume, 4-32
    coils, 8k-200k samples, L = 4-12.  `small=True` shrinks every range (for
    tests).  Slices of one request share maps and image content."""
    rng = Rng(seed, 77)
    items = []
    t_arr = 0.0
    for _ in range(n_requests):
        t_arr += float(-np.log1p(-rng.uniform(1)[0]) / rate_hz)
        u = rng.uniform(8)
        three_d = (u[0] < 0.25) and not small
        if small:
            n = int(32 + 16 * int(u[1] * 2))            # 32 or 48
            nz = 1
            slices = 1 + int(u[2] * 2)
            nc = 2 + int(u[3] * 3)
            M = 2048 + int(u[4] * 6144)
            L = 3 + int(u[5] * 2)
        elif three_d:
            n = int(64 + 32 * int(u[1] * 3))            # 64, 96, 128
            nz = 16 * (1 + int(u[2] * 2))               # 16 or 32
            slices = 1
            nc = 4 + int(u[3] * 29)
            M = 8192 + int(u[4] * (200000 - 8192))
            L = 4 + int(u[5] * 9)
        else:
            n = int(64 + 16 * int(u[1] * 13))           # 64 .. 256
            nz = 1
            slices = 1 + int(u[2] * 32)
            nc = 4 + int(u[3] * 29)
            M = 8192 + int(u[4] * (200000 - 8192))
            L = 4 + int(u[5] * 9)
        t_read = 5e-3 + 20e-3 * float(u[6])
        amp = 50.0 + 150.0 * float(u[7])
        if nz == 1:
            inter = max(1, int(round(M / 8192)))
            per = max(256, M // inter)
            kx, ky, t = spiral(n, inter, per, t_read)
            kz = np.zeros_like(kx)
        else:
            per = max(256, M // nz)
            kx, ky, kz, t = stack_of_spirals(n, nz, 1, per, t_read)
        fm = field_map(rng, n, n, nz, amp)
        sm = coil_maps(rng, n, n, nz, nc)
        x = image(rng, n * n * nz)
        items.append(StreamItem(t_arr, n, n, nz, slices, nc, L, niter, 1e-3, kx, ky, kz, t, fm, sm, x))
    return items
