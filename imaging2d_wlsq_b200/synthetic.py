"""Seeded synthetic workloads standing in for field data (no dataset is available offline).

Each workload carries everything the compact-table entry point needs: velocity model, angular
frequencies, compact operator table and its kappa step, per-shot apertures, and the packed source
and receiver spectra.  Sizes follow the five benchmark configurations of this project:

  plain_small   nz=200  nx=320  dx=dz=10 m, 4 flat layers + Gaussian lens, nf=64 (2-30 Hz),
                nk=1000 x 25 taps, 4 full-aperture shots at x=40,120,200,280, Ricker 15 Hz
  plain_medium  nz=500  nx=1024 dx=dz=10 m, Gaussian random field 1500-4500 m/s (corr. 50 samples),
                nf=256 (2-40 Hz), nk=2000 x 31 taps, 32 evenly spaced full-aperture shots, Ricker 20 Hz
  batched_uneven nz=1000 nx=2048 dx=dz=10 m, same velocity recipe, nf=512 (2-50 Hz), nk=4000 x 35
                taps, 256 shots with aperture NX ~ U[256, 2048] centred on a random x (clipped)
  precision     nz=2000 nx=4096 dx=dz=5 m, random field + 20 thin layers of +-800 m/s (5-15 samples),
                nf=1024 (2-60 Hz), nk=8000 x 55 taps, 64 full-aperture shots
  lsm           nz=500 nx=1024, smooth background as plain_medium, nf=256 (2-40 Hz), nk=2000 x 31,
                64 full-aperture shots (data synthesised by the adjoint kernel)

Receiver spectra are Ricker(f0) amplitude x seeded complex unit-variance Gaussian per trace; the
source is a Ricker(f0) spike at the shot position.  `scale` shrinks every dimension for tests.
"""
import math
from dataclasses import dataclass, field

import numpy as np
from scipy import ndimage

from . import operators


@dataclass
class Workload:
    name: str
    nz: int
    nx: int
    dx: float
    dz: float
    nf: int
    M: int
    nk: int
    dk: float
    omega: np.ndarray          # (nf,) float64
    velocity: np.ndarray       # (nz, nx) float64
    table: np.ndarray          # (nk, 2M+1) complex64 forward operators
    shot_x0: np.ndarray        # (ns,) int32
    shot_nx: np.ndarray        # (ns,) int32
    shot_pos: np.ndarray       # (ns,) int32 source position in model coordinates
    wave: np.ndarray = field(default=None)   # packed source spectra, complex64
    shot: np.ndarray = field(default=None)   # packed receiver spectra, complex64
    nextrap: int = 0
    seed: int = 0
    reflectivity: np.ndarray = field(default=None)  # (nz, nx) float32 (least-squares migration only)

    @property
    def ns(self):
        return len(self.shot_x0)

    @property
    def L(self):
        return 2 * self.M + 1

    @property
    def nt(self):
        return self.nf

    def offsets(self):
        off = np.zeros(self.ns, dtype=np.int64)
        off[1:] = np.cumsum(self.nf * self.shot_nx.astype(np.int64))[:-1]
        return off

    def points(self):
        """Extrapolated points (shot, w, z, x) of one migration."""
        return int(self.shot_nx.astype(np.int64).sum()) * self.nf * self.nextrap

    def block(self, arr, s):
        o = self.offsets()[s]
        return arr[o:o + self.nf * int(self.shot_nx[s])].reshape(self.nf, int(self.shot_nx[s]))


def ricker_spectrum(f, f0):
    """Amplitude spectrum of a Ricker wavelet of peak frequency f0."""
    f = np.asarray(f, dtype=np.float64)
    return (2.0 / math.sqrt(math.pi)) * f ** 2 / f0 ** 3 * np.exp(-(f ** 2) / f0 ** 2)


def gaussian_random_field(nz, nx, corr, vmin, vmax, rng):
    white = rng.standard_normal((nz, nx))
    g = ndimage.gaussian_filter(white, sigma=corr / 2.0, mode="wrap")
    g = (g - g.mean()) / (g.std() + 1e-30)
    mid = 0.5 * (vmin + vmax)
    half = 0.5 * (vmax - vmin)
    return np.clip(mid + half * g / 2.0, vmin, vmax)


def layered_lens(nz, nx):
    v = np.empty((nz, nx), dtype=np.float64)
    speeds = [1500.0, 2200.0, 2800.0, 3500.0]
    for i, c in enumerate(speeds):
        v[i * nz // 4:(i + 1) * nz // 4, :] = c
    zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    zc, xc = 120 * nz / 200.0, 160 * nx / 320.0
    v += 600.0 * np.exp(-((zz - zc) ** 2 + (xx - xc) ** 2) / (2.0 * (20.0 * nz / 200.0) ** 2))
    return ndimage.gaussian_filter(v, sigma=5.0 * nz / 200.0, mode="nearest")


def _finish(w, fmin, fmax, f0, rng, tables=True):
    f = np.linspace(fmin, fmax, w.nf)
    w.omega = 2.0 * math.pi * f
    kmax = w.omega.max() / w.velocity[:w.nextrap].min()
    w.dk = kmax / (w.nk - 1)
    if tables:
        w.table = operators.design_compact_table(w.nx, w.dx, w.dz, w.M, w.nk, w.dk)
    amp = ricker_spectrum(f, f0).astype(np.float32)
    total = int(w.shot_nx.astype(np.int64).sum()) * w.nf
    w.wave = np.zeros(total, dtype=np.complex64)
    w.shot = np.empty(total, dtype=np.complex64)
    off = w.offsets()
    for s in range(w.ns):
        n = int(w.shot_nx[s])
        blk = w.wave[off[s]:off[s] + w.nf * n].reshape(w.nf, n)
        blk[:, int(w.shot_pos[s] - w.shot_x0[s])] = amp
        g = rng.standard_normal((w.nf, n, 2)).astype(np.float32) * np.float32(1.0 / math.sqrt(2.0))
        rec = (g[..., 0] + 1j * g[..., 1]).astype(np.complex64) * amp[:, None]
        w.shot[off[s]:off[s] + w.nf * n] = rec.reshape(-1)
    return w


def _full_aperture(ns, nx, positions):
    x0 = np.zeros(ns, dtype=np.int32)
    wdt = np.full(ns, nx, dtype=np.int32)
    return x0, wdt, np.asarray(positions, dtype=np.int32)


def plain_small(seed=1, scale=1.0, tables=True):
    nz, nx = max(8, int(200 * scale)), max(16, int(320 * scale))
    rng = np.random.default_rng(seed)
    v = layered_lens(nz, nx)
    pos = [int(p * nx / 320.0) for p in (40, 120, 200, 280)]
    x0, wdt, pos = _full_aperture(4, nx, pos)
    w = Workload("plain_small", nz, nx, 10.0, 10.0, max(4, int(64 * scale)), 12, max(64, int(1000 * scale)), 0.0,
                 None, v, None, x0, wdt, pos, nextrap=nz, seed=seed)
    return _finish(w, 2.0, 30.0, 15.0, rng, tables)


def plain_medium(seed=2, scale=1.0, tables=True, ns=32, nz=None, nx=None, nf=None):
    nz = nz or max(8, int(500 * scale))
    nx = nx or max(32, int(1024 * scale))
    rng = np.random.default_rng(seed)
    v = gaussian_random_field(nz, nx, 50.0 * max(scale, 0.1), 1500.0, 4500.0, rng)
    ns = max(1, int(ns * min(1.0, scale * 4))) if scale < 1.0 else ns
    pos = np.linspace(nx / (2 * ns), nx - nx / (2 * ns), ns).astype(np.int32)
    x0, wdt, pos = _full_aperture(ns, nx, pos)
    w = Workload("plain_medium", nz, nx, 10.0, 10.0, nf or max(4, int(256 * scale)), 15,
                 max(64, int(2000 * scale)), 0.0, None, v, None, x0, wdt, pos, nextrap=nz, seed=seed)
    return _finish(w, 2.0, 40.0, 20.0, rng, tables)


def batched_uneven(seed=3, scale=1.0, tables=True, ns=256, nz=None, nx=None, nf=None):
    nz = nz or max(8, int(1000 * scale))
    nx = nx or max(64, int(2048 * scale))
    rng = np.random.default_rng(seed)
    v = gaussian_random_field(nz, nx, 50.0 * max(scale, 0.1), 1500.0, 4500.0, rng)
    ns = max(2, int(ns * scale)) if scale < 1.0 else ns
    lo, hi = max(4, int(256 * scale)), nx
    width = rng.integers(lo, hi + 1, ns)
    centre = rng.integers(0, nx, ns)
    x0 = np.clip(centre - width // 2, 0, nx).astype(np.int32)
    x1 = np.clip(centre - width // 2 + width, 0, nx).astype(np.int32)
    bad = x1 - x0 < 2
    x0[bad] = np.minimum(x0[bad], nx - 2)
    x1[bad] = x0[bad] + 2
    wdt = (x1 - x0).astype(np.int32)
    pos = np.clip(centre, x0, x1 - 1).astype(np.int32)
    w = Workload("batched_uneven", nz, nx, 10.0, 10.0, nf or max(4, int(512 * scale)), 17,
                 max(64, int(4000 * scale)), 0.0, None, v, None, x0, wdt, pos, nextrap=nz, seed=seed)
    return _finish(w, 2.0, 50.0, 20.0, rng, tables)


def precision(seed=4, scale=1.0, tables=True, ns=64, nextrap=None, nf=None, nx=None):
    nz, nx = max(8, int(2000 * scale)), nx or max(64, int(4096 * scale))
    rng = np.random.default_rng(seed)
    v = gaussian_random_field(nz, nx, 50.0 * max(scale, 0.1), 1500.0, 4500.0, rng)
    for _ in range(20):
        thick = int(rng.integers(5, 16) * max(scale, 0.2)) or 1
        z0 = int(rng.integers(0, max(1, nz - thick)))
        v[z0:z0 + thick, :] += rng.choice([-800.0, 800.0])
    v = np.clip(v, 1200.0, 5300.0)
    ns = max(2, int(ns * scale)) if scale < 1.0 else ns
    pos = np.linspace(nx / (2 * ns), nx - nx / (2 * ns), ns).astype(np.int32)
    x0, wdt, pos = _full_aperture(ns, nx, pos)
    w = Workload("precision", nz, nx, 5.0, 5.0, nf or max(4, int(1024 * scale)), 27, max(64, int(8000 * scale)), 0.0,
                 None, v, None, x0, wdt, pos, nextrap=nextrap or nz, seed=seed)
    return _finish(w, 2.0, 60.0, 25.0, rng, tables)


def sparse_reflectivity(nz, nx, density, rng):
    """Seeded sparse spikes (`density` of the samples, amplitudes N(0, 1)) convolved with the
    3-sample smoothing kernel [1, 2, 1]/4 along z and along x."""
    r = np.zeros((nz, nx), dtype=np.float64)
    n = max(1, int(round(density * nz * nx)))
    flat = rng.choice(nz * nx, size=n, replace=False)
    r.reshape(-1)[flat] = rng.standard_normal(n)
    k = np.array([0.25, 0.5, 0.25])
    r = ndimage.convolve1d(r, k, axis=0, mode="constant")
    r = ndimage.convolve1d(r, k, axis=1, mode="constant")
    return r.astype(np.float32)


def lsm(seed=5, scale=1.0, tables=True, ns=64, nz=None, nx=None, nf=None):
    """Least-squares migration configuration: plain_medium's smooth background and operators,
    64 full-aperture shots, and a sparse reflectivity (0.5% spikes) from which the observed data
    are synthesised by demigration on the device."""
    nz = nz or max(8, int(500 * scale))
    nx = nx or max(32, int(1024 * scale))
    rng = np.random.default_rng(seed)
    v = gaussian_random_field(nz, nx, 50.0 * max(scale, 0.1), 1500.0, 4500.0, rng)
    ns = max(1, int(ns * min(1.0, scale * 4))) if scale < 1.0 else ns
    pos = np.linspace(nx / (2 * ns), nx - nx / (2 * ns), ns).astype(np.int32)
    x0, wdt, pos = _full_aperture(ns, nx, pos)
    w = Workload("lsm", nz, nx, 10.0, 10.0, nf or max(4, int(256 * scale)), 15,
                 max(64, int(2000 * scale)), 0.0, None, v, None, x0, wdt, pos, nextrap=nz, seed=seed)
    w = _finish(w, 2.0, 40.0, 20.0, rng, tables)
    w.reflectivity = sparse_reflectivity(nz, nx, 0.005, rng)
    return w


WORKLOADS = {
    "plain_small": plain_small,
    "plain_medium": plain_medium,
    "batched_uneven": batched_uneven,
    "precision": precision,
    "lsm": lsm,
}
