"""Seeded synthetic interferometer data with the shapes of the benchmark configs.

Stands in for a measurement set (the reference simulates with csimulator and
casacore measures; none of that is on the hot path).  Everything is FP64 and
seeded with numpy's default_rng:

  * antennas uniform in a disk of the given diameter in local ENU coordinates,
  * the standard hour-angle rotation ENU -> XYZ -> uvw (uvw in metres),
  * rows ordered time-major (all baselines of one integration together), as a
    measurement set stores them,
  * point sources with log-uniform fluxes, uniform positions in the field,
  * visibilities from the measurement equation
      V = sum_k S_k exp(+2 pi i f/c (l u + m v + (n - 1) w))
    (the sign convention of UnpolarizedPointSource::calcPoint), plus Gaussian
    noise, with unit noise (weight 1).

Cubes are complex64 arrays of shape (nrow, nchan, npol) in Fortran order, the
reference's casacore layout (row fastest).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

C_LIGHT = 299792458.0
SIDEREAL_RATE = 2.0 * math.pi / 86164.0905  # rad per second
ARCSEC = math.pi / (180.0 * 3600.0)
DEG = math.pi / 180.0


@dataclass
class Array:
    enu: np.ndarray          # (nant, 3) metres
    latitude: float          # rad

    @property
    def nant(self):
        return self.enu.shape[0]

    def baselines(self):
        i, j = np.triu_indices(self.nant, k=1)
        return i, j

    def xyz(self):
        lat = self.latitude
        e, n, u = self.enu[:, 0], self.enu[:, 1], self.enu[:, 2]
        x = -math.sin(lat) * n + math.cos(lat) * u
        y = e
        z = math.cos(lat) * n + math.sin(lat) * u
        return np.stack([x, y, z], axis=1)


def random_disk_array(nant: int, diameter_m: float, latitude_deg: float, seed: int) -> Array:
    rng = np.random.default_rng(seed)
    r = 0.5 * diameter_m * np.sqrt(rng.uniform(0.0, 1.0, nant))
    th = rng.uniform(0.0, 2.0 * math.pi, nant)
    enu = np.stack([r * np.cos(th), r * np.sin(th), np.zeros(nant)], axis=1)
    return Array(enu=enu, latitude=latitude_deg * DEG)


def uvw_track(arr: Array, dec: float, duration_s: float, dt_s: float):
    """uvw (nrow, 3) for a track centred on transit; rows time-major."""
    xyz = arr.xyz()
    i, j = arr.baselines()
    b = xyz[j] - xyz[i]                       # (nbl, 3)
    ntime = int(round(duration_s / dt_s))
    t = (np.arange(ntime) + 0.5) * dt_s - 0.5 * duration_s
    h = t * SIDEREAL_RATE                     # hour angle
    sh, ch = np.sin(h)[:, None], np.cos(h)[:, None]
    sd, cd = math.sin(dec), math.cos(dec)
    X, Y, Z = b[None, :, 0], b[None, :, 1], b[None, :, 2]
    u = sh * X + ch * Y
    v = -sd * ch * X + sd * sh * Y + cd * Z
    w = cd * ch * X - cd * sh * Y + sd * Z
    uvw = np.stack([u, v, w], axis=-1).reshape(-1, 3)
    return np.ascontiguousarray(uvw), ntime, b.shape[0]


@dataclass
class Sky:
    """components: (ncomp, 8) [flux, l, m, bmaj, bmin, bpa, spectral_index, ref_freq]."""
    components: np.ndarray


def random_point_sky(nsrc: int, field_deg: float, seed: int, flux_range=(0.01, 1.0)) -> Sky:
    rng = np.random.default_rng(seed)
    lo, hi = math.log(flux_range[0]), math.log(flux_range[1])
    flux = np.exp(rng.uniform(lo, hi, nsrc))
    half = 0.5 * field_deg * DEG
    l = rng.uniform(-half, half, nsrc)
    m = rng.uniform(-half, half, nsrc)
    comp = np.zeros((nsrc, 8))
    comp[:, 0] = flux
    comp[:, 1] = l
    comp[:, 2] = m
    comp[:, 7] = 1.0
    return Sky(comp)


def predict_numpy(uvw: np.ndarray, freq: np.ndarray, sky: Sky, chunk_rows: int = 65536) -> np.ndarray:
    """FP64 measurement equation, complex128 (nrow, nchan), Fortran order."""
    nrow, nchan = uvw.shape[0], freq.shape[0]
    out = np.zeros((nrow, nchan), dtype=np.complex128, order="F")
    comp = sky.components
    l, m = comp[:, 1], comp[:, 2]
    n = np.sqrt(1.0 - (l * l + m * m))
    scale = math.pi ** 2 / (4 * math.log(2.0))
    for r0 in range(0, nrow, chunk_rows):
        r1 = min(nrow, r0 + chunk_rows)
        u, v, w = uvw[r0:r1, 0:1], uvw[r0:r1, 1:2], uvw[r0:r1, 2:3]
        delay = 2.0 * math.pi * (l[None] * u + m[None] * v + (n[None] - 1.0) * w) / C_LIGHT  # (rows, ncomp)
        gauss = (comp[:, 3] > 0) | (comp[:, 4] > 0)
        r = None
        if np.any(gauss):
            bpa = comp[:, 5]
            up = (np.cos(bpa)[None] * u + np.sin(bpa)[None] * v) / C_LIGHT
            vp = (-np.sin(bpa)[None] * u + np.cos(bpa)[None] * v) / C_LIGHT
            r = (comp[:, 3][None] ** 2 * up * up + comp[:, 4][None] ** 2 * vp * vp) * scale
        for c in range(nchan):
            f = freq[c]
            flux = comp[:, 0].copy()
            si = comp[:, 6] != 0
            flux[si] = flux[si] * np.power(f / comp[si, 7], comp[si, 6])
            amp = np.broadcast_to(flux[None], delay.shape)
            if r is not None:
                amp = amp * np.exp(-r * f * f)
            out[r0:r1, c] = np.sum(amp * np.exp(1j * delay * f), axis=1)
    return out


@dataclass
class Dataset:
    uvw: np.ndarray
    freq: np.ndarray
    vis: np.ndarray          # complex64 (nrow, nchan, npol) F-order
    noise: np.ndarray        # complex64 cube (1 + 0j)
    flag: np.ndarray         # bool cube
    sky: Sky
    ntime: int
    nbl: int
    meta: dict = field(default_factory=dict)

    @property
    def nrow(self):
        return self.uvw.shape[0]


def make_dataset(nant=36, diameter_m=6000.0, latitude_deg=-26.7, dec_deg=-45.0, duration_s=3600.0,
                 dt_s=10.0, freq0=940e6, freq1=948e6, nchan=8, npol=1, nsrc=20, field_deg=2.0,
                 noise_sigma=0.01, seed=0, predict=None) -> Dataset:
    arr = random_disk_array(nant, diameter_m, latitude_deg, seed)
    uvw, ntime, nbl = uvw_track(arr, dec_deg * DEG, duration_s, dt_s)
    df = (freq1 - freq0) / nchan
    freq = freq0 + (np.arange(nchan) + 0.5) * df
    sky = random_point_sky(nsrc, field_deg, seed + 1)
    model = (predict or predict_numpy)(uvw, freq, sky)
    rng = np.random.default_rng(seed + 2)
    nrow = uvw.shape[0]
    vis = np.zeros((nrow, nchan, npol), dtype=np.complex64, order="F")
    for p in range(npol):
        # polarisations: XX and YY carry I, cross-hands carry noise only
        sig = model if (npol == 1 or p in (0, npol - 1)) else 0.0
        nz = noise_sigma * (rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan)))
        vis[:, :, p] = (sig + nz).astype(np.complex64)
    noise = np.ones((nrow, nchan, npol), dtype=np.complex64, order="F")
    flag = np.zeros((nrow, nchan, npol), dtype=bool, order="F")
    return Dataset(uvw=uvw, freq=freq, vis=vis, noise=noise, flag=flag, sky=sky, ntime=ntime, nbl=nbl,
                   meta=dict(nant=nant, dec_deg=dec_deg, seed=seed))


def config0(seed: int = 0, predict=None, duration_s: float = 3600.0) -> tuple[Dataset, dict]:
    """Plain WProject grid+degrid case: 36 antennas in a 6 km disk at -26.7 deg,
    1 h at 10 s, dec -45, 8 channels over 940-948 MHz, XX only, 20 sources in a
    2 deg field, noise 0.01 Jy.  Grid 2048^2 at 8 arcsec; 65 w-planes, os 4,
    cutoff 1e-3, maxsupport 1024."""
    ds = make_dataset(duration_s=duration_s, seed=seed, predict=predict)
    wmax_data = float(np.max(np.abs(ds.uvw[:, 2])) * ds.freq.max() / C_LIGHT)
    params = dict(gridder="WProject", nx=2048, ny=2048, cell_arcsec=8.0, nwplanes=65, oversample=4,
                  cutoff=1e-3, maxsupport=1024, wmax=math.ceil(wmax_data * 1.02 / 100.0) * 100.0)
    return ds, params


def beam_footprint(nside: int = 6, pitch_deg: float = 0.9) -> np.ndarray:
    """Pointing offsets (ra, dec) in radians of a square nside x nside beam
    footprint at the given pitch, centred on (0, 0), beams in row-major order."""
    k = (np.arange(nside) - (nside - 1) / 2.0) * pitch_deg * DEG
    dx, dy = np.meshgrid(k, k, indexing="xy")
    return np.stack([dx.ravel(), dy.ravel()], 1)


def multibeam_rows(ntime: int, nbl: int, nbeam: int, first_beam: int = 0):
    """Beam (feed) index per row of a track of ntime integrations x nbl
    baselines when the beams are observed in turn: integration t belongs to
    beam (first_beam + t) mod nbeam."""
    t = np.arange(ntime * nbl) // nbl
    return ((first_beam + t) % nbeam).astype(np.int32)
