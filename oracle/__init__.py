"""ORACLE — test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package; the product (``yandasoft_b200``) never does.

It restates yandasoft's visibility gridder on the CPU:
  * ``liboracle.so`` (C, oracle_gridder.c / oracle_dft.c): the bit-exact index
    block, w-plane mapping, the generic grid/degrid loop with GridKernel
    arithmetic, and an FP64 direct-DFT measurement equation;
  * ``cf.py`` / ``spheroidal.py`` (numpy): convolution-function generation,
    support search, grid correction and the FFT-side finalise steps.

``OracleGridder`` strings them together behind the same call sequence as
IVisGridder (askap/gridding/IVisGridder.h:64-140).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np

from . import cf as cfmod
from .spheroidal import SpheroidalFunction

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
C_LIGHT = 299792458.0


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
        _setup(_LIB)
    return _LIB


P = ctypes.c_void_p
I64 = ctypes.c_int64
I32 = ctypes.c_int
D = ctypes.c_double


class _Cfg(ctypes.Structure):
    _fields_ = [("nx", I32), ("ny", I32), ("npol", I32), ("nchan_img", I32), ("ngrids", I32),
                ("cellu", D), ("cellv", D), ("os", I32), ("ncf", I32),
                ("cf_size", P), ("cf_off", P), ("cf_data", P), ("noffsets", I32), ("cf_offsets", P),
                ("forward", I32), ("psf", I32), ("track_per_os", I32), ("nsumw_rows", I32), ("pcf", I32)]


class _Stats(ctypes.Structure):
    _fields_ = [("samples", D), ("taps", D), ("vectors_flagged", D), ("vectors_wflagged", D)]


def _setup(L):
    L.orc_nint.restype = I32
    L.orc_nint.argtypes = [D]
    L.orc_indices.restype = I32
    L.orc_indices.argtypes = [I64, I32, P, P, D, D, I32, I32, I32, P, P, P, P]
    L.orc_wplane_map.restype = I32
    L.orc_wplane_map.argtypes = [I64, I32, P, P, I32, D, I32, D, D, D, I32, P]
    L.orc_get_wterm.restype = D
    L.orc_get_wterm.argtypes = [I32, D, I32, D, D, D, I32]
    L.orc_gauss_params.restype = I32
    L.orc_gauss_params.argtypes = [D, ctypes.POINTER(D), ctypes.POINTER(D)]
    L.orc_ws_map.restype = D
    L.orc_ws_map.argtypes = [I32, D, D, D, D]
    L.orc_ws_index_pub.restype = D
    L.orc_ws_index_pub.argtypes = [I32, D, D, D, D]
    L.orc_generic.restype = I32
    L.orc_generic.argtypes = [ctypes.POINTER(_Cfg), I64, I32, I32, P, P, P, P, P, P, P, P, P, P, P, P,
                              P, P, P, ctypes.POINTER(_Stats), I64]
    L.orc_last_error.restype = ctypes.c_char_p
    L.orc_wstack_wproj_map.restype = I32
    L.orc_wstack_wproj_map.argtypes = [I64, I32, P, P, I32, D, I32, I32, D, P, P]
    L.orc_set_tap_kernels.restype = None
    L.orc_set_tap_kernels.argtypes = [P, P]
    L.orc_dft.restype = I32
    L.orc_dft.argtypes = [I64, I32, P, P, I32, P, P, P, I32]


def _p(a):
    return None if a is None else a.ctypes.data


REF_GRIDKERNEL = os.path.join(_HERE, "_ref", "libref_gridkernel.so")
_REF = None


def reference_gridkernel():
    """The reference's own GridKernel.cc compiled by oracle/Makefile into
    oracle/_ref (None when it was not built: the reference tree is absent)."""
    global _REF
    if _REF is None and os.path.exists(REF_GRIDKERNEL):
        _REF = ctypes.CDLL(REF_GRIDKERNEL)
        _REF.ref_grid_kernel_info.restype = I32
        _REF.ref_grid_kernel_info.argtypes = [ctypes.c_char_p, I32]
    return _REF


def use_reference_gridkernel(on: bool = True):
    """Makes the generic loop call the reference's compiled GridKernel::grid /
    degrid (on) or the restated tap loops (off, the default)."""
    L = lib()
    if not on:
        L.orc_set_tap_kernels(None, None)
        return
    R = reference_gridkernel()
    if R is None:
        raise OracleError("oracle/_ref/libref_gridkernel.so is not built (the reference tree is absent)")
    L.orc_set_tap_kernels(ctypes.cast(R.ref_grid_kernel, P), ctypes.cast(R.ref_degrid_kernel, P))


class OracleError(RuntimeError):
    pass


def _check(code):
    if code != 0:
        raise OracleError("oracle error %d: %s" % (code, lib().orc_last_error().decode()))


# --------------------------------------------------------------------------
# small helpers
# --------------------------------------------------------------------------
def nint(x: float) -> int:
    return lib().orc_nint(float(x))


def indices(uvw, freq, cellu, cellv, os_, nx, ny):
    """Bit-exact (iu, iv, fracu, fracv) per (row, chan), arrays shaped (nrow, nchan)."""
    uvw = np.ascontiguousarray(uvw, dtype=np.float64)
    freq = np.ascontiguousarray(freq, dtype=np.float64)
    nrow, nchan = uvw.shape[0], freq.shape[0]
    out = [np.zeros((nrow, nchan), dtype=np.int32, order="F") for _ in range(4)]
    _check(lib().orc_indices(nrow, nchan, _p(uvw), _p(freq), cellu, cellv, os_, nx, ny, *[_p(o) for o in out]))
    return tuple(out)


@dataclass
class WSampling:
    """w -> plane mapping of WDependentGridderBase with its IWSampling."""
    nwplanes: int
    wmax: float
    kind: str = "linear"       # linear | powerlaw | gaussian
    exponent: float = 1.0
    nwplanes50: float = 0.0
    wmaxclip: bool = False

    def __post_init__(self):
        if self.nwplanes % 2 != 1:
            raise OracleError("Number of w planes must be odd")
        self.wscale = self.wmax / float((self.nwplanes - 1) // 2) if self.nwplanes > 1 else 1.0
        self.code = {"linear": 0, "powerlaw": 1, "gaussian": 2}[self.kind]
        self.two_sigma2 = 1.0
        self.amplitude = 0.0
        if self.kind == "gaussian":
            a, b = D(), D()
            _check(lib().orc_gauss_params(self.nwplanes50 / self.nwplanes, ctypes.byref(a), ctypes.byref(b)))
            self.two_sigma2, self.amplitude = a.value, b.value

    def wterm(self, plane: int) -> float:
        return lib().orc_get_wterm(self.nwplanes, self.wscale, self.code, self.exponent,
                                   self.two_sigma2, self.amplitude, int(plane))

    def wterms(self):
        return np.array([self.wterm(i) for i in range(self.nwplanes)])

    def plane_map(self, uvw, freq):
        uvw = np.ascontiguousarray(uvw, dtype=np.float64)
        freq = np.ascontiguousarray(freq, dtype=np.float64)
        out = np.zeros((uvw.shape[0], freq.shape[0]), dtype=np.int32, order="F")
        _check(lib().orc_wplane_map(uvw.shape[0], freq.shape[0], _p(uvw), _p(freq), self.nwplanes, self.wscale,
                                    self.code, self.exponent, self.two_sigma2, self.amplitude,
                                    int(self.wmaxclip), _p(out)))
        return out

    def map(self, plane: float) -> float:
        return lib().orc_ws_map(self.code, self.exponent, self.two_sigma2, self.amplitude, plane)

    def index(self, w: float) -> float:
        return lib().orc_ws_index_pub(self.code, self.exponent, self.two_sigma2, self.amplitude, w)


def frequency_map(freqs, nchan_img, start=None, end=None, single_plane=False):
    """FrequencyMapper::setupMapping (askap/gridding/FrequencyMapper.cc:72-107)."""
    freqs = np.asarray(freqs, dtype=np.float64)
    if single_plane or nchan_img == 1:
        return np.zeros(len(freqs), dtype=np.int32)
    inc = (end - start) / float(nchan_img - 1)
    out = np.empty(len(freqs), dtype=np.int32)
    for i, f in enumerate(freqs):
        d = (f - start) / inc
        d += -0.5 if d < 0. else 0.5
        c = int(d)
        out[i] = c if 0 <= c < nchan_img else -1
    return out


def dft(uvw, freq, components, gain=None, nthreads=None):
    """FP64 DFT. components: (ncomp, 8) [flux, l, m, bmaj, bmin, bpa, si, reffreq].
    Returns complex128 (nrow, nchan)."""
    uvw = np.ascontiguousarray(uvw, dtype=np.float64)
    freq = np.ascontiguousarray(freq, dtype=np.float64)
    comp = np.ascontiguousarray(components, dtype=np.float64)
    nrow, nchan = uvw.shape[0], freq.shape[0]
    out = np.zeros((nrow, nchan), dtype=np.complex128, order="F")
    g = None if gain is None else np.asfortranarray(gain, dtype=np.float64)
    nt = nthreads or os.cpu_count() or 1
    _check(lib().orc_dft(nrow, nchan, _p(uvw), _p(freq), comp.shape[0], _p(comp), _p(g), _p(out), nt))
    return out


# --------------------------------------------------------------------------
# the gridder restatement
# --------------------------------------------------------------------------
@dataclass
class Chunk:
    """One accessor chunk (IConstDataAccessor unpacked).  Cubes are (nrow, nchan, npol)
    Fortran-ordered, i.e. the reference's casacore layout (row fastest)."""
    uvw: np.ndarray                 # (nrow, 3) float64, metres
    freq: np.ndarray                # (nchan,) float64, Hz
    vis: np.ndarray                 # complex64 cube
    noise: np.ndarray | None = None  # complex64 cube (default 1)
    flag: np.ndarray | None = None   # bool cube
    delay: np.ndarray | None = None  # (nrow,) float64
    feed1: np.ndarray | None = None  # (nrow,) int32
    pointing: np.ndarray | None = None  # (nrow, 2) float64 (ra, dec)

    @property
    def nrow(self):
        return self.uvw.shape[0]


class OracleGridder:
    """CPU restatement of SphFunc / WProject / WStack / AWProject gridders."""

    def __init__(self, kind: str, **kw):
        self.kind = kind
        self.kw = kw
        self.os = int(kw.get("oversample", {"SphFunc": 128}.get(kind, 8)))
        self.alpha = float(kw.get("alpha", 1.0))
        self.grdsf = SpheroidalFunction(math.pi * int(kw.get("support", 3)) if kind == "SphFunc" else math.pi * 3,
                                        self.alpha)
        self.cache = None
        self.carry = None
        self.track_per_os = bool(kw.get("oversampleweight", False))
        self.model_empty = False
        if kind in ("WProject", "WStack", "AWProject"):
            default_wmax = 10000.0 if kind == "AWProject" else 35000.0
            self.ws = WSampling(int(kw.get("nwplanes", 65)), float(kw.get("wmax", default_wmax)),
                                kw.get("wsampling", "linear"), float(kw.get("exponent", 1.0)),
                                float(kw.get("nwplanes50", 0.0)), bool(kw.get("wmaxclip", False)))
        elif kind == "WStackWProject":
            # w-stacks over (-wmax, wmax); w-projection of the residual over half a stack spacing
            self.stacks = WSampling(int(kw.get("nwstacks", 17)), float(kw.get("wmax", 35000.0)),
                                    wmaxclip=bool(kw.get("wmaxclip", False)))
            self.ws = WSampling(int(kw.get("nwplanes", 33)), 0.5 * self.stacks.wscale)
        else:
            self.ws = None

    # ---- axes -------------------------------------------------------------
    def _init_axes(self, nx, ny, npol, nchan, cell_x, cell_y, freq_axis):
        self.nx, self.ny, self.npol, self.nchan_img = nx, ny, npol, nchan
        self.uvcell = (1.0 / (cell_x * float(nx)), 1.0 / (cell_y * float(ny)))
        self.freq_axis = freq_axis

    def _chan_map(self, freq):
        if self.freq_axis is None:
            return np.zeros(len(freq), dtype=np.int32)
        return frequency_map(freq, self.nchan_img, self.freq_axis[0], self.freq_axis[1])

    def _ngrids(self):
        if self.kind == "WStack":
            return self.ws.nwplanes
        if self.kind == "WStackWProject":
            return self.stacks.nwplanes
        return 1

    def initialise_grid(self, nx, ny, npol, nchan, cell_x, cell_y, freq_axis=None, dopsf=False, dopcf=False):
        self._init_axes(nx, ny, npol, nchan, cell_x, cell_y, freq_axis)
        self.psf = dopsf
        self.pcf = dopcf
        self.forward = False
        n = nx * ny * npol * nchan
        buf = np.zeros(n * self._ngrids(), dtype=np.complex64)
        self.grids = [buf[i * n:(i + 1) * n].reshape((nx, ny, npol, nchan), order="F") for i in range(self._ngrids())]
        self._init_sumw()
        self.first_psf_row = True
        self.rep_feed = None
        self.rep_pointing = None

    def _nsumw_cf(self):
        if self.kind in ("WProject", "WStackWProject"):
            return self.ws.nwplanes
        if self.kind == "WStack":
            return 1
        if self.kind == "AWProject":
            return None  # set when the CF cache is built
        return 1

    def _init_sumw(self):
        n = self._nsumw_cf()
        if n is None:
            self.sumw = None
            return
        rows = n * self.os * self.os if self.track_per_os else n
        self.sumw = np.zeros((rows, self.npol, self.nchan_img), dtype=np.float64, order="F")

    # ---- CF ---------------------------------------------------------------
    def _cf_params(self):
        kw = self.kw
        common = dict(nwplanes=self.ws.nwplanes, wmax=self.ws.wmax, cutoff=float(kw.get("cutoff", 1e-3)),
                      oversample=self.os, limitsupport=int(kw.get("limitsupport", 0)), alpha=self.alpha,
                      variablesupport=bool(kw.get("variablesupport", False)),
                      offsetsupport=bool(kw.get("offsetsupport", False)),
                      cutoff_absolute=bool(kw.get("cutoff_absolute", False)), wterms=self.ws.wterms())
        if self.kind in ("WProject", "WStackWProject"):
            return cfmod.WProjectParams(maxsupport=int(kw.get("maxsupport", 256)), **common)
        return cfmod.AWProjectParams(maxsupport=int(kw.get("maxsupport", 128)),
                                     diameter=float(kw.get("diameter", 12.0)), blockage=float(kw.get("blockage", 2.0)),
                                     maxfeeds=int(kw.get("maxfeeds", 1)), maxfields=int(kw.get("maxfields", 1)),
                                     frequencydependent=bool(kw.get("frequencydependent", True)),
                                     spheroidaltaper=bool(kw.get("spheroidaltaper", False)), **common)

    def init_cf(self, chunk: Chunk | None = None):
        if self.cache is not None and self.kind != "AWProject":
            return
        if self.kind in ("SphFunc", "WStack"):
            sup = int(self.kw.get("support", 3)) if self.kind == "SphFunc" else 3
            os_ = self.os if self.kind == "SphFunc" else 128
            if self.kind == "WStack":
                self.os = os_
            self.cache = cfmod.sphfunc_cf(sup, os_, self.alpha)
        elif self.kind in ("WProject", "WStackWProject"):
            self.cache = cfmod.wproject_cf(self.nx, self.ny, self.uvcell[0], self.uvcell[1], self._cf_params())
        else:
            if self.cache is None:
                p = self._cf_params()
                feeds = {}
                for r in range(chunk.nrow):
                    f = int(chunk.feed1[r]) if chunk.feed1 is not None else 0
                    if f not in feeds:
                        feeds[f] = tuple(chunk.pointing[r]) if chunk.pointing is not None else (0.0, 0.0)
                centre = tuple(self.kw.get("image_centre", (0.0, 0.0)))
                self.aw_nchan = len(chunk.freq) if p.frequencydependent else 1
                self.cache = cfmod.awproject_cf(self.uvcell[0], self.uvcell[1], p, chunk.freq, feeds, centre,
                                                is_psf=self.psf)
                self.aw_params = p
            if self.sumw is None:
                # AWProjectVisGridder's sums of weights have a row per CF plane
                # (initialiseSumOfWeights, after every initialiseGrid)
                p = self.aw_params
                n = p.nwplanes * p.maxfeeds * p.maxfields * self.aw_nchan
                rows = n * self.os * self.os if self.track_per_os else n
                self.sumw = np.zeros((rows, self.npol, self.nchan_img), dtype=np.float64, order="F")
        self._flat = self.cache.flatten()

    # ---- index maps -------------------------------------------------------
    def _maps(self, chunk: Chunk):
        nrow, nchan = chunk.nrow, len(chunk.freq)
        if self.kind == "SphFunc":
            return None, None
        if self.kind == "WStackWProject":
            uvw = np.ascontiguousarray(chunk.uvw, dtype=np.float64)
            freq = np.ascontiguousarray(chunk.freq, dtype=np.float64)
            gmap = np.zeros((nrow, nchan), dtype=np.int32, order="F")
            cmap = np.zeros((nrow, nchan), dtype=np.int32, order="F")
            _check(lib().orc_wstack_wproj_map(nrow, nchan, _p(uvw), _p(freq), self.stacks.nwplanes,
                                              self.stacks.wscale, int(self.stacks.wmaxclip), self.ws.nwplanes,
                                              self.ws.wscale, _p(gmap), _p(cmap)))
            return cmap, gmap
        planes = self.ws.plane_map(chunk.uvw, chunk.freq)
        if self.kind == "WStack":
            return np.zeros((nrow, nchan), dtype=np.int32, order="F"), planes
        if self.kind == "WProject":
            return planes, None
        p = self.aw_params
        feed = chunk.feed1 if chunk.feed1 is not None else np.zeros(nrow, dtype=np.int32)
        field = 0
        nw = p.nwplanes
        ch = np.arange(nchan)[None, :]
        fd = feed.astype(np.int64)[:, None]
        if p.frequencydependent:
            extra = nw * (ch + nchan * (fd + p.maxfeeds * field))
        else:
            extra = nw * (fd + p.maxfeeds * field) + 0 * ch
        cmap = np.where(planes >= 0, planes + extra, planes).astype(np.int32)
        return np.asfortranarray(cmap), None

    def _run(self, chunk: Chunk, forward: bool):
        nrow, nchan = chunk.nrow, len(chunk.freq)
        npol = chunk.vis.shape[2]
        if self.carry is None:
            self.carry = np.zeros(2 * npol, dtype=np.float32)
        cmap, gmap = self._maps(chunk)
        sizes, offs, data = self._flat
        offsets = None
        if self.cache.offsets:
            offsets = np.ascontiguousarray(np.array(self.cache.offsets, dtype=np.int32).reshape(-1))
        cfg = _Cfg(self.nx, self.ny, self.npol, self.nchan_img, len(self.grids), self.uvcell[0], self.uvcell[1],
                   self.os, len(sizes), _p(sizes), _p(offs), _p(data),
                   0 if offsets is None else len(self.cache.offsets), _p(offsets),
                   int(forward), int(getattr(self, "psf", False) and not forward), int(self.track_per_os),
                   self.sumw.shape[0] if self.sumw is not None else 1,
                   int(getattr(self, "pcf", False) and not forward))
        flag = chunk.flag if chunk.flag is not None else np.zeros(chunk.vis.shape, dtype=bool, order="F")
        flag = np.asfortranarray(flag.astype(np.uint8))
        noise = chunk.noise if chunk.noise is not None else np.ones(chunk.vis.shape, dtype=np.complex64, order="F")
        noise = np.asfortranarray(noise.astype(np.complex64))
        chan_map = np.ascontiguousarray(self._chan_map(chunk.freq), dtype=np.int32)
        psf_ok = self._psf_mask(chunk) if (not forward and getattr(self, "psf", False)) else None
        mfs = getattr(self, "mfs", None)
        mfs_arr = None if mfs is None else np.ascontiguousarray(mfs(chunk.freq), dtype=np.float32)
        uvw = np.ascontiguousarray(chunk.uvw, dtype=np.float64)
        freq = np.ascontiguousarray(chunk.freq, dtype=np.float64)
        delay = None if chunk.delay is None else np.ascontiguousarray(chunk.delay, dtype=np.float64)
        assert chunk.vis.flags.f_contiguous and chunk.vis.dtype == np.complex64
        # grids buffer: ngrids consecutive column-major (nx, ny, npol, nchan) blocks
        gbuf = self._grid_buffer()
        sumw = self.sumw if self.sumw is not None else np.zeros((1, self.npol, self.nchan_img), order="F")
        st = _Stats()
        _check(lib().orc_generic(ctypes.byref(cfg), nrow, nchan, npol, _p(uvw), _p(delay), _p(freq), _p(chan_map),
                                 _p(flag), _p(chunk.vis), _p(noise), _p(cmap), _p(gmap), None, _p(psf_ok), _p(mfs_arr),
                                 _p(gbuf), _p(sumw), _p(self.carry), ctypes.byref(st), 0))
        if not forward:
            n = self.nx * self.ny * self.npol * self.nchan_img
            for i in range(len(self.grids)):
                self.grids[i] = gbuf[i * n:(i + 1) * n].reshape((self.nx, self.ny, self.npol, self.nchan_img),
                                                                 order="F")
        self.stats = st
        return st

    def _grid_buffer(self):
        """The grids as one buffer of consecutive column-major blocks: the
        grids themselves when they are already such views of one array (as
        initialise_grid makes them), else a copy."""
        n = self.nx * self.ny * self.npol * self.nchan_img
        g0 = self.grids[0]
        base = g0.base if g0.base is not None else g0
        if (base.ndim == 1 and base.dtype == np.complex64 and base.size == n * len(self.grids)
                and all(g.flags.f_contiguous and g.dtype == np.complex64 and g.size == n
                        and g.ctypes.data == base.ctypes.data + i * n * 8 for i, g in enumerate(self.grids))):
            return base
        return np.concatenate([g.ravel(order="F") for g in self.grids])

    def _psf_mask(self, chunk: Chunk):
        if self.kw.get("alldatapsf", False):
            return None
        feed = chunk.feed1 if chunk.feed1 is not None else np.zeros(chunk.nrow, dtype=np.int32)
        pnt = chunk.pointing if chunk.pointing is not None else np.zeros((chunk.nrow, 2))
        if self.first_psf_row:
            self.rep_feed = int(feed[0])
            self.rep_pointing = tuple(pnt[0])
            self.first_psf_row = False
        sep = _separation(pnt, self.rep_pointing)
        return np.ascontiguousarray(((feed == self.rep_feed) & (sep < 1e-6)).astype(np.uint8))

    def grid(self, chunk: Chunk):
        self.init_cf(chunk)
        return self._run(chunk, forward=False)

    def _stack_sampling(self):
        return self.ws if self.kind == "WStack" else self.stacks

    def finalise_grid(self):
        if self.kind in ("WStack", "WStackWProject"):
            st = self._stack_sampling()
            screens = [cfmod.wstack_screen(self.nx, self.ny, self.uvcell[0], self.uvcell[1], st.wterm(i))
                       for i in range(st.nwplanes)]
            return cfmod.finalise_grid(self.grids, self.grdsf, screens=screens)
        if self.kind == "AWProject" and not self.aw_params.spheroidaltaper:
            s = None
            for g in self.grids:
                r = cfmod.fft2d(g, False).real.astype(np.float32)
                s = r if s is None else s + r
            return (s * np.float32(float(self.nx) * float(self.ny))).astype(np.float32)
        return cfmod.finalise_grid(self.grids, self.grdsf)

    def finalise_weights(self):
        if self.kind == "AWProject":
            p = self.aw_params
            return cfmod.aw_finalise_weights(self.cache.cfs, self.sumw, self.os, self.track_per_os,
                                             self.cache.offsets, p.maxsupport, self.nx, self.ny, self.nx, self.ny,
                                             grdsf=self.grdsf if p.spheroidaltaper else None,
                                             weights_cutoff=float(self.kw.get("spheroidalweightscutoff", 0.0)))
        tot = self.sumw.sum(axis=0)  # (npol, nchan)
        return np.broadcast_to(tot[None, None], (self.nx, self.ny) + tot.shape).astype(np.float32)

    def initialise_degrid(self, image, cell_x, cell_y, freq_axis=None):
        nx, ny, npol, nchan = image.shape
        self._init_axes(nx, ny, npol, nchan, cell_x, cell_y, freq_axis)
        self.psf = False
        self.pcf = False
        self.model_empty = not np.max(np.abs(image)) > 0
        if self.kind in ("WStack", "WStackWProject"):
            st = self._stack_sampling()
            screens = [cfmod.wstack_screen(nx, ny, self.uvcell[0], self.uvcell[1], st.wterm(i))
                       for i in range(st.nwplanes)]
            self.grids = cfmod.wstack_initialise_degrid(image, self.grdsf, screens)
        elif self.kind == "AWProject" and not self.kw.get("spheroidaltaper", False):
            self.grids = [cfmod.fft2d(image.astype(np.complex64), True)]
        else:
            self.grids = [cfmod.initialise_degrid(image, self.grdsf)]
        self.grids = [np.asfortranarray(g.astype(np.complex64)) for g in self.grids]
        self.sumw = None
        if self.kind != "AWProject":
            self._init_sumw()

    def degrid(self, chunk: Chunk):
        if self.model_empty:
            return None
        self.init_cf(chunk)
        if self.sumw is None:
            self.sumw = np.zeros((1, self.npol, self.nchan_img), order="F")
        return self._run(chunk, forward=True)


def _separation(pnt, ref):
    ra, dec = pnt[:, 0], pnt[:, 1]
    ra0, dec0 = ref
    c = np.sin(dec) * np.sin(dec0) + np.cos(dec) * np.cos(dec0) * np.cos(ra - ra0)
    return np.arccos(np.clip(c, -1.0, 1.0))
