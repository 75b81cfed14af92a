"""ORACLE — test infrastructure only (never imported by the product).

numpy restatement of yandasoft's convolution-function (CF) generation and of
the FFT-side finalise/initialise steps, with the reference's FP32/FP64 split.
Arrays are indexed [x, y] (x = u axis); a casacore column-major scan
(x fastest) is ``order='F'``.

Reference files followed:
  - SupportSearcher::findPeak / doSupportSearch / support /
    symmetricalSupport: askap/gridding/SupportSearcher.tcc:88-262,
    SupportSearcher.cc:98-121.
  - SphFuncVisGridder::initConvolutionFunction / correctConvolution:
    askap/gridding/SphFuncVisGridder.cc:90-248; interpolateEdgeValues:
    SphFuncVisGridder.tcc:38-50.
  - WProjectVisGridder::generate / setup / populateThisPlane / extractSupport /
    calcSupport / limitSupportIfNecessary / calcConvFuncOverflow /
    populateItsConvFunc / normalise: askap/gridding/WProjectVisGridder.cc:
    198-284,435-522,538-726.
  - AWProjectVisGridder::initConvolutionFunction:
    askap/gridding/AWProjectVisGridder.cc:259-611; DiskIllumination::getPattern:
    askap/gridding/DiskIllumination.cc:85-181.
  - TableVisGridder::finaliseGrid / initialiseDegrid / finaliseWeights:
    askap/gridding/TableVisGridder.cc:1109-1319.
  - WStackVisGridder::multiply / finaliseGrid / initialiseDegrid:
    askap/gridding/WStackVisGridder.cc:134-337.

``scimath::fft2d`` (un-vendored base-scimath 1.9.0, FFTW) is restated from
its usage: centred transforms (origin at N/2), forward = exp(-2 pi i ...)
unnormalised, backward = exp(+2 pi i ...) normalised by 1/N.  The FFT here is
numpy's single-precision pocketfft, so CF values agree with FFTW only to FP32
rounding; support sizes and indices are compared exactly.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .spheroidal import SpheroidalFunction

C_LIGHT = 299792458.0
F32 = np.float32


# --------------------------------------------------------------------------
# FFT conventions of scimath::fft2d / fft
# --------------------------------------------------------------------------
def fft2d(a: np.ndarray, forward: bool) -> np.ndarray:
    a = np.asarray(a)
    dt = a.dtype
    s = np.fft.ifftshift(a, axes=(0, 1))
    if forward:
        r = np.fft.fft2(s, axes=(0, 1))
    else:
        r = np.fft.ifft2(s, axes=(0, 1))
    return np.fft.fftshift(r, axes=(0, 1)).astype(dt, copy=False)


def fft1d(a: np.ndarray, forward: bool) -> np.ndarray:
    dt = a.dtype
    s = np.fft.ifftshift(a)
    r = np.fft.fft(s) if forward else np.fft.ifft(s)
    return np.fft.fftshift(r).astype(dt, copy=False)


# --------------------------------------------------------------------------
# SupportSearcher
# --------------------------------------------------------------------------
@dataclass
class SupportResult:
    peak_pos: tuple
    peak_val: float
    blc: tuple
    trc: tuple

    def support(self) -> int:
        return max(self.trc[0] - self.blc[0], self.trc[1] - self.blc[1])

    def symmetrical_support(self, shape) -> int:
        cx, cy = shape[0] // 2, shape[1] // 2
        xmax = max(abs(self.trc[0] - cx), abs(cx - self.blc[0]))
        ymax = max(abs(self.trc[1] - cy), abs(cy - self.blc[1]))
        return int(max(xmax, ymax) * 2)


def find_peak(a: np.ndarray):
    """Peak of |a|^2 in double, column-major scan with the reference's tie rules."""
    amp = a.real.astype(np.float64) ** 2 + a.imag.astype(np.float64) ** 2
    col_arg = np.argmax(amp, axis=0)          # first max in each column
    col_max = amp[col_arg, np.arange(amp.shape[1])]
    peak_val = -1.0
    pos = (0, 0)
    for iy in range(amp.shape[1]):
        t = col_max[iy]
        if peak_val < 0 or peak_val * peak_val < t:
            pos = (int(col_arg[iy]), iy)
            peak_val = math.sqrt(t)
    if not peak_val > 0:
        raise ValueError("Unable to find peak in the support searcher")
    return pos, peak_val


def support_search(a: np.ndarray, cutoff: float, value: float = -1.0) -> SupportResult:
    """SupportSearcher::search(in, value) on a complex64 matrix."""
    pos, peak_val = find_peak(a)
    if value > 0:
        peak_val = value
    px, py = pos
    nxr, nyc = a.shape
    if not (px > 0 and py > 0 and px + 1 < nxr and py + 1 < nyc):
        raise ValueError("Peak position of the convolution function is too close to the edge")
    c = cutoff * peak_val
    abs_cut = abs(c) * abs(c)
    # ampFunction on complex<float>: re*re + im*im in float
    row = a[:, py]
    col = a[px, :]
    amp_row = (row.real * row.real + row.imag * row.imag).astype(F32)
    amp_col = (col.real * col.real + col.imag * col.imag).astype(F32)
    above_r = amp_row.astype(np.float64) > abs_cut
    above_c = amp_col.astype(np.float64) > abs_cut
    idx = np.nonzero(above_r[: px + 1])[0]
    blc0 = int(idx[0]) if idx.size else -1
    idx = np.nonzero(above_c[: py + 1])[0]
    blc1 = int(idx[0]) if idx.size else -1
    idx = np.nonzero(above_r[px:])[0]
    trc0 = int(px + idx[-1]) if idx.size else -1
    idx = np.nonzero(above_c[py:])[0]
    trc1 = int(py + idx[-1]) if idx.size else -1
    if min(blc0, blc1, trc0, trc1) < 0:
        raise ValueError("Unable to find the support on one of the coordinates")
    return SupportResult(pos, peak_val, (blc0, blc1), (trc0, trc1))


# --------------------------------------------------------------------------
# helpers shared by the gridders
# --------------------------------------------------------------------------
def interpolate_edge_values(f: np.ndarray) -> np.ndarray:
    """SphFuncVisGridder::interpolateEdgeValues in the vector's own type."""
    f = f.copy()
    t3 = f.dtype.type(3.0)
    f[0] = t3 * (f[1] - f[2]) + f[3]
    if f.shape[0] % 2 == 1:
        f[-1] = f[0]
    return f


def float_sum_sequential(x: np.ndarray) -> np.float32:
    """casacore sum(): std::accumulate in float over column-major order."""
    return np.cumsum(np.asarray(x, dtype=F32).ravel(order="F"), dtype=F32)[-1]


@dataclass
class CFCache:
    """itsConvFunc + itsConvFuncOffsets: CFs as complex64 arrays [x, y]."""
    cfs: list                      # index cInd -> np.ndarray (2S+1, 2S+1) complex64 or None
    offsets: list = field(default_factory=list)   # per plane before oversampling: (offU, offV)
    support: int = 0               # itsSupport

    def flatten(self):
        sizes = np.array([0 if c is None else c.shape[0] for c in self.cfs], dtype=np.int32)
        offs = np.zeros(len(self.cfs), dtype=np.int64)
        tot = 0
        for i, c in enumerate(self.cfs):
            offs[i] = tot
            if c is not None:
                tot += c.size
        data = np.zeros(tot, dtype=np.complex64)
        for i, c in enumerate(self.cfs):
            if c is not None:
                data[offs[i]:offs[i] + c.size] = c.ravel(order="F")
        return sizes, offs, data


# --------------------------------------------------------------------------
# SphFunc
# --------------------------------------------------------------------------
def sphfunc_cf(support: int = 3, oversample: int = 128, alpha: float = 1.0) -> CFCache:
    grdsf = SpheroidalFunction(math.pi * support, alpha)
    csize = 2 * support + 1
    cfs = [None] * (oversample * oversample)
    for fracv in range(oversample):
        for fracu in range(oversample):
            plane = fracu + oversample * fracv
            i = np.arange(csize)
            nux = np.abs((oversample * (i - support) + fracu).astype(np.float64)) / float(support * oversample)
            nuy = np.abs((oversample * (i - support) + fracv).astype(np.float64)) / float(support * oversample)
            bx = (grdsf(nux) * np.power(1.0 - nux * nux, float(alpha))).astype(F32)
            by = (grdsf(nuy) * np.power(1.0 - nuy * nuy, float(alpha))).astype(F32)
            cf = (bx[:, None] * by[None, :]).astype(F32)
            # norm = real(sum(abs(cf))) accumulated in float; cf /= Complex(norm)
            norm = float_sum_sequential(np.abs(cf))
            # limited-range complex division by (norm, 0): (a*c)/(c*c)
            cre = (cf * norm).astype(F32) / F32(norm * norm)
            cfs[plane] = cre.astype(np.complex64)
    return CFCache(cfs=cfs, offsets=[], support=support)


def sph_correction_vectors(shape, grdsf, interp: bool = True):
    """1-D correction factors of SphFuncVisGridder::correctConvolution (x and y)."""
    out = []
    for n in shape[:2]:
        half = n // 2
        nu = np.abs(np.arange(n, dtype=np.float64) - half) / float(half)
        buf = grdsf(nu).astype(np.complex64)
        if interp:
            buf = interpolate_edge_values(buf)
        support = 3
        max_before = buf[n // 2]
        buf = fft1d(buf, True)
        buf[: n // 2 - support] = 0
        buf[n // 2 + support + 1:] = 0
        buf = fft1d(buf, False)
        norm = np.complex64(max_before / buf[n // 2])
        buf = (buf * norm).astype(np.complex64)
        val = buf.real.astype(np.float64)
        ccf = np.where(np.abs(val) > 1e-10, 1.0 / np.where(val == 0, 1, val), 0.0)
        out.append(ccf)
    return out


def correct_convolution(img: np.ndarray, grdsf) -> np.ndarray:
    """Apply the spheroidal grid correction to an image [x, y, ...] (float32)."""
    ccfx, ccfy = sph_correction_vectors(img.shape, grdsf)
    fac = ccfx[:, None] * ccfy[None, :]
    ext = fac.reshape(fac.shape + (1,) * (img.ndim - 2))
    return (img.astype(np.float64) * ext).astype(F32)


# --------------------------------------------------------------------------
# WProject
# --------------------------------------------------------------------------
@dataclass
class WProjectParams:
    nwplanes: int = 65
    wmax: float = 35000.0
    cutoff: float = 1e-3
    oversample: int = 8
    maxsupport: int = 256
    limitsupport: int = 0
    alpha: float = 1.0
    variablesupport: bool = False
    offsetsupport: bool = False
    cutoff_absolute: bool = False
    wterms: np.ndarray | None = None   # w-term per plane (wavelengths)


def _extract_support(plane: np.ndarray, p: WProjectParams):
    ss = support_search(plane, p.cutoff, 1.0 if p.cutoff_absolute else -1.0)
    off_u = off_v = 0
    if p.offsetsupport:
        size = ss.support()
        # C++ integer division truncates toward zero
        off_u = int((ss.peak_pos[0] - plane.shape[0] // 2) / p.oversample)
        off_v = int((ss.peak_pos[1] - plane.shape[1] // 2) / p.oversample)
    else:
        size = ss.symmetrical_support(plane.shape)
        if not size > 0:
            raise ValueError("Unable to determine support of convolution function")
    size //= 2 * p.oversample
    if size < 3:
        size = 3
    return size, off_u, off_v


def _limit_support(s: int, limit: int) -> int:
    return limit if (limit > 0 and s > limit) else s


def wproject_taper(shape_x: int, shape_y: int, uvcell_u: float, uvcell_v: float,
                   p: WProjectParams, grdsf):
    """WProjectVisGridder::setup: buffer sizes, cell sizes, ccfx/ccfy (float)."""
    nx = ny = p.maxsupport
    qnx, qny = nx // p.oversample, ny // p.oversample
    cellx = 1.0 / (float(shape_x) * uvcell_u)
    celly = 1.0 / (float(shape_y) * uvcell_v)
    ccellx = float(shape_x) * cellx / float(qnx)
    ccelly = float(shape_y) * celly / float(qny)

    def ccf(q):
        i = np.arange(q)
        nu = (np.abs((i - q // 2).astype(F32)) / F32(q // 2)).astype(F32)
        v = (grdsf(nu.astype(np.float64)) / float(F32(q))).astype(F32)
        return interpolate_edge_values(v)

    return nx, ny, qnx, qny, ccellx, ccelly, ccf(qnx), ccf(qny)


def wproject_screen(nx, ny, qnx, qny, ccellx, ccelly, ccfx, ccfy, wterm: float) -> np.ndarray:
    """populateThisPlane: spheroidal x w phase screen, FP64 phase, FP32 store."""
    w = 2.0 * math.pi * wterm
    buf = np.zeros((nx, ny), dtype=np.complex64)
    iy = np.arange(qny)
    ix = np.arange(qnx)
    y2 = ((iy - qny // 2).astype(np.float64) * ccelly) ** 2
    x2 = ((ix - qnx // 2).astype(np.float64) * ccellx) ** 2
    r2 = x2[:, None] + y2[None, :]
    inside = r2 < 1.0
    phase = w * (1.0 - np.sqrt(np.where(inside, 1.0 - r2, 1.0)))
    wt = (ccfx[:, None] * ccfy[None, :]).astype(F32).astype(np.float64)
    re = (wt * np.cos(phase)).astype(F32)
    im = (-(wt * np.sin(phase))).astype(F32)
    val = np.where(inside, re + 1j * im, 0).astype(np.complex64)
    buf[nx // 2 - qnx // 2: nx // 2 - qnx // 2 + qnx, ny // 2 - qny // 2: ny // 2 - qny // 2 + qny] = val
    return buf


def _cut_planes(full: np.ndarray, support: int, off_u: int, off_v: int, os: int, rescale=None):
    nx, ny = full.shape
    out = {}
    i = np.arange(-support, support + 1)
    for fracu in range(os):
        kx = (i + off_u) * os + fracu + nx // 2
        for fracv in range(os):
            ky = (i + off_v) * os + fracv + ny // 2
            c = full[np.ix_(kx, ky)].astype(np.complex64)
            if rescale is not None:
                c = (c * F32(rescale)).astype(np.complex64)
            out[(fracu, fracv)] = c
    return out


def _check_overflow(support, off_u, off_v, os, nx, ny):
    kxmin = (-support + off_u) * os + nx // 2
    kxmax = (support + off_u) * os + os - 1 + nx // 2
    kymin = (-support + off_v) * os + ny // 2
    kymax = (support + off_v) * os + os - 1 + ny // 2
    ov = 0
    if kxmin < 0:
        ov = -kxmin
    if kxmax >= nx:
        ov = max(ov, kxmax - (nx - 1))
    if kymin < 0:
        ov = max(ov, -kymin)
    if kymax >= ny:
        ov = max(ov, kymax - (ny - 1))
    if ov != 0:
        raise ValueError("Convolution function overflowing - increase maxsupport or cutoff or decrease oversample")


def normalise_cf(c: np.ndarray) -> np.ndarray:
    """WProjectVisGridder::normalise for one CF: float sum of real parts, scale."""
    norm = float(float_sum_sequential(c.real))
    inv = F32(1.0 / norm)
    return (c * inv).astype(np.complex64)


def wproject_cf(shape_x, shape_y, uvcell_u, uvcell_v, p: WProjectParams,
                keep_planes: bool = False):
    """Full WProject CF cache. Returns CFCache (+ FFT'd planes when asked)."""
    grdsf = SpheroidalFunction(math.pi * 3, p.alpha)
    nx, ny, qnx, qny, ccellx, ccelly, ccfx, ccfy = wproject_taper(shape_x, shape_y, uvcell_u, uvcell_v, p, grdsf)
    os = p.oversample
    cfs = [None] * (p.nwplanes * os * os)
    offsets = [(0, 0)] * p.nwplanes
    its_support = 0
    planes = []
    for iw in range(p.nwplanes):
        buf = wproject_screen(nx, ny, qnx, qny, ccellx, ccelly, ccfx, ccfy, float(p.wterms[iw]))
        full = fft2d(buf, True)
        if keep_planes:
            planes.append(full)
        s_plane, off_u, off_v = its_support, 0, 0
        if p.variablesupport or its_support == 0:
            s_plane, off_u, off_v = _extract_support(full, p)
            if not ((s_plane + 1) * os < nx // 2):
                raise ValueError("Overflowing convolution function for w-plane %d" % iw)
            s_plane = _limit_support(s_plane, p.limitsupport)
            if its_support == 0:
                its_support = s_plane
        if p.offsetsupport:
            offsets[iw] = (off_u, off_v)
        support = s_plane if p.variablesupport else its_support
        _check_overflow(support, off_u, off_v, os, nx, ny)
        for (fu, fv), c in _cut_planes(full, support, off_u, off_v, os).items():
            cfs[fu + os * (fv + os * iw)] = c
    cfs = [normalise_cf(c) for c in cfs]
    cache = CFCache(cfs=cfs, offsets=offsets if p.offsetsupport else [], support=its_support)
    if keep_planes:
        return cache, planes
    return cache


# --------------------------------------------------------------------------
# AWProject with DiskIllumination
# --------------------------------------------------------------------------
@dataclass
class AWProjectParams(WProjectParams):
    diameter: float = 12.0
    blockage: float = 2.0
    maxfeeds: int = 1
    maxfields: int = 1
    frequencydependent: bool = True
    spheroidaltaper: bool = False
    maxsupport: int = 128
    oversample: int = 8
    wmax: float = 10000.0


def disk_pattern(nu_, nv_, uvcell_u, uvcell_v, os, freq, diameter, blockage, l, m):
    """DiskIllumination::getPattern into a (nU, nV) complex64 buffer."""
    cell_u = uvcell_u / os
    cell_v = uvcell_v / os
    l_scaled = 2. * math.pi * cell_u * l
    m_scaled = 2. * math.pi * cell_v * m
    if not abs(abs(cell_u / cell_v) - 1.) < 1e-7:
        raise ValueError("Rectangular cells are not supported at the moment")
    cell = abs(cell_u * (C_LIGHT / freq))
    radius = diameter / (2.0 * cell)
    rmax2 = radius * radius
    rmin2 = (blockage / (2.0 * cell)) ** 2
    if not rmax2 > rmin2:
        raise ValueError("Disk hole is supposed to be less than the disk size")
    if not (float(nu_) ** 2 > rmax2 and float(nv_) ** 2 > rmax2):
        raise ValueError("The pattern buffer passed to DiskIllumination::getPattern is too small")
    if rmin2 + 1 >= rmax2:
        rmin2 -= 1
    ou = np.arange(nu_, dtype=np.float64) - float(nu_) / 2.
    ov = np.arange(nv_, dtype=np.float64) - float(nv_) / 2.
    r2 = ou[:, None] ** 2 + ov[None, :] ** 2
    inside = (r2 >= rmin2) & (r2 <= rmax2)
    phase = l_scaled * ou[:, None] + m_scaled * ov[None, :]
    pat = np.where(inside, np.cos(phase).astype(F32) + 1j * (-np.sin(phase)).astype(F32), 0).astype(np.complex64)
    total = float(np.count_nonzero(inside))
    if not total > 0:
        raise ValueError("Integral of the disk should be non-zero")
    scale = F32(F32(F32(nu_) * F32(nv_)) / F32(total))
    return (pat * scale).astype(np.complex64)


def beam_offset_lm(image_centre, beam_centre):
    """(l, m) of a beam pointing relative to the image centre (DiskIllumination.cc:104-107)."""
    ra0, dec0 = image_centre
    ra, dec = beam_centre
    l = math.sin(ra - ra0) * math.cos(dec)
    m = math.sin(dec) * math.cos(dec0) - math.cos(dec) * math.sin(dec0) * math.cos(ra - ra0)
    return l, m


def awproject_plane(pattern_img: np.ndarray, p: AWProjectParams, uvcell_u, uvcell_v,
                    wterm: float, ccfx=None, ccfy=None) -> np.ndarray:
    """One w-plane of AWProject: |A|^2 x w screen -> forward FFT / (nx ny)."""
    nx = ny = p.maxsupport
    qnx, qny = nx // p.oversample, ny // p.oversample
    ccellx = 1.0 / (float(qnx) * uvcell_u)
    ccelly = 1.0 / (float(qny) * uvcell_v)
    w = 2.0 * math.pi * wterm
    iy = np.arange(ny)
    ix = np.arange(nx)
    y2 = ((iy.astype(np.float64) - float(ny) / 2) * ccelly) ** 2
    x2 = ((ix.astype(np.float64) - float(nx) / 2) * ccellx) ** 2
    qix = ix + qnx // 2 - nx // 2
    qiy = iy + qny // 2 - ny // 2
    r2 = x2[:, None] + y2[None, :]
    inside = r2 < 1.0
    if p.spheroidaltaper:
        inq = ((qix >= 0) & (qix < qnx))[:, None] & ((qiy >= 0) & (qiy < qny))[None, :]
        inside = inside & inq
        tx = np.where((qix >= 0) & (qix < qnx), ccfx[np.clip(qix, 0, qnx - 1)], 0.0)
        ty = np.where((qiy >= 0) & (qiy < qny), ccfy[np.clip(qiy, 0, qny - 1)], 0.0)
        taper = (tx[:, None] * ty[None, :]).astype(F32)
    else:
        taper = np.ones((nx, ny), dtype=F32)
    phase = w * (1.0 - np.sqrt(np.where(inside, 1.0 - r2, 1.0)))
    pr = pattern_img.real.astype(F32)
    pi_ = pattern_img.imag.astype(F32)
    # pattern * conj(pattern) in float, then * taper
    wre = (pr * pr - pi_ * (-pi_)).astype(F32)
    wim = (pr * (-pi_) + pi_ * pr).astype(F32)
    wre = (wre * taper).astype(F32)
    wim = (wim * taper).astype(F32)
    cr = np.cos(phase).astype(F32)
    ci = (-np.sin(phase)).astype(F32)
    vre = (wre * cr - wim * ci).astype(F32)
    vim = (wre * ci + wim * cr).astype(F32)
    buf = np.where(inside, vre + 1j * vim, 0).astype(np.complex64)
    if not np.any(inside & ((wre != 0) | (wim != 0))):
        raise ValueError("Convolution function is empty")
    full = fft2d(buf, True)
    return (full * F32(1.0 / (float(nx) * float(ny)))).astype(np.complex64)


def awproject_cf(uvcell_u, uvcell_v, p: AWProjectParams, freqs, feeds_pointing: dict,
                 image_centre=(0.0, 0.0), is_psf: bool = False, field: int = 0):
    """CF cache of AWProject for the feeds in ``feeds_pointing`` (feed -> (ra, dec)),
    filled in the order the reference fills it (feeds in first-row order)."""
    from .spheroidal import SpheroidalFunction as _SF
    nchan = len(freqs) if p.frequencydependent else 1
    os = p.oversample
    nw = p.nwplanes
    nplanes_total = nw * p.maxfeeds * p.maxfields * nchan
    cfs = [None] * (os * os * nplanes_total)
    offsets = [(0, 0)] * nplanes_total if p.offsetsupport else []
    nx = ny = p.maxsupport
    qnx, qny = nx // os, ny // os
    ccfx = ccfy = None
    if p.spheroidaltaper:
        g = _SF(math.pi * 3, p.alpha)
        ccfx = interpolate_edge_values(g(np.abs(np.arange(qnx) - float(qnx // 2)) / float(qnx // 2)))
        ccfy = interpolate_edge_values(g(np.abs(np.arange(qny) - float(qny // 2)) / float(qny // 2)))
    its_support = 0
    for feed, pointing in feeds_pointing.items():
        l, m = (0.0, 0.0) if is_psf else beam_offset_lm(image_centre, pointing)
        for chan in range(nchan):
            pat = disk_pattern(nx, ny, uvcell_u, uvcell_v, os, freqs[chan], p.diameter, p.blockage, l, m)
            pat_img = fft2d(pat, False)
            for iw in range(nw):
                full = awproject_plane(pat_img, p, uvcell_u, uvcell_v, float(p.wterms[iw]), ccfx, ccfy)
                z = iw + nw * (chan + nchan * (feed + p.maxfeeds * field))
                s_plane, off_u, off_v = its_support, 0, 0
                if p.variablesupport or its_support == 0:
                    s_plane, off_u, off_v = _extract_support(full, p)
                    if not ((s_plane + 1) * os < nx // 2):
                        raise ValueError("Overflowing convolution function")
                    s_plane = _limit_support(s_plane, p.limitsupport)
                    if its_support == 0:
                        its_support = s_plane
                    if p.offsetsupport:
                        offsets[z] = (off_u, off_v)
                support = s_plane if p.variablesupport else its_support
                _check_overflow(support, off_u, off_v, os, nx, ny)
                for (fu, fv), c in _cut_planes(full, support, off_u, off_v, os, rescale=float(os * os)).items():
                    cfs[fu + os * (fv + os * z)] = c
    return CFCache(cfs=cfs, offsets=offsets, support=its_support)


# --------------------------------------------------------------------------
# finalise / initialise (FFT side)
# --------------------------------------------------------------------------
def finalise_grid(grids, grdsf, padding: float = 1.0, screens=None) -> np.ndarray:
    """TableVisGridder::finaliseGrid (screens=None) or WStackVisGridder::finaliseGrid
    (screens = list of callables applied after the backward FFT).  grids: list of
    complex64 arrays [x, y, pol, chan]."""
    acc = None
    for i, g in enumerate(grids):
        if screens is not None and not np.max(np.abs(g)) > 0:
            continue
        s = fft2d(g.astype(np.complex64), False)
        if screens is not None:
            s = screens[i](s)
        r = s.real.astype(F32)
        acc = r if acc is None else (acc + r).astype(F32)
    acc = correct_convolution(acc, grdsf)
    acc = (acc * F32(float(acc.shape[0]) * float(acc.shape[1]))).astype(F32)
    return extract_padded(acc, padding)


def extract_padded(a: np.ndarray, padding: float):
    if padding == 1.0:
        return a
    nx = int(round(a.shape[0] / padding))
    ny = int(round(a.shape[1] / padding))
    x0 = (a.shape[0] - nx) // 2
    y0 = (a.shape[1] - ny) // 2
    return a[x0:x0 + nx, y0:y0 + ny]


def initialise_degrid(image: np.ndarray, grdsf) -> np.ndarray:
    """TableVisGridder::initialiseDegrid (padding 1): correct, complex, forward FFT."""
    s = correct_convolution(image.astype(F32), grdsf)
    return fft2d(s.astype(np.complex64), True)


def wstack_screen(shape_x, shape_y, uvcell_u, uvcell_v, wterm):
    """Returns a function applying WStackVisGridder::multiply (FP32 screen)."""
    cellx = F32(1.0 / (float(F32(shape_x)) * uvcell_u))
    celly = F32(1.0 / (float(F32(shape_y)) * uvcell_v))
    w = F32(2.0 * math.pi * wterm)
    y = ((np.arange(shape_y) - shape_y // 2).astype(F32) * celly).astype(F32)
    x = ((np.arange(shape_x) - shape_x // 2).astype(F32) * cellx).astype(F32)
    y2 = (y * y).astype(F32)
    x2 = (x * x).astype(F32)
    r2 = (x2[:, None] + y2[None, :]).astype(F32)
    inside = r2 < 1.0
    phase = (w.astype(np.float64) * (1.0 - np.sqrt(1.0 - np.where(inside, r2, 0).astype(np.float64)))).astype(F32)
    cr = np.cos(phase).astype(F32)
    ci = (-np.sin(phase)).astype(F32)

    def apply(m):
        m = m.copy()
        nz = (np.abs(m) > 0) & inside.reshape(inside.shape + (1,) * (m.ndim - 2))
        cre = cr.reshape(cr.shape + (1,) * (m.ndim - 2))
        cim = ci.reshape(ci.shape + (1,) * (m.ndim - 2))
        re = (m.real * cre - m.imag * cim).astype(F32)
        im = (m.real * cim + m.imag * cre).astype(F32)
        return np.where(nz, re + 1j * im, m).astype(np.complex64)

    return apply


def wstack_initialise_degrid(image, grdsf, screens):
    s = correct_convolution(image.astype(F32), grdsf).astype(np.complex64)
    out = []
    for sc in screens:
        work = np.conj(sc(s)).astype(np.complex64)
        out.append(fft2d(work, True))
    return out


# --------------------------------------------------------------------------
# AWProject finaliseWeights
# --------------------------------------------------------------------------
def fft_pad(a: np.ndarray, nxo: int, nyo: int) -> np.ndarray:
    """Fourier-domain interpolation of a real plane to (nxo, nyo), values kept:
    complex copy scaled by the area ratio, forward transform, the spectrum in
    the centre of a zero grid, backward transform, real part.  Restated from
    the steps of SynthesisParamsHelper::oversample with norm = true
    (askap/measurementequation/SynthesisParamsHelper.cc:918-951); the
    reference calls base-scimath's PaddingUtils::fftPad (un-vendored), whose
    exact scaling is not pinned."""
    cnx, cny = a.shape
    if (cnx, cny) == (nxo, nyo):
        return a.astype(F32)
    A = fft2d(a.astype(np.complex64) * F32(float(nxo) * float(nyo) / (float(cnx) * float(cny))), True)
    B = np.zeros((nxo, nyo), dtype=np.complex64)
    x0, y0 = (nxo - cnx) // 2, (nyo - cny) // 2
    B[x0:x0 + cnx, y0:y0 + cny] = A
    return fft2d(B, False).real.astype(F32)


def aw_finalise_weights(cfs, sumw, os_, track_per_os, offsets, maxsupport, nx, ny, onx, ony, grdsf=None,
                        weights_cutoff=0.0):
    """AWProjectVisGridder::finaliseWeights (AWProjectVisGridder.cc:616-766):
    for every sum-of-weights row with data, the CF of its first oversampling
    plane, centred in a min(maxsupport, n) grid, backward-transformed
    (unnormalised); wt |val|^2 summed per (pol, chan) in row order, then
    Fourier-padded to the (padded) image and its centre (onx, ony) kept.
    With a spheroidal taper (grdsf given, :641-664, :735-745) the taper
    grdsf(|i - c| / c), zero at or below weights_cutoff, edge interpolated,
    is divided out of each transformed CF where it is positive."""
    nz, npol, nchan = sumw.shape
    cnx, cny = min(maxsupport, nx), min(maxsupport, ny)
    ccx, ccy = cnx // 2, cny // 2
    taper = None
    if grdsf is not None:
        def tap(n, c):
            val = grdsf(np.abs(np.arange(n, dtype=np.float64) - float(c)) / float(c))
            return interpolate_edge_values(np.where(val > weights_cutoff, val, 0.0))
        taper = (tap(cnx, ccx)[:, None] * tap(cny, ccy)[None, :]).astype(F32)
    cout = np.zeros((cnx, cny, npol, nchan), dtype=F32)
    for iz in range(nz):
        if not np.any(sumw[iz] > 0):
            continue
        plane = iz if track_per_os else os_ * os_ * iz
        c = cfs[plane]
        s = (c.shape[0] - 1) // 2
        ou, ov = offsets[iz] if offsets else (0, 0)
        buf = np.zeros((cnx, cny), dtype=np.complex64)
        for iy in range(-s, s + 1):
            for ix in range(-s, s + 1):
                xp, yp = ix + ccx + ou, iy + ccy + ov
                if 0 <= xp < cnx and 0 <= yp < cny:
                    buf[xp, yp] = c[ix + s, iy + s]
        val = (fft2d(buf, False) * F32(float(cnx) * float(cny))).astype(np.complex64)
        vr, vi = val.real.astype(F32), val.imag.astype(F32)
        if taper is not None:
            pos = taper > 0
            safe = np.where(pos, taper, F32(1.0))
            vr = np.where(pos, vr / safe, F32(0.0)).astype(F32)
            vi = np.where(pos, vi / safe, F32(0.0)).astype(F32)
        r = (vr * vr - vi * (-vi)).astype(F32)
        for ch in range(nchan):
            for p in range(npol):
                wt = float(sumw[iz, p, ch])
                cout[:, :, p, ch] = (cout[:, :, p, ch].astype(np.float64) + wt * r.astype(np.float64)).astype(F32)
    out = np.zeros((onx, ony, npol, nchan), dtype=F32)
    x0, y0 = (nx - onx) // 2, (ny - ony) // 2
    for ch in range(nchan):
        for p in range(npol):
            full = fft_pad(cout[:, :, p, ch], nx, ny)
            out[:, :, p, ch] = full[x0:x0 + onx, y0:y0 + ony]
    return out
