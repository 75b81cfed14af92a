"""Python binding of the B200 gridder's C-ABI (include/yg.h).

Mirrors yandasoft's gridder interface so that callers and tests read like the
reference's own: ``VisGridderFactory.make(parset)`` returns an ``IVisGridder``
with ``initialiseGrid / grid / finaliseGrid / finaliseWeights /
initialiseDegrid / degrid / finaliseDegrid / customiseForContext /
initVisWeights / isModelEmpty / clone`` (askap/gridding/IVisGridder.h:64-140,
VisGridderFactory.cc:112-285).  Failures raise ``AskapError`` carrying the
library's status code, as ASKAPCHECK throws in the reference.

The CUDA library must be built (``yandasoft_b200.build``); there is no CPU
fallback: without the extension every call fails loudly.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libyg_b200.so")
_LIB = None

P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64
D = ctypes.c_double

# names exported by include/yg.h
EXPORTS = [
    "yg_last_error", "yg_create", "yg_clone", "yg_destroy", "yg_initialise_grid", "yg_grid", "yg_finalise_grid",
    "yg_finalise_weights", "yg_initialise_degrid", "yg_degrid", "yg_finalise_degrid", "yg_customise_for_context",
    "yg_init_vis_weights_mfs", "yg_is_model_empty", "yg_get_support", "yg_get_cf", "yg_get_cf_offsets",
    "yg_get_sum_weights", "yg_get_grid", "yg_get_shape", "yg_get_stats", "yg_build_cf", "yg_plan_create",
    "yg_plan_grid", "yg_plan_degrid", "yg_plan_info", "yg_plan_samples", "yg_plan_destroy", "yg_set_tile", "yg_set_item_size",
    "yg_synchronize", "yg_get_stream", "yg_get_kernel_times", "yg_kernel_launch_count",
    "yg_set_grid_variant", "yg_degrid_noalloc", "yg_mlp_nparams", "yg_learned_train", "yg_set_cf_form",
    "yg_learned_get_params", "yg_learned_set_params", "yg_mlp_loss_grad", "yg_mlp_eval",
    "yg_cycle_create", "yg_cycle_run", "yg_cycle_info", "yg_cycle_destroy", "yg_autotune", "yg_autotune_reset",
    "yg_cycle_create_roles", "yg_sort_pairs", "yg_scan_i32",
]


class AskapError(RuntimeError):
    """Error raised by the gridder (status code in ``.code``)."""

    def __init__(self, code, msg):
        super().__init__("%s (code %d)" % (msg, code))
        self.code = code


class yg_axes(ctypes.Structure):
    _fields_ = [("cell", D * 2), ("centre", D * 2), ("tangent", D * 2), ("has_freq", I32), ("reserved", I32),
                ("freq_start", D), ("freq_end", D)]


class yg_learn_params(ctypes.Structure):
    _fields_ = [("ntrain", I64), ("batch", I32), ("steps", I32), ("lr", D), ("seed", ctypes.c_uint64),
                ("nwplanes_train", I32), ("reserved", I32)]


class yg_learn_report(ctypes.Structure):
    _fields_ = [("final_loss", D), ("train_ms", ctypes.c_float), ("steps", I32), ("scale", ctypes.c_float),
                ("cf_table_bytes", D), ("network_bytes", D)]


class yg_tune_report(ctypes.Structure):
    _fields_ = [("tile", I32), ("items", I32), ("variant", I32), ("trials", I32), ("best_ms", ctypes.c_float),
                ("default_ms", ctypes.c_float), ("cf_width", I32), ("npol", I32)]


class yg_chunk(ctypes.Structure):
    _fields_ = [("nrow", I64), ("nchan", I32), ("npol", I32), ("uvw", P), ("delay", P), ("freq", P), ("vis", P),
                ("noise", P), ("flag", P), ("feed1", P), ("pointing", P), ("on_device", I32), ("reserved", I32)]


def load(path: str | None = None):
    """Loads libyg_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    p = path or LIBPATH
    if not os.path.exists(p):
        raise AskapError(2, "CUDA gridder library %s is missing: run yandasoft_b200.build.build()" % p)
    L = ctypes.CDLL(p)
    L.yg_last_error.restype = ctypes.c_char_p
    L.yg_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(P)]
    L.yg_clone.argtypes = [P, ctypes.POINTER(P)]
    L.yg_destroy.argtypes = [P]
    L.yg_destroy.restype = None
    L.yg_initialise_grid.argtypes = [P, ctypes.POINTER(yg_axes), I32, I32, I32, I32, I32, I32]
    L.yg_grid.argtypes = [P, ctypes.POINTER(yg_chunk)]
    L.yg_finalise_grid.argtypes = [P, P, I32]
    L.yg_finalise_weights.argtypes = [P, P, I32]
    L.yg_initialise_degrid.argtypes = [P, ctypes.POINTER(yg_axes), I32, I32, I32, I32, P, I32]
    L.yg_degrid.argtypes = [P, ctypes.POINTER(yg_chunk)]
    L.yg_finalise_degrid.argtypes = [P]
    L.yg_customise_for_context.argtypes = [P, ctypes.c_char_p]
    L.yg_init_vis_weights_mfs.argtypes = [P, D]
    L.yg_is_model_empty.argtypes = [P, ctypes.POINTER(I32)]
    L.yg_get_support.argtypes = [P, ctypes.POINTER(I32), ctypes.POINTER(I32), ctypes.POINTER(I32)]
    L.yg_get_cf.argtypes = [P, P, P, P, I64]
    L.yg_get_cf_offsets.argtypes = [P, P, I32, ctypes.POINTER(I32)]
    L.yg_get_sum_weights.argtypes = [P, P, I64, ctypes.POINTER(I32)]
    L.yg_get_grid.argtypes = [P, P, I64, ctypes.POINTER(I32)]
    L.yg_get_shape.argtypes = [P] + [ctypes.POINTER(I32)] * 4
    L.yg_get_stats.argtypes = [P, P]
    L.yg_build_cf.argtypes = [P]
    L.yg_plan_create.argtypes = [P, ctypes.POINTER(yg_chunk), ctypes.POINTER(P)]
    L.yg_plan_grid.argtypes = [P, P, ctypes.POINTER(yg_chunk)]
    L.yg_plan_degrid.argtypes = [P, P, ctypes.POINTER(yg_chunk)]
    L.yg_plan_info.argtypes = [P, ctypes.POINTER(I64), ctypes.POINTER(I32), ctypes.POINTER(I32)]
    L.yg_plan_samples.argtypes = [P, P, P, P, P, P]
    L.yg_plan_destroy.argtypes = [P]
    L.yg_plan_destroy.restype = None
    L.yg_set_tile.argtypes = [P, I32]
    L.yg_set_item_size.argtypes = [P, I32]
    L.yg_set_grid_variant.argtypes = [P, I32]
    L.yg_degrid_noalloc.argtypes = [P, ctypes.POINTER(yg_chunk)]
    L.yg_cycle_create_roles.argtypes = [I32, P, P, ctypes.POINTER(P)]
    L.yg_synchronize.argtypes = [P]
    L.yg_get_stream.argtypes = [P, ctypes.POINTER(P)]
    L.yg_get_kernel_times.argtypes = [P, P]
    L.yg_kernel_launch_count.restype = I64
    L.yg_kernel_launch_count.argtypes = []
    L.yg_mlp_nparams.restype = I32
    L.yg_mlp_nparams.argtypes = []
    L.yg_learned_train.argtypes = [P, ctypes.POINTER(yg_learn_params), ctypes.POINTER(yg_learn_report)]
    L.yg_set_cf_form.argtypes = [P, I32]
    L.yg_learned_get_params.argtypes = [P, P, ctypes.POINTER(ctypes.c_float)]
    L.yg_learned_set_params.argtypes = [P, P, ctypes.c_float]
    L.yg_mlp_loss_grad.argtypes = [P, P, P, I64, ctypes.c_float, P, ctypes.POINTER(D)]
    L.yg_mlp_eval.argtypes = [P, P, I64, P]
    L.yg_sort_pairs.argtypes = [P, P, I64, I32]
    L.yg_scan_i32.argtypes = [P, P, I64, I32, I32]
    L.yg_cycle_create.argtypes = [I32, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(yg_chunk),
                                  ctypes.POINTER(P)]
    L.yg_cycle_run.argtypes = [P, I32, ctypes.POINTER(ctypes.c_float)]
    L.yg_cycle_info.argtypes = [P, ctypes.POINTER(I64)]
    L.yg_cycle_destroy.argtypes = [P]
    L.yg_cycle_destroy.restype = None
    L.yg_autotune.argtypes = [P, ctypes.POINTER(yg_chunk), I32, ctypes.POINTER(yg_tune_report)]
    L.yg_autotune_reset.argtypes = []
    L.yg_autotune_reset.restype = None
    _LIB = L
    return L


def _check(rc):
    if rc != 0:
        raise AskapError(rc, load().yg_last_error().decode())


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


@dataclass
class Axes:
    """Image axes: direction increments (rad), image centre and tangent point,
    optional FREQUENCY axis (start, end) in Hz."""
    cell_x: float
    cell_y: float
    centre: tuple = (0.0, 0.0)
    tangent: tuple = (0.0, 0.0)
    freq: tuple | None = None

    def c(self):
        a = yg_axes()
        a.cell[0], a.cell[1] = self.cell_x, self.cell_y
        a.centre[0], a.centre[1] = self.centre
        a.tangent[0], a.tangent[1] = self.tangent
        if self.freq is not None:
            a.has_freq = 1
            a.freq_start, a.freq_end = self.freq
        return a


class Accessor:
    """A chunk of visibilities (IConstDataAccessor / IDataAccessor unpacked).

    numpy arrays (host) or torch CUDA tensors (device).  Cubes are
    (nrow, nchan, npol) complex64 in Fortran order (row fastest)."""

    def __init__(self, uvw, freq, vis, noise=None, flag=None, delay=None, feed1=None, pointing=None, shape=None):
        self.uvw, self.freq, self.vis = uvw, freq, vis
        self.noise, self.flag, self.delay, self.feed1, self.pointing = noise, flag, delay, feed1, pointing
        self.on_device = hasattr(vis, "data_ptr")
        if not self.on_device:
            self.uvw = np.ascontiguousarray(uvw, dtype=np.float64)
            self.freq = np.ascontiguousarray(freq, dtype=np.float64)
            if not (vis.dtype == np.complex64 and vis.flags.f_contiguous):
                raise AskapError(1, "vis must be a Fortran-ordered complex64 cube")
            if noise is not None:
                self.noise = np.asfortranarray(noise, dtype=np.complex64)
            if flag is not None:
                self.flag = np.asfortranarray(flag.astype(np.uint8))
            if delay is not None:
                self.delay = np.ascontiguousarray(delay, dtype=np.float64)
            if feed1 is not None:
                self.feed1 = np.ascontiguousarray(feed1, dtype=np.int32)
        if pointing is not None:
            self.pointing = np.ascontiguousarray(pointing, dtype=np.float64)
        shp = tuple(shape) if shape is not None else tuple(vis.shape)
        self.nrow, self.nchan, self.npol = shp

    def to_device(self, device="cuda"):
        """Copy of this host accessor with every array in torch device memory
        (same memory layout; cubes stay column-major)."""
        import torch

        def dev(a, dt=None):
            if a is None:
                return None
            a = np.asarray(a)
            flat = a.ravel(order="K") if (a.flags.f_contiguous or a.flags.c_contiguous) else a.ravel(order="F")
            if np.iscomplexobj(flat):
                flat = flat.view(np.float32 if flat.dtype == np.complex64 else np.float64)
            return torch.from_numpy(np.ascontiguousarray(flat)).to(device)

        return Accessor(dev(self.uvw), dev(self.freq), dev(self.vis), noise=dev(self.noise), flag=dev(self.flag),
                        delay=dev(self.delay), feed1=dev(self.feed1), pointing=self.pointing,
                        shape=(self.nrow, self.nchan, self.npol))

    def vis_numpy(self):
        """The visibility cube as a (nrow, nchan, npol) complex64 Fortran array."""
        if not self.on_device:
            return self.vis
        # the tensor's memory, in its own (contiguous) order, is the column-major cube
        flat = self.vis.detach().contiguous().cpu().numpy().view(np.complex64).reshape(-1)
        return flat.reshape((self.nrow, self.nchan, self.npol), order="F")

    def c(self):
        c = yg_chunk()
        c.nrow, c.nchan, c.npol = self.nrow, self.nchan, self.npol
        c.uvw, c.delay, c.freq = _ptr(self.uvw), _ptr(self.delay), _ptr(self.freq)
        c.vis, c.noise, c.flag = _ptr(self.vis), _ptr(self.noise), _ptr(self.flag)
        c.feed1 = _ptr(self.feed1)
        c.pointing = None if self.pointing is None else self.pointing.ctypes.data
        c.on_device = 1 if self.on_device else 0
        return c


class Plan:
    def __init__(self, gridder, acc: Accessor):
        self._lib = load()
        self.h = P()
        self._chunk = acc.c()
        _check(self._lib.yg_plan_create(gridder.h, ctypes.byref(self._chunk), ctypes.byref(self.h)))

    def samples(self, gridder, acc: "Accessor"):
        """(iu, iv, cfi, status) per sample, (nrow, nchan) Fortran arrays."""
        n = acc.nrow * acc.nchan
        iu = np.zeros(n, dtype=np.int32)
        iv = np.zeros(n, dtype=np.int32)
        c = np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.uint8)
        _check(self._lib.yg_plan_samples(gridder.h, self.h, iu.ctypes.data, iv.ctypes.data, c.ctypes.data,
                                         st.ctypes.data))
        shp = (acc.nrow, acc.nchan)
        return (iu.reshape(shp, order="F"), iv.reshape(shp, order="F"), c.reshape(shp, order="F"),
                st.reshape(shp, order="F"))

    def info(self):
        nv, ni, t = I64(), I32(), I32()
        _check(self._lib.yg_plan_info(self.h, ctypes.byref(nv), ctypes.byref(ni), ctypes.byref(t)))
        return dict(nvalid=nv.value, nitems=ni.value, tile=t.value)

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            self._lib.yg_plan_destroy(self.h)
            self.h = P()


class IVisGridder:
    """Handle on one gridder instance (owns a CUDA stream and device memory)."""

    def __init__(self, handle):
        self._lib = load()
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            self._lib.yg_destroy(self.h)
            self.h = P()

    def clone(self) -> "IVisGridder":
        out = P()
        _check(self._lib.yg_clone(self.h, ctypes.byref(out)))
        return IVisGridder(out)

    # ---- gridding ----
    def initialiseGrid(self, axes: Axes, shape, dopsf=False, dopcf=False):
        nx, ny, npol, nchan = shape
        self._shape = tuple(shape)
        _check(self._lib.yg_initialise_grid(self.h, ctypes.byref(axes.c()), nx, ny, npol, nchan, int(dopsf), int(dopcf)))

    def grid(self, acc: Accessor):
        c = acc.c()
        _check(self._lib.yg_grid(self.h, ctypes.byref(c)))

    def finaliseGrid(self, out=None):
        nx, ny, npol, nchan = self._shape
        if out is None:
            out = np.zeros((nx, ny, npol, nchan), dtype=np.float32, order="F")
        on_dev = 1 if hasattr(out, "data_ptr") else 0
        _check(self._lib.yg_finalise_grid(self.h, _ptr(out), on_dev))
        return out

    def finaliseWeights(self, out=None):
        nx, ny, npol, nchan = self._shape
        if out is None:
            out = np.zeros((nx, ny, npol, nchan), dtype=np.float32, order="F")
        _check(self._lib.yg_finalise_weights(self.h, _ptr(out), 1 if hasattr(out, "data_ptr") else 0))
        return out

    # ---- degridding ----
    def initialiseDegrid(self, axes: Axes, image):
        if hasattr(image, "data_ptr"):
            nx, ny, npol, nchan = image.shape_fortran if hasattr(image, "shape_fortran") else image.shape
            on_dev = 1
        else:
            image = np.asfortranarray(image, dtype=np.float32)
            nx, ny, npol, nchan = image.shape
            on_dev = 0
        self._shape = (nx, ny, npol, nchan)
        self._model = image
        _check(self._lib.yg_initialise_degrid(self.h, ctypes.byref(axes.c()), nx, ny, npol, nchan, _ptr(image), on_dev))

    def degrid(self, acc: Accessor):
        c = acc.c()
        _check(self._lib.yg_degrid(self.h, ctypes.byref(c)))

    def degrid_noalloc(self, acc: Accessor):
        """degrid() for a device-resident chunk that allocates no device memory
        (scratch in a static device array; see include/yg.h)."""
        c = acc.c()
        _check(self._lib.yg_degrid_noalloc(self.h, ctypes.byref(c)))

    def finaliseDegrid(self):
        _check(self._lib.yg_finalise_degrid(self.h))

    def customiseForContext(self, context: str):
        _check(self._lib.yg_customise_for_context(self.h, context.encode()))

    def initVisWeights(self, reffreq: float):
        """VisWeightsMultiFrequency(reffreq)."""
        _check(self._lib.yg_init_vis_weights_mfs(self.h, float(reffreq)))

    def isModelEmpty(self) -> bool:
        v = I32()
        _check(self._lib.yg_is_model_empty(self.h, ctypes.byref(v)))
        return bool(v.value)

    # ---- learned convolution function (no counterpart in the reference) ----
    def learned_train(self, ntrain=1 << 22, batch=16384, steps=60000, lr=1e-2, seed=1, nwplanes_train=0):
        """Trains the CF network on this gridder's tabulated CFs (or a denser
        table of nwplanes_train planes); returns the training report."""
        lp = yg_learn_params(int(ntrain), int(batch), int(steps), float(lr), int(seed), int(nwplanes_train), 0)
        r = yg_learn_report()
        _check(self._lib.yg_learned_train(self.h, ctypes.byref(lp), ctypes.byref(r)))
        return {k: getattr(r, k) for k, _ in yg_learn_report._fields_}

    def set_cf_form(self, form):
        """0: tabulated CFs, 1: the learned network."""
        _check(self._lib.yg_set_cf_form(self.h, int(form)))

    def learned_params(self):
        p = np.zeros(mlp_nparams(), dtype=np.float32)
        sc = ctypes.c_float()
        _check(self._lib.yg_learned_get_params(self.h, p.ctypes.data, ctypes.byref(sc)))
        return p, sc.value

    def set_learned_params(self, params, scale):
        p = np.ascontiguousarray(params, dtype=np.float32)
        _check(self._lib.yg_learned_set_params(self.h, p.ctypes.data, float(scale)))

    # ---- autotuner (no counterpart in the reference) ----
    def autotune(self, acc: Accessor, max_trials=12):
        """Times (tile, samples per item, thread layout) candidates on a
        device-resident chunk; keeps the fastest for this CF width class."""
        c = acc.c()
        r = yg_tune_report()
        _check(self._lib.yg_autotune(self.h, ctypes.byref(c), int(max_trials), ctypes.byref(r)))
        return {k: getattr(r, k) for k, _ in yg_tune_report._fields_}

    # ---- plans (repeated passes over resident data) ----
    def plan(self, acc: Accessor) -> Plan:
        return Plan(self, acc)

    def grid_plan(self, plan: Plan, acc: Accessor):
        c = acc.c()
        _check(self._lib.yg_plan_grid(self.h, plan.h, ctypes.byref(c)))

    def degrid_plan(self, plan: Plan, acc: Accessor):
        c = acc.c()
        _check(self._lib.yg_plan_degrid(self.h, plan.h, ctypes.byref(c)))

    def synchronize(self):
        _check(self._lib.yg_synchronize(self.h))

    def stream_handle(self) -> int:
        """cudaStream_t (as an int) on which this gridder launches its kernels."""
        sp = P()
        _check(self._lib.yg_get_stream(self.h, ctypes.byref(sp)))
        return sp.value or 0

    def set_tile(self, t: int):
        _check(self._lib.yg_set_tile(self.h, int(t)))

    def set_grid_variant(self, v: int):
        _check(self._lib.yg_set_grid_variant(self.h, int(v)))

    def set_item_size(self, v: int):
        _check(self._lib.yg_set_item_size(self.h, int(v)))

    # ---- inspection ----
    def support(self):
        s, o, n = I32(), I32(), I32()
        _check(self._lib.yg_get_support(self.h, ctypes.byref(s), ctypes.byref(o), ctypes.byref(n)))
        return s.value, o.value, n.value

    def build_cf(self):
        _check(self._lib.yg_build_cf(self.h))

    def convolution_functions(self):
        """List of CF matrices (complex64 [x, y]) indexed like itsConvFunc."""
        _, _, ncf = self.support()
        sizes = np.zeros(ncf, dtype=np.int32)
        offs = np.zeros(ncf, dtype=np.int64)
        _check(self._lib.yg_get_cf(self.h, sizes.ctypes.data, offs.ctypes.data, None, 0))
        total = int(np.max(offs + sizes.astype(np.int64) ** 2)) if ncf else 0
        data = np.zeros(total, dtype=np.complex64)
        _check(self._lib.yg_get_cf(self.h, sizes.ctypes.data, offs.ctypes.data, data.ctypes.data, total))
        out = []
        for i in range(ncf):
            n = int(sizes[i])
            out.append(None if n == 0 else data[offs[i]:offs[i] + n * n].reshape((n, n), order="F"))
        return out

    def cf_bytes(self) -> int:
        """Bytes of the tabulated CF cache (every matrix, unpadded)."""
        _, _, ncf = self.support()
        if ncf == 0:
            return 0
        sizes = np.zeros(ncf, dtype=np.int32)
        offs = np.zeros(ncf, dtype=np.int64)
        _check(self._lib.yg_get_cf(self.h, sizes.ctypes.data, offs.ctypes.data, None, 0))
        return int(np.sum(sizes.astype(np.int64) ** 2) * 8)

    def cf_offsets(self):
        n = I32()
        _check(self._lib.yg_get_cf_offsets(self.h, None, 0, ctypes.byref(n)))
        buf = np.zeros(2 * max(1, n.value), dtype=np.int32)
        _check(self._lib.yg_get_cf_offsets(self.h, buf.ctypes.data, n.value, ctypes.byref(n)))
        return [tuple(buf[2 * i:2 * i + 2]) for i in range(n.value)]

    def sum_weights(self):
        rows = I32()
        _check(self._lib.yg_get_sum_weights(self.h, None, 0, ctypes.byref(rows)))
        nx, ny, npol, nchan = self.shape()
        out = np.zeros((rows.value, npol, nchan), dtype=np.float64, order="F")
        _check(self._lib.yg_get_sum_weights(self.h, out.ctypes.data, out.size, ctypes.byref(rows)))
        return out

    def shape(self):
        a, b, c, d = I32(), I32(), I32(), I32()
        _check(self._lib.yg_get_shape(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d)))
        return a.value, b.value, c.value, d.value

    def grids(self):
        n = I32()
        _check(self._lib.yg_get_grid(self.h, None, 0, ctypes.byref(n)))
        nx, ny, npol, nchan = self.shape()
        buf = np.zeros(n.value * nx * ny * npol * nchan, dtype=np.complex64)
        _check(self._lib.yg_get_grid(self.h, buf.ctypes.data, buf.size, ctypes.byref(n)))
        per = nx * ny * npol * nchan
        return [buf[i * per:(i + 1) * per].reshape((nx, ny, npol, nchan), order="F") for i in range(n.value)]

    def kernel_times(self):
        out = np.zeros(4)
        _check(self._lib.yg_get_kernel_times(self.h, out.ctypes.data))
        return dict(kgrid_ms=out[0], kgrid_calls=out[1], kdegrid_ms=out[2], kdegrid_calls=out[3])

    def stats(self):
        out = np.zeros(8)
        _check(self._lib.yg_get_stats(self.h, out.ctypes.data))
        keys = ["samples_gridded", "taps_gridded", "samples_degridded", "taps_degridded", "ms_grid", "ms_degrid",
                "ms_cf", "cf_planes"]
        return dict(zip(keys, out.tolist()))


class yg_cycle_roles(ctypes.Structure):
    _fields_ = [("model", P), ("residual", P), ("psf", P), ("pcf", P)]


class MajorCycle:
    """degrid -> subtract -> grid for n instances, recorded once as one CUDA
    graph (each instance on a branch of its own) and replayed per cycle.
    degridders[i] holds the model (initialiseDegrid), gridders[i] receives the
    residual (initialiseGrid), accessors[i] are device-resident observed
    chunks; psf[i] / pcf[i] (optional, None entries allowed) grid the PSF
    (initialiseGrid with dopsf) and the preconditioner function (dopcf) from
    the same buffer.  See yg_cycle_create and yg_cycle_create_roles."""

    def __init__(self, degridders, gridders, accessors, psf=None, pcf=None):
        self._lib = load()
        n = len(degridders)
        if not (len(gridders) == n == len(accessors)):
            raise AskapError(1, "one degridder, gridder and accessor per instance")
        psf = list(psf) if psf is not None else [None] * n
        pcf = list(pcf) if pcf is not None else [None] * n
        if len(psf) != n or len(pcf) != n:
            raise AskapError(1, "one PSF and one preconditioner entry per instance")
        self._keep = (list(degridders), list(gridders), list(accessors), psf, pcf)
        ch = (yg_chunk * n)(*[a.c() for a in accessors])
        self.h = P()
        if all(g is None for g in psf + pcf):
            dg = (P * n)(*[g.h for g in degridders])
            gg = (P * n)(*[g.h for g in gridders])
            self._arrays = (dg, gg, ch)
            _check(self._lib.yg_cycle_create(n, dg, gg, ch, ctypes.byref(self.h)))
        else:
            roles = (yg_cycle_roles * n)(*[yg_cycle_roles(d.h, g.h, None if s is None else s.h,
                                                          None if c is None else c.h)
                                           for d, g, s, c in zip(degridders, gridders, psf, pcf)])
            self._arrays = (roles, ch)
            _check(self._lib.yg_cycle_create_roles(n, ctypes.cast(roles, P), ctypes.cast(ch, P), ctypes.byref(self.h)))

    def run(self, cycles=1) -> float:
        """Replays the graph `cycles` times; returns the GPU milliseconds."""
        ms = ctypes.c_float()
        _check(self._lib.yg_cycle_run(self.h, int(cycles), ctypes.byref(ms)))
        return ms.value

    def nodes(self) -> int:
        n = I64()
        _check(self._lib.yg_cycle_info(self.h, ctypes.byref(n)))
        return n.value

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            self._lib.yg_cycle_destroy(self.h)
            self.h = P()


def autotune_reset():
    """Forgets every process-wide autotuner choice."""
    load().yg_autotune_reset()


def mlp_nparams() -> int:
    return int(load().yg_mlp_nparams())


def mlp_loss_grad(params, X, T, scale=1.0):
    """(loss, gradient) of the learned-CF network on the GPU for taps X (n x 5)
    with targets T (n x 2): loss = scale * sum |y - t|^2."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    g = np.zeros(mlp_nparams(), dtype=np.float32)
    loss = D()
    _check(load().yg_mlp_loss_grad(p.ctypes.data, X.ctypes.data, T.ctypes.data, X.shape[0], float(scale),
                                   g.ctypes.data, ctypes.byref(loss)))
    return loss.value, g


def mlp_eval(params, X):
    """Network outputs (n x 2) for inputs X (n x 5), weights rounded to FP16."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.zeros((X.shape[0], 2), dtype=np.float32)
    _check(load().yg_mlp_eval(p.ctypes.data, X.ctypes.data, X.shape[0], Y.ctypes.data))
    return Y


def sort_pairs(keys, vals, end_bit=64):
    """The plan builder's stable radix sort on host copies: (keys, vals) sorted
    by bits [0, end_bit) of the uint64 keys, equal keys in input order."""
    k = np.array(keys, dtype=np.uint64, copy=True)
    v = np.array(vals, dtype=np.uint32, copy=True)
    if k.shape != v.shape or k.ndim != 1:
        raise ValueError("keys and vals must be 1-D arrays of one length")
    _check(load().yg_sort_pairs(k.ctypes.data, v.ctypes.data, k.size, int(end_bit)))
    return k, v


def scan_i32(x, op="sum", exclusive=False):
    """The plan builder's device scan of an int32 array (op sum, min or max)."""
    a = np.array(x, dtype=np.int32, copy=True).reshape(-1)
    out = np.empty_like(a)
    _check(load().yg_scan_i32(a.ctypes.data, out.ctypes.data, a.size, {"sum": 0, "min": 1, "max": 2}[op],
                              int(bool(exclusive))))
    return out


def kernel_launch_count() -> int:
    """Process-wide number of the library's own kernel launches."""
    return int(load().yg_kernel_launch_count())


class VisGridderFactory:
    @staticmethod
    def make(parset) -> IVisGridder:
        """parset: dict or 'key = value' text (keys as in a cimager parset)."""
        if isinstance(parset, dict):
            text = "\n".join("%s = %s" % (k, _fmt(v)) for k, v in parset.items())
        else:
            text = parset
        lib = load()
        h = P()
        _check(lib.yg_create(text.encode(), ctypes.byref(h)))
        return IVisGridder(h)


def _fmt(v):
    if isinstance(v, bool):
        return "true" if v else "false"
    return str(v)
