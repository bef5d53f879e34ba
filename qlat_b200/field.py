"""Lattice geometry, RngState and GPU-resident fields, mirroring qlat's
``Geometry``, ``RngState``, ``GaugeField`` (qcd.pyx:45-88), ``GaugeMomentum``
(hmc.pyx:39-53), ``FieldRealD`` and ``GaugeAction`` (gauge_action.pyx:18-36).

A field lives in GPU memory behind a C ABI handle (include/qlat_b200.h).
``np.asarray(field)`` downloads it in the reference memory image
(shape ``(V, multiplicity, 3, 3)`` complex128 for color matrices,
``(V, multiplicity)`` float64 for real fields, sites x-fastest);
``field.from_numpy(arr)`` uploads.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import call

F64 = 64
F32 = 32
KIND_COLOR_MATRIX = 0
KIND_REAL = 1


class Coordinate(tuple):
    """Minimal stand-in for qlat.Coordinate (a 4-tuple of ints)."""

    def __new__(cls, x=(0, 0, 0, 0)):
        v = tuple(int(a) for a in x)
        assert len(v) == 4
        return super().__new__(cls, v)

    def to_list(self):
        return list(self)

    def volume(self):
        return int(np.prod(self))


class Geometry:
    """qlat.Geometry(total_site) for one node (core.h:92-359)."""

    def __init__(self, total_site=None):
        self.total_site = Coordinate(total_site if total_site is not None else (1, 1, 1, 1))

    @property
    def total_volume(self) -> int:
        return self.total_site.volume()

    @property
    def local_volume(self) -> int:
        return self.total_volume

    def __eq__(self, other):
        return isinstance(other, Geometry) and self.total_site == other.total_site

    def __repr__(self):
        return f"Geometry({list(self.total_site)})"

    def show(self):
        return repr(self)

    def xg_arr(self) -> np.ndarray:
        """Global coordinates of the sites, shape (V, 4) int32, x fastest
        (Geometry.xg_arr, geometry.pyx)."""
        X, Y, Z, T = self.total_site
        i = np.arange(self.total_volume, dtype=np.int64)
        return np.stack([i % X, (i // X) % Y, (i // (X * Y)) % Z, i // (X * Y * Z)], axis=1).astype(np.int32)


class RngState:
    """qlat.RngState (rng-state.h:38-99): a SHA-256 counter RNG; the state is
    the 24 x uint32 serialised form of the reference (rng-state.cpp:61-81)."""

    def __init__(self, seed: str | int | None = None):
        self._v = (ctypes.c_uint32 * 24)()
        if seed is None:
            # reset(rs) (rng-state.cpp:150-164): initial SHA-256 hash (first 32
            # fractional bits of the square roots of the first 8 primes), no
            # bytes hashed, type = ULONG_MAX
            h0 = [math.isqrt(p << 64) & 0xFFFFFFFF for p in (2, 3, 5, 7, 11, 13, 17, 19)]
            v = [0, 0] + h0 + [0xFFFFFFFF, 0xFFFFFFFF] + [0] * 12
            for i in range(24):
                self._v[i] = v[i]
        else:
            call("qgb_rng_seed", self._v, str(seed).encode())

    @classmethod
    def _from(cls, arr) -> "RngState":
        r = cls.__new__(cls)
        r._v = (ctypes.c_uint32 * 24)(*list(arr))
        return r

    def copy(self) -> "RngState":
        return RngState._from(list(self._v))

    def split(self, sindex) -> "RngState":
        out = (ctypes.c_uint32 * 24)()
        call("qgb_rng_split", out, self._v, str(sindex).encode())
        return RngState._from(list(out))

    def rand_gen(self) -> int:
        o = ctypes.c_uint64()
        call("qgb_rng_rand_gen", self._v, ctypes.byref(o))
        return int(o.value)

    def u_rand_gen(self, upper: float = 1.0, lower: float = 0.0) -> float:
        o = ctypes.c_double()
        call("qgb_rng_u_rand_gen", self._v, upper, lower, ctypes.byref(o))
        return o.value

    def g_rand_gen(self, center: float = 0.0, sigma: float = 1.0) -> float:
        o = ctypes.c_double()
        call("qgb_rng_g_rand_gen", self._v, center, sigma, ctypes.byref(o))
        return o.value

    def c_rand_gen(self, size) -> Coordinate:
        """c_rand_gen (coordinate.h:305-310): the coordinate of site
        rand_gen() % volume(size), x fastest."""
        size = Coordinate(size)
        ri = self.rand_gen() % size.volume()
        x = []
        for n in size:
            x.append(ri % n)
            ri //= n
        return Coordinate(x)

    def export(self) -> np.ndarray:
        return np.array(list(self._v), dtype=np.uint32)

    @property
    def c(self):
        return self._v


class GaugeAction:
    """qlat.GaugeAction(beta, c1) (gauge-action.h:8-28): Wilson c1 = 0,
    Iwasaki c1 = -0.331, DBW2 c1 = -1.4008."""

    def __init__(self, beta: float = 5.5, c1: float = 0.0):
        self._beta = float(beta)
        self._c1 = float(c1)

    def beta(self) -> float:
        return self._beta

    def c1(self) -> float:
        return self._c1

    def __repr__(self):
        return f"GaugeAction(beta={self._beta}, c1={self._c1})"


class Field:
    """A lattice field in GPU memory (Field<M>, core.h:753-969)."""

    _kind = KIND_COLOR_MATRIX

    def __init__(self, geo: Geometry | None = None, multiplicity: int = 1, *, precision: int = F64,
                 kind: int | None = None):
        self._h = None
        self.geo = geo
        self.multiplicity = int(multiplicity)
        self.precision = int(precision)
        self.kind = self._kind if kind is None else int(kind)
        if geo is not None:
            self._create()

    def _create(self):
        h = ctypes.c_void_p()
        call("qgb_field_create", ctypes.byref(h), _lib.i32x4(*self.geo.total_site), self.multiplicity,
             self.kind, self.precision)
        self._h = h

    def init(self, geo: Geometry, multiplicity: int | None = None):
        self._free()
        self.geo = geo
        if multiplicity is not None:
            self.multiplicity = int(multiplicity)
        self._create()

    def _free(self):
        if self._h is not None and self._h.value:
            try:
                _lib.load().qgb_field_destroy(self._h)
            except Exception:
                pass
        self._h = None

    def __del__(self):
        self._free()

    @property
    def handle(self) -> ctypes.c_void_p:
        if self._h is None:
            raise RuntimeError("field is not initialised (no geometry)")
        return self._h

    def _like(self) -> "Field":
        f = self.__class__.__new__(self.__class__)
        Field.__init__(f, self.geo, self.multiplicity, precision=self.precision, kind=self.kind)
        return f

    def copy(self, precision: int | None = None) -> "Field":
        f = self._like()
        if precision is not None and precision != self.precision:
            f._free()
            f.precision = precision
            f._create()
        call("qgb_field_copy", f.handle, self.handle)
        return f

    def __imatmul__(self, other: "Field"):
        """f @= g: copy (with precision conversion), qlat's field assignment."""
        if self._h is None:
            self.geo = other.geo
            self.multiplicity = other.multiplicity
            self._create()
        call("qgb_field_copy", self.handle, other.handle)
        return self

    def __imul__(self, s: float):
        call("qgb_field_axpby", self.handle, 0.0, None, float(s))
        return self

    def __iadd__(self, other: "Field"):
        call("qgb_field_axpby", self.handle, 1.0, other.handle, 1.0)
        return self

    def __isub__(self, other: "Field"):
        call("qgb_field_axpby", self.handle, -1.0, other.handle, 1.0)
        return self

    def set_zero(self):
        call("qgb_field_set_zero", self.handle)

    def qnorm(self) -> float:
        o = ctypes.c_double()
        call("qgb_field_qnorm", self.handle, ctypes.byref(o))
        return o.value

    def _shape(self):
        V = self.geo.total_volume
        if self.kind == KIND_COLOR_MATRIX:
            return (V, self.multiplicity, 3, 3), np.complex128
        return (V, self.multiplicity), np.float64

    def to_numpy(self) -> np.ndarray:
        shape, dt = self._shape()
        a = np.empty(shape, dtype=dt)
        call("qgb_field_download", self.handle, a.ctypes.data_as(_lib.c_dbl_p))
        return a

    def __array__(self, dtype=None, copy=None):
        a = self.to_numpy()
        return a if dtype is None else a.astype(dtype)

    def from_numpy(self, arr) -> "Field":
        shape, dt = self._shape()
        a = np.ascontiguousarray(np.asarray(arr, dtype=dt).reshape(shape))
        call("qgb_field_upload", self.handle, a.ctypes.data_as(_lib.c_dbl_p))
        return self

    def upload_host(self, ptr: int) -> None:
        """Copy from host memory at address `ptr` (e.g. a pinned torch tensor)
        in the reference memory image."""
        call("qgb_field_upload", self.handle, ctypes.cast(ctypes.c_void_p(ptr), _lib.c_dbl_p))

    def upload_host_pipelined(self, ptr_now: int, ptr_next: int | None = None) -> None:
        """Copy the host image at ``ptr_now`` into the field and start copying the
        one at ``ptr_next`` to the GPU behind the work that follows, for the next
        call to commit (``qgb_field_upload_pipelined``; pinned host memory)."""
        call("qgb_field_upload_pipelined", self.handle, ctypes.c_void_p(ptr_now),
             None if ptr_next is None else ctypes.c_void_p(ptr_next))

    def download_host_async(self, ptr: int) -> None:
        """Queue a copy of the field, in the reference memory image, into host
        memory at ``ptr`` (pinned) without waiting; the data is there after
        ``qlat_b200.synchronize()`` (``qgb_field_download_async``)."""
        call("qgb_field_download_async", self.handle, ctypes.c_void_p(ptr))

    def upload_device(self, ptr: int) -> None:
        """Copy from a device buffer (e.g. a torch CUDA tensor's data_ptr) in
        the reference memory image."""
        call("qgb_field_upload_device", self.handle, ctypes.c_void_p(ptr))

    def download_device(self, ptr: int) -> None:
        call("qgb_field_download_device", self.handle, ctypes.c_void_p(ptr))

    def set_rand(self, rng: RngState, upper: float = 1.0, lower: float = 0.0):
        """set_u_rand (field_types.pyx.in:194-196, core.h:1585-1603): per site
        rng.newtype(site index), one uniform draw in [lower, upper) per real."""
        call("qgb_field_set_u_rand", self.handle, rng.c, float(upper), float(lower))

    def set_rand_g(self, rng: RngState, center: float = 0.0, sigma: float = 1.0):
        """set_g_rand (field_types.pyx.in:198-200, core.h:1617-1636)."""
        call("qgb_field_set_g_rand", self.handle, rng.c, float(center), float(sigma))

    def _selection(self, sel) -> np.ndarray | None:
        """A boolean selection of the (site, component) entries as one byte per
        entry, or None for other indexes."""
        if isinstance(sel, np.ndarray) and sel.dtype == np.bool_ and sel.shape == (self.geo.total_volume,
                                                                                   self.multiplicity):
            return np.ascontiguousarray(sel, dtype=np.uint8)
        return None

    def __getitem__(self, idx):
        """``field[idx]``: a copy of the indexed entries of the reference
        memory image (numpy indexing on the downloaded field)."""
        return self.to_numpy()[idx]

    def __setitem__(self, idx, value):
        """``field[idx] = value``.  A boolean selection of (site, component)
        entries with a scalar (real fields) or with ``other.selected(sel)``
        runs on the GPU; other indexes edit the downloaded image and upload
        it."""
        mask = self._selection(idx)
        if mask is not None and isinstance(value, _Selected) and value.sel is idx:
            call("qgb_field_set_selected", self.handle, value.field.handle, mask.ctypes.data_as(ctypes.c_void_p),
                 mask.size)
            return
        if mask is not None and self.kind == KIND_REAL and np.isscalar(value):
            call("qgb_field_fill", self.handle, float(value), mask.ctypes.data_as(ctypes.c_void_p), mask.size)
            return
        if isinstance(value, _Selected):
            value = value.field.to_numpy()[value.sel]
        a = self.to_numpy()
        a[idx] = value
        self.from_numpy(a)

    def selected(self, sel) -> "_Selected":
        """The entries of a boolean selection, for ``dst[sel] = src.selected(sel)``
        (a GPU copy of the selected entries)."""
        return _Selected(self, sel)


class _Selected:
    def __init__(self, field: Field, sel):
        self.field = field
        self.sel = sel


class FieldColorMatrix(Field):
    _kind = KIND_COLOR_MATRIX


class FieldRealD(Field):
    _kind = KIND_REAL

    def glb_sum(self) -> np.ndarray:
        """Sum over the lattice of each component, shape (1, multiplicity)."""
        from .topo_measure import glb_sum
        return glb_sum(self)

    def glb_sum_tslice(self, *, t_dir: int = 3) -> np.ndarray:
        """Per-timeslice sums (field_base.pyx:750-762), shape (T, multiplicity)."""
        from .topo_measure import glb_sum_tslice
        return glb_sum_tslice(self, t_dir=t_dir)

    def glb_min(self) -> np.ndarray:
        from .topo_measure import glb_min
        return glb_min(self)

    def glb_max(self) -> np.ndarray:
        from .topo_measure import glb_max
        return glb_max(self)


class GaugeField(FieldColorMatrix):
    """qlat.GaugeField (qcd.pyx:45-88)."""

    def __init__(self, geo: Geometry | None = None, multiplicity: int = 4, *, precision: int = F64):
        assert multiplicity == 4
        super().__init__(geo, 4, precision=precision)

    def set_rand(self, rng: RngState, sigma: float = 0.5, n_step: int = 1):
        call("qgb_gf_set_rand", self.handle, rng.c, float(sigma), int(n_step))

    def set_unit(self):
        call("qgb_set_unit", self.handle)

    def unitarize(self):
        call("qgb_unitarize", self.handle)

    def plaq(self) -> float:
        from .hmc import gf_avg_plaq
        return gf_avg_plaq(self)

    def save(self, path: str, *, ensemble_id: str | None = None, ensemble_label: str | None = None,
             creator: str | None = None, beta: float = 0.0, sequence_num: int = 0) -> int:
        """Save in the NERSC format (qcd.pyx:55-60 -> save_gauge_field, qcd.h:146-181);
        returns the number of data bytes written."""
        n = ctypes.c_int64()
        enc = lambda v: None if v is None else str(v).encode()  # noqa: E731
        call("qgb_save_gauge_field", self.handle, str(path).encode(), enc(ensemble_id), enc(ensemble_label),
             enc(creator), float(beta), int(sequence_num), ctypes.byref(n))
        return n.value

    def load(self, path: str) -> int:
        """Load a NERSC file (qcd.pyx:62-67 -> load_gauge_field, qcd.h:183-250),
        taking the file's lattice; returns the number of data bytes read.  A
        checksum mismatch is reported with a warning, as the reference does."""
        info = read_gauge_field_header(path)
        ts = tuple(info["total_site"])
        if self.geo is None or tuple(self.geo.total_site) != ts or self._h is None:
            self.init(Geometry(ts))
        checks = ctypes.c_int32()
        n = ctypes.c_int64()
        call("qgb_load_gauge_field", self.handle, str(path).encode(), ctypes.byref(checks), ctypes.byref(n))
        if not checks.value & 1 or not checks.value & 2:
            import warnings
            warnings.warn(f"load_gauge_field: '{path}': checksum mismatch "
                          f"(CRC32HASH {'ok' if checks.value & 1 else 'differs'}, "
                          f"CHECKSUM {'ok' if checks.value & 2 else 'differs'})")
        return n.value


def read_gauge_field_header(path: str) -> dict:
    """The header of a NERSC gauge file (read_gauge_field_header, qcd.h:94-144)."""
    ts = _lib.i32x4()
    rows, big = ctypes.c_int32(), ctypes.c_int32()
    plaq, trace = ctypes.c_double(), ctypes.c_double()
    simple, crc = ctypes.c_uint32(), ctypes.c_uint32()
    call("qgb_nersc_read_header", str(path).encode(), ts, ctypes.byref(rows), ctypes.byref(big),
         ctypes.byref(plaq), ctypes.byref(trace), ctypes.byref(simple), ctypes.byref(crc))
    return {"total_site": list(ts), "n_rows": rows.value, "big_endian": big.value, "plaq": plaq.value,
            "link_trace": trace.value, "simple_checksum": simple.value, "crc32": crc.value}


class GaugeMomentum(FieldColorMatrix):
    """qlat.GaugeMomentum (hmc.pyx:39-53)."""

    def __init__(self, geo: Geometry | None = None, multiplicity: int = 4, *, precision: int = F64):
        assert multiplicity == 4
        super().__init__(geo, 4, precision=precision)

    def set_rand(self, rng: RngState, sigma: float = 1.0):
        call("qgb_set_rand_gauge_momentum", self.handle, float(sigma), rng.c)

    def set_rand_fa(self, mf: "FieldRealD", rng: RngState):
        """set_rand_gauge_momentum(gm, mf, rs) (hmc.pyx:51-52, hmc.cpp:121-149)."""
        call("qgb_set_rand_gauge_momentum_fa", self.handle, mf.handle, rng.c)


def set_unit(gf: Field, coef: float = 1.0):
    """field.h set_unit (everything.pxd:187): coef times the unit matrix in
    every entry of a color-matrix field, coef in every entry of a real field."""
    if gf.kind == KIND_REAL:
        call("qgb_field_fill", gf.handle, float(coef), None, 0)
        return
    call("qgb_set_unit", gf.handle)
    if coef != 1.0:
        gf *= coef
