"""Field containers mirroring jax-fli's field pytrees (reference _src/base/_core.py:175-516,
fields/particles.py, fields/density.py, fields/lightcone.py, fields/painting.py).

A field holds a CUDA tensor in `array` plus the same static metadata the reference
carries (mesh_size, box_size, observer_position, nside, status, unit, ...). Painting,
readout and power spectra dispatch to the B200 kernels through `jfli_b200.ops`.
"""

from __future__ import annotations

import dataclasses
from enum import Enum, auto
from typing import Any

import numpy as np
import torch

from . import ops

DEFAULT_CHUNK_SIZE = 2**24


class FieldStatus(str, Enum):
    UNKNOWN = auto()
    INITIAL_FIELD = auto()
    LPT1 = auto()
    LPT2 = auto()
    DENSITY_FIELD = auto()
    PARTICLES = auto()
    PROJECTED_DENSITY = auto()
    LIGHTCONE = auto()
    KAPPA = auto()
    GAMMA = auto()


class PhysicalUnit(str, Enum):
    INVALID_UNIT = auto()


class PositionUnit(str, Enum):
    GRID_RELATIVE = auto()
    GRID_ABSOLUTE = auto()
    MPC_H = auto()


class DensityUnit(str, Enum):
    OVERDENSITY = auto()
    DENSITY = auto()
    COUNTS = auto()
    MSUN_H_PER_MPC3 = auto()


class ConvergenceUnit(str, Enum):
    DIMENSIONLESS = auto()
    EFFECTIVE_DENSITY = auto()


@dataclasses.dataclass(frozen=True)
class PaintingOptions:
    """Painting configuration (reference fields/painting.py:15-96)."""

    target: str
    scheme: str = "bilinear"
    kernel_width_arcmin: float | None = None
    smoothing_interpretation: str = "fwhm"
    paint_nside: int | None = None
    ud_grade_power: float = 0.0
    ud_grade_order_in: str = "RING"
    ud_grade_order_out: str = "RING"
    ud_grade_pess: bool = False
    chunk_size: int = DEFAULT_CHUNK_SIZE
    weights: Any = 1.0
    batch_size: int | None = None

    def __post_init__(self):
        if self.target not in ("spherical", "flat", "density", "particles"):
            raise ValueError(f"unknown painting target {self.target!r}")
        if self.scheme not in ("ngp", "bilinear", "rbf_neighbor"):
            raise ValueError(f"unknown spherical scheme {self.scheme!r}")


def _weights_arg(weights):
    """Split a painting weight into (per-particle tensor or None, scalar)."""
    if weights is None:
        return None, 1.0
    if isinstance(weights, torch.Tensor):
        if weights.ndim == 0:
            return None, float(weights)
        return weights.to(torch.float32).contiguous(), 1.0
    if isinstance(weights, np.ndarray):
        if weights.ndim == 0:
            return None, float(weights)
        return torch.as_tensor(weights, dtype=torch.float32, device="cuda").contiguous(), 1.0
    return None, float(weights)


@dataclasses.dataclass(frozen=True, eq=False)
class AbstractField:
    array: Any
    mesh_size: tuple
    box_size: tuple
    z_sources: Any = None
    scale_factors: Any = None
    comoving_centers: Any = None
    density_width: Any = None
    observer_position: tuple = (0.5, 0.5, 0.5)
    sharding: Any = None
    halo_size: tuple = (0, 0)
    nside: int | None = None
    flatsky_npix: tuple | None = None
    field_size: float | None = None
    status: FieldStatus = FieldStatus.UNKNOWN
    unit: Any = PhysicalUnit.INVALID_UNIT

    def __post_init__(self):
        if not (isinstance(self.mesh_size, tuple) and len(self.mesh_size) == 3):
            raise ValueError(f"mesh_size must be a tuple of 3, got {self.mesh_size}")
        if not (isinstance(self.box_size, tuple) and len(self.box_size) == 3):
            raise ValueError(f"box_size must be a tuple of 3, got {self.box_size}")
        if any(not 0.0 <= f <= 1.0 for f in self.observer_position):
            raise ValueError("observer_position entries must lie within [0, 1]")
        if self.sharding is not None:
            raise NotImplementedError("jfli_b200 runs on one GPU; sharded fields are not supported")
        if self.nside is not None and self.nside <= 0:
            raise ValueError(f"nside must be positive, got {self.nside}")

    def replace(self, **kw):
        return dataclasses.replace(self, **kw)

    @property
    def observer_position_mpc(self) -> tuple:
        return tuple(f * L for f, L in zip(self.observer_position, self.box_size))

    @property
    def max_comoving_radius(self) -> float:
        box = np.asarray(self.box_size, dtype=np.float64)
        fr = np.clip(np.asarray(self.observer_position, dtype=np.float64), 0.0, 1.0)
        return float(np.min(box / (1.0 + 2.0 * np.minimum(fr, 1.0 - fr))))

    @classmethod
    def FromDensityMetadata(cls, array, field: "AbstractField", **kw):
        base = dict(mesh_size=field.mesh_size, box_size=field.box_size, observer_position=field.observer_position,
                    halo_size=field.halo_size, nside=field.nside, flatsky_npix=field.flatsky_npix,
                    field_size=field.field_size, status=field.status, unit=field.unit,
                    scale_factors=field.scale_factors, z_sources=field.z_sources,
                    comoving_centers=field.comoving_centers, density_width=field.density_width)
        base.update(kw)
        return cls(array=array, **base)

    def _meta(self, **kw):
        d = {f.name: getattr(self, f.name) for f in dataclasses.fields(self) if f.name != "array"}
        d.update(kw)
        return d

    def is_batched(self) -> bool:
        return self.array.ndim > self._core_ndim()

    def is_multi_batched(self) -> bool:
        """True for an (N, S, ...) field: a simulation batch N and a snapshot batch S
        (reference fields/density.py:491, fields/lightcone.py:441,858, fields/particles.py:635)."""
        return self.array.ndim == self._core_ndim() + 2

    # ------------------------------------------ array shorthands (reference _src/base/_core.py:25-171)
    @property
    def shape(self) -> tuple:
        return tuple(self.array.shape)

    @property
    def ndim(self) -> int:
        return self.array.ndim

    @property
    def size(self) -> int:
        return int(self.array.numel()) if isinstance(self.array, torch.Tensor) else int(np.size(self.array))

    @property
    def dtype(self):
        return self.array.dtype

    def __len__(self) -> int:
        return len(self.array)

    def __iter__(self):
        """The entries along the first dimension, each a field of this class."""
        for i in range(len(self)):
            yield self[i]

    # Arithmetic acts on the array and keeps the metadata of the left-hand field; another
    # field contributes its array.
    @staticmethod
    def _operand(other):
        return other.array if isinstance(other, AbstractField) else other

    def __add__(self, other):
        return self.replace(array=self.array + self._operand(other))

    def __radd__(self, other):
        return self.replace(array=self._operand(other) + self.array)

    def __sub__(self, other):
        return self.replace(array=self.array - self._operand(other))

    def __rsub__(self, other):
        return self.replace(array=self._operand(other) - self.array)

    def __mul__(self, other):
        return self.replace(array=self.array * self._operand(other))

    def __rmul__(self, other):
        return self.replace(array=self._operand(other) * self.array)

    def __truediv__(self, other):
        return self.replace(array=self.array / self._operand(other))

    def __rtruediv__(self, other):
        return self.replace(array=self._operand(other) / self.array)

    def __neg__(self):
        return self.replace(array=-self.array)

    def __pos__(self):
        return self

    def __abs__(self):
        return self.replace(array=abs(self.array))

    def _reduce(self, name: str, axis=None, keepdims: bool = False):
        a = self.array
        if isinstance(a, torch.Tensor):
            if name == "std":  # population standard deviation, as numpy's and jnp's default
                return torch.std(a, correction=0) if axis is None else torch.std(a, dim=axis, correction=0,
                                                                                 keepdim=keepdims)
            fn = {"min": torch.amin, "max": torch.amax, "mean": torch.mean}[name]
            if axis is None:
                return fn(a) if not keepdims else fn(a, dim=tuple(range(a.ndim)), keepdim=True)
            return fn(a, dim=axis, keepdim=keepdims)
        return getattr(np, name)(a, axis=axis, keepdims=keepdims)

    def min(self, axis=None, keepdims: bool = False):
        return self._reduce("min", axis, keepdims)

    def max(self, axis=None, keepdims: bool = False):
        return self._reduce("max", axis, keepdims)

    def mean(self, axis=None, keepdims: bool = False):
        return self._reduce("mean", axis, keepdims)

    def std(self, axis=None, keepdims: bool = False):
        return self._reduce("std", axis, keepdims)

    def transpose(self, *axes):
        a = self.array
        if len(axes) == 1 and isinstance(axes[0], (tuple, list)):
            axes = tuple(axes[0])
        if isinstance(a, torch.Tensor):
            return self.replace(array=a.permute(*(axes or tuple(reversed(range(a.ndim))))))
        return self.replace(array=np.transpose(a, axes or None))

    @property
    def T(self):
        return self.transpose()

    def apply_fn(self, fn, *args, **kwargs):
        """A field of this class holding fn(array, *args, **kwargs)."""
        return self.replace(array=fn(self.array, *args, **kwargs))

    def __array__(self, dtype=None, copy=None):
        a = self.array
        if isinstance(a, torch.Tensor):
            a = a.detach().cpu().numpy()
        return np.asarray(a, dtype=dtype)

    def block_until_ready(self):
        """Waits for the device work that produces the array."""
        if isinstance(self.array, torch.Tensor) and self.array.is_cuda:
            torch.cuda.synchronize(self.array.device)
        return self

    def to_metadata(self) -> "FieldMetadata":
        """The metadata alone, as a FieldMetadata with no array (reference _src/base/_core.py:478-496)."""
        return FieldMetadata(array=None, **self._meta())

    @classmethod
    def full_like(cls, field: "AbstractField", fill_value: float = 0.0):
        """A field of this class with field's metadata, filled with fill_value; each concrete
        class gives its own array shape (reference _src/base/_core.py:339-355)."""
        raise NotImplementedError("full_like must be implemented in subclasses.")

    @staticmethod
    def _full(shape, fill_value, like):
        a = getattr(like, "array", None)
        if isinstance(a, torch.Tensor):
            return torch.full(tuple(shape), float(fill_value), dtype=torch.float32, device=a.device)
        device = "cuda" if torch.cuda.is_available() else "cpu"
        return torch.full(tuple(shape), float(fill_value), dtype=torch.float32, device=device)

    def _core_ndim(self) -> int:
        return 3

    _DYNAMIC = ("z_sources", "scale_factors", "comoving_centers", "density_width")

    @classmethod
    def _join(cls, fields, how: str):
        """Stack or concatenate the arrays and the dynamic metadata of fields whose static
        metadata agree (reference _src/base/_core.py:248-282, a tree map over the array leaves)."""
        first = fields[0]
        static = [f.name for f in dataclasses.fields(first) if f.name != "array" and f.name not in cls._DYNAMIC]
        for f in fields[1:]:
            if type(f) is not type(first):
                raise ValueError(f"cannot {how} fields of types {type(first).__name__} and {type(f).__name__}")
            for name in static:
                a, b = getattr(f, name), getattr(first, name)
                same = (np.array_equal(np.asarray(a), np.asarray(b))
                        if isinstance(a, (np.ndarray, tuple, list)) or isinstance(b, (np.ndarray, tuple, list))
                        else a == b)
                if not same:
                    raise ValueError(f"cannot {how} fields whose {name} differ")
        arrays = [f.array for f in fields]
        if isinstance(arrays[0], torch.Tensor):
            array = torch.stack(arrays) if how == "stack" else torch.cat(arrays)
        else:
            array = np.stack(arrays) if how == "stack" else np.concatenate(arrays)

        def meta(name):
            vals = [getattr(f, name) for f in fields]
            if all(v is None for v in vals):
                return None
            if any(v is None for v in vals):
                raise ValueError(f"cannot {how} fields where only some carry {name}")
            vals = [v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else np.asarray(v, np.float64)
                    for v in vals]
            return np.stack(vals) if how == "stack" else np.concatenate(vals)

        return first.replace(array=array, **{name: meta(name) for name in cls._DYNAMIC})

    @classmethod
    def stack(cls, fields):
        """Stack fields along a new axis 0: (S, ...) inputs give an (N, S, ...) multi-batched
        field. Multi-batched inputs are refused; concat joins those."""
        fields = tuple(fields)
        if not fields:
            raise ValueError("stack requires at least one field.")
        if any(f.is_multi_batched() for f in fields):
            raise ValueError("Cannot stack multi-batched (N, S, ...) fields: the extra leading dimension would be "
                             "ambiguous. Use <FieldClass>.concat(fields) to join along the N axis instead.")
        return cls._join(fields, "stack")

    @classmethod
    def concat(cls, fields):
        """Concatenate multi-batched (N, S, ...) fields along the N axis."""
        fields = tuple(fields)
        if not fields:
            raise ValueError("concat requires at least one field.")
        if any(not f.is_multi_batched() for f in fields):
            raise ValueError("concat only works on multi-batched (N, S, ...) fields. Use stack() to create an "
                             "(N, S, ...) field from (S, ...) inputs.")
        return cls._join(fields, "concat")

    def __getitem__(self, key):
        if not self.is_batched():
            raise ValueError("indexing requires a batched field")
        sub = lambda v: v[key] if (isinstance(v, (torch.Tensor, np.ndarray)) and getattr(v, "ndim", 0) >= 1) else v
        return self.replace(array=self.array[key], scale_factors=sub(self.scale_factors),
                            z_sources=sub(self.z_sources), comoving_centers=sub(self.comoving_centers),
                            density_width=sub(self.density_width))


def _stack(rows):
    return torch.stack(rows) if isinstance(rows[0], torch.Tensor) else np.stack(rows)


def _linear_resize_weights(n_in: int, n_out: int) -> np.ndarray:
    """(n_in, n_out) weights of jax.image.resize's "bilinear" method along one axis (its
    scale_and_translate with a triangle kernel, antialiased, no translation): output pixel j
    samples the input at (j + 0.5) n_in / n_out - 0.5; the kernel is widened by n_in / n_out
    when downsampling; weights are normalised per output pixel (zero when their sum is
    negligible) and zero for samples outside [-0.5, n_in - 0.5]."""
    inv = n_in / n_out
    width = max(inv, 1.0)
    sample = (np.arange(n_out, dtype=np.float64) + 0.5) * inv - 0.5
    w = np.maximum(0.0, 1.0 - np.abs(sample[None, :] - np.arange(n_in, dtype=np.float64)[:, None]) / width)
    total = w.sum(axis=0, keepdims=True)
    w = np.where(np.abs(total) > 1000.0 * float(np.finfo(np.float32).eps), w / np.where(total != 0, total, 1.0), 0.0)
    inside = (sample >= -0.5) & (sample <= n_in - 0.5)
    return np.where(inside[None, :], w, 0.0)


def _cl_transfer(field, other, **kw) -> "PowerSpectrum":
    """sqrt(C_other / C_self) of two map fields (reference fields/lightcone.py:318-365,746-788)."""
    cl_self = field.angular_cl(**kw)
    cl_other = other.angular_cl(**kw)
    return PowerSpectrum(wavenumber=cl_self.wavenumber, array=(cl_other.array / cl_self.array) ** 0.5,
                         name="transfer", scale_factors=field.scale_factors)


def _cl_coherence(field, other, **kw) -> "PowerSpectrum":
    """C_cross / sqrt(C_self C_other) of two map fields (reference fields/lightcone.py:367-421,790-838)."""
    cl_self = field.angular_cl(**kw)
    cl_other = other.angular_cl(**kw)
    cl_cross = field.angular_cl(other, **kw)
    return PowerSpectrum(wavenumber=cl_self.wavenumber, array=cl_cross.array / (cl_self.array * cl_other.array) ** 0.5,
                         name="coherence", scale_factors=field.scale_factors)


@dataclasses.dataclass(frozen=True, eq=False)
class PowerSpectrum:
    """P(k) container (reference power/power_spec.py:20-60)."""

    wavenumber: Any
    array: Any
    name: str | None = None
    scale_factors: Any = None

    @property
    def spectra(self):
        return self.array


@dataclasses.dataclass(frozen=True, eq=False)
class DensityField(AbstractField):
    @classmethod
    def full_like(cls, field: AbstractField, fill_value: float = 0.0) -> "DensityField":
        """A mesh of mesh_size filled with fill_value, with field's metadata (reference
        fields/density.py:476-485)."""
        return cls.FromDensityMetadata(array=cls._full(field.mesh_size, fill_value, field), field=field)

    def to(self, unit, *, omega_m=None, h=None, mean_density=None) -> "DensityField":
        """Unit conversion with the voxel volume prod(L / N) (reference fields/density.py:66-124)."""
        vol = float(np.prod(np.asarray(self.box_size, np.float64) / np.asarray(self.mesh_size, np.float64)))
        return _density_to(self, unit, vol, omega_m, h, mean_density)

    def power(self, mesh2: "DensityField" | None = None, *, kedges=None, multipoles=0, los=(0.0, 0.0, 1.0),
              batch_size=None) -> PowerSpectrum:
        """P(k) of the mesh (reference fields/density.py:275-318)."""
        from .power import power as power_fn

        m2 = mesh2.array if isinstance(mesh2, AbstractField) else mesh2
        k, pk = power_fn(self.array, m2, box_shape=self.box_size, kedges=kedges, multipoles=multipoles, los=los)
        return PowerSpectrum(wavenumber=k, array=pk, name="pk", scale_factors=self.scale_factors)

    def cross_power(self, *, kedges=None, multipoles=0, los=(0.0, 0.0, 1.0), batch_size=None) -> PowerSpectrum:
        """P(k) of every pair (i, j), i <= j, of a batch of B meshes, in upper-triangular
        order (0,0), (0,1), ..., (0,B-1), (1,1), ...: array (B(B+1)/2, ...) (reference
        fields/density.py:319-403)."""
        from .power import power as power_fn

        data = self.array
        if data.ndim != 4:
            raise ValueError(f"cross_power requires batched array with shape (B, X, Y, Z), got array with "
                             f"{data.ndim} dimensions. Use power() for single fields.")
        if data.shape[0] < 2:
            raise ValueError(f"cross_power requires at least 2 maps in batch dimension, got {data.shape[0]}. "
                             f"Use power() for single fields.")
        k, spectra = None, []
        for i in range(data.shape[0]):
            for j in range(i, data.shape[0]):
                k_ij, pk = power_fn(data[i], data[j], box_shape=self.box_size, kedges=kedges,
                                    multipoles=multipoles, los=los)
                k = k_ij if k is None else k
                spectra.append(pk)
        return PowerSpectrum(wavenumber=k, array=_stack(spectra), name="cross_pk", scale_factors=self.scale_factors)

    def _paired(self, other, fn, name, kedges):
        data1, data2 = self.array, other.array
        if data1.ndim not in (3, 4):
            raise ValueError(f"DensityField.{name} expects array shape (X,Y,Z) or (B,X,Y,Z)")
        if tuple(data2.shape) != tuple(data1.shape):
            raise ValueError(f"other array must match shape for {name}")
        rows = [(data1, data2)] if data1.ndim == 3 else list(zip(data1, data2))
        k, spectra = None, []
        for m1, m2 in rows:
            k_i, r = fn(m1, m2, box_shape=self.box_size, kedges=kedges)
            k = k_i if k is None else k
            spectra.append(r)
        arr = _stack(spectra) if data1.ndim == 4 else spectra[0]
        return PowerSpectrum(wavenumber=k, array=arr, name=name, scale_factors=self.scale_factors)

    def transfer(self, other: "DensityField", *, kedges=None, batch_size=None) -> PowerSpectrum:
        """Monopole transfer function sqrt(P_other / P_self), per batch entry (reference
        fields/density.py:404-439)."""
        from .power import transfer

        return self._paired(other, transfer, "transfer", kedges)

    def coherence(self, other: "DensityField", *, kedges=None, batch_size=None) -> PowerSpectrum:
        """Monopole coherence P_cross / sqrt(P_self P_other), per batch entry (reference
        fields/density.py:440-475)."""
        from .power import coherence

        return self._paired(other, coherence, "coherence", kedges)

    def project(self, nz_slices: int = 10) -> "FlatDensity":
        """Sum of the last nz_slices planes along z as a flat map of shape (X, Y) or (B, X, Y),
        status PROJECTED_DENSITY (reference fields/density.py:127-159)."""
        data = self.array
        if data.ndim not in (3, 4):
            raise ValueError(f"project() expects 3D array or batch of 3D arrays, got shape {tuple(data.shape)}")
        sl = data[..., -nz_slices:]
        proj = sl.sum(dim=-1) if isinstance(sl, torch.Tensor) else np.sum(sl, axis=-1)
        npix = tuple(int(v) for v in proj.shape[-2:])
        return FlatDensity.FromDensityMetadata(array=proj, field=self.replace(flatsky_npix=npix),
                                               status=FieldStatus.PROJECTED_DENSITY)


@dataclasses.dataclass(frozen=True, eq=False)
class SphericalDensity(AbstractField):
    def _core_ndim(self) -> int:
        return 1

    @classmethod
    def full_like(cls, field: AbstractField, fill_value: float = 0.0) -> "SphericalDensity":
        """One HEALPix map of field's nside filled with fill_value (reference
        fields/lightcone.py:840-852)."""
        if field.nside is None:
            raise ValueError("nside metadata is required to create full_like SphericalDensity.")
        return cls.FromDensityMetadata(array=cls._full((12 * field.nside * field.nside,), fill_value, field),
                                       field=field)

    def to(self, unit, *, omega_m=None, h=None, mean_density=None) -> "SphericalDensity":
        """Unit conversion with each shell's exact pixel volume (4 pi / npix)(R_max^3 - R_min^3) / 3
        (reference fields/lightcone.py:480-535)."""
        if self.unit == unit:
            return self
        if self.comoving_centers is None or self.density_width is None:
            raise ValueError("comoving_centers and density_width metadata are required for unit conversion.")
        c = np.asarray(self.comoving_centers, np.float64)
        w = np.asarray(self.density_width, np.float64)
        vol = 4.0 * np.pi / (12 * self.nside * self.nside) * ((c + w / 2) ** 3 - (c - w / 2) ** 3) / 3.0
        return _density_to(self, unit, vol, omega_m, h, mean_density)

    def angular_cl(self, mesh2: "SphericalDensity | None" = None, *, lmax: int | None = None, method: str = "jax",
                   batch_size=None) -> PowerSpectrum:
        """C_ell of each map, auto or cross with mesh2 (reference fields/lightcone.py:632-674):
        healpy's anafast algorithm in this library's GPU engine (ring transforms and
        Legendre stages in FP64)."""
        from .power import angular_cl_spherical

        d1 = self.array
        d2 = mesh2.array if mesh2 is not None else None
        if d1.ndim not in (1, 2):
            raise ValueError("SphericalDensity.angular_cl expects array shape (npix) or (B,npix)")
        if d2 is not None and d2.shape != d1.shape:
            raise ValueError("mesh2 must match shape for cross Cl")
        rows1 = [d1] if d1.ndim == 1 else list(d1)
        rows2 = [None] * len(rows1) if d2 is None else ([d2] if d2.ndim == 1 else list(d2))
        ell, spectra = None, []
        for a, b in zip(rows1, rows2):
            ell, cl = angular_cl_spherical(a, b, lmax=lmax, method=method)
            spectra.append(cl)
        arr = torch.stack(spectra) if d1.ndim == 2 else spectra[0]
        return PowerSpectrum(wavenumber=ell, array=arr, name="cl", scale_factors=self.scale_factors)

    def ud_sample(self, new_nside: int) -> "SphericalDensity":
        """The RING maps at new_nside with healpy's ud_grade (reference fields/lightcone.py:625-630)."""
        from .healpix_order import ud_grade

        a = self.array if isinstance(self.array, torch.Tensor) else torch.as_tensor(np.asarray(self.array))
        return self.replace(array=ud_grade(a, int(new_nside)), nside=int(new_nside))

    def transfer(self, other: "SphericalDensity", *, lmax: int | None = None, method: str = "jax",
                 batch_size=None) -> PowerSpectrum:
        """Transfer function sqrt(C_other / C_self) (reference fields/lightcone.py:746-788)."""
        return _cl_transfer(self, other, lmax=lmax, method=method)

    def coherence(self, other: "SphericalDensity", *, lmax: int | None = None, method: str = "jax",
                  batch_size=None) -> PowerSpectrum:
        """Coherence C_cross / sqrt(C_self C_other) (reference fields/lightcone.py:790-838)."""
        return _cl_coherence(self, other, lmax=lmax, method=method)

    def cross_angular_cl(self, *, lmax: int | None = None, method: str = "healpy", batch_size=None) -> PowerSpectrum:
        """All auto and cross C_ell of the batched maps, healpy's alm2cl order (reference
        fields/lightcone.py:676-720)."""
        from .power import cross_angular_cl_spherical

        if self.array.ndim != 2:
            raise ValueError("cross_angular_cl needs batched maps (B, npix)")
        ell, cls = cross_angular_cl_spherical(self.array, lmax=lmax, method=method)
        return PowerSpectrum(wavenumber=ell, array=cls, name="cl", scale_factors=self.scale_factors)


@dataclasses.dataclass(frozen=True, eq=False)
class FlatDensity(AbstractField):
    """Flat-sky planes (reference fields/lightcone.py:20-233): (npx, npy) or (S, npx, npy)
    maps, the shape given by flatsky_npix."""

    def _core_ndim(self) -> int:
        return 2

    @classmethod
    def full_like(cls, field: AbstractField, fill_value: float = 0.0) -> "FlatDensity":
        """One flat map of field's flatsky_npix filled with fill_value (reference
        fields/lightcone.py:423-435, which shapes it by field_size)."""
        if field.flatsky_npix is None:
            raise ValueError("flatsky_npix metadata is required to create full_like FlatDensity.")
        return cls.FromDensityMetadata(array=cls._full(field.flatsky_npix, fill_value, field), field=field)

    def __post_init__(self):
        super().__post_init__()
        if self.array.ndim not in (2, 3, 4):
            raise ValueError("FlatDensity array must have shape (ny, nx), (S, ny, nx), or (N, S, ny, nx).")
        if self.flatsky_npix is None:
            raise ValueError("FlatDensity requires `flatsky_npix`.")
        if tuple(self.array.shape[-2:]) != tuple(self.flatsky_npix):
            raise ValueError(f"Array spatial shape {tuple(self.array.shape[-2:])} does not match flatsky_npix "
                             f"{tuple(self.flatsky_npix)}.")

    def to(self, unit, *, omega_m=None, h=None, mean_density=None) -> "FlatDensity":
        """Unit conversion with the pixel volume the reference's FlatDensity.to uses
        (fields/lightcone.py:51-98): (L_x / flatsky_npix[1]) (L_y / flatsky_npix[0]) width."""
        ny_pix, nx_pix = self.flatsky_npix
        Lx, Ly, _ = self.box_size
        vol = (Lx / nx_pix) * (Ly / ny_pix) * np.asarray(self.density_width, np.float64)
        return _density_to(self, unit, vol, omega_m, h, mean_density)

    def angular_cl(self, mesh2: "FlatDensity | None" = None, *, field_size=None, pixel_size=None, ell_edges=None,
                   batch_size=None) -> PowerSpectrum:
        """Flat-sky C_ell, auto or cross (reference fields/lightcone.py:197-233)."""
        from .power import angular_cl_flat

        data1 = self.array
        data2 = mesh2.array if mesh2 is not None else None
        if data1.ndim not in (2, 3):
            raise ValueError("FlatDensity.angular_cl expects array shape (ny,nx) or (B,ny,nx)")
        if data2 is not None and data2.shape != data1.shape:
            raise ValueError("mesh2 must match shape for cross Cl")
        ell, cl = angular_cl_flat(data1, data2, pixel_size=pixel_size, field_size=field_size or self.field_size,
                                  ell_edges=ell_edges)
        return PowerSpectrum(wavenumber=ell, array=cl, name="cl", scale_factors=self.scale_factors)

    def cross_angular_cl(self, *, field_size=None, pixel_size=None, ell_edges=None, batch_size=None) -> PowerSpectrum:
        """Flat-sky C_ell of every pair (i, j), i <= j, of B maps in upper-triangular order
        (0,0), (0,1), ..., (0,B-1), (1,1), ...: array (B(B+1)/2, nbins) (reference
        fields/lightcone.py:236-316)."""
        from .power import angular_cl_flat

        data = self.array
        if data.ndim != 3:
            raise ValueError(f"cross_angular_cl requires batched array with shape (B, ny, nx), got array with "
                             f"{data.ndim} dimensions. Use angular_cl() for single maps.")
        if data.shape[0] < 2:
            raise ValueError(f"cross_angular_cl requires at least 2 maps in batch dimension, got {data.shape[0]}. "
                             f"Use angular_cl() for single maps.")
        fs = field_size or self.field_size
        ell, spectra = None, []
        for i in range(data.shape[0]):
            for j in range(i, data.shape[0]):
                ell_ij, cl = angular_cl_flat(data[i], data[j], pixel_size=pixel_size, field_size=fs,
                                             ell_edges=ell_edges)
                ell = ell_ij if ell is None else ell
                spectra.append(cl)
        return PowerSpectrum(wavenumber=ell, array=_stack(spectra), name="cross_cl", scale_factors=self.scale_factors)

    def ud_sample(self, new_npix: int) -> "FlatDensity":
        """The maps resampled to (new_npix, new_npix) with jax.image.resize's bilinear rule
        (reference fields/lightcone.py:184-195)."""
        a = self.array
        if a.ndim not in (2, 3):
            raise ValueError("ud_sample expects maps of shape (ny, nx) or (B, ny, nx)")
        w0 = _linear_resize_weights(int(a.shape[-2]), int(new_npix))
        w1 = _linear_resize_weights(int(a.shape[-1]), int(new_npix))
        if isinstance(a, torch.Tensor):
            t0 = torch.as_tensor(w0, dtype=a.dtype, device=a.device)
            t1 = torch.as_tensor(w1, dtype=a.dtype, device=a.device)
            out = torch.einsum("...ij,ik,jl->...kl", a, t0, t1)
        else:
            out = np.einsum("...ij,ik,jl->...kl", a, w0.astype(a.dtype), w1.astype(a.dtype))
        return self.replace(array=out, flatsky_npix=(int(new_npix), int(new_npix)))

    def transfer(self, other: "FlatDensity", *, field_size=None, pixel_size=None, ell_edges=None,
                 batch_size=None) -> PowerSpectrum:
        """Angular transfer function sqrt(C_other / C_self) (reference fields/lightcone.py:318-365)."""
        return _cl_transfer(self, other, field_size=field_size, pixel_size=pixel_size, ell_edges=ell_edges)

    def coherence(self, other: "FlatDensity", *, field_size=None, pixel_size=None, ell_edges=None,
                  batch_size=None) -> PowerSpectrum:
        """Angular coherence C_cross / sqrt(C_self C_other) (reference fields/lightcone.py:367-421)."""
        return _cl_coherence(self, other, field_size=field_size, pixel_size=pixel_size, ell_edges=ell_edges)


@dataclasses.dataclass(frozen=True, eq=False)
class ParticleField(AbstractField):
    def _core_ndim(self) -> int:
        return 4

    @classmethod
    def full_like(cls, field: AbstractField, fill_value: float = 0.0) -> "ParticleField":
        """A (mesh_size, 3) particle grid filled with fill_value (reference fields/particles.py:620-629)."""
        return cls.FromDensityMetadata(array=cls._full(tuple(field.mesh_size) + (3,), fill_value, field),
                                       field=field)

    def to(self, unit: PositionUnit) -> "ParticleField":
        """Unit conversion through GRID_ABSOLUTE (reference fields/units.py:78-130)."""
        if unit == self.unit:
            return self
        n = torch.tensor(self.mesh_size, dtype=torch.float32, device=self.array.device)
        L = torch.tensor(self.box_size, dtype=torch.float32, device=self.array.device)
        if self.unit == PositionUnit.GRID_ABSOLUTE:
            grid = self.array
        elif self.unit == PositionUnit.GRID_RELATIVE:
            grid = self.array + uniform_particles(self.mesh_size, self.array.device)
        elif self.unit == PositionUnit.MPC_H:
            grid = self.array / L * n
        else:
            raise ValueError(f"unknown unit {self.unit}")
        if unit == PositionUnit.GRID_ABSOLUTE:
            out = grid
        elif unit == PositionUnit.GRID_RELATIVE:
            out = grid - uniform_particles(self.mesh_size, self.array.device)
        elif unit == PositionUnit.MPC_H:
            out = grid / n * L
        else:
            raise ValueError(f"unknown unit {unit}")
        return self.replace(array=out.contiguous(), unit=unit)

    def _grid_mode(self):
        if self.unit == PositionUnit.MPC_H:
            raise ValueError("Cannot paint ParticleField with unit MPC_H; convert to GRID_RELATIVE or GRID_ABSOLUTE first.")
        return self.unit == PositionUnit.GRID_ABSOLUTE

    def paint(self, *, mesh=None, weights=1.0, chunk_size: int = DEFAULT_CHUNK_SIZE, batch_size=None) -> DensityField:
        """CIC paint onto the mesh (reference fields/particles.py:119-178)."""
        absolute = self._grid_mode()
        w, ws = _weights_arg(weights)
        out = None
        acc = False
        if torch.is_grad_enabled() and self.array.requires_grad:
            if absolute or w is not None or mesh is not None:
                raise NotImplementedError("gradients of CIC painting: relative displacements, a scalar weight, a new "
                                          "mesh")
            from .painting import CICPaint

            dens = CICPaint.apply(self.array.contiguous(), ws)
            return DensityField(array=dens, **self._meta_for_density(FieldStatus.DENSITY_FIELD))
        if mesh is not None:
            out = (mesh.array if isinstance(mesh, AbstractField) else mesh).clone().contiguous()
            acc = True
        dens = ops.paint_cic(self.array.contiguous(), absolute=absolute, weights=w, weight=ws, out=out,
                             accumulate=acc)
        return DensityField(array=dens, **self._meta_for_density(FieldStatus.DENSITY_FIELD))

    def _meta_for_density(self, status):
        return dict(mesh_size=self.mesh_size, box_size=self.box_size, observer_position=self.observer_position,
                    halo_size=self.halo_size, nside=self.nside, flatsky_npix=self.flatsky_npix,
                    field_size=self.field_size, status=status, scale_factors=self.scale_factors,
                    unit=DensityUnit.DENSITY)

    def read_out(self, density_mesh) -> DensityField:
        """CIC interpolation of a mesh at the particle positions (reference fields/particles.py:182-229)."""
        absolute = self._grid_mode()
        mesh = density_mesh.array if isinstance(density_mesh, AbstractField) else density_mesh
        if torch.is_grad_enabled() and (self.array.requires_grad or mesh.requires_grad):
            if absolute or tuple(mesh.shape) != tuple(self.array.shape[:-1]):
                raise NotImplementedError("gradients of the CIC readout: relative displacements, one mesh per "
                                          "particle set")
            from .painting import CICReadout

            vals = CICReadout.apply(self.array, mesh)
            return DensityField(array=vals, **self._meta_for_density(self.status))
        vals = ops.readout_cic(self.array.contiguous(), mesh.contiguous(), absolute=absolute)
        return DensityField(array=vals, **self._meta_for_density(self.status))

    def paint_2d(self, center, density_plane_width, *, weights=None, batch_size=None) -> FlatDensity:
        """Flat-sky planes (reference fields/particles.py:234-320 -> _src/fields/_painting.py:117-202):
        the particles with center - width/2 < z <= center + width/2 (z measured from the box
        origin; center and width in Mpc/h) painted with 2D CIC on a flatsky_npix grid, x and
        y scaled to it and wrapped, divided by the pixel volume (L_x / npx)(L_y / npy) width.
        As in the reference (its light-cone mode), every plane takes the particles of every
        snapshot of a batched (S, ...) input that fall in its z range."""
        if self.flatsky_npix is None:
            raise ValueError("ParticleField requires `flatsky_npix` for paint_2d.")
        grad = torch.is_grad_enabled() and self.array.requires_grad
        if grad and (self.unit != PositionUnit.GRID_RELATIVE or self.array.ndim != 4 or
                     not isinstance(weights, (type(None), int, float))):
            raise NotImplementedError("gradients of flat-sky planes: one set of relative displacements, a scalar "
                                      "weight")
        field = self if self.unit != PositionUnit.MPC_H else self.to(PositionUnit.GRID_ABSOLUTE)
        absolute = field._grid_mode()
        centers = np.atleast_1d(np.asarray(center, dtype=np.float64))
        widths = np.atleast_1d(np.asarray(density_plane_width, dtype=np.float64))
        if centers.shape != widths.shape:
            raise ValueError(f"center and density_plane_width must have the same shape; got {centers.shape} and "
                             f"{widths.shape}")
        arr = field.array.contiguous()
        if arr.ndim == 5:
            if arr.shape[0] != centers.size:
                raise ValueError(f"Batched input: center must have {arr.shape[0]} elements, got {centers.size}")
        elif arr.ndim != 4:
            raise ValueError(f"paint_2d() expects 4D or 5D array, got shape {tuple(arr.shape)}")
        npx, npy = (int(v) for v in self.flatsky_npix)
        nz = self.mesh_size[2]
        Lx, Ly, Lz = (float(v) for v in self.box_size)
        w, ws = _weights_arg(weights)
        srcs = [arr[i] for i in range(arr.shape[0])] if arr.ndim == 5 else [arr]
        maps = []
        for c, wd in zip(centers, widths):
            cg, wg = c * nz / Lz, wd * nz / Lz  # grid units along z
            vol = (Lx / npx) * (Ly / npy) * wd
            if grad:
                from .painting import PaintFlat

                maps.append(PaintFlat.apply(arr, (npx, npy), cg - wg / 2, cg + wg / 2, ws / vol if vol > 0 else ws))
                continue
            m = None
            for src in srcs:
                m = ops.paint_flat(src, (npx, npy), cg - wg / 2, cg + wg / 2, absolute=absolute, weights=w,
                                   weight=ws / vol if vol > 0 else ws, out=m, accumulate=m is not None)
            maps.append(m)
        out = maps[0] if centers.size == 1 else torch.stack(maps)
        return FlatDensity(array=out, mesh_size=self.mesh_size, box_size=self.box_size,
                           observer_position=self.observer_position, flatsky_npix=(npx, npy),
                           field_size=self.field_size, nside=self.nside, status=FieldStatus.LIGHTCONE,
                           comoving_centers=centers, density_width=widths, scale_factors=self.scale_factors,
                           unit=DensityUnit.DENSITY)

    def paint_spherical(self, center, density_plane_width, *, scheme: str = "bilinear", weights=None,
                        kernel_width_arcmin=None, smoothing_interpretation="fwhm", paint_nside=None,
                        ud_grade_power=0.0, ud_grade_order_in="RING", ud_grade_order_out="RING",
                        ud_grade_pess=False, batch_size=None) -> SphericalDensity:
        """HEALPix shell painting (reference fields/particles.py:326-442)."""
        if self.nside is None:
            raise ValueError("Spherical painting requires `nside`.")
        if kernel_width_arcmin is not None and scheme != "rbf_neighbor":
            raise NotImplementedError("kernel_width_arcmin applies to the rbf_neighbor scheme only")
        from .painting import check_grade_orders, paint_shells, regrade

        # painted at paint_nside when given, then brought to nside with healpy's ud_grade
        check_grade_orders(ud_grade_order_in, ud_grade_order_out)
        grade = dict(power=ud_grade_power, order_in=ud_grade_order_in, order_out=ud_grade_order_out,
                     pess=ud_grade_pess)
        src = self if paint_nside is None else self.replace(nside=int(paint_nside))
        sigma = ops.rbf_sigma(src.nside, kernel_width_arcmin, smoothing_interpretation) \
            if scheme == "rbf_neighbor" else None

        centers = np.atleast_1d(np.asarray(center, dtype=np.float64))
        widths = np.atleast_1d(np.asarray(density_plane_width, dtype=np.float64))
        if centers.shape != widths.shape:
            raise ValueError("center and density_plane_width must have the same shape")
        arr = self.array
        if arr.ndim == 5:
            if arr.shape[0] != centers.size:
                raise ValueError(f"Batched input: center must have {arr.shape[0]} elements")
            maps = torch.stack([paint_shells(src.replace(array=arr[i]), centers[i:i + 1], widths[i:i + 1], scheme,
                                             weights, sigma=sigma)[0] for i in range(arr.shape[0])])
        else:
            maps = paint_shells(src, centers, widths, scheme, weights, sigma=sigma)
        maps = regrade(maps, self.nside, paint_nside, **grade)
        if maps.shape[0] == 1:
            maps = maps[0]
        return SphericalDensity(array=maps, mesh_size=self.mesh_size, box_size=self.box_size,
                                observer_position=self.observer_position, nside=self.nside,
                                status=FieldStatus.LIGHTCONE, comoving_centers=centers, density_width=widths,
                                scale_factors=self.scale_factors, unit=DensityUnit.DENSITY)


def uniform_particles(mesh_size, device="cuda") -> torch.Tensor:
    """Lagrangian grid coordinates (N, N, N, 3) (jaxpm uniform_particles)."""
    axes = [torch.arange(n, dtype=torch.float32, device=device) for n in mesh_size]
    g = torch.meshgrid(*axes, indexing="ij")
    return torch.stack(g, dim=-1)


def convert_units(array, origin, destination, mesh_size, box_size, h=None, omega_m=None, mean_density=None,
                  volume_element=None, sharding=None):
    """Convert an array between units of one family (reference fields/units.py:22-258):
    positions through GRID_ABSOLUTE, densities through DENSITY (particles per (Mpc/h)^3)."""
    if origin == destination:
        return array
    if type(origin) is not type(destination):
        raise TypeError(f"Cannot convert between different unit families: {type(origin).__name__} -> "
                        f"{type(destination).__name__}")
    if isinstance(origin, PositionUnit):
        f = ParticleField(array=array, mesh_size=tuple(mesh_size), box_size=tuple(box_size), unit=origin)
        return f.to(destination).array
    if isinstance(origin, DensityUnit):
        return _convert_density(array, origin, destination, volume_element, omega_m, h, mean_density)
    if isinstance(origin, ConvergenceUnit):  # both are kappa = Sigma / Sigma_crit
        return array
    raise NotImplementedError(f"Conversion not implemented for {type(origin).__name__}")


def _convert_density(array, origin, destination, volume_element, omega_m, h, mean_density):
    """DENSITY as the hub (reference fields/units.py:133-258): COUNTS = DENSITY x V,
    OVERDENSITY = DENSITY / mean - 1 (mean of the array when not given), MSUN_H_PER_MPC3 =
    DENSITY x (Omega_m 2.775e11 h^2 V / h^3) h, V the volume per voxel or pixel in (Mpc/h)^3
    (one value, or one per leading entry)."""
    if volume_element is None:
        raise ValueError("volume_element is required for density unit conversions")
    x = array if isinstance(array, torch.Tensor) else torch.as_tensor(np.asarray(array))
    v = torch.as_tensor(np.asarray(volume_element, dtype=np.float64), dtype=x.dtype, device=x.device)
    v = v.reshape(v.shape + (1,) * (x.ndim - v.ndim))
    mass = None
    if DensityUnit.MSUN_H_PER_MPC3 in (origin, destination):
        if omega_m is None or h is None:
            raise ValueError("omega_m and h required for MSUN_H_PER_MPC3 conversion")
        mass = omega_m * 2.775e11 * h**2 * (v / h**3)  # solar masses per particle at mean 1 per voxel
    if origin == DensityUnit.DENSITY:
        density = x
    elif origin == DensityUnit.COUNTS:
        density = x / v
    elif origin == DensityUnit.OVERDENSITY:
        if mean_density is None:
            raise ValueError("mean_density required to convert from OVERDENSITY")
        density = (x + 1.0) * mean_density
    elif origin == DensityUnit.MSUN_H_PER_MPC3:
        density = (x * v / h) / mass / v
    else:
        raise ValueError(f"Unknown origin unit: {origin}")
    if destination == DensityUnit.DENSITY:
        return density
    if destination == DensityUnit.COUNTS:
        return density * v
    if destination == DensityUnit.OVERDENSITY:
        mean = density.mean() if mean_density is None else torch.as_tensor(mean_density, dtype=x.dtype)
        eps = torch.finfo(density.dtype).eps
        safe = torch.where(mean == 0, torch.as_tensor(eps, dtype=x.dtype, device=x.device), mean)
        return density / safe - 1.0
    if destination == DensityUnit.MSUN_H_PER_MPC3:
        return density * v * mass * h / v
    raise ValueError(f"Unknown destination unit: {destination}")


def _density_to(field, unit, volume_element, omega_m, h, mean_density):
    if field.unit == unit:
        return field
    if not isinstance(unit, DensityUnit):
        raise TypeError(f"{type(field).__name__}.to() expected a DensityUnit for 'unit', got {unit!r}")
    arr = convert_units(field.array, field.unit, unit, field.mesh_size, field.box_size, h=h, omega_m=omega_m,
                        mean_density=mean_density, volume_element=volume_element)
    return field.replace(array=arr, unit=unit)


# ----------------------------------------------------------------------- lensing maps
# Convergence and shear maps (reference fields/lensing_maps.py): the density containers
# with convergence units. The reference does not implement the kappa <-> shear conversions
# either; they raise the same NotImplementedError.
def _convergence_to(field, unit):
    if field.unit == unit:
        return field
    if not isinstance(unit, ConvergenceUnit):
        raise TypeError(f"{type(field).__name__}.to() expected a ConvergenceUnit, got {unit!r}")
    return field.replace(unit=unit)


@dataclasses.dataclass(frozen=True, eq=False)
class SphericalKappaField(SphericalDensity):
    """HEALPix convergence maps (npix,) or (n_sources, npix)."""

    def to(self, unit, **_):
        return _convergence_to(self, unit)

    def get_shear(self, cosmo=None):
        raise NotImplementedError("Shear computation from kappa (spherical) not implemented yet.")


@dataclasses.dataclass(frozen=True, eq=False)
class FlatKappaField(FlatDensity):
    """Flat-sky convergence maps."""

    def to(self, unit, **_):
        return _convergence_to(self, unit)

    def get_shear(self, cosmo=None):
        raise NotImplementedError("Shear computation from kappa (flat-sky) not implemented yet.")


@dataclasses.dataclass(frozen=True, eq=False)
class SphericalShearField(SphericalDensity):
    def to(self, unit, **_):
        return _convergence_to(self, unit)

    def get_convergence(self, cosmo=None):
        raise NotImplementedError("Convergence from shear (spherical) not implemented yet.")


@dataclasses.dataclass(frozen=True, eq=False)
class FlatShearField(FlatDensity):
    def to(self, unit, **_):
        return _convergence_to(self, unit)

    def get_convergence(self, cosmo=None):
        raise NotImplementedError("Convergence from shear (flat-sky) not implemented yet.")


@dataclasses.dataclass(frozen=True, eq=False)
class FieldMetadata(AbstractField):
    """Metadata-only field (array None), as the reference's to_metadata() produces."""

    @classmethod
    def full_like(cls, field: AbstractField, fill_value: float = 0.0):
        raise NotImplementedError("FieldMetadata is metadata-only; use a concrete field class.")

    def is_batched(self) -> bool:
        return False

    def is_multi_batched(self) -> bool:
        return False
