"""Field + cosmology catalog on disk (reference io/catalog.py:1-510, format version 2).

One row per (field, cosmology) entry, written through HuggingFace `datasets` with the
reference's Features schema, so files written here load in jax-fli's `Catalog.from_parquet`
and the reverse:
- "array": the batched array (B, ...) as Array2D (SphericalDensity, SphericalKappaField:
  (B, npix)), Array3D (FlatDensity, FlatKappaField: (B, npx, npy)), Array4D (DensityField)
  or Array5D (ParticleField), first dimension variable;
- dynamic metadata "z_sources", "scale_factors", "comoving_centers", "density_width":
  float64 sequences of length B;
- static metadata "mesh_size", "box_size", "observer_position", "halo_size", enum names
  "status" and "unit", "field_type", "version", and the cosmology "Omega_c", "Omega_b",
  "h", "n_s", "sigma8", "w0", "wa", "Omega_k", "Omega_nu" (float32);
- optional "nside", "flatsky_npix", "field_size" when the field has them.
A batch of 1 is read back as the unbatched field. Arrays are read back as CUDA tensors
when a GPU is present (the `device` argument chooses).
"""

from __future__ import annotations

import numpy as np
import torch

from .cosmology import Cosmology
from .fields import (AbstractField, ConvergenceUnit, DensityField, DensityUnit, FieldStatus, FlatDensity,
                     FlatKappaField, ParticleField, PositionUnit, SphericalDensity, SphericalKappaField)

CATALOG_VERSION = 2

__all__ = ["Catalog", "CATALOG_VERSION"]

_FIELD_CLASSES = {"SphericalDensity": SphericalDensity, "SphericalKappaField": SphericalKappaField,
                  "FlatDensity": FlatDensity, "FlatKappaField": FlatKappaField, "DensityField": DensityField,
                  "ParticleField": ParticleField}
_CORE_NDIM = {"SphericalDensity": 1, "SphericalKappaField": 1, "FlatDensity": 2, "FlatKappaField": 2,
              "DensityField": 3, "ParticleField": 4}


def _batched(array: np.ndarray, field_type: str) -> np.ndarray:
    """The array with its batch dimension (reference io/catalog.py:57-84)."""
    core = _CORE_NDIM.get(field_type)
    if core is None:
        raise ValueError(f"Unknown field type: {field_type}")
    if array.ndim == core:
        return array[None, ...]
    if array.ndim != core + 1:
        raise ValueError(f"Unexpected shape for {field_type}: {array.shape}")
    return array


def _dynamic(value, name: str, batch: int) -> list:
    """Dynamic metadata as a list of length `batch` (reference io/catalog.py:87-110)."""
    if value is None:
        raise ValueError(f"Dynamic metadata '{name}' cannot be None.")
    arr = np.asarray(value.detach().cpu() if isinstance(value, torch.Tensor) else value, dtype=np.float64)
    if arr.ndim == 0:
        arr = arr[None]
    if arr.ndim == 2 and arr.shape[1] == 1:
        arr = arr[:, 0]
    if arr.ndim != 1:
        raise ValueError(f"Dynamic metadata '{name}' must be 0-d or 1-d, got shape {arr.shape}.")
    if arr.shape[0] != batch:
        raise ValueError(f"Dynamic metadata '{name}' length {arr.shape[0]} != batch_size {batch}.")
    return arr.tolist()


def _pair(v) -> list:
    return [float(v), float(v)] if np.ndim(v) == 0 else [float(x) for x in v]


def _features(field_type: str, element_shape, dtype: str, field: AbstractField):
    """The reference's Features schema (io/catalog.py:113-177)."""
    from datasets import Array2D, Array3D, Array4D, Array5D, Features, Sequence, Value

    array_cls = {"SphericalDensity": Array2D, "SphericalKappaField": Array2D, "FlatDensity": Array3D,
                 "FlatKappaField": Array3D, "DensityField": Array4D, "ParticleField": Array5D}[field_type]
    feats = {
        "array": array_cls(shape=(None, *element_shape), dtype=dtype),
        "z_sources": Sequence(Value("float64")),
        "scale_factors": Sequence(Value("float64")),
        "comoving_centers": Sequence(Value("float64")),
        "density_width": Sequence(Value("float64")),
        "mesh_size": Sequence(Value("int32"), length=3),
        "box_size": Sequence(Value("float32"), length=3),
        "observer_position": Sequence(Value("float32"), length=3),
        "halo_size": Sequence(Value("int32"), length=2),
        "status": Value("string"),
        "unit": Value("string"),
    }
    for k in ("Omega_c", "Omega_b", "h", "n_s", "sigma8", "w0", "wa", "Omega_k", "Omega_nu"):
        feats[k] = Value("float32")
    feats["version"] = Value("int32")
    feats["field_type"] = Value("string")
    if field.nside is not None:
        feats["nside"] = Value("int32")
    if field.flatsky_npix is not None:
        feats["flatsky_npix"] = Sequence(Value("int32"), length=2)
    if field.field_size is not None:
        feats["field_size"] = Sequence(Value("float32"), length=2)
    return Features(feats)


def _row(field: AbstractField, cosmo: Cosmology, version: int) -> tuple[dict, object]:
    """One (field, cosmology) entry as a one-row column dict and its Features
    (reference io/catalog.py:180-251)."""
    field_type = type(field).__name__
    if field_type not in _FIELD_CLASSES:
        raise ValueError(f"Unknown field type: {field_type}")
    arr = field.array.detach().cpu().numpy() if isinstance(field.array, torch.Tensor) else np.asarray(field.array)
    arr = _batched(arr, field_type)
    b = arr.shape[0]
    data = {
        "array": [arr],
        "z_sources": [_dynamic(field.z_sources, "z_sources", b)],
        "scale_factors": [_dynamic(field.scale_factors, "scale_factors", b)],
        "comoving_centers": [_dynamic(field.comoving_centers, "comoving_centers", b)],
        "density_width": [_dynamic(field.density_width, "density_width", b)],
        "mesh_size": [list(field.mesh_size)],
        "box_size": [list(field.box_size)],
        "observer_position": [list(field.observer_position)],
        "halo_size": [[int(v) for v in field.halo_size]],
        "status": [field.status.name],
        "unit": [field.unit.name],
        "field_type": [field_type],
        "version": [int(version)],
    }
    if field.nside is not None:
        data["nside"] = [int(field.nside)]
    if field.flatsky_npix is not None:
        data["flatsky_npix"] = [list(field.flatsky_npix)]
    if field.field_size is not None:
        data["field_size"] = [_pair(field.field_size)]
    cos = {"Omega_c": cosmo.Omega_c, "Omega_b": cosmo.Omega_b, "h": cosmo.h, "n_s": cosmo.n_s,
           "sigma8": cosmo.sigma8, "w0": cosmo.w0, "wa": cosmo.wa, "Omega_k": cosmo.Omega_k,
           "Omega_nu": getattr(cosmo, "Omega_nu", 0.0)}
    for k, v in cos.items():
        data[k] = [float(v)]
    return data, _features(field_type, arr.shape[1:], np.dtype(arr.dtype).name, field)


def _field_from_row(item: dict, device) -> tuple[AbstractField, Cosmology, int]:
    """One dataset row back to (field, cosmology, version) (reference io/catalog.py:254-337)."""
    from .fields import PhysicalUnit

    field_type = item["field_type"]
    cls = _FIELD_CLASSES[field_type]
    if cls is ParticleField:
        unit = PositionUnit[item["unit"]]
    elif cls in (SphericalKappaField, FlatKappaField):
        unit = ConvergenceUnit[item["unit"]]
    elif item["unit"] in DensityUnit.__members__:
        unit = DensityUnit[item["unit"]]
    else:
        unit = PhysicalUnit[item["unit"]]
    arr = np.asarray(item["array"])
    unbatched = arr.shape[0] == 1
    if unbatched:
        arr = arr[0]

    def dyn(key):
        v = np.asarray(item[key], dtype=np.float64)
        return float(v[0]) if unbatched else v

    opt = lambda key: item.get(key) is not None
    field = cls(array=torch.as_tensor(np.ascontiguousarray(arr), device=device),
                mesh_size=tuple(int(v) for v in item["mesh_size"]),
                box_size=tuple(float(v) for v in item["box_size"]),
                observer_position=tuple(float(v) for v in item["observer_position"]),
                halo_size=tuple(int(v) for v in item["halo_size"]),
                nside=int(item["nside"]) if opt("nside") else None,
                flatsky_npix=tuple(int(v) for v in item["flatsky_npix"]) if opt("flatsky_npix") else None,
                field_size=tuple(float(v) for v in item["field_size"]) if opt("field_size") else None,
                z_sources=dyn("z_sources"), scale_factors=dyn("scale_factors"),
                comoving_centers=dyn("comoving_centers"), density_width=dyn("density_width"),
                status=FieldStatus[item["status"]], unit=unit)
    if float(item["Omega_nu"]) != 0.0:
        raise ValueError("Omega_nu != 0: massive neutrinos are not in this cosmology model")
    cosmo = Cosmology(Omega_c=float(item["Omega_c"]), Omega_b=float(item["Omega_b"]), h=float(item["h"]),
                      n_s=float(item["n_s"]), sigma8=float(item["sigma8"]), Omega_k=float(item["Omega_k"]),
                      w0=float(item["w0"]), wa=float(item["wa"]))
    return field, cosmo, int(item["version"])


_COSMO_PARAMS = ("Omega_c", "Omega_b", "h", "n_s", "sigma8", "Omega_k", "w0", "wa")


def _cosmology_batch(c: Cosmology) -> int:
    """1 for a cosmology of scalars, N when its parameters are length-N arrays."""
    sizes = {int(np.size(getattr(c, k))) for k in _COSMO_PARAMS}
    sizes.discard(1)
    if len(sizes) > 1:
        raise ValueError(f"batched cosmology parameters have different lengths {sorted(sizes)}")
    return sizes.pop() if sizes else 1


def _cosmology_entry(c: Cosmology, i: int) -> Cosmology:
    """Entry i of a batched cosmology (scalar parameters are shared)."""
    pick = lambda v: float(np.ravel(v)[i]) if np.size(v) > 1 else float(np.ravel(v)[0])
    return Cosmology(**{k: pick(getattr(c, k)) for k in _COSMO_PARAMS})


class Catalog:
    """Fields and their cosmologies (reference io/catalog.py:340-510): lists of equal length;
    a single field and cosmology are wrapped into length-1 lists, or split into N entries
    when the cosmology is batched (parameters given as length-N arrays)."""

    def __init__(self, field, cosmology, version: int = CATALOG_VERSION):
        if isinstance(field, AbstractField) and isinstance(cosmology, Cosmology):
            # one field with one cosmology; a batched cosmology (parameters as length-N
            # arrays) splits a field with leading dimension N into N entries
            # (reference io/catalog.py:361-382)
            cosmo_n = _cosmology_batch(cosmology)
            if cosmo_n > 1:
                field_n = field.array.shape[0] if field.is_batched() else 1
                if field_n != cosmo_n:
                    raise ValueError(f"Cosmology batch size {cosmo_n} != field leading dimension {field_n}.")
                field = [field[i] for i in range(cosmo_n)]
                cosmology = [_cosmology_entry(cosmology, i) for i in range(cosmo_n)]
            elif field.is_multi_batched() and field.array.shape[0] > 1:
                raise ValueError(f"Scalar cosmology cannot pair with a multi-batched field (shape "
                                 f"{tuple(field.array.shape)}, N={field.array.shape[0]} > 1). Pass a batched cosmology "
                                 f"of size N, or split the field first.")
            else:
                field, cosmology = [field], [cosmology]
        if isinstance(field, AbstractField):
            field = [field]
        if isinstance(cosmology, Cosmology):
            cosmology = [cosmology]
        self.field = list(field)
        self.cosmology = list(cosmology)
        self.version = int(version)
        if len(self.field) != len(self.cosmology):
            raise ValueError(f"field and cosmology must have the same length, got {len(self.field)} and "
                             f"{len(self.cosmology)}.")
        if not self.field:
            raise ValueError("Catalog must contain at least one field.")

    def __len__(self) -> int:
        return len(self.field)

    def __getitem__(self, key) -> "Catalog":
        if isinstance(key, int):
            return Catalog(field=[self.field[key]], cosmology=[self.cosmology[key]], version=self.version)
        return Catalog(field=self.field[key], cosmology=self.cosmology[key], version=self.version)

    def __repr__(self) -> str:
        types = {type(f).__name__ for f in self.field}
        return f"Catalog(n_entries={len(self.field)}, field_types={types}, version={self.version})"

    def to_dataset(self):
        """A HuggingFace Dataset with one row per (field, cosmology) entry."""
        import datasets

        parts = []
        for f, c in zip(self.field, self.cosmology):
            data, feats = _row(f, c, self.version)
            parts.append(datasets.Dataset.from_dict(data, features=feats))
        return datasets.concatenate_datasets(parts)

    def to_parquet(self, path: str) -> None:
        self.to_dataset().to_parquet(path)

    @classmethod
    def from_parquet(cls, path: str, device=None) -> "Catalog":
        from datasets import load_dataset

        return cls.from_dataset(load_dataset("parquet", data_files=path, split="train"), device=device)

    @classmethod
    def from_dataset(cls, ds, device=None) -> "Catalog":
        if len(ds) == 0:
            raise ValueError("Cannot reconstruct Catalog from an empty dataset.")
        dev = device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")
        if isinstance(ds, dict):
            f, c, v = _field_from_row(ds, dev)
            return cls(field=[f], cosmology=[c], version=v)
        ds_np = ds.with_format("numpy")
        fields, cosmos, version = [], [], CATALOG_VERSION
        for i in range(len(ds_np)):
            f, c, version = _field_from_row(ds_np[i], dev)
            fields.append(f)
            cosmos.append(c)
        return cls(field=fields, cosmology=cosmos, version=version)
