"""The reference's `jax_fli.io` namespace (io/__init__.py): the field catalog and the
Stage-3 weak-lensing redshift distributions (io/cosmogrid.py:25-67). The package exposes
this module as its attribute `io` (`jfli_b200.io.Catalog`, as `jax_fli.io.Catalog`).

The Stage-3 n(z) tables are data files that ship with jax-fli (io/data/nz_stage3_{1..4}.txt,
two columns: z and n(z) on 1000 points); they are read from a directory given by the caller
or, without one, from an installed jax_fli package (located without importing it).
"""

from __future__ import annotations

import importlib.util
from pathlib import Path

import numpy as np

from .catalog import CATALOG_VERSION, Catalog
from .lensing import RedshiftDistribution, kde_nz

__all__ = ["Catalog", "CATALOG_VERSION", "get_stage3_nz_shear", "stage3_data_dir"]

STAGE3_GALS_PER_ARCMIN2 = (7.0, 8.5, 7.5, 6.0)


def stage3_data_dir() -> Path:
    """The io/data directory of an installed jax_fli package."""
    spec = importlib.util.find_spec("jax_fli")
    if spec is None or not spec.submodule_search_locations:
        raise FileNotFoundError(
            "the Stage-3 n(z) tables ship with jax-fli (jax_fli/io/data/nz_stage3_*.txt); jax_fli is not "
            "installed here, so pass data_dir= the directory that holds them")
    return Path(list(spec.submodule_search_locations)[0]) / "io" / "data"


def get_stage3_nz_shear(gals_per_arcmin2: list[float] | None = None, bw: float = 0.01, zmax: float | None = None,
                        data_dir=None) -> list[RedshiftDistribution]:
    """The 4 tomographic Stage-3 n(z) (reference io/cosmogrid.py:25-67): each file's (z, n(z))
    columns, in file-name order, become a Gaussian KDE (`kde_nz`) with bandwidth `bw`,
    normalised on [0, zmax] (zmax defaults to the file's largest z), with the bin's galaxy
    density (default 7, 8.5, 7.5 and 6 per arcmin^2)."""
    if gals_per_arcmin2 is None:
        gals_per_arcmin2 = list(STAGE3_GALS_PER_ARCMIN2)
    d = Path(data_dir) if data_dir is not None else stage3_data_dir()
    files = sorted(d.glob("nz_stage3_*.txt"))
    if not files:
        raise FileNotFoundError(f"no nz_stage3_*.txt files in {d}")
    out = []
    for f, g in zip(files, gals_per_arcmin2):
        z, nz = np.loadtxt(f, unpack=True)
        out.append(kde_nz(z, nz, bw=bw, zmax=zmax if zmax is not None else float(z.max()),
                          gals_per_arcmin2=float(g)))
    return out
