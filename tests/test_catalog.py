"""Catalog on disk (reference io/catalog.py): the HuggingFace parquet rows written here use
the reference's Features schema (format version 2), and every field type round-trips with
its metadata and cosmology. CPU only."""

import numpy as np
import pytest
import torch

import jfli_b200 as jf

datasets = pytest.importorskip("datasets")


def _fields():
    rng = np.random.default_rng(0)
    meta = dict(mesh_size=(8, 8, 8), box_size=(100.0, 100.0, 100.0), observer_position=(0.5, 0.5, 0.5))
    sph = jf.SphericalDensity(array=torch.as_tensor(rng.random((3, 12 * 4 * 4), dtype=np.float32)), nside=4,
                              status=jf.FieldStatus.LIGHTCONE, unit=jf.DensityUnit.DENSITY,
                              scale_factors=np.array([0.9, 0.8, 0.7]), z_sources=np.array([0.11, 0.25, 0.43]),
                              comoving_centers=np.array([10.0, 30.0, 50.0]), density_width=np.array([20.0] * 3),
                              **meta)
    flat = jf.FlatDensity(array=torch.as_tensor(rng.random((16, 12), dtype=np.float32)), flatsky_npix=(16, 12),
                          field_size=(2.0, 1.5), status=jf.FieldStatus.LIGHTCONE, unit=jf.DensityUnit.DENSITY,
                          scale_factors=0.8, z_sources=0.25, comoving_centers=40.0, density_width=10.0, **meta)
    dens = jf.DensityField(array=torch.as_tensor(rng.random((8, 8, 8), dtype=np.float32)),
                           status=jf.FieldStatus.DENSITY_FIELD, unit=jf.DensityUnit.DENSITY, scale_factors=1.0,
                           z_sources=0.0, comoving_centers=0.0, density_width=0.0, **meta)
    parts = jf.ParticleField(array=torch.as_tensor(rng.standard_normal((2, 8, 8, 8, 3)).astype(np.float32)),
                             status=jf.FieldStatus.PARTICLES, unit=jf.PositionUnit.GRID_RELATIVE,
                             scale_factors=np.array([0.5, 1.0]), z_sources=np.array([1.0, 0.0]),
                             comoving_centers=np.array([0.0, 0.0]), density_width=np.array([0.0, 0.0]), **meta)
    return [sph, flat, dens, parts]


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_catalog_round_trip(tmp_path, kind):
    """One catalog per field type (a catalog's rows share one schema, as in the reference),
    two entries each with their own cosmology."""
    a = _fields()[kind]
    b2 = a.replace(array=a.array * 2)
    fields = [a, b2]
    cosmos = [jf.Planck18(Omega_c=0.25 + 0.01 * i, sigma8=0.8 - 0.01 * i) for i in range(2)]
    path = str(tmp_path / "cat.parquet")
    jf.Catalog(fields, cosmos).to_parquet(path)
    back = jf.Catalog.from_parquet(path, device="cpu")
    assert len(back) == 2 and back.version == jf.CATALOG_VERSION
    for x, y, cx, cy in zip(fields, back.field, cosmos, back.cosmology):
        assert type(x) is type(y)
        assert torch.equal(x.array, y.array)
        assert (x.mesh_size, x.box_size, x.observer_position, x.status, x.unit) == \
               (y.mesh_size, y.box_size, y.observer_position, y.status, y.unit)
        for key in ("scale_factors", "z_sources", "comoving_centers", "density_width"):
            np.testing.assert_allclose(np.asarray(getattr(y, key)), np.asarray(getattr(x, key)))
        assert y.nside == x.nside and y.flatsky_npix == x.flatsky_npix
        np.testing.assert_allclose([cy.Omega_c, cy.sigma8, cy.h], [cx.Omega_c, cx.sigma8, cx.h], rtol=1e-6)
    if kind == 1:
        assert back.field[0].field_size == (2.0, 1.5)
    assert back[1].field[0].array.shape == a.array.shape and len(back[0:2]) == 2


def test_catalog_schema_is_the_reference_schema(tmp_path):
    """The features a reader finds in the file: the reference's names and types."""
    path = str(tmp_path / "one.parquet")
    jf.Catalog(_fields()[0], jf.Planck18()).to_parquet(path)
    ds = datasets.load_dataset("parquet", data_files=path, split="train")
    f = ds.features
    assert type(f["array"]).__name__ == "Array2D" and tuple(f["array"].shape) == (None, 192)
    assert f["array"].dtype == "float32"
    seq = lambda k: (f[k].feature.dtype if hasattr(f[k], "feature") else f[k].dtype)
    for k in ("z_sources", "scale_factors", "comoving_centers", "density_width"):
        assert "float64" in str(seq(k)) or "float64" in str(f[k])
    for k in ("Omega_c", "Omega_b", "h", "n_s", "sigma8", "w0", "wa", "Omega_k", "Omega_nu"):
        assert f[k].dtype == "float32"
    assert f["version"].dtype == "int32" and f["nside"].dtype == "int32"
    row = ds[0]
    assert row["field_type"] == "SphericalDensity" and row["status"] == "LIGHTCONE" and row["unit"] == "DENSITY"
    assert row["version"] == 2 and row["mesh_size"] == [8, 8, 8]


def test_catalog_rejects_mismatched_lengths():
    f = _fields()[2]
    with pytest.raises(ValueError):
        jf.Catalog([f, f], [jf.Planck18()])


def test_catalog_kappa_field(tmp_path):
    """Convergence maps (born's SphericalKappaField) keep their class and unit."""
    sph = _fields()[0]
    kap = jf.SphericalKappaField.FromDensityMetadata(array=sph.array[:2], field=sph, status=jf.FieldStatus.KAPPA,
                                                     unit=jf.ConvergenceUnit.DIMENSIONLESS,
                                                     z_sources=np.array([0.5, 1.0]),
                                                     scale_factors=np.array([0.67, 0.5]),
                                                     comoving_centers=np.array([0.0, 0.0]),
                                                     density_width=np.array([0.0, 0.0]))
    path = str(tmp_path / "kappa.parquet")
    jf.Catalog(kap, jf.Planck18()).to_parquet(path)
    back = jf.Catalog.from_parquet(path, device="cpu").field[0]
    assert type(back) is jf.SphericalKappaField and back.unit == jf.ConvergenceUnit.DIMENSIONLESS
    assert torch.equal(back.array, kap.array)
    assert kap.to(jf.ConvergenceUnit.EFFECTIVE_DENSITY).unit == jf.ConvergenceUnit.EFFECTIVE_DENSITY
    with pytest.raises(NotImplementedError):
        kap.get_shear()


# ------------------------------------------------------- multi-batched fields (N, S, ...)
MESH = (8, 8, 8)


def _density(array, **dyn):
    meta = dict(mesh_size=MESH, box_size=(100.0, 100.0, 100.0), observer_position=(0.5, 0.5, 0.5),
                status=jf.FieldStatus.DENSITY_FIELD, unit=jf.DensityUnit.DENSITY)
    base = dict(z_sources=1.0, scale_factors=0.8, comoving_centers=300.0, density_width=25.0)
    base.update(dyn)
    return jf.DensityField(array=array, **meta, **base)


def _multi(N, S, seed=0):
    rng = np.random.default_rng(seed)
    return _density(torch.as_tensor(rng.standard_normal((N, S, *MESH)).astype(np.float32)),
                    z_sources=rng.uniform(0.5, 2.0, (N, S)), scale_factors=rng.uniform(0.5, 1.0, (N, S)),
                    comoving_centers=rng.uniform(100, 500, (N, S)), density_width=rng.uniform(10, 50, (N, S)))


def _batched_cosmo(n):
    """A cosmology whose parameters are length-n arrays (the reference's batched jc.Cosmology)."""
    return jf.Cosmology(Omega_c=np.full(n, 0.3), Omega_b=np.full(n, 0.05), h=np.full(n, 0.7),
                        n_s=np.full(n, 0.96), sigma8=np.linspace(0.7, 0.9, n), Omega_k=np.zeros(n),
                        w0=np.full(n, -1.0), wa=np.zeros(n))


def test_multi_batched_predicates():
    """(N, S, spatial...) arrays are batched and multi-batched for every field type
    (reference tests/test_catalog.py:306-368)."""
    N, S = 2, 4
    meta = dict(mesh_size=MESH, box_size=(100.0, 100.0, 100.0))
    fields = [jf.SphericalDensity(array=torch.zeros(N, S, 192), nside=4, **meta),
              jf.SphericalKappaField(array=torch.zeros(N, S, 192), nside=4, **meta),
              jf.FlatDensity(array=torch.zeros(N, S, 16, 16), flatsky_npix=(16, 16), **meta),
              jf.FlatKappaField(array=torch.zeros(N, S, 16, 16), flatsky_npix=(16, 16), **meta),
              jf.DensityField(array=torch.zeros(N, S, *MESH), **meta),
              jf.ParticleField(array=torch.zeros(N, S, *MESH, 3), **meta)]
    for f in fields:
        assert f.is_multi_batched() and f.is_batched(), type(f).__name__
        assert not f[0].is_multi_batched() and f[0].is_batched()
        assert not f[0][0].is_batched()


def test_stack_and_concat():
    S = 4
    f1 = _density(torch.zeros(S, *MESH))
    f2 = _density(torch.ones(S, *MESH), z_sources=1.2, scale_factors=0.75, comoving_centers=350.0,
                  density_width=20.0)
    st = jf.DensityField.stack([f1, f2])
    assert tuple(st.array.shape) == (2, S, *MESH) and st.is_multi_batched()
    np.testing.assert_allclose(st.z_sources, [1.0, 1.2])
    assert torch.equal(st[1].array, f2.array)
    with pytest.raises(ValueError, match="concat"):
        jf.DensityField.stack([st, st])
    a, b = _multi(2, S, seed=1), _multi(2, S, seed=2)
    cat = jf.DensityField.concat([a, b])
    assert tuple(cat.array.shape) == (4, S, *MESH) and cat.is_multi_batched()
    assert cat.z_sources.shape == (4, S)
    np.testing.assert_allclose(cat.z_sources[2:], b.z_sources)
    with pytest.raises(ValueError, match="stack"):
        jf.DensityField.concat([f1])
    with pytest.raises(ValueError):
        jf.DensityField.stack([f1, f1.replace(box_size=(200.0, 200.0, 200.0))])
    with pytest.raises(ValueError):
        jf.DensityField.stack([])


def test_catalog_expands_batched_cosmology(tmp_path):
    """(N, S, ...) field + cosmology of N -> N entries of (S, ...); (S, ...) field + cosmology
    of S -> S unbatched entries; a scalar cosmology with N > 1 is refused (reference
    tests/test_catalog.py:447-517)."""
    N, S = 2, 4
    field = _multi(N, S)
    cat = jf.Catalog(field=field, cosmology=_batched_cosmo(N))
    assert len(cat) == N
    for i, entry in enumerate(cat.field):
        assert tuple(entry.array.shape) == (S, *MESH) and entry.is_batched() and not entry.is_multi_batched()
        np.testing.assert_allclose(entry.z_sources, field.z_sources[i])
    assert [c.sigma8 for c in cat.cosmology] == pytest.approx([0.7, 0.9])
    assert all(isinstance(c.Omega_c, float) for c in cat.cosmology)
    path = str(tmp_path / "multi.parquet")
    cat.to_parquet(path)
    back = jf.Catalog.from_parquet(path, device="cpu")
    assert len(back) == N
    for x, y in zip(cat.field, back.field):
        assert tuple(y.array.shape) == (S, *MESH) and y.is_batched() and not y.is_multi_batched()
        assert torch.equal(x.array, y.array)

    snap = _multi(1, 3)[0]
    cat = jf.Catalog(field=snap, cosmology=_batched_cosmo(3))
    assert len(cat) == 3
    assert all(tuple(e.array.shape) == MESH and not e.is_batched() for e in cat.field)

    with pytest.raises(ValueError, match="Scalar cosmology"):
        jf.Catalog(field=field, cosmology=jf.Planck18())
    with pytest.raises(ValueError, match="batch size"):
        jf.Catalog(field=field, cosmology=_batched_cosmo(3))
    single = jf.Catalog(field=_multi(1, S), cosmology=jf.Planck18())
    assert len(single) == 1
