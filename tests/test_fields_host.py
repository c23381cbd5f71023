"""Field containers on the host: the array shorthands, arithmetic, reductions, full_like,
to_metadata and iteration of the reference's field pytrees (_src/base/_core.py:25-171,
fields/*.py full_like), on CPU tensors."""

import importlib

import numpy as np
import pytest
import torch

import jfli_b200 as jf

MESH = (4, 6, 8)
META = dict(mesh_size=MESH, box_size=(100.0, 150.0, 200.0), observer_position=(0.5, 0.5, 0.5))


def _density(array, **kw):
    return jf.DensityField(array=array, status=jf.FieldStatus.DENSITY_FIELD, unit=jf.DensityUnit.DENSITY,
                           scale_factors=kw.pop("scale_factors", 0.8), **META, **kw)


def test_shorthands_and_reductions():
    rng = np.random.default_rng(0)
    a = torch.as_tensor(rng.standard_normal((3, *MESH)).astype(np.float32))
    f = _density(a, scale_factors=np.array([0.5, 0.7, 0.9]))
    assert f.shape == (3, *MESH) and f.ndim == 4 and f.size == a.numel() and f.dtype == torch.float32
    assert len(f) == 3
    entries = list(f)
    assert len(entries) == 3 and all(isinstance(e, jf.DensityField) for e in entries)
    assert torch.equal(entries[2].array, a[2]) and float(entries[2].scale_factors) == 0.9
    x = a.double().numpy()
    assert float(f.mean()) == pytest.approx(x.mean(), rel=1e-6)
    assert float(f.std()) == pytest.approx(x.std(), rel=1e-5)  # population, as jnp.std
    assert float(f.min()) == x.min() and float(f.max()) == x.max()
    np.testing.assert_allclose(f.mean(axis=0).numpy(), x.mean(0), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(f.std(axis=(1, 2, 3)).numpy(), x.std(axis=(1, 2, 3)), rtol=1e-5)
    assert tuple(f.max(axis=1, keepdims=True).shape) == (3, 1, 6, 8)
    np.testing.assert_array_equal(np.asarray(f), a.numpy())
    assert f.T.shape == (8, 6, 4, 3) and f.transpose(0, 2, 1, 3).shape == (3, 6, 4, 8)
    assert f.apply_fn(torch.clamp, min=0.0).min() >= 0
    assert f.block_until_ready() is f
    # numpy-backed fields behave the same way
    g = _density(x[0])
    assert g.mean() == pytest.approx(x[0].mean()) and g.T.shape == MESH[::-1]


def test_arithmetic_keeps_metadata():
    a = torch.full(MESH, 2.0)
    b = torch.full(MESH, 0.5)
    f, g = _density(a), _density(b)
    delta = f / f.mean() - 1
    assert isinstance(delta, jf.DensityField) and delta.box_size == f.box_size and delta.unit == f.unit
    assert torch.equal(delta.array, torch.zeros(MESH))
    assert torch.equal((f + g).array, a + b) and torch.equal((f - g).array, a - b)
    assert torch.equal((f * g).array, a * b) and torch.equal((f / g).array, a / b)
    assert torch.equal((3 * f).array, 3 * a) and torch.equal((1 + f).array, 1 + a)
    assert torch.equal((1 - f).array, 1 - a) and torch.equal((1 / f).array, 1 / a)
    assert torch.equal((-f).array, -a) and (+f) is f and torch.equal(abs(-f).array, a)
    assert torch.equal(sum([f, g]).array, a + b)


def test_full_like_and_metadata():
    base = _density(torch.zeros(MESH), nside=4, flatsky_npix=(5, 7), field_size=(2.0, 3.0))
    d = jf.DensityField.full_like(base, 2.5)
    assert d.shape == MESH and torch.all(d.array == 2.5) and d.box_size == base.box_size
    p = jf.ParticleField.full_like(base)
    assert p.shape == (*MESH, 3) and torch.all(p.array == 0)
    s = jf.SphericalDensity.full_like(base, 1.0)
    assert s.shape == (12 * 16,) and s.nside == 4
    fl = jf.FlatDensity.full_like(base, -1.0)
    assert fl.shape == (5, 7)
    with pytest.raises(ValueError, match="nside"):
        jf.SphericalDensity.full_like(base.replace(nside=None))
    with pytest.raises(ValueError, match="flatsky_npix"):
        jf.FlatDensity.full_like(base.replace(flatsky_npix=None))
    m = base.to_metadata()
    assert isinstance(m, jf.FieldMetadata) and m.array is None
    assert (m.mesh_size, m.box_size, m.nside, m.flatsky_npix, m.status, m.unit) == \
           (base.mesh_size, base.box_size, base.nside, base.flatsky_npix, base.status, base.unit)
    assert not m.is_batched() and not m.is_multi_batched()
    with pytest.raises(NotImplementedError):
        jf.FieldMetadata.full_like(base)


# ---------------------------------------------- spectral comparisons, with the spectra faked
def _fake_power(mesh, mesh2=None, *, box_shape, kedges=None, multipoles=0, los=(0.0, 0.0, 1.0)):
    """Stands in for the GPU P(k): one 'bin' per value of a 3-vector, <m1 m2> times (1, 2, 3)."""
    m2 = mesh if mesh2 is None else mesh2
    v = float((mesh.double() * m2.double()).mean())
    return torch.tensor([0.1, 0.2, 0.3]), torch.tensor([v, 2 * v, 3 * v])


def test_density_cross_power_transfer_coherence(monkeypatch):
    pw = importlib.import_module("jfli_b200.power")  # the package's `power` attribute is the function

    monkeypatch.setattr(pw, "power", _fake_power)
    rng = np.random.default_rng(1)
    a = torch.as_tensor(rng.uniform(1, 2, (3, *MESH)))
    f = _density(a, scale_factors=np.array([0.5, 0.7, 0.9]))
    cp = f.cross_power()
    assert cp.name == "cross_pk" and tuple(cp.array.shape) == (6, 3)
    order = [(i, j) for i in range(3) for j in range(i, 3)]
    for row, (i, j) in zip(cp.array, order):
        assert float(row[0]) == pytest.approx(float((a[i] * a[j]).mean()))
    with pytest.raises(ValueError, match="batched"):
        f[0].cross_power()
    with pytest.raises(ValueError, match="at least 2"):
        _density(a[:1]).cross_power()

    g = f * 2.0
    tr = f.transfer(g)
    assert tr.name == "transfer" and tuple(tr.array.shape) == (3, 3)
    np.testing.assert_allclose(tr.array.numpy(), 2.0, rtol=1e-12)  # sqrt(P(2a) / P(a))
    co = f[0].coherence(g[0])
    assert tuple(co.array.shape) == (3,)
    np.testing.assert_allclose(co.array.numpy(), 1.0, rtol=1e-6)  # P01 / sqrt(P0 P1) of a and 2a
    with pytest.raises(ValueError, match="match shape"):
        f.transfer(g[0])


def test_map_transfer_and_coherence(monkeypatch):
    pw = importlib.import_module("jfli_b200.power")  # the package's `power` attribute is the function

    def fake_flat(m1, m2=None, *, pixel_size=None, field_size=None, ell_edges=None):
        m2 = m1 if m2 is None else m2
        v = (m1.double() * m2.double()).mean(dim=(-2, -1))
        return torch.tensor([10.0, 20.0]), torch.stack([v, 4 * v], -1)

    def fake_sph(m1, m2=None, *, lmax=None, method="jax"):
        m2 = m1 if m2 is None else m2
        v = (m1.double() * m2.double()).mean()
        return torch.arange(3, dtype=torch.float64), torch.stack([v, v, v])

    monkeypatch.setattr(pw, "angular_cl_flat", fake_flat)
    monkeypatch.setattr(pw, "angular_cl_spherical", fake_sph)
    rng = np.random.default_rng(2)
    fl = jf.FlatDensity(array=torch.as_tensor(rng.uniform(1, 2, (2, 5, 7))), flatsky_npix=(5, 7),
                        field_size=(1.0, 1.0), **META)
    tr = fl.transfer(fl * 3.0)
    np.testing.assert_allclose(tr.array.numpy(), 3.0, rtol=1e-12)
    co = fl.coherence(fl * 3.0)
    np.testing.assert_allclose(co.array.numpy(), 1.0, rtol=1e-12)
    sp = jf.SphericalDensity(array=torch.as_tensor(rng.uniform(1, 2, 192)), nside=4, **META)
    np.testing.assert_allclose(sp.transfer(sp * 4.0).array.numpy(), 4.0, rtol=1e-12)
    np.testing.assert_allclose(sp.coherence(-sp).array.numpy(), -1.0, rtol=1e-12)


def test_project():
    rng = np.random.default_rng(3)
    a = torch.as_tensor(rng.standard_normal((2, *MESH)).astype(np.float32))
    f = _density(a)
    p = f[0].project(nz_slices=3)
    assert isinstance(p, jf.FlatDensity) and p.status == jf.FieldStatus.PROJECTED_DENSITY
    assert p.flatsky_npix == (4, 6) and p.box_size == f.box_size
    assert torch.allclose(p.array, a[0, :, :, -3:].sum(-1))
    pb = f.project()
    assert tuple(pb.array.shape) == (2, 4, 6) and torch.allclose(pb.array, a.sum(-1))
    with pytest.raises(ValueError):
        _density(torch.zeros(2, 2, *MESH)).project()


def _resize_loop(a, n_out):
    """jax.image.resize 'bilinear' along both axes, restated with explicit loops."""
    def axis_w(n_in):
        scale = n_out / n_in
        width = max(1.0 / scale, 1.0)
        W = np.zeros((n_in, n_out))
        for j in range(n_out):
            s = (j + 0.5) / scale - 0.5
            col = [max(0.0, 1.0 - abs(s - i) / width) for i in range(n_in)]
            tot = sum(col)
            if abs(tot) > 1000 * np.finfo(np.float32).eps and -0.5 <= s <= n_in - 0.5:
                W[:, j] = np.array(col) / tot
        return W

    return axis_w(a.shape[0]).T @ a @ axis_w(a.shape[1])


@pytest.mark.parametrize("n_in,n_out", [(8, 16), (16, 8), (12, 5), (6, 6)])
def test_flat_ud_sample(n_in, n_out):
    rng = np.random.default_rng(n_in + n_out)
    a = rng.standard_normal((2, n_in, n_in))
    fl = jf.FlatDensity(array=torch.as_tensor(a), flatsky_npix=(n_in, n_in), **META)
    out = fl.ud_sample(n_out)
    assert out.flatsky_npix == (n_out, n_out) and tuple(out.array.shape) == (2, n_out, n_out)
    for b in range(2):
        np.testing.assert_allclose(out.array[b].numpy(), _resize_loop(a[b], n_out), rtol=1e-12, atol=1e-12)
    one = jf.FlatDensity(array=torch.ones(n_in, n_in, dtype=torch.float64), flatsky_npix=(n_in, n_in), **META)
    np.testing.assert_allclose(one.ud_sample(n_out).array.numpy(), 1.0, rtol=1e-12)
    if n_in == n_out:
        np.testing.assert_allclose(out.array.numpy(), a, rtol=1e-12)


def test_flat_ud_sample_linear_ramp():
    ramp = np.tile(np.arange(16, dtype=np.float64)[:, None], (1, 16))
    fl = jf.FlatDensity(array=torch.as_tensor(ramp), flatsky_npix=(16, 16), **META)
    up = fl.ud_sample(32).array.numpy()
    j = np.arange(32)
    np.testing.assert_allclose(up[2:-2, 5], (j / 2 - 0.25)[2:-2], rtol=1e-12)  # interpolation at j/2 - 1/4
    down = fl.ud_sample(8).array.numpy()
    np.testing.assert_allclose(down[1:-1, 3], (2 * np.arange(8) + 0.5)[1:-1], rtol=1e-12)  # antialiased mean


def test_flat_cross_angular_cl_pairs(monkeypatch):
    pw = importlib.import_module("jfli_b200.power")

    def fake_flat(m1, m2=None, *, pixel_size=None, field_size=None, ell_edges=None):
        m2 = m1 if m2 is None else m2
        return torch.tensor([10.0, 20.0]), torch.stack([(m1 * m2).mean(), 2 * (m1 * m2).mean()])

    monkeypatch.setattr(pw, "angular_cl_flat", fake_flat)
    rng = np.random.default_rng(4)
    a = torch.as_tensor(rng.uniform(1, 2, (3, 5, 7)))
    fl = jf.FlatDensity(array=a, flatsky_npix=(5, 7), field_size=(1.0, 1.0), **META)
    cc = fl.cross_angular_cl()
    assert cc.name == "cross_cl" and tuple(cc.array.shape) == (6, 2)
    for row, (i, j) in zip(cc.array, [(i, j) for i in range(3) for j in range(i, 3)]):
        assert float(row[0]) == pytest.approx(float((a[i] * a[j]).mean()))
    with pytest.raises(ValueError, match="batched"):
        fl[0].cross_angular_cl()


def test_spherical_ud_sample_and_base_full_like():
    from oracle import healpix as oh

    rng = np.random.default_rng(7)
    m = rng.uniform(size=(2, 12 * 64))
    sp = jf.SphericalDensity(array=torch.as_tensor(m), nside=8, **META)
    down = sp.ud_sample(2)
    assert down.nside == 2 and tuple(down.array.shape) == (2, 48)
    np.testing.assert_allclose(down.array[1].numpy(), oh.ud_grade_ring(m[1], 2), rtol=1e-12)
    assert sp.ud_sample(16).nside == 16
    with pytest.raises(NotImplementedError):
        jf.AbstractField.full_like(sp)
