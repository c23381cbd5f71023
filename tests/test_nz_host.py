"""Redshift distributions on the host: the Gaussian-KDE n(z) (jax_cosmo.redshift.kde_nz, as
the reference's io/cosmogrid.py:25-67 builds the Stage-3 bins) and the Stage-3 loader, on
synthetic tables written here; Born weights of a narrow KDE against a single source plane."""

import importlib.util
import math

import numpy as np
import pytest

import jfli_b200 as jf
from jfli_b200 import lensing


def _kde_loop(z, zcat, w, bw, zmax):
    """The KDE restated with explicit loops and its Simpson normalisation on [0, zmax]."""
    def raw(t):
        s = 0.0
        for zi, wi in zip(zcat, w):
            s += wi * math.exp(-((t - zi) ** 2) / (2 * bw * bw)) / (math.sqrt(2 * math.pi) * bw)
        return s / sum(w)

    n = 256
    h = zmax / n
    norm = sum((1 if i in (0, n) else (4 if i % 2 else 2)) * raw(i * h) for i in range(n + 1)) * h / 3
    return np.array([raw(t) / norm for t in z])


def test_kde_nz_matches_loop_restatement():
    rng = np.random.default_rng(3)
    zcat = rng.uniform(0.1, 1.8, 40)
    w = rng.uniform(0.0, 2.0, 40)
    nz = jf.kde_nz(zcat, w, bw=0.07, zmax=2.5, gals_per_arcmin2=6.0)
    z = np.linspace(0.0, 2.5, 31)
    np.testing.assert_allclose(nz(z), _kde_loop(z, zcat, w, 0.07, 2.5), rtol=1e-12, atol=1e-14)
    assert nz.gals_per_arcmin2 == 6.0
    assert nz.gals_per_steradian == pytest.approx(6.0 * (180 * 60 / math.pi) ** 2)
    assert float(nz(0.9)) == pytest.approx(float(nz(np.array([0.9]))[0]))


def test_kde_nz_normalised_and_checked():
    nz = jf.kde_nz([0.4, 0.6, 1.1], [1.0, 3.0, 0.5], bw=0.02, zmax=3.0)
    z = np.linspace(0.0, 3.0, 257)
    assert np.sum(lensing.simpson_weights(0.0, 3.0, 256) * nz(z)) == pytest.approx(1.0, abs=1e-12)
    with pytest.raises(ValueError):
        jf.kde_nz([0.4, 0.6], [1.0], bw=0.02)
    with pytest.raises(ValueError):
        jf.kde_nz([], [], bw=0.02)
    with pytest.raises(ValueError):
        jf.kde_nz([0.4], [1.0], bw=0.0)


def _write_tables(d, nbins=4):
    z = np.linspace(0.0, 4.0, 1000)
    tabs = []
    for b in range(nbins):
        nz = np.exp(-0.5 * ((z - 0.3 - 0.25 * b) / 0.15) ** 2)
        np.savetxt(d / f"nz_stage3_{b + 1}.txt", np.stack([z, nz], 1))
        tabs.append((z, nz))
    return tabs


def test_stage3_loader_reads_bins_in_order(tmp_path):
    tabs = _write_tables(tmp_path)
    out = jf.io.get_stage3_nz_shear(data_dir=tmp_path)
    assert len(out) == 4
    assert [d.gals_per_arcmin2 for d in out] == [7.0, 8.5, 7.5, 6.0]
    zt = np.linspace(0.05, 2.0, 13)
    for d, (z, nz) in zip(out, tabs):
        assert d.zmax == pytest.approx(4.0)
        np.testing.assert_allclose(d(zt), jf.kde_nz(z, nz, bw=0.01, zmax=4.0)(zt), rtol=1e-13)
    # the bins peak where their tables do
    peaks = [zt[np.argmax(d(zt))] for d in out]
    assert peaks == sorted(peaks)
    custom = jf.io.get_stage3_nz_shear(gals_per_arcmin2=[1, 2, 3, 4], bw=0.05, zmax=3.0, data_dir=tmp_path)
    assert [d.gals_per_arcmin2 for d in custom] == [1.0, 2.0, 3.0, 4.0]
    assert custom[0].zmax == 3.0


def test_stage3_loader_without_tables(tmp_path):
    with pytest.raises(FileNotFoundError):
        jf.io.get_stage3_nz_shear(data_dir=tmp_path)
    if importlib.util.find_spec("jax_fli") is None:
        with pytest.raises(FileNotFoundError):
            jf.io.get_stage3_nz_shear()


def test_born_weights_of_narrow_kde_approach_a_single_source():
    """A KDE of one sample is a source plane at that z smoothed by the kernel: the Born
    weights differ from the single plane's by a term of order bw^2 (the kernel's variance
    times the lensing efficiency's curvature). The bandwidths stay above the 256-interval
    Simpson step that normalises n(z) on [0, 2]."""
    cosmo = jf.Planck18()
    a = np.linspace(0.6, 0.98, 12)
    w_src, _ = lensing.born_weights(cosmo, a, 1500.0, [0.8])
    dev = []
    for bw in (0.01, 0.02):
        nz = jf.kde_nz([0.8], [1.0], bw=bw, zmax=2.0)
        w_kde, z_eff = lensing.born_weights(cosmo, a, 1500.0, [nz], n_integrate=4000)
        assert z_eff[0] == pytest.approx(0.8, abs=1e-6)
        dev.append(np.abs(w_kde / w_src - 1).max())
    assert dev[0] < 2e-3
    assert dev[1] / dev[0] == pytest.approx(4.0, rel=0.1)
