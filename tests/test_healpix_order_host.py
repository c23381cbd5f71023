"""HEALPix orderings and ud_grade on the host (jfli_b200.healpix_order), and paint_nside in
spherical painting: NESTED <-> RING against healpy's documented examples and against the
RING geometry of the oracle (a child pixel's centre lies in its parent); ud_grade against
the oracle's restatement built on that geometry alone (no NESTED numbering)."""

import importlib
import json
from pathlib import Path

import numpy as np
import pytest
import torch

import jfli_b200 as jf
from jfli_b200 import healpix_order as ho
from oracle import healpix as oh

GOLDEN = json.loads((Path(__file__).parent / "golden" / "healpix_docs.json").read_text())


def test_orderings_match_healpy_examples():
    for case in GOLDEN["nest2ring"]:
        np.testing.assert_array_equal(ho.nest2ring(case["nside"], case["nest"]), case["ring"])
    for case in GOLDEN["ring2nest"]:
        np.testing.assert_array_equal(ho.ring2nest(case["nside"], case["ring"]), case["nest"])


@pytest.mark.parametrize("nside", [1, 2, 8, 64])
def test_orderings_follow_the_ring_geometry(nside):
    n2r = ho._nest2ring_table(nside)
    assert np.array_equal(np.sort(n2r), np.arange(12 * nside * nside))
    assert np.array_equal(ho.ring2nest(nside, n2r), np.arange(12 * nside * nside))
    nest = np.arange(12 * nside * nside)
    for nout in [v for v in (1, 2, 4, 16) if v < nside]:
        k = (nside // nout) ** 2
        parents = oh.ring_parents(nside, nout)[n2r]  # RING parent of each NESTED child
        assert np.array_equal(parents, ho._nest2ring_table(nout)[nest // k])


def test_reorder_round_trip():
    m = torch.arange(12 * 16 * 16, dtype=torch.float32).reshape(1, -1).repeat(2, 1)
    nest = ho.reorder(m, "RING", "NESTED")
    assert torch.equal(nest[0], m[0][torch.as_tensor(ho._nest2ring_table(16))])
    assert torch.equal(ho.reorder(nest, "NEST", "RING"), m)
    with pytest.raises(ValueError):
        ho.reorder(m, "RING", "SPIRAL")


@pytest.mark.parametrize("nin,nout", [(16, 4), (16, 8), (4, 16), (8, 8)])
@pytest.mark.parametrize("power", [None, -2.0, 2.0])
def test_ud_grade_matches_geometric_restatement(nin, nout, power):
    rng = np.random.default_rng(nin * 100 + nout)
    m = rng.uniform(0.5, 2.0, (2, 12 * nin * nin))
    out = ho.ud_grade(torch.as_tensor(m), nout, power=power)
    for row, ref in zip(out.numpy(), m):
        np.testing.assert_allclose(row, oh.ud_grade_ring(ref, nout, power=power), rtol=1e-12)
    if power == -2.0:
        np.testing.assert_allclose(out.sum(-1).numpy(), m.sum(-1), rtol=1e-12)  # sums kept


@pytest.mark.parametrize("pess", [False, True])
def test_ud_grade_unseen_pixels(pess):
    nin, nout = 8, 2
    rng = np.random.default_rng(5)
    m = rng.uniform(0.5, 2.0, 12 * nin * nin)
    m[rng.choice(m.size, 40, replace=False)] = ho.UNSEEN
    m[ho._nest2ring_table(nin)[:16]] = ho.UNSEEN  # every child of NESTED parent 0
    out = ho.ud_grade(torch.as_tensor(m), nout, pess=pess).numpy()
    ref = oh.ud_grade_ring(m, nout, pess=pess)
    np.testing.assert_allclose(out, ref, rtol=1e-12)
    assert out[ho.nest2ring(nout, 0)] == ho.UNSEEN
    assert (out == ho.UNSEEN).sum() >= (1 if not pess else 2)


def test_ud_grade_orders_and_checks():
    rng = np.random.default_rng(6)
    m = torch.as_tensor(rng.uniform(size=12 * 8 * 8))
    ring = ho.ud_grade(m, 4)
    assert torch.equal(ho.ud_grade(m, 4, order_out="NESTED"), ho.reorder(ring, "RING", "NESTED"))
    nested_in = ho.reorder(m, "RING", "NESTED")
    assert torch.allclose(ho.ud_grade(nested_in, 4, order_in="NESTED", order_out="RING"), ring)
    with pytest.raises(ValueError):
        ho.ud_grade(m, 3)
    with pytest.raises(ValueError):
        ho.ud_grade(torch.zeros(100), 2)


def test_paint_spherical_at_paint_nside(monkeypatch):
    """paint_nside: the shells are painted at paint_nside and graded to the field's nside."""
    painting = importlib.import_module("jfli_b200.painting")
    seen = []

    def fake_paint_shells(field, centers, widths, scheme="bilinear", weights=None, out=None, sigma=None):
        seen.append(field.nside)
        npix = 12 * field.nside * field.nside
        return torch.arange(npix, dtype=torch.float64).repeat(len(centers), 1) + 1.0

    monkeypatch.setattr(painting, "paint_shells", fake_paint_shells)
    parts = jf.ParticleField(array=torch.zeros(4, 4, 4, 3), mesh_size=(4, 4, 4), box_size=(10.0, 10.0, 10.0),
                             nside=4, unit=jf.PositionUnit.GRID_RELATIVE, status=jf.FieldStatus.PARTICLES)
    lc = parts.paint_spherical([3.0, 4.0], [1.0, 1.0], paint_nside=16, ud_grade_power=-2.0)
    assert seen == [16] and lc.nside == 4 and tuple(lc.array.shape) == (2, 192)
    ref = oh.ud_grade_ring(np.arange(12 * 256, dtype=np.float64) + 1.0, 4, power=-2.0)
    np.testing.assert_allclose(lc.array[0].numpy(), ref, rtol=1e-12)
    same = parts.paint_spherical(3.0, 1.0)
    assert seen[-1] == 4 and tuple(same.array.shape) == (192,)
    with pytest.raises(NotImplementedError):
        parts.paint_spherical(3.0, 1.0, paint_nside=16, ud_grade_order_in="NESTED")
    with pytest.raises(ValueError):
        parts.paint_spherical(3.0, 1.0, paint_nside=16, ud_grade_order_out="SPIRAL")


def test_tiled_interp_paint_nside_helpers():
    """OnionTiler / TelephotoInterp paint replicas at paint_nside and grade to the field's nside."""
    from jfli_b200.pm import interp

    parts = jf.ParticleField(array=torch.zeros(4, 4, 4, 3), mesh_size=(4, 4, 4), box_size=(10.0, 10.0, 10.0),
                             nside=4, unit=jf.PositionUnit.GRID_RELATIVE, status=jf.FieldStatus.PARTICLES)
    plain = jf.PaintingOptions(target="spherical")
    fine = jf.PaintingOptions(target="spherical", paint_nside=16, ud_grade_power=-2.0, ud_grade_order_out="NESTED")
    assert interp._at_paint_nside(parts, plain) is parts
    assert interp._at_paint_nside(parts, fine).nside == 16
    m = torch.arange(12 * 256, dtype=torch.float64)
    assert interp._regrade(m[:192], parts, plain) is not None
    graded = interp._regrade(m, parts, fine)
    ref = oh.ud_grade_ring(m.numpy(), 4, power=-2.0)
    np.testing.assert_allclose(graded.numpy(), ref[ho._nest2ring_table(4)], rtol=1e-12)  # NESTED out
