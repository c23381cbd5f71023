"""HEALPix orderings and resolution changes for painted shells.

The reference paints a shell at `PaintingOptions.paint_nside` and brings it to the field's
nside with jax-healpy's `ud_grade` (reference _src/fields/_painting.py:249-348, options
from fields/painting.py:78-96; the painter itself is in jax-fli's JaxPM fork, which is not
vendored). jax-healpy follows healpy's `ud_grade`, restated here:
- the map is taken to NESTED order (where the 4^k children of a pixel at nside / 2^k are
  consecutive), unless it is NESTED already (order_in);
- degrading averages each parent's children that are not bad (UNSEEN within healpy's
  tolerance); a parent with no good child, or with pess=True any bad child, is UNSEEN (as
  in healpy, a non-finite child counts as bad but still propagates through the sum);
  upgrading copies each parent to its children;
- power p scales the result by (nside_out / nside_in)^p (p = -2 keeps the sum of the map);
- the result is returned in order_out.

RING <-> NESTED indices follow the HEALPix pixelisation (Gorski et al. 2005): a NESTED
index is (face, x, y) with x, y bit-interleaved inside the face; the RING index of
(face, x, y) follows from the face's ring and phase offsets. The tables are built once per
nside on the host (int64) and moved to the map's device.
"""

from __future__ import annotations

import functools

import numpy as np
import torch

UNSEEN = -1.6375e30

_FACE_RING = np.array([2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4], dtype=np.int64)  # ring of a face's corner, / nside
_FACE_PHASE = np.array([1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7], dtype=np.int64)  # phase of a face's corner


def _check_nside(nside: int) -> int:
    nside = int(nside)
    if nside < 1 or nside & (nside - 1):
        raise ValueError(f"nside must be a power of 2, got {nside}")
    return nside


def npix2nside(npix: int) -> int:
    nside = int(round((npix / 12) ** 0.5))
    if 12 * nside * nside != npix:
        raise ValueError(f"{npix} is not a valid HEALPix pixel count")
    return _check_nside(nside)


def _even_bits(v: np.ndarray) -> np.ndarray:
    """The even-position bits of v packed into the low half (inverse of bit interleaving)."""
    v = v & 0x5555555555555555
    v = (v | (v >> 1)) & 0x3333333333333333
    v = (v | (v >> 2)) & 0x0F0F0F0F0F0F0F0F
    v = (v | (v >> 4)) & 0x00FF00FF00FF00FF
    v = (v | (v >> 8)) & 0x0000FFFF0000FFFF
    v = (v | (v >> 16)) & 0x00000000FFFFFFFF
    return v


def nest2ring(nside: int, ipix) -> np.ndarray:
    """RING index of NESTED pixel(s) ipix."""
    nside = _check_nside(nside)
    n = np.asarray(ipix, dtype=np.int64)
    face = n // (nside * nside)
    inface = n % (nside * nside)
    x, y = _even_bits(inface), _even_bits(inface >> 1)
    ring = _FACE_RING[face] * nside - x - y - 1  # 1 .. 4 nside - 1, north to south
    north, south = ring < nside, ring > 3 * nside
    nr = np.where(north, ring, np.where(south, 4 * nside - ring, nside))  # pixels per ring / 4
    first = np.where(north, 2 * nr * (nr - 1),
                     np.where(south, 12 * nside * nside - 2 * (nr + 1) * nr,
                              2 * nside * (nside - 1) + (ring - nside) * 4 * nside))
    shift = np.where(north | south, 0, (ring - nside) & 1)
    phase = (_FACE_PHASE[face] * nr + x - y + 1 + shift) // 2
    phase = np.where(phase > 4 * nside, phase - 4 * nside, np.where(phase < 1, phase + 4 * nside, phase))
    return first + phase - 1


@functools.lru_cache(maxsize=16)
def _nest2ring_table(nside: int) -> np.ndarray:
    return nest2ring(nside, np.arange(12 * nside * nside, dtype=np.int64))


@functools.lru_cache(maxsize=16)
def _ring2nest_table(nside: int) -> np.ndarray:
    n2r = _nest2ring_table(nside)
    r2n = np.empty_like(n2r)
    r2n[n2r] = np.arange(n2r.size, dtype=np.int64)
    return r2n


def ring2nest(nside: int, ipix) -> np.ndarray:
    """NESTED index of RING pixel(s) ipix."""
    return _ring2nest_table(_check_nside(nside))[np.asarray(ipix, dtype=np.int64)]


_device_tables: dict = {}


def _table(kind: str, nside: int, device) -> torch.Tensor:
    key = (kind, nside, str(device))
    t = _device_tables.get(key)
    if t is None:
        host = _nest2ring_table(nside) if kind == "n2r" else _ring2nest_table(nside)
        t = torch.as_tensor(host, device=device)
        _device_tables[key] = t
    return t


def _order(order: str) -> str:
    o = str(order).upper()
    if o in ("NEST", "NESTED"):
        return "NESTED"
    if o == "RING":
        return "RING"
    raise ValueError(f"order must be 'RING' or 'NESTED', got {order!r}")


def reorder(m: torch.Tensor, order_in: str, order_out: str) -> torch.Tensor:
    """The maps m (..., npix) in order_out."""
    order_in, order_out = _order(order_in), _order(order_out)
    if order_in == order_out:
        return m
    nside = npix2nside(int(m.shape[-1]))
    # RING -> NESTED: nested[n] = ring[nest2ring[n]]; NESTED -> RING: ring[r] = nested[ring2nest[r]]
    idx = _table("n2r" if order_in == "RING" else "r2n", nside, m.device)
    return m.index_select(-1, idx)


def ud_grade(m: torch.Tensor, nside_out: int, *, pess: bool = False, order_in: str = "RING",
             order_out: str | None = None, power: float | None = None) -> torch.Tensor:
    """healpy.ud_grade of the maps m (..., npix) to nside_out (module docstring)."""
    nside_out = _check_nside(nside_out)
    nside_in = npix2nside(int(m.shape[-1]))
    order_out = order_in if order_out is None else order_out
    x = reorder(m, order_in, "NESTED")
    ratio = (nside_out / nside_in) ** float(power) if power else 1.0
    lead = tuple(x.shape[:-1])
    if nside_out > nside_in:
        k = (nside_out // nside_in) ** 2
        out = (x.unsqueeze(-1) * ratio).expand(*lead, x.shape[-1], k).reshape(*lead, 12 * nside_out * nside_out)
    elif nside_out < nside_in:
        k = (nside_in // nside_out) ** 2
        xr = x.reshape(*lead, 12 * nside_out * nside_out, k)
        bad = (torch.abs(xr - UNSEEN) <= 1e-8 + 1e-5 * abs(UNSEEN)) | ~torch.isfinite(xr)
        good = ~bad
        total = (xr * good.to(xr.dtype)).sum(-1)  # as healpy: a non-finite child gives a non-finite sum
        nhit = good.sum(-1).to(total.dtype)
        out = torch.where(nhit > 0, total / torch.where(nhit > 0, nhit, torch.ones_like(nhit)) * ratio, total)
        badout = (nhit < k) if pess else (nhit == 0)
        out = torch.where(badout, torch.full_like(out, UNSEEN), out)
    else:
        out = x
    return reorder(out, "NESTED", order_out)
