"""Lightcone shell geometry (reference utils.py:22-312), host-side NumPy/FP64."""

from __future__ import annotations

import numpy as np

from . import cosmology as cj


def _compute_equal_vol_shells(R_last: float, N_total: int, min_width: float) -> np.ndarray:
    """Equal-volume shells with at most M outer shells of exactly `min_width`
    (reference utils.py:22-71). Returns N_total+1 ascending edges starting at 0."""
    R_start = 0.0
    if N_total * min_width > R_last - R_start:
        raise ValueError(f"Cannot fit {N_total} shells of min_width={min_width} Mpc/h in max_radius={R_last:.2f} Mpc/h")
    for M in range(N_total):
        R_split = R_last - M * min_width
        n_inner = N_total - M
        k = np.arange(n_inner + 1)
        R_inner = (R_start**3 + (k / n_inner) * (R_split**3 - R_start**3)) ** (1.0 / 3.0)
        if R_inner[-1] - R_inner[-2] >= min_width - 1e-10:
            if M > 0:
                return np.concatenate((R_inner, R_split + np.arange(1, M + 1) * min_width))
            return R_inner
    raise ValueError(
        f"No valid equal-volume + min_width partition found for nb_shells={N_total}, min_width={min_width}, "
        f"max_radius={R_last:.2f}"
    )


def compute_lightcone_shells(cosmo, field, nb_shells: int, equal_vol: bool = False, min_width: float = 50.0):
    """(r_center, a_center), both (nb_shells,), far-to-near (reference utils.py:176-230)."""
    max_radius = float(field.max_comoving_radius)
    if equal_vol:
        r_edges = _compute_equal_vol_shells(max_radius, nb_shells, float(min_width))[::-1]
    else:
        width = max_radius / nb_shells
        n_lens = int(max_radius // float(width))
        r_edges = np.linspace(0.0, float(n_lens) * float(width), n_lens + 1)[::-1]
    r_center = 0.5 * (r_edges[1:] + r_edges[:-1])
    return r_center, cj.a_of_chi(cosmo, r_center)


def edges(centers, r_left=None):
    """(2, N) left/right edges from centres (reference utils.py:247-281)."""
    c = np.asarray(centers, dtype=np.float64)
    desc = c[0] > c[-1]
    ca = c[::-1] if desc else c
    if r_left is None:
        r_left = 1.5 * ca[0] - 0.5 * ca[1]
    e = [float(r_left)]
    for ci in ca:
        e.append(2 * ci - e[-1])
    e = np.asarray(e)
    left, right = e[:-1], e[1:]
    if desc:
        left, right = left[::-1], right[::-1]
    return np.stack([left, right])


def distances(centers, r_left=None):
    e = edges(centers, r_left)
    return e[1] - e[0]


def centers(distances, r_left, is_descending=False):
    """Shell centres from shell widths laid out from r_left (reference utils.py:297-312)."""
    d = np.asarray(distances, dtype=np.float64)
    da = d[::-1] if is_descending else d
    r_edges = np.concatenate([[r_left], r_left + np.cumsum(da)])
    c = 0.5 * (r_edges[1:] + r_edges[:-1])
    return c[::-1] if is_descending else c


def compute_box_size_from_redshift(cosmo, max_redshift, observer_position):
    r = float(cj.radial_comoving_distance(cosmo, cj.z2a(max_redshift)))
    f = np.clip(np.asarray(observer_position, dtype=np.float64), 0.0, 1.0)
    return tuple(float(v) for v in (1.0 + 2.0 * np.minimum(f, 1.0 - f)) * r)


def compute_max_redshift_from_box_size(cosmo, box_size, observer_position):
    f = np.clip(np.asarray(observer_position, dtype=np.float64), 0.0, 1.0)
    r_eff = np.min(np.asarray(box_size, dtype=np.float64) / (1.0 + 2.0 * np.minimum(f, 1.0 - f)))
    return float(cj.a2z(cj.a_of_chi(cosmo, r_eff)))


def compute_particle_scale_factors(cosmo, field):
    """Per-particle a(|x - observer|) (reference utils.py:233-244)."""
    from .fields import PositionUnit

    pos = field.to(PositionUnit.MPC_H).array.detach().double().cpu().numpy()
    r = np.linalg.norm(pos - np.asarray(field.observer_position_mpc), axis=-1)
    return cj.a_of_chi(cosmo, r)
