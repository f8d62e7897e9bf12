"""Planar pixel detector geometry and angular tiles.

Restates the reference's pixel-ray and tile construction
(src/pyrite/instrument/geometry.py:99-122 ``angular_tiles``) for a flat
detector whose centre sits at polar angle ``theta_obs`` from the beam
(+z lab), azimuth 0, at ``distance_mm``, facing the sample. Pixel centres are
uniform on the plane; a tile's direction is the solid-angle-weighted mean
of its pixels' unit directions; results are rotated into the sample frame
with the tilt rotation of ``tables.tilted_geometry``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .tables import sample_to_lab


@dataclass(frozen=True)
class PlanarDetector:
    theta_obs_rad: float
    distance_mm: float
    width_mm: float
    height_mm: float
    nx: int
    ny: int

    def pixel_rays(self):
        """Lab unit directions (ny, nx, 3) and solid angles (ny, nx) [sr]."""
        c = np.array([np.sin(self.theta_obs_rad), 0.0, np.cos(self.theta_obs_rad)])
        normal = -c
        x_axis = np.array([np.cos(self.theta_obs_rad), 0.0, -np.sin(self.theta_obs_rad)])
        y_axis = np.array([0.0, 1.0, 0.0])
        px = self.width_mm / self.nx
        py = self.height_mm / self.ny
        xs = (np.arange(self.nx) - (self.nx - 1) / 2.0) * px
        ys = (np.arange(self.ny) - (self.ny - 1) / 2.0) * py
        centre = c * self.distance_mm
        pts = centre[None, None, :] + ys[:, None, None] * y_axis + xs[None, :, None] * x_axis
        r = np.linalg.norm(pts, axis=-1)
        dirs = pts / r[..., None]
        cos_inc = np.abs(np.sum(dirs * -normal, axis=-1))
        omega = px * py * cos_inc / (r * r)
        return dirs, omega

    @property
    def solid_angle_sr(self) -> float:
        return float(self.pixel_rays()[1].sum())


def angular_tiles(det: PlanarDetector, angular_shape):
    """(tile index per pixel (ny, nx), tile lab directions (n_tile, 3),
    tile solid angles (n_tile,)) as instrument/geometry.py:99-122."""
    ay, ax = angular_shape
    if ay <= 0 or ax <= 0 or ay > det.ny or ax > det.nx:
        raise ValueError("angular_shape must be positive and not exceed the pixel shape")
    dirs, omega = det.pixel_rays()
    rows = np.array_split(np.arange(det.ny), ay)
    cols = np.array_split(np.arange(det.nx), ax)
    tile_index = np.empty((det.ny, det.nx), dtype=np.int64)
    out = np.empty((ay * ax, 3))
    w = np.empty(ay * ax)
    t = 0
    for r in rows:
        for c in cols:
            yy, xx = np.ix_(r, c)
            tile_index[yy, xx] = t
            wt = omega[yy, xx]
            v = np.sum(wt[..., None] * dirs[yy, xx, :], axis=(0, 1))
            out[t] = v / np.linalg.norm(v)
            w[t] = wt.sum()
            t += 1
    return tile_index, out, w


def tiles_in_sample_frame(det: PlanarDetector, angular_shape, tilt_polar_rad, tilt_azim_rad=0.0):
    """Tile directions rotated into the sample frame (v_sample = R^T v_lab)."""
    idx, lab, omega = angular_tiles(det, angular_shape)
    R = sample_to_lab(tilt_polar_rad, tilt_azim_rad)
    return idx, lab @ R, omega


def directions_at(det: PlanarDetector, uv, tilt_polar_rad, tilt_azim_rad=0.0):
    """Sample-frame unit directions toward detector-plane points at normalised
    coordinates ``uv[:, 0]`` (along the plane's x axis) and ``uv[:, 1]`` (y),
    each in [-1, 1] across the active area (the surrogate's pixel inputs)."""
    uv = np.atleast_2d(np.asarray(uv, dtype=float))
    c = np.array([np.sin(det.theta_obs_rad), 0.0, np.cos(det.theta_obs_rad)])
    x_axis = np.array([np.cos(det.theta_obs_rad), 0.0, -np.sin(det.theta_obs_rad)])
    y_axis = np.array([0.0, 1.0, 0.0])
    pts = (c * det.distance_mm)[None, :] + (0.5 * det.width_mm * uv[:, 0])[:, None] * x_axis \
        + (0.5 * det.height_mm * uv[:, 1])[:, None] * y_axis
    dirs = pts / np.linalg.norm(pts, axis=1, keepdims=True)
    return dirs @ sample_to_lab(tilt_polar_rad, tilt_azim_rad)


def tile_uv(det: PlanarDetector, angular_shape):
    """Normalised detector coordinates (n_tile, 2) of each angular tile's pixel
    centroid, in the tile order of ``angular_tiles``."""
    ay, ax = angular_shape
    xs = (np.arange(det.nx) - (det.nx - 1) / 2.0) / (det.nx / 2.0)
    ys = (np.arange(det.ny) - (det.ny - 1) / 2.0) / (det.ny / 2.0)
    out = []
    for r in np.array_split(np.arange(det.ny), ay):
        for c in np.array_split(np.arange(det.nx), ax):
            out.append((xs[c].mean(), ys[r].mean()))
    return np.asarray(out)
