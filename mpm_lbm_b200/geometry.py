"""Initial geometry of the FSI cases (host, init-only, not timed).

Restates the parts of the reference's geometry package that the FSI driver
uses to build its initial state:
  duct static geometry   src/mpm_lbm/sim/geometry/duct_flap_proxy.py:190-232
  flap masks             duct_flap_proxy.py:57-87, flap bounds 148-187
  deterministic sampler  src/mpm_lbm/sim/geometry/sampler.py:74-117, 159-180
plus a seeded jittered particle generator and non-cubic duct/plate cases used
by the benchmark configurations (not in the reference).
"""

from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np

DEFAULT_DUCT = {"x": [0.0, 1.0], "y": [0.3, 0.7], "z": [0.45, 0.55]}
DEFAULT_FLAP = {"anchor_x": 0.505, "anchor_y": 0.3, "height_over_duct_height": 0.25,
                "thickness_over_duct_height": 0.075, "normalized_height": 0.10, "normalized_thickness": 0.03,
                "z": [0.45, 0.55], "fixed_base": True, "mirrored_pair": False}
DEFAULT_MATERIAL = {"density": 1600.0, "youngs_modulus": 1.0e6, "poisson_ratio": 0.47,
                    "used_for_exact_structural_model": False}


@dataclass(frozen=True)
class GeometryConfig:
    """The fields of the reference's GeometryConfig (geometry/config.py:30-154) the FSI path reads."""

    geometry_type: str = "box"
    n_particles: int = 4096
    domain_min: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    domain_max: Tuple[float, float, float] = (1.0, 1.0, 1.0)
    box_min: Tuple[float, float, float] = (0.25, 0.35, 0.25)
    box_max: Tuple[float, float, float] = (0.55, 0.65, 0.55)
    center: Tuple[float, float, float] = (0.5, 0.5, 0.5)
    ellipsoid_radii: Tuple[float, float, float] = (0.15, 0.20, 0.12)
    duct: Optional[dict] = None
    flap: Optional[dict] = None
    material_reference: Optional[dict] = None
    dimensional_reference: Optional[dict] = None
    monitor_reference: Optional[dict] = None
    p_rho: float = 1.0
    particles_per_axis_hint: int = 32
    deterministic: bool = True
    quality_check_enabled: bool = False
    quality_check_strict: bool = False
    quality_report_path: Optional[str] = None
    extra: dict = field(default_factory=dict)

    @classmethod
    def from_json(cls, path):
        with open(path, "r", encoding="utf-8") as f:
            data = json.load(f)
        known = {k: v for k, v in data.items() if k in cls.__dataclass_fields__}
        extra = {k: v for k, v in data.items() if k not in cls.__dataclass_fields__}
        for k in ("domain_min", "domain_max", "box_min", "box_max", "center", "ellipsoid_radii"):
            if k in known:
                known[k] = tuple(float(v) for v in known[k])
        return cls(**known, extra=extra)


def _duct(cfg):
    return dict(DEFAULT_DUCT if cfg.duct is None else cfg.duct)


def _flap(cfg):
    return dict(DEFAULT_FLAP if cfg.flap is None else cfg.flap)


def _inside(points, lo, hi):
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    return np.all((points >= lo) & (points <= hi), axis=1)


def flap_bounds(cfg):
    f = _flap(cfg)
    h = 0.5 * float(f["normalized_thickness"])
    lo = np.array([float(f["anchor_x"]) - h, float(f["anchor_y"]), float(f["z"][0])])
    hi = np.array([float(f["anchor_x"]) + h, float(f["anchor_y"]) + float(f["normalized_height"]), float(f["z"][1])])
    out = [(lo, hi, "y_min")]
    if bool(f.get("mirrored_pair", False)):
        d = _duct(cfg)
        lo2 = np.array([lo[0], float(d["y"][1]) - float(f["normalized_height"]), lo[2]])
        hi2 = np.array([hi[0], float(d["y"][1]), hi[2]])
        out.append((lo2, hi2, "y_max"))
    return out


def flap_component_masks(points, cfg):
    pts = np.asarray(points, dtype=np.float64)
    f = _flap(cfg)
    flap = np.zeros(len(pts), bool)
    base = np.zeros(len(pts), bool)
    tip = np.zeros(len(pts), bool)
    bt = max(float(f["normalized_thickness"]), 0.2 * float(f["normalized_height"]))
    for lo, hi, side in flap_bounds(cfg):
        cur = _inside(pts, lo, hi)
        flap |= cur
        if side == "y_max":
            base |= _inside(pts, [lo[0], max(lo[1], hi[1] - bt), lo[2]], hi) & cur
            tip |= _inside(pts, lo, [hi[0], min(hi[1], lo[1] + bt), hi[2]]) & cur
        else:
            base |= _inside(pts, lo, [hi[0], min(hi[1], lo[1] + bt), hi[2]]) & cur
            tip |= _inside(pts, [lo[0], max(lo[1], hi[1] - bt), lo[2]], hi) & cur
    return {"flap": flap, "fixed_base": base, "free_tip_proxy": tip}


def duct_static_geometry(n_grid, cfg):
    """Solid mask (n,n,n): cells whose centre lies outside the duct are solid."""
    c = (np.arange(n_grid, dtype=np.float64) + 0.5) / float(n_grid)
    pts = np.stack(np.meshgrid(c, c, c, indexing="ij"), axis=-1).reshape(-1, 3)
    d = _duct(cfg)
    inside = _inside(pts, [d["x"][0], d["y"][0], d["z"][0]], [d["x"][1], d["y"][1], d["z"][1]])
    solid = np.ones(n_grid ** 3, np.int8)
    solid[inside] = 0
    solid = solid.reshape(n_grid, n_grid, n_grid)
    fluid = solid == 0
    report = {"duct_wall_cell_count": int(np.count_nonzero(solid)), "fluid_cell_count": int(np.count_nonzero(fluid)),
              "inlet_fluid_cell_count": int(np.count_nonzero(fluid[0])),
              "pressure_outlet_fluid_cell_count": int(np.count_nonzero(fluid[-1])),
              "solid_cell_count": int(np.count_nonzero(solid)), "flap_static_cell_count": 0}
    return solid, report


def sample_particles(cfg: GeometryConfig):
    """Deterministic candidate-lattice sampler (sampler.py:74-117)."""
    if cfg.geometry_type not in ("box", "ellipsoid", "duct_flap_proxy"):
        raise NotImplementedError(f"geometry_type={cfg.geometry_type!r} sampling is not supported here")
    dmin = np.asarray(cfg.domain_min, np.float64)
    dmax = np.asarray(cfg.domain_max, np.float64)
    span = dmax - dmin

    def inside(p):
        if cfg.geometry_type == "box":
            return _inside(p, cfg.box_min, cfg.box_max)
        if cfg.geometry_type == "ellipsoid":
            r = np.asarray(cfg.ellipsoid_radii)
            return np.sum(((p - np.asarray(cfg.center)) / r) ** 2, axis=1) <= 1.0
        return flap_component_masks(p, cfg)["flap"]

    min_fraction = 0.025 if cfg.geometry_type == "box" else 0.015
    res = max(int(cfg.particles_per_axis_hint), int(math.ceil((cfg.n_particles / min_fraction) ** (1.0 / 3.0))), 16)
    for _ in range(8):
        coords = dmin + (np.arange(res, dtype=np.float64) + 0.5)[:, None] * (span / float(res))
        x, y, z = np.meshgrid(coords[:, 0], coords[:, 1], coords[:, 2], indexing="ij")
        cand = np.column_stack((x.ravel(), y.ravel(), z.ravel()))
        mask = inside(cand)
        if int(np.count_nonzero(mask)) >= cfg.n_particles:
            break
        res = int(math.ceil(res * 1.35))
    else:
        raise RuntimeError(f"geometry_type={cfg.geometry_type} produced too few inside candidates")
    pts = cand[mask]
    n = cfg.n_particles
    sel = pts.copy() if len(pts) == n else pts[np.linspace(0, len(pts) - 1, n, dtype=np.int64)].copy()
    volume = float(np.prod(span)) * float(np.count_nonzero(mask)) / float(res ** 3)
    vol0 = np.full(n, volume / n, dtype=np.float32)
    cloud = {"x": sel.astype(np.float32), "vol0": vol0, "mass": (vol0 * np.float32(cfg.p_rho)).astype(np.float32),
             "geometry_volume": volume, "sampling_stats": {"candidate_resolution": res,
                                                           "accepted_count": int(len(pts)), "particle_count": n}}
    if cfg.geometry_type == "duct_flap_proxy":
        m = flap_component_masks(sel, cfg)
        cloud["fixed_base_mask"] = m["fixed_base"].astype(np.int8)
        cloud["free_tip_proxy_mask"] = m["free_tip_proxy"].astype(np.int8)
    return cloud


# ------------------------------------------------ benchmark case builders
def jittered_block(lo_cell, hi_cell, dx, ppc_axis=2, seed=0):
    """Particles at the ppc_axis^3 sub-cell centres of every cell in [lo, hi) with
    uniform jitter U(-dx/(2 ppc_axis), +) per axis (seeded); normalised units."""
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo_cell)
    hi = np.asarray(hi_cell)
    cells = np.stack(np.meshgrid(*[np.arange(a, b) for a, b in zip(lo, hi)], indexing="ij"), -1).reshape(-1, 3)
    sub = (np.arange(ppc_axis) + 0.5) / ppc_axis
    offs = np.stack(np.meshgrid(sub, sub, sub, indexing="ij"), -1).reshape(-1, 3)
    pts = (cells[:, None, :] + offs[None, :, :]).reshape(-1, 3) * dx
    pts += rng.uniform(-0.5 / ppc_axis, 0.5 / ppc_axis, pts.shape) * dx
    return pts.astype(np.float32)


def walled_channel(nx, ny, nz):
    """Solid planes at j in {0, ny-1} and k in {0, nz-1}; periodic in x."""
    s = np.zeros((nx, ny, nz), np.int8)
    s[:, 0, :] = s[:, -1, :] = 1
    s[:, :, 0] = s[:, :, -1] = 1
    return s


def duct_plate_case(nx, ny, nz, plate_cells=(2, 32, 48), plate_x0=None, ppc_axis=2, seed=0, base_frac=0.2):
    """Duct of nx x ny x nz cells (walls at j in {0,ny-1}, k in {0,nz-1}) with a
    cantilevered plate: plate_cells = (thickness x, height y, span z) growing
    along +y from the y-min wall (the reference's orientation), fixed base =
    the bottom max(thickness, base_frac * height) cells.  Returns
    (solid, x, fixed_mask, free_tip_mask) in normalised units (dx = 1/nx)."""
    solid = walled_channel(nx, ny, nz)
    dx = 1.0 / nx
    tx, hy, sz = plate_cells
    x0 = nx // 4 if plate_x0 is None else plate_x0
    z0 = (nz - sz) // 2
    lo = (x0, 1, z0)
    hi = (x0 + tx, 1 + hy, z0 + sz)
    x = jittered_block(lo, hi, dx, ppc_axis, seed)
    ycell = x[:, 1] / dx
    base_h = max(tx, base_frac * hy)
    fixed = (ycell < 1 + base_h).astype(np.int8)
    tip = (ycell >= 1 + hy - base_h).astype(np.int8)
    return solid, x, fixed, tip
