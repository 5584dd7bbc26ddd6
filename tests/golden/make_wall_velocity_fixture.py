"""Generate the wall-velocity application fixture with the reference's own code.

TEST INFRASTRUCTURE.  Run in a container that holds the reference checkout
(read-only) at REF_ROOT.  The reference's
src/mpm_lbm/sim/wall_velocity/application.py applies seeded velocity grids
to a seeded solid_vel field (apply_wall_velocity_to_lbm_solid_vel) under both
policies, and validates a few application configs; the results go to
tests/golden/wall_velocity_ref.npz / wall_velocity_ref.json, which pin
mpm_lbm_b200.wall_velocity (tests/test_wall_velocity.py on the CPU,
tests/test_gpu_wall_velocity.py on the device).  ``inputs()`` rebuilds the
seeded arrays.  Usage::

    python tests/golden/make_wall_velocity_fixture.py --ref PATH
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
N = 12
# the four files an application config names, relative to a root directory
CONFIG_FILES = {"wall_velocity_config_path": "configs/wall_velocity_field.json",
                "boundary_motion_config_path": "configs/boundary_motion.json",
                "geometry_config_path": "configs/geometry.json", "region_config_path": "configs/regions.json"}


def inputs(seed=7, n=N):
    rng = np.random.default_rng(seed)
    before = (0.003 * rng.standard_normal((n, n, n, 3))).astype(np.float32)
    grid = 0.006 * rng.standard_normal((n, n, n, 3))
    grid[rng.random((n, n, n)) < 0.4] = 0.0
    grid[1, 2, 3] = (0.02, -0.01, 0.0)  # above the cap on its own
    return before, grid


def config_variants():
    """name -> overrides of the base application config (validation cases)."""
    return {"valid": {}, "replace": {"application_policy": "replace_capped"}, "cap_too_large": {"wall_velocity_cap_lbm": 0.2},
            "bad_policy": {"application_policy": "bogus"}, "populations": {"apply_to_lbm_populations": True},
            "missing_file": {"region_config_path": "configs/absent.json"}, "scope": {"scope_note": "smoke"}}


def make_root(path):
    for rel in CONFIG_FILES.values():
        full = os.path.join(path, rel)
        os.makedirs(os.path.dirname(full), exist_ok=True)
        with open(full, "w") as fh:
            fh.write("{}\n")


class _Field:
    def __init__(self, arr):
        self.arr = np.asarray(arr, dtype=np.float32).copy()

    def to_numpy(self):
        return self.arr.copy()

    def from_numpy(self, arr):
        self.arr[...] = np.asarray(arr, dtype=np.float32)


class _Lattice:
    def __init__(self, before):
        self.solid_vel = _Field(before)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("REF_ROOT"), help="reference checkout (or set REF_ROOT)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or REF_ROOT")
    sys.path.insert(0, HERE)
    import taichi_shim  # noqa: E402

    sys.modules.setdefault("taichi", taichi_shim)
    sys.path.insert(0, args.ref)
    from src.mpm_lbm.sim.wall_velocity import application as app  # noqa: E402
    from src.mpm_lbm.sim.wall_velocity import application_config as appcfg  # noqa: E402

    out_json = {"apply": {}, "validation": {}}
    arrays = {}
    with tempfile.TemporaryDirectory() as root:
        make_root(root)
        base = appcfg.WallVelocityApplicationConfig(
            application_id="fixture_application",
            **{k: os.path.join(root, v) for k, v in CONFIG_FILES.items()},
            scope_note="Step 36 opt-in experimental solid_vel application smoke only")
        before, grid = inputs()
        for policy in ("additive_capped", "replace_capped"):
            cfg = dataclasses.replace(base, application_policy=policy)
            lat = _Lattice(before)
            res = app.apply_wall_velocity_to_lbm_solid_vel(lat, grid, cfg)
            arrays[policy + "_after"] = lat.solid_vel.to_numpy()
            out_json["apply"][policy] = res
        for name, over in config_variants().items():
            fields = dict(over)
            for key, rel in CONFIG_FILES.items():
                fields[key] = os.path.join(root, over.get(key, rel))
            cfg = dataclasses.replace(base, **fields)
            rows = appcfg.validate_wall_velocity_application_config(cfg, root=root)
            out_json["validation"][name] = [[row["check"], bool(row["pass"])] for row in rows]
    np.savez_compressed(os.path.join(HERE, "wall_velocity_ref.npz"), **arrays)
    with open(os.path.join(HERE, "wall_velocity_ref.json"), "w") as fh:
        json.dump(out_json, fh, indent=1, sort_keys=True)
    print("wrote wall_velocity_ref.npz / .json")


if __name__ == "__main__":
    main()
