"""Generate the LBM restart fixture with the reference's own restart writer.

TEST INFRASTRUCTURE.  Run in a container that holds the reference checkout
(read-only) at REF_ROOT.  The reference's restart module
(src/mpm_lbm/sim/lbm/restart.py) needs only numpy and json, so it is loaded
from its file directly.  Seeded arrays of a 6^3 lattice go through its
write_lbm_restart_npz; the file it wrote (tests/golden/lbm_restart_ref.npz) and
the statistics dictionary it returned (tests/golden/lbm_restart_ref_stats.json)
pin mpm_lbm_b200.restart in tests/test_restart.py.  Usage::

    python tests/golden/make_restart_fixture.py --ref PATH
"""

from __future__ import annotations

import argparse
import importlib.util
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
N = 6


def fixture_arrays(seed=0, n=N):
    """The seeded arrays of the fixture (also rebuilt by the tests)."""
    rng = np.random.default_rng(seed)
    solid = np.zeros((n, n, n), np.int8)
    solid[:, 0, :] = 1
    solid[2:4, 2:4, 2:4] = 1
    static = solid.copy()
    static[2:4, 2:4, 2:4] = 0
    F = (rng.uniform(0.01, 0.2, (n, n, n, 19))).astype(np.float32)
    rho = F.sum(axis=-1).astype(np.float32)
    v = (0.01 * rng.standard_normal((n, n, n, 3))).astype(np.float32)
    return {"rho": rho, "v": v, "f": F.copy(), "F": F, "solid": solid, "static_solid": static}


def fixture_metadata(n=N):
    return {"lbm_boundary_condition_mode": "duct_velocity_inlet_pressure_outlet",
            "lbm_restart_scope": "rho_velocity_populations", "n_grid": n, "target_u_lbm": [0.05, 0.0, 0.0]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("REF_ROOT"), help="reference checkout (or set REF_ROOT)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or REF_ROOT")
    path = os.path.join(args.ref, "src", "mpm_lbm", "sim", "lbm", "restart.py")
    spec = importlib.util.spec_from_file_location("reference_lbm_restart", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = os.path.join(HERE, "lbm_restart_ref.npz")
    stats = mod.write_lbm_restart_npz(out, fixture_arrays(), fixture_metadata())
    with open(os.path.join(HERE, "lbm_restart_ref_stats.json"), "w") as fh:
        json.dump(stats, fh, indent=1, sort_keys=True)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
