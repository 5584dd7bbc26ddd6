"""Writes duct_plate_outlet_stability.json: the CPU oracle's per-FSI-step
flow statistics of the 128 x 64 x 64 duct/plate case (tau 0.55, inlet
u_x = 0.05, plate 2 x 32 x 48 cells, 24,576 particles, moving_boundary
subcycled with 120 LBM and 40 MPM substeps per FSI step) under two outlet
semantics:

  - regularized_velocity_pressure_limited (the official campaign's outlet,
    solvers/official_duct_flap_config.py:14);
  - equilibrium_all_population_reset (the reference's default, the one the
    benchmark runs).

Per FSI step it records the largest fluid speed, the fluid density range and
whether every population is finite.  The record is the oracle's evidence of
where the regularized outlet leaves the bounded regime in this case; the GPU
test (tests/test_gpu_duct_plate_parity.py) checks that the CUDA path follows
it.  The oracle is the C++ restatement of the reference's kernels
(oracle/fsi_oracle.cpp, pinned by the reference-generated fixtures); the
reference itself does not run here.

Usage: python tests/golden/make_outlet_stability_record.py [--steps 6] [--threads N]
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "duct_plate_outlet_stability.json")
SEMANTICS = ("regularized_velocity_pressure_limited", "equilibrium_all_population_reset")


def fsi_step_stats(lbm):
    fluid = lbm.solid == 0
    with np.errstate(all="ignore"):
        u = np.linalg.norm(lbm.v[fluid].astype(np.float64), axis=1)
        rho = lbm.rho[fluid].astype(np.float64)
        return {"max_speed": float(np.nanmax(u)) if np.isfinite(u).any() else float("inf"),
                "rho_min": float(np.nanmin(rho)), "rho_max": float(np.nanmax(rho)),
                "finite": bool(np.isfinite(lbm.F).all() and np.isfinite(lbm.v).all())}


def main(argv=None):
    from mpm_lbm_b200.cases import DuctPlateCase
    from oracle import oracle as orc

    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args(argv)
    rec = {"case": "duct_plate_128x64x64 tau 0.55 u_in 0.05 plate 2x32x48, S=120 LBM + M=40 MPM substeps per FSI step",
           "oracle": "oracle/fsi_oracle.cpp, FP32", "semantics": {}}
    for sem in SEMANTICS:
        case = DuctPlateCase(open_boundary=sem)
        drv = orc.fsi_driver_for_case(case, threads=args.threads)
        rows = []
        for k in range(args.steps):
            t0 = time.time()
            drv.step_once()
            row = {"fsi_step": k + 1, "lbm_substeps": (k + 1) * case.lbm_substeps, **fsi_step_stats(drv.lbm)}
            rows.append(row)
            print(sem, row, f"{time.time() - t0:.1f}s", flush=True)
        rec["semantics"][sem] = rows
    with open(OUT, "w") as f:
        json.dump(rec, f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
