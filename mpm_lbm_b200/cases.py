"""Duct-with-cantilevered-plate FSI cases, built for FSIDriver3D.

A case is a walled duct (solid planes at j in {0, ny-1} and k in {0, nz-1}),
a velocity inlet at x = 0 and a pressure outlet at x = nx - 1 (the duct mode
of the reference's driver, src/mpm_lbm/sim/drivers/fsi_driver.py:219-257),
and an elastic plate growing along +y from the y-min wall with a clamped
base (the reference's flap orientation, src/mpm_lbm/sim/geometry/
duct_flap_proxy.py:57-87).  Particles sit at the 2 x 2 x 2 sub-cell centres
of the plate's cells with a seeded uniform jitter.  The coupling is
moving_boundary with the engineering reaction transfer, subcycled: S LBM
substeps and M MPM substeps per FSI step.

tau and the solid's Young's modulus are given in lattice units and mapped to
the driver's physical inputs (fsi_config.py:376-445: nu_lbm = nu_phys dt /
dx^2, tau = 3 nu_lbm + 0.5; the MPM runs in normalised units where
E_norm = E_lu (dx / dt)^2).
"""

from __future__ import annotations

import tempfile
from dataclasses import dataclass, field
from typing import Tuple

import numpy as np

from .config import FSIDriverConfig
from .geometry import duct_plate_case


@dataclass(frozen=True)
class DuctPlateCase:
    lattice: Tuple[int, int, int] = (128, 64, 64)
    tau: float = 0.55
    u_in: float = 0.05
    plate: Tuple[int, int, int] = (2, 32, 48)   # cells: thickness (x), height (y), span (z)
    lbm_substeps: int = 120                     # S
    mpm_substeps: int = 40                      # M per FSI step
    dt_lbm: float = 1.0e-3                      # physical seconds per LBM step
    e_lu: float = 0.02
    nu_poisson: float = 0.3
    rho_s: float = 1.2
    open_boundary: str = "equilibrium_all_population_reset"
    # per-particle reaction cap (normalised units) at 128 cells along x, scaled
    # with the particle volume
    reaction_cap_128: float = 1.0e-8
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def nx(self):
        return self.lattice[0]

    @property
    def cells(self):
        return self.lattice[0] * self.lattice[1] * self.lattice[2]

    @property
    def n_particles(self):
        return self.plate[0] * self.plate[1] * self.plate[2] * 8

    @property
    def reaction_cap(self):
        return self.reaction_cap_128 * (128.0 / self.nx) ** 3

    def config(self, **overrides) -> FSIDriverConfig:
        nx = self.nx
        dx_phys = 1.0 / nx
        nu_phys = (self.tau - 0.5) / 3.0 * dx_phys ** 2 / self.dt_lbm
        S, M = self.lbm_substeps, self.mpm_substeps
        kw = dict(
            coupling_mode="moving_boundary", n_grid=nx, n_particles=self.n_particles, n_lbm_steps=10 ** 6,
            mpm_substeps_per_lbm_step=M, mpm_dt=S * self.dt_lbm / M, target_u_lbm=(self.u_in, 0.0, 0.0),
            lbm_boundary_condition_mode="duct_velocity_inlet_pressure_outlet",
            lbm_open_boundary_semantics=self.open_boundary, mb_force_cap_norm=self.reaction_cap,
            fsi_exchange_mode="lbm_subcycled_per_fsi_step", lbm_substeps_per_fsi_step=S,
            lbm_dt_phys_override_s=self.dt_lbm, official_fsi_dt_s=S * self.dt_lbm,
            target_u_lbm_for_dimensional_mapping=self.u_in, physical_duct_length_m=1.0,
            target_inlet_velocity_mps=self.u_in * dx_phys / self.dt_lbm,
            lbm_viscosity_semantics="physical_nu_mapping", fluid_kinematic_viscosity_m2_s=nu_phys,
            output_interval=10)
        kw.update(self.extra)
        kw.update(overrides)
        return FSIDriverConfig(**kw)

    def geometry(self):
        """(static solid (nx, ny, nz) int8, particle dict) in normalised units."""
        nx, ny, nz = self.lattice
        solid, x, fixed, tip = duct_plate_case(nx, ny, nz, plate_cells=self.plate, seed=self.seed)
        dx = 1.0 / nx
        vol0 = np.full(len(x), dx ** 3 / 8.0, np.float32)
        mass = (vol0 * np.float32(self.rho_s)).astype(np.float32)
        return solid, {"x": x, "vol0": vol0, "mass": mass, "fixed": fixed, "free_tip": tip}

    def material(self):
        e_norm = self.e_lu * ((1.0 / self.nx) / self.dt_lbm) ** 2
        return {"young_modulus": e_norm, "poisson_ratio": self.nu_poisson, "p_rho": self.rho_s}

    def make_driver(self, out_dir=None, storage="fp32", graph=False, device="cuda", **kw):
        from .driver import FSIDriver3D

        solid, parts = self.geometry()
        out = out_dir if out_dir is not None else tempfile.mkdtemp(prefix="fsi_case_")
        drv = FSIDriver3D(self.config(), out, population_storage=storage, lattice_shape=tuple(self.lattice),
                          material=self.material(), static_solid=solid, initial_particles=parts,
                          use_cuda_graph=graph, device=device, **kw)
        drv.initialize()
        return drv
