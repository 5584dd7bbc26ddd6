"""Per-FSI-step reductions of the subcycled-flow campaign, on the device.

The reference's campaign caller
(src/mpm_lbm/solvers/official_subcycled_flow_solver.py) copies rho, v, f and
solid of the whole lattice to the host after every official FSI step
(_copy_lbm_fields, 352-365) and computes its gates there in FP64:
  - _stability_row (465-500): finiteness of rho, v and the populations over
    fluid cells, the density gate 0 < rho_min, rho_max < 5 and the J gate;
  - _mass_flux_row (503-540): the fluid mass sum(rho) over fluid cells, and
    the fluxes sum(rho * u_x) over the inlet, outlet and mid-plane masks.
Here one kernel pass (fsi_campaign_sums) produces the same sums from the
device state and returns about 100 bytes, and the rows are built from them
with the reference's field names, formulas and errors.  copy_lbm_fields is
kept for the steps that write velocity snapshots.
"""

from __future__ import annotations

import ctypes
import math
from typing import Any

import numpy as np
import torch

from ._lib import FSI_CAMPAIGN_REGIONS, FsiCampaignSums, call, ptr, stream_handle
from .fields import ref_to_lattice


def campaign_regions(masks: dict[str, dict[str, np.ndarray]]) -> dict[str, np.ndarray]:
    """The flux regions of _mass_flux_row (solver.py:509-515): the velocity
    inlet and pressure outlet masks, and the static fluid cells of the x
    mid-plane (x = nx // 2)."""
    boundary, geometry = masks["boundary"], masks["geometry"]
    static_fluid = np.asarray(geometry["fluid_mask"]).astype(bool)
    midplane = np.zeros_like(static_fluid, dtype=bool)
    mid = static_fluid.shape[0] // 2
    midplane[mid, :, :] = static_fluid[mid, :, :]
    return {"inlet": np.asarray(boundary["velocity_inlet_mask"]).astype(bool),
            "outlet": np.asarray(boundary["pressure_outlet_mask"]).astype(bool),
            "midplane": midplane}


class CampaignReductions:
    """fsi_campaign_sums for one lattice and a fixed set of named flux
    regions ((nx, ny, nz) boolean masks, at most FSI_CAMPAIGN_REGIONS)."""

    def __init__(self, lbm, regions: dict[str, np.ndarray]):
        if len(regions) > FSI_CAMPAIGN_REGIONS:
            raise ValueError(f"at most {FSI_CAMPAIGN_REGIONS} flux regions")
        self.lbm = lbm
        self.names = list(regions)
        code = np.zeros(lbm.dims, np.uint8)
        for bit, name in enumerate(self.names):
            mask = np.asarray(regions[name])
            if mask.shape != tuple(lbm.dims):
                raise ValueError(f"region {name!r} has shape {mask.shape}, the lattice is {tuple(lbm.dims)}")
            code |= (mask.astype(bool).astype(np.uint8) << bit).astype(np.uint8)
        self.t_regions = torch.zeros(lbm.pitch, dtype=torch.uint8, device=lbm.device)
        ref_to_lattice(code, lbm.dims, 0, self.t_regions)
        size = ctypes.sizeof(FsiCampaignSums)
        self.t_out = torch.zeros((size + 255) // 256 * 256, dtype=torch.uint8, device=lbm.device)

    def __call__(self) -> dict[str, Any]:
        lbm = self.lbm
        call("fsi_campaign_sums", ctypes.byref(lbm.state), ctypes.byref(lbm.params), ctypes.byref(lbm._ctl()),
             ptr(self.t_regions), ptr(self.t_out), stream_handle())
        size = ctypes.sizeof(FsiCampaignSums)
        st = FsiCampaignSums.from_buffer_copy(self.t_out[:size].cpu().numpy().tobytes())
        return {
            "fluid_mass": float(st.fluid_mass),
            "flux": {name: float(st.region_flux[bit]) for bit, name in enumerate(self.names)},
            "fluid_cells": int(st.fluid_cells),
            "rho_finite": st.nonfinite_rho == 0,
            "velocity_finite": st.nonfinite_vel == 0,
            "population_finite": st.nonfinite_pop == 0,
        }


def campaign_sums_from_fields(fields: dict[str, np.ndarray], regions: dict[str, np.ndarray], device="cuda"
                              ) -> dict[str, Any]:
    """The sums of CampaignReductions from host copies in the reference's
    layouts (_copy_lbm_fields, solver.py:352-365: rho (nx, ny, nz), velocity
    (nx, ny, nz, 3), population (nx, ny, nz, 19), solid (nx, ny, nz)), held
    on the device in lattice order (fsi_campaign_sums_arrays)."""
    rho = np.asarray(fields["rho"], np.float32)
    nx, ny, nz = rho.shape
    if len(regions) > FSI_CAMPAIGN_REGIONS:
        raise ValueError(f"at most {FSI_CAMPAIGN_REGIONS} flux regions")
    names = list(regions)
    code = np.zeros((nx, ny, nz), np.uint8)
    for bit, name in enumerate(names):
        code |= (np.asarray(regions[name]).astype(bool).astype(np.uint8) << bit).astype(np.uint8)

    def dev(a, comps=False):
        a = np.asarray(a)
        a = a.transpose(3, 2, 1, 0) if comps else a.transpose(2, 1, 0)
        return torch.from_numpy(np.ascontiguousarray(a)).to(device)

    t_rho = dev(rho)
    t_vel = dev(np.asarray(fields["velocity"], np.float32), True)
    pop = fields.get("population")
    t_pop = dev(np.asarray(pop, np.float32), True) if pop is not None else None
    t_solid = dev((np.asarray(fields["solid"]) != 0).astype(np.uint8))
    t_reg = dev(code)
    size = ctypes.sizeof(FsiCampaignSums)
    t_out = torch.zeros((size + 255) // 256 * 256, dtype=torch.uint8, device=device)
    call("fsi_campaign_sums_arrays", nx, ny, nz, ptr(t_rho), ptr(t_vel), ptr(t_pop), ptr(t_solid), ptr(t_reg),
         ptr(t_out), stream_handle())
    st = FsiCampaignSums.from_buffer_copy(t_out[:size].cpu().numpy().tobytes())
    return {"fluid_mass": float(st.fluid_mass),
            "flux": {name: float(st.region_flux[bit]) for bit, name in enumerate(names)},
            "fluid_cells": int(st.fluid_cells), "rho_finite": st.nonfinite_rho == 0,
            "velocity_finite": st.nonfinite_vel == 0, "population_finite": st.nonfinite_pop == 0}


def _assert_finite_row(row: dict[str, Any]) -> None:
    """solver.py:830-835."""
    for key, value in row.items():
        if isinstance(value, (bool, str)):
            continue
        if isinstance(value, (int, float)) and not math.isfinite(float(value)):
            raise ValueError(f"nonfinite row value {key}={value}")


def stability_row(base: dict[str, Any], diagnostics: dict[str, Any], sums: dict[str, Any]) -> dict[str, Any]:
    """_stability_row (solver.py:465-500) from the device sums."""
    rho_finite, velocity_finite, population_finite = (bool(sums["rho_finite"]), bool(sums["velocity_finite"]),
                                                      bool(sums["population_finite"]))
    density_gate = bool(rho_finite and float(diagnostics["rho_min"]) > 0.0 and float(diagnostics["rho_max"]) < 5.0)
    mpm_j_gate = bool(math.isfinite(float(diagnostics["mpm_min_J"])) and float(diagnostics["mpm_min_J"]) > 0.0)
    row = {
        **base,
        "step": int(base["official_step"]),
        "rho_min": float(diagnostics["rho_min"]),
        "rho_max": float(diagnostics["rho_max"]),
        "rho_finite": rho_finite,
        "velocity_finite": velocity_finite,
        "population_finite": population_finite,
        "lbm_max_v": float(diagnostics["lbm_max_v"]),
        "mpm_min_J": float(diagnostics["mpm_min_J"]),
        "mpm_max_speed": float(diagnostics["mpm_max_speed"]),
        "density_gate_pass_step": density_gate,
        "mpm_j_gate_pass_step": mpm_j_gate,
        "finite_gate_pass_step": bool(rho_finite and velocity_finite and population_finite),
    }
    _assert_finite_row({k: v for k, v in row.items() if not isinstance(v, bool)})
    return row


def mass_flux_row(base: dict[str, Any], sums: dict[str, Any], initial_mass: float | None
                  ) -> tuple[dict[str, Any], float]:
    """_mass_flux_row (solver.py:503-540) from the device sums (regions named
    inlet, outlet and midplane, as campaign_regions builds them)."""
    total_mass = float(sums["fluid_mass"])
    if initial_mass is None:
        initial_mass = total_mass
    inlet_flux, outlet_flux, midplane_flux = (float(sums["flux"][k]) for k in ("inlet", "outlet", "midplane"))
    denom = max(abs(inlet_flux), 1.0e-30)
    row = {
        "official_step": int(base["official_step"]),
        "time_s": float(base["time_s"]),
        "total_lbm_substeps": int(base["total_lbm_substeps"]),
        "total_fluid_mass": total_mass,
        "mass_delta_rel": (total_mass - initial_mass) / max(abs(initial_mass), 1.0e-30),
        "inlet_flux": inlet_flux,
        "outlet_flux": outlet_flux,
        "midplane_flux": midplane_flux,
        "flux_imbalance_rel": (outlet_flux - inlet_flux) / denom,
        "outlet_to_inlet_flux_ratio": outlet_flux / denom,
        "midplane_to_inlet_flux_ratio": midplane_flux / denom,
    }
    _assert_finite_row(row)
    return row, initial_mass


def copy_lbm_fields(driver) -> dict[str, np.ndarray]:
    """_copy_lbm_fields (solver.py:352-365): the host copies a velocity
    snapshot needs."""
    velocity = np.asarray(driver.lbm.v.to_numpy(), dtype=np.float32)
    return {
        "velocity": velocity,
        "rho": np.asarray(driver.lbm.rho.to_numpy(), dtype=np.float32),
        "solid": np.asarray(driver.lbm.solid.to_numpy(), dtype=np.int8),
        "population": np.asarray(driver.lbm.f.to_numpy(), dtype=np.float32),
        "speed": np.linalg.norm(velocity, axis=3).astype(np.float32),
    }
