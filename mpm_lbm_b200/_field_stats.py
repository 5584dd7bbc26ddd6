"""Per-x-plane statistics of the lattice fields, computed on the device in
one pass (fsi_lbm_field_stats / fsi_field_stats_arrays) for the diagnostics
modules lbm_boundary_diagnostics and lbm_stability_diagnostics.

The reference's diagnostics (src/mpm_lbm/sim/diagnostics/*.py) copy rho, v,
solid, f and F to the host and reduce them with numpy in FP64.  Here the
device reduces them into one FsiPlaneStats record per x plane (FP64 sums,
exact FP32 extrema, counts, first outlier per plane) and only those ~160
bytes per plane cross to the host.  A snapshot dict (the reference's
``snapshot_from_lbm`` form) is uploaded and reduced by the same kernel.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import FsiFieldStatsArgs, FsiPlaneStats, call, ptr, stream_handle

KEY_NONE_MIN = 0xFFFFFFFF


def _plane_dtype() -> np.dtype:
    fields = {}
    for name, ctype in FsiPlaneStats._fields_:
        off = getattr(FsiPlaneStats, name).offset
        if issubclass(ctype, ctypes.Array):
            base = np.dtype(ctype._type_)
            fields[name] = ((base, (ctype._length_,)), off)
        else:
            fields[name] = (np.dtype(ctype), off)
    return np.dtype({"names": list(fields), "formats": [f[0] for f in fields.values()],
                     "offsets": [f[1] for f in fields.values()], "itemsize": ctypes.sizeof(FsiPlaneStats)})


PLANE_DTYPE = _plane_dtype()


def decode_keys(keys) -> np.ndarray:
    """FP32 values of order-preserving uint32 keys."""
    k = np.asarray(keys, dtype=np.uint32)
    bits = np.where(k & np.uint32(0x80000000), k & np.uint32(0x7FFFFFFF), ~k).astype(np.uint32)
    return bits.view(np.float32).astype(np.float64)


@dataclass
class PlaneTable:
    """The per-plane records of one pass, as numpy arrays over x."""

    rec: np.ndarray  # PLANE_DTYPE, shape (nx,)
    shape: tuple

    @property
    def nx(self) -> int:
        return self.shape[0]

    def __getitem__(self, name):
        return self.rec[name]

    def key_min(self, name, sel=slice(None)) -> float:
        """Smallest value over the selected planes (nan if none)."""
        k = np.asarray(self.rec[name][sel]).reshape(-1)
        k = k[k != np.uint32(KEY_NONE_MIN)]
        return float(decode_keys(k.min())) if k.size else float("nan")

    def key_max(self, name, sel=slice(None)) -> float:
        k = np.asarray(self.rec[name][sel]).reshape(-1)
        k = k[k != 0]
        return float(decode_keys(k.max())) if k.size else float("nan")

    def speed_max(self, sel=slice(None)) -> float:
        bits = np.asarray(self.rec["speed_max"][sel], dtype=np.uint64).reshape(-1)
        return float(bits.max().view(np.float64)) if bits.size else 0.0


def _is_lbm(obj) -> bool:
    return hasattr(obj, "state") and hasattr(obj, "params") and hasattr(obj, "t_pop")


def field_stats(lbm_or_snapshot, rho_low=0.0, rho_high=1.2, vel_high=0.2, cy=None, cz=None) -> PlaneTable:
    """One device pass over an LBMFluid3D (its readout state) or over a
    snapshot dict with rho (nx, ny, nz), v (nx, ny, nz, 3), solid and
    optionally f, F (nx, ny, nz, 19); cy, cz default to ny // 2, nz // 2."""
    if _is_lbm(lbm_or_snapshot):
        lbm = lbm_or_snapshot
        nx, ny, nz = lbm.dims
        device = lbm.device
    elif isinstance(lbm_or_snapshot, dict):
        nx, ny, nz = np.asarray(lbm_or_snapshot["rho"]).shape
        device = torch.device("cuda")
    else:
        raise TypeError("expected an LBMFluid3D or a snapshot dict with rho, v and solid")
    cy = ny // 2 if cy is None else int(cy)
    cz = nz // 2 if cz is None else int(cz)
    args = FsiFieldStatsArgs(rho_low=float(rho_low), rho_high=float(rho_high), vel_high=float(vel_high), cy=cy,
                             cz=cz)
    out = torch.empty(nx * ctypes.sizeof(FsiPlaneStats), dtype=torch.uint8, device=device)
    if _is_lbm(lbm_or_snapshot):
        call("fsi_lbm_field_stats", ctypes.byref(lbm.state), ctypes.byref(lbm.params), ctypes.byref(lbm._ctl()),
             ctypes.byref(args), ptr(out), stream_handle())
    else:
        snap = lbm_or_snapshot

        def lattice(a, comps):
            t = torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float32))).to(device)
            if comps:
                return t.permute(3, 2, 1, 0).contiguous()
            return t.permute(2, 1, 0).contiguous()

        keep = [lattice(snap["rho"], 0), lattice(snap["v"], 3),
                torch.from_numpy((np.asarray(snap["solid"]) != 0).astype(np.uint8)).to(device).permute(2, 1, 0)
                .contiguous()]
        args.rho, args.vel, args.solid = ptr(keep[0]), ptr(keep[1]), ptr(keep[2])
        for key, attr in (("f", "pop_f"), ("F", "pop_F")):
            if key in snap:
                keep.append(lattice(snap[key], 19))
                setattr(args, attr, ptr(keep[-1]))
        call("fsi_field_stats_arrays", nx, ny, nz, ctypes.byref(args), ptr(out), stream_handle())
    rec = np.frombuffer(out.cpu().numpy().tobytes(), dtype=PLANE_DTYPE).copy()
    return PlaneTable(rec=rec, shape=(nx, ny, nz))
