"""Autotuner for the launch variants of the step kernels.

The variants differ in how a kernel maps onto the SMs: the register budget of
the one-cell LBM step kernel (3 or 4 resident CTAs per SM), with or without an
L2 prefetch of the tile one resident wave ahead (bit-identical results), and
the two-cells-per-thread LBM kernel on the paired FP32 pipe (the
same operator; its contraction of multiply-adds differs, so results agree to
FP32 rounding).  The tuner times each variant with CUDA events
on the caller's own state -- trial steps on a device snapshot that is
restored afterwards -- and keeps the fastest.  It runs before a CUDA graph of
the step is captured (a captured graph keeps the variant it was built with).
"""

from __future__ import annotations

import torch

from ._lib import FSI_TUNE_LBM_OCC3, FSI_TUNE_LBM_OCC3_PF, FSI_TUNE_LBM_OCC4, FSI_TUNE_LBM_OCC4_PF, FSI_TUNE_LBM_PAIR


def _time_ms(fn, steps, reps):
    """Device time per call of fn: `steps` calls captured in a CUDA graph (so
    that host launch overhead does not enter), replayed `reps` times between
    events; the best replay counts.  steps must return the state's alternating
    layouts (AA parity, ping-pong slots) to their start, i.e. be
    even."""
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(steps):
            fn()
    graph.replay()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        graph.replay()
        e1.record(stream)
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / steps)
    del graph
    return best


def lbm_candidates(lbm):
    """Launch variants valid for this lattice: the paired kernel needs an even
    nx, and nx % 64 != 2 with open boundaries."""
    out = [FSI_TUNE_LBM_OCC3, FSI_TUNE_LBM_OCC4, FSI_TUNE_LBM_OCC3_PF, FSI_TUNE_LBM_OCC4_PF]
    if lbm.nx % 2 == 0 and not ((lbm.bc_x_left or lbm.bc_x_right) and lbm.nx % 64 == 2):
        out.append(FSI_TUNE_LBM_PAIR)
    return out


def tune_lbm(lbm, step_fn, candidates=None, steps=10, reps=3):
    """Pick lbm.tune among candidates by timing `step_fn` (one LBM substep of
    the caller's kind) on a snapshot of the state.  Returns
    {"choice": tune, "ms_per_substep": {tune: ms}}."""
    if candidates is None:
        candidates = lbm_candidates(lbm)
    snap = lbm.snapshot()
    times = {}
    try:
        for t in candidates:
            lbm.tune = int(t)
            for _ in range(2):  # warm-up (parity returns to its start value)
                step_fn()
            torch.cuda.synchronize()
            times[int(t)] = _time_ms(step_fn, steps if steps % 2 == 0 else steps + 1, reps)
            lbm.restore(snap)
    finally:
        lbm.restore(snap)
    best = min(times, key=times.get)
    lbm.tune = best
    lbm._sync_params()
    return {"choice": best, "ms_per_substep": times}


def tune_batch(make_drivers, capacity=None, storage="fp32", mpm_substeps=10, device="cuda", steps=4, reps=2):
    """Launch variants of the batched form (FSIBatch): the LBM step kernel
    (one cell per thread, or two on the paired FP32 pipe when every case has
    an even nx) and the CTA count per case of the batched MPM substeps (the
    default of about one per chunk of the largest case, half and twice that).
    make_drivers() builds the cases' initialised drivers; they run in a
    throwaway batch (their state advances and is discarded), each variant as
    a CUDA graph of one batched FSI step replayed `steps` times between
    events, the best of `reps`.  Returns {"lbm_tune", "mpm_ctas",
    "ms_per_step": {(lbm_tune, mpm_ctas): ms}}."""
    from .batch import FSIBatch

    drivers = make_drivers()
    cap = capacity or len(drivers)
    batch = FSIBatch(capacity=cap, storage=storage, mpm_substeps=mpm_substeps, device=device)
    for drv in drivers:
        batch.add(drv)
    lbm_opts = [FSI_TUNE_LBM_OCC3]
    if all(d.lbm.nx % 2 == 0 for d in drivers):
        lbm_opts.append(FSI_TUNE_LBM_PAIR)
    chunks = max(1, int(batch.dims.max_chunks))
    default = min(chunks, 2 * ((int(batch.dims.max_particles) + 127) // 128) + 8)
    mpm_opts = [0] + sorted({max(1, default // 2), min(65535, default * 2)} - {default})
    times = {}
    stream = torch.cuda.current_stream()
    for lt in lbm_opts:
        for mc in mpm_opts:
            batch.lbm_tune, batch.mpm_ctas = lt, mc
            batch._update_dims()
            batch.invalidate_graph()
            batch.step(use_graph=True)  # capture and warm
            torch.cuda.synchronize()
            best = float("inf")
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(steps):
                    batch.step(use_graph=True)
                e1.record(stream)
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1) / steps)
            times[(lt, mc)] = best
    batch.invalidate_graph()
    choice = min(times, key=times.get)
    del batch, drivers
    return {"lbm_tune": int(choice[0]), "mpm_ctas": int(choice[1]),
            "ms_per_step": {f"{k[0]}/{k[1]}": v for k, v in times.items()}}
