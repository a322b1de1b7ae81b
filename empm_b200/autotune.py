"""Launch-option autotuner for the batched engine and the single-instance solver.

Every launch option of the library gives the same results up to FP32
reduction order (the GPU parity tests check each one against the others and
the FP64 oracle), so it can be picked by speed alone. The tuner times a few
substeps of the caller's own workload under each candidate:

* ``sort_every``: the period of the cell sort (8, 16, 32 substeps);
* ``p2g_mode`` / ``tile_cap`` / ``seg_cap``: warp-aggregated reductions into
  the grid over same-cell runs of at most 4 or 8 lanes, or accumulation in a
  per-CTA shared-memory node tile of 512 / 1024 / 2048 nodes (the tile shape);
* ``g2p_tile``: G2P gathering directly from L2 or from a staged tile;
* ``fuse``: the G2P of each substep and the stress + P2G of the next as one
  kernel between cell sorts, or separate kernels.

It restores the state after every trial, keeps the fastest candidate and
applies it. Results are cached in memory (and, when ``path`` is given, in a
JSON file) per workload signature: the sorted instance grid resolutions, the
particle count rounded to a power of two, and the materials.
"""
from __future__ import annotations

import itertools
import json
import math
import os
from typing import Dict, List, Optional, Sequence

CANDIDATES: List[Dict[str, int]] = [
    dict(sort_every=s, p2g_mode=m, tile_cap=c, seg_cap=k, g2p_tile=g, fuse=f)
    for s, (m, c, k), g, f in itertools.product(
        (8, 16, 32), ((2, 1024, 4), (2, 1024, 8), (1, 512, 4), (1, 1024, 4), (1, 2048, 4)), (0, 1), (1, 0))
    if f == 1 or (m == 2 and g == 0)   # fusing applies to warp-aggregated P2G with direct G2P only
]
OPTION_NAMES = ("sort_every", "p2g_mode", "tile_cap", "seg_cap", "g2p_tile", "fuse")
DEFAULTS = dict(sort_every=32, p2g_mode=2, tile_cap=1024, seg_cap=4, g2p_tile=0, fuse=1)

_MEMORY: Dict[str, Dict] = {}


def signature(grids: Sequence[int], n_particles: int, materials: Sequence[str]) -> str:
    """Cache key of a workload: sorted grid resolutions, log2 particle bucket, materials."""
    bucket = int(round(math.log2(max(int(n_particles), 1))))
    return f"G{'-'.join(str(int(g)) for g in sorted(grids))}|n2^{bucket}|{'-'.join(sorted(set(materials)))}"


def _load(path: Optional[str]) -> Dict[str, Dict]:
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def _store(path: Optional[str], key: str, entry: Dict) -> None:
    if not path:
        return
    data = _load(path)
    data[key] = entry
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def lookup(key: str, path: Optional[str] = None) -> Optional[Dict]:
    if key in _MEMORY:
        return _MEMORY[key]
    entry = _load(path).get(key)
    if entry is not None:
        _MEMORY[key] = entry
    return entry


def _snapshot_colliders(solvers) -> List:
    """Host-side collider parameters, which building a schedule advances
    (the modify callbacks of kinematic colliders)."""
    return [(p, dict(p.__dict__)) for sv in solvers for p in getattr(sv, "collider_params", [])]


def _restore_colliders(snap) -> None:
    for p, d in snap:
        p.__dict__.clear()
        p.__dict__.update(d)


def _apply(target, opts: Dict[str, int]) -> None:
    for k in OPTION_NAMES:
        v = opts.get(k, DEFAULTS[k])
        setattr(target, k, bool(v) if k in ("g2p_tile", "fuse") else int(v))


def tune_batch(batch, dt: float, substeps: int = 32, candidates: Optional[List[Dict[str, int]]] = None,
               path: Optional[str] = None, force: bool = False) -> Dict:
    """Pick the fastest launch options for a BatchedMPM on its current state.

    Returns {"key", "options", "ms": {candidate: ms per substep}, "cached"}.
    The batch's particle state, material state and time are restored."""
    import torch

    key = signature([s.n_grid for s in batch.specs], batch.n, [s.material for s in batch.specs])
    if not force:
        hit = lookup(key, path)
        if hit is not None:
            _apply(batch, hit["options"])
            return dict(hit, cached=True)
    cands = candidates or CANDIDATES
    b0 = batch.cur
    saved = dict(x4=batch._x4[b0].clone(), v4=batch._v4[b0].clone(), C=batch._C[b0].clone(), F=batch._F[b0].clone(),
                 mu=batch.mu.clone(), lam=batch.lam.clone(), ys=batch.yield_stress.clone(), time=batch.time,
                 use_graph=batch.use_graph, opts={k: getattr(batch, k) for k in OPTION_NAMES},
                 colliders=_snapshot_colliders(batch.solvers))

    def restore():
        _restore_colliders(saved["colliders"])
        batch.cur = b0
        batch._x4[b0].copy_(saved["x4"])
        batch._v4[b0].copy_(saved["v4"])
        batch._C[b0].copy_(saved["C"])
        batch._F[b0].copy_(saved["F"])
        batch.mu.copy_(saved["mu"])
        batch.lam.copy_(saved["lam"])
        batch.yield_stress.copy_(saved["ys"])
        batch.time = saved["time"]

    times = {}
    batch.use_graph = True
    for cand in cands:
        _apply(batch, cand)
        restore()
        batch.rollout(dt, substeps, block=substeps)        # captures this candidate's graph
        restore()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.rollout(dt, substeps, block=substeps)
        e1.record()
        torch.cuda.synchronize()
        times[json.dumps(cand, sort_keys=True)] = e0.elapsed_time(e1) / substeps
    restore()
    batch.use_graph = saved["use_graph"]
    best = json.loads(min(times, key=times.get))
    _apply(batch, best)
    entry = {"key": key, "options": best, "ms": times}
    _MEMORY[key] = entry
    _store(path, key, entry)
    return dict(entry, cached=False)


def tune_solver(solver, model, state, dt: float, substeps: int = 32,
                candidates: Optional[List[Dict[str, int]]] = None, path: Optional[str] = None,
                force: bool = False) -> Dict:
    """The same for a single-instance MPMWARPDiff rollout from `state`
    (state, material scalars and solver time are restored)."""
    import torch

    from .mpm_solver_diff import MATERIALS

    mat_name = {v: k for k, v in MATERIALS.items()}.get(int(model.material), str(model.material))
    key = signature([int(model.n_grid)], state.n_particles, [mat_name])
    if not force:
        hit = lookup(key, path)
        if hit is not None:
            _apply(solver, hit["options"])
            return dict(hit, cached=True)
    cands = candidates or CANDIDATES
    saved = [t.clone() for t in (state._x4, state._v4, state._C, state._F_trial, model.mu, model.lam,
                                 model.yield_stress)]
    t0 = solver.time
    colliders = _snapshot_colliders([solver])
    other = state.partial_clone(requires_grad=False)
    schedule = solver.build_schedule(t0, dt, substeps)

    def restore():
        _restore_colliders(colliders)
        for dst, src in zip((state._x4, state._v4, state._C, state._F_trial, model.mu, model.lam,
                             model.yield_stress), saved):
            dst.copy_(src)
        solver.time = t0

    times = {}
    for cand in cands:
        _apply(solver, cand)
        restore()
        solver.rollout(model, state, other, dt, substeps, schedule=schedule)
        restore()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        solver.rollout(model, state, other, dt, substeps, schedule=schedule)
        e1.record()
        torch.cuda.synchronize()
        times[json.dumps(cand, sort_keys=True)] = e0.elapsed_time(e1) / substeps
    restore()
    best = json.loads(min(times, key=times.get))
    _apply(solver, best)
    entry = {"key": key, "options": best, "ms": times}
    _MEMORY[key] = entry
    _store(path, key, entry)
    return dict(entry, cached=False)
