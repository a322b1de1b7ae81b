"""Request loop: rollout and gradient requests of mixed sizes on one GPU.

EMPM has no server. Its online loop (``interactive_playground``,
trainer_warp_mpm.py:1309, and ``scripts/interactive_viser.py:216-292``) calls
``advance_to`` for one simulation at a time. This module serves many
independent simulations at once, with continuous batching:

* Every admitted request keeps its particle state resident on the device, in
  one arena shared by all requests in their forward phase. Instance i occupies
  particles ``[poff_i, poff_i + n_i)``.
* Work proceeds in blocks of ``block`` substeps (fewer when every active
  request finishes sooner). Each block is one batched launch sequence
  (``empm_rollout`` on a batch context) over every active request, each
  request on its own grid, dt and boundary conditions. A request that
  finishes inside a block is held for the rest of it (the step tables'
  ``hold`` flag: no P2G contribution, state copied through).
* At block boundaries, finished requests leave and waiting requests are
  admitted as instance slots, arena particles, grid blocks and HBM budget
  free up. The arena is then re-laid out: surviving state is gathered to the
  new offsets, and the context is reconfigured without allocating
  (``empm_batch_reconfigure``).
* At every block boundary a gradient request's state, mu, lam and yield are
  copied to its own checkpoint storage, so its adjoint segments are the
  blocks it took part in (at most ``block`` substeps each).
* A gradient request whose forward is done moves to the adjoint engine. That
  engine runs ``empm_adjoint_segment`` over the request's checkpoints on a
  second CUDA stream, so its work overlaps the forward blocks of the others.

The loss of a gradient request is mean |x_T - target|^2 over its particles.
Its result holds dL/dv0 per particle and dL/dE, dL/dnu and dL/dyield (sums
over particles), computed as in the differentiable rollout.

``Scheduler`` is the host-side policy: admission against capacities and the
byte model, block length, cancellation and deadlines. It runs without a GPU.
``GpuExecutor`` carries a plan out on the device; ``MPMServer`` joins the two
in a background thread. A request that is in its adjoint phase cannot be
cancelled; its deadline applies to the waiting and forward phases.
"""
from __future__ import annotations

import ctypes
import itertools
import math
import threading
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, Deque, Dict, List, Optional

import numpy as np

from .batch import InstanceSpec, _params, register_colliders

# bytes per particle held by the forward arena (two arenas x two ping-pong
# states of x4, v4, C, F at 104 B, elastic F 36 B, vol/mu/lam/yield/density/E/nu
# 28 B) and by the sorted-path buffers of the batch context (2 x 104 B states,
# 36 B elastic F, 2 x (16 + 8) B material/index arrays, keys and ranks 8 B)
ARENA_BYTES_PER_PARTICLE = 4 * 104 + 36 + 28
SORTED_BYTES_PER_PARTICLE = 2 * 104 + 36 + 48 + 8
STATE_BYTES_PER_PARTICLE = 104 + 12          # one checkpoint: state + mu, lam, yield
GRID_BYTES_PER_BLOCK = 2 * 64 * 16 + 1       # momentum + velocity + flag of one 4^3 block


def grid_blocks(n_grid: int) -> int:
    nb = (int(n_grid) + 3) // 4
    return nb * nb * nb


@dataclass
class Request:
    """A rollout (grad=False) or rollout + gradient (grad=True) request."""
    spec: InstanceSpec               # initial state, material and colliders
    n_substeps: int
    dt: float
    grad: bool = False
    target: Optional[np.ndarray] = None   # [N, 3] target positions of the gradient loss
    deadline_s: Optional[float] = None    # relative to submission; None = no deadline

    def validate(self) -> None:
        s = self.spec
        n = s.n
        if n < 1:
            raise ValueError("a request needs at least one particle")
        if s.x.shape != (n, 3):
            raise ValueError(f"x must be [N, 3], got {tuple(s.x.shape)}")
        for name in ("vol", "rho", "E", "nu"):
            a = np.asarray(getattr(s, name))
            if a.shape != (n,):
                raise ValueError(f"{name} must be [N], got {tuple(a.shape)}")
        if s.v is not None and np.asarray(s.v).shape != (n, 3):
            raise ValueError("v must be [N, 3]")
        if not (4 <= int(s.n_grid) <= 1024):
            raise ValueError(f"n_grid {s.n_grid} out of [4, 1024]")
        if int(self.n_substeps) < 1:
            raise ValueError("n_substeps must be >= 1")
        if not (self.dt > 0.0 and math.isfinite(self.dt)):
            raise ValueError("dt must be positive")
        x = np.asarray(s.x)
        if not np.isfinite(x).all() or (x <= 0.0).any() or (x >= s.grid_lim).any():
            raise ValueError("particles must lie strictly inside the domain")
        if self.grad:
            if self.target is None or np.asarray(self.target).shape != (n, 3):
                raise ValueError("a gradient request needs target positions [N, 3]")


@dataclass
class Result:
    status: str                       # "ok", "rejected", "cancelled", "timeout", "error"
    x: Optional[np.ndarray] = None    # final positions [N, 3]
    v: Optional[np.ndarray] = None    # final velocities [N, 3]
    loss: Optional[float] = None
    grads: Optional[Dict[str, np.ndarray]] = None
    error: Optional[str] = None
    submitted: float = 0.0            # host monotonic clock, seconds
    admitted: Optional[float] = None
    finished: Optional[float] = None

    @property
    def latency_s(self) -> Optional[float]:
        return None if self.finished is None else self.finished - self.submitted


class Ticket:
    """Handle of a submitted request."""

    _ids = itertools.count()

    def __init__(self, req: Request, now: float):
        self.id = next(Ticket._ids)
        self.req = req
        self.submitted = now
        self.result: Optional[Result] = None
        self._done = threading.Event()
        self.cancel_requested = False
        # scheduler state
        self.progress = 0                 # forward substeps done
        self.phase = "pending"            # pending -> forward -> (backward) -> done
        self.admitted: Optional[float] = None
        self.ckpt_bytes = 0

    @property
    def n(self) -> int:
        return self.req.spec.n

    @property
    def blocks(self) -> int:
        return grid_blocks(self.req.spec.n_grid)

    def cancel(self) -> None:
        self.cancel_requested = True

    def done(self) -> bool:
        return self._done.is_set()

    def wait(self, timeout: Optional[float] = None) -> Optional[Result]:
        self._done.wait(timeout)
        return self.result

    def _finish(self, result: Result) -> None:
        result.submitted = self.submitted
        result.admitted = self.admitted
        if result.finished is None:
            result.finished = time.monotonic()
        self.result = result
        self.phase = "done"
        self._done.set()


def checkpoint_bytes(req: Request, block: int) -> int:
    """Device bytes a gradient request holds outside the arena: one
    checkpoint per block boundary it passes (at most T // block + 1, since
    only its last block can be short), the initial state and its final
    state."""
    if not req.grad:
        return 0
    n_ckpt = req.n_substeps // block + 3
    return n_ckpt * req.spec.n * STATE_BYTES_PER_PARTICLE


@dataclass
class Capacity:
    particles: int          # arena particles
    blocks: int             # grid blocks of the batch context
    instances: int          # instance slots
    ckpt_bytes: int         # checkpoint pool
    adjoint_particles: int  # largest gradient request the adjoint engine takes
    adjoint_blocks: int


def capacity_for_budget(hbm_budget: int, max_instances: int = 64, grid_share: float = 0.25,
                        ckpt_share: float = 0.35, adjoint_particles: int = 1_000_000,
                        adjoint_grid: int = 160, every: int = 50) -> Capacity:
    """Split an HBM budget (bytes) between the forward arena, the grids, the
    checkpoint pool and the adjoint engine (segment states of up to `every`
    substeps, its own grids and sorted buffers, and the per-substep store of
    touched grid blocks and elastic F that its reverse pass reads)."""
    adj_blocks = grid_blocks(adjoint_grid)
    adjoint = adjoint_particles * ((every + 1) * 104 + every * 12 + 2 * 104 + 3 * 36 + 64 +
                                   SORTED_BYTES_PER_PARTICLE) + adj_blocks * 4 * 64 * 16
    adjoint += every * (adj_blocks * (128 * 16 + 4) + adjoint_particles * 36)
    rest = hbm_budget - adjoint
    if rest <= 0:
        raise ValueError("HBM budget too small for the adjoint engine")
    grid = int(rest * grid_share)
    ckpt = int(rest * ckpt_share)
    arena = rest - grid - ckpt
    return Capacity(particles=int(arena // (ARENA_BYTES_PER_PARTICLE + SORTED_BYTES_PER_PARTICLE)),
                    blocks=int(grid // GRID_BYTES_PER_BLOCK), instances=max_instances, ckpt_bytes=ckpt,
                    adjoint_particles=adjoint_particles, adjoint_blocks=adj_blocks)


@dataclass
class Plan:
    rejected: List[Ticket] = field(default_factory=list)
    cancelled: List[Ticket] = field(default_factory=list)     # removed from pending / forward
    admitted: List[Ticket] = field(default_factory=list)
    active: List[Ticket] = field(default_factory=list)        # forward set of the next block, in arena order
    relayout: bool = False
    block: int = 0                                            # substeps of the next block (0 = idle)


class Scheduler:
    """Admission and block planning (host only)."""

    def __init__(self, cap: Capacity, block: int = 50):
        self.cap = cap
        self.block = int(block)
        self.pending: Deque[Ticket] = deque()
        self.forward: List[Ticket] = []
        self.backward: List[Ticket] = []      # gradient requests in (or waiting for) the adjoint engine
        self.ckpt_in_use = 0

    def fits_at_all(self, t: Ticket) -> Optional[str]:
        c = self.cap
        if t.n > c.particles:
            return f"{t.n} particles exceed the arena capacity of {c.particles}"
        if t.blocks > c.blocks:
            return f"grid {t.req.spec.n_grid}^3 exceeds the grid capacity"
        if t.req.grad:
            if checkpoint_bytes(t.req, self.block) > c.ckpt_bytes:
                return "checkpoints exceed the HBM budget"
            if t.n > c.adjoint_particles or t.blocks > c.adjoint_blocks:
                return "request exceeds the adjoint engine's capacity"
        return None

    def submit(self, t: Ticket) -> Optional[str]:
        why = self.fits_at_all(t)
        if why is None:
            self.pending.append(t)
        return why

    def release_backward(self, t: Ticket) -> None:
        if t in self.backward:
            self.backward.remove(t)
        self.ckpt_in_use -= t.ckpt_bytes
        t.ckpt_bytes = 0

    def block_length(self, active: List[Ticket]) -> int:
        """Substeps of the next block: `block`, or fewer when every active
        request finishes sooner. Requests that finish inside it are held."""
        return max(1, min(self.block, max(t.req.n_substeps - t.progress for t in active)))

    def plan(self, now: float) -> Plan:
        p = Plan()
        prev_ids = [t.id for t in self.forward]
        # cancellations and deadlines
        for q in (self.pending, self.forward):
            for t in list(q):
                expired = t.req.deadline_s is not None and now - t.submitted > t.req.deadline_s
                if t.cancel_requested or expired:
                    q.remove(t)
                    t.phase = "timeout" if expired and not t.cancel_requested else "cancelled"
                    if t.ckpt_bytes:
                        self.ckpt_in_use -= t.ckpt_bytes
                        t.ckpt_bytes = 0
                    p.cancelled.append(t)
        finished = [t for t in self.forward if t.progress >= t.req.n_substeps]
        keep = [t for t in self.forward if t.progress < t.req.n_substeps]
        for t in finished:
            if t.req.grad:
                self.backward.append(t)
        # admission in arrival order, no overtaking
        used_p = sum(t.n for t in keep)
        used_b = sum(t.blocks for t in keep)
        while self.pending:
            t = self.pending[0]
            cb = checkpoint_bytes(t.req, self.block)
            if (len(keep) + 1 > self.cap.instances or used_p + t.n > self.cap.particles or
                    used_b + t.blocks > self.cap.blocks or self.ckpt_in_use + cb > self.cap.ckpt_bytes):
                break
            self.pending.popleft()
            t.phase = "forward"
            t.admitted = now
            t.ckpt_bytes = cb
            self.ckpt_in_use += cb
            keep.append(t)
            p.admitted.append(t)
            used_p += t.n
            used_b += t.blocks
        p.relayout = [t.id for t in keep] != prev_ids
        self.forward = keep
        p.active = list(keep)
        if keep:
            p.block = self.block_length(keep)
        return p

    def advance(self, p: Plan) -> None:
        for t in p.active:
            t.progress = min(t.progress + p.block, t.req.n_substeps)

    def idle(self) -> bool:
        return not self.pending and not self.forward and not self.backward


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
class GpuExecutor:
    """Device state of the server: the batch context and its particle arena,
    the per-request checkpoints and the adjoint engine."""

    def __init__(self, cap: Capacity, device="cuda:0", sort_every: int = 32):
        import torch

        from . import _native as N
        from .mpm_data_structure import DTYPE

        self.torch, self.N, self.DTYPE = torch, N, DTYPE
        self.cap = cap
        self.device = torch.device(device)
        dev = self.device
        self.L = N.lib()
        self.fwd_stream = torch.cuda.Stream(device=dev)
        self.bwd_stream = torch.cuda.Stream(device=dev)
        P = cap.particles
        # two arenas (swapped at each re-layout), each with two ping-pong states
        self.arenas = []
        for _ in range(2):
            a = dict(x4=[torch.zeros((P, 4), dtype=DTYPE, device=dev) for _ in range(2)],
                     v4=[torch.zeros((P, 4), dtype=DTYPE, device=dev) for _ in range(2)],
                     C=[torch.zeros(9 * P, dtype=DTYPE, device=dev) for _ in range(2)],
                     F=[torch.zeros(9 * P, dtype=DTYPE, device=dev) for _ in range(2)])
            self.arenas.append(a)
        self.mat = {k: [torch.zeros(P, dtype=DTYPE, device=dev) for _ in range(2)]
                    for k in ("vol", "mu", "lam", "ys")}
        self.Fe = torch.zeros(9 * P, dtype=DTYPE, device=dev)
        # first plane chunks of an identity F (float4 planes A, B)
        self._id_row = torch.tensor([1.0, 0.0, 0.0, 0.0], dtype=DTYPE, device=dev)
        self.ai = 0        # current arena
        self.cur = 0       # current ping-pong state within it
        self.layout: List[Ticket] = []      # tickets in arena order
        self.offsets: Dict[int, int] = {}
        self.n_total = 0
        # forward batch context, reserved at capacity
        self.ctx = self._make_ctx(cap.particles, cap.blocks, cap.instances, sort_every)
        # adjoint engine: one single-instance context re-laid for each request
        self.actx = self._make_ctx(cap.adjoint_particles, cap.adjoint_blocks, 1, sort_every)
        self.solvers: Dict[int, object] = {}
        self.tables: Dict[int, tuple] = {}
        self.ckpts: Dict[int, List] = {}
        self.pending_results = []   # (ticket, event, fill-callback)

    def _make_ctx(self, particles, blocks, instances, sort_every):
        N = self.N
        p = (N.EmpmModelParams * 1)()
        p[0].n_grid, p[0].grid_lim = 8, 1.0
        counts = (ctypes.c_int * 1)(1)
        ptr = ctypes.c_void_p()
        with self.torch.cuda.device(self.device):
            N.check(self.L.empm_batch_create(p, counts, 1, 64, ctypes.byref(ptr)))
            N.check(self.L.empm_batch_reserve(ptr, int(particles), int(blocks), int(instances)), ptr)
            N.check(self.L.empm_ctx_set_option(ptr, N.OPT_SORT_EVERY, int(sort_every)), ptr)
        return ptr

    def close(self):
        for name in ("ctx", "actx"):
            ptr = getattr(self, name, None)
            if ptr:
                self.L.empm_ctx_destroy(ptr)
                setattr(self, name, None)

    # -- helpers ----------------------------------------------------------------
    @staticmethod
    def _planes(buf, n):
        return buf[: 4 * n].view(n, 4), buf[4 * n: 8 * n].view(n, 4), buf[8 * n: 9 * n]

    @staticmethod
    def _sptr(stream):
        return ctypes.c_void_p(stream.cuda_stream)

    def _solver(self, t: Ticket):
        """Per-request schedule: the collider list and time gates of a
        single-instance MPMWARPDiff. Boundary conditions without time windows
        or host callbacks give one step table for every substep; otherwise
        the whole schedule is built up front."""
        from .mpm_solver_diff import MPMWARPDiff

        s = t.req.spec
        sv = MPMWARPDiff()
        sv.initialize(s.n, n_grid=s.n_grid, grid_lim=s.grid_lim, device=self.device)
        register_colliders(sv, s.colliders)
        static = not any(m is not None for m in sv.modify_bc) and all(
            float(c.start_time) <= 0.0 and float(c.end_time) >= 999.0 for c in sv.collider_params)
        if static:
            table = (self.N.EmpmStep * 1)()
            sv._fill_step(table[0], 0.0, t.req.dt)
        else:
            table, _ = sv.build_schedule(0.0, t.req.dt, t.req.n_substeps)
        self.solvers[t.id] = sv
        self.tables[t.id] = (table, static)

    def _steps(self, t: Ticket, k0: int, k1: int):
        """Step tables of substeps [k0, k1) of request t."""
        N = self.N
        table, static = self.tables[t.id]
        out = (N.EmpmStep * (k1 - k0))()
        sz = ctypes.sizeof(N.EmpmStep)
        for k in range(k0, k1):
            ctypes.memmove(ctypes.addressof(out) + (k - k0) * sz, ctypes.addressof(table) + (0 if static else k) * sz,
                           sz)
        return out

    # -- re-layout ----------------------------------------------------------------
    def relayout(self, active: List[Ticket], admitted: List[Ticket]) -> None:
        torch = self.torch
        new_ids = {t.id for t in admitted}
        old = self.arenas[self.ai]
        new_ai = 1 - self.ai
        new = self.arenas[new_ai]
        n_old = self.n_total
        counts = [t.n for t in active]
        n_new = int(sum(counts))
        offs = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64) if counts else np.zeros(0, np.int64)
        with torch.cuda.stream(self.fwd_stream):
            # surviving instances keep their order: copy them as contiguous runs
            # (survivors that were neighbours stay neighbours), device to device,
            # so that the host never waits for the GPU here
            runs = []   # [src, dst, n]
            for t, o in zip(active, offs):
                if t.id in new_ids:
                    continue
                so = self.offsets[t.id]
                if runs and runs[-1][0] + runs[-1][2] == so and runs[-1][1] + runs[-1][2] == o:
                    runs[-1][2] += t.n
                else:
                    runs.append([so, int(o), t.n])
            c = self.cur
            old_planes = {k: self._planes(old[k][c], n_old) for k in ("C", "F")}
            new_planes = {k: self._planes(new[k][0], n_new) for k in ("C", "F")}
            for so, do, n in runs:
                src, dst = slice(so, so + n), slice(do, do + n)
                new["x4"][0][dst].copy_(old["x4"][c][src])
                new["v4"][0][dst].copy_(old["v4"][c][src])
                for k in ("C", "F"):
                    for po, pn in zip(old_planes[k], new_planes[k]):
                        pn[dst].copy_(po[src])
                for k in ("vol", "mu", "lam", "ys"):
                    self.mat[k][new_ai][dst].copy_(self.mat[k][self.ai][src])
            # admitted instances: initial state from the host
            for t, o in zip(active, offs):
                if t.id in new_ids:
                    self._load(t, int(o), new, new_ai, n_new)
        self.ai, self.cur = new_ai, 0
        self.layout = list(active)
        self.offsets = {t.id: int(o) for t, o in zip(active, offs)}
        self.n_total = n_new
        if active:
            N = self.N
            params = (N.EmpmModelParams * len(active))(*[_params(t.req.spec) for t in active])
            cnt = (ctypes.c_int * len(active))(*counts)
            N.check(self.L.empm_batch_reconfigure(self.ctx, params, cnt, len(active), self._sptr(self.fwd_stream)),
                    self.ctx)

    def _load(self, t: Ticket, o: int, arena, ai: int, n_total: int) -> None:
        torch, N = self.torch, self.N
        s = t.req.spec
        n = s.n
        dev = self.device
        h = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).pin_memory().to(  # noqa: E731
            dev, non_blocking=True)
        sl = slice(o, o + n)
        arena["x4"][0][sl, :3] = h(s.x)
        arena["v4"][0][sl, :3] = h(s.v) if s.v is not None else 0.0
        arena["v4"][0][sl, 3] = 0.0
        A, B, Cc = self._planes(arena["C"][0], n_total)
        A[sl] = 0.0
        B[sl] = 0.0
        Cc[sl] = 0.0
        A, B, Cc = self._planes(arena["F"][0], n_total)
        A[sl] = self._id_row
        B[sl] = self._id_row
        Cc[sl] = 1.0
        vol = self.mat["vol"][ai][sl]
        vol.copy_(h(s.vol))
        ys = self.mat["ys"][ai][sl]
        ys.copy_(h(s.yield_stress) if s.yield_stress is not None else torch.zeros(n, device=dev))
        E, nu, rho = h(s.E), h(s.nu), h(s.rho)
        N.check(self.L.empm_prepare(None, E.data_ptr(), nu.data_ptr(), self.mat["mu"][ai][sl].data_ptr(),
                                    self.mat["lam"][ai][sl].data_ptr(), rho.data_ptr(), vol.data_ptr(),
                                    arena["x4"][0][sl].data_ptr(), n, self._sptr(self.fwd_stream)))
        t._E, t._nu, t._rho = E, nu, rho      # kept alive; E and nu feed the gradient's prepare adjoint
        self._solver(t)
        if t.req.grad:
            self.ckpts[t.id] = []
            self._checkpoint(t, arena, 0, ai, o, n_total)

    def _checkpoint(self, t: Ticket, arena, c: int, ai: int, o: int, n_total: int) -> None:
        """Copy a gradient request's slice of the arena into its own
        single-instance layout (stream-ordered on the forward stream)."""
        torch = self.torch
        n = t.n
        sl = slice(o, o + n)
        with torch.cuda.stream(self.fwd_stream):
            x4 = arena["x4"][c][sl].clone()
            v4 = arena["v4"][c][sl].clone()
            Cb = torch.empty(9 * n, dtype=self.DTYPE, device=self.device)
            Fb = torch.empty(9 * n, dtype=self.DTYPE, device=self.device)
            for src, dst in ((arena["C"][c], Cb), (arena["F"][c], Fb)):
                for ps, pd in zip(self._planes(src, n_total), self._planes(dst, n)):
                    pd.copy_(ps[sl])
            mu = self.mat["mu"][ai][sl].clone()
            lam = self.mat["lam"][ai][sl].clone()
            ys = self.mat["ys"][ai][sl].clone()
        self.ckpts[t.id].append((t.progress, x4, v4, Cb, Fb, mu, lam, ys))

    # -- forward block --------------------------------------------------------------
    def run_block(self, active: List[Ticket], L: int) -> None:
        N = self.N
        n_inst = len(active)
        sz = ctypes.sizeof(N.EmpmStep)
        uniform = all(self.tables[t.id][1] and t.req.n_substeps - t.progress >= L for t in active)
        n_tables = 1 if uniform else L
        table = (N.EmpmStep * (n_tables * n_inst))()
        for i, t in enumerate(active):
            src, static = self.tables[t.id]
            remaining = t.req.n_substeps - t.progress
            for s in range(n_tables):
                e = s * n_inst + i
                k = min(t.progress + s, t.req.n_substeps - 1)
                ctypes.memmove(ctypes.addressof(table) + e * sz, ctypes.addressof(src) + (0 if static else k) * sz, sz)
                if s >= remaining:
                    table[e].hold = 1
        a = self.arenas[self.ai]
        c = self.cur
        views = [N.EmpmParticles(a["x4"][k].data_ptr(), a["v4"][k].data_ptr(), a["C"][k].data_ptr(),
                                 a["F"][k].data_ptr()) for k in (c, 1 - c)]
        mat = N.EmpmMaterial(self.mat["vol"][self.ai].data_ptr(), self.mat["mu"][self.ai].data_ptr(),
                             self.mat["lam"][self.ai].data_ptr(), self.mat["ys"][self.ai].data_ptr(), None,
                             self.Fe.data_ptr())
        N.check(self.L.empm_rollout(self.ctx, views[0], views[1], mat, table, n_tables, L, 0,
                                    self._sptr(self.fwd_stream)), self.ctx)
        if L % 2 == 1:
            self.cur = 1 - c

    def after_block(self, active: List[Ticket]) -> None:
        """Checkpoints of gradient requests at their boundaries (progress
        already advanced)."""
        a = self.arenas[self.ai]
        for t in active:
            if t.req.grad and t.progress < t.req.n_substeps:
                self._checkpoint(t, a, self.cur, self.ai, self.offsets[t.id], self.n_total)

    # -- results ------------------------------------------------------------------------
    def finish_forward(self, t: Ticket) -> None:
        """Final state of a request leaving the arena: the result of a rollout
        request, or the start of a gradient request's adjoint."""
        torch = self.torch
        a = self.arenas[self.ai]
        o, n = self.offsets[t.id], t.n
        sl = slice(o, o + n)
        with torch.cuda.stream(self.fwd_stream):
            if not t.req.grad:
                hx = torch.empty((n, 3), dtype=self.DTYPE, pin_memory=True)
                hv = torch.empty((n, 3), dtype=self.DTYPE, pin_memory=True)
                hx.copy_(a["x4"][self.cur][sl, :3], non_blocking=True)
                hv.copy_(a["v4"][self.cur][sl, :3], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.fwd_stream)
                self.pending_results.append((t, ev, lambda hx=hx, hv=hv: Result("ok", x=hx.numpy(), v=hv.numpy())))
                return
            x_final = a["x4"][self.cur][sl, :3].clone()
            ev = torch.cuda.Event()
            ev.record(self.fwd_stream)
        self._adjoint(t, x_final, ev)

    def _adjoint(self, t: Ticket, x_final, ready_event) -> None:
        torch, N = self.torch, self.N
        from .adjoint import PackedGrad, prepare_adjoint

        n = t.n
        dev = self.device
        s = self.bwd_stream
        s.wait_event(ready_event)
        with torch.cuda.stream(s):
            target = torch.as_tensor(np.ascontiguousarray(t.req.target, dtype=np.float32)).pin_memory().to(
                dev, non_blocking=True)
            diff = x_final - target
            loss = (diff * diff).sum(1).mean()
            grad = PackedGrad(n, dev)
            grad.add(g_x=2.0 * diff / n)
            g_mu = torch.zeros(n, dtype=self.DTYPE, device=dev)
            g_lam, g_ys, g_mass = (torch.zeros_like(g_mu) for _ in range(3))
            gmat = N.EmpmMaterialGrad(g_mu.data_ptr(), g_lam.data_ptr(), g_ys.data_ptr(), g_mass.data_ptr())
            spec = t.req.spec
            vol = torch.as_tensor(np.ascontiguousarray(spec.vol, dtype=np.float32)).pin_memory().to(
                dev, non_blocking=True)
            params = (N.EmpmModelParams * 1)(_params(spec))
            cnt = (ctypes.c_int * 1)(n)
            N.check(self.L.empm_batch_reconfigure(self.actx, params, cnt, 1, self._sptr(s)), self.actx)
            mat = N.EmpmMaterial(vol.data_ptr(), None, None, None, None, None)
            ck = self.ckpts[t.id]
            bounds = [c[0] for c in ck] + [t.req.n_substeps]
            for (k0, x4, v4, Cb, Fb, mu, lam, ys), k1 in reversed(list(zip(ck, bounds[1:]))):
                seg = self._steps(t, k0, k1)
                part = N.EmpmParticles(x4.data_ptr(), v4.data_ptr(), Cb.data_ptr(), Fb.data_ptr())
                N.check(self.L.empm_adjoint_segment(self.actx, part, mu.data_ptr(), lam.data_ptr(), ys.data_ptr(),
                                                    mat, seg, k1 - k0, grad.particles(), gmat, self._sptr(s)),
                        self.actx)
            g_E, g_nu, _ = prepare_adjoint(t._E, t._nu, g_mu, g_lam)
            out = torch.stack([loss, g_E.sum(), g_nu.sum(), g_ys.sum()])
            hs = torch.empty(4, dtype=self.DTYPE, pin_memory=True)
            hgv = torch.empty((n, 3), dtype=self.DTYPE, pin_memory=True)
            hx = torch.empty((n, 3), dtype=self.DTYPE, pin_memory=True)
            hs.copy_(out, non_blocking=True)
            hgv.copy_(grad.v4[:, :3], non_blocking=True)
            hx.copy_(x_final, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
            # tensors written by another stream or read by the adjoint stay
            # referenced until its completion event has been observed
            keep = (grad, g_mu, g_lam, g_ys, g_mass, vol, target, ck, x_final, diff, loss, out, g_E, g_nu)

        def fill(hs=hs, hgv=hgv, hx=hx, keep=keep):
            v = hs.numpy()
            return Result("ok", x=hx.numpy(), loss=float(v[0]),
                          grads={"v0": hgv.numpy(), "E": float(v[1]), "nu": float(v[2]), "yield_stress": float(v[3])})

        self.pending_results.append((t, ev, fill))

    def poll(self) -> List:
        """(ticket, Result) of every request whose device work has completed."""
        done, rest = [], []
        for t, ev, fill in self.pending_results:
            if ev.query():
                done.append((t, fill()))
            else:
                rest.append((t, ev, fill))
        self.pending_results = rest
        return done

    def forget(self, t: Ticket) -> None:
        for d in (self.solvers, self.tables, self.ckpts):
            d.pop(t.id, None)


class MPMServer:
    """Continuous-batching request loop on one GPU (see the module docstring)."""

    def __init__(self, hbm_budget: int = 40 << 30, device="cuda:0", block: int = 50, max_instances: int = 64,
                 capacity: Optional[Capacity] = None, sort_every: int = 32, max_blocks_in_flight: int = 2):
        self.cap = capacity or capacity_for_budget(hbm_budget, max_instances=max_instances, every=block)
        self.sched = Scheduler(self.cap, block=block)
        self.exec = GpuExecutor(self.cap, device=device, sort_every=sort_every)
        self.max_in_flight = max_blocks_in_flight
        self._lock = threading.Lock()
        self._wake = threading.Event()
        self._stop = False
        self._thread: Optional[threading.Thread] = None
        self.fault_hook: Optional[Callable[[Ticket], None]] = None   # test hook: raise to fail a request
        self.stats = {"blocks": 0, "substeps": 0, "particle_substeps": 0, "relayouts": 0}
        self._inflight: Deque = deque()

    # -- client side ---------------------------------------------------------------
    def submit(self, req: Request) -> Ticket:
        req.validate()
        t = Ticket(req, time.monotonic())
        with self._lock:
            why = self.sched.submit(t)
        if why is not None:
            t._finish(Result("rejected", error=why))
        self._wake.set()
        return t

    def start(self) -> "MPMServer":
        self._thread = threading.Thread(target=self._run, name="empm-server", daemon=True)
        self._thread.start()
        return self

    def stop(self, drain: bool = True, timeout: Optional[float] = None) -> None:
        """Stop the engine thread (after draining, by default) and free the
        device contexts. The thread is stopped even if draining times out."""
        try:
            if drain:
                self.drain(timeout)
        finally:
            self._stop = True
            self._wake.set()
            if self._thread is not None:
                self._thread.join(timeout)
            self.exec.torch.cuda.synchronize(self.exec.device)
            self.exec.close()

    def drain(self, timeout: Optional[float] = None) -> None:
        t0 = time.monotonic()
        while True:
            with self._lock:
                idle = self.sched.idle() and not self.exec.pending_results
            if idle:
                return
            if timeout is not None and time.monotonic() - t0 > timeout:
                raise TimeoutError("server did not drain in time")
            time.sleep(0.002)

    # -- engine ----------------------------------------------------------------------
    def _run(self) -> None:
        torch = self.exec.torch
        torch.cuda.set_device(self.exec.device)
        while not self._stop:
            try:
                worked = self.step()
            except Exception as e:   # a failure of the engine fails every request it holds
                self._fail_all(f"{type(e).__name__}: {e}")
                worked = False
            if not worked:
                self._wake.wait(0.002)
                self._wake.clear()

    def _fail_all(self, why: str) -> None:
        with self._lock:
            for t in list(self.sched.pending) + list(self.sched.forward) + list(self.sched.backward):
                t._finish(Result("error", error=why))
                self.exec.forget(t)
            self.sched.pending.clear()
            self.sched.forward = []
            self.sched.backward = []
            self.sched.ckpt_in_use = 0
            self.exec.layout, self.exec.offsets, self.exec.n_total = [], {}, 0
            self.exec.pending_results = []

    def step(self) -> bool:
        """One engine iteration; returns whether any work was issued or finished."""
        ex = self.exec
        worked = False
        for t, res in ex.poll():
            ex.forget(t)
            with self._lock:
                if t.req.grad:
                    self.sched.release_backward(t)
            t._finish(res)
            worked = True
        # bound the look-ahead of the host over the GPU
        while len(self._inflight) >= self.max_in_flight:
            self._inflight.popleft().synchronize()
        now = time.monotonic()
        with self._lock:
            prev_forward = list(self.sched.forward)
            plan = self.sched.plan(now)
        for t in plan.cancelled:
            ex.forget(t)
            t._finish(Result(t.phase, error="deadline exceeded" if t.phase == "timeout" else "cancelled"))
            worked = True
        # requests that completed their forward in the previous block (read
        # from the arena before it is re-laid out)
        for t in prev_forward:
            if t.progress >= t.req.n_substeps and t.phase == "forward":
                t.phase = "backward" if t.req.grad else "results"
                try:
                    ex.finish_forward(t)
                except Exception as e:
                    self._fail(t, e)
                    if t.req.grad:
                        with self._lock:
                            self.sched.release_backward(t)
                worked = True
        # per-request host faults while admitting: fail that request only
        ok_admitted = []
        for t in plan.admitted:
            try:
                if self.fault_hook is not None:
                    self.fault_hook(t)
                ok_admitted.append(t)
            except Exception as e:
                self._fail(t, e)
                with self._lock:
                    self.sched.forward.remove(t)
                    self.sched.ckpt_in_use -= t.ckpt_bytes
                    t.ckpt_bytes = 0
                plan.active.remove(t)
                plan.relayout = True
        if plan.relayout:
            ex.relayout(plan.active, ok_admitted)
            self.stats["relayouts"] += 1
            worked = True
        if plan.active:
            with self._lock:
                plan.block = self.sched.block_length(plan.active)
            ex.run_block(plan.active, plan.block)
            ev = ex.torch.cuda.Event()
            ev.record(ex.fwd_stream)
            self._inflight.append(ev)
            advanced = sum(min(plan.block, t.req.n_substeps - t.progress) * t.n for t in plan.active)
            with self._lock:
                self.sched.advance(plan)
            ex.after_block(plan.active)
            self.stats["blocks"] += 1
            self.stats["substeps"] += plan.block
            self.stats["particle_substeps"] += advanced          # held substeps excluded
            worked = True
        return worked

    def _fail(self, t: Ticket, e: Exception) -> None:
        self.exec.forget(t)
        t._finish(Result("error", error=f"{type(e).__name__}: {e}"))
