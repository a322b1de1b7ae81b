"""Reverse-mode rollouts: a checkpointed forward and adjoint segments.

The reference differentiates a rollout by recording every kernel launch on a
Warp tape and replaying Warp's generated adjoints (interface.py:130-251,
391-472, 579-774, 899-986). All T substep states stay alive on that tape
(``partial_clone`` per substep, mpm_data_structure.py:356-387). Here the
forward keeps one checkpoint every ``checkpoint_every`` substeps: the packed
particle state plus mu, lam and the yield stress, which the plastic return
maps update in place. The backward walks the segments in reverse through
``empm_adjoint_segment``. That call recomputes a segment from its checkpoint
on the GPU, then runs the per-substep adjoint kernels.

Gradients are exact for the FP32 forward map up to rounding. They are taken
with respect to the state at the start of the taped rollout (x, v, C,
F_trial), the per-particle mu, lam, yield stress and mass, and, through
``prepare_adjoint``, E, nu and density.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import torch
from torch import Tensor

from . import _native as N
from .mpm_data_structure import DTYPE, MPMModelStruct, MPMStateStruct, _f9_pack, _f9_unpack, _stream_ptr


class PackedGrad:
    """Adjoint of a particle state in the library layout: x and v as float4
    rows (w unused), C and F_trial as f9 planes."""

    def __init__(self, n: int, device):
        self.n = n
        self.x4 = torch.zeros((n, 4), dtype=DTYPE, device=device)
        self.v4 = torch.zeros((n, 4), dtype=DTYPE, device=device)
        self.C = torch.zeros(9 * n, dtype=DTYPE, device=device)
        self.F = torch.zeros(9 * n, dtype=DTYPE, device=device)

    def particles(self) -> N.EmpmParticles:
        return N.EmpmParticles(self.x4.data_ptr(), self.v4.data_ptr(), self.C.data_ptr(), self.F.data_ptr())

    def add(self, g_x: Optional[Tensor] = None, g_v: Optional[Tensor] = None, g_C: Optional[Tensor] = None,
            g_F: Optional[Tensor] = None) -> None:
        n = self.n
        if g_x is not None:
            self.x4[:, :3] += g_x.detach().reshape(n, 3).to(self.x4)
        if g_v is not None:
            self.v4[:, :3] += g_v.detach().reshape(n, 3).to(self.v4)
        if g_C is not None:
            tmp = torch.empty_like(self.C)
            _f9_pack(tmp, g_C.detach().reshape(n, 9).to(self.C))
            self.C += tmp
        if g_F is not None:
            tmp = torch.empty_like(self.F)
            _f9_pack(tmp, g_F.detach().reshape(n, 9).to(self.F))
            self.F += tmp

    def x(self) -> Tensor:
        return self.x4[:, :3].clone()

    def v(self) -> Tensor:
        return self.v4[:, :3].clone()

    def C_mat(self) -> Tensor:
        return _f9_unpack(self.C, self.n).clone()

    def F_mat(self) -> Tensor:
        return _f9_unpack(self.F, self.n).clone()


@dataclass
class _Checkpoint:
    step: int            # substep index the segment starts at
    x4: Tensor
    v4: Tensor
    C: Tensor
    F: Tensor
    mu: Tensor
    lam: Tensor
    ys: Tensor

    def particles(self) -> N.EmpmParticles:
        return N.EmpmParticles(self.x4.data_ptr(), self.v4.data_ptr(), self.C.data_ptr(), self.F.data_ptr())


class _StoredSegment:
    """A segment kept on the device by empm_segment_forward for its reverse
    pass. Released segments go back to their context's pool."""

    def __init__(self, ctx, ptr: ctypes.c_void_p, step: int, n_steps: int, block_cap: int):
        self.ctx = ctx
        self.ptr = ptr
        self.step = step
        self.n_steps = n_steps
        self.block_cap = block_cap

    def release(self) -> None:
        if self.ptr is not None:
            need = self.ctx.touched_blocks
            if need is not None and self.block_cap > 2 * int(need * 1.25) + 64:
                self.destroy()   # sized by a first guess far above what the rollouts touch
                return
            self.ctx.give_segment(self.ptr, self.n_steps, self.block_cap)
        self.ptr = None

    def destroy(self) -> None:
        if self.ptr is not None:
            N.lib().empm_segment_destroy(self.ptr)
        self.ptr = None


class CheckpointedRollout:
    """Forward rollout that can be differentiated afterwards.

    ``record_every`` records positions after every substep ``i`` with
    ``i % record_every == 0`` (the Trail function's recording). Segments end at
    those substeps, so the adjoint of a record is injected exactly where the
    record was taken.

    Segments are either stored or checkpointed. A stored segment keeps, from
    the forward pass, everything its reverse pass reads (empm_segment_*). The
    reverse pass then runs only the adjoint kernels, as Warp's tape replays the
    recorded launches. A checkpointed segment keeps its start state, and its
    reverse pass recomputes it first (empm_adjoint_segment). ``store``: True
    stores every segment and raises MemoryError when they do not fit; False
    checkpoints. None stores when the whole rollout fits ``store_budget`` bytes
    (default: half of the device memory free at the forward pass) and the
    allocation succeeds, and checkpoints otherwise. Released segments return
    to the solver context's pool and are reused in stream order, so one
    solver's rollouts should run on one CUDA stream.
    """

    def __init__(self, solver, model: MPMModelStruct, state: MPMStateStruct, dt: float, n_steps: int,
                 checkpoint_every: int = 20, record_every: Optional[int] = None, step_callback=None,
                 store: Optional[bool] = None, store_budget: Optional[int] = None):
        if n_steps < 1:
            raise ValueError("n_steps must be >= 1")
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be >= 1")
        self.solver = solver
        self.model = model
        self.dt = float(dt)
        self.n_steps = int(n_steps)
        self.every = int(checkpoint_every)
        self.record_steps: List[int] = [] if record_every is None else list(range(0, self.n_steps, int(record_every)))
        self.step_callback = step_callback
        self.state = state
        self.store = store
        self.store_budget = store_budget
        self.records: List[Tensor] = []
        self.ckpts: List[_Checkpoint] = []
        self.segments: List[_StoredSegment] = []
        self.final: Optional[MPMStateStruct] = None

    @property
    def stored(self) -> bool:
        """True when the forward pass stored its segments."""
        return bool(self.segments)

    def release(self) -> None:
        """Hand the stored segments back to the pool and drop the checkpoints
        (a later backward then raises)."""
        for sg in self.segments:
            sg.release()
        self.segments = []
        self.ckpts = []

    def __del__(self):
        try:
            self.release()
        except Exception:   # interpreter shutdown: the library may be gone
            pass

    def _block_cap(self, ctx, n: int) -> int:
        """Grid blocks per substep to keep: the largest count a stored forward
        pass of this context touched, with a margin; before any, a guess from
        the particle count (an overflow is detected and the pass repeated).
        Segments sized by a guess far above the observed counts are freed when
        released rather than pooled."""
        if ctx.touched_blocks is not None:
            return int(ctx.touched_blocks * 1.25) + 16
        return max(512, n // 256)

    def _allocate_segments(self, ctx, dev, block_cap: int) -> bool:
        """Stored segments for every segment of the rollout, or False (nothing
        kept) when they exceed the budget or do not fit."""
        if self.store is False:
            return False
        L = N.lib()
        lengths = [s1 - s0 for s0, s1 in zip(self.bounds[:-1], self.bounds[1:])]
        total = new = 0
        nb = ctypes.c_size_t()
        for n_seg in set(lengths):
            N.check(L.empm_segment_bytes(ctx.ptr, n_seg, block_cap, ctypes.byref(nb)), ctx.ptr)
            total += nb.value * lengths.count(n_seg)
            new += nb.value * max(0, lengths.count(n_seg) - ctx.pooled(n_seg, block_cap))
        budget = self.store_budget
        if budget is None:
            # segments already in the pool count as available
            budget = torch.cuda.mem_get_info(dev)[0] // 2 + (total - new)
        if total > budget:
            if self.store:
                raise MemoryError(f"storing the rollout needs {total} bytes, over the budget of {budget}")
            return False
        segs = []
        for s0, n_seg in zip(self.bounds[:-1], lengths):
            pooled = ctx.take_segment(n_seg, block_cap)
            if pooled is not None:
                segs.append(_StoredSegment(ctx, pooled[0], s0, n_seg, pooled[1]))
                continue
            p = ctypes.c_void_p()
            with torch.cuda.device(dev):
                rc = L.empm_segment_create(ctx.ptr, n_seg, block_cap, ctypes.byref(p))
            if rc != N.EMPM_OK:
                for sg in segs:
                    sg.release()
                if rc == N.EMPM_ERR_OOM and not self.store:
                    return False
                if rc == N.EMPM_ERR_OOM:
                    raise MemoryError(N.last_error(ctx.ptr))
                N.check(rc, ctx.ptr)
            segs.append(_StoredSegment(ctx, p, s0, n_seg, block_cap))
        self.segments = segs
        return True

    def _blocks_overflowed(self, ctx, stream) -> bool:
        """Read the touched-block maxima of the stored forward pass (one wait
        for the stream) into the context's estimate; True when a segment could
        not keep its grids."""
        L = N.lib()
        mx, cap = ctypes.c_int(), ctypes.c_int()
        over = False
        seen = 0
        for sg in self.segments:
            N.check(L.empm_segment_blocks(sg.ptr, ctypes.byref(mx), ctypes.byref(cap), stream), ctx.ptr)
            seen = max(seen, mx.value)
            over |= mx.value > cap.value
        ctx.touched_blocks = seen if ctx.touched_blocks is None else max(ctx.touched_blocks, seen)
        return over

    def _bounds(self) -> List[int]:
        b = set(range(0, self.n_steps, self.every))
        b.update(i + 1 for i in self.record_steps if i + 1 < self.n_steps)
        b.add(self.n_steps)
        return sorted(b)

    def forward(self) -> MPMStateStruct:
        solver, model, st = self.solver, self.model, self.state
        n = st.n_particles
        ctx = solver._context(model, n, st.device, max_steps=self.n_steps)
        t0 = solver.time
        self.table, t_end = solver.build_schedule(t0, self.dt, self.n_steps, self.step_callback)
        times = [t0]
        for _ in range(self.n_steps):
            times.append(times[-1] + self.dt)
        self.bounds = self._bounds()
        self.release()
        stream = _stream_ptr(st.device)
        material0 = (model.mu.clone(), model.lam.clone(), model.yield_stress.clone())
        for attempt in range(2):
            store = self._allocate_segments(ctx, st.device, self._block_cap(ctx, n))
            cur = self._run(ctx, store, times, stream)
            if not store or not self._blocks_overflowed(ctx, stream):
                break
            # a substep touched more grid blocks than the segments hold: run the
            # pass again from the start with room for the counts just observed
            for sg in self.segments:
                sg.destroy()
            self.segments = []
            for dst, src in zip((model.mu, model.lam, model.yield_stress), material0):
                dst.copy_(src)
            if attempt == 1:
                raise RuntimeError("stored forward pass overflowed its grid store twice")
        solver.time = t_end
        self._ctx = ctx
        self.final = cur
        return cur

    def _run(self, ctx, store: bool, times, stream) -> MPMStateStruct:
        """The forward pass over all segments, stored or checkpointed."""
        solver, model, st = self.solver, self.model, self.state
        self.ckpts = []
        self.records = []
        a = st.partial_clone(requires_grad=False)
        for src, dst in ((st._x4, a._x4), (st._v4, a._v4), (st._C, a._C), (st._F_trial, a._F_trial)):
            dst.copy_(src)
        b = st.partial_clone(requires_grad=False)
        cur, other = a, b
        record_set = set(self.record_steps)
        for i, (s0, s1) in enumerate(zip(self.bounds[:-1], self.bounds[1:])):
            L = s1 - s0
            seg = (N.EmpmStep * L).from_buffer(self.table, s0 * ctypes.sizeof(N.EmpmStep))
            solver.time = times[s0]
            if store:
                mat = N.EmpmMaterial(cur.particle_vol.data_ptr(), model.mu.data_ptr(), model.lam.data_ptr(),
                                     model.yield_stress.data_ptr(), cur._sel_ptr(), other._F.data_ptr())
                with torch.cuda.device(st.device):
                    N.check(N.lib().empm_segment_forward(ctx.ptr, self.segments[i].ptr, cur._particles(),
                                                         model.mu.data_ptr(), model.lam.data_ptr(),
                                                         model.yield_stress.data_ptr(), mat, seg, L,
                                                         other._particles(), stream), ctx.ptr)
                cur, other = other, cur
            else:
                self.ckpts.append(_Checkpoint(s0, cur._x4.clone(), cur._v4.clone(), cur._C.clone(),
                                              cur._F_trial.clone(), model.mu.clone(), model.lam.clone(),
                                              model.yield_stress.clone()))
                res = solver.rollout(model, cur, other, self.dt, L, schedule=(seg, times[s1]))
                if res is not cur:
                    cur, other = other, cur
            if (s1 - 1) in record_set:
                self.records.append(cur.particle_x.clone())
        return cur

    def backward(self, g_x: Optional[Tensor] = None, g_v: Optional[Tensor] = None, g_C: Optional[Tensor] = None,
                 g_F: Optional[Tensor] = None, g_records: Optional[Sequence[Optional[Tensor]]] = None
                 ) -> Dict[str, Tensor]:
        """Adjoint of the whole rollout. g_* are dL/d(final state); g_records[r]
        is dL/d(record r). Returns dL/d(initial x, v, C, F_trial, mu, lam,
        yield_stress, mass)."""
        if not self.segments and not self.ckpts:
            raise RuntimeError("nothing to differentiate: forward() has not run, or its tape was released "
                               "(release(), or a later differentiable forward pass on the same solver)")
        st, model = self.state, self.model
        n = st.n_particles
        dev = st.device
        grad = PackedGrad(n, dev)
        grad.add(g_x, g_v, g_C, g_F)
        g_mu = torch.zeros(n, dtype=DTYPE, device=dev)
        g_lam = torch.zeros_like(g_mu)
        g_ys = torch.zeros_like(g_mu)
        g_mass = torch.zeros_like(g_mu)
        gmat = N.EmpmMaterialGrad(g_mu.data_ptr(), g_lam.data_ptr(), g_ys.data_ptr(), g_mass.data_ptr())
        mat = N.EmpmMaterial(st.particle_vol.data_ptr(), model.mu.data_ptr(), model.lam.data_ptr(),
                             model.yield_stress.data_ptr(), st._sel_ptr(), None)
        rec_index = {s: r for r, s in enumerate(self.record_steps)}
        ctx = self.solver._context(model, n, dev, max_steps=self.n_steps)
        L = N.lib()
        stream = _stream_ptr(dev)
        if self.segments:
            for sg, s1 in reversed(list(zip(self.segments, self.bounds[1:]))):
                r = rec_index.get(s1 - 1)
                if r is not None and g_records is not None and g_records[r] is not None:
                    grad.add(g_x=g_records[r])
                with torch.cuda.device(dev):
                    N.check(L.empm_segment_reverse(ctx.ptr, sg.ptr, grad.particles(), gmat, stream), ctx.ptr)
            return {"x": grad.x(), "v": grad.v(), "C": grad.C_mat(), "F": grad.F_mat(), "mu": g_mu, "lam": g_lam,
                    "yield_stress": g_ys, "mass": g_mass}
        for ck, s1 in reversed(list(zip(self.ckpts, self.bounds[1:]))):
            r = rec_index.get(s1 - 1)
            if r is not None and g_records is not None and g_records[r] is not None:
                grad.add(g_x=g_records[r])
            steps = s1 - ck.step
            seg = (N.EmpmStep * steps).from_buffer(self.table, ck.step * ctypes.sizeof(N.EmpmStep))
            with torch.cuda.device(dev):
                N.check(L.empm_adjoint_segment(ctx.ptr, ck.particles(), ck.mu.data_ptr(), ck.lam.data_ptr(),
                                               ck.ys.data_ptr(), mat, seg, steps, grad.particles(), gmat, stream),
                        ctx.ptr)
        return {"x": grad.x(), "v": grad.v(), "C": grad.C_mat(), "F": grad.F_mat(), "mu": g_mu, "lam": g_lam,
                "yield_stress": g_ys, "mass": g_mass}


def prepare_adjoint(E: Tensor, nu: Tensor, g_mu: Tensor, g_lam: Tensor, vol: Optional[Tensor] = None,
                    g_mass: Optional[Tensor] = None):
    """(dL/dE, dL/dnu, dL/ddensity) from dL/dmu, dL/dlam and dL/dmass through
    mu, lam = f(E, nu) and mass = density * vol. E and nu are the per-particle
    arrays the forward used."""
    n = g_mu.shape[0]
    dev = g_mu.device
    E = E.detach().reshape(-1).to(dev, DTYPE).contiguous()
    nu = nu.detach().reshape(-1).to(dev, DTYPE).contiguous()
    if E.numel() == 1:
        E = E.expand(n).contiguous()
    if nu.numel() == 1:
        nu = nu.expand(n).contiguous()
    g_E = torch.empty(n, dtype=DTYPE, device=dev)
    g_nu = torch.empty_like(g_E)
    g_rho = None
    if vol is not None and g_mass is not None:
        g_rho = torch.empty_like(g_E)
    N.check(N.lib().empm_prepare_adjoint(E.data_ptr(), nu.data_ptr(), g_mu.data_ptr(), g_lam.data_ptr(),
                                         g_E.data_ptr(), g_nu.data_ptr(),
                                         None if g_rho is None else vol.data_ptr(),
                                         None if g_rho is None else g_mass.data_ptr(),
                                         None if g_rho is None else g_rho.data_ptr(), n, _stream_ptr(dev)))
    return g_E, g_nu, g_rho
