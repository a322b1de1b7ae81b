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


class CheckpointedRollout:
    """Forward rollout that can be differentiated afterwards.

    ``record_every`` records positions after every substep ``i`` with
    ``i % record_every == 0`` (the Trail function's recording). Segments end at
    those substeps, so the adjoint of a record is injected exactly where the
    record was taken.
    """

    def __init__(self, solver, model: MPMModelStruct, state: MPMStateStruct, dt: float, n_steps: int,
                 checkpoint_every: int = 20, record_every: Optional[int] = None, step_callback=None):
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
        self.records: List[Tensor] = []
        self.ckpts: List[_Checkpoint] = []
        self.final: Optional[MPMStateStruct] = None

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
        a = st.partial_clone(requires_grad=False)
        for src, dst in ((st._x4, a._x4), (st._v4, a._v4), (st._C, a._C), (st._F_trial, a._F_trial)):
            dst.copy_(src)
        b = st.partial_clone(requires_grad=False)
        cur, other = a, b
        record_set = set(self.record_steps)
        for s0, s1 in zip(self.bounds[:-1], self.bounds[1:]):
            self.ckpts.append(_Checkpoint(s0, cur._x4.clone(), cur._v4.clone(), cur._C.clone(), cur._F_trial.clone(),
                                          model.mu.clone(), model.lam.clone(), model.yield_stress.clone()))
            L = s1 - s0
            seg = (N.EmpmStep * L).from_buffer(self.table, s0 * ctypes.sizeof(N.EmpmStep))
            solver.time = times[s0]
            res = solver.rollout(model, cur, other, self.dt, L, schedule=(seg, times[s1]))
            if res is not cur:
                cur, other = other, cur
            if (s1 - 1) in record_set:
                self.records.append(cur.particle_x.clone())
        solver.time = t_end
        self._ctx = ctx
        self.final = cur
        return cur

    def backward(self, g_x: Optional[Tensor] = None, g_v: Optional[Tensor] = None, g_C: Optional[Tensor] = None,
                 g_F: Optional[Tensor] = None, g_records: Optional[Sequence[Optional[Tensor]]] = None
                 ) -> Dict[str, Tensor]:
        """Adjoint of the whole rollout. g_* are dL/d(final state); g_records[r]
        is dL/d(record r). Returns dL/d(initial x, v, C, F_trial, mu, lam,
        yield_stress, mass)."""
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
