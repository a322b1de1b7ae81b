"""torch.autograd.Function boundary of the simulator.

Mirrors the four Functions of phys_sim/diff_simulator/warp_mpm/interface.py
(same positional signatures and returned tuples):

* MPMDifferentiableSimulationTrail (:20-251) — positions every ``substep``
  substeps, ``[T, N, 3]``; a scalar E is scaled by 1e6 in the forward (:70)
* MPMDifferentiableSimulation (:254-472) — final positions
* MPMDifferentiableSimulationWCheckpoint (:476-774) — (x, v, F, C) of a segment
* MPMDifferentiableSimulationClean (:777-986) — (x, v, F, C, cov)

The forward passes run the CUDA substep. With requires_grad the rollout is
checkpointed (``empm_b200.adjoint.CheckpointedRollout``), and the backward passes
run the library's adjoint kernels segment by segment. The gradients returned,
and their quirks, follow the reference's backward passes:

* a scalar (0-d) E or nu gets the per-particle gradients summed and divided by
  the particle count (interface.py:210-236). For the Trail function that
  gradient is taken with respect to the 1e6-scaled value;
* the Trail backward sums the gradient of all records over time and injects it
  at the final state (interface.py:178-197);
* MPMDifferentiableSimulation / Trail return no position gradient, and the
  density gradient restricted to ``density_change_mask`` (interface.py:238-251);
* gradients are taken at the start of the taped substeps. With
  extra_no_grad_steps > 0, Simulation and Trail therefore return zero velocity
  and density gradients (their inputs are not on the tape), while
  WCheckpoint / Clean return the gradients at the state after the extra steps.

A forward pass keeps its tape (stored segments or checkpoints) until the next
differentiable forward pass on the same solver, or until its graph is freed.
So a graph may be backpropagated more than once (retain_graph=True) until
then, as the reference's Warp tape allows; the next forward hands the tape's
segments back to the solver's pool before it allocates its own, so two sets
are never held at once, and a backward through the older graph then raises.
"""
from __future__ import annotations

import weakref
from typing import Optional

import torch
import torch.autograd as autograd
from torch import Tensor

from .adjoint import CheckpointedRollout, prepare_adjoint
from .mpm_data_structure import MPMModelStruct, MPMStateStruct

#: substeps between checkpoints of a differentiable rollout (MPMWARPDiff.checkpoint_every overrides it)
CHECKPOINT_EVERY = 20


def _set_E_nu(mpm_solver, mpm_model, E: Tensor, nu: Tensor, scale_scalar_E: float = 1.0):
    E_inp = E.item() * scale_scalar_E if E.ndim == 0 else E.detach()
    nu_inp = nu.item() if nu.ndim == 0 else nu.detach()
    mpm_solver.set_E_nu(mpm_model, E_inp, nu_inp)
    return E.ndim == 0, nu.ndim == 0


def _run(mpm_solver, mpm_model, state, n_steps, dt, record_every=None, step_callback=None):
    """Ping-pong rollout from `state`; returns (final_state, recorded positions)."""
    recorded = []
    other = state.partial_clone(requires_grad=False)
    cur = state
    first = True
    for i in range(n_steps):
        if step_callback is not None:
            step_callback(i)
        mpm_solver.p2g2p_differentiable(mpm_model, cur, other, dt)
        if record_every is not None and i % record_every == 0:
            recorded.append(other.particle_x.clone())
        if first:
            # never write into the caller's state object again
            cur = state.partial_clone(requires_grad=False)
            first = False
        cur, other = other, cur
    return cur, recorded


def _new_tape(mpm_solver, *args, **kw) -> CheckpointedRollout:
    """A tape for a differentiable forward pass. The solver's previous tape
    (if its graph is still alive) is released first: its segments go back to
    the pool and this pass reuses them."""
    prev = getattr(mpm_solver, "_live_tape", None)
    prev = prev() if prev is not None else None
    if prev is not None:
        prev.release()
    tape = CheckpointedRollout(mpm_solver, *args, **kw)
    mpm_solver._live_tape = weakref.ref(tape)
    return tape


def _taped_run(mpm_solver, mpm_model, state, n_steps, dt, step_callback=None):
    tape = _new_tape(mpm_solver, mpm_model, state, dt, n_steps,
                     checkpoint_every=int(getattr(mpm_solver, "checkpoint_every", CHECKPOINT_EVERY)),
                     step_callback=step_callback)
    return tape, tape.forward()


def _param_grads(ctx, res):
    """(E_grad, nu_grad, density_grad) from the tape's mu / lam / mass adjoints."""
    model, state = ctx.mpm_model, ctx.tape_state
    n = state.n_particles
    g_E, g_nu, g_rho = prepare_adjoint(model.E, model.nu, res["mu"], res["lam"], state.particle_vol, res["mass"])
    E_grad = g_E.sum() / n if ctx.aggregating_E else g_E
    nu_grad = g_nu.sum() / n if ctx.aggregating_nu else g_nu
    return E_grad, nu_grad, g_rho


def _fast_run(mpm_solver, mpm_model, state, n_steps, dt):
    if n_steps <= 0:
        return state
    other = state.partial_clone(requires_grad=False)
    work = state.partial_clone(requires_grad=False)
    work._x4.copy_(state._x4)
    work._v4.copy_(state._v4)
    work._C.copy_(state._C)
    work._F_trial.copy_(state._F_trial)
    return mpm_solver.rollout(mpm_model, work, other, dt, n_steps)


def _masked_density(g_rho: Tensor, mask: Optional[Tensor]) -> Tensor:
    return g_rho if mask is None else g_rho[mask.to(g_rho.device).bool()]


class MPMDifferentiableSimulationTrail(autograd.Function):
    @staticmethod
    def forward(ctx, mpm_solver, mpm_state: MPMStateStruct, mpm_model: MPMModelStruct, substep: int,
                substep_size: float, num_substeps: int, init_pos: Tensor, init_velocity: Tensor, E: Tensor, nu: Tensor,
                particle_density: Optional[Tensor] = None, density_change_mask: Optional[Tensor] = None,
                static_pos: Optional[Tensor] = None, device: str = "cuda:0", requires_grad: bool = True,
                extra_no_grad_steps: int = 0):
        if static_pos is not None:
            mpm_state.reset_state(static_pos.clone(), None, init_velocity, device=device, requires_grad=requires_grad)
            mpm_solver.restart_and_compute_F_C(mpm_model, mpm_state, init_pos, device=device)
        else:
            mpm_state.reset_state(init_pos.clone(), None, init_velocity, device=device, requires_grad=requires_grad)
        ctx.aggregating_E, ctx.aggregating_nu = _set_E_nu(mpm_solver, mpm_model, E, nu, scale_scalar_E=1e6)
        mpm_state.reset_density(tensor_density=particle_density, selection_mask=density_change_mask, device=device,
                                requires_grad=requires_grad)
        prev = mpm_state
        if extra_no_grad_steps > 0:
            mpm_state.update_mass()
            mpm_solver.prepare_mu_lam(mpm_model, mpm_state, device=device)
            prev, _ = _run(mpm_solver, mpm_model, prev, extra_no_grad_steps, substep_size)
        prev.update_mass()
        mpm_solver.prepare_mu_lam(mpm_model, prev, device=device)
        ctx.taped = requires_grad   # (ctx.requires_grad is reserved by torch.autograd)
        if not requires_grad:
            final, recorded = _run(mpm_solver, mpm_model, prev, num_substeps, substep_size, record_every=substep,
                                   step_callback=mpm_solver.step_callback)
            ctx.final_state = final
            return torch.stack(recorded, dim=0)
        tape = _new_tape(mpm_solver, mpm_model, prev, substep_size, num_substeps,
                         checkpoint_every=int(getattr(mpm_solver, "checkpoint_every", CHECKPOINT_EVERY)),
                         record_every=substep, step_callback=mpm_solver.step_callback)
        ctx.final_state = tape.forward()
        ctx.tape, ctx.tape_state, ctx.mpm_model = tape, prev, mpm_model
        ctx.on_tape = extra_no_grad_steps == 0
        ctx.save_for_backward(density_change_mask)
        return torch.stack(tape.records, dim=0)

    @staticmethod
    def backward(ctx, out_pos_grad):
        # interface.py:178-197: the record gradients are summed over time and
        # injected at the final state
        res = ctx.tape.backward(g_x=out_pos_grad.sum(dim=0))
        E_grad, nu_grad, density_grad = _param_grads(ctx, res)
        velo_grad = res["v"] if ctx.on_tape else torch.zeros_like(res["v"])
        density_grad = _masked_density(density_grad if ctx.on_tape else torch.zeros_like(density_grad),
                                       ctx.saved_tensors[0])
        return (None, None, None, None, None, None, None, velo_grad, E_grad, nu_grad, density_grad, None, None,
                None, None, None)


class MPMDifferentiableSimulation(autograd.Function):
    @staticmethod
    def forward(ctx, mpm_solver, mpm_state: MPMStateStruct, mpm_model: MPMModelStruct, substep: int,
                substep_size: float, num_substeps: int, init_pos: Tensor, init_velocity: Tensor, E: Tensor, nu: Tensor,
                particle_density: Optional[Tensor] = None, density_change_mask: Optional[Tensor] = None,
                static_pos: Optional[Tensor] = None, device: str = "cuda:0", requires_grad: bool = True,
                extra_no_grad_steps: int = 0):
        if static_pos is not None:
            mpm_state.reset_state(static_pos.clone(), None, init_velocity, device=device, requires_grad=requires_grad)
            mpm_solver.restart_and_compute_F_C(mpm_model, mpm_state, init_pos, device=device)
        else:
            mpm_state.reset_state(init_pos.clone(), None, init_velocity, device=device, requires_grad=requires_grad)
        ctx.aggregating_E, ctx.aggregating_nu = _set_E_nu(mpm_solver, mpm_model, E, nu)
        mpm_state.reset_density(tensor_density=particle_density, selection_mask=density_change_mask, device=device,
                                requires_grad=requires_grad)
        prev = mpm_state
        if extra_no_grad_steps > 0:
            mpm_state.update_mass()
            mpm_solver.prepare_mu_lam(mpm_model, mpm_state, device=device)
            prev = _fast_run(mpm_solver, mpm_model, prev, extra_no_grad_steps, substep_size)
        prev.update_mass()
        mpm_solver.prepare_mu_lam(mpm_model, prev, device=device)
        if not requires_grad:
            return _fast_run(mpm_solver, mpm_model, prev, num_substeps, substep_size).particle_x.clone()
        ctx.tape, final = _taped_run(mpm_solver, mpm_model, prev, num_substeps, substep_size)
        ctx.tape_state, ctx.mpm_model = prev, mpm_model
        ctx.on_tape = extra_no_grad_steps == 0
        ctx.save_for_backward(density_change_mask)
        return final.particle_x.clone()

    @staticmethod
    def backward(ctx, out_pos_grad):
        res = ctx.tape.backward(g_x=out_pos_grad)
        E_grad, nu_grad, density_grad = _param_grads(ctx, res)
        velo_grad = res["v"] if ctx.on_tape else torch.zeros_like(res["v"])
        density_grad = _masked_density(density_grad if ctx.on_tape else torch.zeros_like(density_grad),
                                       ctx.saved_tensors[0])
        return (None, None, None, None, None, None, None, velo_grad, E_grad, nu_grad, density_grad, None, None,
                None, None, None)


class MPMDifferentiableSimulationWCheckpoint(autograd.Function):
    @staticmethod
    @torch.no_grad()
    def forward(ctx, mpm_solver, mpm_state: MPMStateStruct, mpm_model: MPMModelStruct, substep_size: float,
                num_substeps: int, particle_x: Tensor, particle_v: Tensor, particle_F: Tensor, particle_C: Tensor,
                E: Tensor, nu: Tensor, particle_density: Optional[Tensor] = None, query_mask: Optional[Tensor] = None,
                device: str = "cuda:0", requires_grad: bool = True, extra_no_grad_steps: int = 0):
        mpm_state.continue_from_torch(particle_x, particle_v, particle_F, particle_C, device=device,
                                      requires_grad=True)
        ctx.aggregating_E, ctx.aggregating_nu = _set_E_nu(mpm_solver, mpm_model, E, nu)
        mpm_solver.prepare_mu_lam(mpm_model, mpm_state, device=device)
        mpm_state.reset_density(tensor_density=particle_density, selection_mask=query_mask, device=device,
                                requires_grad=True, update_mass=True)
        prev = mpm_state
        if extra_no_grad_steps > 0:
            prev = _fast_run(mpm_solver, mpm_model, prev, extra_no_grad_steps, substep_size)
        ctx.tape, final = _taped_run(mpm_solver, mpm_model, prev, num_substeps, substep_size)
        ctx.tape_state, ctx.mpm_model = prev, mpm_model
        n = final.n_particles
        return (final.particle_x.clone(), final.particle_v.clone(), final.particle_F_trial.reshape(n, 3, 3).clone(),
                final.particle_C.reshape(n, 3, 3).clone())

    @staticmethod
    def backward(ctx, out_pos_grad, out_velo_grad, out_F_grad, out_C_grad):
        res = ctx.tape.backward(g_x=out_pos_grad, g_v=out_velo_grad, g_C=out_C_grad, g_F=out_F_grad)
        E_grad, nu_grad, density_grad = _param_grads(ctx, res)
        return (None, None, None, None, None, res["x"], res["v"], res["F"], res["C"], E_grad, nu_grad, density_grad,
                None, None, None, None)


class MPMDifferentiableSimulationClean(autograd.Function):
    @staticmethod
    @torch.no_grad()
    def forward(ctx, mpm_solver, mpm_state: MPMStateStruct, mpm_model: MPMModelStruct, substep_size: float,
                num_substeps: int, particle_x: Tensor, particle_v: Tensor, particle_F: Tensor, particle_C: Tensor,
                E: Tensor, nu: Tensor, particle_density: Optional[Tensor] = None, query_mask: Optional[Tensor] = None,
                device: str = "cuda:0", requires_grad: bool = True, extra_no_grad_steps: int = 0):
        mpm_state.continue_from_torch(particle_x, particle_v, particle_F, particle_C, device=device,
                                      requires_grad=True)
        ctx.aggregating_E, ctx.aggregating_nu = _set_E_nu(mpm_solver, mpm_model, E, nu)
        mpm_solver.prepare_mu_lam(mpm_model, mpm_state, device=device)
        mpm_state.reset_density(tensor_density=particle_density, selection_mask=query_mask, device=device,
                                requires_grad=True, update_mass=True)
        prev = mpm_state
        if extra_no_grad_steps > 0:
            prev = _fast_run(mpm_solver, mpm_model, prev, extra_no_grad_steps, substep_size)
        prev.update_mass()
        mpm_solver.prepare_mu_lam(mpm_model, prev, device=device)
        ctx.tape, final = _taped_run(mpm_solver, mpm_model, prev, num_substeps, substep_size)
        ctx.tape_state, ctx.mpm_model = prev, mpm_model
        n = final.n_particles
        return (final.particle_x.clone(), final.particle_v.clone(), final.particle_F_trial.reshape(n, 3, 3).clone(),
                final.particle_C.reshape(n, 3, 3).clone(), final.particle_cov.view(-1, 6).clone())

    @staticmethod
    def backward(ctx, out_pos_grad, out_velo_grad, out_F_grad, out_C_grad, out_cov_grad):
        # the covariance output is a pass-through (its update is disabled in the
        # reference, mpm_utils.py:578), so its gradient does not reach the inputs
        res = ctx.tape.backward(g_x=out_pos_grad, g_v=out_velo_grad, g_C=out_C_grad, g_F=out_F_grad)
        E_grad, nu_grad, density_grad = _param_grads(ctx, res)
        return (None, None, None, None, None, res["x"], res["v"], res["F"], res["C"], E_grad, nu_grad, density_grad,
                None, None, None, None)
