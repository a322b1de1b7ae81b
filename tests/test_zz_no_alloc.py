"""The allocation-free substep (empm_substep_noalloc) against the regular one.

Some callers cannot allocate device memory when they step the simulation,
for example an application that reserves all device memory at start-up and
steps the simulator inside a fixed-budget control or rendering loop.
empm_substep_noalloc serves them with statically sized grid scratch. These
tests call it through the C ABI and check two calls in a row against the
context-based empm_substep on identical inputs, within the tolerance used by
the other GPU tests (positions 1e-6, other fields relative 1e-5: the two runs
differ only in the order of the floating-point reductions), on grids of 32^3,
61^3 (not a multiple of the 4^3 block) and 64^3 (the maximum, which fills the
static arrays), and a 32^3 grid right after a 64^3 one (the arrays keep the
previous call's contents beyond the cleared range). They also check the
status word the caller passes, and that grids beyond the static maximum are
rejected with a clear error.

This file is named so that pytest collects it last.
"""
import numpy as np
import pytest
import torch

from empm_b200 import MPMModelStruct, MPMStateStruct, MPMWARPDiff
from empm_b200 import _native as N
from empm_b200.mpm_data_structure import _stream_ptr
from tests.gpu_helpers import max_abs

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
N_MAX = 64


def _setup(n=3000, G=32, seed=7, x=None):
    rng = np.random.default_rng(seed)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=DEV)  # noqa: E731
    if x is None:
        x = rng.uniform(0.3, 0.7, (n, 3))
    st = MPMStateStruct()
    st.init(n, device=DEV)
    st.from_torch(t(x), t(np.full(n, 0.064 / n)), None, t(rng.standard_normal((n, 3)) * 0.3), n_grid=G, device=DEV)
    st.particle_F_trial = t(np.eye(3)[None] + 0.05 * rng.standard_normal((n, 3, 3)))
    st.reset_density(t(np.full(n, 1e3)), update_mass=True)
    md = MPMModelStruct()
    md.init(n, device=DEV)
    md.init_other_params(n_grid=G)
    md.material = 5
    md.gravitational_accelaration = (0.0, -9.8, 0.0)
    md.E.copy_(t(np.exp(rng.uniform(np.log(5e3), np.log(5e4), n))))
    md.nu.copy_(t(rng.uniform(0.25, 0.4, n)))
    md.finalize_mu_lam(n)
    md.yield_stress.copy_(t(rng.uniform(5e2, 3e3, n)))
    solver = MPMWARPDiff()
    solver.initialize(n, n_grid=G)
    solver.add_surface_collider((0.0, 3.0 / G, 0.0), (0.0, 1.0, 0.0), "sticky", 0.0)
    solver.add_bounding_box()
    return st, md, solver


def _noalloc_step(solver, md, st, nxt, dt, status=None):
    step = N.EmpmStep()
    solver._fill_step(step, solver.time, dt)
    mat = solver._material(md, st)
    rc = N.lib().empm_substep_noalloc(md._params(), st._particles(), nxt._particles(), mat, step, st.n_particles,
                                      None if status is None else status.data_ptr(), _stream_ptr(st.device))
    N.check(rc)
    solver._modify(solver.time, dt)
    solver.time = solver.time + dt


def _compare_two_calls(G, seed=7):
    dt = 2e-4
    st_a, md_a, sv_a = _setup(G=G, seed=seed)
    st_b, md_b, sv_b = _setup(G=G, seed=seed)
    a0, a1 = st_a, st_a.partial_clone()
    b0, b1 = st_b, st_b.partial_clone()
    for call in range(2):
        sv_a.p2g2p_differentiable(md_a, a0, a1, dt)       # context-based entry point
        _noalloc_step(sv_b, md_b, b0, b1, dt)             # allocation-free entry point
        torch.cuda.synchronize()
        err = max_abs(b1.particle_x, a1.particle_x)
        print(f"G={G} call {call + 1}: max |x_noalloc - x_ctx| = {err:.2e}")
        assert err <= 1e-6
        for name in ("particle_v", "particle_C", "particle_F_trial"):
            ref = getattr(a1, name).reshape(st_a.n_particles, -1)
            got = getattr(b1, name).reshape(st_a.n_particles, -1)
            scale = max(float(ref.abs().max()), 1.0)
            assert float((got - ref).abs().max()) <= 1e-5 * scale, name
        assert float((md_b.yield_stress - md_a.yield_stress).abs().max()) <= 1e-5 * float(md_a.yield_stress.max())
        a0, a1 = a1, a0
        b0, b1 = b1, b0


@pytest.mark.parametrize("G", [32, 61, N_MAX])
def test_noalloc_matches_context_substep_twice(G):
    _compare_two_calls(G)


def test_noalloc_smaller_grid_after_the_largest():
    """A 32^3 call right after a 64^3 call: only the 32^3 range is cleared,
    the rest of the arrays still holds the larger call's data."""
    _compare_two_calls(N_MAX, seed=11)
    _compare_two_calls(32, seed=12)


def test_noalloc_status_word_reports_out_of_band():
    n, G = 500, 32
    rng = np.random.default_rng(3)
    x = rng.uniform(0.3, 0.7, (n, 3))
    x[17] = (0.99, 0.5, 0.5)          # its stencil reaches past the last node: skipped and flagged
    st, md, solver = _setup(n=n, G=G, x=x)
    nxt = st.partial_clone()
    status = torch.zeros(1, dtype=torch.int32, device=DEV)
    _noalloc_step(solver, md, st, nxt, 1e-4, status)
    torch.cuda.synchronize()
    assert int(status.item()) & N.EMPM_STATUS_OUT_OF_BAND
    # the word accumulates until the caller clears it; an in-band step adds nothing
    status.zero_()
    st2, md2, solver2 = _setup(n=n, G=G)
    nxt2 = st2.partial_clone()
    _noalloc_step(solver2, md2, st2, nxt2, 1e-4, status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0


def test_noalloc_rejects_grids_beyond_its_maximum_and_aliasing():
    st, md, solver = _setup(n=100, G=32)
    nxt = st.partial_clone()
    step = N.EmpmStep()
    solver._fill_step(step, 0.0, 1e-4)
    md.init_other_params(n_grid=N_MAX + 1)
    rc = N.lib().empm_substep_noalloc(md._params(), st._particles(), nxt._particles(), solver._material(md, st), step,
                                      st.n_particles, None, _stream_ptr(st.device))
    assert rc == N.EMPM_ERR_INVALID
    assert "allocation-free maximum" in N.last_error()
    md.init_other_params(n_grid=32)
    out = nxt._particles()
    out.v = st._particles().v          # in and out share the velocity plane
    rc = N.lib().empm_substep_noalloc(md._params(), st._particles(), out, solver._material(md, st), step,
                                      st.n_particles, None, _stream_ptr(st.device))
    assert rc == N.EMPM_ERR_INVALID
    assert "distinct" in N.last_error()
