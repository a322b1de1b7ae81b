"""CPU-side checks of the C ABI: the library loads, exports every symbol that
include/empm_b200.h declares, and rejects bad arguments before touching the
device. No compute runs here."""
import ctypes

import pytest

from empm_b200 import _native as N


def test_library_exports_header_symbols():
    L = N.lib()
    declared = N.header_symbols()
    assert "empm_substep" in declared and "empm_rollout" in declared
    for name in declared:
        assert hasattr(L, name), f"{name} declared in include/empm_b200.h but not exported"


def test_version():
    assert N.lib().empm_version() >= 100


def test_struct_sizes_match_header():
    # the library static_asserts the same numbers
    assert ctypes.sizeof(N.EmpmCollider) == 104
    assert ctypes.sizeof(N.EmpmModifier) == 88
    assert ctypes.sizeof(N.EmpmStep) == 2392


def test_ctx_create_rejects_bad_params_without_gpu():
    L = N.lib()
    out = ctypes.c_void_p()
    assert L.empm_ctx_create(None, 10, 4, ctypes.byref(out)) == -1
    p = N.EmpmModelParams()
    p.n_grid = 2          # below the minimum
    p.grid_lim = 1.0
    assert L.empm_ctx_create(p, 10, 4, ctypes.byref(out)) == -1
    assert "n_grid" in N.last_error()
    p.n_grid = 32
    p.material = 9        # unknown material id
    assert L.empm_ctx_create(p, 10, 4, ctypes.byref(out)) == -4
    p.material = 0
    assert L.empm_ctx_create(p, 10, 0, ctypes.byref(out)) == -1   # max_steps < 1


def test_null_context_is_rejected():
    L = N.lib()
    st = N.EmpmStep()
    assert L.empm_substep(None, None, None, None, st, None) == -1
    assert L.empm_rollout(None, None, None, None, None, 1, 1, 0, None) == -1
    with pytest.raises(N.EmpmError):
        N.check(L.empm_ctx_destroy(None) - 1)


def test_batch_create_rejects_bad_arguments_without_gpu():
    L = N.lib()
    out = ctypes.c_void_p()
    p = (N.EmpmModelParams * 2)()
    for q in p:
        q.n_grid, q.grid_lim = 32, 1.0
    counts = (ctypes.c_int * 2)(100, -5)
    assert L.empm_batch_create(p, counts, 2, 4, ctypes.byref(out)) == -1        # negative count
    counts[1] = 10
    assert L.empm_batch_create(p, counts, 0, 4, ctypes.byref(out)) == -1        # no instances
    p[1].n_grid = 3
    assert L.empm_batch_create(p, counts, 2, 4, ctypes.byref(out)) == -1        # bad grid in instance 1


def test_adjoint_entry_points_reject_bad_arguments_without_gpu():
    L = N.lib()
    g = N.EmpmParticles()
    gm = N.EmpmMaterialGrad()
    mat = N.EmpmMaterial()
    st = (N.EmpmStep * 1)()
    assert L.empm_adjoint_segment(None, g, None, None, None, mat, st, 1, g, gm, None) == -1
    assert "ctx" in N.last_error()
    assert L.empm_prepare_adjoint(None, None, None, None, None, None, None, None, None, -1, None) == -1
    # g_E without E / nu / g_mu / g_lam
    buf = (ctypes.c_float * 4)()
    assert L.empm_prepare_adjoint(None, None, None, None, buf, buf, None, None, None, 4, None) == -1
    # g_density without vol / g_mass
    assert L.empm_prepare_adjoint(None, None, None, None, None, None, None, None, buf, 4, None) == -1
    # nothing to do: accepted without touching the device
    assert L.empm_prepare_adjoint(None, None, None, None, None, None, None, None, None, 0, None) == 0
    p = N.EmpmModelParams()
    p.n_grid, p.grid_lim = 16, 1.0
    assert L.empm_debug_stress_adjoint(p, None, None, None, None, 0.0, None, None, None, None, None, None, 3,
                                       None) == -1


def test_option_ids_match_header():
    """Every launch option the header defines (EMPM_OPT_*) has the same id in
    the Python binding."""
    import os
    import re

    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "empm_b200.h")).read()
    opts = dict(re.findall(r"#define\s+EMPM_OPT_(\w+)\s+(\d+)", hdr))
    assert "SEGMENT_GRAPH" in opts and "FUSE" in opts
    for name, value in opts.items():
        assert getattr(N, "OPT_" + name) == int(value), name
