"""FP64 oracle fixtures for the accuracy checks at the benchmarked sizes.

TEST INFRASTRUCTURE: runs the FP64 OpenMP build of the CPU oracle
(oracle/mpm_oracle.c, itself pinned to the reference's kernels by
tests/golden/make_golden.py) over the full seeded workloads and stores what
the GPU tests in tests/test_gpu_fullsize.py compare against:

  fullsize_c2.npz  large single rollout: 500,000 plasticine particles, 128^3,
                   descending-then-lifting cuboid collider, dt=1e-4 x 1000.
                   Positions of a seeded subset of particles every 100
                   substeps (the error-growth curve) and after the last
                   substep (a larger subset); and, over ALL particles, the
                   max / mean / p99 distance between the FP32 and the FP64
                   builds of the oracle every 100 substeps (the error an
                   FP32 evaluation of the same algorithm has by itself).
  fullsize_c4.npz  batched population: 32 plasticine members (3.17M
                   particles, grids 48..128^3), dt=2e-4 x 300. Final
                   positions of a seeded subset of every member.
  fullsize_c3.npz  differentiable rollout: 200,000 particles, 96^3, dt=2e-4
                   x 400, loss = mean |x_T - x_T(target)|^2 with the target
                   material (3e4, 0.35, 2e3) and the guess (1e4, 0.25, 1e3).
                   Central finite differences (h = 1e-3 relative) of the loss
                   in E, nu, yield stress and along a seeded direction of the
                   initial velocities, in the Lame parameters mu and lam
                   separately (scaled by 1 +- h), and the FP64 residual
                   x_T - x_T(target) of every particle.

The workloads come from empm_b200.workloads (seeded numpy generators; no
GPU is involved). The oracle keeps the colliders as the reference does, in
float32 (OracleSim(collider_f32=True)): the moving cuboid of c2 has faces at
x = 0.25 and z = 0.25, exactly on the node planes i = 32 and k = 32 of the
128^3 grid, where a float64 inside test and the reference's float32 one
disagree. With float64 tests the FP32 and FP64 oracles drift apart by
2.2e-3 (max over particles) within 100 substeps; with the float32 tests, by
6e-7. Runtime on 8 host cores: about 12 min (c2), 12 min (c4)
and 10 min (c3).

    python tests/golden/make_fullsize.py [c2] [c4] [c3] [c3_residual] [c3_lame]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from empm_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import specs as OS  # noqa: E402

C2_EVERY = 100
C2_CURVE_SUBSET = 2048
C2_FINAL_SUBSET = 16384
C4_SUBSET = 512
C3_H = 1e-3
C3_DIR_SEED = 303


def subset(n: int, k: int, seed: int) -> np.ndarray:
    return np.sort(np.random.default_rng(seed).choice(n, size=min(k, n), replace=False)).astype(np.int64)


def make_c2(path: str) -> None:
    w = W.c2()
    cb = OS.workload_callback(w)
    s64 = OS.sim_from_workload(w, precision="fp64_omp", collider_f32=True)
    s32 = OS.sim_from_workload(w, precision="fp32_omp", collider_f32=True)
    curve_idx = subset(w.n, C2_CURVE_SUBSET, 2002)
    final_idx = subset(w.n, C2_FINAL_SUBSET, 2003)
    marks, curve, fp32 = [], [], []
    t0 = time.time()
    for s in range(w.T):
        cb(s64, s)
        cb(s32, s)
        s64.substep(w.dt)
        s32.substep(w.dt)
        if (s + 1) % C2_EVERY == 0:
            d = np.linalg.norm(s32.x.astype(np.float64) - s64.x, axis=1)
            marks.append(s + 1)
            curve.append(s64.x[curve_idx].astype(np.float32))
            fp32.append((d.max(), d.mean(), np.percentile(d, 99)))
            print(f"c2 substep {s + 1}: FP32 oracle vs FP64 max {d.max():.3e} mean {d.mean():.3e} "
                  f"({time.time() - t0:.0f} s)", flush=True)
    np.savez_compressed(path, marks=np.array(marks, np.int32), curve_idx=curve_idx, curve_x=np.stack(curve),
                        final_idx=final_idx, final_x=s64.x[final_idx].astype(np.float32),
                        fp32_vs_fp64=np.array(fp32, np.float64), n=w.n, T=w.T)


def oracle_member(spec, precision="fp64_omp"):
    sim = O.OracleSim(spec.x, spec.v, spec.vol, spec.rho.astype(np.float64) * spec.vol, spec.E, spec.nu,
                      n_grid=spec.n_grid, material=OS.MATERIAL_IDS[spec.material], gravity=tuple(spec.gravity),
                      yield_stress=spec.yield_stress, softening=spec.softening, precision=precision,
                      collider_f32=True)
    sim.colliders = OS.oracle_colliders(spec.colliders)
    return sim


def make_c4(path: str) -> None:
    specs, dt, T = W.c4()
    idx, xs, offs = [], [], [0]
    t0 = time.time()
    for i, spec in enumerate(specs):
        sim = oracle_member(spec)
        sim.rollout(dt, T)
        k = subset(spec.n, C4_SUBSET, 4000 + i)
        idx.append(k)
        xs.append(sim.x[k].astype(np.float32))
        offs.append(offs[-1] + len(k))
        print(f"c4 member {i}: n={spec.n} G={spec.n_grid} ({time.time() - t0:.0f} s)", flush=True)
    np.savez_compressed(path, idx=np.concatenate(idx), x=np.concatenate(xs), offsets=np.array(offs, np.int64),
                        T=T, dt=dt)


def c3_direction(n: int) -> np.ndarray:
    """Seeded direction in initial-velocity space (same scale as v0)."""
    return (np.random.default_rng(C3_DIR_SEED).standard_normal((n, 3)) * 0.05).astype(np.float32)


def c3_final(w, E=None, nu=None, ys=None, v=None, mu_scale=1.0, lam_scale=1.0) -> np.ndarray:
    sim = O.OracleSim(w.x, w.v if v is None else v, w.vol, w.rho.astype(np.float64) * w.vol,
                      w.E if E is None else E, w.nu if nu is None else nu, n_grid=w.G,
                      material=OS.MATERIAL_IDS[w.material], gravity=w.gravity,
                      yield_stress=w.ys if ys is None else ys, precision="fp64_omp", collider_f32=True)
    sim.mu *= mu_scale
    sim.lam *= lam_scale
    sim.colliders = OS.oracle_colliders(w.colliders)
    sim.rollout(w.dt, w.T)
    return sim.x


def c3_loss(w, target, **kw) -> float:
    d = c3_final(w, **kw) - target
    return float((d * d).sum(1).mean())


def c3_residual(w, target) -> np.ndarray:
    """x_T(guess) - x_T(target) of every particle in FP64, stored as float32
    (its values are about 2e-5, so float32 keeps 7 digits of it): the
    residual whose 2/N multiple is dL/dx_T."""
    return (c3_final(w) - target).astype(np.float32)


def make_c3(path: str) -> None:
    w = W.c3()
    tw = W.c3(guess=False)
    t0 = time.time()
    ts = OS.sim_from_workload(tw, precision="fp64_omp", collider_f32=True)
    ts.rollout(tw.dt, tw.T)
    target = ts.x.copy()
    residual = c3_residual(w, target)
    base = float((residual.astype(np.float64) ** 2).sum(1).mean())
    print(f"c3 target + base loss {base:.9e} ({time.time() - t0:.0f} s)", flush=True)
    E0, nu0, ys0 = float(w.E[0]), float(w.nu[0]), float(w.ys[0])
    v64 = w.v.astype(np.float64)
    d = c3_direction(w.n).astype(np.float64)
    fd, lp, lm = {}, {}, {}
    cases = {
        "E": (C3_H * E0, lambda s: dict(E=np.full(w.n, E0 + s, np.float64))),
        "nu": (C3_H * nu0, lambda s: dict(nu=np.full(w.n, nu0 + s, np.float64))),
        "yield_stress": (C3_H * ys0, lambda s: dict(ys=np.full(w.n, ys0 + s, np.float64))),
        "v0_dir": (C3_H, lambda s: dict(v=v64 + s * d)),
    }
    for name, (h, kw) in cases.items():
        lp[name] = c3_loss(w, target, **kw(h))
        lm[name] = c3_loss(w, target, **kw(-h))
        fd[name] = (lp[name] - lm[name]) / (2.0 * h)
        print(f"c3 dL/d{name} = {fd[name]:.9e} ({time.time() - t0:.0f} s)", flush=True)
    names = list(cases)
    np.savez_compressed(path, names=np.array(names), fd=np.array([fd[k] for k in names]),
                        loss_plus=np.array([lp[k] for k in names]), loss_minus=np.array([lm[k] for k in names]),
                        step=np.array([cases[k][0] for k in names]), loss=base, h=C3_H, dir_seed=C3_DIR_SEED,
                        residual=residual)
    add_c3_lame(path)


def add_c3_lame(path: str) -> None:
    """Central differences of an existing c3 fixture's loss in the Lame
    parameters separately (mu and lam scaled by 1 +- h): dL/dnu is a
    difference of the two, which these resolve one at a time."""
    w = W.c3()
    tw = W.c3(guess=False)
    ts = OS.sim_from_workload(tw, precision="fp64_omp", collider_f32=True)
    ts.rollout(tw.dt, tw.T)
    target = ts.x.copy()
    old = dict(np.load(path))
    for name in ("mu", "lam"):
        kw = lambda sc: {f"{name}_scale": sc}  # noqa: E731
        lp = c3_loss(w, target, **kw(1.0 + C3_H))
        lm = c3_loss(w, target, **kw(1.0 - C3_H))
        old[f"fd_log_{name}"] = np.float64((lp - lm) / (2.0 * C3_H))
        print(f"c3 dL/dlog({name}) = {old[f'fd_log_{name}']:.9e}", flush=True)
    np.savez_compressed(path, **old)


def add_c3_residual(path: str) -> None:
    """Recompute only the FP64 residual of an existing c3 fixture."""
    w = W.c3()
    tw = W.c3(guess=False)
    ts = OS.sim_from_workload(tw, precision="fp64_omp", collider_f32=True)
    ts.rollout(tw.dt, tw.T)
    old = dict(np.load(path))
    old.pop("target_subset_idx", None)
    old.pop("target_subset_x", None)
    old["residual"] = c3_residual(w, ts.x.copy())
    np.savez_compressed(path, **old)


def main(argv) -> None:
    O.build()
    jobs = argv or ["c2", "c4", "c3"]
    make = {"c2": make_c2, "c4": make_c4, "c3": make_c3, "c3_residual": add_c3_residual, "c3_lame": add_c3_lame}
    for j in jobs:
        make[j](os.path.join(HERE, f"fullsize_{j.split('_')[0]}.npz"))


if __name__ == "__main__":
    main(sys.argv[1:])
