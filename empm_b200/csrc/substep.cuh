// substep.cuh — per-particle and per-node device code of one MLS-MPM substep.
//
// The device functions here are shared by the single-instance kernels
// (substep.cu) and the batched kernels. Formulas follow
// phys_sim/diff_simulator/warp_mpm/mpm_utils.py (line numbers cited per function).
#pragma once
#include "../../include/empm_b200.h"
#include "mat3.cuh"
#include "constitutive.cuh"

namespace empm {

// Quadratic B-spline stencil of one particle (mpm_utils.py:368-383):
// base = int(x * inv_dx - 0.5) (truncation), fx = x * inv_dx - base,
// w[axis][offset], dw[axis][offset] = dw/dfx. The three weights sum to one
// for any fx, so a base that rounds to the neighbouring node at a half-integer
// boundary changes the contributions only by O(fx error^2).
struct Stencil {
    int   b[3];
    float fx[3];
    float w[3][3];
    float dw[3][3];
};

// Base node of one coordinate: int(x * inv_dx - 0.5), with the product and the
// subtraction fused into one rounding. Every kernel derives a particle's base
// node from this function (stencils, cell keys, shared-memory tile boxes),
// so they agree bit for bit whatever the compiler does with separate
// multiply-adds.
EMPM_HD int base_node(float x, float inv_dx) { return (int)fmaf(x, inv_dx, -0.5f); }

// fx = x * inv_dx - base, rounded once.
EMPM_HD float base_frac(float x, float inv_dx, int b) { return fmaf(x, inv_dx, -(float)b); }

EMPM_HD Stencil make_stencil(V3 x, float inv_dx) {
    Stencil st;
    const float xs[3] = {x.x, x.y, x.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        st.b[a] = base_node(xs[a], inv_dx);
        const float f = base_frac(xs[a], inv_dx, st.b[a]);
        st.fx[a] = f;
        const float wa = 1.5f - f, wb = f - 1.f, wc = f - 0.5f;
        st.w[a][0] = (wa * wa) * 0.5f;
        st.w[a][1] = (0.f - wb * wb) + 0.75f;
        st.w[a][2] = (wc * wc) * 0.5f;
        st.dw[a][0] = f - 1.5f;
        st.dw[a][1] = -2.f * (f - 1.f);
        st.dw[a][2] = f - 0.5f;
    }
    return st;
}

// Quadratic B-spline weight and its derivative in fx at stencil offset i,
// formed from fx (the same expressions as make_stencil): loops over a
// run-time offset then need no table of the three weights.
EMPM_HD void bspline_at(float f, int i, float& w, float& dw) {
    if (i == 1) {
        const float x = f - 1.f;
        w = (0.f - x * x) + 0.75f;
        dw = -2.f * x;
        return;
    }
    const float t = i == 0 ? 1.5f - f : f - 0.5f;
    w = (t * t) * 0.5f;
    dw = i == 0 ? -t : t;
}

EMPM_HD bool stencil_in_grid(const Stencil& st, int G) {
    return st.b[0] >= 0 && st.b[1] >= 0 && st.b[2] >= 0 &&
           st.b[0] + 2 < G && st.b[1] + 2 < G && st.b[2] + 2 < G;
}

// Pre-P2G particle velocity modifiers (mpm_solver_diff.py:977-991, 1022-1036,
// 1098-1142, 1146-1171, 1198-1212, 1332-1348, 1391-1410). Returns true when v
// changed.
__device__ __forceinline__ bool apply_modifiers(const EmpmStep& st, int mask_index, V3 x, float mass, V3& v) {
    bool changed = false;
    const float dt = st.dt;
    for (int m = 0; m < st.n_modifiers; ++m) {
        const EmpmModifier& md = st.modifiers[m];
        if (md.gate != EMPM_GATE_APPLY) continue;
        const int mk = md.mask ? __ldg(md.mask + mask_index) : 0;
        const V3 vec = v3(md.vec[0], md.vec[1], md.vec[2]);
        switch (md.kind) {
            case EMPM_MOD_IMPULSE:
                if (mk == 1) {
                    const V3 imp = v3(vec.x / mass, vec.y / mass, vec.z / mass);
                    v = v + imp * dt;
                    changed = true;
                }
                break;
            case EMPM_MOD_IMPULSE_MASK:
                if (mk >= 1) { v = v + vec * dt; changed = true; }
                break;
            case EMPM_MOD_SET_VELOCITY:
                if (mk == 1) { v = vec; changed = true; }
                break;
            case EMPM_MOD_SET_VELOCITY_LAYERED:
                if (mk >= (int)md.scale[0]) { v = vec; changed = true; }
                break;
            case EMPM_MOD_ROTATION:
                if (mk == 1) {
                    const V3 n = v3(md.normal[0], md.normal[1], md.normal[2]);
                    const V3 a1 = v3(md.axis1[0], md.axis1[1], md.axis1[2]);
                    const V3 a2 = v3(md.axis2[0], md.axis2[1], md.axis2[2]);
                    const V3 off = x - v3(md.point[0], md.point[1], md.point[2]);
                    const float hd = length(off - dot(off, n) * n);
                    const float cosine = dot(off, a1) / hd;
                    float theta = acosf(cosine);
                    if (!(dot(off, a2) > 0.f)) theta = -theta;
                    const float s1 = -hd * sinf(theta) * md.scale[0];
                    const float s2 = hd * cosf(theta) * md.scale[0];
                    v = s1 * a1 + s2 * a2 + md.scale[1] * n;
                    changed = true;
                }
                break;
            case EMPM_MOD_MOVER:
                if (mk == 1) {
                    V3 nv = v + vec;
                    const V3 off = x - v3(md.point[0], md.point[1], md.point[2]);
                    nv = nv + md.scale[0] * cross(v3(md.normal[0], md.normal[1], md.normal[2]), off);
                    v = nv;
                    changed = true;
                }
                break;
            default: break;
        }
    }
    return changed;
}

// Grid boundary conditions for node (i, j, k), applied in registration order
// (the collide closures of mpm_solver_diff.py:473-528, 612-672, 756-793,
// 835-858, 878-935, 1275-1286). v is the node velocity after normalisation.
//
// Each collider acts on v as a diagonal projection (plus a constant). The
// recorder receives, for every collider that changed v, a code: bit a
// (a = 0, 1, 2) means component a was overwritten by a constant, and bit 3
// means the remaining components were scaled by 0.3 (surface type 11). The
// adjoint replays the sequence and applies the transposed projections in
// reverse order.
struct NoColliderRecord {
    __device__ __forceinline__ void operator()(int, unsigned) const {}
};

template <typename Rec>
__device__ __forceinline__ void apply_colliders_rec(const EmpmStep& st, int i, int j, int k, int G, float dx,
                                                    long long node, V3& v, Rec rec) {
    for (int c = 0; c < st.n_colliders; ++c) {
        const EmpmCollider& cl = st.colliders[c];
        if (cl.gate == EMPM_GATE_OFF) continue;
        if (cl.gate == EMPM_GATE_ZERO_ALL) { v = v3(0.f, 0.f, 0.f); rec(c, 7u); continue; }
        const V3 p = v3(cl.point[0], cl.point[1], cl.point[2]);
        const V3 off = v3((float)i * dx - p.x, (float)j * dx - p.y, (float)k * dx - p.z);
        switch (cl.kind) {
            case EMPM_COLL_SURFACE:
            case EMPM_COLL_GEOMETRY: {
                bool inside = false;
                int shape = (cl.kind == EMPM_COLL_SURFACE) ? EMPM_SHAPE_HALFSPACE : cl.shape;
                if (shape == EMPM_SHAPE_CUBE) {
                    inside = fabsf(off.x) < cl.size[0] && fabsf(off.y) < cl.size[1] && fabsf(off.z) < cl.size[2];
                    if (inside) { v = v3(0.f, 0.f, 0.f); rec(c, 7u); }
                } else if (shape == EMPM_SHAPE_SPHERE) {
                    if (length(off) < cl.radius) { v = v3(0.f, 0.f, 0.f); rec(c, 7u); }
                } else if (shape == EMPM_SHAPE_CYLINDER) {
                    const V3 ax = v3(cl.normal[0], cl.normal[1], cl.normal[2]);
                    const float proj = dot(off, ax);
                    const V3 radial = off - proj * ax;
                    if (fabsf(proj) < cl.half_height && length(radial) < cl.radius) {
                        v = v3(0.f, 0.f, 0.f);
                        rec(c, 7u);
                    }
                } else if (shape == EMPM_SHAPE_HALFSPACE) {
                    const V3 n = v3(cl.normal[0], cl.normal[1], cl.normal[2]);
                    if (dot(off, n) < 0.f) {
                        if (cl.surface_type == 11) {
                            const float z = (float)k * dx;
                            if (z < 0.4f || z > 0.53f) { v = v3(0.f, 0.f, 0.f); rec(c, 7u); }
                            else { v = v3(v.x, 0.f, v.z) * 0.3f; rec(c, 2u | 8u); }
                        } else {
                            // sticky, and (as in the reference) slip / separate as well:
                            // the projected velocity is computed there but zero is written.
                            v = v3(0.f, 0.f, 0.f);
                            rec(c, 7u);
                        }
                    }
                }
                break;
            }
            case EMPM_COLL_GRID_VELOCITY: {
                const V3 vset = v3(cl.velocity[0], cl.velocity[1], cl.velocity[2]) +
                                cl.angular_velocity * cross(v3(cl.rot_axis[0], cl.rot_axis[1], cl.rot_axis[2]), off);
                bool inside = false;
                if (cl.shape == EMPM_SHAPE_CUBE) {
                    inside = fabsf(off.x) < cl.size[0] && fabsf(off.y) < cl.size[1] && fabsf(off.z) < cl.size[2];
                } else if (cl.shape == EMPM_SHAPE_SPHERE) {
                    inside = length(off) < cl.radius;
                } else if (cl.shape == EMPM_SHAPE_CYLINDER) {
                    const V3 ax = v3(cl.normal[0], cl.normal[1], cl.normal[2]);
                    const float proj = dot(off, ax);
                    inside = fabsf(proj) < cl.half_height && length(off - proj * ax) < cl.radius;
                } else if (cl.shape == EMPM_SHAPE_HALFSPACE) {
                    inside = dot(off, v3(cl.normal[0], cl.normal[1], cl.normal[2])) < 0.f;
                }
                if (inside) { v = vset; rec(c, 7u); }
                break;
            }
            case EMPM_COLL_CUBOID_VELOCITY:
                if (fabsf(off.x) < cl.size[0] && fabsf(off.y) < cl.size[1] && fabsf(off.z) < cl.size[2]) {
                    v = v3(cl.velocity[0], cl.velocity[1], cl.velocity[2]);
                    rec(c, 7u);
                }
                break;
            case EMPM_COLL_BOUNDING_BOX: {
                const int pad = 3;
                unsigned code = 0;
                if (i < pad && v.x < 0.f) { v.x = 0.f; code |= 1u; }
                if (i >= G - pad && v.x > 0.f) { v.x = 0.f; code |= 1u; }
                if (j < pad && v.y < 0.f) { v.y = 0.f; code |= 2u; }
                if (j >= G - pad && v.y > 0.f) { v.y = 0.f; code |= 2u; }
                if (k < pad && v.z < 0.f) { v.z = 0.f; code |= 4u; }
                if (k >= G - pad && v.z > 0.f) { v.z = 0.f; code |= 4u; }
                if (code) rec(c, code);
                break;
            }
            case EMPM_COLL_GRID_MASK:
                if (cl.mask && __ldg(cl.mask + node) >= 1) { v = v3(0.f, 0.f, 0.f); rec(c, 7u); }
                break;
            default: break;
        }
    }
}

__device__ __forceinline__ void apply_colliders(const EmpmStep& st, int i, int j, int k, int G, float dx,
                                                long long node, V3& v) {
    apply_colliders_rec(st, i, j, k, G, dx, node, v, NoColliderRecord{});
}

// Grid normalisation, gravity and damping (mpm_utils.py:426-438, 722-734).
__device__ __forceinline__ V3 grid_velocity(float4 a, float dt, V3 g, float damping_scale) {
    V3 v = v3(0.f, 0.f, 0.f);
    if (a.w > 1e-15f) {
        const float inv = 1.f / a.w;
        v = v3(a.x, a.y, a.z) * inv;
        v = v + dt * g;
    }
    if (damping_scale < 1.f) v = v - (1.f - damping_scale) * v;
    return v;
}

// Everything P2G needs about one particle after the return map.
struct P2GParticle {
    Stencil st;
    float   wm_scale;   // particle mass
    V3      v;          // velocity (after modifiers)
    M3      Cd;         // damped affine matrix
    M3      Sv;         // -vol * stress
};

// Contribution of one particle to stencil node (i, j, k) of its stencil:
// (weight * mass) * (v + C dpos) + dt * (-vol * stress * dweight), and weight * mass
// (mpm_utils.py:385-423).
EMPM_HD float4 p2g_node(const P2GParticle& q, int i, int j, int k, float dx, float inv_dx, float dt) {
    const Stencil& st = q.st;
    const V3 dpos = v3(((float)i - st.fx[0]) * dx, ((float)j - st.fx[1]) * dx, ((float)k - st.fx[2]) * dx);
    const float weight = st.w[0][i] * st.w[1][j] * st.w[2][k];
    const V3 dweight = v3(st.dw[0][i] * st.w[1][j] * st.w[2][k],
                          st.w[0][i] * st.dw[1][j] * st.w[2][k],
                          st.w[0][i] * st.w[1][j] * st.dw[2][k]) * inv_dx;
    const float wm = weight * q.wm_scale;
    const V3 force = q.Sv * dweight;
    const V3 add = wm * (q.v + q.Cd * dpos) + dt * force;
    return make_float4(add.x, add.y, add.z, wm);
}

// Per-particle terms of the 27 P2G contributions, arranged so that each node
// costs ~20 flops:
//   (weight*mass)*(v + C dpos) + dt*(-vol*stress*dweight)
// with dpos = ((i,j,k) - fx)*dx becomes  wm*(a + i B0 + j B1 + k B2) + S (f0, f1, f2)
// where a = v - dx*C*fx, B = dx*C, S = dt*inv_dx*(-vol*stress) and
// (f0, f1, f2) = (dwx wy wz, wx dwy wz, wx wy dwz).
struct P2GPre {
    Stencil st;
    float   m;
    V3      a;
    M3      B;
    M3      S;
};

EMPM_HD P2GPre p2g_pre(const P2GParticle& q, float dx, float inv_dx, float dt) {
    P2GPre p;
    p.st = q.st;
    p.m = q.wm_scale;
    p.B = dx * q.Cd;
    const V3 fx = v3(q.st.fx[0], q.st.fx[1], q.st.fx[2]);
    p.a = q.v - p.B * fx;
    p.S = (dt * inv_dx) * q.Sv;
    return p;
}

// Calls emit(i, j, k, contribution) for the 27 stencil nodes in (i, j, k) order.
//
// The contribution of node (i, j, k) factorises over the inner axis:
//   wz_k P_ij + (k wz_k) Q_ij + dwz_k R_ij,   mass wz_k (m wx wy),
// with P_ij = m wx wy (a + i B0 + j B1) + dwx wy S0 + wx dwy S1,
// Q_ij = m wx wy B2 and R_ij = wx wy S2, formed once per stencil row: about
// 10 flops per node instead of 20.
template <typename Emit>
__device__ __forceinline__ void p2g_emit(const P2GPre& p, Emit emit) {
    const Stencil& st = p.st;
    const V3 B0 = col(p.B, 0), B1 = col(p.B, 1), B2 = col(p.B, 2);
    const V3 S0 = col(p.S, 0), S1 = col(p.S, 1), S2 = col(p.S, 2);
    // the outer axis is a loop: a third of the code of the fully unrolled 27
    // nodes, for the instruction cache (a loop over the middle axis as well
    // measured slower). The weights are formed from fx where they are used
    // rather than kept in a table: fewer live registers, fewer spills at the
    // 64-register cap of the particle kernels (population fused kernel 586 ->
    // 563 us for all three axes)
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        const V3 ai = p.a + (float)i * B0;
        float wx, dwx;
        bspline_at(st.fx[0], i, wx, dwx);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const V3 aij = j == 0 ? ai : ai + (float)j * B1;
            float wy_, dwy_;
            bspline_at(st.fx[1], j, wy_, dwy_);
            const float wxy = wx * wy_, dxy = dwx * wy_, xdy = wx * dwy_;
            const float mw = wxy * p.m;
            const V3 P = mw * aij + dxy * S0 + xdy * S1;
            const V3 Q = mw * B2;
            const V3 R = wxy * S2;
            float wz0, uz0, wz1, uz1, wz2, uz2;
            bspline_at(st.fx[2], 0, wz0, uz0);
            bspline_at(st.fx[2], 1, wz1, uz1);
            bspline_at(st.fx[2], 2, wz2, uz2);
            const float kz2 = 2.f * wz2;
            const V3 c0 = wz0 * P + uz0 * R;
            emit(i, j, 0, make_float4(c0.x, c0.y, c0.z, wz0 * mw));
            const V3 c1 = wz1 * (P + Q) + uz1 * R;
            emit(i, j, 1, make_float4(c1.x, c1.y, c1.z, wz1 * mw));
            const V3 c2 = wz2 * P + kz2 * Q + uz2 * R;
            emit(i, j, 2, make_float4(c2.x, c2.y, c2.z, wz2 * mw));
        }
    }
}

__device__ __forceinline__ M3 damp_affine(const M3& C, float rpic) {
    if (rpic < -0.001f) return m3_zero();
    return (1.f - rpic) * C + (rpic / 2.f) * (C - transpose(C));
}

__device__ __forceinline__ void red_add_v4(float4* addr, float4 val) {
    atomicAdd(addr, val);  // red.global.add.v4.f32 on sm_90+
}

// G2P gather for one particle from the node velocities (mpm_utils.py:528-576).
struct G2POut {
    V3 v;
    M3 C;
    M3 gradv;
};

// G2P gather (mpm_utils.py:528-550), rearranged so that each node costs ~25
// flops: with o = (i,j,k) and wg = weight * grid_v,
//   v = sum wg,   C = 4 inv_dx (sum wg (x) o - v (x) fx),
//   grad v = inv_dx sum grid_v (x) (dwx wy wz, wx dwy wz, wx wy dwz).
template <typename Fetch>
__device__ __forceinline__ G2POut g2p_gather(const Stencil& st, float inv_dx, Fetch fetch) {
    V3 vs = v3(0.f, 0.f, 0.f);
    V3 m0 = vs, m1 = vs, m2 = vs;      // sum wg * i, sum wg * j, sum wg * k
    V3 g0 = vs, g1 = vs, g2 = vs;      // columns of sum grid_v (x) dweight / inv_dx
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float wx = st.w[0][i], dwx = st.dw[0][i];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float wxy = wx * st.w[1][j], dxy = dwx * st.w[1][j], xdy = wx * st.dw[1][j];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const V3 g = fetch(i, j, k);
                const float wz = st.w[2][k];
                const V3 wg = (wxy * wz) * g;
                vs = vs + wg;
                if (i) m0 = m0 + (float)i * wg;
                if (j) m1 = m1 + (float)j * wg;
                if (k) m2 = m2 + (float)k * wg;
                g0 = g0 + (dxy * wz) * g;
                g1 = g1 + (xdy * wz) * g;
                g2 = g2 + (wxy * st.dw[2][k]) * g;
            }
        }
    }
    G2POut o;
    o.v = vs;
    const float c4 = 4.f * inv_dx;
    const V3 mc[3] = {m0 - st.fx[0] * vs, m1 - st.fx[1] * vs, m2 - st.fx[2] * vs};
    const V3 gc[3] = {g0, g1, g2};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            o.C.m[3 * r + c] = c4 * comp(mc[c], r);
            o.gradv.m[3 * r + c] = inv_dx * comp(gc[c], r);
        }
    return o;
}

// g2p_gather with a run-time loop over the outer stencil axis (weights formed
// from fx where they are used): a third of the code, fewer gathers in flight. The kernel that
// runs G2P and P2G back to back uses it where its size is what limits it.
template <typename Fetch>
__device__ __forceinline__ G2POut g2p_gather_rt(const Stencil& st, float inv_dx, Fetch fetch) {
    V3 vs = v3(0.f, 0.f, 0.f);
    V3 m0 = vs, m1 = vs, m2 = vs;
    V3 g0 = vs, g1 = vs, g2 = vs;
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        float wx, dwx;
        bspline_at(st.fx[0], i, wx, dwx);
        V3 si = v3(0.f, 0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float wy_, dwy_;
            bspline_at(st.fx[1], j, wy_, dwy_);
            const float wxy = wx * wy_, dxy = dwx * wy_, xdy = wx * dwy_;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const V3 g = fetch(i, j, k);
                float wz, dwz;
                bspline_at(st.fx[2], k, wz, dwz);
                const V3 wg = (wxy * wz) * g;
                si = si + wg;
                if (j) m1 = m1 + (float)j * wg;
                if (k) m2 = m2 + (float)k * wg;
                g0 = g0 + (dxy * wz) * g;
                g1 = g1 + (xdy * wz) * g;
                g2 = g2 + (wxy * dwz) * g;
            }
        }
        vs = vs + si;
        m0 = m0 + (float)i * si;
    }
    G2POut o;
    o.v = vs;
    const float c4 = 4.f * inv_dx;
    const V3 mc[3] = {m0 - st.fx[0] * vs, m1 - st.fx[1] * vs, m2 - st.fx[2] * vs};
    const V3 gc[3] = {g0, g1, g2};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            o.C.m[3 * r + c] = c4 * comp(mc[c], r);
            o.gradv.m[3 * r + c] = inv_dx * comp(gc[c], r);
        }
    return o;
}

__device__ __forceinline__ bool finite3(V3 a) {
    return isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
}

}  // namespace empm
