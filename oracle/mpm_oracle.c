/*
 * mpm_oracle.c — CPU restatement of EMPM's MLS-MPM substep.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA library and
 * the timed CPU baseline; nothing in the product links or calls it.
 *
 * Built twice by oracle/build_oracle.sh:
 *   liboracle64.so      OR_REAL=double, sequential (the FP64 oracle)
 *   liboracle32_omp.so  OR_REAL=float, OpenMP over particles / nodes, grid
 *                       scatter with atomics (the CPU baseline)
 *
 * Follows, statement by statement, the reference (paths in the EMPM repo):
 *   stage order            phys_sim/diff_simulator/warp_mpm/mpm_solver_diff.py:165-291
 *   return maps / stresses mpm_utils.py:8-84, 87-274, 602-665
 *   mu, lam from E, nu     mpm_utils.py:277-283
 *   P2G                    mpm_utils.py:358-423 (+ compute_dweight :294-303)
 *   grid normalisation     mpm_utils.py:426-438, damping :722-734
 *   colliders              mpm_solver_diff.py:473-528, 612-672, 756-793, 835-858, 878-935, 1275-1286
 *   particle modifiers     mpm_solver_diff.py:977-991, 1022-1036, 1098-1142, 1198-1212, 1332-1348, 1391-1410
 *   G2P                    mpm_utils.py:502-579
 * The reference's wp.svd3 (Warp builtin, not in the repository) is restated
 * as a one-sided Jacobi SVD iterated to convergence, with U, V proper
 * rotations and the sign of det(A) on the last singular value.
 */
#include <math.h>
#include <string.h>
#include <stdlib.h>

#ifndef OR_REAL
#define OR_REAL double
#endif
typedef OR_REAL real;

#ifdef _OPENMP
#include <omp.h>
#define OR_PARALLEL_FOR _Pragma("omp parallel for schedule(static)")
#define OR_ATOMIC _Pragma("omp atomic")
#else
#define OR_PARALLEL_FOR
#define OR_ATOMIC
#endif

typedef struct {
    int  G;
    real grid_lim, dx, inv_dx;
    int  material;
    real gravity[3];
    real rpic_damping, grid_v_damping_scale;
    real softening, hardening, xi, plastic_viscosity, alpha;
    /* 1: the colliders' inside tests are evaluated as the reference's Warp
     * kernels evaluate them, on float32 offsets float(i) * dx - point and
     * float32 extents (mpm_solver_diff.py:612-672, 756-793, 835-858). A node
     * plane can lie exactly on a collider face (x = 0.25 for a face at
     * 0.30 - 0.05), and there the float32 and float64 tests disagree. */
    int  pred32;
} OrModel;

/* gate: 0 off, 1 apply, 2 zero every node (same meaning as the library) */
typedef struct {
    int  kind, gate, shape, surface_type;
    real point[3], normal[3], size[3], velocity[3], rot_axis[3];
    real angular_velocity, radius, half_height, friction;
    const int* mask;
} OrCollider;

typedef struct {
    int  kind, gate;
    real vec[3], point[3], normal[3], axis1[3], axis2[3], scale[2];
    const int* mask;
} OrModifier;

/* ---------------- 3x3 helpers (row-major) ---------------- */
static void mm(const real* a, const real* b, real* c) {
    real t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            t[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
    memcpy(c, t, sizeof(t));
}
static void mt(const real* a, real* b) {
    real t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[3 * i + j] = a[3 * j + i];
    memcpy(b, t, sizeof(t));
}
static real mdet(const real* a) {
    return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) + a[2] * (a[3] * a[7] - a[4] * a[6]);
}
static real len3(const real* v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
static real dot3(const real* a, const real* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void cross3(const real* a, const real* b, real* c) {
    real t[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    c[0] = t[0]; c[1] = t[1]; c[2] = t[2];
}
static real rmax(real a, real b) { return a > b ? a : b; }
static real rmin(real a, real b) { return a < b ? a : b; }

/* U diag(s) V^T */
static void usvt(const real* U, const real* s, const real* V, real* out) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            out[3 * i + j] = U[3 * i] * s[0] * V[3 * j] + U[3 * i + 1] * s[1] * V[3 * j + 1] + U[3 * i + 2] * s[2] * V[3 * j + 2];
}

/* One-sided Jacobi SVD. A = U diag(s) V^T, U,V in SO(3), s0>=s1>=|s2|. */
void or_svd3(const real* A, real* U, real* s, real* V) {
    real b[3][3], v[3][3]; /* columns */
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) { b[c][r] = A[3 * r + c]; v[c][r] = (r == c); }
    const real tol = (sizeof(real) == 8) ? 1e-15 : 1e-7;
    for (int sweep = 0; sweep < 60; ++sweep) {
        int rotated = 0;
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            real al = 0, be = 0, ga = 0;
            for (int r = 0; r < 3; ++r) { al += b[p][r] * b[p][r]; be += b[q][r] * b[q][r]; ga += b[p][r] * b[q][r]; }
            if (fabs(ga) <= tol * sqrt(al * be) || ga == 0) continue;
            rotated = 1;
            const real zeta = (be - al) / (2 * ga);
            const real t = (zeta >= 0 ? 1 : -1) / (fabs(zeta) + sqrt(1 + zeta * zeta));
            const real c = 1 / sqrt(1 + t * t), sn = c * t;
            for (int r = 0; r < 3; ++r) {
                real bp = b[p][r], bq = b[q][r];
                b[p][r] = c * bp - sn * bq; b[q][r] = sn * bp + c * bq;
                real vp = v[p][r], vq = v[q][r];
                v[p][r] = c * vp - sn * vq; v[q][r] = sn * vp + c * vq;
            }
        }
        if (!rotated) break;
    }
    real nrm[3];
    for (int c = 0; c < 3; ++c) nrm[c] = len3(b[c]);
    /* selection sort by norm, descending */
    for (int i = 0; i < 2; ++i)
        for (int j = i + 1; j < 3; ++j)
            if (nrm[j] > nrm[i]) {
                real t = nrm[i]; nrm[i] = nrm[j]; nrm[j] = t;
                for (int r = 0; r < 3; ++r) {
                    t = b[i][r]; b[i][r] = b[j][r]; b[j][r] = t;
                    t = v[i][r]; v[i][r] = v[j][r]; v[j][r] = t;
                }
            }
    real Vm[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) Vm[3 * r + c] = v[c][r];
    if (mdet(Vm) < 0) {
        for (int r = 0; r < 3; ++r) { v[2][r] = -v[2][r]; b[2][r] = -b[2][r]; Vm[3 * r + 2] = -Vm[3 * r + 2]; }
    }
    /* U columns: u0 = b0/|b0|, u1 = b1/|b1| (made orthogonal), u2 = u0 x u1 */
    real u[3][3];
    const real tiny = (sizeof(real) == 8) ? 1e-300 : 1e-30f;
    if (nrm[0] > tiny) { for (int r = 0; r < 3; ++r) u[0][r] = b[0][r] / nrm[0]; }
    else { u[0][0] = 1; u[0][1] = 0; u[0][2] = 0; }
    real proj = dot3(b[1], u[0]);
    real w[3] = {b[1][0] - proj * u[0][0], b[1][1] - proj * u[0][1], b[1][2] - proj * u[0][2]};
    real wl = len3(w);
    if (wl > tiny && wl > 1e-12 * nrm[0]) { for (int r = 0; r < 3; ++r) u[1][r] = w[r] / wl; }
    else {
        /* any unit vector orthogonal to u0 */
        real e[3] = {0, 0, 0};
        int k = fabs(u[0][0]) < fabs(u[0][1]) ? (fabs(u[0][0]) < fabs(u[0][2]) ? 0 : 2) : (fabs(u[0][1]) < fabs(u[0][2]) ? 1 : 2);
        e[k] = 1;
        real pe = dot3(e, u[0]);
        for (int r = 0; r < 3; ++r) w[r] = e[r] - pe * u[0][r];
        wl = len3(w);
        for (int r = 0; r < 3; ++r) u[1][r] = w[r] / wl;
    }
    cross3(u[0], u[1], u[2]);
    s[0] = dot3(b[0], u[0]);
    s[1] = dot3(b[1], u[1]);
    s[2] = dot3(b[2], u[2]);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) { U[3 * r + c] = u[c][r]; V[3 * r + c] = Vm[3 * r + c]; }
}

/* ---------------- constitutive models ---------------- */

/* returns 1 if F changed; s is updated to the singular values of F_e */
static int or_von_mises(const real* U, real* s, const real* V, real* mu, real* lam, real* ys,
                        const OrModel* m, int damage, real* Fe) {
    real sig[3], eps[3], tau[3], cond[3];
    for (int i = 0; i < 3; ++i) { sig[i] = rmax(s[i], 0.01); eps[i] = log(sig[i]); }
    const real temp = (eps[0] + eps[1] + eps[2]) / 3.0;
    for (int i = 0; i < 3; ++i) tau[i] = 2.0 * (*mu) * eps[i] + (*lam) * (eps[0] + eps[1] + eps[2]);
    const real sum_tau = tau[0] + tau[1] + tau[2];
    for (int i = 0; i < 3; ++i) cond[i] = tau[i] - sum_tau / 3.0;
    if (!(len3(cond) > *ys)) return 0;
    if (damage && *ys <= 0) return 0;
    real eh[3];
    for (int i = 0; i < 3; ++i) eh[i] = eps[i] - temp;
    const real ehn = len3(eh) + 1e-6;
    const real dg = ehn - *ys / (2.0 * (*mu));
    for (int i = 0; i < 3; ++i) eps[i] = eps[i] - (dg / ehn) * eh[i];
    if (damage) {
        real d[3] = {(dg / ehn) * eh[0], (dg / ehn) * eh[1], (dg / ehn) * eh[2]};
        *ys = *ys - m->softening * len3(d);
        if (*ys <= 0) { *mu = 0; *lam = 0; }
    }
    for (int i = 0; i < 3; ++i) s[i] = exp(eps[i]);
    usvt(U, s, V, Fe);
    if (m->hardening == 1) *ys = *ys + 2.0 * (*mu) * m->xi * dg;
    return 1;
}

static int or_sand(const real* U, real* s, const real* V, real mu, real lam, const OrModel* m, real* Fe) {
    real eps[3], eh[3];
    for (int i = 0; i < 3; ++i) eps[i] = log(rmax(fabs(s[i]), 1e-14));
    const real tr = eps[0] + eps[1] + eps[2];
    for (int i = 0; i < 3; ++i) eh[i] = eps[i] - tr / 3.0;
    const real ehn = len3(eh);
    const real dg = ehn + (3.0 * lam + 2.0 * mu) / (2.0 * mu) * tr * m->alpha;
    if (dg <= 0) return 0;
    if (tr > 0) { s[0] = s[1] = s[2] = 1.0; }
    else { for (int i = 0; i < 3; ++i) s[i] = exp(eps[i] - eh[i] * (dg / ehn)); }
    usvt(U, s, V, Fe);
    return 1;
}

static int or_visco(const real* U, real* s, const real* V, real mu, real ys, real dt, const OrModel* m, real* Fe) {
    real sig[3], b[3], eps[3], eh[3], st[3];
    for (int i = 0; i < 3; ++i) { sig[i] = rmax(s[i], 0.01); b[i] = sig[i] * sig[i]; eps[i] = log(sig[i]); }
    const real tr = eps[0] + eps[1] + eps[2];
    for (int i = 0; i < 3; ++i) { eh[i] = eps[i] - tr / 3.0; st[i] = 2.0 * mu * eh[i]; }
    const real stn = len3(st);
    const real y = stn - sqrt(2.0 / 3.0) * ys;
    if (!(y > 0)) return 0;
    const real mu_hat = mu * (b[0] + b[1] + b[2]) / 3.0;
    const real snn = stn - y / (1.0 + m->plastic_viscosity / (2.0 * mu_hat * dt));
    for (int i = 0; i < 3; ++i) s[i] = exp(1.0 / (2.0 * mu) * ((snn / stn) * st[i]) + tr / 3.0);
    usvt(U, s, V, Fe);
    return 1;
}

/* stress kernel for one particle (compute_stress_from_F_trial) */
static void or_particle_stress(const OrModel* m, const real* Ft, real* mu, real* lam, real* ys, real dt,
                               real* F, real* stress) {
    real U[9], V[9], s[3];
    or_svd3(Ft, U, s, V);
    memcpy(F, Ft, 9 * sizeof(real));
    switch (m->material) {
        case 1: or_von_mises(U, s, V, mu, lam, ys, m, 0, F); break;
        case 2: or_sand(U, s, V, *mu, *lam, m, F); break;
        case 3: or_visco(U, s, V, *mu, *ys, dt, m, F); break;
        case 5: or_von_mises(U, s, V, mu, lam, ys, m, 1, F); break;
        default: break;
    }
    const real J = mdet(F);
    real tau[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    real Ft_[9];
    mt(F, Ft_);
    if (m->material == 0 || m->material == 5) {
        real R[9], Vt[9], D[9];
        mt(V, Vt);
        mm(U, Vt, R);
        for (int i = 0; i < 9; ++i) D[i] = F[i] - R[i];
        mm(D, Ft_, tau);
        for (int i = 0; i < 9; ++i) tau[i] *= 2.0 * (*mu);
        for (int i = 0; i < 3; ++i) tau[4 * i] += (*lam) * J * (J - 1.0);
    } else if (m->material == 1 || m->material == 3) {
        real sg[3], d[3], M[9];
        for (int i = 0; i < 3; ++i) sg[i] = rmax(s[i], 0.01);
        const real ls = log(sg[0]) + log(sg[1]) + log(sg[2]);
        for (int i = 0; i < 3; ++i) d[i] = 2.0 * (*mu) * log(sg[i]) + (*lam) * ls;
        usvt(U, d, V, M);
        mm(M, Ft_, tau);
    } else if (m->material == 2) {
        real d[3], M[9];
        const real ls = log(s[0]) + log(s[1]) + log(s[2]);
        for (int i = 0; i < 3; ++i) d[i] = 2.0 * (*mu) * log(s[i]) * (1.0 / s[i]) + (*lam) * ls * (1.0 / s[i]);
        usvt(U, d, V, M);
        mm(M, Ft_, tau);
    } else if (m->material == 6) {
        real b[3], d[3], M[9];
        for (int i = 0; i < 3; ++i) b[i] = s[i] * s[i];
        const real bm = (b[0] + b[1] + b[2]) / 3.0;
        for (int i = 0; i < 3; ++i) d[i] = (*mu) * pow(J, -2.0 / 3.0) * (b[i] - bm) + (*lam) / 2.0 * (J * J - 1.0);
        usvt(U, d, V, M);
        mm(M, Ft_, tau);
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) stress[3 * i + j] = (tau[3 * i + j] + tau[3 * j + i]) / 2.0;
}

void or_stress(const OrModel* m, int n, const int* sel, const real* F_trial, real* mu, real* lam, real* ys,
               real dt, real* F, real* stress) {
    OR_PARALLEL_FOR
    for (int p = 0; p < n; ++p) {
        if (sel && sel[p] != 0) continue;
        or_particle_stress(m, F_trial + 9 * p, mu + p, lam + p, ys + p, dt, F + 9 * p, stress + 9 * p);
    }
}

void or_mu_lam(int n, const real* E, const real* nu, real* mu, real* lam) {
    for (int p = 0; p < n; ++p) {
        mu[p] = E[p] / (2.0 * (1.0 + nu[p]));
        lam[p] = E[p] * nu[p] / ((1.0 + nu[p]) * (1.0 - 2.0 * nu[p]));
    }
}

/* quadratic B-spline weights */
static void or_stencil(const real* x, real inv_dx, int* base, real* fx, real w[3][3], real dw[3][3]) {
    for (int a = 0; a < 3; ++a) {
        const real gp = x[a] * inv_dx;
        base[a] = (int)(gp - 0.5);
        fx[a] = gp - (real)base[a];
        const real wa = 1.5 - fx[a], wb = fx[a] - 1.0, wc = fx[a] - 0.5;
        w[a][0] = wa * wa * 0.5;
        w[a][1] = 0.0 - wb * wb + 0.75;
        w[a][2] = wc * wc * 0.5;
        dw[a][0] = fx[a] - 1.5;
        dw[a][1] = -2.0 * (fx[a] - 1.0);
        dw[a][2] = fx[a] - 0.5;
    }
}

void or_modifiers(int n, const OrModifier* mods, int nm, real dt, const real* x, const real* mass, real* v) {
    for (int k = 0; k < nm; ++k) {
        const OrModifier* md = mods + k;
        if (md->gate != 1) continue;
        OR_PARALLEL_FOR
        for (int p = 0; p < n; ++p) {
            const int mk = md->mask ? md->mask[p] : 0;
            real* vp = v + 3 * p;
            if (md->kind == 1 && mk == 1) {
                for (int i = 0; i < 3; ++i) vp[i] = vp[i] + (md->vec[i] / mass[p]) * dt;
            } else if (md->kind == 2 && mk >= 1) {
                for (int i = 0; i < 3; ++i) vp[i] = vp[i] + md->vec[i] * dt;
            } else if (md->kind == 3 && mk == 1) {
                for (int i = 0; i < 3; ++i) vp[i] = md->vec[i];
            } else if (md->kind == 4 && mk == 1) {
                real off[3], h[3];
                for (int i = 0; i < 3; ++i) off[i] = x[3 * p + i] - md->point[i];
                const real dn = dot3(off, md->normal);
                for (int i = 0; i < 3; ++i) h[i] = off[i] - dn * md->normal[i];
                const real hd = len3(h);
                const real cosine = dot3(off, md->axis1) / hd;
                real theta = acos(cosine);
                if (!(dot3(off, md->axis2) > 0)) theta = -theta;
                const real s1 = -hd * sin(theta) * md->scale[0];
                const real s2 = hd * cos(theta) * md->scale[0];
                for (int i = 0; i < 3; ++i) vp[i] = s1 * md->axis1[i] + s2 * md->axis2[i] + md->scale[1] * md->normal[i];
            } else if (md->kind == 5 && mk == 1) {
                real off[3], c[3];
                for (int i = 0; i < 3; ++i) off[i] = x[3 * p + i] - md->point[i];
                cross3(md->normal, off, c);
                for (int i = 0; i < 3; ++i) vp[i] = vp[i] + md->vec[i] + md->scale[0] * c[i];
            }
        }
    }
}

/* grid_m [G^3], grid_v_in [G^3*3] accumulate (caller zeroes) */
void or_p2g(const OrModel* m, int n, const int* sel, const real* x, const real* v, const real* C,
            const real* stress, const real* vol, const real* mass, real dt, real* grid_m, real* grid_v_in) {
    const int G = m->G;
    OR_PARALLEL_FOR
    for (int p = 0; p < n; ++p) {
        if (sel && sel[p] != 0) continue;
        int base[3];
        real fx[3], w[3][3], dw[3][3];
        or_stencil(x + 3 * p, m->inv_dx, base, fx, w, dw);
        const real* Cp = C + 9 * p;
        real Cd[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                Cd[3 * i + j] = (1.0 - m->rpic_damping) * Cp[3 * i + j] + m->rpic_damping / 2.0 * (Cp[3 * i + j] - Cp[3 * j + i]);
        if (m->rpic_damping < -0.001) memset(Cd, 0, sizeof(Cd));
        const real* S = stress + 9 * p;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    const int ix = base[0] + i, iy = base[1] + j, iz = base[2] + k;
                    if (ix < 0 || iy < 0 || iz < 0 || ix >= G || iy >= G || iz >= G) continue;
                    const real dpos[3] = {(i - fx[0]) * m->dx, (j - fx[1]) * m->dx, (k - fx[2]) * m->dx};
                    const real weight = w[0][i] * w[1][j] * w[2][k];
                    const real dwt[3] = {dw[0][i] * w[1][j] * w[2][k] * m->inv_dx,
                                         w[0][i] * dw[1][j] * w[2][k] * m->inv_dx,
                                         w[0][i] * w[1][j] * dw[2][k] * m->inv_dx};
                    const long long node = ((long long)ix * G + iy) * G + iz;
                    for (int r = 0; r < 3; ++r) {
                        const real cdp = Cd[3 * r] * dpos[0] + Cd[3 * r + 1] * dpos[1] + Cd[3 * r + 2] * dpos[2];
                        const real force = -vol[p] * (S[3 * r] * dwt[0] + S[3 * r + 1] * dwt[1] + S[3 * r + 2] * dwt[2]);
                        const real add = weight * mass[p] * (v[3 * p + r] + cdp) + dt * force;
                        OR_ATOMIC
                        grid_v_in[3 * node + r] += add;
                    }
                    OR_ATOMIC
                    grid_m[node] += weight * mass[p];
                }
    }
}

static int inside_shape(int shape, const real* off, const OrCollider* c) {
    if (shape == 1) return fabs(off[0]) < c->size[0] && fabs(off[1]) < c->size[1] && fabs(off[2]) < c->size[2];
    if (shape == 2) return len3(off) < c->radius;
    if (shape == 3) {
        const real proj = dot3(off, c->normal);
        real rad[3] = {off[0] - proj * c->normal[0], off[1] - proj * c->normal[1], off[2] - proj * c->normal[2]};
        return fabs(proj) < c->half_height && len3(rad) < c->radius;
    }
    if (shape == 4) return dot3(off, c->normal) < 0;
    return 0;
}

/* inside_shape on float32 offsets and extents (OrModel.pred32) */
static int inside_shape_f32(int shape, const float* off, const OrCollider* c) {
    if (shape == 1)
        return fabsf(off[0]) < (float)c->size[0] && fabsf(off[1]) < (float)c->size[1] &&
               fabsf(off[2]) < (float)c->size[2];
    const float nrm[3] = {(float)c->normal[0], (float)c->normal[1], (float)c->normal[2]};
    if (shape == 2) return sqrtf(off[0] * off[0] + off[1] * off[1] + off[2] * off[2]) < (float)c->radius;
    if (shape == 3) {
        const float proj = off[0] * nrm[0] + off[1] * nrm[1] + off[2] * nrm[2];
        const float rad[3] = {off[0] - proj * nrm[0], off[1] - proj * nrm[1], off[2] - proj * nrm[2]};
        return fabsf(proj) < (float)c->half_height &&
               sqrtf(rad[0] * rad[0] + rad[1] * rad[1] + rad[2] * rad[2]) < (float)c->radius;
    }
    if (shape == 4) return off[0] * nrm[0] + off[1] * nrm[1] + off[2] * nrm[2] < 0.0f;
    return 0;
}

static int collider_inside(const OrModel* m, int shape, const real* off, const float* off32, const OrCollider* c) {
    return m->pred32 ? inside_shape_f32(shape, off32, c) : inside_shape(shape, off, c);
}

/* grid_normalization_and_gravity + damping + colliders; grid_v_out is zeroed by the caller */
void or_grid_update(const OrModel* m, const real* grid_m, const real* grid_v_in, real* grid_v_out,
                    const OrCollider* coll, int nc, real dt) {
    const int G = m->G;
    const long long total = (long long)G * G * G;
    OR_PARALLEL_FOR
    for (long long node = 0; node < total; ++node) {
        real* vo = grid_v_out + 3 * node;
        if (grid_m[node] > 1e-15) {
            const real inv = 1.0 / grid_m[node];
            for (int r = 0; r < 3; ++r) vo[r] = grid_v_in[3 * node + r] * inv + dt * m->gravity[r];
        }
        if (m->grid_v_damping_scale < 1.0)
            for (int r = 0; r < 3; ++r) vo[r] = vo[r] - (1.0 - m->grid_v_damping_scale) * vo[r];
        const int i = (int)(node / ((long long)G * G)), j = (int)((node / G) % G), k = (int)(node % G);
        for (int c = 0; c < nc; ++c) {
            const OrCollider* cl = coll + c;
            if (cl->gate == 0) continue;
            if (cl->gate == 2) { vo[0] = vo[1] = vo[2] = 0; continue; }
            const real off[3] = {(real)i * m->dx - cl->point[0], (real)j * m->dx - cl->point[1], (real)k * m->dx - cl->point[2]};
            const float dx32 = (float)m->dx;
            const float off32[3] = {(float)i * dx32 - (float)cl->point[0], (float)j * dx32 - (float)cl->point[1],
                                    (float)k * dx32 - (float)cl->point[2]};
            if (cl->kind == 1 || cl->kind == 2) {
                const int shape = cl->kind == 1 ? 4 : cl->shape;
                if (shape == 4) {
                    if (collider_inside(m, 4, off, off32, cl)) {
                        if (cl->surface_type == 11) {
                            const real z = (real)k * m->dx;
                            if (z < 0.4 || z > 0.53) { vo[0] = vo[1] = vo[2] = 0; }
                            else { vo[0] = vo[0] * 0.3; vo[1] = 0; vo[2] = vo[2] * 0.3; }
                        } else {
                            vo[0] = vo[1] = vo[2] = 0;
                        }
                    }
                } else if (collider_inside(m, shape, off, off32, cl)) {
                    vo[0] = vo[1] = vo[2] = 0;
                }
            } else if (cl->kind == 3) {
                if (collider_inside(m, cl->shape, off, off32, cl)) {
                    real c3[3];
                    cross3(cl->rot_axis, off, c3);
                    for (int r = 0; r < 3; ++r) vo[r] = cl->velocity[r] + cl->angular_velocity * c3[r];
                }
            } else if (cl->kind == 4) {
                if (collider_inside(m, 1, off, off32, cl))
                    for (int r = 0; r < 3; ++r) vo[r] = cl->velocity[r];
            } else if (cl->kind == 5) {
                const int pad = 3;
                if (i < pad && vo[0] < 0) vo[0] = 0;
                if (i >= G - pad && vo[0] > 0) vo[0] = 0;
                if (j < pad && vo[1] < 0) vo[1] = 0;
                if (j >= G - pad && vo[1] > 0) vo[1] = 0;
                if (k < pad && vo[2] < 0) vo[2] = 0;
                if (k >= G - pad && vo[2] > 0) vo[2] = 0;
            } else if (cl->kind == 6) {
                if (cl->mask && cl->mask[node] >= 1) { vo[0] = vo[1] = vo[2] = 0; }
            }
        }
    }
}

/* g2p_differentiable: writes the new state. Unsimulated particles get the
 * freshly-cloned values (x = v = C = 0, F_trial = I). */
void or_g2p(const OrModel* m, int n, const int* sel, const real* x, const real* F, const real* grid_v_out, real dt,
            real* x1, real* v1, real* C1, real* Ft1) {
    const int G = m->G;
    OR_PARALLEL_FOR
    for (int p = 0; p < n; ++p) {
        if (sel && sel[p] != 0) {
            for (int r = 0; r < 3; ++r) { x1[3 * p + r] = 0; v1[3 * p + r] = 0; }
            for (int r = 0; r < 9; ++r) { C1[9 * p + r] = 0; Ft1[9 * p + r] = (r % 4 == 0); }
            continue;
        }
        int base[3];
        real fx[3], w[3][3], dw[3][3];
        or_stencil(x + 3 * p, m->inv_dx, base, fx, w, dw);
        real nv[3] = {0, 0, 0}, nC[9], nF[9];
        memset(nC, 0, sizeof(nC));
        memset(nF, 0, sizeof(nF));
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    const int ix = base[0] + i, iy = base[1] + j, iz = base[2] + k;
                    if (ix < 0 || iy < 0 || iz < 0 || ix >= G || iy >= G || iz >= G) continue;
                    const real dpos[3] = {i - fx[0], j - fx[1], k - fx[2]};
                    const real weight = w[0][i] * w[1][j] * w[2][k];
                    const real* gv = grid_v_out + 3 * (((long long)ix * G + iy) * G + iz);
                    const real dwt[3] = {dw[0][i] * w[1][j] * w[2][k] * m->inv_dx,
                                         w[0][i] * dw[1][j] * w[2][k] * m->inv_dx,
                                         w[0][i] * w[1][j] * dw[2][k] * m->inv_dx};
                    for (int r = 0; r < 3; ++r) {
                        nv[r] = nv[r] + gv[r] * weight;
                        for (int c = 0; c < 3; ++c) {
                            nC[3 * r + c] = nC[3 * r + c] + gv[r] * dpos[c] * (weight * m->inv_dx * 4.0);
                            nF[3 * r + c] = nF[3 * r + c] + gv[r] * dwt[c];
                        }
                    }
                }
        const real dx = 1.0 / m->inv_dx;
        const real lo = dx * 2.0, hi = m->grid_lim - dx * 2.0;
        for (int r = 0; r < 3; ++r) {
            v1[3 * p + r] = nv[r];
            x1[3 * p + r] = rmin(rmax(x[3 * p + r] + dt * nv[r], lo), hi);
        }
        memcpy(C1 + 9 * p, nC, sizeof(nC));
        real A[9];
        for (int r = 0; r < 9; ++r) A[r] = (r % 4 == 0) + nF[r] * dt;
        mm(A, F + 9 * p, Ft1 + 9 * p);
    }
}

/* Full substep in the reference's launch order. grid buffers are scratch of
 * G^3, 3 G^3 and 3 G^3 reals; F and stress receive the old state's outputs. */
void or_substep(const OrModel* m, int n, const int* sel, real* mu, real* lam, real* ys, const real* vol,
                const real* mass, const real* x, real* v, const real* C, const real* Ft, real* F, real* stress,
                real* x1, real* v1, real* C1, real* Ft1, real* grid_m, real* grid_v_in, real* grid_v_out,
                const OrCollider* coll, int nc, const OrModifier* mods, int nm, real dt) {
    const long long g3 = (long long)m->G * m->G * m->G;
    memset(grid_m, 0, sizeof(real) * g3);
    memset(grid_v_in, 0, sizeof(real) * 3 * g3);
    memset(grid_v_out, 0, sizeof(real) * 3 * g3);
    or_modifiers(n, mods, nm, dt, x, mass, v);
    or_stress(m, n, sel, Ft, mu, lam, ys, dt, F, stress);
    or_p2g(m, n, sel, x, v, C, stress, vol, mass, dt, grid_m, grid_v_in);
    or_grid_update(m, grid_m, grid_v_in, grid_v_out, coll, nc, dt);
    or_g2p(m, n, sel, x, F, grid_v_out, dt, x1, v1, C1, Ft1);
}

/* MPMWARPDiff.restart_and_compute_F_C (mpm_solver_diff.py:1214-1262): the
 * displacement target - x is scattered to the grid with weight * mass
 * (set_F_C_p2g, mpm_utils.py:836-866), normalised by the grid mass
 * (grid_normalization_and_gravity with dt = 0, :426-438) and gathered back as
 * F_trial = I + sum grid_v (x) dweight (set_F_C_g2p, :869-919); every x then
 * becomes its target (set_vec3_to_vec3). C is not touched. Nodes outside the
 * grid are skipped. grid_m / grid_v: scratch of G^3 / 3 G^3 reals. */
/* cov (optional, packed c00 c01 c02 c11 c12 c22 per particle): update_cov
 * with the displacement gradient and dt = 1 (mpm_utils.py:306-326, 918-919). */
void or_restart(const OrModel* m, int n, const int* sel, real* x, const real* mass, const real* target, real* Ft,
                real* grid_m, real* grid_v, real* cov) {
    const int G = m->G;
    const long long g3 = (long long)G * G * G;
    memset(grid_m, 0, sizeof(real) * g3);
    memset(grid_v, 0, sizeof(real) * 3 * g3);
    for (int p = 0; p < n; ++p) {
        if (sel && sel[p] != 0) continue;
        int base[3];
        real fx[3], w[3][3], dw[3][3];
        or_stencil(x + 3 * p, m->inv_dx, base, fx, w, dw);
        const real disp[3] = {target[3 * p] - x[3 * p], target[3 * p + 1] - x[3 * p + 1],
                              target[3 * p + 2] - x[3 * p + 2]};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    const int ix = base[0] + i, iy = base[1] + j, iz = base[2] + k;
                    if (ix < 0 || iy < 0 || iz < 0 || ix >= G || iy >= G || iz >= G) continue;
                    const real weight = w[0][i] * w[1][j] * w[2][k];
                    const long long node = ((long long)ix * G + iy) * G + iz;
                    for (int r = 0; r < 3; ++r) grid_v[3 * node + r] += weight * mass[p] * disp[r];
                    grid_m[node] += weight * mass[p];
                }
    }
    for (long long node = 0; node < g3; ++node) {
        if (grid_m[node] > 1e-15) {
            for (int r = 0; r < 3; ++r) grid_v[3 * node + r] = grid_v[3 * node + r] / grid_m[node];
        }
    }
    for (int p = 0; p < n; ++p) {
        if (sel && sel[p] != 0) continue;
        int base[3];
        real fx[3], w[3][3], dw[3][3];
        or_stencil(x + 3 * p, m->inv_dx, base, fx, w, dw);
        real nF[9];
        memset(nF, 0, sizeof(nF));
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    const int ix = base[0] + i, iy = base[1] + j, iz = base[2] + k;
                    if (ix < 0 || iy < 0 || iz < 0 || ix >= G || iy >= G || iz >= G) continue;
                    const real* gv = grid_v + 3 * (((long long)ix * G + iy) * G + iz);
                    const real dwt[3] = {dw[0][i] * w[1][j] * w[2][k] * m->inv_dx,
                                         w[0][i] * dw[1][j] * w[2][k] * m->inv_dx,
                                         w[0][i] * w[1][j] * dw[2][k] * m->inv_dx};
                    for (int r = 0; r < 3; ++r)
                        for (int c = 0; c < 3; ++c) nF[3 * r + c] += gv[r] * dwt[c];
                }
        for (int r = 0; r < 9; ++r) Ft[9 * p + r] = (r % 4 == 0) + nF[r];
        if (cov) {
            real* c = cov + 6 * p;
            const real S[9] = {c[0], c[1], c[2], c[1], c[3], c[4], c[2], c[4], c[5]};
            real N[9];
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) {
                    real gs = 0, sg = 0;
                    for (int t = 0; t < 3; ++t) {
                        gs += nF[3 * r + t] * S[3 * t + q];
                        sg += S[3 * r + t] * nF[3 * q + t];
                    }
                    N[3 * r + q] = S[3 * r + q] + (gs + sg);
                }
            c[0] = N[0]; c[1] = N[1]; c[2] = N[2]; c[3] = N[4]; c[4] = N[5]; c[5] = N[8];
        }
    }
    for (int p = 0; p < 3 * n; ++p) x[p] = target[p];
}

int or_real_size(void) { return (int)sizeof(real); }
int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
