// spectral.cuh — the constitutive update written in singular values, and its
// adjoint.
//
// Every return map and stress of the material switch
// (phys_sim/diff_simulator/warp_mpm/mpm_utils.py:602-665) is isotropic. With
// F_trial = U diag(s) V^T:
//   F_elastic = U diag(f(s)) V^T,
//   tau       = U diag(h(s)) U^T   (symmetric, so its symmetrisation is exact),
// where f and h also depend on mu, lam and the yield stress, and the return
// map updates those three. `spectral_map` evaluates f, h and the updated
// scalars. It mirrors constitutive() in constitutive.cuh operation for
// operation, so it takes the same branches. Evaluated on Dual<6> numbers
// seeded on (s0, s1, s2, mu, lam, yield), it yields the Jacobian that the
// adjoint needs.
//
// Adjoint of a spectral function. Let M = U^T dF V. Then diag(M) = ds, and the
// off-diagonal part of M rotates U and V. For i != j, with
//   Df = (f_j - f_i) / (s_j - s_i),  Sf = (f_j + f_i) / (s_j + s_i),
//   Dh = (h_j - h_i) / (s_j - s_i),
// the first variations in the U/V frames are
//   (U^T dF_e V)_ij = p M_ij + q M_ji,          p = (Df + Sf)/2, q = (Df - Sf)/2,
//   (U^T dtau U)_ij = c (s_j M_ij + s_i M_ji),  c = Dh / (s_i + s_j).
// Transposing these gives the gradient in F_trial as U B V^T, with
//   B_ij = p A_ij + q A_ji + c s_j (T_ij + T_ji),
//   A = U^T gF_e V,  T = U^T sym(g_tau) U,
// and B_kk the chain rule through the singular values. When s_i and s_j
// (nearly) coincide, the divided differences Df and Dh are replaced by their
// limits from the Jacobian, (J_ii - J_ij + J_jj - J_ji) / 2.
#pragma once
#include "mat3.cuh"
#include "svd3.cuh"
#include "dual.cuh"
#include "constitutive.cuh"

namespace empm {

EMPM_HD float sconst(float, float v) { return v; }
template <int N> EMPM_HD Dual<N> sconst(const Dual<N>&, float v) { return dconst<N>(v); }

template <class T>
EMPM_HD T slen3(const T a[3]) { return ssqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

template <class T>
struct SpectralOut {
    T f[3];      // singular values of F_elastic (in the frame of F_trial's SVD)
    T h[3];      // eigenvalues of tau (eigenvectors: columns of U)
    T mu, lam, ys;
};

// von Mises on Hencky strain; `damage` adds softening (mpm_utils.py:87-186)
template <class T>
EMPM_HD void spectral_von_mises(T s[3], T& mu, T& lam, T& ys, const MaterialScalars& ms, bool damage) {
    T eps[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) eps[a] = slog(smaxc(s[a], 0.01f));
    const T tr = eps[0] + eps[1] + eps[2];
    const T temp = tr / 3.f;
    T tau[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) tau[a] = (2.f * mu) * eps[a] + lam * tr;
    const T sum_tau = tau[0] + tau[1] + tau[2];
    T cond[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) cond[a] = tau[a] - sum_tau / 3.f;
    if (!(sval(slen3(cond)) > sval(ys))) return;
    if (damage && sval(ys) <= 0.f) return;
    T eh[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) eh[a] = eps[a] - temp;
    const T ehn = slen3(eh) + 1e-6f;
    const T dg = ehn - ys / (2.f * mu);
    const T k = dg / ehn;
#pragma unroll
    for (int a = 0; a < 3; ++a) eps[a] = eps[a] - k * eh[a];
    if (damage) {
        T keh[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) keh[a] = k * eh[a];
        ys = ys - ms.softening * slen3(keh);
        if (sval(ys) <= 0.f) { mu = sconst(mu, 0.f); lam = sconst(lam, 0.f); }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) s[a] = sexp(eps[a]);
    if (ms.hardening == 1.f) ys = ys + (2.f * mu) * ms.xi * dg;
}

// Drucker-Prager sand (mpm_utils.py:237-274)
template <class T>
EMPM_HD void spectral_sand(T s[3], const T& mu, const T& lam, const MaterialScalars& ms) {
    T eps[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) eps[a] = slog(smaxc(sabs(s[a]), 1e-14f));
    const T tr = eps[0] + eps[1] + eps[2];
    T eh[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) eh[a] = eps[a] - tr / 3.f;
    const T ehn = slen3(eh);
    const T dg = ehn + (3.f * lam + 2.f * mu) / (2.f * mu) * tr * ms.alpha;
    if (sval(dg) <= 0.f) return;
    if (sval(tr) > 0.f) {
#pragma unroll
        for (int a = 0; a < 3; ++a) s[a] = sconst(s[a], 1.f);
    } else {
        const T r = dg / ehn;
#pragma unroll
        for (int a = 0; a < 3; ++a) s[a] = sexp(eps[a] - r * eh[a]);
    }
}

// viscoplastic with StVK (mpm_utils.py:189-234)
template <class T>
EMPM_HD void spectral_viscoplastic(T s[3], const T& mu, const T& ys, float dt, const MaterialScalars& ms) {
    T sig[3], eps[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) { sig[a] = smaxc(s[a], 0.01f); eps[a] = slog(sig[a]); }
    const T btr = sig[0] * sig[0] + sig[1] * sig[1] + sig[2] * sig[2];
    const T tr = eps[0] + eps[1] + eps[2];
    T st[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) st[a] = (2.f * mu) * (eps[a] - tr / 3.f);
    const T stn = slen3(st);
    const T y = stn - sqrtf(2.f / 3.f) * ys;
    if (!(sval(y) > 0.f)) return;
    const T mu_hat = mu * btr / 3.f;
    const T snn = stn - y / (1.f + ms.plastic_viscosity / ((2.f * mu_hat) * dt));
    const T r = snn / stn;
    const T i2mu = 1.f / (2.f * mu);
#pragma unroll
    for (int a = 0; a < 3; ++a) s[a] = sexp(i2mu * (r * st[a]) + tr / 3.f);
}

// MAT >= 0 compiles the map for that material alone (a batch whose instances
// all use it); -1 switches on ms.material.
template <class T, int MAT = -1>
EMPM_HD SpectralOut<T> spectral_map(const T s_in[3], T mu, T lam, T ys, float dt, const MaterialScalars& ms) {
    T s[3] = {s_in[0], s_in[1], s_in[2]};
    const int material = MAT >= 0 ? MAT : ms.material;
    switch (material) {
        case 1: spectral_von_mises(s, mu, lam, ys, ms, false); break;
        case 2: spectral_sand(s, mu, lam, ms); break;
        case 3: spectral_viscoplastic(s, mu, ys, dt, ms); break;
        case 5: spectral_von_mises(s, mu, lam, ys, ms, true); break;
        default: break;
    }
    SpectralOut<T> o;
#pragma unroll
    for (int a = 0; a < 3; ++a) { o.f[a] = s[a]; o.h[a] = sconst(s[a], 0.f); }
    const T J = s[0] * s[1] * s[2];
    switch (material) {
        case 0:
        case 5: {  // fixed-corotated: 2 mu (F - R) F^T + lam J (J - 1) I
            const T vol = lam * J * (J - 1.f);
#pragma unroll
            for (int a = 0; a < 3; ++a) o.h[a] = (2.f * mu) * (s[a] - 1.f) * s[a] + vol;
            break;
        }
        case 1:
        case 3: {  // StVK with Hencky strain
            T e[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) e[a] = slog(smaxc(s[a], 0.01f));
            const T ls = e[0] + e[1] + e[2];
#pragma unroll
            for (int a = 0; a < 3; ++a) o.h[a] = ((2.f * mu) * e[a] + lam * ls) * s[a];
            break;
        }
        case 2: {  // Drucker-Prager
            T e[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) e[a] = slog(s[a]);
            const T ls = e[0] + e[1] + e[2];
#pragma unroll
            for (int a = 0; a < 3; ++a) o.h[a] = (2.f * mu) * e[a] + lam * ls;
            break;
        }
        case 6: {  // compressible neo-Hookean
            T b[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) b[a] = s[a] * s[a];
            const T bm = (b[0] + b[1] + b[2]) / 3.f;
            const T ca = mu * spow(J, -2.f / 3.f);
            const T cc = lam / 2.f * (J * J - 1.f);
#pragma unroll
            for (int a = 0; a < 3; ++a) o.h[a] = (ca * (b[a] - bm) + cc) * s[a];
            break;
        }
        default: break;  // snow (4): zero stress
    }
    o.mu = mu;
    o.lam = lam;
    o.ys = ys;
    return o;
}

// One particle's constitutive update, factorised and differentiated.
typedef Dual<6> D6;   // tangent directions: s0, s1, s2, mu, lam, yield

struct SpectralEval {
    M3 U, V;
    float s[3];
    SpectralOut<D6> o;
};

// Fixed-corotated stress with no return map (jelly, and plasticine inside its
// yield surface), with its Jacobian written out: f = s, the scalars pass
// through, h_a = 2 mu (s_a - 1) s_a + lam J (J - 1) with J = s0 s1 s2, so
//   dh_a/ds_b = 2 mu (2 s_a - 1) [a = b] + lam (2 J - 1) J_b,  J_b = dJ/ds_b,
//   dh_a/dmu = 2 (s_a - 1) s_a,  dh_a/dlam = J (J - 1).
// The same values and derivatives as spectral_map on Dual<6> numbers on that
// branch, for a fraction of its arithmetic.
EMPM_HD void spectral_fcr_elastic(const float s[3], float mu, float lam, float ys, SpectralOut<D6>& o) {
    const float J = s[0] * s[1] * s[2];
    const float Jb[3] = {s[1] * s[2], s[0] * s[2], s[0] * s[1]};
    const float vol = lam * J * (J - 1.f);
    const float cv = lam * (2.f * J - 1.f);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        o.f[a] = dseed<6>(s[a], a);
        o.h[a].v = (2.f * mu) * (s[a] - 1.f) * s[a] + vol;
#pragma unroll
        for (int b = 0; b < 3; ++b) o.h[a].d[b] = cv * Jb[b] + (a == b ? (2.f * mu) * (2.f * s[a] - 1.f) : 0.f);
        o.h[a].d[3] = 2.f * (s[a] - 1.f) * s[a];
        o.h[a].d[4] = J * (J - 1.f);
        o.h[a].d[5] = 0.f;
    }
    o.mu = dseed<6>(mu, 3);
    o.lam = dseed<6>(lam, 4);
    o.ys = dseed<6>(ys, 5);
}

// The von Mises yield test of constitutive() (constitutive.cuh) on the
// singular values: true when the return map changes nothing.
EMPM_HD bool von_mises_inside(const float s[3], float mu, float lam, float ys, bool damage) {
    const V3 sig = v3(fmaxf(s[0], 0.01f), fmaxf(s[1], 0.01f), fmaxf(s[2], 0.01f));
    const V3 eps = v3(logf(sig.x), logf(sig.y), logf(sig.z));
    const float tr = eps.x + eps.y + eps.z;
    const V3 tau = 2.f * mu * eps + v3(lam * tr, lam * tr, lam * tr);
    const float sum_tau = tau.x + tau.y + tau.z;
    const V3 cond = tau - v3(sum_tau / 3.f, sum_tau / 3.f, sum_tau / 3.f);
    if (!(length(cond) > ys)) return true;
    return damage && ys <= 0.f;
}

template <int MAT = -1>
EMPM_HD void spectral_eval(const M3& Ft, float mu, float lam, float ys, float dt, const MaterialScalars& ms,
                           SpectralEval& e) {
    V3 sv;
    svd3(Ft, e.U, sv, e.V);
    e.s[0] = sv.x; e.s[1] = sv.y; e.s[2] = sv.z;
    const int material = MAT >= 0 ? MAT : ms.material;
    if (material == 0 || (material == 5 && von_mises_inside(e.s, mu, lam, ys, true))) {
        spectral_fcr_elastic(e.s, mu, lam, ys, e.o);
        return;
    }
    const D6 s[3] = {dseed<6>(sv.x, 0), dseed<6>(sv.y, 1), dseed<6>(sv.z, 2)};
    e.o = spectral_map<D6, MAT>(s, dseed<6>(mu, 3), dseed<6>(lam, 4), dseed<6>(ys, 5), dt, ms);
}

// tau = U diag(h) U^T
EMPM_HD M3 spectral_tau(const SpectralEval& e) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[3 * i + j] = e.U.m[3 * i + 0] * e.o.h[0].v * e.U.m[3 * j + 0] +
                             e.U.m[3 * i + 1] * e.o.h[1].v * e.U.m[3 * j + 1] +
                             e.U.m[3 * i + 2] * e.o.h[2].v * e.U.m[3 * j + 2];
    return r;
}

struct SpectralGrad {
    M3    gFt;                 // gradient in F_trial
    float g_mu, g_lam, g_ys;   // gradient in the material scalars before the update
};

// Divided difference (x_j - x_i) / (s_j - s_i), or its limit from the Jacobian
// when the singular values (nearly) coincide.
EMPM_HD float spectral_divdiff(const D6& xi, const D6& xj, float si, float sj, int i, int j) {
    const float ds = sj - si;
    if (fabsf(ds) > 1e-4f * (fabsf(si) + fabsf(sj)) + 1e-30f) return (xj.v - xi.v) / ds;
    return 0.5f * (xi.d[i] - xi.d[j] + xj.d[j] - xj.d[i]);
}

// g_Fe: gradient in F_elastic; g_tau: gradient in the (symmetrised) stress;
// g_mu_out, g_lam_out, g_ys_out: gradients in the updated material scalars.
EMPM_HD SpectralGrad spectral_adjoint(const SpectralEval& e, const M3& g_Fe, const M3& g_tau, float g_mu_out,
                                      float g_lam_out, float g_ys_out) {
    const M3 A = transpose(e.U) * g_Fe * e.V;
    const M3 gs = 0.5f * (g_tau + transpose(g_tau));
    const M3 T = transpose(e.U) * gs * e.U;
    float gseed[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) {
        float acc = g_mu_out * e.o.mu.d[d] + g_lam_out * e.o.lam.d[d] + g_ys_out * e.o.ys.d[d];
#pragma unroll
        for (int k = 0; k < 3; ++k) acc += A.m[4 * k] * e.o.f[k].d[d] + T.m[4 * k] * e.o.h[k].d[d];
        gseed[d] = acc;
    }
    M3 B = m3_diag(gseed[0], gseed[1], gseed[2]);
    const int PI[3] = {0, 0, 1}, PJ[3] = {1, 2, 2};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int i = PI[q], j = PJ[q];
        const float si = e.s[i], sj = e.s[j];
        const float Df = spectral_divdiff(e.o.f[i], e.o.f[j], si, sj, i, j);
        const float Dh = spectral_divdiff(e.o.h[i], e.o.h[j], si, sj, i, j);
        float sum = si + sj;
        if (fabsf(sum) < 1e-6f) sum = sum < 0.f ? -1e-6f : 1e-6f;
        const float Sf = (e.o.f[i].v + e.o.f[j].v) / sum;
        const float p = 0.5f * (Df + Sf), qq = 0.5f * (Df - Sf), c = Dh / sum;
        const float Aij = A.m[3 * i + j], Aji = A.m[3 * j + i];
        const float Ts = T.m[3 * i + j] + T.m[3 * j + i];
        B.m[3 * i + j] = p * Aij + qq * Aji + c * sj * Ts;
        B.m[3 * j + i] = p * Aji + qq * Aij + c * si * Ts;
    }
    SpectralGrad g;
    g.gFt = e.U * B * transpose(e.V);
    g.g_mu = gseed[3];
    g.g_lam = gseed[4];
    g.g_ys = gseed[5];
    return g;
}

}  // namespace empm
