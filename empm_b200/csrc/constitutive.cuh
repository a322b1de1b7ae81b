// constitutive.cuh — return maps and Kirchhoff stresses of the reference's
// material switch (phys_sim/diff_simulator/warp_mpm/mpm_utils.py:602-665).
//
// One SVD per particle: the return map factorises F_trial, and the stress
// reuses that factorisation for the elastic F (U diag(sigma_e) V^T with the
// same U, V), where the reference factorises F a second time
// (mpm_utils.py:641). Every stress below is a spectral function of F, so the
// result is independent of which valid factorisation is used.
#pragma once
#include "mat3.cuh"
#include "svd3.cuh"

namespace empm {

struct MaterialScalars {
    int   material;
    float softening;
    float hardening;
    float xi;
    float plastic_viscosity;
    float alpha;
};

struct ConstitutiveOut {
    M3   F;            // elastic deformation gradient (particle_F)
    M3   tau;          // symmetrised Kirchhoff stress (particle_stress)
    bool mat_changed;  // yield / mu / lam were modified
};

EMPM_HD M3 usv(const M3& U, V3 s, const M3& V) {
    // U diag(s) V^T
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[3 * i + j] = U.m[3 * i + 0] * s.x * V.m[3 * j + 0] +
                             U.m[3 * i + 1] * s.y * V.m[3 * j + 1] +
                             U.m[3 * i + 2] * s.z * V.m[3 * j + 2];
    return r;
}

// U diag(t) U^T (symmetric)
EMPM_HD M3 u_diag_ut(const M3& U, V3 t) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float a0 = U.m[3 * i + 0] * t.x, a1 = U.m[3 * i + 1] * t.y, a2 = U.m[3 * i + 2] * t.z;
#pragma unroll
        for (int j = i; j < 3; ++j) {
            const float v = a0 * U.m[3 * j + 0] + a1 * U.m[3 * j + 1] + a2 * U.m[3 * j + 2];
            r.m[3 * i + j] = v;
            r.m[3 * j + i] = v;
        }
    }
    return r;
}

// The stresses below have the form tau = U diag(d) V^T F^T with F the elastic
// F = U diag(s) V^T, i.e. tau = U diag(d * s) U^T, symmetric already (the
// reference symmetrises its explicit products, mpm_utils.py:665).
EMPM_HD M3 spectral_stress(const M3& U, V3 d, V3 s) { return u_diag_ut(U, v3(d.x * s.x, d.y * s.y, d.z * s.z)); }

// Von Mises projection on Hencky strain (mpm_utils.py:87-130; with damage
// and softening :133-186 when `damage` is set). Updates s (singular values of
// the returned F) and the material scalars; returns true when F changed.
EMPM_HD bool von_mises(const M3& U, V3& s, const M3& V, float& mu, float& lam, float& ys,
                       const MaterialScalars& ms, bool damage, bool& mat_changed, M3& Fe) {
    const V3 sig = v3(fmaxf(s.x, 0.01f), fmaxf(s.y, 0.01f), fmaxf(s.z, 0.01f));
    V3 eps = v3(logf(sig.x), logf(sig.y), logf(sig.z));
    const float tr = eps.x + eps.y + eps.z;
    const float temp = tr / 3.f;
    const V3 tau = 2.f * mu * eps + v3(lam * tr, lam * tr, lam * tr);
    const float sum_tau = tau.x + tau.y + tau.z;
    const V3 cond = tau - v3(sum_tau / 3.f, sum_tau / 3.f, sum_tau / 3.f);
    if (!(length(cond) > ys)) return false;
    if (damage && ys <= 0.f) return false;
    const V3 eps_hat = eps - v3(temp, temp, temp);
    const float eps_hat_norm = length(eps_hat) + 1e-6f;
    const float delta_gamma = eps_hat_norm - ys / (2.f * mu);
    const float k = delta_gamma / eps_hat_norm;
    eps = eps - k * eps_hat;
    if (damage) {
        ys = ys - ms.softening * length(k * eps_hat);
        if (ys <= 0.f) { mu = 0.f; lam = 0.f; }
    }
    s = v3(expf(eps.x), expf(eps.y), expf(eps.z));
    Fe = usv(U, s, V);
    if (ms.hardening == 1.f) ys = ys + 2.f * mu * ms.xi * delta_gamma;
    mat_changed = true;
    return true;
}

// Drucker-Prager sand projection (mpm_utils.py:237-274).
EMPM_HD bool sand(const M3& U, V3& s, const M3& V, float mu, float lam, const MaterialScalars& ms, M3& Fe) {
    const V3 eps = v3(logf(fmaxf(fabsf(s.x), 1e-14f)), logf(fmaxf(fabsf(s.y), 1e-14f)),
                      logf(fmaxf(fabsf(s.z), 1e-14f)));
    const float tr = eps.x + eps.y + eps.z;
    const V3 eps_hat = eps - v3(tr / 3.f, tr / 3.f, tr / 3.f);
    const float ehn = length(eps_hat);
    const float dg = ehn + (3.f * lam + 2.f * mu) / (2.f * mu) * tr * ms.alpha;
    if (dg <= 0.f) return false;
    if (tr > 0.f) {
        s = v3(1.f, 1.f, 1.f);
    } else {
        const V3 H = eps - (dg / ehn) * eps_hat;
        s = v3(expf(H.x), expf(H.y), expf(H.z));
    }
    Fe = usv(U, s, V);
    return true;
}

// Viscoplastic projection with StVK (mpm_utils.py:189-234).
EMPM_HD bool viscoplastic(const M3& U, V3& s, const M3& V, float mu, float ys, float dt,
                          const MaterialScalars& ms, M3& Fe) {
    const V3 sig = v3(fmaxf(s.x, 0.01f), fmaxf(s.y, 0.01f), fmaxf(s.z, 0.01f));
    const V3 b_trial = v3(sig.x * sig.x, sig.y * sig.y, sig.z * sig.z);
    const V3 eps = v3(logf(sig.x), logf(sig.y), logf(sig.z));
    const float tr = eps.x + eps.y + eps.z;
    const V3 eps_hat = eps - v3(tr / 3.f, tr / 3.f, tr / 3.f);
    const V3 s_trial = 2.f * mu * eps_hat;
    const float s_trial_norm = length(s_trial);
    const float y = s_trial_norm - sqrtf(2.f / 3.f) * ys;
    if (!(y > 0.f)) return false;
    const float mu_hat = mu * (b_trial.x + b_trial.y + b_trial.z) / 3.f;
    const float s_new_norm = s_trial_norm - y / (1.f + ms.plastic_viscosity / (2.f * mu_hat * dt));
    const V3 s_new = (s_new_norm / s_trial_norm) * s_trial;
    const V3 eps_new = (1.f / (2.f * mu)) * s_new + v3(tr / 3.f, tr / 3.f, tr / 3.f);
    s = v3(expf(eps_new.x), expf(eps_new.y), expf(eps_new.z));
    Fe = usv(U, s, V);
    return true;
}

// Return map + stress for one particle. mu, lam, ys are read and, for the
// von Mises models, updated in place.
// MAT >= 0 compiles the update for that material only (a batch whose
// instances all use it); -1 switches on ms.material.
template <int MAT = -1>
EMPM_HD ConstitutiveOut constitutive(const M3& Ft, float& mu, float& lam, float& ys, float dt,
                                     const MaterialScalars& ms) {
    ConstitutiveOut out;
    out.mat_changed = false;
    M3 U, V;
    V3 s;
    svd3(Ft, U, s, V);
    M3 F = Ft;
    const int material = MAT >= 0 ? MAT : ms.material;
    switch (material) {
        case 1: von_mises(U, s, V, mu, lam, ys, ms, false, out.mat_changed, F); break;
        case 2: sand(U, s, V, mu, lam, ms, F); break;
        case 3: viscoplastic(U, s, V, mu, ys, dt, ms, F); break;
        case 5: von_mises(U, s, V, mu, lam, ys, ms, true, out.mat_changed, F); break;
        default: break;
    }
    // F = U diag(s) V^T (after the return maps too), so det F = s.x s.y s.z
    const float J = s.x * s.y * s.z;
    M3 tau = m3_zero();
    switch (material) {
        case 0:
        case 5: {  // fixed-corotated (mpm_utils.py:8-15): 2 mu (F - R) F^T + lam J (J - 1) I, R = U V^T
            const float d = lam * J * (J - 1.f);
            tau = u_diag_ut(U, v3(2.f * mu * (s.x - 1.f) * s.x + d, 2.f * mu * (s.y - 1.f) * s.y + d,
                                  2.f * mu * (s.z - 1.f) * s.z + d));
            break;
        }
        case 1:
        case 3: {  // StVK with Hencky strain (mpm_utils.py:50-66)
            const V3 sg = v3(fmaxf(s.x, 0.01f), fmaxf(s.y, 0.01f), fmaxf(s.z, 0.01f));
            const V3 e = v3(logf(sg.x), logf(sg.y), logf(sg.z));
            const float ls = logf(sg.x) + logf(sg.y) + logf(sg.z);
            const V3 d = 2.f * mu * e + v3(lam * ls, lam * ls, lam * ls);
            tau = spectral_stress(U, d, s);
            break;
        }
        case 2: {  // Drucker-Prager (mpm_utils.py:69-84)
            const float ls = logf(s.x) + logf(s.y) + logf(s.z);
            const V3 d = v3(2.f * mu * logf(s.x) * (1.f / s.x) + lam * ls * (1.f / s.x),
                            2.f * mu * logf(s.y) * (1.f / s.y) + lam * ls * (1.f / s.y),
                            2.f * mu * logf(s.z) * (1.f / s.z) + lam * ls * (1.f / s.z));
            tau = spectral_stress(U, d, s);
            break;
        }
        case 6: {  // compressible neo-Hookean (mpm_utils.py:18-47)
            const V3 b = v3(s.x * s.x, s.y * s.y, s.z * s.z);
            const float bm = (b.x + b.y + b.z) / 3.f;
            const V3 bh = b - v3(bm, bm, bm);
            const float a = mu * powf(J, -2.f / 3.f);
            const float c = lam / 2.f * (J * J - 1.f);
            const V3 d = a * bh + v3(c, c, c);
            tau = spectral_stress(U, d, s);
            break;
        }
        default: break;  // snow (4) and unknown ids: zero stress
    }
    out.F = F;
    out.tau = tau;
    return out;
}

}  // namespace empm
