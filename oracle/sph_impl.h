/*
 * sph_impl.h — WCSPH step and integrate_particles, written once over REAL
 * and included by sph_f32.c (REAL=float) and sph_f64.c (REAL=double).
 * TEST INFRASTRUCTURE ONLY (the checker; see nsph_oracle.h).
 *
 * Neighbour topology is always fp32 (oracle_neighbors_of); only the physics
 * arithmetic follows REAL.
 *
 * Step definition (no SPH exists in the reference; published methods):
 *   W(r)    = sigma * (6(q^3-q^2)+1)   q <= 1/2       sigma = 8/(pi h^3), q = r/h
 *           = sigma * 2(1-q)^3         1/2 < q < 1    (Monaghan 1992, support h)
 *   rho_i   = sum_{j in N(i), self incl.} m_j W(r_ij)
 *   p_i     = B((rho_i/rho0)^gamma - 1), clamped at 0   (Tait; B = rho0 c0^2/gamma)
 *   a_i     = - sum_{j != i} m_j (p_i/rho_i^2 + p_j/rho_j^2) grad_i W_ij
 *   dv_i    = sum_{j != i} (m_j/rho_j)(v_j - v_i) W_ij    (XSPH, old velocities)
 * Every fp32 operation is written out (explicit fma where the device uses
 * one, no other contraction), and neighbours are summed in the grid's query
 * order, so the fp32 instance reproduces the device's per-particle sums.
 * Integration follows integrate_particles (newton/_src/solvers/solver.py:24-47):
 *   inactive: x1 = x0, v untouched
 *   w > 0:    v1 = v0 + (a_i + f_i w + g[max(world,0)]) dt + eps dv_i
 *   w == 0:   v1 = v0
 *   |v1| > v_max: v1 *= v_max/|v1|;  x1 = x0 + v1 dt
 *   w > 0 and box: x clamped to [lo, hi], the velocity component into the
 *   wall set to 0.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct SFX(phys) {
    REAL h, inv_h, sigma, dsigma, rho0, inv_rho0, eos_b, xsph_eps, v_max, dt;
    REAL c_near; /* 6 dsigma / h */
    REAL c_far;  /* -6 dsigma    */
    REAL box_lo[3], box_hi[3];
    int eos_gamma, clamp_pressure, use_box;
} SFX(phys);

/* W(q): near = fma((6q)q, q-1, 1), far = ((2t)t)t with t = 1-q */
static inline REAL SFX(kernel_w)(REAL q, const SFX(phys) * ph)
{
    const REAL t = (REAL)1 - q;
    const REAL nearv = RFMA((REAL)6 * q * q, q - (REAL)1, (REAL)1);
    const REAL farv = (REAL)2 * t * t * t;
    return ph->sigma * (q <= (REAL)0.5 ? nearv : (q < (REAL)1 ? farv : (REAL)0));
}

/* (dW/dr)/r: near = (6 dsigma/h)(3q-2) with 3q-2 = fma(3,q,-2),
 * far = ((-6 dsigma) t) t * (1/r) */
static inline REAL SFX(kernel_f)(REAL q, REAL inv_r, const SFX(phys) * ph)
{
    const REAL t = (REAL)1 - q;
    const REAL nearv = ph->c_near * RFMA((REAL)3, q, (REAL)-2);
    const REAL farv = ph->c_far * t * t * inv_r;
    return q <= (REAL)0.5 ? nearv : (q < (REAL)1 ? farv : (REAL)0);
}

static inline REAL SFX(eos)(REAL rho, const SFX(phys) * ph)
{
    const REAL ratio = rho * ph->inv_rho0;
    REAL pw = (REAL)1;
    for (int k = 0; k < ph->eos_gamma; ++k) pw *= ratio;
    REAL p = ph->eos_b * (pw - (REAL)1);
    if (ph->clamp_pressure && p < (REAL)0) p = (REAL)0;
    return p;
}

static inline int SFX(gravity_index)(const int* world, int i, int world_count)
{
    int w = world ? world[i] : 0;
    if (w < 0) w = 0;
    if (w >= world_count) w = world_count - 1;
    return w;
}

static int SFX(sph_step_impl)(const nsph_sph_params* p, const SFX(phys) * ph, const int* grid_dims, int n,
                              const float* x_in, const float* v_in, const float* f_ext, const float* mass,
                              const float* inv_mass, const int* flags, const int* world,
                              const float* gravity, int world_count, REAL* x_out, REAL* v_out,
                              REAL* rho_out, REAL* p_out, REAL* a_out, REAL* a_scale_out)
{
    if (n < 0 || world_count < 1) return NSPH_ERR_INVALID_ARG;
    if (n == 0) return NSPH_OK;
    grid_tables g;
    int st = oracle_build_tables(&g, p, grid_dims, n, x_in);
    if (st != NSPH_OK) return st;
    REAL* rho = (REAL*)malloc(sizeof(REAL) * (size_t)n);
    REAL* prs = (REAL*)malloc(sizeof(REAL) * (size_t)n);
    REAL* pr2 = (REAL*)malloc(sizeof(REAL) * (size_t)n); /* p / rho^2 */
    REAL* mor = (REAL*)malloc(sizeof(REAL) * (size_t)n); /* m / rho   */
    if (!rho || !prs || !pr2 || !mor) {
        free(rho);
        free(prs);
        free(pr2);
        free(mor);
        oracle_free_tables(&g);
        return NSPH_ERR_OUT_OF_MEMORY;
    }
    int fail = 0;

    /* ---- pass 1: density and equation of state ---- */
#pragma omp parallel
    {
        long long cap = 256;
        int* nb = (int*)malloc(sizeof(int) * (size_t)cap);
#pragma omp for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            rho[i] = prs[i] = pr2[i] = mor[i] = (REAL)0;
            if (!(flags[i] & NSPH_PARTICLE_ACTIVE) || !nb) continue;
            long long cnt = oracle_neighbors_of(&g, p, x_in, flags, i, nb, cap);
            if (cnt > cap) {
                cap = cnt * 2;
                free(nb);
                nb = (int*)malloc(sizeof(int) * (size_t)cap);
                if (!nb) {
#pragma omp atomic write
                    fail = 1;
                    continue;
                }
                cnt = oracle_neighbors_of(&g, p, x_in, flags, i, nb, cap);
            }
            const float* xi = x_in + 3 * (size_t)i;
            REAL acc = (REAL)0;
            for (long long t = 0; t < cnt; ++t) {
                const int j = nb[t];
                const float* xj = x_in + 3 * (size_t)j;
                const REAL dx = (REAL)xi[0] - (REAL)xj[0];
                const REAL dy = (REAL)xi[1] - (REAL)xj[1];
                const REAL dz = (REAL)xi[2] - (REAL)xj[2];
                const REAL r = RSQRT(RFMA(dz, dz, RFMA(dy, dy, dx * dx)));
                acc = RFMA((REAL)mass[j], SFX(kernel_w)(r * ph->inv_h, ph), acc);
            }
            rho[i] = acc;
            if (acc > (REAL)0) {
                prs[i] = SFX(eos)(acc, ph);
                pr2[i] = prs[i] / (acc * acc);
                mor[i] = (REAL)mass[i] / acc;
            }
        }
        free(nb);
    }

    /* ---- pass 2: pressure force, XSPH, integrate ---- */
#pragma omp parallel
    {
        long long cap = 256;
        int* nb = (int*)malloc(sizeof(int) * (size_t)cap);
#pragma omp for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            const float* xi = x_in + 3 * (size_t)i;
            if (rho_out) rho_out[i] = rho[i];
            if (p_out) p_out[i] = prs[i];
            if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) {
                for (int c = 0; c < 3; ++c) {
                    x_out[3 * (size_t)i + c] = (REAL)xi[c];
                    if (a_out) a_out[3 * (size_t)i + c] = (REAL)0;
                }
                if (a_scale_out) a_scale_out[i] = (REAL)0;
                continue;
            }
            if (!nb) continue;
            long long cnt = oracle_neighbors_of(&g, p, x_in, flags, i, nb, cap);
            if (cnt > cap) {
                cap = cnt * 2;
                free(nb);
                nb = (int*)malloc(sizeof(int) * (size_t)cap);
                if (!nb) {
#pragma omp atomic write
                    fail = 1;
                    continue;
                }
                cnt = oracle_neighbors_of(&g, p, x_in, flags, i, nb, cap);
            }
            const float* vi = v_in + 3 * (size_t)i;
            REAL a[3] = {0, 0, 0}, dv[3] = {0, 0, 0}, ascale = 0;
            for (long long t = 0; t < cnt; ++t) {
                const int j = nb[t];
                if (j == i) continue;
                const float* xj = x_in + 3 * (size_t)j;
                const float* vj = v_in + 3 * (size_t)j;
                const REAL d[3] = {(REAL)xi[0] - (REAL)xj[0], (REAL)xi[1] - (REAL)xj[1],
                                   (REAL)xi[2] - (REAL)xj[2]};
                const REAL r2 = RFMA(d[2], d[2], RFMA(d[1], d[1], d[0] * d[0]));
                const REAL r = RSQRT(r2);
                const REAL q = r * ph->inv_h;
                const REAL w = SFX(kernel_w)(q, ph);
                if (r2 > (REAL)0) {
                    const REAL inv_r = (REAL)1 / r;
                    const REAL s = (REAL)mass[j] * (pr2[i] + pr2[j]) * SFX(kernel_f)(q, inv_r, ph);
                    for (int c = 0; c < 3; ++c) a[c] = RFMA(-s, d[c], a[c]);
                    ascale += RABS(s) * r;
                }
                const REAL cw = mor[j] * w;
                for (int c = 0; c < 3; ++c) dv[c] = RFMA(cw, (REAL)vj[c] - (REAL)vi[c], dv[c]);
            }
            if (a_out)
                for (int c = 0; c < 3; ++c) a_out[3 * (size_t)i + c] = a[c];
            if (a_scale_out) a_scale_out[i] = ascale;

            const REAL wi = (REAL)inv_mass[i];
            REAL v1[3] = {(REAL)vi[0], (REAL)vi[1], (REAL)vi[2]};
            if (wi > (REAL)0) {
                const float* gv = gravity + 3 * (size_t)SFX(gravity_index)(world, i, world_count);
                for (int c = 0; c < 3; ++c) {
                    const REAL fe = f_ext ? (REAL)f_ext[3 * (size_t)i + c] * wi : (REAL)0;
                    const REAL acc = (a[c] + fe) + (REAL)gv[c];
                    v1[c] = RFMA(ph->xsph_eps, dv[c], RFMA(acc, ph->dt, (REAL)vi[c]));
                }
            }
            const REAL vmag = RSQRT(RFMA(v1[2], v1[2], RFMA(v1[1], v1[1], v1[0] * v1[0])));
            if (vmag > ph->v_max) {
                const REAL s = ph->v_max / vmag;
                for (int c = 0; c < 3; ++c) v1[c] *= s;
            }
            REAL x1[3];
            for (int c = 0; c < 3; ++c) x1[c] = RFMA(v1[c], ph->dt, (REAL)xi[c]);
            if (wi > (REAL)0 && ph->use_box) {
                for (int c = 0; c < 3; ++c) {
                    if (x1[c] < ph->box_lo[c]) {
                        x1[c] = ph->box_lo[c];
                        if (v1[c] < (REAL)0) v1[c] = (REAL)0;
                    }
                    if (x1[c] > ph->box_hi[c]) {
                        x1[c] = ph->box_hi[c];
                        if (v1[c] > (REAL)0) v1[c] = (REAL)0;
                    }
                }
            }
            for (int c = 0; c < 3; ++c) {
                x_out[3 * (size_t)i + c] = x1[c];
                v_out[3 * (size_t)i + c] = v1[c];
            }
        }
        free(nb);
    }

    free(rho);
    free(prs);
    free(pr2);
    free(mor);
    oracle_free_tables(&g);
    return fail ? NSPH_ERR_OUT_OF_MEMORY : NSPH_OK;
}

/* integrate_particles, newton/_src/solvers/solver.py:10-47 */
static void SFX(integrate_impl)(const float* x, const float* v, const float* f, const float* inv_mass,
                                const int* flags, const int* world, const float* gravity, int world_count,
                                int n, REAL dt, REAL v_max, REAL* x_new, REAL* v_new)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const float* x0 = x + 3 * (size_t)i;
        if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) {
            for (int c = 0; c < 3; ++c) x_new[3 * (size_t)i + c] = (REAL)x0[c];
            continue;
        }
        const float* v0 = v + 3 * (size_t)i;
        const float* f0 = f + 3 * (size_t)i;
        const REAL w = (REAL)inv_mass[i];
        const float* g = gravity + 3 * (size_t)SFX(gravity_index)(world, i, world_count);
        const REAL gate = (-w < (REAL)0) ? (REAL)1 : (REAL)0; /* wp.step(-w) */
        REAL v1[3];
        for (int c = 0; c < 3; ++c) {
            const REAL acc = (REAL)f0[c] * w + (REAL)g[c] * gate;
            v1[c] = RFMA(acc, dt, (REAL)v0[c]);
        }
        const REAL m = RSQRT(RFMA(v1[2], v1[2], RFMA(v1[1], v1[1], v1[0] * v1[0])));
        if (m > v_max) {
            const REAL s = v_max / m;
            for (int c = 0; c < 3; ++c) v1[c] *= s;
        }
        for (int c = 0; c < 3; ++c) {
            x_new[3 * (size_t)i + c] = RFMA(v1[c], dt, (REAL)x0[c]);
            v_new[3 * (size_t)i + c] = v1[c];
        }
    }
}
