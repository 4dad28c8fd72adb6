/*
 * contact.c — particle-particle contact on the HashGrid, restated in fp32.
 * TEST INFRASTRUCTURE ONLY (the checker; see nsph_oracle.h).
 *
 * Restates, operation by operation:
 *   particle_force + eval_particle_contact
 *     newton/_src/solvers/semi_implicit/kernels_contact.py:11-32, 35-84
 *   solve_particle_particle_contacts
 *     newton/_src/solvers/xpbd/kernels.py:225-289
 * with the candidates of hash_grid_query(grid, x_i, r_i + max_radius +
 * cohesion) in Warp's order (oracle_grid_query on a grid built with cell
 * width `grid_radius`). fp32, every operation rounded as written (dot
 * products ((x + y) + z), -ffp-contract=off), so the device results match
 * bit for bit. Warp's normalize returns the zero vector for a zero-length
 * input.
 */
#include <math.h>
#include <stdlib.h>

#include "nsph_oracle.h"

static inline float dot3(const float a[3], const float b[3])
{
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

static void particle_force(const float n[3], const float v[3], float c, const nsph_contact_params* p, float out[3])
{
    const float vn = dot3(n, v);
    const float jn = c * p->k_contact;
    const float jd = fminf(vn, 0.0f) * p->k_damp;
    const float fn = jn + jd;
    float vt[3];
    for (int k = 0; k < 3; ++k) vt[k] = v[k] - n[k] * vn;
    const float vs = sqrtf(dot3(vt, vt));
    if (vs > 0.0f)
        for (int k = 0; k < 3; ++k) vt[k] = vt[k] / vs;
    const float ft = fminf(vs * p->k_friction, p->k_mu * fabsf(fn));
    for (int k = 0; k < 3; ++k) out[k] = (-n[k]) * fn - vt[k] * ft;
}

typedef struct contact_grid {
    int *cells, *ids, *starts, *ends;
    int dims[3];
    float inv;
} contact_grid;

static int build(contact_grid* g, const float* x, int n, float grid_radius, const int* dims)
{
    const size_t nc = (size_t)dims[0] * dims[1] * dims[2];
    g->cells = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    g->ids = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    g->starts = (int*)malloc(sizeof(int) * nc);
    g->ends = (int*)malloc(sizeof(int) * nc);
    for (int k = 0; k < 3; ++k) g->dims[k] = dims[k];
    g->inv = 1.0f / grid_radius;
    if (!g->cells || !g->ids || !g->starts || !g->ends) return NSPH_ERR_OUT_OF_MEMORY;
    return oracle_grid_build(x, n, grid_radius, dims[0], dims[1], dims[2], g->cells, g->ids, g->starts, g->ends);
}

static void release(contact_grid* g)
{
    free(g->cells);
    free(g->ids);
    free(g->starts);
    free(g->ends);
}

/* candidates of particle i (Warp order) into *buf (grown as needed) */
static long long candidates(const contact_grid* g, const float pos[3], float r, int** buf, long long* cap)
{
    long long cnt = oracle_grid_query(g->ids, g->starts, g->ends, g->dims[0], g->dims[1], g->dims[2], g->inv, pos, r,
                                      *buf, *cap);
    if (cnt > *cap) {
        free(*buf);
        *cap = cnt * 2;
        *buf = (int*)malloc(sizeof(int) * (size_t)*cap);
        if (!*buf) return -1;
        cnt = oracle_grid_query(g->ids, g->starts, g->ends, g->dims[0], g->dims[1], g->dims[2], g->inv, pos, r, *buf,
                                *cap);
    }
    return cnt;
}

int oracle_particle_contact_forces(const nsph_contact_params* p, float grid_radius, const int* dims, int n,
                                   const float* x, const float* v, const float* radius, const int* flags,
                                   float* f_out)
{
    if (!p || !dims || n < 0 || !(grid_radius > 0.0f)) return NSPH_ERR_INVALID_ARG;
    if (n == 0) return NSPH_OK;
    contact_grid g;
    int st = build(&g, x, n, grid_radius, dims);
    if (st != NSPH_OK) {
        release(&g);
        return st;
    }
    int fail = 0;
#pragma omp parallel
    {
        long long cap = 256;
        int* buf = (int*)malloc(sizeof(int) * (size_t)cap);
#pragma omp for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            if (!(flags[i] & NSPH_PARTICLE_ACTIVE) || !buf) continue;
            const float* xi = x + 3 * (size_t)i;
            const float* vi = v + 3 * (size_t)i;
            const float qr = (radius[i] + p->max_radius) + p->k_cohesion;
            const long long cnt = candidates(&g, xi, qr, &buf, &cap);
            if (cnt < 0) {
#pragma omp atomic write
                fail = 1;
                continue;
            }
            float f[3] = {0.0f, 0.0f, 0.0f};
            for (long long t = 0; t < cnt; ++t) {
                const int j = buf[t];
                if (!(flags[j] & NSPH_PARTICLE_ACTIVE) || j == i) continue;
                float nv[3];
                for (int k = 0; k < 3; ++k) nv[k] = xi[k] - x[3 * (size_t)j + k];
                const float d = sqrtf(dot3(nv, nv));
                const float err = (d - radius[i]) - radius[j];
                if (err <= p->k_cohesion) {
                    float vr[3], pf[3];
                    for (int k = 0; k < 3; ++k) {
                        nv[k] = nv[k] / d;
                        vr[k] = vi[k] - v[3 * (size_t)j + k];
                    }
                    particle_force(nv, vr, err, p, pf);
                    for (int k = 0; k < 3; ++k) f[k] = f[k] + pf[k];
                }
            }
            for (int k = 0; k < 3; ++k) f_out[3 * (size_t)i + k] = f[k];
        }
        free(buf);
    }
    release(&g);
    return fail ? NSPH_ERR_OUT_OF_MEMORY : NSPH_OK;
}

int oracle_particle_contact_deltas(float grid_radius, const int* dims, int n, const float* x, const float* v,
                                   const float* inv_mass, const float* radius, const int* flags, float k_mu,
                                   float k_cohesion, float max_radius, float dt, float relaxation, float* deltas)
{
    return oracle_particle_contact_deltas_grid(x, grid_radius, dims, n, x, v, inv_mass, radius, flags, k_mu,
                                               k_cohesion, max_radius, dt, relaxation, deltas);
}

int oracle_particle_contact_deltas_grid(const float* grid_x, float grid_radius, const int* dims, int n,
                                        const float* x, const float* v, const float* inv_mass, const float* radius,
                                        const int* flags, float k_mu, float k_cohesion, float max_radius, float dt,
                                        float relaxation, float* deltas)
{
    if (!dims || n < 0 || !(grid_radius > 0.0f)) return NSPH_ERR_INVALID_ARG;
    if (n == 0) return NSPH_OK;
    contact_grid g;
    int st = build(&g, grid_x, n, grid_radius, dims);
    if (st != NSPH_OK) {
        release(&g);
        return st;
    }
    int fail = 0;
#pragma omp parallel
    {
        long long cap = 256;
        int* buf = (int*)malloc(sizeof(int) * (size_t)cap);
#pragma omp for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            if (!(flags[i] & NSPH_PARTICLE_ACTIVE) || !buf) continue;
            const float* xi = x + 3 * (size_t)i;
            const float* vi = v + 3 * (size_t)i;
            const float w1 = inv_mass[i];
            const float qr = (radius[i] + max_radius) + k_cohesion;
            const long long cnt = candidates(&g, xi, qr, &buf, &cap);
            if (cnt < 0) {
#pragma omp atomic write
                fail = 1;
                continue;
            }
            float delta[3] = {0.0f, 0.0f, 0.0f};
            for (long long t = 0; t < cnt; ++t) {
                const int j = buf[t];
                if (!(flags[j] & NSPH_PARTICLE_ACTIVE) || j == i) continue;
                float nv[3];
                for (int k = 0; k < 3; ++k) nv[k] = xi[k] - x[3 * (size_t)j + k];
                const float d = sqrtf(dot3(nv, nv));
                const float err = (d - radius[i]) - radius[j];
                const float denom = w1 + inv_mass[j];
                if (err <= k_cohesion && denom > 0.0f) {
                    float vr[3], dn[3], vt[3];
                    for (int k = 0; k < 3; ++k) {
                        nv[k] = nv[k] / d;
                        vr[k] = vi[k] - v[3 * (size_t)j + k];
                    }
                    const float lambda_n = err;
                    for (int k = 0; k < 3; ++k) dn[k] = nv[k] * lambda_n;
                    const float vn = dot3(nv, vr);
                    for (int k = 0; k < 3; ++k) vt[k] = vr[k] - nv[k] * vn;
                    const float lt = sqrtf(dot3(vt, vt));
                    const float lambda_f = fmaxf(k_mu * lambda_n, (-lt) * dt);
                    for (int k = 0; k < 3; ++k) {
                        const float u = lt > 0.0f ? vt[k] / lt : 0.0f;
                        delta[k] = delta[k] + (u * lambda_f - dn[k]) / denom;
                    }
                }
            }
            for (int k = 0; k < 3; ++k)
                deltas[3 * (size_t)i + k] = deltas[3 * (size_t)i + k] + (delta[k] * w1) * relaxation;
        }
        free(buf);
    }
    release(&g);
    return fail ? NSPH_ERR_OUT_OF_MEMORY : NSPH_OK;
}
