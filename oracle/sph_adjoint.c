/*
 * sph_adjoint.c — the WCSPH step on an fp64 state and its reverse-mode
 * derivative (vector-Jacobian product), in fp64.
 * TEST INFRASTRUCTURE ONLY (the checker; see nsph_oracle.h). Finite
 * differences of oracle_adj_step_f64 pin oracle_adj_vjp_f64; the device
 * adjoint is then compared with both.
 *
 * The forward map is the step of sph_impl.h (same W, (dW/dr)/r, Tait EOS,
 * pressure force, XSPH, integrate_particles semantics, box), except that the
 * state is double and the neighbour sets are found in double (a cell list of
 * width h over the points' bounding box). The order of the neighbours does
 * not matter in fp64. Inactive particles keep x and v (the velocity output is
 * defined as a copy of the input).
 *
 * The neighbour set is piecewise constant in x; the cubic spline and its
 * derivative vanish at r = h, so the step is continuous with a continuous
 * derivative across a change of neighbour set. The other kinks (pressure
 * clamp at 0, |v| clamp, box) are differentiated on the side the forward
 * took, as the device does.
 *
 * The reverse is written as the plain transposition of the forward, term by
 * term, scattering into both particles of each pair (serial loops), so that
 * it is an independent restatement of the device's gather formulation.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "nsph_oracle.h"

typedef struct adj_lists {
    long long* off; /* n+1 */
    int* ids;       /* neighbours j != i, active, r2 < h2 */
} adj_lists;

static void free_lists(adj_lists* L)
{
    free(L->off);
    free(L->ids);
    L->off = NULL;
    L->ids = NULL;
}

/* neighbour lists in double: cell list of width h over the bounding box */
static int build_lists(const oracle_phys_f64* ph, int n, const double* x, const int* flags, adj_lists* L)
{
    L->off = NULL;
    L->ids = NULL;
    const double h = ph->h, h2 = ph->h * ph->h;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    int any = 0;
    for (int i = 0; i < n; ++i) {
        if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) continue;
        for (int c = 0; c < 3; ++c) {
            const double v = x[3 * (size_t)i + c];
            if (!isfinite(v)) return NSPH_ERR_INVALID_ARG;
            lo[c] = v < lo[c] ? v : lo[c];
            hi[c] = v > hi[c] ? v : hi[c];
        }
        any = 1;
    }
    long long dims[3] = {1, 1, 1};
    if (any)
        for (int c = 0; c < 3; ++c) dims[c] = (long long)floor((hi[c] - lo[c]) / h) + 1;
    const long long ncell = dims[0] * dims[1] * dims[2];
    if (ncell > (1LL << 28)) return NSPH_ERR_CAPACITY;
    int* cell = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    long long* start = (long long*)calloc((size_t)ncell + 1, sizeof(long long));
    int* sorted = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    L->off = (long long*)calloc((size_t)n + 1, sizeof(long long));
    if (!cell || !start || !sorted || !L->off) {
        free(cell);
        free(start);
        free(sorted);
        free_lists(L);
        return NSPH_ERR_OUT_OF_MEMORY;
    }
    for (int i = 0; i < n; ++i) {
        cell[i] = -1;
        if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) continue;
        long long cc[3];
        for (int c = 0; c < 3; ++c) {
            cc[c] = (long long)floor((x[3 * (size_t)i + c] - lo[c]) / h);
            if (cc[c] >= dims[c]) cc[c] = dims[c] - 1;
        }
        cell[i] = (int)((cc[2] * dims[1] + cc[1]) * dims[0] + cc[0]);
        start[cell[i] + 1]++;
    }
    for (long long c = 0; c < ncell; ++c) start[c + 1] += start[c];
    {
        long long* fill = (long long*)malloc(sizeof(long long) * (size_t)ncell);
        if (!fill) {
            free(cell);
            free(start);
            free(sorted);
            free_lists(L);
            return NSPH_ERR_OUT_OF_MEMORY;
        }
        memcpy(fill, start, sizeof(long long) * (size_t)ncell);
        for (int i = 0; i < n; ++i)
            if (cell[i] >= 0) sorted[fill[cell[i]]++] = i;
        free(fill);
    }
    /* two passes: count, then fill */
    for (int pass = 0; pass < 2; ++pass) {
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            if (cell[i] < 0) continue;
            const double* xi = x + 3 * (size_t)i;
            long long cc[3];
            long long rem = cell[i];
            cc[0] = rem % dims[0];
            rem /= dims[0];
            cc[1] = rem % dims[1];
            cc[2] = rem / dims[1];
            long long o = pass ? L->off[i] : 0, cnt = 0;
            for (long long z = cc[2] - 1; z <= cc[2] + 1; ++z)
                for (long long y = cc[1] - 1; y <= cc[1] + 1; ++y)
                    for (long long xx = cc[0] - 1; xx <= cc[0] + 1; ++xx) {
                        if (z < 0 || y < 0 || xx < 0 || z >= dims[2] || y >= dims[1] || xx >= dims[0]) continue;
                        const long long id = (z * dims[1] + y) * dims[0] + xx;
                        for (long long t = start[id]; t < start[id + 1]; ++t) {
                            const int j = sorted[t];
                            if (j == i) continue;
                            const double* xj = x + 3 * (size_t)j;
                            const double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
                            if (dx * dx + dy * dy + dz * dz < h2) {
                                if (pass) L->ids[o++] = j;
                                ++cnt;
                            }
                        }
                    }
            if (!pass) L->off[i + 1] = cnt;
        }
        if (!pass) {
            for (int i = 0; i < n; ++i) L->off[i + 1] += L->off[i];
            L->ids = (int*)malloc(sizeof(int) * (size_t)(L->off[n] > 0 ? L->off[n] : 1));
            if (!L->ids) {
                free(cell);
                free(start);
                free(sorted);
                free_lists(L);
                return NSPH_ERR_OUT_OF_MEMORY;
            }
        }
    }
    free(cell);
    free(start);
    free(sorted);
    return NSPH_OK;
}

static inline double w_of(double q, const oracle_phys_f64* ph)
{
    const double t = 1.0 - q;
    return ph->sigma * (q <= 0.5 ? 6.0 * q * q * (q - 1.0) + 1.0 : (q < 1.0 ? 2.0 * t * t * t : 0.0));
}

/* F = (dW/dr)/r and dF/dr */
static inline void f_of(double r, const oracle_phys_f64* ph, double* F, double* dF)
{
    const double q = r * ph->inv_h, t = 1.0 - q;
    if (q <= 0.5) {
        *F = ph->c_near * (3.0 * q - 2.0);
        *dF = 3.0 * ph->c_near * ph->inv_h;
    } else if (q < 1.0) {
        *F = ph->c_far * t * t / r;
        *dF = -ph->c_far * t * (2.0 * ph->inv_h / r + t / (r * r));
    } else {
        *F = 0.0;
        *dF = 0.0;
    }
}

/* per-particle intermediates of one forward step */
typedef struct adj_fwd {
    double *rho, *prs, *praw, *pr2, *mor, *a, *dv, *u;
} adj_fwd;

static void free_fwd(adj_fwd* F)
{
    free(F->rho);
    free(F->prs);
    free(F->praw);
    free(F->pr2);
    free(F->mor);
    free(F->a);
    free(F->dv);
    free(F->u);
}

static int gravity_row(const int* world, int i, int world_count)
{
    int w = world ? world[i] : 0;
    if (w < 0) w = 0;
    if (w >= world_count) w = world_count - 1;
    return w;
}

static int forward(const oracle_phys_f64* ph, int n, const double* x, const double* v, const double* f_ext,
                   const double* mass, const double* inv_mass, const int* flags, const int* world,
                   const double* gravity, int world_count, const adj_lists* L, adj_fwd* F, double* x_out,
                   double* v_out)
{
    const size_t s1 = sizeof(double) * (size_t)(n > 0 ? n : 1), s3 = 3 * s1;
    F->rho = (double*)calloc(1, s1);
    F->prs = (double*)calloc(1, s1);
    F->praw = (double*)calloc(1, s1);
    F->pr2 = (double*)calloc(1, s1);
    F->mor = (double*)calloc(1, s1);
    F->a = (double*)calloc(1, s3);
    F->dv = (double*)calloc(1, s3);
    F->u = (double*)calloc(1, s3);
    if (!F->rho || !F->prs || !F->praw || !F->pr2 || !F->mor || !F->a || !F->dv || !F->u) return NSPH_ERR_OUT_OF_MEMORY;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
        if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) continue;
        const double* xi = x + 3 * (size_t)i;
        double rho = mass[i] * ph->sigma; /* self term, W(0) = sigma */
        for (long long t = L->off[i]; t < L->off[i + 1]; ++t) {
            const int j = L->ids[t];
            const double* xj = x + 3 * (size_t)j;
            const double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
            rho += mass[j] * w_of(sqrt(dx * dx + dy * dy + dz * dz) * ph->inv_h, ph);
        }
        F->rho[i] = rho;
        if (rho > 0.0) {
            const double raw = ph->eos_b * (pow(rho * ph->inv_rho0, ph->eos_gamma) - 1.0);
            F->praw[i] = raw;
            F->prs[i] = (ph->clamp_pressure && raw < 0.0) ? 0.0 : raw;
            F->pr2[i] = F->prs[i] / (rho * rho);
            F->mor[i] = mass[i] / rho;
        }
    }
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
        const double* xi = x + 3 * (size_t)i;
        const double* vi = v + 3 * (size_t)i;
        if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) {
            for (int c = 0; c < 3; ++c) {
                x_out[3 * (size_t)i + c] = xi[c];
                v_out[3 * (size_t)i + c] = vi[c];
            }
            continue;
        }
        double a[3] = {0, 0, 0}, dv[3] = {0, 0, 0};
        for (long long t = L->off[i]; t < L->off[i + 1]; ++t) {
            const int j = L->ids[t];
            const double* xj = x + 3 * (size_t)j;
            const double* vj = v + 3 * (size_t)j;
            const double d[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            const double w = w_of(r * ph->inv_h, ph);
            if (r > 0.0) {
                double Fk, dF;
                f_of(r, ph, &Fk, &dF);
                const double s = mass[j] * (F->pr2[i] + F->pr2[j]) * Fk;
                for (int c = 0; c < 3; ++c) a[c] -= s * d[c];
            }
            for (int c = 0; c < 3; ++c) dv[c] += F->mor[j] * w * (vj[c] - vi[c]);
        }
        const double wi = inv_mass[i];
        double u[3] = {vi[0], vi[1], vi[2]};
        if (wi > 0.0) {
            const double* g = gravity + 3 * (size_t)gravity_row(world, i, world_count);
            for (int c = 0; c < 3; ++c) {
                const double fe = f_ext ? f_ext[3 * (size_t)i + c] * wi : 0.0;
                u[c] = vi[c] + (a[c] + fe + g[c]) * ph->dt + ph->xsph_eps * dv[c];
            }
        }
        for (int c = 0; c < 3; ++c) {
            F->a[3 * (size_t)i + c] = a[c];
            F->dv[3 * (size_t)i + c] = dv[c];
            F->u[3 * (size_t)i + c] = u[c];
        }
        double v1[3] = {u[0], u[1], u[2]};
        const double vm = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        if (vm > ph->v_max)
            for (int c = 0; c < 3; ++c) v1[c] = u[c] * (ph->v_max / vm);
        double x1[3];
        for (int c = 0; c < 3; ++c) x1[c] = xi[c] + v1[c] * ph->dt;
        if (wi > 0.0 && ph->use_box)
            for (int c = 0; c < 3; ++c) {
                if (x1[c] < ph->box_lo[c]) {
                    x1[c] = ph->box_lo[c];
                    if (v1[c] < 0.0) v1[c] = 0.0;
                }
                if (x1[c] > ph->box_hi[c]) {
                    x1[c] = ph->box_hi[c];
                    if (v1[c] > 0.0) v1[c] = 0.0;
                }
            }
        for (int c = 0; c < 3; ++c) {
            x_out[3 * (size_t)i + c] = x1[c];
            v_out[3 * (size_t)i + c] = v1[c];
        }
    }
    return NSPH_OK;
}

int oracle_adj_step_f64(const oracle_phys_f64* ph, int n, const double* x, const double* v, const double* f_ext,
                        const double* mass, const double* inv_mass, const int* flags, const int* world,
                        const double* gravity, int world_count, double* x_out, double* v_out, double* rho_out)
{
    if (!ph || n < 0 || world_count < 1) return NSPH_ERR_INVALID_ARG;
    if (n == 0) return NSPH_OK;
    adj_lists L;
    int st = build_lists(ph, n, x, flags, &L);
    if (st != NSPH_OK) return st;
    adj_fwd F;
    memset(&F, 0, sizeof(F));
    st = forward(ph, n, x, v, f_ext, mass, inv_mass, flags, world, gravity, world_count, &L, &F, x_out, v_out);
    if (st == NSPH_OK && rho_out) memcpy(rho_out, F.rho, sizeof(double) * (size_t)n);
    free_fwd(&F);
    free_lists(&L);
    return st;
}

int oracle_adj_vjp_f64(const oracle_phys_f64* ph, int n, const double* x, const double* v, const double* f_ext,
                       const double* mass, const double* inv_mass, const int* flags, const int* world,
                       const double* gravity, int world_count, const double* x_out_adj, const double* v_out_adj,
                       const double* rho_out_adj, double* x_adj, double* v_adj, double* f_adj, double* b_adj)
{
    if (!ph || n < 0 || world_count < 1 || !x_out_adj || !v_out_adj || !x_adj || !v_adj) return NSPH_ERR_INVALID_ARG;
    if (b_adj) *b_adj = 0.0;
    if (n == 0) return NSPH_OK;
    adj_lists L;
    int st = build_lists(ph, n, x, flags, &L);
    if (st != NSPH_OK) return st;
    adj_fwd F;
    memset(&F, 0, sizeof(F));
    const size_t s1 = sizeof(double) * (size_t)n;
    double* xo = (double*)malloc(3 * s1);
    double* vo = (double*)malloc(3 * s1);
    double* G = (double*)calloc(3, s1);     /* adjoint of a_i   */
    double* D = (double*)calloc(3, s1);     /* adjoint of dv_i  */
    double* pr2b = (double*)calloc(1, s1);  /* adjoint of p/rho^2 */
    double* morb = (double*)calloc(1, s1);  /* adjoint of m/rho */
    double* rhob = (double*)calloc(1, s1);  /* adjoint of rho   */
    if (!xo || !vo || !G || !D || !pr2b || !morb || !rhob) st = NSPH_ERR_OUT_OF_MEMORY;
    if (st == NSPH_OK)
        st = forward(ph, n, x, v, f_ext, mass, inv_mass, flags, world, gravity, world_count, &L, &F, xo, vo);
    if (st != NSPH_OK) goto done;

    /* (1) integrate, reversed particle by particle */
    for (int i = 0; i < n; ++i) {
        const double* xb1 = x_out_adj + 3 * (size_t)i;
        const double* vb1 = v_out_adj + 3 * (size_t)i;
        if (f_adj)
            for (int c = 0; c < 3; ++c) f_adj[3 * (size_t)i + c] = 0.0;
        if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) {
            for (int c = 0; c < 3; ++c) {
                x_adj[3 * (size_t)i + c] = xb1[c];
                v_adj[3 * (size_t)i + c] = vb1[c];
            }
            continue;
        }
        const double* xi = x + 3 * (size_t)i;
        const double* u = F.u + 3 * (size_t)i;
        const double wi = inv_mass[i];
        const double vm = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        const int vclamp = vm > ph->v_max;
        double vc[3], xp[3];
        for (int c = 0; c < 3; ++c) {
            vc[c] = vclamp ? u[c] * (ph->v_max / vm) : u[c];
            xp[c] = xi[c] + vc[c] * ph->dt;
        }
        double xpb[3], vcb[3];
        for (int c = 0; c < 3; ++c) {
            xpb[c] = xb1[c];
            vcb[c] = vb1[c];
            if (wi > 0.0 && ph->use_box) {
                if (xp[c] < ph->box_lo[c]) {
                    xpb[c] = 0.0;
                    if (vc[c] < 0.0) vcb[c] = 0.0;
                } else if (xp[c] > ph->box_hi[c]) {
                    xpb[c] = 0.0;
                    if (vc[c] > 0.0) vcb[c] = 0.0;
                }
            }
        }
        double ub[3];
        for (int c = 0; c < 3; ++c) {
            x_adj[3 * (size_t)i + c] = xpb[c];
            vcb[c] += xpb[c] * ph->dt;
        }
        if (vclamp) {
            const double uh[3] = {u[0] / vm, u[1] / vm, u[2] / vm};
            const double dot = uh[0] * vcb[0] + uh[1] * vcb[1] + uh[2] * vcb[2];
            for (int c = 0; c < 3; ++c) ub[c] = (ph->v_max / vm) * (vcb[c] - uh[c] * dot);
        } else {
            for (int c = 0; c < 3; ++c) ub[c] = vcb[c];
        }
        for (int c = 0; c < 3; ++c) {
            v_adj[3 * (size_t)i + c] = ub[c];
            if (wi > 0.0) {
                G[3 * (size_t)i + c] = ub[c] * ph->dt;
                D[3 * (size_t)i + c] = ub[c] * ph->xsph_eps;
                if (f_adj && f_ext) f_adj[3 * (size_t)i + c] = ub[c] * ph->dt * wi;
            }
        }
    }

    /* (2) pressure and XSPH terms, each pair term transposed into both particles */
    for (int i = 0; i < n; ++i) {
        if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) continue;
        const double* xi = x + 3 * (size_t)i;
        const double* vi = v + 3 * (size_t)i;
        const double* Gi = G + 3 * (size_t)i;
        const double* Di = D + 3 * (size_t)i;
        for (long long t = L.off[i]; t < L.off[i + 1]; ++t) {
            const int j = L.ids[t];
            const double* xj = x + 3 * (size_t)j;
            const double* vj = v + 3 * (size_t)j;
            const double d[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            const double w = w_of(r * ph->inv_h, ph);
            double Fk = 0.0, dF = 0.0;
            if (r > 0.0) f_of(r, ph, &Fk, &dF);
            /* a_i -= m_j (pr2_i + pr2_j) F(r) d */
            if (r > 0.0) {
                const double S = F.pr2[i] + F.pr2[j];
                const double gd = Gi[0] * d[0] + Gi[1] * d[1] + Gi[2] * d[2];
                pr2b[i] -= mass[j] * Fk * gd;
                pr2b[j] -= mass[j] * Fk * gd;
                /* d/dd of F(|d|) d is F I + (F'/r) d d^T */
                for (int c = 0; c < 3; ++c) {
                    const double gx = -mass[j] * S * (Fk * Gi[c] + (dF / r) * d[c] * gd);
                    x_adj[3 * (size_t)i + c] += gx;
                    x_adj[3 * (size_t)j + c] -= gx;
                }
            }
            /* dv_i += mor_j W(r) (v_j - v_i) */
            double dvd = 0.0;
            for (int c = 0; c < 3; ++c) dvd += Di[c] * (vj[c] - vi[c]);
            morb[j] += w * dvd;
            for (int c = 0; c < 3; ++c) {
                v_adj[3 * (size_t)j + c] += F.mor[j] * w * Di[c];
                v_adj[3 * (size_t)i + c] -= F.mor[j] * w * Di[c];
                /* dW/dd = F d */
                const double gx = F.mor[j] * dvd * Fk * d[c];
                x_adj[3 * (size_t)i + c] += gx;
                x_adj[3 * (size_t)j + c] -= gx;
            }
        }
    }

    /* (3) equation of state and the m/rho, p/rho^2 factors */
    {
        double bsum = 0.0;
        for (int i = 0; i < n; ++i) {
            if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) continue;
            double rb = rho_out_adj ? rho_out_adj[i] : 0.0;
            const double rho = F.rho[i];
            if (rho > 0.0) {
                const double ratio = rho * ph->inv_rho0;
                const int live = !(ph->clamp_pressure && F.praw[i] < 0.0);
                const double dp = live ? ph->eos_b * ph->eos_gamma * pow(ratio, ph->eos_gamma - 1) * ph->inv_rho0 : 0.0;
                rb += pr2b[i] * (dp / (rho * rho) - 2.0 * F.prs[i] / (rho * rho * rho));
                rb -= morb[i] * mass[i] / (rho * rho);
                if (live) bsum += pr2b[i] * (pow(ratio, ph->eos_gamma) - 1.0) / (rho * rho);
            }
            rhob[i] = rb;
        }
        if (b_adj) *b_adj = bsum;
    }

    /* (4) density sum: rho_i += m_j W(r_ij) */
    for (int i = 0; i < n; ++i) {
        if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) continue;
        const double* xi = x + 3 * (size_t)i;
        for (long long t = L.off[i]; t < L.off[i + 1]; ++t) {
            const int j = L.ids[t];
            const double* xj = x + 3 * (size_t)j;
            const double d[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (!(r > 0.0)) continue;
            double Fk, dF;
            f_of(r, ph, &Fk, &dF);
            for (int c = 0; c < 3; ++c) {
                const double gx = rhob[i] * mass[j] * Fk * d[c];
                x_adj[3 * (size_t)i + c] += gx;
                x_adj[3 * (size_t)j + c] -= gx;
            }
        }
    }

done:
    free(xo);
    free(vo);
    free(G);
    free(D);
    free(pr2b);
    free(morb);
    free(rhob);
    free_fwd(&F);
    free_lists(&L);
    return st;
}
