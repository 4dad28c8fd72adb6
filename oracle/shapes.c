/*
 * shapes.c — particles against static analytic shapes and the XPBD particle
 * update, restated in fp32. TEST INFRASTRUCTURE ONLY (the checker; see
 * nsph_oracle.h).
 *
 * Restates, operation by operation, for shapes without a body (identity
 * body transform, zero body velocity):
 *   create_soft_contacts              newton/_src/geometry/kernels.py:1001-1140
 *     with sdf_sphere / sdf_box / sdf_capsule / sdf_cylinder / sdf_cone /
 *     sdf_ellipsoid / sdf_plane and their gradients (:132-600; capsules,
 *     cylinders and cones along local +Z), contacts in (particle, shape)
 *     order
 *   eval_particle_body_contact        newton/_src/solvers/semi_implicit/kernels_contact.py:143-262
 *   solve_particle_shape_contacts     newton/_src/solvers/xpbd/kernels.py:115-222
 *   apply_particle_shape_restitution  newton/_src/solvers/xpbd/kernels.py:34-112
 *   apply_particle_deltas             newton/_src/solvers/xpbd/kernels.py:777-808
 * Contacts are processed sequentially in contact order and accumulated into
 * their particle in that order (the reference's atomic adds, serialised).
 * fp32, every operation rounded as written (-ffp-contract=off); dot
 * products are ((x + y) + z); quaternion rotation is
 * v (2w^2 - 1) + (u x v) 2w + u (u.v) 2.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "nsph_oracle.h"

typedef struct { float x, y, z; } v3;

static inline v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 divs(v3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
static inline float dot(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline v3 cross(v3 a, v3 b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float len(v3 a) { return sqrtf(dot(a, a)); }
static inline v3 normalize(v3 a)
{
    const float l = len(a);
    return l > 0.0f ? divs(a, l) : mk(0.0f, 0.0f, 0.0f);
}
static inline v3 ld(const float* p, size_t i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
static inline void st(float* p, size_t i, v3 a)
{
    p[3 * i] = a.x;
    p[3 * i + 1] = a.y;
    p[3 * i + 2] = a.z;
}

static inline v3 qrot(v3 u, float w, v3 v)
{
    const float c = (2.0f * w) * w - 1.0f;
    const v3 a = mul(v, c);
    const v3 b = mul(mul(cross(u, v), w), 2.0f);
    const v3 d = mul(mul(u, dot(u, v)), 2.0f);
    return add(add(a, b), d);
}

static inline float sgn(float v) { return v < 0.0f ? -1.0f : 1.0f; }
static inline float len2(float a, float b) { return sqrtf(a * a + b * b); }
static inline v3 unit_or(v3 v, v3 fallback)
{
    const float l = len(v);
    return l > 1.0e-8f ? divs(v, l) : fallback;
}

/* _sdf_capped_cone_z (kernels.py:141-161): bottom radius rb at z = -hh, top rt at +hh */
static float capped_cone_z(float rb, float rt, float hh, v3 x)
{
    const float qx = len2(x.x, x.y), qy = x.z;
    const float k1x = rt, k1y = hh, k2x = rt - rb, k2y = 2.0f * hh;
    const float cax = qx - fminf(qx, qy < 0.0f ? rb : rt), cay = fabsf(qy) - hh;
    const float denom = k2x * k2x + k2y * k2y;
    float t = 0.0f;
    if (denom > 0.0f) t = fminf(fmaxf(((k1x - qx) * k2x + (k1y - qy) * k2y) / denom, 0.0f), 1.0f);
    const float cbx = (qx - k1x) + k2x * t, cby = (qy - k1y) + k2y * t;
    const float sign = (cbx < 0.0f && cay < 0.0f) ? -1.0f : 1.0f;
    return sign * sqrtf(fminf(cax * cax + cay * cay, cbx * cbx + cby * cby));
}

static int sdf(const nsph_shape* s, v3 x, float* d, v3* n)
{
    if (s->type == NSPH_GEO_CAPSULE) { /* sdf_capsule / _grad, kernels.py:262-329 */
        const float r = s->scale[0], hh = s->scale[1];
        v3 v, fb;
        if (x.z > hh) {
            v = mk(x.x, x.y, x.z - hh);
            fb = mk(0.0f, 0.0f, 1.0f);
        } else if (x.z < -hh) {
            v = mk(x.x, x.y, x.z + hh);
            fb = mk(0.0f, 0.0f, -1.0f);
        } else {
            v = mk(x.x, x.y, 0.0f);
            fb = mk(0.0f, 0.0f, 1.0f);
        }
        *d = len(v) - r;
        *n = unit_or(v, fb);
        return 1;
    }
    if (s->type == NSPH_GEO_CYLINDER) { /* sdf_cylinder / _grad, kernels.py:332-446 */
        const float r = s->scale[0], hh = s->scale[1];
        const v3 v = mk(x.x, x.y, 0.0f);
        const float vl = len(v);
        const float dx = vl - r, dy = fabsf(x.z) - hh;
        *d = fminf(fmaxf(dx, dy), 0.0f) + len2(fmaxf(dx, 0.0f), fmaxf(dy, 0.0f));
        const v3 radial = vl > 1.0e-8f ? divs(v, vl) : mk(0.0f, 0.0f, 1.0f);
        const v3 axial = mk(0.0f, 0.0f, sgn(x.z));
        if (dx > 0.0f && dy > 0.0f)
            *n = unit_or(add(mul(radial, dx), mul(axial, dy)), radial);
        else
            *n = dx > dy ? radial : axial;
        return 1;
    }
    if (s->type == NSPH_GEO_CONE) { /* sdf_cone / _grad, kernels.py:515-565 */
        const float r = s->scale[0], hh = s->scale[1];
        *d = capped_cone_z(r, 0.0f, hh, x);
        if (hh <= 0.0f) {
            *n = mk(0.0f, 0.0f, sgn(x.z));
            return 1;
        }
        const float rl = len(mk(x.x, x.y, 0.0f));
        const float h2 = 2.0f * hh;
        const float dx = rl - (r * (hh - x.z)) / h2, dy = fabsf(x.z) - hh;
        if (dx > dy)
            *n = rl > 0.0f ? normalize(add(divs(mk(x.x, x.y, 0.0f), rl), mk(0.0f, 0.0f, r / h2)))
                           : mk(0.0f, 0.0f, 1.0f);
        else
            *n = mk(0.0f, 0.0f, sgn(x.z));
        return 1;
    }
    if (s->type == NSPH_GEO_ELLIPSOID) { /* sdf_ellipsoid / _grad, kernels.py:449-512 */
        const float e = 1.0e-8f;
        const v3 r = mk(fmaxf(fabsf(s->scale[0]), e), fmaxf(fabsf(s->scale[1]), e), fmaxf(fabsf(s->scale[2]), e));
        const v3 ir = mk(1.0f / r.x, 1.0f / r.y, 1.0f / r.z);
        const v3 ir2 = mk(ir.x * ir.x, ir.y * ir.y, ir.z * ir.z);
        const v3 q0 = mk(x.x * ir.x, x.y * ir.y, x.z * ir.z);
        const v3 q1 = mk(x.x * ir2.x, x.y * ir2.y, x.z * ir2.z);
        const float k0 = len(q0), k1 = len(q1);
        *d = k1 > e ? (k0 * (k0 - 1.0f)) / k1 : -fminf(fminf(r.x, r.y), r.z);
        *n = k1 < e ? mk(0.0f, 0.0f, 1.0f) : unit_or(mul(q1, k0 / k1), mk(0.0f, 0.0f, 1.0f));
        return 1;
    }
    if (s->type == NSPH_GEO_SPHERE) {
        const float l = len(x);
        *d = l - s->scale[0];
        *n = l > 1.0e-8f ? divs(x, l) : mk(0.0f, 0.0f, 1.0f);
        return 1;
    }
    if (s->type == NSPH_GEO_BOX) {
        const float hx = s->scale[0], hy = s->scale[1], hz = s->scale[2];
        const float qx = fabsf(x.x) - hx, qy = fabsf(x.y) - hy, qz = fabsf(x.z) - hz;
        const v3 e = mk(fmaxf(qx, 0.0f), fmaxf(qy, 0.0f), fmaxf(qz, 0.0f));
        *d = len(e) + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.0f);
        if (qx > 0.0f || qy > 0.0f || qz > 0.0f) {
            const v3 c = mk(fminf(fmaxf(x.x, -hx), hx), fminf(fmaxf(x.y, -hy), hy), fminf(fmaxf(x.z, -hz), hz));
            *n = normalize(sub(x, c));
        } else {
            const float sx = x.x < 0.0f ? -1.0f : 1.0f, sy = x.y < 0.0f ? -1.0f : 1.0f,
                        sz = x.z < 0.0f ? -1.0f : 1.0f;
            if ((qx > qy && qx > qz) || (qy == 0.0f && qz == 0.0f))
                *n = mk(sx, 0.0f, 0.0f);
            else if ((qy > qx && qy > qz) || (qx == 0.0f && qz == 0.0f))
                *n = mk(0.0f, sy, 0.0f);
            else
                *n = mk(0.0f, 0.0f, sz);
        }
        return 1;
    }
    if (s->type == NSPH_GEO_PLANE) {
        const float w = s->scale[0] * 0.5f, l = s->scale[1] * 0.5f;
        if (w > 0.0f && l > 0.0f)
            *d = fmaxf(fmaxf(fabsf(x.x) - w, fabsf(x.y) - l), fabsf(x.z));
        else
            *d = x.z;
        *n = mk(0.0f, 0.0f, 1.0f);
        return 1;
    }
    return 0;
}

static int contact(const nsph_shape* s, v3 px, float r, int pw, float margin, v3* bp, v3* nw)
{
    if (!(s->flags & (1 << 2))) return 0;
    if (pw != -1 && s->world != -1 && pw != s->world) return 0;
    const v3 p = mk(s->pos[0], s->pos[1], s->pos[2]);
    const v3 u = mk(s->rot[0], s->rot[1], s->rot[2]);
    const float w = s->rot[3];
    const v3 ui = mk(-u.x, -u.y, -u.z);
    const v3 t = qrot(ui, w, p);
    const v3 ti = mk(-t.x, -t.y, -t.z);
    const v3 xl = add(qrot(ui, w, px), ti);
    float d = 1.0e6f;
    v3 n = mk(0.0f, 0.0f, 0.0f);
    if (!sdf(s, xl, &d, &n)) return 0;
    if (!(d < margin + r)) return 0;
    *bp = add(qrot(u, w, sub(xl, mul(n, d))), p);
    *nw = qrot(u, w, n);
    return 1;
}

int oracle_soft_contacts_create(const nsph_shape* shapes, int shape_count, int n, const float* x,
                                const float* radius, const int* flags, const int* world, float margin, int max,
                                int* count, int* particle, int* shape, float* body_pos, float* body_vel,
                                float* normal)
{
    int c = 0;
    for (int p = 0; p < n; ++p) {
        if (!(flags[p] & NSPH_PARTICLE_ACTIVE)) continue;
        const v3 px = ld(x, (size_t)p);
        const int pw = world ? world[p] : -1;
        for (int s = 0; s < shape_count; ++s) {
            v3 bp, nw;
            if (!contact(&shapes[s], px, radius[p], pw, margin, &bp, &nw)) continue;
            if (c < max) {
                particle[c] = p;
                shape[c] = s;
                st(body_pos, (size_t)c, bp);
                st(body_vel, (size_t)c, mk(0.0f, 0.0f, 0.0f));
                st(normal, (size_t)c, nw);
            }
            ++c;
        }
    }
    *count = c;
    return NSPH_OK;
}

int oracle_shape_contact_forces(const nsph_shape* shapes, int count, const int* particle, const int* shape,
                                const float* body_pos, const float* body_vel, const float* normal,
                                const nsph_soft_contact_params* prm, const float* x, const float* v,
                                const float* radius, const int* flags, float* f)
{
    for (int t = 0; t < count; ++t) {
        const int p = particle[t];
        if (!(flags[p] & NSPH_PARTICLE_ACTIVE)) continue;
        const nsph_shape* s = &shapes[shape[t]];
        const v3 px = ld(x, (size_t)p), pv = ld(v, (size_t)p);
        const v3 bx = ld(body_pos, (size_t)t), n = ld(normal, (size_t)t);
        const float c = dot(n, sub(px, bx)) - radius[p];
        if (c > prm->adhesion) continue;
        const float ke = 0.5f * (prm->ke + s->ke);
        const float kd = 0.5f * (prm->kd + s->kd);
        const float kf = 0.5f * (prm->kf + s->kf);
        const float mu = 0.5f * (prm->mu + s->mu);
        const v3 vr = sub(pv, ld(body_vel, (size_t)t));
        const float vn = dot(n, vr);
        const v3 vt = sub(vr, mul(n, vn));
        const v3 fn = mul(mul(n, c), ke);
        const v3 fd = mul(mul(n, fminf(vn, 0.0f)), kd);
        const v3 ft = mul(normalize(vt), fminf(kf * len(vt), fabsf((mu * c) * ke)));
        st(f, (size_t)p, sub(ld(f, (size_t)p), add(fn, add(fd, ft))));
    }
    return NSPH_OK;
}

int oracle_shape_contact_deltas(const nsph_shape* shapes, int count, const int* particle, const int* shape,
                                const float* body_pos, const float* body_vel, const float* normal,
                                const nsph_soft_contact_params* prm, const float* x, const float* v,
                                const float* inv_mass, const float* radius, const int* flags, float* delta)
{
    for (int t = 0; t < count; ++t) {
        const int p = particle[t];
        if (!(flags[p] & NSPH_PARTICLE_ACTIVE)) continue;
        const nsph_shape* s = &shapes[shape[t]];
        const v3 px = ld(x, (size_t)p), pv = ld(v, (size_t)p);
        const v3 bx = ld(body_pos, (size_t)t), n = ld(normal, (size_t)t);
        const float c = dot(n, sub(px, bx)) - radius[p];
        if (c > prm->adhesion) continue;
        const float mu = 0.5f * (prm->mu + s->mu);
        const v3 vr = sub(pv, ld(body_vel, (size_t)t));
        const v3 delta_n = mul(n, c);
        const float vn = dot(n, vr);
        const v3 vt = sub(vr, mul(n, vn));
        const float w1 = inv_mass[p];
        const float denom = w1;
        if (denom == 0.0f) continue;
        const float lambda_f = fmaxf(mu * c, (-len(vt)) * prm->dt);
        const v3 delta_f = mul(normalize(vt), lambda_f);
        const v3 delta_total = mul(divs(sub(delta_f, delta_n), denom), prm->relaxation);
        st(delta, (size_t)p, add(ld(delta, (size_t)p), mul(delta_total, w1)));
    }
    return NSPH_OK;
}

int oracle_shape_restitution(int n, int count, const int* particle, const float* body_pos, const float* body_vel,
                             const float* normal, const nsph_soft_contact_params* prm, const float* v_new,
                             const float* x_old, const float* v_old, const float* radius, const int* flags,
                             float* v_out)
{
    /* every contact reads v_new as it was before any restitution update */
    float* vn1 = (float*)malloc(sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
    if (!vn1) return NSPH_ERR_OUT_OF_MEMORY;
    memcpy(vn1, v_new, sizeof(float) * 3 * (size_t)n);
    for (int t = 0; t < count; ++t) {
        const int p = particle[t];
        if (!(flags[p] & NSPH_PARTICLE_ACTIVE)) continue;
        const v3 px = ld(x_old, (size_t)p);
        const v3 bx = ld(body_pos, (size_t)t), nn = ld(normal, (size_t)t);
        const float c = dot(nn, sub(px, bx)) - radius[p];
        if (c > prm->adhesion) continue;
        const v3 bv = ld(body_vel, (size_t)t);
        const float rel_old = dot(nn, sub(ld(v_old, (size_t)p), bv));
        const float rel_new = dot(nn, sub(ld(vn1, (size_t)p), bv));
        if (rel_old < 0.0f) {
            const v3 dv = mul(nn, (-rel_new) + fmaxf((-prm->restitution) * rel_old, 0.0f));
            st(v_out, (size_t)p, add(ld(v_out, (size_t)p), dv));
        }
    }
    free(vn1);
    return NSPH_OK;
}

void oracle_apply_particle_deltas(int n, const float* x_orig, const float* x_pred, const int* flags,
                                  const float* delta, float dt, float v_max, float* x_out, float* v_out)
{
    for (int p = 0; p < n; ++p) {
        if (!(flags[p] & NSPH_PARTICLE_ACTIVE)) continue;
        const v3 xn = add(ld(x_pred, (size_t)p), ld(delta, (size_t)p));
        v3 vn = divs(sub(xn, ld(x_orig, (size_t)p)), dt);
        const float m = len(vn);
        if (m > v_max) vn = mul(vn, v_max / m);
        st(x_out, (size_t)p, xn);
        st(v_out, (size_t)p, vn);
    }
}
