// shapes.cu — particles against static analytic collision shapes, and the
// XPBD particle update:
//
//   nsph_soft_contacts_create            create_soft_contacts
//       (newton/_src/geometry/kernels.py:1001-1140, launched by the
//       collision pipeline, newton/_src/sim/collide.py:1194-1228) for
//       shapes of type PLANE, SPHERE, BOX, CAPSULE, CYLINDER, CONE and
//       ELLIPSOID without a body
//   nsph_particle_shape_contact_forces   eval_particle_body_contact
//       (newton/_src/solvers/semi_implicit/kernels_contact.py:143-262)
//   nsph_particle_shape_contact_deltas   solve_particle_shape_contacts
//       (newton/_src/solvers/xpbd/kernels.py:115-222)
//   nsph_particle_shape_restitution      apply_particle_shape_restitution
//       (newton/_src/solvers/xpbd/kernels.py:34-112)
//   nsph_apply_particle_deltas           apply_particle_deltas
//       (newton/_src/solvers/xpbd/kernels.py:777-808)
//
// Shapes here are static (body -1), so the body transform is the identity
// and the body velocity is zero; the per-contact arithmetic keeps the
// reference's expressions for that case.
//
// Determinism. The reference appends soft contacts with an atomic counter
// (their order depends on scheduling) and accumulates each contact into its
// particle with atomic adds. Here the contacts are written in (particle,
// shape) order by a block-ordered compaction (count per block, scan of the
// block totals, write), so a particle's contacts are consecutive, and the
// accumulating kernels walk each particle's run of contacts with one thread,
// in contact order: out[p] = ((out[p] + c_1) + c_2) + ... . Every fp32
// operation is an explicit round-to-nearest intrinsic (no contraction), so
// the CPU restatement reproduces the results bit for bit.
#include "nsph_internal.cuh"

namespace nsph {

NSPH_BOUNDS_READER(shapes)
namespace {

constexpr int kShapeThreads = 256;
constexpr int kScanMaxThreads = 1024;
constexpr int kCollideParticles = 1 << 2;  // ShapeFlags.COLLIDE_PARTICLES
constexpr int kMaxShapes = 1024;

struct V3 {
    float x, y, z;
};

__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 add(V3 a, V3 b) { return v3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return v3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
__device__ __forceinline__ V3 mul(V3 a, float s) { return v3(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)); }
__device__ __forceinline__ V3 divs(V3 a, float s) { return v3(__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s)); }
__device__ __forceinline__ float dot(V3 a, V3 b)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ V3 cross(V3 a, V3 b)
{
    return v3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
              __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float length(V3 a) { return __fsqrt_rn(dot(a, a)); }
// normalize: v / |v|, the zero vector for |v| = 0
__device__ __forceinline__ V3 normalize(V3 a)
{
    const float l = length(a);
    return l > 0.f ? divs(a, l) : v3(0.f, 0.f, 0.f);
}
__device__ __forceinline__ V3 load3(const float* p, size_t i) { return v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ void store3(float* p, size_t i, V3 a)
{
    p[3 * i] = a.x;
    p[3 * i + 1] = a.y;
    p[3 * i + 2] = a.z;
}

// rotate v by the unit quaternion (u, w): v (2w^2 - 1) + (u x v) 2w + u (u.v) 2
__device__ __forceinline__ V3 quat_rotate(V3 u, float w, V3 v)
{
    const float c = __fsub_rn(__fmul_rn(__fmul_rn(2.f, w), w), 1.f);
    const V3 a = mul(v, c);
    const V3 b = mul(mul(cross(u, v), w), 2.f);
    const V3 d = mul(mul(u, dot(u, v)), 2.f);
    return add(add(a, b), d);
}

struct Xform {
    V3 p;
    V3 u;
    float w;
};

__device__ __forceinline__ Xform shape_xform(const nsph_shape& s)
{
    return Xform{v3(s.pos[0], s.pos[1], s.pos[2]), v3(s.rot[0], s.rot[1], s.rot[2]), s.rot[3]};
}
// transform_point(X, x) = rotate(q, x) + p
__device__ __forceinline__ V3 xform_point(const Xform& X, V3 x) { return add(quat_rotate(X.u, X.w, x), X.p); }
// transform_inverse(X) = (-rotate(q*, p), q*), q* the conjugate
__device__ __forceinline__ Xform xform_inverse(const Xform& X)
{
    const V3 ui = v3(-X.u.x, -X.u.y, -X.u.z);
    const V3 t = quat_rotate(ui, X.w, X.p);
    return Xform{v3(-t.x, -t.y, -t.z), ui, X.w};
}

__device__ __forceinline__ float sgnf(float v) { return v < 0.f ? -1.f : 1.f; }
__device__ __forceinline__ float len2(float a, float b) { return __fsqrt_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b))); }
// v / |v| when |v| > 1e-8, else the fallback direction
__device__ __forceinline__ V3 unit_or(V3 v, V3 fallback)
{
    const float l = length(v);
    return l > 1.0e-8f ? divs(v, l) : fallback;
}

// signed distance of the capped cone about +Z with the given bottom (z =
// -hh) and top (z = +hh) radii (_sdf_capped_cone_z,
// newton/_src/geometry/kernels.py:141-161)
__device__ __forceinline__ float capped_cone_z(float rb, float rt, float hh, V3 x)
{
    const float qx = len2(x.x, x.y), qy = x.z;
    const float k1x = rt, k1y = hh;
    const float k2x = __fsub_rn(rt, rb), k2y = __fmul_rn(2.f, hh);
    const float cax = __fsub_rn(qx, fminf(qx, qy < 0.f ? rb : rt));
    const float cay = __fsub_rn(fabsf(qy), hh);
    const float denom = __fadd_rn(__fmul_rn(k2x, k2x), __fmul_rn(k2y, k2y));
    float t = 0.f;
    if (denom > 0.f) {
        const float num = __fadd_rn(__fmul_rn(__fsub_rn(k1x, qx), k2x), __fmul_rn(__fsub_rn(k1y, qy), k2y));
        t = fminf(fmaxf(__fdiv_rn(num, denom), 0.f), 1.f);
    }
    const float cbx = __fadd_rn(__fsub_rn(qx, k1x), __fmul_rn(k2x, t));
    const float cby = __fadd_rn(__fsub_rn(qy, k1y), __fmul_rn(k2y, t));
    const float sign = (cbx < 0.f && cay < 0.f) ? -1.f : 1.f;
    const float da = __fadd_rn(__fmul_rn(cax, cax), __fmul_rn(cay, cay));
    const float db = __fadd_rn(__fmul_rn(cbx, cbx), __fmul_rn(cby, cby));
    return __fmul_rn(sign, __fsqrt_rn(fminf(da, db)));
}

// signed distance and outward direction of a shape in its local frame
// (sdf_* / sdf_*_grad, newton/_src/geometry/kernels.py:165-600; capsules,
// cylinders and cones along local +Z as create_soft_contacts uses them)
__device__ __forceinline__ bool shape_sdf(const nsph_shape& s, V3 x, float& d, V3& n)
{
    if (s.type == NSPH_GEO_CAPSULE) {
        const float r = s.scale[0], hh = s.scale[1];
        if (x.z > hh) {
            const V3 v = v3(x.x, x.y, __fsub_rn(x.z, hh));
            d = __fsub_rn(length(v), r);
            n = unit_or(v, v3(0.f, 0.f, 1.f));
        } else if (x.z < -hh) {
            const V3 v = v3(x.x, x.y, __fadd_rn(x.z, hh));
            d = __fsub_rn(length(v), r);
            n = unit_or(v, v3(0.f, 0.f, -1.f));
        } else {
            const V3 v = v3(x.x, x.y, 0.f);
            d = __fsub_rn(length(v), r);
            n = unit_or(v, v3(0.f, 0.f, 1.f));
        }
        return true;
    }
    if (s.type == NSPH_GEO_CYLINDER) {
        const float r = s.scale[0], hh = s.scale[1];
        const V3 v = v3(x.x, x.y, 0.f);
        const float vl = length(v);
        const float dx = __fsub_rn(vl, r), dy = __fsub_rn(fabsf(x.z), hh);
        d = __fadd_rn(fminf(fmaxf(dx, dy), 0.f), len2(fmaxf(dx, 0.f), fmaxf(dy, 0.f)));
        const V3 radial = vl > 1.0e-8f ? divs(v, vl) : v3(0.f, 0.f, 1.f);
        const V3 axial = v3(0.f, 0.f, sgnf(x.z));
        if (dx > 0.f && dy > 0.f)
            n = unit_or(add(mul(radial, dx), mul(axial, dy)), radial);
        else
            n = dx > dy ? radial : axial;
        return true;
    }
    if (s.type == NSPH_GEO_CONE) {
        const float r = s.scale[0], hh = s.scale[1];
        d = capped_cone_z(r, 0.f, hh, x);
        if (hh <= 0.f) {
            n = v3(0.f, 0.f, sgnf(x.z));
            return true;
        }
        const float rl = length(v3(x.x, x.y, 0.f));
        const float h2 = __fmul_rn(2.f, hh);
        const float dx = __fsub_rn(rl, __fdiv_rn(__fmul_rn(r, __fsub_rn(hh, x.z)), h2));
        const float dy = __fsub_rn(fabsf(x.z), hh);
        if (dx > dy) {
            n = rl > 0.f ? normalize(add(divs(v3(x.x, x.y, 0.f), rl), v3(0.f, 0.f, __fdiv_rn(r, h2))))
                         : v3(0.f, 0.f, 1.f);
        } else {
            n = v3(0.f, 0.f, sgnf(x.z));
        }
        return true;
    }
    if (s.type == NSPH_GEO_ELLIPSOID) {
        const float e = 1.0e-8f;
        const V3 r = v3(fmaxf(fabsf(s.scale[0]), e), fmaxf(fabsf(s.scale[1]), e), fmaxf(fabsf(s.scale[2]), e));
        const V3 ir = v3(__fdiv_rn(1.f, r.x), __fdiv_rn(1.f, r.y), __fdiv_rn(1.f, r.z));
        const V3 ir2 = v3(__fmul_rn(ir.x, ir.x), __fmul_rn(ir.y, ir.y), __fmul_rn(ir.z, ir.z));
        const V3 q0 = v3(__fmul_rn(x.x, ir.x), __fmul_rn(x.y, ir.y), __fmul_rn(x.z, ir.z));
        const V3 q1 = v3(__fmul_rn(x.x, ir2.x), __fmul_rn(x.y, ir2.y), __fmul_rn(x.z, ir2.z));
        const float k0 = length(q0), k1 = length(q1);
        d = k1 > e ? __fdiv_rn(__fmul_rn(k0, __fsub_rn(k0, 1.f)), k1) : -fminf(fminf(r.x, r.y), r.z);
        n = k1 < e ? v3(0.f, 0.f, 1.f) : unit_or(mul(q1, __fdiv_rn(k0, k1)), v3(0.f, 0.f, 1.f));
        return true;
    }
    if (s.type == NSPH_GEO_SPHERE) {
        const float l = length(x);
        d = __fsub_rn(l, s.scale[0]);
        n = l > 1.0e-8f ? divs(x, l) : v3(0.f, 0.f, 1.f);
        return true;
    }
    if (s.type == NSPH_GEO_BOX) {
        const float hx = s.scale[0], hy = s.scale[1], hz = s.scale[2];
        const float qx = __fsub_rn(fabsf(x.x), hx), qy = __fsub_rn(fabsf(x.y), hy), qz = __fsub_rn(fabsf(x.z), hz);
        const V3 e = v3(fmaxf(qx, 0.f), fmaxf(qy, 0.f), fmaxf(qz, 0.f));
        d = __fadd_rn(length(e), fminf(fmaxf(qx, fmaxf(qy, qz)), 0.f));
        if (qx > 0.f || qy > 0.f || qz > 0.f) {
            const V3 c = v3(fminf(fmaxf(x.x, -hx), hx), fminf(fmaxf(x.y, -hy), hy), fminf(fmaxf(x.z, -hz), hz));
            n = normalize(sub(x, c));
        } else {
            auto sgn = [](float v) { return v < 0.f ? -1.f : 1.f; };
            if ((qx > qy && qx > qz) || (qy == 0.f && qz == 0.f))
                n = v3(sgn(x.x), 0.f, 0.f);
            else if ((qy > qx && qy > qz) || (qx == 0.f && qz == 0.f))
                n = v3(0.f, sgn(x.y), 0.f);
            else
                n = v3(0.f, 0.f, sgn(x.z));
        }
        return true;
    }
    if (s.type == NSPH_GEO_PLANE) {
        const float width = __fmul_rn(s.scale[0], 0.5f), len = __fmul_rn(s.scale[1], 0.5f);
        if (width > 0.f && len > 0.f) {
            const float a = fmaxf(__fsub_rn(fabsf(x.x), width), __fsub_rn(fabsf(x.y), len));
            d = fmaxf(a, fabsf(x.z));
        } else {
            d = x.z;
        }
        n = v3(0.f, 0.f, 1.f);
        return true;
    }
    return false;
}

// contact of particle (x, r, world) with shape s: true (and the contact's
// body-frame point and world normal) when d < margin + r
__device__ __forceinline__ bool shape_contact(const nsph_shape& s, V3 px, float radius, int pworld, float margin,
                                              V3& body_pos, V3& normal)
{
    if (!(s.flags & kCollideParticles)) return false;
    if (pworld != -1 && s.world != -1 && pworld != s.world) return false;
    const Xform X = shape_xform(s);
    const Xform Xi = xform_inverse(X);
    const V3 xl = xform_point(Xi, px);
    float d = 1.0e6f;
    V3 n = v3(0.f, 0.f, 0.f);
    if (!shape_sdf(s, xl, d, n)) return false;
    if (!(d < __fadd_rn(margin, radius))) return false;
    body_pos = xform_point(X, sub(xl, mul(n, d)));
    normal = quat_rotate(X.u, X.w, n);
    return true;
}

struct ContactArrays {
    int* count;
    int* particle;
    int* shape;
    float* body_pos;
    float* body_vel;
    float* normal;
    int max;
};

__device__ __forceinline__ int particle_contact_count(const nsph_shape* __restrict__ shapes, int shape_count, V3 px,
                                                      float r, int pworld, float margin)
{
    int c = 0;
    for (int s = 0; s < shape_count; ++s) {
        V3 bp, nn;
        c += shape_contact(shapes[s], px, r, pworld, margin, bp, nn);
    }
    return c;
}

// exclusive scan of one value per thread over the block; returns the block total
__device__ __forceinline__ int block_exclusive_scan(int v, int& total)
{
    __shared__ int warp_sums[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        int w = lane < nw ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        warp_sums[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    total = warp_sums[((blockDim.x + 31) >> 5) - 1];
    const int base = warp > 0 ? warp_sums[warp - 1] : 0;
    __syncthreads();
    return base + inc - v;
}

__device__ __forceinline__ bool particle_active(const int* flags, int p) { return (flags[p] & 1) != 0; }

// pass 1: contacts per block of particles
__global__ void k_soft_count(const nsph_shape* __restrict__ shapes, int shape_count, int n, const float* __restrict__ x,
                             const float* __restrict__ radius, const int* __restrict__ flags,
                             const int* __restrict__ world, float margin, int* __restrict__ block_counts)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    int c = 0;
    if (p < n && particle_active(flags, p))
        c = particle_contact_count(shapes, shape_count, load3(x, p), radius[p], world ? world[p] : -1, margin);
    int total = 0;
    block_exclusive_scan(c, total);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = total;
}

// pass 2 (one block): exclusive scan of the block totals in place, and the
// contact count (soft_contact_count[0], the total before the max clamp)
__global__ void k_soft_scan(int* __restrict__ block_counts, int blocks, int* __restrict__ count)
{
    const int per = (blocks + blockDim.x - 1) / blockDim.x;
    const int lo = threadIdx.x * per, hi = min(lo + per, blocks);
    int s = 0;
    for (int b = lo; b < hi; ++b) s += block_counts[b];
    int total = 0;
    const int base = block_exclusive_scan(s, total);
    int run = base;
    for (int b = lo; b < hi; ++b) {
        const int v = block_counts[b];
        block_counts[b] = run;
        run += v;
    }
    if (threadIdx.x == 0) count[0] = total;
}

// pass 3: every particle writes its contacts (shape order) at its offset
__global__ void k_soft_write(const nsph_shape* __restrict__ shapes, int shape_count, int n,
                             const float* __restrict__ x, const float* __restrict__ radius,
                             const int* __restrict__ flags, const int* __restrict__ world, float margin,
                             const int* __restrict__ block_offsets, ContactArrays out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = p < n && particle_active(flags, p);
    V3 px = v3(0.f, 0.f, 0.f);
    float r = 0.f;
    int pw = -1, c = 0;
    if (live) {
        px = load3(x, p);
        r = radius[p];
        pw = world ? world[p] : -1;
        c = particle_contact_count(shapes, shape_count, px, r, pw, margin);
    }
    int total = 0;
    int idx = block_offsets[blockIdx.x] + block_exclusive_scan(c, total);
    if (!c) return;
    for (int s = 0; s < shape_count && idx < out.max; ++s) {
        V3 bp, nn;
        if (!shape_contact(shapes[s], px, r, pw, margin, bp, nn)) continue;
        out.particle[idx] = p;
        out.shape[idx] = s;
        store3(out.body_pos, idx, bp);
        store3(out.body_vel, idx, v3(0.f, 0.f, 0.f));
        store3(out.normal, idx, nn);
        ++idx;
    }
}

struct ContactView {
    const int* count;
    const int* particle;
    const int* shape;
    const float* body_pos;
    const float* body_vel;
    const float* normal;
    int max;
};

__device__ __forceinline__ int contact_total(const ContactView& c) { return min(c.max, c.count[0]); }

// true for the first contact of a particle's run (whose thread walks the run)
__device__ __forceinline__ bool run_head(const ContactView& c, int t, int total, int& p)
{
    if (t >= total) return false;
    p = c.particle[t];
    return t == 0 || c.particle[t - 1] != p;
}

// eval_particle_body_contact for a static shape (body velocity zero):
// f[p] -= fn + (fd + ft)
__global__ void k_shape_forces(const nsph_shape* __restrict__ shapes, ContactView c, nsph_soft_contact_params prm,
                               const float* __restrict__ x, const float* __restrict__ v,
                               const float* __restrict__ radius, const int* __restrict__ flags, float* __restrict__ f)
{
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int total = contact_total(c);
    int p = 0;
    if (!run_head(c, t0, total, p)) return;
    if (!particle_active(flags, p)) return;
    const V3 px = load3(x, p), pv = load3(v, p);
    const float rad = radius[p];
    V3 acc = load3(f, p);
    for (int t = t0; t < total && c.particle[t] == p; ++t) {
        const nsph_shape& s = shapes[c.shape[t]];
        const V3 bx = load3(c.body_pos, t);
        const V3 n = load3(c.normal, t);
        const float cc = __fsub_rn(dot(n, sub(px, bx)), rad);
        if (cc > prm.adhesion) continue;
        const float ke = __fmul_rn(0.5f, __fadd_rn(prm.ke, s.ke));
        const float kd = __fmul_rn(0.5f, __fadd_rn(prm.kd, s.kd));
        const float kf = __fmul_rn(0.5f, __fadd_rn(prm.kf, s.kf));
        const float mu = __fmul_rn(0.5f, __fadd_rn(prm.mu, s.mu));
        const V3 bv = load3(c.body_vel, t);
        const V3 vr = sub(pv, bv);
        const float vn = dot(n, vr);
        const V3 vt = sub(vr, mul(n, vn));
        const V3 fn = mul(mul(n, cc), ke);
        const V3 fd = mul(mul(n, fminf(vn, 0.f)), kd);
        const V3 ft = mul(normalize(vt), fminf(__fmul_rn(kf, length(vt)), fabsf(__fmul_rn(__fmul_rn(mu, cc), ke))));
        acc = sub(acc, add(fn, add(fd, ft)));
    }
    store3(f, p, acc);
}

// solve_particle_shape_contacts for a static shape: delta[p] += w1 * delta_total
__global__ void k_shape_deltas(const nsph_shape* __restrict__ shapes, ContactView c, nsph_soft_contact_params prm,
                               const float* __restrict__ x, const float* __restrict__ v,
                               const float* __restrict__ inv_mass, const float* __restrict__ radius,
                               const int* __restrict__ flags, float* __restrict__ delta)
{
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int total = contact_total(c);
    int p = 0;
    if (!run_head(c, t0, total, p)) return;
    if (!particle_active(flags, p)) return;
    const V3 px = load3(x, p), pv = load3(v, p);
    const float rad = radius[p];
    const float w1 = inv_mass[p];
    V3 acc = load3(delta, p);
    for (int t = t0; t < total && c.particle[t] == p; ++t) {
        const nsph_shape& s = shapes[c.shape[t]];
        const V3 bx = load3(c.body_pos, t);
        const V3 n = load3(c.normal, t);
        const float cc = __fsub_rn(dot(n, sub(px, bx)), rad);
        if (cc > prm.adhesion) continue;
        const float mu = __fmul_rn(0.5f, __fadd_rn(prm.mu, s.mu));
        const V3 bv = load3(c.body_vel, t);
        const V3 vr = sub(pv, bv);
        const float lambda_n = cc;
        const V3 delta_n = mul(n, lambda_n);
        const float vn = dot(n, vr);
        const V3 vt = sub(vr, mul(n, vn));
        const float denom = w1;  // w1 + w2 with w2 = 0 for a static shape
        if (denom == 0.f) continue;
        const float lambda_f = fmaxf(__fmul_rn(mu, lambda_n), __fmul_rn(-length(vt), prm.dt));
        const V3 delta_f = mul(normalize(vt), lambda_f);
        const V3 delta_total = mul(divs(sub(delta_f, delta_n), denom), prm.relaxation);
        acc = add(acc, mul(delta_total, w1));
    }
    store3(delta, p, acc);
}

// apply_particle_shape_restitution for a static shape: v_out[p] += dv; every
// contact of p reads v_new[p] as it was before this kernel
__global__ void k_shape_restitution(ContactView c, nsph_soft_contact_params prm, const float* __restrict__ v_new,
                                    const float* __restrict__ x_old, const float* __restrict__ v_old,
                                    const float* __restrict__ radius, const int* __restrict__ flags,
                                    float* __restrict__ v_out)
{
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int total = contact_total(c);
    int p = 0;
    if (!run_head(c, t0, total, p)) return;
    if (!particle_active(flags, p)) return;
    const V3 vn1 = load3(v_new, p), px = load3(x_old, p), v0 = load3(v_old, p);
    const float rad = radius[p];
    V3 acc = load3(v_out, p);
    for (int t = t0; t < total && c.particle[t] == p; ++t) {
        const V3 bx = load3(c.body_pos, t);
        const V3 n = load3(c.normal, t);
        const float cc = __fsub_rn(dot(n, sub(px, bx)), rad);
        if (cc > prm.adhesion) continue;
        const V3 bv = load3(c.body_vel, t);
        const float rel_old = dot(n, sub(v0, bv));
        const float rel_new = dot(n, sub(vn1, bv));
        if (rel_old < 0.f) {
            const V3 dv = mul(n, __fadd_rn(-rel_new, fmaxf(__fmul_rn(-prm.restitution, rel_old), 0.f)));
            acc = add(acc, dv);
        }
    }
    store3(v_out, p, acc);
}

// apply_particle_deltas: x = x_pred + delta, v = (x - x0)/dt clamped to v_max
__global__ void k_apply_deltas(int n, const float* __restrict__ x_orig, const float* __restrict__ x_pred,
                               const int* __restrict__ flags, const float* __restrict__ delta, float dt, float v_max,
                               float* __restrict__ x_out, float* __restrict__ v_out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n || !particle_active(flags, p)) return;
    const V3 x0 = load3(x_orig, p);
    const V3 xn = add(load3(x_pred, p), load3(delta, p));
    V3 vn = divs(sub(xn, x0), dt);
    const float m = length(vn);
    if (m > v_max) vn = mul(vn, __fdiv_rn(v_max, m));
    store3(x_out, p, xn);
    store3(v_out, p, vn);
}

int check_shapes(const nsph_shape* shapes, int shape_count)
{
    if (shape_count < 0 || shape_count > kMaxShapes)
        return fail(NSPH_ERR_INVALID_ARG, "shape_count must be in [0, " + std::to_string(kMaxShapes) + "]");
    if (shape_count > 0 && !shapes) return fail(NSPH_ERR_INVALID_ARG, "null shapes");
    return NSPH_OK;
}

int check_contacts(const nsph_soft_contacts* c)
{
    if (!c) return fail(NSPH_ERR_INVALID_ARG, "null contacts");
    if (c->max < 0) return fail(NSPH_ERR_INVALID_ARG, "negative soft_contact_max");
    if (!c->count) return fail(NSPH_ERR_INVALID_ARG, "null contact count");
    if (c->max > 0 && (!c->particle || !c->shape || !c->body_pos || !c->body_vel || !c->normal))
        return fail(NSPH_ERR_INVALID_ARG, "null contact array");
    return NSPH_OK;
}

ContactView view_of(const nsph_soft_contacts* c)
{
    return ContactView{c->count, c->particle, c->shape, c->body_pos, c->body_vel, c->normal, c->max};
}

int contact_blocks(const nsph_soft_contacts* c) { return std::max(1, (c->max + kShapeThreads - 1) / kShapeThreads); }

}  // namespace
}  // namespace nsph

using namespace nsph;

extern "C" int nsph_soft_contacts_scratch_ints(int num_particles)
{
    return std::max(1, (std::max(num_particles, 0) + kShapeThreads - 1) / kShapeThreads);
}

extern "C" int nsph_soft_contacts_create(const nsph_shape* shapes, int shape_count, int n, const float* x,
                                         const float* radius, const int* flags, const int* world, float margin,
                                         nsph_soft_contacts* contacts, int* scratch, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_soft_contacts_create");
    int st = check_shapes(shapes, shape_count);
    if (st != NSPH_OK) return st;
    st = check_contacts(contacts);
    if (st != NSPH_OK) return st;
    if (n < 0) return fail(NSPH_ERR_INVALID_ARG, "negative particle count");
    if (n > 0 && (!x || !radius || !flags)) return fail(NSPH_ERR_INVALID_ARG, "null particle array");
    if (!scratch) return fail(NSPH_ERR_INVALID_ARG, "null scratch");
    cudaStream_t cs = (cudaStream_t)stream;
    if (n == 0 || shape_count == 0) {
        NSPH_CUDA_TRY(cudaMemsetAsync(contacts->count, 0, sizeof(int), cs));
        return NSPH_OK;
    }
    const int blocks = (n + kShapeThreads - 1) / kShapeThreads;
    k_soft_count<<<blocks, kShapeThreads, 0, cs>>>(shapes, shape_count, n, x, radius, flags, world, margin, scratch);
    NSPH_LAUNCH_CHECK("k_soft_count");
    k_soft_scan<<<1, kScanMaxThreads, 0, cs>>>(scratch, blocks, contacts->count);
    NSPH_LAUNCH_CHECK("k_soft_scan");
    ContactArrays out{contacts->count, contacts->particle, contacts->shape, contacts->body_pos, contacts->body_vel,
                      contacts->normal, contacts->max};
    k_soft_write<<<blocks, kShapeThreads, 0, cs>>>(shapes, shape_count, n, x, radius, flags, world, margin, scratch,
                                                   out);
    NSPH_LAUNCH_CHECK("k_soft_write");
    return NSPH_OK;
}

extern "C" int nsph_particle_shape_contact_forces(const nsph_shape* shapes, int shape_count,
                                                  const nsph_soft_contacts* contacts,
                                                  const nsph_soft_contact_params* params, const float* x,
                                                  const float* v, const float* radius, const int* flags, float* f,
                                                  void* stream)
{
    clear_error();
    int st = check_shapes(shapes, shape_count);
    if (st != NSPH_OK) return st;
    st = check_contacts(contacts);
    if (st != NSPH_OK) return st;
    if (!params) return fail(NSPH_ERR_INVALID_ARG, "null params");
    if (contacts->max == 0 || shape_count == 0) return NSPH_OK;
    if (!x || !v || !radius || !flags || !f) return fail(NSPH_ERR_INVALID_ARG, "null particle array");
    k_shape_forces<<<contact_blocks(contacts), kShapeThreads, 0, (cudaStream_t)stream>>>(
        shapes, view_of(contacts), *params, x, v, radius, flags, f);
    NSPH_LAUNCH_CHECK("k_shape_forces");
    return NSPH_OK;
}

extern "C" int nsph_particle_shape_contact_deltas(const nsph_shape* shapes, int shape_count,
                                                  const nsph_soft_contacts* contacts,
                                                  const nsph_soft_contact_params* params, const float* x,
                                                  const float* v, const float* inv_mass, const float* radius,
                                                  const int* flags, float* deltas, void* stream)
{
    clear_error();
    int st = check_shapes(shapes, shape_count);
    if (st != NSPH_OK) return st;
    st = check_contacts(contacts);
    if (st != NSPH_OK) return st;
    if (!params) return fail(NSPH_ERR_INVALID_ARG, "null params");
    if (contacts->max == 0 || shape_count == 0) return NSPH_OK;
    if (!x || !v || !inv_mass || !radius || !flags || !deltas) return fail(NSPH_ERR_INVALID_ARG, "null particle array");
    k_shape_deltas<<<contact_blocks(contacts), kShapeThreads, 0, (cudaStream_t)stream>>>(
        shapes, view_of(contacts), *params, x, v, inv_mass, radius, flags, deltas);
    NSPH_LAUNCH_CHECK("k_shape_deltas");
    return NSPH_OK;
}

extern "C" int nsph_particle_shape_restitution(const nsph_soft_contacts* contacts,
                                               const nsph_soft_contact_params* params, const float* v_new,
                                               const float* x_old, const float* v_old, const float* radius,
                                               const int* flags, float* v_out, void* stream)
{
    clear_error();
    int st = check_contacts(contacts);
    if (st != NSPH_OK) return st;
    if (!params) return fail(NSPH_ERR_INVALID_ARG, "null params");
    if (contacts->max == 0) return NSPH_OK;
    if (!v_new || !x_old || !v_old || !radius || !flags || !v_out)
        return fail(NSPH_ERR_INVALID_ARG, "null particle array");
    k_shape_restitution<<<contact_blocks(contacts), kShapeThreads, 0, (cudaStream_t)stream>>>(
        view_of(contacts), *params, v_new, x_old, v_old, radius, flags, v_out);
    NSPH_LAUNCH_CHECK("k_shape_restitution");
    return NSPH_OK;
}

extern "C" int nsph_apply_particle_deltas(int n, const float* x_orig, const float* x_pred, const int* flags,
                                          const float* deltas, float dt, float v_max, float* x_out, float* v_out,
                                          void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_apply_particle_deltas");
    if (n < 0) return fail(NSPH_ERR_INVALID_ARG, "negative particle count");
    if (n == 0) return NSPH_OK;
    if (!x_orig || !x_pred || !flags || !deltas || !x_out || !v_out)
        return fail(NSPH_ERR_INVALID_ARG, "null particle array");
    k_apply_deltas<<<(n + kShapeThreads - 1) / kShapeThreads, kShapeThreads, 0, (cudaStream_t)stream>>>(
        n, x_orig, x_pred, flags, deltas, dt, v_max, x_out, v_out);
    NSPH_LAUNCH_CHECK("k_apply_deltas");
    return NSPH_OK;
}
