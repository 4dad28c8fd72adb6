// contact.cu — particle-particle contact on the HashGrid: the other
// consumers of the grid in the reference, rebuilt on this library's grid.
//
//   nsph_particle_contact_forces   eval_particle_contact + particle_force
//       (newton/_src/solvers/semi_implicit/kernels_contact.py:11-84, launched
//       by eval_particle_contact_forces, :559-579): spring-damper normal
//       force and Coulomb friction, written to f[i].
//   nsph_particle_contact_deltas   solve_particle_particle_contacts
//       (newton/_src/solvers/xpbd/kernels.py:225-289, launched at
//       newton/_src/solvers/xpbd/solver_xpbd.py:420-440): XPBD position
//       corrections, added to deltas[i].
//
// One thread per grid point, taken in sorted order (the reference's
// hash_grid_point_id(grid, tid)); each particle gathers over the candidates
// of hash_grid_query(grid, x_i, r_i + max_radius + cohesion) in Warp's
// iteration order. A first kernel copies the particles into sorted float4
// mirrors held by the grid object, m0 = (x, r) and m1 = (v, inverse mass),
// so that the candidates of a cell run are read contiguously; an inactive
// particle's radius slot holds -inf (radii of active particles are
// finite). Every fp32 operation is an explicit round-to-nearest
// intrinsic in the order the reference's expressions are written (dot
// products ((x + y) + z), no contraction), so the CPU restatement reproduces
// the results bit for bit.
#include "nsph_internal.cuh"

namespace nsph {

NSPH_BOUNDS_READER(contact)
namespace {

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// particle_force (kernels_contact.py:11-32): normal force c k_n + min(v.n, 0) k_d
// along -n, Coulomb friction min(|vt| k_f, mu |fn|) along -vt/|vt|
__device__ __forceinline__ void particle_force(float nx, float ny, float nz, float vx, float vy, float vz, float c,
                                               const nsph_contact_params& p, float& fx, float& fy, float& fz)
{
    const float vn = dot3(nx, ny, nz, vx, vy, vz);
    const float jn = __fmul_rn(c, p.k_contact);
    const float jd = __fmul_rn(fminf(vn, 0.f), p.k_damp);
    const float fn = __fadd_rn(jn, jd);
    float tx = __fsub_rn(vx, __fmul_rn(nx, vn));
    float ty = __fsub_rn(vy, __fmul_rn(ny, vn));
    float tz = __fsub_rn(vz, __fmul_rn(nz, vn));
    const float vs = __fsqrt_rn(dot3(tx, ty, tz, tx, ty, tz));
    if (vs > 0.f) {
        tx = __fdiv_rn(tx, vs);
        ty = __fdiv_rn(ty, vs);
        tz = __fdiv_rn(tz, vs);
    }
    const float ft = fminf(__fmul_rn(vs, p.k_friction), __fmul_rn(p.k_mu, fabsf(fn)));
    fx = __fsub_rn(__fmul_rn(-nx, fn), __fmul_rn(tx, ft));
    fy = __fsub_rn(__fmul_rn(-ny, fn), __fmul_rn(ty, ft));
    fz = __fsub_rn(__fmul_rn(-nz, fn), __fmul_rn(tz, ft));
}

__device__ __forceinline__ bool mirror_active(float4 m0) { return m0.w != -INFINITY; }

// sorted mirrors: m0[k] = (x, r or -inf if inactive), m1[k] = (v, inverse mass or 0)
__global__ void k_contact_gather(const int* __restrict__ ids, int n, const float* __restrict__ x,
                                 const float* __restrict__ v, const float* __restrict__ radius,
                                 const int* __restrict__ flags, const float* __restrict__ inv_mass,
                                 float4* __restrict__ m0, float4* __restrict__ m1)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t i = (size_t)ids[k];
    const bool active = (flags[i] & NSPH_PARTICLE_ACTIVE) != 0;
    m0[k] = make_float4(x[3 * i], x[3 * i + 1], x[3 * i + 2], active ? radius[i] : -INFINITY);
    m1[k] = make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], inv_mass ? inv_mass[i] : 0.f);
}

// bounded to 48 registers (from 64): 40 resident warps per SM
__global__ void __launch_bounds__(128, 10) k_contact_forces(GridDev g, int n, const float4* __restrict__ m0, const float4* __restrict__ m1,
                                 const nsph_contact_params p, float* __restrict__ f_out)
{
    const int kk = blockIdx.x * blockDim.x + threadIdx.x;
    if (kk >= n) return;
    const float4 a = m0[kk];
    if (!mirror_active(a)) return;
    const float4 va = m1[kk];
    const float ri = a.w;
    const float qr = __fadd_rn(__fadd_rn(ri, p.max_radius), p.k_cohesion);
    float fx = 0.f, fy = 0.f, fz = 0.f;
    for_each_candidate(g, a.x, a.y, a.z, qr, [&](int k) {
        const float4 b = __ldg(m0 + k);
        if (!mirror_active(b) || k == kk) return;
        float nx = __fsub_rn(a.x, b.x);
        float ny = __fsub_rn(a.y, b.y);
        float nz = __fsub_rn(a.z, b.z);
        const float d = __fsqrt_rn(dot3(nx, ny, nz, nx, ny, nz));
        const float err = __fsub_rn(__fsub_rn(d, ri), b.w);
        if (err <= p.k_cohesion) {
            const float4 vb = __ldg(m1 + k);
            nx = __fdiv_rn(nx, d);
            ny = __fdiv_rn(ny, d);
            nz = __fdiv_rn(nz, d);
            float cx, cy, cz;
            particle_force(nx, ny, nz, __fsub_rn(va.x, vb.x), __fsub_rn(va.y, vb.y), __fsub_rn(va.z, vb.z), err, p,
                           cx, cy, cz);
            fx = __fadd_rn(fx, cx);
            fy = __fadd_rn(fy, cy);
            fz = __fadd_rn(fz, cz);
        }
    });
    const size_t i = (size_t)g.ids[kk];
    f_out[3 * i] = fx;
    f_out[3 * i + 1] = fy;
    f_out[3 * i + 2] = fz;
}

// solve_particle_particle_contacts (xpbd/kernels.py:225-289)
__global__ void k_contact_deltas(GridDev g, int n, const float4* __restrict__ m0, const float4* __restrict__ m1,
                                 float k_mu, float k_cohesion, float max_radius, float dt, float relaxation,
                                 float* __restrict__ deltas)
{
    const int kk = blockIdx.x * blockDim.x + threadIdx.x;
    if (kk >= n) return;
    const float4 a = m0[kk];
    if (!mirror_active(a)) return;
    const float4 va = m1[kk];
    const float ri = a.w;
    const float w1 = va.w;
    const float qr = __fadd_rn(__fadd_rn(ri, max_radius), k_cohesion);
    float dx = 0.f, dy = 0.f, dz = 0.f;
    for_each_candidate(g, a.x, a.y, a.z, qr, [&](int k) {
        const float4 b = __ldg(m0 + k);
        if (!mirror_active(b) || k == kk) return;
        float nx = __fsub_rn(a.x, b.x);
        float ny = __fsub_rn(a.y, b.y);
        float nz = __fsub_rn(a.z, b.z);
        const float d = __fsqrt_rn(dot3(nx, ny, nz, nx, ny, nz));
        const float err = __fsub_rn(__fsub_rn(d, ri), b.w);
        const float4 vb = __ldg(m1 + k);
        const float denom = __fadd_rn(w1, vb.w);
        if (err <= k_cohesion && denom > 0.f) {
            nx = __fdiv_rn(nx, d);
            ny = __fdiv_rn(ny, d);
            nz = __fdiv_rn(nz, d);
            const float rx = __fsub_rn(va.x, vb.x);
            const float ry = __fsub_rn(va.y, vb.y);
            const float rz = __fsub_rn(va.z, vb.z);
            // normal
            const float lambda_n = err;
            const float dnx = __fmul_rn(nx, lambda_n), dny = __fmul_rn(ny, lambda_n), dnz = __fmul_rn(nz, lambda_n);
            // friction
            const float vn = dot3(nx, ny, nz, rx, ry, rz);
            float tx = __fsub_rn(rx, __fmul_rn(nx, vn));
            float ty = __fsub_rn(ry, __fmul_rn(ny, vn));
            float tz = __fsub_rn(rz, __fmul_rn(nz, vn));
            const float lt = __fsqrt_rn(dot3(tx, ty, tz, tx, ty, tz));
            const float lambda_f = fmaxf(__fmul_rn(k_mu, lambda_n), __fmul_rn(-lt, dt));
            if (lt > 0.f) {  // normalize(vt); the zero vector stays zero
                tx = __fdiv_rn(tx, lt);
                ty = __fdiv_rn(ty, lt);
                tz = __fdiv_rn(tz, lt);
            } else {
                tx = ty = tz = 0.f;
            }
            dx = __fadd_rn(dx, __fdiv_rn(__fsub_rn(__fmul_rn(tx, lambda_f), dnx), denom));
            dy = __fadd_rn(dy, __fdiv_rn(__fsub_rn(__fmul_rn(ty, lambda_f), dny), denom));
            dz = __fadd_rn(dz, __fdiv_rn(__fsub_rn(__fmul_rn(tz, lambda_f), dnz), denom));
        }
    });
    // deltas[i] += delta * w1 * relaxation (one writer per particle: no atomics)
    const size_t i = (size_t)g.ids[kk];
    deltas[3 * i] = __fadd_rn(deltas[3 * i], __fmul_rn(__fmul_rn(dx, w1), relaxation));
    deltas[3 * i + 1] = __fadd_rn(deltas[3 * i + 1], __fmul_rn(__fmul_rn(dy, w1), relaxation));
    deltas[3 * i + 2] = __fadd_rn(deltas[3 * i + 2], __fmul_rn(__fmul_rn(dz, w1), relaxation));
}

int check_grid(const nsph_grid* grid, int n)
{
    if (!grid) return fail(NSPH_ERR_INVALID_ARG, "null grid");
    if (grid->g.world_count > 0) return fail(NSPH_ERR_INVALID_ARG, "contacts need a single-world grid");
    if (!grid->g.built) return fail(NSPH_ERR_NOT_BUILT, "the grid has not been built");
    if (n < 0) return fail(NSPH_ERR_INVALID_ARG, "negative particle count");
    if (n != grid->g.num_points)
        return fail(NSPH_ERR_INVALID_ARG, "particle count differs from the points of the grid's last build");
    if (n > grid->mirror_cap) return fail(NSPH_ERR_CAPACITY, "grid not reserved through nsph_grid_reserve");
    return NSPH_OK;
}

}  // namespace
}  // namespace nsph

using namespace nsph;

extern "C" int nsph_particle_contact_forces(const nsph_grid* grid, const nsph_contact_params* params, int n,
                                            const float* x, const float* v, const float* radius, const int* flags,
                                            float* f_out, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_particle_contact_forces");
    int st = check_grid(grid, n);
    if (st != NSPH_OK) return st;
    if (!params) return fail(NSPH_ERR_INVALID_ARG, "null params");
    if (n == 0) return NSPH_OK;
    if (!x || !v || !radius || !flags || !f_out) return fail(NSPH_ERR_INVALID_ARG, "null array");
    DeviceGuard guard(grid->g.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    float4* m0 = grid->mirror;
    float4* m1 = grid->mirror + grid->mirror_cap;
    k_contact_gather<<<(n + 255) / 256, 256, 0, cs>>>(grid->g.point_ids, n, x, v, radius, flags, nullptr, m0, m1);
    NSPH_LAUNCH_CHECK("k_contact_gather");
    k_contact_forces<<<(n + 127) / 128, 128, 0, cs>>>(grid->g.view(), n, m0, m1, *params, f_out);
    NSPH_LAUNCH_CHECK("k_contact_forces");
    return NSPH_OK;
}

extern "C" int nsph_particle_contact_deltas(const nsph_grid* grid, int n, const float* x, const float* v,
                                            const float* inv_mass, const float* radius, const int* flags, float k_mu,
                                            float k_cohesion, float max_radius, float dt, float relaxation,
                                            float* deltas, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_particle_contact_deltas");
    int st = check_grid(grid, n);
    if (st != NSPH_OK) return st;
    if (n == 0) return NSPH_OK;
    if (!x || !v || !inv_mass || !radius || !flags || !deltas) return fail(NSPH_ERR_INVALID_ARG, "null array");
    DeviceGuard guard(grid->g.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    float4* m0 = grid->mirror;
    float4* m1 = grid->mirror + grid->mirror_cap;
    k_contact_gather<<<(n + 255) / 256, 256, 0, cs>>>(grid->g.point_ids, n, x, v, radius, flags, inv_mass, m0, m1);
    NSPH_LAUNCH_CHECK("k_contact_gather");
    k_contact_deltas<<<(n + 127) / 128, 128, 0, cs>>>(grid->g.view(), n, m0, m1, k_mu, k_cohesion, max_radius, dt,
                                                       relaxation, deltas);
    NSPH_LAUNCH_CHECK("k_contact_deltas");
    return NSPH_OK;
}
