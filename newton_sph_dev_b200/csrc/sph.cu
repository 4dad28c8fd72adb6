// sph.cu — the WCSPH step: grid build on x_n, density/EOS pass, then the
// pressure + XSPH + integrate pass that writes x_{n+1}, v_{n+1}.
//
// The reference has no SPH solver (its particle hot path is the HashGrid
// gather of newton/_src/solvers/semi_implicit/kernels_contact.py:35-84 plus
// integrate_particles, newton/_src/solvers/solver.py:10-47); the step keeps
// that structure and replaces the contact law with published WCSPH math:
//   W      cubic spline with support h (Monaghan 1992), sigma = 8/(pi h^3)
//   rho_i  = sum_j m_j W_ij (self included)
//   p_i    = B((rho_i/rho0)^gamma - 1) clamped at 0 (Tait EOS)
//   a_i    = -sum_{j!=i} m_j (p_i/rho_i^2 + p_j/rho_j^2) grad W_ij
//   dv_i   = eps sum_{j!=i} (m_j/rho_j)(v_j - v_i) W_ij (XSPH on v_n)
// and integrates with integrate_particles' semantics (gravity and forces
// only for inv_mass > 0, |v| clamp, inactive particles keep x and v).
//
// Layout in HBM (sorted by cell, written by the last radix pass):
//   xs[k]  float4 (x, y, z, m_eff)   m_eff = 0 for inactive particles
//   vs[k]  float4 (vx, vy, vz, attr) attr = active | dynamic<<1 | gravity<<2
//   aux[k] float2 (m/rho, p/rho^2)   written by the density pass
//   rp[k]  float2 (rho, p)           written by the density pass
// Outputs are scattered back to original particle order through point_ids.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "mlp.cuh"
#include "nsph_internal.cuh"

namespace nsph {

NSPH_BOUNDS_READER(sph)

namespace {

constexpr int kSphThreads = 256;

// the neighbour test shared with the oracle (no contraction beyond the two
// explicit FMAs): r2 = fma(dz, dz, fma(dy, dy, dx*dx))
__device__ __forceinline__ float dist2(float4 a, float4 b, float& dx, float& dy, float& dz)
{
    dx = __fsub_rn(a.x, b.x);
    dy = __fsub_rn(a.y, b.y);
    dz = __fsub_rn(a.z, b.z);
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// Every fp32 operation below is written with an explicit rounding intrinsic
// (no compiler contraction), in the same order as the fp32 oracle, and each
// particle's neighbours are summed in the grid's query order, so the device
// reproduces the fp32 restatement's sums.

// W(q) = sigma * {fma((6q)q, q-1, 1) for q <= 1/2; ((2t)t)t with t = 1-q for q < 1}
__device__ __forceinline__ float kernel_w(float q, const nsph_sph_params& p)
{
    const float t = __fsub_rn(1.f, q);
    const float nearv = __fmaf_rn(__fmul_rn(__fmul_rn(6.f, q), q), __fsub_rn(q, 1.f), 1.f);
    const float farv = __fmul_rn(__fmul_rn(__fmul_rn(2.f, t), t), t);
    return __fmul_rn(p.sigma, q <= 0.5f ? nearv : (q < 1.f ? farv : 0.f));
}

// (dW/dr)/r = {c_near * fma(3, q, -2) for q <= 1/2; ((c_far t) t)(1/r) for q < 1}
__device__ __forceinline__ float kernel_f(float q, float inv_r, const nsph_sph_params& p)
{
    const float t = __fsub_rn(1.f, q);
    const float nearv = __fmul_rn(p.c_near, __fmaf_rn(3.f, q, -2.f));
    const float farv = __fmul_rn(__fmul_rn(__fmul_rn(p.c_far, t), t), inv_r);
    return q <= 0.5f ? nearv : (q < 1.f ? farv : 0.f);
}

__device__ __forceinline__ float eos(float rho, const nsph_sph_params& p)
{
    const float ratio = __fmul_rn(rho, p.inv_rho0);
    float pw = 1.f;
    for (int k = 0; k < p.eos_gamma; ++k) pw = __fmul_rn(pw, ratio);
    float pr = __fmul_rn(p.eos_b, __fsub_rn(pw, 1.f));
    if (p.clamp_pressure && pr < 0.f) pr = 0.f;
    return pr;
}

__device__ __forceinline__ float wterm(float r2, const nsph_sph_params& p)
{
    return kernel_w(__fmul_rn(__fsqrt_rn(r2), p.inv_h), p);
}

// ---- tolerance ("fast") arithmetic ---------------------------------------------
// The same kernel values with the hardware reciprocal square root instead of
// the correctly rounded square root, reciprocal and division, and with the
// compiler free to contract multiply-adds: r = r2 * rsqrt(r2), 1/r = rsqrt(r2).
// The neighbour test r2 < h2 is unchanged, so neighbour sets stay bit-exact;
// sums keep the query order. Results are within the fp64 oracle's tolerance
// (checked by the tests), not bit-exact with the fp32 oracle.
__device__ __forceinline__ float kernel_w_fast(float q, const nsph_sph_params& p)
{
    const float t = 1.f - q;
    const float v = q <= 0.5f ? fmaf(6.f * q * q, q - 1.f, 1.f) : (q < 1.f ? 2.f * t * t * t : 0.f);
    return p.sigma * v;
}

__device__ __forceinline__ float wterm_fast(float r2, const nsph_sph_params& p)
{
    const float r = r2 > 0.f ? r2 * rsqrtf(r2) : 0.f;
    return kernel_w_fast(r * p.inv_h, p);
}

// ---- density + EOS -----------------------------------------------------------
template <bool Fast = false>
__device__ __forceinline__ void density_finish(int k, float m, float rho, const nsph_sph_params& p,
                                               float2* __restrict__ aux, float2* __restrict__ rp,
                                               unsigned* __restrict__ status)
{
    float pr = 0.f, mor = 0.f, pr2 = 0.f;
    if (rho > 0.f) {
        pr = eos(rho, p);
        if (Fast) {
            const float ir = __frcp_rn(rho);
            mor = m * ir;
            pr2 = pr * ir * ir;
        } else {
            mor = __fdiv_rn(m, rho);
            pr2 = __fdiv_rn(pr, __fmul_rn(rho, rho));
        }
    } else if (status) {
        atomicOr(status, (unsigned)NSPH_STATUS_ZERO_DENSITY);
    }
    aux[k] = make_float2(mor, pr2);
    rp[k] = make_float2(rho, pr);
}

// ---- neighbour lists (the plain step) -----------------------------------------
// The density pass of the plain step first tests every candidate (in query
// order) and appends the sorted index of each neighbour to the particle's
// list, in groups of four: group g (slots 4g .. 4g+3) at nbr[g * n + k] as
// one int4 (group-major, so that a warp reading group g of 32 consecutive
// particles reads one contiguous 512-byte span), for the first kNbrSlots
// neighbours, and their number in ncnt[k]. A thread keeps the last four hits
// in registers and stores a full group at once (a store per four neighbours
// instead of one per neighbour). The cubic-spline terms are then evaluated
// by a second loop over the list, in the same order, so every lane of a warp
// runs the term code only for its own neighbours (evaluated inside the
// candidate loop, a warp runs it for every candidate slot at which any of
// its 32 lanes has a hit, which at a ~15% hit rate is nearly all of them).
// Readers load a whole group ahead of its use. The force pass walks the same
// list with one uniform loop and no grid traversal. A particle with more
// than kNbrSlots neighbours (dense clusters) is summed by re-testing its
// candidates, in the same order. Sums, their order and every rounding are
// those of the fp32 oracle.
constexpr int kNbrSlots = 64;
constexpr int kNbrGroups = kNbrSlots / 4;
// entries every sorted-position array that neighbor_list reads holds past
// its last particle (the candidate groups' reads past a run's end)
constexpr int kXsPad = 4;

// One candidate's hit bit pushed into `acc` from the right: the sign bit of
// fl(r2 - h2), by one funnel shift. fl(r2 - h2) is negative exactly when
// r2 < h2: an IEEE subtraction of two unequal values is never zero and its
// rounding keeps the sign, and r2 == h2 gives +0. A NaN difference (from a
// non-finite position) is the GPU's canonical NaN, whose sign bit is clear,
// as r2 < h2 is false for it. So the bits are those of the comparison, at
// one FADD and one shift per candidate instead of a compare, a select, a
// variable shift and an OR.
__device__ __forceinline__ unsigned push_hit(unsigned acc, float r2, float h2)
{
    return __funnelshift_l(__float_as_uint(__fsub_rn(r2, h2)), acc, 1);
}

template <bool kPaddedGroups>
__device__ __forceinline__ int neighbor_list(const GridDev& g, const float4* __restrict__ xs,
                                             const nsph_sph_params& p, float4 xi, int4* __restrict__ nbr, int n,
                                             int k)
{
    int cnt = 0;
    int b0 = 0, b1 = 0, b2 = 0, b3 = 0;
    auto append = [&](int j) {
        b0 = b1;
        b1 = b2;
        b2 = b3;
        b3 = j;
        ++cnt;
        if ((cnt & 3) == 0 && cnt <= kNbrSlots) nbr[(size_t)((cnt >> 2) - 1) * n + k] = make_int4(b0, b1, b2, b3);
    };
    // Candidates are tested branch-free into a bit mask per chunk of up to 32
    // of a run; the hits are appended after the chunk, so the append code runs
    // once per neighbour (a warp iterates over its lanes' largest hit count of
    // the chunk) instead of at every candidate where any lane has a hit.
    // Candidates go in groups of four (four loads issued together). With
    // kPaddedGroups there is no scalar tail loop: a run's last group reads
    // up to three entries past the run, whose bits are then cleared. Those
    // reads stay inside the array: every xs array the density passes read
    // holds at least kXsPad entries past its last particle. (Padded groups
    // took the 1M tank's density pass from 0.330 to 0.315 ms but the batched
    // worlds' from 5.18 to 5.39 ms, so the worlds pass keeps the tail loop.)
    // The padded path takes each hit bit from push_hit (0.318 -> 0.303 ms on
    // the 1M tank); the worlds pass keeps the comparison, which spilled less.
    for_each_run(g, xi.x, xi.y, xi.z, p.h, [&](int lo, int hi) {
        for (int c0 = lo; c0 < hi; c0 += 32) {
            const int m = min(32, hi - c0);
            unsigned bits;
            if constexpr (kPaddedGroups) {
                unsigned acc = 0u;  // candidate t of the chunk at bit mp - 1 - t
#pragma unroll 1
                for (int j = 0; j < m; j += 4) {
                    float4 xj[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) xj[u] = __ldg(xs + c0 + j + u);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        float dx, dy, dz;
                        acc = push_hit(acc, dist2(xi, xj[u], dx, dy, dz), p.h2);
                    }
                }
                // reversed, candidate t sits at bit t; the group's reads past
                // the run (bits m .. mp - 1) are cleared
                const int mp = (m + 3) & ~3;
                bits = __brev(acc) >> (32 - mp);
                if (m < 32) bits &= (1u << m) - 1u;
            } else {
                bits = 0u;
                int j = 0;
                for (; j + 4 <= m; j += 4) {
                    float4 xj[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) xj[u] = __ldg(xs + c0 + j + u);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        float dx, dy, dz;
                        bits |= (unsigned)(dist2(xi, xj[u], dx, dy, dz) < p.h2) << (j + u);
                    }
                }
                for (; j < m; ++j) {
                    float dx, dy, dz;
                    bits |= (unsigned)(dist2(xi, __ldg(xs + c0 + j), dx, dy, dz) < p.h2) << j;
                }
            }
            while (bits) {
                append(c0 + __ffs(bits) - 1);
                bits &= bits - 1u;
            }
        }
    });
    const int r = cnt & 3;  // the last, partial group: its r hits are b(4-r) .. b3
    if (r && cnt <= kNbrSlots)
        nbr[(size_t)(cnt >> 2) * n + k] = r == 1 ? make_int4(b3, 0, 0, 0)
                                                 : (r == 2 ? make_int4(b2, b3, 0, 0) : make_int4(b1, b2, b3, 0));
    return cnt;
}

// Element u (0..3, a constant after unrolling) of a list group.
__device__ __forceinline__ int group_item(const int4& gr, int u)
{
    return u == 0 ? gr.x : (u == 1 ? gr.y : (u == 2 ? gr.z : gr.w));
}

// Walk of a particle's list by whole groups: visit(j) for its neighbours in
// order. The group after the current one is loaded when the current one
// starts; the four items of a group are unrolled, so each index is a fixed
// register (no per-item select, as a reader returning one item at a time
// needs) and the visits' loads can issue together. kReadOnly: the list was
// written by an earlier kernel (read-only path); otherwise it is read back by
// the thread that wrote it (plain loads). kUnrolled = false keeps a rolled
// loop over a group's items (one item per iteration, selected at run time):
// the batched worlds' force pass spills more when unrolled (2.16 -> 2.38 ms
// on worlds_4096).
template <bool kReadOnly, bool kUnrolled = true, class F>
__device__ __forceinline__ void for_each_listed(const int4* __restrict__ nbr, int n, int k, int cnt, F&& visit)
{
    in_bounds(cnt >= 0 && cnt <= kNbrSlots);
    const int4* a = nbr + k;
    auto load = [&](int gi) { return kReadOnly ? __ldg(a + (size_t)gi * n) : a[(size_t)gi * n]; };
    int4 cur = cnt > 0 ? load(0) : make_int4(0, 0, 0, 0);
    int4 nxt = cnt > 4 ? load(1) : make_int4(0, 0, 0, 0);
    for (int t = 0; t < cnt; t += 4) {
        const int4 gr = cur;
        cur = nxt;
        if (t + 8 < cnt) nxt = load((t >> 2) + 2);
        auto item = [&](int u) {
            if (t + u < cnt) {
                const int j = group_item(gr, u);
                visit(in_bounds(j >= 0 && j < n) ? j : 0);
            }
        };
        if constexpr (kUnrolled) {
#pragma unroll
            for (int u = 0; u < 4; ++u) item(u);
        } else {
#pragma unroll 1
            for (int u = 0; u < 4; ++u) item(u);
        }
    }
}

// rho of particle k from its list (read back by the thread that wrote it,
// with plain loads), or by re-testing its candidates when the list overflowed
template <bool Fast>
__device__ __forceinline__ float density_from_list(const GridDev& g, const float4* __restrict__ xs,
                                                   const nsph_sph_params& p, float4 xi, const int4* nbr, int cnt,
                                                   int n, int k)
{
    float rho = 0.f;
    auto w = [&](float r2) { return Fast ? wterm_fast(r2, p) : wterm(r2, p); };
    if (cnt <= kNbrSlots) {
        for_each_listed<false>(nbr, n, k, cnt, [&](int j) {
            const float4 xj = __ldg(xs + j);
            float dx, dy, dz;
            rho = __fmaf_rn(xj.w, w(dist2(xi, xj, dx, dy, dz)), rho);
        });
    } else {
        for_each_candidate(g, xi.x, xi.y, xi.z, p.h, [&](int j) {
            const float4 xj = __ldg(xs + j);
            float dx, dy, dz;
            const float r2 = dist2(xi, xj, dx, dy, dz);
            if (r2 < p.h2) rho = __fmaf_rn(xj.w, w(r2), rho);
        });
    }
    return rho;
}

struct ForceAcc {
    float ax, ay, az, dvx, dvy, dvz;
};

// pressure and XSPH terms of one neighbour (not self), accumulated in order
__device__ __forceinline__ void force_term_data(float4 xj, float4 vj, float2 aj, float4 xi, float4 vi, float pr2_i,
                                                const nsph_sph_params& p, ForceAcc& acc)
{
    if (!(__float_as_int(vj.w) & kAttrActive)) return;
    float dx, dy, dz;
    const float r2 = dist2(xi, xj, dx, dy, dz);
    const float r = __fsqrt_rn(r2);
    const float q = __fmul_rn(r, p.inv_h);
    const float w = kernel_w(q, p);
    if (r2 > 0.f) {
        const float f = kernel_f(q, __frcp_rn(r), p);
        const float s = __fmul_rn(__fmul_rn(xj.w, __fadd_rn(pr2_i, aj.y)), f);
        acc.ax = __fmaf_rn(-s, dx, acc.ax);
        acc.ay = __fmaf_rn(-s, dy, acc.ay);
        acc.az = __fmaf_rn(-s, dz, acc.az);
    }
    const float c = __fmul_rn(aj.x, w);
    acc.dvx = __fmaf_rn(c, __fsub_rn(vj.x, vi.x), acc.dvx);
    acc.dvy = __fmaf_rn(c, __fsub_rn(vj.y, vi.y), acc.dvy);
    acc.dvz = __fmaf_rn(c, __fsub_rn(vj.z, vi.z), acc.dvz);
}

// force_term_data in the tolerance arithmetic (see kernel_w_fast)
__device__ __forceinline__ void force_term_fast(float4 xj, float4 vj, float2 aj, float4 xi, float4 vi, float pr2_i,
                                                const nsph_sph_params& p, ForceAcc& acc)
{
    if (!(__float_as_int(vj.w) & kAttrActive)) return;
    const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
    const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
    float w = p.sigma;
    if (r2 > 0.f) {
        const float ir = rsqrtf(r2);
        const float q = r2 * ir * p.inv_h;
        const float t = 1.f - q;
        w = kernel_w_fast(q, p);
        const float f = q <= 0.5f ? p.c_near * fmaf(3.f, q, -2.f) : (q < 1.f ? p.c_far * t * t * ir : 0.f);
        const float s = xj.w * (pr2_i + aj.y) * f;
        acc.ax -= s * dx;
        acc.ay -= s * dy;
        acc.az -= s * dz;
    }
    const float c = aj.x * w;
    acc.dvx += c * (vj.x - vi.x);
    acc.dvy += c * (vj.y - vi.y);
    acc.dvz += c * (vj.z - vi.z);
}

struct StepOut {
    const float* f_ext;
    const float* inv_mass;
    const float* gravity;
    float* x_out;
    float* v_out;
    float* rho_out;
    float* p_out;
    float* a_out;
    unsigned* status;
    float4* acc_sorted;  // or null: (a, 0), (dv, 0) of sorted particle k at 2k, 2k + 1 (the segment tape)
};

// integrate particle k (original index i) and scatter its outputs
__device__ __forceinline__ void integrate_out(size_t i, float4 xi, float4 vi, int attr, float2 rpk,
                                              const ForceAcc& acc, const nsph_sph_params& p, float dt,
                                              const StepOut& o)
{
    if (o.rho_out) o.rho_out[i] = rpk.x;
    if (o.p_out) o.p_out[i] = rpk.y;
    if (!(attr & kAttrActive)) {
        o.x_out[3 * i + 0] = xi.x;
        o.x_out[3 * i + 1] = xi.y;
        o.x_out[3 * i + 2] = xi.z;
        if (o.a_out) o.a_out[3 * i + 0] = o.a_out[3 * i + 1] = o.a_out[3 * i + 2] = 0.f;
        return;
    }
    const float ax = acc.ax, ay = acc.ay, az = acc.az;
    if (o.a_out) {
        o.a_out[3 * i + 0] = ax;
        o.a_out[3 * i + 1] = ay;
        o.a_out[3 * i + 2] = az;
    }
    float v1x = vi.x, v1y = vi.y, v1z = vi.z;
    const bool dynamic = (attr & kAttrDynamic) != 0;
    if (dynamic) {
        const int gw = attr >> kAttrGravShift;
        float fx = 0.f, fy = 0.f, fz = 0.f;
        if (o.f_ext) {
            const float w = o.inv_mass[i];
            fx = __fmul_rn(o.f_ext[3 * i + 0], w);
            fy = __fmul_rn(o.f_ext[3 * i + 1], w);
            fz = __fmul_rn(o.f_ext[3 * i + 2], w);
        }
        const float gx = o.gravity[3 * gw + 0], gy = o.gravity[3 * gw + 1], gz = o.gravity[3 * gw + 2];
        // v1 = fma(eps, dv, fma((a + f w) + g, dt, v0))
        v1x = __fmaf_rn(p.xsph_eps, acc.dvx, __fmaf_rn(__fadd_rn(__fadd_rn(ax, fx), gx), dt, vi.x));
        v1y = __fmaf_rn(p.xsph_eps, acc.dvy, __fmaf_rn(__fadd_rn(__fadd_rn(ay, fy), gy), dt, vi.y));
        v1z = __fmaf_rn(p.xsph_eps, acc.dvz, __fmaf_rn(__fadd_rn(__fadd_rn(az, fz), gz), dt, vi.z));
    }
    const float vm = __fsqrt_rn(__fmaf_rn(v1z, v1z, __fmaf_rn(v1y, v1y, __fmul_rn(v1x, v1x))));
    if (vm > p.v_max) {
        const float s = __fdiv_rn(p.v_max, vm);
        v1x = __fmul_rn(v1x, s);
        v1y = __fmul_rn(v1y, s);
        v1z = __fmul_rn(v1z, s);
    }
    float x1x = __fmaf_rn(v1x, dt, xi.x), x1y = __fmaf_rn(v1y, dt, xi.y), x1z = __fmaf_rn(v1z, dt, xi.z);
    if (dynamic && p.use_box) {
        if (x1x < p.box_lo[0]) { x1x = p.box_lo[0]; v1x = fmaxf(v1x, 0.f); }
        if (x1x > p.box_hi[0]) { x1x = p.box_hi[0]; v1x = fminf(v1x, 0.f); }
        if (x1y < p.box_lo[1]) { x1y = p.box_lo[1]; v1y = fmaxf(v1y, 0.f); }
        if (x1y > p.box_hi[1]) { x1y = p.box_hi[1]; v1y = fminf(v1y, 0.f); }
        if (x1z < p.box_lo[2]) { x1z = p.box_lo[2]; v1z = fmaxf(v1z, 0.f); }
        if (x1z > p.box_hi[2]) { x1z = p.box_hi[2]; v1z = fminf(v1z, 0.f); }
    }
    if (o.status && !(isfinite(x1x) && isfinite(x1y) && isfinite(x1z) && isfinite(v1x) && isfinite(v1y) &&
                      isfinite(v1z)))
        atomicOr(o.status, (unsigned)NSPH_STATUS_NONFINITE_OUTPUT);
    o.x_out[3 * i + 0] = x1x;
    o.x_out[3 * i + 1] = x1y;
    o.x_out[3 * i + 2] = x1z;
    o.v_out[3 * i + 0] = v1x;
    o.v_out[3 * i + 1] = v1y;
    o.v_out[3 * i + 2] = v1z;
}

// ---- the plain step's passes on neighbour lists ----------------------------------
// Bounded to 48 registers (4 bytes of spills): 40 resident warps per SM.
template <bool Fast>
__global__ void __launch_bounds__(kSphThreads, 5) k_density_list(GridDev g, const float4* __restrict__ xs,
                                                                 const float4* __restrict__ vs, int n,
                                                                 const __grid_constant__ nsph_sph_params p,
                                                                 float2* __restrict__ aux, float2* __restrict__ rp,
                                                                 int4* __restrict__ nbr, int* __restrict__ ncnt,
                                                                 unsigned* __restrict__ status)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float4 xi = xs[k];
        if (!(__float_as_int(vs[k].w) & kAttrActive)) {
            aux[k] = make_float2(0.f, 0.f);
            rp[k] = make_float2(0.f, 0.f);
            ncnt[k] = 0;
            continue;
        }
        const int cnt = neighbor_list<true>(g, xs, p, xi, nbr, n, k);
        ncnt[k] = cnt;
        const float rho = density_from_list<Fast>(g, xs, p, xi, nbr, cnt, n, k);
        density_finish<Fast>(k, xi.w, rho, p, aux, rp, status);
    }
}

// pressure and XSPH sums of particle k over its list, in order (loads of
// neighbour t+1 issued before the terms of neighbour t), or by re-testing
// its candidates when the list overflowed
template <bool Fast, bool kUnrolledWalk = true>
__device__ __forceinline__ void force_from_list(const GridDev& g, const float4* __restrict__ xs,
                                                const float4* __restrict__ vs, const float2* __restrict__ aux,
                                                const int4* __restrict__ nbr, int cnt, int n, int k, float4 xi,
                                                float4 vi, float pr2_i, const nsph_sph_params& p, ForceAcc& acc)
{
    if (cnt <= kNbrSlots) {
        bool have = false;
        float4 pxj = make_float4(0.f, 0.f, 0.f, 0.f), pvj = pxj;
        float2 paj = make_float2(0.f, 0.f);
        for_each_listed<true, kUnrolledWalk>(nbr, n, k, cnt, [&](int j) {
            if (j == k) return;
            const float4 nxj = __ldg(xs + j);
            const float4 nvj = __ldg(vs + j);
            const float2 naj = __ldg(aux + j);
            if (have) {
                if (Fast)
                    force_term_fast(pxj, pvj, paj, xi, vi, pr2_i, p, acc);
                else
                    force_term_data(pxj, pvj, paj, xi, vi, pr2_i, p, acc);
            }
            pxj = nxj;
            pvj = nvj;
            paj = naj;
            have = true;
        });
        if (have) {
            if (Fast)
                force_term_fast(pxj, pvj, paj, xi, vi, pr2_i, p, acc);
            else
                force_term_data(pxj, pvj, paj, xi, vi, pr2_i, p, acc);
        }
    } else {
        for_each_run(g, xi.x, xi.y, xi.z, p.h, [&](int lo, int hi) {
            for (int j = lo; j < hi; ++j) {
                float dx, dy, dz;
                if (dist2(xi, __ldg(xs + j), dx, dy, dz) < p.h2 && j != k) {
                    if (Fast)
                        force_term_fast(__ldg(xs + j), __ldg(vs + j), __ldg(aux + j), xi, vi, pr2_i, p, acc);
                    else
                        force_term_data(__ldg(xs + j), __ldg(vs + j), __ldg(aux + j), xi, vi, pr2_i, p, acc);
                }
            }
        });
    }
}

template <bool Fast>
__global__ void __launch_bounds__(kSphThreads, 4) k_force_list(GridDev g, const float4* __restrict__ xs,
                                                               const float4* __restrict__ vs,
                                                               const float2* __restrict__ aux,
                                                               const float2* __restrict__ rp, int n,
                                                               const __grid_constant__ nsph_sph_params p,
                                                               const int4* __restrict__ nbr,
                                                               const int* __restrict__ ncnt, const StepOut o)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float4 xi = xs[k], vi = vs[k];
        const int attr = __float_as_int(vi.w);
        ForceAcc acc{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (attr & kAttrActive) force_from_list<Fast>(g, xs, vs, aux, nbr, ncnt[k], n, k, xi, vi, aux[k].y, p, acc);
        if (o.acc_sorted) {  // the force sums, for the adjoint's segment tape
            o.acc_sorted[2 * (size_t)k] = make_float4(acc.ax, acc.ay, acc.az, 0.f);
            o.acc_sorted[2 * (size_t)k + 1] = make_float4(acc.dvx, acc.dvy, acc.dvz, 0.f);
        }
        integrate_out((size_t)g.ids[k], xi, vi, attr, rp[k], acc, p, p.dt, o);
    }
}

// ---- batched worlds ------------------------------------------------------------
// One launch per pass covers every world. The kernels are persistent: a grid
// of (SMs x resident blocks) threads strides over all particles, whose work
// is similar whatever their world, so no work queue is needed. A particle's
// world (attr >> kAttrGravShift, clamped at the gather) selects its grid
// (dims, 1/cell width, cell-table offset) and its parameter block; its
// neighbours are found and summed exactly as in the single-world kernels, in
// its own world's query order.
__device__ __forceinline__ GridDev world_grid(const WorldCells& c, const int2* __restrict__ ranges,
                                              const int* __restrict__ ids, int n)
{
    return GridDev{c.dx, c.dy, c.dz, c.inv, ranges + c.off, ids, n};
}

// Bounded to 64 registers (36 bytes of spills outside the candidate loop):
// 5.81 -> 5.18 ms per pass on worlds_4096 against its unbounded 80 (same
// box, back to back); a reference into the parameter table instead of the
// copy was slower at 64 (5.41) and at 48 registers (5.53).
__global__ void __launch_bounds__(kSphThreads, 4) k_density_worlds(const WorldCells* __restrict__ wc,
                                                                   const nsph_sph_params* __restrict__ wp,
                                                                   const int2* __restrict__ ranges,
                                                                   const int* __restrict__ ids,
                                                                   const float4* __restrict__ xs,
                                                                   const float4* __restrict__ vs, int n,
                                                                   float2* __restrict__ aux, float2* __restrict__ rp,
                                                                   int4* __restrict__ nbr, int* __restrict__ ncnt,
                                                                   unsigned* __restrict__ status)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float4 xi = xs[k];
        const int attr = __float_as_int(vs[k].w);
        if (!(attr & kAttrActive)) {
            aux[k] = make_float2(0.f, 0.f);
            rp[k] = make_float2(0.f, 0.f);
            ncnt[k] = 0;
            continue;
        }
        const int w = attr >> kAttrGravShift;
        const nsph_sph_params p = wp[w];  // a copy: its fields stay in registers across the candidate loop
        const GridDev g = world_grid(wc[w], ranges, ids, n);
        const int cnt = neighbor_list<false>(g, xs, p, xi, nbr, n, k);
        ncnt[k] = cnt;
        const float rho = density_from_list<false>(g, xs, p, xi, nbr, cnt, n, k);
        density_finish(k, xi.w, rho, p, aux, rp, status);
    }
}

// Bounded to 64 registers: 2.39 -> 2.11 ms per pass on worlds_4096 against
// 80 at three blocks per SM (same box, back to back).
__global__ void __launch_bounds__(kSphThreads, 4) k_force_worlds(const WorldCells* __restrict__ wc,
                                                                 const nsph_sph_params* __restrict__ wp,
                                                                 const int2* __restrict__ ranges,
                                                                 const int* __restrict__ ids,
                                                                 const float4* __restrict__ xs,
                                                                 const float4* __restrict__ vs,
                                                                 const float2* __restrict__ aux,
                                                                 const float2* __restrict__ rp, int n, float dt,
                                                                 const int4* __restrict__ nbr,
                                                                 const int* __restrict__ ncnt, const StepOut o)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float4 xi = xs[k], vi = vs[k];
        const int attr = __float_as_int(vi.w);
        const int w = attr >> kAttrGravShift;
        const nsph_sph_params& p = wp[w];
        const GridDev g = world_grid(wc[w], ranges, ids, n);
        ForceAcc acc{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (attr & kAttrActive) force_from_list<false, false>(g, xs, vs, aux, nbr, ncnt[k], n, k, xi, vi, aux[k].y, p, acc);
        integrate_out((size_t)ids[k], xi, vi, attr, rp[k], acc, p, dt, o);
    }
}

__global__ void k_neighbors_worlds(const WorldCells* __restrict__ wc, const nsph_sph_params* __restrict__ wp,
                                   const int2* __restrict__ ranges, const int* __restrict__ ids,
                                   const float4* __restrict__ xs, const float4* __restrict__ vs, int n,
                                   int* __restrict__ counts, const long long* __restrict__ offsets,
                                   int* __restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = ids[k];
    const float4 xi = xs[k];
    const int attr = __float_as_int(vs[k].w);
    long long o = out ? offsets[i] : 0;
    int c = 0;
    if (attr & kAttrActive) {
        const int w = attr >> kAttrGravShift;
        const float h = wp[w].h, h2 = wp[w].h2;
        const GridDev g = world_grid(wc[w], ranges, ids, n);
        for_each_candidate(g, xi.x, xi.y, xi.z, h, [&](int j) {
            float dx, dy, dz;
            if (dist2(xi, xs[j], dx, dy, dz) < h2 && (__float_as_int(vs[j].w) & kAttrActive)) {
                if (out) out[o++] = ids[j];
                ++c;
            }
        });
    }
    if (!out) counts[i] = c;
}

// ---- neighbour lists of the last build (parity export) ----------------------
__global__ void k_neighbors(GridDev g, const float4* __restrict__ xs, const float4* __restrict__ vs, int n,
                            nsph_sph_params p, int* __restrict__ counts, const long long* __restrict__ offsets,
                            int* __restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = g.ids[k];
    const float4 xi = xs[k];
    const bool active = (__float_as_int(vs[k].w) & kAttrActive) != 0;
    long long o = out ? offsets[i] : 0;
    int c = 0;
    if (active) {
        for_each_candidate(g, xi.x, xi.y, xi.z, p.h, [&](int j) {
            const float4 xj = xs[j];
            float dx, dy, dz;
            if (dist2(xi, xj, dx, dy, dz) < p.h2 && (__float_as_int(vs[j].w) & kAttrActive)) {
                if (out) out[o++] = g.ids[j];
                ++c;
            }
        });
    }
    if (!out) counts[i] = c;
}

// ==========================================================================
// Adjoint of the step (reverse mode): given the adjoints of x_{n+1}, v_{n+1}
// (and optionally of rho), the adjoints of x_n, v_n, f_ext and of the EOS
// stiffness B. The neighbour set is held fixed (it is piecewise constant in
// x; W and dW/dr vanish at r = h, so the step is C1 across its changes); the
// pressure clamp, |v| clamp and box are differentiated on the side the
// forward step took, which the reverse pass recomputes bit for bit.
//
// The forward step sums pair terms into particle i only (a gather), so its
// transpose scatters into both particles of a pair. Because the neighbour
// relation is symmetric (the fp32 r2 of (i, j) and (j, i) are equal) every
// scatter is rewritten as a gather over the same neighbour lists, with no
// atomics, and each particle's adjoint is written by one thread:
//   local   G_i = adj(a_i), D_i = adj(dv_i), and the integrate reverse
//   pair    adj(p_i/rho_i^2) = sum_j F_ij (Z_ij . d_ij)
//           adj(m_i/rho_i)   = sum_j W_ij D_j . (v_i - v_j)
//           adj(x_i)        += sum_j S_ij [F Z + (F'/r)(d.Z) d]
//                              + F ((v_j - v_i) . Y_ij) d
//           adj(v_i)        -= sum_j W_ij Y_ij
//           with Z = m_i G_j - m_j G_i, Y = mor_j D_i - mor_i D_j,
//           S = p_i/rho_i^2 + p_j/rho_j^2, d = x_i - x_j, F = (dW/dr)/r
//           then adj(rho_i) through the EOS and the m/rho, p/rho^2 factors
//   density adj(x_i)        += sum_j F_ij (adj(rho_i) m_j + adj(rho_j) m_i) d_ij
// ==========================================================================

// (dF/dr)/r of F = (dW/dr)/r: near 3 c_near / (h r); far -c_far t (2/(h r^2) + t/r^3)
__device__ __forceinline__ float kernel_df_over_r(float q, float inv_r, const nsph_sph_params& p)
{
    const float t = 1.f - q;
    if (q <= 0.5f) return 3.f * p.c_near * p.inv_h * inv_r;
    if (q < 1.f) return -p.c_far * t * (2.f * p.inv_h + t * inv_r) * inv_r * inv_r;
    return 0.f;
}

// visit(j) for every neighbour j != k of sorted particle k, in query order,
// from the density pass's neighbour list (re-testing its candidates when the
// list overflowed)
template <class V>
__device__ __forceinline__ void for_each_neighbor(const GridDev& g, const float4* __restrict__ xs,
                                                  const int4* __restrict__ nbr, int cnt, int n, int k, float4 xi,
                                                  const nsph_sph_params& p, V&& visit)
{
    if (cnt <= kNbrSlots) {
        for_each_listed<true>(nbr, n, k, cnt, [&](int j) {
            if (j != k) visit(j);
        });
    } else {
        for_each_run(g, xi.x, xi.y, xi.z, p.h, [&](int lo, int hi) {
            for (int j = lo; j < hi; ++j) {
                float dx, dy, dz;
                if (j != k && dist2(xi, __ldg(xs + j), dx, dy, dz) < p.h2) visit(j);
            }
        });
    }
}

struct AdjIO {
    const float* x_out_adj;
    const float* v_out_adj;
    const float* rho_out_adj;
    float* x_in_adj;
    float* v_in_adj;
    float* f_ext_adj;
    const float* f_ext;
    const float* inv_mass;
    const float* gravity;
    float4* g;     // sorted: adj(a)
    float4* d;     // sorted: adj(dv)
    float* rho;    // sorted: adj(rho)
    float* bpart;  // per block: partial adj(B)
    const float4* acc;  // or null: the forward's sorted (a, 0), (dv, 0) (the segment tape), else recomputed
};

// reverse of integrate: recompute the forward particle update (bit for bit,
// so the clamp decisions are the forward's), then transpose it. The force
// sums a, dv are the forward's, stored (io.acc) or recomputed here.
__global__ void __launch_bounds__(kSphThreads, 2) k_adj_local(GridDev g, const float4* __restrict__ xs,
                                                              const float4* __restrict__ vs,
                                                              const float2* __restrict__ aux, int n,
                                                              const __grid_constant__ nsph_sph_params p,
                                                              const int4* __restrict__ nbr,
                                                              const int* __restrict__ ncnt, const AdjIO io)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float4 xi = xs[k], vi = vs[k];
        const int attr = __float_as_int(vi.w);
        const size_t i = (size_t)g.ids[k];
        const float xb1[3] = {io.x_out_adj[3 * i], io.x_out_adj[3 * i + 1], io.x_out_adj[3 * i + 2]};
        const float vb1[3] = {io.v_out_adj[3 * i], io.v_out_adj[3 * i + 1], io.v_out_adj[3 * i + 2]};
        float fb[3] = {0.f, 0.f, 0.f};
        float4 gk = make_float4(0.f, 0.f, 0.f, 0.f), dk = gk;
        if (!(attr & kAttrActive)) {
            for (int c = 0; c < 3; ++c) {
                io.x_in_adj[3 * i + c] = xb1[c];
                io.v_in_adj[3 * i + c] = vb1[c];
            }
        } else {
            ForceAcc acc{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (io.acc) {
                const float4 a = io.acc[2 * (size_t)k], d = io.acc[2 * (size_t)k + 1];
                acc = ForceAcc{a.x, a.y, a.z, d.x, d.y, d.z};
            } else {
                force_from_list<false>(g, xs, vs, aux, nbr, ncnt[k], n, k, xi, vi, aux[k].y, p, acc);
            }
            const bool dynamic = (attr & kAttrDynamic) != 0;
            float w = 0.f;
            float u[3] = {vi.x, vi.y, vi.z};
            if (dynamic) {  // the forward update of integrate_out, same rounding
                const int gw = attr >> kAttrGravShift;
                float fe[3] = {0.f, 0.f, 0.f};
                if (io.f_ext) {
                    w = io.inv_mass[i];
                    for (int c = 0; c < 3; ++c) fe[c] = __fmul_rn(io.f_ext[3 * i + c], w);
                }
                const float a[3] = {acc.ax, acc.ay, acc.az}, dv[3] = {acc.dvx, acc.dvy, acc.dvz};
                for (int c = 0; c < 3; ++c)
                    u[c] = __fmaf_rn(p.xsph_eps, dv[c],
                                     __fmaf_rn(__fadd_rn(__fadd_rn(a[c], fe[c]), io.gravity[3 * gw + c]), p.dt, u[c]));
            }
            const float vm = __fsqrt_rn(__fmaf_rn(u[2], u[2], __fmaf_rn(u[1], u[1], __fmul_rn(u[0], u[0]))));
            const bool vclamp = vm > p.v_max;
            const float s = vclamp ? __fdiv_rn(p.v_max, vm) : 1.f;
            const float xin[3] = {xi.x, xi.y, xi.z};
            float vcb[3], xpb[3];
            for (int c = 0; c < 3; ++c) {
                const float vc = vclamp ? __fmul_rn(u[c], s) : u[c];
                const float xp = __fmaf_rn(vc, p.dt, xin[c]);
                xpb[c] = xb1[c];
                vcb[c] = vb1[c];
                if (dynamic && p.use_box) {
                    if (xp < p.box_lo[c]) {  // x = lo, v = max(v, 0)
                        xpb[c] = 0.f;
                        if (vc < 0.f) vcb[c] = 0.f;
                    } else if (xp > p.box_hi[c]) {  // x = hi, v = min(v, 0)
                        xpb[c] = 0.f;
                        if (vc > 0.f) vcb[c] = 0.f;
                    }
                }
                vcb[c] += xpb[c] * p.dt;
            }
            float ub[3] = {vcb[0], vcb[1], vcb[2]};
            if (vclamp) {  // v = v_max u/|u|: adj(u) = (v_max/|u|)(adj(v) - u^ (u^ . adj(v)))
                const float inv = 1.f / vm;
                const float uh[3] = {u[0] * inv, u[1] * inv, u[2] * inv};
                const float dot = uh[0] * vcb[0] + uh[1] * vcb[1] + uh[2] * vcb[2];
                for (int c = 0; c < 3; ++c) ub[c] = s * (vcb[c] - uh[c] * dot);
            }
            for (int c = 0; c < 3; ++c) {
                io.x_in_adj[3 * i + c] = xpb[c];
                io.v_in_adj[3 * i + c] = ub[c];
            }
            if (dynamic) {
                gk = make_float4(ub[0] * p.dt, ub[1] * p.dt, ub[2] * p.dt, 0.f);
                dk = make_float4(ub[0] * p.xsph_eps, ub[1] * p.xsph_eps, ub[2] * p.xsph_eps, 0.f);
                if (io.f_ext)
                    for (int c = 0; c < 3; ++c) fb[c] = ub[c] * p.dt * w;
            }
        }
        if (io.f_ext_adj)
            for (int c = 0; c < 3; ++c) io.f_ext_adj[3 * i + c] += fb[c];
        io.g[k] = gk;
        io.d[k] = dk;
    }
}

// sum of v over the block, valid in thread 0 (a second call needs a
// __syncthreads() in between: the shared partials are reused)
__device__ __forceinline__ float block_sum(float v)
{
    __shared__ float part[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) part[warp] = v;
    __syncthreads();
    v = 0.f;
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? part[lane] : 0.f;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

// gather of the transposed pressure and XSPH terms, then adj(rho) through
// the EOS; per-block partial sums of adj(B)
__global__ void __launch_bounds__(kSphThreads, 2) k_adj_pair(GridDev g, const float4* __restrict__ xs,
                                                             const float4* __restrict__ vs,
                                                             const float2* __restrict__ aux,
                                                             const float2* __restrict__ rp, int n,
                                                             const __grid_constant__ nsph_sph_params p,
                                                             const int4* __restrict__ nbr,
                                                             const int* __restrict__ ncnt, const AdjIO io)
{
    float bsum = 0.f;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float4 xi = xs[k], vi = vs[k];
        const size_t i = (size_t)g.ids[k];
        if (!(__float_as_int(vi.w) & kAttrActive)) {
            io.rho[k] = 0.f;
            continue;
        }
        const float2 ak = aux[k];
        const float4 gk = io.g[k], dk = io.d[k];
        const float mk = xi.w;
        float pr2b = 0.f, morb = 0.f;
        float xb[3] = {0.f, 0.f, 0.f}, vb[3] = {0.f, 0.f, 0.f};
        for_each_neighbor(g, xs, nbr, ncnt[k], n, k, xi, p, [&](int j) {
            const float4 vj = __ldg(vs + j);
            if (!(__float_as_int(vj.w) & kAttrActive)) return;
            const float4 xj = __ldg(xs + j);
            const float2 aj = __ldg(aux + j);
            const float4 gj = __ldg(io.g + j), dj = __ldg(io.d + j);
            float dx, dy, dz;
            const float r2 = dist2(xi, xj, dx, dy, dz);
            const float r = __fsqrt_rn(r2);
            const float q = r * p.inv_h;
            const float w = kernel_w(q, p);
            const float yx = aj.x * dk.x - ak.x * dj.x, yy = aj.x * dk.y - ak.x * dj.y, yz = aj.x * dk.z - ak.x * dj.z;
            const float rvx = vj.x - vi.x, rvy = vj.y - vi.y, rvz = vj.z - vi.z;
            if (r2 > 0.f) {
                const float inv_r = 1.f / r;
                const float f = kernel_f(q, inv_r, p);
                const float dfr = kernel_df_over_r(q, inv_r, p);
                const float zx = mk * gj.x - xj.w * gk.x, zy = mk * gj.y - xj.w * gk.y, zz = mk * gj.z - xj.w * gk.z;
                const float zd = zx * dx + zy * dy + zz * dz;
                pr2b += f * zd;
                const float sp = ak.y + aj.y;
                const float cx = sp * dfr * zd + f * (rvx * yx + rvy * yy + rvz * yz);
                xb[0] += sp * f * zx + cx * dx;
                xb[1] += sp * f * zy + cx * dy;
                xb[2] += sp * f * zz + cx * dz;
            }
            vb[0] -= w * yx;
            vb[1] -= w * yy;
            vb[2] -= w * yz;
            morb -= w * (dj.x * rvx + dj.y * rvy + dj.z * rvz);
        });
        // adj(rho) from p/rho^2 (through the EOS) and m/rho
        const float2 rpk = rp[k];
        float rb = io.rho_out_adj ? io.rho_out_adj[i] : 0.f;
        if (rpk.x > 0.f) {
            const float rho = rpk.x, ratio = __fmul_rn(rho, p.inv_rho0);
            float pw1 = 1.f;  // ratio^(gamma-1)
            for (int e = 1; e < p.eos_gamma; ++e) pw1 = __fmul_rn(pw1, ratio);
            const float pw = p.eos_gamma > 0 ? __fmul_rn(pw1, ratio) : 1.f;
            const float praw = __fmul_rn(p.eos_b, __fsub_rn(pw, 1.f));
            const bool live = !(p.clamp_pressure && praw < 0.f);
            const float inv_rho = 1.f / rho, inv_rho2 = inv_rho * inv_rho;
            const float dp = (live && p.eos_gamma > 0) ? p.eos_b * (float)p.eos_gamma * pw1 * p.inv_rho0 : 0.f;
            rb += pr2b * (dp - 2.f * rpk.y * inv_rho) * inv_rho2 - morb * mk * inv_rho2;
            if (live) bsum += pr2b * (pw - 1.f) * inv_rho2;
        }
        io.rho[k] = rb;
        for (int c = 0; c < 3; ++c) {
            io.x_in_adj[3 * i + c] += xb[c];
            io.v_in_adj[3 * i + c] += vb[c];
        }
    }
    bsum = block_sum(bsum);
    if (threadIdx.x == 0) io.bpart[blockIdx.x] = bsum;
}

// gather of the transposed density sum
__global__ void __launch_bounds__(kSphThreads, 3) k_adj_density(GridDev g, const float4* __restrict__ xs,
                                                                const float4* __restrict__ vs, int n,
                                                                const __grid_constant__ nsph_sph_params p,
                                                                const int4* __restrict__ nbr,
                                                                const int* __restrict__ ncnt,
                                                                const float* __restrict__ rho_adj,
                                                                float* __restrict__ x_in_adj)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        if (!(__float_as_int(vs[k].w) & kAttrActive)) continue;
        const float4 xi = xs[k];
        const float rbk = rho_adj[k], mk = xi.w;
        float xb[3] = {0.f, 0.f, 0.f};
        for_each_neighbor(g, xs, nbr, ncnt[k], n, k, xi, p, [&](int j) {
            const float4 xj = __ldg(xs + j);
            float dx, dy, dz;
            const float r2 = dist2(xi, xj, dx, dy, dz);
            if (!(r2 > 0.f)) return;
            const float r = __fsqrt_rn(r2);
            const float c = kernel_f(r * p.inv_h, 1.f / r, p) * (rbk * xj.w + __ldg(rho_adj + j) * mk);
            xb[0] += c * dx;
            xb[1] += c * dy;
            xb[2] += c * dz;
        });
        const size_t i = (size_t)g.ids[k];
        for (int c = 0; c < 3; ++c) x_in_adj[3 * i + c] += xb[c];
    }
}

// adj(B) += sum of the per-block partials, in a fixed order
__global__ void k_adj_b_reduce(const float* __restrict__ bpart, int blocks, float* __restrict__ b_adj)
{
    float v = 0.f;
    for (int b = threadIdx.x; b < blocks; b += blockDim.x) v += bpart[b];
    v = block_sum(v);
    if (threadIdx.x == 0) *b_adj += v;
}

// ==========================================================================
// Surrogate step: the plain step's build and density pass (neighbour lists),
// then one kernel (k_surrogate_fused) that gathers each particle's force
// sums and 16 neighbour features, evaluates the MLP on the tensor cores
// (mlp.cuh) and integrates with the corrected acceleration a + da. The
// feature pass alone (k_force_features_list) serves the training data. The
// features are dimensionless (lengths / h, velocities / c0, accelerations
// h / c0^2, with c0^2 = B gamma / rho0):
//   0 rho/rho0   1 rho/rho0 - 1   2-4 sum V_j W (x_j - x_i) / h
//   5-7 sum V_j W (v_j - v_i) / c0 (the XSPH sum)   8-10 a h / c0^2
//   11 sum V_j W r^2 / h^2   12 Shepard sum V_i W(0) + sum V_j W
//   13 sum V_j F (v_j - v_i).(x_i - x_j) h / c0 (velocity divergence)
//   14 p / (rho0 c0^2)   15 |a| h / c0^2
// with V_j = m_j / rho_j and F = (dW/dr)/r.
// ==========================================================================
constexpr int kFeat = kMlpIn;

struct FeatAcc {
    float sw, mx, my, mz, m2, dvg;
};

// the pressure and XSPH terms of force_term_data (same statements, so the
// same rounding) plus the feature sums
__device__ __forceinline__ void force_feature_term(float4 xj, float4 vj, float2 aj, float4 xi, float4 vi, float pr2_i,
                                                   const nsph_sph_params& p, ForceAcc& acc, FeatAcc& fa)
{
    if (!(__float_as_int(vj.w) & kAttrActive)) return;
    float dx, dy, dz;
    const float r2 = dist2(xi, xj, dx, dy, dz);
    const float r = __fsqrt_rn(r2);
    const float q = __fmul_rn(r, p.inv_h);
    const float w = kernel_w(q, p);
    float f = 0.f;
    if (r2 > 0.f) {
        f = kernel_f(q, __frcp_rn(r), p);
        const float s = __fmul_rn(__fmul_rn(xj.w, __fadd_rn(pr2_i, aj.y)), f);
        acc.ax = __fmaf_rn(-s, dx, acc.ax);
        acc.ay = __fmaf_rn(-s, dy, acc.ay);
        acc.az = __fmaf_rn(-s, dz, acc.az);
    }
    const float c = __fmul_rn(aj.x, w);
    const float rvx = __fsub_rn(vj.x, vi.x), rvy = __fsub_rn(vj.y, vi.y), rvz = __fsub_rn(vj.z, vi.z);
    acc.dvx = __fmaf_rn(c, rvx, acc.dvx);
    acc.dvy = __fmaf_rn(c, rvy, acc.dvy);
    acc.dvz = __fmaf_rn(c, rvz, acc.dvz);
    fa.sw += c;
    fa.mx -= c * dx;
    fa.my -= c * dy;
    fa.mz -= c * dz;
    fa.m2 += c * r2;
    fa.dvg += aj.x * f * (rvx * dx + rvy * dy + rvz * dz);
}

// pressure and XSPH sums (the statements of force_term_data, so the same
// rounding) and the feature sums of particle k over its neighbour list, in
// order
__device__ __forceinline__ void force_features_from_list(const GridDev& g, const float4* __restrict__ xs,
                                                         const float4* __restrict__ vs,
                                                         const float2* __restrict__ aux, const int4* __restrict__ nbr,
                                                         int cnt, int n, int k, float4 xi, float4 vi, float pr2_i,
                                                         const nsph_sph_params& p, ForceAcc& acc, FeatAcc& fa)
{
    if (cnt <= kNbrSlots) {
        bool have = false;
        float4 pxj = make_float4(0.f, 0.f, 0.f, 0.f), pvj = pxj;
        float2 paj = make_float2(0.f, 0.f);
        for_each_listed<true>(nbr, n, k, cnt, [&](int j) {
            if (j == k) return;
            const float4 nxj = __ldg(xs + j);
            const float4 nvj = __ldg(vs + j);
            const float2 naj = __ldg(aux + j);
            if (have) force_feature_term(pxj, pvj, paj, xi, vi, pr2_i, p, acc, fa);
            pxj = nxj;
            pvj = nvj;
            paj = naj;
            have = true;
        });
        if (have) force_feature_term(pxj, pvj, paj, xi, vi, pr2_i, p, acc, fa);
    } else {
        for_each_run(g, xi.x, xi.y, xi.z, p.h, [&](int lo, int hi) {
            for (int j = lo; j < hi; ++j) {
                float dx, dy, dz;
                if (dist2(xi, __ldg(xs + j), dx, dy, dz) < p.h2 && j != k)
                    force_feature_term(__ldg(xs + j), __ldg(vs + j), __ldg(aux + j), xi, vi, pr2_i, p, acc, fa);
            }
        });
    }
}

// The 16 features of sorted particle k (all zero for an inactive one) and
// its force sums; adds the particle's compression max(0, rho/rho0 - 1) and
// 1 to (csum, ccount) when it is active.
__device__ __forceinline__ void particle_features(const GridDev& g, const float4* __restrict__ xs,
                                                  const float4* __restrict__ vs, const float2* __restrict__ aux,
                                                  const float2* __restrict__ rp, const int4* __restrict__ nbr,
                                                  const int* __restrict__ ncnt, int n, int k, float4 xi, float4 vi,
                                                  const nsph_sph_params& p, float (&f)[kFeat], ForceAcc& acc,
                                                  float& csum, float& ccount)
{
    acc = ForceAcc{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (!(__float_as_int(vi.w) & kAttrActive)) {
#pragma unroll
        for (int j = 0; j < kFeat; ++j) f[j] = 0.f;
        return;
    }
    const float c0sq = fmaxf(p.eos_b * (float)p.eos_gamma * p.inv_rho0, 1e-30f);
    const float inv_c0 = rsqrtf(c0sq);
    const float ascale = p.h / c0sq;
    const float2 ak = aux[k];
    FeatAcc fa{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    force_features_from_list(g, xs, vs, aux, nbr, ncnt[k], n, k, xi, vi, ak.y, p, acc, fa);
    const float2 rpk = rp[k];
    const float ratio = rpk.x * p.inv_rho0;
    f[0] = ratio;
    f[1] = ratio - 1.f;
    f[2] = fa.mx * p.inv_h;
    f[3] = fa.my * p.inv_h;
    f[4] = fa.mz * p.inv_h;
    f[5] = acc.dvx * inv_c0;
    f[6] = acc.dvy * inv_c0;
    f[7] = acc.dvz * inv_c0;
    f[8] = acc.ax * ascale;
    f[9] = acc.ay * ascale;
    f[10] = acc.az * ascale;
    f[11] = fa.m2 * p.inv_h * p.inv_h;
    f[12] = fa.sw + ak.x * p.sigma;
    f[13] = fa.dvg * p.h * inv_c0;
    f[14] = rpk.y * p.inv_rho0 / c0sq;
    f[15] = sqrtf(f[8] * f[8] + f[9] * f[9] + f[10] * f[10]);
    csum += fmaxf(ratio - 1.f, 0.f);
    ccount += 1.f;
}

// per sorted particle k: feat[16 k ..] and sacc[2k] = (a, 0), sacc[2k+1] =
// (dv, 0), from the neighbour lists; per block: (sum of max(0, rho/rho0 - 1),
// active count)
__global__ void __launch_bounds__(kSphThreads, 4) k_force_features_list(GridDev g, const float4* __restrict__ xs,
                                                                        const float4* __restrict__ vs,
                                                                        const float2* __restrict__ aux,
                                                                        const float2* __restrict__ rp, int n,
                                                                        const __grid_constant__ nsph_sph_params p,
                                                                        const int4* __restrict__ nbr,
                                                                        const int* __restrict__ ncnt,
                                                                        float* __restrict__ feat,
                                                                        float4* __restrict__ sacc,
                                                                        float* __restrict__ cpart)
{
    float csum = 0.f, ccount = 0.f;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float4 xi = xs[k], vi = vs[k];
        float f[kFeat];
        ForceAcc acc;
        particle_features(g, xs, vs, aux, rp, nbr, ncnt, n, k, xi, vi, p, f, acc, csum, ccount);
        float4* fo = reinterpret_cast<float4*>(feat + (size_t)k * kFeat);
#pragma unroll
        for (int j = 0; j < kFeat; j += 4) fo[j / 4] = make_float4(f[j], f[j + 1], f[j + 2], f[j + 3]);
        sacc[2 * (size_t)k] = make_float4(acc.ax, acc.ay, acc.az, 0.f);
        sacc[2 * (size_t)k + 1] = make_float4(acc.dvx, acc.dvy, acc.dvz, 0.f);
    }
    csum = block_sum(csum);
    __syncthreads();  // block_sum's shared partials are reused
    ccount = block_sum(ccount);
    if (threadIdx.x == 0) {
        cpart[2 * blockIdx.x] = csum;
        cpart[2 * blockIdx.x + 1] = ccount;
    }
}

// stats[0] = mean compression of this step; stats[1] = max since reset;
// stats[2] += 1; stats[3] += stats[0]
__global__ void k_compression_reduce(const float* __restrict__ cpart, int blocks, float* __restrict__ stats)
{
    float s = 0.f, c = 0.f;
    for (int b = threadIdx.x; b < blocks; b += blockDim.x) {
        s += cpart[2 * b];
        c += cpart[2 * b + 1];
    }
    s = block_sum(s);
    __syncthreads();
    c = block_sum(c);
    if (threadIdx.x == 0) {
        const float e = c > 0.f ? s / c : 0.f;
        stats[0] = e;
        stats[1] = fmaxf(stats[1], e);
        stats[2] += 1.f;
        stats[3] += e;
    }
}

// The surrogate step's force pass fused with the MLP: each CTA takes tiles
// of 128 consecutive sorted particles; every thread gathers its particle's
// pressure / XSPH sums and 16 features from the neighbour list, stages the
// normalised bf16 feature row straight into the A tile of layer 1 in shared
// memory, the tcgen05 chain runs (accumulators in TMEM), and the thread
// integrates with a + da. Features and force sums never leave the SM.
// While one CTA waits on its MMAs, the other resident CTAs gather. If an
// MMA-completion wait gives up (after wait_limit polls), the CTA issues no
// further MMAs, integrates its remaining particles without the correction
// (the plain step at this dt) and flags NSPH_STATUS_SURROGATE_TIMEOUT. Per
// CTA: (sum of max(0, rho/rho0 - 1), active count) into cpart.
__global__ void __launch_bounds__(kMlpTile, 6) k_surrogate_fused(const float* __restrict__ model, float acc_scale,
                                                                 int wait_limit, GridDev g,
                                                                 const float4* __restrict__ xs,
                                                                 const float4* __restrict__ vs,
                                                                 const float2* __restrict__ aux,
                                                                 const float2* __restrict__ rp, int n,
                                                                 const __grid_constant__ nsph_sph_params p,
                                                                 const int4* __restrict__ nbr,
                                                                 const int* __restrict__ ncnt, const StepOut o,
                                                                 float* __restrict__ cpart)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    MlpFwdSmem& s = *reinterpret_cast<MlpFwdSmem*>(smem_raw);
    const uint32_t tmem = mlp_cta_begin(model, s, kMlpFwdCols);
    uint32_t phase = 0;
    bool ok = true;
    float csum = 0.f, ccount = 0.f;
    const int tiles = (n + kMlpTile - 1) / kMlpTile;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int k = t * kMlpTile + threadIdx.x;
        const int kk = k < n ? k : 0;
        const float4 xi = xs[kk], vi = vs[kk];
        float f[kFeat];
        ForceAcc acc;
        if (k < n) {
            particle_features(g, xs, vs, aux, rp, nbr, ncnt, n, k, xi, vi, p, f, acc, csum, ccount);
        } else {
            acc = ForceAcc{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int j = 0; j < kFeat; ++j) f[j] = 0.f;
        }
        float y[kMlpOut] = {0.f, 0.f, 0.f};
        if (ok) {  // uniform across the CTA (mlp_wait makes the outcome uniform)
            mlp_stage_input(s, f);
            mlp_sync();
            ok = mlp_forward_tile(s, tmem, 0, 0, 0, phase, y, wait_limit);
        }
        if (k < n) {
            const int attr = __float_as_int(vi.w);
            if (ok && (attr & kAttrDynamic)) {
                acc.ax = __fadd_rn(acc.ax, acc_scale * mlp_denorm(s, y, 0));
                acc.ay = __fadd_rn(acc.ay, acc_scale * mlp_denorm(s, y, 1));
                acc.az = __fadd_rn(acc.az, acc_scale * mlp_denorm(s, y, 2));
            }
            integrate_out((size_t)g.ids[k], xi, vi, attr, rp[k], acc, p, p.dt, o);
        }
        __syncthreads();
    }
    if (!ok && o.status && threadIdx.x == 0) atomicOr(o.status, (unsigned)NSPH_STATUS_SURROGATE_TIMEOUT);
    csum = block_sum(csum);
    __syncthreads();
    ccount = block_sum(ccount);
    if (threadIdx.x == 0) {
        cpart[2 * blockIdx.x] = csum;
        cpart[2 * blockIdx.x + 1] = ccount;
    }
    mlp_cta_end(s, tmem, kMlpFwdCols, !ok, phase);
}

// k_surrogate_fused with kGroups tiles per CTA: groups of 128 threads share
// one copy of the weights (12 KB) and run their tiles independently (own
// input / hidden tiles, completion barrier, 64 TMEM columns, named barriers),
// so one group's MMA round trips overlap the other groups' gathers, and a CTA
// of 2 groups holds 53 KB of shared memory for 8 warps instead of 67 KB.
// Same per-particle arithmetic as k_surrogate_fused; the timeout rule
// applies per group.
template <int kGroups>
__global__ void __launch_bounds__(kGroups * kMlpTile, 6 / kGroups)
    k_surrogate_fused_groups(const float* __restrict__ model, float acc_scale, int wait_limit, GridDev g,
                             const float4* __restrict__ xs, const float4* __restrict__ vs,
                             const float2* __restrict__ aux, const float2* __restrict__ rp, int n,
                             const __grid_constant__ nsph_sph_params p, const int4* __restrict__ nbr,
                             const int* __restrict__ ncnt, const StepOut o, float* __restrict__ cpart)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    auto& s = *reinterpret_cast<MlpFwdGroupSmem<kGroups>*>(smem_raw);
    const int grp = threadIdx.x / kMlpTile, row = threadIdx.x % kMlpTile;
    mlp_stage_weights(model, s);
    if (threadIdx.x < kGroups) umma::mbar_init(&s.bar[threadIdx.x], 1);
    if (threadIdx.x < 32) umma::tmem_alloc(&s.tmem, kGroups * kMlpFwdCols);
    mlp_sync();
    const uint32_t tmem = s.tmem;
    uint32_t phase = 0;
    bool ok = true;
    float csum = 0.f, ccount = 0.f;
    const int tiles = (n + kMlpTile - 1) / kMlpTile;
    for (int t = blockIdx.x * kGroups + grp; t < tiles; t += gridDim.x * kGroups) {
        const int k = t * kMlpTile + row;
        const int kk = k < n ? k : 0;
        const float4 xi = xs[kk], vi = vs[kk];
        float f[kFeat];
        ForceAcc acc;
        if (k < n) {
            particle_features(g, xs, vs, aux, rp, nbr, ncnt, n, k, xi, vi, p, f, acc, csum, ccount);
        } else {
            acc = ForceAcc{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int j = 0; j < kFeat; ++j) f[j] = 0.f;
        }
        float y[kMlpOut] = {0.f, 0.f, 0.f};
        if (ok) {  // uniform across the group (mlp_group_wait makes the outcome uniform)
            mlp_group_stage_input(s, grp, row, f);
            mlp_group_sync(grp);
            ok = mlp_group_forward_tile(s, grp, row, tmem, phase, y, wait_limit);
        }
        if (k < n) {
            const int attr = __float_as_int(vi.w);
            if (ok && (attr & kAttrDynamic)) {
                acc.ax = __fadd_rn(acc.ax, acc_scale * mlp_denorm(s, y, 0));
                acc.ay = __fadd_rn(acc.ay, acc_scale * mlp_denorm(s, y, 1));
                acc.az = __fadd_rn(acc.az, acc_scale * mlp_denorm(s, y, 2));
            }
            integrate_out((size_t)g.ids[k], xi, vi, attr, rp[k], acc, p, p.dt, o);
        }
    }
    if (!ok && o.status && row == 0) atomicOr(o.status, (unsigned)NSPH_STATUS_SURROGATE_TIMEOUT);
    // a group whose wait gave up waits once more (bounded) for the completion
    // it left outstanding, before the CTA frees its TMEM
    if (!ok) umma::mbar_wait(&s.bar[grp], phase, kMlpWaitLimit);
    csum = block_sum(csum);
    __syncthreads();
    ccount = block_sum(ccount);
    if (threadIdx.x == 0) {
        cpart[2 * blockIdx.x] = csum;
        cpart[2 * blockIdx.x + 1] = ccount;
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (threadIdx.x < 32) umma::tmem_dealloc(tmem, kGroups * kMlpFwdCols);
}

// sorted scratch -> original order: feat (n x 16), acc (n x 6: a, dv)
__global__ void k_scatter_features(const int* __restrict__ ids, int n, const float* __restrict__ sfeat,
                                   const float4* __restrict__ sacc, float* __restrict__ feat_out,
                                   float* __restrict__ acc_out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t i = (size_t)ids[k];
    if (feat_out)
        for (int j = 0; j < kFeat; ++j) feat_out[i * kFeat + j] = sfeat[(size_t)k * kFeat + j];
    if (acc_out) {
        const float4 a = sacc[2 * (size_t)k], dv = sacc[2 * (size_t)k + 1];
        acc_out[6 * i + 0] = a.x;
        acc_out[6 * i + 1] = a.y;
        acc_out[6 * i + 2] = a.z;
        acc_out[6 * i + 3] = dv.x;
        acc_out[6 * i + 4] = dv.y;
        acc_out[6 * i + 5] = dv.z;
    }
}

__global__ void k_scatter_rho(const int* __restrict__ ids, int n, const float2* __restrict__ rp,
                              float* __restrict__ rho_out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) rho_out[ids[k]] = rp[k].x;
}

}  // namespace
}  // namespace nsph

// ==========================================================================
// C ABI: solver context
// ==========================================================================
using namespace nsph;

struct nsph_sph {
    Grid grid;
    int capacity = 0;
    float4* xs = nullptr;
    float4* vs = nullptr;
    float2* aux = nullptr;
    float2* rp = nullptr;
    int4* nbr = nullptr;       // kNbrGroups x capacity neighbour lists (group-major), every step form
    int* ncnt = nullptr;       //   neighbours per particle
    int fast = 0;              // plain step: tolerance arithmetic (nsph_sph_set_arithmetic)
    unsigned* status = nullptr;
    int last_n = 0;
    int last_launches = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // start, built, density, end
    nsph_sph_params* wparams = nullptr;  // batched worlds: per-world parameters (device)
    int wparams_set = 0;
    int persistent_blocks = 0;           // batched worlds: blocks of the persistent passes
    int launch_threads = 0;              // neighbour passes: threads per block (0 = default)
    int launch_blocks_per_sm = -1;       // neighbour passes: persistent blocks per SM (-1 = default, 0 = one thread per particle)
    int sms = 0;
    float4* adj_g = nullptr;             // adjoint scratch (nsph_sph_enable_adjoint), sorted order: adj(a)
    float4* adj_d = nullptr;             //   adj(dv)
    float* adj_rho = nullptr;            //   adj(rho)
    float* adj_bpart = nullptr;          //   per-block partial sums of adj(B)
    int adj_bcap = 0;                    //   entries of adj_bpart
    cudaEvent_t eva[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // adjoint / surrogate phases
    float* sfeat = nullptr;              // surrogate scratch (nsph_sph_enable_surrogate), sorted: 16 features
    float4* sacc = nullptr;              //   (a, 0), (dv, 0)
    float* cpart = nullptr;              //   per-block (compression sum, active count)
    int surr_ctas = 0;                   //   resident CTAs of the fused surrogate kernel (its grid)
    int surr_groups = 1;                 //   tiles of 128 particles per CTA (1: k_surrogate_fused, 2: the grouped kernel)
    int surr_wait_limit = -1;            //   polls of an MMA-completion wait (-1: kMlpWaitLimit)
    char* tape = nullptr;                // segment tape (nsph_sph_segment_adjoint): per step of a segment,
    int tape_steps = 0;                  //   the build and density outputs the step's reverse reads,
    size_t tape_step_bytes = 0;          //   tape_steps slots of tape_step_bytes, then two states
};

// One step's slot of the segment tape: the sorted mirrors, the density
// pass's outputs and neighbour lists, the grid (sorted ids, cell table) and
// the force pass's sums.
struct TapeStep {
    float4* xs;
    float4* vs;
    float2* aux;
    float2* rp;
    int4* nbr;
    int* ncnt;
    int* ids;
    int2* ranges;
    float4* acc;  // the force pass's (a, 0), (dv, 0) per sorted particle
};

static size_t tape_align(size_t b) { return (b + 255) & ~(size_t)255; }

static size_t tape_slot_bytes(size_t c, long long ncells)
{
    return 2 * tape_align(sizeof(float4) * c) + 2 * tape_align(sizeof(float2) * c) +
           tape_align(sizeof(int4) * kNbrGroups * c) + 2 * tape_align(sizeof(int) * c) +
           tape_align(sizeof(int2) * (size_t)ncells) + tape_align(sizeof(float4) * 2 * c);
}

static TapeStep tape_slot(const nsph_sph* s, int t)
{
    const size_t c = (size_t)s->capacity;
    char* b = s->tape + (size_t)t * s->tape_step_bytes;
    TapeStep ts;
    ts.xs = reinterpret_cast<float4*>(b);
    b += tape_align(sizeof(float4) * c);
    ts.vs = reinterpret_cast<float4*>(b);
    b += tape_align(sizeof(float4) * c);
    ts.aux = reinterpret_cast<float2*>(b);
    b += tape_align(sizeof(float2) * c);
    ts.rp = reinterpret_cast<float2*>(b);
    b += tape_align(sizeof(float2) * c);
    ts.nbr = reinterpret_cast<int4*>(b);
    b += tape_align(sizeof(int4) * kNbrGroups * c);
    ts.ncnt = reinterpret_cast<int*>(b);
    b += tape_align(sizeof(int) * c);
    ts.ids = reinterpret_cast<int*>(b);
    b += tape_align(sizeof(int) * c);
    ts.ranges = reinterpret_cast<int2*>(b);
    b += tape_align(sizeof(int2) * (size_t)s->grid.ncells);
    ts.acc = reinterpret_cast<float4*>(b);
    return ts;
}

// the two recompute states (x then v, 3 x capacity floats each) after the slots
static float* tape_state(const nsph_sph* s, int which)
{
    return reinterpret_cast<float*>(s->tape + (size_t)s->tape_steps * s->tape_step_bytes) +
           (size_t)which * 6 * (size_t)s->capacity;
}

// grid of a neighbour pass: one thread per particle, or a persistent grid of
// blocks_per_sm blocks per SM striding over the particles
static void pass_launch(const nsph_sph* s, int n, bool persistent_default, int& blocks, int& threads)
{
    threads = s->launch_threads > 0 ? s->launch_threads : kSphThreads;
    const int full = (n + threads - 1) / threads;
    int bps = s->launch_blocks_per_sm;
    if (bps < 0) bps = persistent_default ? -1 : 0;
    if (bps < 0)
        blocks = std::min(full, s->persistent_blocks > 0 ? s->persistent_blocks : full);
    else if (bps == 0)
        blocks = full;
    else
        blocks = std::min(full, std::max(1, s->sms * bps));
    blocks = std::max(blocks, 1);
}

// Record a timing event: as an external event node while the stream is being
// captured (so a replayed graph records it), as a plain record otherwise.
static cudaError_t record_mark(cudaEvent_t ev, cudaStream_t stream)
{
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(stream, &cap);
    if (e != cudaSuccess) return e;
    return cap == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, stream, cudaEventRecordExternal)
                                                : cudaEventRecord(ev, stream);
}

static void sph_free(nsph_sph* s)
{
    DeviceGuard guard(s->grid.device);
    for (cudaEvent_t& e : s->ev)
        if (e) {
            cudaEventDestroy(e);
            e = nullptr;
        }
    for (cudaEvent_t& e : s->eva)
        if (e) {
            cudaEventDestroy(e);
            e = nullptr;
        }
    cudaFree(s->xs);
    cudaFree(s->vs);
    cudaFree(s->aux);
    cudaFree(s->rp);
    cudaFree(s->nbr);
    cudaFree(s->ncnt);
    cudaFree(s->wparams);
    cudaFree(s->status);
    cudaFree(s->adj_g);
    cudaFree(s->adj_d);
    cudaFree(s->adj_rho);
    cudaFree(s->adj_bpart);
    cudaFree(s->sfeat);
    cudaFree(s->tape);
    cudaFree(s->sacc);
    cudaFree(s->cpart);
    grid_free(s->grid);
}

static int sph_create_common(nsph_sph* s, int device, int capacity);

extern "C" int nsph_sph_create(int device, int capacity, const int grid_dims[3], nsph_sph** out)
{
    clear_error();
    if (!out || !grid_dims) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (capacity < 0) return fail(NSPH_ERR_INVALID_ARG, "negative capacity");
    nsph_sph* s = new (std::nothrow) nsph_sph();
    if (!s) return fail(NSPH_ERR_OUT_OF_MEMORY, "host allocation failed");
    int st = grid_init(s->grid, grid_dims[0], grid_dims[1], grid_dims[2], device);
    if (st == NSPH_OK) st = sph_create_common(s, device, capacity);
    if (st == NSPH_OK) {  // the plain step's kernels
        DeviceGuard guard(device);
        cudaError_t e = cudaSuccess;
        cudaFuncAttributes fa;
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_density_list<false>);
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_force_list<false>);
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_density_list<true>);
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_force_list<true>);
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = fail(NSPH_ERR_OUT_OF_MEMORY, std::string("solver allocation: ") + cudaGetErrorString(e));
        }
    }
    if (st != NSPH_OK) {
        sph_free(s);
        delete s;
        return st;
    }
    *out = s;
    return NSPH_OK;
}

extern "C" int nsph_sph_create_worlds(int device, int capacity, int world_count, const int* world_dims,
                                      nsph_sph** out)
{
    clear_error();
    if (!out || !world_dims) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (capacity < 0) return fail(NSPH_ERR_INVALID_ARG, "negative capacity");
    nsph_sph* s = new (std::nothrow) nsph_sph();
    if (!s) return fail(NSPH_ERR_OUT_OF_MEMORY, "host allocation failed");
    int st = grid_init_worlds(s->grid, world_dims, world_count, device);
    if (st == NSPH_OK) st = sph_create_common(s, device, capacity);
    if (st == NSPH_OK) {
        DeviceGuard guard(device);
        cudaError_t e = cudaMalloc(&s->wparams, sizeof(nsph_sph_params) * (size_t)world_count);
        int sms = 0, per_sm = 0;
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_force_worlds, kSphThreads, 0);
        cudaFuncAttributes fa;
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_density_worlds);
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_neighbors_worlds);
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = fail(NSPH_ERR_CUDA, std::string("worlds setup: ") + cudaGetErrorString(e));
        }
        s->persistent_blocks = std::max(1, sms * std::max(1, per_sm));
    }
    if (st != NSPH_OK) {
        sph_free(s);
        delete s;
        return st;
    }
    *out = s;
    return NSPH_OK;
}

static int sph_create_common(nsph_sph* s, int device, int capacity)
{
    if (cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        s->sms = 1;
    }
    int st = grid_reserve(s->grid, capacity);
    if (st == NSPH_OK) {
        DeviceGuard guard(device);
        const size_t c = (size_t)(capacity > 0 ? capacity : 1);
        cudaError_t e = cudaMalloc(&s->xs, sizeof(float4) * (c + kXsPad));
        if (e == cudaSuccess) e = cudaMemset(s->xs + c, 0, sizeof(float4) * kXsPad);
        if (e == cudaSuccess) e = cudaMalloc(&s->vs, sizeof(float4) * c);
        if (e == cudaSuccess) e = cudaMalloc(&s->aux, sizeof(float2) * c);
        if (e == cudaSuccess) e = cudaMalloc(&s->rp, sizeof(float2) * c);
        if (e == cudaSuccess) e = cudaMalloc(&s->nbr, sizeof(int4) * kNbrGroups * c);
        if (e == cudaSuccess) e = cudaMalloc(&s->ncnt, sizeof(int) * c);
        if (e == cudaSuccess) e = cudaMalloc(&s->status, sizeof(unsigned));
        if (e == cudaSuccess) e = cudaMemset(s->status, 0, sizeof(unsigned));
        cudaFuncAttributes fa;
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_neighbors);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = fail(NSPH_ERR_OUT_OF_MEMORY, std::string("solver allocation: ") + cudaGetErrorString(e));
        }
    }
    if (st == NSPH_OK) s->capacity = capacity;
    return st;
}

extern "C" int nsph_sph_destroy(nsph_sph* solver)
{
    clear_error();
    if (!solver) return NSPH_OK;
    sph_free(solver);
    delete solver;
    return NSPH_OK;
}

static int check_params(const nsph_sph_params* p)
{
    if (!p) return fail(NSPH_ERR_INVALID_ARG, "null params");
    if (!(p->h > 0.f) || !(p->h2 > 0.f) || !(p->cell_inv > 0.f) || !isfinite(p->h) || !isfinite(p->cell_inv))
        return fail(NSPH_ERR_INVALID_ARG, "h and cell width must be positive and finite");
    if (p->eos_gamma < 0 || p->eos_gamma > 16) return fail(NSPH_ERR_INVALID_ARG, "eos_gamma out of [0, 16]");
    if (!(p->rho0 > 0.f)) return fail(NSPH_ERR_INVALID_ARG, "rho0 must be positive");
    return NSPH_OK;
}

// Checks shared by the single-world step entry points (the caller has
// checked the solver handle and the parameter block).
static int check_step_inputs(const nsph_sph* s, int n, const float* x_in, const float* v_in, const float* mass,
                             const float* inv_mass, const int* flags, const float* gravity, int world_count)
{
    if (n < 0) return fail(NSPH_ERR_INVALID_ARG, "negative particle count");
    if (n > s->capacity) return fail(NSPH_ERR_CAPACITY, "more particles than the solver was created for");
    if (world_count < 1 || !gravity) return fail(NSPH_ERR_INVALID_ARG, "gravity needs world_count >= 1");
    if (n > 0 && (!x_in || !v_in || !mass || !inv_mass || !flags))
        return fail(NSPH_ERR_INVALID_ARG, "null state or model array");
    if (s->grid.world_count > 0)
        return fail(NSPH_ERR_INVALID_ARG, "solver was created for batched worlds: use nsph_sph_step_worlds");
    return NSPH_OK;
}

// Enqueue one step on validated inputs: grid build + sorted gather, density,
// force + integrate (with the phase events when enabled).
static int step_enqueue(nsph_sph* s, const nsph_sph_params* p, int n, const float* x_in, const float* v_in,
                        const float* f_ext, const float* mass, const float* inv_mass, const int* flags,
                        const int* world, const float* gravity, int world_count, float* x_out, float* v_out,
                        float* rho_out, float* p_out, float* a_out, cudaStream_t cs, int& launches)
{
    GatherArgs ga{x_in, v_in, mass, inv_mass, flags, world, world_count, s->xs, s->vs};
    if (s->ev[0]) NSPH_CUDA_TRY(record_mark(s->ev[0], cs));
    int st = grid_build(s->grid, x_in, n, p->cell_width, p->cell_inv, &ga, s->status, cs, &launches);
    if (st != NSPH_OK) return st;
    s->last_n = n;
    if (s->ev[1]) NSPH_CUDA_TRY(record_mark(s->ev[1], cs));
    if (n > 0) {
        const GridDev g = s->grid.view();
        int blocks, threads;
        pass_launch(s, n, false, blocks, threads);
        if (s->fast)
            k_density_list<true><<<blocks, threads, 0, cs>>>(g, s->xs, s->vs, n, *p, s->aux, s->rp, s->nbr, s->ncnt,
                                                             s->status);
        else
            k_density_list<false><<<blocks, threads, 0, cs>>>(g, s->xs, s->vs, n, *p, s->aux, s->rp, s->nbr,
                                                              s->ncnt, s->status);
        NSPH_LAUNCH_CHECK("k_density_list");
        ++launches;
        if (s->ev[2]) NSPH_CUDA_TRY(record_mark(s->ev[2], cs));
        const StepOut o{f_ext, inv_mass, gravity, x_out, v_out, rho_out, p_out, a_out, s->status};
        if (s->fast)
            k_force_list<true><<<blocks, threads, 0, cs>>>(g, s->xs, s->vs, s->aux, s->rp, n, *p, s->nbr, s->ncnt, o);
        else
            k_force_list<false><<<blocks, threads, 0, cs>>>(g, s->xs, s->vs, s->aux, s->rp, n, *p, s->nbr, s->ncnt,
                                                            o);
        NSPH_LAUNCH_CHECK("k_force_list");
        ++launches;
    } else if (s->ev[2]) {
        NSPH_CUDA_TRY(record_mark(s->ev[2], cs));
    }
    if (s->ev[3]) NSPH_CUDA_TRY(record_mark(s->ev[3], cs));
    return NSPH_OK;
}

extern "C" int nsph_sph_step(nsph_sph* s, const nsph_sph_params* p, int n, const float* x_in, const float* v_in,
                             const float* f_ext, const float* mass, const float* inv_mass, const int* flags,
                             const int* world, const float* gravity, int world_count, float* x_out,
                             float* v_out, float* rho_out, float* p_out, float* a_out, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_sph_step");
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    int st = check_params(p);
    if (st == NSPH_OK) st = check_step_inputs(s, n, x_in, v_in, mass, inv_mass, flags, gravity, world_count);
    if (st != NSPH_OK) return st;
    if (n > 0 && (!x_out || !v_out)) return fail(NSPH_ERR_INVALID_ARG, "null state or model array");
    if (n > 0 && (x_out == x_in || v_out == v_in))
        return fail(NSPH_ERR_INVALID_ARG, "state_out must not alias state_in");
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    int launches = 0;
    st = step_enqueue(s, p, n, x_in, v_in, f_ext, mass, inv_mass, flags, world, gravity, world_count, x_out, v_out,
                      rho_out, p_out, a_out, (cudaStream_t)stream, launches);
    s->last_launches = launches;
    return st;
}

// [a, a + na) and [b, b + nb) (in floats) share memory
static bool overlaps(const float* a, size_t na, const float* b, size_t nb)
{
    return a < b + nb && b < a + na;
}

extern "C" int nsph_sph_rollout(nsph_sph* s, const nsph_sph_params* p, int n, int steps, const float* x0,
                                const float* v0, const float* f_ext, const float* mass, const float* inv_mass,
                                const int* flags, const int* world, const float* gravity, int world_count,
                                float* x_traj, float* v_traj, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_sph_rollout");
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    int st = check_params(p);
    if (st == NSPH_OK) st = check_step_inputs(s, n, x0, v0, mass, inv_mass, flags, gravity, world_count);
    if (st != NSPH_OK) return st;
    if (steps < 0) return fail(NSPH_ERR_INVALID_ARG, "negative step count");
    const size_t len = 3 * (size_t)n;
    if (n > 0 && steps > 0) {
        if (!x_traj || !v_traj) return fail(NSPH_ERR_INVALID_ARG, "null trajectory array");
        const size_t tot = len * (size_t)steps;
        if (overlaps(x_traj, tot, v_traj, tot) || overlaps(x0, len, x_traj, tot) || overlaps(v0, len, v_traj, tot) ||
            overlaps(x0, len, v_traj, tot) || overlaps(v0, len, x_traj, tot))
            return fail(NSPH_ERR_INVALID_ARG, "trajectory arrays overlap each other or the initial state");
    }
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    int launches = 0;
    for (int t = 0; t < steps && n > 0; ++t) {
        const float* xi = t == 0 ? x0 : x_traj + (size_t)(t - 1) * len;
        const float* vi = t == 0 ? v0 : v_traj + (size_t)(t - 1) * len;
        float* xo = x_traj + (size_t)t * len;
        float* vo = v_traj + (size_t)t * len;
        // inactive particles keep their velocity (the step leaves it untouched)
        NSPH_CUDA_TRY(cudaMemcpyAsync(vo, vi, sizeof(float) * len, cudaMemcpyDeviceToDevice, cs));
        st = step_enqueue(s, p, n, xi, vi, f_ext, mass, inv_mass, flags, world, gravity, world_count, xo, vo, nullptr,
                          nullptr, nullptr, cs, launches);
        if (st != NSPH_OK) return st;
    }
    s->last_launches = launches;
    return NSPH_OK;
}

extern "C" int nsph_sph_set_world_params(nsph_sph* s, const nsph_sph_params* params, int world_count)
{
    clear_error();
    if (!s || !params) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    if (s->grid.world_count <= 0) return fail(NSPH_ERR_INVALID_ARG, "solver was not created for batched worlds");
    if (world_count != s->grid.world_count) return fail(NSPH_ERR_INVALID_ARG, "world_count differs from the solver's");
    for (int w = 0; w < world_count; ++w) {
        const int st = check_params(params + w);
        if (st != NSPH_OK) return fail(st, "world " + std::to_string(w) + ": " + nsph_last_error());
    }
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    std::vector<WorldCells> wc((size_t)world_count);
    NSPH_CUDA_TRY(cudaMemcpy(wc.data(), s->grid.worlds, sizeof(WorldCells) * world_count, cudaMemcpyDeviceToHost));
    for (int w = 0; w < world_count; ++w) wc[w].inv = params[w].cell_inv;
    NSPH_CUDA_TRY(cudaMemcpy(s->grid.worlds, wc.data(), sizeof(WorldCells) * world_count, cudaMemcpyHostToDevice));
    NSPH_CUDA_TRY(cudaMemcpy(s->wparams, params, sizeof(nsph_sph_params) * world_count, cudaMemcpyHostToDevice));
    s->wparams_set = 1;
    return NSPH_OK;
}

extern "C" int nsph_sph_step_worlds(nsph_sph* s, float dt, int n, const float* x_in, const float* v_in,
                                    const float* f_ext, const float* mass, const float* inv_mass, const int* flags,
                                    const int* world, const float* gravity, int world_count, float* x_out,
                                    float* v_out, float* rho_out, float* p_out, float* a_out, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_sph_step_worlds");
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    if (s->grid.world_count <= 0) return fail(NSPH_ERR_INVALID_ARG, "solver was not created for batched worlds");
    if (!s->wparams_set) return fail(NSPH_ERR_INVALID_ARG, "world parameters not set (nsph_sph_set_world_params)");
    if (!isfinite(dt)) return fail(NSPH_ERR_INVALID_ARG, "dt must be finite");
    if (n < 0) return fail(NSPH_ERR_INVALID_ARG, "negative particle count");
    if (n > s->capacity) return fail(NSPH_ERR_CAPACITY, "more particles than the solver was created for");
    if (world_count != s->grid.world_count || !gravity)
        return fail(NSPH_ERR_INVALID_ARG, "gravity must have one row per world of the solver");
    if (n > 0 && (!x_in || !v_in || !mass || !inv_mass || !flags || !x_out || !v_out))
        return fail(NSPH_ERR_INVALID_ARG, "null state or model array");
    if (n > 0 && (x_out == x_in || v_out == v_in))
        return fail(NSPH_ERR_INVALID_ARG, "state_out must not alias state_in");
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    GatherArgs ga{x_in, v_in, mass, inv_mass, flags, world, world_count, s->xs, s->vs};
    int launches = 0;
    if (s->ev[0]) NSPH_CUDA_TRY(record_mark(s->ev[0], cs));
    int st = grid_build(s->grid, x_in, n, 0.f, 0.f, &ga, s->status, cs, &launches, world);
    if (st != NSPH_OK) return st;
    s->last_n = n;
    if (s->ev[1]) NSPH_CUDA_TRY(record_mark(s->ev[1], cs));
    if (n > 0) {
        int blocks, threads;
        pass_launch(s, n, true, blocks, threads);
        k_density_worlds<<<blocks, threads, 0, cs>>>(s->grid.worlds, s->wparams, s->grid.cell_ranges,
                                                         s->grid.point_ids, s->xs, s->vs, n, s->aux, s->rp, s->nbr,
                                                         s->ncnt, s->status);
        NSPH_LAUNCH_CHECK("k_density_worlds");
        ++launches;
        if (s->ev[2]) NSPH_CUDA_TRY(record_mark(s->ev[2], cs));
        const StepOut o{f_ext, inv_mass, gravity, x_out, v_out, rho_out, p_out, a_out, s->status};
        k_force_worlds<<<blocks, threads, 0, cs>>>(s->grid.worlds, s->wparams, s->grid.cell_ranges,
                                                       s->grid.point_ids, s->xs, s->vs, s->aux, s->rp, n, dt, s->nbr,
                                                       s->ncnt, o);
        NSPH_LAUNCH_CHECK("k_force_worlds");
        ++launches;
    } else if (s->ev[2]) {
        NSPH_CUDA_TRY(record_mark(s->ev[2], cs));
    }
    if (s->ev[3]) NSPH_CUDA_TRY(record_mark(s->ev[3], cs));
    s->last_launches = launches;
    return NSPH_OK;
}

extern "C" int nsph_sph_neighbors(const nsph_sph* s, const nsph_sph_params* p, int* counts,
                                  const long long* offsets, int* out_ids, void* stream)
{
    clear_error();
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    if (s->grid.world_count > 0) {
        if (!s->grid.built) return fail(NSPH_ERR_NOT_BUILT, "no step has run yet");
        if (out_ids ? !offsets : !counts)
            return fail(NSPH_ERR_INVALID_ARG, "counts (count call) or offsets (fill call) required");
        const int n = s->last_n;
        if (n == 0) return NSPH_OK;
        DeviceGuard guard(s->grid.device);
        if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
        k_neighbors_worlds<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
            s->grid.worlds, s->wparams, s->grid.cell_ranges, s->grid.point_ids, s->xs, s->vs, n, counts, offsets,
            out_ids);
        NSPH_LAUNCH_CHECK("k_neighbors_worlds");
        return NSPH_OK;
    }
    int st = check_params(p);
    if (st != NSPH_OK) return st;
    if (!s->grid.built) return fail(NSPH_ERR_NOT_BUILT, "no step has run yet");
    if (out_ids ? !offsets : !counts) return fail(NSPH_ERR_INVALID_ARG, "counts (count call) or offsets (fill call) required");
    const int n = s->last_n;
    if (n == 0) return NSPH_OK;
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    k_neighbors<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(s->grid.view(), s->xs, s->vs, n, *p, counts,
                                                                   offsets, out_ids);
    NSPH_LAUNCH_CHECK("k_neighbors");
    return NSPH_OK;
}

extern "C" int nsph_sph_get_grid_view(const nsph_sph* s, nsph_grid_view* view)
{
    clear_error();
    if (!s || !view) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    const Grid& g = s->grid;
    view->point_cells = g.point_cells;
    view->point_ids = g.point_ids;
    view->cell_starts = reinterpret_cast<const int*>(g.cell_ranges);
    view->cell_ends = reinterpret_cast<const int*>(g.cell_ranges) + 1;
    view->cell_stride = 2;
    view->num_points = g.num_points;
    view->dim_x = g.dx;
    view->dim_y = g.dy;
    view->dim_z = g.dz;
    view->cell_width = g.cell_width;
    view->cell_width_inv = g.cell_inv;
    view->built = g.built;
    return NSPH_OK;
}

extern "C" int nsph_sph_enable_phase_timing(nsph_sph* s, int enable)
{
    clear_error();
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    for (cudaEvent_t* set : {s->ev, s->eva}) {
        const int count = set == s->ev ? 4 : 6;
        for (int k = 0; k < count; ++k) {
            cudaEvent_t& e = set[k];
            if (enable && !e) NSPH_CUDA_TRY(cudaEventCreate(&e));
            if (!enable && e) {
                NSPH_CUDA_TRY(cudaEventDestroy(e));
                e = nullptr;
            }
        }
    }
    return NSPH_OK;
}

extern "C" int nsph_sph_phase_times(nsph_sph* s, float ms_out[3])
{
    clear_error();
    if (!s || !ms_out) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    if (!s->ev[0]) return fail(NSPH_ERR_INVALID_ARG, "phase timing is not enabled");
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    NSPH_CUDA_TRY(cudaEventSynchronize(s->ev[3]));
    for (int k = 0; k < 3; ++k) NSPH_CUDA_TRY(cudaEventElapsedTime(ms_out + k, s->ev[k], s->ev[k + 1]));
    return NSPH_OK;
}

extern "C" int nsph_sph_set_launch(nsph_sph* s, int threads, int blocks_per_sm)
{
    clear_error();
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    if (threads != 0 && (threads < 32 || threads > kSphThreads || (threads & 31)))
        return fail(NSPH_ERR_INVALID_ARG, "threads must be 0 or a multiple of 32 in [32, 256]");
    if (blocks_per_sm < -1 || blocks_per_sm > 64) return fail(NSPH_ERR_INVALID_ARG, "blocks_per_sm out of [-1, 64]");
    s->launch_threads = threads;
    s->launch_blocks_per_sm = blocks_per_sm;
    return NSPH_OK;
}

extern "C" int nsph_sph_last_launches(const nsph_sph* s) { return s ? s->last_launches : 0; }

extern "C" int nsph_sph_status(nsph_sph* s, unsigned int* status, void* stream)
{
    clear_error();
    if (!s || !status) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    NSPH_CUDA_TRY(cudaMemcpyAsync(status, s->status, sizeof(unsigned), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    NSPH_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return NSPH_OK;
}

extern "C" int nsph_sph_reset_status(nsph_sph* s, void* stream)
{
    clear_error();
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    NSPH_CUDA_TRY(cudaMemsetAsync(s->status, 0, sizeof(unsigned), (cudaStream_t)stream));
    return NSPH_OK;
}

// ==========================================================================
// C ABI: adjoint of the step
// ==========================================================================
extern "C" int nsph_sph_enable_adjoint(nsph_sph* s)
{
    clear_error();
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    if (s->grid.world_count > 0) return fail(NSPH_ERR_INVALID_ARG, "the adjoint supports single-world solvers only");
    if (s->adj_g) return NSPH_OK;
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    const size_t c = (size_t)(s->capacity > 0 ? s->capacity : 1);
    const int bcap = (int)((c + 31) / 32) + 1;  // blocks of a pass of >= 32 threads per block
    cudaError_t e = cudaMalloc(&s->adj_g, sizeof(float4) * c);
    if (e == cudaSuccess) e = cudaMalloc(&s->adj_d, sizeof(float4) * c);
    if (e == cudaSuccess) e = cudaMalloc(&s->adj_rho, sizeof(float) * c);
    if (e == cudaSuccess) e = cudaMalloc(&s->adj_bpart, sizeof(float) * (size_t)bcap);
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_adj_local);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_adj_pair);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_adj_density);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(s->adj_g);
        cudaFree(s->adj_d);
        cudaFree(s->adj_rho);
        cudaFree(s->adj_bpart);
        s->adj_g = s->adj_d = nullptr;
        s->adj_rho = s->adj_bpart = nullptr;
        return fail(NSPH_ERR_OUT_OF_MEMORY, std::string("adjoint allocation: ") + cudaGetErrorString(e));
    }
    s->adj_bcap = bcap;
    return NSPH_OK;
}

// The adjoint kernels of one step whose build and density outputs are `ts`
// (its grid seen through g). mark: record the adjoint phase events.
static int adjoint_kernels(nsph_sph* s, const nsph_sph_params* p, int n, const GridDev& g, const TapeStep& ts,
                           const AdjIO& io, float* eos_b_adj, cudaStream_t cs, int& launches, bool mark)
{
    int blocks, threads;
    pass_launch(s, n, false, blocks, threads);
    k_adj_local<<<blocks, threads, 0, cs>>>(g, ts.xs, ts.vs, ts.aux, n, *p, ts.nbr, ts.ncnt, io);
    NSPH_LAUNCH_CHECK("k_adj_local");
    if (mark && s->eva[3]) NSPH_CUDA_TRY(record_mark(s->eva[3], cs));
    k_adj_pair<<<blocks, threads, 0, cs>>>(g, ts.xs, ts.vs, ts.aux, ts.rp, n, *p, ts.nbr, ts.ncnt, io);
    NSPH_LAUNCH_CHECK("k_adj_pair");
    if (mark && s->eva[4]) NSPH_CUDA_TRY(record_mark(s->eva[4], cs));
    k_adj_density<<<blocks, threads, 0, cs>>>(g, ts.xs, ts.vs, n, *p, ts.nbr, ts.ncnt, io.rho, io.x_in_adj);
    NSPH_LAUNCH_CHECK("k_adj_density");
    launches += 3;
    if (eos_b_adj) {
        k_adj_b_reduce<<<1, 256, 0, cs>>>(io.bpart, blocks, eos_b_adj);
        NSPH_LAUNCH_CHECK("k_adj_b_reduce");
        ++launches;
    }
    return NSPH_OK;
}

// Enqueue the reverse of one step on validated inputs.
static int adjoint_enqueue(nsph_sph* s, const nsph_sph_params* p, int n, const float* x_in, const float* v_in,
                           const float* f_ext, const float* mass, const float* inv_mass, const int* flags,
                           const int* world, const float* gravity, int world_count, const float* x_out_adj,
                           const float* v_out_adj, const float* rho_out_adj, float* x_in_adj, float* v_in_adj,
                           float* f_ext_adj, float* eos_b_adj, cudaStream_t cs, int& launches)
{
    GatherArgs ga{x_in, v_in, mass, inv_mass, flags, world, world_count, s->xs, s->vs};
    if (s->eva[0]) NSPH_CUDA_TRY(record_mark(s->eva[0], cs));
    int st = grid_build(s->grid, x_in, n, p->cell_width, p->cell_inv, &ga, s->status, cs, &launches);
    if (st != NSPH_OK) return st;
    s->last_n = n;
    if (s->eva[1]) NSPH_CUDA_TRY(record_mark(s->eva[1], cs));
    if (n > 0) {
        const GridDev g = s->grid.view();
        int blocks, threads;
        pass_launch(s, n, false, blocks, threads);
        k_density_list<false><<<blocks, threads, 0, cs>>>(g, s->xs, s->vs, n, *p, s->aux, s->rp, s->nbr, s->ncnt,
                                                          s->status);
        NSPH_LAUNCH_CHECK("k_density_list");
        if (s->eva[2]) NSPH_CUDA_TRY(record_mark(s->eva[2], cs));
        ++launches;
        const AdjIO io{x_out_adj, v_out_adj, rho_out_adj, x_in_adj, v_in_adj, f_ext_adj, f_ext, inv_mass, gravity,
                       s->adj_g, s->adj_d, s->adj_rho, s->adj_bpart};
        const TapeStep ts{s->xs, s->vs, s->aux, s->rp, s->nbr, s->ncnt, nullptr, nullptr, nullptr};
        st = adjoint_kernels(s, p, n, g, ts, io, eos_b_adj, cs, launches, true);
        if (st != NSPH_OK) return st;
    } else {
        for (int k = 2; k < 5; ++k)
            if (s->eva[k]) NSPH_CUDA_TRY(record_mark(s->eva[k], cs));
    }
    if (s->eva[5]) NSPH_CUDA_TRY(record_mark(s->eva[5], cs));
    return NSPH_OK;
}

static int check_adjoint_ready(const nsph_sph* s)
{
    if (s->grid.world_count > 0) return fail(NSPH_ERR_INVALID_ARG, "the adjoint supports single-world solvers only");
    if (!s->adj_g) return fail(NSPH_ERR_INVALID_ARG, "adjoint scratch not allocated (nsph_sph_enable_adjoint)");
    return NSPH_OK;
}

extern "C" int nsph_sph_step_adjoint(nsph_sph* s, const nsph_sph_params* p, int n, const float* x_in,
                                     const float* v_in, const float* f_ext, const float* mass, const float* inv_mass,
                                     const int* flags, const int* world, const float* gravity, int world_count,
                                     const float* x_out_adj, const float* v_out_adj, const float* rho_out_adj,
                                     float* x_in_adj, float* v_in_adj, float* f_ext_adj, float* eos_b_adj,
                                     void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_sph_step_adjoint");
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    int st = check_params(p);
    if (st == NSPH_OK) st = check_adjoint_ready(s);
    if (st == NSPH_OK) st = check_step_inputs(s, n, x_in, v_in, mass, inv_mass, flags, gravity, world_count);
    if (st != NSPH_OK) return st;
    if (n > 0 && (!x_out_adj || !v_out_adj || !x_in_adj || !v_in_adj))
        return fail(NSPH_ERR_INVALID_ARG, "null adjoint array");
    if (n > 0 && ((const float*)x_in_adj == v_out_adj || (const float*)v_in_adj == x_out_adj || x_in_adj == v_in_adj))
        return fail(NSPH_ERR_INVALID_ARG, "position and velocity adjoints must not share memory");
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    int launches = 0;
    st = adjoint_enqueue(s, p, n, x_in, v_in, f_ext, mass, inv_mass, flags, world, gravity, world_count, x_out_adj,
                         v_out_adj, rho_out_adj, x_in_adj, v_in_adj, f_ext_adj, eos_b_adj, (cudaStream_t)stream,
                         launches);
    s->last_launches = launches;
    return st;
}

extern "C" int nsph_sph_rollout_adjoint(nsph_sph* s, const nsph_sph_params* p, int n, int steps,
                                        const float* x_states, const float* v_states, const float* f_ext,
                                        const float* mass, const float* inv_mass, const int* flags, const int* world,
                                        const float* gravity, int world_count, float* x_adj, float* v_adj,
                                        float* f_ext_adj, float* eos_b_adj, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_sph_rollout_adjoint");
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    int st = check_params(p);
    if (st == NSPH_OK) st = check_adjoint_ready(s);
    if (st == NSPH_OK) st = check_step_inputs(s, n, x_states, v_states, mass, inv_mass, flags, gravity, world_count);
    if (st != NSPH_OK) return st;
    if (steps < 0) return fail(NSPH_ERR_INVALID_ARG, "negative step count");
    const size_t len = 3 * (size_t)n;
    if (n > 0 && steps > 0) {
        if (!x_adj || !v_adj) return fail(NSPH_ERR_INVALID_ARG, "null adjoint array");
        const size_t tot = len * (size_t)steps;
        if (overlaps(x_adj, len, v_adj, len) || overlaps(x_adj, len, x_states, tot) ||
            overlaps(x_adj, len, v_states, tot) || overlaps(v_adj, len, x_states, tot) ||
            overlaps(v_adj, len, v_states, tot))
            return fail(NSPH_ERR_INVALID_ARG, "adjoint arrays overlap each other or the states");
    }
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    int launches = 0;
    for (int t = steps - 1; t >= 0 && n > 0; --t) {
        st = adjoint_enqueue(s, p, n, x_states + (size_t)t * len, v_states + (size_t)t * len, f_ext, mass, inv_mass,
                             flags, world, gravity, world_count, x_adj, v_adj, nullptr, x_adj, v_adj, f_ext_adj,
                             eos_b_adj, cs, launches);
        if (st != NSPH_OK) return st;
    }
    s->last_launches = launches;
    return NSPH_OK;
}

extern "C" int nsph_sph_reserve_segment(nsph_sph* s, int steps)
{
    clear_error();
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    if (s->grid.world_count > 0) return fail(NSPH_ERR_INVALID_ARG, "the adjoint supports single-world solvers only");
    if (steps < 0) return fail(NSPH_ERR_INVALID_ARG, "negative step count");
    if (steps <= s->tape_steps) return NSPH_OK;
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    const size_t c = (size_t)(s->capacity > 0 ? s->capacity : 1);
    const size_t slot = tape_slot_bytes(c, s->grid.ncells);
    const size_t bytes = slot * (size_t)steps + tape_align(sizeof(float) * 12 * c);
    char* t = nullptr;
    const cudaError_t e = cudaMalloc(&t, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(NSPH_ERR_OUT_OF_MEMORY, "segment tape of " + std::to_string(bytes) + " bytes: " +
                                                cudaGetErrorString(e));
    }
    cudaFree(s->tape);
    s->tape = t;
    s->tape_steps = steps;
    s->tape_step_bytes = slot;
    return NSPH_OK;
}

extern "C" int nsph_sph_segment_adjoint(nsph_sph* s, const nsph_sph_params* p, int n, int steps, const float* x0,
                                        const float* v0, const float* f_ext, const float* mass,
                                        const float* inv_mass, const int* flags, const int* world,
                                        const float* gravity, int world_count, float* x_adj, float* v_adj,
                                        float* f_ext_adj, float* eos_b_adj, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_sph_segment_adjoint");
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    int st = check_params(p);
    if (st == NSPH_OK) st = check_adjoint_ready(s);
    if (st == NSPH_OK) st = check_step_inputs(s, n, x0, v0, mass, inv_mass, flags, gravity, world_count);
    if (st != NSPH_OK) return st;
    if (steps < 0) return fail(NSPH_ERR_INVALID_ARG, "negative step count");
    const size_t len = 3 * (size_t)n;
    if (n > 0 && steps > 0) {
        if (!x_adj || !v_adj) return fail(NSPH_ERR_INVALID_ARG, "null adjoint array");
        if (overlaps(x_adj, len, v_adj, len) || overlaps(x_adj, len, x0, len) || overlaps(x_adj, len, v0, len) ||
            overlaps(v_adj, len, x0, len) || overlaps(v_adj, len, v0, len))
            return fail(NSPH_ERR_INVALID_ARG, "adjoint arrays overlap each other or the initial state");
    }
    if (n == 0 || steps == 0) {
        s->last_launches = 0;
        return NSPH_OK;
    }
    st = nsph_sph_reserve_segment(s, steps);
    if (st != NSPH_OK) return st;
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    int launches = 0;
    int blocks, threads;
    pass_launch(s, n, false, blocks, threads);
    // forward: the build, density and force passes of every step, their
    // outputs into the step's slot (the last step's new state is not used)
    for (int t = 0; t < steps; ++t) {
        const float* xi = t == 0 ? x0 : tape_state(s, t & 1);
        const float* vi = t == 0 ? v0 : tape_state(s, t & 1) + len;
        const TapeStep ts = tape_slot(s, t);
        GatherArgs ga{xi, vi, mass, inv_mass, flags, world, world_count, ts.xs, ts.vs};
        st = grid_build(s->grid, xi, n, p->cell_width, p->cell_inv, &ga, s->status, cs, &launches);
        if (st != NSPH_OK) return st;
        NSPH_CUDA_TRY(cudaMemcpyAsync(ts.ranges, s->grid.cell_ranges, sizeof(int2) * (size_t)s->grid.ncells,
                                      cudaMemcpyDeviceToDevice, cs));
        NSPH_CUDA_TRY(cudaMemcpyAsync(ts.ids, s->grid.point_ids, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice,
                                      cs));
        GridDev g = s->grid.view();
        g.ranges = ts.ranges;
        g.ids = ts.ids;
        k_density_list<false><<<blocks, threads, 0, cs>>>(g, ts.xs, ts.vs, n, *p, ts.aux, ts.rp, ts.nbr, ts.ncnt,
                                                          s->status);
        NSPH_LAUNCH_CHECK("k_density_list");
        ++launches;
        float* xo = tape_state(s, (t + 1) & 1);
        float* vo = xo + len;
        // inactive particles keep their velocity (the step leaves it untouched)
        if (t + 1 < steps) NSPH_CUDA_TRY(cudaMemcpyAsync(vo, vi, sizeof(float) * len, cudaMemcpyDeviceToDevice, cs));
        const StepOut o{f_ext, inv_mass, gravity, xo, vo, nullptr, nullptr, nullptr, s->status, ts.acc};
        k_force_list<false><<<blocks, threads, 0, cs>>>(g, ts.xs, ts.vs, ts.aux, ts.rp, n, *p, ts.nbr, ts.ncnt, o);
        NSPH_LAUNCH_CHECK("k_force_list");
        ++launches;
    }
    // the solver's mirrors describe its grid's last build (the last step's input)
    const TapeStep last = tape_slot(s, steps - 1);
    NSPH_CUDA_TRY(cudaMemcpyAsync(s->xs, last.xs, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToDevice, cs));
    NSPH_CUDA_TRY(cudaMemcpyAsync(s->vs, last.vs, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToDevice, cs));
    s->last_n = n;
    // reverse, from the slots
    AdjIO io{x_adj, v_adj, nullptr, x_adj, v_adj, f_ext_adj, f_ext, inv_mass, gravity,
             s->adj_g, s->adj_d, s->adj_rho, s->adj_bpart, nullptr};
    for (int t = steps - 1; t >= 0; --t) {
        const TapeStep ts = tape_slot(s, t);
        io.acc = ts.acc;
        GridDev g = s->grid.view();
        g.ranges = ts.ranges;
        g.ids = ts.ids;
        // phase events: the build and density phases of a step reversed from
        // the tape are empty (the recompute ran them)
        for (int k = 0; k < 3; ++k)
            if (s->eva[k]) NSPH_CUDA_TRY(record_mark(s->eva[k], cs));
        st = adjoint_kernels(s, p, n, g, ts, io, eos_b_adj, cs, launches, true);
        if (st != NSPH_OK) return st;
        if (s->eva[5]) NSPH_CUDA_TRY(record_mark(s->eva[5], cs));
    }
    s->last_launches = launches;
    return NSPH_OK;
}

extern "C" int nsph_sph_adjoint_phase_times(nsph_sph* s, float ms_out[5])
{
    clear_error();
    if (!s || !ms_out) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    if (!s->eva[0]) return fail(NSPH_ERR_INVALID_ARG, "phase timing is not enabled");
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    NSPH_CUDA_TRY(cudaEventSynchronize(s->eva[5]));
    for (int k = 0; k < 5; ++k) NSPH_CUDA_TRY(cudaEventElapsedTime(ms_out + k, s->eva[k], s->eva[k + 1]));
    return NSPH_OK;
}

// ==========================================================================
// C ABI: surrogate step
// ==========================================================================
// Default launch of the fused surrogate kernel: CTAs of two 128-particle
// tiles sharing the weights, as many per SM as fit (3: registers), with the
// carveout they need. Measured on the relaxed 1M tank (same box, back to
// back): 0.273 ms per launch; one tile per CTA: 0.292 ms at 5 CTAs per SM,
// 0.319 at 4, 0.395 at 6 (which leaves about 28 KB of L1 for the gathers).
constexpr int kSurrogateCtasPerSm = 5;  // CTAs per SM when tiles_per_cta = 1
constexpr int kSurrogateGroups = 2;

// resident CTAs per SM of a fused surrogate kernel: registers (allocated per
// warp in units of 256), shared memory (plus the per-CTA reservation) and
// the SM's 512 TMEM columns; 0 on a CUDA error
template <class K>
static int surrogate_per_sm(K kernel, int threads, size_t smem, int tmem_cols, int device)
{
    cudaFuncAttributes fa;
    int smem_sm = 0, reserved = 0, regs_sm = 0;
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const int warp_regs = ((fa.numRegs * 32 + 255) / 256) * 256;
    const int by_regs = regs_sm / (warp_regs * (threads / 32));
    const int by_smem = smem_sm / (int)(smem + fa.sharedSizeBytes + reserved);
    return std::min(std::min(by_regs, by_smem), kTmemCols / tmem_cols);
}

static int set_surrogate_ctas(nsph_sph* s, int ctas_per_sm, int groups)
{
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    int sms = 0, smem_sm = 0, reserved = 0;
    NSPH_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->grid.device));
    NSPH_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, s->grid.device));
    NSPH_CUDA_TRY(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, s->grid.device));
    if (groups == 0) groups = kSurrogateGroups;
    const size_t smem = groups == 2 ? sizeof(MlpFwdGroupSmem<2>) : sizeof(MlpFwdSmem);
    const int most = groups == 2 ? surrogate_per_sm(k_surrogate_fused_groups<2>, 2 * kMlpTile, smem,
                                                    2 * (int)kMlpFwdCols, s->grid.device)
                                 : surrogate_per_sm(k_surrogate_fused, kMlpTile, smem, (int)kMlpFwdCols,
                                                    s->grid.device);
    if (most <= 0 || sms <= 0 || smem_sm <= 0) return fail(NSPH_ERR_CUDA, "cannot size the surrogate grid");
    const int def = groups == 2 ? most : kSurrogateCtasPerSm;
    const int per_sm = std::max(1, std::min(ctas_per_sm == 0 ? def : ctas_per_sm, most));
    // the shared-memory carveout that holds per_sm CTAs, so that the rest of
    // the SM's unified L1 / shared storage serves the neighbour gathers
    const int need = per_sm * (int)(smem + reserved);
    const int pct = std::min(100, (need * 100 + smem_sm - 1) / smem_sm);
    if (groups == 2)
        NSPH_CUDA_TRY(
            cudaFuncSetAttribute(k_surrogate_fused_groups<2>, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
    else
        NSPH_CUDA_TRY(cudaFuncSetAttribute(k_surrogate_fused, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
    s->surr_ctas = sms * per_sm;
    s->surr_groups = groups;
    return NSPH_OK;
}

extern "C" int nsph_sph_enable_surrogate(nsph_sph* s)
{
    clear_error();
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    if (s->grid.world_count > 0) return fail(NSPH_ERR_INVALID_ARG, "the surrogate supports single-world solvers only");
    if (s->sfeat) return NSPH_OK;
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    const size_t c = (size_t)(s->capacity > 0 ? s->capacity : 1);
    const size_t blocks = std::max((c + 31) / 32 + 1, (size_t)4096);  // per-block partials of either pass
    cudaError_t e = cudaMalloc(&s->sfeat, sizeof(float) * kFeat * c);
    if (e == cudaSuccess) e = cudaMalloc(&s->sacc, sizeof(float4) * 2 * c);
    if (e == cudaSuccess) e = cudaMalloc(&s->cpart, sizeof(float) * 2 * blocks);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_surrogate_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(MlpFwdSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_surrogate_fused_groups<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(MlpFwdGroupSmem<2>));
    if (e == cudaSuccess) {  // an upper bound on either kernel's grid, for the partials
        const int most = mlp_resident_grid(k_surrogate_fused, sizeof(MlpFwdSmem), s->grid.device);
        if (most <= 0) e = cudaErrorUnknown;
        else if (most + 1 > (int)blocks) e = cudaErrorInvalidValue;
    }
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_force_features_list);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(s->sfeat);
        cudaFree(s->sacc);
        cudaFree(s->cpart);
        s->sfeat = s->cpart = nullptr;
        s->sacc = nullptr;
        return fail(NSPH_ERR_OUT_OF_MEMORY, std::string("surrogate allocation: ") + cudaGetErrorString(e));
    }
    return set_surrogate_ctas(s, 0, 0);  // the default launch and its carveout
}

// grid build, density pass and (with `features`) the feature pass into the
// sorted scratch (with `mark`, records phase events 0-2 when phase timing is
// enabled: start, built, after the density pass)
static int features_enqueue(nsph_sph* s, const nsph_sph_params* p, int n, const float* x_in, const float* v_in,
                            const float* mass, const float* inv_mass, const int* flags, const int* world,
                            int world_count, cudaStream_t cs, int& launches, int& blocks, bool mark = false,
                            bool features = true)
{
    GatherArgs ga{x_in, v_in, mass, inv_mass, flags, world, world_count, s->xs, s->vs};
    if (mark && s->eva[0]) NSPH_CUDA_TRY(record_mark(s->eva[0], cs));
    int st = grid_build(s->grid, x_in, n, p->cell_width, p->cell_inv, &ga, s->status, cs, &launches);
    if (st != NSPH_OK) return st;
    s->last_n = n;
    blocks = 0;
    if (mark && s->eva[1]) NSPH_CUDA_TRY(record_mark(s->eva[1], cs));
    if (n > 0) {
        const GridDev g = s->grid.view();
        int threads;
        pass_launch(s, n, false, blocks, threads);
        k_density_list<false><<<blocks, threads, 0, cs>>>(g, s->xs, s->vs, n, *p, s->aux, s->rp, s->nbr, s->ncnt,
                                                          s->status);
        NSPH_LAUNCH_CHECK("k_density_list");
        ++launches;
        if (mark && s->eva[2]) NSPH_CUDA_TRY(record_mark(s->eva[2], cs));
        if (features) {
            k_force_features_list<<<blocks, threads, 0, cs>>>(g, s->xs, s->vs, s->aux, s->rp, n, *p, s->nbr,
                                                              s->ncnt, s->sfeat, s->sacc, s->cpart);
            NSPH_LAUNCH_CHECK("k_force_features_list");
            ++launches;
        }
    } else if (mark && s->eva[2]) {
        NSPH_CUDA_TRY(record_mark(s->eva[2], cs));
    }
    return NSPH_OK;
}

static int check_surrogate_ready(const nsph_sph* s)
{
    if (s->grid.world_count > 0) return fail(NSPH_ERR_INVALID_ARG, "the surrogate supports single-world solvers only");
    if (!s->sfeat) return fail(NSPH_ERR_INVALID_ARG, "surrogate scratch not allocated (nsph_sph_enable_surrogate)");
    return NSPH_OK;
}

extern "C" int nsph_sph_features(nsph_sph* s, const nsph_sph_params* p, int n, const float* x_in, const float* v_in,
                                 const float* mass, const float* inv_mass, const int* flags, const int* world,
                                 const float* gravity, int world_count, float* feat_out, float* acc_out,
                                 float* rho_out, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_sph_features");
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    int st = check_params(p);
    if (st == NSPH_OK) st = check_surrogate_ready(s);
    if (st == NSPH_OK) st = check_step_inputs(s, n, x_in, v_in, mass, inv_mass, flags, gravity, world_count);
    if (st != NSPH_OK) return st;
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    int launches = 0, blocks = 0;
    st = features_enqueue(s, p, n, x_in, v_in, mass, inv_mass, flags, world, world_count, cs, launches, blocks);
    if (st != NSPH_OK) return st;
    if (n > 0 && (feat_out || acc_out)) {
        k_scatter_features<<<(n + 255) / 256, 256, 0, cs>>>(s->grid.point_ids, n, s->sfeat, s->sacc, feat_out,
                                                              acc_out);
        NSPH_LAUNCH_CHECK("k_scatter_features");
        ++launches;
    }
    if (n > 0 && rho_out) {
        k_scatter_rho<<<(n + 255) / 256, 256, 0, cs>>>(s->grid.point_ids, n, s->rp, rho_out);
        NSPH_LAUNCH_CHECK("k_scatter_rho");
        ++launches;
    }
    s->last_launches = launches;
    return NSPH_OK;
}

extern "C" int nsph_sph_step_surrogate(nsph_sph* s, const nsph_sph_params* p, const float* model, float acc_scale,
                                       int n, const float* x_in, const float* v_in, const float* f_ext,
                                       const float* mass, const float* inv_mass, const int* flags, const int* world,
                                       const float* gravity, int world_count, float* x_out, float* v_out,
                                       float* rho_out, float* p_out, float* stats, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_sph_step_surrogate");
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    int st = check_params(p);
    if (st == NSPH_OK) st = check_surrogate_ready(s);
    if (st == NSPH_OK) st = check_step_inputs(s, n, x_in, v_in, mass, inv_mass, flags, gravity, world_count);
    if (st != NSPH_OK) return st;
    if (n > 0 && (!x_out || !v_out || !model || !stats)) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    if (n > 0 && (x_out == x_in || v_out == v_in))
        return fail(NSPH_ERR_INVALID_ARG, "state_out must not alias state_in");
    if (!isfinite(acc_scale)) return fail(NSPH_ERR_INVALID_ARG, "acc_scale must be finite");
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    int launches = 0, blocks = 0;
    st = features_enqueue(s, p, n, x_in, v_in, mass, inv_mass, flags, world, world_count, cs, launches, blocks,
                          true, false);
    if (st != NSPH_OK) return st;
    if (n > 0) {
        const int tiles = (n + kMlpTile - 1) / kMlpTile;
        const int wait_limit = s->surr_wait_limit >= 0 ? s->surr_wait_limit : kMlpWaitLimit;
        const StepOut o{f_ext, inv_mass, gravity, x_out, v_out, rho_out, p_out, nullptr, s->status};
        int grid;
        if (s->surr_groups == 2) {
            grid = std::min((tiles + 1) / 2, std::max(1, s->surr_ctas));
            k_surrogate_fused_groups<2><<<grid, 2 * kMlpTile, sizeof(MlpFwdGroupSmem<2>), cs>>>(
                model, acc_scale, wait_limit, s->grid.view(), s->xs, s->vs, s->aux, s->rp, n, *p, s->nbr, s->ncnt, o,
                s->cpart);
            NSPH_LAUNCH_CHECK("k_surrogate_fused_groups");
        } else {
            grid = std::min(tiles, std::max(1, s->surr_ctas));
            k_surrogate_fused<<<grid, kMlpTile, sizeof(MlpFwdSmem), cs>>>(model, acc_scale, wait_limit,
                                                                          s->grid.view(), s->xs, s->vs, s->aux, s->rp,
                                                                          n, *p, s->nbr, s->ncnt, o, s->cpart);
            NSPH_LAUNCH_CHECK("k_surrogate_fused");
        }
        if (s->eva[3]) NSPH_CUDA_TRY(record_mark(s->eva[3], cs));
        k_compression_reduce<<<1, 256, 0, cs>>>(s->cpart, grid, stats);
        NSPH_LAUNCH_CHECK("k_compression_reduce");
        launches += 2;
    } else if (s->eva[3]) {
        NSPH_CUDA_TRY(record_mark(s->eva[3], cs));
    }
    if (s->eva[4]) NSPH_CUDA_TRY(record_mark(s->eva[4], cs));
    s->last_launches = launches;
    return NSPH_OK;
}

extern "C" int nsph_sph_set_surrogate_launch(nsph_sph* s, int ctas_per_sm, int tiles_per_cta)
{
    clear_error();
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    if (ctas_per_sm < 0 || ctas_per_sm > 64) return fail(NSPH_ERR_INVALID_ARG, "ctas_per_sm out of [0, 64]");
    if (tiles_per_cta < 0 || tiles_per_cta > 2) return fail(NSPH_ERR_INVALID_ARG, "tiles_per_cta out of [0, 2]");
    if (!s->sfeat) return fail(NSPH_ERR_INVALID_ARG, "surrogate not enabled (nsph_sph_enable_surrogate)");
    return set_surrogate_ctas(s, ctas_per_sm, tiles_per_cta);
}

extern "C" int nsph_sph_set_surrogate_wait_limit(nsph_sph* s, int polls)
{
    clear_error();
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    if (polls < -1) return fail(NSPH_ERR_INVALID_ARG, "poll count below -1");
    s->surr_wait_limit = polls;
    return NSPH_OK;
}

extern "C" int nsph_sph_set_arithmetic(nsph_sph* s, int mode)
{
    clear_error();
    if (!s) return fail(NSPH_ERR_INVALID_ARG, "null solver");
    if (mode != NSPH_ARITH_EXACT && mode != NSPH_ARITH_FAST) return fail(NSPH_ERR_INVALID_ARG, "unknown arithmetic");
    s->fast = mode == NSPH_ARITH_FAST;
    return NSPH_OK;
}

extern "C" int nsph_sph_surrogate_phase_times(nsph_sph* s, float ms_out[4])
{
    clear_error();
    if (!s || !ms_out) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    if (!s->eva[0]) return fail(NSPH_ERR_INVALID_ARG, "phase timing is not enabled");
    DeviceGuard guard(s->grid.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    NSPH_CUDA_TRY(cudaEventSynchronize(s->eva[4]));
    for (int k = 0; k < 4; ++k) NSPH_CUDA_TRY(cudaEventElapsedTime(ms_out + k, s->eva[k], s->eva[k + 1]));
    return NSPH_OK;
}
