// integrate.cu — integrate_particles, newton/_src/solvers/solver.py:10-47,
// launched by SolverBase.integrate_particles (solver.py:266-299).
//   v1 = v0 + (f*w + g[max(world,0)]*step(-w))*dt; |v1| clamped to v_max;
//   x1 = x0 + v1*dt; inactive particles: x1 = x0, v_new not written.
// A pure streaming kernel (48 B read + 24 B written per particle): one thread
// per particle, AoS vec3 loads as three scalar loads that coalesce across the
// warp.
#include "nsph_internal.cuh"

namespace nsph {
namespace {

__global__ void k_integrate(const float* __restrict__ x, const float* __restrict__ v, const float* __restrict__ f,
                            const float* __restrict__ inv_mass, const int* __restrict__ flags,
                            const int* __restrict__ world, const float* __restrict__ gravity, int world_count,
                            int n, float dt, float v_max, float* __restrict__ x_new, float* __restrict__ v_new)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const size_t i = (size_t)t;
    const float x0 = x[3 * i], y0 = x[3 * i + 1], z0 = x[3 * i + 2];
    if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) {
        x_new[3 * i] = x0;
        x_new[3 * i + 1] = y0;
        x_new[3 * i + 2] = z0;
        return;
    }
    const float w = inv_mass[i];
    int gw = world ? world[i] : 0;
    gw = gw < 0 ? 0 : (gw >= world_count ? world_count - 1 : gw);
    const float gate = (-w < 0.f) ? 1.f : 0.f;  // wp.step(-w)
    // v1 = fma(f*w + g*gate, dt, v0), rounded exactly as written
    float v1x = __fmaf_rn(__fadd_rn(__fmul_rn(f[3 * i], w), __fmul_rn(gravity[3 * gw], gate)), dt, v[3 * i]);
    float v1y = __fmaf_rn(__fadd_rn(__fmul_rn(f[3 * i + 1], w), __fmul_rn(gravity[3 * gw + 1], gate)), dt, v[3 * i + 1]);
    float v1z = __fmaf_rn(__fadd_rn(__fmul_rn(f[3 * i + 2], w), __fmul_rn(gravity[3 * gw + 2], gate)), dt, v[3 * i + 2]);
    const float m = __fsqrt_rn(__fmaf_rn(v1z, v1z, __fmaf_rn(v1y, v1y, __fmul_rn(v1x, v1x))));
    if (m > v_max) {
        const float s = __fdiv_rn(v_max, m);
        v1x = __fmul_rn(v1x, s);
        v1y = __fmul_rn(v1y, s);
        v1z = __fmul_rn(v1z, s);
    }
    x_new[3 * i] = __fmaf_rn(v1x, dt, x0);
    x_new[3 * i + 1] = __fmaf_rn(v1y, dt, y0);
    x_new[3 * i + 2] = __fmaf_rn(v1z, dt, z0);
    v_new[3 * i] = v1x;
    v_new[3 * i + 1] = v1y;
    v_new[3 * i + 2] = v1z;
}

}  // namespace
}  // namespace nsph

using namespace nsph;

extern "C" int nsph_integrate_particles(const float* x, const float* v, const float* f, const float* inv_mass,
                                        const int* flags, const int* world, const float* gravity, int world_count,
                                        int num, float dt, float v_max, float* x_new, float* v_new, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_integrate_particles");
    if (num < 0) return fail(NSPH_ERR_INVALID_ARG, "negative particle count");
    if (num == 0) return NSPH_OK;
    if (!x || !v || !f || !inv_mass || !flags || !gravity || !x_new || !v_new)
        return fail(NSPH_ERR_INVALID_ARG, "null array");
    if (world_count < 1) return fail(NSPH_ERR_INVALID_ARG, "gravity needs world_count >= 1");
    k_integrate<<<(num + 255) / 256, 256, 0, (cudaStream_t)stream>>>(x, v, f, inv_mass, flags, world, gravity,
                                                                    world_count, num, dt, v_max, x_new, v_new);
    NSPH_LAUNCH_CHECK("k_integrate");
    return NSPH_OK;
}
