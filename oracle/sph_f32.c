/*
 * sph_f32.c — fp32 instance of sph_impl.h: the same fp32 constants the
 * device receives (nsph_sph_params), fp32 arithmetic.
 * TEST INFRASTRUCTURE ONLY (the checker; see nsph_oracle.h).
 */
#include "oracle_internal.h"

#define REAL float
#define SFX(name) name##_f32
#define RSQRT sqrtf
#define RFMA fmaf
#define RABS fabsf
#include "sph_impl.h"

int oracle_sph_step_f32(const nsph_sph_params* p, const int* grid_dims, int n, const float* x_in,
                        const float* v_in, const float* f_ext, const float* mass, const float* inv_mass,
                        const int* flags, const int* world, const float* gravity, int world_count,
                        float* x_out, float* v_out, float* rho_out, float* p_out, float* a_out,
                        float* a_scale_out)
{
    if (!p || !grid_dims) return NSPH_ERR_INVALID_ARG;
    phys_f32 ph;
    ph.h = p->h;
    ph.inv_h = p->inv_h;
    ph.sigma = p->sigma;
    ph.dsigma = p->dsigma;
    ph.c_near = p->c_near;
    ph.c_far = p->c_far;
    ph.rho0 = p->rho0;
    ph.inv_rho0 = p->inv_rho0;
    ph.eos_b = p->eos_b;
    ph.xsph_eps = p->xsph_eps;
    ph.v_max = p->v_max;
    ph.dt = p->dt;
    for (int c = 0; c < 3; ++c) {
        ph.box_lo[c] = p->box_lo[c];
        ph.box_hi[c] = p->box_hi[c];
    }
    ph.eos_gamma = p->eos_gamma;
    ph.clamp_pressure = p->clamp_pressure;
    ph.use_box = p->use_box;
    return sph_step_impl_f32(p, &ph, grid_dims, n, x_in, v_in, f_ext, mass, inv_mass, flags, world, gravity,
                             world_count, x_out, v_out, rho_out, p_out, a_out, a_scale_out);
}

void oracle_integrate_particles_f32(const float* x, const float* v, const float* f, const float* inv_mass,
                                    const int* flags, const int* world, const float* gravity, int world_count,
                                    int n, float dt, float v_max, float* x_new, float* v_new)
{
    integrate_impl_f32(x, v, f, inv_mass, flags, world, gravity, world_count, n, dt, v_max, x_new, v_new);
}
