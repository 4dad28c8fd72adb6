/*
 * sph_f64.c — fp64 instance of sph_impl.h: the truth the fp32 results are
 * measured against. Same fp32 neighbour topology, double arithmetic and
 * double constants (oracle_phys_f64).
 * TEST INFRASTRUCTURE ONLY (the checker; see nsph_oracle.h).
 */
#include "oracle_internal.h"

#define REAL double
#define SFX(name) name##_f64
#define RSQRT sqrt
#define RFMA fma
#define RABS fabs
#include "sph_impl.h"

int oracle_sph_step_f64(const nsph_sph_params* p, const oracle_phys_f64* phys, const int* grid_dims, int n,
                        const float* x_in, const float* v_in, const float* f_ext, const float* mass,
                        const float* inv_mass, const int* flags, const int* world, const float* gravity,
                        int world_count, double* x_out, double* v_out, double* rho_out, double* p_out,
                        double* a_out, double* a_scale_out)
{
    if (!p || !phys || !grid_dims) return NSPH_ERR_INVALID_ARG;
    phys_f64 ph;
    ph.h = phys->h;
    ph.inv_h = phys->inv_h;
    ph.sigma = phys->sigma;
    ph.dsigma = phys->dsigma;
    ph.c_near = phys->c_near;
    ph.c_far = phys->c_far;
    ph.rho0 = phys->rho0;
    ph.inv_rho0 = phys->inv_rho0;
    ph.eos_b = phys->eos_b;
    ph.xsph_eps = phys->xsph_eps;
    ph.v_max = phys->v_max;
    ph.dt = phys->dt;
    for (int c = 0; c < 3; ++c) {
        ph.box_lo[c] = phys->box_lo[c];
        ph.box_hi[c] = phys->box_hi[c];
    }
    ph.eos_gamma = phys->eos_gamma;
    ph.clamp_pressure = phys->clamp_pressure;
    ph.use_box = phys->use_box;
    return sph_step_impl_f64(p, &ph, grid_dims, n, x_in, v_in, f_ext, mass, inv_mass, flags, world, gravity,
                             world_count, x_out, v_out, rho_out, p_out, a_out, a_scale_out);
}

void oracle_integrate_particles_f64(const float* x, const float* v, const float* f, const float* inv_mass,
                                    const int* flags, const int* world, const float* gravity, int world_count,
                                    int n, double dt, double v_max, double* x_new, double* v_new)
{
    integrate_impl_f64(x, v, f, inv_mass, flags, world, gravity, world_count, n, dt, v_max, x_new, v_new);
}
