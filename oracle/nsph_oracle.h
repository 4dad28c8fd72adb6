/*
 * nsph_oracle.h — CPU oracle for the particle-fluid hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker, not the product: only the
 * tests, the smoke check and the benchmark's CPU-baseline leg load it. The
 * product (libnsph.so) never links or calls it.
 *
 * What it restates:
 *   - Warp's HashGrid (external warp-lang 1.14.0.dev20260511, not vendored in
 *     the reference; call sites newton/_src/sim/builder.py:9853,
 *     newton/_src/solvers/xpbd/solver_xpbd.py:139,315-319,
 *     newton/_src/solvers/semi_implicit/kernels_contact.py:54,68,71):
 *     truncating cell coordinates, 2^20 origin offset, modulo dims, stable
 *     sort by cell id, [start,end) ranges, x-fastest query order. Restated
 *     from Warp's published behaviour.
 *   - integrate_particles, newton/_src/solvers/solver.py:10-47.
 *   - the WCSPH step (no counterpart in the reference; published methods:
 *     Monaghan 1992 cubic spline and symmetric pressure gradient, Tait EOS
 *     per Monaghan 1994 / Becker & Teschner 2007, XSPH per Monaghan 1989),
 *     arranged like the neighbour gather of kernels_contact.py:35-84.
 *
 * Parity status: UNPINNED against the reference itself. The reference holds
 * no golden vectors for HashGrid or particle dynamics and cannot run here
 * (warp-lang is absent), and it has no SPH at all. The oracle is pinned by
 * analytic known answers instead (kernel normalisation, lattice density,
 * free fall, a brute-force O(N^2) neighbour search) — see tests/.
 *
 * Precision: the grid, the neighbour test and the cell ids are always fp32
 * (bit-exact mirror of the device). The SPH arithmetic is compiled twice:
 * *_f32 (same fp32 constants as the device) and *_f64 (truth).
 */
#ifndef NSPH_ORACLE_H
#define NSPH_ORACLE_H

#include "../include/nsph.h"

#ifdef __cplusplus
extern "C" {
#endif

/* float -> int32 like CUDA cvt.rzi.s32.f32: truncate, saturate, NaN -> 0 */
int oracle_trunc_sat(float v);
/* Warp hash_grid_index for virtual cell (x, y, z). */
int oracle_grid_index(int x, int y, int z, int dim_x, int dim_y, int dim_z);

/* HashGrid.build(points, radius) restated. Outputs: point_cells / point_ids
 * (n, sorted), cell_starts / cell_ends (dim_x*dim_y*dim_z, zero for empty). */
int oracle_grid_build(const float* points, int n, float radius, int dim_x, int dim_y, int dim_z,
                      int* point_cells, int* point_ids, int* cell_starts, int* cell_ends);

/* hash_grid_query + hash_grid_query_next restated: candidates of one query
 * in Warp's order, no distance test. Writes at most max_out ids, returns the
 * total count. cell_inv = 1.0f / cell_width. */
long long oracle_grid_query(const int* point_ids, const int* cell_starts, const int* cell_ends,
                            int dim_x, int dim_y, int dim_z, float cell_inv,
                            const float pos[3], float radius, int* out, long long max_out);

/* SPH neighbour lists in original order (self included; active only):
 * counts[i]; and when out_ids != NULL, ids at out_ids[offsets[i] ...]. */
int oracle_sph_neighbors(const nsph_sph_params* p, int n, const float* x, const int* flags,
                         const int* grid_dims, int* counts, const long long* offsets, int* out_ids);

/* Physics constants in double for the fp64 truth path. */
typedef struct oracle_phys_f64 {
    double h, inv_h, sigma, dsigma, rho0, inv_rho0, eos_b, xsph_eps, v_max, dt;
    double c_near, c_far;
    double box_lo[3], box_hi[3];
    int eos_gamma, clamp_pressure, use_box;
} oracle_phys_f64;

/* One WCSPH step. Inputs are the fp32 state; outputs in the function's
 * precision. v_out must hold the previous contents (inactive particles leave
 * it untouched). Any of rho_out, p_out, a_out, a_scale_out may be NULL.
 * a_scale_out[i] = sum_j |m_j (P_i + P_j) dW/dr| (the magnitude of the
 * summands of the pressure acceleration), for normalising sum errors. */
int oracle_sph_step_f32(const nsph_sph_params* p, const int* grid_dims, int n,
                        const float* x_in, const float* v_in, const float* f_ext,
                        const float* mass, const float* inv_mass, const int* flags, const int* world,
                        const float* gravity, int world_count,
                        float* x_out, float* v_out, float* rho_out, float* p_out, float* a_out,
                        float* a_scale_out);
int oracle_sph_step_f64(const nsph_sph_params* p, const oracle_phys_f64* phys, const int* grid_dims, int n,
                        const float* x_in, const float* v_in, const float* f_ext,
                        const float* mass, const float* inv_mass, const int* flags, const int* world,
                        const float* gravity, int world_count,
                        double* x_out, double* v_out, double* rho_out, double* p_out, double* a_out,
                        double* a_scale_out);

/* integrate_particles (solver.py:10-47) in fp32 and fp64. */
void oracle_integrate_particles_f32(const float* x, const float* v, const float* f, const float* inv_mass,
                                    const int* flags, const int* world, const float* gravity, int world_count,
                                    int n, float dt, float v_max, float* x_new, float* v_new);
void oracle_integrate_particles_f64(const float* x, const float* v, const float* f, const float* inv_mass,
                                    const int* flags, const int* world, const float* gravity, int world_count,
                                    int n, double dt, double v_max, double* x_new, double* v_new);

/* ---- adjoint (sph_adjoint.c): fp64 state, fp64 neighbour sets ----------
 * oracle_adj_step_f64: one step on a double state (inactive particles keep x
 * and v). oracle_adj_vjp_f64: given the adjoints of x_out and v_out (and
 * optionally of the step's density), the adjoints of x, v, f_ext (optional)
 * and of the EOS stiffness B (optional, one double, overwritten). */
int oracle_adj_step_f64(const oracle_phys_f64* ph, int n, const double* x, const double* v, const double* f_ext,
                        const double* mass, const double* inv_mass, const int* flags, const int* world,
                        const double* gravity, int world_count, double* x_out, double* v_out, double* rho_out);
int oracle_adj_vjp_f64(const oracle_phys_f64* ph, int n, const double* x, const double* v, const double* f_ext,
                       const double* mass, const double* inv_mass, const int* flags, const int* world,
                       const double* gravity, int world_count, const double* x_out_adj, const double* v_out_adj,
                       const double* rho_out_adj, double* x_adj, double* v_adj, double* f_adj, double* b_adj);

/* ---- particle-particle contact (contact.c), fp32 ------------------------
 * The grid is built on x with cell width grid_radius (HashGrid.build(x,
 * grid_radius)) and dims; f_out rows of inactive particles are not written;
 * deltas are accumulated (+=). */
int oracle_particle_contact_forces(const nsph_contact_params* p, float grid_radius, const int* dims, int n,
                                   const float* x, const float* v, const float* radius, const int* flags,
                                   float* f_out);
int oracle_particle_contact_deltas(float grid_radius, const int* dims, int n, const float* x, const float* v,
                                   const float* inv_mass, const float* radius, const int* flags, float k_mu,
                                   float k_cohesion, float max_radius, float dt, float relaxation, float* deltas);
/* The same with the grid built on grid_x while the particles sit at x (the
 * XPBD iterations query the grid of the predicted positions). */
int oracle_particle_contact_deltas_grid(const float* grid_x, float grid_radius, const int* dims, int n,
                                        const float* x, const float* v, const float* inv_mass, const float* radius,
                                        const int* flags, float k_mu, float k_cohesion, float max_radius, float dt,
                                        float relaxation, float* deltas);

/* Number of OpenMP threads the oracle uses (0 = OpenMP default). */
void oracle_set_threads(int n);
int  oracle_get_threads(void);

/* ---- particle raycast depth camera (raycast.c), fp32 --------------------
 * The grid is built on x with cell width search_radius and dims; depth
 * (height x width) holds the initial nearest hits (negative = none) and
 * receives the nearer particle hits. oracle_raycast_clamp_no_hits turns
 * values >= max_distance into -1. */
int oracle_raycast_particles(const float* x, const float* radius, int n, const int* dims,
                             const nsph_raycast_camera* cam, float search_radius, float march_step, int max_steps,
                             float* depth);
void oracle_raycast_clamp_no_hits(float* depth, int count, float max_distance);

/* Particles against static analytic shapes and the XPBD particle update
 * (shapes.c): soft contacts in (particle, shape) order, processed in contact
 * order; fp32 restatements of create_soft_contacts,
 * eval_particle_body_contact, solve_particle_shape_contacts,
 * apply_particle_shape_restitution and apply_particle_deltas for shapes
 * without a body. */
int oracle_soft_contacts_create(const nsph_shape* shapes, int shape_count, int n, const float* x,
                                const float* radius, const int* flags, const int* world, float margin, int max,
                                int* count, int* particle, int* shape, float* body_pos, float* body_vel,
                                float* normal);
int oracle_shape_contact_forces(const nsph_shape* shapes, int count, const int* particle, const int* shape,
                                const float* body_pos, const float* body_vel, const float* normal,
                                const nsph_soft_contact_params* prm, const float* x, const float* v,
                                const float* radius, const int* flags, float* f);
int oracle_shape_contact_deltas(const nsph_shape* shapes, int count, const int* particle, const int* shape,
                                const float* body_pos, const float* body_vel, const float* normal,
                                const nsph_soft_contact_params* prm, const float* x, const float* v,
                                const float* inv_mass, const float* radius, const int* flags, float* delta);
int oracle_shape_restitution(int n, int count, const int* particle, const float* body_pos, const float* body_vel,
                             const float* normal, const nsph_soft_contact_params* prm, const float* v_new,
                             const float* x_old, const float* v_old, const float* radius, const int* flags,
                             float* v_out);
void oracle_apply_particle_deltas(int n, const float* x_orig, const float* x_pred, const int* flags,
                                  const float* delta, float dt, float v_max, float* x_out, float* v_out);

#ifdef __cplusplus
}
#endif
#endif
