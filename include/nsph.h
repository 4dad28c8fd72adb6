/*
 * nsph.h — C ABI of libnsph.so, the sm_100a implementation of Newton's
 * particle-fluid hot path (hash-grid neighbour search + WCSPH step).
 *
 * Every entry point takes plain pointers and sizes. Pointers named *device*
 * below are CUDA device pointers (e.g. torch.Tensor.data_ptr() of a CUDA
 * tensor). `stream` is a cudaStream_t passed as void* (0 = legacy default
 * stream). Every entry point returns an int status (NSPH_OK == 0); no C++
 * exception crosses this boundary and no kernel traps. The message of the last
 * failure on the calling host thread is returned by nsph_last_error().
 *
 * Entry points that enqueue work are stream-ordered and perform no host
 * synchronisation and no device allocation, so they can be captured into a
 * CUDA graph (the Newton contract exercised by
 * newton/tests/test_runtime_gravity.py:141-210). Allocation happens only in
 * the *_create / *_reserve calls.
 *
 * Reference interfaces replaced (paths inside the Newton source tree):
 *   - wp.HashGrid (external warp-lang 1.14.0.dev20260511), constructed at
 *     newton/_src/sim/builder.py:9853, reserved at
 *     newton/_src/solvers/xpbd/solver_xpbd.py:139, built at
 *     newton/_src/solvers/xpbd/solver_xpbd.py:315-319, queried from kernels at
 *     newton/_src/solvers/semi_implicit/kernels_contact.py:54,68,71.
 *   - the integrate_particles kernel, newton/_src/solvers/solver.py:10-47,
 *     launched by SolverBase.integrate_particles, solver.py:266-299.
 *   - SolverBase.step, newton/_src/solvers/solver.py:301-316, for the new
 *     WCSPH solver (the reference has no SPH solver; the step follows the
 *     neighbour-gather structure of kernels_contact.py:35-84).
 */
#ifndef NSPH_H
#define NSPH_H

#if defined(__GNUC__)
#define NSPH_API __attribute__((visibility("default")))
#else
#define NSPH_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define NSPH_OK                 0
#define NSPH_ERR_INVALID_ARG    1   /* bad pointer, size or parameter           */
#define NSPH_ERR_CAPACITY       2   /* more points than reserved                 */
#define NSPH_ERR_CUDA           3   /* a CUDA runtime call failed                */
#define NSPH_ERR_NOT_BUILT      4   /* query before the first build              */
#define NSPH_ERR_OUT_OF_MEMORY  5   /* allocation in *_create / *_reserve failed */

/* ---- device-side status word bits (nsph_sph_status) -------------------- */
#define NSPH_STATUS_NONFINITE_INPUT   1u  /* a position was NaN/Inf at the build     */
#define NSPH_STATUS_NONFINITE_OUTPUT  2u  /* a new position/velocity was NaN/Inf     */
#define NSPH_STATUS_ZERO_DENSITY      4u  /* an active particle had density <= 0     */
#define NSPH_STATUS_SURROGATE_TIMEOUT 8u  /* a tensor-core completion wait gave up   */

/* Particle flag bit, newton/_src/geometry/flags.py:8-14 (ParticleFlags.ACTIVE). */
#define NSPH_PARTICLE_ACTIVE 1

NSPH_API int         nsph_version(void);
NSPH_API const char* nsph_status_string(int status);
/* Message of the last failed call on this host thread ("" if none). */
NSPH_API const char* nsph_last_error(void);

/* Build flags of this library: NSPH_BUILD_BOUNDS_CHECK when it was compiled
 * with -DNSPH_BOUNDS_CHECK (python -m newton_sph_dev_b200._build
 * --bounds-check, into libnsph_bounds.so). In that build every gather and
 * scatter of the grid, neighbour and build kernels checks its index; a
 * violation is counted and the access redirected or skipped, so the check
 * never faults. */
#define NSPH_BUILD_BOUNDS_CHECK 1
NSPH_API int nsph_build_flags(void);
/* Bounds-check violations counted on the current device since the last
 * call (the counters are reset); always 0 in the release build. */
NSPH_API int nsph_debug_bounds_violations(unsigned long long* count);

/* ======================================================================== *
 *  HashGrid — replaces wp.HashGrid(dim_x, dim_y, dim_z)                    *
 *  (builder.py:9853; reserve solver_xpbd.py:139; build solver_xpbd.py:319) *
 *                                                                          *
 *  Semantics (Warp's public HashGrid behaviour):                           *
 *   cell_width = radius, inv = 1.0f / radius (fp32)                        *
 *   virtual cell c_a = int(p_a * inv)  (truncation toward zero, saturating,*
 *                                      NaN -> 0)                           *
 *   physical  k_a = max(c_a + 2^20, 0) % dim_a                             *
 *   cell id   = k_z*dim_x*dim_y + k_y*dim_x + k_x                          *
 *   points are stably sorted by cell id; cell_starts/cell_ends hold the    *
 *   [start,end) range of each cell in sorted order, 0/0 for empty cells.   *
 * ======================================================================== */
typedef struct nsph_grid nsph_grid;

/* HashGrid(dim_x, dim_y, dim_z) on CUDA device `device`. dim_x*dim_y*dim_z
 * must be <= 2^28. */
NSPH_API int nsph_grid_create(int dim_x, int dim_y, int dim_z, int device, nsph_grid** out);
NSPH_API int nsph_grid_destroy(nsph_grid* grid);
/* HashGrid.reserve(num_points): size the point buffers (allocates). */
NSPH_API int nsph_grid_reserve(nsph_grid* grid, int num_points);
/* HashGrid.build(points, radius). points: device, num_points x 3 float32
 * (AoS vec3). Requires num_points <= reserved capacity (no allocation). */
NSPH_API int nsph_grid_build(nsph_grid* grid, const float* points, int num_points, float radius, void* stream);

/* Device pointers of the last build: sorted cell ids (num_points), sorted
 * point ids (num_points; hash_grid_point_id(grid, tid) == point_ids[tid]),
 * and the cell table: the start and end of cell c are
 * cell_starts[c * cell_stride] and cell_ends[c * cell_stride]
 * (dim_x*dim_y*dim_z cells; the two live interleaved in one table). */
typedef struct nsph_grid_view {
    const int* point_cells;
    const int* point_ids;
    const int* cell_starts;
    const int* cell_ends;
    int   cell_stride;
    int   num_points;
    int   dim_x, dim_y, dim_z;
    float cell_width;
    float cell_width_inv;
    int   built;
} nsph_grid_view;
NSPH_API int nsph_grid_get_view(const nsph_grid* grid, nsph_grid_view* view);
/* Number of kernels the last nsph_grid_build launched. */
NSPH_API int nsph_grid_last_launches(const nsph_grid* grid);

/* Batched hash_grid_query(grid, pos, radius) + hash_grid_query_next:
 * enumerate, for each of num_queries positions (device, num_queries x 3
 * float32), the candidate point ids in Warp's iteration order (cells x
 * fastest, then y, then z; within a cell in sorted order; no distance test).
 * Two calls: with out_ids == NULL it writes counts[q]; with out_ids != NULL
 * it writes the candidates of query q at out_ids[offsets[q] ...]. */
NSPH_API int nsph_grid_query(const nsph_grid* grid, const float* queries, int num_queries, float radius,
                    int* counts, const long long* offsets, int* out_ids, void* stream);

/* Allocation-free HashGrid build. No counterpart in the reference: it exists
 * for callers that must not allocate device memory, such as code that
 * rebuilds the grid while a CUDA stream is being captured (cudaMalloc is not
 * allowed during a global-mode capture) or a host program whose device
 * memory belongs to another allocator (a caching allocator or a fixed arena
 * that a library-side cudaMalloc would compete with).
 *
 * Same semantics as nsph_grid_create + nsph_grid_build(points, radius), but
 * no grid object: the caller passes every output (device memory):
 *   point_cells, point_ids: num_points ints (sorted cell ids / original ids)
 *   cell_starts, cell_ends: dim_x*dim_y*dim_z ints each (cleared by the call,
 *                           then the [start,end) of every occupied cell)
 * The sort scratch is a fixed device array of the library (4.5 MiB, held
 * by every GPU that loads the library until the process exits), so
 * num_points may not exceed NSPH_NOALLOC_MAX_POINTS (NSPH_ERR_CAPACITY).
 * All calls share that scratch: calls that overlap on the GPU (concurrent
 * streams, other host threads) race and must be serialised by the caller.
 * The first call on a device (of any size, num_points == 0 included) looks
 * up the scratch's device address and loads every kernel a build launches
 * (runtime calls, once per device); make that first call before any stream
 * capture. The call calls neither cudaMalloc nor cudaFree. */
#define NSPH_NOALLOC_MAX_POINTS (1 << 18)
NSPH_API int nsph_grid_build_noalloc(const float* points, int num_points, float radius, int dim_x, int dim_y,
                                     int dim_z, int* point_cells, int* point_ids, int* cell_starts, int* cell_ends,
                                     void* stream);

/* ======================================================================== *
 *  integrate_particles — replaces newton/_src/solvers/solver.py:10-47      *
 *  v1 = v0 + (f*w + g[max(world,0)]*(w>0))*dt; |v1| clamped to v_max;     *
 *  x1 = x0 + v1*dt; inactive particles: x1 = x0 and v_new not written.     *
 *  x, v, f, x_new, v_new: device num x 3 float32; inv_mass: float32[n];    *
 *  flags, world: int32[n]; gravity: device world_count x 3 float32.        *
 * ======================================================================== */
NSPH_API int nsph_integrate_particles(const float* x, const float* v, const float* f, const float* inv_mass,
                             const int* flags, const int* world, const float* gravity, int world_count,
                             int num, float dt, float v_max, float* x_new, float* v_new, void* stream);

/* ======================================================================== *
 *  WCSPH solver — the SolverSPH.step hot path                             *
 * ======================================================================== */

/* Scalar parameters of one step, precomputed on the host in fp32 so that the
 * device and the fp32 oracle use bit-identical constants. */
typedef struct nsph_sph_params {
    float h;           /* kernel support radius (neighbour radius)          */
    float h2;          /* h*h rounded to fp32: neighbour test r2 < h2       */
    float inv_h;       /* 1/h                                               */
    float cell_width;  /* grid cell width (== h by default)                 */
    float cell_inv;    /* 1.0f / cell_width (fp32)                          */
    float sigma;       /* 8/(pi h^3): 3-D cubic-spline normalisation        */
    float dsigma;      /* sigma/h: factor of dW/dr                          */
    float c_near;      /* 6 sigma/h^2: (dW/dr)/r = c_near (3q-2), q <= 1/2  */
    float c_far;       /* -6 sigma/h:  (dW/dr)/r = c_far (1-q)^2 / r, q > 1/2 */
    float rho0;        /* rest density                                       */
    float inv_rho0;
    float eos_b;       /* Tait stiffness B = rho0 c0^2 / gamma              */
    int   eos_gamma;   /* Tait exponent (integer, 7)                        */
    int   clamp_pressure; /* 1: p = max(p, 0)                               */
    float xsph_eps;    /* XSPH velocity-smoothing coefficient               */
    float v_max;       /* Model.particle_max_velocity                        */
    float dt;
    int   use_box;     /* 1: clamp positions to [box_lo, box_hi]            */
    float box_lo[3];
    float box_hi[3];
} nsph_sph_params;

typedef struct nsph_sph nsph_sph;

/* Create a solver context on `device` for up to `capacity` particles, with
 * a neighbour grid of grid_dims[0..2] cells (HashGrid semantics above).
 * Allocates all scratch (sort buffers, cell tables, sorted mirrors). */
NSPH_API int nsph_sph_create(int device, int capacity, const int grid_dims[3], nsph_sph** out);
NSPH_API int nsph_sph_destroy(nsph_sph* solver);

/* One WCSPH step, state_in -> state_out (SolverBase.step, solver.py:301-316).
 *   x_in, v_in:   device n x 3 float32 (State.particle_q / particle_qd)
 *   f_ext:        device n x 3 float32 external forces (State.particle_f) or NULL
 *   mass, inv_mass: device float32[n]; flags, world: device int32[n]
 *   gravity:      device world_count x 3 float32 (Model.gravity), read on the device
 *   x_out, v_out: device n x 3 float32 (must not alias x_in / v_in)
 *   rho_out, p_out: device float32[n] or NULL (density / pressure of the step)
 *   a_out:        device n x 3 float32 or NULL (SPH acceleration, no gravity)
 * Kernels (stream-ordered, no allocation, no host sync):
 *   grid build (hash + LSD radix sort + cell ranges + sorted gather),
 *   density/EOS pass, force/XSPH/integrate pass. */
NSPH_API int nsph_sph_step(nsph_sph* solver, const nsph_sph_params* params, int n,
                  const float* x_in, const float* v_in, const float* f_ext,
                  const float* mass, const float* inv_mass, const int* flags, const int* world,
                  const float* gravity, int world_count,
                  float* x_out, float* v_out, float* rho_out, float* p_out, float* a_out,
                  void* stream);

/* ---- batched worlds ------------------------------------------------------
 * Many independent scenes (Newton worlds: ModelBuilder.begin_world /
 * add_world, builder.py:2815-2909, with Model.particle_world) in one solver.
 * Each world has its own grid (dims world_dims[3w..3w+2], HashGrid semantics,
 * cell width from its parameters) and its own parameters; a particle's
 * neighbours are the particles of its own world only (world -1 counts as
 * world 0). Sort keys are (world cell offset + cell), so one build, one
 * density launch and one force launch cover every world.
 *
 * nsph_sph_create_worlds: allocates for `capacity` particles and the sum of
 *   the worlds' cells.
 * nsph_sph_set_world_params: copies world_count parameter blocks to the
 *   device (synchronous; call before the first step and after changes; their
 *   dt fields are ignored).
 * nsph_sph_step_worlds: nsph_sph_step for all worlds with time step dt;
 *   gravity has one row per world. */
NSPH_API int nsph_sph_create_worlds(int device, int capacity, int world_count, const int* world_dims,
                                    nsph_sph** out);
NSPH_API int nsph_sph_set_world_params(nsph_sph* solver, const nsph_sph_params* params, int world_count);
NSPH_API int nsph_sph_step_worlds(nsph_sph* solver, float dt, int n,
                                  const float* x_in, const float* v_in, const float* f_ext,
                                  const float* mass, const float* inv_mass, const int* flags, const int* world,
                                  const float* gravity, int world_count,
                                  float* x_out, float* v_out, float* rho_out, float* p_out, float* a_out,
                                  void* stream);

/* ---- adjoint (reverse mode) of nsph_sph_step ------------------------------
 * Replaces the reference's wp.Tape gradient of a solver step
 * (newton/solvers.py:359-395; examples/diffsim/example_diffsim_ball.py:
 * 115-151): the vector-Jacobian product of one step, written by hand.
 *
 * nsph_sph_enable_adjoint: allocates the adjoint scratch (36 bytes per
 *   particle of capacity); call once, outside graph capture. Single-world
 *   solvers only.
 * nsph_sph_step_adjoint: same model/state inputs as the nsph_sph_step it
 *   reverses (x_in, v_in, f_ext, mass, ... of that step; it recomputes the
 *   step's grid, density and forces from them, bit for bit). Given
 *     x_out_adj, v_out_adj: adjoints of x_out, v_out (n x 3)
 *     rho_out_adj:          adjoint of the step's density (float[n]) or NULL
 *   it writes
 *     x_in_adj, v_in_adj:   adjoints of x_in, v_in (n x 3, overwritten; may
 *                           be the same memory as x_out_adj / v_out_adj
 *                           respectively, which a reverse loop uses)
 *   and accumulates (+=), so a reverse loop sums them over steps,
 *     f_ext_adj:            adjoint of f_ext (n x 3) or NULL
 *     eos_b_adj:            adjoint of params->eos_b (one float) or NULL.
 * The neighbour set is held fixed (W and dW/dr vanish at r = h, so the step
 * is C1 across its changes); the pressure clamp, |v| clamp and box are
 * differentiated on the side the forward step took. Inactive particles
 * pass their adjoints through (their velocity output is taken as a copy of
 * the input). Deterministic: no atomics; adj(B) is reduced in a fixed order
 * for a fixed launch shape. The call overwrites the solver's grid and
 * neighbour scratch (as a step on x_in would). Kernels: grid build, density,
 * force recompute + integrate reverse, pair gather, density gather, and the
 * adj(B) reduction when eos_b_adj is given. */
NSPH_API int nsph_sph_enable_adjoint(nsph_sph* solver);
NSPH_API int nsph_sph_step_adjoint(nsph_sph* solver, const nsph_sph_params* params, int n,
                                   const float* x_in, const float* v_in, const float* f_ext,
                                   const float* mass, const float* inv_mass, const int* flags, const int* world,
                                   const float* gravity, int world_count,
                                   const float* x_out_adj, const float* v_out_adj, const float* rho_out_adj,
                                   float* x_in_adj, float* v_in_adj, float* f_ext_adj, float* eos_b_adj,
                                   void* stream);

/* Multi-step forms used by checkpointed rollouts (one call per segment, the
 * step loop runs in the library).
 * nsph_sph_rollout: `steps` steps from (x0, v0) with constant f_ext; the
 *   state after step t goes to x_traj / v_traj + 3 n t (steps x n x 3 each;
 *   must not overlap each other or x0 / v0, but x0 may directly precede
 *   x_traj). Inactive particles keep their velocity.
 * nsph_sph_rollout_adjoint: reverse of `steps` steps whose input states are
 *   x_states / v_states + 3 n t, t = 0..steps-1 (the layout of x0 followed
 *   by the first steps-1 states of nsph_sph_rollout). x_adj / v_adj hold the
 *   adjoint of the last step's output on entry and of the first step's input
 *   on return; f_ext_adj and eos_b_adj accumulate as in
 *   nsph_sph_step_adjoint. */
NSPH_API int nsph_sph_rollout(nsph_sph* solver, const nsph_sph_params* params, int n, int steps,
                              const float* x0, const float* v0, const float* f_ext,
                              const float* mass, const float* inv_mass, const int* flags, const int* world,
                              const float* gravity, int world_count,
                              float* x_traj, float* v_traj, void* stream);
NSPH_API int nsph_sph_rollout_adjoint(nsph_sph* solver, const nsph_sph_params* params, int n, int steps,
                                      const float* x_states, const float* v_states, const float* f_ext,
                                      const float* mass, const float* inv_mass, const int* flags, const int* world,
                                      const float* gravity, int world_count,
                                      float* x_adj, float* v_adj, float* f_ext_adj, float* eos_b_adj, void* stream);

/* Segment form with a tape: one call recomputes a checkpointed segment and
 * reverses it, replacing nsph_sph_rollout (of steps - 1 steps) followed by
 * nsph_sph_rollout_adjoint, with bit-identical results.
 * nsph_sph_segment_adjoint: `steps` steps from (x0, v0). The forward keeps,
 *   per step, the grid build, density pass and force sums that the step's
 *   reverse reads (sorted mirrors, cell table, sorted ids, m/rho, p/rho^2,
 *   rho, p, neighbour lists, a and the XSPH sum), so the reverse skips the
 *   rebuild, the density pass and the force recompute. x_adj / v_adj hold the adjoint of
 *   the state after `steps` steps on entry and of (x0, v0) on return (they
 *   must not overlap each other or x0 / v0); f_ext_adj and eos_b_adj
 *   accumulate as in nsph_sph_step_adjoint. Afterwards the solver's grid
 *   describes the last step's input.
 * nsph_sph_reserve_segment: allocates the tape for segments of up to
 *   `steps` steps (344 bytes per particle of capacity plus 8 bytes per grid
 *   cell, per step, and two states); nsph_sph_segment_adjoint reserves on
 *   demand, so call this first where the call is captured in a graph. */
NSPH_API int nsph_sph_reserve_segment(nsph_sph* solver, int steps);
NSPH_API int nsph_sph_segment_adjoint(nsph_sph* solver, const nsph_sph_params* params, int n, int steps,
                                      const float* x0, const float* v0, const float* f_ext,
                                      const float* mass, const float* inv_mass, const int* flags, const int* world,
                                      const float* gravity, int world_count,
                                      float* x_adj, float* v_adj, float* f_ext_adj, float* eos_b_adj, void* stream);

/* ---- particle raycast (depth camera) on the HashGrid ----------------------
 * Replaces, for particles, SensorRaycast.update(state, include_particles=True)
 * (newton/_src/sensors/sensor_raycast.py:185-263, 272-320): the launch of
 * sensor_raycast_particles_kernel (newton/_src/geometry/raycast.py:1090-1180)
 * with ray_for_pixel (:727-775) and ray_intersect_particle_sphere
 * (:123-156), and clamp_no_hits_kernel (sensor_raycast.py:18-23).
 *
 * nsph_raycast_particles: `grid` must have been built on x (n points) with
 *   the cell width search_radius (the reference builds its
 *   HashGrid(128, 128, 128) with radius = max particle radius + 1e-6). For
 *   pixel (px, py) the ray from camera->position through the pixel centre
 *   is marched in steps of march_step, at most max_steps samples, while
 *   t <= max_distance and t <= the nearest hit so far; at each sample the
 *   candidates of the grid query (search_radius) with radius > 0 are
 *   intersected as spheres. depth (height x width, row-major) is read as the
 *   initial nearest hit (a negative value means max_distance) and receives
 *   the nearer particle hit, if any.
 *   max_steps is at most NSPH_RAYCAST_MAX_STEPS (the reference's cap on the
 *   samples of one ray, sensor_raycast.py:28).
 * nsph_raycast_clamp_no_hits: depth[i] >= max_distance becomes -1. */
#define NSPH_RAYCAST_MAX_STEPS (1 << 20)

typedef struct nsph_raycast_camera {
    float position[3];
    float direction[3]; /* unit forward */
    float up[3];        /* unit, orthogonal to direction */
    float right[3];     /* unit, direction x up */
    float fov_scale;    /* tan(vertical field of view / 2) */
    float aspect_ratio; /* width / height */
    int width, height;
    float max_distance;
} nsph_raycast_camera;

NSPH_API int nsph_raycast_particles(nsph_grid* grid, const float* x, const float* radius, int n,
                                    const nsph_raycast_camera* camera, float search_radius, float march_step,
                                    int max_steps, float* depth, void* stream);
NSPH_API int nsph_raycast_clamp_no_hits(float* depth, int count, float max_distance, void* stream);

/* ---- particle-particle contact on the HashGrid ------------------------------
 * The reference's other consumers of the grid, rebuilt on nsph_grid (same
 * query: the candidates of hash_grid_query(grid, x_i, r_i + max_radius +
 * cohesion) in Warp's order; one thread per grid point in sorted order).
 * `grid` must have been built on x (n == its point count), with a cell
 * width covering the query radius (the reference builds it with
 * 2 max_radius + cohesion, solver_xpbd.py:315-319).
 *
 * nsph_particle_contact_forces replaces eval_particle_contact
 *   (newton/_src/solvers/semi_implicit/kernels_contact.py:35-84 with
 *   particle_force :11-32, launched by eval_particle_contact_forces
 *   :559-579): for every active particle i, f_out[i] = the sum over active
 *   j != i with err = |x_i - x_j| - r_i - r_j <= cohesion of the normal
 *   force err k_contact + min(v_rel.n, 0) k_damp along -n and the Coulomb
 *   friction min(|v_t| k_friction, mu |f_n|) along -v_t/|v_t|. Inactive
 *   particles' f_out rows are not written.
 * nsph_particle_contact_deltas replaces solve_particle_particle_contacts
 *   (newton/_src/solvers/xpbd/kernels.py:225-289, launched at
 *   solver_xpbd.py:420-440): adds the XPBD position correction of every
 *   active particle to deltas[i] (one writer per particle, no atomics).
 * Every fp32 operation is rounded as written (no contraction). Both calls
 * first copy the particles into sorted mirrors owned by the grid (32 bytes
 * per point, allocated by nsph_grid_reserve), then run the contact kernel:
 * two launches, no allocation. */
typedef struct nsph_contact_params {
    float k_contact;   /* Model.particle_ke */
    float k_damp;      /* Model.particle_kd */
    float k_friction;  /* Model.particle_kf */
    float k_mu;        /* Model.particle_mu */
    float k_cohesion;  /* Model.particle_cohesion */
    float max_radius;  /* Model.particle_max_radius */
} nsph_contact_params;
NSPH_API int nsph_particle_contact_forces(const nsph_grid* grid, const nsph_contact_params* params, int n,
                                          const float* x, const float* v, const float* radius, const int* flags,
                                          float* f_out, void* stream);
NSPH_API int nsph_particle_contact_deltas(const nsph_grid* grid, int n, const float* x, const float* v,
                                          const float* inv_mass, const float* radius, const int* flags, float k_mu,
                                          float k_cohesion, float max_radius, float dt, float relaxation,
                                          float* deltas, void* stream);

/* ---- measurement helper (no counterpart in the reference) -----------------
 * The device's FP32 / instruction-issue peak, the denominator of the issue
 * roofline that bounds the neighbour passes: 64 resident warps per SM, each
 * thread running 8 independent FMA chains of `iters` x 16 FFMA (one warp
 * instruction per FFMA). Writes the FP32 rate (TFLOP/s), the warp
 * instructions issued per second over the device and the timed launch's
 * duration (ms, CUDA events on `stream` after one warm-up launch).
 * Allocates a small sink buffer and synchronises: not for use in a step. */
NSPH_API int nsph_fp32_peak(int device, int iters, float* tflops, float* warp_inst_per_s, float* ms, void* stream);

/* ---- particles against static analytic shapes; the XPBD particle update --
 * Shapes without a body (body -1: ground planes and world-fixed spheres,
 * boxes, capsules, cylinders, cones and ellipsoids), as
 * ModelBuilder.add_shape_plane / add_ground_plane / add_shape_sphere /
 * add_shape_box / add_shape_capsule / add_shape_cylinder / add_shape_cone /
 * add_shape_ellipsoid make them (newton/_src/sim/builder.py:5611-6050).
 * `type` takes the reference's GeoType values. The world transform is (pos,
 * rot) with rot an (x, y, z, w) unit quaternion; scale is (radius, -, -)
 * for a sphere, the half extents for a box, (width, length, -) for a plane
 * (0 = infinite), (radius, half_height, -) for a capsule, cylinder or cone
 * (axis local +Z; a cone's apex at +half_height) and the semi-axes for an
 * ellipsoid. ke/kd/kf/mu are the shape's material (ShapeConfig). */
#define NSPH_GEO_PLANE 1
#define NSPH_GEO_SPHERE 3
#define NSPH_GEO_CAPSULE 4
#define NSPH_GEO_ELLIPSOID 5
#define NSPH_GEO_CYLINDER 6
#define NSPH_GEO_BOX 7
#define NSPH_GEO_CONE 9
typedef struct nsph_shape {
    int   type;      /* GeoType: PLANE 1, SPHERE 3, CAPSULE 4, ELLIPSOID 5, CYLINDER 6, BOX 7, CONE 9
                        (others never make contacts) */
    int   flags;     /* ShapeFlags; COLLIDE_PARTICLES (1 << 2) enables particle contacts */
    int   world;     /* shape_world; -1 = every world */
    int   reserved;
    float pos[3];
    float rot[4];
    float scale[3];
    float ke, kd, kf, mu;
} nsph_shape;

/* Soft contacts (Contacts.soft_contact_*): device arrays owned by the
 * caller; count is one int, the others hold `max` entries (vec3 arrays
 * 3*max floats). */
typedef struct nsph_soft_contacts {
    int*   count;     /* soft_contact_count[0]: contacts found (may exceed max) */
    int*   particle;  /* soft_contact_particle */
    int*   shape;     /* soft_contact_shape */
    float* body_pos;  /* soft_contact_body_pos (shape-body frame = world for static shapes) */
    float* body_vel;  /* soft_contact_body_vel */
    float* normal;    /* soft_contact_normal (world) */
    int    max;       /* soft_contact_max */
} nsph_soft_contacts;

/* The particle side of the soft-contact material and the solver knobs. */
typedef struct nsph_soft_contact_params {
    float ke, kd, kf, mu;  /* Model.soft_contact_ke / kd / kf / mu */
    float adhesion;        /* Model.particle_adhesion (the reference's particle_ka) */
    float restitution;     /* Model.soft_contact_restitution */
    float relaxation;      /* SolverXPBD.soft_contact_relaxation */
    float dt;
} nsph_soft_contact_params;

/* Ints of scratch nsph_soft_contacts_create needs for n particles. */
NSPH_API int nsph_soft_contacts_scratch_ints(int num_particles);
/* Replaces create_soft_contacts (newton/_src/geometry/kernels.py:1001-1140,
 * launched by the collision pipeline, newton/_src/sim/collide.py:1194-1228)
 * for static shapes: a contact for every active particle p and shape s with
 * COLLIDE_PARTICLES, a compatible world and sdf(x_p) < margin + r_p, with
 * the shape-frame contact point x - n d mapped to world and the world
 * normal. The reference appends with an atomic counter; here the contacts
 * come in (particle, shape) order, so each particle's contacts are
 * consecutive (the accumulating calls below rely on it). count[0] gets the
 * number found; entries beyond max are dropped. `shapes` is a device array;
 * `world` may be NULL (all -1). At most 1024 shapes. */
NSPH_API int nsph_soft_contacts_create(const nsph_shape* shapes, int shape_count, int num_particles,
                                       const float* x, const float* radius, const int* flags, const int* world,
                                       float margin, nsph_soft_contacts* contacts, int* scratch, void* stream);
/* Replaces eval_particle_body_contact for static shapes
 * (newton/_src/solvers/semi_implicit/kernels_contact.py:143-262, launched
 * by eval_particle_body_contact_forces :644-690): for each contact with
 * c = n.(x - p) - r <= adhesion, f[particle] -= fn + (fd + ft), material
 * averaged between params and the shape. */
NSPH_API int nsph_particle_shape_contact_forces(const nsph_shape* shapes, int shape_count,
                                                const nsph_soft_contacts* contacts,
                                                const nsph_soft_contact_params* params, const float* x,
                                                const float* v, const float* radius, const int* flags, float* f,
                                                void* stream);
/* Replaces solve_particle_shape_contacts for static shapes
 * (newton/_src/solvers/xpbd/kernels.py:115-222, launched at
 * solver_xpbd.py:386-412): deltas[particle] += w * delta_total. */
NSPH_API int nsph_particle_shape_contact_deltas(const nsph_shape* shapes, int shape_count,
                                                const nsph_soft_contacts* contacts,
                                                const nsph_soft_contact_params* params, const float* x,
                                                const float* v, const float* inv_mass, const float* radius,
                                                const int* flags, float* deltas, void* stream);
/* Replaces apply_particle_shape_restitution for static shapes
 * (newton/_src/solvers/xpbd/kernels.py:34-112, launched at
 * solver_xpbd.py:686-714): v_out[particle] += n (-v_new.n + max(-e v_old.n,
 * 0)) for contacts that were approaching (v_old.n < 0); x_old / v_old are
 * the step's input state. v_new may alias v_out. */
NSPH_API int nsph_particle_shape_restitution(const nsph_soft_contacts* contacts,
                                             const nsph_soft_contact_params* params, const float* v_new,
                                             const float* x_old, const float* v_old, const float* radius,
                                             const int* flags, float* v_out, void* stream);
/* Replaces apply_particle_deltas (newton/_src/solvers/xpbd/kernels.py:
 * 777-808): for active particles x_out = x_pred + delta, v_out = (x_out -
 * x_orig)/dt clamped to |v| <= v_max; inactive particles are not written. */
NSPH_API int nsph_apply_particle_deltas(int num_particles, const float* x_orig, const float* x_pred,
                                        const int* flags, const float* deltas, float dt, float v_max, float* x_out,
                                        float* v_out, void* stream);

/* ---- learned surrogate step (no counterpart in the reference) -------------
 * A WCSPH step with a larger dt whose acceleration is corrected per particle
 * by a small MLP (16 -> 64 -> 64 -> 3, SiLU; bf16 weights and activations,
 * fp32 accumulation on the tcgen05 tensor cores) that reads 16
 * dimensionless neighbour features (density, density error, kernel-weighted
 * relative position and velocity moments, the SPH acceleration, ...; the
 * list is in csrc/sph.cu). `model` is a device buffer of
 * nsph_mlp_model_floats() floats: the fp32 weights W1[16][64], b1[64],
 * W2[64][64], b2[64], W3[64][3], b3[3] at offsets 0, 1024, 1088, 5184, 5248,
 * 5440, the feature means and inverse standard deviations at 5448 and 5464,
 * and the output means and standard deviations at 5480 and 5484. The
 * correction is acc_scale * (y * out_std + out_mean) with acc_scale = c0^2/h.
 *
 * nsph_sph_enable_surrogate: allocates the feature scratch (96 bytes per
 *   particle of capacity); once, outside graph capture.
 * nsph_sph_features: the step's grid build, density pass and feature pass
 *   on (x_in, v_in): feat_out (n x 16) and acc_out (n x 6: SPH acceleration,
 *   XSPH sum), original order, either may be NULL; rho_out optional.
 * nsph_sph_step_surrogate: one surrogate step (time step params->dt).
 *   stats: device float[4]; the step writes stats[0] = mean over active
 *   particles of max(0, rho/rho0 - 1) at x_in (the compression error),
 *   stats[1] = max(stats[1], stats[0]), stats[2] += 1 and
 *   stats[3] += stats[0], so a host that zeroes stats[1..2] reads a
 *   window's worst compression and step count with one copy. Kernels: grid
 *   build, density (neighbour lists), then one kernel that gathers each
 *   particle's force sums and features, stages them into the MLP's input
 *   tile in shared memory, runs the MLP and integrates (the features never
 *   go through HBM), then the compression reduction. If a tensor-core
 *   completion wait gives up, the remaining particles are integrated without
 *   the correction and NSPH_STATUS_SURROGATE_TIMEOUT is set.
 * nsph_sph_set_surrogate_wait_limit: polls of each tensor-core completion
 *   wait of the surrogate step (-1 = the default, about 4M polls). 0 makes
 *   every wait give up before it polls, to exercise the timeout path; the
 *   CTA then still waits, with the default limit, for the completion it
 *   left outstanding before it frees its TMEM. */
NSPH_API int nsph_sph_enable_surrogate(nsph_sph* solver);
NSPH_API int nsph_sph_features(nsph_sph* solver, const nsph_sph_params* params, int n,
                               const float* x_in, const float* v_in,
                               const float* mass, const float* inv_mass, const int* flags, const int* world,
                               const float* gravity, int world_count,
                               float* feat_out, float* acc_out, float* rho_out, void* stream);
NSPH_API int nsph_sph_set_surrogate_wait_limit(nsph_sph* solver, int polls);
NSPH_API int nsph_sph_step_surrogate(nsph_sph* solver, const nsph_sph_params* params, const float* model,
                                     float acc_scale, int n,
                                     const float* x_in, const float* v_in, const float* f_ext,
                                     const float* mass, const float* inv_mass, const int* flags, const int* world,
                                     const float* gravity, int world_count,
                                     float* x_out, float* v_out, float* rho_out, float* p_out, float* stats,
                                     void* stream);
/* Launch shape of the surrogate step's fused kernel: persistent CTAs, each
 * taking tiles of 128 particles. tiles_per_cta = 1: CTAs of 128 threads and
 * about 34 KB of shared memory; 2: CTAs of 256 threads whose two tiles share
 * one copy of the weights (about 53 KB) and run their MMA chains
 * independently; 0 = the default (2). ctas_per_sm: resident CTAs per SM, at
 * most as many as fit (6 of one tile, 3 of two on a B200); 0 = the default
 * (5 of one tile, as many as fit of two). The kernel's preferred
 * shared-memory carveout is set to what those CTAs need, so that the rest of
 * each SM's unified L1 / shared storage caches the neighbour gathers (6 CTAs
 * of one tile leave only about 28 KB of L1). The carveout is a property of
 * the kernel, so it applies to every solver of the process. Results do not
 * depend on the launch shape. nsph_sph_enable_surrogate applies the default;
 * call this after it. */
NSPH_API int nsph_sph_set_surrogate_launch(nsph_sph* solver, int ctas_per_sm, int tiles_per_cta);

/* The MLP on its own (training and checks).
 * nsph_mlp_model_floats: size of the model buffer in floats.
 * nsph_mlp_forward: out (n x 3) = de-normalised MLP outputs of features
 *   (n x 16, raw) on device `device`; err (device uint) gets bit 0 if a
 *   tensor-core wait gave up.
 * nsph_mlp_gradient: gradient of the mean squared error between the
 *   normalised outputs and the normalised targets (n x 3, raw) over the
 *   batch rows batch_idx[0..batch): grad (device, 5443 + 1 floats: the
 *   gradient in model order, then the loss). partials: device scratch of
 *   partial_rows x 5444 floats, partial_rows >= nsph_mlp_gradient_ctas().
 * nsph_mlp_adam: one Adam step on the 5443 trainable floats of `model`
 *   (m, v: device moment buffers of 5443 floats; step counts from 1). */
NSPH_API int nsph_mlp_model_floats(void);
NSPH_API int nsph_mlp_forward(int device, const float* model, const float* features, int n, float* out,
                              unsigned int* err, void* stream);
NSPH_API int nsph_mlp_gradient_ctas(int device, int batch);
NSPH_API int nsph_mlp_gradient(int device, const float* model, const float* features, const float* targets,
                               const int* batch_idx, int batch, float* partials, int partial_rows, float* grad,
                               unsigned int* err, void* stream);
NSPH_API int nsph_mlp_adam(int device, float* model, const float* grad, float* m, float* v, float lr, float beta1,
                           float beta2, float eps, int step, void* stream);

/* Neighbour lists of the last step's build, in original particle order: for
 * each particle i the ids j (self included) of active particles visited by
 * hash_grid_query(x_i, h) with fp32 r2 = fma(dz,dz,fma(dy,dy,dx*dx)) < h2,
 * in Warp's iteration order. Inactive particles have none. Two calls as in
 * nsph_grid_query (counts first, then ids at offsets). */
NSPH_API int nsph_sph_neighbors(const nsph_sph* solver, const nsph_sph_params* params,
                       int* counts, const long long* offsets, int* out_ids, void* stream);

/* The solver's grid of the last step (sorted cell ids, permutation, ranges). */
NSPH_API int nsph_sph_get_grid_view(const nsph_sph* solver, nsph_grid_view* view);

/* Phase timing. When enabled, every later step records four CUDA events on
 * its stream (start, after the grid build and sorted gather, after the
 * density pass, end) with cudaEventRecordExternal, so they also become event
 * record nodes of a captured CUDA graph. nsph_sph_phase_times waits for the
 * end event of the last executed step (eager or replayed) and returns its
 * build / density / force durations in ms. Enable/disable outside capture. */
NSPH_API int nsph_sph_enable_phase_timing(nsph_sph* solver, int enable);
NSPH_API int nsph_sph_phase_times(nsph_sph* solver, float ms_out[3]);
/* With phase timing enabled, every adjoint step also records six events:
 * start, after the grid build, after the density pass, after the force
 * recompute + integrate reverse, after the pair gather, end (density gather
 * and adj(B) reduction). Returns the five durations of the last executed
 * adjoint step in ms. */
NSPH_API int nsph_sph_adjoint_phase_times(nsph_sph* solver, float ms_out[5]);
/* With phase timing enabled, every surrogate step records five events:
 * start, after the grid build, after the density pass, after the fused
 * feature + MLP + integrate kernel, end (compression reduction). Returns the
 * four durations of the last executed surrogate step in ms. */
NSPH_API int nsph_sph_surrogate_phase_times(nsph_sph* solver, float ms_out[4]);

/* Arithmetic of the plain single-world step's density and force passes.
 * NSPH_ARITH_EXACT (the default): every fp32 operation correctly rounded in
 * the fp32 oracle's order, so results are bit-exact with it.
 * NSPH_ARITH_FAST: the kernel terms use the hardware reciprocal square root
 * in place of the correctly rounded square root, reciprocal and division,
 * and multiply-adds may contract; the neighbour test, and so the neighbour
 * sets, are unchanged and sums keep the query order. Results then agree with
 * the fp64 oracle to the same tolerances as the exact mode, not bit for bit
 * with the fp32 oracle. Other steps (worlds, adjoint, surrogate) always use
 * the exact arithmetic. */
#define NSPH_ARITH_EXACT 0
#define NSPH_ARITH_FAST 1
NSPH_API int nsph_sph_set_arithmetic(nsph_sph* solver, int mode);

/* Launch shape of the two neighbour passes (density, force): `threads` per
 * block (0 = default 256; else a multiple of 32 up to 256) and
 * `blocks_per_sm` (-1 = default: one thread per particle for a single world,
 * a persistent grid for batched worlds; 0 = one thread per particle; k > 0 =
 * a persistent grid of k blocks per SM striding over the particles). Results
 * do not depend on the shape; SolverSPH.autotune picks the fastest. */
NSPH_API int nsph_sph_set_launch(nsph_sph* solver, int threads, int blocks_per_sm);

/* Number of kernels the last nsph_sph_step launched. */
NSPH_API int nsph_sph_last_launches(const nsph_sph* solver);

/* Device-side status word (NSPH_STATUS_* bits), OR-accumulated by the step
 * kernels. Reading copies 4 bytes to the host and synchronises the stream;
 * reset clears it (stream-ordered). */
NSPH_API int nsph_sph_status(nsph_sph* solver, unsigned int* status, void* stream);
NSPH_API int nsph_sph_reset_status(nsph_sph* solver, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NSPH_H */
