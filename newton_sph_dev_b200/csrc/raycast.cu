// raycast.cu — the particle path of the raycast depth camera on the HashGrid.
//
// Replaces, for particles, SensorRaycast.update(state, include_particles=True)
// (newton/_src/sensors/sensor_raycast.py:185-263, 272-320): the launch of
// sensor_raycast_particles_kernel (newton/_src/geometry/raycast.py:1090-1180)
// with its helpers ray_for_pixel (raycast.py:727-775) and
// ray_intersect_particle_sphere (raycast.py:123-156), and the final
// clamp_no_hits_kernel (sensor_raycast.py:18-23).
//
// One thread per pixel marches its ray from the camera in steps of
// march_step. At every sample it queries the grid (Warp's query box around
// the sample, radius search_radius) and intersects the ray with the sphere
// of every candidate, keeping the nearest hit; it stops after max_steps
// samples, beyond max_distance, or beyond the nearest hit so far. The depth
// is the minimum over the candidates of the samples taken, which does not
// depend on the order they are tested in.
//
// Each cell is tested once per ray. Along every axis the sample coordinate
// is monotone in t, and so are both ends of the query box, so a cell of this
// sample's box that was in any earlier box was in the previous one. The
// cells of the box that the previous box did not hold are therefore exactly
// the cells no earlier sample tested; testing only those gives the same
// running minimum after every sample, hence the same samples and the same
// result as the reference's per-sample query, at about a sixth of the cell
// visits for a march step of half a cell.
//
// fp32, every operation rounded as written (explicit _rn intrinsics, dot
// products ((x + y) + z)), so the depth image matches the CPU restatement
// bit for bit.
#include <algorithm>

#include "nsph_internal.cuh"

namespace nsph {

NSPH_BOUNDS_READER(raycast)
namespace {

constexpr int kRayTileX = 32;  // a warp: 32 consecutive pixels of a row
constexpr int kRayTileY = 4;

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// sorted mirror (x, y, z, radius) of the grid's points
__global__ void k_raycast_gather(const int* __restrict__ ids, const float* __restrict__ x,
                                 const float* __restrict__ radius, int n, float4* __restrict__ m)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t i = (size_t)ids[k];
    m[k] = make_float4(x[3 * i], x[3 * i + 1], x[3 * i + 2], radius[i]);
}

struct Ray {
    float ox, oy, oz, dx, dy, dz;
};

// ray_for_pixel: pixel centre in normalised device coordinates (y up),
// scaled by tan(fov/2) and the aspect ratio, then right*x + up*y + forward
// normalised (the zero vector for a zero length)
__device__ __forceinline__ Ray ray_for_pixel(const nsph_raycast_camera& c, int px, int py)
{
    const float ndc_x =
        __fsub_rn(__fdiv_rn(__fadd_rn(__fmul_rn(2.f, (float)px), 1.f), (float)c.width), 1.f);
    const float ndc_y =
        __fsub_rn(1.f, __fdiv_rn(__fadd_rn(__fmul_rn(2.f, (float)py), 1.f), (float)c.height));
    const float cx = __fmul_rn(__fmul_rn(ndc_x, c.fov_scale), c.aspect_ratio);
    const float cy = __fmul_rn(ndc_y, c.fov_scale);
    float d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        d[k] = __fadd_rn(__fadd_rn(__fmul_rn(c.right[k], cx), __fmul_rn(c.up[k], cy)), c.direction[k]);
    const float l = __fsqrt_rn(dot3(d[0], d[1], d[2], d[0], d[1], d[2]));
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = l > 0.f ? __fdiv_rn(d[k], l) : 0.f;
    return Ray{c.position[0], c.position[1], c.position[2], d[0], d[1], d[2]};
}

// ray_intersect_particle_sphere: the nearer non-negative root, else -1
__device__ __forceinline__ float ray_sphere(const Ray& r, float4 s)
{
    const float ox = __fsub_rn(r.ox, s.x), oy = __fsub_rn(r.oy, s.y), oz = __fsub_rn(r.oz, s.z);
    const float proj = dot3(r.dx, r.dy, r.dz, ox, oy, oz);
    const float c = __fsub_rn(dot3(ox, oy, oz, ox, oy, oz), __fmul_rn(s.w, s.w));
    const float disc = __fsub_rn(__fmul_rn(proj, proj), c);
    if (disc < 0.f) return -1.f;
    const float sq = __fsqrt_rn(disc);
    float t = __fsub_rn(-proj, sq);
    if (t < 0.f) t = __fadd_rn(-proj, sq);
    if (t < 0.f) return -1.f;
    return t;
}

// physical coordinate of virtual cell lo + i along one axis (i < dim: the
// query box spans at most dim cells): a 32-bit modulo for the first and an
// increment that wraps once at dim for the next; the general mapping when
// the run starts below the 2^20 origin (clamped cells)
struct AxisWalk {
    int first, dim, lo;
    bool general;
    __device__ __forceinline__ int at(int i) const
    {
        if (general) return phys_axis((long long)lo + i, dim);
        const int v = first + i;  // <= 2 dim - 2
        return v < dim ? v : v - dim;
    }
};

__device__ __forceinline__ AxisWalk axis_walk(int lo, int dim)
{
    AxisWalk a;
    a.dim = dim;
    a.lo = lo;
    a.general = (long long)lo + kOrigin < 0;
    a.first = a.general ? 0 : (int)((unsigned)((long long)lo + kOrigin) % (unsigned)dim);
    return a;
}

// query box of one axis as ints (Warp's bounds fit: start >= INT_MIN, and
// end <= the truncated upper bound <= INT_MAX)
__device__ __forceinline__ void box_axis(float p, float r, float inv, int dim, int& lo, int& hi)
{
    long long a, b;
    query_bounds(p, r, inv, dim, a, b);
    lo = (int)a;
    hi = (int)b;
}

__global__ void __launch_bounds__(kRayTileX* kRayTileY) k_raycast(GridDev g, const float4* __restrict__ m,
                                                                   const nsph_raycast_camera cam, float search_radius,
                                                                   float march_step, int max_steps,
                                                                   float* __restrict__ depth)
{
    const int px = blockIdx.x * kRayTileX + threadIdx.x;
    const int py = blockIdx.y * kRayTileY + threadIdx.y;
    if (px >= cam.width || py >= cam.height) return;
    const Ray r = ray_for_pixel(cam, px, py);
    float* out = depth + (size_t)py * cam.width + px;
    float best = *out;
    if (best < 0.f) best = cam.max_distance;
    bool hit = false;
    // previous query box, empty at first (every cell then counts as new)
    int pxl = 0, pxh = -1, pyl = 0, pyh = -1, pzl = 0, pzh = -1;
    int s = 0;
    float t = 0.f;
    while (s < max_steps && t <= cam.max_distance && t <= best) {
        int xl, xh, yl, yh, zl, zh;
        box_axis(__fadd_rn(r.ox, __fmul_rn(r.dx, t)), search_radius, g.inv, g.dx, xl, xh);
        box_axis(__fadd_rn(r.oy, __fmul_rn(r.dy, t)), search_radius, g.inv, g.dy, yl, yh);
        box_axis(__fadd_rn(r.oz, __fmul_rn(r.dz, t)), search_radius, g.inv, g.dz, zl, zh);
        if (xl != pxl || xh != pxh || yl != pyl || yh != pyh || zl != pzl || zh != pzh) {
            const AxisWalk ax = axis_walk(xl, g.dx), ay = axis_walk(yl, g.dy), az = axis_walk(zl, g.dz);
            const int nx = xh - xl + 1, ny = yh - yl + 1, nz = zh - zl + 1;
            for (int iz = 0; iz < nz; ++iz) {
                const int z = zl + iz;
                const bool zin = z >= pzl && z <= pzh;
                const int cz = az.at(iz);
                for (int iy = 0; iy < ny; ++iy) {
                    const int y = yl + iy;
                    const bool yzin = zin && y >= pyl && y <= pyh;
                    const int rowbase = cz * (g.dx * g.dy) + ay.at(iy) * g.dx;
                    for (int ix = 0; ix < nx; ++ix) {
                        const int x = xl + ix;
                        if (yzin && x >= pxl && x <= pxh) continue;  // tested by an earlier sample
                        const int2 se = __ldg(g.ranges + rowbase + ax.at(ix));
                        for (int k = se.x; k < se.y; ++k) {
                            const float4 q = __ldg(m + k);
                            if (q.w <= 0.f) continue;
                            const float th = ray_sphere(r, q);
                            if (th < 0.f) continue;
                            if (th > cam.max_distance) continue;
                            if (th < best) {
                                best = th;
                                hit = true;
                            }
                        }
                    }
                }
            }
            pxl = xl;
            pxh = xh;
            pyl = yl;
            pyh = yh;
            pzl = zl;
            pzh = zh;
        }
        ++s;
        t = __fadd_rn(t, march_step);
    }
    if (hit) *out = best;
}

__global__ void k_clamp_no_hits(float* __restrict__ depth, int count, float max_distance)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count && depth[i] >= max_distance) depth[i] = -1.f;
}

}  // namespace
}  // namespace nsph

using namespace nsph;

extern "C" int nsph_raycast_particles(nsph_grid* grid, const float* x, const float* radius, int n,
                                      const nsph_raycast_camera* camera, float search_radius, float march_step,
                                      int max_steps, float* depth, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_raycast_particles");
    if (!grid || !camera) return fail(NSPH_ERR_INVALID_ARG, "null grid or camera");
    const nsph_raycast_camera& c = *camera;
    if (c.width < 0 || c.height < 0) return fail(NSPH_ERR_INVALID_ARG, "negative image size");
    if ((long long)c.width * c.height > 0x7fffffffLL) return fail(NSPH_ERR_INVALID_ARG, "image too large");
    if (n < 0) return fail(NSPH_ERR_INVALID_ARG, "negative particle count");
    if (!(march_step > 0.f)) return fail(NSPH_ERR_INVALID_ARG, "march_step must be positive");
    if (!(search_radius > 0.f) || !isfinite(search_radius))
        return fail(NSPH_ERR_INVALID_ARG, "search_radius must be positive and finite");
    if (max_steps < 0 || max_steps > NSPH_RAYCAST_MAX_STEPS)
        return fail(NSPH_ERR_INVALID_ARG, "max_steps must be in [0, NSPH_RAYCAST_MAX_STEPS]");
    if (c.width == 0 || c.height == 0 || n == 0 || max_steps == 0) return NSPH_OK;
    if (!x || !radius || !depth) return fail(NSPH_ERR_INVALID_ARG, "null array");
    Grid& g = grid->g;
    if (g.world_count > 0) return fail(NSPH_ERR_INVALID_ARG, "the raycast needs a single-world grid");
    if (!g.built || g.num_points != n)
        return fail(NSPH_ERR_NOT_BUILT, "the grid must be built on the n particle positions first");
    DeviceGuard guard(g.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    if (grid->mirror_cap < n) {
        cudaFree(grid->mirror);
        grid->mirror = nullptr;
        grid->mirror_cap = 0;
        NSPH_CUDA_TRY(cudaMalloc(&grid->mirror, sizeof(float4) * 2 * (size_t)g.capacity));
        grid->mirror_cap = g.capacity;
    }
    cudaStream_t cs = (cudaStream_t)stream;
    k_raycast_gather<<<(n + 255) / 256, 256, 0, cs>>>(g.point_ids, x, radius, n, grid->mirror);
    NSPH_LAUNCH_CHECK("k_raycast_gather");
    const dim3 block(kRayTileX, kRayTileY);
    const dim3 blocks((c.width + kRayTileX - 1) / kRayTileX, (c.height + kRayTileY - 1) / kRayTileY);
    k_raycast<<<blocks, block, 0, cs>>>(g.view(), grid->mirror, c, search_radius, march_step, max_steps, depth);
    NSPH_LAUNCH_CHECK("k_raycast");
    return NSPH_OK;
}

extern "C" int nsph_raycast_clamp_no_hits(float* depth, int count, float max_distance, void* stream)
{
    clear_error();
    if (count < 0) return fail(NSPH_ERR_INVALID_ARG, "negative count");
    if (count == 0) return NSPH_OK;
    if (!depth) return fail(NSPH_ERR_INVALID_ARG, "null depth");
    k_clamp_no_hits<<<(count + 255) / 256, 256, 0, (cudaStream_t)stream>>>(depth, count, max_distance);
    NSPH_LAUNCH_CHECK("k_clamp_no_hits");
    return NSPH_OK;
}
