// nsph_internal.cuh — shared device helpers and host plumbing of libnsph.so.
//
// Hash-grid semantics follow Warp's public HashGrid behaviour (the grid used by
// newton/_src/solvers/semi_implicit/kernels_contact.py:54-71 and
// newton/_src/solvers/xpbd/solver_xpbd.py:315-319): truncating cell
// coordinates, a 2^20 origin offset, modulo dims, x-fastest query order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include <nvtx3/nvToolsExt.h>

#include "nsph.h"

namespace nsph {

// ---------------------------------------------------------------------------
// error reporting (thread-local last message; no exception crosses the ABI)
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);
void clear_error();

// NVTX range over a public entry point (host side; a no-op unless a
// profiler is attached): the enqueue of a step, build or query shows as one
// named range on the timeline.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t err, const char* what);

// ---------------------------------------------------------------------------
// bounds-checked build (-DNSPH_BOUNDS_CHECK): the kernels' gathers and
// scatters check their indices; a violation is counted (one counter per
// translation unit, read by nsph_debug_bounds_violations) and the access is
// redirected to index 0 or skipped, so the check itself never faults. In the
// release build in_bounds() is the constant true and the checks compile away.
// ---------------------------------------------------------------------------
#ifdef NSPH_BOUNDS_CHECK
static __device__ unsigned long long g_bounds_violations;
#endif

__device__ __forceinline__ bool in_bounds(bool ok)
{
#ifdef NSPH_BOUNDS_CHECK
    if (!ok) atomicAdd(&g_bounds_violations, 1ull);
    return ok;
#else
    (void)ok;
    return true;
#endif
}

// defines unsigned long long nsph_bounds_read_<tag>(): this translation
// unit's violation count on the current device, reset to zero (0 in the
// release build)
#ifdef NSPH_BOUNDS_CHECK
#define NSPH_BOUNDS_READER(tag)                                                                    \
    unsigned long long nsph_bounds_read_##tag()                                                    \
    {                                                                                              \
        unsigned long long v = 0, z = 0;                                                           \
        if (cudaMemcpyFromSymbol(&v, g_bounds_violations, sizeof(v)) != cudaSuccess) v = ~0ull;    \
        cudaMemcpyToSymbol(g_bounds_violations, &z, sizeof(z));                                    \
        return v;                                                                                  \
    }
#else
#define NSPH_BOUNDS_READER(tag) \
    unsigned long long nsph_bounds_read_##tag() { return 0; }
#endif
unsigned long long nsph_bounds_read_hashgrid();
unsigned long long nsph_bounds_read_sph();
unsigned long long nsph_bounds_read_contact();
unsigned long long nsph_bounds_read_shapes();
unsigned long long nsph_bounds_read_raycast();

#define NSPH_CUDA_TRY(expr)                                   \
    do {                                                      \
        cudaError_t err__ = (expr);                           \
        if (err__ != cudaSuccess) return ::nsph::cuda_fail(err__, #expr); \
    } while (0)

#define NSPH_LAUNCH_CHECK(what)                                       \
    do {                                                              \
        cudaError_t err__ = cudaGetLastError();                       \
        if (err__ != cudaSuccess) return ::nsph::cuda_fail(err__, what); \
    } while (0)

// Makes `device` current for the lifetime of the guard and restores the
// caller's device afterwards.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int device)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        ok = (prev == device) || (cudaSetDevice(device) == cudaSuccess);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// ---------------------------------------------------------------------------
// grid arithmetic (device side)
// ---------------------------------------------------------------------------
constexpr long long kOrigin = 1LL << 20;

// float -> int like Warp's int(): truncation toward zero. cvt.rzi.s32.f32
// saturates out-of-range values and maps NaN to 0.
__device__ __forceinline__ int trunc_sat(float v) { return __float2int_rz(v); }

__device__ __forceinline__ int phys_axis(long long c, int dim)
{
    long long v = c + kOrigin;
    v = v < 0 ? 0 : v;
    return (int)(v % dim);
}

// Per-axis query bounds, Warp: start = int((p-r)*inv), end = min(int((p+r)*inv),
// start + dim - 1); the start cell is always visited. Rounded exactly as
// written (no contraction).
__device__ __forceinline__ void query_bounds(float p, float r, float inv, int dim, long long& s, long long& e)
{
    const long long a = trunc_sat(__fmul_rn(__fsub_rn(p, r), inv));
    long long b = trunc_sat(__fmul_rn(__fadd_rn(p, r), inv));
    const long long lim = a + dim - 1;
    b = b > lim ? lim : b;
    b = b < a ? a : b;
    s = a;
    e = b;
}

__device__ __forceinline__ int point_cell(float x, float y, float z, float inv, int dx, int dy, int dz)
{
    const int cx = phys_axis(trunc_sat(__fmul_rn(x, inv)), dx);
    const int cy = phys_axis(trunc_sat(__fmul_rn(y, inv)), dy);
    const int cz = phys_axis(trunc_sat(__fmul_rn(z, inv)), dz);
    return cz * (dx * dy) + cy * dx + cx;
}

// Read-only view of a built grid as the kernels see it.
struct GridDev {
    int dx, dy, dz;
    float inv;
    const int2* __restrict__ ranges;  // per cell {start, end} in sorted order, {0,0} if empty
    const int* __restrict__ ids;      // sorted position -> original index
    int n;                            // points of the build (read by the bounds-checked build only)
};

// Visit, in Warp's order, the sorted positions of the cells overlapping the
// query box of (px,py,pz) +- r, as contiguous runs [lo, hi): consecutive
// non-empty cells whose ranges abut in sorted order are merged into one run,
// so the candidate sequence is exactly Warp's while loops restart less often.
//
// Fast path (every visited virtual cell c has 0 <= c + 2^20 < 2^31, i.e. no
// clamping): the physical coordinate of the first cell per axis is computed
// once with a 32-bit modulo and the next ones by an increment that wraps at
// dim, which is what (c + 2^20) mod dim does for consecutive c. Otherwise each
// cell is mapped with the general formula.
template <class R>
__device__ __forceinline__ void for_each_run(const GridDev& g, float px, float py, float pz, float r, R&& run)
{
    long long xs, xe, ys, ye, zs, ze;
    query_bounds(px, r, g.inv, g.dx, xs, xe);
    query_bounds(py, r, g.inv, g.dy, ys, ye);
    query_bounds(pz, r, g.inv, g.dz, zs, ze);
    int lo = 0, hi = 0;
    auto visit = [&](int c) {
        if (!in_bounds(c >= 0 && c < g.dx * g.dy * g.dz)) return;
        const int2 se = __ldg(g.ranges + c);
        if (!in_bounds(se.x >= 0 && se.x <= se.y && se.y <= g.n)) return;
        if (se.y > se.x) {
            if (se.x == hi && hi > lo) {
                hi = se.y;
            } else {
                if (hi > lo) run(lo, hi);
                lo = se.x;
                hi = se.y;
            }
        }
    };
    const long long kMax = 0x7fffffffLL - kOrigin;
    const bool fast = xs >= -kOrigin && ys >= -kOrigin && zs >= -kOrigin && xe < kMax && ye < kMax && ze < kMax;
    if (fast) {
        const int nx = (int)(xe - xs) + 1, ny = (int)(ye - ys) + 1, nz = (int)(ze - zs) + 1;
        const int cx0 = (int)((unsigned)(xs + kOrigin) % (unsigned)g.dx);
        int cy0 = (int)((unsigned)(ys + kOrigin) % (unsigned)g.dy);
        int cz = (int)((unsigned)(zs + kOrigin) % (unsigned)g.dz);
        const int dxy = g.dx * g.dy;
        for (int iz = 0; iz < nz; ++iz) {
            int cy = cy0;
            for (int iy = 0; iy < ny; ++iy) {
                const int rowbase = cz * dxy + cy * g.dx;
                int cx = cx0;
                for (int ix = 0; ix < nx; ++ix) {
                    visit(rowbase + cx);
                    cx = (cx + 1 == g.dx) ? 0 : cx + 1;
                }
                cy = (cy + 1 == g.dy) ? 0 : cy + 1;
            }
            cz = (cz + 1 == g.dz) ? 0 : cz + 1;
        }
    } else {
        for (long long z = zs; z <= ze; ++z) {
            const int cz = phys_axis(z, g.dz);
            for (long long y = ys; y <= ye; ++y) {
                const int rowbase = cz * (g.dx * g.dy) + phys_axis(y, g.dy) * g.dx;
                for (long long x = xs; x <= xe; ++x) visit(rowbase + phys_axis(x, g.dx));
            }
        }
    }
    if (hi > lo) run(lo, hi);
}

// Per-candidate form of for_each_run: f(k) for every k of every run, in order.
template <class F>
__device__ __forceinline__ void for_each_candidate(const GridDev& g, float px, float py, float pz, float r, F&& f)
{
    for_each_run(g, px, py, pz, r, [&](int lo, int hi) {
        for (int k = lo; k < hi; ++k) f(k);
    });
}

// ---------------------------------------------------------------------------
// grid object (shared by the HashGrid API and the SPH solver)
// ---------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per CTA
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

// One world of the batched-worlds mode: the world's own HashGrid dims, its
// 1/cell_width, and where its cells start in the shared cell table. A
// particle's sort key is off + (its cell in the world's grid), so worlds
// occupy disjoint key ranges and never see each other's particles.
struct WorldCells {
    int dx, dy, dz;
    float inv;
    long long off;
};

struct Grid {
    int device = 0;
    int world_count = 0;             // > 0: batched-worlds mode
    WorldCells* worlds = nullptr;    // device table (world_count entries)
    int dx = 0, dy = 0, dz = 0;
    long long ncells = 0;
    int key_bits = 0;
    int capacity = 0;
    int num_points = 0;   // points of the last build
    int last_launches = 0;  // kernels launched by the last nsph_grid_build
    int built = 0;
    float cell_width = 0.f;
    float cell_inv = 0.f;
    // sort buffers (capacity each)
    int* keys_a = nullptr;
    int* vals_a = nullptr;
    int* keys_b = nullptr;
    int* vals_b = nullptr;
    int* point_cells = nullptr;  // sorted cell ids of the last build
    int* point_ids = nullptr;    // sorted original ids of the last build
    unsigned int* hist = nullptr;  // kRadix * ntiles(capacity)
    // cell table (ncells entries of {start, end})
    int2* cell_ranges = nullptr;
    // counting build (single world, at most kCountMaxCells cells): per-cell
    // counts (all zero between builds) and per-tile (8192 cells) counts
    int* cell_count = nullptr;
    int* tile_count = nullptr;

    GridDev view() const { return GridDev{dx, dy, dz, cell_inv, cell_ranges, point_ids, num_points}; }
};

// Gather performed by the last radix pass (SPH mode): writes the sorted
// mirrors xs = (x, y, z, m_eff) and vs = (vx, vy, vz, attr bits).
struct GatherArgs {
    const float* x;
    const float* v;
    const float* mass;
    const float* inv_mass;
    const int* flags;
    const int* world;
    int world_count;
    float4* xs;
    float4* vs;
};

// attr bits stored in vs.w
constexpr int kAttrActive = 1;
constexpr int kAttrDynamic = 2;
constexpr int kAttrGravShift = 2;

int grid_init(Grid& g, int dx, int dy, int dz, int device);
// Batched-worlds grid: world w has dims world_dims[3w..3w+2]; its cells start
// at the sum of the previous worlds' cell counts.
int grid_init_worlds(Grid& g, const int* world_dims, int world_count, int device);
int grid_reserve(Grid& g, int capacity);
void grid_free(Grid& g);
// Build over `points` (n x 3 AoS float). gather may be null. status may be
// null. launches (may be null) is incremented per kernel launched.
// In batched-worlds mode `world` (original order, may be null = world 0) selects
// each point's world; cell_width/cell_inv are ignored (per world).
int grid_build(Grid& g, const float* points, int n, float cell_width, float cell_inv, const GatherArgs* gather,
               unsigned int* status, cudaStream_t stream, int* launches = nullptr, const int* world = nullptr);

}  // namespace nsph

// the opaque handle of the nsph_grid_* C ABI (a HashGrid object)
struct nsph_grid {
    nsph::Grid g;
    float4* mirror = nullptr;  // contact scratch: 2 x mirror_cap sorted float4 ((x, r), (v, inv_mass))
    int mirror_cap = 0;
};
