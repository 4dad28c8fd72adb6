// hashgrid.cu — HashGrid build (hash + stable LSD radix sort + cell ranges)
// and the batched Warp-order query.
//
// Replaces wp.HashGrid (external warp-lang 1.14.0.dev20260511), constructed
// at newton/_src/sim/builder.py:9853, reserved at
// newton/_src/solvers/xpbd/solver_xpbd.py:139 and built at
// solver_xpbd.py:315-319; its device query is used at
// newton/_src/solvers/semi_implicit/kernels_contact.py:54,68,71.
//
// Build pipeline (all stream-ordered, no allocation, no host sync):
//   k_hash_hist   original order: cell id per point + digit-0 tile histograms;
//                 also clears the cell ranges the previous build wrote.
//   per 8-bit digit pass: [k_upsweep] -> k_scan_rows -> k_downsweep
//                 stable multi-split per tile of 256 x kItems keys (2048,
//                 or 512 for builds of at most kSmallBuildPoints points, so
//                 that small builds still spread over the SMs; the sorted
//                 result does not depend on the tile) (warp match_any ranks,
//                 shared-memory staging for coalesced scatter). The last pass
//                 writes point_cells / point_ids and, in SPH mode, gathers the
//                 sorted float4 mirrors of position and velocity.
//   k_ranges      cell_starts / cell_ends from the sorted cell ids.
// Single-world grids whose table holds at most kCountCellsPerPoint cells per
// point (the SPH solver's grids) build by cell counts instead (count_build:
// atomic counts, per-tile sums and a scan of the cell table that writes the
// ranges, scatter, stable rank within each cell): 5 launches instead of 10,
// the same result.
#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "nsph_internal.cuh"

namespace nsph {

NSPH_BOUNDS_READER(hashgrid)

namespace {

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// --------------------------------------------------------------------------
// k_hash_hist: keys/vals in original order + histogram of digit 0 per tile.
// Also clears the previous build's occupied cells (their first sorted entry
// resets start/end to 0), so no full memset of the cell tables is needed.
// --------------------------------------------------------------------------
template <int kItems>
__global__ void __launch_bounds__(kSortThreads) k_hash_hist(
    const float* __restrict__ points, int n, float inv, int dx, int dy, int dz, int* __restrict__ keys,
    int* __restrict__ vals, unsigned* __restrict__ hist, int ntiles, int digit_mask,
    const int* __restrict__ prev_cells, int prev_n, int2* __restrict__ ranges, unsigned* __restrict__ status,
    const int* __restrict__ world, const WorldCells* __restrict__ wcells, int world_count)
{
    __shared__ unsigned wh[kSortThreads / 32][kRadix];
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < (kSortThreads / 32) * kRadix; i += kSortThreads) (&wh[0][0])[i] = 0u;
    __syncthreads();

    const int base = blockIdx.x * (kSortThreads * kItems);
    bool bad = false;
#pragma unroll 4
    for (int it = 0; it < kItems; ++it) {
        const int idx = base + it * kSortThreads + threadIdx.x;
        if (idx < prev_n) {
            const int c = prev_cells[idx];
            if (idx == 0 || prev_cells[idx - 1] != c) ranges[c] = make_int2(0, 0);
        }
        if (idx < n) {
            const float x = points[3 * (size_t)idx + 0];
            const float y = points[3 * (size_t)idx + 1];
            const float z = points[3 * (size_t)idx + 2];
            bad |= !(isfinite(x) && isfinite(y) && isfinite(z));
            int key;
            if (wcells) {
                int w = world ? world[idx] : 0;
                w = w < 0 ? 0 : (w >= world_count ? world_count - 1 : w);
                const WorldCells c = wcells[w];
                key = (int)(c.off + point_cell(x, y, z, c.inv, c.dx, c.dy, c.dz));
            } else {
                key = point_cell(x, y, z, inv, dx, dy, dz);
            }
            keys[idx] = key;
            vals[idx] = idx;
            atomicAdd(&wh[warp][key & digit_mask], 1u);
        }
    }
    if (bad && status) atomicOr(status, (unsigned)NSPH_STATUS_NONFINITE_INPUT);
    __syncthreads();
    if (blockIdx.x < ntiles) {
        for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
            unsigned s = 0;
#pragma unroll
            for (int w = 0; w < kSortThreads / 32; ++w) s += wh[w][d];
            hist[(size_t)d * ntiles + blockIdx.x] = s;
        }
    }
}

// Histogram of one digit per tile (passes after the first).
template <int kItems>
__global__ void __launch_bounds__(kSortThreads) k_upsweep(const int* __restrict__ keys, int n, int shift,
                                                          int digit_mask, unsigned* __restrict__ hist,
                                                          int ntiles)
{
    __shared__ unsigned wh[kSortThreads / 32][kRadix];
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < (kSortThreads / 32) * kRadix; i += kSortThreads) (&wh[0][0])[i] = 0u;
    __syncthreads();
    const int base = blockIdx.x * (kSortThreads * kItems);
#pragma unroll 4
    for (int it = 0; it < kItems; ++it) {
        const int idx = base + it * kSortThreads + threadIdx.x;
        if (idx < n) atomicAdd(&wh[warp][(keys[idx] >> shift) & digit_mask], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
        unsigned s = 0;
#pragma unroll
        for (int w = 0; w < kSortThreads / 32; ++w) s += wh[w][d];
        hist[(size_t)d * ntiles + blockIdx.x] = s;
    }
}

// Row scan of the digit-major histogram table: CTA d turns hist[d][0..ntiles)
// into exclusive offsets within digit d and writes the digit's total to
// digit_tot[d]. The downsweep adds the exclusive scan of the digit totals.
constexpr int kScanThreads = 256;
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned& total, unsigned* ws)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) ws[warp] = incl;
    __syncthreads();
    unsigned base = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kScanThreads / 32; ++w) {
        const unsigned x = ws[w];
        base += (w < warp) ? x : 0u;
        tot += x;
    }
    __syncthreads();  // ws reusable after return
    total = tot;
    return base + incl - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_rows(unsigned* __restrict__ hist, int ntiles,
                                                            unsigned* __restrict__ digit_tot)
{
    __shared__ unsigned ws[kScanThreads / 32];
    unsigned* row = hist + (size_t)blockIdx.x * ntiles;
    unsigned carry = 0;
    for (int base = 0; base < ntiles; base += kScanThreads) {
        const int i = base + threadIdx.x;
        const unsigned v = i < ntiles ? row[i] : 0u;
        unsigned tot;
        const unsigned ex = block_exclusive_scan(v, tot, ws);
        if (i < ntiles) row[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) digit_tot[blockIdx.x] = carry;
}

// --------------------------------------------------------------------------
// k_downsweep: stable scatter of one digit pass.
// Warp w owns tile elements [w*32*kItems, (w+1)*32*kItems) in kItems rounds
// of 32; within a round lanes with equal digits are ranked by __match_any_sync, and a
// per-warp counter carries ranks across rounds, so the order inside a tile
// is exactly the input order per digit. Keys are staged in shared memory in
// tile-sorted order and written out in runs (coalesced).
// --------------------------------------------------------------------------
constexpr int kWarps = kSortThreads / 32;

template <int kItems>
struct DownsweepSmem {
    unsigned warp_cnt[kWarps][kRadix];
    unsigned tile_off[kRadix];
    unsigned glob_off[kRadix];
    int keys[kSortThreads * kItems];
    int vals[kSortThreads * kItems];
};

template <bool kGather, int kItems>
__global__ void __launch_bounds__(kSortThreads) k_downsweep(const int* __restrict__ keys_in,
                                                            const int* __restrict__ vals_in,
                                                            int* __restrict__ keys_out, int* __restrict__ vals_out,
                                                            int n, int shift, int digit_mask,
                                                            const unsigned* __restrict__ hist, int ntiles,
                                                            const unsigned* __restrict__ digit_tot,
                                                            GatherArgs gather)
{
    constexpr int kTile = kSortThreads * kItems;
    constexpr int kPerWarp = kTile / kWarps;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DownsweepSmem<kItems>& sm = *reinterpret_cast<DownsweepSmem<kItems>*>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kSortThreads) (&sm.warp_cnt[0][0])[i] = 0u;
    __syncthreads();

    const int tile_base = blockIdx.x * kTile;
    const int tile_n = min(kTile, n - tile_base);
    int key[kItems], val[kItems];
    unsigned rank[kItems];
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        const int local = warp * kPerWarp + r * 32 + lane;
        const bool valid = local < tile_n;
        key[r] = valid ? keys_in[tile_base + local] : 0;
        val[r] = valid ? vals_in[tile_base + local] : 0;
        const int d = valid ? ((key[r] >> shift) & digit_mask) : kRadix;  // kRadix: sentinel group
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned before = __popc(peers & lt);
        unsigned base = 0;
        if (valid) base = sm.warp_cnt[warp][d];
        __syncwarp();
        if (valid && before == 0) sm.warp_cnt[warp][d] = base + __popc(peers);
        __syncwarp();
        rank[r] = base + before;
    }
    __syncthreads();
    // per digit (thread d): exclusive prefix over warps and this tile's total
    const int d = threadIdx.x;  // kRadix == kSortThreads
    unsigned total = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const unsigned c = sm.warp_cnt[w][d];
        sm.warp_cnt[w][d] = total;
        total += c;
    }
    __shared__ unsigned ws[kWarps];
    unsigned dummy;
    // global offset of digit d from this tile: digits before d (all tiles) +
    // digit d in the tiles before this one
    const unsigned dbase = block_exclusive_scan(digit_tot[d], dummy, ws);
    sm.glob_off[d] = dbase + hist[(size_t)d * ntiles + blockIdx.x];
    // exclusive scan of this tile's digit totals
    sm.tile_off[d] = block_exclusive_scan(total, dummy, ws);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        const int local = warp * kPerWarp + r * 32 + lane;
        if (local < tile_n) {
            const int d = (key[r] >> shift) & digit_mask;
            const unsigned pos = sm.tile_off[d] + sm.warp_cnt[warp][d] + rank[r];
            sm.keys[pos] = key[r];
            sm.vals[pos] = val[r];
        }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < tile_n; p += kSortThreads) {
        const int k = sm.keys[p];
        const int v = sm.vals[p];
        const int d = (k >> shift) & digit_mask;
        const unsigned g = sm.glob_off[d] + (unsigned)p - sm.tile_off[d];
        keys_out[g] = k;
        vals_out[g] = v;
        if constexpr (kGather) {
            const size_t i = (size_t)v;
            const float x = gather.x[3 * i + 0], y = gather.x[3 * i + 1], z = gather.x[3 * i + 2];
            const float vx = gather.v[3 * i + 0], vy = gather.v[3 * i + 1], vz = gather.v[3 * i + 2];
            const int fl = gather.flags[i];
            const bool active = (fl & NSPH_PARTICLE_ACTIVE) != 0;
            const float m = gather.mass[i];
            const float w = gather.inv_mass[i];
            int gw = gather.world ? gather.world[i] : 0;
            gw = gw < 0 ? 0 : (gw >= gather.world_count ? gather.world_count - 1 : gw);
            const int attr = (active ? kAttrActive : 0) | (w > 0.f ? kAttrDynamic : 0) | (gw << kAttrGravShift);
            gather.xs[g] = make_float4(x, y, z, active ? m : 0.f);
            gather.vs[g] = make_float4(vx, vy, vz, __int_as_float(attr));
        }
    }
}

// Cell [start, end) ranges from sorted cell ids (Warp's compute_cell_offsets
// semantics; cells not written keep the {0,0} of an empty cell).
__global__ void k_ranges(const int* __restrict__ cells, int n, int2* __restrict__ ranges)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int c = cells[k];
    int* r = reinterpret_cast<int*>(ranges + c);
    if (k == 0 || cells[k - 1] != c) r[0] = k;
    if (k == n - 1 || cells[k + 1] != c) r[1] = k + 1;
}

// --------------------------------------------------------------------------
// Counting build (single-world grids whose cell table is at most a few times
// the point count): the stable (cell, index) order from cell counts instead
// of three radix passes.
//   k_cc_count        cell of each point (original order), its slot in the
//                     cell from an atomic counter (an arbitrary order within a
//                     cell); clears the ranges of the previous build's cells
//   k_cc_tile_sums    the points of each tile of kCsTile cells
//   k_cc_scan_ranges  per tile: its offset (the sum of the earlier tiles'
//                     counts), the exclusive scan of its cells' counts, the
//                     ranges of its occupied cells
//   k_cc_scatter      point -> start + slot (the arbitrary order), with its cell
//   k_cc_rank         per cell-ordered position: its point goes to start +
//                     (points of its cell with a smaller index), the stable
//                     order; writes point_cells / point_ids, gathers the
//                     sorted mirrors in SPH mode, and zeroes the cell's count
// No kernel waits on another block. The result is identical to the stable
// radix sort's.
// --------------------------------------------------------------------------
constexpr int kCcPoints = 4;     // points per thread of k_cc_count / k_cc_scatter
constexpr int kCsThreads = 256;  // k_cc_scan_ranges
constexpr int kCsPer = 32;       // cells per thread (eight int4 loads)
constexpr int kCsTile = kCsThreads * kCsPer;

__global__ void __launch_bounds__(256) k_cc_count(const float* __restrict__ points, int n, float inv, int dx, int dy,
                                                  int dz, int* __restrict__ count, int* __restrict__ cells,
                                                  int* __restrict__ slots, const int* __restrict__ prev_cells,
                                                  int prev_n, int2* __restrict__ ranges,
                                                  unsigned* __restrict__ status)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    // the previous build's cells: the first sorted entry of each clears its range
    for (int k = t; k < prev_n; k += stride) {
        const int c = prev_cells[k];
        if (k == 0 || prev_cells[k - 1] != c) ranges[c] = make_int2(0, 0);
    }
    bool bad = false;
    int c[kCcPoints];
#pragma unroll
    for (int u = 0; u < kCcPoints; ++u) {
        const int i = t + u * stride;
        c[u] = -1;
        if (i < n) {
            const float x = points[3 * (size_t)i + 0];
            const float y = points[3 * (size_t)i + 1];
            const float z = points[3 * (size_t)i + 2];
            bad |= !(isfinite(x) && isfinite(y) && isfinite(z));
            c[u] = point_cell(x, y, z, inv, dx, dy, dz);
            cells[i] = c[u];
        }
    }
#pragma unroll
    for (int u = 0; u < kCcPoints; ++u) {
        const int i = t + u * stride;
        if (i < n) slots[i] = atomicAdd(count + c[u], 1);
    }
    if (bad && status) atomicOr(status, (unsigned)NSPH_STATUS_NONFINITE_INPUT);
}

// this thread's kCsPer counts of the tile (int4 loads where the tile is whole)
__device__ __forceinline__ void cc_load_counts(const int* __restrict__ count, long long ncells, long long c0,
                                               int (&v)[kCsPer])
{
    if (c0 + kCsPer <= ncells) {  // count is 256-byte aligned and c0 a multiple of 32
        const int4* p4 = reinterpret_cast<const int4*>(count + c0);
#pragma unroll
        for (int q = 0; q < kCsPer / 4; ++q) {
            const int4 a = p4[q];
            v[4 * q + 0] = a.x;
            v[4 * q + 1] = a.y;
            v[4 * q + 2] = a.z;
            v[4 * q + 3] = a.w;
        }
    } else {
#pragma unroll
        for (int u = 0; u < kCsPer; ++u) v[u] = c0 + u < ncells ? count[c0 + u] : 0;
    }
}

__global__ void __launch_bounds__(kCsThreads) k_cc_tile_sums(const int* __restrict__ count, long long ncells,
                                                             int* __restrict__ tile_count)
{
    __shared__ int part[kCsThreads / 32];
    const long long c0 = (long long)blockIdx.x * kCsTile + (long long)threadIdx.x * kCsPer;
    int v[kCsPer];
    cc_load_counts(count, ncells, c0, v);
    int sum = 0;
#pragma unroll
    for (int u = 0; u < kCsPer; ++u) sum += v[u];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        int total = 0;
#pragma unroll
        for (int w = 0; w < kCsThreads / 32; ++w) total += part[w];
        tile_count[blockIdx.x] = total;
    }
}

__global__ void __launch_bounds__(kCsThreads) k_cc_scan_ranges(const int* __restrict__ count,
                                                               const int* __restrict__ tile_count, long long ncells,
                                                               int2* __restrict__ ranges)
{
    __shared__ int ws[kCsThreads / 32];
    __shared__ int s_base[kCsThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile = blockIdx.x;
    // the tile's offset: the counts of the tiles before it
    int before = 0;
    for (int q = threadIdx.x; q < tile; q += kCsThreads) before += tile_count[q];
    const long long c0 = (long long)tile * kCsTile + (long long)threadIdx.x * kCsPer;
    int v[kCsPer];
    cc_load_counts(count, ncells, c0, v);
    int sum = 0;
#pragma unroll
    for (int u = 0; u < kCsPer; ++u) sum += v[u];
    int inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
        before += __shfl_xor_sync(0xffffffffu, before, o);
    }
    if (lane == 31) ws[warp] = inc;
    if (lane == 0) s_base[warp] = before;
    __syncthreads();
    int base = 0, warp_off = 0;
#pragma unroll
    for (int w = 0; w < kCsThreads / 32; ++w) {
        base += s_base[w];
        warp_off += w < warp ? ws[w] : 0;
    }
    int start = base + warp_off + inc - sum;
#pragma unroll
    for (int u = 0; u < kCsPer; ++u) {
        if (v[u]) ranges[c0 + u] = make_int2(start, start + v[u]);  // empty cells keep {0, 0}
        start += v[u];
    }
}

__global__ void __launch_bounds__(256) k_cc_scatter(const int* __restrict__ cells, const int* __restrict__ slots,
                                                    const int2* __restrict__ ranges, int n, int* __restrict__ tmp,
                                                    int* __restrict__ tmp_cells)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    int c[kCcPoints], s[kCcPoints];
#pragma unroll
    for (int u = 0; u < kCcPoints; ++u) {
        const int i = t + u * stride;
        c[u] = i < n ? cells[i] : 0;
        s[u] = i < n ? slots[i] : 0;
    }
#pragma unroll
    for (int u = 0; u < kCcPoints; ++u) {
        const int i = t + u * stride;
        if (i < n) s[u] += ranges[c[u]].x;
    }
#pragma unroll
    for (int u = 0; u < kCcPoints; ++u) {
        const int i = t + u * stride;
        if (i < n && in_bounds(s[u] >= 0 && s[u] < n)) {
            tmp[s[u]] = i;
            tmp_cells[s[u]] = c[u];
        }
    }
}

// one thread per position q of the cell-ordered (not yet stable) array: its
// point i, the rank of i among its cell's points, and the stable position
// start + rank, which lies in the same cell's range, so neighbouring threads
// write neighbouring positions
__global__ void __launch_bounds__(256) k_cc_rank(const int* __restrict__ tmp_cells, const int2* __restrict__ ranges,
                                                 const int* __restrict__ tmp, int n, int* __restrict__ count,
                                                 int* __restrict__ point_cells, int* __restrict__ point_ids,
                                                 GatherArgs gather, bool do_gather)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int i = tmp[q];
    const int c = tmp_cells[q];
    if (!in_bounds(i >= 0 && i < n)) return;
    float4 xs, vs;
    if (do_gather) {  // the gathered loads go out before the rank loop
        const size_t ii = (size_t)i;
        const float x = gather.x[3 * ii + 0], y = gather.x[3 * ii + 1], z = gather.x[3 * ii + 2];
        const float vx = gather.v[3 * ii + 0], vy = gather.v[3 * ii + 1], vz = gather.v[3 * ii + 2];
        const int fl = gather.flags[ii];
        const bool active = (fl & NSPH_PARTICLE_ACTIVE) != 0;
        const float m = gather.mass[ii];
        const float w = gather.inv_mass[ii];
        int gw = gather.world ? gather.world[ii] : 0;
        gw = gw < 0 ? 0 : (gw >= gather.world_count ? gather.world_count - 1 : gw);
        const int attr = (active ? kAttrActive : 0) | (w > 0.f ? kAttrDynamic : 0) | (gw << kAttrGravShift);
        xs = make_float4(x, y, z, active ? m : 0.f);
        vs = make_float4(vx, vy, vz, __int_as_float(attr));
    }
    const int2 se = ranges[c];
    if (!in_bounds(se.x >= 0 && se.x <= q && q < se.y && se.y <= n)) return;
    int rank = 0;
    for (int t = se.x; t < se.y; ++t) rank += tmp[t] < i;
    if (rank == 0) count[c] = 0;  // the counts start at zero for the next build
    const int g = se.x + rank;
    point_cells[g] = c;
    point_ids[g] = i;
    if (do_gather) {
        gather.xs[g] = xs;
        gather.vs[g] = vs;
    }
}

// Batched Warp-order query: counts, or ids at offsets.
__global__ void k_query(GridDev g, const float* __restrict__ q, int nq, float radius, int* __restrict__ counts,
                        const long long* __restrict__ offsets, int* __restrict__ out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nq) return;
    const float px = q[3 * (size_t)t], py = q[3 * (size_t)t + 1], pz = q[3 * (size_t)t + 2];
    if (out) {
        long long o = offsets[t];
        for_each_candidate(g, px, py, pz, radius, [&](int k) { out[o++] = g.ids[k]; });
    } else {
        int c = 0;
        for_each_candidate(g, px, py, pz, radius, [&](int) { ++c; });
        counts[t] = c;
    }
}

inline int ntiles_of(int n, int items = kSortItems)
{
    const int tile = kSortThreads * items;
    return (n + tile - 1) / tile;
}

// Small builds use tiles of 512 keys (2 per thread), so that a build of 65k
// points runs 128 CTAs instead of 32.
constexpr int kSmallItems = 2;
// the counting build runs on single-world grids of at most kCountMaxCells
// cells when the table has at most kCountCellsPerPoint cells per point (its
// scan reads every cell; the radix sort's cost does not grow with the table)
constexpr long long kCountMaxCells = 1LL << 26;
constexpr int kCountCellsPerPoint = 16;
constexpr int kSmallBuildPoints = 1 << 18;
inline int items_for(int n) { return n <= kSmallBuildPoints ? kSmallItems : kSortItems; }

// per-tile histogram rows the table needs for builds of up to `capacity` points
inline int hist_tiles(int capacity)
{
    return std::max(ntiles_of(capacity, kSortItems), ntiles_of(std::min(capacity, kSmallBuildPoints), kSmallItems));
}

template <int kItems>
cudaError_t load_sort_kernels()
{
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k_hash_hist<kItems>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_upsweep<kItems>);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_downsweep<false, kItems>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(DownsweepSmem<kItems>));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_downsweep<true, kItems>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(DownsweepSmem<kItems>));
    return e;
}

}  // namespace

// --------------------------------------------------------------------------
// host side
// --------------------------------------------------------------------------
int grid_init(Grid& g, int dx, int dy, int dz, int device)
{
    if (dx <= 0 || dy <= 0 || dz <= 0) return fail(NSPH_ERR_INVALID_ARG, "grid dims must be positive");
    const long long nc = (long long)dx * dy * dz;
    if (nc > (1LL << 28)) return fail(NSPH_ERR_INVALID_ARG, "grid has more than 2^28 cells");
    g.device = device;
    g.dx = dx;
    g.dy = dy;
    g.dz = dz;
    g.ncells = nc;
    int bits = 1;
    while ((1LL << bits) < nc) ++bits;
    g.key_bits = bits;
    DeviceGuard guard(device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    NSPH_CUDA_TRY(cudaMalloc(&g.cell_ranges, sizeof(int2) * nc));
    NSPH_CUDA_TRY(cudaMemset(g.cell_ranges, 0, sizeof(int2) * nc));
    if (nc <= kCountMaxCells) {  // the counting build's per-cell counts
        NSPH_CUDA_TRY(cudaMalloc(&g.cell_count, sizeof(int) * nc));
        NSPH_CUDA_TRY(cudaMemset(g.cell_count, 0, sizeof(int) * nc));
        const size_t tiles = (size_t)((nc + kCsTile - 1) / kCsTile);
        NSPH_CUDA_TRY(cudaMalloc(&g.tile_count, sizeof(int) * tiles));
    }
    // load every kernel now, so that a later stream capture never triggers
    // lazy module loading
    cudaFuncAttributes fa;
    NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_cc_count));
    NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_cc_tile_sums));
    NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_cc_scan_ranges));
    NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_cc_scatter));
    NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_cc_rank));
    NSPH_CUDA_TRY(load_sort_kernels<kSortItems>());
    NSPH_CUDA_TRY(load_sort_kernels<kSmallItems>());
    NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_scan_rows));
    NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_ranges));
    NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_query));
    NSPH_CUDA_TRY(cudaDeviceSynchronize());
    return NSPH_OK;
}

int grid_init_worlds(Grid& g, const int* world_dims, int world_count, int device)
{
    if (world_count <= 0 || !world_dims) return fail(NSPH_ERR_INVALID_ARG, "world_count must be positive");
    std::vector<WorldCells> wc((size_t)world_count);
    long long off = 0;
    for (int w = 0; w < world_count; ++w) {
        const int dx = world_dims[3 * w], dy = world_dims[3 * w + 1], dz = world_dims[3 * w + 2];
        if (dx <= 0 || dy <= 0 || dz <= 0) return fail(NSPH_ERR_INVALID_ARG, "world grid dims must be positive");
        wc[w] = WorldCells{dx, dy, dz, 0.f, off};
        off += (long long)dx * dy * dz;
        if (off > (1LL << 30)) return fail(NSPH_ERR_INVALID_ARG, "the worlds' grids hold more than 2^30 cells");
    }
    g.device = device;
    g.dx = g.dy = g.dz = 0;
    g.ncells = off;
    int bits = 1;
    while ((1LL << bits) < off) ++bits;
    g.key_bits = bits;
    g.world_count = world_count;
    DeviceGuard guard(device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    NSPH_CUDA_TRY(cudaMalloc(&g.cell_ranges, sizeof(int2) * off));
    NSPH_CUDA_TRY(cudaMemset(g.cell_ranges, 0, sizeof(int2) * off));
    NSPH_CUDA_TRY(cudaMalloc(&g.worlds, sizeof(WorldCells) * world_count));
    NSPH_CUDA_TRY(cudaMemcpy(g.worlds, wc.data(), sizeof(WorldCells) * world_count, cudaMemcpyHostToDevice));
    cudaFuncAttributes fa;
    NSPH_CUDA_TRY(load_sort_kernels<kSortItems>());
    NSPH_CUDA_TRY(load_sort_kernels<kSmallItems>());
    NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_scan_rows));
    NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_ranges));
    NSPH_CUDA_TRY(cudaDeviceSynchronize());
    return NSPH_OK;
}

int grid_reserve(Grid& g, int capacity)
{
    if (capacity < 0) return fail(NSPH_ERR_INVALID_ARG, "negative capacity");
    if (capacity <= g.capacity) return NSPH_OK;
    DeviceGuard guard(g.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    // a grown reservation drops the previous build (the Warp contract)
    if (g.built && g.num_points > 0) {
        NSPH_CUDA_TRY(cudaDeviceSynchronize());
        NSPH_CUDA_TRY(cudaMemset(g.cell_ranges, 0, sizeof(int2) * g.ncells));
    }
    g.built = 0;
    g.num_points = 0;
    int* bufs[6] = {g.keys_a, g.vals_a, g.keys_b, g.vals_b, g.point_cells, g.point_ids};
    for (int* b : bufs) cudaFree(b);
    cudaFree(g.hist);
    g.keys_a = g.vals_a = g.keys_b = g.vals_b = g.point_cells = g.point_ids = nullptr;
    g.hist = nullptr;
    g.capacity = 0;
    const size_t sz = sizeof(int) * (size_t)capacity;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc(&g.keys_a, sz);
    if (e == cudaSuccess) e = cudaMalloc(&g.vals_a, sz);
    if (e == cudaSuccess) e = cudaMalloc(&g.keys_b, sz);
    if (e == cudaSuccess) e = cudaMalloc(&g.vals_b, sz);
    if (e == cudaSuccess) e = cudaMalloc(&g.point_cells, sz);
    if (e == cudaSuccess) e = cudaMalloc(&g.point_ids, sz);
    // per-tile digit histograms plus kRadix digit totals
    if (e == cudaSuccess)
        e = cudaMalloc(&g.hist, sizeof(unsigned) * kRadix * ((size_t)std::max(1, hist_tiles(capacity)) + 1));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(NSPH_ERR_OUT_OF_MEMORY, std::string("reserve: ") + cudaGetErrorString(e));
    }
    g.capacity = capacity;
    return NSPH_OK;
}

void grid_free(Grid& g)
{
    DeviceGuard guard(g.device);
    int* bufs[6] = {g.keys_a, g.vals_a, g.keys_b, g.vals_b, g.point_cells, g.point_ids};
    for (int* b : bufs) cudaFree(b);
    cudaFree(g.hist);
    cudaFree(g.cell_ranges);
    cudaFree(g.cell_count);
    cudaFree(g.tile_count);
    cudaFree(g.worlds);
    g = Grid();
}

namespace {

// hash, digit passes and ranges of one build with tiles of 256 x kItems keys
template <int kItems>
int build_passes(Grid& g, const float* points, int n, float cell_inv, const GatherArgs* gather, unsigned int* status,
                 cudaStream_t stream, int& nl, const int* world, int prev_n)
{
    constexpr size_t kSmem = sizeof(DownsweepSmem<kItems>);
    const int ntiles = ntiles_of(n, kItems);
    const int launch_tiles = std::max(ntiles, ntiles_of(prev_n, kItems));
    const int passes = (g.key_bits + kRadixBits - 1) / kRadixBits;
    auto mask_of = [&](int p) {
        const int bits = std::min(kRadixBits, g.key_bits - p * kRadixBits);
        return (1 << bits) - 1;
    };
    if (launch_tiles > 0) {
        k_hash_hist<kItems><<<launch_tiles, kSortThreads, 0, stream>>>(
            points, n, cell_inv, g.dx, g.dy, g.dz, g.keys_a, g.vals_a, g.hist, ntiles, mask_of(0), g.point_cells,
            prev_n, g.cell_ranges, status, world, g.worlds, g.world_count);
        NSPH_LAUNCH_CHECK("k_hash_hist");
        ++nl;
    }
    if (n > 0) {
        const int* kin = g.keys_a;
        const int* vin = g.vals_a;
        unsigned* digit_tot = g.hist + (size_t)kRadix * hist_tiles(g.capacity);
        for (int p = 0; p < passes; ++p) {
            const bool last = (p == passes - 1);
            int* kout = last ? g.point_cells : ((p & 1) ? g.keys_a : g.keys_b);
            int* vout = last ? g.point_ids : ((p & 1) ? g.vals_a : g.vals_b);
            const int shift = p * kRadixBits;
            if (p > 0) {
                k_upsweep<kItems><<<ntiles, kSortThreads, 0, stream>>>(kin, n, shift, mask_of(p), g.hist, ntiles);
                NSPH_LAUNCH_CHECK("k_upsweep");
                ++nl;
            }
            k_scan_rows<<<kRadix, kScanThreads, 0, stream>>>(g.hist, ntiles, digit_tot);
            NSPH_LAUNCH_CHECK("k_scan_rows");
            ++nl;
            GatherArgs ga{};
            if (last && gather) {
                ga = *gather;
                k_downsweep<true, kItems><<<ntiles, kSortThreads, kSmem, stream>>>(
                    kin, vin, kout, vout, n, shift, mask_of(p), g.hist, ntiles, digit_tot, ga);
            } else {
                k_downsweep<false, kItems><<<ntiles, kSortThreads, kSmem, stream>>>(
                    kin, vin, kout, vout, n, shift, mask_of(p), g.hist, ntiles, digit_tot, ga);
            }
            NSPH_LAUNCH_CHECK("k_downsweep");
            ++nl;
            kin = kout;
            vin = vout;
        }
        k_ranges<<<(n + 255) / 256, 256, 0, stream>>>(g.point_cells, n, g.cell_ranges);
        NSPH_LAUNCH_CHECK("k_ranges");
        ++nl;
    }
    return NSPH_OK;
}

// the counting build (see k_cc_count): 5 launches
int count_build(Grid& g, const float* points, int n, float cell_inv, const GatherArgs* gather, unsigned int* status,
                cudaStream_t stream, int& nl, int prev_n)
{
    const int tiles = (int)((g.ncells + kCsTile - 1) / kCsTile);
    const int per_block = 256 * kCcPoints;
    const int blocks = (n + per_block - 1) / per_block;
    k_cc_count<<<blocks, 256, 0, stream>>>(points, n, cell_inv, g.dx, g.dy, g.dz, g.cell_count, g.keys_a, g.vals_a,
                                           g.point_cells, prev_n, g.cell_ranges, status);
    NSPH_LAUNCH_CHECK("k_cc_count");
    k_cc_tile_sums<<<tiles, kCsThreads, 0, stream>>>(g.cell_count, g.ncells, g.tile_count);
    NSPH_LAUNCH_CHECK("k_cc_tile_sums");
    k_cc_scan_ranges<<<tiles, kCsThreads, 0, stream>>>(g.cell_count, g.tile_count, g.ncells, g.cell_ranges);
    NSPH_LAUNCH_CHECK("k_cc_scan_ranges");
    k_cc_scatter<<<blocks, 256, 0, stream>>>(g.keys_a, g.vals_a, g.cell_ranges, n, g.keys_b, g.vals_b);
    NSPH_LAUNCH_CHECK("k_cc_scatter");
    k_cc_rank<<<(n + 255) / 256, 256, 0, stream>>>(g.vals_b, g.cell_ranges, g.keys_b, n, g.cell_count,
                                                   g.point_cells, g.point_ids, gather ? *gather : GatherArgs{},
                                                   gather != nullptr);
    NSPH_LAUNCH_CHECK("k_cc_rank");
    nl += 5;
    return NSPH_OK;
}

}  // namespace

int grid_build(Grid& g, const float* points, int n, float cell_width, float cell_inv, const GatherArgs* gather,
               unsigned int* status, cudaStream_t stream, int* launches, const int* world)
{
    int local_launches = 0;
    int& nl = launches ? *launches : local_launches;
    if (n < 0) return fail(NSPH_ERR_INVALID_ARG, "negative point count");
    if (n > g.capacity) return fail(NSPH_ERR_CAPACITY, "build: more points than reserved");
    if (n > 0 && !points) return fail(NSPH_ERR_INVALID_ARG, "build: null points");
    const int prev_n = g.built ? g.num_points : 0;
    if (g.world_count == 0 && g.cell_count && n > 0 && g.ncells <= (long long)kCountCellsPerPoint * n) {
        const int st = count_build(g, points, n, cell_inv, gather, status, stream, nl, prev_n);
        if (st != NSPH_OK) return st;
        g.num_points = n;
        g.cell_width = cell_width;
        g.cell_inv = cell_inv;
        g.built = 1;
        return NSPH_OK;
    }
    const int st = items_for(n) == kSmallItems
                       ? build_passes<kSmallItems>(g, points, n, cell_inv, gather, status, stream, nl, world, prev_n)
                       : build_passes<kSortItems>(g, points, n, cell_inv, gather, status, stream, nl, world, prev_n);
    if (st != NSPH_OK) return st;
    g.num_points = n;
    g.cell_width = cell_width;
    g.cell_inv = cell_inv;
    g.built = 1;
    return NSPH_OK;
}

}  // namespace nsph

// ==========================================================================
// C ABI: HashGrid
// ==========================================================================

using namespace nsph;

extern "C" int nsph_grid_create(int dim_x, int dim_y, int dim_z, int device, nsph_grid** out)
{
    clear_error();
    if (!out) return fail(NSPH_ERR_INVALID_ARG, "null out pointer");
    *out = nullptr;
    nsph_grid* h = new (std::nothrow) nsph_grid();
    if (!h) return fail(NSPH_ERR_OUT_OF_MEMORY, "host allocation failed");
    const int st = grid_init(h->g, dim_x, dim_y, dim_z, device);
    if (st != NSPH_OK) {
        grid_free(h->g);
        delete h;
        return st;
    }
    *out = h;
    return NSPH_OK;
}

extern "C" int nsph_grid_destroy(nsph_grid* grid)
{
    clear_error();
    if (!grid) return NSPH_OK;
    {
        DeviceGuard guard(grid->g.device);
        cudaFree(grid->mirror);
    }
    grid_free(grid->g);
    delete grid;
    return NSPH_OK;
}

extern "C" int nsph_grid_reserve(nsph_grid* grid, int num_points)
{
    clear_error();
    if (!grid) return fail(NSPH_ERR_INVALID_ARG, "null grid");
    const int st = grid_reserve(grid->g, num_points);
    if (st != NSPH_OK || grid->mirror_cap >= grid->g.capacity) return st;
    // sorted mirrors for the contact kernels (32 bytes per point)
    DeviceGuard guard(grid->g.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    cudaFree(grid->mirror);
    grid->mirror = nullptr;
    grid->mirror_cap = 0;
    const size_t c = (size_t)std::max(1, grid->g.capacity);
    if (cudaMalloc(&grid->mirror, sizeof(float4) * 2 * c) != cudaSuccess) {
        cudaGetLastError();
        grid->mirror = nullptr;
        return fail(NSPH_ERR_OUT_OF_MEMORY, "grid reserve: contact mirror allocation failed");
    }
    grid->mirror_cap = grid->g.capacity;
    return NSPH_OK;
}

extern "C" int nsph_grid_build(nsph_grid* grid, const float* points, int num_points, float radius, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_grid_build");
    if (!grid) return fail(NSPH_ERR_INVALID_ARG, "null grid");
    if (!(radius > 0.f) || !isfinite(radius)) return fail(NSPH_ERR_INVALID_ARG, "radius must be positive and finite");
    DeviceGuard guard(grid->g.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    const float inv = 1.0f / radius;
    int launches = 0;
    const int st = grid_build(grid->g, points, num_points, radius, inv, nullptr, nullptr, (cudaStream_t)stream,
                              &launches);
    grid->g.last_launches = launches;
    return st;
}

extern "C" int nsph_grid_last_launches(const nsph_grid* grid) { return grid ? grid->g.last_launches : 0; }

extern "C" int nsph_grid_get_view(const nsph_grid* grid, nsph_grid_view* view)
{
    clear_error();
    if (!grid || !view) return fail(NSPH_ERR_INVALID_ARG, "null argument");
    const Grid& g = grid->g;
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

extern "C" int nsph_grid_query(const nsph_grid* grid, const float* queries, int num_queries, float radius,
                               int* counts, const long long* offsets, int* out_ids, void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_grid_query");
    if (!grid) return fail(NSPH_ERR_INVALID_ARG, "null grid");
    if (!grid->g.built) return fail(NSPH_ERR_NOT_BUILT, "query before build");
    if (num_queries < 0) return fail(NSPH_ERR_INVALID_ARG, "negative query count");
    if (num_queries == 0) return NSPH_OK;
    if (!queries) return fail(NSPH_ERR_INVALID_ARG, "null queries");
    if (out_ids ? !offsets : !counts) return fail(NSPH_ERR_INVALID_ARG, "counts (count call) or offsets (fill call) required");
    DeviceGuard guard(grid->g.device);
    if (!guard.ok) return fail(NSPH_ERR_CUDA, "cannot select CUDA device");
    k_query<<<(num_queries + 127) / 128, 128, 0, (cudaStream_t)stream>>>(grid->g.view(), queries, num_queries,
                                                                         radius, counts, offsets, out_ids);
    NSPH_LAUNCH_CHECK("k_query");
    return NSPH_OK;
}

// ==========================================================================
// C ABI: allocation-free HashGrid build
//
// For callers that must not allocate device memory: code that rebuilds the
// grid while a CUDA stream is being captured (cudaMalloc is not allowed
// during a global-mode capture), and host programs whose device memory is
// owned by another allocator (a framework's caching allocator or a fixed
// arena, where a library-side cudaMalloc would compete for memory and
// synchronise the device). The caller passes the points and every output;
// the sort scratch lives in the fixed device array below.
// ==========================================================================
namespace nsph {
namespace {

// Every accepted size is a small build, so the sort uses the small builds'
// 512-key tiles, like nsph_grid_build does for the same point count.
static_assert(NSPH_NOALLOC_MAX_POINTS <= kSmallBuildPoints, "allocation-free builds are small builds");
constexpr int kNoAllocItems = kSmallItems;
constexpr int kNoAllocTiles = (NSPH_NOALLOC_MAX_POINTS + kSortThreads * kNoAllocItems - 1) /
                              (kSortThreads * kNoAllocItems);
// keys_a, vals_a, keys_b, vals_b (NSPH_NOALLOC_MAX_POINTS ints each), then
// the per-tile digit histograms and the kRadix digit totals
constexpr size_t kNoAllocSortInts = 4 * (size_t)NSPH_NOALLOC_MAX_POINTS;
constexpr size_t kNoAllocHistUints = (size_t)kRadix * (kNoAllocTiles + 1);
constexpr size_t kNoAllocBytes = sizeof(int) * kNoAllocSortInts + sizeof(unsigned) * kNoAllocHistUints;

// Held by every GPU that loads the library until the process exits. Shared by
// all calls: the last call's contents stay behind, and calls that overlap on
// the GPU race on it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// start / end of each cell into two caller arrays (Warp's layout)
__global__ void k_ranges_split(const int* __restrict__ cells, int n, int* __restrict__ starts, int* __restrict__ ends)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int c = cells[k];
    if (k == 0 || cells[k - 1] != c) starts[c] = k;
    if (k == n - 1 || cells[k + 1] != c) ends[c] = k + 1;
}

constexpr int kNoAllocMaxDevices = 64;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};  // device address per device
std::mutex g_noalloc_mutex;

// Device address of g_noalloc_scratch on the current device (looked up once
// per device with that device current; in host code the symbol itself is only
// a host-side stand-in and must never be handed to a kernel).
int noalloc_scratch(int device, unsigned char** out)
{
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(NSPH_ERR_INVALID_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void* ptr = nullptr;
        NSPH_CUDA_TRY(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        // load every kernel a build may launch now, so that no later call
        // (whatever its size, even the first one inside a stream capture)
        // triggers lazy module loading
        cudaFuncAttributes fa;
        NSPH_CUDA_TRY(load_sort_kernels<kNoAllocItems>());
        NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_scan_rows));
        NSPH_CUDA_TRY(cudaFuncGetAttributes(&fa, k_ranges_split));
        g_noalloc_ptr[device] = static_cast<unsigned char*>(ptr);
    }
    *out = g_noalloc_ptr[device];
    return NSPH_OK;
}

}  // namespace
}  // namespace nsph

extern "C" int nsph_grid_build_noalloc(const float* points, int num_points, float radius, int dim_x, int dim_y,
                                       int dim_z, int* point_cells, int* point_ids, int* cell_starts, int* cell_ends,
                                       void* stream)
{
    clear_error();
    NvtxRange nvtx_range("nsph_grid_build_noalloc");
    if (num_points < 0) return fail(NSPH_ERR_INVALID_ARG, "negative point count");
    if (num_points > NSPH_NOALLOC_MAX_POINTS)
        return fail(NSPH_ERR_CAPACITY, "nsph_grid_build_noalloc: more than NSPH_NOALLOC_MAX_POINTS (" +
                                           std::to_string(NSPH_NOALLOC_MAX_POINTS) + ") points");
    if (dim_x <= 0 || dim_y <= 0 || dim_z <= 0) return fail(NSPH_ERR_INVALID_ARG, "grid dims must be positive");
    const long long ncells = (long long)dim_x * dim_y * dim_z;
    if (ncells > (1LL << 28)) return fail(NSPH_ERR_INVALID_ARG, "grid has more than 2^28 cells");
    if (!(radius > 0.f) || !isfinite(radius)) return fail(NSPH_ERR_INVALID_ARG, "radius must be positive and finite");
    if (!cell_starts || !cell_ends || (num_points > 0 && (!points || !point_cells || !point_ids)))
        return fail(NSPH_ERR_INVALID_ARG, "null pointer");
    int device = 0;
    NSPH_CUDA_TRY(cudaGetDevice(&device));
    unsigned char* scratch = nullptr;
    int st = noalloc_scratch(device, &scratch);
    if (st != NSPH_OK) return st;
    cudaStream_t cs = (cudaStream_t)stream;
    int* keys_a = reinterpret_cast<int*>(scratch);
    int* vals_a = keys_a + NSPH_NOALLOC_MAX_POINTS;
    int* keys_b = vals_a + NSPH_NOALLOC_MAX_POINTS;
    int* vals_b = keys_b + NSPH_NOALLOC_MAX_POINTS;
    unsigned* hist = reinterpret_cast<unsigned*>(vals_b + NSPH_NOALLOC_MAX_POINTS);
    unsigned* digit_tot = hist + (size_t)kRadix * kNoAllocTiles;
    // empty cells read 0/0
    NSPH_CUDA_TRY(cudaMemsetAsync(cell_starts, 0, sizeof(int) * ncells, cs));
    NSPH_CUDA_TRY(cudaMemsetAsync(cell_ends, 0, sizeof(int) * ncells, cs));
    const int n = num_points;
    if (n == 0) return NSPH_OK;
    int bits = 1;
    while ((1LL << bits) < ncells) ++bits;
    const int passes = (bits + kRadixBits - 1) / kRadixBits;
    auto mask_of = [&](int p) { return (1 << std::min(kRadixBits, bits - p * kRadixBits)) - 1; };
    const int ntiles = ntiles_of(n, kNoAllocItems);
    const float inv = 1.0f / radius;
    k_hash_hist<kNoAllocItems><<<ntiles, kSortThreads, 0, cs>>>(points, n, inv, dim_x, dim_y, dim_z, keys_a, vals_a,
                                                             hist, ntiles, mask_of(0), nullptr, 0, nullptr, nullptr,
                                                             nullptr, nullptr, 0);
    NSPH_LAUNCH_CHECK("k_hash_hist");
    const int* kin = keys_a;
    const int* vin = vals_a;
    for (int p = 0; p < passes; ++p) {
        const bool last = (p == passes - 1);
        int* kout = last ? point_cells : ((p & 1) ? keys_a : keys_b);
        int* vout = last ? point_ids : ((p & 1) ? vals_a : vals_b);
        const int shift = p * kRadixBits;
        if (p > 0) {
            k_upsweep<kNoAllocItems><<<ntiles, kSortThreads, 0, cs>>>(kin, n, shift, mask_of(p), hist, ntiles);
            NSPH_LAUNCH_CHECK("k_upsweep");
        }
        k_scan_rows<<<kRadix, kScanThreads, 0, cs>>>(hist, ntiles, digit_tot);
        NSPH_LAUNCH_CHECK("k_scan_rows");
        k_downsweep<false, kNoAllocItems><<<ntiles, kSortThreads, sizeof(DownsweepSmem<kNoAllocItems>), cs>>>(
            kin, vin, kout, vout, n, shift, mask_of(p), hist, ntiles, digit_tot, GatherArgs{});
        NSPH_LAUNCH_CHECK("k_downsweep");
        kin = kout;
        vin = vout;
    }
    k_ranges_split<<<(n + 255) / 256, 256, 0, cs>>>(point_cells, n, cell_starts, cell_ends);
    NSPH_LAUNCH_CHECK("k_ranges_split");
    return NSPH_OK;
}
