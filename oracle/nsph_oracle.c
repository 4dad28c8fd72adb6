/*
 * nsph_oracle.c — fp32 HashGrid restatement and SPH neighbour lists.
 * TEST INFRASTRUCTURE ONLY (the checker; see nsph_oracle.h).
 *
 * Compile with -ffp-contract=off: every fp32 expression here must round
 * exactly like the device code it checks.
 */
#include "nsph_oracle.h"
#include "oracle_internal.h"

#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORIGIN (1LL << 20)

int oracle_trunc_sat(float v)
{
    if (v != v) return 0;
    if (v >= 2147483648.0f) return INT_MAX;
    if (v <= -2147483648.0f) return INT_MIN;
    return (int)v; /* C conversion truncates toward zero */
}

/* physical coordinate of a virtual cell along one axis */
static inline int phys_axis(long long c, int dim)
{
    long long v = c + ORIGIN;
    if (v < 0) v = 0;
    return (int)(v % dim);
}

int oracle_grid_index(int x, int y, int z, int dim_x, int dim_y, int dim_z)
{
    int cx = phys_axis(x, dim_x), cy = phys_axis(y, dim_y), cz = phys_axis(z, dim_z);
    return cz * (dim_x * dim_y) + cy * dim_x + cx;
}

static inline int point_cell(const float* p, float inv, int dx, int dy, int dz)
{
    return oracle_grid_index(oracle_trunc_sat(p[0] * inv), oracle_trunc_sat(p[1] * inv),
                             oracle_trunc_sat(p[2] * inv), dx, dy, dz);
}

/* Warp's build: keys per point, stable key/value sort, then start/end per
 * cell (memset to 0 first, so empty cells read 0/0). A counting sort in
 * index order is stable, so it yields the same permutation as a stable
 * radix sort. */
static int grid_build_inv(const float* points, int n, float inv, int dx, int dy, int dz,
                          int* point_cells, int* point_ids, int* cell_starts, int* cell_ends)
{
    const long long ncells = (long long)dx * dy * dz;
    if (n < 0 || ncells <= 0) return NSPH_ERR_INVALID_ARG;
    memset(cell_starts, 0, sizeof(int) * (size_t)ncells);
    memset(cell_ends, 0, sizeof(int) * (size_t)ncells);
    if (n == 0) return NSPH_OK;
    int* keys = (int*)malloc(sizeof(int) * (size_t)n);
    int* count = (int*)calloc((size_t)ncells + 1, sizeof(int));
    if (!keys || !count) {
        free(keys);
        free(count);
        return NSPH_ERR_OUT_OF_MEMORY;
    }
    for (int i = 0; i < n; ++i) {
        keys[i] = point_cell(points + 3 * (size_t)i, inv, dx, dy, dz);
        count[keys[i] + 1]++;
    }
    for (long long c = 0; c < ncells; ++c) count[c + 1] += count[c];
    for (int i = 0; i < n; ++i) {
        int pos = count[keys[i]]++;
        point_cells[pos] = keys[i];
        point_ids[pos] = i;
    }
    for (int k = 0; k < n; ++k) {
        int c = point_cells[k];
        if (k == 0 || point_cells[k - 1] != c) cell_starts[c] = k;
        if (k == n - 1 || point_cells[k + 1] != c) cell_ends[c] = k + 1;
    }
    free(keys);
    free(count);
    return NSPH_OK;
}

int oracle_grid_build(const float* points, int n, float radius, int dim_x, int dim_y, int dim_z,
                      int* point_cells, int* point_ids, int* cell_starts, int* cell_ends)
{
    const float inv = 1.0f / radius;
    return grid_build_inv(points, n, inv, dim_x, dim_y, dim_z, point_cells, point_ids, cell_starts,
                          cell_ends);
}

/* Query bounds per axis as Warp computes them: start = int((p - r) * inv),
 * end = min(int((p + r) * inv), start + dim - 1). The first cell is always
 * visited, so an empty range degenerates to the start cell. */
static inline void query_bounds(float p, float r, float inv, int dim, long long* s, long long* e)
{
    long long a = oracle_trunc_sat((p - r) * inv);
    long long b = oracle_trunc_sat((p + r) * inv);
    long long lim = a + dim - 1;
    if (b > lim) b = lim;
    if (b < a) b = a;
    *s = a;
    *e = b;
}

long long oracle_grid_query(const int* point_ids, const int* cell_starts, const int* cell_ends,
                            int dim_x, int dim_y, int dim_z, float cell_inv,
                            const float pos[3], float radius, int* out, long long max_out)
{
    long long xs, xe, ys, ye, zs, ze;
    query_bounds(pos[0], radius, cell_inv, dim_x, &xs, &xe);
    query_bounds(pos[1], radius, cell_inv, dim_y, &ys, &ye);
    query_bounds(pos[2], radius, cell_inv, dim_z, &zs, &ze);
    long long cnt = 0;
    for (long long z = zs; z <= ze; ++z) {
        const int cz = phys_axis(z, dim_z);
        for (long long y = ys; y <= ye; ++y) {
            const int cy = phys_axis(y, dim_y);
            for (long long x = xs; x <= xe; ++x) {
                const int c = cz * (dim_x * dim_y) + cy * dim_x + phys_axis(x, dim_x);
                for (int k = cell_starts[c]; k < cell_ends[c]; ++k) {
                    if (cnt < max_out && out) out[cnt] = point_ids[k];
                    ++cnt;
                }
            }
        }
    }
    return cnt;
}

/* The neighbour test shared with the device: r2 = fma(dz,dz,fma(dy,dy,dx*dx)) < h2 */
static inline int is_neighbor(const float* xi, const float* xj, float h2)
{
    const float dx = xi[0] - xj[0];
    const float dy = xi[1] - xj[1];
    const float dz = xi[2] - xj[2];
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    return r2 < h2;
}

static int tables_alloc(grid_tables* g, const int* dims, int n)
{
    g->dx = dims[0];
    g->dy = dims[1];
    g->dz = dims[2];
    const size_t ncells = (size_t)g->dx * g->dy * g->dz;
    g->point_cells = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    g->point_ids = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    g->starts = (int*)malloc(sizeof(int) * ncells);
    g->ends = (int*)malloc(sizeof(int) * ncells);
    if (!g->point_cells || !g->point_ids || !g->starts || !g->ends) return NSPH_ERR_OUT_OF_MEMORY;
    return NSPH_OK;
}

static void tables_free(grid_tables* g)
{
    free(g->point_cells);
    free(g->point_ids);
    free(g->starts);
    free(g->ends);
}

/* Neighbours of particle i: Warp query order, fp32 test, active filter.
 * Writes at most max_out ids to out and returns the total count. Used by the
 * SPH step (sph_impl.h) and by oracle_sph_neighbors below. */
long long oracle_neighbors_of(const grid_tables* g, const nsph_sph_params* p, const float* x,
                              const int* flags, int i, int* out, long long max_out)
{
    long long xs, xe, ys, ye, zs, ze;
    const float* xi = x + 3 * (size_t)i;
    query_bounds(xi[0], p->h, p->cell_inv, g->dx, &xs, &xe);
    query_bounds(xi[1], p->h, p->cell_inv, g->dy, &ys, &ye);
    query_bounds(xi[2], p->h, p->cell_inv, g->dz, &zs, &ze);
    long long cnt = 0;
    for (long long z = zs; z <= ze; ++z) {
        const int cz = phys_axis(z, g->dz);
        for (long long y = ys; y <= ye; ++y) {
            const int cy = phys_axis(y, g->dy);
            for (long long xx = xs; xx <= xe; ++xx) {
                const int c = cz * (g->dx * g->dy) + cy * g->dx + phys_axis(xx, g->dx);
                for (int k = g->starts[c]; k < g->ends[c]; ++k) {
                    const int j = g->point_ids[k];
                    if (!(flags[j] & NSPH_PARTICLE_ACTIVE)) continue;
                    if (!is_neighbor(xi, x + 3 * (size_t)j, p->h2)) continue;
                    if (cnt < max_out && out) out[cnt] = j;
                    ++cnt;
                }
            }
        }
    }
    return cnt;
}

int oracle_build_tables(grid_tables* g, const nsph_sph_params* p, const int* dims, int n, const float* x)
{
    int st = tables_alloc(g, dims, n);
    if (st != NSPH_OK) {
        tables_free(g);
        return st;
    }
    st = grid_build_inv(x, n, p->cell_inv, g->dx, g->dy, g->dz, g->point_cells, g->point_ids, g->starts,
                        g->ends);
    if (st != NSPH_OK) tables_free(g);
    return st;
}

void oracle_free_tables(grid_tables* g) { tables_free(g); }

int oracle_sph_neighbors(const nsph_sph_params* p, int n, const float* x, const int* flags,
                         const int* grid_dims, int* counts, const long long* offsets, int* out_ids)
{
    grid_tables g;
    int st = oracle_build_tables(&g, p, grid_dims, n, x);
    if (st != NSPH_OK) return st;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
        if (!(flags[i] & NSPH_PARTICLE_ACTIVE)) {
            counts[i] = 0;
            continue;
        }
        if (out_ids) {
            long long c = oracle_neighbors_of(&g, p, x, flags, i, out_ids + offsets[i], counts[i]);
            (void)c;
        } else {
            counts[i] = (int)oracle_neighbors_of(&g, p, x, flags, i, NULL, 0);
        }
    }
    tables_free(&g);
    return NSPH_OK;
}

void oracle_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int oracle_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
