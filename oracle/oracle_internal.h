/*
 * oracle_internal.h — grid tables shared by the oracle's translation units.
 * TEST INFRASTRUCTURE ONLY (the checker; see nsph_oracle.h).
 */
#ifndef NSPH_ORACLE_INTERNAL_H
#define NSPH_ORACLE_INTERNAL_H
#include "nsph_oracle.h"

typedef struct grid_tables {
    int dx, dy, dz;
    int* point_cells;
    int* point_ids;
    int* starts;
    int* ends;
} grid_tables;

int  oracle_build_tables(grid_tables* g, const nsph_sph_params* p, const int* dims, int n, const float* x);
void oracle_free_tables(grid_tables* g);
long long oracle_neighbors_of(const grid_tables* g, const nsph_sph_params* p, const float* x,
                              const int* flags, int i, int* out, long long max_out);
#endif
