/*
 * raycast.c — the particle raycast depth camera, restated in fp32.
 * TEST INFRASTRUCTURE ONLY (the checker; see nsph_oracle.h).
 *
 * Restates, operation by operation, the particle path of
 * SensorRaycast.update(state, include_particles=True)
 * (newton/_src/sensors/sensor_raycast.py:185-263, 272-320):
 *   sensor_raycast_particles_kernel  newton/_src/geometry/raycast.py:1090-1180
 *   ray_for_pixel                    raycast.py:727-775
 *   ray_intersect_particle_sphere    raycast.py:123-156
 * as the reference writes it: at every march sample the full grid query
 * (oracle_grid_query, Warp's order) on a grid built on x with cell width
 * search_radius, every candidate intersected. fp32, every operation rounded
 * as written (dot products ((x + y) + z), -ffp-contract=off). Warp's
 * normalize returns the zero vector for a zero-length input.
 */
#include <math.h>
#include <stdlib.h>

#include "nsph_oracle.h"

static inline float dot3(const float a[3], const float b[3])
{
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

static void ray_for_pixel(const nsph_raycast_camera* c, int px, int py, float dir[3])
{
    const float ndc_x = (2.0f * (float)px + 1.0f) / (float)c->width - 1.0f;
    const float ndc_y = 1.0f - (2.0f * (float)py + 1.0f) / (float)c->height;
    const float cx = ndc_x * c->fov_scale * c->aspect_ratio;
    const float cy = ndc_y * c->fov_scale;
    for (int k = 0; k < 3; ++k) dir[k] = (c->right[k] * cx + c->up[k] * cy) + c->direction[k];
    const float l = sqrtf(dot3(dir, dir));
    for (int k = 0; k < 3; ++k) dir[k] = l > 0.0f ? dir[k] / l : 0.0f;
}

static float ray_sphere(const float o[3], const float d[3], const float ctr[3], float radius)
{
    float oc[3];
    for (int k = 0; k < 3; ++k) oc[k] = o[k] - ctr[k];
    const float proj = dot3(d, oc);
    const float c = dot3(oc, oc) - radius * radius;
    const float disc = proj * proj - c;
    if (disc < 0.0f) return -1.0f;
    const float sq = sqrtf(disc);
    float t = -proj - sq;
    if (t < 0.0f) t = -proj + sq;
    if (t < 0.0f) return -1.0f;
    return t;
}

int oracle_raycast_particles(const float* x, const float* radius, int n, const int* dims,
                             const nsph_raycast_camera* cam, float search_radius, float march_step, int max_steps,
                             float* depth)
{
    if (!dims || !cam || n < 0 || cam->width < 0 || cam->height < 0 || !(march_step > 0.0f) ||
        !(search_radius > 0.0f) || max_steps < 0)
        return NSPH_ERR_INVALID_ARG;
    if (n == 0 || cam->width == 0 || cam->height == 0 || max_steps == 0) return NSPH_OK;
    const size_t nc = (size_t)dims[0] * dims[1] * dims[2];
    int* cells = (int*)malloc(sizeof(int) * (size_t)n);
    int* ids = (int*)malloc(sizeof(int) * (size_t)n);
    int* starts = (int*)malloc(sizeof(int) * nc);
    int* ends = (int*)malloc(sizeof(int) * nc);
    int st = (cells && ids && starts && ends) ? NSPH_OK : NSPH_ERR_OUT_OF_MEMORY;
    if (st == NSPH_OK) st = oracle_grid_build(x, n, search_radius, dims[0], dims[1], dims[2], cells, ids, starts, ends);
    const float inv = 1.0f / search_radius;
    int fail = 0;
    if (st == NSPH_OK) {
#pragma omp parallel
        {
            long long cap = 1024;
            int* buf = (int*)malloc(sizeof(int) * (size_t)cap);
#pragma omp for schedule(dynamic, 16)
            for (int pix = 0; pix < cam->width * cam->height; ++pix) {
                if (!buf) continue;
                const int px = pix % cam->width, py = pix / cam->width;
                float d[3];
                ray_for_pixel(cam, px, py, d);
                const float* o = cam->position;
                float* out = depth + (size_t)py * cam->width + px;
                float best = *out;
                if (best < 0.0f) best = cam->max_distance;
                int s = 0;
                float t = 0.0f;
                while (s < max_steps && t <= cam->max_distance && t <= best) {
                    const float p[3] = {o[0] + d[0] * t, o[1] + d[1] * t, o[2] + d[2] * t};
                    long long cnt = oracle_grid_query(ids, starts, ends, dims[0], dims[1], dims[2], inv, p,
                                                      search_radius, buf, cap);
                    if (cnt > cap) {
                        free(buf);
                        cap = cnt * 2;
                        buf = (int*)malloc(sizeof(int) * (size_t)cap);
                        if (!buf) {
#pragma omp atomic write
                            fail = 1;
                            break;
                        }
                        cnt = oracle_grid_query(ids, starts, ends, dims[0], dims[1], dims[2], inv, p, search_radius,
                                                buf, cap);
                    }
                    for (long long q = 0; q < cnt; ++q) {
                        const int j = buf[q];
                        const float r = radius[j];
                        if (r <= 0.0f) continue;
                        const float th = ray_sphere(o, d, x + 3 * (size_t)j, r);
                        if (th < 0.0f) continue;
                        if (th > cam->max_distance) continue;
                        if (th < best) {
                            *out = th;
                            best = th;
                        }
                    }
                    s += 1;
                    t += march_step;
                }
            }
            free(buf);
        }
    }
    free(cells);
    free(ids);
    free(starts);
    free(ends);
    if (st != NSPH_OK) return st;
    return fail ? NSPH_ERR_OUT_OF_MEMORY : NSPH_OK;
}

void oracle_raycast_clamp_no_hits(float* depth, int count, float max_distance)
{
    for (int i = 0; i < count; ++i)
        if (depth[i] >= max_distance) depth[i] = -1.0f;
}
