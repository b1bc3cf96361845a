// sph_mc.cuh — density grid, grid normals and marching cubes on the device.
//
// Replaces integrate_dens / integrate_normal (SPH-3D-2/sph_system.cu:1842-2351)
// and the host marching cubes SPHSystem::marching_cube(_cell)
// (SPH-3D-2/sph_system.cpp:406-542), which the reference runs on the CPU
// after copying the whole grid back every step.
//
// Grid: ndens[0] x ndens[1] x ndens[2] nodes at (i * den_size), node index
// g = z*R*C + y*R + x.  Cubes are numbered in the reference's loop order
// (x outer, y, z inner): q = (x*(C-1) + y)*(L-1) + z, so the scan over cube
// triangle counts appends triangles in the reference's order.
#pragma once
#include <cstdint>
#include <vector>
#include "../../include/sph/sph.h"
#include "sph_kernels.cuh"
#include "sph_mc_tables.h"

namespace sph {

struct McBuffers {
    uint32_t nodes = 0, cubes = 0, max_tri = 0;
    float *dens = nullptr;        // [nodes]
    float4 *normal = nullptr;     // [nodes]
    uint32_t *cube_cnt = nullptr; // [cubes]
    uint32_t *cube_off = nullptr; // [cubes]
    uint32_t *num_tri = nullptr;  // [1] total triangles of the last extraction
    float *tri = nullptr;         // [6][max_tri][3]: v0 v1 v2 n0 n1 n2
};

inline int mc_alloc(McBuffers &mc, const sph_config &c, std::vector<void *> &allocs)
{
    if (c.dim != 3 || c.ndens[0] < 2 || c.ndens[1] < 2 || c.ndens[2] < 2) return SPH_OK;
    mc.nodes = c.ndens[0] * c.ndens[1] * c.ndens[2];
    mc.cubes = (c.ndens[0] - 1) * (c.ndens[1] - 1) * (c.ndens[2] - 1);
    mc.max_tri = c.max_triangles ? c.max_triangles : 3u * mc.nodes;
    auto alloc = [&](void **p, size_t bytes) {
        if (cudaMalloc(p, bytes ? bytes : 4) != cudaSuccess) return SPH_ERR_CUDA;
        cudaMemset(*p, 0, bytes ? bytes : 4);
        allocs.push_back(*p);
        return SPH_OK;
    };
    int rc = 0;
    rc |= alloc((void **)&mc.dens, sizeof(float) * mc.nodes);
    rc |= alloc((void **)&mc.normal, sizeof(float4) * mc.nodes);
    rc |= alloc((void **)&mc.cube_cnt, sizeof(uint32_t) * mc.cubes);
    rc |= alloc((void **)&mc.cube_off, sizeof(uint32_t) * mc.cubes);
    rc |= alloc((void **)&mc.num_tri, sizeof(uint32_t) * 4);
    rc |= alloc((void **)&mc.tri, sizeof(float) * 18ull * mc.max_tri);
    return rc ? SPH_ERR_CUDA : SPH_OK;
}

// Density splat at every node from the particles of the 27 cells around the
// node's cell, on the given (stale) cell ranges and positions
// (integrate_dens_kernel, SPH-3D-2/sph_system.cu:1905-2183).  Nodes on the
// lower faces stay 0 (the reference's upper-face test never fires).  The
// weight is m * poly6(R) * (R^2 - r^2)^3 with R the particle radius, or the
// kernel length when splat_with_kernel is set.
//
// One thread per pair of x-adjacent nodes (2m-1, 2m): with two nodes per cell
// edge both usually map to the same cell, so each candidate is loaded once
// for two nodes.  Each node still sums exactly its own stencil's particles in
// its own walk order (a node whose cell differs from its partner's takes the
// candidates of the joint row range that fall in its own range).
__global__ void __launch_bounds__(kThreads) k_splat(sph_config c, const uint32_t *__restrict__ off,
                                                   const float4 *__restrict__ pos, float *__restrict__ dens)
{
    const uint32_t R = c.ndens[0], Cn = c.ndens[1], L = c.ndens[2];
    const uint32_t GX = R / 2 + 1;   // groups {0}, {1, 2}, {3, 4}, ...
    const uint32_t G = GX * Cn * L;
    // per level: the squared splat radius and m * W's coefficient
    const float rad0 = c.splat_with_kernel ? c.kernel[0] : c.radius[0];
    const float rad1 = c.splat_with_kernel ? c.kernel[1] : c.radius[1];
    const float rs0 = __fmul_rn(rad0, rad0), rs1 = __fmul_rn(rad1, rad1);
    const float cf0 = __fmul_rn(c.mass[0], c.splat_with_kernel ? c.poly6[0] : c.poly6_radius[0]);
    const float cf1 = __fmul_rn(c.mass[1], c.splat_with_kernel ? c.poly6[1] : c.poly6_radius[1]);
    for (uint32_t g = grid_stride_start(); g < G; g += grid_stride()) {
        const uint32_t gx = g % GX, vy = (g / GX) % Cn, vz = g / (GX * Cn);
        const size_t row = ((size_t)vz * Cn + vy) * R;
        const uint32_t va = 2u * gx - 1u, vb = 2u * gx;   // va is not a node when gx = 0
        const bool has_b = vb < R;
        if (gx == 0 || vy == 0 || vz == 0) {
            if (gx > 0) dens[row + va] = 0.0f;
            if (has_b) dens[row + vb] = 0.0f;
            continue;
        }
        auto cell_x = [&](uint32_t vx) {
            return min((uint32_t)floorf(__fmul_rn(__fdiv_rn((float)vx, (float)R), (float)c.ncell[0])),
                       c.ncell[0] - 1);
        };
        uint3 q;
        q.x = cell_x(va);
        q.y = (uint32_t)floorf(__fmul_rn(__fdiv_rn((float)vy, (float)Cn), (float)c.ncell[1]));
        q.z = (uint32_t)floorf(__fmul_rn(__fdiv_rn((float)vz, (float)L), (float)c.ncell[2]));
        q.y = min(q.y, c.ncell[1] - 1); q.z = min(q.z, c.ncell[2] - 1);
        const uint32_t qbx = has_b ? cell_x(vb) : q.x;
        const float ny = __fmul_rn((float)vy, c.den_size), nz = __fmul_rn((float)vz, c.den_size);
        const float4 npa = make_float4(__fmul_rn((float)va, c.den_size), ny, nz, 0.f);
        const float4 npb = make_float4(__fmul_rn((float)vb, c.den_size), ny, nz, 0.f);
        float acc_a = 0.0f, acc_b = 0.0f;
        // acc += (m * W) * (rad^2 - r^2)^3 over r^2 < rad^2
        auto add = [&](float &acc, const float4 &np, const float4 &pj, bool l1) {
            float dx, dyy, dzz;
            const float r2 = r2_of<3>(pj, np, dx, dyy, dzz);
            const float rad2 = l1 ? rs0 : rs1;
            const float x = __fsub_rn(rad2, r2);
            if (r2 < rad2) acc = __fmaf_rn(l1 ? cf0 : cf1, __fmul_rn(__fmul_rn(x, x), x), acc);
        };
        const uint3 qb = make_uint3(qbx, q.y, q.z);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy) {
                uint32_t ba, ea;
                if (!row_range<3>(c, off, q, dy, dz, ba, ea)) continue;
                if (qbx == q.x) {   // one stencil for both nodes
                    for (uint32_t t = ba; t < ea; ++t) {
                        const float4 pj = pos[t];
                        const bool l1 = pj.w == 1.0f;
                        add(acc_a, npa, pj, l1);
                        add(acc_b, npb, pj, l1);
                    }
                } else {   // node b's row range starts and ends later in slot order
                    uint32_t bb, eb;
                    row_range<3>(c, off, qb, dy, dz, bb, eb);
                    for (uint32_t t = ba; t < eb; ++t) {
                        const float4 pj = pos[t];
                        const bool l1 = pj.w == 1.0f;
                        if (t < ea) add(acc_a, npa, pj, l1);
                        if (t >= bb) add(acc_b, npb, pj, l1);
                    }
                }
            }
        dens[row + va] = acc_a;
        if (has_b) dens[row + vb] = acc_b;
    }
}

__global__ void __launch_bounds__(kThreads) k_grid_normals(sph_config c, const float *__restrict__ dens,
                                                          float4 *__restrict__ normal)
{
    const uint32_t R = c.ndens[0], Cn = c.ndens[1], L = c.ndens[2];
    const uint32_t G = R * Cn * L;
    for (uint32_t g = grid_stride_start(); g < G; g += grid_stride()) {
        const uint32_t v[3] = {g % (R * Cn) % R, g % (R * Cn) / R, g / (R * Cn)};
        const uint32_t dims[3] = {R, Cn, L};
        const uint32_t stride[3] = {1u, R, R * Cn};
        float n[3];
        for (int a = 0; a < 3; ++a) {
            const float lo = v[a] == 0 ? 0.0f : dens[g - stride[a]];
            const float hi = v[a] == dims[a] - 1 ? 0.0f : dens[g + stride[a]];
            n[a] = (lo - hi) / c.den_size;
        }
        const float len = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        normal[g] = len == 0.0f ? make_float4(0.f, 0.f, 0.f, 0.f)
                                : make_float4(n[0] / len, n[1] / len, n[2] / len, 0.f);
    }
}

__device__ __forceinline__ uint32_t mc_cube_case(const sph_config &c, const float *__restrict__ dens, uint32_t x,
                                                 uint32_t y, uint32_t z, uint32_t *corner_node)
{
    const uint32_t R = c.ndens[0], Cn = c.ndens[1];
    uint32_t flags = 0;
    for (int v = 0; v < 8; ++v) {
        const uint32_t g = (z + kMcCornerOffset[v][2]) * R * Cn + (y + kMcCornerOffset[v][1]) * R +
                           (x + kMcCornerOffset[v][0]);
        corner_node[v] = g;
        if (dens[g] > c.iso_value) flags |= 1u << v;   // SPH-3D-2/sph_system.cpp:459-466
    }
    return flags;
}

__device__ __forceinline__ uint32_t mc_tri_count(uint32_t flags)
{
    uint32_t k = 0;
    while (k < 5 && kMcTriangles[flags][3 * k] >= 0) ++k;
    return k;
}

__global__ void __launch_bounds__(kThreads) k_mc_count(sph_config c, const float *__restrict__ dens,
                                                      uint32_t *__restrict__ cnt)
{
    const uint32_t Cm = c.ndens[1] - 1, Lm = c.ndens[2] - 1;
    const uint32_t Q = (c.ndens[0] - 1) * Cm * Lm;
    for (uint32_t q = grid_stride_start(); q < Q; q += grid_stride()) {
        const uint32_t z = q % Lm, y = (q / Lm) % Cm, x = q / (Lm * Cm);
        uint32_t nodes[8];
        cnt[q] = mc_tri_count(mc_cube_case(c, dens, x, y, z, nodes));
    }
}

// Triangles of every cube at its scanned offset.  Edge vertices are the edge
// midpoints (a + b) / 2 of the node positions i * den_size, as the reference
// places them (SPH-3D-2/sph_system.cpp:479-480), or linear interpolation at
// the iso value when mc_interpolate is set; vertex normals are the mean of
// the two node normals.
__global__ void __launch_bounds__(kThreads) k_mc_emit(sph_config c, const float *__restrict__ dens,
                                                     const float4 *__restrict__ normal,
                                                     const uint32_t *__restrict__ cnt,
                                                     const uint32_t *__restrict__ off, uint32_t max_tri,
                                                     float *__restrict__ tri)
{
    const uint32_t R = c.ndens[0], Cn = c.ndens[1];
    const uint32_t Cm = Cn - 1, Lm = c.ndens[2] - 1;
    const uint32_t Q = (R - 1) * Cm * Lm;
    float *v0 = tri, *v1 = tri + 3ull * max_tri, *v2 = tri + 6ull * max_tri;
    float *n0 = tri + 9ull * max_tri, *n1 = tri + 12ull * max_tri, *n2 = tri + 15ull * max_tri;
    for (uint32_t q = grid_stride_start(); q < Q; q += grid_stride()) {
        if (cnt[q] == 0) continue;
        const uint32_t z = q % Lm, y = (q / Lm) % Cm, x = q / (Lm * Cm);
        uint32_t node[8];
        const uint32_t flags = mc_cube_case(c, dens, x, y, z, node);
        const uint32_t base = off[q];
        for (uint32_t k = 0; k < 5; ++k) {
            if (kMcTriangles[flags][3 * k] < 0) break;
            const uint32_t t = base + k;
            if (t >= max_tri) break;
            float *vo[3] = {v0, v1, v2}, *no[3] = {n0, n1, n2};
            for (int j = 0; j < 3; ++j) {
                const int e = kMcTriangles[flags][3 * k + j];
                const int a = kMcEdgeCorner[e][0], b = kMcEdgeCorner[e][1];
                const uint32_t ga = node[a], gb = node[b];
                float pa[3] = {__fmul_rn((float)(x + kMcCornerOffset[a][0]), c.den_size),
                               __fmul_rn((float)(y + kMcCornerOffset[a][1]), c.den_size),
                               __fmul_rn((float)(z + kMcCornerOffset[a][2]), c.den_size)};
                float pb[3] = {__fmul_rn((float)(x + kMcCornerOffset[b][0]), c.den_size),
                               __fmul_rn((float)(y + kMcCornerOffset[b][1]), c.den_size),
                               __fmul_rn((float)(z + kMcCornerOffset[b][2]), c.den_size)};
                const float4 na = normal[ga], nb = normal[gb];
                float p[3];
                if (c.mc_interpolate) {
                    const float da = dens[ga], db = dens[gb];
                    const float s = db != da ? (c.iso_value - da) / (db - da) : 0.5f;
                    for (int d = 0; d < 3; ++d) p[d] = pa[d] + s * (pb[d] - pa[d]);
                } else {
                    for (int d = 0; d < 3; ++d) p[d] = __fdiv_rn(__fadd_rn(pa[d], pb[d]), 2.0f);
                }
                const float nrm[3] = {__fdiv_rn(__fadd_rn(na.x, nb.x), 2.0f), __fdiv_rn(__fadd_rn(na.y, nb.y), 2.0f),
                                      __fdiv_rn(__fadd_rn(na.z, nb.z), 2.0f)};
                for (int d = 0; d < 3; ++d) {
                    vo[j][3ull * t + d] = p[d];
                    no[j][3ull * t + d] = nrm[d];
                }
            }
        }
    }
}

}  // namespace sph
