// sph_pov.cpp — headless POV-Ray scene files for the surface and the particles.
//
// The reference renders offline by writing POV-Ray scenes from its GLUT app
// (make_mesh, make_particle: SPH-3D-2/sph_main.cpp:114-220): one
// smooth_triangle per marching-cubes triangle (vertices scaled by the
// display ratio and shifted by the display origin, normals as computed), or
// one coloured sphere per particle (red radius 0.3 for level 1, yellow 0.24
// for level 2).  These writers produce the same object lines from a mesh or
// particle arrays so that pipeline keeps working without a window.
#include "../../include/sph/sph.h"

#include <cstdio>

namespace {

const char *kMeshHeader =
    "#include \"colors.inc\"\n"
    "camera { location <5,10,-35> look_at <0,0,0> }\n"
    "light_source { <13, 13, -20> color White }\n"
    "mesh {\n";
const char *kMeshFooter =
    "pigment { color red 0.8 green 0.8 blue 0.8 transmit 0.6 } finish { ambient 0.2 diffuse 0.5 } }\n"
    "plane { <0,-1,0>, 10 pigment { checker color White, color Black } }\n";
const char *kParticleHeader =
    "#include \"colors.inc\"\n"
    "camera { location <5,10,-35> look_at <0,0,0> }\n"
    "light_source { <13, 13, -20> color White }\n";
const char *kParticleFooter = "plane { <0,-1,0>, 10 pigment { checker color White, color Black } }\n";

float tr(const float *v, int a, const float *scale, const float *offset)
{
    return v[a] * (scale ? scale[a] : 1.0f) + (offset ? offset[a] : 0.0f);
}

}  // namespace

extern "C" int sph_write_pov_mesh(const sph_mesh_view *mesh, const float *scale, const float *offset, const char *path)
{
    if (!mesh || !path) return SPH_ERR_INVALID;
    FILE *fp = fopen(path, "w");
    if (!fp) return SPH_ERR_INVALID;
    fputs(kMeshHeader, fp);
    const uint32_t nt = mesh->num_triangles < mesh->max_triangles ? mesh->num_triangles : mesh->max_triangles;
    const float *v[3] = {mesh->v0, mesh->v1, mesh->v2}, *nn[3] = {mesh->n0, mesh->n1, mesh->n2};
    for (uint32_t t = 0; t < nt; ++t) {
        fprintf(fp, "smooth_triangle { ");
        for (int k = 0; k < 3; ++k) {
            const float *p = v[k] + 3ull * t, *q = nn[k] + 3ull * t;
            fprintf(fp, "<%f, %f, %f>, <%f, %f, %f>%s", tr(p, 0, scale, offset), tr(p, 1, scale, offset),
                    tr(p, 2, scale, offset), q[0], q[1], q[2], k < 2 ? ", " : "");
        }
        fprintf(fp, " }  \n");
    }
    fputs(kMeshFooter, fp);
    return fclose(fp) == 0 ? SPH_OK : SPH_ERR_INVALID;
}

extern "C" int sph_write_pov_particles(const float *pos, const uint32_t *level, uint32_t n, uint32_t dim,
                                       const float *scale, const float *offset, const char *path)
{
    if ((n && (!pos || !level)) || !path || (dim != 2 && dim != 3)) return SPH_ERR_INVALID;
    FILE *fp = fopen(path, "w");
    if (!fp) return SPH_ERR_INVALID;
    fputs(kParticleHeader, fp);
    for (uint32_t i = 0; i < n; ++i) {
        const float p3[3] = {pos[(size_t)i * dim], pos[(size_t)i * dim + 1], dim == 3 ? pos[(size_t)i * dim + 2] : 0.0f};
        const float x = tr(p3, 0, scale, offset), y = tr(p3, 1, scale, offset), z = tr(p3, 2, scale, offset);
        if (level[i] == 1)
            fprintf(fp, "sphere { <%f, %f, %f>, %f texture { pigment { color Red } } }\n", x, y, z, 0.3f);
        else
            fprintf(fp, "sphere { <%f, %f, %f>, %f texture { pigment { color Yellow } } }\n", x, y, z, 0.24f);
    }
    fputs(kParticleFooter, fp);
    return fclose(fp) == 0 ? SPH_OK : SPH_ERR_INVALID;
}
