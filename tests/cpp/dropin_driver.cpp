// Drives the drop-in SPHSystem the way the reference's GLUT application does
// (construct, add the default scene, switch split/merge on, call the step,
// read m_host_mem / the mesh) and dumps the result for
// tests/test_gpu_dropin.py.
//   dropin_driver <steps> <out.bin>
#include "sph_system.h"

#include <cstdio>
#include <cstdlib>

int main(int argc, char **argv)
{
    if (argc < 3) return 2;
    const int steps = atoi(argv[1]);
    SPHSystem *sys = new SPHSystem();
    if (sys->last_status() != SPH_OK) return 3;
#if SCA2012_VARIANT == 2
    sys->add_init_particle();
    sys->m_enable_split = 1;
    sys->m_enable_merge = 1;
#else
    sys->add_box_particle();
    sys->m_use_split = 1;
    sys->m_use_merge = 1;
#endif
    sys->m_sys_running = 1;
    for (int k = 0; k < steps; ++k) {
#if SCA2012_VARIANT == 2
        sys->animate();
#else
        if (k == steps - 1) sys->m_disp_mode = 2;
        sys->animation();
#endif
        if (sys->last_status() != SPH_OK) return 4;
    }
    FILE *f = fopen(argv[2], "wb");
    if (!f) return 5;
    unsigned n = sys->m_num_particle, rec = sizeof(Particle);
    fwrite(&n, 4, 1, f);
    fwrite(&rec, 4, 1, f);
    fwrite(sys->m_host_mem, rec, n, f);
#if SCA2012_VARIANT != 2
    unsigned nt = sys->m_num_triangle;
    fwrite(&nt, 4, 1, f);
    fwrite(sys->m_host_triangle0, sizeof(float3), nt, f);
#endif
    fclose(f);
    delete sys;
    return 0;
}
