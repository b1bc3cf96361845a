// sph_mc.cuh — density grid, grid normals and marching cubes on the device.
#pragma once
#include <cstdint>
#include <vector>
#include "../../include/sph/sph.h"

namespace sph {

struct McBuffers {
    uint32_t nodes = 0;
};

inline int mc_alloc(McBuffers &mc, const sph_config &c, std::vector<void *> &)
{
    mc.nodes = c.dim == 3 ? c.ndens[0] * c.ndens[1] * c.ndens[2] : 0u;
    return SPH_OK;
}

}  // namespace sph
