// Structured-box addressing shared by the host launchers and the kernels.
#pragma once

namespace vfb {

// a structured box in the addressing of the boundary, drag and init kernels: node k = x + nx (y +
// ny z); on a periodic axis (bits 0-2 of `periodic` for x, y, z) the +1 neighbour wraps
struct NodeAddr {
    int nx, ny, nz, periodic;
};

} // namespace vfb
