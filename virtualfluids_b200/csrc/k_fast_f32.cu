// Kernels of the fast arithmetic variant for float population storage (see launch_impl.cuh).
#define VFB_NS fast
#define VFB_EXACT false
#include "launch_impl.cuh"

template struct vfb::fast::Launchers<float>;
