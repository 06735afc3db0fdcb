// Kernels of the exact arithmetic variant for float population storage (see launch_impl.cuh).
#define VFB_NS exact
#define VFB_EXACT true
#include "launch_impl.cuh"

template struct vfb::exact::Launchers<float>;
