// Kernels of the fast arithmetic variant for E3M12 population storage (see launch_impl.cuh).
#define VFB_NS fast
#define VFB_EXACT false
#include "launch_impl.cuh"

template struct vfb::fast::Launchers<vfb::e3m12_t>;
