// Explicit instantiation of the float pass kernels and their launchers for
// the grid sizes 2^a 3^b 5^c other than the sub-grid sizes (48, 60, 96, 300, 600).
#include "ps_launch.cuh"

namespace ps {
PS_INSTANTIATE_L3_MIXED(float)
}  // namespace ps
