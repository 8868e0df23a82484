// Explicit instantiation of the double pass kernels and their launchers.
#include "ps_launch.cuh"

namespace ps {
PS_INSTANTIATE_L3_POW2(double)
}  // namespace ps
