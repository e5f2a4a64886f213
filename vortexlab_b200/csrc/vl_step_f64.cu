// FP64 step kernels. This translation unit is compiled with -fmad=false: no multiply-add is
// fused, so every FP64 result is bit-identical to the reference's CPU path.
#include "vl_launch_impl.cuh"

namespace vl {
const Launchers& launchers_f64() { return LaunchImpl<double>::table(); }
}  // namespace vl
