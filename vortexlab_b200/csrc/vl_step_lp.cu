// Reduced-precision step kernels: FP32 storage, IEEE FP16 storage of f_i - w_i, the custom
// 16-bit storage of f_i - w_i (c16) and its 16-bit fixed point (q16), all with FP32 collision
// arithmetic; the force accumulation and
// every reduction stay in FP64. Compiled without multiply-add contraction like the FP64 kernels:
// the narrow collision states its fused multiply-adds with intrinsics, and every other expression
// (link rules, decoding) then rounds the same way in every kernel that evaluates it.
#include "vl_launch_impl.cuh"

namespace vl {
const Launchers& launchers_f32() { return LaunchImpl<float>::table(); }
const Launchers& launchers_f16s() { return LaunchImpl<__half>::table(); }
const Launchers& launchers_f16c() { return LaunchImpl<c16>::table(); }
const Launchers& launchers_f16x() { return LaunchImpl<q16>::table(); }
}  // namespace vl
