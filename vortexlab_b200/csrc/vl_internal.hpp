// Declarations shared by the host translation units (not part of the C ABI).
#pragma once

#include <memory>
#include <vector>

#include "../../include/vortexlab.h"
#include "vl_host.hpp"

struct vl_shape {
  std::unique_ptr<vl::Shape> s;
};

namespace vl {

// Channel::new / Channel::step host decisions for a channel spec; takes the body shape.
int plan_channel(const vl_channel_spec* sp, std::unique_ptr<Shape> body, ChannelPlan& out);
// The developed inflow profile as a (rho, ux, uy) start field.
void profile_field(const ChannelPlan& plan, std::vector<double>& rho, std::vector<double>& ux,
                   std::vector<double>& uy);

}  // namespace vl
