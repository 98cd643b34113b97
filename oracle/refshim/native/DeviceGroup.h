// TEST INFRASTRUCTURE ONLY -- stand-in for the reference's
// native/DeviceGroup.h, reduced to the names that the compiled reference
// headers (TransferFunction.h, Volume.h) declare members with.  No object of
// these types is ever created by the harness.
#pragma once
#include "native/common/barney-common.h"
#include <memory>

namespace BARNEY_NS {
namespace native {
struct Device;
struct DevGroup {
  typedef std::shared_ptr<DevGroup> SP;
};
}  // namespace native
}  // namespace BARNEY_NS
