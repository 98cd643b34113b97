// TEST INFRASTRUCTURE ONLY -- stand-in for the reference's
// native/volume/ScalarField.h (which pulls in the macrocell grid, the model
// slot and the context), reduced to what Volume.h names: ScalarField::SP and
// ScalarField::DD.
#pragma once
#include "native/Object.h"

namespace BARNEY_NS {
namespace native {
struct ScalarField : public SlottedObject {
  typedef std::shared_ptr<ScalarField> SP;
  struct DD {
    box3f worldBounds;
  };
  DD getDD(Device *device);
};
}  // namespace native
}  // namespace BARNEY_NS
