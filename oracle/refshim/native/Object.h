// TEST INFRASTRUCTURE ONLY -- stand-in for the reference's native/Object.h,
// reduced to the base classes and virtual setters that the compiled reference
// headers (TransferFunction.h, Volume.h) derive from and override.
#pragma once
#include "native/common/barney-common.h"
#include "native/DeviceGroup.h"
#include <string>

namespace BARNEY_NS {
namespace native {
struct Context;
struct Object : public std::enable_shared_from_this<Object> {
  typedef std::shared_ptr<Object> SP;
  Object(Context *context = nullptr) : context(context) {}
  virtual ~Object() = default;
  virtual std::string toString() const { return "Object"; }
  virtual void commit() {}
  virtual bool set1i(const std::string &, const int &) { return false; }
  virtual bool set1f(const std::string &, const float &) { return false; }
  virtual bool set2f(const std::string &, const vec2f &) { return false; }
  virtual bool set3f(const std::string &, const vec3f &) { return false; }
  Context *const context;
};
struct SlottedObject : public Object {
  SlottedObject(Context *context, const DevGroup::SP &devices) : Object(context), devices(devices) {}
  const DevGroup::SP devices;
};
}  // namespace native
}  // namespace BARNEY_NS
