// Stand-in for rmm/mr/device/per_device_resource.hpp (see
// device_memory_resource.hpp in this folder for what the stand-ins are).
#pragma once

#include "rmm/mr/device/device_memory_resource.hpp"

namespace rmm {
namespace mr {

inline device_memory_resource *initial_resource() {
  static cuda_memory_resource res;
  return &res;
}

inline device_memory_resource *&current_resource_slot() {
  static device_memory_resource *cur = nullptr;
  return cur;
}

inline device_memory_resource *get_current_device_resource() {
  device_memory_resource *cur = current_resource_slot();
  return cur != nullptr ? cur : initial_resource();
}

// Returns the previous resource; nullptr restores the initial one.
inline device_memory_resource *set_current_device_resource(device_memory_resource *mr) {
  device_memory_resource *prev = get_current_device_resource();
  current_resource_slot() = mr;
  return prev;
}

}  // namespace mr
}  // namespace rmm
