// Stand-in for rmm/mr/device/binning_memory_resource.hpp.  rmm's binning
// resource routes an allocation to the smallest bin whose block size holds
// it (each bin a fixed-size block pool fed by the upstream) and anything
// larger than the largest bin to the upstream.  Here a bin is a free list of
// blocks of the bin's size: a freed block is reused by the next allocation
// of that bin in stream order (the reference issues all work on one stream,
// so reuse needs no synchronisation), and blocks go back to the upstream
// when the resource is destroyed.
#pragma once

#include <algorithm>
#include <map>
#include <unordered_map>
#include <vector>

#include "rmm/mr/device/device_memory_resource.hpp"

namespace rmm {
namespace mr {

template <typename Upstream>
class binning_memory_resource final : public device_memory_resource {
 public:
  explicit binning_memory_resource(Upstream *upstream) : upstream_(upstream) {}
  ~binning_memory_resource() override {
    for (auto &kv : free_) {
      for (void *p : kv.second) upstream_->deallocate(p, kv.first, stream_of_release_);
    }
  }
  binning_memory_resource(const binning_memory_resource &) = delete;
  binning_memory_resource &operator=(const binning_memory_resource &) = delete;

  void add_bin(std::size_t allocation_size) { free_[allocation_size]; }

 protected:
  void *do_allocate(std::size_t bytes, cudaStream_t stream) override {
    auto it = free_.lower_bound(bytes);
    if (it == free_.end()) return upstream_->allocate(bytes, stream);
    std::vector<void *> &list = it->second;
    void *p;
    if (list.empty()) {
      p = upstream_->allocate(it->first, stream);
    } else {
      p = list.back();
      list.pop_back();
    }
    return p;
  }
  void do_deallocate(void *p, std::size_t bytes, cudaStream_t stream) override {
    auto it = free_.lower_bound(bytes);
    if (it == free_.end()) {
      upstream_->deallocate(p, bytes, stream);
      return;
    }
    it->second.push_back(p);
  }

 private:
  Upstream *upstream_;
  std::map<std::size_t, std::vector<void *>> free_;
  cudaStream_t stream_of_release_ = cudaStreamLegacy;
};

}  // namespace mr
}  // namespace rmm
