// Stand-in for rmm/mr/device/cuda_async_memory_resource.hpp: stream-ordered
// allocation from a CUDA memory pool (cudaMallocFromPoolAsync /
// cudaFreeAsync).  As in rmm, the pool's release threshold is raised so that
// freed memory stays in the pool across synchronisations.
#pragma once

#include <cstdint>

#include "rmm/mr/device/device_memory_resource.hpp"

namespace rmm {
namespace mr {

class cuda_async_memory_resource final : public device_memory_resource {
 public:
  cuda_async_memory_resource() {
    int dev = 0;
    shim_check(cudaGetDevice(&dev), "cudaGetDevice");
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    shim_check(cudaMemPoolCreate(&pool_, &props), "cudaMemPoolCreate");
    uint64_t threshold = UINT64_MAX;
    shim_check(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &threshold),
               "cudaMemPoolSetAttribute");
  }
  ~cuda_async_memory_resource() override {
    cudaDeviceSynchronize();
    cudaMemPoolDestroy(pool_);
  }
  cuda_async_memory_resource(const cuda_async_memory_resource &) = delete;
  cuda_async_memory_resource &operator=(const cuda_async_memory_resource &) = delete;

 protected:
  void *do_allocate(std::size_t bytes, cudaStream_t stream) override {
    void *p = nullptr;
    shim_check(cudaMallocFromPoolAsync(&p, bytes, pool_, stream), "cudaMallocFromPoolAsync");
    return p;
  }
  void do_deallocate(void *p, std::size_t, cudaStream_t stream) override {
    shim_check(cudaFreeAsync(p, stream), "cudaFreeAsync");
  }

 private:
  cudaMemPool_t pool_ = nullptr;
};

}  // namespace mr
}  // namespace rmm
