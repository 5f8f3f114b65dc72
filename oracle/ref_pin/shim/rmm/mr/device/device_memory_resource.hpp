// Project-written stand-in for the small part of RAPIDS rmm (branch-22.12,
// the tag the reference's CMakeLists.txt:21-28 fetches) that the reference's
// include/core/DeviceVector.h:80-125 and include/core/MemoryPool.h:13-25 use.
// rmm is not installed here (its build needs the network), so the reference
// sources compile against this instead.  Test infrastructure only: it backs
// the reference build that the parity tests and the reference timing run.
//
// Semantics kept from rmm's published API:
//  * a device_memory_resource hands out stream-ordered device allocations;
//  * the "current device resource" is process-wide (one device here) and a
//    buffer remembers the resource it was allocated from;
//  * set_current_device_resource(nullptr) restores the initial resource
//    (plain cudaMalloc / cudaFree).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdio>
#include <cstdlib>

namespace rmm {

inline void shim_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "rmm shim: %s failed: %s\n", what, cudaGetErrorString(e));
    std::abort();
  }
}

namespace mr {

class device_memory_resource {
 public:
  virtual ~device_memory_resource() = default;
  void *allocate(std::size_t bytes, cudaStream_t stream) {
    return bytes == 0 ? nullptr : do_allocate(bytes, stream);
  }
  void deallocate(void *p, std::size_t bytes, cudaStream_t stream) {
    if (p != nullptr) do_deallocate(p, bytes, stream);
  }

 protected:
  virtual void *do_allocate(std::size_t bytes, cudaStream_t stream) = 0;
  virtual void do_deallocate(void *p, std::size_t bytes, cudaStream_t stream) = 0;
};

// rmm::mr::cuda_memory_resource: synchronous cudaMalloc / cudaFree.
class cuda_memory_resource final : public device_memory_resource {
 protected:
  void *do_allocate(std::size_t bytes, cudaStream_t) override {
    void *p = nullptr;
    shim_check(cudaMalloc(&p, bytes), "cudaMalloc");
    return p;
  }
  void do_deallocate(void *p, std::size_t, cudaStream_t) override {
    shim_check(cudaFree(p), "cudaFree");
  }
};

}  // namespace mr
}  // namespace rmm
