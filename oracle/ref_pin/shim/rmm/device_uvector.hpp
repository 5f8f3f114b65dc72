// Stand-in for rmm/device_uvector.hpp: an uninitialised, typed device array
// that allocates from the current device resource at construction, keeps
// that resource for its lifetime, and is movable but not copyable.
// resize() keeps the leading min(old, new) elements: it reallocates only
// when the new size exceeds the capacity, copying on the vector's stream.
#pragma once

#include <cstddef>
#include <utility>

#include "rmm/mr/device/per_device_resource.hpp"

namespace rmm {

template <typename T>
class device_uvector {
 public:
  using value_type = T;
  using pointer = T *;
  using const_pointer = const T *;
  using iterator = T *;
  using const_iterator = const T *;

  device_uvector(std::size_t size, cudaStream_t stream)
      : stream_(stream), mr_(mr::get_current_device_resource()) {
    allocate_exact(size);
  }
  device_uvector(const device_uvector &) = delete;
  device_uvector &operator=(const device_uvector &) = delete;
  device_uvector(device_uvector &&o) noexcept
      : data_(o.data_), size_(o.size_), capacity_(o.capacity_), stream_(o.stream_), mr_(o.mr_) {
    o.data_ = nullptr;
    o.size_ = 0;
    o.capacity_ = 0;
  }
  device_uvector &operator=(device_uvector &&o) noexcept {
    if (this != &o) {
      release_storage();
      data_ = o.data_;
      size_ = o.size_;
      capacity_ = o.capacity_;
      stream_ = o.stream_;
      mr_ = o.mr_;
      o.data_ = nullptr;
      o.size_ = 0;
      o.capacity_ = 0;
    }
    return *this;
  }
  ~device_uvector() { release_storage(); }

  T *data() noexcept { return data_; }
  const T *data() const noexcept { return data_; }
  std::size_t size() const noexcept { return size_; }
  std::size_t capacity() const noexcept { return capacity_; }
  bool is_empty() const noexcept { return size_ == 0; }
  T *begin() noexcept { return data_; }
  T *end() noexcept { return data_ + size_; }
  const T *begin() const noexcept { return data_; }
  const T *end() const noexcept { return data_ + size_; }
  cudaStream_t stream() const noexcept { return stream_; }
  void set_stream(cudaStream_t s) noexcept { stream_ = s; }

  void resize(std::size_t new_size, cudaStream_t stream) {
    stream_ = stream;
    if (new_size <= capacity_) {
      size_ = new_size;
      return;
    }
    T *old = data_;
    std::size_t old_size = size_, old_cap = capacity_;
    data_ = static_cast<T *>(mr_->allocate(new_size * sizeof(T), stream_));
    if (old_size > 0) {
      shim_check(cudaMemcpyAsync(data_, old, old_size * sizeof(T), cudaMemcpyDeviceToDevice, stream_),
                 "cudaMemcpyAsync");
    }
    mr_->deallocate(old, old_cap * sizeof(T), stream_);
    size_ = new_size;
    capacity_ = new_size;
  }

  void shrink_to_fit(cudaStream_t stream) {
    if (size_ == capacity_) return;
    device_uvector tmp(size_, stream);
    if (size_ > 0) {
      shim_check(cudaMemcpyAsync(tmp.data_, data_, size_ * sizeof(T), cudaMemcpyDeviceToDevice, stream),
                 "cudaMemcpyAsync");
    }
    *this = std::move(tmp);
  }

 private:
  void allocate_exact(std::size_t n) {
    data_ = static_cast<T *>(mr_->allocate(n * sizeof(T), stream_));
    size_ = n;
    capacity_ = n;
  }
  void release_storage() {
    if (data_ != nullptr) mr_->deallocate(data_, capacity_ * sizeof(T), stream_);
    data_ = nullptr;
    size_ = 0;
    capacity_ = 0;
  }

  T *data_ = nullptr;
  std::size_t size_ = 0;
  std::size_t capacity_ = 0;
  cudaStream_t stream_;
  mr::device_memory_resource *mr_;
};

}  // namespace rmm
