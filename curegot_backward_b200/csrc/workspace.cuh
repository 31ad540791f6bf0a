// Stream-ordered workspace: one block from the library pool carved into
// 256-byte-aligned pieces, released with cudaFreeAsync on the same stream.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "common.cuh"

namespace cg {

class Workspace {
 public:
  explicit Workspace(cudaStream_t s) : stream_(s) {}
  ~Workspace() { release(); }
  Workspace(const Workspace&) = delete;
  Workspace& operator=(const Workspace&) = delete;

  // Reserve `bytes` (first pass: sizing).  Returns the offset.
  template <typename T>
  size_t reserve(size_t count) {
    const size_t off = (size_ + 255) & ~size_t(255);
    size_ = off + count * sizeof(T);
    offsets_.push_back(off);
    return off;
  }
  int allocate() {
    if (size_ == 0) return CG_OK;
    CG_TRY(pool_alloc_async(&base_, size_, stream_));
    return CG_OK;
  }
  template <typename T>
  T* at(size_t off) const {
    return reinterpret_cast<T*>(static_cast<char*>(base_) + off);
  }
  void* base() const { return base_; }
  size_t size() const { return size_; }
  void release() {
    if (base_) {
      cudaFreeAsync(base_, stream_);
      base_ = nullptr;
    }
  }

 private:
  cudaStream_t stream_;
  void* base_ = nullptr;
  size_t size_ = 0;
  std::vector<size_t> offsets_;
};

}  // namespace cg
