/*
 * Test-infrastructure stand-in for the pinned allocator header that CUDA 12
 * no longer ships.  The oracle's reference build compiles the reference's host
 * sources for the CPU only (no -DGPU), where these declarations name buffers
 * that the CPU aligner never allocates; a std::allocator keeps them valid.
 */
#ifndef GZ_REFSTUB_THRUST_PINNED_ALLOCATOR_H_
#define GZ_REFSTUB_THRUST_PINNED_ALLOCATOR_H_
#include <memory>

namespace thrust {
namespace cuda {
namespace experimental {
template <typename T>
class pinned_allocator : public std::allocator<T> {
 public:
  template <typename U>
  struct rebind {
    typedef pinned_allocator<U> other;
  };
  pinned_allocator() {}
  template <typename U>
  pinned_allocator(const pinned_allocator<U> &) {}
};
}  // namespace experimental
}  // namespace cuda
}  // namespace thrust
#endif
