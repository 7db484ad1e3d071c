// Stand-in (test infrastructure only) for the two Boost.Serialization names that frame-aligner's
// Cv3dUtils.h mentions in uninstantiated templates. Nothing here is ever executed.
#pragma once
#include <cstddef>
#define BOOST_SERIALIZATION_SPLIT_FREE(T)
namespace boost {
namespace serialization {
struct binary_object {
  binary_object(void* p, std::size_t n) : ptr(p), size(n) {}
  void* ptr;
  std::size_t size;
};
}  // namespace serialization
}  // namespace boost
