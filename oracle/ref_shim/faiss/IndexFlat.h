/* Stand-in for faiss/IndexFlat.h: the oracle never trains with faiss
 * (Index::train(..., faiss=true)); these types only let Index.cpp compile. */
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstdint>
namespace faiss {
struct IndexFlatL2 {
  explicit IndexFlatL2(size_t) {}
  const float* get_xb() const { std::fprintf(stderr, "oracle: faiss training unavailable\n"); std::abort(); }
};
}  // namespace faiss
