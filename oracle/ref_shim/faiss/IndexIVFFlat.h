/* Stand-in for faiss/IndexIVFFlat.h; see IndexFlat.h. */
#pragma once
#include "IndexFlat.h"
namespace faiss {
struct IndexIVFFlat {
  IndexIVFFlat(IndexFlatL2*, size_t, size_t) {}
  void train(size_t, const float*) { std::fprintf(stderr, "oracle: faiss training unavailable\n"); std::abort(); }
};
}  // namespace faiss
