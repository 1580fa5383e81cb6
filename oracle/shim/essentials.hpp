/* Build shim for oracle/_ref only: the two helpers the reference's encoders take
 * from the (empty) `essentials` submodule. */
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace essentials {
inline uint64_t words_for(uint64_t bits) { return (bits + 63) / 64; }
template <typename T>
inline size_t vec_bytes(std::vector<T> const &v) { return sizeof(T) * v.size() + sizeof(size_t); }
}  // namespace essentials
