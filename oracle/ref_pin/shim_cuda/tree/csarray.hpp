// Interface stand-in (test infrastructure): the tree index type and the leaf-array helpers
// the reference's headers name.  nodeRange and nNodes return zero; nothing here builds a
// tree.
#pragma once
#include <cstdint>
#include "util/annotation.hpp"

namespace cstone {

using TreeNodeIndex = int;

template<class KeyType>
struct maxTreeLevel
{
    constexpr operator unsigned() const { return 0u; }
};

template<class KeyType>
HOST_DEVICE_FUN constexpr KeyType nodeRange(unsigned) { return KeyType(0); }

template<class V>
inline TreeNodeIndex nNodes(const V&) { return 0; }

} // namespace cstone
