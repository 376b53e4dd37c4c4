// Interface stand-in (test infrastructure): the linked-octree container the reference's
// GpuState holds, with the members its sources touch.  Nothing here fills it.
#pragma once
#include <cstdint>
#include <thrust/device_vector.h>
#include "tree/csarray.hpp"

namespace cstone {

struct GpuTag {};
struct CpuTag {};

template<class KeyType, class Tag>
struct OctreeData
{
    thrust::device_vector<KeyType> prefixes;
    thrust::device_vector<TreeNodeIndex> childOffsets;
    thrust::device_vector<TreeNodeIndex> parents;
    thrust::device_vector<TreeNodeIndex> internalToLeaf;
    thrust::device_vector<TreeNodeIndex> leafToInternal;
    thrust::device_vector<TreeNodeIndex> levelRange;
    TreeNodeIndex numNodes = 0;
    TreeNodeIndex numLeafNodes = 0;
};

} // namespace cstone
