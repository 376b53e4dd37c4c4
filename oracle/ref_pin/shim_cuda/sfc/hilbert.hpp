// Interface stand-in (test infrastructure): names of the space-filling-curve functions the
// reference's headers mention.  Every body returns zero; the kernels that call them (key
// generation and node centres) are never launched by the probe.
#pragma once
#include <cstdint>
#include "sfc/box.hpp"

namespace cstone {

struct IBox
{
    int lo[3], hi[3];
};

template<class KeyType>
HOST_DEVICE_FUN KeyType hilbert3D(double, double, double, const Box<double>&) { return KeyType(0); }

template<class KeyType>
HOST_DEVICE_FUN KeyType decodePlaceholderBit(KeyType) { return KeyType(0); }

template<class KeyType>
HOST_DEVICE_FUN unsigned decodePrefixLength(KeyType) { return 0u; }

template<class KeyType>
HOST_DEVICE_FUN IBox hilbertIBox(KeyType, unsigned) { return IBox{{0, 0, 0}, {0, 0, 0}}; }

template<class A, class B>
struct CenterSize
{
    A first;
    B second;
};

template<class KeyType, class T>
HOST_DEVICE_FUN CenterSize<Vec3<T>, Vec3<T>> centerAndSize(const IBox&, const Box<T>&)
{
    return CenterSize<Vec3<T>, Vec3<T>>{Vec3<T>{{T(0), T(0), T(0)}}, Vec3<T>{{T(0), T(0), T(0)}}};
}

} // namespace cstone
