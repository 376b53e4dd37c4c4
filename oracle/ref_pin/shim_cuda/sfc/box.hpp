// Interface stand-in (test infrastructure): the box, boundary and 3-vector types the
// reference's kernels take by value.  Box keeps its limits and reports each length as
// max - min.  minDistance and norm2 return zero: only the never-launched j-leaf walk
// calls them.
#pragma once
#include "util/annotation.hpp"

namespace util {
template<class A, class B>
struct TiePair
{
    A& a;
    B& b;
    template<class P>
    HOST_DEVICE_FUN TiePair& operator=(const P& p) { a = p.first; b = p.second; return *this; }
};
template<class A, class B>
HOST_DEVICE_FUN TiePair<A, B> tie(A& a, B& b) { return TiePair<A, B>{a, b}; }
} // namespace util

namespace cstone {

enum class BoundaryType : int { open = 0, periodic = 1, fixed = 2 };

template<class T>
struct Vec3
{
    T v[3];
    HOST_DEVICE_FUN T& operator[](int i) { return v[i]; }
    HOST_DEVICE_FUN const T& operator[](int i) const { return v[i]; }
};

template<class T>
class Box
{
public:
    HOST_DEVICE_FUN Box(T xyzMin, T xyzMax, BoundaryType b = BoundaryType::open)
        : Box(xyzMin, xyzMax, xyzMin, xyzMax, xyzMin, xyzMax, b, b, b) {}
    HOST_DEVICE_FUN Box(T xmin, T xmax, T ymin, T ymax, T zmin, T zmax, BoundaryType bx = BoundaryType::open,
                        BoundaryType by = BoundaryType::open, BoundaryType bz = BoundaryType::open)
        : lo_{xmin, ymin, zmin}, hi_{xmax, ymax, zmax}, b_{bx, by, bz} {}
    HOST_DEVICE_FUN T xmin() const { return lo_[0]; }
    HOST_DEVICE_FUN T xmax() const { return hi_[0]; }
    HOST_DEVICE_FUN T ymin() const { return lo_[1]; }
    HOST_DEVICE_FUN T ymax() const { return hi_[1]; }
    HOST_DEVICE_FUN T zmin() const { return lo_[2]; }
    HOST_DEVICE_FUN T zmax() const { return hi_[2]; }
    HOST_DEVICE_FUN T lx() const { return hi_[0] - lo_[0]; }
    HOST_DEVICE_FUN T ly() const { return hi_[1] - lo_[1]; }
    HOST_DEVICE_FUN T lz() const { return hi_[2] - lo_[2]; }
    HOST_DEVICE_FUN BoundaryType boundaryX() const { return b_[0]; }
    HOST_DEVICE_FUN BoundaryType boundaryY() const { return b_[1]; }
    HOST_DEVICE_FUN BoundaryType boundaryZ() const { return b_[2]; }

private:
    T lo_[3], hi_[3];
    BoundaryType b_[3];
};

template<class T>
HOST_DEVICE_FUN Vec3<T> minDistance(const Vec3<T>&, const Vec3<T>&, const Vec3<T>&)
{
    return Vec3<T>{{T(0), T(0), T(0)}};
}
template<class T>
HOST_DEVICE_FUN Vec3<T> minDistance(const Vec3<T>&, const Vec3<T>&, const Vec3<T>&, const Vec3<T>&)
{
    return Vec3<T>{{T(0), T(0), T(0)}};
}
template<class T>
HOST_DEVICE_FUN Vec3<T> minDistance(const Vec3<T>&, const Vec3<T>&, const Vec3<T>&, const Vec3<T>&, const Box<T>&)
{
    return Vec3<T>{{T(0), T(0), T(0)}};
}
template<class T>
HOST_DEVICE_FUN T norm2(const Vec3<T>&) { return T(0); }

} // namespace cstone
