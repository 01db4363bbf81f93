// Declaration-only stand-in for the third-party wykobi header that src/linalg/Geom.hpp includes
// (the submodule is not vendored). The oracle harness never evaluates the closest-point
// projections that use it; declarations let the reference's dg/Basis.cpp compile unchanged.
#pragma once
namespace wykobi {
template <typename T, unsigned int D> class triangle;
template <typename T> class point2d;
template <typename T> class point3d;
template <typename T> point2d<T> closest_point_on_triangle_from_point(const triangle<T, 2> &, const point2d<T> &);
template <typename T> point3d<T> closest_point_on_triangle_from_point(const triangle<T, 3> &, const point3d<T> &);
template <typename T> T distance(const point3d<T> &, const point3d<T> &);
template <typename T> T robust_cartesian_angle(const T &, const T &);
}  // namespace wykobi
