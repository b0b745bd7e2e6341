// Stand-in for Core/transfer-stencil.h, which the reference's sources include
// (FluidSim/src/cpu/advect-solver.cc:1, util.cc:1) but which is absent from the
// reference snapshot.  core::CubicKernel::weight<Real, Dim>(h, d) is the
// tensor-product cubic B-spline N(|d_i| / h) -- the same documented policy as
// the oracle restatement (fluid_oracle.cc, bspline/kweight) and the GPU path,
// with the same operation order.
#pragma once
#include <cmath>
namespace sim::core {
struct CubicKernel {
  static double N(double r) {
    if (r < 1.0) return 2.0 / 3.0 - r * r + 0.5 * r * r * r;
    if (r < 2.0) {
      double t = 2.0 - r;
      return t * t * t / 6.0;
    }
    return 0.0;
  }
  // isotropic spacing (sampleVelocity, util.cc:40-85 passes gridSpacing().x)
  template <typename T, int Dim, class V>
  static T weight(T h, const V& d) {
    T w = N(std::fabs(d[0]) / h);
    for (int i = 1; i < Dim; i++) w = w * N(std::fabs(d[i]) / h);
    return w;
  }
  // per-axis spacing (solveP2G, advect-solver.cc:204-230 passes gridSpacing())
  template <typename T, int Dim, class V>
  static T weight(const V& h, const V& d) {
    T w = N(std::fabs(d[0]) / h[0]);
    for (int i = 1; i < Dim; i++) w = w * N(std::fabs(d[i]) / h[i]);
    return w;
  }
};
}  // namespace sim::core
