// host_lattice.h -- host-side wing lattice generation (set-up, once per case).
#pragma once

#include <cmath>
#include <vector>

#include "../../include/uvlm_b200.h"

namespace uvlm {

// RectGenerator (src/wing/rect.cpp:18-45) with linspace (src/util.h:36-43)
// and TransformChebyshev (src/wing/rect.h:16-25); host set-up, once per case.
inline std::vector<double> linspace(double a, double b, size_t N) {
  const double dx = (b - a) / (N - 1);
  std::vector<double> r;
  for (size_t i = 0; i < N; i++) r.push_back(a + i * dx);
  return r;
}
inline std::vector<double> chebyshev(size_t N, double xmin, double xmax) {
  auto th = linspace(-M_PI_2, 0, N);
  std::vector<double> r;
  for (double t : th) r.push_back(xmin + (xmax - xmin) * std::cos(t));
  r.front() = xmin;
  r.back() = xmax;
  return r;
}
// WholeWing (src/wing/wing.cpp:12-52) of the half wing (chord, span/2,
// rows, cols/2), shifted by the wing origin (simple_simulator.cpp:159-166).
inline std::vector<double> whole_wing_nodes(const uvlm_wing_desc& w) {
  const size_t rows = (size_t)w.rows, hc = (size_t)w.cols / 2;
  auto xs = w.chebyshev_chord ? chebyshev(rows + 1, 0, w.chord) : linspace(0, w.chord, rows + 1);
  auto ys = w.chebyshev_span ? chebyshev(hc + 1, 0, w.span / 2) : linspace(0, w.span / 2, hc + 1);
  std::vector<double> out;
  out.reserve((rows + 1) * (2 * hc + 1) * 3);
  for (size_t i = 0; i <= rows; i++) {
    for (size_t q = 0; q <= hc; q++) {  // mirrored half, reversed
      const size_t jj = hc - q;
      out.push_back(xs[i] + 0.0 + w.origin[0]);
      out.push_back(ys[jj] * -1 + w.origin[1]);
      out.push_back(0.0 + w.origin[2]);
    }
    for (size_t jj = 1; jj <= hc; jj++) {
      out.push_back(xs[i] + w.origin[0]);
      out.push_back(ys[jj] + w.origin[1]);
      out.push_back(0.0 + w.origin[2]);
    }
  }
  return out;
}

}  // namespace uvlm
