// uvlm_b200.hpp -- header-only C++17 adapter: the reference's C++ API
// (namespace UVLM) implemented on the uvlm_b200 C-ABI.
//
// A C++ host that used xeno14/UVLM includes this header instead of
// src/uvlm.h (src/uvlm.h:1-23) and links libuvlm_b200.so.  Mirrored surfaces:
//   UVLM::InducedVelocity(x, pos, gamma)            src/velocity.h:14-24
//   UVLM::advect::Advection / Euler / RungeKutta2 /
//     RungeKutta4 / AdamsBashforth2, AdvectFactory   src/advect.h:48-121,
//                                                    src/advect_factory.cpp:43-60
//   UVLM::Morphing (closed-form sinusoid setters)    src/morphing.h:25-108
//   UVLM::wing::{WingGenerator, RectGenerator, NACA4digitGenerator,
//     NACA00XXGenerator, WholeWing}, proto::Wing     src/wing/*, proto/uvlm.proto:6-30
//   UVLM::simulator::SimpleSimulator                 src/simulator/simple_simulator.h:33-108
//   multiple_sheet::MultipleSheet<T> (layout of the missing submodule,
//     contiguous [num][rows][cols])
//   the legacy AoS API (VortexRing, VortexContainer, shed, linear,
//     calc_load, WingBuilder, simulator::Start)  uvlm_b200_legacy.hpp
// The element type of node sheets is UVLM_B200_VECTOR3 (default UVLM::Vec3);
// any type of three packed doubles works, e.g. define it to Eigen::Vector3d
// before including this header.  Errors throw UVLM::Error where the
// reference would LOG(FATAL) / CHECK-fail; defining UVLM_B200_FATAL_ON_ERROR
// before including it makes them print the message to stderr and abort, as
// the reference's LOG(FATAL) does.
#pragma once

#include <array>
#include <cmath>
#include <typeinfo>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "uvlm_b200.h"

namespace UVLM {

struct Vec3 {
  double v[3] = {0, 0, 0};
  Vec3() = default;
  Vec3(double x, double y, double z) : v{x, y, z} {}
  double& operator[](std::size_t i) { return v[i]; }
  double operator[](std::size_t i) const { return v[i]; }
  double x() const { return v[0]; }
  double y() const { return v[1]; }
  double z() const { return v[2]; }
};

}  // namespace UVLM

#ifndef UVLM_B200_VECTOR3
#define UVLM_B200_VECTOR3 ::UVLM::Vec3
#endif

namespace multiple_sheet {

// MultipleSheet<T>(num, rows, cols): contiguous storage, index
// K = j + cols * (i + rows * n) (the order of the reference's call sites).
template <class T>
class MultipleSheet {
 public:
  MultipleSheet() = default;
  MultipleSheet(std::size_t num, std::size_t rows, std::size_t cols) { resize(num, rows, cols); }
  void resize(std::size_t num, std::size_t rows, std::size_t cols) {
    num_ = num;
    rows_ = rows;
    cols_ = cols;
    data_.assign(num * rows * cols, T{});
  }
  template <class U>
  void resize(const MultipleSheet<U>& o) {
    resize(o.num(), o.rows(), o.cols());
  }
  std::size_t num() const { return num_; }
  std::size_t rows() const { return rows_; }
  std::size_t cols() const { return cols_; }
  std::size_t size() const { return data_.size(); }
  std::size_t index(std::size_t n, std::size_t i, std::size_t j) const { return j + cols_ * (i + rows_ * n); }
  T& at(std::size_t n, std::size_t i, std::size_t j) { return data_[index(n, i, j)]; }
  const T& at(std::size_t n, std::size_t i, std::size_t j) const { return data_[index(n, i, j)]; }
  T& operator[](std::size_t k) { return data_[k]; }
  const T& operator[](std::size_t k) const { return data_[k]; }
  typename std::vector<T>::iterator begin() { return data_.begin(); }
  typename std::vector<T>::iterator end() { return data_.end(); }
  typename std::vector<T>::const_iterator begin() const { return data_.begin(); }
  typename std::vector<T>::const_iterator end() const { return data_.end(); }
  T* data() { return data_.data(); }
  const T* data() const { return data_.data(); }

 private:
  std::size_t num_ = 0, rows_ = 0, cols_ = 0;
  std::vector<T> data_;
};

}  // namespace multiple_sheet

namespace UVLM {

using multiple_sheet::MultipleSheet;
using Vector3 = UVLM_B200_VECTOR3;
static_assert(sizeof(Vector3) == 3 * sizeof(double), "node sheets need three packed doubles per element");

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

namespace detail {
inline void check(int rc, const char* what, const char* detail_msg = nullptr) {
  if (rc == UVLM_OK) return;
  std::string m = std::string(what) + ": " + uvlm_status_string(rc);
  const char* d = detail_msg ? detail_msg : uvlm_global_last_error();
  if (d && *d) m += std::string(" (") + d + ")";
#ifdef UVLM_B200_FATAL_ON_ERROR
  std::fprintf(stderr, "F uvlm_b200] Check failed: %s\n", m.c_str());
  std::fflush(stderr);
  std::abort();
#else
  throw Error(rc, m);
#endif
}
template <class S>
inline const double* dptr(const S& sheet) {
  return sheet.size() ? reinterpret_cast<const double*>(&*sheet.begin()) : nullptr;
}
template <class S>
inline double* dptr_mut(S& sheet) {
  return sheet.size() ? reinterpret_cast<double*>(&*sheet.begin()) : nullptr;
}
}  // namespace detail

// UVLM::InducedVelocity(x, pos, gamma) (src/velocity.h:14-24): the velocity
// that every ring of the sheets induces at x.  pos holds (rows + 1) x
// (cols + 1) nodes per sheet, gamma rows x cols circulations.
template <class SheetV, class SheetD>
inline Vector3 InducedVelocity(const Vector3& x, const SheetV& pos, const SheetD& gamma,
                               int precision = UVLM_PRECISION_FP64) {
  Vector3 out{};
  detail::check(uvlm_sheet_induced_velocity(detail::dptr(pos), detail::dptr(gamma), (int64_t)gamma.num(),
                                            (int64_t)gamma.rows(), (int64_t)gamma.cols(),
                                            reinterpret_cast<const double*>(&x), 1,
                                            reinterpret_cast<double*>(&out), precision),
                "InducedVelocity");
  return out;
}

// Many targets in one call (the form every N-body stage uses).
template <class SheetV, class SheetD>
inline std::vector<Vector3> InducedVelocity(const std::vector<Vector3>& xs, const SheetV& pos, const SheetD& gamma,
                                            int precision = UVLM_PRECISION_FP64) {
  std::vector<Vector3> out(xs.size());
  if (xs.empty()) return out;
  detail::check(uvlm_sheet_induced_velocity(detail::dptr(pos), detail::dptr(gamma), (int64_t)gamma.num(),
                                            (int64_t)gamma.rows(), (int64_t)gamma.cols(),
                                            reinterpret_cast<const double*>(xs.data()), (int64_t)xs.size(),
                                            reinterpret_cast<double*>(out.data()), precision),
                "InducedVelocity");
  return out;
}

// Morphing (src/morphing.h:25-108) with each motion a closed-form sinusoid
// (the reference takes std::function objects; the device needs the form).
class Morphing {
 public:
  Morphing() { k_ = uvlm_kinematics{}; }
  void set_alpha(double a) { k_.alpha = a; }
  void set_plug(double amp, double omega, double phase = 0) {
    k_.plug_amp = amp;
    k_.plug_omega = omega;
    k_.plug_phase = phase;
  }
  void set_flap(double amp, double omega, double phase = 0) {
    k_.flap_amp = amp;
    k_.flap_omega = omega;
    k_.flap_phase = phase;
  }
  void set_twist(double amp, double omega, double phase = 0, double span_slope = 0) {
    k_.twist_amp = amp;
    k_.twist_omega = omega;
    k_.twist_phase = phase;
    k_.twist_span_slope = span_slope;
  }
  void set_bend(double cx, double cy, double omega, double phase = 0) {
    k_.bend_cx = cx;
    k_.bend_cy = cy;
    k_.bend_omega = omega;
    k_.bend_phase = phase;
  }
  void set_origin(const Vector3& o) {
    const double* p = reinterpret_cast<const double*>(&o);
    for (int d = 0; d < 3; ++d) k_.origin[d] = p[d];
  }
  const uvlm_kinematics& kinematics() const { return k_; }
  // Morphing::Perfome / Velocity (src/morphing.cpp:23-52) of one reference
  // point, evaluated by the library's kinematics kernel.
  void Perfome(Vector3* x, const Vector3& x0, double t) const {
    detail::check(uvlm_kinematics_perfome(&k_, reinterpret_cast<const double*>(&x0), 1, t,
                                          reinterpret_cast<double*>(x)),
                  "Morphing::Perfome");
  }
  void Velocity(Vector3* v, const Vector3& x0, double t) const {
    detail::check(uvlm_kinematics_velocity(&k_, reinterpret_cast<const double*>(&x0), 1, t,
                                           reinterpret_cast<double*>(v)),
                  "Morphing::Velocity");
  }

 private:
  uvlm_kinematics k_;
};

namespace advect {

// advect::Advection (src/advect.h:48-59).  Advect may be called with
// next == &wake_pos (the simulator advects in place).
class Advection {
 public:
  explicit Advection(const char* name, int precision = UVLM_PRECISION_FP64) {
    uvlm_advection* h = nullptr;
    detail::check(uvlm_advection_create(name, precision, &h), "AdvectFactory");
    h_.reset(h);
  }
  virtual ~Advection() = default;
  virtual void Advect(MultipleSheet<Vector3>* next, const MultipleSheet<Vector3>& wing_pos,
                      const MultipleSheet<double>& wing_gamma, const MultipleSheet<Vector3>& wake_pos,
                      const MultipleSheet<double>& wake_gamma, const Vector3& forward_flight,
                      const double dt) const {
    if (next != &wake_pos) next->resize(wake_pos);  // aliasing next == &wake_pos is allowed
    detail::check(uvlm_advection_advect(h_.get(), detail::dptr_mut(*next), detail::dptr(wing_pos),
                                        detail::dptr(wing_gamma), (int64_t)wing_gamma.num(),
                                        (int64_t)wing_gamma.rows(), (int64_t)wing_gamma.cols(),
                                        detail::dptr(wake_pos),
                                        detail::dptr(wake_gamma), (int64_t)wake_gamma.rows(),
                                        reinterpret_cast<const double*>(&forward_flight), dt),
                  "Advection::Advect");
  }

 private:
  struct Del {
    void operator()(uvlm_advection* p) const { uvlm_advection_destroy(p); }
  };
  std::unique_ptr<uvlm_advection, Del> h_;
};

class Euler : public Advection {
 public:
  Euler() : Advection("euler") {}
};
class RungeKutta2 : public Advection {
 public:
  RungeKutta2() : Advection("RK2") {}
};
class RungeKutta4 : public Advection {
 public:
  RungeKutta4() : Advection("RK4") {}
};
class AdamsBashforth2 : public Advection {
 public:
  AdamsBashforth2() : Advection("AB2") {}
};

// AdvectFactory (src/advect_factory.cpp:43-60): "euler", "RK2", "RK4", "AB2".
inline std::unique_ptr<Advection> AdvectFactory(const std::string& name) {
  return std::unique_ptr<Advection>(new Advection(name.c_str()));
}

}  // namespace advect

// ---------------------------------------------------------------- proto
// The subset of the generated proto::Point / proto::Wing accessors that the
// wing generators and the legacy code use (proto/uvlm.proto:6-30).
namespace proto {
struct Point {
  double x_ = 0, y_ = 0, z_ = 0;
  double x() const { return x_; }
  double y() const { return y_; }
  double z() const { return z_; }
  void set_x(double v) { x_ = v; }
  void set_y(double v) { y_ = v; }
  void set_z(double v) { z_ = v; }
};
class Wing {
 public:
  std::uint64_t rows() const { return rows_; }
  std::uint64_t cols() const { return cols_; }
  void set_rows(std::uint64_t v) { rows_ = v; }
  void set_cols(std::uint64_t v) { cols_ = v; }
  double chord() const { return chord_; }
  double span() const { return span_; }
  void set_chord(double v) { chord_ = v; }
  void set_span(double v) { span_ = v; }
  Point* add_points() {
    points_.emplace_back();
    return &points_.back();
  }
  const std::vector<Point>& points() const { return points_; }
  int points_size() const { return (int)points_.size(); }
  const Point& points(int i) const { return points_[(std::size_t)i]; }
  Point* mutable_points(int i) { return &points_[(std::size_t)i]; }
  bool has_origin() const { return has_origin_; }
  const Point& origin() const { return origin_; }
  Point* mutable_origin() {
    has_origin_ = true;
    return &origin_;
  }
  void CopyFrom(const Wing& w) { *this = w; }
  void Clear() { *this = Wing(); }

 private:
  std::uint64_t rows_ = 0, cols_ = 0;
  double chord_ = 0, span_ = 0;
  std::vector<Point> points_;
  Point origin_;
  bool has_origin_ = false;
};
}  // namespace proto

namespace wing {

// WingGenerator (src/wing/wing_generator.h:12-32): fills a half wing's
// lattice; SimpleSimulator::AddWing takes ownership of any generator.
class WingGenerator {
 public:
  WingGenerator() = default;
  virtual ~WingGenerator() = default;
  virtual void Generate(proto::Wing* wing, const double chord, const double span, const std::size_t rows,
                        const std::size_t cols) const {
    wing->Clear();
    wing->set_chord(chord);
    wing->set_span(span);
    wing->set_cols(cols);
    wing->set_rows(rows);
  }
  void operator()(proto::Wing* wing, const double chord, const double span, const std::size_t rows,
                  const std::size_t cols) const {
    this->Generate(wing, chord, span, rows, cols);
  }
};

// linspace (src/util.h:36-43).
inline std::vector<double> linspace(double a, double b, std::size_t N) {
  const double dx = (b - a) / (N - 1);
  std::vector<double> res;
  for (std::size_t i = 0; i < N; i++) res.push_back(a + i * dx);
  return res;
}

// TransformChebyshev (src/wing/rect.h:16-25).
inline void TransformChebyshev(std::vector<double>* res, std::size_t N, double xmin, double xmax) {
  const auto theta = linspace(-M_PI_2, 0, N);
  res->clear();
  for (double t : theta) res->push_back(xmin + (xmax - xmin) * std::cos(t));
  res->front() = xmin;
  res->back() = xmax;
}

// RectGenerator (src/wing/rect.{h,cpp}): flat lattice, linspace or Chebyshev
// spacing (the reference's --chebyshev_chord / --chebyshev_span flags are the
// two members).  AddWing builds a plain RectGenerator wing inside the library.
class RectGenerator : public WingGenerator {
 public:
  RectGenerator(bool cheb_chord = false, bool cheb_span = false)
      : chebyshev_chord(cheb_chord), chebyshev_span(cheb_span) {}
  void Generate(proto::Wing* wing, const double chord, const double span, const std::size_t rows,
                const std::size_t cols) const override {
    WingGenerator::Generate(wing, chord, span, rows, cols);
    std::vector<double> xs, ys;
    if (chebyshev_chord)
      TransformChebyshev(&xs, rows + 1, 0, chord);
    else
      xs = linspace(0, chord, rows + 1);
    if (chebyshev_span)
      TransformChebyshev(&ys, cols + 1, 0, span);
    else
      ys = linspace(0, span, cols + 1);
    for (const double x : xs)
      for (const double y : ys) {
        auto* p = wing->add_points();
        p->set_x(x);
        p->set_y(y);
        p->set_z(0);
      }
  }
  bool chebyshev_chord = false, chebyshev_span = false;
};

// NACA4digit / NACA4digitGenerator (src/wing/naca4digit.{h,cpp}): mean camber
// line of a 4-digit section (first digit: camber in %, second: its position
// in tenths of the chord) on the rectangular lattice.
inline double NACA4digit(double x, double c, int xx) {
  const int first = xx / 10, second = xx % 10;
  const double m = first / 100.0, p = second / 10.0;
  double res = 0;
  if (0 <= x && x <= p * c)
    res = m * x / p / p * (2 * p - x / c);
  else if (p * c <= x && x <= c)
    res = m * (c - x) / (1 - p) / (1 - p) * (1 + x / c - 2 * p);
  return res;
}
class NACA4digitGenerator : public RectGenerator {
 public:
  explicit NACA4digitGenerator(int digit) : RectGenerator(), digit_(digit) {}
  void Generate(proto::Wing* wing, const double chord, const double span, const std::size_t rows,
                const std::size_t cols) const override {
    RectGenerator::Generate(wing, chord, span, rows, cols);
    for (int i = 0; i < wing->points_size(); i++) {
      auto* p = wing->mutable_points(i);
      p->set_z(NACA4digit(p->x(), chord, digit_));
    }
  }
  void set_verbose(bool) {}

 private:
  int digit_;
};

// NACA00XX / NACA00XXGenerator (src/wing/naca00XX.{h,cpp}): half thickness of
// a symmetric 4-digit section on the rectangular lattice.
inline double NACA00XX(double x, double c, int xx) {
  const double t = xx * 0.01;
  const double z = x / c;
  return 5 * t * c *
         (0.2969 * std::sqrt(z) + (-0.1260) * (z) + (-0.3516) * z * z + 0.2843 * z * z * z +
          (-0.1015) * z * z * z * z);
}
class NACA00XXGenerator : public RectGenerator {
 public:
  explicit NACA00XXGenerator(int digit) : RectGenerator(), digit_(digit) {}
  void Generate(proto::Wing* wing, const double chord, const double span, const std::size_t rows,
                const std::size_t cols) const override {
    RectGenerator::Generate(wing, chord, span, rows, cols);
    for (int i = 0; i < wing->points_size(); i++) {
      auto* p = wing->mutable_points(i);
      p->set_z(NACA00XX(p->x(), chord, digit_));
    }
  }
  void set_verbose(bool) {}

 private:
  int digit_;
};

// WholeWing (src/wing/wing.cpp:12-52): per node row, the mirror image (y ->
// -y) of the half row in reverse order, then the half row without its first
// point; finally + the half's origin.
inline void WholeWing(proto::Wing* wing, const proto::Wing& half) {
  wing->Clear();
  wing->set_cols(half.cols() * 2);
  wing->set_rows(half.rows());
  *wing->mutable_origin() = half.origin();
  wing->set_chord(half.chord());
  wing->set_span(half.span());
  const std::size_t COLS = half.cols() + 1;
  const std::size_t ROWS = half.points().size() / COLS;
  const proto::Point& o = half.origin();
  auto put = [&](double x, double y, double z) {
    auto* p = wing->add_points();
    p->set_x(x + o.x());
    p->set_y(y + o.y());
    p->set_z(z + o.z());
  };
  for (std::size_t i = 0; i < ROWS; ++i) {
    for (std::size_t q = COLS; q-- > 0;) {
      const proto::Point& p = half.points()[i * COLS + q];
      put(p.x(), p.y() * -1, p.z());
    }
    for (std::size_t q = 1; q < COLS; ++q) {
      const proto::Point& p = half.points()[i * COLS + q];
      put(p.x(), p.y(), p.z());
    }
  }
}

}  // namespace wing

namespace simulator {

// SimpleSimulator (src/simulator/simple_simulator.h:33-108) with the whole
// MainLoop on the GPU.  The extra Config selects the B200 arithmetic.
class SimpleSimulator {
 public:
  static const std::size_t STEP_MIN = 0;

  explicit SimpleSimulator(const uvlm_config* cfg = nullptr) {
    uvlm_config c;
    uvlm_config_default(&c);
    if (cfg) c = *cfg;
    uvlm_ctx* h = nullptr;
    detail::check(uvlm_create(&c, &h), "SimpleSimulator");
    h_.reset(h);
  }

  // AddWing (simple_simulator.cpp:126-140) with any wing::WingGenerator, as
  // the reference's (it takes ownership of the generator): BuildWing's
  // lattice (:155-166) is the generator's half wing (chord, span/2, rows,
  // cols/2) through WholeWing, moved to `origin` by the library.
  void AddWing(wing::WingGenerator* generator, const Morphing& morphing, const double chord, const double span,
               const std::size_t rows, const std::size_t cols, const Vector3& origin) {
    std::unique_ptr<wing::WingGenerator> gen(generator);
    if (!gen) detail::check(UVLM_ERR_INVALID, "AddWing", "NULL wing generator");
    if (cols & 1) detail::check(UVLM_ERR_INVALID, "AddWing", "columns must be even.");
    if (auto* rect = dynamic_cast<wing::RectGenerator*>(gen.get()); rect && typeid(*gen) == typeid(wing::RectGenerator)) {
      AddWing(*rect, morphing, chord, span, rows, cols, origin);
      return;
    }
    proto::Wing half, whole;
    gen->Generate(&half, chord, span / 2, rows, cols / 2);
    wing::WholeWing(&whole, half);
    std::vector<double> nodes;
    nodes.reserve(whole.points().size() * 3);
    for (const auto& p : whole.points()) {
      nodes.push_back(p.x());
      nodes.push_back(p.y());
      nodes.push_back(p.z());
    }
    const double* o = reinterpret_cast<const double*>(&origin);
    num_ += 1;
    detail::check(uvlm_add_wing_nodes(h_.get(), (int64_t)rows, (int64_t)cols, nodes.data(), chord, span, o,
                                      &morphing.kinematics()),
                  "AddWing", uvlm_last_error(h_.get()));
  }
  void AddWing(const wing::RectGenerator& gen, const Morphing& morphing, const double chord, const double span,
               const std::size_t rows, const std::size_t cols, const Vector3& origin) {
    uvlm_wing_desc w{};
    w.chord = chord;
    w.span = span;
    w.rows = (int64_t)rows;
    w.cols = (int64_t)cols;
    const double* o = reinterpret_cast<const double*>(&origin);
    for (int d = 0; d < 3; ++d) w.origin[d] = o[d];
    w.chebyshev_chord = gen.chebyshev_chord;
    w.chebyshev_span = gen.chebyshev_span;
    num_ += 1;
    detail::check(uvlm_add_wing(h_.get(), &w, &morphing.kinematics()), "AddWing", uvlm_last_error(h_.get()));
  }
  void set_forward_flight(const Vector3& v) {
    detail::check(uvlm_set_forward_flight(h_.get(), reinterpret_cast<const double*>(&v)), "set_forward_flight");
  }
  void set_advection(const std::string& name) {
    detail::check(uvlm_set_advection(h_.get(), name.c_str()), "set_advection", uvlm_last_error(h_.get()));
  }
  // set_sheet_path / set_result_path (simple_simulator.cpp:53-66): one
  // AllVortexSheets / Snapshot2 record per step, length-prefixed protobuf.
  void set_sheet_path(const std::string& path) {
    sheet_path_ = path;
    detail::check(uvlm_set_output_paths(h_.get(), sheet_path_.c_str(), result_path_.c_str()), "set_sheet_path",
                  uvlm_last_error(h_.get()));
  }
  void set_result_path(const std::string& path) {
    result_path_ = path;
    detail::check(uvlm_set_output_paths(h_.get(), sheet_path_.c_str(), result_path_.c_str()), "set_result_path",
                  uvlm_last_error(h_.get()));
  }
  void FlushOutput() { detail::check(uvlm_flush_output(h_.get()), "FlushOutput", uvlm_last_error(h_.get())); }

  // Run (simple_simulator.cpp:288-313): MainLoop(step, dt) for step =
  // 0..steps.  Returns the load rows t, CD_0, CL_0, CD_1, CL_1, ...
  std::vector<std::vector<double>> Run(const std::size_t steps, const double dt) {
    detail::check(uvlm_begin(h_.get()), "Run", uvlm_last_error(h_.get()));
    std::vector<std::vector<double>> rows;
    for (std::size_t s = 0; s <= steps; ++s) rows.push_back(Step(s, dt));
    return rows;
  }
  // One MainLoop after Begin (for callers that drive the loop themselves).
  void Begin() { detail::check(uvlm_begin(h_.get()), "Begin", uvlm_last_error(h_.get())); }
  std::vector<double> Step(const std::size_t step, const double dt) {
    std::vector<double> row(1 + 2 * num_);
    detail::check(uvlm_step(h_.get(), (int64_t)step, dt, row.data()), "MainLoop", uvlm_last_error(h_.get()));
    return row;
  }
  // The same MainLoop in its six stages (uvlm_stage_*), in this order.
  void StageKinematics(const std::size_t step, const double dt) {
    detail::check(uvlm_stage_kinematics(h_.get(), (int64_t)step, dt), "StageKinematics", uvlm_last_error(h_.get()));
  }
  void StageAssemble() { detail::check(uvlm_stage_assemble(h_.get()), "StageAssemble", uvlm_last_error(h_.get())); }
  void StageRhs() { detail::check(uvlm_stage_rhs(h_.get()), "StageRhs", uvlm_last_error(h_.get())); }
  void StageSolve() { detail::check(uvlm_stage_solve(h_.get()), "StageSolve", uvlm_last_error(h_.get())); }
  void StageLoads() { detail::check(uvlm_stage_loads(h_.get()), "StageLoads", uvlm_last_error(h_.get())); }
  std::vector<double> StageAdvect() {
    std::vector<double> row(1 + 2 * num_);
    detail::check(uvlm_stage_advect(h_.get(), row.data()), "StageAdvect", uvlm_last_error(h_.get()));
    return row;
  }
  // SimpleSimulator::Velocity (simple_simulator.h:98-100): -ff + U_bound + U_wake
  // at x for the current state.
  Vector3 Velocity(const Vector3& x) const {
    Vector3 out{};
    detail::check(uvlm_velocity_at(h_.get(), reinterpret_cast<const double*>(&x), 1, 1,
                                   reinterpret_cast<double*>(&out)),
                  "Velocity", uvlm_last_error(h_.get()));
    return out;
  }
  // State of the last step in the reference's member layout.
  void GetState(MultipleSheet<Vector3>* wing_pos, MultipleSheet<double>* wing_gamma, MultipleSheet<Vector3>* wake_pos,
                MultipleSheet<double>* wake_gamma) const {
    int64_t num, rows, cols, wr, wn;
    detail::check(uvlm_get_sizes(h_.get(), &num, &rows, &cols, &wr, &wn), "GetState");
    if (wing_pos) wing_pos->resize(num, rows + 1, cols + 1);
    if (wing_gamma) wing_gamma->resize(num, rows, cols);
    if (wake_pos) wake_pos->resize(num, wn, cols + 1);
    if (wake_gamma) wake_gamma->resize(num, wr, cols);
    detail::check(uvlm_get_state(h_.get(), wing_pos ? detail::dptr_mut(*wing_pos) : nullptr, nullptr,
                                 wake_pos ? detail::dptr_mut(*wake_pos) : nullptr,
                                 wing_gamma ? detail::dptr_mut(*wing_gamma) : nullptr, nullptr,
                                 wake_gamma ? detail::dptr_mut(*wake_gamma) : nullptr),
                  "GetState");
  }

 private:
  struct Del {
    void operator()(uvlm_ctx* p) const { uvlm_destroy(p); }
  };
  std::unique_ptr<uvlm_ctx, Del> h_;
  std::size_t num_ = 0;
  std::string sheet_path_, result_path_;
};

}  // namespace simulator
}  // namespace UVLM

#include "uvlm_b200_legacy.hpp"
