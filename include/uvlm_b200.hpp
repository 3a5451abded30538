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
//   UVLM::wing::RectGenerator                        src/wing/rect.h:10-30
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
#include <cstddef>
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

namespace wing {
// RectGenerator (src/wing/rect.h:10-30); Chebyshev spacing as
// TransformChebyshev (src/wing/rect.h:16-25).
struct RectGenerator {
  bool chebyshev_chord = false, chebyshev_span = false;
};
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
