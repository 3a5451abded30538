// uvlm_b200_legacy.hpp -- the reference's legacy (AoS) C++ API on the
// uvlm_b200 C-ABI; included by uvlm_b200.hpp.
//
// Mirrored surfaces (namespace UVLM):
//   VortexRing                                   src/vortex.h:25-150
//   VortexContainer, CountTotalSize,
//     CopyContainers, GetWake                    src/vortex_container.h:22-190
//   InducedVelocity / ChordwiseInducedVelocity
//     over ring iterators, ConnectTrailingEdge,
//     Advect, AdvectParallel                     src/shed.h:14-46, src/shed.inl:8-86
//   SolveLinearProblem (ring iterators and
//     containers), internal::CalcMorphingVelocityOnWing
//                                                src/linear.h:95-125, src/linear.inl:78-157
//   UVLMVortexRing (InitWing, PlaneSymmetry,
//     TrailingEdgeIterators, velocity queries)   src/uvlm_vortex_ring.{h,cpp}
//   calc_load::AerodynamicLoad, CalcUm,
//     CalcLoadKatzPlotkin, CalcLoadJoukowski     src/calc_load/{functions,katz_plotkin,joukowski}.h
//   internal::TransformRow, WingBuilder          src/wing_builder.{h,cpp}
//   simulator::{InitSimulator, AddWing, SetInlet,
//     SetOutputPath, SetOutputLoadPath, Start}   src/simulator/simulator.{h,cpp}
// Every N-body, solve and load evaluation is one C-ABI call (CUDA kernels,
// FP64); ring geometry accessors (Normal, Area, ...) are host arithmetic on
// the ring's four nodes.  Advect and AdvectParallel both take every velocity
// before any node moves, which is what every reference caller relies on
// (the wake rings are never among the sources).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <functional>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace UVLM {

struct VecX {
  std::vector<double> v;
  VecX() = default;
  explicit VecX(std::size_t n) : v(n) {}
  double& operator()(std::size_t i) { return v[i]; }
  double operator()(std::size_t i) const { return v[i]; }
  double& operator[](std::size_t i) { return v[i]; }
  double operator[](std::size_t i) const { return v[i]; }
  std::size_t size() const { return v.size(); }
  double* data() { return v.data(); }
  const double* data() const { return v.data(); }
};

}  // namespace UVLM

#ifndef UVLM_B200_VECTORX
#define UVLM_B200_VECTORX ::UVLM::VecX
#endif

namespace UVLM {

using VectorX = UVLM_B200_VECTORX;

namespace detail {
inline const double* c3(const Vector3& v) { return reinterpret_cast<const double*>(&v); }
inline Vector3 v3(double x, double y, double z) { return Vector3(x, y, z); }
inline Vector3 sub(const Vector3& a, const Vector3& b) {
  return v3(c3(a)[0] - c3(b)[0], c3(a)[1] - c3(b)[1], c3(a)[2] - c3(b)[2]);
}
inline Vector3 add(const Vector3& a, const Vector3& b) {
  return v3(c3(a)[0] + c3(b)[0], c3(a)[1] + c3(b)[1], c3(a)[2] + c3(b)[2]);
}
inline Vector3 scale(const Vector3& a, double s) { return v3(c3(a)[0] * s, c3(a)[1] * s, c3(a)[2] * s); }
inline double dot(const Vector3& a, const Vector3& b) {
  return c3(a)[0] * c3(b)[0] + c3(a)[1] * c3(b)[1] + c3(a)[2] * c3(b)[2];
}
inline Vector3 cross(const Vector3& a, const Vector3& b) {
  const double* p = c3(a);
  const double* q = c3(b);
  return v3(p[1] * q[2] - p[2] * q[1], p[2] * q[0] - p[0] * q[2], p[0] * q[1] - p[1] * q[0]);
}
inline double norm(const Vector3& a) { return std::sqrt(dot(a, a)); }
inline Vector3 normalized(const Vector3& a) {
  const double n = norm(a);
  return n > 0 ? scale(a, 1.0 / n) : a;
}
}  // namespace detail

// ------------------------------------------------------------- VortexRing
class VortexRing {
 public:
  static const std::size_t DEFAULT_NODE_SIZE = 4;

  VortexRing() = default;

  // Biot-Savart law of the ring's four segments at pos (src/vortex.cpp:41-65).
  void BiotSavartLaw(Vector3* result, const Vector3& pos, double gamma) const { eval(result, pos, gamma, 0); }
  void ChordwiseBiotSavartLaw(Vector3* result, const Vector3& pos, double gamma) const {
    eval(result, pos, gamma, 1);
  }
  void BiotSavartLaw(Vector3* result, const Vector3& pos) const { BiotSavartLaw(result, pos, gamma_); }
  void ChordwiseBiotSavartLaw(Vector3* result, const Vector3& pos) const {
    ChordwiseBiotSavartLaw(result, pos, gamma_);
  }

  VortexRing& PushNode(const Vector3& pos) {
    nodes_.push_back(pos);
    return *this;
  }
  VortexRing& PushNode(double x, double y, double z) { return PushNode(Vector3(x, y, z)); }
  void SaveReferenceNode() { nodes0_ = nodes_; }

  // src/vortex.cpp:82-143
  Vector3 Normal() const {
    return detail::normalized(
        detail::cross(detail::sub(nodes_[1], nodes_[3]), detail::sub(nodes_[2], nodes_[0])));
  }
  Vector3 Tangent() const {
    return detail::normalized(detail::add(detail::sub(nodes_[1], nodes_[3]), detail::sub(nodes_[2], nodes_[0])));
  }
  Vector3 Tangent2() const { return detail::cross(Normal(), Tangent()); }
  Vector3 Centroid() const { return centroid(nodes_); }
  Vector3 ReferenceCentroid() const { return centroid(nodes0_); }
  Vector3 TanVecChord() const { return detail::normalized(detail::sub(nodes_[1], nodes_[0])); }
  Vector3 TanVecSpan() const { return detail::normalized(detail::sub(nodes_[3], nodes_[0])); }
  double AngleOfAttack(const Vector3& Q) const { return std::atan2(detail::dot(Q, Normal()), detail::dot(Q, Tangent())); }
  double CalcC() const { return detail::norm(detail::sub(nodes_[0], nodes_[1])); }
  double CalcB() const { return detail::norm(detail::sub(nodes_[0], nodes_[3])); }
  double Area() const {
    using namespace detail;
    return (norm(cross(sub(nodes_[1], nodes_[0]), sub(nodes_[3], nodes_[0]))) +
            norm(cross(sub(nodes_[3], nodes_[2]), sub(nodes_[1], nodes_[2])))) /
           2;
  }
  Vector3 Impulse() const { return detail::scale(Normal(), gamma_ * Area() * (-1)); }

  double gamma() const { return gamma_; }
  void set_gamma(double gamma) { gamma_ = gamma; }
  std::vector<Vector3>& nodes() { return nodes_; }
  const std::vector<Vector3>& nodes() const { return nodes_; }
  const std::vector<Vector3>& nodes0() const { return nodes0_; }
  void Clear() { nodes_.clear(); }

  // ForEachSegment (src/vortex.h:132-150): start = nodes[i+1], end = nodes[i].
  void ForEachSegment(std::function<void(const Vector3&, const Vector3&)> func) const {
    for (std::size_t i = 0; i < nodes_.size(); i++) func(nodes_[(i + 1) % nodes_.size()], nodes_[i]);
  }
  void ForEachSegment(
      std::function<void(const Vector3&, const Vector3&, const Vector3&, const Vector3&)> func) const {
    for (std::size_t i = 0; i < nodes_.size(); i++)
      func(nodes_[(i + 1) % nodes_.size()], nodes_[i], nodes0_[(i + 1) % nodes_.size()], nodes0_[i]);
  }

 private:
  static Vector3 centroid(const std::vector<Vector3>& n) {
    return detail::scale(detail::add(detail::add(n[0], n[1]), detail::add(n[2], n[3])), 0.25);
  }
  void eval(Vector3* result, const Vector3& pos, double gamma, int chordwise) const;

  double gamma_ = 0;
  std::vector<Vector3> nodes_, nodes0_;
};

namespace detail {
// AoS rings (12 doubles each) and circulations of a ring range.
template <class It>
inline void pack_rings(It first, It last, std::vector<double>* rings, std::vector<double>* gammas,
                       bool reference_nodes = false) {
  rings->clear();
  gammas->clear();
  for (; first != last; ++first) {
    const auto& n = reference_nodes ? first->nodes0() : first->nodes();
    if (n.size() != 4) throw Error(UVLM_ERR_INVALID, "a VortexRing needs 4 nodes");
    for (int q = 0; q < 4; ++q)
      for (int d = 0; d < 3; ++d) rings->push_back(c3(n[q])[d]);
    gammas->push_back(first->gamma());
  }
}
}  // namespace detail

inline void VortexRing::eval(Vector3* result, const Vector3& pos, double gamma, int chordwise) const {
  std::vector<double> r, g;
  const VortexRing* self = this;
  detail::pack_rings(self, self + 1, &r, &g);
  g[0] = gamma;
  detail::check(uvlm_rings_induced_velocity(r.data(), g.data(), 1, detail::c3(pos), 1, chordwise,
                                            reinterpret_cast<double*>(result)),
                "VortexRing::BiotSavartLaw");
}

// -------------------------------------------------------- VortexContainer
class VortexContainer {
  typedef std::vector<VortexRing> container_t;
  typedef std::shared_ptr<container_t> vortices_ptr_t;

 public:
  VortexContainer() = default;
  VortexContainer(const vortices_ptr_t& vortices, std::size_t rows, std::size_t cols, std::size_t id, double chord,
                  double span)
      : vortices_(vortices), rows_(rows), cols_(cols), id_(id), chord_(chord), span_(span) {}

  std::size_t Offset() const { return id_ * rows_ * cols_; }
  std::size_t Index(std::size_t i) const { return Offset() + i; }
  std::size_t Index(std::size_t i, std::size_t j) const { return Offset() + j + i * cols_; }
  VortexRing& operator[](std::size_t i) { return (*vortices_)[Index(i)]; }
  const VortexRing& operator[](std::size_t i) const { return (*vortices_)[Index(i)]; }
  VortexRing& at(std::size_t i, std::size_t j) { return (*vortices_)[Index(i, j)]; }
  const VortexRing& at(std::size_t i, std::size_t j) const { return (*vortices_)[Index(i, j)]; }
  bool ShapeEquals(const VortexContainer& c) const { return rows_ == c.rows() && cols_ == c.cols() && id_ == c.id(); }
  void alloc(std::size_t sz) {
    if (vortices_->size() < sz) vortices_->resize(sz);
  }
  // vortex_container.h:87-96
  double DeltaGamma(std::size_t i, std::size_t j) const {
    return at(i, j).gamma() - (i == 0 ? 0.0 : at(i - 1, j).gamma());
  }
  Vector3 Grad(std::size_t i, std::size_t j) const {
    return detail::scale(at(i, j).Tangent(), DeltaGamma(i, j) / at(i, j).CalcC());
  }
  const vortices_ptr_t& vortices() const { return vortices_; }
  std::size_t cols() const { return cols_; }
  std::size_t rows() const { return rows_; }
  std::size_t id() const { return id_; }
  double chord() const { return chord_; }
  double span() const { return span_; }
  void set_vortices(const vortices_ptr_t& vortices, std::size_t r, std::size_t c, std::size_t i, double chord,
                    double span) {
    vortices_ = vortices;
    rows_ = r;
    cols_ = c;
    id_ = i;
    chord_ = chord;
    span_ = span;
  }
  std::size_t size() const { return cols_ * rows_; }
  container_t::iterator begin() { return vortices_->begin() + Index(0); }
  container_t::const_iterator begin() const { return vortices_->cbegin() + Index(0); }
  container_t::iterator end() { return vortices_->begin() + Index(rows_ * cols_); }
  container_t::const_iterator end() const { return vortices_->cbegin() + Index(rows_ * cols_); }
  container_t::iterator edge_begin() { return vortices_->begin() + Index(rows_ - 1, 0); }
  container_t::iterator edge_end() { return end(); }
  container_t::const_iterator edge_begin() const { return vortices_->cbegin() + Index(rows_ - 1, 0); }
  container_t::const_iterator edge_end() const { return end(); }
  container_t::const_iterator cbegin() const { return vortices_->cbegin() + Index(0); }
  container_t::const_iterator cend() const { return vortices_->cbegin() + Index(rows_ * cols_); }

 private:
  vortices_ptr_t vortices_;
  std::size_t rows_ = 0, cols_ = 0, id_ = 0;
  double chord_ = 0, span_ = 0;
};

template <class InputIterator>
std::size_t CountTotalSize(InputIterator first, InputIterator last) {
  std::size_t res = 0;
  for (; first != last; ++first) res += first->size();
  return res;
}

// CopyContainers (vortex_container.h:153-170): the containers' rings are
// copied into a new pool shared by the copies.
template <class InputIterator, class OutputIterator>
void CopyContainers(InputIterator first, InputIterator last, OutputIterator result) {
  auto vortices = first->vortices();
  const auto total = CountTotalSize(first, last);
  auto copied = std::make_shared<std::vector<VortexRing>>(vortices->begin(), vortices->begin() + total);
  for (; first != last; ++first, ++result)
    *result = VortexContainer(copied, first->rows(), first->cols(), first->id(), first->chord(), first->span());
}

template <class Range>
auto GetWake(const Range& containers) {
  const auto off = CountTotalSize(std::begin(containers), std::end(containers));
  auto vortices = std::begin(containers)->vortices();
  return std::make_pair(vortices->begin() + off, vortices->end());
}

// -------------------------------------------------------------- shed.inl
template <class InputIterator>
void InducedVelocity(Vector3* result, const Vector3& pos, InputIterator first, InputIterator last) {
  std::vector<double> r, g;
  detail::pack_rings(first, last, &r, &g);
  detail::check(uvlm_rings_induced_velocity(r.data(), g.data(), (int64_t)g.size(), detail::c3(pos), 1, 0,
                                            reinterpret_cast<double*>(result)),
                "InducedVelocity");
}

template <class InputIterator>
void ChordwiseInducedVelocity(Vector3* result, const Vector3& pos, InputIterator first, InputIterator last) {
  std::vector<double> r, g;
  detail::pack_rings(first, last, &r, &g);
  detail::check(uvlm_rings_induced_velocity(r.data(), g.data(), (int64_t)g.size(), detail::c3(pos), 1, 1,
                                            reinterpret_cast<double*>(result)),
                "ChordwiseInducedVelocity");
}

template <class InputIterator, class OutputIterator>
void ConnectTrailingEdge(InputIterator edge_first, InputIterator edge_last, OutputIterator wake) {
  for (auto edge = edge_first; edge != edge_last; ++edge, ++wake) {
    wake->nodes()[0] = edge->nodes()[1];
    wake->nodes()[3] = edge->nodes()[2];
  }
}

template <class InputIterator, class OutputIterator>
void AdvectParallel(InputIterator vortex_first, InputIterator vortex_last, OutputIterator wake_first,
                    OutputIterator wake_last, const Vector3& freestream, const double dt) {
  std::vector<double> vr, vg, wr, wg;
  detail::pack_rings(vortex_first, vortex_last, &vr, &vg);
  detail::pack_rings(wake_first, wake_last, &wr, &wg);
  detail::check(uvlm_rings_advect(vr.data(), vg.data(), (int64_t)vg.size(), wr.data(), (int64_t)wg.size(),
                                  detail::c3(freestream), dt),
                "AdvectParallel");
  std::size_t k = 0;
  for (auto w = wake_first; w != wake_last; ++w, ++k)
    for (int q = 0; q < 4; ++q) w->nodes()[q] = Vector3(wr[12 * k + 3 * q], wr[12 * k + 3 * q + 1], wr[12 * k + 3 * q + 2]);
}

template <class InputIterator, class OutputIterator>
void Advect(InputIterator vortex_first, InputIterator vortex_last, OutputIterator wake_first,
            OutputIterator wake_last, const Vector3& freestream, const double dt) {
  AdvectParallel(vortex_first, vortex_last, wake_first, wake_last, freestream, dt);
}

// --------------------------------------------------------- linear.inl
namespace internal {
// CalcMorphingVelocityOnWing (src/linear.inl:78-90): Vls(reference centroid) . normal.
template <class InputIterator, class OutputIterator>
OutputIterator CalcMorphingVelocityOnWing(InputIterator panel_first, InputIterator panel_last,
                                          const Morphing& morphing, double t, OutputIterator result) {
  std::vector<Vector3> c, n;
  for (auto p = panel_first; p != panel_last; ++p) {
    c.push_back(p->ReferenceCentroid());
    n.push_back(p->Normal());
  }
  std::vector<Vector3> v(c.size());
  if (!c.empty())
    detail::check(uvlm_kinematics_velocity(&morphing.kinematics(), reinterpret_cast<const double*>(c.data()),
                                           (int64_t)c.size(), t, reinterpret_cast<double*>(v.data())),
                  "CalcMorphingVelocityOnWing");
  for (std::size_t k = 0; k < c.size(); ++k, ++result) *result = detail::dot(v[k], n[k]);
  return result;
}
}  // namespace internal

// SolveLinearProblem (src/linear.inl:113-130).  drop_wake_term = true keeps
// the reference's behaviour, whose wake RHS term is a discarded statement.
template <class InputIterator1, class InputIterator2>
VectorX SolveLinearProblem(InputIterator1 bound_first, InputIterator1 bound_last, InputIterator2 wake_first,
                           InputIterator2 wake_last, const Vector3 freestream, const Morphing& morphing,
                           const double t, bool drop_wake_term = true) {
  std::vector<double> br, bg, b0, b0g, wr, wg;
  detail::pack_rings(bound_first, bound_last, &br, &bg);
  detail::pack_rings(bound_first, bound_last, &b0, &b0g, true);
  detail::pack_rings(wake_first, wake_last, &wr, &wg);
  VectorX x(bg.size());
  detail::check(uvlm_rings_solve_linear_problem(br.data(), b0.data(), (int64_t)bg.size(), wr.data(), wg.data(),
                                                (int64_t)wg.size(), detail::c3(freestream), &morphing.kinematics(),
                                                t, drop_wake_term ? 1 : 0, x.data()),
                "SolveLinearProblem");
  return x;
}

// SolveLinearProblem(containers, morphings, freestream, t) (src/linear.inl:132-157).
inline VectorX SolveLinearProblem(const std::vector<VortexContainer>& containers,
                                  const std::vector<Morphing>& morphings, const Vector3& freestream, const double t,
                                  bool drop_wake_term = true) {
  if (containers.size() != morphings.size())
    throw Error(UVLM_ERR_INVALID, "containers and morphings have to be same size");
  const auto& vortices = containers.begin()->vortices();
  const std::size_t off = CountTotalSize(containers.begin(), containers.end());
  std::vector<double> br, bg, b0, b0g, wr, wg;
  detail::pack_rings(vortices->cbegin(), vortices->cbegin() + off, &br, &bg);
  detail::pack_rings(vortices->cbegin(), vortices->cbegin() + off, &b0, &b0g, true);
  detail::pack_rings(vortices->cbegin() + off, vortices->cend(), &wr, &wg);
  std::vector<int64_t> sizes;
  std::vector<uvlm_kinematics> kins;
  for (std::size_t c = 0; c < containers.size(); ++c) {
    sizes.push_back((int64_t)containers[c].size());
    kins.push_back(morphings[c].kinematics());
  }
  VectorX x(off);
  detail::check(uvlm_rings_solve_linear_problem_containers(
                    br.data(), b0.data(), sizes.data(), (int32_t)sizes.size(), kins.data(), wr.data(), wg.data(),
                    (int64_t)wg.size(), detail::c3(freestream), t, drop_wake_term ? 1 : 0, x.data()),
                "SolveLinearProblem");
  return x;
}

// ------------------------------------------------------ UVLMVortexRing
// The bound / wake ring sets with their velocity queries
// (src/uvlm_vortex_ring.h:43-130).
class UVLMVortexRing {
 public:
  void InducedVelocity(Vector3* result, const Vector3& pos) const {
    Vector3 a, b;
    InducedVelocityByBound(&a, pos);
    InducedVelocityByWake(&b, pos);
    *result = detail::add(a, b);
  }
  void InducedVelocityByBound(Vector3* result, const Vector3& pos) const {
    ::UVLM::InducedVelocity(result, pos, bound_vortices_.cbegin(), bound_vortices_.cend());
  }
  void InducedVelocityByWake(Vector3* result, const Vector3& pos) const {
    ::UVLM::InducedVelocity(result, pos, wake_vortices_.cbegin(), wake_vortices_.cend());
  }
  void InducedVelocityByChordwiseBound(Vector3* result, const Vector3& pos) const {
    ::UVLM::ChordwiseInducedVelocity(result, pos, bound_vortices_.cbegin(), bound_vortices_.cend());
  }
  template <class InputIterator>
  void AppendWake(InputIterator first, InputIterator last) {
    wake_vortices_.insert(wake_vortices_.end(), first, last);
  }
  std::vector<VortexRing>& bound_vortices() { return bound_vortices_; }
  const std::vector<VortexRing>& bound_vortices() const { return bound_vortices_; }
  std::vector<VortexRing>& wake_vortices() { return wake_vortices_; }
  const std::vector<VortexRing>& wake_vortices() const { return wake_vortices_; }

  // InitWing (src/uvlm_vortex_ring.cpp:37-72): the half-wing lattice pos
  // ((rows + 1) x (cols + 1) points at y >= 0, index j + i (cols + 1)) as
  // rings p(i,j), p(i+1,j), p(i+1,j+1), p(i,j+1); each row of rings is
  // followed by its mirror image in y (PlaneSymmetry); all nodes are shifted
  // by the origin and saved as the reference nodes.
  void InitWing(const std::vector<Vector3>& pos, std::size_t cols) {
    const std::size_t cp = cols + 1;
    cols_ = cols;
    rows_ = pos.size() / cp - 1;
    for (std::size_t i = 0; i < rows_; ++i) {
      for (std::size_t j = 0; j < cols_; ++j) {
        VortexRing v;
        for (std::size_t idx : {j + i * cp, j + (i + 1) * cp, j + 1 + (i + 1) * cp, j + 1 + i * cp})
          v.nodes().push_back(pos[idx]);
        bound_vortices_.push_back(v);
      }
      for (std::size_t j = 0; j < cols_; ++j) {
        bound_vortices_.emplace_back();
        bound_vortices_.back().nodes().resize(4);
      }
    }
    PlaneSymmetry();
    for (auto& v : bound_vortices_)
      for (auto& n : v.nodes()) n = detail::add(n, origin_);
    for (auto& v : bound_vortices_) v.SaveReferenceNode();
  }
  // PlaneSymmetry (src/uvlm_vortex_ring.cpp:81-94): ring (i, cols + j) of a
  // row is the mirror of ring (i, j) in the x-z plane, its nodes reversed.
  void PlaneSymmetry() {
    auto mirror = [](const Vector3& p) { return detail::v3(detail::c3(p)[0], -detail::c3(p)[1], detail::c3(p)[2]); };
    for (std::size_t i = 0; i < rows_; ++i)
      for (std::size_t j = 0; j < cols_; ++j) {
        const std::size_t idx = j + i * 2 * cols_;
        auto& to = bound_vortices_[idx + cols_].nodes();
        const auto& from = bound_vortices_[idx].nodes();
        for (int q = 0; q < 4; ++q) to[q] = mirror(from[3 - q]);
      }
  }
  // TrailingEdgeIterators (src/uvlm_vortex_ring.h:89-94): the last row of
  // bound rings, both halves.
  std::pair<std::vector<VortexRing>::iterator, std::vector<VortexRing>::iterator> TrailingEdgeIterators() {
    return {bound_vortices_.begin() + (rows_ - 1) * 2 * cols_, bound_vortices_.begin() + rows_ * 2 * cols_};
  }
  const Vector3& origin() const { return origin_; }
  void set_origin(const Vector3& pos) { origin_ = pos; }
  std::size_t rows() const { return rows_; }
  std::size_t cols() const { return cols_; }

 private:
  std::vector<VortexRing> bound_vortices_, wake_vortices_;
  std::size_t cols_ = 0, rows_ = 0;
  Vector3 origin_ = detail::v3(0, 0, 0);
};

// ------------------------------------------------------------ calc_load
namespace calc_load {

struct AerodynamicLoad {
  Vector3 F;
  double Pin, Pout;
};

namespace internal {
// CalcUm (src/calc_load/functions.h:23-31): freestream - Vls(x0).
inline Vector3 CalcUm(const Morphing& morphing, const Vector3& x0, const Vector3& freestream, const double t) {
  Vector3 v;
  detail::check(uvlm_kinematics_velocity(&morphing.kinematics(), detail::c3(x0), 1, t,
                                         reinterpret_cast<double*>(&v)),
                "CalcUm");
  return detail::sub(freestream, v);
}
}  // namespace internal

// CalcLoadKatzPlotkin (src/calc_load/katz_plotkin.cpp:16-68); F starts at zero.
inline AerodynamicLoad CalcLoadKatzPlotkin(const VortexContainer& c, const VortexContainer& cp,
                                           const Morphing& morphing, const UVLMVortexRing& rings,
                                           const Vector3& freestream, const double rho, const double t,
                                           const double dt) {
  std::vector<double> r, g, r0, gp, br, bg, wr, wg;
  detail::pack_rings(c.cbegin(), c.cend(), &r, &g);
  detail::pack_rings(cp.cbegin(), cp.cend(), &r0, &gp);
  detail::pack_rings(rings.bound_vortices().cbegin(), rings.bound_vortices().cend(), &br, &bg);
  detail::pack_rings(rings.wake_vortices().cbegin(), rings.wake_vortices().cend(), &wr, &wg);
  double out[5];
  detail::check(uvlm_rings_load_katz_plotkin(r.data(), g.data(), gp.data(), (int64_t)c.rows(), (int64_t)c.cols(),
                                             &morphing.kinematics(), br.data(), bg.data(), (int64_t)bg.size(),
                                             wr.data(), wg.data(), (int64_t)wg.size(), detail::c3(freestream), rho,
                                             t, dt, out),
                "CalcLoadKatzPlotkin");
  return AerodynamicLoad{Vector3(out[0], out[1], out[2]), out[3], out[4]};
}

// CalcLoadJoukowski over a container (src/calc_load/joukowski.h:59-104);
// the induced velocity comes from the container's whole ring pool.
inline AerodynamicLoad CalcLoadJoukowski(const VortexContainer& vb, const VortexContainer& vb_prev,
                                         const Morphing& morphing, const Vector3& freestream, const double rho,
                                         const double t, const double dt) {
  std::vector<double> r, g, r0, g0, rp, gp, pr, pg;
  detail::pack_rings(vb.cbegin(), vb.cend(), &r, &g);
  detail::pack_rings(vb.cbegin(), vb.cend(), &r0, &g0, true);
  detail::pack_rings(vb_prev.cbegin(), vb_prev.cend(), &rp, &gp);
  detail::pack_rings(vb.vortices()->cbegin(), vb.vortices()->cend(), &pr, &pg);
  double out[5];
  detail::check(uvlm_rings_load_joukowski(r.data(), r0.data(), g.data(), gp.data(), (int64_t)vb.rows(),
                                          (int64_t)vb.cols(), &morphing.kinematics(), pr.data(), pg.data(),
                                          (int64_t)pg.size(), detail::c3(freestream), rho, t, dt, out),
                "CalcLoadJoukowski");
  return AerodynamicLoad{Vector3(out[0], out[1], out[2]), out[3], out[4]};
}

}  // namespace calc_load

// proto::Point / proto::Wing are declared in uvlm_b200.hpp (shared with the wing generators).

inline Vector3 PointToVector3d(const proto::Point& p) { return Vector3(p.x(), p.y(), p.z()); }

// --------------------------------------------------------- WingBuilder
namespace internal {
struct WingHolder {
  std::vector<Vector3> points;
  Vector3 origin;
  std::size_t rows = 0, cols = 0;
  double chord = 0, span = 0;
};

// TransformRow (src/wing_builder.h:21-35)
template <class InputIterator>
std::vector<Vector3> TransformRow(InputIterator first, InputIterator last) {
  std::vector<Vector3> row(first, last);
  std::vector<Vector3> res;
  for (std::size_t k = row.size(); k-- > 1;) {
    const double* p = detail::c3(row[k]);
    res.push_back(Vector3(p[0], -p[1], p[2]));
  }
  res.insert(res.end(), row.begin(), row.end());
  return res;
}
}  // namespace internal

// WingBuilder (src/wing_builder.{h,cpp}): half wings -> mirrored full wings,
// rings (i, j) = p(i, j), p(i+1, j), p(i+1, j+1), p(i, j+1) with their
// reference nodes saved.
class WingBuilder {
 public:
  WingBuilder(std::vector<VortexContainer>* containers, std::shared_ptr<std::vector<VortexRing>> vortices)
      : containers_(containers), vortices_(std::move(vortices)) {}
  ~WingBuilder() {
    if (is_modified_) Build();
  }
  WingBuilder& AddWing(const proto::Wing& wing) {
    is_modified_ = true;
    const std::size_t point_rows = wing.rows() + 1, point_cols = wing.cols() + 1;
    internal::WingHolder h;
    h.rows = wing.rows();
    h.cols = wing.cols() * 2;
    h.chord = wing.chord();
    h.span = wing.span();
    h.origin = wing.has_origin() ? PointToVector3d(wing.origin()) : Vector3(0, 0, 0);
    std::vector<Vector3> points;
    for (const auto& p : wing.points()) points.push_back(PointToVector3d(p));
    for (std::size_t i = 0; i < point_rows; i++) {
      auto first = points.begin() + i * point_cols;
      auto row = internal::TransformRow(first, first + point_cols);
      h.points.insert(h.points.end(), row.begin(), row.end());
    }
    for (auto& p : h.points) p = detail::add(p, h.origin);
    holders_.push_back(h);
    return *this;
  }
  void Build() {
    if (!is_modified_) return;
    vortices_->resize(CountTotalSize(holders_));
    containers_->resize(holders_.size());
    for (std::size_t i = 0; i < containers_->size(); i++) {
      containers_->at(i).set_vortices(vortices_, holders_[i].rows, holders_[i].cols, i, holders_[i].chord,
                                      holders_[i].span);
      BuildWing(&containers_->at(i), holders_[i]);
    }
    is_modified_ = false;
  }
  static void BuildWing(VortexContainer* container, const internal::WingHolder& h) {
    const std::size_t pc = h.cols + 1;
    for (std::size_t i = 0; i < h.rows; i++)
      for (std::size_t j = 0; j < h.cols; j++) {
        const std::size_t idx[4] = {j + i * pc, j + (i + 1) * pc, j + 1 + (i + 1) * pc, j + 1 + i * pc};
        VortexRing v;
        for (auto k : idx) v.nodes().push_back(h.points[k]);
        v.SaveReferenceNode();
        container->at(i, j) = v;
      }
  }
  static std::size_t CountTotalSize(const std::vector<internal::WingHolder>& holders) {
    std::size_t res = 0;
    for (const auto& h : holders) res += h.rows * h.cols;
    return res;
  }
  const std::vector<internal::WingHolder>& holders() const { return holders_; }

 private:
  std::vector<VortexContainer>* containers_;
  std::shared_ptr<std::vector<VortexRing>> vortices_;
  std::vector<internal::WingHolder> holders_;
  bool is_modified_ = false;
};

// ------------------------------------------------- legacy simulator
// UVLM::simulator free functions (src/simulator/simulator.cpp:202-270) over
// one process-wide state.  The reference's gflags become LegacyOptions.
// Snapshot2 files (SetOutputPath) are not written.
namespace simulator {

struct LegacyOptions {
  bool disable_wake = false;    // --disable_wake
  bool use_joukowski = false;   // --use_joukowski
  bool drop_wake_term = true;   // the reference's discarded wake RHS term
};

namespace legacy_detail {
struct State {
  LegacyOptions options;
  std::vector<proto::Wing> wings;
  std::vector<Morphing> morphings;
  std::shared_ptr<std::vector<VortexRing>> vortices = std::make_shared<std::vector<VortexRing>>();
  std::vector<VortexContainer> containers, containers_prev;
  UVLMVortexRing rings;  // empty, as in the reference
  Vector3 inlet = Vector3(1, 0, 0);
  std::string output_path, output_load_path;
  std::vector<std::vector<double>> load_rows;
};
inline State& state() {
  static State s;
  return s;
}
}  // namespace legacy_detail

inline LegacyOptions& legacy_options() { return legacy_detail::state().options; }
// Load rows of the last Start (t, then per wing C_x, C_y, C_z, Pin, Pout).
inline const std::vector<std::vector<double>>& legacy_load_rows() { return legacy_detail::state().load_rows; }
inline void ResetLegacySimulator() {
  const LegacyOptions o = legacy_options();
  legacy_detail::state() = legacy_detail::State();
  legacy_options() = o;
}

namespace legacy_detail {
// OutputSnapshot2 (simulator.cpp:118-160) to output_path/%08lu: the container
// shapes, every ring of the pool with its reference nodes, and per bound ring
// the morphing velocity at its reference centroid and at (start0 + end0) / 2
// of each segment (ForEachSegment order), with the inlet.
inline void OutputSnapshot2(State& s, std::size_t step, double t) {
  std::vector<int64_t> rows, cols;
  std::vector<double> chord, span, rings, rings0, gamma, center, nodes, inlet;
  for (const auto& c : s.containers) {
    rows.push_back((int64_t)c.rows());
    cols.push_back((int64_t)c.cols());
    chord.push_back(c.chord());
    span.push_back(c.span());
  }
  bool all0 = true;
  for (const auto& v : *s.vortices) {
    gamma.push_back(v.gamma());
    all0 = all0 && v.nodes0().size() == 4;
    for (std::size_t q = 0; q < 4; ++q)
      for (int d = 0; d < 3; ++d) {
        rings.push_back(detail::c3(v.nodes()[q])[d]);
        rings0.push_back(all0 ? detail::c3(v.nodes0()[q])[d] : 0.0);
      }
  }
  for (std::size_t i = 0; i < s.containers.size(); ++i) {
    std::vector<Vector3> x;  // per ring: reference centroid, then the four segment midpoints
    for (const auto& v : s.containers[i]) {
      x.push_back(v.ReferenceCentroid());
      const auto& n0 = v.nodes0();
      for (std::size_t q = 0; q < 4; ++q) x.push_back(detail::scale(detail::add(n0[(q + 1) % 4], n0[q]), 0.5));
    }
    std::vector<Vector3> vel(x.size());
    if (!x.empty())
      detail::check(uvlm_kinematics_velocity(&s.morphings[i].kinematics(), reinterpret_cast<const double*>(x.data()),
                                             (int64_t)x.size(), t, reinterpret_cast<double*>(vel.data())),
                    "OutputSnapshot2");
    for (std::size_t k = 0; k < vel.size(); ++k)
      for (int d = 0; d < 3; ++d) (k % 5 ? nodes : center).push_back(detail::c3(vel[k])[d]);
    for (std::size_t k = 0; k < vel.size() / 5; ++k)
      for (int d = 0; d < 3; ++d) inlet.push_back(detail::c3(s.inlet)[d]);
  }
  char name[32];
  std::snprintf(name, sizeof name, "/%08lu", (unsigned long)step);
  const std::string path = s.output_path + name;
  detail::check(uvlm_write_legacy_snapshot2(path.c_str(), t, (int64_t)rows.size(), rows.data(), cols.data(),
                                            chord.data(), span.data(), rings.data(), all0 ? rings0.data() : nullptr,
                                            gamma.data(), (int64_t)gamma.size(), center.data(), nodes.data(),
                                            inlet.data(), (int64_t)(center.size() / 3)),
                "OutputSnapshot2");
}
}  // namespace legacy_detail

inline void InitSimulator() {}
inline void AddWing(const proto::Wing& wing, const Morphing& m) {
  auto& s = legacy_detail::state();
  s.wings.push_back(wing);
  s.morphings.push_back(m);
  s.morphings.back().set_origin(PointToVector3d(wing.origin()));
}
inline void SetInlet(double x, double y, double z) { legacy_detail::state().inlet = Vector3(x, y, z); }
inline void SetOutputPath(const std::string& path) { legacy_detail::state().output_path = path; }
inline void SetOutputLoadPath(const std::string& path) { legacy_detail::state().output_load_path = path; }

// Start (simulator.cpp:220-270).
inline void Start(const std::size_t steps, const double dt) {
  auto& s = legacy_detail::state();
  if (s.morphings.empty()) throw Error(UVLM_ERR_INVALID, "No morphing");
  if (s.wings.empty()) throw Error(UVLM_ERR_INVALID, "No wing");
  if (!s.output_load_path.empty()) std::ofstream(s.output_load_path).close();
  {
    WingBuilder builder(&s.containers, s.vortices);
    for (const auto& w : s.wings) builder.AddWing(w);
    builder.Build();
  }
  s.load_rows.clear();
  const std::size_t wake_offset = CountTotalSize(s.containers.begin(), s.containers.end());
  for (std::size_t step = 0; step <= steps; ++step) {
    const double t = dt * step;
    s.containers_prev.resize(s.containers.size());
    CopyContainers(s.containers.begin(), s.containers.end(), s.containers_prev.begin());
    // MorphingProcess + ConnectProcess (:82-108)
    for (std::size_t i = 0; i < s.containers.size(); i++) {
      std::vector<Vector3> x0;
      for (const auto& v : s.containers[i])
        for (const auto& n : v.nodes0()) x0.push_back(n);
      std::vector<Vector3> x(x0.size());
      detail::check(uvlm_kinematics_perfome(&s.morphings[i].kinematics(), reinterpret_cast<const double*>(x0.data()),
                                            (int64_t)x0.size(), t, reinterpret_cast<double*>(x.data())),
                    "MorphingProcess");
      std::size_t k = 0;
      for (auto& v : s.containers[i])
        for (auto& n : v.nodes()) n = x[k++];
    }
    {
      const std::size_t shed = std::distance(s.containers[0].edge_begin(), s.containers[0].edge_end());
      if (wake_offset + shed <= s.vortices->size()) {
        auto edge = s.containers[0].edge_begin();
        for (auto it = s.vortices->begin() + wake_offset; it != s.vortices->begin() + wake_offset + shed;
             ++it, ++edge) {
          it->nodes().resize(4);
          it->nodes()[0] = edge->nodes()[1];
          it->nodes()[3] = edge->nodes()[2];
        }
      }
    }
    // SolveLinearProblem (:110-116)
    const VectorX gamma = SolveLinearProblem(s.containers, s.morphings, s.inlet, t, s.options.drop_wake_term);
    for (std::size_t i = 0; i < wake_offset; i++) s.vortices->at(i).set_gamma(gamma[i]);
    if (!s.output_path.empty()) legacy_detail::OutputSnapshot2(s, step, t);
    // CalcLoadProcess (:162-200)
    std::vector<double> row{t};
    for (std::size_t i = 0; i < s.containers.size(); i++) {
      const double rho = 1, S = s.containers[i].chord() * s.containers[i].span();
      const calc_load::AerodynamicLoad load =
          s.options.use_joukowski
              ? calc_load::CalcLoadJoukowski(s.containers[i], s.containers_prev[i], s.morphings[i], s.inlet, rho, t,
                                             dt)
              : calc_load::CalcLoadKatzPlotkin(s.containers[i], s.containers_prev[i], s.morphings[i], s.rings,
                                               s.inlet, rho, t, dt);
      const double U = detail::norm(s.inlet);
      const Vector3 coeff = detail::scale(load.F, 1.0 / (0.5 * rho * U * U * S));
      for (int d = 0; d < 3; ++d) row.push_back(detail::c3(coeff)[d]);
      row.push_back(load.Pin);
      row.push_back(load.Pout);
    }
    s.load_rows.push_back(row);
    if (!s.output_load_path.empty()) {
      std::ofstream ofs(s.output_load_path, std::ios::app);
      for (std::size_t k = 0; k < row.size(); ++k) ofs << (k ? "\t" : "") << row[k];
      ofs << "\n";
    }
    if (step == steps) break;
    if (!s.options.disable_wake) {  // :252-266
      std::vector<VortexRing> wake_next(s.containers[0].edge_begin(), s.containers[0].edge_end());
      wake_next.insert(wake_next.end(), s.vortices->cbegin() + wake_offset, s.vortices->cend());
      AdvectParallel(s.vortices->cbegin(), s.vortices->cend(), wake_next.begin(), wake_next.end(), s.inlet, dt);
      s.vortices->resize(wake_offset + wake_next.size());
      std::copy(wake_next.cbegin(), wake_next.cend(), s.vortices->begin() + wake_offset);
    }
  }
}

}  // namespace simulator
}  // namespace UVLM
