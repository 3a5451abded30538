// legacy_parity.cpp -- the legacy AoS C++ API of include/uvlm_b200.hpp used the
// way the reference's own tests use it (test/vortex_container_test.cpp,
// test/wing_builder_test.cpp, test/shed_test.cpp, test/linear_test.cpp),
// plus the container loads against the FP64 CPU oracle.
//   legacy_parity cpu    containers, wing builder, ring geometry (no GPU)
//   legacy_parity gpu    shed, linear and load checks on the GPU
//   legacy_parity start [dir]  prints the load rows of simulator::Start
//                              (and writes its Snapshot2 files to dir)
// Exit status 0 when every check passes.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "uvlm_b200.hpp"
#include "uvlm_oracle.h"

using UVLM::Vector3;
using UVLM::VortexContainer;
using UVLM::VortexRing;

static int failures = 0;
static void expect(bool ok, const char* what) {
  if (!ok) {
    std::printf("FAIL %s\n", what);
    ++failures;
  }
}
static bool near(double a, double b, double tol) { return std::fabs(a - b) <= tol; }
static bool vnear(const Vector3& v, double x, double y, double z, double tol) {
  return near(v.x(), x, tol) && near(v.y(), y, tol) && near(v.z(), z, tol);
}

// GetSquareRing(l, x0, y0) (test/testutil.h:36-46)
static VortexRing square(double l, double x0, double y0) {
  VortexRing r;
  x0 -= l / 2;
  y0 -= l / 2;
  r.PushNode(x0, y0, 0).PushNode(x0 + l, y0, 0).PushNode(x0 + l, y0 + l, 0).PushNode(x0, y0 + l, 0);
  return r;
}

static void uvlm_vortex_ring_checks() {
  // uvlm_vortex_ring_test.cpp:7-85: a 5 x 10 half-wing lattice of spacing 0.1
  const double dx = 0.1;
  const std::size_t rows = 5, cols = 10;
  std::vector<Vector3> pos;
  for (std::size_t i = 0; i <= rows; i++)
    for (std::size_t j = 0; j <= cols; j++) pos.push_back(Vector3(i * dx, j * dx, 0));
  UVLM::UVLMVortexRing rings;
  rings.InitWing(pos, cols);
  const auto& v = rings.bound_vortices();
  bool ok = v.size() == 2 * rows * cols && rings.rows() == rows && rings.cols() == cols;
  for (std::size_t i = 0; i < rows; i++) {
    for (std::size_t j = 0; j < cols; j++) {  // y >= 0
      const auto& n = v[j + i * (2 * cols)].nodes();
      ok = ok && vnear(n[0], i * dx, j * dx, 0, 0) && vnear(n[1], (i + 1) * dx, j * dx, 0, 0) &&
           vnear(n[2], (i + 1) * dx, (j + 1) * dx, 0, 0) && vnear(n[3], i * dx, (j + 1) * dx, 0, 0);
    }
    for (std::size_t j = 0; j < cols; j++) {  // y <= 0
      const auto& n = v[j + cols + i * (2 * cols)].nodes();
      ok = ok && vnear(n[3], i * dx, -1. * j * dx, 0, 0) && vnear(n[2], (i + 1) * dx, -1. * j * dx, 0, 0) &&
           vnear(n[1], (i + 1) * dx, -1. * (j + 1) * dx, 0, 0) && vnear(n[0], i * dx, -1. * (j + 1) * dx, 0, 0);
    }
  }
  expect(ok, "UVLMVortexRing::InitWing");
  auto te = rings.TrailingEdgeIterators();
  std::size_t i = 0;
  bool ok2 = true;
  for (auto it = te.first; it != te.second; ++it, ++i)
    ok2 = ok2 && (i < cols ? near(it->nodes()[0].y(), i * dx, 0)
                           : near(it->nodes()[3].y(), ((int)cols - (int)i) * dx, 0));
  expect(ok2 && i == 2 * cols, "UVLMVortexRing::TrailingEdgeIterators");
}

static void cpu_checks() {
  uvlm_vortex_ring_checks();
  // vortex_container_test.cpp:8-60: four 2 x 3 containers, gamma = running index
  auto vortices = std::make_shared<std::vector<VortexRing>>();
  for (int val = 0; val < 24; ++val) {
    vortices->emplace_back();
    vortices->back().set_gamma(val);
  }
  std::vector<VortexContainer> containers;
  for (int id = 0; id < 4; ++id) containers.emplace_back(vortices, 2, 3, 4, 1.0, 2.0);
  VortexContainer v(vortices, 2, 3, 1, 1, 1);
  expect(v.rows() == 2 && v.cols() == 3 && v.id() == 1, "container shape");
  expect(v.Index(0) == 6 && v.Index(0, 1) == 7 && v.Index(1, 2) == 11, "container index");
  VortexContainer v2(vortices, 2, 3, 2, 1, 1);
  expect(v2.Index(0) == 12 && v2.Index(1, 1) == 16 && v2.Offset() == 12, "container index2");
  expect(v[3].gamma() == 9 && v.at(1, 2).gamma() == 11, "container access");
  VortexContainer v0(vortices, 2, 3, 0, 1, 1);
  v0[0].set_gamma(10);
  expect((*vortices)[0].gamma() == 10 && &v0[0] == &vortices->at(0), "container shares the pool");
  vortices->at(0).set_gamma(0);
  {
    double g = 6;
    bool ok = true;
    for (auto it = v.begin(); it != v.end(); ++it) ok = ok && it->gamma() == g++;
    expect(ok && g == 12, "container iterator");
    g = 9;
    ok = true;
    for (auto it = v.edge_begin(); it != v.edge_end(); ++it) ok = ok && it->gamma() == g++;
    expect(ok && g == 12, "container edge iterator");
  }
  expect(UVLM::CountTotalSize(containers.begin(), containers.end()) == 24, "CountTotalSize");
  {
    std::vector<VortexContainer> copied(containers.size());
    UVLM::CopyContainers(containers.begin(), containers.end(), copied.begin());
    bool ok = copied[0].vortices().get() != vortices.get();
    for (std::size_t i = 0; i < containers.size(); ++i)
      ok = ok && containers[i].ShapeEquals(copied[i]) && copied[i].chord() == 1.0 && copied[i].span() == 2.0;
    expect(ok, "CopyContainers");
  }

  // wing_builder_test.cpp:31-123
  {
    std::vector<Vector3> row{{1, 0, 2}, {1, 1, 2}, {1, 2, 2}};
    auto r = UVLM::internal::TransformRow(row.begin(), row.end());
    bool ok = r.size() == 5;
    const double ys[5] = {-2, -1, 0, 1, 2};
    for (int k = 0; ok && k < 5; ++k) ok = r[k].y() == ys[k] && r[k].x() == 1 && r[k].z() == 2;
    expect(ok, "TransformRow");
  }
  UVLM::proto::Wing wing;
  wing.set_rows(2);
  wing.set_cols(3);
  for (int i = 0; i <= 2; i++)
    for (int j = 0; j <= 3; j++) {
      auto* p = wing.add_points();
      p->set_x(i);
      p->set_y(j);
      p->set_z(0);
    }
  {
    std::vector<VortexContainer> cs;
    auto pool = std::make_shared<std::vector<VortexRing>>();
    UVLM::WingBuilder builder(&cs, pool);
    UVLM::proto::Wing wing2;
    wing2.CopyFrom(wing);
    auto* o = wing2.mutable_origin();
    o->set_x(0);
    o->set_y(0);
    o->set_z(1);
    builder.AddWing(wing).AddWing(wing2);
    const auto& h = builder.holders();
    expect(h.size() == 2 && h[1].rows == 2 && h[1].cols == 6, "WingBuilder holders");
    expect(h[1].points[0].x() == 0 && h[1].points[0].y() == -3 && h[1].points[0].z() == 1 &&
               h[1].points[6].z() == 1,
           "WingBuilder mirrored points with origin");
    builder.Build();
    expect(pool->size() == 24 && cs.size() == 2 && cs[0].rows() == 2 && cs[0].cols() == 6, "WingBuilder::Build");
    const auto& n = cs[0].at(0, 0);
    expect(n.nodes()[0].x() == 0 && n.nodes()[0].y() == -3 && n.nodes0()[0].y() == -3, "built ring nodes");
  }

  // ring geometry against the oracle (vortex.cpp:82-143)
  {
    VortexRing r;
    r.PushNode(0.1, -0.2, 0.05).PushNode(1.2, -0.1, 0.0).PushNode(1.0, 0.9, -0.1).PushNode(-0.1, 1.1, 0.02);
    r.set_gamma(1.7);
    double nodes[12];
    for (int q = 0; q < 4; ++q)
      for (int d = 0; d < 3; ++d) nodes[3 * q + d] = reinterpret_cast<const double*>(&r.nodes()[q])[d];
    double o[3];
    orc_ring_vector(nodes, 1.7, 0, o);
    expect(vnear(r.Normal(), o[0], o[1], o[2], 1e-14), "Normal");
    orc_ring_vector(nodes, 1.7, 1, o);
    expect(vnear(r.Tangent(), o[0], o[1], o[2], 1e-14), "Tangent");
    orc_ring_vector(nodes, 1.7, 6, o);
    expect(vnear(r.Impulse(), o[0], o[1], o[2], 1e-14), "Impulse");
    expect(near(r.Area(), orc_ring_scalar(nodes, 0), 1e-14) && near(r.CalcC(), orc_ring_scalar(nodes, 1), 1e-14) &&
               near(r.CalcB(), orc_ring_scalar(nodes, 2), 1e-14),
           "Area, CalcC, CalcB");
    const double Q[3] = {1.0, 0.1, 0.2};
    expect(near(r.AngleOfAttack(Vector3(1.0, 0.1, 0.2)), orc_ring_angle_of_attack(nodes, Q), 1e-14),
           "AngleOfAttack");
  }
}

static void gpu_checks() {
  const double PI = 3.14159265358979323846, SQ2 = std::sqrt(2.0);
  // shed_test.cpp:8-50
  VortexRing v;
  v.set_gamma(4 * PI);
  v.PushNode(1, 1, 0).PushNode(-1, 1, 0).PushNode(-1, -1, 0).PushNode(1, -1, 0);
  std::vector<VortexRing> rings(20, v);
  Vector3 res;
  UVLM::InducedVelocity(&res, Vector3(0, 0, 0), rings.begin(), rings.end());
  expect(vnear(res, 0, 0, -4 * SQ2 * 20, 1e-12), "InducedVelocity many rings");
  UVLM::ChordwiseInducedVelocity(&res, Vector3(0, 0, 0), rings.begin(), rings.end());
  expect(vnear(res, 0, 0, -2 * SQ2 * 20, 1e-12), "ChordwiseInducedVelocity many rings");
  {
    std::vector<VortexRing> edge{square(2, 1, 1), square(2, 1, 3)}, wake{square(2, 99, 1), square(2, 99, 3)};
    UVLM::ConnectTrailingEdge(edge.cbegin(), edge.cend(), wake.begin());
    expect(vnear(wake[0].nodes()[0], 2, 0, 0, 0) && vnear(wake[0].nodes()[1], 100, 0, 0, 0) &&
               vnear(wake[1].nodes()[3], 2, 4, 0, 0),
           "ConnectTrailingEdge");
  }
  for (int parallel = 0; parallel < 2; ++parallel) {
    std::vector<VortexRing> wake{square(2, 0, 0)}, dummy;
    if (parallel)
      UVLM::AdvectParallel(dummy.begin(), dummy.end(), wake.begin(), wake.end(), Vector3(1, 0, 0), 0.1);
    else
      UVLM::Advect(dummy.begin(), dummy.end(), wake.begin(), wake.end(), Vector3(1, 0, 0), 0.1);
    const auto& n = wake[0].nodes();
    expect(vnear(n[0], -0.9, -1, 0, 1e-15) && vnear(n[2], 1.1, 1, 0, 1e-15), "Advect without vortices");
  }

  // linear_test.cpp:27-49 (flap = sin t) and :51-140
  {
    UVLM::Morphing m;
    m.set_flap(1.0, 1.0);
    m.set_origin(Vector3(0, 0, 0));
    std::vector<VortexRing> panels{square(1, 0, 1), square(1, 0, -2)};
    for (auto& p : panels) p.SaveReferenceNode();
    std::vector<double> out(2);
    auto it = UVLM::internal::CalcMorphingVelocityOnWing(panels.cbegin(), panels.cend(), m, 0, out.begin());
    expect(it == out.end() && near(out[0], 1, 1e-10) && near(out[1], 2, 1e-10), "CalcMorphingVelocityOnWing flap");
  }
  {
    const double alpha = PI / 6, U = 2, a = 0.1;
    UVLM::Morphing m;
    std::vector<VortexRing> vs, dummy;
    VortexRing r;
    r.PushNode(0, 0, 0).PushNode(a * std::cos(alpha), 0, -a * std::sin(alpha));
    r.PushNode(a * std::cos(alpha), a, -a * std::sin(alpha)).PushNode(0, a, 0);
    r.SaveReferenceNode();
    vs.push_back(r);
    auto g = UVLM::SolveLinearProblem(vs.begin(), vs.end(), dummy.begin(), dummy.end(), Vector3(U, 0, 0), m, 0);
    expect(near(g(0), SQ2 * PI * a * U * std::sin(alpha) / 4, 1e-10), "SolveLinearProblem no_wake");
  }
  for (int mode = 0; mode < 3; ++mode) {  // no_wake_no_morphing, no_wake_morphing, wake_morphing
    std::vector<VortexRing> vs{square(2, -1, 0), square(2, 1, 0)}, wake;
    for (auto& r : vs) r.SaveReferenceNode();
    if (mode == 2) wake.push_back(square(2, 2, 0));
    UVLM::Morphing m;
    if (mode > 0) m.set_plug(0.1, 1.0);
    auto g = UVLM::SolveLinearProblem(vs.cbegin(), vs.cend(), wake.cbegin(), wake.cend(), Vector3(0, 0, 1), m, 0);
    vs[0].set_gamma(g(0));
    vs[1].set_gamma(g(1));
    Vector3 v0, v1, w0(0, 0, 0), w1(0, 0, 0);
    UVLM::InducedVelocity(&v0, Vector3(-1, 0, 0), vs.cbegin(), vs.cend());
    UVLM::InducedVelocity(&v1, Vector3(1, 0, 0), vs.cbegin(), vs.cend());
    if (mode == 2) {
      UVLM::InducedVelocity(&w0, Vector3(-1, 0, 0), wake.cbegin(), wake.cend());
      UVLM::InducedVelocity(&w1, Vector3(1, 0, 0), wake.cbegin(), wake.cend());
    }
    const double e = mode > 0 ? 0.1 : 0.0;
    expect(vnear(v0, 0, 0, -1 + e + w0.z(), 1e-10) && vnear(v1, 0, 0, -1 + e + w1.z(), 1e-10),
           "SolveLinearProblem no-penetration");
  }

  // container loads against the oracle on a built, morphed 3 x 8 wing
  {
    UVLM::proto::Wing wing;
    wing.set_rows(3);
    wing.set_cols(4);
    wing.set_chord(1.0);
    wing.set_span(2.0);
    for (int i = 0; i <= 3; i++)
      for (int j = 0; j <= 4; j++) {
        auto* p = wing.add_points();
        p->set_x(i / 3.0);
        p->set_y(j / 2.0);
        p->set_z(0.02 * i * j);
      }
    std::vector<VortexContainer> cs, prev;
    auto pool = std::make_shared<std::vector<VortexRing>>();
    UVLM::WingBuilder(&cs, pool).AddWing(wing).Build();
    UVLM::Morphing m;
    m.set_alpha(0.1);
    m.set_plug(0.1, 1.0, 0.3);
    m.set_twist(0.05, 1.0, 0.5);
    const double t = 0.7, dt = 0.1;
    for (auto& r : cs[0]) {
      for (std::size_t q = 0; q < 4; ++q) m.Perfome(&r.nodes()[q], r.nodes0()[q], t);
    }
    for (std::size_t k = 0; k < pool->size(); ++k) (*pool)[k].set_gamma(0.3 + 0.01 * k);
    prev.resize(1);
    UVLM::CopyContainers(cs.begin(), cs.end(), prev.begin());
    for (std::size_t k = 0; k < pool->size(); ++k) (*pool)[k].set_gamma(0.3 + 0.012 * k);
    // a few wake rings behind the wing in the pool
    for (int j = 0; j < 8; ++j) {
      VortexRing w = square(0.4, 1.3, -1.75 + 0.5 * j);
      w.set_gamma(0.05 * (j - 3));
      pool->push_back(w);
    }
    std::vector<double> rr, g, r0, g0, rp, gp, pr, pg;
    UVLM::detail::pack_rings(cs[0].cbegin(), cs[0].cend(), &rr, &g);          // nodes(), gamma
    UVLM::detail::pack_rings(cs[0].cbegin(), cs[0].cend(), &r0, &g0, true);   // nodes0()
    UVLM::detail::pack_rings(prev[0].cbegin(), prev[0].cend(), &rp, &gp);     // previous gamma
    UVLM::detail::pack_rings(pool->cbegin(), pool->cend(), &pr, &pg);         // the whole pool
    orc_kinematics k;
    std::memcpy(&k, &m.kinematics(), sizeof(k));
    const double fs[3] = {1.0, 0.0, 0.05};
    double ref[5];
    UVLM::UVLMVortexRing empty;
    auto kp = UVLM::calc_load::CalcLoadKatzPlotkin(cs[0], prev[0], m, empty, Vector3(1, 0, 0.05), 1.0, t, dt);
    orc_load_katz_plotkin(rr.data(), g.data(), gp.data(), 3, 8, &k, nullptr, nullptr, 0, nullptr, nullptr, 0, fs,
                          1.0, t, dt, ref);
    const double s1 = std::fmax(std::fabs(ref[2]), 1e-3);
    expect(vnear(kp.F, ref[0], ref[1], ref[2], 1e-11 * s1) && near(kp.Pin, ref[3], 1e-11 * s1) && kp.Pout == 0,
           "CalcLoadKatzPlotkin vs oracle");
    auto jk = UVLM::calc_load::CalcLoadJoukowski(cs[0], prev[0], m, Vector3(1, 0, 0.05), 1.0, t, dt);
    orc_load_joukowski_rings(rr.data(), r0.data(), g.data(), gp.data(), 3, 8, &k, pr.data(), pg.data(),
                             (int64_t)pg.size(), fs, 1.0, t, dt, ref);
    const double s2 = std::fmax(std::fabs(ref[2]), 1e-3);
    expect(vnear(jk.F, ref[0], ref[1], ref[2], 1e-11 * s2) && near(jk.Pin, ref[3], 1e-11 * s2) &&
               near(jk.Pout, ref[4], 1e-11 * s2),
           "CalcLoadJoukowski vs oracle");
  }
}

static void start_rows(bool joukowski, const char* out_dir) {
  // two half wings 3 x 4 (chord 1, half span 2), the second 0.8 above
  namespace S = UVLM::simulator;
  S::ResetLegacySimulator();
  S::legacy_options().use_joukowski = joukowski;
  for (int w = 0; w < 2; ++w) {
    UVLM::proto::Wing wing;
    wing.set_rows(3);
    wing.set_cols(4);
    wing.set_chord(1.0);
    wing.set_span(2.0);
    for (int i = 0; i <= 3; i++)
      for (int j = 0; j <= 4; j++) {
        auto* p = wing.add_points();
        p->set_x(i / 3.0);
        p->set_y(j / 2.0);
        p->set_z(0);
      }
    auto* o = wing.mutable_origin();
    o->set_x(0);
    o->set_y(0);
    o->set_z(0.8 * w);
    UVLM::Morphing m;
    m.set_alpha(0.08);
    m.set_plug(0.1, 1.0, 0.5 * w);
    m.set_twist(0.05, 1.0, 0.3);
    S::AddWing(wing, m);
  }
  S::SetInlet(1, 0, 0);
  if (out_dir) S::SetOutputPath(out_dir);
  S::Start(10, 2 * 3.14159265358979323846 / 40);
  for (const auto& row : S::legacy_load_rows()) {
    for (std::size_t k = 0; k < row.size(); ++k) std::printf("%s%.17g", k ? " " : "", row[k]);
    std::printf("\n");
  }
}

int main(int argc, char** argv) {
  const char* mode = argc > 1 ? argv[1] : "cpu";
  if (!std::strcmp(mode, "cpu")) cpu_checks();
  if (!std::strcmp(mode, "gpu")) gpu_checks();
  const char* out_dir = argc > 2 ? argv[2] : nullptr;
  if (!std::strcmp(mode, "start")) start_rows(false, out_dir);
  if (!std::strcmp(mode, "start_joukowski")) start_rows(true, out_dir);
  if (failures) std::printf("%d check(s) failed\n", failures);
  return failures ? 1 : 0;
}
