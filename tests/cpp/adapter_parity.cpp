// adapter_parity.cpp -- the C++ adapter (include/uvlm_b200.hpp) used the way a
// C++ host of the reference uses src/uvlm.h, checked against the FP64 CPU
// oracle.  Exit status 0 when every check passes.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "uvlm_b200.hpp"
#include "uvlm_oracle.h"

using UVLM::MultipleSheet;
using UVLM::Vector3;

static int failures = 0;
static void expect(bool ok, const char* what, double err) {
  std::printf("%-44s max err %.3e  %s\n", what, err, ok ? "ok" : "FAIL");
  if (!ok) ++failures;
}

int main() {
  // 1. UVLM::InducedVelocity on a wavy 2 x 3 x 5 sheet set
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> U(-0.1, 0.1);
  MultipleSheet<Vector3> pos(2, 4, 6);
  MultipleSheet<double> gamma(2, 3, 5);
  for (std::size_t n = 0; n < 2; ++n)
    for (std::size_t i = 0; i < 4; ++i)
      for (std::size_t j = 0; j < 6; ++j) pos.at(n, i, j) = Vector3(0.3 * i + U(rng), 0.5 * j + U(rng), 0.4 * n + U(rng));
  for (auto& g : gamma) g = 1.0 + U(rng);
  std::vector<Vector3> xs;
  for (int k = 0; k < 17; ++k) xs.emplace_back(U(rng) * 10, 1.2 + U(rng) * 10, 0.2 + U(rng) * 5);
  const auto got = UVLM::InducedVelocity(xs, pos, gamma);
  std::vector<double> ref(3 * xs.size());
  orc_sheet_induced_velocity(reinterpret_cast<const double*>(pos.data()), 2, 4, 6, gamma.data(), 3, 5,
                             reinterpret_cast<const double*>(xs.data()), (int64_t)xs.size(), ref.data());
  double e1 = 0, s1 = 0;
  for (std::size_t k = 0; k < xs.size(); ++k)
    for (int d = 0; d < 3; ++d) {
      e1 = std::fmax(e1, std::fabs(got[k][d] - ref[3 * k + d]));
      s1 = std::fmax(s1, std::fabs(ref[3 * k + d]));
    }
  expect(e1 <= 1e-12 * s1 + 1e-15, "InducedVelocity vs oracle", e1);
  const Vector3 one = UVLM::InducedVelocity(xs[3], pos, gamma);
  expect(std::fabs(one[2] - ref[3 * 3 + 2]) <= 1e-12 * s1, "InducedVelocity single point", std::fabs(one[2] - ref[11]));

  // 2. SimpleSimulator::Run, RK2 heave + pitch, 4 x 8 rings, 14 steps
  const double PI = 3.14159265358979323846, dt = 2 * PI / 40;
  UVLM::Morphing m;
  m.set_plug(0.2, 1.0);
  m.set_twist(10 * PI / 180, 1.0, PI / 2);
  UVLM::simulator::SimpleSimulator sim;
  sim.AddWing(UVLM::wing::RectGenerator{}, m, 1.0, 4.0, 4, 8, Vector3(0, 0, 0));
  sim.set_forward_flight(Vector3(-1, 0, 0));
  sim.set_advection("RK2");
  const auto rows = sim.Run(14, dt);

  orc_kinematics k{};
  k.plug_amp = 0.2;
  k.plug_omega = 1.0;
  k.twist_amp = 10 * PI / 180;
  k.twist_omega = 1.0;
  k.twist_phase = PI / 2;
  const double origin[3] = {0, 0, 0}, ff[3] = {-1, 0, 0};
  void* o = orc_sim_create();
  orc_sim_add_wing(o, 1.0, 4.0, 4, 8, origin, &k, 0, 0);
  orc_sim_set_forward_flight(o, ff);
  orc_sim_set_advection(o, "RK2");
  orc_sim_begin(o);
  double e2 = 0, s2 = 0;
  for (int s = 0; s <= 14; ++s) {
    double row[3];
    orc_sim_step(o, s, dt, row);
    for (int q = 1; q < 3; ++q) {
      e2 = std::fmax(e2, std::fabs(rows[s][q] - row[q]));
      s2 = std::fmax(s2, std::fabs(row[q]));
    }
  }
  orc_sim_destroy(o);
  expect(e2 <= 1e-8 * s2, "SimpleSimulator::Run loads vs oracle", e2);

  // 3. advect::AdvectFactory("RK2") in place == out of place, on the run's state
  MultipleSheet<Vector3> wing_pos, wake_pos, next;
  MultipleSheet<double> wing_gamma, wake_gamma;
  sim.GetState(&wing_pos, &wing_gamma, &wake_pos, &wake_gamma);
  auto adv = UVLM::advect::AdvectFactory("RK2");
  adv->Advect(&next, wing_pos, wing_gamma, wake_pos, wake_gamma, Vector3(-1, 0, 0), dt);
  MultipleSheet<Vector3> inplace = wake_pos;
  adv->Advect(&inplace, wing_pos, wing_gamma, inplace, wake_gamma, Vector3(-1, 0, 0), dt);
  double e3 = 0;
  for (std::size_t q = 0; q < next.size(); ++q)
    for (int d = 0; d < 3; ++d) e3 = std::fmax(e3, std::fabs(next[q][d] - inplace[q][d]));
  expect(e3 == 0.0 && next.size() == wake_pos.size(), "Advection::Advect aliasing next == wake_pos", e3);

  // 4. the set-up of src/multiple_flapping_wings_main.cpp:40-73 with its flag
  // defaults: three NACA 83 wings (AddWing takes the generator, as the
  // reference's does), flap -pi/4 cos(w t) = pi/4 sin(w t - pi/2), alpha 5 deg,
  // w = 2 U k / c with k = 0.1, 6 x 20 rings, Euler; 30 steps
  {
    const double w = 2 * 1.0 * 0.1 / 1.0, dtw = 2 * PI / w / 40, alpha = 5 * PI / 180;
    const double origins[3][3] = {{0, 0, 0}, {3, 6, 0}, {3, -6, 0}};
    UVLM::simulator::SimpleSimulator ms;
    UVLM::Morphing mf;
    mf.set_flap(PI / 4, w, -PI / 2);
    mf.set_alpha(alpha);
    for (auto& og : origins)
      ms.AddWing(new UVLM::wing::NACA4digitGenerator(83), mf, 1.0, 6.0, 6, 20, Vector3(og[0], og[1], og[2]));
    ms.set_forward_flight(Vector3(-1, 0, 0));
    ms.set_advection("euler");
    const auto mrows = ms.Run(30, dtw);

    orc_kinematics kf{};
    kf.alpha = alpha;
    kf.flap_amp = PI / 4;
    kf.flap_omega = w;
    kf.flap_phase = -PI / 2;
    void* om = orc_sim_create();
    for (auto& og : origins) orc_sim_add_wing_generator(om, 1, 83, 1.0, 6.0, 6, 20, og, &kf, 0, 0);
    orc_sim_set_forward_flight(om, ff);
    orc_sim_set_advection(om, "euler");
    orc_sim_begin(om);
    double e4 = 0, s4 = 0;
    for (int s = 0; s <= 30; ++s) {
      double row[7];
      orc_sim_step(om, s, dtw, row);
      for (int q = 1; q < 7; ++q) {
        e4 = std::fmax(e4, std::fabs(mrows[s][q] - row[q]));
        s4 = std::fmax(s4, std::fabs(row[q]));
      }
    }
    orc_sim_destroy(om);
    expect(e4 <= 1e-8 * s4, "NACA 83 three-wing flap loads vs oracle", e4);
  }

  // 5. errors surface as UVLM::Error (the reference aborts)
  bool threw = false;
  try {
    UVLM::advect::AdvectFactory("RK3");
  } catch (const UVLM::Error& e) {
    threw = e.code() == UVLM_ERR_INVALID;
  }
  expect(threw, "AdvectFactory rejects an unknown name", 0.0);
  return failures ? 1 : 0;
}
