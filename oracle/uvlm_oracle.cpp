// uvlm_oracle.cpp -- CPU FP64 restatement of xeno14/UVLM's time-stepper.
//
// TEST INFRASTRUCTURE ONLY: the correctness oracle and the timed CPU baseline
// for the CUDA product.  Every function cites the reference file:line it
// restates.  Arithmetic is FP64 and follows the reference's evaluation order
// (Eigen 3-vector expressions expanded component-wise), OpenMP sits on the
// loops the reference parallelises, and the dense solve is a complete
// (full) pivoting LU like Eigen::FullPivLU.
//
// MultipleSheet (the reference's missing submodule) is re-created from its
// call sites: a dense num x rows x cols buffer with K = j + cols*(i + rows*n),
// prepend_row() inserting a new row i=0 in every sheet and erase_last_row()
// dropping the last row of every sheet.

#include "uvlm_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <tuple>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

struct V3 {
  double x = 0, y = 0, z = 0;
  V3() = default;
  V3(double a, double b, double c) : x(a), y(b), z(c) {}
  explicit V3(const double* p) : x(p[0]), y(p[1]), z(p[2]) {}
  void store(double* p) const { p[0] = x; p[1] = y; p[2] = z; }
};
inline V3 operator+(const V3& a, const V3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(const V3& a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(const V3& a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(const V3& a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3& operator+=(V3& a, const V3& b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
inline double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double sqnorm(const V3& a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline double norm(const V3& a) { return std::sqrt(sqnorm(a)); }
inline V3 cross(const V3& a, const V3& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 normalized(const V3& a) {
  const double n = norm(a);
  return n > 0 ? a / n : a;
}

// Re-created multiple_sheet::MultipleSheet<T> (layout only, no arithmetic).
template <class T>
class Sheet {
 public:
  Sheet() = default;
  Sheet(size_t num, size_t rows, size_t cols) { resize(num, rows, cols); }
  void resize(size_t num, size_t rows, size_t cols) {
    num_ = num; rows_ = rows; cols_ = cols;
    data_.assign(num * rows * cols, T());
  }
  template <class U>
  void resize(const Sheet<U>& o) { resize(o.num(), o.rows(), o.cols()); }
  size_t num() const { return num_; }
  size_t rows() const { return rows_; }
  size_t cols() const { return cols_; }
  size_t size() const { return data_.size(); }
  size_t index(size_t n, size_t i, size_t j) const { return j + cols_ * (i + rows_ * n); }
  T& at(size_t n, size_t i, size_t j) { return data_[index(n, i, j)]; }
  const T& at(size_t n, size_t i, size_t j) const { return data_[index(n, i, j)]; }
  T& operator[](size_t k) { return data_[k]; }
  const T& operator[](size_t k) const { return data_[k]; }
  T* sheet_begin(size_t n) { return data_.data() + index(n, 0, 0); }
  const T* sheet_begin(size_t n) const { return data_.data() + index(n, 0, 0); }
  // prepend_row(first, last): the input is num x cols values, one row per
  // sheet; it becomes row i=0 of every sheet
  // (src/simulator/simple_simulator.cpp:179,186).
  void prepend_row(const std::vector<T>& row) {
    std::vector<T> nd(num_ * (rows_ + 1) * cols_);
    for (size_t n = 0; n < num_; n++) {
      for (size_t j = 0; j < cols_; j++) nd[j + cols_ * ((rows_ + 1) * n)] = row[n * cols_ + j];
      for (size_t i = 0; i < rows_; i++)
        for (size_t j = 0; j < cols_; j++)
          nd[j + cols_ * (i + 1 + (rows_ + 1) * n)] = data_[index(n, i, j)];
    }
    rows_ += 1;
    data_.swap(nd);
  }
  // erase_last_row() (src/simulator/simple_simulator.cpp:236-237).
  void erase_last_row() {
    if (rows_ == 0) return;
    std::vector<T> nd(num_ * (rows_ - 1) * cols_);
    for (size_t n = 0; n < num_; n++)
      for (size_t i = 0; i + 1 < rows_; i++)
        for (size_t j = 0; j < cols_; j++)
          nd[j + cols_ * (i + (rows_ - 1) * n)] = data_[index(n, i, j)];
    rows_ -= 1;
    data_.swap(nd);
  }
  std::vector<T>& data() { return data_; }
  const std::vector<T>& data() const { return data_; }

 private:
  size_t num_ = 0, rows_ = 0, cols_ = 0;
  std::vector<T> data_;
};

// ---------------------------------------------------------------- vortex.cpp
// src/vortex.cpp:13-19
double DistanceLineAndPoint(const V3& start, const V3& end, const V3& pos) {
  V3 direction = normalized(end - start);
  V3 diff = pos - start;
  return norm(diff - direction * dot(direction, diff));
}

// src/vortex.cpp:21-39 (Katz & Plotkin p.255), cutoff 1e-10, no core.
inline V3 BiotSavartLaw(const V3& start, const V3& end, const V3& pos) {
  const V3 r0 = end - start;
  const V3 r1 = pos - start;
  const V3 r2 = pos - end;
  const V3 d = cross(r1, r2);
  const double d_len = norm(d);
  const double r1_len = norm(r1);
  const double r2_len = norm(r2);
  const double eps = 1e-10;
  if (d_len * d_len < eps || r1_len < eps || r2_len < eps) return V3();
  const double K = 1. / 4. / M_PI / sqnorm(d) * dot(r0, r1 / norm(r1) - r2 / norm(r2));
  return d * K;
}

// src/vortex.h:173-182
inline V3 VORTEX(const V3& x, const V3& x1, const V3& x2, double gamma) {
  return BiotSavartLaw(x1, x2, x) * gamma;
}

// src/vortex.cpp:145-160
inline V3 VORING(const V3& x, const Sheet<V3>& pos, const Sheet<double>& gamma,
                 size_t n, size_t i, size_t j) {
  V3 u;
  const double g = gamma.at(n, i, j);
  const V3& p0 = pos.at(n, i, j);
  const V3& p1 = pos.at(n, i, j + 1);
  const V3& p2 = pos.at(n, i + 1, j + 1);
  const V3& p3 = pos.at(n, i + 1, j);
  u += VORTEX(x, p0, p1, g);
  u += VORTEX(x, p1, p2, g);
  u += VORTEX(x, p2, p3, g);
  u += VORTEX(x, p3, p0, g);
  return u;
}

// src/velocity.h:14-24 (serial over gamma.list_index()).
inline V3 InducedVelocity(const V3& x, const Sheet<V3>& pos, const Sheet<double>& gamma) {
  V3 res;
  for (size_t n = 0; n < gamma.num(); n++)
    for (size_t i = 0; i < gamma.rows(); i++)
      for (size_t j = 0; j < gamma.cols(); j++) res += VORING(x, pos, gamma, n, i, j);
  return res;
}

// ---------------------------------------------------- AoS ring (vortex.h/.cpp)
struct Ring {
  V3 nodes[4];
  V3 nodes0[4];
  double gamma = 0;
};

// ForEachSegment: start = nodes[(i+1)%4], end = nodes[i] (src/vortex.h:132-140)
// VortexRing::BiotSavartLaw (src/vortex.cpp:41-50)
inline V3 RingBiotSavart(const Ring& v, const V3& pos, double gamma) {
  V3 res;
  for (int i = 0; i < 4; i++) res += BiotSavartLaw(v.nodes[(i + 1) % 4], v.nodes[i], pos);
  return res * gamma;
}
// src/vortex.cpp:52-65
inline V3 RingChordwiseBiotSavart(const Ring& v, const V3& pos, double gamma) {
  V3 res;
  const int idx[2] = {0, 2};
  for (int i : idx) res += BiotSavartLaw(v.nodes[(i + 1) % 4], v.nodes[i], pos);
  return res * gamma;
}
// src/vortex.cpp:82-87
inline V3 RingNormal(const Ring& v) {
  return normalized(cross(v.nodes[1] - v.nodes[3], v.nodes[2] - v.nodes[0]));
}
// src/vortex.cpp:89-94
inline V3 RingTangent(const Ring& v) {
  return normalized((v.nodes[1] - v.nodes[3]) + (v.nodes[2] - v.nodes[0]));
}
// src/vortex.cpp:98-104
inline V3 RingCentroid(const Ring& v) {
  return (v.nodes[0] + v.nodes[1] + v.nodes[2] + v.nodes[3]) / 4;
}
inline V3 RingRefCentroid(const Ring& v) {
  return (v.nodes0[0] + v.nodes0[1] + v.nodes0[2] + v.nodes0[3]) / 4;
}
// src/vortex.cpp:132-138
inline double RingArea(const Ring& v) {
  V3 u1 = v.nodes[1] - v.nodes[0];
  V3 u2 = v.nodes[3] - v.nodes[0];
  V3 v1 = v.nodes[3] - v.nodes[2];
  V3 v2 = v.nodes[1] - v.nodes[2];
  return (norm(cross(u1, u2)) + norm(cross(v1, v2))) / 2;
}

// ------------------------------------------------------------- morphing.cpp
inline double Sine(double amp, double omega, double phase, double t) {
  return amp * std::sin(omega * t + phase);
}

struct Morphing {
  orc_kinematics k{};
  V3 origin() const { return V3(k.origin); }
  double plug(double t) const { return Sine(k.plug_amp, k.plug_omega, k.plug_phase, t); }
  double flap(double t) const { return Sine(k.flap_amp, k.flap_omega, k.flap_phase, t); }
  double twist(const V3& x0, double t) const {
    return (k.twist_amp + k.twist_span_slope * std::fabs(x0.y)) *
           std::sin(k.twist_omega * t + k.twist_phase);
  }
  double bend(const V3& x0, double t) const {
    return (k.bend_cx * x0.x * (1 - x0.x) + k.bend_cy * x0.y * x0.y) *
           std::sin(k.bend_omega * t + k.bend_phase);
  }
  // src/morphing.cpp:54-76: m = attack * flap * twist (Eigen 3x3 products).
  void PrepareMatrix(double m[3][3], const V3& x0, double t) const {
    const double phi = flap(t);
    const double F[3][3] = {{1, 0, 0}, {0, std::cos(phi), -std::sin(phi)},
                            {0, std::sin(phi), std::cos(phi)}};
    const double alpha = k.alpha;
    const double A[3][3] = {{std::cos(alpha), 0, std::sin(alpha)}, {0, 1, 0},
                            {-std::sin(alpha), 0, std::cos(alpha)}};
    const double beta = twist(x0, t);
    const double T[3][3] = {{std::cos(beta), 0, std::sin(beta)}, {0, 1, 0},
                            {-std::sin(beta), 0, std::cos(beta)}};
    double AF[3][3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) AF[i][j] = A[i][0] * F[0][j] + A[i][1] * F[1][j] + A[i][2] * F[2][j];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) m[i][j] = AF[i][0] * T[0][j] + AF[i][1] * T[1][j] + AF[i][2] * T[2][j];
  }
  // src/morphing.cpp:23-43
  V3 Perfome(const V3& x0, double t) const {
    V3 x_ref = x0 - origin();
    const bool is_negative = x_ref.y < 0;
    if (is_negative) x_ref.y *= -1;
    double T[3][3];
    PrepareMatrix(T, x_ref, t);
    const double gamma_z = plug(t);
    const double gamma_b = bend(x_ref, t);
    const V3 v(x_ref.x, x_ref.y, x_ref.z + gamma_b);
    V3 x(T[0][0] * v.x + T[0][1] * v.y + T[0][2] * v.z,
         T[1][0] * v.x + T[1][1] * v.y + T[1][2] * v.z,
         T[2][0] * v.x + T[2][1] * v.y + T[2][2] * v.z);
    x = V3(0, 0, gamma_z) + x;
    if (x_ref.y == 0) x.y = 0;
    if (is_negative) x.y *= -1;
    return x + origin();
  }
  // src/morphing.cpp:45-52 (central difference, default h = 1e-6).
  V3 Velocity(const V3& x0, double t, double h = 1e-6) const {
    const V3 x1 = Perfome(x0, t - h);
    const V3 x2 = Perfome(x0, t + h);
    return (x2 - x1) / (2 * h);
  }
};

// ------------------------------------------------------------ dense solve
// Complete-pivoting LU with the semantics of Eigen::FullPivLU<MatrixXd>:
// P A Q = L U, pivot = largest |a_ij| of the trailing block, solve through
// L, U and the two permutations.  Row-major storage.  The elimination is
// resumable one column at a time (Step), so that a timed run can be cut into
// slices.  threads > 1 splits the pivot search (each thread keeps the first
// maximum of its row block in row-major order; blocks are merged in order, so
// the pivot is the serial one) and the row updates (independent per row):
// the result is bit-identical to the single-threaded elimination, which is
// the default because Eigen's FullPivLU is single-threaded.
struct FullPivLU {
  std::vector<double>* A = nullptr;
  size_t n = 0;
  std::vector<size_t> rp, cp;
  int threads = 1;
  bool singular = false;

  void Init(std::vector<double>& a, size_t nn, int th = 1) {
    A = &a;
    n = nn;
    threads = th;
    singular = false;
    rp.resize(n);
    cp.resize(n);
    for (size_t i = 0; i < n; i++) rp[i] = cp[i] = i;
  }

  // Elimination of column k; false once the trailing block is zero.
  bool Step(size_t k) {
    if (singular) return false;
    std::vector<double>& M = *A;
    size_t pi = k, pj = k;
    double best = -1;
    // The first maximum of |a_ij| in row-major order: per row a vectorised
    // max (as Eigen's packet maxCoeff), then the first column attaining it
    // when the row beats every earlier row (the same pivot as a scalar scan).
    auto search = [&](size_t i0, size_t i1, double& b, size_t& bi, size_t& bj) {
      for (size_t i = i0; i < i1; i++) {
        const double* row = &M[i * n];
        double m = -1;
#pragma omp simd reduction(max : m)
        for (size_t j = k; j < n; j++) m = std::max(m, std::fabs(row[j]));
        if (m > b) {
          size_t j = k;
          while (std::fabs(row[j]) != m) j++;
          b = m; bi = i; bj = j;
        }
      }
    };
#ifdef _OPENMP
    if (threads > 1 && n - k >= 64) {
      const int T = threads;
      std::vector<double> tb(T, -1);
      std::vector<size_t> ti(T, k), tj(T, k);
#pragma omp parallel num_threads(T)
      {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        const size_t rows = n - k;
        search(k + rows * t / nt, k + rows * (t + 1) / nt, tb[t], ti[t], tj[t]);
      }
      for (int t = 0; t < T; t++)
        if (tb[t] > best) { best = tb[t]; pi = ti[t]; pj = tj[t]; }
    } else {
      search(k, n, best, pi, pj);
    }
#else
    search(k, n, best, pi, pj);
#endif
    if (best == 0) { singular = true; return false; }
    if (pi != k) {
      for (size_t j = 0; j < n; j++) std::swap(M[k * n + j], M[pi * n + j]);
      std::swap(rp[k], rp[pi]);
    }
    if (pj != k) {
      for (size_t i = 0; i < n; i++) std::swap(M[i * n + k], M[i * n + pj]);
      std::swap(cp[k], cp[pj]);
    }
    const double piv = M[k * n + k];
    const double* rowk = &M[k * n];
    auto update = [&](size_t i) {
      double* rowi = &M[i * n];
      const double l = rowi[k] / piv;
      rowi[k] = l;
      if (l != 0) {
#pragma omp simd
        for (size_t j = k + 1; j < n; j++) rowi[j] -= l * rowk[j];
      }
    };
#ifdef _OPENMP
    if (threads > 1 && n - k >= 64) {
#pragma omp parallel for num_threads(threads) schedule(static)
      for (long long i = (long long)k + 1; i < (long long)n; i++) update((size_t)i);
    } else {
      for (size_t i = k + 1; i < n; i++) update(i);
    }
#else
    for (size_t i = k + 1; i < n; i++) update(i);
#endif
    return true;
  }

  void Solve(const std::vector<double>& b, std::vector<double>& x) const {
    const std::vector<double>& M = *A;
    std::vector<double> y(n);
    for (size_t i = 0; i < n; i++) y[i] = b[rp[i]];
    for (size_t i = 0; i < n; i++) {
      double s = y[i];
      const double* row = &M[i * n];
      for (size_t j = 0; j < i; j++) s -= row[j] * y[j];
      y[i] = s;
    }
    for (size_t ii = n; ii-- > 0;) {
      double s = y[ii];
      const double* row = &M[ii * n];
      for (size_t j = ii + 1; j < n; j++) s -= row[j] * y[j];
      y[ii] = s / row[ii];
    }
    x.assign(n, 0);
    for (size_t i = 0; i < n; i++) x[cp[i]] = y[i];
  }
};

int FullPivLUSolve(std::vector<double>& A, size_t n, const std::vector<double>& b, std::vector<double>& x,
                   int threads = 1) {
  FullPivLU lu;
  lu.Init(A, n, threads);
  for (size_t k = 0; k < n; k++)
    if (!lu.Step(k)) break;
  if (lu.singular) return 1;
  lu.Solve(b, x);
  return 0;
}

// --------------------------------------------------------------- advect.*
struct SimState;

// src/advect.h:26-46: velocity at every wake node, TE row forced to -ff.
void SheetVelocity(Sheet<V3>* result, const Sheet<V3>& wing_pos, const Sheet<double>& wing_gamma,
                   const Sheet<V3>& wake_pos, const Sheet<double>& wake_gamma, const V3& ff) {
  result->resize(wake_pos);
  const long long K_n = (long long)wake_pos.size();
#pragma omp parallel for schedule(dynamic, 16)
  for (long long K = 0; K < K_n; K++) {
    (*result)[K] = -ff + InducedVelocity(wake_pos[K], wing_pos, wing_gamma) +
                   InducedVelocity(wake_pos[K], wake_pos, wake_gamma);
  }
  for (size_t n = 0; n < result->num(); n++)
    if (result->rows() > 0)
      for (size_t j = 0; j < result->cols(); j++) result->at(n, 0, j) = -ff;
}

// Velocity with the moved wake as source (src/advect.cpp:40-46, 54-63).
static void StageVelocity(Sheet<V3>* k, const Sheet<V3>& pos, const Sheet<V3>& wing_pos,
                          const Sheet<double>& wing_gamma, const Sheet<double>& wake_gamma,
                          const V3& ff) {
  SheetVelocity(k, wing_pos, wing_gamma, pos, wake_gamma, ff);
}

struct Advection {
  virtual ~Advection() = default;
  virtual void Advect(Sheet<V3>* next, const Sheet<V3>& wing_pos, const Sheet<double>& wing_gamma,
                      const Sheet<V3>& wake_pos, const Sheet<double>& wake_gamma, const V3& ff,
                      double dt) = 0;
  virtual void Reset() {}
};

// src/advect.cpp:11-22
struct Euler : Advection {
  Sheet<V3> vel;
  void Advect(Sheet<V3>* next, const Sheet<V3>& wing_pos, const Sheet<double>& wing_gamma,
              const Sheet<V3>& wake_pos, const Sheet<double>& wake_gamma, const V3& ff,
              double dt) override {
    SheetVelocity(&vel, wing_pos, wing_gamma, wake_pos, wake_gamma, ff);
    for (size_t K = 0; K < wake_pos.size(); K++) (*next)[K] = wake_pos[K] + vel[K] * dt;
  }
};

// src/advect.cpp:24-80 (Euler for rows i <= ignore_steps_, src/advect.h:77).
struct RK2 : Advection {
  size_t ignore;
  Sheet<V3> k1, k2, pos1, pos2;
  explicit RK2(size_t s = 5) : ignore(s) {}
  void Advect(Sheet<V3>* next, const Sheet<V3>& wing_pos, const Sheet<double>& wing_gamma,
              const Sheet<V3>& wake_pos, const Sheet<double>& wake_gamma, const V3& ff,
              double dt) override {
    pos1 = wake_pos;
    StageVelocity(&k1, pos1, wing_pos, wing_gamma, wake_gamma, ff);
    pos2.resize(wake_pos);
    for (size_t K = 0; K < wake_pos.size(); K++) pos2[K] = wake_pos[K] + k1[K] * dt;
    StageVelocity(&k2, pos2, wing_pos, wing_gamma, wake_gamma, ff);
    for (size_t n = 0; n < wake_pos.num(); n++)
      for (size_t i = 0; i < wake_pos.rows(); i++)
        for (size_t j = 0; j < wake_pos.cols(); j++) {
          const size_t K = wake_pos.index(n, i, j);
          if (i > ignore)
            (*next)[K] = wake_pos[K] + (k1[K] + k2[K]) * dt / 2;
          else
            (*next)[K] = wake_pos[K] + k1[K] * dt;
        }
  }
};

// src/advect.cpp:82-179.  The update uses k3 twice and never k4 (:173).
struct RK4 : Advection {
  size_t ignore;
  Sheet<V3> k1, k2, k3, k4, pos, pos4;
  explicit RK4(size_t s = 5) : ignore(s) {}
  void Advect(Sheet<V3>* next, const Sheet<V3>& wing_pos, const Sheet<double>& wing_gamma,
              const Sheet<V3>& wake_pos, const Sheet<double>& wake_gamma, const V3& ff,
              double dt) override {
    pos = wake_pos;
    StageVelocity(&k1, pos, wing_pos, wing_gamma, wake_gamma, ff);
    for (size_t K = 0; K < wake_pos.size(); K++) pos[K] = wake_pos[K] + k1[K] * dt / 2;
    StageVelocity(&k2, pos, wing_pos, wing_gamma, wake_gamma, ff);
    for (size_t K = 0; K < wake_pos.size(); K++) pos[K] = wake_pos[K] + k2[K] * dt / 2;
    StageVelocity(&k3, pos, wing_pos, wing_gamma, wake_gamma, ff);
    for (size_t K = 0; K < wake_pos.size(); K++) pos[K] = wake_pos[K] + k3[K] * dt;
    StageVelocity(&k4, pos, wing_pos, wing_gamma, wake_gamma, ff);
    for (size_t n = 0; n < wake_pos.num(); n++)
      for (size_t i = 0; i < wake_pos.rows(); i++)
        for (size_t j = 0; j < wake_pos.cols(); j++) {
          const size_t K = wake_pos.index(n, i, j);
          if (i > ignore)
            (*next)[K] = wake_pos[K] + (k1[K] + k2[K] * 2 + k3[K] * 2 + k3[K]) * dt / 6;
          else
            (*next)[K] = wake_pos[K] + k1[K] * dt;
        }
  }
};

// src/advect.cpp:181-217.  First call Euler; afterwards v(n,i,j) pairs with
// v_prev(n,i-1,j); row i=0 does next += v*dt on the aliased input.
struct AB2 : Advection {
  Sheet<V3> v, v_prev;
  void Reset() override { v_prev = Sheet<V3>(); }
  void Advect(Sheet<V3>* next, const Sheet<V3>& wing_pos, const Sheet<double>& wing_gamma,
              const Sheet<V3>& wake_pos, const Sheet<double>& wake_gamma, const V3& ff,
              double dt) override {
    SheetVelocity(&v, wing_pos, wing_gamma, wake_pos, wake_gamma, ff);
    if (v_prev.size() == 0) {
      for (size_t K = 0; K < wake_pos.size(); K++) (*next)[K] = wake_pos[K] + v[K] * dt;
    } else {
      for (size_t n = 0; n < wake_pos.num(); n++)
        for (size_t i = 0; i < wake_pos.rows(); i++)
          for (size_t j = 0; j < wake_pos.cols(); j++) {
            if (i >= 1) {
              next->at(n, i, j) =
                  wake_pos.at(n, i, j) + (v.at(n, i, j) * 3 - v_prev.at(n, i - 1, j)) * dt / 2;
            } else {
              next->at(n, i, j) += v.at(n, i, j) * dt;
            }
          }
    }
    v_prev = v;
  }
};

std::unique_ptr<Advection> AdvectFactory(const std::string& name) {
  // src/advect_factory.cpp:22-27, 43-60
  if (name == "euler") return std::unique_ptr<Advection>(new Euler);
  if (name == "RK2") return std::unique_ptr<Advection>(new RK2);
  if (name == "RK4") return std::unique_ptr<Advection>(new RK4);
  if (name == "AB2") return std::unique_ptr<Advection>(new AB2);
  return nullptr;
}

// ------------------------------------------------------------ joukowski.*
struct VortexLine {
  V3 p0, p1, p0_init, p1_init;
  double gamma;
};

// src/calc_load/joukowski.cpp:12-34 (TE segment of the last row skipped).
std::vector<VortexLine> GetLines(const Sheet<V3>& pos, const Sheet<V3>& pos_init,
                                 const Sheet<double>& gamma, size_t n) {
  std::vector<VortexLine> res;
  for (size_t i = 0; i < gamma.rows(); i++)
    for (size_t j = 0; j < gamma.cols(); j++) {
      const V3 c[4] = {pos.at(n, i, j), pos.at(n, i, j + 1), pos.at(n, i + 1, j + 1), pos.at(n, i + 1, j)};
      const V3 c0[4] = {pos_init.at(n, i, j), pos_init.at(n, i, j + 1), pos_init.at(n, i + 1, j + 1),
                        pos_init.at(n, i + 1, j)};
      for (size_t k = 0; k < 4; k++) {
        if (i == pos.rows() - 1 - 1 && k == 2) continue;
        res.push_back(VortexLine{c[k], c[(k + 1) % 4], c0[k], c0[(k + 1) % 4], gamma.at(n, i, j)});
      }
    }
  return res;
}

// src/calc_load/joukowski.cpp:55-67
std::vector<double> CalcPanelArea(const Sheet<V3>& pos, size_t n) {
  std::vector<double> res;
  for (size_t i = 0; i + 1 < pos.rows(); i++)
    for (size_t j = 0; j + 1 < pos.cols(); j++)
      res.push_back(norm(cross(pos.at(n, i + 1, j) - pos.at(n, i, j), pos.at(n, i, j + 1) - pos.at(n, i, j))));
  return res;
}

// ------------------------------------------------------- SimpleSimulator
// generator: 0 RectGenerator, 1 NACA4digitGenerator(digit), 2 NACA00XXGenerator(digit)
struct WingInfo {
  double chord, span;
  size_t rows, cols;
  V3 origin;
  Morphing morphing;
  int cheb_chord, cheb_span;
  int generator = 0, digit = 0;
};

// src/util.h:36-43
std::vector<double> linspace(double a, double b, size_t N) {
  const double dx = (b - a) / (N - 1);
  std::vector<double> res;
  for (size_t i = 0; i < N; i++) res.push_back(a + i * dx);
  return res;
}

// src/wing/rect.h:16-25
std::vector<double> TransformChebyshev(size_t N, double xmin, double xmax) {
  auto theta = linspace(-M_PI_2, 0, N);
  std::vector<double> res;
  for (double t : theta) res.push_back(xmin + (xmax - xmin) * std::cos(t));
  res.front() = xmin;
  res.back() = xmax;
  return res;
}

// src/wing/rect.cpp:18-45
std::vector<V3> RectGenerate(double chord, double span, size_t rows, size_t cols, int cc, int cs) {
  std::vector<double> xs = cc ? TransformChebyshev(rows + 1, 0, chord) : linspace(0, chord, rows + 1);
  std::vector<double> ys = cs ? TransformChebyshev(cols + 1, 0, span) : linspace(0, span, cols + 1);
  std::vector<V3> pts;
  for (double x : xs)
    for (double y : ys) pts.emplace_back(x, y, 0.0);
  return pts;
}

// src/wing/naca4digit.cpp:12-27: mean camber line of a 4-digit NACA section
// (only the first two digits matter: m = first/100, p = second/10).
double NACA4digit(double x, double c, int xx) {
  const int first = xx / 10;
  const int second = xx % 10;
  const double m = first / 100.0;
  const double p = second / 10.0;
  double res = 0;
  if (0 <= x && x <= p * c) {
    res = m * x / p / p * (2 * p - x / c);
  } else if (p * c <= x && x <= c) {
    res = m * (c - x) / (1 - p) / (1 - p) * (1 + x / c - 2 * p);
  }
  return res;
}

// src/wing/naca00XX.cpp:14-19: half thickness of a symmetric 4-digit section.
double NACA00XX(double x, double c, int xx) {
  const double t = xx * 0.01;
  const double z = x / c;
  return 5 * t * c * (0.2969 * std::sqrt(z) + (-0.1260) * (z) + (-0.3516) * z * z + 0.2843 * z * z * z +
                      (-0.1015) * z * z * z * z);
}

// WingGenerator::Generate of the three generators: the rectangular lattice
// (src/wing/rect.cpp:18-45), then z = NACA4digit(x) (src/wing/naca4digit.cpp:29-39)
// or z = NACA00XX(x) (src/wing/naca00XX.cpp:21-32) at every point.
std::vector<V3> GenerateWing(int generator, int digit, double chord, double span, size_t rows, size_t cols, int cc,
                             int cs) {
  auto pts = RectGenerate(chord, span, rows, cols, cc, cs);
  if (generator == 1)
    for (auto& p : pts) p.z = NACA4digit(p.x, chord, digit);
  if (generator == 2)
    for (auto& p : pts) p.z = NACA00XX(p.x, chord, digit);
  return pts;
}

// src/wing/wing.cpp:12-52: per row, mirrored half reversed then the half
// without its first point; finally + origin.
std::vector<V3> WholeWing(const std::vector<V3>& half, size_t half_cols, const V3& origin) {
  const size_t COLS = half_cols + 1;
  const size_t ROWS = half.size() / COLS;
  std::vector<V3> whole;
  for (size_t i = 0; i < ROWS; i++) {
    std::vector<V3> row(half.begin() + i * COLS, half.begin() + (i + 1) * COLS);
    std::vector<V3> mirror(COLS);
    for (size_t j = 0; j < COLS; j++) { mirror[j] = row[j]; mirror[j].y *= -1; }
    whole.insert(whole.end(), mirror.rbegin(), mirror.rend());
    whole.insert(whole.end(), row.begin() + 1, row.end());
  }
  for (auto& p : whole) p += origin;
  return whole;
}

// src/simulator/simple_simulator.cpp:19-32
std::vector<V3> CollocationPoints(const Sheet<V3>& pos) {
  std::vector<V3> res;
  for (size_t n = 0; n < pos.num(); n++)
    for (size_t i = 0; i + 1 < pos.rows(); i++)
      for (size_t j = 0; j + 1 < pos.cols(); j++)
        res.push_back((pos.at(n, i, j) + pos.at(n, i + 1, j) + pos.at(n, i + 1, j + 1) + pos.at(n, i, j + 1)) / 4);
  return res;
}

// src/simulator/simple_simulator.cpp:34-50
std::vector<V3> Normals(const Sheet<V3>& pos) {
  std::vector<V3> res;
  for (size_t n = 0; n < pos.num(); n++)
    for (size_t i = 0; i + 1 < pos.rows(); ++i)
      for (size_t j = 0; j + 1 < pos.cols(); ++j)
        res.push_back(normalized(cross(pos.at(n, i + 1, j + 1) - pos.at(n, i, j),
                                       pos.at(n, i, j + 1) - pos.at(n, i + 1, j))));
  return res;
}

struct Simulator {
  std::vector<WingInfo> info;
  std::vector<Morphing> morphings;
  Sheet<V3> wing_pos, wing_pos_init, wake_pos;
  Sheet<double> wing_gamma, wing_gamma_prev, wake_gamma;
  V3 ff;
  std::unique_ptr<Advection> advection;
  long long erase_after = 0;
  bool built = false;
  int lu_threads = 1;  // FullPivLU threads (1 = Eigen's single-threaded elimination)

  // src/simulator/simple_simulator.cpp:126-140
  int AddWing(const WingInfo& w) {
    if (!info.empty() && (info.back().rows != w.rows || info.back().cols != w.cols)) return 2;
    if ((w.cols & 1) != 0) return 3;
    info.push_back(w);
    return 0;
  }

  // src/simulator/simple_simulator.cpp:142-169
  void BuildWing() {
    const size_t num = info.size(), rows = info.back().rows, cols = info.back().cols;
    wing_pos.resize(num, rows + 1, cols + 1);
    wing_pos_init.resize(num, rows + 1, cols + 1);
    wing_gamma.resize(num, rows, cols);
    wing_gamma_prev.resize(num, rows, cols);
    morphings.clear();
    size_t n = 0;
    for (const auto& w : info) {
      Morphing m = w.morphing;
      w.origin.store(m.k.origin);
      morphings.push_back(m);
      auto half = GenerateWing(w.generator, w.digit, w.chord, w.span / 2, w.rows, w.cols / 2, w.cheb_chord,
                               w.cheb_span);
      auto pts = WholeWing(half, w.cols / 2, V3());
      for (auto& p : pts) p = p + w.origin;
      std::copy(pts.begin(), pts.end(), wing_pos_init.sheet_begin(n));
      ++n;
    }
  }

  // src/simulator/simple_simulator.cpp:288-303 (up to the step loop)
  int Begin() {
    if (info.empty()) return 4;
    BuildWing();
    wake_pos.resize(wing_pos.num(), 0, wing_pos.cols());
    wake_gamma.resize(wing_gamma.num(), 0, wing_gamma.cols());
    if (!advection) advection.reset(new Euler);
    advection->Reset();
    built = true;
    return 0;
  }

  V3 Velocity(const V3& x) const {
    return -ff + InducedVelocity(x, wing_pos, wing_gamma) + InducedVelocity(x, wake_pos, wake_gamma);
  }

  // src/simulator/simple_simulator.cpp:76-101
  std::vector<double> CalcMatrix(const std::vector<V3>& cpos, const std::vector<V3>& normal,
                                 size_t stride = 1) const {
    const size_t N = wing_gamma.size();
    std::vector<double> A(stride == 1 ? N * N : 0);
    Sheet<double> gamma(wing_gamma);
    std::fill(gamma.data().begin(), gamma.data().end(), 1.0);
    double sink = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : sink)
    for (long long K = 0; K < (long long)N; K += (long long)stride) {
      const V3& cp = cpos[K];
      const V3& nl = normal[K];
      size_t L = 0;
      for (size_t nn = 0; nn < gamma.num(); nn++)
        for (size_t ii = 0; ii < gamma.rows(); ii++)
          for (size_t jj = 0; jj < gamma.cols(); jj++, L++) {
            const double a = dot(VORING(cp, wing_pos, gamma, nn, ii, jj), nl);
            if (stride == 1) A[K * N + L] = a; else sink += a;
          }
    }
    (void)sink;
    return A;
  }

  // src/simulator/simple_simulator.cpp:103-124
  std::vector<double> CalcRhs(const std::vector<V3>& cpos, const std::vector<V3>& cpos_init,
                              const std::vector<V3>& normal, double t, size_t stride = 1) const {
    const size_t N = wing_gamma.size();
    const size_t per = wing_gamma.rows() * wing_gamma.cols();
    std::vector<double> res(N, 0.0);
#pragma omp parallel for schedule(dynamic, 4)
    for (long long K = 0; K < (long long)N; K += (long long)stride) {
      const size_t n = (size_t)K / per;
      const V3 Uw = InducedVelocity(cpos[K], wake_pos, wake_gamma);
      const V3 Uls = morphings[n].Velocity(cpos_init[K], t);
      const V3 u = Uw - (Uls + ff);
      res[K] = -dot(u, normal[K]);
    }
    return res;
  }

  // src/simulator/simple_simulator.cpp:171-188
  void Shed(size_t step) {
    std::vector<V3> te_pos;
    for (size_t n = 0; n < wing_pos.num(); n++)
      for (size_t j = 0; j < wing_pos.cols(); j++) te_pos.push_back(wing_pos.at(n, wing_pos.rows() - 1, j));
    wake_pos.prepend_row(te_pos);
    if (step > 0) {
      std::vector<double> te_gamma;
      for (size_t n = 0; n < wing_gamma.num(); n++)
        for (size_t j = 0; j < wing_gamma.cols(); j++)
          te_gamma.push_back(wing_gamma.at(n, wing_gamma.rows() - 1, j));
      wake_gamma.prepend_row(te_gamma);
    }
  }

  // src/simulator/simple_simulator.cpp:195-233
  V3 LoadLineVelocity(const VortexLine& line, size_t n, double t) const {
    const V3 mp = (line.p0 + line.p1) / 2;
    const V3 mp_init = (line.p0_init + line.p1_init) / 2;
    return Velocity(mp) - morphings[n].Velocity(mp_init, t);
  }
  // JoukowskiSteady + JoukowskiUnsteady of wing n from its line velocities U.
  void LoadSums(size_t n, const std::vector<VortexLine>& lines, const V3* U, const std::vector<V3>& normal,
                double dt, double* row) const {
    const auto area = CalcPanelArea(wing_pos, n);
    // JoukowskiSteady (src/calc_load/joukowski.cpp:36-53)
    double Fx = 0, Fy = 0, Fz = 0;
    for (size_t i = 0; i < lines.size(); i++) {
      const V3 df = cross(U[i], lines[i].p1 - lines[i].p0) * lines[i].gamma;
      Fx += df.x; Fy += df.y; Fz += df.z;
    }
    // JoukowskiUnsteady range form (src/calc_load/joukowski.h:132-148)
    double Gx = 0, Gy = 0, Gz = 0;
    const size_t off = wing_gamma.index(n, 0, 0);
    const size_t cnt = wing_gamma.rows() * wing_gamma.cols();
    for (size_t k = 0; k < cnt; k++) {
      const double g = wing_gamma[off + k], gp = wing_gamma_prev[off + k];
      const double dg_dt = (g - gp) / dt;
      const V3 df = normal[off + k] * dg_dt * area[k];
      Gx += df.x; Gy += df.y; Gz += df.z;
    }
    const V3 F = V3(Fx, Fy, Fz) + V3(Gx, Gy, Gz);
    const double Q = norm(ff);
    const double S = info[n].chord * info[n].span;
    const V3 C = F / (0.5 * Q * Q * S);
    if (row) { row[1 + 2 * n] = C.x; row[2 + 2 * n] = C.z; }
  }

  void CalcLoad(const std::vector<V3>& normal, double t, double dt, double* row,
                size_t stride = 1) const {
    if (row) row[0] = t;
    for (size_t n = 0; n < wing_pos.num(); n++) {
      const auto lines = GetLines(wing_pos, wing_pos_init, wing_gamma, n);
      std::vector<V3> U(lines.size());
#pragma omp parallel for schedule(dynamic, 8)
      for (long long i = 0; i < (long long)lines.size(); i += (long long)stride)
        U[i] = LoadLineVelocity(lines[i], n, t);
      LoadSums(n, lines, U.data(), normal, dt, row);
    }
  }

  // src/simulator/simple_simulator.cpp:240-286 (+ the erase of :307-311)
  int MainLoop(size_t step, double dt, double* row) {
    const double t = step * dt;
    wing_gamma_prev = wing_gamma;
    for (size_t n = 0; n < wing_pos.num(); n++) {
      const V3* src = wing_pos_init.sheet_begin(n);
      V3* dst = wing_pos.sheet_begin(n);
      const size_t cnt = wing_pos.rows() * wing_pos.cols();
      for (size_t k = 0; k < cnt; k++) dst[k] = morphings[n].Perfome(src[k], t);
    }
    Shed(step);
    const auto cpos = CollocationPoints(wing_pos);
    const auto cpos_init = CollocationPoints(wing_pos_init);
    const auto normal = Normals(wing_pos);
    auto A = CalcMatrix(cpos, normal);
    auto rhs = CalcRhs(cpos, cpos_init, normal, t);
    std::vector<double> g;
    if (FullPivLUSolve(A, rhs.size(), rhs, g, lu_threads)) return 5;
    for (size_t K = 0; K < wing_gamma.size(); K++) wing_gamma[K] = g[K];
    CalcLoad(normal, t, dt, row);
    advection->Advect(&wake_pos, wing_pos, wing_gamma, wake_pos, wake_gamma, ff, dt);
    if (erase_after > 0 && (long long)step >= erase_after) {
      wake_pos.erase_last_row();
      wake_gamma.erase_last_row();
    }
    return 0;
  }
  // ---- MainLoop(step, dt) cut into slices ------------------------------------
  // The CPU reference timing runs one MainLoop at full size as a sequence of
  // slices of about equal estimated time (one slice per timed bench step).
  // The loop is broken into work items -- the kinematics and shed, row ranges
  // of CalcMatrix and CalcRhs, single columns of the FullPivLU elimination,
  // its substitutions, ranges of load lines, ranges of wake nodes of each
  // advection stage, the updates -- which evaluate the same expressions as
  // MainLoop for every output element, so running all slices in order is
  // exactly MainLoop(step, dt).  Euler and RK2 advection are cut into node
  // ranges; RK4 and AB2 run as one item.
  enum SliceKind { kKin, kMat, kRhs, kLu, kLuSolve, kLoadPrep, kLoadVel, kLoadFin, kAdvPrep, kAdvVel1, kAdvMid,
                   kAdvVel2, kAdvEnd, kAdvAll, kErase };
  struct SliceItem {
    int kind;
    size_t a, b;
    double cost;
  };
  struct SlicedLoop {
    size_t step = 0;
    double dt = 0, t = 0;
    int scheme = 0;  // 0 Euler, 1 RK2, 2 other (one item)
    size_t rk_ignore = 5;
    std::vector<SliceItem> items;
    std::vector<size_t> first;  // first item of every slice, then items.size()
    size_t next_slice = 0;
    std::vector<V3> cpos, cpos_init, normal;
    std::vector<double> A, rhs, g;
    FullPivLU lu;
    std::vector<std::vector<VortexLine>> lines;
    std::vector<size_t> line_off;
    std::vector<V3> U;
    Sheet<V3> k1, k2, pos2;
    double* row = nullptr;
    bool failed = false;
  } sl;

  // Plans MainLoop(step, dt) in `slices` slices; `threads` is the OpenMP
  // thread count the N-body items run with (for the time estimate only).
  int SlicedBegin(size_t step, double dt, size_t slices, int threads) {
    if (!built || slices < 1) return 4;
    SlicedLoop& L = sl;
    L = SlicedLoop();
    L.step = step;
    L.dt = dt;
    L.t = step * dt;
    if (auto* e = dynamic_cast<Euler*>(advection.get())) { (void)e; L.scheme = 0; }
    else if (auto* r = dynamic_cast<RK2*>(advection.get())) { L.scheme = 1; L.rk_ignore = r->ignore; }
    else L.scheme = 2;
    // sizes after the shed of this step
    const size_t num = wing_gamma.num(), N = wing_gamma.size();
    const size_t wake_rings = num * (wake_gamma.rows() + (step > 0 ? 1 : 0)) * wing_gamma.cols();
    const size_t wake_nodes = num * (wake_pos.rows() + 1) * wake_pos.cols();
    const size_t lines = num * (4 * wing_gamma.rows() * wing_gamma.cols() - wing_gamma.cols());
    // estimated seconds: one FP64 segment evaluation ~18 ns on one thread;
    // one elimination element (pivot search + update) ~1.2 ns on one thread
    const double seg = 18e-9 / std::max(threads, 1), elem = 1.2e-9 / std::max(lu_threads, 1);
    auto add = [&](int kind, size_t a, size_t b, double cost) { L.items.push_back(SliceItem{kind, a, b, cost}); };
    auto ranges = [&](int kind, size_t n, size_t chunk, double per) {
      for (size_t a = 0; a < n; a += chunk) add(kind, a, std::min(n, a + chunk), per * (double)(std::min(n, a + chunk) - a));
    };
    add(kKin, 0, 0, 1e-4);
    ranges(kMat, N, 16, seg * 4.0 * N);
    ranges(kRhs, N, 64, seg * 4.0 * wake_rings);
    for (size_t k = 0; k < N; k++) add(kLu, k, k + 1, elem * (double)(N - k) * (double)(N - k));
    add(kLuSolve, 0, 0, 2e-9 * (double)N * (double)N);
    add(kLoadPrep, 0, 0, 1e-4);
    ranges(kLoadVel, lines, 64, seg * 4.0 * (N + wake_rings));
    add(kLoadFin, 0, 0, 1e-4);
    const double per_node = seg * 4.0 * (N + wake_rings);
    if (L.scheme == 2) {
      add(kAdvAll, 0, 0, per_node * wake_nodes * 4.0);
    } else {
      add(kAdvPrep, 0, 0, 1e-5);
      ranges(kAdvVel1, wake_nodes, 64, per_node);
      add(kAdvMid, 0, 0, 1e-5);
      if (L.scheme == 1) ranges(kAdvVel2, wake_nodes, 64, per_node);
      add(kAdvEnd, 0, 0, 1e-5);
    }
    add(kErase, 0, 0, 1e-6);
    double total = 0;
    for (const auto& it : L.items) total += it.cost;
    L.first.push_back(0);
    double acc = 0;
    for (size_t q = 0; q < L.items.size(); q++) {
      acc += L.items[q].cost;
      if (L.first.size() < slices && acc >= total * (double)L.first.size() / (double)slices && q + 1 < L.items.size())
        L.first.push_back(q + 1);
    }
    while (L.first.size() < slices) L.first.push_back(L.items.size());
    L.first.push_back(L.items.size());
    return 0;
  }

  void SliceItemRun(const SliceItem& it) {
    SlicedLoop& L = sl;
    const size_t N = wing_gamma.size();
    switch (it.kind) {
      case kKin: {
        wing_gamma_prev = wing_gamma;
        for (size_t n = 0; n < wing_pos.num(); n++) {
          const V3* src = wing_pos_init.sheet_begin(n);
          V3* dst = wing_pos.sheet_begin(n);
          const size_t cnt = wing_pos.rows() * wing_pos.cols();
          for (size_t k = 0; k < cnt; k++) dst[k] = morphings[n].Perfome(src[k], L.t);
        }
        Shed(L.step);
        L.cpos = CollocationPoints(wing_pos);
        L.cpos_init = CollocationPoints(wing_pos_init);
        L.normal = Normals(wing_pos);
        L.A.assign(N * N, 0.0);
        L.rhs.assign(N, 0.0);
        break;
      }
      case kMat: {  // CalcMatrix rows (src/simulator/simple_simulator.cpp:76-101)
        Sheet<double> gamma(wing_gamma);
        std::fill(gamma.data().begin(), gamma.data().end(), 1.0);
#pragma omp parallel for schedule(dynamic, 4)
        for (long long K = (long long)it.a; K < (long long)it.b; K++) {
          size_t Lc = 0;
          for (size_t nn = 0; nn < gamma.num(); nn++)
            for (size_t ii = 0; ii < gamma.rows(); ii++)
              for (size_t jj = 0; jj < gamma.cols(); jj++, Lc++)
                L.A[K * N + Lc] = dot(VORING(L.cpos[K], wing_pos, gamma, nn, ii, jj), L.normal[K]);
        }
        break;
      }
      case kRhs: {  // CalcRhs rows (:103-124)
        const size_t per = wing_gamma.rows() * wing_gamma.cols();
#pragma omp parallel for schedule(dynamic, 4)
        for (long long K = (long long)it.a; K < (long long)it.b; K++) {
          const size_t n = (size_t)K / per;
          const V3 Uw = InducedVelocity(L.cpos[K], wake_pos, wake_gamma);
          const V3 Uls = morphings[n].Velocity(L.cpos_init[K], L.t);
          const V3 u = Uw - (Uls + ff);
          L.rhs[K] = -dot(u, L.normal[K]);
        }
        break;
      }
      case kLu:
        if (it.a == 0) L.lu.Init(L.A, N, lu_threads);
        L.lu.Step(it.a);
        break;
      case kLuSolve:
        if (L.lu.singular) { L.failed = true; break; }
        L.lu.Solve(L.rhs, L.g);
        for (size_t K = 0; K < N; K++) wing_gamma[K] = L.g[K];
        break;
      case kLoadPrep: {
        L.lines.clear();
        L.line_off.assign(1, 0);
        for (size_t n = 0; n < wing_pos.num(); n++) {
          L.lines.push_back(GetLines(wing_pos, wing_pos_init, wing_gamma, n));
          L.line_off.push_back(L.line_off.back() + L.lines.back().size());
        }
        L.U.assign(L.line_off.back(), V3());
        break;
      }
      case kLoadVel: {
#pragma omp parallel for schedule(dynamic, 8)
        for (long long q = (long long)it.a; q < (long long)it.b; q++) {
          size_t n = 0;
          while ((size_t)q >= L.line_off[n + 1]) n++;
          L.U[q] = LoadLineVelocity(L.lines[n][q - L.line_off[n]], n, L.t);
        }
        break;
      }
      case kLoadFin:
        if (L.row) L.row[0] = L.t;
        for (size_t n = 0; n < wing_pos.num(); n++) LoadSums(n, L.lines[n], L.U.data() + L.line_off[n], L.normal, L.dt, L.row);
        break;
      case kAdvPrep:
        L.k1.resize(wake_pos);
        break;
      case kAdvVel1: {  // advect::Velocity of the wake nodes (src/advect.h:26-46)
#pragma omp parallel for schedule(dynamic, 16)
        for (long long K = (long long)it.a; K < (long long)it.b; K++)
          L.k1[K] = -ff + InducedVelocity(wake_pos[K], wing_pos, wing_gamma) +
                    InducedVelocity(wake_pos[K], wake_pos, wake_gamma);
        break;
      }
      case kAdvMid: {
        for (size_t n = 0; n < L.k1.num(); n++)
          if (L.k1.rows() > 0)
            for (size_t j = 0; j < L.k1.cols(); j++) L.k1.at(n, 0, j) = -ff;
        if (L.scheme == 1) {  // RK2 (src/advect.cpp:24-80): the whole wake moved to pos2
          L.pos2.resize(wake_pos);
          for (size_t K = 0; K < wake_pos.size(); K++) L.pos2[K] = wake_pos[K] + L.k1[K] * L.dt;
          L.k2.resize(L.pos2);
        }
        break;
      }
      case kAdvVel2: {
#pragma omp parallel for schedule(dynamic, 16)
        for (long long K = (long long)it.a; K < (long long)it.b; K++)
          L.k2[K] = -ff + InducedVelocity(L.pos2[K], wing_pos, wing_gamma) +
                    InducedVelocity(L.pos2[K], L.pos2, wake_gamma);
        break;
      }
      case kAdvEnd: {
        if (L.scheme == 0) {  // Euler (src/advect.cpp:11-22)
          for (size_t K = 0; K < wake_pos.size(); K++) wake_pos[K] = wake_pos[K] + L.k1[K] * L.dt;
          break;
        }
        for (size_t n = 0; n < L.k2.num(); n++)
          if (L.k2.rows() > 0)
            for (size_t j = 0; j < L.k2.cols(); j++) L.k2.at(n, 0, j) = -ff;
        for (size_t n = 0; n < wake_pos.num(); n++)
          for (size_t i = 0; i < wake_pos.rows(); i++)
            for (size_t j = 0; j < wake_pos.cols(); j++) {
              const size_t K = wake_pos.index(n, i, j);
              if (i > L.rk_ignore)
                wake_pos[K] = wake_pos[K] + (L.k1[K] + L.k2[K]) * L.dt / 2;
              else
                wake_pos[K] = wake_pos[K] + L.k1[K] * L.dt;
            }
        break;
      }
      case kAdvAll:
        advection->Advect(&wake_pos, wing_pos, wing_gamma, wake_pos, wake_gamma, ff, L.dt);
        break;
      case kErase:
        if (erase_after > 0 && (long long)L.step >= erase_after) {
          wake_pos.erase_last_row();
          wake_gamma.erase_last_row();
        }
        break;
      default:
        break;
    }
  }

  // Runs slice `s` (slices run in order 0, 1, ...); the load row is written
  // by the slice that finishes the loads.  0, or 5 if the matrix is singular,
  // 6 if out of order.
  int SlicedRun(size_t s, double* row) {
    SlicedLoop& L = sl;
    if (s != L.next_slice || s + 1 >= L.first.size()) return 6;
    L.row = row;
    for (size_t q = L.first[s]; q < L.first[s + 1]; q++) {
      SliceItemRun(L.items[q]);
      if (L.failed) return 5;
    }
    L.next_slice++;
    return 0;
  }
};

}  // namespace orc

using namespace orc;

namespace {
Ring LoadRing(const double* p, double gamma = 0) {
  Ring r;
  for (int k = 0; k < 4; k++) r.nodes[k] = r.nodes0[k] = V3(p + 3 * k);
  r.gamma = gamma;
  return r;
}
void StoreRing(const Ring& r, double* p) {
  for (int k = 0; k < 4; k++) r.nodes[k].store(p + 3 * k);
}
Morphing MakeMorphing(const orc_kinematics* k) {
  Morphing m;
  if (k) m.k = *k;
  return m;
}
Sheet<V3> SheetFrom(const double* p, size_t num, size_t rows, size_t cols) {
  Sheet<V3> s(num, rows, cols);
  for (size_t k = 0; k < s.size(); k++) s[k] = V3(p + 3 * k);
  return s;
}
Sheet<double> GammaFrom(const double* p, size_t num, size_t rows, size_t cols) {
  Sheet<double> s(num, rows, cols);
  if (p) std::memcpy(s.data().data(), p, sizeof(double) * s.size());
  return s;
}
}  // namespace

extern "C" {

void orc_biot_savart(const double start[3], const double end[3], const double pos[3], double out[3]) {
  BiotSavartLaw(V3(start), V3(end), V3(pos)).store(out);
}

double orc_distance_line_and_point(const double start[3], const double end[3], const double pos[3]) {
  return DistanceLineAndPoint(V3(start), V3(end), V3(pos));
}

void orc_voring(const double* pos, int64_t pnum, int64_t prows, int64_t pcols, const double* gamma,
                int64_t grows, int64_t gcols, int64_t n, int64_t i, int64_t j, const double x[3],
                double out[3]) {
  auto P = SheetFrom(pos, pnum, prows, pcols);
  auto G = GammaFrom(gamma, pnum, grows, gcols);
  VORING(V3(x), P, G, n, i, j).store(out);
}

void orc_sheet_induced_velocity(const double* pos, int64_t pnum, int64_t prows, int64_t pcols,
                                const double* gamma, int64_t grows, int64_t gcols,
                                const double* targets, int64_t n_targets, double* out) {
  auto P = SheetFrom(pos, pnum, prows, pcols);
  auto G = GammaFrom(gamma, pnum, grows, gcols);
#pragma omp parallel for schedule(dynamic, 8)
  for (long long t = 0; t < (long long)n_targets; t++)
    InducedVelocity(V3(targets + 3 * t), P, G).store(out + 3 * t);
}

void orc_ring_biot_savart(const double nodes[12], double gamma, const double pos[3], double out[3]) {
  RingBiotSavart(LoadRing(nodes), V3(pos), gamma).store(out);
}

void orc_ring_chordwise_biot_savart(const double nodes[12], double gamma, const double pos[3],
                                    double out[3]) {
  RingChordwiseBiotSavart(LoadRing(nodes), V3(pos), gamma).store(out);
}

void orc_ring_vector(const double nodes[12], double gamma, int what, double out[3]) {
  Ring r = LoadRing(nodes, gamma);
  V3 v;
  switch (what) {
    case 0: v = RingNormal(r); break;
    case 1: v = RingTangent(r); break;
    case 2: v = cross(RingNormal(r), RingTangent(r)); break;               // vortex.cpp:96
    case 3: v = RingCentroid(r); break;
    case 4: v = normalized(r.nodes[1] - r.nodes[0]); break;                // vortex.cpp:106-110
    case 5: v = normalized(r.nodes[3] - r.nodes[0]); break;                // vortex.cpp:112-116
    case 6: v = RingNormal(r) * gamma * RingArea(r) * (-1); break;          // vortex.cpp:140-143
    default: break;
  }
  v.store(out);
}

double orc_ring_scalar(const double nodes[12], int what) {
  Ring r = LoadRing(nodes);
  switch (what) {
    case 0: return RingArea(r);
    case 1: return norm(r.nodes[0] - r.nodes[1]);  // CalcC vortex.cpp:124-126
    case 2: return norm(r.nodes[0] - r.nodes[3]);  // CalcB vortex.cpp:128-130
    default: return 0;
  }
}

double orc_ring_angle_of_attack(const double nodes[12], const double Q[3]) {
  // src/vortex.cpp:118-122
  Ring r = LoadRing(nodes);
  return std::atan2(dot(V3(Q), RingNormal(r)), dot(V3(Q), RingTangent(r)));
}

void orc_vortex_impulse(const double* rings, const double* gammas, int64_t n, double out[3]) {
  // CalcVortexImpulse (calc_impulse_main.cpp:34-41): sum of VortexRing::Impulse()
  // = Normal() * gamma * Area() * (-1) (vortex.cpp:140-143)
  V3 res;
  for (int64_t k = 0; k < n; k++) {
    Ring r = LoadRing(rings + 12 * k, gammas[k]);
    res += RingNormal(r) * gammas[k] * RingArea(r) * (-1);
  }
  res.store(out);
}

void orc_lamb_vector(const double* panels, const double* panel_gamma, const double* v_nodes, int64_t n_panels,
                     const double* freestreams, const double* vortices, const double* vortex_gamma,
                     int64_t n_vortices, double out[3]) {
  // CalcLambVectorOnPanel (calc_impulse.h:15-30), summed over the panels as
  // calc_impulse_main.cpp:79-82 does: for each segment (ForEachSegment order,
  // start = nodes[k+1], end = nodes[k]) ue = v_node[k] + u(mid) - freestream_i,
  // res += (ue x dl) * gamma with u the velocity of every vortex
  // (InducedVelocityByVortices, uvlm_vortex_ring.cpp:13-22).
  std::vector<Ring> vort(n_vortices);
  for (int64_t k = 0; k < n_vortices; k++) vort[k] = LoadRing(vortices + 12 * k, vortex_gamma[k]);
  V3 res;
  for (int64_t i = 0; i < n_panels; i++) {
    Ring p = LoadRing(panels + 12 * i, panel_gamma[i]);
    const V3 fs(freestreams + 3 * i);
    V3 acc;
    for (int k = 0; k < 4; k++) {
      const V3 start = p.nodes[(k + 1) % 4], end = p.nodes[k];
      const V3 dl = end - start;
      const V3 pos = (start + end) / 2;
      V3 u;
      for (const auto& v : vort) u += RingBiotSavart(v, pos, v.gamma);
      const V3 ue = V3(v_nodes + 12 * i + 3 * k) + u - fs;
      acc += cross(ue, dl) * panel_gamma[i];
    }
    res += acc;
  }
  res.store(out);
}

void orc_rings_induced_velocity(const double* rings, const double* gammas, int64_t n_rings,
                                const double pos[3], int chordwise_only, double out[3]) {
  // src/shed.inl:22-33, 66-77
  V3 res;
  for (int64_t k = 0; k < n_rings; k++) {
    Ring r = LoadRing(rings + 12 * k);
    res += chordwise_only ? RingChordwiseBiotSavart(r, V3(pos), gammas[k])
                          : RingBiotSavart(r, V3(pos), gammas[k]);
  }
  res.store(out);
}

void orc_rings_advect(const double* vortex_rings, const double* vortex_gamma, int64_t n_vortex,
                      double* wake_rings, int64_t n_wake, const double freestream[3], double dt,
                      int parallel) {
  // src/shed.inl:8-19 (AdvectKernel), :43-49 (Advect), :52-64 (AdvectParallel)
  std::vector<Ring> src(n_vortex);
  for (int64_t k = 0; k < n_vortex; k++) src[k] = LoadRing(vortex_rings + 12 * k, vortex_gamma[k]);
  const V3 fs(freestream);
  auto kernel = [&](int64_t w) {
    Ring r = LoadRing(wake_rings + 12 * w);
    for (int q = 0; q < 4; q++) {
      V3 vel;
      for (const auto& s : src) vel += RingBiotSavart(s, r.nodes[q], s.gamma);
      vel += fs;
      r.nodes[q] += vel * dt;
    }
    StoreRing(r, wake_rings + 12 * w);
  };
  if (parallel) {
#pragma omp parallel for
    for (long long w = 0; w < (long long)n_wake; w++) kernel(w);
  } else {
    for (int64_t w = 0; w < n_wake; w++) kernel(w);
  }
}

void orc_connect_trailing_edge(const double* edge_rings, int64_t n_edge, double* wake_rings) {
  // src/shed.inl:79-86: wake.nodes[0] = edge.nodes[1]; wake.nodes[3] = edge.nodes[2]
  for (int64_t k = 0; k < n_edge; k++) {
    std::memcpy(wake_rings + 12 * k + 0, edge_rings + 12 * k + 3, 3 * sizeof(double));
    std::memcpy(wake_rings + 12 * k + 9, edge_rings + 12 * k + 6, 3 * sizeof(double));
  }
}

// src/linear.inl:14-32 (CalcMatrix), :34-45 (FreeStream), :47-61 (Wake),
// :63-104 (Morphing, per container), :113-157 (SolveLinearProblem).  Ring k
// moves with morphs[kin_of[k]].
static int SolveRings(const double* bound_rings, const double* bound_rings0, int64_t n_bound,
                      const double* wake_rings, const double* wake_gamma, int64_t n_wake,
                      const double freestream[3], const std::vector<Morphing>& morphs,
                      const std::vector<int>& kin_of, double t, int drop_wake_term, double* gamma_out) {
  std::vector<Ring> b(n_bound);
  for (int64_t k = 0; k < n_bound; k++) {
    b[k] = LoadRing(bound_rings + 12 * k);
    if (bound_rings0)
      for (int q = 0; q < 4; q++) b[k].nodes0[q] = V3(bound_rings0 + 12 * k + 3 * q);
  }
  const size_t n = (size_t)n_bound;
  std::vector<double> A(n * n);
  for (size_t i = 0; i < n; i++)
    for (size_t j = 0; j < n; j++)
      A[i * n + j] = dot(RingBiotSavart(b[j], RingCentroid(b[i]), 1.), RingNormal(b[i]));
  std::vector<double> rhs(n);
  for (size_t i = 0; i < n; i++) {
    const double morph = dot(morphs[kin_of[i]].Velocity(RingRefCentroid(b[i]), t), RingNormal(b[i]));
    const double fs = dot(V3(freestream), RingNormal(b[i]));
    rhs[i] = morph - fs;
    if (!drop_wake_term) {
      V3 w;
      for (int64_t k = 0; k < n_wake; k++)
        w += RingBiotSavart(LoadRing(wake_rings + 12 * k), RingCentroid(b[i]), wake_gamma[k]);
      rhs[i] -= dot(w, RingNormal(b[i]));
    }
  }
  std::vector<double> x;
  if (FullPivLUSolve(A, n, rhs, x)) return 1;
  std::memcpy(gamma_out, x.data(), n * sizeof(double));
  return 0;
}

int orc_solve_linear_problem(const double* bound_rings, const double* bound_rings0, int64_t n_bound,
                             const double* wake_rings, const double* wake_gamma, int64_t n_wake,
                             const double freestream[3], const orc_kinematics* mk, double t,
                             int drop_wake_term, double* gamma_out) {
  return SolveRings(bound_rings, bound_rings0, n_bound, wake_rings, wake_gamma, n_wake, freestream,
                    {MakeMorphing(mk)}, std::vector<int>((size_t)n_bound, 0), t, drop_wake_term, gamma_out);
}

int orc_solve_linear_problem_containers(const double* bound_rings, const double* bound_rings0,
                                        const int64_t* container_rings, int n_containers,
                                        const orc_kinematics* kins, const double* wake_rings,
                                        const double* wake_gamma, int64_t n_wake, const double freestream[3],
                                        double t, int drop_wake_term, double* gamma_out) {
  std::vector<Morphing> morphs;
  std::vector<int> kin_of;
  for (int c = 0; c < n_containers; c++) {
    morphs.push_back(MakeMorphing(kins + c));
    kin_of.insert(kin_of.end(), (size_t)container_rings[c], c);
  }
  return SolveRings(bound_rings, bound_rings0, (int64_t)kin_of.size(), wake_rings, wake_gamma, n_wake,
                    freestream, morphs, kin_of, t, drop_wake_term, gamma_out);
}

void orc_load_katz_plotkin(const double* rings, const double* gamma, const double* gamma_prev, int64_t rows,
                           int64_t cols, const orc_kinematics* mk, const double* bound_rings,
                           const double* bound_gamma, int64_t n_bound, const double* wake_rings,
                           const double* wake_gamma, int64_t n_wake, const double freestream[3], double rho,
                           double t, double dt, double out[5]) {
  // CalcLoadKatzPlotkin (src/calc_load/katz_plotkin.cpp:16-68) with
  // CalcLocalLiftSt / CalcLocalDragSt (katz_plotkin.h:21-34), CalcUm and
  // CalcProjectionOperator (functions.h:14-31), DeltaGamma / Grad
  // (vortex_container.h:87-96).  F starts from zero.
  const Morphing m = MakeMorphing(mk);
  const V3 fs(freestream);
  V3 F;
  double Pin = 0;
  auto g = [&](int64_t i, int64_t j) { return gamma[i * cols + j]; };
  auto gp = [&](int64_t i, int64_t j) { return gamma_prev[i * cols + j]; };
  for (int64_t i = 0; i < rows; i++) {
    for (int64_t j = 0; j < cols; j++) {
      const Ring v = LoadRing(rings + 12 * (i * cols + j));
      const V3 centroid = RingCentroid(v);
      const double db = norm(v.nodes[0] - v.nodes[3]);
      const double dc = norm(v.nodes[0] - v.nodes[1]);
      const V3 Um = fs - m.Velocity(centroid, t);
      const V3 uh = normalized(Um);
      const V3 n = RingNormal(v);
      const V3 Pn = n - uh * dot(uh, n);  // (I - u u^T) n
      const double alpha = std::atan2(dot(Um, n), dot(Um, RingTangent(v)));
      V3 Uw, Ubc;
      for (int64_t k = 0; k < n_wake; k++)
        Uw += RingBiotSavart(LoadRing(wake_rings + 12 * k), centroid, wake_gamma[k]);
      for (int64_t k = 0; k < n_bound; k++)
        Ubc += RingChordwiseBiotSavart(LoadRing(bound_rings + 12 * k), centroid, bound_gamma[k]);
      const double dg = g(i, j) - (i == 0 ? 0.0 : g(i - 1, j));
      const V3 grad = RingTangent(v) * dg / dc;
      const double Lst = rho * dot(Um + Uw, grad) * db * dc * std::cos(alpha);
      const double Dst = rho * (-dot(Um + Ubc, Pn) * dg * db);
      double dg_dt = (g(i, j) - gp(i, j)) / dt;
      if (i > 0) dg_dt += (g(i - 1, j) - gp(i - 1, j)) / dt;
      dg_dt /= 2;
      const double Lunst = rho * dg_dt * db * dc * std::cos(alpha);
      const double Dunst = rho * dg_dt * db * dc * std::sin(alpha);
      const V3 dF = Um / norm(Um) * (Dst + Dunst) + Pn * (Lst + Lunst);
      F += dF;
      Pin += (-1) * dot(Um, n) * dot(dF, n);
    }
  }
  F.store(out);
  out[3] = Pin;
  out[4] = 0;
}

void orc_load_joukowski_rings(const double* rings, const double* rings0, const double* gamma,
                              const double* gamma_prev, int64_t rows, int64_t cols, const orc_kinematics* mk,
                              const double* vortices, const double* vortex_gamma, int64_t n_vortices,
                              const double freestream[3], double rho, double t, double dt, double out[5]) {
  // CalcLoadJoukowski (src/calc_load/joukowski.h:24-104): steady part per
  // segment with U = u_ind(mid) + CalcUm(mid0) (the trailing-edge segment of
  // the last row skipped), unsteady part Normal rho dG/dt B C, Pin = sum dF .
  // Vls(reference centroid), Pout = -Fx |freestream|.
  const Morphing m = MakeMorphing(mk);
  const V3 fs(freestream);
  std::vector<Ring> pool(n_vortices);
  for (int64_t k = 0; k < n_vortices; k++) pool[k] = LoadRing(vortices + 12 * k, vortex_gamma[k]);
  V3 F;
  double Pin = 0;
  for (int64_t i = 0; i < rows; i++) {
    for (int64_t j = 0; j < cols; j++) {
      const int64_t K = i * cols + j;
      Ring v = LoadRing(rings + 12 * K, gamma[K]);
      for (int q = 0; q < 4; q++) v.nodes0[q] = V3(rings0 + 12 * K + 3 * q);
      V3 st;
      for (int q = 0; q < 4; q++) {
        if (i + 1 == rows && q == 1) continue;
        const V3 a = v.nodes[(q + 1) % 4], b = v.nodes[q];
        const V3 mid = (a + b) / 2, mid0 = (v.nodes0[(q + 1) % 4] + v.nodes0[q]) / 2;
        V3 uind;
        for (const auto& r : pool) uind += RingBiotSavart(r, mid, r.gamma);
        const V3 U = uind + (fs - m.Velocity(mid0, t));
        st += cross(U, b - a) * rho * v.gamma;
      }
      const double B = norm(v.nodes[0] - v.nodes[3]), Cc = norm(v.nodes[0] - v.nodes[1]);
      const V3 unst = RingNormal(v) * rho * ((gamma[K] - gamma_prev[K]) / dt) * B * Cc;
      const V3 dF = st + unst;
      F += dF;
      Pin += dot(dF, m.Velocity(RingRefCentroid(v), t));
    }
  }
  F.store(out);
  out[3] = Pin;
  out[4] = F.x * norm(fs) * (-1);
}

void orc_calc_morphing_velocity_on_wing(const double* rings, const double* rings0, int64_t n,
                                        const orc_kinematics* mk, double t, double* out) {
  // src/linear.inl:78-90
  Morphing m = MakeMorphing(mk);
  for (int64_t k = 0; k < n; k++) {
    Ring r = LoadRing(rings + 12 * k);
    for (int q = 0; q < 4; q++) r.nodes0[q] = V3(rings0 + 12 * k + 3 * q);
    out[k] = dot(m.Velocity(RingRefCentroid(r), t), RingNormal(r));
  }
}

void orc_kin_perfome(const orc_kinematics* mk, const double x0[3], double t, double out[3]) {
  MakeMorphing(mk).Perfome(V3(x0), t).store(out);
}

void orc_kin_velocity(const orc_kinematics* mk, const double x0[3], double t, double h, double out[3]) {
  MakeMorphing(mk).Velocity(V3(x0), t, h).store(out);
}

void orc_calc_um(const orc_kinematics* mk, const double x0[3], const double freestream[3], double t,
                 double out[3]) {
  // src/calc_load/functions.h:23-30
  (V3(freestream) - MakeMorphing(mk).Velocity(V3(x0), t)).store(out);
}

void orc_transform_chebyshev(int64_t N, double xmin, double xmax, double* out) {
  auto v = TransformChebyshev(N, xmin, xmax);
  std::memcpy(out, v.data(), sizeof(double) * v.size());
}

void orc_rect_generate(double chord, double span, int64_t rows, int64_t cols, int cc, int cs, double* out) {
  auto v = RectGenerate(chord, span, rows, cols, cc, cs);
  for (size_t k = 0; k < v.size(); k++) v[k].store(out + 3 * k);
}

void orc_whole_wing(const double* half, int64_t rows, int64_t half_cols, const double origin[3], double* out) {
  std::vector<V3> h((rows + 1) * (half_cols + 1));
  for (size_t k = 0; k < h.size(); k++) h[k] = V3(half + 3 * k);
  auto w = WholeWing(h, half_cols, V3(origin));
  for (size_t k = 0; k < w.size(); k++) w[k].store(out + 3 * k);
}

int orc_fullpiv_lu_solve(double* A, int64_t n, const double* b, double* x) {
  std::vector<double> a(A, A + n * n), bb(b, b + n), xx;
  const int rc = FullPivLUSolve(a, n, bb, xx);
  std::memcpy(A, a.data(), sizeof(double) * n * n);
  if (rc == 0) std::memcpy(x, xx.data(), sizeof(double) * n);
  return rc;
}

void* orc_sim_create(void) { return new Simulator(); }
void orc_sim_destroy(void* s) { delete static_cast<Simulator*>(s); }

int orc_sim_add_wing(void* s, double chord, double span, int64_t rows, int64_t cols, const double origin[3],
                     const orc_kinematics* m, int cc, int cs) {
  WingInfo w{chord, span, (size_t)rows, (size_t)cols, V3(origin), MakeMorphing(m), cc, cs};
  return static_cast<Simulator*>(s)->AddWing(w);
}

int orc_sim_add_wing_generator(void* s, int generator, int digit, double chord, double span, int64_t rows,
                               int64_t cols, const double origin[3], const orc_kinematics* m, int cc, int cs) {
  if (generator < 0 || generator > 2) return 1;
  WingInfo w{chord, span, (size_t)rows, (size_t)cols, V3(origin), MakeMorphing(m), cc, cs, generator, digit};
  return static_cast<Simulator*>(s)->AddWing(w);
}

double orc_naca4digit(double x, double c, int xx) { return NACA4digit(x, c, xx); }
double orc_naca00xx(double x, double c, int xx) { return NACA00XX(x, c, xx); }

void orc_generate_wing(int generator, int digit, double chord, double span, int64_t rows, int64_t cols, int cc,
                       int cs, double* out) {
  auto v = GenerateWing(generator, digit, chord, span, rows, cols, cc, cs);
  for (size_t k = 0; k < v.size(); k++) v[k].store(out + 3 * k);
}

void orc_sim_set_lu_threads(void* s, int threads) { static_cast<Simulator*>(s)->lu_threads = threads > 1 ? threads : 1; }

int orc_sim_sliced_begin(void* s, int64_t step, double dt, int64_t slices, int threads) {
  return static_cast<Simulator*>(s)->SlicedBegin((size_t)step, dt, (size_t)std::max<int64_t>(slices, 1), threads);
}

int orc_sim_sliced_run(void* s, int64_t slice, double* load_row) {
  return static_cast<Simulator*>(s)->SlicedRun((size_t)slice, load_row);
}

void orc_sim_set_forward_flight(void* s, const double ff[3]) { static_cast<Simulator*>(s)->ff = V3(ff); }

int orc_sim_set_advection(void* s, const char* name) {
  auto a = AdvectFactory(name ? name : "");
  if (!a) return 1;
  static_cast<Simulator*>(s)->advection = std::move(a);
  return 0;
}

void orc_sim_set_erase_wake_after(void* s, int64_t step) { static_cast<Simulator*>(s)->erase_after = step; }

void orc_sim_set_threads(void*, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
}

int orc_sim_begin(void* s) { return static_cast<Simulator*>(s)->Begin(); }

int orc_sim_step(void* s, int64_t step, double dt, double* row) {
  auto* sim = static_cast<Simulator*>(s);
  if (!sim->built) return 4;
  return sim->MainLoop((size_t)step, dt, row);
}

void orc_sim_sizes(void* s, int64_t* num, int64_t* rows, int64_t* cols, int64_t* wake_rows) {
  auto* sim = static_cast<Simulator*>(s);
  *num = sim->wing_gamma.num();
  *rows = sim->wing_gamma.rows();
  *cols = sim->wing_gamma.cols();
  *wake_rows = sim->wake_gamma.rows();
}

int64_t orc_sim_wake_node_rows(void* s) { return static_cast<Simulator*>(s)->wake_pos.rows(); }

void orc_sim_get_state(void* s, double* wing_pos, double* wing_pos_init, double* wake_pos, double* wing_gamma,
                       double* wing_gamma_prev, double* wake_gamma) {
  auto* sim = static_cast<Simulator*>(s);
  auto put = [](const Sheet<V3>& sh, double* p) {
    if (p) for (size_t k = 0; k < sh.size(); k++) sh[k].store(p + 3 * k);
  };
  auto putg = [](const Sheet<double>& sh, double* p) {
    if (p && sh.size()) std::memcpy(p, sh.data().data(), sizeof(double) * sh.size());
  };
  put(sim->wing_pos, wing_pos);
  put(sim->wing_pos_init, wing_pos_init);
  put(sim->wake_pos, wake_pos);
  putg(sim->wing_gamma, wing_gamma);
  putg(sim->wing_gamma_prev, wing_gamma_prev);
  putg(sim->wake_gamma, wake_gamma);
}

int orc_sim_set_state(void* s, int64_t wake_rows, const double* wing_pos, const double* wake_pos,
                      const double* wing_gamma, const double* wing_gamma_prev, const double* wake_gamma) {
  auto* sim = static_cast<Simulator*>(s);
  if (!sim->built) return 4;
  const size_t num = sim->wing_gamma.num(), cols = sim->wing_gamma.cols();
  for (size_t k = 0; k < sim->wing_pos.size(); k++) sim->wing_pos[k] = V3(wing_pos + 3 * k);
  sim->wake_pos = SheetFrom(wake_pos, num, wake_rows + 1, cols + 1);
  std::memcpy(sim->wing_gamma.data().data(), wing_gamma, sizeof(double) * sim->wing_gamma.size());
  std::memcpy(sim->wing_gamma_prev.data().data(), wing_gamma_prev, sizeof(double) * sim->wing_gamma.size());
  sim->wake_gamma = GammaFrom(wake_gamma, num, wake_rows, cols);
  sim->advection->Reset();
  return 0;
}

int orc_sim_time_step_sampled(void* s, int64_t step, double dt, int64_t stride, int64_t lu_n,
                              double* sec) {
  using clk = std::chrono::steady_clock;
  auto* base = static_cast<Simulator*>(s);
  if (!base->built) return 4;
  Simulator sim;  // work on a copy; the advection stage is timed on the copy
  sim.info = base->info;
  sim.morphings = base->morphings;
  sim.wing_pos = base->wing_pos; sim.wing_pos_init = base->wing_pos_init; sim.wake_pos = base->wake_pos;
  sim.wing_gamma = base->wing_gamma; sim.wing_gamma_prev = base->wing_gamma_prev;
  sim.wake_gamma = base->wake_gamma;
  sim.ff = base->ff;
  const size_t st = stride > 0 ? (size_t)stride : 1;
  const double t = step * dt;
  auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };

  auto t0 = clk::now();
  sim.wing_gamma_prev = sim.wing_gamma;
  for (size_t n = 0; n < sim.wing_pos.num(); n++) {
    const V3* src = sim.wing_pos_init.sheet_begin(n);
    V3* dst = sim.wing_pos.sheet_begin(n);
    for (size_t k = 0; k < sim.wing_pos.rows() * sim.wing_pos.cols(); k++) dst[k] = sim.morphings[n].Perfome(src[k], t);
  }
  sim.Shed(step);
  const auto cpos = CollocationPoints(sim.wing_pos);
  const auto cpos_init = CollocationPoints(sim.wing_pos_init);
  const auto normal = Normals(sim.wing_pos);
  auto t1 = clk::now();
  sec[0] = secs(t0, t1);
  sim.CalcMatrix(cpos, normal, st);
  auto t2 = clk::now();
  sec[1] = secs(t1, t2) * st;
  sim.CalcRhs(cpos, cpos_init, normal, t, st);
  auto t3 = clk::now();
  sec[2] = secs(t2, t3) * st;
  // FullPivLU on the leading lu_n x lu_n block of a full-size-like matrix.
  const size_t N = sim.wing_gamma.size();
  size_t ln = lu_n > 0 ? std::min((size_t)lu_n, N) : N;
  std::vector<double> Asub(ln * ln), bsub(ln, 1.0), xsub;
  {
    // leading block of the influence matrix, assembled without timing
    Sheet<double> one(sim.wing_gamma);
    std::fill(one.data().begin(), one.data().end(), 1.0);
#pragma omp parallel for
    for (long long K = 0; K < (long long)ln; K++) {
      size_t L = 0;
      for (size_t nn = 0; nn < one.num() && L < ln; nn++)
        for (size_t ii = 0; ii < one.rows() && L < ln; ii++)
          for (size_t jj = 0; jj < one.cols() && L < ln; jj++, L++)
            Asub[K * ln + L] = dot(VORING(cpos[K], sim.wing_pos, one, nn, ii, jj), normal[K]);
    }
  }
  auto t4 = clk::now();
  FullPivLUSolve(Asub, ln, bsub, xsub);
  auto t5 = clk::now();
  const double scale = std::pow((double)N / (double)ln, 3.0);
  sec[3] = secs(t4, t5) * scale;
  sim.CalcLoad(normal, t, dt, nullptr, st);
  auto t6 = clk::now();
  sec[4] = secs(t5, t6) * st;
  // advection: velocity evaluations on every st-th wake node
  {
    const size_t stages = dynamic_cast<Euler*>(base->advection.get()) ? 1
                          : dynamic_cast<RK2*>(base->advection.get()) ? 2
                          : dynamic_cast<RK4*>(base->advection.get()) ? 4 : 1;
    auto t7 = clk::now();
    double sink = 0;
    for (size_t sgi = 0; sgi < stages; sgi++) {
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : sink)
      for (long long K = 0; K < (long long)sim.wake_pos.size(); K += (long long)st) {
        const V3 u = -sim.ff + InducedVelocity(sim.wake_pos[K], sim.wing_pos, sim.wing_gamma) +
                     InducedVelocity(sim.wake_pos[K], sim.wake_pos, sim.wake_gamma);
        sink += u.x;
      }
    }
    (void)sink;
    auto t8 = clk::now();
    sec[5] = secs(t7, t8) * st;
  }
  return 0;
}

}  // extern "C"
