// shore_oracle.cpp - CPU FP64 oracle for cs_dmri's SHORE fit.
//
// TEST INFRASTRUCTURE.  This file restates, in plain C++17 and IEEE double,
// the reference algorithm of the masked-voxel 3D-SHORE fit so that the CUDA
// product can be checked against it.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load it; the product library never does.
//
// Every function names the reference file:line it follows (paths inside the
// cs_dmri project).  The reference is Rust (nalgebra 0.33.3 for dense linear
// algebra); where nalgebra supplies the arithmetic (SVD for sigma_max,
// Cholesky, gemv) the oracle uses textbook algorithms with the same
// mathematical result: cyclic Jacobi eigenvalues of M^T M for sigma_max^2,
// an LL^T Cholesky with forward/back substitution, and sequential dot products.
// Built with -ffp-contract=off so no product is fused into an FMA.

#include "shore_oracle.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <utility>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;
using Vec = std::vector<double>;

// Row-major dense matrix.
struct Mat {
  int rows = 0, cols = 0;
  Vec a;
  Mat() = default;
  Mat(int r, int c) : rows(r), cols(c), a(static_cast<size_t>(r) * c, 0.0) {}
  double& operator()(int i, int j) { return a[static_cast<size_t>(i) * cols + j]; }
  double operator()(int i, int j) const { return a[static_cast<size_t>(i) * cols + j]; }
};

void set_err(char* err, size_t len, const std::string& msg) {
  if (err && len > 0) {
    std::snprintf(err, len, "%s", msg.c_str());
  }
}

// ---------------------------------------------------------------- math.rs

double gamma_fn(double x);

// factorial: exact table for n <= 20, gamma(n + 1) above (math.rs:8-37).
double factorial(uint32_t n) {
  static const double table[21] = {1.0,
                                   1.0,
                                   2.0,
                                   6.0,
                                   24.0,
                                   120.0,
                                   720.0,
                                   5040.0,
                                   40320.0,
                                   362880.0,
                                   3628800.0,
                                   39916800.0,
                                   479001600.0,
                                   6227020800.0,
                                   87178291200.0,
                                   1307674368000.0,
                                   20922789888000.0,
                                   355687428096000.0,
                                   6402373705728000.0,
                                   121645100408832000.0,
                                   2432902008176640000.0};
  if (n < 21) return table[n];
  return gamma_fn(static_cast<double>(n + 1));
}

// Lanczos approximation of Gamma with g = 7 and the nine published Lanczos
// coefficients (Numerical Recipes / Godfrey), reflection below 0.5
// (math.rs:40-64).
double gamma_fn(double x) {
  if (x < 0.5) return kPi / (std::sin(kPi * x) * gamma_fn(1.0 - x));
  const double g = 7.0;
  static const double c[9] = {0.99999999999980993,  676.5203681218851,     -1259.1392167224028,
                              771.32342877765313,   -176.61502916214059,   12.507343278686905,
                              -0.13857109526572012, 9.9843695780195716e-6, 1.5056327351493116e-7};
  x -= 1.0;
  double a = c[0];
  const double t = x + g + 0.5;
  for (int i = 1; i < 9; ++i) a += c[i] / (x + static_cast<double>(i));
  return std::sqrt(2.0 * kPi) * std::pow(t, x + 0.5) * std::exp(-t) * a;
}

// P_l^m(x) with the Condon-Shortley phase by upward recurrence in l
// (math.rs:70-100).
double assoc_legendre(uint32_t l, uint32_t m, double x) {
  double pmm = 1.0;
  if (m > 0) {
    const double somx2 = std::sqrt(std::max((1.0 - x) * (1.0 + x), 0.0));
    double fact = 1.0;
    for (uint32_t i = 0; i < m; ++i) {
      pmm *= -fact * somx2;
      fact += 2.0;
    }
  }
  if (l == m) return pmm;
  double pmmp1 = x * (2.0 * m + 1.0) * pmm;
  if (l == m + 1) return pmmp1;
  double pll = 0.0;
  for (uint32_t ll = m + 2; ll <= l; ++ll) {
    const double llf = ll, mf = m;
    pll = ((2.0 * llf - 1.0) * x * pmmp1 - (llf + mf - 1.0) * pmm) / (llf - mf);
    pmm = pmmp1;
    pmmp1 = pll;
  }
  return pll;
}

// Generalised Laguerre L_n^alpha(x) by three-term recurrence (math.rs:108-124).
double gen_laguerre(uint32_t n, double alpha, double x) {
  if (n == 0) return 1.0;
  double lkm1 = 1.0;
  double lk = 1.0 + alpha - x;
  if (n == 1) return lk;
  for (uint32_t k = 1; k < n; ++k) {
    const double kf = k;
    const double lkp1 = ((2.0 * kf + 1.0 + alpha - x) * lk - (kf + alpha) * lkm1) / (kf + 1.0);
    lkm1 = lk;
    lk = lkp1;
  }
  return lk;
}

// Gauss 2F1 power series, terminating (math.rs:130-145).
double hyp2f1(double a, double b, double c, double z) {
  double sum = 1.0, term = 1.0;
  for (int k = 0; k < 200; ++k) {
    const double kf = k;
    term *= (a + kf) * (b + kf) / ((c + kf) * (kf + 1.0)) * z;
    sum += term;
    if (term == 0.0) break;
    if (std::fabs(term) < 1e-15 * std::max(std::fabs(sum), 1.0)) break;
  }
  return sum;
}

// (x, y, z) -> (r, theta azimuth, phi polar) (math.rs:157-166).
void cart2sphere(double x, double y, double z, double* r, double* theta, double* phi) {
  *r = std::sqrt(x * x + y * y + z * z);
  *theta = std::atan2(y, x);
  *phi = (*r > 0.0) ? std::acos(std::min(std::max(z / *r, -1.0), 1.0)) : 0.0;
}

// -------------------------------------------------------------- qspace.rs

constexpr double kTortoiseGmax = 80e-3;       // qspace.rs:262
constexpr double kGyro = 267.51532e6;         // qspace.rs:265
constexpr double kShellTolerance = 50.0;      // fit.rs:618
constexpr size_t kMinShoreShells = 2;         // fit.rs:615

// TORTOISE (Delta, delta) heuristic from the largest b (qspace.rs:213-227).
void tortoise_deltas(const double* bvals, int n, double gmax, double* big, double* small) {
  double max_b = 0.0;
  for (int i = 0; i < n; ++i) max_b = std::max(max_b, bvals[i]);
  if (max_b <= 0.0) {
    const double small_ms = std::pow(1.0, 1.0 / 3.0);
    *big = 3.0 * small_ms * 1e-3;
    *small = small_ms * 1e-3;
    return;
  }
  const double temp = max_b / kGyro / kGyro / gmax / gmax / 2.0 * 1e6;
  const double small_ms = std::pow(temp, 1.0 / 3.0) * 1000.0;
  const double big_ms = small_ms * 3.0;
  *big = big_ms * 1e-3;
  *small = small_ms * 1e-3;
}

struct Gtab {
  Vec bvals;
  std::vector<std::array<double, 3>> bvecs;
  double big_delta = 0, small_delta = 0, b0_threshold = 50.0;
  int delta_source = 0;  // 0 user, 1 TORTOISE
  int n() const { return static_cast<int>(bvals.size()); }
  double tau() const { return big_delta - small_delta / 3.0; }  // qspace.rs:130-132
  // q = sqrt(b / (4 pi^2 tau)), 0 at b <= threshold (qspace.rs:136-149).
  Vec qvals() const {
    const double denom = 4.0 * kPi * kPi * tau();
    Vec q(bvals.size());
    for (size_t i = 0; i < bvals.size(); ++i)
      q[i] = (bvals[i] <= b0_threshold) ? 0.0 : std::sqrt(bvals[i] / denom);
    return q;
  }
};

// GradientTable::new with the PyO3 b0_threshold override (qspace.rs:90-118,
// python/src/lib.rs:89-105).
Gtab make_gtab(const csd_gtab* g) {
  Gtab t;
  t.bvals.assign(g->bvals, g->bvals + g->n);
  t.bvecs.resize(g->n);
  for (int i = 0; i < g->n; ++i)
    t.bvecs[i] = {g->bvecs[3 * i], g->bvecs[3 * i + 1], g->bvecs[3 * i + 2]};
  if (!std::isnan(g->big_delta) && !std::isnan(g->small_delta)) {
    t.big_delta = g->big_delta;
    t.small_delta = g->small_delta;
    t.delta_source = 0;
  } else {
    tortoise_deltas(g->bvals, g->n, kTortoiseGmax, &t.big_delta, &t.small_delta);
    t.delta_source = 1;
  }
  t.b0_threshold = g->b0_threshold;
  return t;
}

struct Shell {
  double b;
  std::vector<int> idx;
};

// Shell partition: b0 first, then shells by ascending running-mean b; a
// gradient joins the first shell within `tol` (qspace.rs:171-197).
std::vector<Shell> shells(const Vec& bvals, double b0_threshold, double tol) {
  std::vector<Shell> sh;
  Shell b0{0.0, {}};
  for (size_t i = 0; i < bvals.size(); ++i) {
    const double b = bvals[i];
    if (b <= b0_threshold) {
      b0.idx.push_back(static_cast<int>(i));
      continue;
    }
    Shell* slot = nullptr;
    for (auto& s : sh) {
      if (std::fabs(s.b - b) <= tol) {
        slot = &s;
        break;
      }
    }
    if (slot) {
      const double nn = static_cast<double>(slot->idx.size());
      slot->b = (slot->b * nn + b) / (nn + 1.0);
      slot->idx.push_back(static_cast<int>(i));
    } else {
      sh.push_back(Shell{b, {static_cast<int>(i)}});
    }
  }
  std::stable_sort(sh.begin(), sh.end(), [](const Shell& a, const Shell& b) { return a.b < b.b; });
  std::vector<Shell> out;
  if (!b0.idx.empty()) out.push_back(b0);
  for (auto& s : sh) out.push_back(s);
  return out;
}

// Mean b of the non-zero shells (fit.rs:621-623).
Vec dwi_shells(const Gtab& g) {
  Vec out;
  for (auto& s : shells(g.bvals, g.b0_threshold, kShellTolerance))
    if (s.b > 0.0) out.push_back(s.b);
  return out;
}

// ------------------------------------------------------- basis/shore.rs

struct Idx {
  int n, l, m;
};

// Coefficient order: n ascending, even l <= n, m = -l..l (shore.rs:29-44).
std::vector<Idx> shore_indices(int radial_order) {
  std::vector<Idx> v;
  for (int n = 0; n <= radial_order; ++n)
    for (int l = 0; l <= n; l += 2)
      for (int m = -l; m <= l; ++m) v.push_back({n, l, m});
  return v;
}

// kappa = sqrt(2 (n-l)! / (zeta^1.5 Gamma(n + 3/2))) (shore.rs:56-61).
double kappa(double zeta, uint32_t n, uint32_t l) {
  const double num = 2.0 * factorial(n - l);
  const double den = std::pow(zeta, 1.5) * gamma_fn(static_cast<double>(n) + 1.5);
  return std::sqrt(num / den);
}

// Radial function R_nl(q) (shore.rs:64-70).
double shore_radial(uint32_t n, uint32_t l, double q, double zeta) {
  const double u = q * q / zeta;
  const double lag = gen_laguerre(n - l, static_cast<double>(l) + 0.5, u);
  const double env = std::exp(-u * 0.5);
  const double rp = std::pow(u, static_cast<double>(l) / 2.0);
  return kappa(zeta, n, l) * lag * env * rp;
}

// BrainSuite real-SH block of degree l: cosine terms m = l..1, the m = 0
// term, then signed sine terms m = 1..l (shore.rs:76-115).
void brainsuite_sh_block(uint32_t l, double theta, double phi, double* out) {
  if (l == 0) {
    out[0] = 1.0 / std::sqrt(4.0 * kPi);
    return;
  }
  const double cphi = std::cos(phi);
  const double tlp1 = 2.0 * l + 1.0;
  double p[32];
  for (uint32_t k = 0; k <= l; ++k) {
    const double norm = std::sqrt(tlp1 / (4.0 * kPi) * factorial(l - k) / factorial(l + k));
    p[k] = norm * assoc_legendre(l, k, cphi);
  }
  const double s2 = std::sqrt(2.0);
  for (uint32_t k = 1; k <= l; ++k) out[l - k] = s2 * p[k] * std::cos(static_cast<double>(k) * theta);
  out[l] = p[0];
  for (uint32_t k = 1; k <= l; ++k) {
    const double sign = ((k + 1) % 2 == 0) ? 1.0 : -1.0;
    out[l + k] = s2 * sign * p[k] * std::sin(static_cast<double>(k) * theta);
  }
}

// Design matrix M[i, col] = R_nl(q_i) Y_l^k(theta_i, phi_i) (shore.rs:122-178).
Mat design_matrix(const Gtab& g, int radial_order, double zeta) {
  const int rows = g.n();
  const int cols = static_cast<int>(shore_indices(radial_order).size());
  const Vec q = g.qvals();
  Mat m(rows, cols);
  std::vector<double> r(rows), th(rows), ph(rows);
  for (int i = 0; i < rows; ++i) {
    cart2sphere(g.bvecs[i][0] * q[i], g.bvecs[i][1] * q[i], g.bvecs[i][2] * q[i], &r[i], &th[i],
                &ph[i]);
    if (std::isnan(th[i])) th[i] = 0.0;
  }
  int col = 0;
  double blk[64];
  for (int n = 0; n <= radial_order; ++n) {
    for (int l = 0; l <= n; l += 2) {
      const int bs = 2 * l + 1;
      for (int i = 0; i < rows; ++i) {
        const double rad = shore_radial(n, l, r[i], zeta);
        brainsuite_sh_block(l, th[i], ph[i], blk);
        for (int k = 0; k < bs; ++k) m(i, col + k) = rad * blk[k];
      }
      col += bs;
    }
  }
  return m;
}

// Regularisation diagonals N_ii = (n(n+1))^2, L_ii = (l(l+1))^2 (shore.rs:180-195).
void regularization(int radial_order, Vec& nd, Vec& ld) {
  auto idx = shore_indices(radial_order);
  nd.resize(idx.size());
  ld.resize(idx.size());
  for (size_t i = 0; i < idx.size(); ++i) {
    const double nn = static_cast<double>(idx[i].n * (idx[i].n + 1));
    const double ll = static_cast<double>(idx[i].l * (idx[i].l + 1));
    nd[i] = nn * nn;
    ld[i] = ll * ll;
  }
}

// ----------------------------------------------------------------- odf.rs

// Largest even l <= radial order (odf.rs:22-24).
int default_lmax(int radial_order) { return radial_order - (radial_order % 2); }

// (lmax+1)(lmax+2)/2 Tournier coefficients (odf.rs:30-32).
int n_tournier(int lmax) { return (lmax + 1) * (lmax + 2) / 2; }

// Radial factor C*G*F of the analytic SHORE ODF (odf.rs:35-49).
double radial_factor(uint32_t n, uint32_t l, double zeta) {
  const double nf = n, lf = l;
  const double sign = (((static_cast<int>(n) - static_cast<int>(l) / 2) % 2) == 0) ? 1.0 : -1.0;
  const double c_nl =
      sign * std::sqrt(2.0 * factorial(n - l) / (std::pow(zeta, 1.5) * gamma_fn(nf + 1.5)));
  const double g_nl = (gamma_fn(lf / 2.0 + 1.5) * gamma_fn(nf + 1.5)) /
                      (gamma_fn(lf + 1.5) * factorial(n - l)) * std::pow(0.5, -lf / 2.0 - 1.5);
  const double f_nl = hyp2f1(-nf + lf, lf / 2.0 + 1.5, lf + 1.5, 2.0);
  return c_nl * g_nl * f_nl;
}

// BrainSuite block column k -> (Tournier index, sign) (odf.rs:57-73).
void brainsuite_to_tournier(uint32_t l, int k, int* idx, double* sign) {
  const int base = static_cast<int>(l * (l + 1) / 2);
  const int kl = static_cast<int>(l);
  if (k < kl) {
    *idx = base + (kl - k);
    *sign = 1.0;
  } else if (k == kl) {
    *idx = base;
    *sign = 1.0;
  } else {
    const int j = k - kl;
    *sign = (j % 2 == 1) ? 1.0 : -1.0;
    *idx = base - j;
  }
}

// SHORE -> Tournier SH projection, n_sh x K (odf.rs:79-102).
Mat shore_to_tournier(int radial_order, double zeta, int lmax) {
  const int K = static_cast<int>(shore_indices(radial_order).size());
  Mat m(n_tournier(lmax), K);
  int col = 0;
  for (int n = 0; n <= radial_order; ++n) {
    for (int l = 0; l <= n; l += 2) {
      const int bs = 2 * l + 1;
      if (l <= lmax) {
        const double rad = radial_factor(n, l, zeta);
        for (int k = 0; k < bs; ++k) {
          int row;
          double sign;
          brainsuite_to_tournier(l, k, &row, &sign);
          m(row, col + k) = rad * sign;
        }
      }
      col += bs;
    }
  }
  return m;
}

// Tournier (MRtrix) real SH of even degree up to lmax at cartesian unit
// directions, index l(l+1)/2 + m; the convention restated in the reference's
// own test helper (odf.rs:113-146) for odx-rs's sh2amp_cart.  Values are
// rounded through float32 because the reference receives them as f32
// (shore_icls.rs:54-63).
Mat sh2amp_cart(const std::vector<std::array<double, 3>>& dirs, int lmax) {
  const int nsh = n_tournier(lmax);
  Mat y(static_cast<int>(dirs.size()), nsh);
  const double s2 = std::sqrt(2.0);
  for (size_t d = 0; d < dirs.size(); ++d) {
    double r, th, ph;
    cart2sphere(dirs[d][0], dirs[d][1], dirs[d][2], &r, &th, &ph);
    const double cphi = std::cos(ph);
    for (int l = 0; l <= lmax; l += 2) {
      for (int m = -l; m <= l; ++m) {
        const uint32_t am = static_cast<uint32_t>(std::abs(m));
        const double norm =
            std::sqrt((2.0 * l + 1.0) / (4.0 * kPi) * factorial(l - am) / factorial(l + am));
        const double p = norm * assoc_legendre(l, am, cphi);
        double v;
        if (m < 0)
          v = s2 * p * std::sin(am * th);
        else if (m == 0)
          v = p;
        else
          v = s2 * p * std::cos(am * th);
        y(static_cast<int>(d), l * (l + 1) / 2 + m) = static_cast<double>(static_cast<float>(v));
      }
    }
  }
  return y;
}

// 642-vertex geodesic icosphere (icosahedron, three midpoint subdivisions,
// vertices projected to the unit sphere) and one direction of each antipodal
// pair: the 321-direction hemisphere used as the amplitude-constraint set.
// The reference takes DSI Studio's ODF8 hemisphere from odx-rs
// (shore_icls.rs:52), whose vertex table is not available; this is the same
// construction, not the same table.
std::vector<std::array<double, 3>> odf8_hemisphere() {
  const double phi = (1.0 + std::sqrt(5.0)) / 2.0;
  std::vector<std::array<double, 3>> v = {
      {-1, phi, 0}, {1, phi, 0}, {-1, -phi, 0}, {1, -phi, 0}, {0, -1, phi}, {0, 1, phi},
      {0, -1, -phi}, {0, 1, -phi}, {phi, 0, -1}, {phi, 0, 1}, {-phi, 0, -1}, {-phi, 0, 1}};
  for (auto& p : v) {
    const double n = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    for (auto& c : p) c /= n;
  }
  std::vector<std::array<int, 3>> f = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11},
                                       {1, 5, 9},  {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                                       {3, 9, 4},  {3, 4, 2},  {3, 2, 6},   {3, 6, 8},  {3, 8, 9},
                                       {4, 9, 5},  {2, 4, 11}, {6, 2, 10},  {8, 6, 7},  {9, 8, 1}};
  for (int level = 0; level < 3; ++level) {
    std::map<std::pair<int, int>, int> mid;
    auto midpoint = [&](int a, int b) {
      auto key = std::make_pair(std::min(a, b), std::max(a, b));
      auto it = mid.find(key);
      if (it != mid.end()) return it->second;
      std::array<double, 3> p = {v[a][0] + v[b][0], v[a][1] + v[b][1], v[a][2] + v[b][2]};
      const double n = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
      for (auto& c : p) c /= n;
      v.push_back(p);
      const int id = static_cast<int>(v.size()) - 1;
      mid[key] = id;
      return id;
    };
    std::vector<std::array<int, 3>> nf;
    for (auto& t : f) {
      const int a = midpoint(t[0], t[1]), b = midpoint(t[1], t[2]), c = midpoint(t[2], t[0]);
      nf.push_back({t[0], a, c});
      nf.push_back({t[1], b, a});
      nf.push_back({t[2], c, b});
      nf.push_back({a, b, c});
    }
    f.swap(nf);
  }
  std::vector<std::array<double, 3>> hemi;
  const double e = 1e-12;
  for (auto& p : v) {
    const bool keep = (p[2] > e) || (std::fabs(p[2]) <= e && p[1] > e) ||
                      (std::fabs(p[2]) <= e && std::fabs(p[1]) <= e && p[0] > 0.0);
    if (keep) hemi.push_back(p);
  }
  return hemi;
}

// ------------------------------------------------------ dense helpers

// y = A x with sequential accumulation per output element.
void gemv(const Mat& A, const double* x, double* y) {
  for (int i = 0; i < A.rows; ++i) {
    double acc = 0.0;
    for (int j = 0; j < A.cols; ++j) acc += A(i, j) * x[j];
    y[i] = acc;
  }
}

// y = A^T x.
void gemv_t(const Mat& A, const double* x, double* y) {
  for (int j = 0; j < A.cols; ++j) {
    double acc = 0.0;
    for (int i = 0; i < A.rows; ++i) acc += A(i, j) * x[i];
    y[j] = acc;
  }
}

double norm2(const double* v, int n) {
  double acc = 0.0;
  for (int i = 0; i < n; ++i) acc += v[i] * v[i];
  return std::sqrt(acc);
}

Mat gram(const Mat& M) {
  Mat G(M.cols, M.cols);
  for (int i = 0; i < M.cols; ++i)
    for (int j = 0; j < M.cols; ++j) {
      double acc = 0.0;
      for (int r = 0; r < M.rows; ++r) acc += M(r, i) * M(r, j);
      G(i, j) = acc;
    }
  return G;
}

// Largest eigenvalue of a symmetric matrix by cyclic Jacobi rotations.
double sym_max_eig(Mat A) {
  const int n = A.rows;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) (i == j ? diag : off) += A(i, j) * A(i, j);
    if (off <= 1e-32 * diag || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p) {
      for (int q = p + 1; q < n; ++q) {
        const double apq = A(p, q);
        if (apq == 0.0) continue;
        const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = A(k, p), akq = A(k, q);
          A(k, p) = c * akp - s * akq;
          A(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = A(p, k), aqk = A(q, k);
          A(p, k) = c * apk - s * aqk;
          A(q, k) = s * apk + c * aqk;
        }
      }
    }
  }
  double mx = -std::numeric_limits<double>::infinity();
  for (int i = 0; i < n; ++i) mx = std::max(mx, A(i, i));
  return mx;
}

// sigma_max(M) = sqrt(lambda_max(M^T M)); stands in for nalgebra's SVD
// (fista.rs:45-50).
double sigma_max(const Mat& M) {
  const double l = sym_max_eig(gram(M));
  return std::sqrt(std::max(l, 0.0));
}

// In-place LL^T Cholesky (lower factor); false if not positive definite.
bool cholesky(Mat& A) {
  const int n = A.rows;
  for (int j = 0; j < n; ++j) {
    double d = A(j, j);
    for (int k = 0; k < j; ++k) d -= A(j, k) * A(j, k);
    if (!(d > 0.0)) return false;
    const double ljj = std::sqrt(d);
    A(j, j) = ljj;
    for (int i = j + 1; i < n; ++i) {
      double s = A(i, j);
      for (int k = 0; k < j; ++k) s -= A(i, k) * A(j, k);
      A(i, j) = s / ljj;
    }
    for (int k = j + 1; k < n; ++k) A(j, k) = 0.0;
  }
  return true;
}

// Solve L L^T x = b (forward then backward substitution).
void chol_solve(const Mat& L, const double* b, double* x) {
  const int n = L.rows;
  for (int i = 0; i < n; ++i) {
    double s = b[i];
    for (int k = 0; k < i; ++k) s -= L(i, k) * x[k];
    x[i] = s / L(i, i);
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = x[i];
    for (int k = i + 1; k < n; ++k) s -= L(k, i) * x[k];
    x[i] = s / L(i, i);
  }
}

// ------------------------------------------------------ solver/mod.rs

struct Diag {
  uint32_t iterations = 0;
  double residual_l2 = 0;
  bool converged = false;
  double alpha = 0;
  uint8_t kind = 0;
};

// --------------------------------------------------------- solver/fista.rs

// FISTA for (1/(2n))||Mc - s||^2 + alpha ||c||_1 (fista.rs:88-143).
struct Fista {
  double alpha;
  uint32_t max_iter;
  double tol;
  bool non_negative;
  double lipschitz;
  const Mat* design;
  Mat mt;
  double n_inv;

  Fista(const Mat& M, double a, uint32_t mi, double t, bool nn, double sigma)
      : alpha(a), max_iter(mi), tol(t), non_negative(nn), design(&M) {
    const double n = M.rows;
    n_inv = 1.0 / n;
    lipschitz = std::max(sigma * sigma * n_inv, std::numeric_limits<double>::epsilon());
    mt = Mat(M.cols, M.rows);
    for (int i = 0; i < M.rows; ++i)
      for (int j = 0; j < M.cols; ++j) mt(j, i) = M(i, j);
  }

  // fit_with_warm_start (fista.rs:70-143).
  Diag fit(const double* s, const double* warm, double* x_out) const {
    const int K = design->cols, N = design->rows;
    Vec x(K, 0.0), y, xn(K), yn(K), my(N), res(N), grad(K);
    if (warm) x.assign(warm, warm + K);
    y = x;
    double t = 1.0;
    const double step = 1.0 / lipschitz;
    const double thr = step * alpha;
    uint32_t iters = 0;
    bool conv = false;
    for (uint32_t it = 0; it < max_iter; ++it) {
      gemv(*design, y.data(), my.data());
      for (int i = 0; i < N; ++i) res[i] = my[i] - s[i];
      gemv(mt, res.data(), grad.data());
      for (int k = 0; k < K; ++k) grad[k] = grad[k] * n_inv;
      for (int k = 0; k < K; ++k) {
        const double v = y[k] - step * grad[k];
        double sv;
        if (v > thr)
          sv = v - thr;
        else if (v < -thr)
          sv = v + thr;
        else
          sv = 0.0;
        xn[k] = non_negative ? std::max(sv, 0.0) : sv;
      }
      const double tn = 0.5 * (1.0 + std::sqrt(1.0 + 4.0 * t * t));
      const double mom = (t - 1.0) / tn;
      double dx2 = 0.0, xn2 = 0.0;
      for (int k = 0; k < K; ++k) {
        yn[k] = xn[k] + mom * (xn[k] - x[k]);
        const double d = xn[k] - x[k];
        dx2 += d * d;
        xn2 += xn[k] * xn[k];
      }
      const double rel = std::sqrt(dx2) / std::max(std::sqrt(xn2), 1e-12);
      x.swap(xn);
      y.swap(yn);
      t = tn;
      iters = it + 1;
      if (rel < tol) {
        conv = true;
        break;
      }
    }
    gemv(*design, x.data(), my.data());
    for (int i = 0; i < N; ++i) res[i] = s[i] - my[i];
    Diag d;
    d.iterations = iters;
    d.residual_l2 = norm2(res.data(), N);
    d.converged = conv;
    d.alpha = alpha;
    d.kind = 1;
    std::copy(x.begin(), x.end(), x_out);
    return d;
  }
};

// ------------------------------------------------------ solver/tikhonov.rs

// Cholesky of M^T M + lambda_N N + lambda_L L once, then per voxel
// c = chol.solve(M^T s) and ||s - Mc|| (tikhonov.rs:26-76).
struct Tikhonov {
  const Mat* design;
  Mat L;
  bool ok = false;
  Tikhonov(const Mat& M, const Vec& nd, const Vec& ld, double ln, double ll) : design(&M) {
    L = gram(M);
    for (int i = 0; i < L.rows; ++i) L(i, i) += ln * nd[i];
    for (int i = 0; i < L.rows; ++i) L(i, i) += ll * ld[i];
    ok = cholesky(L);
  }
  Diag fit(const double* s, double* c) const {
    const int K = design->cols, N = design->rows;
    Vec rhs(K), my(N);
    gemv_t(*design, s, rhs.data());
    chol_solve(L, rhs.data(), c);
    gemv(*design, c, my.data());
    for (int i = 0; i < N; ++i) my[i] = s[i] - my[i];
    Diag d;
    d.iterations = 1;
    d.residual_l2 = norm2(my.data(), N);
    d.converged = true;
    d.alpha = 0.0;
    d.kind = 2;
    return d;
  }
};

// --------------------------------------------------------- solver/icls.rs

struct IclsCfg {
  int max_iter;
  double tol;
  double epsilon;
};

struct IclsDiag {
  int iterations = 0, final_active = 0;
  bool converged = false, infeasible = false;
};

// Goldfarb-Idnani dual active-set solver for min 1/2||Hx - b||^2 s.t. Cx >= 0
// (icls.rs:137-411).
struct Icls {
  const Mat* h;
  Mat ht, C, L, J0;
  IclsCfg cfg;
  int n, m;
  bool ok = false;

  Icls(const Mat& H, const Mat& Cm, IclsCfg c) : h(&H), C(Cm), cfg(c) {
    n = H.cols;
    m = Cm.rows;
    ht = Mat(H.cols, H.rows);
    for (int i = 0; i < H.rows; ++i)
      for (int j = 0; j < H.cols; ++j) ht(j, i) = H(i, j);
    // G = H^T H + eps I (icls.rs:174-208).
    L = gram(H);
    for (int i = 0; i < n; ++i) L(i, i) += cfg.epsilon;
    ok = cholesky(L);
    if (!ok) return;
    // J0 = L^{-T} by back-substitution per column (icls.rs:417-431).
    J0 = Mat(n, n);
    for (int j = 0; j < n; ++j) {
      for (int i = n - 1; i >= 0; --i) {
        double sum = (i == j) ? 1.0 : 0.0;
        for (int k = i + 1; k < n; ++k) sum -= L(k, i) * J0(k, j);
        J0(i, j) = sum / L(i, i);
      }
    }
  }

  static void rotate_columns(Mat& M, int i, double c, double s) {
    for (int r = 0; r < M.rows; ++r) {
      const double a = M(r, i), b = M(r, i + 1);
      M(r, i) = c * a + s * b;
      M(r, i + 1) = -s * a + c * b;
    }
  }

  // icls.rs:436-460.
  static void add_active(Mat& R, Mat& J, Vec& d, int q, int n) {
    for (int i = n - 1; i >= q + 1; --i) {
      const double a = d[i - 1], b = d[i];
      if (b == 0.0) continue;
      const double rn = std::sqrt(a * a + b * b);
      const double c = a / rn, s = b / rn;
      d[i - 1] = rn;
      d[i] = 0.0;
      rotate_columns(J, i - 1, c, s);
    }
    for (int i = 0; i <= q; ++i) R(i, q) = d[i];
  }

  // icls.rs:465-501.
  static void drop_active(Mat& R, Mat& J, int k, int q) {
    for (int col = k; col < q - 1; ++col)
      for (int row = 0; row < q; ++row) R(row, col) = R(row, col + 1);
    for (int row = 0; row < q; ++row) R(row, q - 1) = 0.0;
    for (int i = k; i < q - 1; ++i) {
      const double a = R(i, i), b = R(i + 1, i);
      if (b == 0.0) continue;
      const double rn = std::sqrt(a * a + b * b);
      const double c = a / rn, s = b / rn;
      for (int col = i; col < q - 1; ++col) {
        const double ri = R(i, col), rip1 = R(i + 1, col);
        R(i, col) = c * ri + s * rip1;
        R(i + 1, col) = -s * ri + c * rip1;
      }
      rotate_columns(J, i, c, s);
    }
  }

  // solve_into (icls.rs:261-410).
  IclsDiag solve(const double* b, double* x_out) const {
    const int maxq = std::min(n, m);
    Mat J = J0, R(maxq, maxq);
    Vec d(n), z(n), rdir(maxq > 0 ? maxq : 1);
    std::vector<int> active;
    Vec mult;
    std::vector<char> is_active(m, 0);
    Vec htb(n), x(n);
    gemv(ht, b, htb.data());
    chol_solve(L, htb.data(), x.data());
    int q = 0, iters = 0;
    bool converged = false, infeasible = false;
    Vec np(n);
    while (true) {
      iters += 1;
      if (iters > cfg.max_iter) break;
      int worst = -1;
      double worst_val = -cfg.tol;
      for (int p = 0; p < m; ++p) {
        if (is_active[p]) continue;
        double sp = 0.0;
        for (int k = 0; k < n; ++k) sp += C(p, k) * x[k];
        if (sp < worst_val) {
          worst_val = sp;
          worst = p;
        }
      }
      if (worst < 0) {
        converged = true;
        break;
      }
      const int p = worst;
      for (int k = 0; k < n; ++k) np[k] = C(p, k);
      double sp = 0.0;
      for (int k = 0; k < n; ++k) sp += C(p, k) * x[k];
      bool stop = false;
      while (true) {
        for (int c = 0; c < n; ++c) {
          double acc = 0.0;
          for (int r = 0; r < n; ++r) acc += J(r, c) * np[r];
          d[c] = acc;
        }
        std::fill(z.begin(), z.end(), 0.0);
        if (q < n) {
          for (int r = 0; r < n; ++r) {
            double acc = 0.0;
            for (int c = q; c < n; ++c) acc += J(r, c) * d[c];
            z[r] = acc;
          }
        }
        for (int i = q - 1; i >= 0; --i) {
          double sum = d[i];
          for (int k = i + 1; k < q; ++k) sum -= R(i, k) * rdir[k];
          rdir[i] = sum / R(i, i);
        }
        double t1 = std::numeric_limits<double>::infinity();
        int drop = -1;
        for (int i = 0; i < q; ++i) {
          if (rdir[i] > cfg.tol) {
            const double ratio = mult[i] / rdir[i];
            if (ratio < t1) {
              t1 = ratio;
              drop = i;
            }
          }
        }
        double zdn = 0.0;
        for (int k = 0; k < n; ++k) zdn += z[k] * np[k];
        const double t2 = (zdn > cfg.tol) ? -sp / zdn : std::numeric_limits<double>::infinity();
        const double t = std::min(t1, t2);
        if (!std::isfinite(t)) {
          infeasible = true;
          stop = true;
          break;
        }
        for (int i = 0; i < q; ++i) mult[i] -= t * rdir[i];
        if (std::isfinite(t2) && t == t2) {
          for (int k = 0; k < n; ++k) x[k] += t * z[k];
          add_active(R, J, d, q, n);
          active.push_back(p);
          is_active[p] = 1;
          mult.push_back(t);
          q += 1;
          break;
        } else {
          for (int k = 0; k < n; ++k) x[k] += t * z[k];
          sp += t * zdn;
          const int k = drop;
          const int dropped = active[k];
          drop_active(R, J, k, q);
          active.erase(active.begin() + k);
          is_active[dropped] = 0;
          mult.erase(mult.begin() + k);
          q -= 1;
        }
      }
      if (stop) break;
    }
    IclsDiag dg;
    dg.iterations = iters - 1;
    dg.final_active = q;
    dg.converged = converged;
    dg.infeasible = infeasible;
    std::copy(x.begin(), x.end(), x_out);
    return dg;
  }
};

// ---------------------------------------------------------- solver/alpha.rs

// ||M^T s||_inf / n (alpha.rs:47-53).
double alpha_max(const Mat& M, const double* s) {
  if (M.rows == 0) return 0.0;
  Vec xty(M.cols);
  gemv_t(M, s, xty.data());
  double m = 0.0;
  for (double v : xty) m = std::max(m, std::fabs(v));
  return m / static_cast<double>(M.rows);
}

// Log-spaced descending path alpha_max .. alpha_max * eps (alpha.rs:57-69).
Vec log_path(double amax, int n, double eps) {
  Vec p(n);
  const double lmax = std::log(amax), lmin = std::log(amax * eps);
  for (int i = 0; i < n; ++i) {
    const double t = static_cast<double>(i) / static_cast<double>(n - 1);
    p[i] = std::exp(lmax + t * (lmin - lmax));
  }
  return p;
}

// n ln(RSS/n) + ln(n) k with RSS floored at the smallest normal (alpha.rs:99-103).
double bic(int n_grads, double rss, int k) {
  const double n = n_grads;
  const double rc = std::max(rss, std::numeric_limits<double>::min());
  return n * std::log(rc / n) + std::log(n) * static_cast<double>(k);
}

int count_nonzero(const double* c, int K) {
  int k = 0;
  for (int i = 0; i < K; ++i) k += (c[i] != 0.0);
  return k;
}

struct VoxelAlpha {
  double alpha = 0, residual_l2 = 0, bic = 0, rss_l2 = 0;
  uint32_t iterations = 0;
  bool converged = true;
};

// ---------------------------------------------------------------- fit.rs

struct VoxelOut {
  double r2;
  double residual_l2;
  uint32_t iterations;
  uint8_t kind;
  double alpha, bic, rss_l2;
  bool converged;
};

}  // namespace

// ======================================================================
// C ABI
// ======================================================================

extern "C" {

double oracle_factorial(uint32_t n) { return factorial(n); }
double oracle_gamma(double x) { return gamma_fn(x); }
double oracle_assoc_legendre(uint32_t l, uint32_t m, double x) { return assoc_legendre(l, m, x); }
double oracle_gen_laguerre(uint32_t n, double a, double x) { return gen_laguerre(n, a, x); }
double oracle_hyp2f1(double a, double b, double c, double z) { return hyp2f1(a, b, c, z); }

int oracle_qvals(const csd_gtab* g, double* q_out, double* big, double* small, int32_t* src) {
  Gtab t = make_gtab(g);
  Vec q = t.qvals();
  std::copy(q.begin(), q.end(), q_out);
  *big = t.big_delta;
  *small = t.small_delta;
  *src = t.delta_source;
  return 0;
}

int oracle_shells(const double* bvals, int32_t n, double thr, double tol, double* shell_b,
                  int32_t* shell_of) {
  Vec b(bvals, bvals + n);
  auto sh = shells(b, thr, tol);
  for (size_t s = 0; s < sh.size(); ++s) {
    shell_b[s] = sh[s].b;
    for (int i : sh[s].idx) shell_of[i] = static_cast<int32_t>(s);
  }
  return static_cast<int>(sh.size());
}

void oracle_tortoise_deltas(const double* bvals, int32_t n, double gmax, double* big,
                            double* small) {
  tortoise_deltas(bvals, n, gmax, big, small);
}

int oracle_n_coeffs(int32_t r) { return static_cast<int>(shore_indices(r).size()); }

void oracle_shore_indices(int32_t r, int32_t* n_out, int32_t* l_out, int32_t* m_out) {
  auto idx = shore_indices(r);
  for (size_t i = 0; i < idx.size(); ++i) {
    n_out[i] = idx[i].n;
    l_out[i] = idx[i].l;
    m_out[i] = idx[i].m;
  }
}

double oracle_kappa(double zeta, uint32_t n, uint32_t l) { return kappa(zeta, n, l); }
double oracle_shore_radial(uint32_t n, uint32_t l, double q, double zeta) {
  return shore_radial(n, l, q, zeta);
}
void oracle_brainsuite_sh_block(uint32_t l, double th, double ph, double* out) {
  brainsuite_sh_block(l, th, ph, out);
}

int oracle_design_matrix(const csd_gtab* g, int32_t r, double zeta, double* out) {
  Gtab t = make_gtab(g);
  Mat m = design_matrix(t, r, zeta);
  std::copy(m.a.begin(), m.a.end(), out);
  return 0;
}

void oracle_regularization(int32_t r, double* nd, double* ld) {
  Vec a, b;
  regularization(r, a, b);
  std::copy(a.begin(), a.end(), nd);
  std::copy(b.begin(), b.end(), ld);
}

double oracle_radial_factor(uint32_t n, uint32_t l, double zeta) { return radial_factor(n, l, zeta); }
void oracle_brainsuite_to_tournier(uint32_t l, int32_t k, int32_t* idx, double* sign) {
  int i;
  brainsuite_to_tournier(l, k, &i, sign);
  *idx = i;
}
int oracle_shore_to_tournier(int32_t r, double zeta, int32_t lmax, double* out) {
  Mat m = shore_to_tournier(r, zeta, lmax);
  std::copy(m.a.begin(), m.a.end(), out);
  return m.rows;
}
int oracle_odf8_hemisphere(double* out) {
  auto h = odf8_hemisphere();
  for (size_t i = 0; i < h.size(); ++i)
    for (int c = 0; c < 3; ++c) out[3 * i + c] = h[i][c];
  return static_cast<int>(h.size());
}
void oracle_sh2amp_cart(const double* dirs, int32_t nd, int32_t lmax, double* out) {
  std::vector<std::array<double, 3>> d(nd);
  for (int i = 0; i < nd; ++i) d[i] = {dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]};
  Mat y = sh2amp_cart(d, lmax);
  std::copy(y.a.begin(), y.a.end(), out);
}

static Mat wrap(const double* a, int m, int n) {
  Mat M(m, n);
  std::copy(a, a + static_cast<size_t>(m) * n, M.a.begin());
  return M;
}

double oracle_sigma_max(const double* design, int32_t m, int32_t n) {
  return sigma_max(wrap(design, m, n));
}

int oracle_fista_fit(const double* design, int32_t m, int32_t n, const double* signal, double alpha,
                     int32_t max_iter, double tol, int32_t nn, const double* warm, double* coef,
                     int32_t* iterations, int32_t* converged, double* resid) {
  Mat M = wrap(design, m, n);
  Fista f(M, alpha, static_cast<uint32_t>(max_iter), tol, nn != 0, sigma_max(M));
  Diag d = f.fit(signal, warm, coef);
  *iterations = static_cast<int32_t>(d.iterations);
  *converged = d.converged;
  *resid = d.residual_l2;
  return 0;
}

int oracle_tikhonov_fit(const double* design, int32_t m, int32_t n, const double* nd,
                        const double* ld, double ln, double ll, const double* s, double* c,
                        double* resid) {
  Mat M = wrap(design, m, n);
  Vec a(nd, nd + n), b(ld, ld + n);
  Tikhonov t(M, a, b, ln, ll);
  if (!t.ok) return CSD_ERR_NUMERICAL;
  Diag d = t.fit(s, c);
  *resid = d.residual_l2;
  return 0;
}

int oracle_icls_solve(const double* h, int32_t m, int32_t n, const double* c, int32_t mc,
                      const double* b, int32_t max_iter, double tol, double eps, double* x,
                      int32_t* iterations, int32_t* final_active, int32_t* converged,
                      int32_t* infeasible) {
  Mat H = wrap(h, m, n), C = wrap(c, mc, n);
  Icls s(H, C, IclsCfg{max_iter, tol, eps});
  if (!s.ok) return CSD_ERR_NUMERICAL;
  IclsDiag d = s.solve(b, x);
  *iterations = d.iterations;
  *final_active = d.final_active;
  *converged = d.converged;
  *infeasible = d.infeasible;
  return 0;
}

double oracle_alpha_max(const double* design, int32_t m, int32_t n, const double* s) {
  return alpha_max(wrap(design, m, n), s);
}

int oracle_log_path(double amax, int32_t n, double eps, double* out) {
  if (n < 2 || !(amax > 0.0) || !(eps > 0.0 && eps < 1.0)) return CSD_ERR_INVALID;
  Vec p = log_path(amax, n, eps);
  std::copy(p.begin(), p.end(), out);
  return 0;
}

double oracle_bic(int32_t n, double rss, int32_t k) { return bic(n, rss, k); }

void oracle_default_spec(csd_shore_spec* s) {
  // ShoreFitSpec::default + PyO3 kwargs (fit.rs:647-669, models.rs:70-76).
  s->radial_order = 6;
  s->zeta = 700.0;
  s->regularization = CSD_REG_L1;
  s->alpha_mode = CSD_ALPHA_L2_ANCHORED;
  s->alpha = 1.0;
  s->alpha_ratio = 1e-3;
  s->path_n_alphas = 20;
  s->path_eps = 0.0;
  s->slack = 0.05;
  s->max_iter = 1000;
  s->tol = 1e-6;
  s->non_negative = 0;
  s->lambda_n = 1e-8;
  s->lambda_l = 1e-8;
  s->nonneg_max_iter = 200;
  s->nonneg_tol = 1e-9;
  s->nonneg_epsilon = 1e-10;
  s->diagnostics = 0;
  s->allow_single_shell = 0;
  s->precision = CSD_PRECISION_FP64;
}

int oracle_shore_fit_volume(const float* data, const uint8_t* mask, int64_t X, int64_t Y, int64_t Z,
                            const csd_gtab* gtab, const csd_shore_spec* spec, csd_fit_result* out,
                            int32_t n_threads, char* err, size_t err_len) {
  if (!data || !mask || !gtab || !spec || !out || !out->coefficients || X < 0 || Y < 0 || Z < 0) {
    set_err(err, err_len, "invalid argument: null pointer or negative shape");
    return CSD_ERR_INVALID;
  }
  if (spec->radial_order <= 0 || spec->radial_order % 2 != 0) {
    set_err(err, err_len,
            "radial_order must be a positive even number, got " + std::to_string(spec->radial_order));
    return CSD_ERR_INVALID;
  }
  // build_alpha_strategy validation (fit.rs:555-591).
  double path_eps = spec->path_eps;
  if (spec->regularization == CSD_REG_L1) {
    const int mode = spec->alpha_mode;
    if (mode == CSD_ALPHA_RATIO && !(spec->alpha_ratio > 0.0 && spec->alpha_ratio < 1.0)) {
      set_err(err, err_len, "--alpha-ratio must lie in (0, 1)");
      return CSD_ERR_INVALID;
    }
    if (mode == CSD_ALPHA_PATH_BIC || mode == CSD_ALPHA_L2_ANCHORED) {
      if (spec->path_n_alphas < 2) {
        set_err(err, err_len, "--path-n-alphas must be >= 2");
        return CSD_ERR_INVALID;
      }
      if (!(path_eps > 0.0)) path_eps = (mode == CSD_ALPHA_PATH_BIC) ? 1e-3 : 1e-4;
      if (!(path_eps > 0.0 && path_eps < 1.0)) {
        set_err(err, err_len, "--path-eps must lie in (0, 1)");
        return CSD_ERR_INVALID;
      }
      if (mode == CSD_ALPHA_L2_ANCHORED && spec->slack < 0.0) {
        set_err(err, err_len, "--slack must be >= 0");
        return CSD_ERR_INVALID;
      }
    }
  } else if (spec->regularization != CSD_REG_L2 && spec->regularization != CSD_REG_NONNEG) {
    set_err(err, err_len, "regularization must be l1, l2 or nonneg");
    return CSD_ERR_INVALID;
  }
  Gtab g = make_gtab(gtab);
  const int N = g.n();
  // Shell guard (fit.rs:691-717).
  Vec sh = dwi_shells(g);
  std::string warnings;
  if (sh.empty()) {
    set_err(err, err_len,
            "3D-SHORE needs diffusion-weighted data; every volume is at or below the b=0 threshold");
    return CSD_ERR_FIT_REFUSED;
  }
  if (sh.size() < kMinShoreShells) {
    char what[128];
    if (sh.size() == 1)
      std::snprintf(what, sizeof what, "a single shell (b = %.0f s/mm\xc2\xb2)", sh[0]);
    else
      std::snprintf(what, sizeof what, "%zu shells", sh.size());
    if (!spec->allow_single_shell) {
      set_err(err, err_len,
              std::string("3D-SHORE needs diffusion-weighted data on at least 2 b-value shells; "
                          "this series has ") +
                  what +
                  ". With a single shell the radial decay of the signal is not determined by the "
                  "data. To fit anyway for orientation information only, allow single-shell data "
                  "(allow_single_shell=True).");
      return CSD_ERR_FIT_REFUSED;
    }
    warnings += std::string("the data have ") + what +
                ": only the orientation information of this fit is meaningful, and "
                "propagator-derived scalars are not computed\n";
  }
  const int K = oracle_n_coeffs(spec->radial_order);
  if (N < K && spec->regularization != CSD_REG_L1) {
    warnings += std::to_string(N) + " measurements for " + std::to_string(K) +
                " coefficients (radial order " + std::to_string(spec->radial_order) +
                "): without L1 regularization the fit is underdetermined and its fit statistics "
                "are not meaningful; use a lower radial order or L1\n";
  }
  Mat M = design_matrix(g, spec->radial_order, spec->zeta);
  Vec nd, ld;
  regularization(spec->radial_order, nd, ld);

  // Masked voxels in x-y-z order (voxel_loop.rs:28-42).
  std::vector<int64_t> vox;
  const int64_t nvol = X * Y * Z;
  for (int64_t i = 0; i < nvol; ++i)
    if (mask[i]) vox.push_back(i);
  const int64_t V = static_cast<int64_t>(vox.size());

  // Solvers, built once (fit.rs:731-795).
  const bool is_l1 = spec->regularization == CSD_REG_L1;
  const bool need_tik =
      spec->regularization == CSD_REG_L2 || (is_l1 && spec->alpha_mode == CSD_ALPHA_L2_ANCHORED);
  std::unique_ptr<Tikhonov> tik;
  if (need_tik) {
    tik.reset(new Tikhonov(M, nd, ld, spec->lambda_n, spec->lambda_l));
    if (!tik->ok) {
      set_err(err, err_len, "normal-equations matrix should be PD");
      return CSD_ERR_NUMERICAL;
    }
  }
  std::unique_ptr<Fista> fista;
  if (is_l1) {
    fista.reset(new Fista(M, std::max(spec->alpha, 1e-12), static_cast<uint32_t>(spec->max_iter),
                          spec->tol, spec->non_negative != 0, sigma_max(M)));
  }
  std::unique_ptr<Icls> icls;
  int lmax = 0, ndirs = 0;
  if (spec->regularization == CSD_REG_NONNEG) {
    lmax = default_lmax(spec->radial_order);
    Mat P = shore_to_tournier(spec->radial_order, spec->zeta, lmax);
    auto dirs = odf8_hemisphere();
    ndirs = static_cast<int>(dirs.size());
    Mat Ys = sh2amp_cart(dirs, lmax);
    Mat Cm(ndirs, K);
    for (int i = 0; i < ndirs; ++i)
      for (int j = 0; j < K; ++j) {
        double acc = 0.0;
        for (int k = 0; k < P.rows; ++k) acc += Ys(i, k) * P(k, j);
        Cm(i, j) = acc;
      }
    icls.reset(new Icls(M, Cm, IclsCfg{spec->nonneg_max_iter, spec->nonneg_tol, spec->nonneg_epsilon}));
    if (!icls->ok) {
      set_err(err, err_len, "H^T H + eps I must be positive definite");
      return CSD_ERR_NUMERICAL;
    }
  }

  std::vector<VoxelOut> vo(V);
  std::vector<double> coefs(static_cast<size_t>(V) * K, 0.0);
  const int mode = spec->alpha_mode;

  auto fit_one = [&](int64_t vi) {
    const float* src = data + vox[vi] * N;
    Vec s(N);
    for (int i = 0; i < N; ++i) s[i] = static_cast<double>(src[i]);
    double mean = 0.0;
    for (int i = 0; i < N; ++i) mean += s[i];
    mean /= static_cast<double>(N);
    double* c = &coefs[static_cast<size_t>(vi) * K];
    VoxelOut o{};
    double resid = 0.0;
    if (spec->regularization == CSD_REG_L2) {
      Diag d = tik->fit(s.data(), c);
      resid = d.residual_l2;
      o.iterations = d.iterations;
      o.kind = d.kind;
      o.converged = d.converged;
    } else if (spec->regularization == CSD_REG_NONNEG) {
      IclsDiag d = icls->solve(s.data(), c);
      Vec hx(N);
      gemv(M, c, hx.data());
      for (int i = 0; i < N; ++i) hx[i] -= s[i];
      resid = norm2(hx.data(), N);
      o.iterations = static_cast<uint32_t>(d.iterations);
      o.kind = 3;
      o.converged = d.converged;
    } else {
      // AlphaStrategy::resolve / resolve_with_l2_ref (alpha.rs:207-318).
      Fista f = *fista;
      double rss_l2 = 0.0;
      if (mode == CSD_ALPHA_L2_ANCHORED) {
        Vec tmp(K);
        Diag dl = tik->fit(s.data(), tmp.data());
        rss_l2 = dl.residual_l2 * dl.residual_l2;
      }
      Diag d;
      double a_used = 0.0;
      bool zero = false;
      if (mode == CSD_ALPHA_FIXED) {
        f.alpha = spec->alpha;
        d = f.fit(s.data(), nullptr, c);
        a_used = spec->alpha;
      } else {
        const double amax = alpha_max(M, s.data());
        if (amax == 0.0) {
          zero = true;
        } else if (mode == CSD_ALPHA_RATIO) {
          a_used = amax * spec->alpha_ratio;
          f.alpha = a_used;
          d = f.fit(s.data(), nullptr, c);
        } else {
          // fit_path, warm-started descending (fista.rs:164-178).
          Vec alphas = log_path(amax, spec->path_n_alphas, path_eps);
          const int P = spec->path_n_alphas;
          std::vector<Vec> cs(P, Vec(K));
          std::vector<Diag> ds(P);
          const double* warm = nullptr;
          for (int i = 0; i < P; ++i) {
            f.alpha = alphas[i];
            ds[i] = f.fit(s.data(), warm, cs[i].data());
            warm = cs[i].data();
          }
          int idx = 0;
          if (mode == CSD_ALPHA_PATH_BIC) {
            // bic_argmin (alpha.rs:107-128).
            double best = std::numeric_limits<double>::infinity();
            for (int i = 0; i < P; ++i) {
              const double b =
                  bic(N, ds[i].residual_l2 * ds[i].residual_l2, count_nonzero(cs[i].data(), K));
              if (b < best) {
                best = b;
                idx = i;
              }
            }
          } else {
            // l2_anchored_argmax (alpha.rs:140-165).
            const double thr = (1.0 + spec->slack) * rss_l2;
            idx = -1;
            for (int i = 0; i < P; ++i)
              if (ds[i].residual_l2 * ds[i].residual_l2 <= thr) {
                idx = i;
                break;
              }
            if (idx < 0) {
              double best = std::numeric_limits<double>::infinity();
              idx = 0;
              for (int i = 0; i < P; ++i) {
                const double r = ds[i].residual_l2 * ds[i].residual_l2;
                if (r < best) {
                  best = r;
                  idx = i;
                }
              }
            }
          }
          std::copy(cs[idx].begin(), cs[idx].end(), c);
          d = ds[idx];
          a_used = alphas[idx];
        }
      }
      if (zero) {
        std::fill(c, c + K, 0.0);
        o.alpha = 0.0;
        o.bic = 0.0;
        o.iterations = 0;
        o.converged = true;
        resid = 0.0;
      } else {
        resid = d.residual_l2;
        o.alpha = a_used;
        o.bic = bic(N, d.residual_l2 * d.residual_l2, count_nonzero(c, K));
        o.iterations = d.iterations;
        o.converged = d.converged;
      }
      o.kind = 1;
      o.rss_l2 = rss_l2;
    }
    // R^2 = 1 - RSS / sum (s - mean)^2 (fit.rs:120-128).
    const double ss_res = resid * resid;
    double ss_tot = 0.0;
    for (int i = 0; i < N; ++i) ss_tot += (s[i] - mean) * (s[i] - mean);
    o.r2 = ss_tot > 0.0 ? 1.0 - ss_res / ss_tot : 0.0;
    o.residual_l2 = resid;
    vo[vi] = o;
  };

  // Parallel voxel loop with per-worker state (voxel_loop.rs:79-103).
  int nt = n_threads > 0 ? n_threads : static_cast<int>(std::thread::hardware_concurrency());
  if (nt < 1) nt = 1;
  std::atomic<int64_t> next(0);
  auto worker = [&]() {
    while (true) {
      const int64_t start = next.fetch_add(16);
      if (start >= V) break;
      const int64_t end = std::min<int64_t>(start + 16, V);
      for (int64_t i = start; i < end; ++i) fit_one(i);
    }
  };
  std::vector<std::thread> th;
  for (int i = 1; i < nt; ++i) th.emplace_back(worker);
  worker();
  for (auto& t : th) t.join();

  // Scatter (fit.rs:139-155 / 294-318 / 456-483).
  std::memset(out->coefficients, 0, sizeof(float) * static_cast<size_t>(nvol) * K);
  const bool diag = spec->diagnostics != 0;
  if (diag) {
    if (out->r2) std::memset(out->r2, 0, sizeof(float) * nvol);
    if (out->residual_l2) std::memset(out->residual_l2, 0, sizeof(float) * nvol);
    if (out->iterations) std::memset(out->iterations, 0, sizeof(uint32_t) * nvol);
    if (out->regularization_kind) std::memset(out->regularization_kind, 0, nvol);
    if (out->alpha && is_l1) std::memset(out->alpha, 0, sizeof(float) * nvol);
    if (out->bic && is_l1) std::memset(out->bic, 0, sizeof(float) * nvol);
    if (out->rss_l2 && is_l1 && mode == CSD_ALPHA_L2_ANCHORED)
      std::memset(out->rss_l2, 0, sizeof(float) * nvol);
  }
  uint64_t total_it = 0;
  std::vector<double> alphas_seen;
  for (int64_t vi = 0; vi < V; ++vi) {
    const int64_t li = vox[vi];
    for (int k = 0; k < K; ++k)
      out->coefficients[li * K + k] = static_cast<float>(coefs[static_cast<size_t>(vi) * K + k]);
    if (out->coef64)
      std::copy(&coefs[static_cast<size_t>(vi) * K], &coefs[static_cast<size_t>(vi) * K] + K,
                out->coef64 + vi * K);
    if (out->converged) out->converged[vi] = vo[vi].converged ? 1 : 0;
    total_it += vo[vi].iterations;
    if (is_l1) alphas_seen.push_back(vo[vi].alpha);
    if (!diag) continue;
    if (out->r2) out->r2[li] = static_cast<float>(vo[vi].r2);
    if (out->residual_l2) out->residual_l2[li] = static_cast<float>(vo[vi].residual_l2);
    if (out->iterations) out->iterations[li] = vo[vi].iterations;
    if (out->regularization_kind) out->regularization_kind[li] = vo[vi].kind;
    if (is_l1) {
      if (out->alpha) out->alpha[li] = static_cast<float>(vo[vi].alpha);
      if (out->bic) out->bic[li] = static_cast<float>(vo[vi].bic);
      if (out->rss_l2 && mode == CSD_ALPHA_L2_ANCHORED)
        out->rss_l2[li] = static_cast<float>(vo[vi].rss_l2);
    }
  }
  // alpha distribution (fit.rs:334-352).
  out->has_alpha_distribution = 0;
  out->representative_alpha = 0.0;
  if (is_l1) {
    if (mode == CSD_ALPHA_FIXED) {
      out->representative_alpha = spec->alpha;
    } else {
      out->has_alpha_distribution = 1;
      std::sort(alphas_seen.begin(), alphas_seen.end());
      if (alphas_seen.empty()) {
        out->alpha_distribution[0] = out->alpha_distribution[1] = out->alpha_distribution[2] = 0.0;
      } else {
        auto pct = [&](double q) {
          size_t i = static_cast<size_t>(std::round(static_cast<double>(alphas_seen.size() - 1) * q));
          return alphas_seen[std::min(i, alphas_seen.size() - 1)];
        };
        out->alpha_distribution[0] = pct(0.5);
        out->alpha_distribution[1] = pct(0.10);
        out->alpha_distribution[2] = pct(0.90);
      }
      out->representative_alpha = out->alpha_distribution[0];
    }
  }
  out->n_coeffs = K;
  out->n_voxels = V;
  out->big_delta_seconds = g.big_delta;
  out->small_delta_seconds = g.small_delta;
  out->tau_seconds = g.tau();
  out->delta_source = g.delta_source;
  out->n_shells = static_cast<int32_t>(std::min<size_t>(sh.size(), 32));
  for (int i = 0; i < out->n_shells; ++i) out->dwi_shells[i] = sh[i];
  out->lmax = lmax;
  out->n_constraint_dirs = ndirs;
  out->total_iterations = total_it;
  std::snprintf(out->warnings, sizeof out->warnings, "%s", warnings.c_str());
  return 0;
}

}  // extern "C"


// ------------------------------------------------- synth.rs / odf projection

namespace {

// y = A c with A (R x K) and the products summed in column order, as the
// reference's gemv / per-row loop (synth.rs:60, models.rs:238-243).
void apply_rows(const Mat& A, const double* c, double* y) {
  for (int i = 0; i < A.rows; ++i) {
    double acc = 0.0;
    for (int k = 0; k < A.cols; ++k) acc += A(i, k) * c[k];
    y[i] = acc;
  }
}

}  // namespace

int oracle_shore_predict(const float* coeffs, int64_t X, int64_t Y, int64_t Z, int32_t radial_order,
                         double zeta, const csd_gtab* target, float* out, char* err, size_t err_len) {
  try {
    const Gtab g = make_gtab(target);
    const Mat M = design_matrix(g, radial_order, zeta);
    const int K = M.cols, N = M.rows;
    std::vector<double> c(K), y(N);
    for (int64_t v = 0; v < X * Y * Z; ++v) {
      const float* cv = coeffs + v * K;
      float* ov = out + v * N;
      bool any = false;
      for (int k = 0; k < K; ++k) any |= (cv[k] != 0.0f);  // synth.rs:55-58
      if (!any) {
        for (int t = 0; t < N; ++t) ov[t] = 0.0f;
        continue;
      }
      for (int k = 0; k < K; ++k) c[k] = static_cast<double>(cv[k]);
      apply_rows(M, c.data(), y.data());
      for (int t = 0; t < N; ++t) ov[t] = static_cast<float>(y[t]);
    }
    return 0;
  } catch (const std::exception& e) {
    set_err(err, err_len, e.what());
    return 1;
  }
}

int oracle_shore_odf_sh(const float* coeffs, int64_t X, int64_t Y, int64_t Z, int32_t radial_order,
                        double zeta, int32_t lmax, const uint8_t* mask, float* out, char* err,
                        size_t err_len) {
  try {
    const Mat P = shore_to_tournier(radial_order, zeta, lmax);
    const int K = P.cols, R = P.rows;
    std::vector<double> c(K), y(R);
    for (int64_t v = 0; v < X * Y * Z; ++v) {
      float* ov = out + v * R;
      if (mask && !mask[v]) {
        for (int i = 0; i < R; ++i) ov[i] = 0.0f;
        continue;
      }
      for (int k = 0; k < K; ++k) c[k] = static_cast<double>(coeffs[v * K + k]);
      apply_rows(P, c.data(), y.data());
      for (int i = 0; i < R; ++i) ov[i] = static_cast<float>(y[i]);
    }
    return 0;
  } catch (const std::exception& e) {
    set_err(err, err_len, e.what());
    return 1;
  }
}

// ------------------------------------------------ scalars/microstructure.rs

namespace {

double binomial_float(double n, uint32_t k) {  // math.rs:150-152
  return gamma_fn(n + 1.0) / (factorial(k) * gamma_fn(n - static_cast<double>(k) + 1.0));
}

struct NlBlock {
  int n, l, start, len;
};

std::vector<NlBlock> nl_blocks(int radial_order) {  // microstructure.rs:42-58
  std::vector<NlBlock> b;
  int start = 0;
  for (int n = 0; n <= radial_order; ++n)
    for (int l = 0; l <= n; l += 2) {
      b.push_back({n, l, start, 2 * l + 1});
      start += 2 * l + 1;
    }
  return b;
}

int n00_index(const std::vector<NlBlock>& b, int n) {  // microstructure.rs:62-71
  for (const auto& x : b)
    if (x.n == n && x.l == 0) return x.start;
  return -1;
}

// Ê(0) = sum_n c_(n,0,0) kappa(n, 0) L_n^(1/2)(0) / sqrt(4 pi) (:76-88).
double predict_e0(const double* c, int radial_order, double zeta, const std::vector<NlBlock>& b) {
  double e0 = 0.0;
  const double inv = 1.0 / std::sqrt(4.0 * kPi);
  for (int n = 0; n <= radial_order; ++n) {
    const double r0 = kappa(zeta, n, 0) * gen_laguerre(n, 0.5, 0.0);
    e0 += c[n00_index(b, n)] * r0 * inv;
  }
  return e0;
}

double alpha_factor(uint32_t n, uint32_t l, double zeta) {  // :272-278
  const double sign = ((l / 2) % 2 == 0) ? 1.0 : -1.0;
  const double num = 2.0 * kPi * std::pow(zeta, 1.5) * gamma_fn(static_cast<double>(n) + 1.5);
  const double den = std::pow(2.0, static_cast<int>(l)) * factorial(n - l);
  return sign * std::sqrt(num / den);
}

double rtap_kappa(uint32_t j, uint32_t l) {  // :284-298
  const double jf = j, lf = l;
  const double kap = std::pow(-1.0, static_cast<int>(j) - 1) * std::pow(2.0, -(lf + 3.0) / 2.0) / kPi;
  double sum = 0.0;
  for (uint32_t k = 0; k < j; ++k) {
    const double kf = k;
    const double sign = (k % 2 == 0) ? 1.0 : -1.0;
    const double bin = binomial_float(jf + lf - 0.5, j - k - 1);
    const double g = gamma_fn((lf + 1.0) / 2.0 + kf);
    const double hp = std::pow(0.5, (lf + 1.0) / 2.0 + kf);
    sum += sign * bin * g / (factorial(k) * hp);
  }
  return 2.0 * kap * sum;
}

double rtpp_kappa(uint32_t j, uint32_t l) {  // :301-315
  const double jf = j, lf = l;
  const double pre = std::pow(-0.5, lf / 2.0) / std::sqrt(kPi);
  double sum = 0.0;
  for (uint32_t k = 0; k < j; ++k) {
    const double kf = k;
    const double sign = (k % 2 == 0) ? 1.0 : -1.0;
    const double bin = binomial_float(jf + lf - 0.5, j - k - 1);
    const double g = gamma_fn(lf / 2.0 + kf + 0.5);
    const double hp = std::pow(0.5, lf / 2.0 + 0.5 + kf);
    sum += sign * bin * g / (factorial(k) * hp);
  }
  return pre * sum;
}

// RTAP (rtap = true) / RTPP along `dir` (:209-270).
double direction_scalar(const double* c, int radial_order, double zeta, const std::vector<NlBlock>& b,
                        const double* dir, bool rtap) {
  if (!dir) return std::nan("");
  const double norm = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  if (!std::isfinite(norm) || norm == 0.0) return std::nan("");
  const double e0 = predict_e0(c, radial_order, zeta, b);
  if (!std::isfinite(e0) || e0 == 0.0) return std::nan("");
  const double inv = 1.0 / norm;
  double r, theta, phi;
  cart2sphere(dir[0] * inv, dir[1] * inv, dir[2] * inv, &r, &theta, &phi);
  double acc = 0.0;
  double sh[32];
  for (const auto& blk : b) {
    const uint32_t j = static_cast<uint32_t>(blk.n - blk.l + 1);
    const double kern = rtap ? rtap_kappa(j, blk.l) : rtpp_kappa(j, blk.l);
    if (kern == 0.0) continue;
    const double scale = kern / alpha_factor(blk.n, blk.l, zeta);
    brainsuite_sh_block(blk.l, theta, phi, sh);
    double inner = 0.0;
    for (int k = 0; k < blk.len; ++k) inner += (c[blk.start + k] / e0) * sh[k];
    acc += scale * inner;
  }
  const double mu = 1.0 / (2.0 * kPi * std::sqrt(zeta));
  const double pre = rtap ? 1.0 / (mu * mu) : 1.0 / mu;
  return std::max(pre * acc, 0.0);
}

void micro_voxel(const double* c, int K, int radial_order, double zeta, const std::vector<NlBlock>& b,
                 const double* dir, double* out) {
  const double nan = std::nan("");
  const double e0 = predict_e0(c, radial_order, zeta, b);
  const bool bad = !std::isfinite(e0) || e0 == 0.0;
  // RTOP (:98-118)
  double rtop = nan;
  if (!bad) {
    double acc = 0.0;
    for (int n = 0; n <= radial_order; ++n) {
      const double cn = c[n00_index(b, n)] / e0;
      const double sign = (n % 2 == 0) ? 1.0 : -1.0;
      const double w = std::sqrt(16.0 * kPi * std::pow(zeta, 1.5) * gamma_fn(n + 1.5) / factorial(n));
      acc += cn * sign * w;
    }
    rtop = std::max(acc, 0.0);
  }
  // MSD (:122-140)
  double msd = nan;
  if (!bad) {
    double acc = 0.0;
    for (int n = 0; n <= radial_order; ++n) {
      const double cn = c[n00_index(b, n)] / e0;
      const double sign = (n % 2 == 0) ? 1.0 : -1.0;
      const double w = std::sqrt(9.0 * gamma_fn(n + 1.5) /
                                 (8.0 * std::pow(kPi, 6) * std::pow(zeta, 3.5) * factorial(n)));
      const double hyp = hyp2f1(-static_cast<double>(n), 2.5, 1.5, 2.0);
      acc += cn * sign * w * hyp;
    }
    msd = std::max(acc, 0.0);
  }
  // QIV (:155-182)
  double qiv = nan;
  if (!bad) {
    const double pre = 6.0 * std::sqrt(2.0 * kPi) * std::pow(zeta, 2.5);
    double q2i = 0.0;
    for (int n = 0; n <= radial_order; ++n) {
      const double cn = c[n00_index(b, n)] / e0;
      q2i += cn * kappa(zeta, n, 0) * gamma_fn(n + 1.5) / factorial(n) *
             hyp2f1(-static_cast<double>(n), 2.5, 1.5, 2.0);
    }
    const double q2 = pre * q2i;
    if (std::isfinite(q2) && q2 > 0.0) qiv = 1.0 / q2;
  }
  // NG (:186-198)
  double ng = nan;
  if (!bad) {
    double total = 0.0;
    for (int k = 0; k < K; ++k) {
      const double cn = c[k] / e0;
      total += cn * cn;
    }
    if (total == 0.0) {
      ng = 0.0;
    } else {
      const double c0 = c[0] / e0;
      ng = std::sqrt(std::max(1.0 - (c0 * c0) / total, 0.0));
    }
  }
  out[0] = rtop;
  out[1] = msd;
  out[2] = qiv;
  out[3] = ng;
  out[4] = direction_scalar(c, radial_order, zeta, b, dir, true);
  out[5] = direction_scalar(c, radial_order, zeta, b, dir, false);
}

// Nearest-rank percentile of the finite values (io/microstructure.rs:303-313).
bool percentile_value(const std::vector<float>& xs, double percentile, float* out) {
  std::vector<float> f;
  for (float v : xs)
    if (std::isfinite(v)) f.push_back(v);
  if (f.empty()) return false;
  std::sort(f.begin(), f.end());
  const size_t n = f.size();
  const double p = std::min(std::max(percentile, 0.0), 100.0) / 100.0;
  const size_t idx = std::min(static_cast<size_t>(std::round(p * static_cast<double>(n - 1))), n - 1);
  *out = f[idx];
  return true;
}

}  // namespace

void oracle_microstructure_voxel(const double* coefs, int32_t radial_order, double zeta, const double* dir,
                                 double* out) {
  const auto b = nl_blocks(radial_order);
  const int K = static_cast<int>(shore_indices(radial_order).size());
  micro_voxel(coefs, K, radial_order, zeta, b, dir, out);
}

double oracle_micro_alpha_factor(uint32_t n, uint32_t l, double zeta) { return alpha_factor(n, l, zeta); }

int oracle_shore_microstructure(const float* coeffs, int64_t X, int64_t Y, int64_t Z, int32_t radial_order,
                                double zeta, const uint8_t* mask, const float* directions, int32_t units,
                                int32_t reject, float outlier_factor, float* rtop, float* rtap, float* rtpp,
                                float* msd, float* qiv, float* ng, char* err, size_t err_len) {
  try {
    const int K = static_cast<int>(shore_indices(radial_order).size());
    const auto b = nl_blocks(radial_order);
    // unit scales (io/microstructure.rs:162-173): rtop, rtap, rtpp, msd, qiv, ng
    const float sc_um[6] = {1e-9f, 1e-6f, 1e-3f, 1e6f, 1e15f, 1.0f};
    const float sc_mm[6] = {1.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f};
    const float* sc = units == 1 ? sc_mm : sc_um;
    const int64_t nvox = X * Y * Z;
    std::vector<int64_t> idx;
    for (int64_t v = 0; v < nvox; ++v)
      if (mask[v]) idx.push_back(v);
    std::vector<float> s[6];  // rtop, rtap, rtpp, msd, qiv, ng (masked order)
    for (auto& a : s) a.resize(idx.size());
    std::vector<double> c(K);
    double out[6];
    for (size_t i = 0; i < idx.size(); ++i) {
      const int64_t v = idx[i];
      for (int k = 0; k < K; ++k) c[k] = static_cast<double>(coeffs[v * K + k]);
      double dir[3];
      const double* dp = nullptr;
      if (directions) {
        const float* d = directions + v * 3;
        const bool any = d[0] != 0.0f || d[1] != 0.0f || d[2] != 0.0f;
        const bool fin = std::isfinite(d[0]) && std::isfinite(d[1]) && std::isfinite(d[2]);
        if (any && fin) {
          dir[0] = d[0];
          dir[1] = d[1];
          dir[2] = d[2];
          dp = dir;
        }
      }
      micro_voxel(c.data(), K, radial_order, zeta, b, dp, out);
      // out = {rtop, msd, qiv, ng, rtap, rtpp}; f64 -> f32, then the f32 unit scale
      s[0][i] = static_cast<float>(out[0]) * sc[0];
      s[1][i] = static_cast<float>(out[4]) * sc[1];
      s[2][i] = static_cast<float>(out[5]) * sc[2];
      s[3][i] = static_cast<float>(out[1]) * sc[3];
      s[4][i] = static_cast<float>(out[2]) * sc[4];
      s[5][i] = static_cast<float>(out[3]) * sc[5];
    }
    if (reject) {  // io/microstructure.rs:222-270 and nan_above (:317-326)
      for (auto& a : s) {
        float p99;
        if (!percentile_value(a, 99.0, &p99)) continue;
        const float thr = outlier_factor * p99;
        for (float& v : a)
          if (std::isfinite(v) && v > thr) v = std::nanf("");
      }
    }
    float* maps[6] = {rtop, rtap, rtpp, msd, qiv, ng};
    for (int m = 0; m < 6; ++m) {
      for (int64_t v = 0; v < nvox; ++v) maps[m][v] = 0.0f;
      for (size_t i = 0; i < idx.size(); ++i) maps[m][idx[i]] = s[m][i];
    }
    return 0;
  } catch (const std::exception& e) {
    set_err(err, err_len, e.what());
    return 1;
  }
}
