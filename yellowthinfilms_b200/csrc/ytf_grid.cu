// ytf_grid.cu -- host side of the Sommerfeld k-grid builder; see ytf_grid.h.
#include "ytf_grid.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <limits>
#include <stdexcept>

namespace ytf {
namespace grid {

namespace {

using cplx = std::complex<double>;

// merge sorted values closer than rtol (relative)
std::vector<double> merge_close(const std::vector<double>& ks, double rtol = 1e-9) {
  std::vector<double> out;
  for (double k : ks)
    if (out.empty() || k - out.back() > rtol * std::max(std::fabs(k), 1e-300)) out.push_back(k);
  return out;
}

cplx det3(const cplx A[3][3]) {
  return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
         A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

// inverse by cofactors over the determinant
void inv3(const cplx A[3][3], cplx B[3][3]) {
  const cplx d = det3(A);
  B[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) / d;
  B[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) / d;
  B[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) / d;
  B[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) / d;
  B[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) / d;
  B[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) / d;
  B[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) / d;
  B[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) / d;
  B[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) / d;
}

void matmul3(const cplx X[3][3], const cplx Y[3][3], cplx Z[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      cplx a = 0;
      for (int k = 0; k < 3; ++k) a += X[i][k] * Y[k][j];
      Z[i][j] = a;
    }
}

}  // namespace

std::vector<double> layer_light_lines(const double* eps, const double* mu, double w, double phi) {
  cplx e[3][3], m[3][3], mi[3][3], K[3][3], T[3][3], M[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      e[i][j] = cplx(eps[2 * (i + 3 * j)], eps[2 * (i + 3 * j) + 1]);
      m[i][j] = cplx(mu[2 * (i + 3 * j)], mu[2 * (i + 3 * j) + 1]);
      K[i][j] = 0.0;
    }
  // K(φ) k_t: the in-plane wave vector's cross-product matrix for the unit direction (c, s, 0)
  const double c = std::cos(phi), s = std::sin(phi);
  K[0][2] = s; K[1][2] = -c; K[2][0] = -s; K[2][1] = c;
  inv3(m, mi);
  matmul3(K, mi, T);
  matmul3(T, K, M);
  double me = 0, mm = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      me = std::max(me, std::abs(e[i][j]));
      mm = std::max(mm, std::abs(m[i][j]));
    }
  // p(q) = det(ω² ε + q M) is a quadratic in q: sample it at q = 0, sc, 2 sc
  const double w2 = w * w;
  const double sc = w2 * std::max(me * mm, std::numeric_limits<double>::epsilon());
  cplx A0[3][3], A1[3][3], A2[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      A0[i][j] = w2 * e[i][j];
      A1[i][j] = A0[i][j] + sc * M[i][j];
      A2[i][j] = A0[i][j] + (2 * sc) * M[i][j];
    }
  const cplx p0 = det3(A0), p1 = det3(A1), p2 = det3(A2);
  const cplx c2 = (p2 - 2.0 * p1 + p0) / (2 * sc * sc);
  const cplx c1 = (p1 - p0) / sc - c2 * sc;
  const cplx c0 = p0;
  std::vector<cplx> roots;
  if (std::abs(c2) * sc * sc <= 1e-12 * (std::abs(c1) * sc + std::abs(c0))) {
    if (std::abs(c1) > 0) roots.push_back(-c0 / c1);
  } else {
    const cplx D = c1 * c1 - 4.0 * c2 * c0;
    const cplx Dl = std::abs(D) <= 1e-10 * std::norm(c1) ? cplx(0.0, 0.0) : std::sqrt(D);
    roots.push_back((-c1 + Dl) / (2.0 * c2));
    roots.push_back((-c1 - Dl) / (2.0 * c2));
  }
  std::vector<double> out;
  for (auto& q : roots)
    if (q.real() > 0) out.push_back(std::sqrt(q).real());
  std::sort(out.begin(), out.end());
  return merge_close(out, 1e-7);
}

int real_axis_poles(const Eval& f, double phi, double k_lo, double k_hi, double scan_step, double prominence,
                    const std::vector<double>& exclude, std::vector<Pole>& out, double floor_rel, double floor_abs) {
  const double span = std::log(k_hi / k_lo);
  const int n = (int)std::floor(span / scan_step + 1e-10) + 1;
  std::vector<double> ks(n), v;
  for (int i = 0; i < n; ++i) ks[i] = k_lo * std::exp(i * scan_step);
  const int Wn = (int)std::ceil(std::log(4.0) / scan_step);
  int rc = f(ks, v);
  if (rc) return rc;
  std::vector<double> y(n);
  for (int i = 0; i < n; ++i) y[i] = std::log(v[i] + 1e-300);
  const double ymax = *std::max_element(y.begin(), y.end());
  const double ymin = std::max(ymax + std::log(floor_rel), std::log(floor_abs));
  struct Peak {
    int i, jl, jr;
    double lmin, rmin, base, prom;
    double a, b, c, d, fc, fd;  // golden-section bracket
    bool open;
    double q, lvl, lo[2], hi[2];  // crossings: [0] left, [1] right
    bool bis[2];
  };
  std::vector<Peak> P;
  for (int i = 1; i < n - 1; ++i) {
    if (!(y[i] > y[i - 1] && y[i] >= y[i + 1] && y[i] >= ymin)) continue;
    int jl = i;
    double lmin = y[i];
    while (jl > std::max(0, i - Wn) && y[jl - 1] <= y[i]) { --jl; lmin = std::min(lmin, y[jl]); }
    int jr = i;
    double rmin = y[i];
    while (jr < std::min(n - 1, i + Wn) && y[jr + 1] <= y[i]) { ++jr; rmin = std::min(rmin, y[jr]); }
    const double base = std::max(lmin, rmin);
    const double prom = y[i] - base;
    if (!(prom >= std::log(prominence))) continue;
    Peak p{};
    p.i = i; p.jl = jl; p.jr = jr; p.lmin = lmin; p.rmin = rmin; p.base = base; p.prom = prom;
    P.push_back(p);
  }
  const double g = (std::sqrt(5.0) - 1) / 2;
  // golden section on [ks[i-1], ks[i+1]], all peaks in lockstep
  std::vector<double> pts;
  for (auto& p : P) {
    p.a = ks[p.i - 1];
    p.b = ks[p.i + 1];
    p.c = p.b - g * (p.b - p.a);
    p.d = p.a + g * (p.b - p.a);
    p.open = true;
    pts.push_back(p.c);
    pts.push_back(p.d);
  }
  if (!P.empty()) {
    if ((rc = f(pts, v))) return rc;
    for (size_t k = 0; k < P.size(); ++k) { P[k].fc = v[2 * k]; P[k].fd = v[2 * k + 1]; }
  }
  for (int it = 0; it < 60; ++it) {
    pts.clear();
    std::vector<std::pair<int, bool>> need;  // (peak, new point is c)
    for (size_t k = 0; k < P.size(); ++k) {
      Peak& p = P[k];
      if (!p.open) continue;
      if ((p.b - p.a) <= 1e-12 * p.b) { p.open = false; continue; }
      if (p.fc >= p.fd) {
        p.b = p.d; p.d = p.c; p.fd = p.fc; p.c = p.b - g * (p.b - p.a);
        pts.push_back(p.c);
        need.push_back({(int)k, true});
      } else {
        p.a = p.c; p.c = p.d; p.fc = p.fd; p.d = p.a + g * (p.b - p.a);
        pts.push_back(p.d);
        need.push_back({(int)k, false});
      }
    }
    if (pts.empty()) break;
    if ((rc = f(pts, v))) return rc;
    for (size_t t = 0; t < need.size(); ++t) {
      Peak& p = P[need[t].first];
      if (need[t].second) p.fc = v[t];
      else p.fd = v[t];
    }
  }
  pts.clear();
  for (auto& p : P) {
    p.q = (p.a + p.b) / 2;
    pts.push_back(p.q);
  }
  if (!P.empty() && (rc = f(pts, v))) return rc;
  std::vector<bool> keep(P.size(), true);
  for (size_t k = 0; k < P.size(); ++k) {
    Peak& p = P[k];
    const double Pk = std::max(v[k], std::exp(y[p.i]));
    for (double L : exclude)
      if (std::fabs(p.q - L) <= 1e-6 * p.q) keep[k] = false;
    p.lvl = std::exp(p.base) + (Pk - std::exp(p.base)) / std::sqrt(2.0);
    int jlast = p.jl;
    for (int j = p.jl; j <= p.i; ++j)
      if (y[j] == p.lmin) jlast = j;
    int jfirst = p.i;
    for (int j = p.i; j <= p.jr; ++j)
      if (y[j] == p.rmin) { jfirst = j; break; }
    p.lo[0] = p.q; p.hi[0] = ks[jlast];
    p.lo[1] = p.q; p.hi[1] = ks[jfirst];
    p.bis[0] = p.bis[1] = keep[k];
  }
  // half-power crossings by bisection, both sides of every kept peak in lockstep
  for (int it = 0; it < 50; ++it) {
    pts.clear();
    std::vector<std::pair<int, int>> need;
    for (size_t k = 0; k < P.size(); ++k)
      for (int sd = 0; sd < 2; ++sd) {
        Peak& p = P[k];
        if (!p.bis[sd]) continue;
        if (std::fabs(p.hi[sd] - p.lo[sd]) <= 1e-12 * p.q) { p.bis[sd] = false; continue; }
        pts.push_back((p.lo[sd] + p.hi[sd]) / 2);
        need.push_back({(int)k, sd});
      }
    if (pts.empty()) break;
    if ((rc = f(pts, v))) return rc;
    for (size_t t = 0; t < need.size(); ++t) {
      Peak& p = P[need[t].first];
      const int sd = need[t].second;
      const double mid = (p.lo[sd] + p.hi[sd]) / 2;
      if (v[t] > p.lvl) p.lo[sd] = mid;
      else p.hi[sd] = mid;
    }
  }
  for (size_t k = 0; k < P.size(); ++k) {
    if (!keep[k]) continue;
    const Peak& p = P[k];
    const double cl = (p.lo[0] + p.hi[0]) / 2, cr = (p.lo[1] + p.hi[1]) / 2;
    const double G = std::min(p.q - cl, cr - p.q);
    out.push_back({p.q, std::max(G, 1e-12 * p.q), phi, p.prom});
  }
  return 0;
}

std::vector<Cluster> clusters(std::vector<Pole> ps, double merge_rel) {
  std::stable_sort(ps.begin(), ps.end(), [](const Pole& x, const Pole& y) { return x.q < y.q; });
  std::vector<Cluster> cl;
  auto add = [&](Cluster c) {
    for (auto& e : cl)
      if (e.a == c.a && e.b == c.b && e.G == c.G) return;
    cl.push_back(c);
  };
  for (size_t i = 0; i < ps.size(); ++i) {
    add({ps[i].q, ps[i].q, ps[i].G});
    if (i > 0) {
      const Pole& r = ps[i - 1];
      const Pole& p = ps[i];
      if (p.q - r.q <= std::max(merge_rel * p.q, 4 * std::min(p.G, r.G)) && p.q > r.q)
        add({r.q, p.q, std::min(p.G, r.G)});
    }
  }
  return cl;
}

int features_1d(const std::vector<const double*>& eps, const std::vector<const double*>& mu, double w, double h_min,
                double rho_max, double target_decay, double kr_cap, double kr_cap_rel, bool scan, double scan_step,
                double prominence, const Eval& f, Features& F) {
  const int N = (int)eps.size();
  std::vector<double> ll, sing;
  for (int j = 0; j < N; ++j) {
    auto L = layer_light_lines(eps[j], mu[j], w, 0.0);
    ll.insert(ll.end(), L.begin(), L.end());
    if (j == 0 || j == N - 1) sing.insert(sing.end(), L.begin(), L.end());
  }
  std::sort(ll.begin(), ll.end());
  std::sort(sing.begin(), sing.end());
  F.light_lines = merge_close(ll);
  F.singular_lines = merge_close(sing);
  F.kmax = F.light_lines.empty() ? w : F.light_lines.back();
  F.K_geom = target_decay / h_min;
  F.K_cap = kr_cap > 0 ? kr_cap : kr_cap_rel * F.kmax;
  F.Kcut = std::min(std::max(F.K_geom, 2.0 * F.kmax), F.K_cap);
  F.capped = F.Kcut < F.K_geom;
  F.h_min = h_min;
  F.rho_max = rho_max;
  F.poles.clear();
  if (scan) {
    const double k_lo = 0.5 * (F.light_lines.empty() ? w : F.light_lines[0]);
    int rc = real_axis_poles(f, 0.0, k_lo, F.Kcut, scan_step, prominence, F.light_lines, F.poles);
    if (rc) return rc;
  }
  F.cl = clusters(F.poles, 0.0);
  return 0;
}

double pole_track_eta(const std::vector<Pole>& poles, std::vector<double> phis) {
  std::sort(phis.begin(), phis.end());
  phis.erase(std::unique(phis.begin(), phis.end()), phis.end());
  if (phis.size() < 2) return INFINITY;
  std::vector<std::array<double, 3>> pairs;  // (φ1, φ2, dφ)
  for (size_t i = 0; i + 1 < phis.size(); ++i) pairs.push_back({phis[i], phis[i + 1], phis[i + 1] - phis[i]});
  const double step = phis[1] - phis[0];
  if (std::fabs(phis.back() - phis.front() + step - 2 * M_PI) < 1e-9) pairs.push_back({phis.back(), phis.front(), step});
  double eta = INFINITY;
  for (const auto& pr : pairs)
    for (const auto& p : poles) {
      if (p.phi != pr[0]) continue;
      for (const auto& r : poles) {
        if (r.phi != pr[1]) continue;
        const double dq = std::fabs(p.q - r.q);
        if (!(0 < dq && dq <= pr[2] * std::max(p.q, r.q))) continue;
        eta = std::min(eta, std::min(p.G, r.G) * pr[2] / dq);
      }
    }
  return eta;
}

int features_2d(const std::vector<const double*>& eps, const std::vector<const double*>& mu, bool sym, bool diag,
                double w, double h_min, double rho_max, double target_decay, double kr_cap, double kr_cap_rel,
                bool scan, double scan_step, double prominence, int n_phi_scan, double c_phi, int n_phi_min,
                double rtol, double c_eta, const EvalAt& f, Features& F) {
  const int N = (int)eps.size();
  std::vector<double> phis;
  double merge_rel = 0.0;
  if (sym) {
    phis = {0.0};
  } else if (diag) {
    const int m = std::max(2, n_phi_scan / 4 + 1);
    for (int p = 0; p < m; ++p) phis.push_back((M_PI / 2) * p / (m - 1));
    merge_rel = (M_PI / 2) / std::max(1, n_phi_scan / 4);
  } else {
    for (int p = 0; p < n_phi_scan; ++p) phis.push_back(2 * M_PI * p / n_phi_scan);
    merge_rel = 2 * M_PI / n_phi_scan;
  }
  std::vector<double> phi_ll;  // light lines are even in the direction: φ mod π, first occurrences
  if (sym) {
    phi_ll = {0.0};
  } else {
    for (double ph : phis) {
      const double m = std::fmod(ph, M_PI);
      if (std::find(phi_ll.begin(), phi_ll.end(), m) == phi_ll.end()) phi_ll.push_back(m);
    }
  }
  std::vector<double> ll, sing;
  for (int j = 0; j < N; ++j)
    for (double ph : phi_ll) {
      auto L = layer_light_lines(eps[j], mu[j], w, ph);
      ll.insert(ll.end(), L.begin(), L.end());
      if (j == 0 || j == N - 1) sing.insert(sing.end(), L.begin(), L.end());
    }
  std::sort(ll.begin(), ll.end());
  std::sort(sing.begin(), sing.end());
  F.light_lines = merge_close(ll);
  F.singular_lines = merge_close(sing);
  F.kmax = F.light_lines.empty() ? w : F.light_lines.back();
  F.K_geom = target_decay / h_min;
  F.K_cap = kr_cap > 0 ? kr_cap : kr_cap_rel * F.kmax;
  F.Kcut = std::min(std::max(F.K_geom, 2.0 * F.kmax), F.K_cap);
  F.capped = F.Kcut < F.K_geom;
  F.h_min = h_min;
  F.rho_max = rho_max;
  F.phi_scan = phis;
  F.poles.clear();
  if (scan) {
    const double k_lo = 0.5 * (F.light_lines.empty() ? w : F.light_lines[0]);
    for (double ph : phis) {
      int rc = real_axis_poles(f(ph), ph, k_lo, F.Kcut, scan_step, prominence, F.light_lines, F.poles);
      if (rc) return rc;
    }
  }
  F.cl = clusters(F.poles, merge_rel);
  F.N_phi_lateral = (long)std::ceil(c_phi * F.Kcut * rho_max);
  F.eta_min = pole_track_eta(F.poles, phis);
  F.N_phi_poles = std::isfinite(F.eta_min) ? (long)std::ceil(c_eta * std::log(10 / rtol) / F.eta_min) : 0;
  const long m = std::max(std::max((long)n_phi_min, F.N_phi_lateral), F.N_phi_poles);
  F.N_phi = 2 * ((m + 1) / 2);
  return 0;
}

void sampled_peaks(const double* ks, const double* y, int n, double prominence, double floor_rel,
                   std::vector<std::pair<double, double>>& out) {
  if (n < 3) return;
  double ymax = -INFINITY;
  for (int i = 0; i < n; ++i) ymax = std::max(ymax, y[i]);
  const double ymin = std::max(ymax + std::log(floor_rel), std::log(1e-10));
  const double l0 = std::log(ks[0]), step = std::log(ks[1]) - l0;
  const int W = (int)std::ceil(std::log(4.0) / step);
  for (int i = 1; i < n - 1; ++i) {
    if (!(y[i] > y[i - 1] && y[i] >= y[i + 1] && y[i] >= ymin)) continue;
    const int lo = std::max(0, i - W), hi = std::min(n - 1, i + W);
    int jl = lo, jr = hi;
    for (int j = i - 1; j >= lo; --j)
      if (y[j] > y[i]) { jl = j + 1; break; }
    for (int j = i + 1; j <= hi; ++j)
      if (y[j] > y[i]) { jr = j - 1; break; }
    double lmin = y[i], rmin = y[i];
    for (int j = jl; j <= i; ++j) lmin = std::min(lmin, y[j]);
    for (int j = i; j <= jr; ++j) rmin = std::min(rmin, y[j]);
    const double base = std::max(lmin, rmin);
    if (y[i] - base < prominence) continue;
    const double den = y[i - 1] - 2 * y[i] + y[i + 1];
    const double off = den < 0 ? 0.5 * (y[i - 1] - y[i + 1]) / den : 0.0;
    const double lki = std::log(ks[i]);
    const double q = std::exp(lki + std::min(0.5, std::max(-0.5, off)) * step);
    const double P = std::exp(y[i]), eb = std::exp(base);
    const double lvl = std::log(eb + (P - eb) / std::sqrt(2.0));
    double G = INFINITY;
    for (int side = 0; side < 2; ++side) {
      const int dj = side == 0 ? 1 : -1;  // towards the peak
      for (int j = side == 0 ? i - 1 : i + 1; side == 0 ? j >= jl : j <= jr; j += side == 0 ? -1 : 1) {
        if (y[j] <= lvl) {
          const int prev = j + dj;
          const double t = (y[prev] - lvl) / (y[prev] - y[j]);
          const double lp = std::log(ks[prev]), lj = std::log(ks[j]);
          G = std::min(G, std::fabs(std::exp(lp + t * (lj - lp)) - q));
          break;
        }
      }
    }
    if (std::isfinite(G) && G > 0) out.push_back({q, G});
  }
}

std::vector<double> adaptive_seeds(const Features& F, double rtol, double n_gamma, int grade) {
  if (grade <= 0) grade = std::min(50, (int)std::ceil(2 * std::log2(10 / rtol)));
  std::vector<double> s(F.light_lines);
  for (double L : F.singular_lines)
    for (int j = 1; j <= grade; ++j)
      for (int sg : {-1, 1}) s.push_back(L * (1 + sg * std::ldexp(1.0, -j)));
  for (const auto& c : F.cl) {
    s.push_back(c.a - n_gamma * c.G);
    s.push_back(c.a);
    s.push_back(c.b);
    s.push_back(c.b + n_gamma * c.G);
  }
  for (double k = 2 * F.kmax; k < F.Kcut; k *= 2) s.push_back(k);
  std::vector<double> out;
  for (double x : s)
    if (0 < x && x < F.Kcut) out.push_back(x);
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

std::vector<std::pair<double, double>> fixed_kr_panels(const Features& F, int order, double rtol, double alpha,
                                                       int grade, double r_rel, double c_h, double c_rho,
                                                       double pole_safety) {
  if (!(r_rel <= alpha)) throw std::runtime_error("fixed_kρ_rule: r_rel must be ≤ α");
  // Bernstein-ellipse width that keeps a pole at distance Γ outside the panel's ellipse
  const double rB = std::pow(1 / rtol, 1.0 / (2 * order));
  const double eB = (rB - 1 / rB) / 2;
  auto wG = [&](double G) { return pole_safety * (2 * G) / eB; };
  const double w_flat = std::min(c_h / F.h_min, F.rho_max > 0 ? c_rho / F.rho_max : INFINITY);
  const double w_floor = F.kmax / 40;
  const double g2 = std::ldexp(1.0, -grade);
  auto width = [&](double k) {
    double wd = std::min(w_flat, std::max(r_rel * k, w_floor));
    for (double L : F.singular_lines) wd = std::min(wd, std::max(L * g2, alpha * std::fabs(k - L)));
    for (auto& c : F.cl) {
      const double dist = k < c.a ? c.a - k : (k > c.b ? k - c.b : 0.0);
      wd = std::min(wd, std::max(wG(c.G), alpha * dist));
    }
    return wd;
  };
  std::vector<double> bs;
  bs.push_back(0.0);
  for (double L : F.light_lines)
    if (L < F.Kcut) bs.push_back(L);
  bs.push_back(F.Kcut);
  // graded_panels (mod_KxGrid.jl:331-347)
  std::sort(bs.begin(), bs.end());
  bs.erase(std::unique(bs.begin(), bs.end()), bs.end());
  std::vector<std::pair<double, double>> panels;
  const long max_panels = 10000000;
  for (size_t i = 0; i + 1 < bs.size(); ++i) {
    const double a = bs[i], b = bs[i + 1];
    double x = a;
    while (x < b) {
      const double s = width(x) / (1 + alpha);
      if (!(s > 0)) throw std::runtime_error("graded_panels: non-positive width");
      const double yv = x + s >= b - 1e-14 * std::fabs(b) ? b : x + s;
      panels.push_back({x, yv});
      if ((long)panels.size() > max_panels) throw std::runtime_error("graded_panels: too many panels");
      x = yv;
    }
  }
  return panels;
}

}  // namespace grid
}  // namespace ytf
