// ytf_grid.h -- host side of the Sommerfeld k-grid builder (the :fixed point rule):
// light lines, the real-axis pole scan over a device-evaluated cavity response, pole
// clusters and graded Gauss-Legendre panels. The cavity response comes in through an
// evaluator callback (ytf_cavity_response on the device), so this code holds no GPU state.
#pragma once
#include <functional>
#include <utility>
#include <vector>

namespace ytf {
namespace grid {

// light lines of one layer at azimuth φ (mod_KxGrid.jl:41-59): √Re of the roots q = kt² with
// positive real part of det(ω² ε + q K(φ) μ⁻¹ K(φ)) = 0, ascending, merged at 1e-7 relative.
// eps, mu: column-major 3x3, interleaved re/im (18 doubles each)
std::vector<double> layer_light_lines(const double* eps, const double* mu, double w, double phi);

// values of the cavity response at the given kρ (one device solve per call)
using Eval = std::function<int(const std::vector<double>& k, std::vector<double>& out)>;

struct Pole {
  double q, G, phi, prom;
};
struct Cluster {
  double a, b, G;
};

// real_axis_poles (mod_KSpaceFeatures.jl:151-204) at one azimuth: log-grid scan, local maxima
// with prominence, golden-section peak, half-power crossings by bisection. The refinements of
// all peaks run in lockstep so that each iteration is one evaluator call; per peak the
// sequence of operations is the sequential algorithm's.
int real_axis_poles(const Eval& f, double phi, double k_lo, double k_hi, double scan_step, double prominence,
                    const std::vector<double>& exclude, std::vector<Pole>& out, double floor_rel = 1e-6,
                    double floor_abs = 1e-10);

// _clusters (mod_KSpaceFeatures.jl:217-229)
std::vector<Cluster> clusters(std::vector<Pole> ps, double merge_rel);

struct Features {
  std::vector<double> light_lines, singular_lines;
  double kmax = 0, Kcut = 0, h_min = 0, rho_max = 0, K_geom = 0, K_cap = 0;
  bool capped = false;
  std::vector<Pole> poles;
  std::vector<Cluster> cl;
  std::vector<double> phi_scan;  // 2D: the scanned directions
  long N_phi = 0;                // 2D: size of the uniform φ trapezoid
  long N_phi_lateral = 0, N_phi_poles = 0;
  double eta_min = 0;
};

// kspace_features for a point rule at φ = 0 (mod_KSpaceFeatures.jl:295-360): light lines of
// every layer (singular lines: those of the two half-spaces), Kcut, and the pole scan
int features_1d(const std::vector<const double*>& eps, const std::vector<const double*>& mu, double w, double h_min,
                double rho_max, double target_decay, double kr_cap, double kr_cap_rel, bool scan, double scan_step,
                double prominence, const Eval& f, Features& F);

// the cavity response along one direction φ
using EvalAt = std::function<Eval(double phi)>;

// _pole_track_η (mod_KSpaceFeatures.jl:243-259): the smallest φ-width Γ dφ / |dq| of a pole
// moving between neighbouring scanned directions; ∞ with fewer than two or no track
double pole_track_eta(const std::vector<Pole>& poles, std::vector<double> phis);

// kspace_features with dims = 2 (mod_KSpaceFeatures.jl:295-360): scanned directions (φ = 0
// for an azimuthally symmetric stack, (π/2) p / (n - 1) for p < n = N_φ_scan/4 + 1 when every
// tensor is diagonal, 2π p / N_φ_scan otherwise), light lines at every direction mod π, the
// poles of every direction, clusters merged at the φ step, and N_φ = the largest of N_φ_min,
// c_φ Kcut ρ_max and c_η log(10/rtol)/η_min, rounded up to even. sym/diag describe the stack.
int features_2d(const std::vector<const double*>& eps, const std::vector<const double*>& mu, bool sym, bool diag,
                double w, double h_min, double rho_max, double target_decay, double kr_cap, double kr_cap_rel,
                bool scan, double scan_step, double prominence, int n_phi_scan, double c_phi, int n_phi_min,
                double rtol, double c_eta, const EvalAt& f, Features& F);

// peaks of a sampled log-response on a log-uniform k grid (the scan's peak rule of
// real_axis_poles applied to samples, mod_KSpaceFeatures.jl:151-204, without the refinement
// rounds): local maxima at or above max(y) + log(floor_rel) (and log 1e-10) that stand at
// least `prominence` (log) above the higher of their two valleys (searched over a factor 4 in
// k), position by a parabola through the three samples in log k (offset clipped to half a
// step), Γ from the nearer crossing of the half-power level, linear in log k. Appends (q, Γ).
void sampled_peaks(const double* ks, const double* y, int n, double prominence, double floor_rel,
                   std::vector<std::pair<double, double>>& out);

// adaptive_seeds (mod_KSpaceFeatures.jl:421-445): starting breakpoints of the adaptive engine
// -- the light lines, L (1 ± 2^-j), j = 1..grade, at every singular line, each cluster's
// [a - nΓ Γ, a, b, b + nΓ Γ], and 2 kmax, 4 kmax, ... below Kcut; those in (0, Kcut), sorted,
// duplicates removed. grade <= 0: min(50, ceil(2 log2(10 / rtol))).
std::vector<double> adaptive_seeds(const Features& F, double rtol, double n_gamma = 4.0, int grade = 0);

// fixed_kρ_rule (mod_KSpaceFeatures.jl:396-419) up to the panels: graded_panels
// (mod_KxGrid.jl:331-347) between 0, the light lines below Kcut and Kcut. Throws
// std::runtime_error with the reference's messages.
std::vector<std::pair<double, double>> fixed_kr_panels(const Features& F, int order, double rtol, double alpha,
                                                       int grade, double r_rel, double c_h, double c_rho,
                                                       double pole_safety);

}  // namespace grid
}  // namespace ytf
