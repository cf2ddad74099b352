// Host plan-time geometry of the stretched leaf: sizes, colatitude periodisation, window,
// polar-optimisation limits. Restates src/Windows.jl, src/Stretch.jl:52-81,151-213 and
// src/Legendre.jl:31-145,194-293 of PartialFSHT.jl (plan time only; nothing here runs
// per apply).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace pf {

enum Kind { kPole = 0, kInterior = 1, kFull = 2, kDirect = 3, kMultiBox = 4 };

struct Geom {
    int kind = kPole;
    int lmax = 0;
    double eps = 0, beta = 0, h = 0, lo = 0, hi = 0, eps_apo = 0, period = 0;
    int64_t K = 0;
    double Theta1 = 0, sigma = 0, ThetaT = 0, invZ = 0;
};

int64_t next_smooth(int64_t n);        // src/Stretch.jl:61-81
int64_t next_smooth_even(int64_t n);   // src/Stretch.jl:52
int polar_mmax(double theta, int lmax, double eps);  // src/Legendre.jl:48-57
void sectorial_log2c(int lmax, std::vector<double>& out);  // src/Legendre.jl:65-75
// src/Legendre.jl:89-127; returns false when mlim is not unimodal
bool nested_ranges(const std::vector<int>& mlim, int lmax, std::vector<int>& jlo,
                   std::vector<int>& jhi);
double es_cdf(double beta, double u);  // src/Windows.jl:208-226
// src/Windows.jl:84-141: 1 admissible, 0 none, -1 bad interval
int try_geometry(double lo, double hi, int lmax, double eps, double eps_apo_max, Geom* g);
double window(const Geom& g, double Th);     // src/Windows.jl:237-250
double to_theta(const Geom& g, double Th);   // src/Windows.jl:272-282
double to_stretch(const Geom& g, double th); // src/Windows.jl:289-298
double jl_mod(double x, double y);           // Julia's floating mod()

// Everything StretchLeaf derives at construction (src/Stretch.jl:129-238), host side.
struct Leaf {
    Geom g;
    bool flip = false;
    int lmax = 0, ntrans = 1;
    int nth_half = 0, nth = 0, nph = 0, mmax = 0;
    std::vector<double> theta_rings, Theta_rings, w, cos_t, log2sin, log2c;
    std::vector<int> mlim, jlo, jhi;
    int64_t ring_work = 0;
    int spin = 0;
};

// 0 ok, 1 refused geometry, 2 bad arguments (message in err)
int build_leaf(double box_lo, double box_hi, int lmax, int ntrans, double tol,
               double eps_apo_max, double ovs_theta, double ovs_phi, Leaf* out,
               std::string* err, int spin = 0);

// ES kernel parameters of the NUFFT (published FINUFFT choice at upsampling 2)
int es_width(double tol);
double es_kernel(double z, double beta);
double es_deconv(int k, int nf, int w, double beta);  // 1 / Phi(k)

}  // namespace pf
