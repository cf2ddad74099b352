// Host plan-time geometry (see geometry.hpp). Each function cites the PartialFSHT.jl
// routine it restates; the arithmetic is kept in the reference's order so plan sizes
// agree exactly.
#include "geometry.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>

namespace pf {

int64_t next_smooth(int64_t n) {
    if (n <= 1) return 1;
    int64_t best = INT64_MAX;
    for (int64_t p2 = 1; p2 < 2 * n + 2; p2 *= 2)
        for (int64_t p3 = p2; p3 < 2 * n + 2; p3 *= 3)
            for (int64_t p5 = p3; p5 < 2 * n + 2; p5 *= 5)
                if (p5 >= n && p5 < best) best = p5;
    return best == INT64_MAX ? n : best;
}

int64_t next_smooth_even(int64_t n) {
    int64_t h = n > 0 ? (n + 1) / 2 : -((-n) / 2);  // cld(n, 2)
    return 2 * next_smooth(h);
}

int polar_mmax(double theta, int L, double eps) {
    if (L <= 0) return 0;
    const double pad_factor = 0.5 * std::cbrt(9.0);
    double s = std::fabs(std::sin(theta));
    double z = ((double)L + 0.5) * s;
    double le = std::fabs(std::log(std::fmax(eps, DBL_MIN)));
    double pad = pad_factor * std::cbrt(std::fmax(z, 1.0)) * std::cbrt(le * le) + 2.0;
    double c = std::ceil(z + pad);
    if (c < 0) return 0;
    if (c > L) return L;
    return (int)c;
}

void sectorial_log2c(int L, std::vector<double>& v) {
    v.assign(L + 1, 0.0);
    double acc = -std::log2(std::sqrt(4.0 * M_PI));
    v[0] = acc;
    for (int m = 1; m <= L; ++m) {
        acc += std::log2(std::sqrt((double)(2 * m + 1) / (double)(2 * m)));
        v[m] = acc;
    }
}

bool nested_ranges(const std::vector<int>& mlim, int L, std::vector<int>& jlo,
                   std::vector<int>& jhi) {
    const int n = (int)mlim.size();
    if (n < 1) return false;
    int peak = 0;
    for (int j = 1; j < n; ++j)
        if (mlim[j] > mlim[peak]) peak = j;
    for (int j = 1; j <= peak; ++j)
        if (mlim[j] < mlim[j - 1]) return false;
    for (int j = peak + 1; j < n; ++j)
        if (mlim[j] > mlim[j - 1]) return false;
    jlo.assign(L + 1, 0);
    jhi.assign(L + 1, -1);
    int lo = peak, hi = peak;
    int mtop = std::min(mlim[peak], L);
    for (int m = mtop; m >= 0; --m) {
        while (lo > 0 && mlim[lo - 1] >= m) --lo;
        while (hi < n - 1 && mlim[hi + 1] >= m) ++hi;
        jlo[m] = lo;
        jhi[m] = hi;
    }
    return true;
}

// 10-point Gauss-Legendre nodes and weights on [-1, 1] (standard published values)
static const double kGLX[10] = {-0.9739065285171717, -0.8650633666889845, -0.6794095682990244,
                                -0.4333953941292472, -0.1488743389816312, 0.1488743389816312,
                                0.4333953941292472,  0.6794095682990244,  0.8650633666889845,
                                0.9739065285171717};
static const double kGLW[10] = {0.0666713443086881, 0.1494513491505806, 0.2190863625159820,
                                0.2692667193099963, 0.2955242247147529, 0.2955242247147529,
                                0.2692667193099963, 0.2190863625159820, 0.1494513491505806,
                                0.0666713443086881};

double es_cdf(double beta, double u) {
    const double panel = 0.05;
    double a = -M_PI / 2;
    if (u <= a) return 0.0;
    double b = std::fmin(u, M_PI / 2);
    int n = std::max(1, (int)std::ceil((b - a) / panel));
    double hw = (b - a) / (2 * n);
    double acc = 0.0;
    for (int p = 0; p < n; ++p) {
        double c = a + (2 * p + 1) * hw;
        double s = 0.0;
        for (int q = 0; q < 10; ++q) {
            double t = c + hw * kGLX[q];
            double ct = std::cos(t);
            s += kGLW[q] * std::exp(beta * (ct - 1)) * ct;
        }
        acc += hw * s;
    }
    return acc;
}

int try_geometry(double lo, double hi, int L, double eps, double eps_apo_max, Geom* out) {
    if (!(lo <= hi)) return -1;
    if (!(lo >= 0 && hi <= M_PI)) return -1;
    double beta = std::fabs(std::log(eps));
    double tiny = std::sqrt(DBL_EPSILON);
    double Z = es_cdf(beta, M_PI / 2);
    double invZ = Z > 0 ? 1.0 / Z : 0.0;
    if (lo <= tiny && hi >= M_PI - tiny) {
        Geom g;
        g.kind = kFull; g.lmax = L; g.eps = eps; g.beta = beta; g.h = M_PI / 2; g.lo = 0.0;
        g.hi = M_PI; g.eps_apo = 0.0; g.period = 2 * M_PI; g.K = L; g.Theta1 = M_PI;
        g.sigma = 0.0; g.ThetaT = M_PI; g.invZ = 1.0;
        *out = g;
        return 1;
    }
    struct Cand { int kind; double h, klo, khi; };
    const Cand cands[3] = {{kPole, hi, 0.0, hi}, {kPole, M_PI - lo, lo, M_PI},
                           {kInterior, (hi - lo) / 2, lo, hi}};
    int64_t bestK = INT64_MAX;
    int found = 0;
    for (const Cand& c : cands) {
        double h = c.h;
        if (!(h > 0)) continue;
        double Lh = (double)L * h;
        if (!(Lh >= 2 * beta / (eps_apo_max * eps_apo_max))) continue;
        double ea = std::sqrt(2 * beta / Lh);
        double pad = h * ea;
        if (c.kind == kInterior) {
            if (!(c.klo - pad >= 0 && c.khi + pad <= M_PI)) continue;
        } else if (!(h * (1 + ea) <= M_PI)) {
            continue;
        }
        int64_t K = std::max<int64_t>(1, (int64_t)std::ceil(Lh * ((1 + ea) * (1 + ea)) / M_PI));
        if (K < bestK) {
            bestK = K;
            Geom g;
            g.kind = c.kind; g.lmax = L; g.eps = eps; g.beta = beta; g.h = h; g.lo = c.klo;
            g.hi = c.khi; g.eps_apo = ea; g.period = 2 * h * (1 + ea); g.K = K;
            g.Theta1 = M_PI / (1 + ea); g.sigma = (M_PI - g.Theta1) / 2;
            g.ThetaT = g.Theta1 + g.sigma; g.invZ = invZ;
            *out = g;
            found = 1;
        }
    }
    return found;
}

double window(const Geom& g, double Th) {
    if (g.kind == kFull) return 1.0;
    double d = g.kind == kPole ? std::fabs(Th) : std::fabs(Th - M_PI);
    if (d <= g.Theta1) return 1.0;
    if (d >= M_PI) return 0.0;
    double sg = g.sigma;
    if (!(sg > 0)) return d <= g.ThetaT ? 1.0 : 0.0;
    double zlo = std::fmin(std::fmax((d - g.ThetaT) / sg, -1.0), 1.0);
    double zhi = std::fmin(std::fmax((d + g.ThetaT) / sg, -1.0), 1.0);
    double v = (es_cdf(g.beta, std::asin(zhi)) - es_cdf(g.beta, std::asin(zlo))) * g.invZ;
    return std::fmin(std::fmax(v, 0.0), 1.0);
}

double to_theta(const Geom& g, double Th) {
    if (g.kind == kFull) return Th;
    if (g.kind == kPole) {
        double thmax = g.h * (1 + g.eps_apo);
        double t = Th * thmax / M_PI;
        return g.lo <= std::sqrt(DBL_EPSILON) ? t : M_PI - t;
    }
    double lo = g.lo - g.h * g.eps_apo;
    return lo + g.period * Th / (2 * M_PI);
}

double to_stretch(const Geom& g, double th) {
    if (g.kind == kFull) return th;
    if (g.kind == kPole) {
        double thmax = g.h * (1 + g.eps_apo);
        double d = g.lo <= std::sqrt(DBL_EPSILON) ? th : M_PI - th;
        return M_PI * d / thmax;
    }
    double lo = g.lo - g.h * g.eps_apo;
    return 2 * M_PI * (th - lo) / g.period;
}

double jl_mod(double x, double y) {
    double r = std::fmod(x, y);
    if (r == 0.0) return std::copysign(r, y);
    if ((r > 0) != (y > 0)) return r + y;
    return r;
}

int build_leaf(double lo, double hi, int L, int B, double tol, double eps_apo_max,
               double ovs_th, double ovs_ph, Leaf* out, std::string* err, int spin) {
    const double tiny = std::sqrt(DBL_EPSILON);
    Geom g0, g;
    int r = try_geometry(lo, hi, L, tol, eps_apo_max, &g0);
    if (r < 0) { *err = "colatitudes must lie in [0, pi] with theta_lo <= theta_hi"; return 2; }
    if (r == 0) {
        *err = "stretched transform is degenerate for this colatitude extent at this lmax and "
               "tol: every periodisation needs an apodisation wider than the data "
               "(src/Windows.jl:66-75); use the direct method";
        return 1;
    }
    // south periodisation is reflected to the north (src/Stretch.jl:151-158)
    bool flip = g0.kind == kPole && g0.hi >= M_PI - tiny && g0.lo > tiny;
    if (flip) {
        if (try_geometry(M_PI - hi, M_PI - lo, L, tol, eps_apo_max, &g) != 1) {
            *err = "reflected geometry refused";
            return 1;
        }
    } else {
        g = g0;
    }
    Leaf& lf = *out;
    lf.g = g;
    lf.flip = flip;
    lf.lmax = L;
    lf.ntrans = B;
    // grid sizes (src/Stretch.jl:164-171)
    int64_t Kth = (int64_t)std::ceil((double)(g.K + 2) * ovs_th);
    if (g.kind == kInterior) {
        lf.nth = (int)next_smooth(2 * Kth + 1);
        lf.nth_half = lf.nth;
    } else {
        lf.nth_half = (int)next_smooth(Kth + 1);
        lf.nth = 2 * lf.nth_half;
    }
    // rings (src/Windows.jl:307-320)
    const int n = lf.nth_half;
    lf.theta_rings.resize(n);
    lf.Theta_rings.resize(n);
    for (int i = 1; i <= n; ++i) {
        double T = g.kind == kInterior ? 2 * M_PI * (i - 1) / n : M_PI * (i - 0.5) / n;
        lf.Theta_rings[i - 1] = T;
        lf.theta_rings[i - 1] = to_theta(g, T);
    }
    for (int i = 1; i < n; ++i)
        if (lf.theta_rings[i] < lf.theta_rings[i - 1]) {
            *err = "ring colatitudes are not ascending";
            return 2;
        }
    // ring engine tables (src/Legendre.jl:194-255); reflect flips cos(theta)
    const double csgn = flip ? -1.0 : 1.0;
    lf.cos_t.resize(n);
    lf.log2sin.resize(n);
    lf.mlim.resize(n);
    for (int j = 0; j < n; ++j) {
        double s = std::sin(lf.theta_rings[j]), c = std::cos(lf.theta_rings[j]);
        double as = std::fabs(s);
        lf.cos_t[j] = csgn * c;
        lf.log2sin[j] = as > 0 ? std::log2(as) : -INFINITY;
        // spin: never below |s|, where d^l_{m,-s} is not small (src/Spin.jl:222-225)
        lf.mlim[j] = std::max(polar_mmax(lf.theta_rings[j], L, tol), std::abs(spin));
    }
    if (!nested_ranges(lf.mlim, L, lf.jlo, lf.jhi)) {
        *err = "retained-order limits are not unimodal in colatitude";
        return 2;
    }
    sectorial_log2c(L, lf.log2c);
    lf.mmax = *std::max_element(lf.mlim.begin(), lf.mlim.end());
    lf.spin = spin;
    lf.nph = (int)next_smooth_even(
        (int64_t)std::ceil((2.0 * std::max(lf.mmax, std::abs(spin)) + 1) * ovs_ph));
    lf.w.resize(n);
    for (int i = 0; i < n; ++i) lf.w[i] = window(g, lf.Theta_rings[i]);
    int64_t wk = 0;
    if (spin == 0) {
        for (int m = 0; m <= L; ++m) {
            int nj = lf.jhi[m] - lf.jlo[m] + 1;
            if (nj > 0) wk += (int64_t)nj * (L - m + 1);
        }
    } else {
        // the spin walk: every order m = -L..L separately, from l0 = max(|m|, |s|)
        for (int m = -L; m <= L; ++m) {
            const int am = std::abs(m), l0 = std::max(am, std::abs(spin));
            int nj = lf.jhi[am] - lf.jlo[am] + 1;
            if (nj > 0 && l0 <= L) wk += (int64_t)nj * (L - l0 + 1);
        }
    }
    lf.ring_work = wk;
    return 0;
}

int es_width(double tol) {
    int w = (int)std::ceil(-std::log10(tol / 10.0));
    return std::min(16, std::max(2, w));
}

double es_kernel(double z, double beta) {
    if (std::fabs(z) >= 1.0) return 0.0;
    return std::exp(beta * (std::sqrt(1.0 - z * z) - 1.0));
}

// Phi(k) = int phi(2s/w) cos(2 pi k s / nf) ds over [-w/2, w/2], by composite Gauss-Legendre
// after z = sin t (removes the square-root branch point at |z| = 1).
double es_deconv(int k, int nf, int w, double beta) {
    const int npan = 40;
    double hw = (M_PI / 2) / (2 * npan);
    double om = M_PI * (double)k * (double)w / (double)nf;
    double acc = 0.0;
    for (int p = 0; p < npan; ++p) {
        double c = (2 * p + 1) * hw;
        double s = 0.0;
        for (int q = 0; q < 10; ++q) {
            double t = c + hw * kGLX[q];
            s += kGLW[q] * std::exp(beta * (std::cos(t) - 1.0)) * std::cos(om * std::sin(t)) *
                 std::cos(t);
        }
        acc += hw * s;
    }
    return 1.0 / ((double)w * acc);
}

}  // namespace pf
