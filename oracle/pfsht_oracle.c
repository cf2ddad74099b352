/*
 * pfsht_oracle.c -- CPU restatement of PartialFSHT.jl's partial-sky SHT (test infrastructure).
 *
 * This is the parity oracle and the timed CPU baseline, nothing else: the product library
 * never links or calls it. It follows the reference's CPU path step by step, citing
 * path:line in the PartialFSHT.jl tree at each routine. Built with -ffp-contract=off so
 * that, like Julia, no product and sum are fused into one rounding.
 *
 * The reference has no golden vectors (its tests draw from Julia's seeded RNG), so the
 * restatement is pinned by the known-answer and property tests of test/test_legendre.jl,
 * test/test_geometry_windows.jl, test/test_transforms.jl and test/test_backends.jl, re-run
 * in tests/ against this library and against mpmath fixtures in tests/golden/.
 */
#include "pfsht_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define RESCALE_STRIDE 64        /* src/Legendre.jl:16 */
#define CHUNK_HEADROOM_BITS 800  /* src/Legendre.jl:20 */
#define CHUNK_MAX 256            /* src/Legendre.jl:23 */
#define K_MARGIN 2               /* src/Stretch.jl:86 */

typedef struct { double re, im; } cplx;

static inline cplx c_add(cplx a, cplx b) { cplx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cplx c_sub(cplx a, cplx b) { cplx r = {a.re - b.re, a.im - b.im}; return r; }
static inline cplx c_mul(cplx a, cplx b) {
    cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static inline cplx c_scale(cplx a, double s) { cplx r = {a.re * s, a.im * s}; return r; }
static inline cplx c_conj(cplx a) { cplx r = {a.re, -a.im}; return r; }
static inline cplx c_cis(double x) { cplx r = {cos(x), sin(x)}; return r; }

/* Julia's max(): NaN propagates (C's fmax drops it). */
static inline double jl_max(double a, double b) {
    if (isnan(a) || isnan(b)) return NAN;
    return a > b ? a : b;
}
/* Julia's mod(x, y) for floats: result carries the sign of y. */
static inline double jl_mod(double x, double y) {
    double r = fmod(x, y);
    if (r == 0.0) return copysign(r, y);
    if ((r > 0) != (y > 0)) return r + y;
    return r;
}

static int nthreads_ok(int n) {
#ifdef _OPENMP
    return n > 1 ? n : 1;
#else
    (void)n;
    return 1;
#endif
}

/* ------------------------------------------------------------------------------------ */
/* sizes: next_smooth / next_smooth_even (src/Stretch.jl:52-81)                          */
/* ------------------------------------------------------------------------------------ */
int64_t orc_next_smooth(int64_t n) {
    if (n <= 1) return 1;
    int64_t best = INT64_MAX;
    for (int64_t p2 = 1; p2 < 2 * n + 2; p2 *= 2) {
        for (int64_t p3 = p2; p3 < 2 * n + 2; p3 *= 3) {
            for (int64_t p5 = p3; p5 < 2 * n + 2; p5 *= 5) {
                if (p5 >= n && p5 < best) best = p5;
            }
        }
    }
    return best == INT64_MAX ? n : best;
}

int64_t orc_next_smooth_even(int64_t n) {
    /* 2 * next_smooth(cld(n, 2)) */
    int64_t h = n > 0 ? (n + 1) / 2 : -((-n) / 2);
    return 2 * orc_next_smooth(h);
}

/* ------------------------------------------------------------------------------------ */
/* Legendre tables (src/Legendre.jl:31-145)                                              */
/* ------------------------------------------------------------------------------------ */
double orc_polar_pad_factor(void) { return 0.5 * cbrt(9.0); }

/* polar_mmax (src/Legendre.jl:48-57) */
int orc_polar_mmax(double theta, int lmax, double eps) {
    int L = lmax;
    if (L <= 0) return 0;
    double s = fabs(sin(theta));
    double z = ((double)L + 0.5) * s;
    double le = fabs(log(fmax(eps, DBL_MIN)));
    double pad = orc_polar_pad_factor() * cbrt(fmax(z, 1.0)) * cbrt(le * le) + 2.0;
    double c = ceil(z + pad);
    if (c < 0) return 0;
    if (c > L) return L;
    return (int)c;
}

/* sectorial_log2c (src/Legendre.jl:65-75) */
void orc_sectorial_log2c(int lmax, double* v) {
    double acc = -log2(sqrt(4.0 * M_PI));
    v[0] = acc;
    for (int m = 1; m <= lmax; ++m) {
        acc += log2(sqrt((double)(2 * m + 1) / (double)(2 * m)));
        v[m] = acc;
    }
}

/* _nested_ranges (src/Legendre.jl:89-127), 0-based and non-symmetric */
int orc_nested_ranges(const int* mlim, int n, int lmax, int* jlo, int* jhi) {
    if (n < 1) return -1;
    int peak = 0;
    for (int j = 1; j < n; ++j)
        if (mlim[j] > mlim[peak]) peak = j;
    for (int j = 1; j <= peak; ++j)
        if (mlim[j] < mlim[j - 1]) return -1;
    for (int j = peak + 1; j < n; ++j)
        if (mlim[j] > mlim[j - 1]) return -1;
    for (int m = 0; m <= lmax; ++m) { jlo[m] = 0; jhi[m] = -1; }
    int lo = peak, hi = peak;
    int mtop = mlim[peak] < lmax ? mlim[peak] : lmax;
    for (int m = mtop; m >= 0; --m) {
        while (lo > 0 && mlim[lo - 1] >= m) --lo;
        while (hi < n - 1 && mlim[hi + 1] >= m) ++hi;
        jlo[m] = lo;
        jhi[m] = hi;
    }
    return 0;
}

/* retained_triples (src/Legendre.jl:136-145) */
int64_t orc_retained_triples(const int* mlim, int n, int lmax) {
    int* jlo = (int*)malloc(sizeof(int) * (lmax + 1));
    int* jhi = (int*)malloc(sizeof(int) * (lmax + 1));
    int64_t w = 0;
    if (orc_nested_ranges(mlim, n, lmax, jlo, jhi) == 0) {
        for (int m = 0; m <= lmax; ++m) {
            int nj = jhi[m] - jlo[m] + 1;
            if (nj > 0) w += (int64_t)nj * (lmax - m + 1);
        }
    } else {
        w = -1;
    }
    free(jlo);
    free(jhi);
    return w;
}

/* alf (src/Legendre.jl:555-596) */
double orc_alf(int l, int m, double theta) {
    int am = abs(m);
    if (am > l) return 0.0;
    double s = fabs(sin(theta)), x = cos(theta);
    double log2c = -log2(sqrt(4.0 * M_PI));
    for (int k = 1; k <= am; ++k) log2c += log2(sqrt((double)(2 * k + 1) / (double)(2 * k)));
    double e0 = am == 0 ? log2c : (double)am * (s > 0 ? log2(s) : -INFINITY) + log2c;
    if (!isfinite(e0)) return 0.0;
    double E = ceil(e0);
    double p2 = ((am % 2 == 0) ? 1.0 : -1.0) * exp2(e0 - E);
    double flip = (m < 0 && (am % 2 == 1)) ? -1.0 : 1.0;
    if (l == am) return flip * (p2 * exp2(E));
    double p1 = sqrt((double)(2 * am + 3)) * x * p2;
    int steps = 0;
    for (int el = am + 2; el <= l; ++el) {
        double a = sqrt((double)(2 * el - 1) * (double)(2 * el + 1) /
                        ((double)(el - am) * (double)(el + am)));
        double b = sqrt((double)(2 * el + 1) / (double)(2 * el - 3) * (double)(el - am - 1) /
                        (double)(el - am) * (double)(el + am - 1) / (double)(el + am));
        double p = a * x * p1 - b * p2;
        p2 = p1;
        p1 = p;
        if (++steps == RESCALE_STRIDE) {
            steps = 0;
            double mx = fmax(fabs(p1), fabs(p2));
            if (mx > 0 && isfinite(mx)) {
                double sh = ceil(log2(mx));
                if (sh != 0) {
                    double f = exp2(-sh);
                    p1 *= f;
                    p2 *= f;
                    E += sh;
                }
            }
        }
    }
    return flip * (p1 * exp2(E));
}

/* ------------------------------------------------------------------------------------ */
/* RingLegendre (src/Legendre.jl:174-283) and the ring walk (src/Legendre.jl:310-542)    */
/* ------------------------------------------------------------------------------------ */
struct orc_rings {
    int n, L, B, mmax, reflect;
    double eps;
    double *theta, *cos_t, *sin_t, *log2sin, *log2c;
    int *mlim, *jlo, *jhi;
    int nchunks;
    int *clo, *chi;
};

/* _ring_chunks (src/Legendre.jl:262-283) */
static int ring_chunks(const double* sinth, const int* mlim, int n, int* clo, int* chi) {
    int i = 0, nc = 0;
    while (i < n) {
        int stop = i;
        int mm = mlim[i];
        while (stop < n - 1) {
            int nxt = stop + 1;
            if (nxt - i + 1 > CHUNK_MAX) break;
            double slo = sinth[i], shi = sinth[nxt];
            double span = (slo > 0 && shi > 0) ? fabs(log2(shi / slo)) : INFINITY;
            int m2 = mm > mlim[nxt] ? mm : mlim[nxt];
            if ((double)m2 * span > CHUNK_HEADROOM_BITS) break; /* 0*Inf = NaN: not > */
            mm = m2;
            stop = nxt;
        }
        clo[nc] = i;
        chi[nc] = stop;
        ++nc;
        i = stop + 1;
    }
    return nc;
}

orc_rings* orc_rings_create(const double* theta, int n, int lmax, double eps, int ntrans,
                            int reflect) {
    if (lmax < 0 || ntrans < 1 || n < 1) return NULL;
    for (int j = 1; j < n; ++j)
        if (theta[j] < theta[j - 1]) return NULL;
    orc_rings* e = (orc_rings*)calloc(1, sizeof(orc_rings));
    e->n = n;
    e->L = lmax;
    e->B = ntrans;
    e->eps = eps;
    e->reflect = reflect;
    e->theta = (double*)malloc(sizeof(double) * n);
    e->cos_t = (double*)malloc(sizeof(double) * n);
    e->sin_t = (double*)malloc(sizeof(double) * n);
    e->log2sin = (double*)malloc(sizeof(double) * n);
    e->log2c = (double*)malloc(sizeof(double) * (lmax + 1));
    e->mlim = (int*)malloc(sizeof(int) * n);
    e->jlo = (int*)malloc(sizeof(int) * (lmax + 1));
    e->jhi = (int*)malloc(sizeof(int) * (lmax + 1));
    e->clo = (int*)malloc(sizeof(int) * n);
    e->chi = (int*)malloc(sizeof(int) * n);
    double csgn = reflect ? -1.0 : 1.0;
    for (int j = 0; j < n; ++j) {
        double s = sin(theta[j]), c = cos(theta[j]);
        double as = fabs(s);
        e->theta[j] = theta[j];
        e->sin_t[j] = as;
        e->cos_t[j] = csgn * c;
        e->log2sin[j] = as > 0 ? log2(as) : -INFINITY;
        e->mlim[j] = orc_polar_mmax(theta[j], lmax, eps);
    }
    if (orc_nested_ranges(e->mlim, n, lmax, e->jlo, e->jhi) != 0) {
        orc_rings_destroy(e);
        return NULL;
    }
    orc_sectorial_log2c(lmax, e->log2c);
    e->nchunks = ring_chunks(e->sin_t, e->mlim, n, e->clo, e->chi);
    int mx = 0;
    for (int j = 0; j < n; ++j) mx = e->mlim[j] > mx ? e->mlim[j] : mx;
    e->mmax = mx;
    return e;
}

void orc_rings_destroy(orc_rings* e) {
    if (!e) return;
    free(e->theta); free(e->cos_t); free(e->sin_t); free(e->log2sin); free(e->log2c);
    free(e->mlim); free(e->jlo); free(e->jhi); free(e->clo); free(e->chi);
    free(e);
}

int orc_rings_n(const orc_rings* e) { return e->n; }
int orc_rings_mmax(const orc_rings* e) { return e->mmax; }
int orc_rings_nchunks(const orc_rings* e) { return e->nchunks; }

/* ring_work (src/Legendre.jl:286-293) */
int64_t orc_rings_work(const orc_rings* e) {
    int64_t w = 0;
    for (int m = 0; m <= e->L; ++m) {
        int nj = e->jhi[m] - e->jlo[m] + 1;
        if (nj > 0) w += (int64_t)nj * (e->L - m + 1);
    }
    return w;
}

void orc_rings_tables(const orc_rings* e, int* mlim, int* jlo, int* jhi, int* clo, int* chi,
                      double* cos_t, double* log2sin, double* log2c) {
    if (mlim) memcpy(mlim, e->mlim, sizeof(int) * e->n);
    if (jlo) memcpy(jlo, e->jlo, sizeof(int) * (e->L + 1));
    if (jhi) memcpy(jhi, e->jhi, sizeof(int) * (e->L + 1));
    if (clo) memcpy(clo, e->clo, sizeof(int) * e->nchunks);
    if (chi) memcpy(chi, e->chi, sizeof(int) * e->nchunks);
    if (cos_t) memcpy(cos_t, e->cos_t, sizeof(double) * e->n);
    if (log2sin) memcpy(log2sin, e->log2sin, sizeof(double) * e->n);
    if (log2c) memcpy(log2c, e->log2c, sizeof(double) * (e->L + 1));
}

/* sph_mode packing: 0-based linear index of (l, m, b) */
static inline int64_t alm_idx(int L, int l, int m, int b) {
    int am = abs(m);
    int col = m >= 0 ? 2 * am : 2 * am - 1;
    return (int64_t)(l - am) + (int64_t)(L + 1) * col + (int64_t)(L + 1) * (2 * L + 1) * b;
}

typedef struct {
    double *p1, *p2;
    cplx *accp, *accm; /* nr x B, ring index fastest */
} scratch;

static scratch scratch_new(int nr, int B) {
    scratch s;
    s.p1 = (double*)malloc(sizeof(double) * nr);
    s.p2 = (double*)malloc(sizeof(double) * nr);
    s.accp = (cplx*)malloc(sizeof(cplx) * nr * B);
    s.accm = (cplx*)malloc(sizeof(cplx) * nr * B);
    return s;
}
static void scratch_free(scratch* s) { free(s->p1); free(s->p2); free(s->accp); free(s->accm); }

/* _seed_exponent (src/Legendre.jl:475-481) */
static double seed_exponent(const orc_rings* e, int m, int r0, int r1) {
    double ex = -INFINITY;
    for (int j = r0; j <= r1; ++j) ex = jl_max(ex, (double)m * e->log2sin[j] + e->log2c[m]);
    return isfinite(ex) ? ceil(ex) : 0.0;
}

/* _renorm! (src/Legendre.jl:521-542) */
static double renorm(int fwd, scratch* sc, int nr, int B) {
    double mx = 0.0;
    for (int k = 0; k < nr; ++k) mx = jl_max(mx, jl_max(fabs(sc->p1[k]), fabs(sc->p2[k])));
    if (mx == 0 || !isfinite(mx)) return 0.0;
    double s = ceil(log2(mx));
    if (s == 0) return 0.0;
    double f = exp2(-s);
    for (int k = 0; k < nr; ++k) { sc->p1[k] *= f; sc->p2[k] *= f; }
    if (fwd) {
        for (int b = 0; b < B; ++b)
            for (int k = 0; k < nr; ++k) {
                sc->accp[k + nr * b] = c_scale(sc->accp[k + nr * b], f);
                sc->accm[k + nr * b] = c_scale(sc->accm[k + nr * b], f);
            }
    }
    return s;
}

static inline cplx get_c(const double* a, int64_t i) { cplx r = {a[2 * i], a[2 * i + 1]}; return r; }
static inline void add_c(double* a, int64_t i, cplx v) { a[2 * i] += v.re; a[2 * i + 1] += v.im; }

/* _touch!(::_Fwd) (src/Legendre.jl:484-496) */
static void touch_fwd(const orc_rings* e, const double* alm, scratch* sc, const double* P,
                      int l, int m, double sgn, int nr) {
    for (int b = 0; b < e->B; ++b) {
        cplx ap = get_c(alm, alm_idx(e->L, l, m, b));
        cplx am = {0.0, 0.0};
        if (m != 0) am = get_c(alm, alm_idx(e->L, l, -m, b));
        if (ap.re == 0 && ap.im == 0 && am.re == 0 && am.im == 0) continue;
        cplx ams = c_scale(am, sgn);
        cplx* accp = sc->accp + nr * b;
        cplx* accm = sc->accm + nr * b;
        for (int k = 0; k < nr; ++k) {
            accp[k] = c_add(accp[k], c_scale(ap, P[k]));
            accm[k] = c_add(accm[k], c_scale(ams, P[k]));
        }
    }
}

/* _touch!(::_Adj) (src/Legendre.jl:501-514) */
static void touch_adj(const orc_rings* e, double* alm, const scratch* sc, const double* P,
                      int l, int m, double sgn, int nr, double E) {
    double f = exp2(E);
    for (int b = 0; b < e->B; ++b) {
        cplx sp = {0, 0}, sm = {0, 0};
        const cplx* accp = sc->accp + nr * b;
        const cplx* accm = sc->accm + nr * b;
        for (int k = 0; k < nr; ++k) {
            sp = c_add(sp, c_scale(accp[k], P[k]));
            sm = c_add(sm, c_scale(accm[k], P[k]));
        }
        add_c(alm, alm_idx(e->L, l, m, b), c_scale(sp, f));
        if (m > 0) add_c(alm, alm_idx(e->L, l, -m, b), c_scale(c_scale(sm, sgn), f));
    }
}

/* _ring_chunk! (src/Legendre.jl:367-472) */
static void ring_chunk(int fwd, const orc_rings* e, double* G, const double* almin,
                       double* almout, int m, int r0, int r1, scratch* sc) {
    const int L = e->L, B = e->B, off = L, n = e->n;
    const int nr = r1 - r0 + 1;
    const double sgn = (m % 2 == 0) ? 1.0 : -1.0;
    double E = seed_exponent(e, m, r0, r1);
    for (int k = 0; k < nr; ++k) {
        int j = r0 + k;
        sc->p2[k] = sgn * exp2((double)m * e->log2sin[j] + e->log2c[m] - E);
    }
    if (fwd) {
        memset(sc->accp, 0, sizeof(cplx) * nr * B);
        memset(sc->accm, 0, sizeof(cplx) * nr * B);
    } else {
        for (int b = 0; b < B; ++b)
            for (int k = 0; k < nr; ++k) {
                int j = r0 + k;
                sc->accp[k + nr * b] = get_c(G, j + (int64_t)n * (m + off) + (int64_t)n * (2 * L + 1) * b);
                cplx z = {0, 0};
                sc->accm[k + nr * b] =
                    m == 0 ? z : get_c(G, j + (int64_t)n * (-m + off) + (int64_t)n * (2 * L + 1) * b);
            }
    }
    if (fwd) touch_fwd(e, almin, sc, sc->p2, m, m, sgn, nr);
    else touch_adj(e, almout, sc, sc->p2, m, m, sgn, nr, E);

    if (m < L) {
        for (int k = 0; k < nr; ++k) sc->p1[k] = sqrt((double)(2 * m + 3)) * e->cos_t[r0 + k] * sc->p2[k];
        if (fwd) touch_fwd(e, almin, sc, sc->p1, m + 1, m, sgn, nr);
        else touch_adj(e, almout, sc, sc->p1, m + 1, m, sgn, nr, E);
        const double* cs = e->cos_t + r0;
        int steps = 0;
        for (int l = m + 2; l <= L; ++l) {
            double a = sqrt((double)(2 * l - 1) * (double)(2 * l + 1) /
                            ((double)(l - m) * (double)(l + m)));
            double b = sqrt((double)(2 * l + 1) / (double)(2 * l - 3) * (double)(l - m - 1) /
                            (double)(l - m) * (double)(l + m - 1) / (double)(l + m));
            if (fwd && B == 1) {
                cplx ap = get_c(almin, alm_idx(L, l, m, 0));
                cplx z = {0, 0};
                cplx ams = c_scale(m == 0 ? z : get_c(almin, alm_idx(L, l, -m, 0)), sgn);
                for (int k = 0; k < nr; ++k) {
                    double p = a * cs[k] * sc->p1[k] - b * sc->p2[k];
                    sc->p2[k] = sc->p1[k];
                    sc->p1[k] = p;
                    sc->accp[k] = c_add(sc->accp[k], c_scale(ap, p));
                    sc->accm[k] = c_add(sc->accm[k], c_scale(ams, p));
                }
            } else if (!fwd && B == 1) {
                double f = exp2(E);
                cplx sp = {0, 0}, sm = {0, 0};
                for (int k = 0; k < nr; ++k) {
                    double p = a * cs[k] * sc->p1[k] - b * sc->p2[k];
                    sc->p2[k] = sc->p1[k];
                    sc->p1[k] = p;
                    sp = c_add(sp, c_scale(sc->accp[k], p));
                    sm = c_add(sm, c_scale(sc->accm[k], p));
                }
                add_c(almout, alm_idx(L, l, m, 0), c_scale(sp, f));
                if (m > 0) add_c(almout, alm_idx(L, l, -m, 0), c_scale(c_scale(sm, sgn), f));
            } else {
                for (int k = 0; k < nr; ++k) {
                    double p = a * cs[k] * sc->p1[k] - b * sc->p2[k];
                    sc->p2[k] = sc->p1[k];
                    sc->p1[k] = p;
                }
                if (fwd) touch_fwd(e, almin, sc, sc->p1, l, m, sgn, nr);
                else touch_adj(e, almout, sc, sc->p1, l, m, sgn, nr, E);
            }
            ++steps;
            if (steps == RESCALE_STRIDE && l < L) {
                steps = 0;
                E += renorm(fwd, sc, nr, B);
            }
        }
    }
    if (fwd) {
        double f = exp2(E);
        for (int b = 0; b < B; ++b)
            for (int k = 0; k < nr; ++k) {
                int j = r0 + k;
                add_c(G, j + (int64_t)n * (m + off) + (int64_t)n * (2 * L + 1) * b,
                      c_scale(sc->accp[k + nr * b], f));
                if (m > 0)
                    add_c(G, j + (int64_t)n * (-m + off) + (int64_t)n * (2 * L + 1) * b,
                          c_scale(sc->accm[k + nr * b], f));
            }
    }
}

/* _walk_orders! (src/Legendre.jl:354-365) over m = t, t+ns, ... */
static void walk_orders(int fwd, const orc_rings* e, double* G, const double* almin,
                        double* almout, int t, int ns, scratch* sc) {
    for (int m = t; m <= e->L; m += ns) {
        int lo = e->jlo[m], hi = e->jhi[m];
        if (hi < lo) continue;
        for (int c = 0; c < e->nchunks; ++c) {
            int r0 = e->clo[c] > lo ? e->clo[c] : lo;
            int r1 = e->chi[c] < hi ? e->chi[c] : hi;
            if (r1 < r0) continue;
            ring_chunk(fwd, e, G, almin, almout, m, r0, r1, sc);
        }
    }
}

static int max_chunk_len(const orc_rings* e) {
    int cw = 1;
    for (int c = 0; c < e->nchunks; ++c) {
        int l = e->chi[c] - e->clo[c] + 1;
        cw = l > cw ? l : cw;
    }
    return cw;
}

static void walk(int fwd, const orc_rings* e, double* G, const double* almin, double* almout,
                 int nthreads) {
    int ns = nthreads_ok(nthreads);
    if (ns > e->L + 1) ns = e->L + 1;
    int cw = max_chunk_len(e);
    if (ns <= 1) {
        scratch sc = scratch_new(cw, e->B);
        walk_orders(fwd, e, G, almin, almout, 0, 1, &sc);
        scratch_free(&sc);
        return;
    }
#ifdef _OPENMP
#pragma omp parallel num_threads(ns)
    {
        int t = omp_get_thread_num();
        scratch sc = scratch_new(cw, e->B);
        walk_orders(fwd, e, G, almin, almout, t, ns, &sc);
        scratch_free(&sc);
    }
#endif
}

/* rings_from_alm! (src/Legendre.jl:310-323) */
void orc_rings_from_alm(const orc_rings* e, const double* alm, double* G, int nthreads) {
    memset(G, 0, sizeof(double) * 2 * (size_t)e->n * (2 * e->L + 1) * e->B);
    walk(1, e, G, alm, NULL, nthreads);
}

/* alm_from_rings! (src/Legendre.jl:332-341) */
void orc_alm_from_rings(const orc_rings* e, const double* G, double* alm, int nthreads) {
    memset(alm, 0, sizeof(double) * 2 * (size_t)(e->L + 1) * (2 * e->L + 1) * e->B);
    walk(0, e, (double*)G, NULL, alm, nthreads);
}

/* ------------------------------------------------------------------------------------ */
/* geometry and window (src/Windows.jl)                                                  */
/* ------------------------------------------------------------------------------------ */
static const double GL10_X[10] = {-0.9739065285171717, -0.8650633666889845, -0.6794095682990244,
                                  -0.4333953941292472, -0.1488743389816312, 0.1488743389816312,
                                  0.4333953941292472,  0.6794095682990244,  0.8650633666889845,
                                  0.9739065285171717};
static const double GL10_W[10] = {0.0666713443086881, 0.1494513491505806, 0.2190863625159820,
                                  0.2692667193099963, 0.2955242247147529, 0.2955242247147529,
                                  0.2692667193099963, 0.2190863625159820, 0.1494513491505806,
                                  0.0666713443086881};
#define ES_PANEL 0.05 /* src/Windows.jl:197 */

double orc_es_beta(double eps) { return fabs(log(eps)); }

/* es_cdf (src/Windows.jl:208-226) */
double orc_es_cdf(double beta, double u) {
    double a = -M_PI / 2;
    if (u <= a) return 0.0;
    double b = fmin(u, M_PI / 2);
    int n = (int)ceil((b - a) / ES_PANEL);
    if (n < 1) n = 1;
    double hw = (b - a) / (2 * n);
    double acc = 0.0;
    for (int p = 0; p < n; ++p) {
        double c = a + (2 * p + 1) * hw;
        double s = 0.0;
        for (int q = 0; q < 10; ++q) {
            double t = c + hw * GL10_X[q];
            double ct = cos(t);
            s += GL10_W[q] * exp(beta * (ct - 1)) * ct;
        }
        acc += hw * s;
    }
    return acc;
}

/* try_stretch_geometry (src/Windows.jl:84-141) */
int orc_try_stretch_geometry(double lo, double hi, int L, double eps, double eps_apo_max,
                             orc_geom* out) {
    if (!(lo <= hi)) return -1;
    if (!(lo >= 0 && hi <= M_PI)) return -1;
    double beta = orc_es_beta(eps);
    double tiny = sqrt(DBL_EPSILON);
    double Z = orc_es_cdf(beta, M_PI / 2);
    double invZ = Z > 0 ? 1.0 / Z : 0.0;
    if (lo <= tiny && hi >= M_PI - tiny) {
        orc_geom g = {ORC_FULL, L, eps, beta, M_PI / 2, 0.0, M_PI, 0.0, 2 * M_PI, L,
                      M_PI, 0.0, M_PI, 1.0};
        *out = g;
        return 1;
    }
    struct { int kind; double h, klo, khi; } cands[3] = {
        {ORC_POLE, hi, 0.0, hi}, {ORC_POLE, M_PI - lo, lo, M_PI}, {ORC_INTERIOR, (hi - lo) / 2, lo, hi}};
    int64_t bestK = INT64_MAX;
    int found = 0;
    for (int c = 0; c < 3; ++c) {
        double h = cands[c].h;
        if (!(h > 0)) continue;
        double Lh = (double)L * h;
        if (!(Lh >= 2 * beta / (eps_apo_max * eps_apo_max))) continue;
        double ea = sqrt(2 * beta / Lh);
        double pad = h * ea;
        if (cands[c].kind == ORC_INTERIOR) {
            if (!(cands[c].klo - pad >= 0 && cands[c].khi + pad <= M_PI)) continue;
        } else {
            if (!(h * (1 + ea) <= M_PI)) continue;
        }
        double Kf = ceil(Lh * ((1 + ea) * (1 + ea)) / M_PI);
        int64_t K = (int64_t)Kf;
        if (K < 1) K = 1;
        if (K < bestK) {
            bestK = K;
            double T1 = M_PI / (1 + ea);
            double sg = (M_PI - T1) / 2;
            orc_geom g = {cands[c].kind, L, eps, beta, h, cands[c].klo, cands[c].khi, ea,
                          2 * h * (1 + ea), K, T1, sg, T1 + sg, invZ};
            *out = g;
            found = 1;
        }
    }
    return found;
}

/* stretch_window (src/Windows.jl:237-250) */
double orc_stretch_window(const orc_geom* g, double Th) {
    if (g->kind == ORC_FULL) return 1.0;
    double d = g->kind == ORC_POLE ? fabs(Th) : fabs(Th - M_PI);
    if (d <= g->Theta1) return 1.0;
    if (d >= M_PI) return 0.0;
    double sg = g->sigma;
    if (!(sg > 0)) return d <= g->ThetaT ? 1.0 : 0.0;
    double zlo = fmin(fmax((d - g->ThetaT) / sg, -1.0), 1.0);
    double zhi = fmin(fmax((d + g->ThetaT) / sg, -1.0), 1.0);
    double v = (orc_es_cdf(g->beta, asin(zhi)) - orc_es_cdf(g->beta, asin(zlo))) * g->invZ;
    return fmin(fmax(v, 0.0), 1.0);
}

/* stretch_to_theta / theta_to_stretch (src/Windows.jl:272-298) */
double orc_stretch_to_theta(const orc_geom* g, double Th) {
    if (g->kind == ORC_FULL) return Th;
    if (g->kind == ORC_POLE) {
        double thmax = g->h * (1 + g->eps_apo);
        double t = Th * thmax / M_PI;
        return g->theta_lo <= sqrt(DBL_EPSILON) ? t : M_PI - t;
    }
    double lo = g->theta_lo - g->h * g->eps_apo;
    return lo + g->period * Th / (2 * M_PI);
}

double orc_theta_to_stretch(const orc_geom* g, double th) {
    if (g->kind == ORC_FULL) return th;
    if (g->kind == ORC_POLE) {
        double thmax = g->h * (1 + g->eps_apo);
        double d = g->theta_lo <= sqrt(DBL_EPSILON) ? th : M_PI - th;
        return M_PI * d / thmax;
    }
    double lo = g->theta_lo - g->h * g->eps_apo;
    return 2 * M_PI * (th - lo) / g->period;
}

/* stretch_rings (src/Windows.jl:307-320) */
void orc_stretch_rings(const orc_geom* g, int n, double* th, double* Th) {
    for (int i = 1; i <= n; ++i) {
        double T;
        if (g->kind == ORC_INTERIOR) T = 2 * M_PI * (i - 1) / n;
        else T = M_PI * (i - 0.5) / n;
        Th[i - 1] = T;
        th[i - 1] = orc_stretch_to_theta(g, T);
    }
}

/* ------------------------------------------------------------------------------------ */
/* DFS periodisation (src/DFS.jl:13-56)                                                  */
/* ------------------------------------------------------------------------------------ */
void orc_dfs_double(const double* F, double* Ft, int Nth, int Nph, int B, int spin) {
    int half = Nph / 2;
    double sgn = (spin % 2 == 0) ? 1.0 : -1.0;
    const cplx* f = (const cplx*)F;
    cplx* ft = (cplx*)Ft;
    for (int b = 0; b < B; ++b) {
        for (int j = 0; j < Nph; ++j)
            for (int i = 0; i < Nth; ++i)
                ft[i + (int64_t)2 * Nth * j + (int64_t)2 * Nth * Nph * b] =
                    f[i + (int64_t)Nth * j + (int64_t)Nth * Nph * b];
        for (int j = 0; j < Nph; ++j) {
            int js = (j + half) % Nph;
            for (int i = 0; i < Nth; ++i)
                ft[Nth + i + (int64_t)2 * Nth * j + (int64_t)2 * Nth * Nph * b] =
                    c_scale(f[(Nth - 1 - i) + (int64_t)Nth * js + (int64_t)Nth * Nph * b], sgn);
        }
    }
}

void orc_dfs_fold(double* F, const double* Ft, int Nth, int Nph, int B, int spin) {
    int half = Nph / 2;
    double sgn = (spin % 2 == 0) ? 1.0 : -1.0;
    cplx* f = (cplx*)F;
    const cplx* ft = (const cplx*)Ft;
    for (int b = 0; b < B; ++b)
        for (int j = 0; j < Nph; ++j) {
            int js = ((j - half) % Nph + Nph) % Nph;
            for (int i = 0; i < Nth; ++i)
                f[i + (int64_t)Nth * j + (int64_t)Nth * Nph * b] =
                    c_add(ft[i + (int64_t)2 * Nth * j + (int64_t)2 * Nth * Nph * b],
                          c_scale(ft[(2 * Nth - 1 - i) + (int64_t)2 * Nth * js +
                                     (int64_t)2 * Nth * Nph * b], sgn));
        }
}

/* ------------------------------------------------------------------------------------ */
/* mixed-radix FFT (FFTW's role at src/Stretch.jl:222-225; own code, radix 4/2/generic)  */
/* ------------------------------------------------------------------------------------ */
typedef struct {
    int n, nf;
    int fac[64]; /* (p, m) pairs */
    cplx* tw;    /* e^{-2 pi i j / n} */
} fftplan;

static fftplan* fftplan_new(int n) {
    fftplan* P = (fftplan*)calloc(1, sizeof(fftplan));
    P->n = n;
    P->tw = (cplx*)malloc(sizeof(cplx) * (n > 0 ? n : 1));
    for (int j = 0; j < n; ++j) {
        double ang = -2.0 * M_PI * (double)j / (double)n;
        P->tw[j].re = cos(ang);
        P->tw[j].im = sin(ang);
    }
    int m = n, k = 0;
    while (m > 1) {
        int p;
        if (m % 4 == 0) p = 4;
        else if (m % 2 == 0) p = 2;
        else if (m % 3 == 0) p = 3;
        else if (m % 5 == 0) p = 5;
        else {
            p = 7;
            while (m % p) p += 2;
        }
        m /= p;
        P->fac[k++] = p;
        P->fac[k++] = m;
    }
    P->nf = k / 2;
    return P;
}
static void fftplan_free(fftplan* P) { if (P) { free(P->tw); free(P); } }

static inline cplx twid(const fftplan* P, int64_t idx, int sign) {
    cplx w = P->tw[idx % P->n];
    if (sign > 0) w.im = -w.im;
    return w;
}

static void fft_work(const fftplan* P, cplx* out, const cplx* in, int fstride, int istride,
                     const int* fac, int sign, cplx* tmp) {
    int p = fac[0], m = fac[1];
    if (m == 1) {
        for (int q = 0; q < p; ++q) out[q] = in[(int64_t)q * fstride * istride];
    } else {
        for (int q = 0; q < p; ++q)
            fft_work(P, out + (int64_t)q * m, in + (int64_t)q * fstride * istride, fstride * p,
                     istride, fac + 2, sign, tmp);
    }
    /* butterflies: X[k + q2 m] = sum_q W_n^{q k fstride} Y_q[k] W_p^{q q2} */
    if (p == 2) {
        for (int k = 0; k < m; ++k) {
            cplx t1 = c_mul(out[k + m], twid(P, (int64_t)k * fstride, sign));
            cplx t0 = out[k];
            out[k] = c_add(t0, t1);
            out[k + m] = c_sub(t0, t1);
        }
    } else if (p == 4) {
        for (int k = 0; k < m; ++k) {
            cplx a0 = out[k];
            cplx a1 = c_mul(out[k + m], twid(P, (int64_t)k * fstride, sign));
            cplx a2 = c_mul(out[k + 2 * m], twid(P, (int64_t)2 * k * fstride, sign));
            cplx a3 = c_mul(out[k + 3 * m], twid(P, (int64_t)3 * k * fstride, sign));
            cplx s02 = c_add(a0, a2), d02 = c_sub(a0, a2);
            cplx s13 = c_add(a1, a3), d13 = c_sub(a1, a3);
            /* multiply d13 by -i (sign -1) or +i (sign +1) */
            cplx rd13 = sign < 0 ? (cplx){d13.im, -d13.re} : (cplx){-d13.im, d13.re};
            out[k] = c_add(s02, s13);
            out[k + m] = c_add(d02, rd13);
            out[k + 2 * m] = c_sub(s02, s13);
            out[k + 3 * m] = c_sub(d02, rd13);
        }
    } else {
        for (int k = 0; k < m; ++k) {
            for (int q = 0; q < p; ++q)
                tmp[q] = c_mul(out[k + (int64_t)q * m], twid(P, (int64_t)q * k * fstride, sign));
            for (int q2 = 0; q2 < p; ++q2) {
                cplx acc = tmp[0];
                for (int q = 1; q < p; ++q)
                    acc = c_add(acc, c_mul(tmp[q], twid(P, (int64_t)((q * q2) % p) * fstride * m, sign)));
                out[k + (int64_t)q2 * m] = acc;
            }
        }
    }
}

/* in-place transform of x[0], x[stride], ... (stride in complex elements) */
static void fft_1d(const fftplan* P, cplx* x, int stride, int sign, cplx* buf, cplx* tmp) {
    int n = P->n;
    if (n <= 1) return;
    fft_work(P, buf, x, 1, stride, P->fac, sign, tmp);
    for (int j = 0; j < n; ++j) x[(int64_t)j * stride] = buf[j];
}

void orc_fft_cols(double* a, int n1, int n2, int sign, int nthreads) {
    fftplan* P = fftplan_new(n1);
    int nt = nthreads_ok(nthreads);
#ifdef _OPENMP
#pragma omp parallel num_threads(nt)
#endif
    {
        cplx* buf = (cplx*)malloc(sizeof(cplx) * n1);
        cplx* tmp = (cplx*)malloc(sizeof(cplx) * 64);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int j = 0; j < n2; ++j) fft_1d(P, (cplx*)a + (int64_t)n1 * j, 1, sign, buf, tmp);
        free(buf);
        free(tmp);
    }
    (void)nt;
    fftplan_free(P);
}

void orc_fft_rows(double* a, int n1, int n2, int sign, int nthreads) {
    fftplan* P = fftplan_new(n2);
    int nt = nthreads_ok(nthreads);
#ifdef _OPENMP
#pragma omp parallel num_threads(nt)
#endif
    {
        cplx* row = (cplx*)malloc(sizeof(cplx) * n2);
        cplx* buf = (cplx*)malloc(sizeof(cplx) * n2);
        cplx* tmp = (cplx*)malloc(sizeof(cplx) * 64);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int i = 0; i < n1; ++i) {
            for (int j = 0; j < n2; ++j) row[j] = ((cplx*)a)[i + (int64_t)n1 * j];
            fft_1d(P, row, 1, sign, buf, tmp);
            for (int j = 0; j < n2; ++j) ((cplx*)a)[i + (int64_t)n1 * j] = row[j];
        }
        free(row);
        free(buf);
        free(tmp);
    }
    (void)nt;
    fftplan_free(P);
}

/* ------------------------------------------------------------------------------------ */
/* NUFFT: mode order and DirectSum (src/NUFFT.jl:85-129)                                */
/* ------------------------------------------------------------------------------------ */
int orc_mode_k(int i0, int n, int modeord) {
    if (modeord == 0) return i0 - n / 2;
    int k = i0;
    return k < (n + 1) / 2 ? k : k - n;
}

void orc_nufft_direct(int type, int n1, int n2, int iflag, int ntrans, const double* x,
                      const double* y, int64_t M, const double* in, double* out) {
    double s = (double)iflag;
    const cplx* ci = (const cplx*)in;
    cplx* co = (cplx*)out;
    if (type == 2) {
        memset(out, 0, sizeof(cplx) * (size_t)M * ntrans);
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static)
#endif
        for (int b = 0; b < ntrans; ++b)
            for (int64_t j = 0; j < M; ++j) {
                cplx acc = {0, 0};
                for (int i2 = 0; i2 < n2; ++i2) {
                    int k2 = orc_mode_k(i2, n2, 1);
                    for (int i1 = 0; i1 < n1; ++i1) {
                        int k1 = orc_mode_k(i1, n1, 1);
                        cplx c = ci[i1 + (int64_t)n1 * i2 + (int64_t)n1 * n2 * b];
                        acc = c_add(acc, c_mul(c, c_cis(s * ((double)k1 * x[j] + (double)k2 * y[j]))));
                    }
                }
                co[j + M * b] = acc;
            }
    } else {
        memset(out, 0, sizeof(cplx) * (size_t)n1 * n2 * ntrans);
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static)
#endif
        for (int b = 0; b < ntrans; ++b)
            for (int i2 = 0; i2 < n2; ++i2) {
                int k2 = orc_mode_k(i2, n2, 1);
                for (int i1 = 0; i1 < n1; ++i1) {
                    int k1 = orc_mode_k(i1, n1, 1);
                    cplx acc = {0, 0};
                    for (int64_t j = 0; j < M; ++j) {
                        cplx fj = ci[j + M * b];
                        if (fj.re == 0 && fj.im == 0) continue;
                        acc = c_add(acc, c_mul(fj, c_cis(s * ((double)k1 * x[j] + (double)k2 * y[j]))));
                    }
                    co[i1 + (int64_t)n1 * i2 + (int64_t)n1 * n2 * b] = acc;
                }
            }
    }
}

/* ------------------------------------------------------------------------------------ */
/* ES-kernel NUFFT (own implementation of the published FINUFFT algorithm; used as the   */
/* fast CPU NUFFT of the timed baseline and to pin the device NUFFT)                      */
/* ------------------------------------------------------------------------------------ */
struct orc_esnufft {
    int n1, n2, B, w, nf1, nf2;
    double tol, beta;
    double *dec1, *dec2;
    int64_t M;
    double *x, *y;
    cplx* grid;
    int kermode;  /* ORC_KER_EXACT or ORC_KER_POLY */
    double* cheb; /* w x (w + 3) Chebyshev coefficients per tap */
};

/* Per-tap Chebyshev interpolant of the ES kernel (FINUFFT's default piecewise-polynomial
 * kernel evaluation): tap a as a function of s = i0 - g + w/2 in [0, 1), interpolated at
 * the w + 3 Chebyshev points of the first kind (degree w + 2). */
static void es_cheb_fit(int w, double beta, double* cheb) {
    const int n = w + 3;
    double ys[32];
    for (int a = 0; a < w; ++a) {
        for (int i = 0; i < n; ++i) {
            double t = cos(M_PI * (i + 0.5) / n);
            double z = ((t + 1.0) / 2.0 + a - 0.5 * w) / (0.5 * w);
            ys[i] = orc_es_kernel(z, beta);
        }
        for (int k = 0; k < n; ++k) {
            double acc = 0.0;
            for (int i = 0; i < n; ++i) acc += ys[i] * cos(k * M_PI * (i + 0.5) / n);
            cheb[a * n + k] = (k == 0 ? 1.0 : 2.0) * acc / n;
        }
    }
}

static double es_cheb_eval(const double* c, int n, double t) {
    double b1 = 0.0, b2 = 0.0;
    for (int k = n - 1; k >= 1; --k) {
        double b0 = c[k] + 2.0 * t * b1 - b2;
        b2 = b1;
        b1 = b0;
    }
    return c[0] + t * b1 - b2;
}

double orc_es_kernel(double z, double beta) {
    if (fabs(z) >= 1.0) return 0.0;
    return exp(beta * (sqrt(1.0 - z * z) - 1.0));
}

/* 1 / Phi(k), Phi(k) = int_{-w/2}^{w/2} phi(2s/w) cos(2 pi k s / nf) ds, by composite
 * Gauss-Legendre after z = sin t (the branch point at |z| = 1 disappears). */
double orc_es_deconv(int k, int nf, int w, double beta) {
    const int npan = 40;
    double a = 0.0, b = M_PI / 2;
    double hw = (b - a) / (2 * npan);
    double acc = 0.0;
    double om = M_PI * (double)k * (double)w / (double)nf;
    for (int p = 0; p < npan; ++p) {
        double c = a + (2 * p + 1) * hw;
        double s = 0.0;
        for (int q = 0; q < 10; ++q) {
            double t = c + hw * GL10_X[q];
            double st = sin(t), ct = cos(t);
            s += GL10_W[q] * exp(beta * (ct - 1.0)) * cos(om * st) * ct;
        }
        acc += hw * s;
    }
    return 1.0 / ((double)w * acc);
}

static int es_width(double tol) {
    int w = (int)ceil(-log10(tol / 10.0));
    if (w < 2) w = 2;
    if (w > 16) w = 16;
    return w;
}

orc_esnufft* orc_esnufft_create(int n1, int n2, int ntrans, double tol, const double* x,
                                const double* y, int64_t M) {
    return orc_esnufft_create_k(n1, n2, ntrans, tol, x, y, M, ORC_KER_POLY);
}

orc_esnufft* orc_esnufft_create_k(int n1, int n2, int ntrans, double tol, const double* x,
                                  const double* y, int64_t M, int kermode) {
    orc_esnufft* p = (orc_esnufft*)calloc(1, sizeof(orc_esnufft));
    p->kermode = kermode;
    p->n1 = n1;
    p->n2 = n2;
    p->B = ntrans;
    p->tol = tol;
    p->w = es_width(tol);
    p->beta = 2.30 * p->w;
    int64_t a = 2 * (int64_t)n1 > 2 * p->w ? 2 * (int64_t)n1 : 2 * p->w;
    int64_t c = 2 * (int64_t)n2 > 2 * p->w ? 2 * (int64_t)n2 : 2 * p->w;
    p->nf1 = (int)orc_next_smooth(a);
    p->nf2 = (int)orc_next_smooth(c);
    p->dec1 = (double*)malloc(sizeof(double) * n1);
    p->dec2 = (double*)malloc(sizeof(double) * n2);
    for (int i = 0; i < n1; ++i) p->dec1[i] = orc_es_deconv(orc_mode_k(i, n1, 1), p->nf1, p->w, p->beta);
    for (int i = 0; i < n2; ++i) p->dec2[i] = orc_es_deconv(orc_mode_k(i, n2, 1), p->nf2, p->w, p->beta);
    p->M = M;
    p->x = (double*)malloc(sizeof(double) * (M > 0 ? M : 1));
    p->y = (double*)malloc(sizeof(double) * (M > 0 ? M : 1));
    memcpy(p->x, x, sizeof(double) * M);
    memcpy(p->y, y, sizeof(double) * M);
    p->grid = (cplx*)malloc(sizeof(cplx) * (size_t)p->nf1 * p->nf2);
    p->cheb = (double*)malloc(sizeof(double) * p->w * (p->w + 3));
    es_cheb_fit(p->w, p->beta, p->cheb);
    return p;
}

void orc_esnufft_destroy(orc_esnufft* p) {
    if (!p) return;
    free(p->dec1); free(p->dec2); free(p->x); free(p->y); free(p->grid); free(p->cheb);
    free(p);
}

/* Fine-grid lengths other than the minimum (any nf1 >= max(2 n1, 2 w), likewise nf2): the
 * per-mode deconvolution follows the lengths. Used to mirror a device plan's lengths. */
int orc_esnufft_set_grid(orc_esnufft* p, int nf1, int nf2) {
    if (nf1 < 2 * p->n1 || nf1 < 2 * p->w || nf2 < 2 * p->n2 || nf2 < 2 * p->w) return 1;
    p->nf1 = nf1;
    p->nf2 = nf2;
    for (int i = 0; i < p->n1; ++i) p->dec1[i] = orc_es_deconv(orc_mode_k(i, p->n1, 1), nf1, p->w, p->beta);
    for (int i = 0; i < p->n2; ++i) p->dec2[i] = orc_es_deconv(orc_mode_k(i, p->n2, 1), nf2, p->w, p->beta);
    free(p->grid);
    p->grid = (cplx*)malloc(sizeof(cplx) * (size_t)nf1 * nf2);
    return 0;
}

void orc_esnufft_params(const orc_esnufft* p, int* w, double* beta, int* nf1, int* nf2) {
    if (w) *w = p->w;
    if (beta) *beta = p->beta;
    if (nf1) *nf1 = p->nf1;
    if (nf2) *nf2 = p->nf2;
}

static inline int wrapi(int64_t i, int n) {
    int64_t r = i % n;
    return (int)(r < 0 ? r + n : r);
}

/* kernel taps of one coordinate: first cell index and w weights */
static inline int64_t es_taps_p(const orc_esnufft* p, double xg, double* ker) {
    const int w = p->w;
    double hw = 0.5 * w;
    int64_t i0 = (int64_t)ceil(xg - hw);
    if (p->kermode == ORC_KER_POLY) {
        double v = ((double)i0 - xg) + (hw - 0.5);
        for (int a = 0; a < w; ++a) ker[a] = es_cheb_eval(p->cheb + a * (w + 3), w + 3, 2.0 * v);
    } else {
        for (int a = 0; a < w; ++a) ker[a] = orc_es_kernel(((double)(i0 + a) - xg) / hw, p->beta);
    }
    return i0;
}

void orc_esnufft_exec(orc_esnufft* p, int type, int iflag, const double* in, double* out,
                      int nthreads) {
    const int n1 = p->n1, n2 = p->n2, nf1 = p->nf1, nf2 = p->nf2, w = p->w;
    const int64_t M = p->M;
    const double s1 = nf1 / (2 * M_PI), s2 = nf2 / (2 * M_PI);
    int nt = nthreads_ok(nthreads);
    const cplx* ci = (const cplx*)in;
    cplx* co = (cplx*)out;
    for (int b = 0; b < p->B; ++b) {
        memset(p->grid, 0, sizeof(cplx) * (size_t)nf1 * nf2);
        if (type == 2) {
            for (int i2 = 0; i2 < n2; ++i2) {
                int k2 = orc_mode_k(i2, n2, 1);
                int q2 = wrapi(k2, nf2);
                for (int i1 = 0; i1 < n1; ++i1) {
                    int k1 = orc_mode_k(i1, n1, 1);
                    int q1 = wrapi(k1, nf1);
                    p->grid[q1 + (int64_t)nf1 * q2] =
                        c_scale(ci[i1 + (int64_t)n1 * i2 + (int64_t)n1 * n2 * b], p->dec1[i1] * p->dec2[i2]);
                }
            }
            orc_fft_cols((double*)p->grid, nf1, nf2, iflag, nt);
            orc_fft_rows((double*)p->grid, nf1, nf2, iflag, nt);
#ifdef _OPENMP
#pragma omp parallel for num_threads(nt) schedule(static)
#endif
            for (int64_t j = 0; j < M; ++j) {
                double k1w[16], k2w[16];
                int64_t i10 = es_taps_p(p, p->x[j] * s1, k1w);
                int64_t i20 = es_taps_p(p, p->y[j] * s2, k2w);
                cplx acc = {0, 0};
                for (int bb = 0; bb < w; ++bb) {
                    int c2 = wrapi(i20 + bb, nf2);
                    cplx row = {0, 0};
                    for (int a = 0; a < w; ++a)
                        row = c_add(row, c_scale(p->grid[wrapi(i10 + a, nf1) + (int64_t)nf1 * c2], k1w[a]));
                    acc = c_add(acc, c_scale(row, k2w[bb]));
                }
                co[j + M * b] = acc;
            }
        } else {
            /* spread: thread t owns a band of grid columns and takes every point whose
             * stencil reaches it, so no two threads write one cell */
#ifdef _OPENMP
#pragma omp parallel num_threads(nt)
#endif
            {
                int t = 0, T = 1;
#ifdef _OPENMP
                t = omp_get_thread_num();
                T = omp_get_num_threads();
#endif
                int c0 = (int)((int64_t)nf2 * t / T), c1 = (int)((int64_t)nf2 * (t + 1) / T);
                for (int64_t j = 0; j < M; ++j) {
                    cplx fj = ci[j + M * b];
                    double g2 = p->y[j] * s2;
                    int64_t i20 = (int64_t)ceil(g2 - 0.5 * w);
                    int hit = 0;
                    for (int bb = 0; bb < w && !hit; ++bb) {
                        int c2 = wrapi(i20 + bb, nf2);
                        if (c2 >= c0 && c2 < c1) hit = 1;
                    }
                    if (!hit) continue;
                    double k1w[16], k2w[16];
                    int64_t i10 = es_taps_p(p, p->x[j] * s1, k1w);
                    es_taps_p(p, g2, k2w);
                    for (int bb = 0; bb < w; ++bb) {
                        int c2 = wrapi(i20 + bb, nf2);
                        if (c2 < c0 || c2 >= c1) continue;
                        cplx v = c_scale(fj, k2w[bb]);
                        for (int a = 0; a < w; ++a) {
                            cplx* g = &p->grid[wrapi(i10 + a, nf1) + (int64_t)nf1 * c2];
                            *g = c_add(*g, c_scale(v, k1w[a]));
                        }
                    }
                }
            }
            orc_fft_cols((double*)p->grid, nf1, nf2, iflag, nt);
            orc_fft_rows((double*)p->grid, nf1, nf2, iflag, nt);
            for (int i2 = 0; i2 < n2; ++i2) {
                int q2 = wrapi(orc_mode_k(i2, n2, 1), nf2);
                for (int i1 = 0; i1 < n1; ++i1) {
                    int q1 = wrapi(orc_mode_k(i1, n1, 1), nf1);
                    co[i1 + (int64_t)n1 * i2 + (int64_t)n1 * n2 * b] =
                        c_scale(p->grid[q1 + (int64_t)nf1 * q2], p->dec1[i1] * p->dec2[i2]);
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------------------ */
/* Direct leaf (src/Direct.jl:15-117). Points are sorted by colatitude and walked as their */
/* own rings with eps = 0 (no polar truncation); blocks of sorted points bound memory.    */
/* ------------------------------------------------------------------------------------ */
#define DIRECT_BLOCK 256
struct orc_direct {
    int L, B;
    int64_t M;
    int64_t* perm;
    double *ths, *phs;
    int nblocks;
    orc_rings** eng;
};

static const double* g_sort_key;
static int cmp_perm(const void* a, const void* b) {
    int64_t i = *(const int64_t*)a, j = *(const int64_t*)b;
    double x = g_sort_key[i], y = g_sort_key[j];
    if (x < y) return -1;
    if (x > y) return 1;
    return i < j ? -1 : (i > j);
}

orc_direct* orc_direct_create(const double* theta, const double* phi, int64_t M, int lmax,
                              int ntrans) {
    if (M < 1 || lmax < 0 || ntrans < 1) return NULL;
    orc_direct* d = (orc_direct*)calloc(1, sizeof(orc_direct));
    d->L = lmax;
    d->B = ntrans;
    d->M = M;
    d->perm = (int64_t*)malloc(sizeof(int64_t) * M);
    for (int64_t i = 0; i < M; ++i) d->perm[i] = i;
    g_sort_key = theta;
    qsort(d->perm, M, sizeof(int64_t), cmp_perm); /* stable via the index tie-break */
    d->ths = (double*)malloc(sizeof(double) * M);
    d->phs = (double*)malloc(sizeof(double) * M);
    for (int64_t i = 0; i < M; ++i) {
        d->ths[i] = theta[d->perm[i]];
        d->phs[i] = phi[d->perm[i]];
    }
    d->nblocks = (int)((M + DIRECT_BLOCK - 1) / DIRECT_BLOCK);
    d->eng = (orc_rings**)calloc(d->nblocks, sizeof(orc_rings*));
    for (int k = 0; k < d->nblocks; ++k) {
        int64_t i0 = (int64_t)k * DIRECT_BLOCK;
        int n = (int)((M - i0) < DIRECT_BLOCK ? (M - i0) : DIRECT_BLOCK);
        d->eng[k] = orc_rings_create(d->ths + i0, n, lmax, 0.0, ntrans, 0);
    }
    return d;
}

void orc_direct_destroy(orc_direct* d) {
    if (!d) return;
    for (int k = 0; k < d->nblocks; ++k) orc_rings_destroy(d->eng[k]);
    free(d->eng); free(d->perm); free(d->ths); free(d->phs);
    free(d);
}

/* synthesize_direct! (src/Direct.jl:60-86) */
void orc_direct_forward(orc_direct* d, const double* alm, double* f, int nthreads) {
    const int L = d->L, B = d->B;
    const int64_t M = d->M;
    cplx* fo = (cplx*)f;
    memset(f, 0, sizeof(cplx) * (size_t)M * B);
    int nt = nthreads_ok(nthreads);
#ifdef _OPENMP
#pragma omp parallel for num_threads(nt) schedule(dynamic)
#endif
    for (int k = 0; k < d->nblocks; ++k) {
        const orc_rings* e = d->eng[k];
        int n = e->n;
        int64_t i0 = (int64_t)k * DIRECT_BLOCK;
        cplx* G = (cplx*)malloc(sizeof(cplx) * (size_t)n * (2 * L + 1) * B);
        orc_rings_from_alm(e, alm, (double*)G, 1);
        for (int b = 0; b < B; ++b)
            for (int i = 0; i < n; ++i) {
                const cplx* Gb = G + (int64_t)n * (2 * L + 1) * b;
                cplx acc = Gb[i + (int64_t)n * L];
                double ph0 = d->phs[i0 + i];
                for (int m = 1; m <= L; ++m) {
                    cplx ph = c_cis((double)m * ph0);
                    acc = c_add(acc, c_add(c_mul(Gb[i + (int64_t)n * (m + L)], ph),
                                           c_mul(Gb[i + (int64_t)n * (-m + L)], c_conj(ph))));
                }
                fo[d->perm[i0 + i] + M * b] = acc;
            }
        free(G);
    }
}

/* adjoint_direct! (src/Direct.jl:94-117), summed over point blocks */
void orc_direct_adjoint(orc_direct* d, const double* f, double* alm, int nthreads) {
    const int L = d->L, B = d->B;
    const int64_t M = d->M;
    const size_t na = (size_t)(L + 1) * (2 * L + 1) * B;
    const cplx* fi = (const cplx*)f;
    memset(alm, 0, sizeof(cplx) * na);
    int nt = nthreads_ok(nthreads);
#ifdef _OPENMP
#pragma omp parallel num_threads(nt)
#endif
    {
        double* part = (double*)calloc(2 * na, sizeof(double));
        double* tmp = (double*)malloc(sizeof(double) * 2 * na);
#ifdef _OPENMP
#pragma omp for schedule(dynamic)
#endif
        for (int k = 0; k < d->nblocks; ++k) {
            const orc_rings* e = d->eng[k];
            int n = e->n;
            int64_t i0 = (int64_t)k * DIRECT_BLOCK;
            cplx* G = (cplx*)calloc((size_t)n * (2 * L + 1) * B, sizeof(cplx));
            for (int b = 0; b < B; ++b)
                for (int i = 0; i < n; ++i) {
                    cplx fv = fi[d->perm[i0 + i] + M * b];
                    if (fv.re == 0 && fv.im == 0) continue;
                    cplx* Gb = G + (int64_t)n * (2 * L + 1) * b;
                    double ph0 = d->phs[i0 + i];
                    Gb[i + (int64_t)n * L] = fv;
                    for (int m = 1; m <= L; ++m) {
                        cplx ph = c_cis((double)m * ph0);
                        Gb[i + (int64_t)n * (m + L)] = c_mul(fv, c_conj(ph));
                        Gb[i + (int64_t)n * (-m + L)] = c_mul(fv, ph);
                    }
                }
            orc_alm_from_rings(e, (const double*)G, tmp, 1);
            for (size_t q = 0; q < 2 * na; ++q) part[q] += tmp[q];
            free(G);
        }
#ifdef _OPENMP
#pragma omp critical
#endif
        for (size_t q = 0; q < 2 * na; ++q) alm[q] += part[q];
        free(part);
        free(tmp);
    }
}

/* ------------------------------------------------------------------------------------ */
/* stretched leaf (src/Stretch.jl:129-295)                                               */
/* ------------------------------------------------------------------------------------ */
struct orc_stretch {
    orc_stretch_info info;
    orc_geom geom;
    double *th_r, *Th_r, *w, *Thp, *php;
    cplx *phase;
    orc_rings* eng;
    int spin;
    orc_spin_rings* seng;  /* spin != 0: the Wigner-d engine (src/Stretch.jl:190-192) */
    int nufft_kind;
    orc_esnufft* es;
    cplx *G, *Fphi, *F, *Ft, *Fhat;
};

orc_stretch* orc_stretch_create(const double* theta, const double* phi, int64_t M, int lmax,
                                int ntrans, double tol, int nufft_kind, double eps_apo_max,
                                double ovs_th, double ovs_ph, int* status) {
    return orc_stretch_create_spin(theta, phi, M, lmax, ntrans, tol, nufft_kind, eps_apo_max,
                                   ovs_th, ovs_ph, 0, status);
}

orc_stretch* orc_stretch_create_spin(const double* theta, const double* phi, int64_t M, int lmax,
                                     int ntrans, double tol, int nufft_kind, double eps_apo_max,
                                     double ovs_th, double ovs_ph, int spin, int* status) {
    *status = 0;
    if (M < 1 || lmax < 0 || ntrans < 1) { *status = 2; return NULL; }
    /* bounding_box colatitude extent (src/Box.jl:51-59) */
    double lo = INFINITY, hi = -INFINITY;
    for (int64_t i = 0; i < M; ++i) { lo = fmin(lo, theta[i]); hi = fmax(hi, theta[i]); }
    lo = fmax(lo, 0.0);
    hi = fmin(hi, M_PI);
    double tiny = sqrt(DBL_EPSILON);
    orc_geom g0, g;
    int r = orc_try_stretch_geometry(lo, hi, lmax, tol, eps_apo_max, &g0);
    if (r < 0) { *status = 2; return NULL; }
    if (r == 0) { *status = 1; return NULL; }
    int flip = g0.kind == ORC_POLE && g0.theta_hi >= M_PI - tiny && g0.theta_lo > tiny;
    if (flip) {
        r = orc_try_stretch_geometry(M_PI - hi, M_PI - lo, lmax, tol, eps_apo_max, &g);
        if (r != 1) { *status = 1; return NULL; }
    } else {
        g = g0;
    }
    orc_stretch* s = (orc_stretch*)calloc(1, sizeof(orc_stretch));
    s->geom = g;
    int64_t Kth = (int64_t)ceil((double)(g.K + K_MARGIN) * ovs_th);
    int nth, nth_half;
    if (g.kind == ORC_INTERIOR) {
        nth = (int)orc_next_smooth(2 * Kth + 1);
        nth_half = nth;
    } else {
        nth_half = (int)orc_next_smooth(Kth + 1);
        nth = 2 * nth_half;
    }
    s->th_r = (double*)malloc(sizeof(double) * nth_half);
    s->Th_r = (double*)malloc(sizeof(double) * nth_half);
    orc_stretch_rings(&g, nth_half, s->th_r, s->Th_r);
    s->spin = spin;
    int mmax;
    if (spin == 0) {
        s->eng = orc_rings_create(s->th_r, nth_half, lmax, tol, ntrans, flip);
        if (!s->eng) { *status = 2; orc_stretch_destroy(s); return NULL; }
        mmax = s->eng->mmax;
    } else {
        s->seng = orc_spin_rings_create(s->th_r, nth_half, lmax, spin, tol, ntrans, flip);
        if (!s->seng) { *status = 2; orc_stretch_destroy(s); return NULL; }
        mmax = orc_spin_rings_mmax(s->seng);
    }
    int mm = mmax > abs(spin) ? mmax : abs(spin);
    int nph = (int)orc_next_smooth_even((int64_t)ceil((2.0 * mm + 1) * ovs_ph));
    s->w = (double*)malloc(sizeof(double) * nth_half);
    for (int i = 0; i < nth_half; ++i) s->w[i] = orc_stretch_window(&g, s->Th_r[i]);
    s->Thp = (double*)malloc(sizeof(double) * M);
    s->php = (double*)malloc(sizeof(double) * M);
    for (int64_t i = 0; i < M; ++i) {
        double t = theta[i];
        s->Thp[i] = orc_theta_to_stretch(&g, flip ? M_PI - t : t);
        s->php[i] = jl_mod(phi[i], 2 * M_PI);
    }
    double shift = g.kind == ORC_INTERIOR ? 0.0 : M_PI / nth;
    double N = (double)nth * (double)nph;
    s->phase = (cplx*)malloc(sizeof(cplx) * nth);
    for (int i = 0; i < nth; ++i) {
        cplx c = c_cis(-(double)orc_mode_k(i, nth, 1) * shift);
        s->phase[i].re = c.re / N;
        s->phase[i].im = c.im / N;
    }
    s->nufft_kind = nufft_kind;
    if (nufft_kind == ORC_NUFFT_ES || nufft_kind == ORC_NUFFT_ES_EXACT)
        s->es = orc_esnufft_create_k(nth, nph, ntrans, tol, s->Thp, s->php, M,
                                     nufft_kind == ORC_NUFFT_ES ? ORC_KER_POLY : ORC_KER_EXACT);
    size_t B = ntrans;
    s->G = (cplx*)calloc((size_t)nth_half * (2 * lmax + 1) * B, sizeof(cplx));
    s->Fphi = (cplx*)calloc((size_t)nth_half * nph * B, sizeof(cplx));
    s->F = (cplx*)calloc((size_t)nth_half * nph * B, sizeof(cplx));
    s->Ft = (cplx*)calloc((size_t)nth * nph * B, sizeof(cplx));
    s->Fhat = (cplx*)calloc((size_t)nth * nph * B, sizeof(cplx));
    orc_stretch_info* in = &s->info;
    in->kind = g.kind;
    in->flip = flip;
    in->lmax = lmax;
    in->ntrans = ntrans;
    in->nth_half = nth_half;
    in->nth = nth;
    in->nph = nph;
    in->mmax = mmax;
    in->nrings = nth_half;
    in->K = g.K;
    in->ring_work = spin == 0 ? orc_rings_work(s->eng) : orc_spin_rings_work(s->seng);
    in->M = M;
    in->eps = g.eps;
    in->beta = g.beta;
    in->h = g.h;
    in->theta_lo = g.theta_lo;
    in->theta_hi = g.theta_hi;
    in->eps_apo = g.eps_apo;
    in->Theta1 = g.Theta1;
    in->sigma = g.sigma;
    in->ThetaT = g.ThetaT;
    in->box_lo = lo;
    in->box_hi = hi;
    return s;
}

void orc_stretch_destroy(orc_stretch* s) {
    if (!s) return;
    free(s->th_r); free(s->Th_r); free(s->w); free(s->Thp); free(s->php); free(s->phase);
    orc_rings_destroy(s->eng);
    orc_spin_rings_destroy(s->seng);
    orc_esnufft_destroy(s->es);
    free(s->G); free(s->Fphi); free(s->F); free(s->Ft); free(s->Fhat);
    free(s);
}

void orc_stretch_info_get(const orc_stretch* s, orc_stretch_info* out) { *out = s->info; }

int orc_stretch_set_nufft_grid(orc_stretch* s, int nf1, int nf2) {
    return s->es ? orc_esnufft_set_grid(s->es, nf1, nf2) : 1;
}
const orc_rings* orc_stretch_rings_engine(const orc_stretch* s) { return s->eng; }

void orc_stretch_tables(const orc_stretch* s, double* th_r, double* Th_r, double* w,
                        double* Thp, double* php) {
    int n = s->info.nth_half;
    if (th_r) memcpy(th_r, s->th_r, sizeof(double) * n);
    if (Th_r) memcpy(Th_r, s->Th_r, sizeof(double) * n);
    if (w) memcpy(w, s->w, sizeof(double) * n);
    if (Thp) memcpy(Thp, s->Thp, sizeof(double) * s->info.M);
    if (php) memcpy(php, s->php, sizeof(double) * s->info.M);
}

/* _order_blocks (src/Stretch.jl:332-339) */
static int mkeep_of(int nph, int L) { int a = (nph - 1) / 2; return L < a ? L : a; }

void orc_stretch_forward(orc_stretch* s, const double* alm, double* f, int nthreads) {
    const orc_stretch_info* in = &s->info;
    const int L = in->lmax, B = in->ntrans, nh = in->nth_half, nth = in->nth, nph = in->nph;
    const int64_t M = in->M;
    /* _fill_rings! */
    if (s->spin == 0) orc_rings_from_alm(s->eng, alm, (double*)s->G, nthreads);
    else orc_spin_rings_from_alm(s->seng, alm, (double*)s->G, nthreads);
    /* _rings_to_grid!: _pack_orders! (src/Stretch.jl:341-350) then bfft along phi */
    int mk = mkeep_of(nph, L);
    memset(s->Fphi, 0, sizeof(cplx) * (size_t)nh * nph * B);
    for (int b = 0; b < B; ++b) {
        for (int m = 0; m <= mk; ++m)
            memcpy(s->Fphi + (int64_t)nh * m + (int64_t)nh * nph * b,
                   s->G + (int64_t)nh * (m + L) + (int64_t)nh * (2 * L + 1) * b, sizeof(cplx) * nh);
        for (int m = 1; m <= mk; ++m)
            memcpy(s->Fphi + (int64_t)nh * (nph - m) + (int64_t)nh * nph * b,
                   s->G + (int64_t)nh * (L - m) + (int64_t)nh * (2 * L + 1) * b, sizeof(cplx) * nh);
    }
    memcpy(s->F, s->Fphi, sizeof(cplx) * (size_t)nh * nph * B);
    for (int b = 0; b < B; ++b) orc_fft_rows((double*)(s->F + (int64_t)nh * nph * b), nh, nph, +1, nthreads);
    /* F .*= w */
    for (int b = 0; b < B; ++b)
        for (int j = 0; j < nph; ++j)
            for (int i = 0; i < nh; ++i) {
                cplx* v = &s->F[i + (int64_t)nh * j + (int64_t)nh * nph * b];
                *v = c_scale(*v, s->w[i]);
            }
    /* _periodize! */
    if (in->kind == ORC_INTERIOR) memcpy(s->Ft, s->F, sizeof(cplx) * (size_t)nh * nph * B);
    else orc_dfs_double((double*)s->F, (double*)s->Ft, nh, nph, B, s->spin);
    /* 2-D fft, then phase */
    memcpy(s->Fhat, s->Ft, sizeof(cplx) * (size_t)nth * nph * B);
    for (int b = 0; b < B; ++b) {
        double* blk = (double*)(s->Fhat + (int64_t)nth * nph * b);
        orc_fft_cols(blk, nth, nph, -1, nthreads);
        orc_fft_rows(blk, nth, nph, -1, nthreads);
    }
    for (int b = 0; b < B; ++b)
        for (int j = 0; j < nph; ++j)
            for (int i = 0; i < nth; ++i) {
                cplx* v = &s->Fhat[i + (int64_t)nth * j + (int64_t)nth * nph * b];
                *v = c_mul(*v, s->phase[i]);
            }
    /* type-2 NUFFT, iflag +1 */
    if (s->es) orc_esnufft_exec(s->es, 2, +1, (double*)s->Fhat, f, nthreads);
    else orc_nufft_direct(2, nth, nph, +1, B, s->Thp, s->php, M, (double*)s->Fhat, f);
}

void orc_stretch_adjoint(orc_stretch* s, const double* f, double* alm, int nthreads) {
    const orc_stretch_info* in = &s->info;
    const int L = in->lmax, B = in->ntrans, nh = in->nth_half, nth = in->nth, nph = in->nph;
    const int64_t M = in->M;
    /* type-1 NUFFT, iflag -1 */
    if (s->es) orc_esnufft_exec(s->es, 1, -1, f, (double*)s->Fhat, nthreads);
    else orc_nufft_direct(1, nth, nph, -1, B, s->Thp, s->php, M, f, (double*)s->Fhat);
    for (int b = 0; b < B; ++b)
        for (int j = 0; j < nph; ++j)
            for (int i = 0; i < nth; ++i) {
                cplx* v = &s->Fhat[i + (int64_t)nth * j + (int64_t)nth * nph * b];
                *v = c_mul(*v, c_conj(s->phase[i]));
            }
    memcpy(s->Ft, s->Fhat, sizeof(cplx) * (size_t)nth * nph * B);
    for (int b = 0; b < B; ++b) {
        double* blk = (double*)(s->Ft + (int64_t)nth * nph * b);
        orc_fft_cols(blk, nth, nph, +1, nthreads);
        orc_fft_rows(blk, nth, nph, +1, nthreads);
    }
    if (in->kind == ORC_INTERIOR) memcpy(s->F, s->Ft, sizeof(cplx) * (size_t)nh * nph * B);
    else orc_dfs_fold((double*)s->F, (const double*)s->Ft, nh, nph, B, s->spin);
    for (int b = 0; b < B; ++b)
        for (int j = 0; j < nph; ++j)
            for (int i = 0; i < nh; ++i) {
                cplx* v = &s->F[i + (int64_t)nh * j + (int64_t)nh * nph * b];
                *v = c_scale(*v, s->w[i]);
            }
    /* _grid_to_rings!: fft along phi then _unpack_orders! (src/Stretch.jl:352-364) */
    memcpy(s->Fphi, s->F, sizeof(cplx) * (size_t)nh * nph * B);
    for (int b = 0; b < B; ++b) orc_fft_rows((double*)(s->Fphi + (int64_t)nh * nph * b), nh, nph, -1, nthreads);
    int mk = mkeep_of(nph, L);
    memset(s->G, 0, sizeof(cplx) * (size_t)nh * (2 * L + 1) * B);
    for (int b = 0; b < B; ++b) {
        for (int m = 0; m <= mk; ++m)
            memcpy(s->G + (int64_t)nh * (m + L) + (int64_t)nh * (2 * L + 1) * b,
                   s->Fphi + (int64_t)nh * m + (int64_t)nh * nph * b, sizeof(cplx) * nh);
        for (int m = 1; m <= mk; ++m)
            memcpy(s->G + (int64_t)nh * (L - m) + (int64_t)nh * (2 * L + 1) * b,
                   s->Fphi + (int64_t)nh * (nph - m) + (int64_t)nh * nph * b, sizeof(cplx) * nh);
    }
    if (s->spin == 0) orc_alm_from_rings(s->eng, (const double*)s->G, alm, nthreads);
    else orc_spin_alm_from_rings(s->seng, (const double*)s->G, alm, nthreads);
}

/* ------------------------------------------------------------------------------------ */
/* spin-weighted transforms (src/Spin.jl)                                                 */
/* ------------------------------------------------------------------------------------ */
static double spin_Nl(int l) { return sqrt((2.0 * l + 1) / (4 * M_PI)); }
static inline cplx c_make(double re, double im) { cplx r = {re, im}; return r; }

/* log sqrt(C(2l, l - a)) (src/Spin.jl:26-29) */
static double half_lbinom(int l, int a) {
    return (lgamma(2.0 * l + 1) - lgamma((double)(l - a) + 1) - lgamma((double)(l + a) + 1)) / 2;
}

/* _d_extremal (src/Spin.jl:38-51): log|d^l_{a,b}(beta)| and its sign, |b| = l */
static void d_extremal(int l, int a, int b, double beta, double* lg, double* sg) {
    double c = cos(beta / 2), s = sin(beta / 2);
    double lb = half_lbinom(l, a);
    int pc, ps;
    double sgn;
    if (b == l) { pc = l + a; ps = l - a; sgn = 1.0; }
    else { pc = l - a; ps = l + a; sgn = ((l - a) % 2 == 0) ? 1.0 : -1.0; }
    double lc = pc == 0 ? 0.0 : (c > 0 ? (double)pc * log(c) : -INFINITY);
    double ls = ps == 0 ? 0.0 : (s > 0 ? (double)ps * log(s) : -INFINITY);
    *lg = lb + lc + ls;
    *sg = sgn;
}

/* wigner_d (src/Spin.jl:58-131): block-scaled degree recurrence at fixed (m, n) */
double orc_wigner_d(int l, int mm, int nn, double b) {
    if (abs(mm) > l || abs(nn) > l) return 0.0;
    double tiny = sqrt(DBL_EPSILON);
    if (b <= tiny) return mm == nn ? 1.0 : 0.0;
    if (b >= M_PI - tiny) return mm == -nn ? (((l - nn) % 2 == 0) ? 1.0 : -1.0) : 0.0;
    int l0 = abs(mm) > abs(nn) ? abs(mm) : abs(nn);
    double lg, sg;
    if (abs(nn) == l0) {
        d_extremal(l0, mm, nn == l0 ? l0 : -l0, b, &lg, &sg);
    } else {
        d_extremal(l0, nn, mm == l0 ? l0 : -l0, b, &lg, &sg);
        if (((nn - mm) % 2 + 2) % 2 == 1) sg = -sg;
    }
    if (!isfinite(lg)) return 0.0;
    double E = ceil(lg / log(2.0));
    double d1 = sg * exp(lg - E * log(2.0));
    if (l == l0) return d1 * exp2(E);
    double cb = cos(b);
    double d0 = 0.0;
    int Lc = l0;
    if (l0 == 0) {
        d0 = d1;
        d1 = d1 * cb;
        Lc = 1;
        if (l == 1) return d1 * exp2(E);
    }
    int steps = 0;
    while (Lc < l) {
        int L1 = Lc + 1;
        double sm1 = sqrt(fmax(0.0, (double)(L1 * L1 - mm * mm)));
        double sn1 = sqrt(fmax(0.0, (double)(L1 * L1 - nn * nn)));
        double den = (double)Lc * sm1 * sn1;
        if (den <= 0) { d0 = d1; d1 = 0.0; Lc = L1; continue; }
        double sm0 = sqrt(fmax(0.0, (double)(Lc * Lc - mm * mm)));
        double sn0 = sqrt(fmax(0.0, (double)(Lc * Lc - nn * nn)));
        double c1 = (double)(2 * Lc + 1) * ((double)Lc * (double)L1 * cb - (double)mm * (double)nn) / den;
        double c0 = (double)L1 * sm0 * sn0 / den;
        double dn = c1 * d1 - c0 * d0;
        d0 = d1;
        d1 = dn;
        Lc = L1;
        if (++steps == RESCALE_STRIDE) {
            steps = 0;
            double mx = fmax(fabs(d1), fabs(d0));
            if (mx > 0 && isfinite(mx)) {
                double sh = ceil(log2(mx));
                if (sh != 0) { double f = exp2(-sh); d1 *= f; d0 *= f; E += sh; }
            }
        }
    }
    return d1 * exp2(E);
}

/* SpinRings (src/Spin.jl:175-280) */
struct orc_spin_rings {
    int n, L, s, B, mmax;
    double eps;
    double *cos_t, *log2cos, *log2sin, *Nl, *lb2, *sg;
    int *pc, *ps, *mlim, *jlo, *jhi; /* jlo/jhi over m = -L..L */
    int nchunks, *clo, *chi;
};

orc_spin_rings* orc_spin_rings_create(const double* theta, int n, int lmax, int spin, double eps,
                                      int ntrans, int reflect) {
    if (lmax < 0 || ntrans < 1 || n < 1) return NULL;
    for (int j = 1; j < n; ++j)
        if (theta[j] < theta[j - 1]) return NULL;
    orc_spin_rings* e = (orc_spin_rings*)calloc(1, sizeof(orc_spin_rings));
    const int L = lmax, nm = 2 * lmax + 1, as = abs(spin);
    e->n = n; e->L = L; e->s = spin; e->B = ntrans; e->eps = eps;
    e->cos_t = (double*)malloc(sizeof(double) * n);
    e->log2cos = (double*)malloc(sizeof(double) * n);
    e->log2sin = (double*)malloc(sizeof(double) * n);
    e->mlim = (int*)malloc(sizeof(int) * n);
    e->Nl = (double*)malloc(sizeof(double) * (L + 1));
    e->lb2 = (double*)malloc(sizeof(double) * nm);
    e->sg = (double*)malloc(sizeof(double) * nm);
    e->pc = (int*)malloc(sizeof(int) * nm);
    e->ps = (int*)malloc(sizeof(int) * nm);
    e->jlo = (int*)malloc(sizeof(int) * nm);
    e->jhi = (int*)malloc(sizeof(int) * nm);
    e->clo = (int*)malloc(sizeof(int) * n);
    e->chi = (int*)malloc(sizeof(int) * n);
    double csgn = reflect ? -1.0 : 1.0;
    for (int j = 0; j < n; ++j) {
        double t = theta[j];
        e->cos_t[j] = csgn * cos(t);
        double ch = cos(t / 2), sh = fabs(sin(t / 2));
        if (reflect) { double x = ch; ch = sh; sh = x; }
        e->log2cos[j] = ch > 0 ? log2(ch) : -INFINITY;
        e->log2sin[j] = sh > 0 ? log2(sh) : -INFINITY;
        int ml = orc_polar_mmax(t, L, eps);
        e->mlim[j] = ml > as ? ml : as;
    }
    int* jlo0 = (int*)malloc(sizeof(int) * (L + 1));
    int* jhi0 = (int*)malloc(sizeof(int) * (L + 1));
    if (orc_nested_ranges(e->mlim, n, L, jlo0, jhi0) != 0) {
        free(jlo0); free(jhi0);
        orc_spin_rings_destroy(e);
        return NULL;
    }
    for (int m = 0; m <= L; ++m) {
        e->jlo[m + L] = e->jlo[L - m] = jlo0[m];
        e->jhi[m + L] = e->jhi[L - m] = jhi0[m];
    }
    free(jlo0); free(jhi0);
    const int nn = -spin;
    const double inv_ln2 = 1.0 / log(2.0);
    for (int m = -L; m <= L; ++m) {
        int idx = m + L;
        int l0 = abs(m) > abs(nn) ? abs(m) : abs(nn);
        if (l0 > L) { e->lb2[idx] = -INFINITY; e->pc[idx] = 0; e->ps[idx] = 0; e->sg[idx] = 1.0; continue; }
        int a, b;
        double extra;
        if (abs(nn) == l0) { a = m; b = nn == l0 ? l0 : -l0; extra = 1.0; }
        else { a = nn; b = m == l0 ? l0 : -l0; extra = ((((nn - m) % 2) + 2) % 2 == 1) ? -1.0 : 1.0; }
        double sgn;
        if (b == l0) { e->pc[idx] = l0 + a; e->ps[idx] = l0 - a; sgn = 1.0; }
        else { e->pc[idx] = l0 - a; e->ps[idx] = l0 + a; sgn = ((l0 - a) % 2 == 0) ? 1.0 : -1.0; }
        e->lb2[idx] = half_lbinom(l0, a) * inv_ln2;
        e->sg[idx] = sgn * extra;
    }
    /* _spin_ring_chunks (src/Spin.jl:291-317) */
    int i = 0, nc = 0;
    while (i < n) {
        int stop = i;
        int l0max = e->mlim[i] > as ? e->mlim[i] : as;
        while (stop < n - 1) {
            int nxt = stop + 1;
            if (nxt - i + 1 > CHUNK_MAX) break;
            double spanc = fabs(e->log2cos[nxt] - e->log2cos[i]);
            double spans = fabs(e->log2sin[nxt] - e->log2sin[i]);
            double span = fmax(isfinite(spanc) ? spanc : INFINITY, isfinite(spans) ? spans : INFINITY);
            int l0 = l0max;
            if (e->mlim[nxt] > l0) l0 = e->mlim[nxt];
            if (as > l0) l0 = as;
            if (2.0 * l0 * span > CHUNK_HEADROOM_BITS) break;
            l0max = l0;
            stop = nxt;
        }
        e->clo[nc] = i;
        e->chi[nc] = stop;
        ++nc;
        i = stop + 1;
    }
    e->nchunks = nc;
    for (int l = 0; l <= L; ++l) e->Nl[l] = spin_Nl(l);
    int mx = 0;
    for (int j = 0; j < n; ++j) mx = e->mlim[j] > mx ? e->mlim[j] : mx;
    e->mmax = mx;
    return e;
}

void orc_spin_rings_destroy(orc_spin_rings* e) {
    if (!e) return;
    free(e->cos_t); free(e->log2cos); free(e->log2sin); free(e->mlim); free(e->Nl); free(e->lb2);
    free(e->sg); free(e->pc); free(e->ps); free(e->jlo); free(e->jhi); free(e->clo); free(e->chi);
    free(e);
}

int orc_spin_rings_mmax(const orc_spin_rings* e) { return e->mmax; }
int orc_spin_rings_nchunks(const orc_spin_rings* e) { return e->nchunks; }

/* retained (l, m, ring) triples of the spin walk: m = -L..L, l from max(|m|, |s|) */
int64_t orc_spin_rings_work(const orc_spin_rings* e) {
    int64_t w = 0;
    for (int m = -e->L; m <= e->L; ++m) {
        int nj = e->jhi[m + e->L] - e->jlo[m + e->L] + 1;
        int l0 = abs(m) > abs(e->s) ? abs(m) : abs(e->s);
        if (nj > 0 && l0 <= e->L) w += (int64_t)nj * (e->L - l0 + 1);
    }
    return w;
}

static double spin_seed_log2(const orc_spin_rings* e, int j, double lb2, int pc, int ps) {
    double v = lb2;
    if (pc != 0) v += (double)pc * e->log2cos[j];
    if (ps != 0) v += (double)ps * e->log2sin[j];
    return v;
}

/* spin coefficient (l, m) of transform b in the (l+1, m+lmax+1) layout (src/Layout.jl:28-29) */
static size_t spin_idx(int l, int m, int L, int b) {
    return (size_t)l + (size_t)(L + 1) * (m + L) + (size_t)(L + 1) * (2 * L + 1) * b;
}

/* _spin_chunk! (src/Spin.jl:376-490) */
static void spin_chunk(int fwd, const orc_spin_rings* e, cplx* G, const cplx* almin, cplx* almout,
                       int m, int r0, int r1, double* d1, double* d0, cplx* acc) {
    const int L = e->L, B = e->B, off = L, nn = -e->s, nr = r1 - r0 + 1;
    int l0 = abs(m) > abs(nn) ? abs(m) : abs(nn);
    if (l0 > L) return;
    const int mi = m + L;
    const double lb2 = e->lb2[mi], sg = e->sg[mi];
    const int pc = e->pc[mi], ps = e->ps[mi];
    double E = -INFINITY;
    for (int j = r0; j <= r1; ++j) E = fmax(E, spin_seed_log2(e, j, lb2, pc, ps));
    E = isfinite(E) ? ceil(E) : 0.0;
    for (int k = 0; k < nr; ++k) {
        double v = spin_seed_log2(e, r0 + k, lb2, pc, ps);
        d1[k] = isfinite(v) ? sg * exp2(v - E) : 0.0;
        d0[k] = 0.0;
    }
    const size_t gs = (size_t)e->n * (2 * L + 1);
    for (int b = 0; b < B; ++b)
        for (int k = 0; k < nr; ++k)
            acc[k + (size_t)nr * b] = fwd ? c_make(0, 0) : G[(r0 + k) + (size_t)e->n * (m + off) + gs * b];
    /* touch at l0 */
    if (fwd) {
        for (int b = 0; b < B; ++b) {
            cplx a = c_scale(almin[spin_idx(l0, m, L, b)], e->Nl[l0]);
            if (a.re == 0 && a.im == 0) continue;
            for (int k = 0; k < nr; ++k) acc[k + (size_t)nr * b] = c_add(acc[k + (size_t)nr * b], c_scale(a, d1[k]));
        }
    } else {
        double f = exp2(E) * e->Nl[l0];
        for (int b = 0; b < B; ++b) {
            cplx s = c_make(0, 0);
            for (int k = 0; k < nr; ++k) s = c_add(s, c_scale(acc[k + (size_t)nr * b], d1[k]));
            cplx* t = &almout[spin_idx(l0, m, L, b)];
            *t = c_add(*t, c_scale(s, f));
        }
    }
    int steps = 0, Lc = l0;
    while (Lc < L) {
        int L1 = Lc + 1;
        double sm1 = sqrt(fmax(0.0, (double)(L1 * L1 - m * m)));
        double sn1 = sqrt(fmax(0.0, (double)(L1 * L1 - nn * nn)));
        double den = (double)Lc * sm1 * sn1;
        if (den <= 0) {
            for (int k = 0; k < nr; ++k) { d0[k] = d1[k]; d1[k] = 0.0; }
            Lc = L1;
            continue;
        }
        double sm0 = sqrt(fmax(0.0, (double)(Lc * Lc - m * m)));
        double sn0 = sqrt(fmax(0.0, (double)(Lc * Lc - nn * nn)));
        double a1 = (double)(2 * Lc + 1) * (double)Lc * (double)L1 / den;
        double a2 = (double)(2 * Lc + 1) * (double)m * (double)nn / den;
        double a0 = (double)L1 * sm0 * sn0 / den;
        for (int k = 0; k < nr; ++k) {
            double dn = (a1 * e->cos_t[r0 + k] - a2) * d1[k] - a0 * d0[k];
            d0[k] = d1[k];
            d1[k] = dn;
        }
        Lc = L1;
        if (fwd) {
            double N = e->Nl[Lc];
            for (int b = 0; b < B; ++b) {
                cplx a = c_scale(almin[spin_idx(Lc, m, L, b)], N);
                if (a.re == 0 && a.im == 0) continue;
                for (int k = 0; k < nr; ++k) acc[k + (size_t)nr * b] = c_add(acc[k + (size_t)nr * b], c_scale(a, d1[k]));
            }
        } else {
            double f = exp2(E) * e->Nl[Lc];
            for (int b = 0; b < B; ++b) {
                cplx s = c_make(0, 0);
                for (int k = 0; k < nr; ++k) s = c_add(s, c_scale(acc[k + (size_t)nr * b], d1[k]));
                cplx* t = &almout[spin_idx(Lc, m, L, b)];
                *t = c_add(*t, c_scale(s, f));
            }
        }
        if (++steps == RESCALE_STRIDE && Lc < L) {
            steps = 0;
            double mx = 0.0;
            for (int k = 0; k < nr; ++k) mx = fmax(mx, fmax(fabs(d1[k]), fabs(d0[k])));
            if (mx > 0 && isfinite(mx)) {
                double sh = ceil(log2(mx));
                if (sh != 0) {
                    double f = exp2(-sh);
                    for (int k = 0; k < nr; ++k) { d1[k] *= f; d0[k] *= f; }
                    if (fwd)
                        for (int q = 0; q < nr * B; ++q) acc[q] = c_scale(acc[q], f);
                    E += sh;
                }
            }
        }
    }
    if (fwd) {
        double f = exp2(E);
        for (int b = 0; b < B; ++b)
            for (int k = 0; k < nr; ++k) {
                cplx* t = &G[(r0 + k) + (size_t)e->n * (m + off) + gs * b];
                *t = c_add(*t, c_scale(acc[k + (size_t)nr * b], f));
            }
    }
}

static void spin_walk(int fwd, const orc_spin_rings* e, cplx* G, const cplx* almin, cplx* almout,
                      int nthreads) {
    int cw = 1;
    for (int c = 0; c < e->nchunks; ++c) cw = (e->chi[c] - e->clo[c] + 1) > cw ? (e->chi[c] - e->clo[c] + 1) : cw;
    int ns = nthreads_ok(nthreads);
#ifdef _OPENMP
#pragma omp parallel num_threads(ns > 0 ? ns : 1)
#endif
    {
        int t = 0, nt = 1;
#ifdef _OPENMP
        t = omp_get_thread_num();
        nt = omp_get_num_threads();
#endif
        double* d1 = (double*)malloc(sizeof(double) * cw);
        double* d0 = (double*)malloc(sizeof(double) * cw);
        cplx* acc = (cplx*)malloc(sizeof(cplx) * (size_t)cw * e->B);
        /* orders are independent: each touches its own G column and coefficients */
        for (int m = -e->L + t; m <= e->L; m += nt) {
            int lo = e->jlo[m + e->L], hi = e->jhi[m + e->L];
            if (hi < lo) continue;
            for (int c = 0; c < e->nchunks; ++c) {
                int r0 = e->clo[c] > lo ? e->clo[c] : lo;
                int r1 = e->chi[c] < hi ? e->chi[c] : hi;
                if (r1 < r0) continue;
                spin_chunk(fwd, e, G, almin, almout, m, r0, r1, d1, d0, acc);
            }
        }
        free(d1); free(d0); free(acc);
    }
}

/* spin_rings_from_alm! / spin_alm_from_rings! (src/Spin.jl:319-341) */
void orc_spin_rings_from_alm(const orc_spin_rings* e, const double* alm, double* G, int nthreads) {
    memset(G, 0, sizeof(double) * 2 * (size_t)e->n * (2 * e->L + 1) * e->B);
    spin_walk(1, e, (cplx*)G, (const cplx*)alm, NULL, nthreads);
}

void orc_spin_alm_from_rings(const orc_spin_rings* e, const double* G, double* alm, int nthreads) {
    memset(alm, 0, sizeof(double) * 2 * (size_t)(e->L + 1) * (2 * e->L + 1) * e->B);
    spin_walk(0, e, (cplx*)G, NULL, (cplx*)alm, nthreads);
}

/* SpinDirectLeaf (src/Spin.jl:557-630): sorted points, spin rings with eps = 0, phases */
typedef struct { double t; int64_t i; } th_idx;
static int cmp_th(const void* a, const void* b) {
    const th_idx* x = (const th_idx*)a; const th_idx* y = (const th_idx*)b;
    if (x->t < y->t) return -1;
    if (x->t > y->t) return 1;
    return x->i < y->i ? -1 : (x->i > y->i);
}

void orc_spin_direct(int fwd, const double* theta, const double* phi, int64_t M, int L, int spin,
                     int ntrans, const double* in, double* out, int nthreads) {
    th_idx* srt = (th_idx*)malloc(sizeof(th_idx) * M);
    for (int64_t i = 0; i < M; ++i) { srt[i].t = theta[i]; srt[i].i = i; }
    qsort(srt, M, sizeof(th_idx), cmp_th);
    double* ths = (double*)malloc(sizeof(double) * M);
    for (int64_t i = 0; i < M; ++i) ths[i] = srt[i].t;
    orc_spin_rings* e = orc_spin_rings_create(ths, (int)M, L, spin, 0.0, ntrans, 0);
    const int B = ntrans, off = L;
    const size_t gs = (size_t)M * (2 * L + 1);
    cplx* G = (cplx*)calloc(gs * B, sizeof(cplx));
    if (fwd) {
        orc_spin_rings_from_alm(e, in, (double*)G, nthreads);
        cplx* f = (cplx*)out;
        for (int b = 0; b < B; ++b)
            for (int64_t i = 0; i < M; ++i) {
                double ph0 = phi[srt[i].i];
                cplx acc = G[i + (size_t)M * off + gs * b];
                for (int m = 1; m <= L; ++m) {
                    cplx ph = c_cis((double)m * ph0);
                    acc = c_add(acc, c_add(c_mul(G[i + (size_t)M * (m + off) + gs * b], ph),
                                           c_mul(G[i + (size_t)M * (off - m) + gs * b], c_conj(ph))));
                }
                f[srt[i].i + (size_t)M * b] = acc;
            }
    } else {
        const cplx* f = (const cplx*)in;
        for (int b = 0; b < B; ++b)
            for (int64_t i = 0; i < M; ++i) {
                cplx fi = f[srt[i].i + (size_t)M * b];
                if (fi.re == 0 && fi.im == 0) continue;
                double ph0 = phi[srt[i].i];
                G[i + (size_t)M * off + gs * b] = fi;
                for (int m = 1; m <= L; ++m) {
                    cplx ph = c_cis((double)m * ph0);
                    G[i + (size_t)M * (m + off) + gs * b] = c_mul(fi, c_conj(ph));
                    G[i + (size_t)M * (off - m) + gs * b] = c_mul(fi, ph);
                }
            }
        orc_spin_alm_from_rings(e, (const double*)G, out, nthreads);
    }
    orc_spin_rings_destroy(e);
    free(G); free(ths); free(srt);
}
