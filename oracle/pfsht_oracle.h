/*
 * pfsht_oracle.h -- CPU restatement of PartialFSHT.jl's partial-sky SHT apply.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the parity oracle and the timed CPU baseline.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load it, and only as the
 * checker; the product library (libpfsht_b200) never links, loads or calls it.
 *
 * Every routine restates the reference's algorithm in plain C (double precision,
 * compiled with -ffp-contract=off so no multiply-add is fused that the reference keeps
 * separate). Citations are path:line inside the PartialFSHT.jl source tree.
 *
 * Layout conventions (all column-major, as in Julia):
 *   alm  : (L+1) x (2L+1) x B complex, sph_mode packing (src/Layout.jl:13-20);
 *          0-based column of order m is 2m for m>=0 and 2|m|-1 for m<0, row is l-|m|.
 *   G    : (nrings) x (2L+1) x B complex, column m+L for order m (src/Legendre.jl:306).
 *   f    : (M) x B complex.
 * Complex numbers are interleaved (re, im) doubles.
 */
#ifndef PFSHT_ORACLE_H
#define PFSHT_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- sizes (src/Stretch.jl:52-81) ---- */
int64_t orc_next_smooth(int64_t n);
int64_t orc_next_smooth_even(int64_t n);

/* ---- Legendre (src/Legendre.jl) ---- */
double orc_polar_pad_factor(void);
int orc_polar_mmax(double theta, int lmax, double eps);
void orc_sectorial_log2c(int lmax, double* out /* L+1 */);
/* returns 0 on success, -1 if mlim is not unimodal; jlo/jhi are 0-based, inclusive, sized L+1 */
int orc_nested_ranges(const int* mlim, int n, int lmax, int* jlo, int* jhi);
int64_t orc_retained_triples(const int* mlim, int n, int lmax);
double orc_alf(int l, int m, double theta);

typedef struct orc_rings orc_rings;
/* RingLegendre (src/Legendre.jl:194-255). theta must be ascending. */
orc_rings* orc_rings_create(const double* theta, int n, int lmax, double eps, int ntrans,
                            int reflect);
void orc_rings_destroy(orc_rings*);
int orc_rings_n(const orc_rings*);
int orc_rings_mmax(const orc_rings*);
int64_t orc_rings_work(const orc_rings*);
int orc_rings_nchunks(const orc_rings*);
void orc_rings_tables(const orc_rings*, int* mlim, int* jlo, int* jhi, int* chunk_lo,
                      int* chunk_hi, double* cos_theta, double* log2sin, double* log2c);
/* rings_from_alm! / alm_from_rings! (src/Legendre.jl:310-341); nthreads<=1 is the serial
 * walk, >1 the interleaved-order threaded walk of ext/PartialFSHTOhMyThreadsExt.jl:31-42 */
void orc_rings_from_alm(const orc_rings*, const double* alm, double* G, int nthreads);
void orc_alm_from_rings(const orc_rings*, const double* G, double* alm, int nthreads);

/* ---- geometry and window (src/Windows.jl) ---- */
enum { ORC_POLE = 0, ORC_INTERIOR = 1, ORC_FULL = 2 };
typedef struct {
    int kind, lmax;
    double eps, beta, h, theta_lo, theta_hi, eps_apo, period;
    int64_t K;
    double Theta1, sigma, ThetaT, invZ;
} orc_geom;
double orc_es_beta(double eps);
double orc_es_cdf(double beta, double u);
/* 1 if admissible (filled), 0 if no periodisation is admissible, -1 on bad arguments */
int orc_try_stretch_geometry(double lo, double hi, int lmax, double eps, double eps_apo_max,
                             orc_geom* out);
double orc_stretch_window(const orc_geom*, double Theta);
double orc_stretch_to_theta(const orc_geom*, double Theta);
double orc_theta_to_stretch(const orc_geom*, double theta);
void orc_stretch_rings(const orc_geom*, int n, double* theta, double* Theta);

/* ---- DFS (src/DFS.jl:13-56) ---- */
void orc_dfs_double(const double* F, double* Ft, int Nth, int Nph, int B, int spin);
void orc_dfs_fold(double* F, const double* Ft, int Nth, int Nph, int B, int spin);

/* ---- FFT (own mixed-radix; FFTW's role in src/Stretch.jl:222-225) ---- */
/* sign -1: X_k = sum x_j e^{-2 pi i jk/n}; sign +1: unnormalised inverse (bfft) */
void orc_fft_cols(double* a, int n1, int n2, int sign, int nthreads);   /* along dim 1 */
void orc_fft_rows(double* a, int n1, int n2, int sign, int nthreads);   /* along dim 2 */

/* ---- NUFFT (src/NUFFT.jl) ---- */
int orc_mode_k(int i0 /* 0-based */, int n, int modeord);
/* DirectSum (src/NUFFT.jl:85-129): exact O(M n1 n2); modes in FFT order (modeord=1) */
void orc_nufft_direct(int type, int n1, int n2, int iflag, int ntrans, const double* x,
                      const double* y, int64_t M, const double* in, double* out);
/* ES-kernel NUFFT (the published FINUFFT algorithm: exponential-of-semicircle kernel,
 * width w = ceil(log10(10/tol)), beta = 2.30 w, upsampling 2; the kernel evaluated exactly
 * or, as FINUFFT does by default, by a per-tap polynomial of degree w + 2) */
typedef struct orc_esnufft orc_esnufft;
enum { ORC_KER_EXACT = 0, ORC_KER_POLY = 1 };
orc_esnufft* orc_esnufft_create(int n1, int n2, int ntrans, double tol, const double* x,
                                const double* y, int64_t M);  /* polynomial kernel */
orc_esnufft* orc_esnufft_create_k(int n1, int n2, int ntrans, double tol, const double* x,
                                  const double* y, int64_t M, int kermode);
void orc_esnufft_destroy(orc_esnufft*);
void orc_esnufft_params(const orc_esnufft*, int* w, double* beta, int* nf1, int* nf2);
int orc_esnufft_set_grid(orc_esnufft*, int nf1, int nf2);  /* 0 = ok, 1 = lengths too short */
void orc_esnufft_exec(orc_esnufft*, int type, int iflag, const double* in, double* out,
                      int nthreads);
double orc_es_kernel(double z, double beta);
/* deconvolution 1/Phi(k) for the grid of nf cells (k signed) */
double orc_es_deconv(int k, int nf, int w, double beta);

/* ---- Direct leaf (src/Direct.jl) ---- */
typedef struct orc_direct orc_direct;
orc_direct* orc_direct_create(const double* theta, const double* phi, int64_t M, int lmax,
                              int ntrans);
void orc_direct_destroy(orc_direct*);
void orc_direct_forward(orc_direct*, const double* alm, double* f, int nthreads);
void orc_direct_adjoint(orc_direct*, const double* f, double* alm, int nthreads);

/* ---- stretched leaf (src/Stretch.jl) ---- */
enum { ORC_NUFFT_DIRECT = 0, ORC_NUFFT_ES = 1, ORC_NUFFT_ES_EXACT = 2 };
typedef struct orc_stretch orc_stretch;
typedef struct {
    int kind, flip, lmax, ntrans, nth_half, nth, nph, mmax, nrings;
    int64_t K, ring_work, M;
    double eps, beta, h, theta_lo, theta_hi, eps_apo, Theta1, sigma, ThetaT;
    double box_lo, box_hi;
} orc_stretch_info;
/* returns NULL with *status = 1 for a refused geometry, 2 for bad arguments */
orc_stretch* orc_stretch_create(const double* theta, const double* phi, int64_t M, int lmax,
                                int ntrans, double tol, int nufft_kind, double eps_apo_max,
                                double oversample_theta, double oversample_phi, int* status);
orc_stretch* orc_stretch_create_spin(const double* theta, const double* phi, int64_t M, int lmax,
                                     int ntrans, double tol, int nufft_kind, double eps_apo_max,
                                     double oversample_theta, double oversample_phi, int spin,
                                     int* status);
void orc_stretch_destroy(orc_stretch*);
void orc_stretch_info_get(const orc_stretch*, orc_stretch_info*);
int orc_stretch_set_nufft_grid(orc_stretch*, int nf1, int nf2);  /* ES NUFFT leaves only */
void orc_stretch_tables(const orc_stretch*, double* theta_rings, double* Theta_rings,
                        double* window, double* Theta_pts, double* phi_pts);
void orc_stretch_forward(orc_stretch*, const double* alm, double* f, int nthreads);
void orc_stretch_adjoint(orc_stretch*, const double* f, double* alm, int nthreads);
/* the ring engine of the leaf (for stage-level parity) */
const orc_rings* orc_stretch_rings_engine(const orc_stretch*);


/* spin-weighted transforms (src/Spin.jl) */
double orc_wigner_d(int l, int m, int n, double beta);
typedef struct orc_spin_rings orc_spin_rings;
orc_spin_rings* orc_spin_rings_create(const double* theta, int n, int lmax, int spin, double eps,
                                      int ntrans, int reflect);
void orc_spin_rings_destroy(orc_spin_rings*);
int orc_spin_rings_mmax(const orc_spin_rings*);
int orc_spin_rings_nchunks(const orc_spin_rings*);
int64_t orc_spin_rings_work(const orc_spin_rings*);
void orc_spin_rings_from_alm(const orc_spin_rings*, const double* alm, double* G, int nthreads);
void orc_spin_alm_from_rings(const orc_spin_rings*, const double* G, double* alm, int nthreads);
/* SpinDirectLeaf: fwd 1: alm -> f; fwd 0: f -> alm (spin layout (l+1, m+lmax+1)) */
void orc_spin_direct(int fwd, const double* theta, const double* phi, int64_t M, int lmax, int spin,
                     int ntrans, const double* in, double* out, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
