"""ctypes front end of the CPU oracle (liboracle_pfsht.so).

TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline. Only tests/,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may import this module; the product
package never does.

Arrays follow the reference's column-major layout: a coefficient array is a complex128
numpy array of shape ``(lmax+1, 2lmax+1, B)`` in Fortran order (``sph_mode`` packing,
src/Layout.jl:13-20), a ring array ``(nrings, 2lmax+1, B)``, a field ``(M, B)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_pfsht.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle with its Makefile; returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class _Geom(C.Structure):
    _fields_ = [("kind", C.c_int), ("lmax", C.c_int), ("eps", C.c_double),
                ("beta", C.c_double), ("h", C.c_double), ("theta_lo", C.c_double),
                ("theta_hi", C.c_double), ("eps_apo", C.c_double), ("period", C.c_double),
                ("K", C.c_int64), ("Theta1", C.c_double), ("sigma", C.c_double),
                ("ThetaT", C.c_double), ("invZ", C.c_double)]


class _StretchInfo(C.Structure):
    _fields_ = [("kind", C.c_int), ("flip", C.c_int), ("lmax", C.c_int), ("ntrans", C.c_int),
                ("nth_half", C.c_int), ("nth", C.c_int), ("nph", C.c_int), ("mmax", C.c_int),
                ("nrings", C.c_int), ("K", C.c_int64), ("ring_work", C.c_int64),
                ("M", C.c_int64), ("eps", C.c_double), ("beta", C.c_double),
                ("h", C.c_double), ("theta_lo", C.c_double), ("theta_hi", C.c_double),
                ("eps_apo", C.c_double), ("Theta1", C.c_double), ("sigma", C.c_double),
                ("ThetaT", C.c_double), ("box_lo", C.c_double), ("box_hi", C.c_double)]


KINDS = {0: "pole", 1: "interior", 2: "full"}


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    vp = C.c_void_p
    sig = {
        "orc_next_smooth": (C.c_int64, [C.c_int64]),
        "orc_next_smooth_even": (C.c_int64, [C.c_int64]),
        "orc_polar_pad_factor": (C.c_double, []),
        "orc_polar_mmax": (C.c_int, [C.c_double, C.c_int, C.c_double]),
        "orc_sectorial_log2c": (None, [C.c_int, _dp]),
        "orc_nested_ranges": (C.c_int, [_ip, C.c_int, C.c_int, _ip, _ip]),
        "orc_retained_triples": (C.c_int64, [_ip, C.c_int, C.c_int]),
        "orc_alf": (C.c_double, [C.c_int, C.c_int, C.c_double]),
        "orc_rings_create": (vp, [_dp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int]),
        "orc_rings_destroy": (None, [vp]),
        "orc_rings_n": (C.c_int, [vp]),
        "orc_rings_mmax": (C.c_int, [vp]),
        "orc_rings_work": (C.c_int64, [vp]),
        "orc_rings_nchunks": (C.c_int, [vp]),
        "orc_rings_tables": (None, [vp, _ip, _ip, _ip, _ip, _ip, _dp, _dp, _dp]),
        "orc_rings_from_alm": (None, [vp, vp, vp, C.c_int]),
        "orc_alm_from_rings": (None, [vp, vp, vp, C.c_int]),
        "orc_es_beta": (C.c_double, [C.c_double]),
        "orc_es_cdf": (C.c_double, [C.c_double, C.c_double]),
        "orc_try_stretch_geometry": (C.c_int, [C.c_double, C.c_double, C.c_int, C.c_double,
                                               C.c_double, C.POINTER(_Geom)]),
        "orc_stretch_window": (C.c_double, [C.POINTER(_Geom), C.c_double]),
        "orc_stretch_to_theta": (C.c_double, [C.POINTER(_Geom), C.c_double]),
        "orc_theta_to_stretch": (C.c_double, [C.POINTER(_Geom), C.c_double]),
        "orc_stretch_rings": (None, [C.POINTER(_Geom), C.c_int, _dp, _dp]),
        "orc_dfs_double": (None, [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int]),
        "orc_dfs_fold": (None, [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int]),
        "orc_fft_cols": (None, [vp, C.c_int, C.c_int, C.c_int, C.c_int]),
        "orc_fft_rows": (None, [vp, C.c_int, C.c_int, C.c_int, C.c_int]),
        "orc_mode_k": (C.c_int, [C.c_int, C.c_int, C.c_int]),
        "orc_nufft_direct": (None, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp,
                                    C.c_int64, vp, vp]),
        "orc_esnufft_create": (vp, [C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, C.c_int64]),
        "orc_esnufft_create_k": (vp, [C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, C.c_int64,
                                      C.c_int]),
        "orc_esnufft_destroy": (None, [vp]),
        "orc_esnufft_params": (None, [vp, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                      C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "orc_esnufft_exec": (None, [vp, C.c_int, C.c_int, vp, vp, C.c_int]),
        "orc_esnufft_set_grid": (C.c_int, [vp, C.c_int, C.c_int]),
        "orc_stretch_set_nufft_grid": (C.c_int, [vp, C.c_int, C.c_int]),
        "orc_es_kernel": (C.c_double, [C.c_double, C.c_double]),
        "orc_es_deconv": (C.c_double, [C.c_int, C.c_int, C.c_int, C.c_double]),
        "orc_direct_create": (vp, [_dp, _dp, C.c_int64, C.c_int, C.c_int]),
        "orc_direct_destroy": (None, [vp]),
        "orc_direct_forward": (None, [vp, vp, vp, C.c_int]),
        "orc_direct_adjoint": (None, [vp, vp, vp, C.c_int]),
        "orc_stretch_create": (vp, [_dp, _dp, C.c_int64, C.c_int, C.c_int, C.c_double, C.c_int,
                                    C.c_double, C.c_double, C.c_double, C.POINTER(C.c_int)]),
        "orc_stretch_create_spin": (vp, [_dp, _dp, C.c_int64, C.c_int, C.c_int, C.c_double, C.c_int,
                                         C.c_double, C.c_double, C.c_double, C.c_int,
                                         C.POINTER(C.c_int)]),
        "orc_wigner_d": (C.c_double, [C.c_int, C.c_int, C.c_int, C.c_double]),
        "orc_spin_rings_create": (vp, [_dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int]),
        "orc_spin_rings_destroy": (None, [vp]),
        "orc_spin_rings_mmax": (C.c_int, [vp]),
        "orc_spin_rings_nchunks": (C.c_int, [vp]),
        "orc_spin_rings_work": (C.c_int64, [vp]),
        "orc_spin_rings_from_alm": (None, [vp, vp, vp, C.c_int]),
        "orc_spin_alm_from_rings": (None, [vp, vp, vp, C.c_int]),
        "orc_spin_direct": (None, [C.c_int, _dp, _dp, C.c_int64, C.c_int, C.c_int, C.c_int, vp, vp,
                                   C.c_int]),
        "orc_stretch_destroy": (None, [vp]),
        "orc_stretch_info_get": (None, [vp, C.POINTER(_StretchInfo)]),
        "orc_stretch_tables": (None, [vp, _dp, _dp, _dp, _dp, _dp]),
        "orc_stretch_forward": (None, [vp, vp, vp, C.c_int]),
        "orc_stretch_adjoint": (None, [vp, vp, vp, C.c_int]),
        "orc_stretch_rings_engine": (vp, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


# ---------------------------------------------------------------------------------------
# layout helpers (src/Layout.jl)
# ---------------------------------------------------------------------------------------
def coeff_size(lmax: int):
    return (lmax + 1, 2 * lmax + 1)


def sph_mode(l: int, m: int):
    """0-based (row, col) of (l, m) in the (lmax+1, 2lmax+1) array (src/Layout.jl:20)."""
    am = abs(m)
    return (l - am, 2 * am if m >= 0 else 2 * am - 1)


def zeros_alm(lmax: int, ntrans: int = 1) -> np.ndarray:
    return np.zeros((lmax + 1, 2 * lmax + 1, ntrans), dtype=np.complex128, order="F")


def valid_mask(lmax: int) -> np.ndarray:
    """Boolean (lmax+1, 2lmax+1) mask of the slots that hold a real mode."""
    mask = np.zeros(coeff_size(lmax), dtype=bool)
    for m in range(-lmax, lmax + 1):
        _, c = sph_mode(abs(m), m)
        mask[0: lmax + 1 - abs(m), c] = True
    return mask


def rand_alm(lmax: int, ntrans: int = 1, rng=None, weight=None) -> np.ndarray:
    """Complex N(0,1) in every valid mode, padding zero (test/runtests.jl:24-36).
    ``weight(l)`` optionally scales degree l."""
    rng = np.random.default_rng(0) if rng is None else rng
    a = zeros_alm(lmax, ntrans)
    mask = valid_mask(lmax)
    n = int(mask.sum())
    ls = np.zeros(coeff_size(lmax), dtype=np.float64)
    for c in range(2 * lmax + 1):
        am = (c + 1) // 2
        ls[:, c] = np.arange(lmax + 1) + am
    for b in range(ntrans):
        v = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        blk = np.zeros(coeff_size(lmax), dtype=np.complex128)
        blk[mask] = v
        if weight is not None:
            blk = blk * np.where(mask, weight(ls), 0.0)
        a[:, :, b] = blk
    return a


def alm_reldiff(a, b, lmax: int) -> float:
    """Max relative difference over valid modes (test/runtests.jl:39-48)."""
    mask = valid_mask(lmax)
    a = np.asarray(a)
    b = np.asarray(b)
    if a.ndim == 2:
        a = a[:, :, None]
        b = b[:, :, None]
    num = np.abs(a - b)[mask].max()
    den = np.abs(b)[mask].max()
    return float(num / max(den, np.finfo(float).eps))


def _as3(a, shape2):
    a = np.asarray(a, dtype=np.complex128)
    if a.ndim == 2:
        a = a[:, :, None]
    return np.asfortranarray(a)


# ---------------------------------------------------------------------------------------
# scalar functions
# ---------------------------------------------------------------------------------------
def next_smooth(n):
    return int(lib().orc_next_smooth(int(n)))


def next_smooth_even(n):
    return int(lib().orc_next_smooth_even(int(n)))


def polar_mmax(theta, lmax, eps):
    return int(lib().orc_polar_mmax(float(theta), int(lmax), float(eps)))


def alf(l, m, theta):
    return float(lib().orc_alf(int(l), int(m), float(theta)))


def ylm(l, m, theta, phi):
    return alf(l, m, theta) * np.exp(1j * m * phi)


def sectorial_log2c(lmax):
    v = np.zeros(lmax + 1)
    lib().orc_sectorial_log2c(int(lmax), v)
    return v


def nested_ranges(mlim, lmax):
    mlim = np.ascontiguousarray(mlim, dtype=np.int32)
    jlo = np.zeros(lmax + 1, np.int32)
    jhi = np.zeros(lmax + 1, np.int32)
    rc = lib().orc_nested_ranges(mlim, len(mlim), int(lmax), jlo, jhi)
    if rc != 0:
        raise ValueError("retained-order limits are not unimodal in colatitude")
    return jlo, jhi


def retained_triples(mlim, lmax):
    mlim = np.ascontiguousarray(mlim, dtype=np.int32)
    return int(lib().orc_retained_triples(mlim, len(mlim), int(lmax)))


def counted_ring_work(theta_rings, lmax, tol):
    """counted_ring_work (src/Cost.jl:88-99)."""
    mlim = [polar_mmax(t, lmax, tol) for t in theta_rings]
    return retained_triples(mlim, lmax), max(mlim)


def es_beta(eps):
    return float(lib().orc_es_beta(float(eps)))


def es_cdf(beta, u):
    return float(lib().orc_es_cdf(float(beta), float(u)))


def es_kernel(z, beta):
    return float(lib().orc_es_kernel(float(z), float(beta)))


def es_deconv(k, nf, w, beta):
    return float(lib().orc_es_deconv(int(k), int(nf), int(w), float(beta)))


class Geometry:
    """StretchGeometry (src/Windows.jl:42-57)."""

    def __init__(self, g: _Geom):
        self._g = g
        self.kind = KINDS[g.kind]
        for name, _ in _Geom._fields_:
            if name != "kind":
                setattr(self, name, getattr(g, name))

    def window(self, Th):
        return float(lib().orc_stretch_window(C.byref(self._g), float(Th)))

    def to_theta(self, Th):
        return float(lib().orc_stretch_to_theta(C.byref(self._g), float(Th)))

    def to_stretch(self, th):
        return float(lib().orc_theta_to_stretch(C.byref(self._g), float(th)))

    def rings(self, n):
        th = np.zeros(n)
        Th = np.zeros(n)
        lib().orc_stretch_rings(C.byref(self._g), int(n), th, Th)
        return th, Th


def try_stretch_geometry(lo, hi, lmax, eps, eps_apo_max=1.0):
    g = _Geom()
    rc = lib().orc_try_stretch_geometry(float(lo), float(hi), int(lmax), float(eps),
                                        float(eps_apo_max), C.byref(g))
    if rc < 0:
        raise ValueError("bad colatitude interval")
    return Geometry(g) if rc == 1 else None


def stretch_geometry(lo, hi, lmax, eps, eps_apo_max=1.0):
    g = try_stretch_geometry(lo, hi, lmax, eps, eps_apo_max)
    if g is None:
        raise ValueError("stretched transform is degenerate for this interval, lmax and tol")
    return g


# ---------------------------------------------------------------------------------------
# ring engine
# ---------------------------------------------------------------------------------------
class Rings:
    """RingLegendre (src/Legendre.jl:174-255) with rings_from_alm! / alm_from_rings!."""

    def __init__(self, theta, lmax, eps, ntrans=1, reflect=False):
        self.theta = _f64(theta)
        self.lmax = int(lmax)
        self.ntrans = int(ntrans)
        self._h = lib().orc_rings_create(self.theta, len(self.theta), self.lmax, float(eps),
                                         self.ntrans, int(bool(reflect)))
        if not self._h:
            raise ValueError("ring colatitudes must be sorted ascending")
        self._own = True

    @classmethod
    def _borrow(cls, handle, lmax, ntrans):
        obj = cls.__new__(cls)
        obj._h = handle
        obj.lmax = lmax
        obj.ntrans = ntrans
        obj._own = False
        return obj

    def __del__(self):
        if getattr(self, "_own", False) and self._h:
            lib().orc_rings_destroy(self._h)
            self._h = None

    @property
    def n(self):
        return int(lib().orc_rings_n(self._h))

    @property
    def mmax(self):
        return int(lib().orc_rings_mmax(self._h))

    def work(self):
        return int(lib().orc_rings_work(self._h))

    def tables(self):
        n, L = self.n, self.lmax
        nc = int(lib().orc_rings_nchunks(self._h))
        mlim = np.zeros(n, np.int32)
        jlo = np.zeros(L + 1, np.int32)
        jhi = np.zeros(L + 1, np.int32)
        clo = np.zeros(max(nc, 1), np.int32)
        chi = np.zeros(max(nc, 1), np.int32)
        cs = np.zeros(n)
        l2s = np.zeros(n)
        l2c = np.zeros(L + 1)
        lib().orc_rings_tables(self._h, mlim, jlo, jhi, clo, chi, cs, l2s, l2c)
        return dict(mlim=mlim, jlo=jlo, jhi=jhi, chunks=list(zip(clo[:nc], chi[:nc])),
                    cos_theta=cs, log2sin=l2s, log2c=l2c)

    def rings_from_alm(self, alm, nthreads=1):
        alm = _as3(alm, None)
        assert alm.shape == (self.lmax + 1, 2 * self.lmax + 1, self.ntrans)
        G = np.zeros((self.n, 2 * self.lmax + 1, self.ntrans), np.complex128, order="F")
        lib().orc_rings_from_alm(self._h, _ptr(alm), _ptr(G), int(nthreads))
        return G

    def alm_from_rings(self, G, nthreads=1):
        G = _as3(G, None)
        assert G.shape == (self.n, 2 * self.lmax + 1, self.ntrans)
        alm = zeros_alm(self.lmax, self.ntrans)
        lib().orc_alm_from_rings(self._h, _ptr(G), _ptr(alm), int(nthreads))
        return alm


# ---------------------------------------------------------------------------------------
# DFS, FFT, NUFFT
# ---------------------------------------------------------------------------------------
def dfs_double(F, spin=0):
    F = _as3(F, None)
    nt, nph, B = F.shape
    Ft = np.zeros((2 * nt, nph, B), np.complex128, order="F")
    lib().orc_dfs_double(_ptr(F), _ptr(Ft), nt, nph, B, int(spin))
    return Ft


def dfs_fold(Ft, spin=0):
    Ft = _as3(Ft, None)
    n2, nph, B = Ft.shape
    F = np.zeros((n2 // 2, nph, B), np.complex128, order="F")
    lib().orc_dfs_fold(_ptr(F), _ptr(Ft), n2 // 2, nph, B, int(spin))
    return F


def fft_cols(a, sign, nthreads=1):
    a = np.asfortranarray(np.array(a, dtype=np.complex128))
    lib().orc_fft_cols(_ptr(a), a.shape[0], a.shape[1], int(sign), int(nthreads))
    return a


def fft_rows(a, sign, nthreads=1):
    a = np.asfortranarray(np.array(a, dtype=np.complex128))
    lib().orc_fft_rows(_ptr(a), a.shape[0], a.shape[1], int(sign), int(nthreads))
    return a


def mode_k(i0, n, modeord=1):
    return int(lib().orc_mode_k(int(i0), int(n), int(modeord)))


def nufft_direct(typ, n1, n2, iflag, x, y, inp):
    """DirectSum NUFFT (src/NUFFT.jl:85-129). type 2: modes (n1,n2,B) -> (M,B);
    type 1: (M,B) -> (n1,n2,B)."""
    x = _f64(x)
    y = _f64(y)
    M = len(x)
    inp = np.asfortranarray(np.asarray(inp, dtype=np.complex128))
    if typ == 2:
        if inp.ndim == 2:
            inp = inp[:, :, None]
        B = inp.shape[2]
        out = np.zeros((M, B), np.complex128, order="F")
    else:
        if inp.ndim == 1:
            inp = inp[:, None]
        B = inp.shape[1]
        out = np.zeros((n1, n2, B), np.complex128, order="F")
    inp = np.asfortranarray(inp)
    lib().orc_nufft_direct(int(typ), int(n1), int(n2), int(iflag), int(B), x, y, M,
                           _ptr(inp), _ptr(out))
    return out


class ESNufft:
    """CPU ES-kernel NUFFT (published FINUFFT algorithm)."""

    def __init__(self, n1, n2, x, y, tol, ntrans=1, kernel="poly", grid=None):
        self.x = _f64(x)
        self.y = _f64(y)
        self.n1, self.n2, self.B = int(n1), int(n2), int(ntrans)
        self._h = lib().orc_esnufft_create_k(self.n1, self.n2, self.B, float(tol), self.x,
                                             self.y, len(self.x), 1 if kernel == "poly" else 0)
        if grid is not None and lib().orc_esnufft_set_grid(self._h, int(grid[0]), int(grid[1])):
            raise ValueError("fine-grid lengths below the minimum")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_esnufft_destroy(self._h)
            self._h = None

    def params(self):
        w = C.c_int()
        beta = C.c_double()
        nf1 = C.c_int()
        nf2 = C.c_int()
        lib().orc_esnufft_params(self._h, C.byref(w), C.byref(beta), C.byref(nf1), C.byref(nf2))
        return dict(w=w.value, beta=beta.value, nf1=nf1.value, nf2=nf2.value)

    def exec(self, typ, iflag, inp, nthreads=1):
        M = len(self.x)
        inp = np.asarray(inp, dtype=np.complex128)
        if typ == 2:
            if inp.ndim == 2:
                inp = inp[:, :, None]
            out = np.zeros((M, self.B), np.complex128, order="F")
        else:
            if inp.ndim == 1:
                inp = inp[:, None]
            out = np.zeros((self.n1, self.n2, self.B), np.complex128, order="F")
        inp = np.asfortranarray(inp)
        lib().orc_esnufft_exec(self._h, int(typ), int(iflag), _ptr(inp), _ptr(out), int(nthreads))
        return out


# ---------------------------------------------------------------------------------------
# leaves
# ---------------------------------------------------------------------------------------
class Direct:
    """DirectLeaf (src/Direct.jl): the O(M L^2) oracle."""

    def __init__(self, theta, phi, lmax, ntrans=1):
        self.theta = _f64(theta)
        self.phi = _f64(phi)
        self.lmax, self.ntrans, self.M = int(lmax), int(ntrans), len(self.theta)
        self._h = lib().orc_direct_create(self.theta, self.phi, self.M, self.lmax, self.ntrans)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_direct_destroy(self._h)
            self._h = None

    def forward(self, alm, nthreads=1):
        alm = _as3(alm, None)
        f = np.zeros((self.M, self.ntrans), np.complex128, order="F")
        lib().orc_direct_forward(self._h, _ptr(alm), _ptr(f), int(nthreads))
        return f

    def adjoint(self, f, nthreads=1):
        f = np.asfortranarray(np.asarray(f, dtype=np.complex128).reshape(self.M, self.ntrans, order="F"))
        alm = zeros_alm(self.lmax, self.ntrans)
        lib().orc_direct_adjoint(self._h, _ptr(f), _ptr(alm), int(nthreads))
        return alm


class RefusedGeometry(ValueError):
    pass


class Stretch:
    """StretchLeaf (src/Stretch.jl:94-295) with DirectSum (exact, nufft="direct"), the ES
    NUFFT with FINUFFT's polynomial kernel evaluation (nufft="es") or with the exact kernel
    (nufft="es_exact"). nufft_grid = (nf1, nf2) sets the ES NUFFT's fine-grid lengths (default:
    the minimum 2,3,5-smooth lengths), e.g. to those of a device plan."""

    def __init__(self, theta, phi, lmax, tol, ntrans=1, nufft="es", eps_apo_max=1.0,
                 oversample_theta=1.0, oversample_phi=1.0, nufft_grid=None, spin=0):
        self.theta = _f64(theta)
        self.phi = _f64(phi)
        self.M = len(self.theta)
        self.spin = int(spin)
        st = C.c_int(0)
        kind = {"direct": 0, "es": 1, "es_exact": 2}[nufft]
        self._h = lib().orc_stretch_create_spin(self.theta, self.phi, self.M, int(lmax), int(ntrans),
                                                float(tol), kind, float(eps_apo_max),
                                                float(oversample_theta), float(oversample_phi),
                                                self.spin, C.byref(st))
        if not self._h:
            if st.value == 1:
                raise RefusedGeometry("stretched transform is degenerate at this lmax and tol")
            raise ValueError("bad arguments")
        if nufft_grid is not None and lib().orc_stretch_set_nufft_grid(
                self._h, int(nufft_grid[0]), int(nufft_grid[1])):
            raise ValueError("nufft_grid needs an ES NUFFT and lengths >= the minimum")
        i = _StretchInfo()
        lib().orc_stretch_info_get(self._h, C.byref(i))
        self.info = {name: getattr(i, name) for name, _ in _StretchInfo._fields_}
        self.info["kind"] = KINDS[i.kind]
        self.lmax, self.ntrans = int(lmax), int(ntrans)
        self.rings = (Rings._borrow(lib().orc_stretch_rings_engine(self._h), self.lmax, self.ntrans)
                      if self.spin == 0 else None)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_stretch_destroy(self._h)
            self._h = None

    def tables(self):
        n = self.info["nth_half"]
        th = np.zeros(n)
        Th = np.zeros(n)
        w = np.zeros(n)
        Tp = np.zeros(self.M)
        pp = np.zeros(self.M)
        lib().orc_stretch_tables(self._h, th, Th, w, Tp, pp)
        return dict(theta_rings=th, Theta_rings=Th, window=w, Theta_pts=Tp, phi_pts=pp)

    def ring_work(self):
        return int(self.info["ring_work"])

    def forward(self, alm, nthreads=1):
        alm = _as3(alm, None)
        f = np.zeros((self.M, self.ntrans), np.complex128, order="F")
        lib().orc_stretch_forward(self._h, _ptr(alm), _ptr(f), int(nthreads))
        return f

    def adjoint(self, f, nthreads=1):
        f = np.asfortranarray(np.asarray(f, dtype=np.complex128).reshape(self.M, self.ntrans, order="F"))
        alm = zeros_alm(self.lmax, self.ntrans)
        lib().orc_stretch_adjoint(self._h, _ptr(f), _ptr(alm), int(nthreads))
        return alm


def cdot(a, b) -> complex:
    """Julia's dot(a, b) = sum(conj(a) .* b)."""
    return complex(np.vdot(np.ravel(a, order="F"), np.ravel(b, order="F")))


# ---------------------------------------------------------------------------------------
# spin-weighted transforms (src/Spin.jl); coefficients in the (l+1, m+lmax+1) layout
# ---------------------------------------------------------------------------------------
def wigner_d(l, m, n, beta):
    """wigner_d (src/Spin.jl:58-131)."""
    return float(lib().orc_wigner_d(int(l), int(m), int(n), float(beta)))


def sylm(s, l, m, theta, phi):
    """sYlm (src/Spin.jl:138-142): N_l d^l_{m,-s}(theta) e^{i m phi}."""
    if abs(s) > l:
        return 0j
    return np.sqrt((2 * l + 1) / (4 * np.pi)) * wigner_d(l, m, -s, theta) * np.exp(1j * m * phi)


def spin_coeff_index(l, m, lmax):
    """spin_coeff_index (src/Layout.jl:28-29), 0-based (row, column)."""
    return l, m + lmax


def spin_valid_mask(lmax, spin):
    """Slots holding a spin-s mode: |m| <= l and l >= |s|."""
    l = np.arange(lmax + 1)[:, None]
    m = np.arange(-lmax, lmax + 1)[None, :]
    return (np.abs(m) <= l) & (l >= abs(spin))


def rand_spin_alm(lmax, spin, ntrans=1, rng=None):
    rng = np.random.default_rng(0) if rng is None else rng
    a = np.zeros((lmax + 1, 2 * lmax + 1, ntrans), np.complex128, order="F")
    mask = spin_valid_mask(lmax, spin)
    for b in range(ntrans):
        a[:, :, b][mask] = rng.standard_normal(mask.sum()) + 1j * rng.standard_normal(mask.sum())
    return a


class SpinRings:
    """SpinRings (src/Spin.jl:175-280) on ascending ring colatitudes."""

    def __init__(self, theta_rings, lmax, spin, eps, ntrans=1, reflect=False):
        self.theta = np.ascontiguousarray(theta_rings, dtype=np.float64)
        self.lmax, self.spin, self.ntrans = int(lmax), int(spin), int(ntrans)
        self._h = lib().orc_spin_rings_create(self.theta, len(self.theta), self.lmax, self.spin,
                                              float(eps), self.ntrans, 1 if reflect else 0)
        if not self._h:
            raise ValueError("ring colatitudes must be ascending and unimodal in their limits")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_spin_rings_destroy(self._h)
            self._h = None

    @property
    def mmax(self):
        return int(lib().orc_spin_rings_mmax(self._h))

    @property
    def nchunks(self):
        return int(lib().orc_spin_rings_nchunks(self._h))

    def ring_work(self):
        return int(lib().orc_spin_rings_work(self._h))

    def rings_from_alm(self, alm, nthreads=1):
        alm = _as3(alm, None)
        G = np.zeros((len(self.theta), 2 * self.lmax + 1, self.ntrans), np.complex128, order="F")
        lib().orc_spin_rings_from_alm(self._h, _ptr(alm), _ptr(G), int(nthreads))
        return G

    def alm_from_rings(self, G, nthreads=1):
        G = np.asfortranarray(np.asarray(G, dtype=np.complex128).reshape(
            (len(self.theta), 2 * self.lmax + 1, self.ntrans), order="F"))
        alm = np.zeros((self.lmax + 1, 2 * self.lmax + 1, self.ntrans), np.complex128, order="F")
        lib().orc_spin_alm_from_rings(self._h, _ptr(G), _ptr(alm), int(nthreads))
        return alm


class SpinDirect:
    """SpinDirectLeaf (src/Spin.jl:557-630): the O(M L^2) spin oracle."""

    def __init__(self, theta, phi, lmax, spin, ntrans=1):
        self.theta, self.phi = _f64(theta), _f64(phi)
        self.lmax, self.spin, self.ntrans = int(lmax), int(spin), int(ntrans)

    def forward(self, alm, nthreads=1):
        alm = _as3(alm, None)
        f = np.zeros((len(self.theta), self.ntrans), np.complex128, order="F")
        lib().orc_spin_direct(1, self.theta, self.phi, len(self.theta), self.lmax, self.spin,
                              self.ntrans, _ptr(alm), _ptr(f), int(nthreads))
        return f

    def adjoint(self, f, nthreads=1):
        f = np.asfortranarray(np.asarray(f, dtype=np.complex128).reshape(
            (len(self.theta), self.ntrans), order="F"))
        alm = np.zeros((self.lmax + 1, 2 * self.lmax + 1, self.ntrans), np.complex128, order="F")
        lib().orc_spin_direct(0, self.theta, self.phi, len(self.theta), self.lmax, self.spin,
                              self.ntrans, _ptr(f), _ptr(alm), int(nthreads))
        return alm
