"""pfsht_b200: PartialFSHT.jl's partial-sky SHT apply on one B200, behind the reference's API.

Mirrors the reference's public operator (src/Plan.jl):

    plan = Plan(theta, phi, lmax=L, tol=1e-8)     # Plan(θ, φ; lmax, tol)
    mul(f, plan, alm)                              # mul!(f, plan, alm)
    mul(alm, plan.H, f)                            # mul!(alm, plan', f)
    f = plan * alm;  alm = plan.H * f              # Base.:* (src/Plan.jl:190-199)

Arrays keep the reference's column-major layout. A coefficient array has Julia shape
(lmax+1, 2lmax+1[, ntrans]) with sph_mode packing (src/Layout.jl:13-20); a field has shape
(npts[, ntrans]). On the device these are torch complex128 CUDA tensors with Fortran strides
(``zeros_alm`` / ``zeros_field`` make them); host numpy arrays (Fortran order) go through
the library's host-buffer entry points. All compute is the CUDA library libpfsht_b200.so:
there is no CPU fallback and the package refuses to import without it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import DimensionMismatch, PFSHTError, RefusedGeometry  # noqa: F401

__all__ = ["Plan", "AdjointPlan", "Batch", "Server", "mul", "coeff_size", "sph_mode", "zeros_alm", "zeros_field",
           "plan_geometry", "ring_forward", "ring_adjoint", "NUFFT", "DimensionMismatch",
           "RefusedGeometry", "PFSHTError", "version", "bounding_box", "box_fsky", "cost_direct",
           "cost_stretch", "partition_boxes", "select_method", "cost_constants",
           "set_cost_constants", "cost_calibrated", "solve", "shannon_number", "spectral_resolution"]

_lib.load()


def version() -> str:
    return _lib.load().pfsht_version().decode()


# ---------------------------------------------------------------------------------------
# layout (src/Layout.jl)
# ---------------------------------------------------------------------------------------
def coeff_size(lmax: int):
    """(lmax+1, 2lmax+1) (src/Layout.jl:13)."""
    return (int(lmax) + 1, 2 * int(lmax) + 1)


def sph_mode(l: int, m: int):
    """0-based (row, column) of degree l, order m (src/Layout.jl:20)."""
    am = abs(int(m))
    return (int(l) - am, 2 * am if m >= 0 else 2 * am - 1)


def _torch():
    import torch
    return torch


def _pinned(shape):
    """Zero complex128 numpy array of `shape` in page-locked host memory, column-major."""
    torch = _torch()
    t = torch.zeros(tuple(reversed(shape)), dtype=torch.complex128).pin_memory()
    return t.numpy().T  # the array's base keeps the pinned tensor alive


def zeros_alm(lmax: int, ntrans: int = 1, device="cuda"):
    """Zero coefficient array, Julia shape (lmax+1, 2lmax+1[, ntrans]), column-major.
    ``device`` is a torch device, "cpu" (numpy) or "pinned" (numpy in page-locked memory)."""
    nr, nc = coeff_size(lmax)
    if device == "pinned":
        return _pinned((nr, nc) if ntrans == 1 else (nr, nc, ntrans))
    if device in (None, "cpu", "host"):
        shape = (nr, nc) if ntrans == 1 else (nr, nc, ntrans)
        return np.zeros(shape, dtype=np.complex128, order="F")
    torch = _torch()
    t = torch.zeros((ntrans, nc, nr), dtype=torch.complex128, device=device).permute(2, 1, 0)
    return t[:, :, 0] if ntrans == 1 else t


def zeros_field(npts: int, ntrans: int = 1, device="cuda"):
    """Zero field, Julia shape (npts[, ntrans]), column-major (devices as for zeros_alm)."""
    if device == "pinned":
        return _pinned((npts,) if ntrans == 1 else (npts, ntrans))
    if device in (None, "cpu", "host"):
        shape = (npts,) if ntrans == 1 else (npts, ntrans)
        return np.zeros(shape, dtype=np.complex128, order="F")
    torch = _torch()
    t = torch.zeros((ntrans, npts), dtype=torch.complex128, device=device).permute(1, 0)
    return t[:, 0] if ntrans == 1 else t


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _colmajor_ok(a, shape) -> bool:
    """True when `a` holds `shape` (Julia order) in column-major memory."""
    if tuple(a.shape) != tuple(shape):
        return False
    if _is_torch(a):
        strides = a.stride()
        item = 1
    else:
        strides = a.strides
        item = a.itemsize
    expect = item
    for n, s in zip(shape, strides):
        if n > 1 and s != expect:
            return False
        expect *= n
    return True


def _check_array(a, shapes, what):
    if _is_torch(a):
        torch = _torch()
        if a.dtype != torch.complex128:
            raise TypeError(f"{what} must be complex128, got {a.dtype}")
    else:
        if not isinstance(a, np.ndarray) or a.dtype != np.complex128:
            raise TypeError(f"{what} must be a complex128 numpy array or torch tensor")
    for shp in shapes:
        if tuple(a.shape) == tuple(shp):
            if not _colmajor_ok(a, shp):
                raise ValueError(f"{what} must be column-major (Fortran order), as in Julia")
            return
    raise DimensionMismatch(f"{what} is {tuple(a.shape)}, expected {' or '.join(map(str, shapes))}")


def _coeff_shapes(lmax, B):
    nr, nc = coeff_size(lmax)
    return [(nr, nc), (nr, nc, 1)] if B == 1 else [(nr, nc, B)]


def _field_shapes(npts, B):
    return [(npts,), (npts, 1)] if B == 1 else [(npts, B)]


def _ptr(a) -> int:
    return a.data_ptr() if _is_torch(a) else a.ctypes.data


def _stream_of(a, stream):
    if stream is not None:
        return int(getattr(stream, "cuda_stream", stream))
    torch = _torch()
    return torch.cuda.current_stream(a.device).cuda_stream


# ---------------------------------------------------------------------------------------
# Plan (src/Plan.jl)
# ---------------------------------------------------------------------------------------
class Plan:
    """Plan(theta, phi; lmax, tol=1e-10, ntrans=1, method="auto") (src/Plan.jl:84-116).

    ``method`` is "auto" (the cost model's choice among the stretched leaf, the direct leaf
    and the multi-box leaf, src/Cost.jl:171-201), "stretch" (refusal raises RefusedGeometry),
    "direct" or "multibox" (one stretched leaf per box of the partition, at most ``maxboxes``,
    src/MultiBox.jl; ``boxes()`` lists them).
    ``precision`` is "fp64" (plain form) or "mixed". Points may be host arrays or CUDA
    tensors (float64). ``rings_per_lane`` / ``bin_rows`` / ``bin_cols`` are device tile
    shapes (0 = defaults); ``segment_degrees`` splits the adjoint ring pass along the degree
    axis (0 = auto, negative = never). ``fft_lengths`` is "timed" (NUFFT fine-grid lengths
    picked by timing the library FFT, the default), "minimal" (the smallest 2,3,5-smooth
    lengths, deterministic) or a pair (nf1, nf2) of lengths at or above the minimum;
    ``info["nf1"]``, ``info["nf2"]`` give the lengths in use. ``transpose`` is "tma" (the NUFFT's
    fine-row transposes load their tiles with TMA tensor copies where the layout allows, the
    default) or "plain" (plain loads only; the results are the same bit for bit). ``spread`` is
    "registers" (the spreading holds each bin's whole tile in registers where it fits, the
    default) or "window" (a sliding window of the kernel's rows); both add the same values in
    the same order.
    ``deterministic=True`` makes adjoints bitwise reproducible run to run (fixed-order sums in
    the ring pass and the spreading) at some cost in speed; by default floating-point atomic
    additions let two adjoints differ at round-off.
    ``spin`` (|spin| <= lmax) transforms spin-weighted fields, f = sum sa_lm sY_lm, with the
    coefficient (l, m) at ``alm[l, m + lmax]`` (src/Layout.jl:28-29, ``spin_coeff_index``);
    entries below l = max(|m|, |spin|) are ignored by the forward and zeroed by the adjoint.
    """

    def __init__(self, theta, phi, *, lmax, tol=1e-10, ntrans=1, method="auto",
                 precision="fp64", oversample_theta=1.0, oversample_phi=1.0, eps_apo_max=1.0,
                 device=None, rings_per_lane=0, bin_rows=0, bin_cols=0, segment_degrees=0,
                 fft_lengths="timed", maxboxes=8, spin=0, transpose="tma", deterministic=False,
                 spread="registers"):
        self._h = None
        if len(theta) != len(phi):
            raise DimensionMismatch("θ and φ must have the same length")
        if lmax < 0:
            raise ValueError("lmax must be nonnegative")
        if spin != 0 and abs(spin) > lmax:
            raise ValueError(f"(|spin| = {abs(spin)}) > lmax = {lmax}")
        if ntrans < 1:
            raise ValueError("ntrans must be ≥ 1")
        if method not in _lib.METHODS:
            raise ValueError(f"unknown method {method!r}")
        if precision not in _lib.PRECISIONS:
            raise ValueError(f"unknown precision {precision!r}")
        o = _lib.default_opts()
        o.method = _lib.METHODS[method]
        o.oversample_theta = float(oversample_theta)
        o.oversample_phi = float(oversample_phi)
        o.eps_apo_max = float(eps_apo_max)
        o.ring_rings_per_lane = int(rings_per_lane)
        o.nufft_bin_rows = int(bin_rows)
        o.nufft_bin_cols = int(bin_cols)
        o.ring_segment_degrees = int(segment_degrees)
        if maxboxes < 1:
            raise ValueError("maxboxes must be >= 1")
        o.maxboxes = int(maxboxes)
        o.spin = int(spin)
        if transpose not in ("tma", "plain"):
            raise ValueError(f"unknown transpose {transpose!r}")
        o.nufft_transpose = 0 if transpose == "tma" else 1
        o.deterministic = 1 if deterministic else 0
        if spread not in ("registers", "window"):
            raise ValueError(f"unknown spread {spread!r}")
        o.nufft_spread = 0 if spread == "registers" else 1
        if isinstance(fft_lengths, (tuple, list)) and len(fft_lengths) == 2:
            o.nufft_fft_lengths = 2
            o.nufft_nf1, o.nufft_nf2 = int(fft_lengths[0]), int(fft_lengths[1])
        elif fft_lengths in ("timed", "minimal"):
            o.nufft_fft_lengths = 0 if fft_lengths == "timed" else 1
        else:
            raise ValueError(f"unknown fft_lengths {fft_lengths!r}")
        if _is_torch(theta):
            torch = _torch()
            th = theta.to(torch.float64).contiguous()
            ph = phi.to(dtype=torch.float64, device=th.device).contiguous()
            if th.is_cuda:
                # the plan is built on the library's own stream: finish torch's writes first
                torch.cuda.current_stream(th.device).synchronize()
                o.points_on_device = 1
                o.device = th.device.index if device is None else int(device)
            else:
                o.device = -1 if device is None else int(device)
            keep = (th, ph)
            pth, pph = th.data_ptr(), ph.data_ptr()
        else:
            th = np.ascontiguousarray(theta, dtype=np.float64)
            ph = np.ascontiguousarray(phi, dtype=np.float64)
            o.device = -1 if device is None else int(device)
            keep = (th, ph)
            pth, pph = th.ctypes.data, ph.ctypes.data
        h = C.c_void_p()
        _lib.check(_lib.load().pfsht_plan_create(pth, pph, len(th), int(lmax), int(ntrans),
                                                 float(tol), _lib.PRECISIONS[precision],
                                                 C.byref(o), C.byref(h)), "Plan")
        self._points = keep  # the plan's points (bounding box for solve's info)
        self._h = h
        self.lmax = int(lmax)
        self.ntrans = int(ntrans)
        self.tol = float(tol)
        self.npts = len(theta)
        self.spin = int(spin)
        self.precision = precision
        inf = _lib.PlanInfo()
        _lib.check(_lib.load().pfsht_plan_get_info(self._h, C.byref(inf)))
        self.info = {k: getattr(inf, k) for k, _ in _lib.PlanInfo._fields_}
        self.info["kind"] = _lib.KINDS[inf.kind]
        self.device = o.device

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None and _lib._lib is not None:
            _lib._lib.pfsht_plan_destroy(h)
        self._h = None

    def close(self):
        self.__del__()

    # -- reference queries --------------------------------------------------------------
    @property
    def algorithm(self) -> str:
        """algorithm(plan) (src/Plan.jl:36)."""
        return {"direct": "DirectAlgorithm", "multibox": "MultiBoxAlgorithm"}.get(
            self.info["kind"], "StretchAlgorithm")

    def boxes(self) -> list:
        """The plan's boxes (src/MultiBox.jl:75-79): for each, its leaf's info and the indices of
        its points (ascending, 0-based). A single-leaf plan is its own one box."""
        lib = _lib.load()
        out = []
        for i in range(int(lib.pfsht_plan_num_boxes(self._h))):
            inf = _lib.PlanInfo()
            _lib.check(lib.pfsht_plan_box(self._h, i, C.byref(inf), None), "plan_box")
            idx = np.empty(inf.npts, dtype=np.int64)
            _lib.check(lib.pfsht_plan_box(self._h, i, C.byref(inf), idx.ctypes.data), "plan_box")
            d = {k: getattr(inf, k) for k, _ in _lib.PlanInfo._fields_}
            d["kind"] = _lib.KINDS[inf.kind]
            d["indices"] = idx
            out.append(d)
        return out

    def ring_work(self) -> int:
        """ring_work(plan) (src/Plan.jl:44): retained (l, m, ring) triples per apply."""
        return int(_lib.load().pfsht_ring_work(self._h))

    def host_bytes(self) -> dict:
        """Bytes one host-buffer forward / adjoint moves between host and device."""
        v = [C.c_int64() for _ in range(4)]
        _lib.check(_lib.load().pfsht_host_bytes(self._h, *[C.byref(x) for x in v]), "host_bytes")
        return {"h2d_forward": v[0].value, "d2h_forward": v[1].value,
                "h2d_adjoint": v[2].value, "d2h_adjoint": v[3].value}

    def workspace_bytes(self) -> int:
        return int(_lib.load().pfsht_workspace_bytes(self._h))

    def profile_start(self, max_marks: int = 4096):
        """Start per-stage CUDA-event timing of this plan's applies."""
        _lib.check(_lib.load().pfsht_profile_start(self._h, int(max_marks)), "profile_start")

    def profile_stop(self) -> dict:
        """Stop stage timing; returns {stage: (total_ms, launches)} for stages that ran."""
        lib = _lib.load()
        n = int(lib.pfsht_num_stages())
        ms = (C.c_double * n)()
        cnt = (C.c_int32 * n)()
        _lib.check(lib.pfsht_profile_stop(self._h, ms, cnt), "profile_stop")
        return {lib.pfsht_stage_name(i).decode(): (ms[i], cnt[i]) for i in range(n) if cnt[i]}

    def __repr__(self):
        return (f"PartialFSHT.Plan(lmax={self.lmax}, npts={self.npts}, ntrans={self.ntrans}, "
                f"spin={self.spin}, algorithm={self.algorithm})")

    @property
    def H(self) -> "AdjointPlan":
        """plan' (src/Plan.jl:22)."""
        return AdjointPlan(self)

    adjoint = H

    # -- applies ------------------------------------------------------------------------
    def mul(self, f, alm, stream=None):
        """mul!(f, plan, alm) (src/Plan.jl:137-141)."""
        _check_array(alm, _coeff_shapes(self.lmax, self.ntrans), "coefficient array")
        _check_array(f, _field_shapes(self.npts, self.ntrans), "field")
        lib = _lib.load()
        if _is_torch(alm) and alm.is_cuda:
            if not (_is_torch(f) and f.is_cuda):
                raise ValueError("alm and f must both be CUDA tensors or both host arrays")
            _lib.check(lib.pfsht_forward(self._h, _ptr(alm), _ptr(f), _stream_of(alm, stream)), "mul!")
        else:
            if _is_torch(f) and f.is_cuda:
                raise ValueError("alm and f must both be CUDA tensors or both host arrays")
            _lib.check(lib.pfsht_forward_host(self._h, _ptr(alm), _ptr(f)), "mul!")
        return f

    def mul_adjoint(self, alm, f, stream=None):
        """mul!(alm, plan', f) (src/Plan.jl:143-148); overwrites alm."""
        _check_array(alm, _coeff_shapes(self.lmax, self.ntrans), "coefficient array")
        _check_array(f, _field_shapes(self.npts, self.ntrans), "field")
        lib = _lib.load()
        if _is_torch(f) and f.is_cuda:
            if not (_is_torch(alm) and alm.is_cuda):
                raise ValueError("alm and f must both be CUDA tensors or both host arrays")
            _lib.check(lib.pfsht_adjoint(self._h, _ptr(f), _ptr(alm), _stream_of(f, stream)), "mul!")
        else:
            if _is_torch(alm) and alm.is_cuda:
                raise ValueError("alm and f must both be CUDA tensors or both host arrays")
            _lib.check(lib.pfsht_adjoint_host(self._h, _ptr(f), _ptr(alm)), "mul!")
        return alm

    def mul_async(self, f, alm):
        """mul!(f, plan, alm) on page-locked host arrays without waiting: the result is in f
        once host_sync() returns (pfsht_forward_host_async)."""
        _check_array(alm, _coeff_shapes(self.lmax, self.ntrans), "coefficient array")
        _check_array(f, _field_shapes(self.npts, self.ntrans), "field")
        if (_is_torch(alm) and alm.is_cuda) or (_is_torch(f) and f.is_cuda):
            raise ValueError("mul_async takes host arrays")
        _lib.check(_lib.load().pfsht_forward_host_async(self._h, _ptr(alm), _ptr(f), None), "mul!")
        return f

    def mul_adjoint_async(self, alm, f):
        """mul!(alm, plan', f) on page-locked host arrays without waiting; alm is complete once
        host_sync() returns (pfsht_adjoint_host_async)."""
        _check_array(alm, _coeff_shapes(self.lmax, self.ntrans), "coefficient array")
        _check_array(f, _field_shapes(self.npts, self.ntrans), "field")
        if (_is_torch(alm) and alm.is_cuda) or (_is_torch(f) and f.is_cuda):
            raise ValueError("mul_adjoint_async takes host arrays")
        _lib.check(_lib.load().pfsht_adjoint_host_async(self._h, _ptr(f), _ptr(alm), None), "mul!")
        return alm

    def host_sync(self):
        """Waits for the plan's host-buffer applies issued so far (pfsht_host_sync)."""
        _lib.check(_lib.load().pfsht_host_sync(self._h), "host_sync")

    def __mul__(self, alm):
        """plan * alm (src/Plan.jl:190-193)."""
        dev = alm.device if (_is_torch(alm) and alm.is_cuda) else "cpu"
        f = zeros_field(self.npts, self.ntrans, device=dev)
        return self.mul(f, alm)

    __matmul__ = __mul__


class AdjointPlan:
    """plan' (src/Plan.jl:18-23)."""

    def __init__(self, parent: Plan):
        self.parent = parent

    @property
    def H(self) -> Plan:
        return self.parent

    def mul(self, alm, f, stream=None):
        return self.parent.mul_adjoint(alm, f, stream)

    def __mul__(self, f):
        """plan' * f (src/Plan.jl:195-199)."""
        dev = f.device if (_is_torch(f) and f.is_cuda) else "cpu"
        alm = zeros_alm(self.parent.lmax, self.parent.ntrans, device=dev)
        return self.parent.mul_adjoint(alm, f)

    __matmul__ = __mul__


def mul(out, op, x, stream=None):
    """mul!(out, op, x): forward for a Plan, adjoint for an AdjointPlan."""
    if isinstance(op, Plan):
        return op.mul(out, x, stream)
    if isinstance(op, AdjointPlan):
        return op.mul(out, x, stream)
    raise TypeError("op must be a Plan or an AdjointPlan")


# ---------------------------------------------------------------------------------------
# lower seams used by parity tests
# ---------------------------------------------------------------------------------------
def ring_forward(plan: Plan, alm, G, stream=None):
    """rings_from_alm! on the plan's ring set (src/Legendre.jl:310-323); G is a CUDA tensor
    of Julia shape (nrings, 2lmax+1[, ntrans])."""
    _lib.check(_lib.load().pfsht_ring_forward(plan._h, _ptr(alm), _ptr(G), _stream_of(alm, stream)),
               "rings_from_alm!")
    return G


def ring_adjoint(plan: Plan, G, alm, stream=None):
    """alm_from_rings! (src/Legendre.jl:332-341)."""
    _lib.check(_lib.load().pfsht_ring_adjoint(plan._h, _ptr(G), _ptr(alm), _stream_of(G, stream)),
               "alm_from_rings!")
    return alm


def dfs_double(F, Ft, spin=0, stream=None):
    """dfs_double!(Ft, F, spin) (src/DFS.jl:13-33): CUDA tensors, F of Julia shape
    (Nth, Nph[, B]) and Ft (2Nth, Nph[, B])."""
    nth, nph = int(F.shape[0]), int(F.shape[1])
    B = int(F.shape[2]) if F.dim() > 2 else 1
    _check_array(Ft, [(2 * nth, nph, B)] + ([(2 * nth, nph)] if B == 1 else []), "Ft")
    _lib.check(_lib.load().pfsht_dfs_double(_ptr(F), _ptr(Ft), nth, nph, B, int(spin),
                                            _stream_of(F, stream)), "dfs_double!")
    return Ft


def dfs_fold(Ft, F, spin=0, stream=None):
    """dfs_fold!(F, Ft, spin) (src/DFS.jl:35-56), the transpose of dfs_double!."""
    nth, nph = int(F.shape[0]), int(F.shape[1])
    B = int(F.shape[2]) if F.dim() > 2 else 1
    _check_array(Ft, [(2 * nth, nph, B)] + ([(2 * nth, nph)] if B == 1 else []), "Ft")
    _lib.check(_lib.load().pfsht_dfs_fold(_ptr(F), _ptr(Ft), nth, nph, B, int(spin),
                                          _stream_of(Ft, stream)), "dfs_fold!")
    return F


def plan_geometry(theta, phi, *, lmax, tol=1e-10, ntrans=1, method="auto",
                  oversample_theta=1.0, oversample_phi=1.0, eps_apo_max=1.0, maxboxes=8,
                  spin=0) -> dict:
    """Host-only: the geometry and sizes pfsht_plan_create would choose (no device used)."""
    th = np.ascontiguousarray(theta, dtype=np.float64)
    ph = np.ascontiguousarray(phi, dtype=np.float64)
    o = _lib.default_opts()
    o.method = _lib.METHODS[method]
    o.maxboxes = int(maxboxes)
    o.spin = int(spin)
    o.oversample_theta = float(oversample_theta)
    o.oversample_phi = float(oversample_phi)
    o.eps_apo_max = float(eps_apo_max)
    inf = _lib.PlanInfo()
    _lib.check(_lib.load().pfsht_plan_geometry(th.ctypes.data, ph.ctypes.data, len(th), int(lmax),
                                               int(ntrans), float(tol), C.byref(o), C.byref(inf)),
               "plan_geometry")
    d = {k: getattr(inf, k) for k, _ in _lib.PlanInfo._fields_}
    d["kind"] = _lib.KINDS[inf.kind]
    return d


# ---------------------------------------------------------------------------------------
# planner (src/Box.jl, src/Cost.jl), host only
# ---------------------------------------------------------------------------------------
def _box_dict(b) -> dict:
    return {"theta_lo": b.theta_lo, "theta_hi": b.theta_hi, "phi_start": b.phi_start,
            "phi_extent": b.phi_extent, "touches_north": bool(b.touches_north),
            "touches_south": bool(b.touches_south)}


def _box_struct(d) -> "_lib.Box":
    return _lib.Box(float(d["theta_lo"]), float(d["theta_hi"]), float(d["phi_start"]),
                    float(d["phi_extent"]), int(bool(d["touches_north"])),
                    int(bool(d["touches_south"])))


def _points(theta, phi):
    th = np.ascontiguousarray(theta, dtype=np.float64)
    ph = np.ascontiguousarray(phi, dtype=np.float64)
    if th.shape != ph.shape or th.ndim != 1:
        raise DimensionMismatch("θ and φ must have the same length")
    return th, ph


def _device_points(theta, phi):
    """CUDA float64 tensors (the planner's device scans), or None for host arrays."""
    if not (_is_torch(theta) and theta.is_cuda):
        return None
    torch = _torch()
    th = theta.to(torch.float64).contiguous()
    ph = phi.to(dtype=torch.float64, device=th.device).contiguous()
    if th.shape != ph.shape or th.dim() != 1:
        raise DimensionMismatch("θ and φ must have the same length")
    torch.cuda.current_stream(th.device).synchronize()
    return th, ph


def bounding_box(theta, phi) -> dict:
    """bounding_box(θ, φ) (src/Box.jl:42-73): the exactly minimal colatitude x longitude box.
    CUDA tensors are scanned on their device."""
    b = _lib.Box()
    dp = _device_points(theta, phi)
    if dp is not None:
        _lib.check(_lib.load().pfsht_bounding_box_device(dp[0].data_ptr(), dp[1].data_ptr(),
                                                         len(dp[0]), C.byref(b), None), "bounding_box")
        return _box_dict(b)
    th, ph = _points(theta, phi)
    _lib.check(_lib.load().pfsht_bounding_box(th.ctypes.data, ph.ctypes.data, len(th), C.byref(b)),
               "bounding_box")
    return _box_dict(b)


def box_fsky(box) -> float:
    """box_fsky (src/Box.jl:98-104): fraction of the sphere the box covers."""
    return (np.cos(box["theta_lo"]) - np.cos(box["theta_hi"])) * box["phi_extent"] / (4 * np.pi)


def cost_direct(npts, lmax, ntrans=1) -> float:
    """cost_direct (src/Cost.jl:107-108)."""
    return float(_lib.load().pfsht_cost_direct(int(npts), int(lmax), int(ntrans)))


def cost_stretch(box, npts, lmax, ntrans=1, tol=1e-10) -> float:
    """cost_stretch (src/Cost.jl:117-142); inf where the stretched geometry is refused."""
    b = _box_struct(box)
    return float(_lib.load().pfsht_cost_stretch(C.byref(b), int(npts), int(lmax), int(ntrans),
                                                float(tol)))


def partition_boxes(theta, phi, *, lmax, ntrans=1, tol=1e-10, maxboxes=8):
    """partition_boxes_costed(θ, φ, cost_stretch; maxboxes) (src/Box.jl:156-200): the groups
    (ascending 0-based indices), their boxes and their predicted costs. CUDA tensors are scanned
    on their device (the same result)."""
    nb = C.c_int32()
    boxes = (_lib.Box * int(maxboxes))()
    costs = (C.c_double * int(maxboxes))()
    dp = _device_points(theta, phi)
    if dp is not None:
        gop = np.empty(len(dp[0]), dtype=np.int32)
        _lib.check(_lib.load().pfsht_partition_boxes_device(
            dp[0].data_ptr(), dp[1].data_ptr(), len(dp[0]), int(lmax), int(ntrans), float(tol),
            int(maxboxes), gop.ctypes.data, C.byref(nb), boxes, costs, None), "partition_boxes")
    else:
        th, ph = _points(theta, phi)
        gop = np.empty(len(th), dtype=np.int32)
        _lib.check(_lib.load().pfsht_partition_boxes(th.ctypes.data, ph.ctypes.data, len(th),
                                                     int(lmax), int(ntrans), float(tol),
                                                     int(maxboxes), gop.ctypes.data, C.byref(nb),
                                                     boxes, costs), "partition_boxes")
    n = nb.value
    groups = [np.flatnonzero(gop == i) for i in range(n)]
    return groups, [_box_dict(boxes[i]) for i in range(n)], [costs[i] for i in range(n)]


def select_method(theta, phi, *, lmax, tol=1e-10, ntrans=1) -> str:
    """select_method(θ, φ, lmax, tol, AutoAlgorithm(), ntrans) (src/Cost.jl:171-201):
    "stretch", "direct" or "multibox" (CUDA tensors: scans on their device)."""
    m = C.c_int32()
    dp = _device_points(theta, phi)
    if dp is not None:
        _lib.check(_lib.load().pfsht_select_method_device(dp[0].data_ptr(), dp[1].data_ptr(),
                                                          len(dp[0]), int(lmax), int(ntrans),
                                                          float(tol), C.byref(m), None),
                   "select_method")
        return {v: k for k, v in _lib.METHODS.items()}[m.value]
    th, ph = _points(theta, phi)
    _lib.check(_lib.load().pfsht_select_method(th.ctypes.data, ph.ctypes.data, len(th), int(lmax),
                                               int(ntrans), float(tol), C.byref(m)), "select_method")
    return {v: k for k, v in _lib.METHODS.items()}[m.value]


def shannon_number(lmax, box_or_fsky) -> float:
    """shannon_number (src/Box.jl:123-132): (lmax+1)^2 f_sky."""
    fsky = box_fsky(box_or_fsky) if isinstance(box_or_fsky, dict) else float(box_or_fsky)
    return (int(lmax) + 1) ** 2 * fsky


def spectral_resolution(box) -> float:
    """spectral_resolution (src/Box.jl:141-154): pi / (the box's larger angular extent)."""
    tiny = np.sqrt(np.finfo(np.float64).eps)
    mid = min(max((box["theta_lo"] + box["theta_hi"]) / 2, tiny), np.pi - tiny)
    lam = max(box["theta_hi"] - box["theta_lo"], box["phi_extent"] * np.sin(mid))
    return np.inf if lam <= 0 else np.pi / lam


_SOLVE_MODES = {"cg": 0, "wiener": 1, "minnorm": 2}


def solve(alm, plan, f, *, mode="cg", rtol=1e-6, maxiter=500, prior=None, w=None, stream=None):
    """solve!(alm, plan, f; mode, rtol, maxiter, prior, w) (src/Analysis.jl:375-436):
    conjugate gradients on (A^H W A + C^-1) alm = A^H W f, run on the device (one CUDA graph per
    iteration, scalars on the device). ``alm`` (overwritten) and ``f`` are CUDA tensors or host
    arrays; ``prior`` is C_l for l = 0..lmax ("wiener" only); ``w`` per-point weights. Returns
    (alm, info) with info's mode, iters, relres, shannon and Δℓ."""
    if mode not in _SOLVE_MODES:
        raise ValueError(f"mode must be cg, wiener or minnorm, got {mode!r}")
    if mode == "wiener" and prior is None:
        raise ValueError("wiener needs a prior C_l: that prior is what makes the problem well posed")
    _check_array(alm, _coeff_shapes(plan.lmax, plan.ntrans), "coefficient array")
    _check_array(f, _field_shapes(plan.npts, plan.ntrans), "field")
    torch = _torch()
    dev = torch.device("cuda", plan.device if plan.device >= 0 else torch.cuda.current_device())
    on_dev = _is_torch(alm) and alm.is_cuda
    if on_dev != (_is_torch(f) and f.is_cuda):
        raise ValueError("alm and f must both be CUDA tensors or both host arrays")
    if on_dev:
        a_d, f_d = alm, f
    else:
        a_d = zeros_alm(plan.lmax, plan.ntrans, device=dev)
        f_d = zeros_field(plan.npts, plan.ntrans, device=dev)
        f_d.copy_(torch.from_numpy(np.asarray(f)))
    pr = None
    if prior is not None:
        pr = np.ascontiguousarray(prior, dtype=np.float64)
        if len(pr) < plan.lmax + 1:
            raise DimensionMismatch(f"prior must cover l = 0:{plan.lmax}, got {len(pr)} entries")
    wd = None
    if w is not None:
        wd = (w if _is_torch(w) else torch.from_numpy(np.ascontiguousarray(w, dtype=np.float64)))
        wd = wd.to(device=dev, dtype=torch.float64).contiguous()
        if wd.numel() != plan.npts:
            raise DimensionMismatch(f"weights have {wd.numel()} entries, field has {plan.npts}")
    s = _stream_of(a_d, stream)
    torch.cuda.current_stream(dev).synchronize()
    it = C.c_int32()
    rel = C.c_double()
    _lib.check(_lib.load().pfsht_solve(plan._h, _ptr(f_d), _ptr(a_d), _SOLVE_MODES[mode], float(rtol),
                                       int(maxiter), pr.ctypes.data if pr is not None else None,
                                       wd.data_ptr() if wd is not None else None, s,
                                       C.byref(it), C.byref(rel)), "solve!")
    if not on_dev:
        torch.cuda.synchronize(dev)
        np.copyto(alm, a_d.cpu().numpy(), casting="no")
    box = getattr(plan, "_box", None)
    if box is None:
        box = plan._box = bounding_box(*plan._points)
    info = {"mode": mode, "iters": it.value, "relres": rel.value,
            "shannon": shannon_number(plan.lmax, box), "Δℓ": spectral_resolution(box)}
    return alm, info


def cost_constants() -> dict:
    """The planner's per-unit costs (src/Cost.jl:39-58) and whether they were installed."""
    v = [C.c_double() for _ in range(4)]
    cal = C.c_int32()
    _lib.check(_lib.load().pfsht_get_cost_constants(*[C.byref(x) for x in v], C.byref(cal)))
    return {"ring": v[0].value, "fft": v[1].value, "spread": v[2].value, "ft_conn": v[3].value,
            "calibrated": bool(cal.value)}


def set_cost_constants(*, ring=None, fft=None, spread=None, ft_conn=None) -> dict:
    """set_cost_constants! (src/Cost.jl:60-71): install measured per-unit costs (process-wide);
    the model then reports itself calibrated."""
    c = cost_constants()
    new = [c["ring"] if ring is None else ring, c["fft"] if fft is None else fft,
           c["spread"] if spread is None else spread, c["ft_conn"] if ft_conn is None else ft_conn]
    _lib.check(_lib.load().pfsht_set_cost_constants(*[float(x) for x in new]), "set_cost_constants")
    return cost_constants()


def cost_calibrated() -> bool:
    """cost_calibrated() (src/Cost.jl:74)."""
    return cost_constants()["calibrated"]


class Batch:
    """Many plans applied together (pfsht_batch_*): one captured CUDA graph per direction, the
    ring passes of all plans in a few launches, the other stages on ``nstreams`` streams. The
    batch borrows the plans: keep them alive and do not apply them elsewhere meanwhile."""

    def __init__(self, plans, nstreams=0):
        self._h = None
        self.plans = list(plans)
        if not self.plans:
            raise ValueError("a batch needs at least one plan")
        arr = (C.c_void_p * len(self.plans))(*[p._h for p in self.plans])
        h = C.c_void_p()
        _lib.check(_lib.load().pfsht_batch_create(arr, len(self.plans), int(nstreams), C.byref(h)),
                   "batch")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None and _lib._lib is not None:
            _lib._lib.pfsht_batch_destroy(h)
        self._h = None

    def _ptrs(self, arrays, shapes, what):
        if len(arrays) != len(self.plans):
            raise DimensionMismatch(f"{len(arrays)} {what} arrays for {len(self.plans)} plans")
        for a, shp in zip(arrays, shapes):
            _check_array(a, shp, what)
            if not (_is_torch(a) and a.is_cuda):
                raise ValueError("batch applies take CUDA tensors")
        return (C.c_void_p * len(arrays))(*[_ptr(a) for a in arrays])

    def forward(self, fs, alms, stream=None):
        """mul!(f_i, plan_i, alm_i) for every plan of the batch."""
        pa = self._ptrs(alms, [_coeff_shapes(p.lmax, p.ntrans) for p in self.plans], "coefficient")
        pf_ = self._ptrs(fs, [_field_shapes(p.npts, p.ntrans) for p in self.plans], "field")
        _lib.check(_lib.load().pfsht_batch_forward(self._h, pa, pf_, _stream_of(alms[0], stream)),
                   "batch forward")
        return fs

    def adjoint(self, alms, fs, stream=None):
        """mul!(alm_i, plan_i', f_i) for every plan of the batch."""
        pa = self._ptrs(alms, [_coeff_shapes(p.lmax, p.ntrans) for p in self.plans], "coefficient")
        pf_ = self._ptrs(fs, [_field_shapes(p.npts, p.ntrans) for p in self.plans], "field")
        _lib.check(_lib.load().pfsht_batch_adjoint(self._h, pf_, pa, _stream_of(fs[0], stream)),
                   "batch adjoint")
        return alms

    def info(self) -> dict:
        a, b = C.c_int32(), C.c_int32()
        c, d = C.c_int64(), C.c_int64()
        _lib.check(_lib.load().pfsht_batch_info(self._h, C.byref(a), C.byref(b), C.byref(c),
                                                C.byref(d)), "batch info")
        return {"ring_launches_fwd": a.value, "ring_launches_adj": b.value,
                "graph_nodes_fwd": c.value, "graph_nodes_adj": d.value}


class Server:
    """Serving loop (pfsht_server_*): plans resident on one device, synthesis and adjoint
    requests on host arrays run as they arrive, concurrently across plans, within an HBM
    budget for the resident plans. Registered plans must outlive the server."""

    def __init__(self, hbm_budget_gb=120.0, nslots=8, device=None):
        self._h = None
        h = C.c_void_p()
        dev = -1 if device is None else int(device)
        _lib.check(_lib.load().pfsht_server_create(dev, int(hbm_budget_gb * 1e9), int(nslots),
                                                   C.byref(h)), "server")
        self._h = h
        self.plans = []
        self._keep = {}

    def add(self, plan) -> int:
        pid = C.c_int32()
        _lib.check(_lib.load().pfsht_server_add_plan(self._h, plan._h, C.byref(pid)), "add_plan")
        self.plans.append(plan)
        return pid.value

    def submit(self, plan_id, forward, inp, out) -> int:
        """Queue mul!(out, plan, inp) (forward) or mul!(out, plan', inp); host arrays."""
        p = self.plans[plan_id]
        cs, fs = _coeff_shapes(p.lmax, p.ntrans), _field_shapes(p.npts, p.ntrans)
        _check_array(inp, cs if forward else fs, "input")
        _check_array(out, fs if forward else cs, "output")
        if _is_torch(inp) or _is_torch(out):
            raise ValueError("server requests take host (numpy) arrays")
        rid = C.c_int64()
        _lib.check(_lib.load().pfsht_server_submit(self._h, int(plan_id), 1 if forward else 0,
                                                   _ptr(inp), _ptr(out), C.byref(rid)), "submit")
        self._keep[rid.value] = (inp, out)
        return rid.value

    def wait(self, rid, timeout=None) -> float:
        """Block until request `rid` is done; returns its latency in seconds."""
        lat = C.c_double()
        _lib.check(_lib.load().pfsht_server_wait(self._h, int(rid), -1.0 if timeout is None
                                                 else float(timeout), C.byref(lat)), "wait")
        return lat.value

    def times(self, rid):
        """(submitted, started, done) in seconds since the server was created."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        _lib.check(_lib.load().pfsht_server_request_times(self._h, int(rid), C.byref(a),
                                                          C.byref(b), C.byref(c)), "times")
        return a.value, b.value, c.value

    def release(self, rid):
        _lib.check(_lib.load().pfsht_server_release(self._h, int(rid)), "release")
        self._keep.pop(rid, None)

    def stats(self) -> dict:
        v = [C.c_int64() for _ in range(4)]
        _lib.check(_lib.load().pfsht_server_stats(self._h, *[C.byref(x) for x in v]), "stats")
        return dict(zip(("completed", "queued", "running", "bytes_resident"), [x.value for x in v]))

    def close(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None and _lib._lib is not None:
            _lib._lib.pfsht_server_destroy(h)
        self._h = None
        self._keep = {}

    __del__ = close


class NUFFT:
    """The NUFFT seam (src/NUFFT.jl:17-25): 2-D type-1/2 NUFFT, modes (n1, n2) in FFT order,
    host points; exec on CUDA tensors."""

    def __init__(self, type, n1, n2, iflag, x, y, tol, ntrans=1):
        xx = np.ascontiguousarray(x, dtype=np.float64)
        yy = np.ascontiguousarray(y, dtype=np.float64)
        h = C.c_void_p()
        _lib.check(_lib.load().pfsht_nufft_create(int(type), int(n1), int(n2), int(iflag),
                                                  int(ntrans), float(tol), xx.ctypes.data,
                                                  yy.ctypes.data, len(xx), C.byref(h)),
                   "_nufft_makeplan")
        self._h = h
        self.type, self.n1, self.n2, self.ntrans, self.M = int(type), int(n1), int(n2), int(ntrans), len(xx)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None and _lib._lib is not None:
            _lib._lib.pfsht_nufft_destroy(h)
        self._h = None

    def exec(self, inp, out, stream=None):
        _lib.check(_lib.load().pfsht_nufft_exec(self._h, _ptr(inp), _ptr(out), _stream_of(inp, stream)),
                   "_nufft_exec!")
        return out
