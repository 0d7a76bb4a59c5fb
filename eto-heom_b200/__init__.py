"""Python face of the B200 HEOM-ETO 2DES propagation library (libheom.so, C ABI).

Mirrors the reference's solver interface (etoheom-cpu/lib/dynamics.h:19-25,
param.h:38-82) over the C ABI declared in include/heom.h:

    prob = Problem.from_key("key.key")        # param::param_2des + construct_ADO_set
    prob.prepare_sample()                      # construct_Hal + polar_mat_ranrot + ...
    plan = Plan(prob, precision="fp64-exact")  # device plan
    P = plan.run_traj(1, 1, 0)                 # twoD_spectrum_solver(key, H, 1, 1, 0, P)
    P, trajs = plan.run_2des()                 # CPU_2DES's p111 - p110 - p101
    P = plan.run_scan(points)                  # a whole delay scan in one launch

    prob = Problem.from_key("population.key", dynamics=True)   # param::param_dynamics
    pops = Plan(prob, "fp64-exact").run_populations((1, 2))    # dynamics_solver

There is no CPU fallback: every propagation runs in the CUDA kernels of libheom.so,
and constructing a Plan without a CUDA device raises HeomError.  The package
directory name contains a hyphen, so load it by path (see load_package()).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libheom.so")

FP64_EXACT, FP64, FP32_BULK = 0, 1, 2
PRECISIONS = {"fp64-exact": FP64_EXACT, "fp64": FP64, "fp32-bulk": FP32_BULK}
MAT_H, MAT_X0, MAT_X1, MAT_X2, MAT_X3, MAT_HKEY = range(6)
KEY_SINGLE_MANIFOLD = 1
KEY_DYNAMICS = 2

ERRORS = {-1: "argument", -2: "io", -3: "parse", -4: "cuda", -5: "nomem", -6: "capacity",
          -7: "unsupported", -8: "numeric", -9: "timeout"}


class HeomError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)} error ({code}): {msg}")
        self.code = code


class ProblemInfo(ctypes.Structure):
    _fields_ = [("single_size", ctypes.c_int), ("sys_size", ctypes.c_int), ("K", ctypes.c_int),
                ("K_m", ctypes.c_int), ("L", ctypes.c_int), ("n_ado", ctypes.c_int),
                ("n_sample", ctypes.c_int), ("seed", ctypes.c_ulong), ("n_steps", ctypes.c_int),
                ("print_stride", ctypes.c_int), ("n_record", ctypes.c_int),
                ("t_start", ctypes.c_float), ("t_end", ctypes.c_float), ("step_size", ctypes.c_float),
                ("print_step", ctypes.c_float), ("E0", ctypes.c_double * 3), ("tau", ctypes.c_double * 3),
                ("taup", ctypes.c_double * 3), ("w0", ctypes.c_double * 3)]


class Opts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("device", ctypes.c_int), ("stream", ctypes.c_void_p),
                ("max_points", ctypes.c_int), ("autotune", ctypes.c_int), ("single_pass", ctypes.c_int)]


class ScanPoint(ctypes.Structure):
    _fields_ = [("tau1", ctypes.c_double), ("tau2", ctypes.c_double), ("tau3", ctypes.c_double),
                ("t_end", ctypes.c_float), ("flags", ctypes.c_int)]


SCAN_POINT_DTYPE = np.dtype([("tau1", "<f8"), ("tau2", "<f8"), ("tau3", "<f8"), ("t_end", "<f4"),
                             ("flags", "<i4")])

_lib = None


def lib() -> ctypes.CDLL:
    """Load libheom.so once; raise (never fall back) if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise HeomError(-4, f"{LIB_PATH} is not built; run eto-heom_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    sig = {
        "heom_last_error": (ctypes.c_char_p, []),
        "heom_abi_version": (I, []),
        "heom_problem_from_key": (I, [ctypes.c_char_p, I, ctypes.POINTER(P)]),
        "heom_problem_info_get": (I, [P, ctypes.POINTER(ProblemInfo)]),
        "heom_problem_prepare_sample": (I, [P]),
        "heom_problem_scan_compatible": (I, [P, P]),
        "heom_problem_prepare_identity": (I, [P]),
        "heom_problem_reset_rng": (I, [P]),
        "heom_problem_get_matrix": (I, [P, I, D]),
        "heom_problem_set_matrix": (I, [P, I, D]),
        "heom_problem_get_ado": (I, [P, ctypes.POINTER(ctypes.c_ubyte)]),
        "heom_problem_destroy": (None, [P]),
        "heom_plan_create": (I, [P, ctypes.POINTER(Opts), ctypes.POINTER(P)]),
        "heom_plan_update": (I, [P, P]),
        "heom_run_traj": (I, [P, I, I, I, D, I, ctypes.POINTER(I)]),
        "heom_run_2des": (I, [P, D, D, I, ctypes.POINTER(I)]),
        "heom_run_populations": (I, [P, ctypes.POINTER(I), I, D, I, ctypes.POINTER(I)]),
        "heom_scan_layout": (I, [P, P, I, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(I),
                                 ctypes.POINTER(ctypes.c_longlong)]),
        "heom_run_scan": (I, [P, P, I, D, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(I)]),
        "heom_run_scan_device": (I, [P, P, I, P, P]),
        "heom_host_alloc": (I, [ctypes.c_size_t, ctypes.POINTER(P)]),
        "heom_host_free": (I, [P]),
        "heom_plan_describe": (I, [P, ctypes.c_char_p, I]),
        "heom_plan_launch_count": (ctypes.c_longlong, [P]),
        "heom_plan_scan_work": (ctypes.c_longlong, [P]),
        "heom_plan_sync": (I, [P]),
        "heom_plan_inject_wait_fault": (I, [P, ctypes.c_ulonglong, I]),
        "heom_plan_destroy": (None, [P]),
        "heom_measure_fma_peak": (I, [I, I, D]),
        "heom_run_scan_noalloc": (I, [P, I, P, I, P, P, P]),
        "heom_problem_param_count": (I, [P]),
        "heom_problem_param_dH": (I, [P, I, D]),
        "heom_problem_set_bath_scale": (I, [P, I, I, ctypes.c_double]),
        "heom_adjoint_scan": (I, [P, P, I, ctypes.POINTER(ctypes.c_longlong), ctypes.c_longlong, D, D, D]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != 0:
        raise HeomError(rc, lib().heom_last_error().decode())


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Problem:
    """A parsed key file plus its current disorder/orientation sample."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_key(cls, path: str, single_manifold: bool = False, dynamics: bool = False) -> "Problem":
        """Parse a 2DES key file (param::param_2des) or, with dynamics=True, a
        population-dynamics key file (param::param_dynamics)."""
        h = ctypes.c_void_p()
        flags = (KEY_SINGLE_MANIFOLD if single_manifold else 0) | (KEY_DYNAMICS if dynamics else 0)
        _check(lib().heom_problem_from_key(os.fsencode(path), flags, ctypes.byref(h)))
        return cls(h)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.heom_problem_destroy(self._h)
            self._h = None

    @property
    def info(self) -> ProblemInfo:
        inf = ProblemInfo()
        _check(lib().heom_problem_info_get(self._h, ctypes.byref(inf)))
        return inf

    def prepare_sample(self) -> None:
        _check(lib().heom_problem_prepare_sample(self._h))

    def prepare_identity(self) -> None:
        _check(lib().heom_problem_prepare_identity(self._h))

    def scan_compatible(self, other: "Problem") -> bool:
        """True if the two key files differ at most in pulse times and end time."""
        rc = lib().heom_problem_scan_compatible(self._h, other._h)
        if rc < 0:
            _check(rc)
        return rc == 1

    def reset_rng(self) -> None:
        _check(lib().heom_problem_reset_rng(self._h))

    def matrix(self, which: int) -> np.ndarray:
        N = self.info.sys_size
        out = np.zeros((N, N), dtype=np.complex128)
        _check(lib().heom_problem_get_matrix(self._h, which, _dptr(out)))
        return out

    def set_matrix(self, which: int, m: np.ndarray) -> None:
        a = np.ascontiguousarray(m, dtype=np.complex128)
        _check(lib().heom_problem_set_matrix(self._h, which, _dptr(a)))

    def ado(self) -> np.ndarray:
        inf = self.info
        out = np.zeros((inf.n_ado, inf.K * inf.K_m), dtype=np.uint8)
        _check(lib().heom_problem_get_ado(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))))
        return out

    # ---- gradient parameters: site energies, couplings (cm^-1), bath amplitude scales
    def param_count(self) -> int:
        n = lib().heom_problem_param_count(self._h)
        if n < 0:
            _check(n)
        return n

    def param_dH(self, i: int) -> np.ndarray:
        N = self.info.sys_size
        out = np.zeros((N, N), dtype=np.complex128)
        _check(lib().heom_problem_param_dH(self._h, i, _dptr(out)))
        return out

    def set_bath_scale(self, site: int, line: int, scale: float) -> None:
        _check(lib().heom_problem_set_bath_scale(self._h, site, line, float(scale)))


@dataclass
class ScanResult:
    P: np.ndarray          # concatenated complex points
    offsets: np.ndarray    # int64 per point
    counts: np.ndarray     # int32 per point

    def point(self, i: int) -> np.ndarray:
        return self.P[self.offsets[i]:self.offsets[i] + self.counts[i]]


class Plan:
    """A device plan for one problem (one CUDA device and stream)."""

    def __init__(self, problem: Problem, precision="fp64-exact", device: int = 0, max_points: int = 1024,
                 autotune: bool = False, stream: int | None = None, single_pass: bool = False):
        self.problem = problem
        prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        o = Opts(prec, device, ctypes.c_void_p(stream) if stream else None, max_points, 1 if autotune else 0,
                 1 if single_pass else 0)
        h = ctypes.c_void_p()
        _check(lib().heom_plan_create(problem._h, ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.precision = prec

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.heom_plan_destroy(self._h)
            self._h = None

    def close(self) -> None:
        self.__del__()

    def update(self) -> None:
        _check(lib().heom_plan_update(self._h, self.problem._h))

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(512)
        _check(lib().heom_plan_describe(self._h, buf, 512))
        return buf.value.decode()

    @property
    def launches(self) -> int:
        return int(lib().heom_plan_launch_count(self._h))

    @property
    def scan_work(self) -> int:
        """Component-steps propagated by the last staged scan (0: single pass)."""
        return int(lib().heom_plan_scan_work(self._h))

    def run_traj(self, nv1: int, nv2: int, nv3: int) -> np.ndarray:
        cap = max(self.problem.info.n_record, 1)
        out = np.zeros(cap, dtype=np.complex128)
        n = ctypes.c_int()
        _check(lib().heom_run_traj(self._h, nv1, nv2, nv3, _dptr(out), cap, ctypes.byref(n)))
        return out[:n.value]

    def run_populations(self, sites=(1, 2)) -> np.ndarray:
        """Populations Re rho_0[s-1][s-1] of the given 1-based sites, every print_step from
        t_start, with site 1 initially excited (dynamics_solver, dynamics.cpp:202-295)."""
        s = np.ascontiguousarray(sites, dtype=np.int32)
        cap = max(self.problem.info.n_record, 1)
        out = np.zeros((len(s), cap), dtype=np.float64)
        n = ctypes.c_int()
        _check(lib().heom_run_populations(self._h, s.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(s),
                                          _dptr(out), cap, ctypes.byref(n)))
        return out[:, :n.value]

    def run_2des(self, trajectories: bool = True):
        """CPU_2DES's combined p111 - p110 - p101 and, unless trajectories=False, the
        three mask trajectories (None otherwise; the staged path then propagates the
        combined point only)."""
        cap = max(self.problem.info.n_record, 1)
        P = np.zeros(cap, dtype=np.complex128)
        tr = np.zeros((3, cap), dtype=np.complex128) if trajectories else None
        n = ctypes.c_int()
        _check(lib().heom_run_2des(self._h, _dptr(P), _dptr(tr) if trajectories else None, cap, ctypes.byref(n)))
        return P[:n.value], (tr[:, :n.value] if trajectories else None)

    def scan_layout(self, points: np.ndarray):
        pts = np.ascontiguousarray(points, dtype=SCAN_POINT_DTYPE)
        n = len(pts)
        off = np.zeros(n, dtype=np.int64)
        cnt = np.zeros(n, dtype=np.int32)
        tot = ctypes.c_longlong()
        _check(lib().heom_scan_layout(self._h, pts.ctypes.data_as(ctypes.c_void_p), n,
                                      off.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                                      cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(tot)))
        return pts, off, cnt, int(tot.value)

    def run_scan(self, points: np.ndarray, layout=None, out: np.ndarray | None = None) -> ScanResult:
        """heom_run_scan.  out: an optional complex128 buffer of at least the layout's total
        to write P into (reused across calls, it saves the allocation and first touch of a
        new output array); the result's P is a view of it."""
        pts, off, cnt, tot = layout if layout is not None else self.scan_layout(points)
        if out is not None:
            if out.dtype != np.complex128 or not out.flags.c_contiguous or out.size < max(tot, 1):
                raise ValueError("out must be a contiguous complex128 array of at least the scan's total points")
            P = out
        else:
            P = np.empty(max(tot, 1), dtype=np.complex128)  # every value is written by the call
        _check(lib().heom_run_scan(self._h, pts.ctypes.data_as(ctypes.c_void_p), len(pts), _dptr(P),
                                   off.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                                   cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return ScanResult(P[:tot], off, cnt)

    def adjoint_scan(self, points: np.ndarray, dLdP: np.ndarray, layout=None):
        """Forward scan P (FP64, mixed-difference basis) and the gradient of
        Re sum conj(dLdP) P with respect to the problem's parameters."""
        pts, off, cnt, tot = layout if layout is not None else self.scan_layout(points)
        g = np.ascontiguousarray(dLdP, dtype=np.complex128)
        assert g.shape == (tot,)
        P = np.zeros(max(tot, 1), dtype=np.complex128)
        grad = np.zeros(self.problem.param_count(), dtype=np.float64)
        _check(lib().heom_adjoint_scan(self._h, pts.ctypes.data_as(ctypes.c_void_p), len(pts),
                                       off.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), tot, _dptr(g),
                                       _dptr(P), _dptr(grad)))
        return ScanResult(P[:tot], off, cnt), grad

    def run_scan_device(self, d_pts: int, n: int, d_P: int, d_offsets: int) -> None:
        """Device-pointer form (e.g. torch tensors' data_ptr()); asynchronous on the plan's
        stream.  Errors found on the device are reported by sync() (or the next scan call)."""
        _check(lib().heom_run_scan_device(self._h, ctypes.c_void_p(d_pts), n, ctypes.c_void_p(d_P),
                                          ctypes.c_void_p(d_offsets)))

    def sync(self) -> None:
        """Wait for the plan's queued work; raises HeomError with its deferred status."""
        _check(lib().heom_plan_sync(self._h))

    def inject_wait_fault(self, wait_ns: int, unmet: bool = True) -> None:
        """Test hook: the next staged scan waits at most wait_ns per dependency and, with
        unmet, one job waits for a flag that no producer sets (heom_plan_inject_wait_fault)."""
        _check(lib().heom_plan_inject_wait_fault(self._h, int(wait_ns), 1 if unmet else 0))


def fma_peak_tflops(device: int = 0, fp64: bool = False) -> float:
    """Measured FP32/FP64 FMA throughput of a device (TFLOP/s)."""
    v = ctypes.c_double()
    _check(lib().heom_measure_fma_peak(device, 1 if fp64 else 0, ctypes.byref(v)))
    return float(v.value)


class _PinnedBuffer:
    """Page-locked host memory from heom_host_alloc, exposed to numpy; freed when the
    last array that uses it goes away."""

    def __init__(self, n: int, dtype: np.dtype):
        p = ctypes.c_void_p()
        _check(lib().heom_host_alloc(max(n, 1) * dtype.itemsize, ctypes.byref(p)))
        self._ptr = p.value
        self.__array_interface__ = {"shape": (n,), "typestr": dtype.str, "data": (self._ptr, False), "version": 3}

    def __del__(self):
        if getattr(self, "_ptr", None) and _lib is not None:
            _lib.heom_host_free(ctypes.c_void_p(self._ptr))
            self._ptr = None


def pinned_empty(n: int, dtype=np.complex128) -> np.ndarray:
    """A 1-D array of n elements in page-locked host memory (heom_host_alloc).  As the
    out= buffer of Plan.run_scan it receives P by DMA, checked for Inf/NaN on the device,
    with no staging copy on the host."""
    return np.asarray(_PinnedBuffer(int(n), np.dtype(dtype)))


def make_points(rows) -> np.ndarray:
    """Scan points from (tau1, tau2, tau3, t_end) rows."""
    pts = np.zeros(len(rows), dtype=SCAN_POINT_DTYPE)
    for i, r in enumerate(rows):
        pts[i] = (r[0], r[1], r[2], r[3], 0)
    return pts
