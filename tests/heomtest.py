"""Shared test helpers: load the package by path, bind the CPU oracle, read fixtures.

The oracle (oracle/liboracle.so) is test infrastructure: it is only ever used here as
the checker, never as the thing under test.
"""
from __future__ import annotations

import ctypes
import importlib.util
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "eto-heom_b200")
KEYS = os.path.join(ROOT, "tests", "golden", "keys")
REF = os.path.join(ROOT, "tests", "golden", "ref")
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle.so")


def load_pkg():
    if "eto_heom_b200" in sys.modules:
        return sys.modules["eto_heom_b200"]
    spec = importlib.util.spec_from_file_location("eto_heom_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["eto_heom_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def key(name: str) -> str:
    return os.path.join(KEYS, name)


def golden(name: str):
    d = np.load(os.path.join(REF, name.replace(".key", ".npz")))
    return d["traj"], d["combined"]


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


# ------------------------------------------------------------------ oracle binding
class Oracle:
    HO_DENSE, HO_STRUCTURED = 0, 1

    def __init__(self):
        if not os.path.exists(ORACLE_LIB):
            subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"])
        L = ctypes.CDLL(ORACLE_LIB)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
        L.ho_load_key.argtypes = [ctypes.c_char_p, I, ctypes.POINTER(P), ctypes.c_char_p, I]
        L.ho_free.argtypes = [P]
        L.ho_info.argtypes = [P, ctypes.POINTER(I)]
        for f in ("ho_rng_reset", "ho_prepare_sample", "ho_prepare_identity"):
            getattr(L, f).argtypes = [P]
        L.ho_get_matrix.argtypes = [P, I, D]
        L.ho_set_matrix.argtypes = [P, I, D]
        L.ho_get_ado.argtypes = [P, ctypes.POINTER(ctypes.c_ubyte)]
        L.ho_rhs.argtypes = [P, D, D, D, I]
        L.ho_traj.argtypes = [P, I, I, I, I, I, D, I, ctypes.POINTER(I)]
        L.ho_2des.argtypes = [P, I, I, D, I, ctypes.POINTER(I), D]
        L.ho_2des_q.argtypes = [P, I, D, I, ctypes.POINTER(I), D]
        self.L = L

    def load(self, path: str, single_manifold: bool = False):
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = self.L.ho_load_key(os.fsencode(path), 1 if single_manifold else 0, ctypes.byref(h), err, 512)
        if rc:
            raise ValueError(err.value.decode())
        return OracleProblem(self, h)


class OracleProblem:
    def __init__(self, o: Oracle, h):
        self.o, self.h = o, h
        info = (ctypes.c_int * 10)()
        o.L.ho_info(h, info)
        (self.single_size, self.N, self.K, self.K_m, self.L, self.n_ado, self.n_sample, self.n_steps,
         self.stride, _) = list(info)

    def __del__(self):
        if self.h:
            self.o.L.ho_free(self.h)
            self.h = None

    def matrix(self, which: int) -> np.ndarray:
        out = np.zeros((self.N, self.N), dtype=np.complex128)
        self.o.L.ho_get_matrix(self.h, which, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def ado(self) -> np.ndarray:
        out = np.zeros((self.n_ado, self.K * self.K_m), dtype=np.uint8)
        self.o.L.ho_get_ado(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
        return out

    def prepare_sample(self):
        self.o.L.ho_prepare_sample(self.h)

    def prepare_identity(self):
        self.o.L.ho_prepare_identity(self.h)

    def rng_reset(self):
        self.o.L.ho_rng_reset(self.h)

    def rhs(self, V: np.ndarray, rho: np.ndarray, mode: int = 1) -> np.ndarray:
        V = np.ascontiguousarray(V, dtype=np.complex128)
        rho = np.ascontiguousarray(rho, dtype=np.complex128)
        out = np.zeros_like(rho)
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
        self.o.L.ho_rhs(self.h, dp(V), dp(rho), dp(out), mode)
        return out

    def traj(self, nv, mode=1, max_steps=0) -> np.ndarray:
        cap = self.n_steps + 1
        out = np.zeros(cap, dtype=np.complex128)
        n = ctypes.c_int()
        rc = self.o.L.ho_traj(self.h, nv[0], nv[1], nv[2], mode, max_steps,
                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cap, ctypes.byref(n))
        assert rc == 0
        return out[:n.value]

    def run_2des(self, mode=1, max_steps=0):
        cap = self.n_steps + 1
        P = np.zeros(cap, dtype=np.complex128)
        tr = np.zeros((self.n_sample, 3, cap), dtype=np.complex128)
        n = ctypes.c_int()
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
        rc = self.o.L.ho_2des(self.h, mode, max_steps, dp(P), cap, ctypes.byref(n), dp(tr))
        assert rc == 0
        return P[:n.value], tr[:, :, :n.value]


    def run_2des_truth(self, max_steps=0):
        """ho_2des_q: the reference's scheme in binary128 (the true combined output)."""
        cap = self.n_steps + 1
        P = np.zeros(cap, dtype=np.complex128)
        tr = np.zeros((self.n_sample, 3, cap), dtype=np.complex128)
        n = ctypes.c_int()
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
        rc = self.o.L.ho_2des_q(self.h, max_steps, dp(P), cap, ctypes.byref(n), dp(tr))
        assert rc == 0
        return P[:n.value], tr[:, :, :n.value]


def truth(name: str):
    """Binary128 truth fixture tests/golden/ref/truth_<name>.npz (make_fixtures.py --truth):
    (rows, [P_true per point], [reference build P per point] or None, grid indices or None)."""
    d = np.load(os.path.join(REF, f"truth_{name}.npz"))
    off = d["offsets"]
    cut = lambda a: [a[off[i]:off[i + 1]] for i in range(len(off) - 1)]  # noqa: E731
    return (d["rows"], cut(d["truth"]), cut(d["reference"]) if "reference" in d else None,
            d["grid_index"] if "grid_index" in d else None)


_oracle = None


def oracle() -> Oracle:
    global _oracle
    if _oracle is None:
        _oracle = Oracle()
    return _oracle


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max_t |a - b| / max_t |b| (the parity metric)."""
    a, b = np.asarray(a), np.asarray(b)
    den = np.abs(b).max() if b.size else 0.0
    num = np.abs(a - b).max() if b.size else 0.0
    return float(num / den) if den > 0 else float(num)
