"""ctypes front end of the tuned CPU port (oracle/cpu_port.cpp): the CPU
baseline that bench.py times beside the GPU.  Test and benchmark
infrastructure only, like the oracle: the product never loads it.

The port is compiled with -march=native for the host that runs it, into
oracle/_native/<host key>/, the first time that host asks for it.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import platform
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class _Desc(C.Structure):
    _fields_ = [("degree", C.c_int), ("nc", C.c_int * 3), ("vertices", C.POINTER(C.c_double)),
                ("dirichlet_mask", C.POINTER(C.c_uint8)), ("uniform", C.c_int), ("kind", C.c_int),
                ("dt", C.c_double), ("rho_cp", C.c_double), ("k0", C.c_double), ("k_alpha", C.c_double),
                ("temperature", C.POINTER(C.c_double)), ("theta", C.c_double), ("diffusivity", C.c_double),
                ("vel_kind", C.c_int)]


def host_key():
    """The CPU model and instruction-set flags of this host: a build made with
    -march=native is only loaded on hosts with the same key."""
    text = platform.machine()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    text += line
                    if line.startswith("flags"):
                        break
    except OSError:
        pass
    return hashlib.sha1(text.encode()).hexdigest()[:12]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "_native", host_key(), "libmpdg_cpu_port.so")
        src = os.path.join(HERE, "cpu_port.cpp")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            subprocess.run(["make", "-s", "-C", HERE, "port", f"PORT_OUT={path}"], check=True)
        L = C.CDLL(path)
        L.port_create.restype = C.c_void_p
        L.port_create.argtypes = [C.POINTER(_Desc)]
        L.port_destroy.argtypes = [C.c_void_p]
        L.port_n_dofs.restype = C.c_long
        L.port_n_dofs.argtypes = [C.c_void_p]
        L.port_vmult.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.port_diagonal.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.port_cg_jacobi.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                     C.c_double, C.c_int, C.POINTER(C.c_double)]
        _lib = L
    return _lib


def threads():
    return int(lib().port_threads())


def _p(a, t=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


class PortOperator:
    """Heat (k(T) = k0 (1 + k_alpha T), optional Dirichlet mask) or
    advection-diffusion (vortex velocity) operator on a structured hexahedral
    mesh, lexicographic DoF numbering as the library's and the oracle's."""

    def __init__(self, vertices, nc, degree, mask=None, uniform=False, kind=0, dt=1e-3, rho_cp=1.0, k0=1.0,
                 k_alpha=0.0, temperature=None, theta=0.5, diffusivity=0.0, velocity=None):
        self._keep = [np.ascontiguousarray(vertices, np.float64).reshape(-1, 3),
                      None if mask is None else np.ascontiguousarray(mask, np.uint8),
                      None if temperature is None else np.ascontiguousarray(temperature, np.float64)]
        V, m, T = self._keep
        d = _Desc(int(degree), (C.c_int * 3)(*[int(v) for v in nc]), _p(V), _p(m, C.c_uint8), int(bool(uniform)),
                  int(kind), dt, rho_cp, k0, k_alpha, _p(T), theta, diffusivity, 2 if velocity == "vortex" else 0)
        self._h = lib().port_create(C.byref(d))
        if not self._h:
            raise ValueError("port_create failed")
        self.n_dofs = int(lib().port_n_dofs(self._h))

    def vmult(self, dst, src):
        lib().port_vmult(self._h, _p(dst), _p(np.ascontiguousarray(src, np.float64)))
        return dst

    def diagonal(self):
        d = np.zeros(self.n_dofs)
        lib().port_diagonal(self._h, _p(d))
        return d

    def cg_jacobi(self, b, rel_tol=1e-10, abs_tol=0.0, max_it=10000):
        x = np.zeros(self.n_dofs)
        res = C.c_double()
        it = lib().port_cg_jacobi(self._h, _p(x), _p(np.ascontiguousarray(b, np.float64)), rel_tol, abs_tol,
                                  max_it, C.byref(res))
        return x, it, res.value

    def close(self):
        if getattr(self, "_h", None):
            lib().port_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
