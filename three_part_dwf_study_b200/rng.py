"""The reference's host random streams (libstdc++ engines via the C ABI).

    Rng(seed).normals(n)        std::normal_distribution<double>(0, 1) draws
    Rng(seed).uniform()         std::uniform_real_distribution<double>(0, 1)
    Rng(seed).pseudofermion(n)  Complex(normal, normal)/sqrt(2), imaginary first
    z4_digits(seed, n)          std::uniform_int_distribution<int>(0, 3) digits
All draws of one Rng share one mt19937_64, as the reference's generators do.
"""
import ctypes as C

import numpy as np

from . import _capi as A


class Rng:
    def __init__(self, seed):
        h = C.c_void_p()
        A.check(A.lib().dwf_rng_create(C.c_uint64(int(seed) % (1 << 64)), C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            A.lib().dwf_rng_destroy(self._h)
            self._h = None

    def normals(self, n):
        out = np.empty(int(n))
        A.check(A.lib().dwf_rng_normals(self._h, int(n), C.c_void_p(out.ctypes.data)))
        return out

    def uniform(self):
        v = C.c_double()
        A.check(A.lib().dwf_rng_uniform(self._h, C.byref(v)))
        return v.value

    def pseudofermion(self, n):
        out = np.empty(int(n), np.complex128)
        A.check(A.lib().dwf_rng_pseudofermion(self._h, int(n), C.c_void_p(out.ctypes.data)))
        return out


def z4_digits(seed, n):
    out = np.empty(int(n), np.int8)
    A.check(A.lib().dwf_z4_digits(C.c_uint64(int(seed) % (1 << 64)), int(n),
                                  C.c_void_p(out.ctypes.data)))
    return out
