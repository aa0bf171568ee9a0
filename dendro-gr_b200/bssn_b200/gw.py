"""Gravitational-wave extraction from psi4 (csrc/gw.cu; the reference's
extractFarFieldPsi4, BSSN_GR/include/gwExtract.h:48-190): psi4 on spheres
about the origin decomposed into spin-weight -2 spherical-harmonic modes.

    modes, coeff, l2 = extract(re, im, spec, radii=(50.0, 100.0), lmax=4)
    # coeff[r, k]: complex mode (l, m) = modes[k] at radius r

re / im: zipped psi4 fields of a single-level mesh (e.g. rows 4 and 5 of
bssn_constraints_psi4_f64's output), CUDA tensors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import check, lib, stream_ptr

lib.bssn_gw_modes_count.argtypes = [C.c_int]
lib.bssn_gw_extract_f64.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                    C.c_double, C.c_int, C.POINTER(C.c_double), C.c_int, C.c_int,
                                    C.c_void_p, C.c_void_p, C.c_void_p]
lib.bssn_gw_sphere_tables.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 4


def modes(lmax):
    return [(l, m) for l in range(2, lmax + 1) for m in range(-l, l + 1)]


def sphere_tables(lmax, ntheta):
    """(theta, phi, w, Y[mode, point] complex) of the extraction rule."""
    n = 2 * ntheta * ntheta
    th, ph, w = np.zeros(n), np.zeros(n), np.zeros(n)
    nm = lib.bssn_gw_modes_count(lmax)
    y = np.zeros((nm, n, 2))
    check(lib.bssn_gw_sphere_tables(lmax, ntheta, th.ctypes.data, ph.ctypes.data, w.ctypes.data, y.ctypes.data),
          "gw_sphere_tables")
    return th, ph, w, y[..., 0] + 1j * y[..., 1]


def extract(re, im, spec, radii, lmax=4, ntheta=24, stream=None):
    import torch
    nm = lib.bssn_gw_modes_count(lmax)
    coeff = torch.zeros((len(radii), nm, 2), dtype=torch.float64, device="cuda")
    l2 = torch.zeros((len(radii), 2), dtype=torch.float64, device="cuda")
    G = (C.c_int32 * 3)(*spec.G)
    xm = (C.c_double * 3)(*spec.origin3)
    rr = (C.c_double * len(radii))(*radii)
    check(lib.bssn_gw_extract_f64(C.c_void_p(re.data_ptr()), C.c_void_p(im.data_ptr()), G, xm, spec.h,
                                  len(radii), rr, lmax, ntheta, C.c_void_p(coeff.data_ptr()),
                                  C.c_void_p(l2.data_ptr()), stream_ptr(stream)), "gw_extract")
    c = coeff.cpu().numpy()
    return modes(lmax), c[..., 0] + 1j * c[..., 1], l2.cpu().numpy()
