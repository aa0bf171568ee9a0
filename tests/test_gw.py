"""The extraction rule of the gravitational-wave modes (csrc/gw.cu) on the
CPU: the spin-weight -2 harmonics in the stated convention and orthonormal
under the quadrature, whose weights sum to 4 pi."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dendro-gr_b200"))
B = pytest.importorskip("bssn_b200")
from bssn_b200 import gw  # noqa: E402


def test_harmonics_and_quadrature():
    lmax, nt = 4, 12
    th, ph, w, Y = gw.sphere_tables(lmax, nt)
    md = gw.modes(lmax)
    assert abs(w.sum() - 4 * np.pi) < 1e-12
    y22 = np.sqrt(5 / np.pi) / 8 * (1 + np.cos(th)) ** 2 * np.exp(2j * ph)
    y2m2 = np.sqrt(5 / np.pi) / 8 * (1 - np.cos(th)) ** 2 * np.exp(-2j * ph)
    assert np.abs(Y[md.index((2, 2))] - y22).max() < 1e-14
    assert np.abs(Y[md.index((2, -2))] - y2m2).max() < 1e-14
    # -2Y_20 = sqrt(15/(32 pi)) sin^2 theta
    assert np.abs(Y[md.index((2, 0))] - np.sqrt(15 / (32 * np.pi)) * np.sin(th) ** 2).max() < 1e-14
    gram = (Y * w) @ Y.conj().T
    assert np.abs(gram - np.eye(len(md))).max() < 1e-12
