"""Gravitational-wave extraction on the GPU (bssn_gw_extract_f64): psi4
fields that are polynomials of degree <= 6 in x, y, z are reproduced
exactly by the octant interpolation, so the modes and sums from the grid
equal the same quadrature of the analytic fields (rounding only).  The
harmonics and the rule themselves are checked on the CPU (test_gw.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_modes_of_polynomial_fields():
    import bssn_b200 as B
    from bssn_b200 import gw
    spec = B.generate_mesh(0, (4, 4, 4))  # [-8, 8]^3, 25 nodes per axis
    G, h, x0 = spec.G, spec.h, spec.xmin
    g = np.arange(spec.n_nodes)
    x = x0 + (g % G[0]) * h
    y = x0 + ((g // G[0]) % G[1]) * h
    z = x0 + (g // (G[0] * G[1])) * h

    def f_re(x, y, z):
        return 0.3 + x * x - y * z + 0.01 * x * y * z * z

    def f_im(x, y, z):
        return 0.2 * y - 0.05 * x ** 3 + 1e-3 * z ** 4 * x * x

    re = torch.from_numpy(f_re(x, y, z)).cuda()
    im = torch.from_numpy(f_im(x, y, z)).cuda()
    radii = (2.0, 5.5)
    lmax, nt = 4, 16
    md, coeff, l2 = gw.extract(re, im, spec, radii, lmax=lmax, ntheta=nt)
    th, ph, w, Y = gw.sphere_tables(lmax, nt)
    for r, R in enumerate(radii):
        px, py, pz = R * np.sin(th) * np.cos(ph), R * np.sin(th) * np.sin(ph), R * np.cos(th)
        psi = f_re(px, py, pz) + 1j * f_im(px, py, pz)
        ref = 4 * np.pi * (Y.conj() * (w * psi)).sum(axis=1)
        assert np.abs(coeff[r] - ref).max() <= 1e-10 * np.abs(ref).max(), r
        assert np.allclose(l2[r], [(psi.real ** 2).sum(), (psi.imag ** 2).sum()], rtol=1e-10)

