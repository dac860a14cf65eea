"""Shared stacks and rules of the parity tests (the reference's validation scripts'
materials and helpers: Gz_ClosedForm_TestHelpers.jl, Gz_ClosedForm_Point_Validation.jl,
Gz_ClosedForm_Foundation_Validation.jl)."""
import numpy as np

from yellowthinfilms_b200.materials import (BiaxialMaterial, FlatLayer, FlatOpticalLayer, GyrotropicMaterial,
                                            IsotropicMaterial, UniaxialMaterial)

lay = FlatOpticalLayer
m_vac = IsotropicMaterial(1.0 + 0.001j)
m_gl = IsotropicMaterial(2.25 + 0.001j)
m_hi = IsotropicMaterial(6.0 + 0.3j)
m_uni = UniaxialMaterial(2.0 + 0.01j, 3.5 + 0.01j)
m_bi = BiaxialMaterial(2.0 + 0.01j, 3.0 + 0.01j, 4.0 + 0.01j)
m_biT = BiaxialMaterial(3.0 + 0.01j, 2.0 + 0.01j, 4.0 + 0.01j)
m_gyr4 = GyrotropicMaterial([[4.0 + 0.01j, 0.3j, 0], [-0.3j, 4.0 + 0.01j, 0], [0, 0, 3.0 + 0.01j]])
m_gyr = GyrotropicMaterial([[2.1 + 0.1j, 1.2j, 0], [-1.2j, 2.1 + 0.1j, 0], [0, 0, 1.5 + 0.05j]])

FOUNDATION_STACKS = [
    ("iso 3-layer vac/glass/vac", [lay(m_vac, 2.0), lay(m_gl, 2.0), lay(m_vac, 2.0)]),
    ("iso 5-layer lossy", [lay(m_vac, 1.0), lay(m_gl, 0.7), lay(m_hi, 0.3), lay(m_gl, 1.1), lay(m_vac, 1.0)]),
    ("uniaxial 4-layer", [lay(m_vac, 1.0), lay(m_uni, 0.8), lay(m_gl, 0.5), lay(m_vac, 1.0)]),
    ("biaxial 4-layer", [lay(m_vac, 1.0), lay(m_bi, 0.8), lay(m_gl, 0.5), lay(m_vac, 1.0)]),
    ("gyrotropic 4-layer", [lay(m_gyr4, 1.0), lay(m_gl, 0.6), lay(m_gyr4, 0.9), lay(m_vac, 1.0)]),
]


def gauss_legendre(n):
    x, w = np.polynomial.legendre.leggauss(n)
    return x, w


def krho_grid(stack, omega, kmax=20.0, width=0.5, order=8):
    """Fixed GL reference rule broken at the light lines (Gz_ClosedForm_TestHelpers.jl:10-24)."""
    brk = sorted(set([0.0, kmax] + [float(np.real(np.sqrt(complex(l.eps[i, i]))) * omega) for l in stack for i in range(2)]))
    brk = [b for b in brk if 0 <= b <= kmax]
    x, w = gauss_legendre(order)
    ks, ws = [], []
    for a, b in zip(brk[:-1], brk[1:]):
        npan = max(1, int(np.ceil((b - a) / width)))
        for j in range(npan):
            lo = a + j * (b - a) / npan
            hi = lo + (b - a) / npan
            ks.extend((hi - lo) / 2 * x + (hi + lo) / 2)
            ws.extend((hi - lo) / 2 * w)
    return np.array(ks), np.array(ws)


def uniform_phi(n):
    return 2 * np.pi * np.arange(n) / n, np.full(n, 2 * np.pi / n)


def relerr(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def e_free(r, p, k, eps):
    """Analytic free-space dipole field, ϵ0 = μ0 = c = 1, e^{-iωt}
    (Gz_ClosedForm_Point_Validation.jl:164-167)."""
    R = np.linalg.norm(r)
    n = r / R
    return (np.exp(1j * k * R) / (4 * np.pi * eps)) * (
        k ** 2 * np.cross(np.cross(n, p), n) / R + (3 * n * np.dot(n, p) - p) * (1 / R ** 3 - 1j * k / R ** 2))


def config1_like_stack():
    """Air / uniaxial hyperbolic film / glass in wavelength units (600 nm → 1): the film is
    εo = -3+0.4i, εe = 4+0.2i, 50 nm; air 200 nm above it. It carries guided-mode poles
    for the pole scan."""
    return [lay(IsotropicMaterial(1.0), 200.0 / 600.0), lay(UniaxialMaterial(-3.0 + 0.4j, 4.0 + 0.2j), 50.0 / 600.0),
            lay(IsotropicMaterial(2.25), 100.0 / 600.0)]
