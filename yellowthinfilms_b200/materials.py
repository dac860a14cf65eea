"""Material and layer descriptors, mirroring the reference's types.

Reference: ``mod_ModeSolver.jl:20-80`` (``IsotropicMaterial``, ``UniaxialMaterial``,
``BiaxialMaterial``, ``GyrotropicMaterial``, ``FlatOpticalLayer(ϵ, d)``,
``FlatLayer(ϵ, μ, d)``). The material's TYPE, not only its values, selects the mode
solver: isotropic or uniaxial ε with isotropic μ takes the closed-form TE/TM modes
(``mod_ModeSolver.jl:243-265``), everything else the general 4x4 eigen solve
(``mod_ModeSolver.jl:207-211``). ``kind`` carries that type across the C ABI.

Tensors are 3x3 complex; the C ABI takes them column-major (Julia's order).
"""
from __future__ import annotations

import numpy as np

ISO, UNI, BIAX, GEN = 0, 1, 2, 3
KIND_NAMES = {ISO: "isotropic", UNI: "uniaxial", BIAX: "biaxial", GEN: "gyrotropic"}


class Material:
    kind: int
    tensor: np.ndarray

    def __getitem__(self, ij):
        i, j = ij
        return self.tensor[i - 1, j - 1]

    def __repr__(self):
        return f"{type(self).__name__}({np.array2string(self.tensor, precision=4)})"


class IsotropicMaterial(Material):
    kind = ISO

    def __init__(self, eps):
        self.tensor = complex(eps) * np.eye(3, dtype=np.complex128)


class UniaxialMaterial(Material):
    kind = UNI

    def __init__(self, eps_t, eps_z):
        self.tensor = np.diag([complex(eps_t), complex(eps_t), complex(eps_z)]).astype(np.complex128)


class BiaxialMaterial(Material):
    kind = BIAX

    def __init__(self, eps_x, eps_y, eps_z):
        self.tensor = np.diag([complex(eps_x), complex(eps_y), complex(eps_z)]).astype(np.complex128)


class GyrotropicMaterial(Material):
    kind = GEN

    def __init__(self, eps):
        t = np.asarray(eps, dtype=np.complex128)
        if t.shape != (3, 3):
            raise ValueError("GyrotropicMaterial needs a 3x3 tensor")
        self.tensor = t.copy()


_VACUUM_MU = IsotropicMaterial(1.0)


class FlatLayer:
    """A layer of thickness ``d`` with permittivity ``eps`` and permeability ``mu``."""

    def __init__(self, eps: Material, mu: Material, d: float):
        self.eps_material, self.mu_material, self.d = eps, mu, float(d)

    @property
    def eps_kind(self):
        return self.eps_material.kind

    @property
    def mu_kind(self):
        return self.mu_material.kind

    @property
    def eps(self):
        return self.eps_material.tensor

    @property
    def mu(self):
        return self.mu_material.tensor

    def __repr__(self):
        return f"FlatLayer({self.eps_material!r}, {self.mu_material!r}, d={self.d})"


class FlatOpticalLayer(FlatLayer):
    """Non-magnetic layer (μ = 1), ``FlatOpticalLayer(ϵ, d)`` of the reference."""

    def __init__(self, eps: Material, d: float):
        super().__init__(eps, _VACUUM_MU, d)

    def __repr__(self):
        return f"FlatOpticalLayer({self.eps_material!r}, d={self.d})"


def is_azimuthally_symmetric(stack) -> bool:
    """``_is_azimuthally_symmetric_stack`` (mod_ModeSolver.jl:427-434)."""
    return all(l.eps_kind in (ISO, UNI) and l.mu_kind == ISO for l in stack)


def stack_arrays(stack):
    """Flat arrays for the C ABI: kinds (int32), ε and μ (complex128, nL x 9 column-major), d."""
    ek = np.array([l.eps_kind for l in stack], dtype=np.int32)
    mk = np.array([l.mu_kind for l in stack], dtype=np.int32)
    eps = np.ascontiguousarray(np.stack([np.asarray(l.eps, np.complex128).T.reshape(9) for l in stack]))
    mu = np.ascontiguousarray(np.stack([np.asarray(l.mu, np.complex128).T.reshape(9) for l in stack]))
    d = np.array([l.d for l in stack], dtype=np.float64)
    return ek, mk, eps, mu, d
