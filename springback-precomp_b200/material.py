"""Materials of the element loop: the reference's material block
(include/sparlab/material/Material.hpp:103-257, python/precomp/materials.py)
as a plain dataclass, and its conversion to the C ABI's sbk_material.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Sequence, Tuple

from . import _capi


@dataclasses.dataclass
class Material:
    """Isotropic elasticity, sigma_y(a) = sy0 + H a + Q (1 - exp(-delta a)),
    Prager's H_kin, von Mises or Hill48 (r-values in the frame of the rolling
    direction and the sheet normal) and Chaboche backstresses (C_i, gamma_i)."""

    youngs_modulus: float
    poisson_ratio: float
    yield_stress: float = 0.0
    hardening_modulus: float = 0.0
    kinematic_hardening_modulus: float = 0.0
    saturation_stress: float = 0.0
    saturation_rate: float = 0.0
    criterion: str = "von_mises"  # or "hill48"
    r0: float = 1.0
    r45: float = 1.0
    r90: float = 1.0
    shear_l: float = 1.5
    shear_m: float = 1.5
    rolling_direction: Tuple[float, float, float] = (1.0, 0.0, 0.0)
    sheet_normal: Tuple[float, float, float] = (0.0, 0.0, 1.0)
    backstresses: Sequence[Tuple[float, float]] = ()
    kinematic_integration: str = "exponential"  # or "backward_euler"
    name: str = "material"

    def to_c(self) -> _capi.sbk_material:
        m = _capi.sbk_material()
        m.youngs_modulus = self.youngs_modulus
        m.poisson_ratio = self.poisson_ratio
        m.yield_stress = self.yield_stress
        m.hardening_modulus = self.hardening_modulus
        m.kinematic_hardening_modulus = self.kinematic_hardening_modulus
        m.saturation_stress = self.saturation_stress
        m.saturation_rate = self.saturation_rate
        m.criterion = 1 if self.criterion == "hill48" else 0
        back = list(self.backstresses)
        m.num_backstresses = len(back)
        m.kinematic_integration = 1 if self.kinematic_integration == "backward_euler" else 0
        for i, (c, g) in enumerate(back):
            m.backstress_modulus[i] = c
            m.backstress_recovery[i] = g
        m.r0, m.r45, m.r90 = self.r0, self.r45, self.r90
        m.shear_l, m.shear_m = self.shear_l, self.shear_m
        for i in range(3):
            m.rolling_direction[i] = self.rolling_direction[i]
            m.sheet_normal[i] = self.sheet_normal[i]
        return m

    def as_dict(self) -> dict:
        d = dataclasses.asdict(self)
        d["backstresses"] = [tuple(b) for b in self.backstresses]
        return d

    @property
    def general(self) -> bool:
        return self.criterion == "hill48" or len(self.backstresses) > 0

    @property
    def kinematic_terms(self) -> int:
        if not self.general:
            return 0
        return len(self.backstresses) + (1 if self.kinematic_hardening_modulus > 0.0 else 0)

    @property
    def state_fields(self) -> int:
        """Doubles per point of the device state layout (sbk_state_fields)."""
        return 14 + 6 * self.kinematic_terms

    @property
    def symmetric(self) -> bool:
        return all(g <= 0.0 for _, g in self.backstresses)

    @classmethod
    def from_swift(cls, name: str, youngs_modulus: float, poisson_ratio: float, K: float, eps0: float, n: float,
                   fit_range: Tuple[float, float] = (0.0, 0.6), points: int = 200, **extra) -> "Material":
        """Linear + Voce hardening standing for the Swift law sigma = K (eps0
        + a)^n, as python/precomp/materials.py:205-254 builds it (the
        parameters must come out the same, so the fit is the same): sy0 =
        K eps0^n exactly; H, Q >= 0 by non-negative least squares on the
        Swift excess over sy0 at `points` equally spaced plastic strains of
        `fit_range`; delta by a bounded scalar search over ln delta in
        [ln 0.1, ln 500] (x tolerance 1e-6); delta = 0 when Q vanishes."""
        if not (K > 0 and eps0 > 0 and n >= 0):
            raise ValueError("from_swift needs K > 0, eps0 > 0 and n >= 0")
        lo, hi = float(fit_range[0]), float(fit_range[1])
        if not 0.0 <= lo < hi:
            raise ValueError("fit_range must satisfy 0 <= low < high")
        sy0 = K * eps0 ** n
        H, Q, delta = _voce_fit(lo, hi, points, lambda a: K * (eps0 + a) ** n - sy0)
        return cls(name=name, youngs_modulus=youngs_modulus, poisson_ratio=poisson_ratio, yield_stress=sy0,
                   hardening_modulus=H, saturation_stress=Q, saturation_rate=delta, **extra)

    @classmethod
    def from_hollomon(cls, name: str, youngs_modulus: float, poisson_ratio: float, K: float, n: float,
                      yield_stress: float, **extra) -> "Material":
        """Hollomon sigma = K eps^n from the yield point on
        (python/precomp/materials.py:256-270): the Swift law whose eps0 puts
        its start at `yield_stress`, eps0 = (yield_stress / K)^(1/n)."""
        if not (K > 0 and n > 0 and yield_stress > 0):
            raise ValueError("from_hollomon needs K, n and yield_stress > 0")
        return cls.from_swift(name, youngs_modulus, poisson_ratio, K, (yield_stress / K) ** (1.0 / n), n, **extra)


def _voce_fit(lo: float, hi: float, points: int, excess):
    """(H, Q, delta) of H a + Q (1 - exp(-delta a)) closest to excess(a) in
    least squares over `points` plastic strains a in [lo, hi]."""
    import numpy as np
    from scipy.optimize import minimize_scalar, nnls

    a = np.linspace(lo, hi, points)
    y = excess(a)

    def nnls_at(log_rate):
        basis = np.column_stack([a, 1.0 - np.exp(-math.exp(log_rate) * a)])
        return nnls(basis, y)

    search = minimize_scalar(lambda t: float(nnls_at(t)[1]), bounds=(math.log(0.1), math.log(500.0)),
                             method="bounded", options={"xatol": 1e-6})
    (H, Q), _ = nnls_at(search.x)
    H, Q = float(H), float(Q)
    return H, Q, (math.exp(search.x) if Q > 0.0 else 0.0)


def yield_matrix(m: Material):
    """The yield matrix P of the material's criterion (6x6, tensorial Voigt)."""
    import numpy as np

    out = (_capi.ctypes.c_double * 36)()
    _capi.check(_capi.lib().sbk_yield_matrix(_capi.ctypes.byref(m.to_c()), out))
    return np.array(list(out)).reshape(6, 6)


def rule_c(stiffness_points: int = 2, thickness_points: int = 0, thickness_axis: int = 2) -> _capi.sbk_rule:
    r = _capi.sbk_rule()
    r.stiffness_points = stiffness_points
    r.thickness_points = thickness_points
    r.thickness_axis = thickness_axis
    return r


def rule_size(stiffness_points: int = 2, thickness_points: int = 0, thickness_axis: int = 2) -> int:
    r = rule_c(stiffness_points, thickness_points, thickness_axis)
    return int(_capi.lib().sbk_rule_size(_capi.ctypes.byref(r)))


# Materials of the configurations and of the reference's own element tests
# (tests/test_incompatible_modes.cpp:394-430), SI units.
def aluminium_swift() -> Material:
    """E = 70 GPa, nu = 0.33, Swift K = 425 MPa, eps0 = 0.003, n = 0.29,
    converted to linear + Voce hardening as precomp does."""
    return Material.from_swift("al_swift", 70.0e9, 0.33, 425.0e6, 0.003, 0.29)


def hill_chaboche_sheet() -> Material:
    """The element microbenchmark's law: the aluminium's elasticity and
    isotropic hardening, Hill48 r0 = 0.73, r45 = 0.80, r90 = 0.70 (RD = x,
    ND = z), Chaboche C1 = 8000 MPa, g1 = 200; C2 = 1200 MPa, g2 = 20,
    exponential integration."""
    base = aluminium_swift()
    return dataclasses.replace(base, name="hill_chaboche", criterion="hill48", r0=0.73, r45=0.80, r90=0.70,
                               backstresses=((8000.0e6, 200.0), (1200.0e6, 20.0)))


# The built-in sheet materials of python/precomp/materials.py:272-299
# (Hollomon K, n, yield stress; r-values; E, nu), by name.
_HOLLOMON = {
    "AA5754-O": (70.0e9, 0.33, 420e6, 0.30, 100e6, (0.75, 0.70, 0.80)),
    "AA2024-O": (73.1e9, 0.33, 330e6, 0.20, 75e6, (0.70, 0.80, 0.70)),
    "AA6061-T6": (68.9e9, 0.33, 410e6, 0.06, 276e6, (0.60, 0.70, 0.65)),
    "AA7075-O": (71.7e9, 0.33, 400e6, 0.17, 103e6, (0.70, 0.90, 0.80)),
    "DC04": (210.0e9, 0.30, 530e6, 0.22, 170e6, (1.90, 1.50, 2.20)),
    "Ti-6Al-4V-annealed": (113.8e9, 0.342, 1100e6, 0.04, 880e6, None),
}


def library_material(name: str, anisotropic: bool = False) -> Material:
    """A built-in material by name (case-insensitive), J2 with its linear +
    Voce fit; with `anisotropic`, Hill48 from its r-values (RD = x, ND =
    z). The reference stores the r-values beside a von Mises criterion
    unless a deck asks for Hill48."""
    for key, (E, nu, K, n, sy, r) in _HOLLOMON.items():
        if key.lower() == name.lower():
            m = Material.from_hollomon(key, E, nu, K, n, sy)
            if anisotropic and r is not None:
                m = dataclasses.replace(m, criterion="hill48", r0=r[0], r45=r[1], r90=r[2])
            return m
    raise KeyError(f"unknown material {name!r}; the library has {sorted(_HOLLOMON)}")


def j2_steel() -> Material:
    return Material(200.0e9, 0.3, yield_stress=250.0e6, hardening_modulus=2.0e9, kinematic_hardening_modulus=1.0e9,
                    name="j2")


def hill_sheet() -> Material:
    return Material(200.0e9, 0.3, yield_stress=250.0e6, hardening_modulus=1.5e9, criterion="hill48", r0=1.9, r45=1.5,
                    r90=2.3, rolling_direction=(1.0, 0.5, 0.0), name="hill")


def chaboche_steel() -> Material:
    return Material(200.0e9, 0.3, yield_stress=250.0e6, saturation_stress=100.0e6, saturation_rate=20.0,
                    backstresses=((40.0e9, 400.0), (5.0e9, 20.0)), name="chaboche")


def elastic_steel() -> Material:
    return Material(200.0e9, 0.3, name="elastic")


def perfectly_plastic() -> Material:
    return Material(200.0e9, 0.3, yield_stress=250.0e6, name="perfectly plastic")
