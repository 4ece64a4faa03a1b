"""Term algebra of fvm::terms, restricted to what the device assembly runs.

Mirrors src/fvm/terms/mod.rs:24-40 (Term), operations.rs:86-199 (+, -, unary
-), laplacian.rs:21 (laplacian), convection.rs:24 (convection),
source.rs:22 (source), with the schemes facengrad::Orthogonal
(orthogonal.rs:26-46), facengrad::Corrected (corrected.rs:36-67) and
faceinterp::Upwind (upwind.rs:26-33).

An expression is kept as a signed combination of at most one laplacian, one
convection and one source term, which is exactly what the term tree computes:
every value is a sum of +/- the individual terms.  The transient and extra
terms time (Euler / Backward), linear_source and divergence are kept the same
way.  Anything else (Linear/LimitedLinear interpolation in convection)
raises NotImplementedError at construction.
"""
from __future__ import annotations

from dataclasses import dataclass, field


class Orthogonal:
    """facengrad::Orthogonal: two-point flux gradient 1/|c_j - c_i|."""


class Corrected:
    """facengrad::Corrected(gradients, corrector_reduction): coefficient
    1/(n.d) plus the explicit non-orthogonal correction from the cell
    gradients (a DistributedVector / array of n_cells*dim, e.g. filled by
    compute_gradients); corrector_reduction 0 = none ... 1 = full."""

    def __init__(self, gradients, corrector_reduction: float = 1.0):
        self.gradients = gradients
        self.corrector_reduction = float(corrector_reduction)


class Upwind:
    """faceinterp::Upwind(flux)."""

    def __init__(self, flux):
        self.flux = flux


class Linear:  # pragma: no cover - name kept for API parity
    def __init__(self, *a, **k):
        raise NotImplementedError("faceinterp::Linear is not implemented on the device path")


@dataclass
class TermExpr:
    """Signed combination c_lap*laplacian + c_conv*convection + c_src*source."""

    coef: dict = field(default_factory=dict)   # kind -> +/-1
    data: dict = field(default_factory=dict)   # kind -> field array

    def _combine(self, other: "TermExpr", sign: float) -> "TermExpr":
        if not isinstance(other, TermExpr):
            return NotImplemented
        coef = dict(self.coef)
        data = dict(self.data)
        for k, c in other.coef.items():
            if k in coef:
                raise NotImplementedError(f"two {k} terms in one expression")
            coef[k] = sign * c
            data[k] = other.data[k]
            if k + "_scheme" in other.data:
                data[k + "_scheme"] = other.data[k + "_scheme"]
        return TermExpr(coef, data)

    def __add__(self, other):
        return self._combine(other, 1.0)

    def __sub__(self, other):
        return self._combine(other, -1.0)

    def __neg__(self):
        return TermExpr({k: -c for k, c in self.coef.items()}, dict(self.data))

    def coefficients(self):
        return (self.coef.get("laplacian", 0.0), self.coef.get("convection", 0.0), self.coef.get("source", 0.0))

    def coefficient(self, kind: str) -> float:
        return self.coef.get(kind, 0.0)


def laplacian(scheme, diffusivity) -> TermExpr:
    if not isinstance(scheme, (Orthogonal, Corrected)):
        raise NotImplementedError("only facengrad::Orthogonal and facengrad::Corrected run on the device")
    return TermExpr({"laplacian": 1.0}, {"laplacian": diffusivity, "laplacian_scheme": scheme})


def convection(scheme, flux) -> TermExpr:
    if not isinstance(scheme, Upwind):
        raise NotImplementedError("only faceinterp::Upwind runs on the device")
    if scheme.flux is not flux:
        raise NotImplementedError("Upwind must use the convected flux field")
    return TermExpr({"convection": 1.0}, {"convection": flux})


def source(values) -> TermExpr:
    return TermExpr({"source": 1.0}, {"source": values})


class Euler:
    """schemes::time::Euler (euler.rs): cell lhs (1/dt) rho, rhs previous/dt rho_previous."""

    def __init__(self, previous, dt: float, density=None, density_previous=None):
        if (density is None) != (density_previous is None):
            raise ValueError("Euler: give both densities or neither")
        self.previous, self.dt = previous, float(dt)
        self.densities = None if density is None else (density, density_previous)


class Backward:
    """schemes::time::Backward (backward.rs): second-order backward difference
    with variable step (dt now, dt_2 the previous step)."""

    def __init__(self, previous, previous_2, dt: float, dt_2: float, densities=None):
        self.previous, self.previous_2, self.dt, self.dt_2 = previous, previous_2, float(dt), float(dt_2)
        if densities is not None and len(densities) != 3:
            raise ValueError("Backward: densities = (now, previous, previous_2)")
        self.densities = densities


def time(scheme) -> TermExpr:
    """terms::time (time.rs:19-35) with Euler or Backward."""
    if not isinstance(scheme, (Euler, Backward)):
        raise NotImplementedError("terms::time runs with schemes::time::Euler or Backward")
    return TermExpr({"time": 1.0}, {"time": scheme})


def linear_source(coefficients) -> TermExpr:
    """terms::linear_source (source.rs:61-79): cell lhs = coefficient."""
    return TermExpr({"linear_source": 1.0}, {"linear_source": coefficients})


def divergence(flux) -> TermExpr:
    """terms::divergence (divergence.rs:22-43): face rhs -flux."""
    return TermExpr({"divergence": 1.0}, {"divergence": flux})
