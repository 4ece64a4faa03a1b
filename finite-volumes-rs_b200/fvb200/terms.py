"""Term algebra of fvm::terms, restricted to what the device assembly runs.

Mirrors src/fvm/terms/mod.rs:24-40 (Term), operations.rs:86-199 (+, -, unary
-), laplacian.rs:21 (laplacian), convection.rs:24 (convection),
source.rs:22 (source), with the schemes facengrad::Orthogonal
(orthogonal.rs:26-46), facengrad::Corrected (corrected.rs:36-67) and
faceinterp::Upwind (upwind.rs:26-33).

An expression is kept as a signed combination of at most one laplacian, one
convection and one source term, which is exactly what the term tree computes:
every value is a sum of +/- the individual terms.  Anything else
(Linear/LimitedLinear interpolation in convection, time, divergence,
linear_source) raises NotImplementedError at construction.
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


def time(*a, **k):  # pragma: no cover - name kept for API parity
    raise NotImplementedError("terms::time is not implemented on the device path")


def divergence(*a, **k):  # pragma: no cover
    raise NotImplementedError("terms::divergence is not implemented on the device path")


def linear_source(*a, **k):  # pragma: no cover
    raise NotImplementedError("terms::linear_source is not implemented on the device path")
