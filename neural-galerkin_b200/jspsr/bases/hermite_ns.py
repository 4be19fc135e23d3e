"""Additive basis with polynomial part constrained to vanish with its derivative at +-1.5
(reference: ``jspsr/bases/hermite_ns.py:7-80``): the Neural Galerkin learned basis."""
import numpy as np
import torch
from scipy.linalg import null_space

from .additive import AdditiveBasis
from .additive_components import Power


def _get_ns(n_degrees):
    """Rows: a basis of the polynomials of degree <= n_degrees (ascending coefficients) with
    b(+-1.5) = b'(+-1.5) = 0."""
    cols = []
    for deg in range(n_degrees, -1, -1):          # descending degree, as the constraint matrix columns
        cols.append([1.5 ** deg, (-1.5) ** deg, deg * 1.5 ** (deg - 1) if deg else 0.0,
                     deg * (-1.5) ** (deg - 1) if deg else 0.0])
    a = np.asarray(cols).T
    return null_space(a)[::-1].T


class AdditiveHermite(AdditiveBasis):
    def __init__(self, n_degrees, components, init_vals):
        if n_degrees <= 3:
            raise ValueError(f"a polynomial part of degree {n_degrees} leaves no freedom once value and slope "
                             "vanish at both ends; use degree 4 or more")
        comps = list(components)
        super().__init__(comps + [Power(p) for p in range(n_degrees + 1)],
                         list(init_vals) + [0.0] * (n_degrees + 1))
        self.n_degrees = n_degrees
        self.n_acomp = len(comps)
        ns = torch.from_numpy(_get_ns(n_degrees).copy()).float()
        self.register_buffer("ns", torch.kron(ns, torch.eye(3)))

    def feature_to_coefficient(self, feat: torch.Tensor) -> torch.Tensor:
        k = 3 * self.n_acomp
        ns = self.ns if self.ns.device == feat.device else self.ns.to(feat.device)
        return torch.cat([feat[:, :k], feat[:, k:] @ ns], dim=1)

    def initialize_feature_value(self, feat: torch.Tensor) -> None:
        assert feat.size(1) == self.get_feature_size()
        for ci in range(self.n_acomp):
            feat[:, 3 * ci:3 * ci + 3] = self.init_vals[ci]
        ns4 = _get_ns(4)
        target = np.zeros(self.n_degrees + 1)
        target[[0, 2, 4]] = ns4[0, [0, 2, 4]]
        w = np.linalg.lstsq(_get_ns(self.n_degrees).T, target, rcond=None)[0]
        base = 3 * self.n_acomp
        for k, v in enumerate(w):
            feat[:, base + 3 * k:base + 3 * k + 3] = float(v)

    def get_feature_size(self) -> int:
        return 3 * self.n_acomp + self.ns.size(0)
