"""Elementary 1-D functions q(x) of the additive (learned) basis, supported on [-1.5, 1.5)
(reference: ``jspsr/bases/additive_components.py:7-164``).

Each component provides torch evaluation (values and derivatives for the solver), numpy
evaluation plus breakpoints (for the integral tables), and a sympy form (``symbolic``)
for callers that want the closed expression.
"""
import math
from abc import ABC, abstractmethod

import numpy as np
import torch


def _inside(x):
    return (x >= -1.5) & (x < 1.5)


class AdditiveComponent(ABC):
    breaks = (-1.5, 1.5)

    @abstractmethod
    def __repr__(self):
        """Name used to identify the component's integral tables."""

    @abstractmethod
    def evaluate(self, xyz: torch.Tensor) -> torch.Tensor:
        """q(x), elementwise (no support mask: callers evaluate inside the support)."""

    @abstractmethod
    def evaluate_derivative(self, xyz: torch.Tensor) -> torch.Tensor:
        """q'(x), elementwise."""

    @abstractmethod
    def f(self, x: np.ndarray) -> np.ndarray:
        """q(x) with the support mask, numpy."""

    @abstractmethod
    def df(self, x: np.ndarray) -> np.ndarray:
        """q'(x) with the support mask, numpy."""

    def symbolic(self, x):
        import sympy as sp
        return sp.Piecewise((0, x < -1.5), (self._sym(x), x < 1.5), (0, True))


class Product(AdditiveComponent):
    """q(x) = a(x) * b(x)."""

    def __init__(self, ca, cb):
        self.ca, self.cb = ca, cb
        self.breaks = tuple(sorted(set(ca.breaks) | set(cb.breaks)))

    def __repr__(self):
        return f"Product({self.ca}|{self.cb})"

    def evaluate(self, xyz):
        return self.ca.evaluate(xyz) * self.cb.evaluate(xyz)

    def evaluate_derivative(self, xyz):
        return self.ca.evaluate(xyz) * self.cb.evaluate_derivative(xyz) + \
            self.ca.evaluate_derivative(xyz) * self.cb.evaluate(xyz)

    def f(self, x):
        return self.ca.f(x) * self.cb.f(x)

    def df(self, x):
        return self.ca.f(x) * self.cb.df(x) + self.ca.df(x) * self.cb.f(x)

    def _sym(self, x):
        return self.ca._sym(x) * self.cb._sym(x)


class Power(AdditiveComponent):
    """q(x) = x ** p."""

    def __init__(self, power):
        self.power = power

    def __repr__(self):
        return f"Power({self.power:.2f})"

    def evaluate(self, xyz):
        return torch.ones_like(xyz) if self.power == 0 else xyz ** self.power

    def evaluate_derivative(self, xyz):
        if self.power == 0:
            return torch.zeros_like(xyz)
        if self.power == 1:
            return torch.ones_like(xyz)
        return self.power * xyz ** (self.power - 1)

    def f(self, x):
        return np.where(_inside(x), np.ones_like(x) if self.power == 0 else x ** self.power, 0.0)

    def df(self, x):
        if self.power == 0:
            return np.zeros_like(x)
        return np.where(_inside(x), self.power * x ** (self.power - 1) if self.power > 1 else np.ones_like(x), 0.0)

    def _sym(self, x):
        return x ** self.power


class Bezier(AdditiveComponent):
    """The quadratic B-spline (x2) of the fixed basis."""
    breaks = (-1.5, -0.5, 0.5, 1.5)

    def __repr__(self):
        return "Bezier()"

    def evaluate(self, xyz):
        return torch.where((xyz >= -1.5) & (xyz < -0.5), (xyz + 1.5) ** 2,
               torch.where((xyz >= -0.5) & (xyz < 0.5), 1.5 - 2 * xyz ** 2,
               torch.where((xyz >= 0.5) & (xyz < 1.5), (xyz - 1.5) ** 2, torch.zeros_like(xyz))))

    def evaluate_derivative(self, xyz):
        return torch.where((xyz >= -1.5) & (xyz < -0.5), 2 * xyz + 3,
               torch.where((xyz >= -0.5) & (xyz < 0.5), -4 * xyz,
               torch.where((xyz >= 0.5) & (xyz < 1.5), 2 * xyz - 3, torch.zeros_like(xyz))))

    def f(self, x):
        return np.where((x >= -1.5) & (x < -0.5), (x + 1.5) ** 2,
               np.where((x >= -0.5) & (x < 0.5), 1.5 - 2 * x * x,
               np.where((x >= 0.5) & (x < 1.5), (x - 1.5) ** 2, 0.0)))

    def df(self, x):
        return np.where((x >= -1.5) & (x < -0.5), 2 * x + 3,
               np.where((x >= -0.5) & (x < 0.5), -4 * x,
               np.where((x >= 0.5) & (x < 1.5), 2 * x - 3, 0.0)))

    def symbolic(self, x):
        import sympy as sp
        return sp.Piecewise((0, x < -1.5), ((x + 1.5) ** 2, x < -0.5), (-2 * x ** 2 + 1.5, x < 0.5),
                            ((x - 1.5) ** 2, x < 1.5), (0, True))


class Sinusoid(AdditiveComponent):
    """q(x) = sin(beta x + gamma)."""

    def __init__(self, beta, gamma):
        self.beta, self.gamma = beta, gamma

    def __repr__(self):
        return f"Sin({self.beta:.2f}-{self.gamma:.2f})"

    def evaluate(self, xyz):
        return torch.sin(self.beta * xyz + self.gamma)

    def evaluate_derivative(self, xyz):
        return self.beta * torch.cos(self.beta * xyz + self.gamma)

    def f(self, x):
        return np.where(_inside(x), np.sin(self.beta * x + self.gamma), 0.0)

    def df(self, x):
        return np.where(_inside(x), self.beta * np.cos(self.beta * x + self.gamma), 0.0)

    def _sym(self, x):
        import sympy as sp
        return sp.sin(self.beta * x + self.gamma)


class SinPeaks(Sinusoid):
    """Sinusoid with n half-periods over the support (zero at both ends for odd patterns)."""

    def __init__(self, n_peaks):
        super().__init__(math.pi * n_peaks / 3, -0.5 * math.pi * n_peaks + math.pi)
        self.n_peaks = n_peaks

    def __repr__(self):
        return f"SinPeaks({self.n_peaks})"
