"""Fixed quadratic B-spline tensor basis (reference: ``jspsr/bases/bezier_tensor.py:11-128``).

B(x) = (x+1.5)^2 on [-1.5,-0.5), 1.5-2x^2 on [-0.5,0.5), (x-1.5)^2 on [0.5,1.5); the 3-D basis
is the product over axes.  Galerkin integrals are separable and come from exact 1-D tables
(``jspsr.bases.tables``), which replace the reference's unpublished ``bezier_integrals.pkl``.
"""
import torch

from .abc import BaseBasis
from . import tables as T


def _pieces(x):
    return ((x >= -1.5) & (x < -0.5), (x >= -0.5) & (x < 0.5), (x >= 0.5) & (x < 1.5))


class BezierTensorBasis(BaseBasis):
    _cache = {}

    @classmethod
    def _table(cls, name, m, device):
        key = (name, m, str(device))
        if key not in cls._cache:
            src = {"ssi": lambda: T.shifted(m)[0], "sdi": lambda: T.shifted(m)[1],
                   "dpi": lambda: T.partial(m)[0], "pi": lambda: T.partial(m)[1],
                   "idpi": lambda: T.inverse_partial(m)[0], "ipi": lambda: T.inverse_partial(m)[1]}[name]()
            cls._cache[key] = torch.tensor(src, dtype=torch.float32, device=device)
        return cls._cache[key]

    @classmethod
    def evaluate_single(cls, x):
        a, b, c = _pieces(x)
        return a * (x + 1.5) ** 2 + b * (-2 * x ** 2 + 1.5) + c * (x - 1.5) ** 2

    @classmethod
    def evaluate_derivative_single(cls, x):
        a, b, c = _pieces(x)
        return a * (2 * x + 3) + b * (-4 * x) + c * (2 * x - 3)

    def evaluate(self, feat, xyz, feat_ids):
        return self.evaluate_single(xyz[..., 0]) * self.evaluate_single(xyz[..., 1]) * \
            self.evaluate_single(xyz[..., 2])

    def evaluate_derivative(self, feat, xyz, feat_ids, stride: int):
        b = [self.evaluate_single(xyz[..., i]) for i in range(3)]
        d = [self.evaluate_derivative_single(xyz[..., i]) / stride for i in range(3)]
        return torch.stack([d[0] * b[1] * b[2], b[0] * d[1] * b[2], b[0] * b[1] * d[2]], dim=1)

    def integrate_deriv_deriv_product(self, rel_pos, source_stride: int, target_stride: int, **kwargs):
        assert source_stride <= target_stride, "Source stride cannot be larger than target stride."
        M = target_stride // source_stride
        m = T.ratio_log2(M)
        idx = (rel_pos + 1.5 * M + 0.5).round().long()
        ssi, sdi = self._table("ssi", m, rel_pos.device), self._table("sdi", m, rel_pos.device)
        ok = (idx >= 0) & (idx < ssi.numel())
        idx = idx.clamp(0, ssi.numel() - 1)
        c = torch.where(ok, ssi[idx] * source_stride, torch.zeros((), device=rel_pos.device))
        g = torch.where(ok, sdi[idx] / target_stride, torch.zeros((), device=rel_pos.device))
        return g[:, 0] * c[:, 1] * c[:, 2] + c[:, 0] * g[:, 1] * c[:, 2] + c[:, 0] * c[:, 1] * g[:, 2]

    def integrate_const_deriv_product(self, data, rel_pos, data_stride: int, target_stride: int, **kwargs):
        dev = rel_pos.device
        if target_stride >= data_stride:
            M = target_stride // data_stride
            idx = (rel_pos + (3 * M - 1) / 2.0).round().long()
            m = T.ratio_log2(M)
            c = self._table("dpi", m, dev)[idx] * data_stride
            g = self._table("pi", m, dev)[idx] * (data_stride / target_stride)
        else:
            M = data_stride // target_stride
            idx = (rel_pos * M + M / 2 + 0.5).round().long()
            m = T.ratio_log2(M)
            c = self._table("idpi", m, dev)[idx] * target_stride
            g = self._table("ipi", m, dev)[idx]
        return data[:, 0] * g[:, 0] * c[:, 1] * c[:, 2] + data[:, 1] * c[:, 0] * g[:, 1] * c[:, 2] + \
            data[:, 2] * c[:, 0] * c[:, 1] * g[:, 2]

    def initialize_feature_value(self, feat) -> None:
        pass
