"""Bases of the Galerkin solver (reference: ``jspsr/bases/__init__.py``)."""


def get_basis(name, **kwargs):
    """Basis instance by name: ``BezierTensorBasis`` or ``AdditiveHermite``."""
    if name == "BezierTensorBasis":
        from .bezier_tensor import BezierTensorBasis
        return BezierTensorBasis()
    if name == "AdditiveHermite":
        from .hermite_ns import AdditiveHermite
        return AdditiveHermite(**kwargs)
    raise NotImplementedError(name)
