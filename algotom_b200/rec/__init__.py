"""Reconstruction functions (drop-in for ``algotom.rec.reconstruction``)."""
from . import reconstruction  # noqa: F401
