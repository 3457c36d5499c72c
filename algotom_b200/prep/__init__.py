"""Pre-processing functions (drop-in for ``algotom.prep``)."""
from . import conversion  # noqa: F401
