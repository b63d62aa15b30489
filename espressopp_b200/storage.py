"""storage.DomainDecomposition."""
from .core import DomainDecomposition  # noqa: F401
