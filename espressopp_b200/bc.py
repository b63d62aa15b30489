"""bc.OrthorhombicBC."""
from .core import OrthorhombicBC  # noqa: F401
