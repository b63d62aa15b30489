"""esutil.RNG."""
from .core import RNG  # noqa: F401
