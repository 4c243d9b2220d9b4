"""Import-path compatibility for the reference package name (wp_sph/__init__.py:1)."""
from . import solver  # noqa: F401
