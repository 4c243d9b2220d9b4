"""``wp_sph.solver.IISPH`` (wp_sph/solver/__init__.py:1), backed by libwpsph.so."""
from warpsph_b200.solver import IISPH  # noqa: F401
