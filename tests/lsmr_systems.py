"""Seeded sparse least-squares systems shaped like DAzi's G matrix (the
generator lives in the package, dazi_current_release_b200.synthetic, so that
bench.py times the solver on the same kind of system)."""
from dazi_current_release_b200.synthetic import g_like_system  # noqa: F401
