"""nessi_b200: B200-native Kadanoff-Baym time stepping (libcntr hot path)."""
from .herm_matrix import herm_matrix, function, distance_norm2  # noqa: F401
