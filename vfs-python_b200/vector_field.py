"""Reference-compatible module name: re-exports vfs_b200.vector_field."""
from vfs_b200.vector_field import get_vector_fields, get_grid_zero, get_grid_one, default_normalizer  # noqa: F401
