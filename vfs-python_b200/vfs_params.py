"""Reference-compatible module name: re-exports vfs_b200.vfs_params."""
from vfs_b200.vfs_params import vfs_params  # noqa: F401
