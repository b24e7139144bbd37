"""Reference-compatible module name: re-exports vfs_b200.vfs."""
from vfs_b200.vfs import VFS  # noqa: F401
