"""Reference-compatible module name: re-exports vfs_b200.texture."""
from vfs_b200.texture import create_texture_object  # noqa: F401
