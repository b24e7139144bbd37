"""Reference-compatible module name: re-exports vfs_b200.colormap."""
from vfs_b200.colormap import colormap, depth_to_colormap, jet  # noqa: F401
