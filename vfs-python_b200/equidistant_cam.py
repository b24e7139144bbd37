"""Reference-compatible module name: re-exports vfs_b200.equidistant_cam."""
from vfs_b200.equidistant_cam import EquidistantCam  # noqa: F401
