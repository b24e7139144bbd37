"""Reference-compatible module name: re-exports vfs_b200.icra_dataset."""
from vfs_b200.icra_dataset import dataset_loader, read_flo, write_flo, write_sample  # noqa: F401
