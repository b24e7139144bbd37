"""Test infrastructure: the checkers for the B200 stereo path.

Nothing in the product imports this package.  ``oracle.np64`` is a float64
NumPy restatement of the reference algorithm; ``oracle.refgpu`` drives the
reference's own CUDA kernels (built from the reference sources into
``oracle/_ref``) with the reference's host-side call order.
"""
