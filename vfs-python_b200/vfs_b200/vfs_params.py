"""Solver parameter bag, attribute-for-attribute the reference's
``vfs_params`` (Python/vfs_params.py:25-43).

Unlike the reference, which bakes most of these into the CUDA source as text
(Python/vfs.py:57-68), every value here reaches the kernels as a run-time
argument, so changing a parameter needs no recompilation.
"""


class vfs_params:
    def __init__(self, img=None):
        if img is None:
            self.width = 848
            self.height = 800
        else:
            self.width = img.shape[1]
            self.height = img.shape[0]
        self.beta = 9.0
        self.gamma = 0.85
        self.alpha0 = 17.0
        self.alpha1 = 1.2
        self.timeStepLambda = 1.0
        self.Lambda = 5.0
        self.nLevel = 11
        self.fScale = 1.2
        self.nWarpIters = 100
        self.nSolverIters = 100
        self.limitRange = 0.1
