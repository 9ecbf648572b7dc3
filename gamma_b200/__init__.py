"""B200-native moving-mesh relativistic hydro step (the GAMMA 1D track path).

``gpu`` binds the C ABI of include/gamma_gpu.h; ``problems`` builds initial
tracks on the host.  The step runs only as sm_100a CUDA (gamma_b200/lib).
"""
from . import gpu, problems  # noqa: F401
