"""The seeded workloads, kept in the CUDA-free package ``bhgrid``."""
from bhgrid.configs import *  # noqa: F401,F403
from bhgrid.configs import con2prim_batch, magnetised_box  # noqa: F401
