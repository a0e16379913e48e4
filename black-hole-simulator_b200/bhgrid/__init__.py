"""bhgrid -- host-side tables and seeded workloads of the GRMHD block update.

Pure numpy: the patch quilt (geometry, neighbour table, ghost-fill order,
amrtree's bookkeeping) and the synthetic inputs.  Importing it loads no CUDA
library, so CPU-only callers (the timed reference arm, the oracle harness)
can build the same inputs the GPU path consumes.
"""
from .mesh import Quilt, BLOCK, GHOST, CPN, NC, NF, NE  # noqa: F401
from . import configs  # noqa: F401
