"""The host-side patch quilt, kept in the CUDA-free package ``bhgrid``."""
from bhgrid.mesh import *  # noqa: F401,F403
from bhgrid.mesh import (BLOCK, CPN, GHOST, NB_BNDY, NB_COPY, NB_PROLONG, NC, NE, NF, Patch, Quilt,  # noqa: F401
                         RegridPlan, cell_index, interior_mask, xface_index, yface_index, zface_index)
