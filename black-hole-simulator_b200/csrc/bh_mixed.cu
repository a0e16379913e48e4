// bh_mixed.cu -- the mixed-precision variant: reconstruction, face ptoc,
// HLLD and the geometric source in FP32; the metric (evaluated in FP64 and
// rounded), constrained transport, the flux divergence, the RK combine and
// con2prim stay FP64.  Compiled with FMA contraction and fast FP32
// division/square root; logf/expf keep their full accuracy.
#define BH_VARIANT vmixed
#define BH_RCP   // reciprocals formed once for repeated divisors (quo)
#define BH_REAL float
#define BH_MINB_FLUX 6   // the FP32 face computation needs fewer registers
#include "bh_variant.cuh"
