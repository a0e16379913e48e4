// bh_fp64fma.cu -- the same FP64 kernels with fused multiply-add
// contraction (compiled with --fmad=true): fewer instructions, results that
// differ from the reference's in the last bits.
#define BH_VARIANT vfma
#define BH_RCP   // reciprocals formed once for repeated divisors (quo)
#include "bh_variant.cuh"
