// bh_fp64.cu -- the reference-faithful variant: FP64 with the reference's
// separate multiply and add roundings (compiled with --fmad=false).
#define BH_VARIANT vfp64
#include "bh_variant.cuh"
