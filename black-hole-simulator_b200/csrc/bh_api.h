// bh_api.h -- the launch sequences each arithmetic variant provides
// (defined in bh_variant.cuh, instantiated by bh_fp64.cu, bh_fp64fma.cu and
// bh_mixed.cu)
#pragma once
#include <stdint.h>
#include "bhgpu.h"

// launch-bound candidates of the tuned kernels (BH_TUNE_*), zero-terminated;
// bh_variant.cuh instantiates each kernel for exactly its list
constexpr int32_t bh_tune_cands[BH_TUNE_NKERNEL][5] = {
    {3, 4, 5, 6, 0}, {3, 4, 5, 6, 0}, {4, 6, 8, 0, 0}, {4, 6, 8, 0, 0}, {4, 6, 8, 0, 0}};
inline bool bh_tune_valid(int32_t kernel, int32_t ctas) {
    if (kernel < 0 || kernel >= BH_TUNE_NKERNEL) return false;
    for (int i = 0; i < 5 && bh_tune_cands[kernel][i]; i++)
        if (bh_tune_cands[kernel][i] == ctas) return true;
    return false;
}

#define BH_VARIANT_API(NS)                                                                                       \
    namespace NS {                                                                                              \
    int metric_comp(const bh_params*, const double*, const double*, int64_t, double*, void*);                  \
    int ptoc(const bh_params*, const double*, const double*, const double*, int64_t, double*, double*, void*);  \
    int ctop(const bh_params*, const double*, const double*, const double*, int64_t, double*, double*, int32_t*, \
             int32_t*, int32_t*, void*);                                                                        \
    int hlld(const bh_params*, const double*, const double*, const double*, const double*, const double*,      \
             const double*, int32_t, int64_t, double*, double*, void*);                                         \
    int geometry(const bh_pool*, void*);                                                                        \
    int reconfp(const bh_params*, const bh_pool*, int32_t, int32_t, double*, double*, void*);                  \
    int fluxcomp(const bh_params*, const bh_pool*, void*);                                                     \
    int emfcomp(const bh_pool*, void*);                                                                         \
    int bfupdate(const bh_pool*, const double*, void*);                                                        \
    int f2cb(const bh_params*, const bh_pool*, void*);                                                         \
    int maxdivb(const bh_pool*, double*, void*);                                                                \
    int div_source(const bh_params*, const bh_pool*, double*, double*, void*);                                 \
    int ghosts(const bh_params*, const bh_pool*, const int32_t*, int32_t, void*);                              \
    int prims(const bh_params*, const bh_pool*, void*);                                                        \
    int ghosts_prims_status(const bh_params*, const bh_pool*, uint8_t*, void*);                                \
    int ghosts_prims(const bh_params*, const bh_pool*, void*);                                                 \
    int update(const bh_params*, const bh_pool*, const double*, int32_t, void*);                               \
    int floors(const bh_params*, const bh_pool*, void*);                                                       \
    int dtcomp(const bh_params*, const bh_pool*, double, double*, void*);                                      \
    int regrid_flags(const bh_params*, const bh_pool*, const int32_t*, uint8_t*, void*);                       \
    int analysis(const bh_params*, const bh_pool*, const bh_analysis_params*, double*, double*, void*);       \
    int torus_init(const bh_params*, const bh_pool*, double, double, double*, void*);                          \
    int ctop_guess(const bh_params*, const double*, const double*, const double*, int64_t, const double*,      \
                   double*, double*, int32_t*, int32_t*, int32_t*, void*);                                     \
    int ctop_pre(const bh_params*, const double*, const double*, const double*, int64_t, double*, void*);    \
    int tune_set(int32_t, int32_t);                                                                         \
    int tune_get(int32_t, int32_t*);                                                                        \
    int ctop_learned(const bh_params*, const bh_mlp*, const double*, const double*, const double*, int64_t,   \
                     double*, double*, double*, int32_t*, int32_t*, int32_t*, int32_t*, void*);               \
    int refine(const bh_params*, const bh_pool*, const int32_t*, int32_t, void*);                              \
    int ccrstr(const bh_params*, const bh_pool*, const int32_t*, int32_t, void*);                              \
    int b_init(const bh_params*, const bh_pool*, const int32_t*, int32_t, void*);                              \
    int rkstg(const bh_params*, const bh_pool*, const double*, int32_t, const int32_t*, const int32_t*, int32_t, \
              void*);                                                                                           \
    int step(const bh_params*, const bh_pool*, double, double*, const int32_t*, const int32_t*, int32_t, void*); \
    int fx_prims(const bh_fx_params*, const bh_fx_grid*, int32_t, int32_t, void*);                           \
    int fx_ghosts(const bh_fx_params*, const bh_fx_grid*, int32_t, void*);                                    \
    int fx_ghost_pass(const bh_fx_params*, const bh_fx_grid*, int32_t, int32_t, void*);                       \
    int fx_fluxes(const bh_fx_params*, const bh_fx_grid*, int32_t, void*);                                    \
    int fx_update(const bh_fx_params*, const bh_fx_grid*, int32_t, void*);                                    \
    int fx_update_parts(const bh_fx_params*, const bh_fx_grid*, int32_t, int32_t, void*);                     \
    int fx_step(const bh_fx_params*, const bh_fx_grid*, void*);                                               \
    int fx_divb(const bh_fx_grid*, double*, void*);                                                           \
    int fx_pack_state(const bh_fx_grid*, const int64_t*, void*, int32_t, void*);                              \
    int fx_torus_init(const bh_fx_params*, const bh_fx_grid*, const bh_fx_torus*, double*, double*, void*);   \
    int fx_tune_set(int32_t, int32_t);                                                                        \
    int fx_tune_get(int32_t, int32_t*);                                                                       \
    }

BH_VARIANT_API(vfp64)
BH_VARIANT_API(vfma)
BH_VARIANT_API(vmixed)
