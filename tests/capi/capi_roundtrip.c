/* A plain C99 caller of the library: only include/bhgpu.h and the CUDA
 * runtime's C API.  Without arguments it makes host-only calls (the ABI
 * version, the tuning table); with "gpu" it converts n static primitive
 * states to conserved variables (bh_ptoc) and back (bh_ctop) on the device
 * and prints the largest density error and the number of cells that did not
 * recover.  Test code only. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <cuda_runtime_api.h>
#include "bhgpu.h"

int main(int argc, char** argv) {
    int32_t cand[8];
    int nc = bh_tune_candidates(BH_TUNE_FLUX, cand, 8);
    printf("abi %d flux_candidates %d first %d\n", bh_abi_version(), nc, nc > 0 ? cand[0] : -1);
    if (argc < 2 || strcmp(argv[1], "gpu") != 0) return 0;
    enum { N = 4096 };
    static double hW[8 * N], hr[N], hth[N], hW2[8 * N];
    static int32_t hst[N];
    for (int q = 0; q < N; q++) {
        hW[q] = 1.0 + 1e-3 * (q % 17);        /* rho */
        hW[N + q] = 0.1 + 1e-4 * (q % 13);    /* eps */
        for (int v = 2; v < 8; v++) hW[v * N + q] = 0.0;
        hr[q] = 10.0 + 0.001 * q;
        hth[q] = 1.0 + 1e-4 * q;
    }
    double *W, *U, *r, *th, *W2;
    int32_t* st;
    if (cudaMalloc((void**)&W, sizeof hW) || cudaMalloc((void**)&U, sizeof hW) || cudaMalloc((void**)&W2, sizeof hW) ||
        cudaMalloc((void**)&r, sizeof hr) || cudaMalloc((void**)&th, sizeof hth) || cudaMalloc((void**)&st, sizeof hst))
        return 2;
    cudaMemcpy(W, hW, sizeof hW, cudaMemcpyHostToDevice);
    cudaMemcpy(r, hr, sizeof hr, cudaMemcpyHostToDevice);
    cudaMemcpy(th, hth, sizeof hth, cudaMemcpyHostToDevice);
    bh_params P;
    memset(&P, 0, sizeof P);
    P.M = 0.0; P.a = 0.0; P.Q = 0.0; P.gamma = 4.0 / 3.0; P.limiter = 1; P.maxiter = 500; P.tol = 1e-10;
    P.cM = 1.0; P.precision = BH_FP64;
    if (bh_ptoc(&P, W, r, th, N, U, NULL, NULL) != BH_OK) return 3;
    if (bh_ctop(&P, U, r, th, N, W2, NULL, st, NULL, NULL, NULL) != BH_OK) return 4;
    if (cudaDeviceSynchronize() != cudaSuccess) return 5;
    cudaMemcpy(hW2, W2, sizeof hW2, cudaMemcpyDeviceToHost);
    cudaMemcpy(hst, st, sizeof hst, cudaMemcpyDeviceToHost);
    double err = 0.0;
    int bad = 0;
    for (int q = 0; q < N; q++) {
        double e = fabs(hW2[q] - hW[q]) / hW[q];
        if (e > err) err = e;
        if (hst[q] != 1) bad++;
    }
    printf("rho_max_rel_err %.3e not_recovered %d\n", err, bad);
    cudaFree(W); cudaFree(U); cudaFree(W2); cudaFree(r); cudaFree(th); cudaFree(st);
    return 0;
}
