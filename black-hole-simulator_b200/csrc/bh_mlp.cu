// bh_mlp.cu -- the learned con2prim initial guess: a 6 -> 64 -> 64 -> 2
// network (tanh hidden layers) mapping scale-free features of a cell's
// conserved state to y0 = log(xi / D) and y1 = log W (xi = rho h W^2, the
// unknown of conserved::ctop's Newton iteration, conserved.cpp:170-187).
// Inference reads BF16 weights and accumulates in FP32; training keeps FP32
// master weights, evaluates the forward pass with their BF16 roundings (the
// weights inference will see), back-propagates in FP32 and takes Adam steps.
// The solver's own FP64 con2prim produces the training pairs and still
// decides every cell: the guess only moves Newton's starting point.
//
// Parameters, FP32, one flat array (and its BF16 copy), in this order:
//   W1 [64][6], b1 [64], W2 [64][64], b2 [64], W3 [2][64], b3 [2]
// followed by 12 floats of feature normalisation (mean[6], 1/std[6]).
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <math.h>
#include "bhgpu.h"
#include "bh_tc.cuh"

namespace {

constexpr int NI = 6, NH = 64, NO = 2;
constexpr int OW1 = 0, OB1 = OW1 + NH * NI, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH,
              OB3 = OW3 + NO * NH, NPAR = OB3 + NO, ONORM = NPAR;
static_assert(NPAR == BH_MLP_NPARAM, "parameter count");
constexpr int TPB = 128;

inline cudaStream_t S(void* s) { return (cudaStream_t)s; }
inline int launched() { return cudaGetLastError() == cudaSuccess ? BH_OK : BH_ECUDA; }

// features of cell q from the con2prim preamble pre [5][n] and r
__device__ inline void features(const double* pre, const double* r, int64_t n, int64_t q, float x[NI]) {
    double p5[5] = {pre[q], pre[n + q], pre[2 * n + q], pre[3 * n + q], pre[4 * n + q]};
    bh_tc::features(p5, r[q], x);
}

__device__ inline float bf(__nv_bfloat16 v) { return __bfloat162float(v); }

// inference: xi0 = D exp(y0); NaN where a feature is not finite
__global__ void k_guess(const __nv_bfloat16* wb, const float* norm, const double* pre, const double* r, int64_t n,
                        double* xi0) {
    int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    float x[NI], h1[NH], h2[NH], y[NO];
    features(pre, r, n, q, x);
    bool ok = true;
    for (int i = 0; i < NI; i++) ok &= isfinite(x[i]);
    if (!ok) { xi0[q] = NAN; return; }
    float xn[NI];
    for (int i = 0; i < NI; i++) xn[i] = (x[i] - norm[i]) * norm[NI + i];
    for (int j = 0; j < NH; j++) {
        float a = bf(wb[OB1 + j]);
        for (int i = 0; i < NI; i++) a += bf(wb[OW1 + j * NI + i]) * xn[i];
        h1[j] = tanhf(a);
    }
    for (int j = 0; j < NH; j++) {
        float a = bf(wb[OB2 + j]);
        for (int i = 0; i < NH; i++) a += bf(wb[OW2 + j * NH + i]) * h1[i];
        h2[j] = tanhf(a);
    }
    for (int o = 0; o < NO; o++) {
        float a = bf(wb[OB3 + o]);
        for (int i = 0; i < NH; i++) a += bf(wb[OW3 + o * NH + i]) * h2[i];
        y[o] = a;
    }
    xi0[q] = pre[q] * exp((double)y[0]);
}

// training: forward with the BF16 roundings of the FP32 weights, loss
// L = mean over cells of sum_o (y_o - t_o)^2, and the per-cell factors the
// weight gradients need: act0 = x (normalised), act1 = h1, act2 = h2,
// d1 = dL/d(pre-activation 1), d2 = dL/d(pre-activation 2), d3 = dL/dy
__global__ void k_train_fwd_bwd(const __nv_bfloat16* wb, const float* norm, const double* pre, const double* r,
                                const float* target, int64_t n, float* act0, float* act1, float* act2, float* d1,
                                float* d2, float* d3, float* loss) {
    int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    float x[NI], h1[NH], h2[NH], y[NO];
    features(pre, r, n, q, x);
    float xn[NI];
    for (int i = 0; i < NI; i++) xn[i] = (x[i] - norm[i]) * norm[NI + i];
    for (int j = 0; j < NH; j++) {
        float a = bf(wb[OB1 + j]);
        for (int i = 0; i < NI; i++) a += bf(wb[OW1 + j * NI + i]) * xn[i];
        h1[j] = tanhf(a);
    }
    for (int j = 0; j < NH; j++) {
        float a = bf(wb[OB2 + j]);
        for (int i = 0; i < NH; i++) a += bf(wb[OW2 + j * NH + i]) * h1[i];
        h2[j] = tanhf(a);
    }
    float dy[NO], l = 0.0f;
    for (int o = 0; o < NO; o++) {
        float a = bf(wb[OB3 + o]);
        for (int i = 0; i < NH; i++) a += bf(wb[OW3 + o * NH + i]) * h2[i];
        y[o] = a;
        float e = y[o] - target[o * n + q];
        l += e * e;
        dy[o] = 2.0f * e / (float)n;
    }
    loss[q] = l;
    float g2[NH];
    for (int i = 0; i < NH; i++) {
        float a = 0.0f;
        for (int o = 0; o < NO; o++) a += bf(wb[OW3 + o * NH + i]) * dy[o];
        g2[i] = a * (1.0f - h2[i] * h2[i]);
    }
    for (int i = 0; i < NH; i++) {
        float a = 0.0f;
        for (int j = 0; j < NH; j++) a += bf(wb[OW2 + j * NH + i]) * g2[j];
        d1[i * n + q] = a * (1.0f - h1[i] * h1[i]);
        d2[i * n + q] = g2[i];
        act1[i * n + q] = h1[i];
        act2[i * n + q] = h2[i];
    }
    for (int i = 0; i < NI; i++) act0[i * n + q] = xn[i];
    for (int o = 0; o < NO; o++) d3[o * n + q] = dy[o];
}

// grad[off + j*K + i] = sum_q delta[j][q] act[i][q] (and the bias sums), one
// thread per weight, the cells in order
__global__ void k_wgrad(const float* delta, const float* act, int64_t n, int J, int K, float* grad, int offW,
                        int offB) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < J * K) {
        int j = t / K, i = t % K;
        float s = 0.0f;
        for (int64_t q = 0; q < n; q++) s += delta[j * n + q] * act[i * n + q];
        grad[offW + t] = s;
    } else if (t < J * K + J) {
        int j = t - J * K;
        float s = 0.0f;
        for (int64_t q = 0; q < n; q++) s += delta[j * n + q];
        grad[offB + j] = s;
    }
}

// Adam step (Kingma & Ba 2015) on the FP32 master weights, then their BF16 copy
__global__ void k_adam(float* w, const float* g, float* m, float* v, __nv_bfloat16* wb, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= NPAR) return;
    float gi = g[t];
    float mi = b1 * m[t] + (1.0f - b1) * gi;
    float vi = b2 * v[t] + (1.0f - b2) * gi * gi;
    m[t] = mi; v[t] = vi;
    w[t] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    wb[t] = __float2bfloat16_rn(w[t]);
}
__global__ void k_to_bf16(const float* w, __nv_bfloat16* wb) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < NPAR) wb[t] = __float2bfloat16_rn(w[t]);
}
__global__ void k_sum(const float* x, int64_t n, float* out) {
    __shared__ float red[256];
    float s = 0.0f;
    for (int64_t q = threadIdx.x; q < n; q += 256) s += x[q];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// the bounded wait of the tensor-core kernels on an mbarrier that nothing
// arrives on: it must give up and report, never hang
__global__ void k_wait_selftest(int32_t* err) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) bh_tc::mbar_init(&bar);
    __syncthreads();
    bool ok = bh_tc::mbar_wait(&bar, 0);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(err, BH_ERR_TIMEOUT);
}

}  // namespace

extern "C" {

int bh_wait_selftest(int32_t* err, void* stream) {
    if (!err) return BH_EINVAL;
    k_wait_selftest<<<1, 32, 0, S(stream)>>>(err);
    return launched();
}

int bh_mlp_sync_bf16(bh_mlp* m, void* stream) {
    if (!m || !m->w || !m->wb) return BH_EINVAL;
    k_to_bf16<<<(NPAR + 255) / 256, 256, 0, S(stream)>>>(m->w, (__nv_bfloat16*)m->wb);
    return launched();
}

int bh_mlp_guess(const bh_mlp* m, const double* pre, const double* r, int64_t n, double* xi0, void* stream) {
    if (!m || !m->wb || !pre || !r || !xi0 || n < 0) return BH_EINVAL;
    if (n == 0) return BH_OK;
    k_guess<<<(unsigned)((n + TPB - 1) / TPB), TPB, 0, S(stream)>>>((const __nv_bfloat16*)m->wb, m->w + ONORM, pre,
                                                                  r, n, xi0);
    return launched();
}

int bh_mlp_train_step(bh_mlp* m, const double* pre, const double* r, const float* target, int64_t n, float lr,
                      float* scratch, float* loss_out, void* stream) {
    if (!m || !m->w || !m->wb || !m->adam_m || !m->adam_v || !pre || !r || !target || !scratch || n <= 0)
        return BH_EINVAL;
    cudaStream_t st = S(stream);
    float* act0 = scratch;
    float* act1 = act0 + NI * n;
    float* act2 = act1 + NH * n;
    float* d1 = act2 + NH * n;
    float* d2 = d1 + NH * n;
    float* d3 = d2 + NH * n;
    float* loss = d3 + NO * n;
    float* grad = loss + n;
    const __nv_bfloat16* wb = (const __nv_bfloat16*)m->wb;
    k_train_fwd_bwd<<<(unsigned)((n + TPB - 1) / TPB), TPB, 0, st>>>(wb, m->w + ONORM, pre, r, target, n, act0, act1,
                                                                    act2, d1, d2, d3, loss);
    k_wgrad<<<(NH * NI + NH + 127) / 128, 128, 0, st>>>(d1, act0, n, NH, NI, grad, OW1, OB1);
    k_wgrad<<<(NH * NH + NH + 127) / 128, 128, 0, st>>>(d2, act1, n, NH, NH, grad, OW2, OB2);
    k_wgrad<<<(NO * NH + NO + 127) / 128, 128, 0, st>>>(d3, act2, n, NO, NH, grad, OW3, OB3);
    if (loss_out) k_sum<<<1, 256, 0, st>>>(loss, n, loss_out);
    if (lr > 0.0f) {
        m->step += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        float c1 = 1.0f - powf(b1, (float)m->step), c2 = 1.0f - powf(b2, (float)m->step);
        k_adam<<<(NPAR + 255) / 256, 256, 0, st>>>(m->w, grad, m->adam_m, m->adam_v, (__nv_bfloat16*)m->wb, lr, b1, b2,
                                                   1e-8f, c1, c2);
    }
    return launched();
}

}  // extern "C"
