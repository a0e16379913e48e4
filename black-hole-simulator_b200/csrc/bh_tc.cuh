// bh_tc.cuh -- the con2prim-guess network (6 -> 64 -> 64 -> 2, tanh) on the
// fifth-generation tensor cores.  One CTA of 128 threads holds 128 cells:
// they are the M = 128 rows of two BF16 x BF16 -> FP32 products
// (tcgen05.mma.cta_group::1.kind::f16) whose accumulator, 64 FP32 columns,
// lives in tensor memory and is read back with tcgen05.ld (thread t of the
// CTA owns TMEM lane t = its own cell's row).
//
// Operands sit in shared memory, K-major without swizzle: 8-row x 16-byte
// core matrices, LBO = 128 bytes between the two core matrices of one
// K = 16 step, SBO = (K / 8) x 128 bytes between 8-row groups.
//
// The weights are BF16 (the trained network's own BF16 copy).  Activations
// enter as two BF16 halves, hi = bf16(x) and lo = bf16(x - hi), placed side
// by side along K against the same weight columns, so the product is that
// of the FP32 activation to ~2^-16 relative: the network the CUDA-core
// inference (bh_mlp.cu) evaluates, up to the FP32 summation order.
//
// Layer 1 (K = 16): [x_hi(6) | x_lo(6) | 1 | 0 0 0] . [W1 | W1 | b1 | 0 0 0]
// Layer 2 (K = 128, eight K = 16 steps): [h1_hi(64) | h1_lo(64)] . [W2 | W2]
// Layer 3 (64 -> 2) and the biases of layer 2 run in FP32 on the CUDA cores
// in the epilogue.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace bh_tc {

constexpr int NI = 6, NH = 64, NO = 2;
constexpr int OW1 = 0, OB1 = OW1 + NH * NI, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH,
              OB3 = OW3 + NO * NH, NPAR = OB3 + NO;
constexpr int ROWS = 128;        // cells per tile: the MMA's M
constexpr int K1 = 16;           // layer-1 K (6 + 6 + bias column, padded)
constexpr int K2 = 2 * NH;       // layer-2 K (hi and lo halves)
constexpr uint32_t TMEM_COLS = NH;   // one FP32 accumulator of N = 64 columns (power of 2, >= 32)
// resident CTAs per SM allowed to hold TMEM at once (512 columns per SM)
constexpr int MAX_CTAS_PER_SM = 512 / (int)TMEM_COLS;

// byte offset of element (row, k) in a K-major, unswizzled BF16 operand of K columns
__host__ __device__ constexpr uint32_t kmaj(int row, int k, int K) {
    return (uint32_t)((row >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// the operand layouts the descriptors below assume: every element inside
// its buffer, the layer-1 operand inside the first 4 KB of the shared one,
// and each K = 16 step 256 bytes (two 128-byte core-matrix columns) on
static_assert(kmaj(ROWS - 1, K2 - 1, K2) + 2 <= ROWS * K2 * 2, "layer-2 A in its buffer");
static_assert(kmaj(ROWS - 1, K1 - 1, K1) + 2 <= ROWS * K1 * 2, "layer-1 A in the first 4 KB");
static_assert(kmaj(NH - 1, K1 - 1, K1) + 2 <= NH * K1 * 2, "layer-1 B in its buffer");
static_assert(kmaj(NH - 1, NH - 1, NH) + 2 <= NH * NH * 2, "layer-2 B in its buffer");
static_assert(kmaj(0, 16, K2) == 256 && kmaj(0, 48, NH) == 3 * 256, "K-step stride of the descriptors");
static_assert(kmaj(8, 0, K2) == (K2 / 8) * 128 && kmaj(8, 0, K1) == (K1 / 8) * 128, "8-row group stride (SBO)");
static_assert(kmaj(0, 8, K2) == 128, "core-matrix column stride (LBO)");
// kind::f16 with M = 128: N a multiple of 16 in [16, 256]; the fields fit
static_assert(ROWS == 128 && NH % 16 == 0 && NH >= 16 && NH <= 256, "MMA shape");
static_assert((NH >> 3) < 64 && (ROWS >> 4) < 32, "instruction-descriptor fields");
static_assert(2 * NI + 1 <= K1, "features, their low halves and the bias column fit layer 1's K");

struct Smem {
    alignas(128) uint8_t a[ROWS * K2 * 2];   // 32 KB: layer-1 A (K = 16, first 4 KB) or layer-2 A (K = 128)
    alignas(128) uint8_t b1[NH * K1 * 2];    // 2 KB
    alignas(128) uint8_t b2[NH * NH * 2];    // 8 KB: W2, K = 64
    float b2f[NH], w3[NO * NH], b3[NO], norm[2 * NI];
    alignas(8) uint64_t mbar;
    uint32_t tmem;
};

// instruction descriptor, kind::f16: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at
// bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NH >> 3) << 17) |
                           ((uint32_t)(ROWS >> 4) << 24);

__device__ inline uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start >> 4 (bits 0-13), LBO >> 4 (16-29),
// SBO >> 4 (32-45), version 1 (bits 46-47), base offset 0, no swizzle (61-63 = 0)
__device__ inline uint64_t sdesc(uint32_t start, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ inline void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory made visible to the tensor core's (async) proxy
__device__ inline void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM allocation: one whole warp executes these
__device__ inline void tmem_alloc(uint32_t* dst) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(dst)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ inline void tmem_free(uint32_t taddr) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(TMEM_COLS) : "memory");
}

__device__ inline void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ inline bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ inline uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// bounded wait for the phase with the given parity to complete: at most
// WAIT_LIMIT polls and WAIT_NS nanoseconds; false if either ran out
constexpr int WAIT_LIMIT = 1 << 24;
constexpr uint64_t WAIT_NS = 1000000000ull;
__device__ inline bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint64_t t0 = globaltimer_ns();
    for (int i = 0; i < WAIT_LIMIT; i++) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 255) == 255 && globaltimer_ns() - t0 > WAIT_NS) return false;
    }
    return false;
}

// D[tmem] (+)= A[smem] . B[smem]^T, issued by one thread
__device__ inline void mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(IDESC), "r"(accumulate)
        : "memory");
}
// arrive on the mbarrier once every MMA this thread issued has completed
__device__ inline void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane; the wait is tied
// to the destination registers so no use of them moves above it
__device__ inline void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r0, r1, r2, r3, r4, r5, r6, r7, r8, r9, r10, r11, r12, r13, r14, r15;
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7), "=r"(r8), "=r"(r9),
          "=r"(r10), "=r"(r11), "=r"(r12), "=r"(r13), "=r"(r14), "=r"(r15)
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3), "+r"(r4), "+r"(r5), "+r"(r6), "+r"(r7), "+r"(r8),
                   "+r"(r9), "+r"(r10), "+r"(r11), "+r"(r12), "+r"(r13), "+r"(r14), "+r"(r15)
                 :
                 : "memory");
    v[0] = __uint_as_float(r0); v[1] = __uint_as_float(r1); v[2] = __uint_as_float(r2);
    v[3] = __uint_as_float(r3); v[4] = __uint_as_float(r4); v[5] = __uint_as_float(r5);
    v[6] = __uint_as_float(r6); v[7] = __uint_as_float(r7); v[8] = __uint_as_float(r8);
    v[9] = __uint_as_float(r9); v[10] = __uint_as_float(r10); v[11] = __uint_as_float(r11);
    v[12] = __uint_as_float(r12); v[13] = __uint_as_float(r13); v[14] = __uint_as_float(r14);
    v[15] = __uint_as_float(r15);
}

__device__ inline uint16_t bf16_bits(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ inline float bf16_val(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }
__device__ inline uint32_t pack2(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }

// the network's inputs from con2prim's preamble p5 = (D, tau, Ssq, Bsq, SB)
// and r: log D, asinh(tau / D), log(1 + S^2 / D^2), log(1 + B^2 / D),
// asinh(S.B / D^1.5), log r
__device__ inline void features(const double* p5, double r, float* x) {
    double D = p5[0], tau = p5[1], Ssq = p5[2], Bsq = p5[3], SB = p5[4];
    x[0] = (float)log(D);
    x[1] = (float)asinh(tau / D);
    x[2] = (float)log1p(Ssq / (D * D));
    x[3] = (float)log1p(Bsq / D);
    x[4] = (float)asinh(SB / (D * sqrt(D)));
    x[5] = (float)log(r);
}

// the network's weights into this CTA's shared memory (all threads)
__device__ inline void stage_weights(Smem& s, const __nv_bfloat16* wb, const float* norm) {
    const uint16_t* w = reinterpret_cast<const uint16_t*>(wb);
    for (int e = threadIdx.x; e < NH * K1; e += blockDim.x) {
        int n = e / K1, k = e % K1;
        uint16_t v = 0;
        if (k < NI) v = w[OW1 + n * NI + k];
        else if (k < 2 * NI) v = w[OW1 + n * NI + k - NI];
        else if (k == 2 * NI) v = w[OB1 + n];
        *reinterpret_cast<uint16_t*>(s.b1 + kmaj(n, k, K1)) = v;
    }
    for (int e = threadIdx.x; e < NH * NH; e += blockDim.x) {
        int n = e / NH, k = e % NH;
        *reinterpret_cast<uint16_t*>(s.b2 + kmaj(n, k, NH)) = w[OW2 + n * NH + k];
    }
    for (int e = threadIdx.x; e < NH; e += blockDim.x) s.b2f[e] = bf16_val(w[OB2 + e]);
    for (int e = threadIdx.x; e < NO * NH; e += blockDim.x) s.w3[e] = bf16_val(w[OW3 + e]);
    if (threadIdx.x < NO) s.b3[threadIdx.x] = bf16_val(w[OB3 + threadIdx.x]);
    if (threadIdx.x < 2 * NI) s.norm[threadIdx.x] = norm[threadIdx.x];
}

// row `row` of the layer-1 operand from the normalised features (zeros when
// the cell has none: its accumulator row is then zero and unused)
__device__ inline void put_row1(Smem& s, int row, const float* xn, bool valid) {
    uint16_t v[K1];
#pragma unroll
    for (int k = 0; k < K1; k++) v[k] = 0;
    if (valid) {
#pragma unroll
        for (int i = 0; i < NI; i++) {
            uint16_t hi = bf16_bits(xn[i]);
            v[i] = hi;
            v[NI + i] = bf16_bits(xn[i] - bf16_val(hi));
        }
        v[2 * NI] = bf16_bits(1.0f);
    }
#pragma unroll
    for (int c = 0; c < K1 / 8; c++) {
        uint4 q = make_uint4(pack2(v[8 * c], v[8 * c + 1]), pack2(v[8 * c + 2], v[8 * c + 3]),
                             pack2(v[8 * c + 4], v[8 * c + 5]), pack2(v[8 * c + 6], v[8 * c + 7]));
        *reinterpret_cast<uint4*>(s.a + kmaj(row, 8 * c, K1)) = q;
    }
}

// 16 hidden values (columns c0..c0+15) of row `row` into the layer-2 operand
// as hi (k = c0..) and lo (k = 64 + c0..) halves
__device__ inline void put_row2(Smem& s, int row, int c0, const float* h) {
#pragma unroll
    for (int c = 0; c < 2; c++) {
        uint16_t hi[8], lo[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            hi[j] = bf16_bits(h[8 * c + j]);
            lo[j] = bf16_bits(h[8 * c + j] - bf16_val(hi[j]));
        }
        *reinterpret_cast<uint4*>(s.a + kmaj(row, c0 + 8 * c, K2)) =
            make_uint4(pack2(hi[0], hi[1]), pack2(hi[2], hi[3]), pack2(hi[4], hi[5]), pack2(hi[6], hi[7]));
        *reinterpret_cast<uint4*>(s.a + kmaj(row, NH + c0 + 8 * c, K2)) =
            make_uint4(pack2(lo[0], lo[1]), pack2(lo[2], lo[3]), pack2(lo[4], lo[5]), pack2(lo[6], lo[7]));
    }
}

// issue layer 1 (one K = 16 step) or layer 2 (eight K = 16 steps), then commit
__device__ inline void issue_layer1(Smem& s, uint32_t tmem) {
    uint64_t da = sdesc(saddr(s.a), 128, (K1 / 8) * 128);
    uint64_t db = sdesc(saddr(s.b1), 128, (K1 / 8) * 128);
    mma(tmem, da, db, 0);
    mma_commit(&s.mbar);
}
__device__ inline void issue_layer2(Smem& s, uint32_t tmem) {
#pragma unroll
    for (int st = 0; st < K2 / 16; st++) {
        uint64_t da = sdesc(saddr(s.a) + st * 256, 128, (K2 / 8) * 128);
        uint64_t db = sdesc(saddr(s.b2) + (st % (NH / 16)) * 256, 128, (NH / 8) * 128);
        mma(tmem, da, db, st > 0);
    }
    mma_commit(&s.mbar);
}

// the whole network for the CTA's 128 cells; thread t passes its cell's
// normalised features (valid = all finite) and receives y0 = log(xi / D).
// Every thread of the CTA calls it (it synchronises the CTA).  `phase`
// tracks the mbarrier's parity across calls; returns false, for the whole
// CTA alike, if an MMA did not complete within the wait limit.
__device__ inline bool network(Smem& s, uint32_t tmem, uint32_t& phase, const float* xn, bool valid, float& y0) {
    const int t = threadIdx.x;
    const uint32_t lane_base = tmem + ((uint32_t)(t & ~31) << 16);   // this warp's 32 TMEM lanes
    put_row1(s, t, xn, valid);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    if (t == 0) issue_layer1(s, tmem);
    bool ok = mbar_wait(&s.mbar, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) return false;
    fence_after();
#pragma unroll
    for (int c0 = 0; c0 < NH; c0 += 16) {
        float h[16];
        tmem_ld16(lane_base + c0, h);
#pragma unroll
        for (int j = 0; j < 16; j++) h[j] = tanhf(h[j]);
        put_row2(s, t, c0, h);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    if (t == 0) issue_layer2(s, tmem);
    ok = mbar_wait(&s.mbar, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) return false;
    fence_after();
    float a = s.b3[0];
#pragma unroll
    for (int c0 = 0; c0 < NH; c0 += 16) {
        float h[16];
        tmem_ld16(lane_base + c0, h);
#pragma unroll
        for (int j = 0; j < 16; j++) a += s.w3[c0 + j] * tanhf(h[j] + s.b2f[c0 + j]);
    }
    y0 = a;
    // the next call's MMA overwrites the accumulator after its barrier
    fence_before();
    return true;
}

}  // namespace bh_tc
