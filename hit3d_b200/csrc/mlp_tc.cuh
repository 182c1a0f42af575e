// Tensor-core inference of the learned subgrid closure (sm_100a, tcgen05).
//
// A CTA of 128 threads takes tiles of 128 points, one point per thread.  The
// two 64x64 hidden layers (92 % of the multiply-adds) run as
//   D[128 x 64] (fp32, TMEM) = A[128 x 64] (bf16, smem) * W^T (bf16, smem)
// with four tcgen05.mma of K = 16 each, issued by one thread and completed
// through tcgen05.commit on an mbarrier.  The input layer (6 -> 64), the GELUs
// (tanh form with the hardware tanh approximation), the output layer (64 -> 5)
// and the tensor basis stay on the CUDA cores in fp32.  The activations that feed
// the tensor cores are rounded to bf16 (round to nearest even).
//
// Shared-memory operands use the no-swizzle K-major canonical layout: 8 x 8
// "core matrices" of 128 contiguous bytes (row r at 16 r bytes, element k at
// 2 k bytes), K chunks of 8 elements LBO bytes apart, 8-row groups SBO bytes
// apart.  Here every K chunk holds all row groups contiguously, so
//   A (128 rows): offset(r, k) = ((k/8) 16 + r/8) 128 + (r%8) 16 + (k%8) 2,  LBO 2048, SBO 128
//   W ( 64 rows): offset(n, k) = ((k/8)  8 + n/8) 128 + (n%8) 16 + (k%8) 2,  LBO 1024, SBO 128
// and k-step s of an MMA starts 2 chunks further (4096 and 2048 bytes).
#pragma once
#include "mlp.cuh"

constexpr int TC_TILE = 128;
constexpr int TC_COLS = 64;  // TMEM columns: one 128 x 64 fp32 accumulator
constexpr uint32_t TC_A_BYTES = TC_TILE * MLP_H * 2, TC_W_BYTES = MLP_H * MLP_H * 2;
constexpr uint32_t TC_OFF_A = 0, TC_OFF_W2 = TC_A_BYTES, TC_OFF_W3 = TC_OFF_W2 + TC_W_BYTES,
                   TC_OFF_F = TC_OFF_W3 + TC_W_BYTES;
// fp32 parameters: W1t[6][64], b1, b2, b3 [64], W4[5][64], b4[5]
constexpr int TCF_W1 = 0, TCF_B1 = TCF_W1 + MLP_IN * MLP_H, TCF_B2 = TCF_B1 + MLP_H, TCF_B3 = TCF_B2 + MLP_H,
              TCF_W4 = TCF_B3 + MLP_H, TCF_B4 = TCF_W4 + MLP_OUT * MLP_H, TCF_N = TCF_B4 + 8;
constexpr uint32_t TC_OFF_BAR = TC_OFF_F + 4 * TCF_N;  // 8-byte mbarrier, then the TMEM address slot
constexpr size_t TC_SMEM = TC_OFF_BAR + 16;
static_assert(TC_OFF_BAR % 8 == 0, "mbarrier alignment");
// kind::f16 instruction descriptor: fp32 accumulator, bf16 A and B, both
// K-major, N = 64, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(MLP_H >> 3) << 17) |
                              ((uint32_t)(TC_TILE >> 4) << 24);
constexpr uint32_t TC_WAIT_LIMIT = 1u << 22;  // bounded mbarrier polls

H3D_D uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle, descriptor version 1
H3D_D uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

H3D_D void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
                 "l"(a), "l"(b), "r"(TC_IDESC), "r"(accumulate));
}
H3D_D void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
H3D_D bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (uint32_t it = 0; it < TC_WAIT_LIMIT; it++) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(ok)
                     : "r"(bar), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}
H3D_D void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
H3D_D void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
H3D_D void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 consecutive TMEM columns of this warp's 32 lanes: thread i gets lane i
H3D_D void tmem_ld32(uint32_t taddr, float *v)
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                 "[%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}
H3D_D void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// bf16 of gelu(acc[j] + b[j]) into this thread's row of the A tile
H3D_D void store_act_row(unsigned char *sA, int r, const float *acc, const float *b)
{
#pragma unroll
    for (int c = 0; c < MLP_H / 8; c++) {
        uint32_t w[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const float lo = gelu_fast(acc[8 * c + 2 * e] + b[8 * c + 2 * e]);
            const float hi = gelu_fast(acc[8 * c + 2 * e + 1] + b[8 * c + 2 * e + 1]);
            const __nv_bfloat162 h2 = __floats2bfloat162_rn(lo, hi);
            w[e] = *reinterpret_cast<const uint32_t *>(&h2);
        }
        *reinterpret_cast<uint4 *>(sA + ((c * (TC_TILE / 8) + r / 8) * 128 + (r % 8) * 16)) =
            make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// one hidden layer on the tensor cores: acc (fp32, this thread's row) = A * W^T
H3D_D bool tc_layer(unsigned char *sm, uint32_t sW, uint32_t tmem, uint32_t bar, uint32_t &phase, float *acc)
{
    proxy_fence();  // the A tile written by the threads, to the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) {
        const uint32_t sA = smem_addr(sm + TC_OFF_A);
#pragma unroll
        for (int s = 0; s < MLP_H / 16; s++)
            umma_bf16(tmem, umma_desc(sA + s * 2 * 2048, 2048, 128), umma_desc(sW + s * 2 * 1024, 1024, 128), s > 0);
        umma_commit(bar);
    }
    const bool ok = mbar_wait(bar, phase);
    phase ^= 1u;
    tc_fence_after();
    const uint32_t ta = tmem + ((uint32_t)(threadIdx.x & ~31) << 16);
    tmem_ld32(ta, acc);
    tmem_ld32(ta + 32, acc + 32);
    tmem_wait_ld();
    return ok;
}

// Inference, as k_mlp_apply, with the hidden layers on the tensor cores.
// err: set to 1 if an MMA completion wait ran out (the results are then invalid).
template <typename TS>
__global__ void __launch_bounds__(TC_TILE) k_mlp_apply_tc(int64_t np, int64_t n, int64_t rp, int64_t fs, float delta,
                                                         int clip, const __nv_bfloat16 *__restrict__ wb, TS *G,
                                                         int *err)
{
    extern __shared__ __align__(1024) unsigned char tsm[];
    unsigned char *sm = tsm;
    float *F = reinterpret_cast<float *>(sm + TC_OFF_F);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + TC_OFF_BAR);
    uint32_t *slot = reinterpret_cast<uint32_t *>(sm + TC_OFF_BAR + 8);
    const int tid = threadIdx.x;

    // weights: hidden layers in the K-major core-matrix layout (16-byte copies),
    // the rest as fp32
    const uint4 *w4 = reinterpret_cast<const uint4 *>(wb);
    for (int q = tid; q < 2 * MLP_H * (MLP_H / 8); q += TC_TILE) {
        const int l = q / (MLP_H * MLP_H / 8), e = q % (MLP_H * MLP_H / 8), nrow = e / 8, c = e % 8;
        const int src = ((l == 0 ? MLP_W2 : MLP_W3) + nrow * MLP_H + 8 * c) / 8;
        *reinterpret_cast<uint4 *>(sm + (l == 0 ? TC_OFF_W2 : TC_OFF_W3) + (c * (MLP_H / 8) + nrow / 8) * 128 +
                                   (nrow % 8) * 16) = w4[src];
    }
    for (int q = tid; q < MLP_IN * MLP_H; q += TC_TILE) {
        const int j = q / MLP_IN, i = q % MLP_IN;
        F[TCF_W1 + i * MLP_H + j] = __bfloat162float(wb[MLP_W1 + q]);
    }
    for (int q = tid; q < MLP_H; q += TC_TILE) {
        F[TCF_B1 + q] = __bfloat162float(wb[MLP_B1 + q]);
        F[TCF_B2 + q] = __bfloat162float(wb[MLP_B2 + q]);
        F[TCF_B3 + q] = __bfloat162float(wb[MLP_B3 + q]);
    }
    for (int q = tid; q < MLP_OUT * MLP_H + MLP_OUT; q += TC_TILE)
        F[TCF_W4 + q] = __bfloat162float(wb[MLP_W4 + q]);  // W4 then b4, contiguous in both layouts
    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                     "r"(TC_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot, sbar = smem_addr(bar);
    const uint32_t sW2 = smem_addr(sm + TC_OFF_W2), sW3 = smem_addr(sm + TC_OFF_W3);
    uint32_t phase = 0;
    bool ok = true;

    const int64_t ntile = (np + TC_TILE - 1) / TC_TILE;
    for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int64_t t = tile * TC_TILE + tid;
        const bool valid = t < np;
        int64_t o = 0;
        float Am[3][3];
        if (valid) {
            const int64_t row = t / n;
            o = row * rp + (t - row * n);
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) Am[i][j] = (float)G[(3 * i + j) * fs + o];
        } else {
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) Am[i][j] = (i == j) ? 1.0f : 0.0f;
        }
        Feat f;
        features(Am, delta, f);
        float acc[MLP_H];
#pragma unroll
        for (int j = 0; j < MLP_H; j++) {
            float s = 0.0f;
#pragma unroll
            for (int i = 0; i < MLP_IN; i++) s = fmaf(F[TCF_W1 + i * MLP_H + j], f.x[i], s);
            acc[j] = s;
        }
        store_act_row(sm + TC_OFF_A, tid, acc, F + TCF_B1);
        ok &= tc_layer(sm, sW2, tmem, sbar, phase, acc);
        store_act_row(sm + TC_OFF_A, tid, acc, F + TCF_B2);
        ok &= tc_layer(sm, sW3, tmem, sbar, phase, acc);
#pragma unroll
        for (int j = 0; j < MLP_H; j++) acc[j] = gelu_fast(acc[j] + F[TCF_B3 + j]);
        float g[MLP_OUT], tau[MLP_TC];
#pragma unroll
        for (int q = 0; q < MLP_OUT; q++) {
            float s = F[TCF_B4 + q];
#pragma unroll
            for (int i = 0; i < MLP_H; i++) s = fmaf(F[TCF_W4 + q * MLP_H + i], acc[i], s);
            g[q] = s;
        }
        basis_sum(f, g, tau);
        const bool zero = clip && sgs_diss(tau, f.sbar) < 0.f;
        if (valid) {
#pragma unroll
            for (int c = 0; c < MLP_TC; c++) G[c * fs + o] = zero ? (TS)0 : (TS)tau[c];
        }
    }
    if (!ok) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_COLS));
}
