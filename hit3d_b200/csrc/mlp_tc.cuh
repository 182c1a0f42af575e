// Tensor-core inference of the learned subgrid closure (sm_100a, tcgen05).
//
// A CTA of 128 threads takes tiles of 128 points, one point per thread.  All
// four layers run on the tensor cores as
//   D[128 x N] (fp32, TMEM) = A[128 x K] (bf16, smem) * W^T (bf16, smem)
// with tcgen05.mma of K = 16 each, issued by one thread and completed through
// tcgen05.commit on an mbarrier:
//   input layer   K = 16 (the six features, a 1 that carries the bias b1 in
//                 W1's seventh column, zeros), N = 64, one MMA;
//   hidden layers K = 64, N = 64, four MMAs each;
//   output layer  K = 64, N = 16 (W4's five rows, zeros), four MMAs.
// The features, the GELUs (tanh form with the hardware tanh approximation),
// the biases b2, b3, b4 and the tensor basis run on the CUDA cores in fp32.
// The features and every activation that feeds the tensor cores are rounded
// to bf16 (round to nearest even).
//
// Shared-memory operands use the no-swizzle K-major canonical layout: 8 x 8
// "core matrices" of 128 contiguous bytes (row r at 16 r bytes, element k at
// 2 k bytes), K chunks of 8 elements LBO bytes apart, 8-row groups SBO bytes
// apart.  Here every K chunk holds all row groups contiguously, so
//   A   (128 rows): offset(r, k) = ((k/8) 16 + r/8) 128 + (r%8) 16 + (k%8) 2,  LBO 2048, SBO 128
//   W   ( 64 rows): offset(n, k) = ((k/8)  8 + n/8) 128 + (n%8) 16 + (k%8) 2,  LBO 1024, SBO 128
//   W4p ( 16 rows): offset(n, k) = ((k/8)  2 + n/8) 128 + (n%8) 16 + (k%8) 2,  LBO  256, SBO 128
// and k-step s of an MMA starts 2 chunks further (4096, 2048 and 512 bytes).
// The input layer's A is the first two chunks of the A tile, its W1p the
// first two chunks of a 64-row W layout.
#pragma once
#include "mlp.cuh"

constexpr int TC_TILE = 128;
constexpr int TC_COLS = 64;  // TMEM columns: one 128 x 64 fp32 accumulator, reused by every layer
constexpr int TC_K1 = 16, TC_N4 = 16;  // padded K of the input layer, padded N of the output layer
constexpr uint32_t TC_A_BYTES = TC_TILE * MLP_H * 2, TC_W_BYTES = MLP_H * MLP_H * 2;
constexpr uint32_t TC_W1_BYTES = MLP_H * TC_K1 * 2, TC_W4_BYTES = TC_N4 * MLP_H * 2;
constexpr uint32_t TC_OFF_A = 0, TC_OFF_W2 = TC_A_BYTES, TC_OFF_W3 = TC_OFF_W2 + TC_W_BYTES,
                   TC_OFF_W1 = TC_OFF_W3 + TC_W_BYTES, TC_OFF_W4 = TC_OFF_W1 + TC_W1_BYTES,
                   TC_OFF_F = TC_OFF_W4 + TC_W4_BYTES;
// fp32 parameters kept for the CUDA cores: b2, b3 [64], b4 [5]
constexpr int TCF_B2 = 0, TCF_B3 = TCF_B2 + MLP_H, TCF_B4 = TCF_B3 + MLP_H, TCF_N = TCF_B4 + 8;
constexpr uint32_t TC_OFF_BAR = TC_OFF_F + 4 * TCF_N;  // 8-byte mbarrier, then the TMEM address slot
constexpr size_t TC_SMEM = TC_OFF_BAR + 16;
static_assert(TC_OFF_BAR % 8 == 0, "mbarrier alignment");
static_assert(TC_SMEM <= 48 * 1024, "the closure kernel runs with the default shared-memory limit");
// kind::f16 instruction descriptors: fp32 accumulator, bf16 A and B, both
// K-major, M = 128; N = 64 (input and hidden layers) or 16 (output layer)
constexpr uint32_t tc_idesc(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_TILE >> 4) << 24);
}
constexpr uint32_t TC_IDESC = tc_idesc(MLP_H), TC_IDESC_OUT = tc_idesc(TC_N4);
constexpr uint32_t TC_WAIT_LIMIT = 1u << 22;  // bounded mbarrier polls

H3D_D uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle, descriptor version 1
H3D_D uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

H3D_D void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate, uint32_t idesc = TC_IDESC)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
                 "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
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

// 16 consecutive TMEM columns of this warp's 32 lanes: thread i gets lane i
H3D_D void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// row r of the A tile, K chunk c (8 bf16 values)
H3D_D uint4 *a_chunk(unsigned char *sA, int r, int c)
{
    return reinterpret_cast<uint4 *>(sA + ((c * (TC_TILE / 8) + r / 8) * 128 + (r % 8) * 16));
}
H3D_D uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 h2 = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&h2);
}

// bf16 of the features, then 1 (the bias column of W1p), then zeros: the
// input layer's A (the first two K chunks of the A tile)
H3D_D void store_input_row(unsigned char *sA, int r, const float *x)
{
    *a_chunk(sA, r, 0) = make_uint4(pack_bf16(x[0], x[1]), pack_bf16(x[2], x[3]), pack_bf16(x[4], x[5]),
                                    pack_bf16(1.0f, 0.0f));
    *a_chunk(sA, r, 1) = make_uint4(0u, 0u, 0u, 0u);
}

// two fp32 lanes in one 64-bit register, and the packed two-lane operations of
// sm_100 (each lane rounded as the scalar operation rounds it)
H3D_D uint64_t f2_pack(float lo, float hi)
{
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
H3D_D void f2_unpack(uint64_t r, float &lo, float &hi) { asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(r)); }
H3D_D uint64_t f2_add(uint64_t a, uint64_t b)
{
    uint64_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
H3D_D uint64_t f2_mul(uint64_t a, uint64_t b)
{
    uint64_t r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
H3D_D uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c)
{
    uint64_t r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
// gelu_fast of two values, the same operations in the same order on each lane
// (so the same results), the multiply-adds two lanes per instruction
H3D_D void gelu_fast2(float z0, float z1, float &g0, float &g1)
{
    const uint64_t z = f2_pack(z0, z1);
    const uint64_t zz = f2_mul(z, z);
    const uint64_t p = f2_fma(f2_pack(GELU_B, GELU_B), zz, f2_pack(1.0f, 1.0f));
    const uint64_t u = f2_mul(f2_mul(f2_pack(GELU_A, GELU_A), z), p);
    float u0, u1, t0, t1;
    f2_unpack(u, u0, u1);
    asm("tanh.approx.f32 %0, %1;" : "=f"(t0) : "f"(u0));
    asm("tanh.approx.f32 %0, %1;" : "=f"(t1) : "f"(u1));
    const uint64_t h = f2_mul(f2_pack(0.5f, 0.5f), z);
    f2_unpack(f2_fma(h, f2_pack(t0, t1), h), g0, g1);
}

// bf16 of gelu(acc[j] + b[j]) (b may be null) into this thread's row of the A tile
H3D_D void store_act_row(unsigned char *sA, int r, const float *acc, const float *b)
{
#pragma unroll
    for (int c = 0; c < MLP_H / 8; c++) {
        uint32_t w[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int j = 8 * c + 2 * e;
            uint64_t z = f2_pack(acc[j], acc[j + 1]);
            if (b) z = f2_add(z, f2_pack(b[j], b[j + 1]));
            float z0, z1, lo, hi;
            f2_unpack(z, z0, z1);
            gelu_fast2(z0, z1, lo, hi);
            w[e] = pack_bf16(lo, hi);
        }
        *a_chunk(sA, r, c) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// one layer on the tensor cores: the A tile written by the threads times W^T,
// nk MMAs of K = 16 (A chunks 2 apart, W chunks `wstep` bytes apart), then this
// thread's row of the accumulator: ncol (64 or 16) columns into acc
H3D_D bool tc_layer(unsigned char *sm, uint32_t sW, uint32_t lboW, uint32_t wstep, int nk, uint32_t idesc, int ncol,
                    uint32_t tmem, uint32_t bar, uint32_t &phase, float *acc)
{
    proxy_fence();  // the A tile written by the threads, to the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) {
        const uint32_t sA = smem_addr(sm + TC_OFF_A);
        for (int s = 0; s < nk; s++)
            umma_bf16(tmem, umma_desc(sA + s * 2 * 2048, 2048, 128), umma_desc(sW + s * wstep, lboW, 128), s > 0, idesc);
        umma_commit(bar);
    }
    const bool ok = mbar_wait(bar, phase);
    phase ^= 1u;
    tc_fence_after();
    const uint32_t ta = tmem + ((uint32_t)(threadIdx.x & ~31) << 16);
    if (ncol == MLP_H) {
        tmem_ld32(ta, acc);
        tmem_ld32(ta + 32, acc + 32);
    } else {
        tmem_ld16(ta, acc);
    }
    tmem_wait_ld();
    return ok;
}

// Inference, as k_mlp_apply, with all four layers on the tensor cores.
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

    // weights: hidden layers in the K-major core-matrix layout (16-byte copies)
    const uint4 *w4 = reinterpret_cast<const uint4 *>(wb);
    for (int q = tid; q < 2 * MLP_H * (MLP_H / 8); q += TC_TILE) {
        const int l = q / (MLP_H * MLP_H / 8), e = q % (MLP_H * MLP_H / 8), nrow = e / 8, c = e % 8;
        const int src = ((l == 0 ? MLP_W2 : MLP_W3) + nrow * MLP_H + 8 * c) / 8;
        *reinterpret_cast<uint4 *>(sm + (l == 0 ? TC_OFF_W2 : TC_OFF_W3) + (c * (MLP_H / 8) + nrow / 8) * 128 +
                                   (nrow % 8) * 16) = w4[src];
    }
    // W1p [64 x 16]: W1's six columns, b1, zeros; W4p [16 x 64]: W4's five rows, zeros
    const __nv_bfloat16 bz = __float2bfloat16(0.0f);
    for (int q = tid; q < MLP_H * TC_K1; q += TC_TILE) {
        const int nrow = q / TC_K1, k = q % TC_K1;
        const __nv_bfloat16 v = k < MLP_IN ? wb[MLP_W1 + nrow * MLP_IN + k] : k == MLP_IN ? wb[MLP_B1 + nrow] : bz;
        *reinterpret_cast<__nv_bfloat16 *>(sm + TC_OFF_W1 + ((k / 8) * (MLP_H / 8) + nrow / 8) * 128 + (nrow % 8) * 16 +
                                           (k % 8) * 2) = v;
    }
    for (int q = tid; q < TC_N4 * MLP_H; q += TC_TILE) {
        const int nrow = q / MLP_H, k = q % MLP_H;
        const __nv_bfloat16 v = nrow < MLP_OUT ? wb[MLP_W4 + nrow * MLP_H + k] : bz;
        *reinterpret_cast<__nv_bfloat16 *>(sm + TC_OFF_W4 + ((k / 8) * (TC_N4 / 8) + nrow / 8) * 128 + (nrow % 8) * 16 +
                                           (k % 8) * 2) = v;
    }
    for (int q = tid; q < MLP_H; q += TC_TILE) {
        F[TCF_B2 + q] = __bfloat162float(wb[MLP_B2 + q]);
        F[TCF_B3 + q] = __bfloat162float(wb[MLP_B3 + q]);
    }
    if (tid < MLP_OUT) F[TCF_B4 + tid] = __bfloat162float(wb[MLP_B4 + tid]);
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
    const uint32_t sW1 = smem_addr(sm + TC_OFF_W1), sW2 = smem_addr(sm + TC_OFF_W2), sW3 = smem_addr(sm + TC_OFF_W3),
                   sW4 = smem_addr(sm + TC_OFF_W4);
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
        store_input_row(sm + TC_OFF_A, tid, f.x);
        ok &= tc_layer(sm, sW1, 1024, 2 * 1024, 1, TC_IDESC, MLP_H, tmem, sbar, phase, acc);
        store_act_row(sm + TC_OFF_A, tid, acc, nullptr);  // b1 came with the input layer
        ok &= tc_layer(sm, sW2, 1024, 2 * 1024, MLP_H / 16, TC_IDESC, MLP_H, tmem, sbar, phase, acc);
        store_act_row(sm + TC_OFF_A, tid, acc, F + TCF_B2);
        ok &= tc_layer(sm, sW3, 1024, 2 * 1024, MLP_H / 16, TC_IDESC, MLP_H, tmem, sbar, phase, acc);
        store_act_row(sm + TC_OFF_A, tid, acc, F + TCF_B3);
        ok &= tc_layer(sm, sW4, 256, 2 * 256, MLP_H / 16, TC_IDESC_OUT, TC_N4, tmem, sbar, phase, acc);
        float g[MLP_OUT], tau[MLP_TC];
#pragma unroll
        for (int q = 0; q < MLP_OUT; q++) g[q] = acc[q] + F[TCF_B4 + q];
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
