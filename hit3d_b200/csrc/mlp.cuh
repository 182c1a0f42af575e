// Learned subgrid closure (no reference counterpart; Smagorinsky, m_les.f90:1142-1215,
// is the fallback and the baseline).
//
// Per point, from the filtered velocity gradient A_ij = d ubar_i / dx_j:
//   S = (A + A^T)/2, R = (A - A^T)/2, |S| = sqrt(2 S:S), s = S/|S|, r = R/|S|
//   inputs  x = [tr(s^2), tr(r^2), tr(s^3), tr(s r^2), tr(s^2 r^2), Delta / (2 pi / 32)]
//   basis   T1 = s, T2 = s r - r s, T3 = s^2 - tr(s^2) I/3, T4 = r^2 - tr(r^2) I/3,
//           T5 = r s^2 - s^2 r
//   stress  tau = Delta^2 |S|^2 sum_n g_n(x) T_n   (deviatoric)
// g = MLP(x): 6 -> 64 -> 64 -> 64 -> 5 with GELU; the weights are stored as bf16
// and every product is accumulated in fp32.  Smagorinsky is g = (-2 Cs^2, 0, 0, 0, 0).
//
// Kernels run one thread per point.  The weights sit in shared memory (fp32
// values of the bf16 weights), the running layer's 64 accumulators in
// registers, and the previous layer's activations in a per-thread column of
// shared memory, so that no register array is indexed by a loop variable.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

constexpr int MLP_IN = 6, MLP_H = 64, MLP_OUT = 5, MLP_NB = 5, MLP_TC = 6;
// flat parameter layout (floats): W_l is [out][in] row-major, then b_l
constexpr int MLP_W1 = 0, MLP_B1 = MLP_W1 + MLP_H * MLP_IN, MLP_W2 = MLP_B1 + MLP_H, MLP_B2 = MLP_W2 + MLP_H * MLP_H,
              MLP_W3 = MLP_B2 + MLP_H, MLP_B3 = MLP_W3 + MLP_H * MLP_H, MLP_W4 = MLP_B3 + MLP_H,
              MLP_B4 = MLP_W4 + MLP_OUT * MLP_H, MLP_NPARAM = MLP_B4 + MLP_OUT;
constexpr int MLP_NT = 128;                                               // threads per block
constexpr int MLP_WPAD = (MLP_NPARAM + 3) / 4 * 4;                        // weights in shared memory
constexpr size_t MLP_SMEM = sizeof(float) * (MLP_WPAD + MLP_H * MLP_NT);  // + activation columns
static_assert(MLP_W2 % 4 == 0 && MLP_W3 % 4 == 0, "float4 rows");

// GELU in its tanh form (Hendrycks and Gimpel, "Gaussian Error Linear Units",
// 2016): gelu(z) = z/2 (1 + tanh(a (z + b z^3))), a = sqrt(2/pi), b = 0.044715;
// the activation of the network, in training and inference
constexpr float GELU_A = 0.79788456080286535588f, GELU_B = 0.044715f;
H3D_D float gelu(float z)
{
    const float u = GELU_A * (z + GELU_B * (z * z * z));
    return 0.5f * z * (1.0f + tanhf(u));
}
H3D_D float gelu_d(float z)
{
    const float u = GELU_A * (z + GELU_B * (z * z * z)), t = tanhf(u);
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * GELU_A * (1.0f + 3.0f * GELU_B * (z * z));
}
// the same with the hardware tanh approximation (tanh.approx.f32, one special
// function unit instruction), for the tensor-core inference kernel, whose
// activations are rounded to bf16 afterwards anyway
H3D_D float gelu_fast(float z)
{
    const float u = GELU_A * z * fmaf(GELU_B, z * z, 1.0f);
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
    const float h = 0.5f * z;
    return fmaf(h, t, h);
}

struct Feat {
    float x[MLP_IN];
    float T[MLP_NB][MLP_TC];  // symmetric 3x3 as (11, 12, 13, 22, 23, 33)
    float sbar[MLP_TC];       // unnormalised strain rate
    float pref;               // Delta^2 |S|^2
};
// Frobenius weights of the (11, 12, 13, 22, 23, 33) storage
H3D_HD float frob_w(int c) { return (c == 1 || c == 2 || c == 4) ? 2.0f : 1.0f; }

H3D_D void mat_mul3(const float a[3][3], const float b[3][3], float c[3][3])
{
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) c[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
}

H3D_D void features(const float A[3][3], float delta, Feat &f)
{
    float S[3][3], R[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            S[i][j] = 0.5f * (A[i][j] + A[j][i]);
            R[i][j] = 0.5f * (A[i][j] - A[j][i]);
        }
    const int ii[6] = {0, 0, 0, 1, 1, 2}, jj[6] = {0, 1, 2, 1, 2, 2};
    float ss = 0.f;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        f.sbar[q] = S[ii[q]][jj[q]];
        ss += frob_w(q) * f.sbar[q] * f.sbar[q];
    }
    const float smag = sqrtf(2.0f * ss) + 1e-30f;
    const float inv = 1.0f / smag;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) { S[i][j] *= inv; R[i][j] *= inv; }
    float s2[3][3], r2[3][3], s3[3][3], sr[3][3], rs[3][3], sr2[3][3], s2r2[3][3], rs2[3][3], s2r[3][3];
    mat_mul3(S, S, s2);
    mat_mul3(R, R, r2);
    mat_mul3(s2, S, s3);
    mat_mul3(S, R, sr);
    mat_mul3(R, S, rs);
    mat_mul3(S, r2, sr2);
    mat_mul3(s2, r2, s2r2);
    mat_mul3(R, s2, rs2);
    mat_mul3(s2, R, s2r);
    const float ts2 = s2[0][0] + s2[1][1] + s2[2][2], tr2 = r2[0][0] + r2[1][1] + r2[2][2];
    f.x[0] = ts2;
    f.x[1] = tr2;
    f.x[2] = s3[0][0] + s3[1][1] + s3[2][2];
    f.x[3] = sr2[0][0] + sr2[1][1] + sr2[2][2];
    f.x[4] = s2r2[0][0] + s2r2[1][1] + s2r2[2][2];
    f.x[5] = delta * (32.0f / 6.283185307179586f);
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const int i = ii[q], j = jj[q];
        const float d = (i == j) ? 1.0f : 0.0f;
        f.T[0][q] = S[i][j];
        f.T[1][q] = sr[i][j] - rs[i][j];
        f.T[2][q] = s2[i][j] - d * ts2 * (1.0f / 3.0f);
        f.T[3][q] = r2[i][j] - d * tr2 * (1.0f / 3.0f);
        f.T[4][q] = rs2[i][j] - s2r[i][j];
    }
    f.pref = delta * delta * smag * smag;
}

// weights into shared memory as fp32; TRANS stores each W_l as [in][out]
// (forward passes), otherwise as [out][in] (backward pass)
template <bool TRANS> H3D_D int param_slot(int q)
{
    if (!TRANS) return q;
    int off = -1, nin = 0, nout = 0;
    if (q < MLP_B1) { off = MLP_W1; nin = MLP_IN; nout = MLP_H; }
    else if (q >= MLP_W2 && q < MLP_B2) { off = MLP_W2; nin = MLP_H; nout = MLP_H; }
    else if (q >= MLP_W3 && q < MLP_B3) { off = MLP_W3; nin = MLP_H; nout = MLP_H; }
    else if (q >= MLP_W4 && q < MLP_B4) { off = MLP_W4; nin = MLP_H; nout = MLP_OUT; }
    if (off < 0) return q;
    const int j = (q - off) / nin, i = (q - off) % nin;
    return off + i * nout + j;
}
// wb must be 16-byte aligned (eight bf16 per load)
template <bool TRANS> H3D_D void load_params(const __nv_bfloat16 *__restrict__ wb, float *sw)
{
    constexpr int NV = MLP_NPARAM / 8;
    for (int k = threadIdx.x; k < NV; k += blockDim.x) {
        const uint4 v = reinterpret_cast<const uint4 *>(wb)[k];
        const uint32_t u[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int e = 0; e < 4; e++) {
            sw[param_slot<TRANS>(8 * k + 2 * e)] = __uint_as_float(u[e] << 16);
            sw[param_slot<TRANS>(8 * k + 2 * e + 1)] = __uint_as_float(u[e] & 0xffff0000u);
        }
    }
    for (int q = 8 * NV + threadIdx.x; q < MLP_NPARAM; q += blockDim.x) sw[param_slot<TRANS>(q)] = __bfloat162float(wb[q]);
    __syncthreads();
}

// acc[j] = b[j] + sum_i Wt[i][j] act[i], act a column of stride MLP_NT
template <int NIN, int NOUT>
H3D_D void dense_col(const float *__restrict__ Wt, const float *__restrict__ b, const float *act, float acc[NOUT])
{
#pragma unroll
    for (int j = 0; j < NOUT; j++) acc[j] = b ? b[j] : 0.0f;
#pragma unroll 2
    for (int i = 0; i < NIN; i++) {
        const float ai = act[i * MLP_NT];
        if constexpr (NOUT % 4 == 0) {
            const float4 *w4 = reinterpret_cast<const float4 *>(Wt + i * NOUT);
#pragma unroll
            for (int q = 0; q < NOUT / 4; q++) {
                const float4 w = w4[q];
                acc[4 * q] = fmaf(w.x, ai, acc[4 * q]);
                acc[4 * q + 1] = fmaf(w.y, ai, acc[4 * q + 1]);
                acc[4 * q + 2] = fmaf(w.z, ai, acc[4 * q + 2]);
                acc[4 * q + 3] = fmaf(w.w, ai, acc[4 * q + 3]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < NOUT; j++) acc[j] = fmaf(Wt[i * NOUT + j], ai, acc[j]);
        }
    }
}

// forward pass of one point; sw holds the transposed weights, act is this
// thread's activation column; Z (optional) receives the pre-activations
// [3][64] at stride zs
H3D_D void mlp_forward(const float *__restrict__ sw, float *act, const float x[MLP_IN], float g[MLP_OUT],
                       float *Z = nullptr, int64_t zs = 0)
{
    float acc[MLP_H];
#pragma unroll
    for (int j = 0; j < MLP_H; j++) {
        float s = sw[MLP_B1 + j];
#pragma unroll
        for (int i = 0; i < MLP_IN; i++) s = fmaf(sw[MLP_W1 + i * MLP_H + j], x[i], s);
        acc[j] = s;
    }
#pragma unroll
    for (int l = 0; l < 2; l++) {
#pragma unroll
        for (int j = 0; j < MLP_H; j++) {
            if (Z) Z[(l * MLP_H + j) * zs] = acc[j];
            act[j * MLP_NT] = gelu(acc[j]);
        }
        dense_col<MLP_H, MLP_H>(sw + (l == 0 ? MLP_W2 : MLP_W3), sw + (l == 0 ? MLP_B2 : MLP_B3), act, acc);
    }
#pragma unroll
    for (int j = 0; j < MLP_H; j++) {
        if (Z) Z[(2 * MLP_H + j) * zs] = acc[j];
        act[j * MLP_NT] = gelu(acc[j]);
    }
    dense_col<MLP_H, MLP_OUT>(sw + MLP_W4, sw + MLP_B4, act, g);
}

H3D_D void basis_sum(const Feat &f, const float g[MLP_OUT], float tau[MLP_TC])
{
#pragma unroll
    for (int c = 0; c < MLP_TC; c++) {
        float t = 0.f;
#pragma unroll
        for (int n = 0; n < MLP_NB; n++) t = fmaf(g[n], f.T[n][c], t);
        tau[c] = f.pref * t;
    }
}
// subgrid dissipation -tau : S
H3D_D float sgs_diss(const float tau[MLP_TC], const float sbar[MLP_TC])
{
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < MLP_TC; c++) s = fmaf(frob_w(c) * tau[c], sbar[c], s);
    return -s;
}

struct MlpBatch {
    int64_t np;          // points in this minibatch
    const int32_t *idx;  // indices into the dataset
    const float *A;      // dataset gradients [9][P]
    const float *tau;    // dataset deviatoric stresses [6][P]
    int64_t P;
    float delta;         // filter width
    float inv_norm;      // 1 / mean |tau|_F^2 over the dataset
    float inv_norm_p;    // 1 / mean (tau:S)^2 over the dataset
    float lam;           // weight of the dissipation term
    float *z;            // [3][64][np] pre-activations
    float *x;            // [6][np] inputs
    float *d;            // [3][64][np] deltas of the hidden layers
    float *d4;           // [5][np] dL/dg
    float *loss;         // per-block partial losses
};

// forward + loss + dL/dg of a minibatch, one thread per point:
//   L = inv_norm/np sum_p |tau_pred - tau|_F^2 + lam inv_norm_p/np sum_p (Pi_pred - Pi)^2
// with Pi = -tau : S the subgrid dissipation
static __global__ void __launch_bounds__(MLP_NT) k_mlp_fwd(const MlpBatch b, const __nv_bfloat16 *__restrict__ wb)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ float red[MLP_NT / 32];
    load_params<true>(wb, sm);
    const int64_t p = blockIdx.x * (int64_t)MLP_NT + threadIdx.x;
    float lsum = 0.f;
    if (p < b.np) {
        const int64_t q = b.idx[p];
        float Am[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) Am[i][j] = b.A[(3 * i + j) * b.P + q];
        Feat f;
        features(Am, b.delta, f);
        float g[MLP_OUT];
        mlp_forward(sm, sm + MLP_WPAD + threadIdx.x, f.x, g, b.z + p, b.np);
#pragma unroll
        for (int i = 0; i < MLP_IN; i++) b.x[i * b.np + p] = f.x[i];
        float tp[MLP_TC], tt[MLP_TC], e[MLP_TC];
        basis_sum(f, g, tp);
#pragma unroll
        for (int c = 0; c < MLP_TC; c++) {
            tt[c] = b.tau[c * b.P + q];
            e[c] = tp[c] - tt[c];
        }
        float lt = 0.f;
#pragma unroll
        for (int c = 0; c < MLP_TC; c++) lt = fmaf(frob_w(c) * e[c], e[c], lt);
        const float ep = sgs_diss(tp, f.sbar) - sgs_diss(tt, f.sbar);
        const float inp = 1.0f / (float)b.np;
        lsum = (b.inv_norm * lt + b.lam * b.inv_norm_p * ep * ep) * inp;
        const float st = 2.0f * b.inv_norm * inp * f.pref, sp = -2.0f * b.lam * b.inv_norm_p * inp * ep * f.pref;
#pragma unroll
        for (int n = 0; n < MLP_NB; n++) {
            float a1 = 0.f, a2 = 0.f;
#pragma unroll
            for (int c = 0; c < MLP_TC; c++) {
                a1 = fmaf(frob_w(c) * e[c], f.T[n][c], a1);
                a2 = fmaf(frob_w(c) * f.sbar[c], f.T[n][c], a2);
            }
            b.d4[n * b.np + p] = st * a1 + sp * a2;
        }
    }
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < MLP_NT / 32; w++) s += red[w];
        b.loss[blockIdx.x] = s;
    }
}

// dL/dz of the three hidden layers, one thread per point
static __global__ void __launch_bounds__(MLP_NT) k_mlp_bwd(const MlpBatch b, const __nv_bfloat16 *__restrict__ wb)
{
    extern __shared__ __align__(16) float sm[];
    load_params<false>(wb, sm);
    const int64_t p = blockIdx.x * (int64_t)MLP_NT + threadIdx.x;
    if (p >= b.np) return;
    float *act = sm + MLP_WPAD + threadIdx.x;
    float d4[MLP_OUT], acc[MLP_H];
#pragma unroll
    for (int o = 0; o < MLP_OUT; o++) d4[o] = b.d4[o * b.np + p];
#pragma unroll
    for (int j = 0; j < MLP_H; j++) {
        float s = 0.f;
#pragma unroll
        for (int o = 0; o < MLP_OUT; o++) s = fmaf(sm[MLP_W4 + o * MLP_H + j], d4[o], s);
        acc[j] = s;
    }
#pragma unroll
    for (int l = 2; l >= 0; l--) {
#pragma unroll
        for (int j = 0; j < MLP_H; j++) {
            const int64_t o = (l * MLP_H + j) * b.np + p;
            const float dj = acc[j] * gelu_d(b.z[o]);
            b.d[o] = dj;
            act[j * MLP_NT] = dj;
        }
        // W_{l+1} rows are [out][in]: d_l[j] = sum_k W[k][j] d_{l+1}[k]
        if (l > 0) dense_col<MLP_H, MLP_H>(sm + (l == 2 ? MLP_W3 : MLP_W2), nullptr, act, acc);
    }
}

// weight gradients over chunks of WG_C points into part[chunk][param]; the
// partials are summed over chunks in order by k_mlp_wgrad_sum
constexpr int WG_C = 64;
static __global__ void __launch_bounds__(256) k_mlp_wgrad_part(const MlpBatch b, float *__restrict__ part)
{
    __shared__ float Ds[MLP_H][WG_C + 1], As[MLP_H][WG_C + 1];
    const int layer = blockIdx.y;
    const int nin = layer == 0 ? MLP_IN : MLP_H, nout = layer == 3 ? MLP_OUT : MLP_H;
    const int64_t p0 = (int64_t)blockIdx.x * WG_C;
    const float *D = layer < 3 ? b.d + (int64_t)layer * MLP_H * b.np : b.d4;
    for (int e = threadIdx.x; e < nout * WG_C; e += blockDim.x) {
        const int j = e / WG_C, q = e % WG_C;
        Ds[j][q] = p0 + q < b.np ? D[j * b.np + p0 + q] : 0.f;
    }
    for (int e = threadIdx.x; e < nin * WG_C; e += blockDim.x) {
        const int i = e / WG_C, q = e % WG_C;
        float a = 0.f;
        if (p0 + q < b.np)
            a = layer == 0 ? b.x[i * b.np + p0 + q] : gelu(b.z[((layer - 1) * MLP_H + i) * b.np + p0 + q]);
        As[i][q] = a;
    }
    __syncthreads();
    const int wo = layer == 0 ? MLP_W1 : layer == 1 ? MLP_W2 : layer == 2 ? MLP_W3 : MLP_W4;
    const int bo = layer == 0 ? MLP_B1 : layer == 1 ? MLP_B2 : layer == 2 ? MLP_B3 : MLP_B4;
    float *out = part + (int64_t)blockIdx.x * MLP_NPARAM;
    for (int o = threadIdx.x; o < nout * (nin + 1); o += blockDim.x) {
        const int j = o / (nin + 1), i = o % (nin + 1);
        float s = 0.f;
        if (i < nin) {
#pragma unroll 8
            for (int q = 0; q < WG_C; q++) s = fmaf(Ds[j][q], As[i][q], s);
            out[wo + j * nin + i] = s;
        } else {
#pragma unroll 8
            for (int q = 0; q < WG_C; q++) s += Ds[j][q];
            out[bo + j] = s;
        }
    }
}

static __global__ void k_mlp_wgrad_sum(int nchunk, const float *__restrict__ part, float *__restrict__ grad)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= MLP_NPARAM) return;
    float s = 0.f;
    for (int c = 0; c < nchunk; c++) s += part[(int64_t)c * MLP_NPARAM + q];
    grad[q] = s;
}

// in-order sum of per-block partial losses into *out
static __global__ void k_sum_partials(int n, const float *__restrict__ part, float *__restrict__ out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        float s = 0.f;
        for (int i = 0; i < n; i++) s += part[i];
        *out = s;
    }
}

H3D_HD uint64_t splitmix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// minibatch indices drawn uniformly from [0, P) by a counter-based hash
static __global__ void k_sample_idx(int64_t np, int64_t P, uint64_t key, int32_t *__restrict__ idx)
{
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p < np) idx[p] = (int32_t)(splitmix64(key ^ ((uint64_t)p * 0xd1b54a32d192ed03ull)) % (uint64_t)P);
}

// Adam on the fp32 master parameters; the bf16 copy used by the kernels follows
static __global__ void k_adam(int n, float lr, float b1, float b2, float eps, float c1, float c2,
                              const float *__restrict__ g, float *__restrict__ w, float *__restrict__ m,
                              float *__restrict__ v, __nv_bfloat16 *__restrict__ wb)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        wb[i] = __float2bfloat16_rn(wi);
    }
}

static __global__ void k_to_bf16(int n, const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

// inference on gradient fields of precision TS: point t of np reads A_ij at
// G[(3i+j) fs + off(t)] and writes tau_c to G[c fs + off(t)] (each point is
// read completely before it is written, by the same thread), where off(t)
// maps the x-fastest point index onto rows of n points at pitch rp.  With
// clip, points whose predicted dissipation -tau:S is negative get tau = 0.
template <typename TS>
__global__ void __launch_bounds__(MLP_NT) k_mlp_apply(int64_t np, int64_t n, int64_t rp, int64_t fs, float delta,
                                                      int clip, const __nv_bfloat16 *__restrict__ wb, TS *G)
{
    extern __shared__ __align__(16) float sm[];
    load_params<true>(wb, sm);
    float *act = sm + MLP_WPAD + threadIdx.x;
    const int64_t t = blockIdx.x * (int64_t)MLP_NT + threadIdx.x;
    if (t < np) {
        const int64_t row = t / n, o = row * rp + (t - row * n);
        float Am[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) Am[i][j] = (float)G[(3 * i + j) * fs + o];
        Feat f;
        features(Am, delta, f);
        float g[MLP_OUT], tau[MLP_TC];
        mlp_forward(sm, act, f.x, g);
        basis_sum(f, g, tau);
        const bool zero = clip && sgs_diss(tau, f.sbar) < 0.f;
#pragma unroll
        for (int c = 0; c < MLP_TC; c++) G[c * fs + o] = zero ? (TS)0 : (TS)tau[c];
    }
}
