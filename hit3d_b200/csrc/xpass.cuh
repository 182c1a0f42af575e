// Launchers of the fused x pass: every launch-shape variant the tuner picks
// from, dispatched on the grid size.  Instantiated once per compute precision
// (xpass_f64.cu, xpass_f32.cu) so that the two compile in parallel.
#pragma once
#include "ctx.cuh"
#include "launch_cfg.cuh"
#include "passes.cuh"
#include "xfused2.cuh"

// launch-shape variants of the fused x pass (picked by the tuner):
//   0: 1024/L pairs x 128 threads   1: 2048/L pairs x 128 threads
//   2: 1024/L pairs x  64 threads   3: 512/L pairs x 64 threads
template <typename T, int L, int V> struct RowCfgV {
    static constexpr int W = V == 1 ? 2048 : V == 3 ? 512 : 1024;
    static constexpr int TC = L >= W ? 1 : W / L;
    static constexpr int NT = (V >= 2) ? 64 : 128;
    static constexpr size_t SMEM = (size_t)Lay<L, TC, true>::elems * sizeof(cx<T>);
};
//   4: register-resident kernel (k_xfused_reg), 1024/L pairs x 128 threads
//   5, 6, 7: lockstep kernel (k_xfused_ms), forward transforms in groups of 3 / 2 / 1,
//            the last with registers capped for 3 (FP64) or 4 (FP32) CTAs per SM
//   8, 9, 10: staged lockstep kernel (k_xfused_st), the same three groupings,
//            each CTA walking tiles with the next tile's input prefetched
//   11: staged lockstep kernel, groups of 3, with 512/L row pairs (at least one)
//       on 64 threads (128 from L = 1024), so that the CTAs of an SM pass their
//       barriers independently
//   12: as 11 with six CTAs per SM for FP32 (the register file holds 384
//       threads at 168 registers), groups of 2 for FP64
//   13: the launch shape of 12, forward transforms in groups of 2, input rows
//       staged by bulk copies and the Hermitian split done in registers
//       (k_xfused_v2); FP64 at L >= 512 keeps the last physical field in
//       shared memory between the inverse and forward transforms
//   14: as 13 with two physical fields in shared memory (FP64), one (FP32)
template <typename T, int L> struct RowCfgSmall {
    static constexpr int TC = L >= 512 ? 1 : 512 / L;
    static constexpr int NT = L >= 1024 ? 128 : 64;
    static constexpr size_t SMEM = (size_t)Lay<L, TC, true>::elems * sizeof(cx<T>);
};
constexpr int kFusedVariants = HIT3D_FUSED_VARIANTS;


template <typename T, template <class> class OP, int L, int V> static int xfused_LV(hit3d_ctx *c, FusedArgs a)
{
    using RC = RowCfgV<T, L, V>;
    auto k = k_xfused<T, L, RC::TC, RC::NT, T, OP<T>>;
    // transform buffer + the CTA's physical field; one cluster of NIN CTAs per tile
    const size_t smem = 2 * RC::SMEM;
    H3D_TRY(set_smem(k, smem));
    const int tiles = (a.npairs + RC::TC - 1) / RC::TC;
    k<<<dim3(tiles * OP<T>::NIN), RC::NT, smem, c->st>>>(a, twid<T>(c));
    H3D_LAUNCH_CHECK();
    return 0;
}
template <typename T, template <class> class OP, int L> static int xfused_reg_L(hit3d_ctx *c, FusedArgs a)
{
    using RC = RowCfg<T, L>;
    auto k = k_xfused_reg<T, L, RC::TC, RC::NT, T, OP<T>>;
    H3D_TRY(set_smem(k, RC::SMEM));
    k<<<dim3((a.npairs + RC::TC - 1) / RC::TC), RC::NT, RC::SMEM, c->st>>>(a, twid<T>(c));
    H3D_LAUNCH_CHECK();
    return 0;
}
template <typename T, template <class> class OP, int L, int GF, int MINB = 1>
static int xfused_ms_L(hit3d_ctx *c, FusedArgs a)
{
    using RC = RowCfg<T, L>;
    constexpr int NB = OP<T>::NIN > GF ? OP<T>::NIN : GF;  // shared-memory buffers
    auto k = k_xfused_ms<T, L, RC::TC, RC::NT, T, OP<T>, GF, MINB>;
    H3D_TRY(set_smem(k, NB * RC::SMEM));
    k<<<dim3((a.npairs + RC::TC - 1) / RC::TC), RC::NT, NB * RC::SMEM, c->st>>>(a, twid<T>(c));
    H3D_LAUNCH_CHECK();
    return 0;
}
// staged lockstep kernel: a grid of the CTAs that fit at once, each walking tiles
// with the next tile's input rows prefetched into shared memory
template <typename T, template <class> class OP, int L, int GF, int MINB, class RC = RowCfg<T, L>>
static int xfused_st_L(hit3d_ctx *c, FusedArgs a)
{
    constexpr int NIN = OP<T>::NIN;
    constexpr int NB = NIN > GF ? NIN : GF;
    auto k = k_xfused_st<T, L, RC::TC, RC::NT, T, OP<T>, GF, MINB>;
    for (int f = 0; f < NIN; f++)
        if (reinterpret_cast<uintptr_t>(a.in[f]) % 16 != 0)
            return h3d_set_error_msg(-1, "fused x pass: input field not 16-byte aligned");
    if ((a.pitch * (int64_t)sizeof(cx<T>)) % 16 != 0)
        return h3d_set_error_msg(-1, "fused x pass: row pitch not a multiple of 16 bytes");
    auto stage_bytes = [&](int lim) {
        return (size_t)NIN * 2 * RC::TC * StageRow<T>::chunks(lim) * StageRow<T>::PER * sizeof(cx<T>);
    };
    const int lim = a.kx_lim > 0 ? a.kx_lim : L / 2 + 1;
    const size_t soff = (NB * RC::SMEM + 15) / 16 * 16;  // the stage starts on a 16-byte boundary
    const size_t smax = soff + stage_bytes(L / 2 + 1), smem = soff + stage_bytes(lim);
    H3D_TRY(set_smem(k, smax));
    // CTAs per SM: the register cap of the kernel, or fewer if shared memory says so
    // (233472 bytes per SM, 1 KB reserved per CTA)
    int per_sm = (int)(233472 / (smem + 1024));
    per_sm = per_sm < MINB ? per_sm : MINB;
    if (per_sm < 1) return h3d_set_error_msg(-1, "fused x pass: stage does not fit in shared memory");
    const int tiles = (a.npairs + RC::TC - 1) / RC::TC;
    int grid = c->nsm * per_sm;
    grid = grid < tiles ? grid : tiles;
    k<<<dim3(grid), RC::NT, smem, c->st>>>(a, twid<T>(c));
    H3D_LAUNCH_CHECK();
    return 0;
}
// bulk-copy staged form with the split in registers (k_xfused_v2)
template <typename T, template <class> class OP, int L, int MINB, class RC, int NSMF>
static int xfused_v2_L(hit3d_ctx *c, FusedArgs a)
{
    constexpr int NIN = OP<T>::NIN;
    constexpr int NB = (NIN > 2 ? NIN : 2) > 2 + NSMF ? (NIN > 2 ? NIN : 2) : 2 + NSMF;
    auto k = k_xfused_v2<T, L, RC::TC, RC::NT, T, OP<T>, MINB, NSMF>;
    for (int f = 0; f < NIN; f++)
        if (reinterpret_cast<uintptr_t>(a.in[f]) % 16 != 0)
            return h3d_set_error_msg(-1, "fused x pass: input field not 16-byte aligned");
    if ((a.pitch * (int64_t)sizeof(cx<T>)) % 16 != 0)
        return h3d_set_error_msg(-1, "fused x pass: row pitch not a multiple of 16 bytes");
    const int lim = a.kx_lim > 0 ? a.kx_lim : L / 2 + 1;
    // the copied rows are rounded up to 16 bytes and must stay inside the pitch
    if ((int64_t)StageRow<T>::chunks(L / 2 + 1) * StageRow<T>::PER > a.pitch)
        return h3d_set_error_msg(-1, "fused x pass: row pitch too small for the staged rows");
    auto stage_bytes = [&](int l) {
        return (size_t)NIN * 2 * RC::TC * StageRow<T>::chunks(l) * StageRow<T>::PER * sizeof(cx<T>);
    };
    const size_t soff = (NB * RC::SMEM + 15) / 16 * 16;
    const size_t smax = soff + stage_bytes(L / 2 + 1) + 8, smem = soff + stage_bytes(lim) + 8;
    H3D_TRY(set_smem(k, smax));
    int per_sm = (int)(233472 / (smem + 1024));
    per_sm = per_sm < MINB ? per_sm : MINB;
    if (per_sm < 1) return h3d_set_error_msg(-1, "fused x pass: stage does not fit in shared memory");
    const int tiles = (a.npairs + RC::TC - 1) / RC::TC;
    int grid = c->nsm * per_sm;
    grid = grid < tiles ? grid : tiles;
    k<<<dim3(grid), RC::NT, smem, c->st>>>(a, twid<T>(c));
    H3D_LAUNCH_CHECK();
    return 0;
}

template <typename T, template <class> class OP, int L> static int xfused_L(hit3d_ctx *c, FusedArgs a)
{
    if constexpr (OP<T>::NIN <= 3) {
        if (c->xcfg == 13 || c->xcfg == 14) {
            // 13: FP64 at L >= 512 keeps one physical field in shared memory
            // (registers), the rest none; 14: two (FP64) or one (FP32)
            using RS = RowCfgSmall<T, L>;
            constexpr int N13 = (sizeof(T) == 8 && L >= 512 && OP<T>::NIN == 3) ? 1 : 0;
            constexpr int N14 = OP<T>::NIN < 3 ? 0 : sizeof(T) == 8 ? 2 : 1;
            if constexpr (sizeof(T) == 4) {
                if (c->xcfg == 13) return xfused_v2_L<T, OP, L, 384 / RS::NT, RS, N13>(c, a);
                return xfused_v2_L<T, OP, L, 384 / RS::NT, RS, N14>(c, a);
            } else {
                if (c->xcfg == 13) return xfused_v2_L<T, OP, L, 256 / RS::NT, RS, N13>(c, a);
                return xfused_v2_L<T, OP, L, 256 / RS::NT, RS, N14>(c, a);
            }
        }
        if (c->xcfg == 8) return xfused_st_L<T, OP, L, 3, 2>(c, a);
        if (c->xcfg == 9) return xfused_st_L<T, OP, L, 2, 2>(c, a);
        if (c->xcfg == 10) return xfused_st_L<T, OP, L, 1, sizeof(T) == 4 ? 4 : 3>(c, a);
        if (c->xcfg == 11) {
            using RS = RowCfgSmall<T, L>;  // 256 threads per SM at the full register file
            return xfused_st_L<T, OP, L, 3, 256 / RS::NT, RS>(c, a);
        }
        if (c->xcfg == 12) {
            using RS = RowCfgSmall<T, L>;
            if constexpr (sizeof(T) == 4) return xfused_st_L<T, OP, L, 3, 384 / RS::NT, RS>(c, a);  // 168 registers
            else return xfused_st_L<T, OP, L, 2, 256 / RS::NT, RS>(c, a);
        }
        if (c->xcfg == 5) return xfused_ms_L<T, OP, L, 3>(c, a);
        if (c->xcfg == 6) return xfused_ms_L<T, OP, L, 2>(c, a);
        if (c->xcfg == 7) return xfused_ms_L<T, OP, L, 1, sizeof(T) == 4 ? 4 : 3>(c, a);
    }
    if (c->xcfg >= 4) return xfused_reg_L<T, OP, L>(c, a);
    if constexpr (L >= 128) {
        switch (c->xcfg) {
        case 1: return xfused_LV<T, OP, L, 1>(c, a);
        case 2: return xfused_LV<T, OP, L, 2>(c, a);
        case 3: return xfused_LV<T, OP, L, 3>(c, a);
        default: break;
        }
    }
    return xfused_LV<T, OP, L, 0>(c, a);
}
template <typename T, template <class> class OP> int xfused(hit3d_ctx *c, FusedArgs a)
{
    a.npairs = c->n * c->n / 2;
    if (c->bruns > 0) {
        // every run of a batch class: only the staged kernels walk the tiles of
        // several runs (variants 8-13); others take variant 13's
        if constexpr (OP<T>::NIN > 3) return h3d_set_error_msg(-1, "fused x pass: batch classes carry the velocity only");
        a.nruns = c->bruns;
        a.rstride = c->brw;
        a.cmax = nullptr;
        a.phys = nullptr;
        if (c->xcfg < 8) {
            const int saved = c->xcfg;
            c->xcfg = 13;
            a.norm = 1.0 / ((double)c->n * c->n * c->n);
            a.kx_lim = c->kc_active >= 0 ? c->kc_active + 1 : 0;
#define CALL(L) xfused_L<T, OP, L>(c, a)
            int rc = 0;
            switch (c->n) {
            case 32: rc = CALL(32); break;
            case 48: rc = CALL(48); break;
            case 64: rc = CALL(64); break;
            case 128: rc = CALL(128); break;
            case 256: rc = CALL(256); break;
            case 512: rc = CALL(512); break;
            case 1024: rc = CALL(1024); break;
            default: rc = h3d_set_error_msg(-3, "unsupported grid size");
            }
#undef CALL
            c->xcfg = saved;
            return rc;
        }
    }
    const double n3 = (double)c->n * c->n * c->n;
    a.norm = 1.0 / n3;
    a.kx_lim = c->kc_active >= 0 ? c->kc_active + 1 : 0;
#define CALL(L) xfused_L<T, OP, L>(c, a)
    H3D_DISPATCH(c->n, CALL)
#undef CALL
}


#define H3D_XPASS_INSTANTIATE(T)                                  \
    template int xfused<T, OpVel>(hit3d_ctx *, FusedArgs);        \
    template int xfused<T, OpScal>(hit3d_ctx *, FusedArgs);       \
    template int xfused<T, OpSmag>(hit3d_ctx *, FusedArgs);
