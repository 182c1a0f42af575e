// Launch shapes of the transform passes per transform length, shared by every
// translation unit that launches them (the context path and the allocation-free
// entry point), so that both run the configurations the tests cover.
#pragma once
#include "passes.cuh"

H3D_HD constexpr int plan_rmax(int L)
{
    int r = 0;
    for (int s = 0; s < plan_stages(L); s++) r = plan_radix_fwd(L, s) > r ? plan_radix_fwd(L, s) : r;
    return r;
}
template <typename T, int L, bool YPASS = false> struct ColCfg {
    // 128-byte rows of kx columns; the FP64 y passes at L = 1024 take 64-byte
    // rows, so that a CTA's shared memory (TC x L elements) leaves room for two
    // CTAs per SM (measured faster there, slower for the z passes and FP32)
    static constexpr int TC = sizeof(T) == 8 ? ((L >= 1024 && YPASS) ? 4 : 8) : 16;
    static constexpr int NT0 = TC * L / plan_rmax(L);
    // one 8-element butterfly set per thread where 512 threads allow it; the
    // FP64 y passes at L = 1024 keep 256 threads (measured faster there)
    static constexpr int NTMAX = (sizeof(T) == 8 && L >= 1024 && YPASS) ? 256 : 512;
    static constexpr int NT = NT0 > NTMAX ? NTMAX : NT0;
    static constexpr size_t SMEM = (size_t)Lay<L, TC, false>::elems * sizeof(cx<T>);
};
template <typename T, int L> struct RowCfg {
    static constexpr int TC = L >= 1024 ? 1 : 1024 / L;  // row pairs per CTA
    static constexpr int NT = 128;
    static constexpr size_t SMEM = (size_t)Lay<L, TC, true>::elems * sizeof(cx<T>);
};

// Column-tile shapes the tuners pick from (ct = the context's `ctile`): 0 the
// default ColCfg, 1 half as many kx columns per CTA, 2 twice as many (grids up
// to 512; at least one warp per CTA), 3 the pipelined pass (k_colfft_pipe,
// every grid)
constexpr int kColTiles = 4;
template <typename T, int L, bool YPASS, int CT> struct ColCfgT {
    using B = ColCfg<T, L, YPASS>;
    static constexpr int TC = CT == 0 ? B::TC : CT == 1 ? B::TC / 2 : B::TC * 2;
    static constexpr int NT0 = TC * L / plan_rmax(L);
    static constexpr int NT = CT == 0 ? B::NT : NT0 < 32 ? 32 : NT0 > 512 ? 512 : NT0;
    static constexpr size_t SMEM = (size_t)Lay<L, TC, false>::elems * sizeof(cx<T>);
    // resident CTAs the register cap allows: the default shape's, or four for
    // the narrow tiles of up to 256 threads and 56 KB
    static constexpr int MINB = CT == 1 && NT <= 256 && SMEM <= 56 * 1024 ? 4 : ColMinBlocks<T, L, TC, NT>::value;
};
