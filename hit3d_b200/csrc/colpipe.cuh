// Pipelined form of the strided (y and z) passes.
//
// k_colfft loads a CTA's tile of TC kx columns x L positions straight into
// registers, transforms it and stores it: a CTA's loads and its shared-memory
// stages do not overlap, and at the column passes' two resident CTAs per SM the
// global-load latency shows (the passes reach 0.7-0.8 of the copy bandwidth
// in FP64, 0.6-0.7 in FP32).  Here a grid of resident CTAs walks the tiles, and
// each CTA brings the tile after next into one of two shared-memory buffers by
// cp.async (16- or 8-byte copies, zero-filled for the positions the 2/3 rule
// prunes and for columns beyond the last) while it transforms the current tile
// in the other buffer, which then serves as the exchange buffer of the radix
// stages.  The arithmetic is k_colfft's, operation for operation: the two
// forms give bit-identical fields.
//
// Supported inputs: IOPlain (every y and z pass) and IOSpec<PRE_COPY> (the z
// pass that reads the FP64 state); other pre-operations keep k_colfft.
#pragma once
#include "launch_cfg.cuh"

// a cp.async of one element (8 or 16 bytes) that writes zeros when !valid
template <int BYTES> H3D_D void cp_async_elem(void *smem, const void *gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const unsigned src_size = valid ? BYTES : 0;
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_size) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gmem), "n"(BYTES), "r"(src_size)
                     : "memory");
}
H3D_D void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// raw source of element (f, o, c, p) of a pass's input, and whether it is
// loaded (false: the element is zero: a column beyond ncol or a pruned position)
template <typename T, typename TI, typename TO> H3D_D const cx<TI> *col_src(const IOPlain<T, TI, TO> &io, int f, int o,
                                                                         int c, int p, bool &valid)
{
    valid = c < io.ncol && (io.kl < 0 || kept(p, io.n, io.kl));
    return io.src + (valid ? f * io.fs_src + p * io.sa_src + o * io.so_src + c : 0);
}
template <typename T, typename TO> H3D_D const double2 *col_src(const IOSpec<T, TO, PRE_COPY> &io, int f, int o, int c,
                                                              int p, bool &valid)
{
    valid = c < io.ncol && (io.kl < 0 || kept(p, io.n, io.kl));
    return io.src + (valid ? f * io.fs_src + ((int64_t)p * io.n + o) * io.psrc + c : 0);
}
template <class IO> struct ColIn;
template <typename T, typename TI, typename TO> struct ColIn<IOPlain<T, TI, TO>> { using type = TI; };
template <typename T, typename TO> struct ColIn<IOSpec<T, TO, PRE_COPY>> { using type = double; };

// launch shape: 64-byte rows of input columns, at most 32 KB per buffer, so
// that several CTAs share an SM
template <typename T, typename TI, int L> struct ColPipeCfg {
    static constexpr int ES = sizeof(cx<TI>) > sizeof(cx<T>) ? (int)sizeof(cx<TI>) : (int)sizeof(cx<T>);
    static constexpr int TC0 = 64 / (int)sizeof(cx<TI>);
    static constexpr int TC = (size_t)TC0 * L * ES <= 32 * 1024 ? TC0 : (int)(32 * 1024 / ((size_t)L * ES));
    static constexpr int NT0 = TC * L / plan_rmax(L);
    static constexpr int NT = NT0 > 512 ? 512 : NT0 < 32 ? 32 : NT0;
    static constexpr size_t BUF = (size_t)Lay<L, TC, false>::elems * ES;  // bytes of one buffer
    static constexpr size_t SMEM = 2 * BUF;
    // CTAs per SM: as many as the shared memory holds, keeping 64 registers a thread
    static constexpr int BY_SMEM = (int)(220 * 1024 / SMEM), BY_REGS = 1024 / NT;
    static constexpr int MINB = BY_SMEM < 1 ? 1 : BY_SMEM > BY_REGS ? BY_REGS : BY_SMEM;
};

// tile t -> (grid index z of the field, outer index y, column tile x)
struct ColTiles {
    int nx, ny;
    H3D_D void at(int t, int &x, int &y, int &z) const
    {
        x = t % nx;
        const int r = t / nx;
        y = r % ny;
        z = r / ny;
    }
};

template <typename T, int L, int TC, int NT, bool FWD, class IO, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_colfft_pipe(const IO io, const cx<T> *__restrict__ tw, ColTiles tl, int ntiles)
{
    using TI = typename ColIn<IO>::type;
    using F = ColFFT<T, L, TC, NT, false, FWD, false>;
    using LY = Lay<L, TC, false>;
    constexpr int ES = sizeof(cx<TI>) > sizeof(cx<T>) ? (int)sizeof(cx<TI>) : (int)sizeof(cx<T>);
    constexpr size_t BUF = (size_t)LY::elems * ES;
    extern __shared__ __align__(16) unsigned char smraw[];

    // copies of tile t's stage-0 inputs into buffer b (each thread its own slots)
    auto issue = [&](int t, int b) {
        if (t < ntiles) {
            int x, y, z, f;
            tl.at(t, x, y, z);
            const IO iob = io.at(z, f);
            const int col0 = x * TC, outer = iob.outer(y);
            cx<TI> *buf = reinterpret_cast<cx<TI> *>(smraw + b * BUF);
#pragma unroll
            for (int i = 0; i < F::NB0; i++)
#pragma unroll
                for (int m = 0; m < F::R0; m++) {
                    int c, p;
                    if (F::in_slot(i, m, c, p)) {
                        bool valid;
                        const cx<TI> *src = col_src(iob, f, outer, col0 + c, p, valid);
                        cp_async_elem<(int)sizeof(cx<TI>)>(buf + LY::idx(c, p), src, valid);
                    }
                }
        }
        cp_async_commit();  // an empty group past the last tile keeps the counting uniform
    };

    const int t0 = blockIdx.x;
    issue(t0, 0);
    issue(t0 + (int)gridDim.x, 1);
    int b = 0;
#pragma unroll 1
    for (int t = t0; t < ntiles; t += gridDim.x, b ^= 1) {
        cp_async_wait_one();  // this tile's copies are done (the next tile's may still run)
        int x, y, z, f;
        tl.at(t, x, y, z);
        const IO iob = io.at(z, f);
        const int col0 = x * TC, outer = iob.outer(y);
        const cx<TI> *buf = reinterpret_cast<const cx<TI> *>(smraw + b * BUF);
        cx<T> in[F::NIN];
#pragma unroll
        for (int i = 0; i < F::NB0; i++)
#pragma unroll
            for (int m = 0; m < F::R0; m++) {
                int c, p;
                if (F::in_slot(i, m, c, p)) in[i * F::R0 + m] = to_cx<T>(buf[LY::idx(c, p)]);
            }
        __syncthreads();  // every thread has read its inputs: the buffer turns into the exchange buffer
        cx<T> *sm = reinterpret_cast<cx<T> *>(smraw + b * BUF);
        F::run_store(in, sm, tw, [&](int c, int p, cx<T> v) { iob.store(f, outer, col0 + c, p, v); });
        __syncthreads();  // the last stage has read the buffer: it may be refilled
        issue(t + 2 * (int)gridDim.x, b);
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
