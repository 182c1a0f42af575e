// The z forward pass of the six velocity products fused with the 2/3-rule
// update (rhs_velocity.f90:85-142, m_force.f90:158-171, main.f90:156-164,
// pressure.f90:13-47) and, when asked, with the next step's z inverse of the
// new state (the first pass of xFFT3d(-1), x_fftw.f90:976-1082).
//
// A grid of resident CTAs walks the tiles: one ky row (a kept one when the
// state is pruned) x TC kx columns x every z.  Per tile a CTA
//  A. transforms the six product columns along z one after the other.  Their
//     columns reach shared memory by cp.async, NB product tiles ahead of the
//     transform (each thread copies its own stage-0 slots, so the staging ring
//     needs no barrier of its own), and every last-stage output adds k_j P_ij
//     to three per-slot accumulators in registers;
//  B. updates the tile's modes as k_update_vel_23 does (RHS, band forcing,
//     AB2, projection), the sums k.P rounded in the same order (kdot3), so the
//     two paths give identical fields;
//  C. (zinv) transforms the new u, v, w back along z from the registers the
//     update left them in and writes them over the tile's first three work
//     fields, which hold only this tile's products, already read: the next
//     step's y inverse starts from them, and its own z inverse is skipped.
// The six product spectra never reach HBM, and the next step does not read
// the new state back for its z inverse: per step this saves 12 + 3 kept-mode
// field passes of the 2/3-rule pipeline's HBM traffic.  It is nonetheless
// slower than the separate passes (every CTA runs nine transforms, an update
// and their waits one after another, at 8 warps per SM), so the context keeps
// it off unless hit3d_gpu_set_update_fusion turns it on.
#pragma once
#include "fft.cuh"
#include "passes.cuh"
#include "spectral.cuh"
#include "launch_cfg.cuh"
#include "colpipe.cuh"

template <int N> H3D_D void cp_async_wait_n() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// k v and k v + a, each rounded once, in the accumulator precision
H3D_D double zmul(double k, double v) { return __dmul_rn(k, v); }
H3D_D float zmul(float k, float v) { return __fmul_rn(k, v); }
H3D_D double zfma(double k, double v, double a) { return __fma_rn(k, v, a); }
H3D_D float zfma(float k, float v, float a) { return __fmaf_rn(k, v, a); }

// last-stage slot m of a z transform of length L with radix RL holds
// positions j + m L/RL (j < L/RL): true when all of them lie beyond the
// 2/3-rule cutoff L/3, so that a pruned step never reads or writes them
H3D_HD constexpr bool zdead(int L, int RL, int m)
{
    return (m * (L / RL) > L / 3) && ((m + 1) * (L / RL) - 1 < L - L / 3);
}

// The sums k_j P_cj are accumulated in FP64 in both precisions, rounded as
// kdot3 rounds them, so the fused and the separate passes agree exactly (FP32
// accumulators in the FP32 form measured no faster: the kernel is bound by
// the latency of its sequential phases, not by their registers).
template <typename T> using ZAcc = double;

template <typename T, int L> struct ZUpdCfg {
    // 32-byte column segments (2 FP64 or 4 FP32 kx columns)
    static constexpr int TC = 32 / (int)sizeof(cx<T>);
    static constexpr int NT0 = TC * L / plan_rmax(L);
    static constexpr int NT = NT0 < 32 ? 32 : NT0 > 512 ? 512 : NT0;
    // resident CTAs: as many as leave each thread 255 registers (the three
    // FP64 accumulators per slot and a transform in flight spill below that)
    static constexpr int BY_REGS0 = 65536 / (NT * 256);
    static constexpr int MINB = BY_REGS0 < 1 ? 1 : BY_REGS0 > 4 ? 4 : BY_REGS0;
    static constexpr size_t BUF = (size_t)Lay<L, TC, false>::elems * sizeof(cx<T>);
    // product tiles in the staging ring: as many as about 200 KB of shared
    // memory per SM holds next to the exchange buffers, 2 to 8
    static constexpr int NB0 = (int)(200 * 1024 / ((size_t)MINB * BUF)) - 1;
    static constexpr int NB = NB0 < 2 ? 2 : NB0 > 8 ? 8 : NB0;
    static constexpr size_t SMEM = (size_t)(1 + NB) * BUF;  // exchange buffer + ring
};

template <typename T> struct ZUpdArgs {
    StepArgs a;      // update parameters; a.ppitch / a.pfs: pitch and field stride of W
    cx<T> *W;        // work fields [z][ky][kx]: the six products after their y pass; z inverse out in W[0..2]
    double2 *U, *RO;
    int ncol, nrows;  // kx columns and ky rows the pass visits
    int zinv;         // write the z inverse of the new u, v, w into W[0..2]
};

template <typename T, int L, int TC, int NT, int NB, int MINB, bool PRUNED>
__global__ void __launch_bounds__(NT, MINB) k_zfwd_update(const ZUpdArgs<T> za, const cx<T> *__restrict__ tw)
{
    using F = ColFFT<T, L, TC, NT, false, true, false>;    // forward z, as the plain z pass
    using FI = ColFFT<T, L, TC, NT, false, false, false>;  // inverse z, as the plain z inverse
    using LY = Lay<L, TC, false>;
    constexpr int E = LY::elems;
    constexpr int RL = F::RL, NOUT = F::NOUT;
    // the update's slots feed the inverse's stage 0 directly when both stages
    // map threads to the same butterflies
    constexpr bool HANDOFF = F::RL == FI::R0 && F::NBL == FI::NB0;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    cx<T> *stg = sm + E;
    const StepArgs &a = za.a;
    const int n = a.n, kc = a.kc;
    const int nxt = (za.ncol + TC - 1) / TC;
    const int ntiles = nxt * za.nrows;
    const int64_t zs = (int64_t)n * a.ppitch;  // z stride of the work fields

    auto tile_of = [&](int t, int &col0, int &kyi) {
        const int y = t / nxt;
        col0 = (t - y * nxt) * TC;
        kyi = PRUNED ? kept_index(y, n, kc) : y;
    };
    // item k of this CTA: product k % 6 of its (k / 6)-th tile, into ring buffer k % NB
    auto issue = [&](int k) {
        const int t = (int)blockIdx.x + (k / 6) * (int)gridDim.x;
        if (t < ntiles) {
            int col0, kyi;
            tile_of(t, col0, kyi);
            const cx<T> *P = za.W + (int64_t)(k % 6) * a.pfs + (int64_t)kyi * a.ppitch + col0;
            cx<T> *buf = stg + (k % NB) * E;
#pragma unroll
            for (int i = 0; i < F::NB0; i++)
#pragma unroll
                for (int m = 0; m < F::R0; m++) {
                    int c, p;
                    if (F::in_slot(i, m, c, p)) {
                        const bool v = col0 + c < za.ncol;
                        cp_async_elem<(int)sizeof(cx<T>)>(buf + LY::idx(c, p), v ? P + p * zs + c : za.W, v);
                    }
                }
        }
        cp_async_commit();  // an empty group past the last tile keeps the counting uniform
    };

#pragma unroll 1
    for (int k = 0; k < NB; k++) issue(k);
    const double nu = a.nu, dt = a.dt;
    const double fac = (a.flow_type == 1) ? a.famp / *a.fenergy : 0.0;
    int k = 0;
#pragma unroll 1
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, k += 6) {
        int col0, kyi;
        tile_of(t, col0, kyi);
        const double ky = kwave(kyi, n);
        // acc[c][q] = k_x P_c1 + k_y P_c2 + k_z P_c3 of slot q, rounded as kdot3
        using A = ZAcc<T>;
        cx<A> acc[3][NOUT];
        const A kya = (A)ky;
#pragma unroll
        for (int f = 0; f < 6; f++) {
            cp_async_wait_n<NB - 1>();  // item k + f has landed (in this thread's slots)
            cx<T> in[F::NIN];
            const cx<T> *buf = stg + ((k + f) % NB) * E;
#pragma unroll
            for (int i = 0; i < F::NB0; i++)
#pragma unroll
                for (int m = 0; m < F::R0; m++) {
                    int c, p;
                    if (F::in_slot(i, m, c, p)) in[i * F::R0 + m] = buf[LY::idx(c, p)];
                }
            // the twiddles are the same for every transform: an opaque copy of the
            // table pointer per transform keeps the compiler from holding them
            // in registers across the six (they are L1 hits)
            const cx<T> *twf = tw;
            asm volatile("" : "+l"(twf));
            F::run_slots_t(in, sm, GlobalTw<T>{twf}, [&](int i, int m, int c, int p, cx<T> v) {
                if (PRUNED && zdead(L, RL, m)) return;
                const int q = i * RL + m;
                const A kx = (A)(col0 + c), kz = (A)kwave(p, n), ky = kya;
                const A vx = (A)v.x, vy = (A)v.y;
                // products uu uv uw vv vw ww
                if (f == 0) acc[0][q] = mk<A>(zmul(kx, vx), zmul(kx, vy));
                if (f == 1) {
                    acc[0][q] = mk<A>(zfma(ky, vx, acc[0][q].x), zfma(ky, vy, acc[0][q].y));
                    acc[1][q] = mk<A>(zmul(kx, vx), zmul(kx, vy));
                }
                if (f == 2) {
                    acc[0][q] = mk<A>(zfma(kz, vx, acc[0][q].x), zfma(kz, vy, acc[0][q].y));
                    acc[2][q] = mk<A>(zmul(kx, vx), zmul(kx, vy));
                }
                if (f == 3) acc[1][q] = mk<A>(zfma(ky, vx, acc[1][q].x), zfma(ky, vy, acc[1][q].y));
                if (f == 4) {
                    acc[1][q] = mk<A>(zfma(kz, vx, acc[1][q].x), zfma(kz, vy, acc[1][q].y));
                    acc[2][q] = mk<A>(zfma(ky, vx, acc[2][q].x), zfma(ky, vy, acc[2][q].y));
                }
                if (f == 5) acc[2][q] = mk<A>(zfma(kz, vx, acc[2][q].x), zfma(kz, vy, acc[2][q].y));
            });
            __syncthreads();  // the exchange buffer is free again; every thread has read its staged slots
            issue(k + f + NB);
        }

        // B: the update of the tile's modes; the new state stays in un[][] for C
        cx<T> un[3][NOUT];
#pragma unroll
        for (int i = 0; i < F::NBL; i++)
#pragma unroll
            for (int m = 0; m < RL; m++) {
                const int q = i * RL + m;
#pragma unroll
                for (int cc = 0; cc < 3; cc++) un[cc][q] = mk<T>(0, 0);
                int c, p;
                if (!F::out_slot(i, m, c, p)) continue;
                if (PRUNED && (zdead(L, RL, m) || !kept(p, n, kc))) continue;
                if (col0 + c >= za.ncol) continue;
                const ModeIdx md = mode_from(col0 + c, kyi, p, n);
                const int64_t o = soff(md, n, a.pitch);
                double2 u[3] = {za.U[o], za.U[o + a.fs], za.U[o + 2 * a.fs]};
                double2 r[3];
                if (md.ialias > 0) {
                    r[0] = r[1] = r[2] = make_double2(0.0, 0.0);
                } else {
                    const double2 s[3] = {make_double2((double)acc[0][q].x, (double)acc[0][q].y),
                                          make_double2((double)acc[1][q].x, (double)acc[1][q].y),
                                          make_double2((double)acc[2][q].x, (double)acc[2][q].y)};
                    vel23_rhs(md, s, u, nu, r);
                }
                if (a.flow_type == 1 && forced(md, n, a.kfmax)) {
#pragma unroll
                    for (int cc = 0; cc < 3; cc++) { r[cc].x = r[cc].x + fac * u[cc].x; r[cc].y = r[cc].y + fac * u[cc].y; }
                }
                double2 ro[3] = {za.RO[o], za.RO[o + a.fs], za.RO[o + 2 * a.fs]};
#pragma unroll
                for (int cc = 0; cc < 3; cc++) ab2(u[cc], ro[cc], r[cc], dt, a.euler_v);
                project(md, u[0], u[1], u[2]);
#pragma unroll
                for (int cc = 0; cc < 3; cc++) {
                    za.U[o + cc * a.fs] = u[cc];
                    za.RO[o + cc * a.fs] = ro[cc];
                    un[cc][q] = to_cx<T>(u[cc]);
                }
            }

        // C: the next step's z inverse of u, v, w over the tile's first three work fields
        if (za.zinv) {
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
                cx<T> in[FI::NIN];
                if constexpr (HANDOFF) {
#pragma unroll
                    for (int q = 0; q < FI::NIN; q++) in[q] = un[cc][q];
                } else {
                    // different butterfly maps: through the exchange buffer
#pragma unroll
                    for (int i = 0; i < F::NBL; i++)
#pragma unroll
                        for (int m = 0; m < RL; m++) {
                            int c, p;
                            if (F::out_slot(i, m, c, p)) sm[LY::idx(c, p)] = un[cc][i * RL + m];
                        }
                    __syncthreads();
#pragma unroll
                    for (int i = 0; i < FI::NB0; i++)
#pragma unroll
                        for (int m = 0; m < FI::R0; m++) {
                            int c, p;
                            if (FI::in_slot(i, m, c, p)) in[i * FI::R0 + m] = sm[LY::idx(c, p)];
                        }
                    __syncthreads();
                }
                cx<T> *dst = za.W + (int64_t)cc * a.pfs + (int64_t)kyi * a.ppitch + col0;
                const cx<T> *twf = tw;
                asm volatile("" : "+l"(twf));
                FI::run_store(in, sm, twf, [&](int c, int p, cx<T> v) {
                    if (col0 + c < za.ncol) dst[p * zs + c] = v;
                });
                __syncthreads();  // the exchange buffer is read: the next transform may overwrite it
            }
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
