// Fused x pass, form with bulk-copy staging and the Hermitian split in registers
// (launch-shape variant 13).
//
// Same work as k_xfused_st (inverse c2r of the NIN inputs in lockstep, the
// per-point operator, forward r2c of the NOUT outputs in groups of two), with
// two changes to the data movement:
//
//  * the next row pair's input rows reach shared memory as whole-row bulk
//    copies (cp.async.bulk, one thread, completion counted in bytes on an
//    mbarrier) instead of one 16-byte cp.async per thread and chunk;
//  * the last radix stage of the forward transforms maps each thread to the
//    two butterflies j and B - j (B butterflies per stage) whose outputs are
//    the Hermitian partners Z[k] and Z[L - k] of the two packed real rows.  The
//    thread splits them into the two rows' half spectra in registers and
//    stores them to HBM directly (coalesced: neighbouring threads hold
//    neighbouring k), so the last stage's outputs never go back through shared
//    memory and the split needs no extra barrier.
//
// The arithmetic is k_xfused_st's except for the last-stage twiddles of the
// butterflies B - q, formed from those of q by a root of unity (one table load
// per pair of butterflies): the two forms agree to rounding.
#pragma once
#include "passes.cuh"

constexpr unsigned XF_WAIT_LIMIT = 1u << 24;  // polls of the stage barrier before the kernel gives up

H3D_D unsigned xf_smem(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

H3D_D void xf_mbar_init(uint64_t *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(xf_smem(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait for the phase of the given parity to complete
H3D_D bool xf_mbar_wait(uint64_t *bar, unsigned parity)
{
    const unsigned b = xf_smem(bar);
    for (unsigned it = 0; it < XF_WAIT_LIMIT; it++) {
        unsigned ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(ok)
                     : "r"(b), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}

// One thread: the input rows (kx < lim, rounded up to 16 bytes) of the TC row
// pairs starting at pair0, NIN fields, into the stage [f][row][rs], completion
// counted in bytes on `bar`.  Rows of pairs beyond npairs are not copied.
// Sources: 16-byte aligned fields and a row pitch of a multiple of 16 bytes
// (checked by the host), and the rounded row stays inside the pitch.
template <typename TS, int NIN, int TC>
H3D_D void xf_stage_issue(const FusedArgs &a, cx<TS> *st, uint64_t *bar, int pair0, int rs, int64_t roff)
{
    const int np = a.npairs - pair0 < TC ? a.npairs - pair0 : TC;
    const unsigned row_bytes = (unsigned)rs * (unsigned)sizeof(cx<TS>);
    // the stage was last read by generic loads of every thread (ordered before
    // this point by a barrier); order them before the asynchronous writes
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(xf_smem(bar)),
                 "r"((unsigned)(NIN * 2 * np) * row_bytes)
                 : "memory");
#pragma unroll
    for (int f = 0; f < NIN; f++)
        for (int r = 0; r < 2 * np; r++) {
            const cx<TS> *src = reinterpret_cast<const cx<TS> *>(a.in[f]) + roff + (int64_t)(2 * pair0 + r) * a.pitch;
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             xf_smem(st + (f * 2 * TC + r) * rs)),
                         "l"(src), "r"(row_bytes), "r"(xf_smem(bar))
                         : "memory");
        }
}

// Hermitian split of Z[k] (zk) with its partner Z[L - k] (zm) into the half
// spectra of the two packed rows (the arithmetic of store_split), stored at k.
template <typename T, typename TS>
H3D_D void xf_split_store(cx<TS> *A, int64_t pitch, int k, cx<T> zk, cx<T> zm, T half)
{
    cx<TS> xa, xb;
    xa.x = (TS)(half * (zk.x + zm.x));
    xa.y = (TS)(half * (zk.y - zm.y));
    xb.x = (TS)(half * (zk.y + zm.y));
    xb.y = (TS)(-half * (zk.x - zm.x));
    A[k] = xa;
    A[pitch + k] = xb;
}

// exp(-2 pi i m / R) for the radices of the last stages (R = 3, 4, 8) and
// exp(-2 pi i m / (2 R)), correctly rounded: the twiddle of butterfly B - q is
// w_R^m conj(w^(q m)), and that of butterfly B / 2 is w_(2R)^m
template <typename T, int R> H3D_D cx<T> root_of_unity(int m)
{
    constexpr double h = 0.70710678118654752440084436210484904;   // sqrt(1/2)
    constexpr double c8 = 0.92387953251128675612818318939678829;  // cos(pi/8)
    constexpr double s8 = 0.38268343236508977172845998403039887;  // sin(pi/8)
    constexpr double s3 = 0.86602540378443864676372317075293618;  // sin(pi/3)
    double re = 1.0, im = 0.0;
    if constexpr (R == 16) {
        const double c[16] = {1, c8, h, s8, 0, -s8, -h, -c8, -1, -c8, -h, -s8, 0, s8, h, c8};
        const double s[16] = {0, -s8, -h, -c8, -1, -c8, -h, -s8, 0, s8, h, c8, 1, c8, h, s8};
        re = c[m]; im = s[m];
    } else if constexpr (R == 8) {
        const double c[8] = {1, h, 0, -h, -1, -h, 0, h};
        const double s[8] = {0, -h, -1, -h, 0, h, 1, h};
        re = c[m]; im = s[m];
    } else if constexpr (R == 6) {
        const double c[6] = {1, 0.5, -0.5, -1, -0.5, 0.5};
        const double s[6] = {0, -s3, -s3, 0, s3, s3};
        re = c[m]; im = s[m];
    } else if constexpr (R == 4) {
        const double c[4] = {1, 0, -1, 0};
        const double s[4] = {0, -1, 0, 1};
        re = c[m]; im = s[m];
    } else if constexpr (R == 3) {
        const double c[3] = {1, -0.5, -0.5};
        const double s[3] = {0, -s3, s3};
        re = c[m]; im = s[m];
    } else {
        static_assert(R == 3 || R == 4 || R == 6 || R == 8 || R == 16, "root of unity");
    }
    return mk<T>((T)re, (T)im);
}

// Last radix stage of NF forward row transforms whose inputs sit in buffers
// sm + f * elems (after FF::run_multi_front), with the split and the stores.
// Unit u of a transform takes butterflies j1 = q and j2 = B - q (q > 0), or 0
// and B / 2 (q = 0); q runs fastest over the threads.  out[f] == nullptr skips
// transform f.
template <typename T, int L, int TC, int NT, int NF, typename TS>
H3D_D void xf_last_split(const cx<T> *sm, const cx<T> *__restrict__ tw, void *const (&out)[NF], int64_t pitch,
                         int pair0, int npairs, int lim, T half)
{
    using P = Plan<L, false>;
    using LY = Lay<L, TC, true>;
    constexpr int S = P::S, RL = P::R(S - 1), B = L / RL, HU = B / 2;
    static_assert(P::Ns(S - 1) == B, "last stage");
    constexpr int TOT = TC * NF * HU, UPT = (TOT + NT - 1) / NT, E = LY::elems;
#pragma unroll
    for (int i = 0; i < UPT; i++) {
        const int u = threadIdx.x + i * NT;
        if (TOT % NT != 0 && u >= TOT) continue;
        const int q = u % HU, fc = u / HU, f = fc % NF, c = fc / NF;
        const int j1 = q, j2 = q == 0 ? B / 2 : B - q;
        const cx<T> *b = sm + f * E;
        cx<T> v1[RL], v2[RL];
#pragma unroll
        for (int m = 0; m < RL; m++) {
            cx<T> x1 = b[LY::idx(c, j1 + m * B)], x2 = b[LY::idx(c, j2 + m * B)];
            if (m > 0) {
                // one table twiddle per m: w^((B - q) m) = w_RL^m conj(w^(q m))
                const cx<T> w1 = twid<T, true>(tw, j1 * m);
                const cx<T> w2 = q == 0 ? root_of_unity<T, 2 * RL>(m) : cmul(root_of_unity<T, RL>(m), conjg(w1));
                x1 = cmul(x1, w1);
                x2 = cmul(x2, w2);
            }
            v1[m] = x1;
            v2[m] = x2;
        }
        dft<T, RL, true>(v1);
        dft<T, RL, true>(v2);
        if (out[f] == nullptr || pair0 + c >= npairs) continue;
        cx<TS> *A = reinterpret_cast<cx<TS> *>(out[f]) + (int64_t)(2 * (pair0 + c)) * pitch;
#pragma unroll
        for (int m = 0; m < RL; m++) {
            const int k1 = j1 + m * B, k2 = j2 + m * B;
            if (k1 < lim) xf_split_store<T, TS>(A, pitch, k1, v1[m], q == 0 ? v1[(RL - m) % RL] : v2[RL - 1 - m], half);
            if (k2 < lim) xf_split_store<T, TS>(A, pitch, k2, v2[m], q == 0 ? v2[RL - 1 - m] : v1[RL - 1 - m], half);
        }
    }
}

// NSMF: the last NSMF input fields wait in shared memory between the inverse
// and the forward transforms (in the exchange buffers the forward groups of
// two leave free), each thread at its own slots, which frees their registers
// for the forward transforms (FP64 at L >= 512 otherwise spills)
template <typename T, int L, int TC, int NT, typename TS, class OP, int MINB, int NSMF = 0>
__global__ void __launch_bounds__(NT, MINB) k_xfused_v2(const FusedArgs a, const cx<T> *__restrict__ tw)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    using FI = RowFFT<T, L, TC, NT, true>;
    using FF = RowFFT<T, L, TC, NT, false>;
    static_assert(FI::NOUT == FF::NIN, "slot hand-off mismatch");
    constexpr int GF = 2;
    constexpr int NP = FI::NOUT;
    constexpr int E = Lay<L, TC, true>::elems;
    constexpr int NB = (OP::NIN > GF ? OP::NIN : GF) > GF + NSMF ? (OP::NIN > GF ? OP::NIN : GF) : GF + NSMF;
    static_assert(NSMF >= 0 && NSMF < OP::NIN, "fields kept in shared memory");
    constexpr size_t SOFF = ((size_t)NB * E * sizeof(cx<T>) + 15) / 16 * 16;
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    cx<TS> *st = reinterpret_cast<cx<TS> *>(smraw + SOFF);
    const T norm = (T)a.norm;
    const int lim = a.kx_lim > 0 ? a.kx_lim : L / 2 + 1;
    const int nch = StageRow<TS>::chunks(lim);
    const int rs = nch * StageRow<TS>::PER;
    // the stage barrier follows the stage (rs * sizeof(cx<TS>) is a multiple of 16)
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + SOFF + (size_t)OP::NIN * 2 * TC * rs * sizeof(cx<TS>));
    const TileMap tm{(a.npairs + TC - 1) / TC, a.nruns > 1 ? a.nruns : 1};
    const int ntiles = tm.total();
    OP op{(T)a.p0, (T)a.p1};
    __shared__ double cwarp[NT / 32];
    if ((threadIdx.x & 31) == 0) cwarp[threadIdx.x >> 5] = 0.0;
    if (threadIdx.x == 0) xf_mbar_init(bar);
    __syncthreads();
    if (threadIdx.x == 0 && (int)blockIdx.x < ntiles) {
        int r0, p0;
        tm.at(blockIdx.x, TC, r0, p0);
        xf_stage_issue<TS, OP::NIN, TC>(a, st, bar, p0, rs, r0 * a.rstride);
    }
    unsigned parity = 0;

#pragma unroll 1
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int run, pair0;
        tm.at(tile, TC, run, pair0);
        const int64_t roff = run * a.rstride;
        const bool ok = xf_mbar_wait(bar, parity);
        if (__syncthreads_or(!ok)) {
            // the copies never completed: report, and leave without touching the stage
            if (threadIdx.x == 0 && a.err != nullptr) atomicOr(a.err, 2);
            return;
        }
        parity ^= 1u;
        cx<T> phys[OP::NIN][NP];
        {
            cx<T> in[OP::NIN][FI::NIN];
#pragma unroll
            for (int f = 0; f < OP::NIN; f++) {
#pragma unroll
                for (int i = 0; i < FI::NB0; i++)
#pragma unroll
                    for (int m = 0; m < FI::R0; m++) {
                        int c, p;
                        if (FI::in_slot(i, m, c, p) && pair0 + c < a.npairs) {
                            const cx<TS> *A = st + (f * 2 * TC + 2 * c) * rs;
                            in[f][i * FI::R0 + m] = load_packed<T, L, TS>(A, A + rs, p, lim);
                        } else in[f][i * FI::R0 + m] = mk<T>(0, 0);
                    }
#pragma unroll
                for (int q = 0; q < NP; q++) phys[f][q] = mk<T>(0, 0);
            }
            __syncthreads();  // the stage is free: bring in the next tile
            if (threadIdx.x == 0 && tile + (int)gridDim.x < ntiles) {
                int rn, pn;
                tm.at(tile + gridDim.x, TC, rn, pn);
                xf_stage_issue<TS, OP::NIN, TC>(a, st, bar, pn, rs, rn * a.rstride);
            }
            FI::template run_multi<OP::NIN>(in, sm, phys, tw);
        }
        // quadratic products: the 1/N^3 of the inverse transforms is applied
        // once, as norm^2 in the split of the forward outputs (and norm to the
        // Courant maximum and the physical fields written out)
        if constexpr (!OP::QUAD) {
#pragma unroll
            for (int f = 0; f < OP::NIN; f++)
#pragma unroll
                for (int q = 0; q < NP; q++) phys[f][q] = mk<T>(phys[f][q].x * norm, phys[f][q].y * norm);
        }
        __syncthreads();
        if (a.phys != nullptr) {
            double *pb = a.phys;
#pragma unroll
            for (int i = 0; i < FI::NBL; i++)
#pragma unroll
                for (int m = 0; m < FI::RL; m++) {
                    int c, p;
                    if (FI::out_slot(i, m, c, p) && pair0 + c < a.npairs) {
                        int64_t r = 2 * (pair0 + c);
#pragma unroll
                        for (int f = 0; f < OP::NPHYS; f++) {
                            pb[f * a.phys_fs + r * a.phys_pitch + p] = (double)(phys[f][i * FI::RL + m].x * (OP::QUAD ? (T)a.norm : (T)1));
                            pb[f * a.phys_fs + (r + 1) * a.phys_pitch + p] = (double)(phys[f][i * FI::RL + m].y * (OP::QUAD ? (T)a.norm : (T)1));
                        }
                    }
                }
        }
        if (a.cmax != nullptr) {
            double cm = 0.0;
#pragma unroll
            for (int q = 0; q < NP; q++) {
                T va[OP::NIN], vb[OP::NIN];
#pragma unroll
                for (int f = 0; f < OP::NIN; f++) { va[f] = phys[f][q].x; vb[f] = phys[f][q].y; }
                cm = fmax(cm, (double)op.cour(va));
                cm = fmax(cm, (double)op.cour(vb));
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) cm = fmax(cm, __shfl_xor_sync(0xffffffffu, cm, off));
            if ((threadIdx.x & 31) == 0) cwarp[threadIdx.x >> 5] = fmax(cwarp[threadIdx.x >> 5], cm);
        }
        cx<T> aux[NP];
#pragma unroll
        for (int q = 0; q < NP; q++) {
            T va[OP::NIN], vb[OP::NIN];
#pragma unroll
            for (int f = 0; f < OP::NIN; f++) { va[f] = phys[f][q].x; vb[f] = phys[f][q].y; }
            aux[q] = mk<T>(op.aux(va), op.aux(vb));
        }
        constexpr int NG = (OP::NOUT + GF - 1) / GF;
        const T half = OP::QUAD ? (T)0.5 * (T)a.norm * (T)a.norm : (T)0.5;
        // fields NIN-NSMF..NIN-1 to buffers GF.., at this thread's own slots (the
        // barrier above ended the inverse's reads of every buffer)
        cx<T> *pw = sm + GF * E;
        if constexpr (NSMF > 0) {
#pragma unroll
            for (int i = 0; i < FI::NBL; i++)
#pragma unroll
                for (int m = 0; m < FI::RL; m++) {
                    int c, p;
                    if (FI::out_slot(i, m, c, p))
#pragma unroll
                        for (int f = OP::NIN - NSMF; f < OP::NIN; f++)
                            pw[(f - (OP::NIN - NSMF)) * E + Lay<L, TC, true>::idx(c, p)] = phys[f][i * FI::RL + m];
                }
        }
#pragma unroll
        for (int g = 0; g < NG; g++) {
            cx<T> in[GF][FF::NIN];
#pragma unroll
            for (int gf = 0; gf < GF; gf++) {
                const int o = g * GF + gf;
#pragma unroll
                for (int q = 0; q < NP; q++) {
                    T va[OP::NIN], vb[OP::NIN];
#pragma unroll
                    for (int f = 0; f < OP::NIN; f++) { va[f] = phys[f][q].x; vb[f] = phys[f][q].y; }
                    if constexpr (NSMF > 0) {
                        // the same slot the inverse left this thread (FI::NOUT == FF::NIN)
                        int c, p;
                        FF::in_slot(q / FF::R0, q % FF::R0, c, p);
#pragma unroll
                        for (int f = OP::NIN - NSMF; f < OP::NIN; f++)
                            if (o < OP::NOUT && OP::uses(o, f)) {
                                const cx<T> v = pw[(f - (OP::NIN - NSMF)) * E + Lay<L, TC, true>::idx(c, p)];
                                va[f] = v.x;
                                vb[f] = v.y;
                            }
                    }
                    in[gf][q] = o < OP::NOUT ? mk<T>(op.out(o, va, aux[q].x), op.out(o, vb, aux[q].y)) : mk<T>(0, 0);
                }
            }
            FF::template run_multi_front<GF>(in, sm, tw);
            void *const outs[GF] = {g * GF < OP::NOUT ? (void *)(reinterpret_cast<cx<TS> *>(a.out[g * GF]) + roff) : nullptr,
                                    g * GF + 1 < OP::NOUT ? (void *)(reinterpret_cast<cx<TS> *>(a.out[g * GF + 1]) + roff)
                                                          : nullptr};
            xf_last_split<T, L, TC, NT, GF, TS>(sm, tw, outs, a.pitch, pair0, a.npairs, lim, half);
            __syncthreads();  // the buffers are read: the next group may overwrite them
        }
    }
    if (a.cmax != nullptr && (threadIdx.x & 31) == 0)
        atomicMax(a.cmax, (unsigned long long)__double_as_longlong(cwarp[threadIdx.x >> 5] * (OP::QUAD ? (double)(T)a.norm : 1.0)));
}
