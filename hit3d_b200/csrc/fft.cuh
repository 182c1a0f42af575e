// Radix-2/3/4/8 Stockham FFT on columns staged through shared memory.
//
// One CTA transforms TC independent sticks ("columns") of length L.  Stage 0 takes
// its inputs straight from registers (loaded from HBM by the caller), the middle
// stages exchange through shared memory, and the last stage leaves its outputs in
// registers for the caller to store (or to combine with other fields first).  With
// Stockham ordering the stage-0 inputs and the last-stage outputs of butterfly j
// both sit at positions j + m*L/R, so a pass over HBM reads and writes the same
// addresses and can run in place.
//
// Two shared-memory layouts:
//   COLS (ROWS=false): element (c,p) at p*TC + c -- columns interleaved, used for
//        the strided y/z passes where TC adjacent kx columns form one 128-byte row;
//   ROWS (ROWS=true):  element (c,p) at c*(L+L/8) + p + p/8 -- each stick
//        contiguous with one pad slot per 8 elements, used for the x passes.
#pragma once
#include "common.cuh"

// ---------------------------------------------------------------------------
// radix plans: forward order; the inverse x pass uses the reversed plan so that
// its last radix equals the forward plan's first radix (register hand-off).
// ---------------------------------------------------------------------------
H3D_HD constexpr int plan_stages(int L)
{
    return L == 16 ? 2 : L == 32 ? 2 : L == 48 ? 3 : L == 64 ? 2 : L == 96 ? 3 : L == 128 ? 3 :
           L == 192 ? 3 : L == 256 ? 3 : L == 384 ? 4 : L == 512 ? 3 : L == 768 ? 4 : L == 1024 ? 4 : 0;
}

H3D_HD constexpr int plan_radix_fwd(int L, int s)
{
    // 16=4.4 32=8.4 48=4.4.3 64=8.8 96=8.4.3 128=8.4.4 192=8.8.3 256=8.8.4
    // 384=8.4.4.3 512=8.8.8 768=8.8.4.3 1024=8.8.4.4
    return L == 16 ? 4 :
           L == 32 ? (s == 0 ? 8 : 4) :
           L == 48 ? (s < 2 ? 4 : 3) :
           L == 64 ? 8 :
           L == 96 ? (s == 0 ? 8 : s == 1 ? 4 : 3) :
           L == 128 ? (s == 0 ? 8 : 4) :
           L == 192 ? (s < 2 ? 8 : 3) :
           L == 256 ? (s < 2 ? 8 : 4) :
           L == 384 ? (s == 0 ? 8 : s < 3 ? 4 : 3) :
           L == 512 ? 8 :
           L == 768 ? (s < 2 ? 8 : s == 2 ? 4 : 3) :
           L == 1024 ? (s < 2 ? 8 : 4) : 0;
}

template <int L, bool REV> struct Plan {
    static constexpr int S = plan_stages(L);
    static H3D_HD constexpr int R(int s) { return REV ? plan_radix_fwd(L, S - 1 - s) : plan_radix_fwd(L, s); }
    // product of the radices of stages [0, s)
    static H3D_HD constexpr int Ns(int s) { return s == 0 ? 1 : Ns(s - 1) * R(s - 1); }
};

// ---------------------------------------------------------------------------
// small DFTs in registers, natural order in and out
// ---------------------------------------------------------------------------
template <typename T, bool FWD> H3D_D void dft2(cx<T> &a, cx<T> &b)
{
    cx<T> t = a;
    a = t + b;
    b = t - b;
}

// d + (-i t) (FWD) or d + i t, and d - (-i t) or d - i t, lane by lane (no
// swapped pair is formed, so the packed FP32 adds serve only the plain sums)
template <typename T, bool FWD> H3D_D cx<T> addmi(cx<T> d, cx<T> t)
{
    return FWD ? mk<T>(d.x + t.y, d.y - t.x) : mk<T>(d.x - t.y, d.y + t.x);
}
template <typename T, bool FWD> H3D_D cx<T> submi(cx<T> d, cx<T> t)
{
    return FWD ? mk<T>(d.x - t.y, d.y + t.x) : mk<T>(d.x + t.y, d.y - t.x);
}

// a + b and a - b; PK (FP32 only): one packed two-lane instruction
// (add/sub.rn.f32x2, each lane rounded as the scalar operation), which the
// strided passes of the FP32 form use
template <typename T, bool PK> H3D_D cx<T> cadd(cx<T> a, cx<T> b)
{
    if constexpr (PK) {
        static_assert(sizeof(T) == 4, "packed sums are FP32");
        unsigned long long pa, pb, r;
        asm("mov.b64 %0, {%1, %2};" : "=l"(pa) : "f"(a.x), "f"(a.y));
        asm("mov.b64 %0, {%1, %2};" : "=l"(pb) : "f"(b.x), "f"(b.y));
        asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pa), "l"(pb));
        cx<T> o;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(o.x), "=f"(o.y) : "l"(r));
        return o;
    } else {
        return a + b;
    }
}
template <typename T, bool PK> H3D_D cx<T> csub(cx<T> a, cx<T> b)
{
    if constexpr (PK) {
        static_assert(sizeof(T) == 4, "packed sums are FP32");
        unsigned long long pa, pb, r;
        asm("mov.b64 %0, {%1, %2};" : "=l"(pa) : "f"(a.x), "f"(a.y));
        asm("mov.b64 %0, {%1, %2};" : "=l"(pb) : "f"(b.x), "f"(b.y));
        asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pa), "l"(pb));
        cx<T> o;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(o.x), "=f"(o.y) : "l"(r));
        return o;
    } else {
        return a - b;
    }
}

template <typename T, bool FWD, bool PK = false> H3D_D void dft4(cx<T> &a0, cx<T> &a1, cx<T> &a2, cx<T> &a3)
{
    cx<T> s0 = cadd<T, PK>(a0, a2), d0 = csub<T, PK>(a0, a2), s1 = cadd<T, PK>(a1, a3), t = csub<T, PK>(a1, a3);
    a0 = cadd<T, PK>(s0, s1);
    a2 = csub<T, PK>(s0, s1);
    a1 = addmi<T, FWD>(d0, t);
    a3 = submi<T, FWD>(d0, t);
}

template <typename T, bool FWD> H3D_D void dft3(cx<T> &a0, cx<T> &a1, cx<T> &a2)
{
    const T h = (T)0.5;
    const T s3 = (T)0.86602540378443864676372317075293618;  // sin(2 pi/3)
    cx<T> s = a1 + a2, d = a1 - a2;
    cx<T> m = mk<T>(a0.x - h * s.x, a0.y - h * s.y);
    // forward: X1 = m - i s3 d, X2 = m + i s3 d
    cx<T> r = mk<T>(s3 * d.y, -s3 * d.x);  // -i*s3*d
    if (!FWD) r = mk<T>(-r.x, -r.y);
    a0 = a0 + s;
    a1 = m + r;
    a2 = m - r;
}

template <typename T, bool FWD, bool PK = false> H3D_D void dft8(cx<T> (&a)[8])
{
    const T r2 = (T)0.70710678118654752440084436210484904;
    cx<T> e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6];
    cx<T> o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
    dft4<T, FWD, PK>(e0, e1, e2, e3);
    dft4<T, FWD, PK>(o0, o1, o2, o3);
    // twiddles w8^k, w8 = exp(-+ i pi/4)
    cx<T> t1 = FWD ? mk<T>(r2 * (o1.x + o1.y), r2 * (o1.y - o1.x)) : mk<T>(r2 * (o1.x - o1.y), r2 * (o1.y + o1.x));
    cx<T> t3 = FWD ? mk<T>(r2 * (-o3.x + o3.y), r2 * (-o3.y - o3.x)) : mk<T>(r2 * (-o3.x - o3.y), r2 * (-o3.y + o3.x));
    a[0] = cadd<T, PK>(e0, o0); a[4] = csub<T, PK>(e0, o0);
    a[1] = cadd<T, PK>(e1, t1); a[5] = csub<T, PK>(e1, t1);
    a[2] = addmi<T, FWD>(e2, o2); a[6] = submi<T, FWD>(e2, o2);  // e2 +- w8^2 o2
    a[3] = cadd<T, PK>(e3, t3); a[7] = csub<T, PK>(e3, t3);
}

template <typename T, int R, bool FWD, bool PK = false> H3D_D void dft(cx<T> *a)
{
    if constexpr (R == 2) dft2<T, FWD>(a[0], a[1]);
    else if constexpr (R == 3) dft3<T, FWD>(a[0], a[1], a[2]);
    else if constexpr (R == 4) dft4<T, FWD, PK>(a[0], a[1], a[2], a[3]);
    else if constexpr (R == 8) {
        cx<T> t[8];
#pragma unroll
        for (int m = 0; m < 8; m++) t[m] = a[m];
        dft8<T, FWD, PK>(t);
#pragma unroll
        for (int m = 0; m < 8; m++) a[m] = t[m];
    }
}

// ---------------------------------------------------------------------------
// thread <-> butterfly mapping and shared-memory layout
// ---------------------------------------------------------------------------
template <int L, int TC, bool ROWS> struct Lay {
    static constexpr int RS = L + L / 8;  // padded stick length in ROWS layout
    static constexpr int elems = ROWS ? TC * RS : TC * L;
    static H3D_D int idx(int c, int p) { return ROWS ? c * RS + p + (p >> 3) : p * TC + c; }
    template <int R> static H3D_D void bf(int b, int &c, int &j)
    {
        constexpr int nbpc = L / R;
        if (ROWS) { j = b % nbpc; c = b / nbpc; }
        else { c = b % TC; j = b / TC; }
    }
};

template <int L, int TC, int NT, int R> struct Cnt {
    static constexpr int total = TC * (L / R);           // butterflies per stage per CTA
    static constexpr int NB = (total + NT - 1) / NT;      // per thread
};

// twiddle w^(k*m) for a stage whose sub-transform length is Ns*R;
// tw[t] = exp(-2 pi i t / L)
template <typename T, bool FWD> H3D_D cx<T> twid(const cx<T> *__restrict__ tw, int t)
{
    cx<T> w = __ldg(tw + t);
    if (!FWD) w.y = -w.y;
    return w;
}

// ---------------------------------------------------------------------------
// the column transform: in[] (stage-0 inputs) -> out[] (last-stage outputs)
//   in[i*R0+m]  : column c, position j + m*L/R0 of butterfly b = tid + i*NT
//   out[i*RL+m] : column c, position j + m*L/RL of butterfly b = tid + i*NT
// The caller must __syncthreads() before reusing sm after this returns.
// ---------------------------------------------------------------------------
// Twiddle sources.  GlobalTw reads the table for every butterfly; CachedTw holds
// the twiddles of this thread's butterflies in registers (they depend only on
// the thread's fixed position in each stage, so a kernel that runs many
// transforms with the same mapping loads them once).  Both return the forward
// twiddle w^(k m) of stage s, butterfly slot i; conjugated for inverse transforms.
template <typename T> struct GlobalTw {
    const cx<T> *__restrict__ tw;
    template <int L, int Ns, int R, bool FWD, int s>
    H3D_D cx<T> get(int i, int m, int k) const
    {
        (void)i;
        return twid<T, FWD>(tw, k * m * (L / (Ns * R)));
    }
};
// packed FP32 sums in the butterflies of the strided passes (COLS layout);
// the row passes keep scalar sums (measured faster there)
template <typename T, bool ROWS> constexpr bool kPackSums = !ROWS && sizeof(T) == 4;

template <typename T, int L, int TC, int NT, bool ROWS, bool FWD, bool REV, int s, class TWS>
H3D_D void fft_mid_stage(cx<T> *sm, const TWS &tws)
{
    using P = Plan<L, REV>;
    using LY = Lay<L, TC, ROWS>;
    constexpr int R = P::R(s), Ns = P::Ns(s), nbpc = L / R;
    using CN = Cnt<L, TC, NT, R>;
    cx<T> a[CN::NB * R];
    const int tid = threadIdx.x;
#pragma unroll
    for (int i = 0; i < CN::NB; i++) {
        int b = tid + i * NT;
        if (CN::total % NT == 0 || b < CN::total) {
            int c, j;
            LY::template bf<R>(b, c, j);
            int k = j % Ns;
#pragma unroll
            for (int m = 0; m < R; m++) {
                cx<T> v = sm[LY::idx(c, j + m * nbpc)];
                if (m > 0) v = cmul(v, tws.template get<L, Ns, R, FWD, s>(i, m, k));
                a[i * R + m] = v;
            }
            dft<T, R, FWD, kPackSums<T, ROWS>>(a + i * R);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < CN::NB; i++) {
        int b = tid + i * NT;
        if (CN::total % NT == 0 || b < CN::total) {
            int c, j;
            LY::template bf<R>(b, c, j);
            int k = j % Ns;
            int base = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int m = 0; m < R; m++) sm[LY::idx(c, base + m * Ns)] = a[i * R + m];
        }
    }
    __syncthreads();
}

template <typename T, int L, int TC, int NT, bool ROWS, bool FWD, bool REV>
struct ColFFT {
    using P = Plan<L, REV>;
    using LY = Lay<L, TC, ROWS>;
    static constexpr int S = P::S;
    static constexpr int R0 = P::R(0), RL = P::R(S - 1);
    static constexpr int NB0 = Cnt<L, TC, NT, R0>::NB, NBL = Cnt<L, TC, NT, RL>::NB;
    static constexpr int TOT0 = Cnt<L, TC, NT, R0>::total, TOTL = Cnt<L, TC, NT, RL>::total;
    static constexpr int NIN = NB0 * R0, NOUT = NBL * RL;

    // register twiddle cache: stages 1..S-1, NB_s butterflies, R_s - 1 twiddles each
    static H3D_HD constexpr int tw_count(int s)
    {
        return ((TC * (L / P::R(s)) + NT - 1) / NT) * (P::R(s) - 1);
    }
    static H3D_HD constexpr int tw_off(int s) { return s <= 1 ? 0 : tw_off(s - 1) + tw_count(s - 1); }
    static constexpr int TWN = tw_off(S);
    struct CachedTw {
        cx<T> w[TWN > 0 ? TWN : 1];  // forward twiddles
        template <int L_, int Ns, int R, bool FWD_, int s>
        H3D_D cx<T> get(int i, int m, int) const
        {
            cx<T> v = w[tw_off(s) + i * (R - 1) + (m - 1)];
            if (!FWD_) v.y = -v.y;
            return v;
        }
    };
    // fill the cache for this thread's butterflies (same mapping in every transform)
    static H3D_D void load_twiddles(CachedTw &c, const cx<T> *__restrict__ tw)
    {
        load_tw_stage<1>(c, tw);
    }
    template <int s> static H3D_D void load_tw_stage(CachedTw &cache, const cx<T> *__restrict__ tw)
    {
        if constexpr (s < S) {
            constexpr int R = P::R(s), Ns = P::Ns(s);
            using CN = Cnt<L, TC, NT, R>;
#pragma unroll
            for (int i = 0; i < CN::NB; i++) {
                int b = threadIdx.x + i * NT;
                int c, j;
                LY::template bf<R>(b, c, j);
                int k = j % Ns;
#pragma unroll
                for (int m = 1; m < R; m++)
                    cache.w[tw_off(s) + i * (R - 1) + (m - 1)] =
                        (CN::total % NT == 0 || b < CN::total) ? __ldg(tw + k * m * (L / (Ns * R))) : mk<T>(1, 0);
            }
            load_tw_stage<s + 1>(cache, tw);
        }
    }

    // (c, position) of in[i*R0+m]; valid() false for idle slots
    static H3D_D bool in_slot(int i, int m, int &c, int &p)
    {
        int b = threadIdx.x + i * NT;
        int j;
        LY::template bf<R0>(b, c, j);
        p = j + m * (L / R0);
        return TOT0 % NT == 0 || b < TOT0;
    }
    static H3D_D bool out_slot(int i, int m, int &c, int &p)
    {
        int b = threadIdx.x + i * NT;
        int j;
        LY::template bf<RL>(b, c, j);
        p = j + m * (L / RL);
        return TOTL % NT == 0 || b < TOTL;
    }

    // stage 0 and the middle stages; afterwards sm holds the input of the last stage
    template <class TWS> static H3D_D void stages_to_last_t(cx<T> (&in)[NIN], cx<T> *sm, const TWS &tws)
    {
        const int tid = threadIdx.x;
#pragma unroll
        for (int i = 0; i < NB0; i++) {
            int b = tid + i * NT;
            if (TOT0 % NT == 0 || b < TOT0) {
                int c, j;
                LY::template bf<R0>(b, c, j);
                dft<T, R0, FWD, kPackSums<T, ROWS>>(in + i * R0);
#pragma unroll
                for (int m = 0; m < R0; m++) sm[LY::idx(c, j * R0 + m)] = in[i * R0 + m];
            }
        }
        __syncthreads();
        if constexpr (S > 2) fft_mid_stage<T, L, TC, NT, ROWS, FWD, REV, 1>(sm, tws);
        if constexpr (S > 3) fft_mid_stage<T, L, TC, NT, ROWS, FWD, REV, 2>(sm, tws);
    }

    // the transform, handing each last-stage butterfly to st(c, p, v) as soon as
    // it is computed so that its outputs need not stay live in registers
    template <class TWS, class ST>
    static H3D_D void run_store_t(cx<T> (&in)[NIN], cx<T> *sm, const TWS &tws, ST &&st)
    {
        stages_to_last_t(in, sm, tws);
        constexpr int NsL = P::Ns(S - 1), nbpc = L / RL;
        const int tid = threadIdx.x;
#pragma unroll
        for (int i = 0; i < NBL; i++) {
            int b = tid + i * NT;
            if (TOTL % NT == 0 || b < TOTL) {
                int c, j;
                LY::template bf<RL>(b, c, j);
                int k = j % NsL;
                cx<T> v[RL];
#pragma unroll
                for (int m = 0; m < RL; m++) {
                    cx<T> x = sm[LY::idx(c, j + m * nbpc)];
                    if (m > 0) x = cmul(x, tws.template get<L, NsL, RL, FWD, S - 1>(i, m, k));
                    v[m] = x;
                }
                dft<T, RL, FWD, kPackSums<T, ROWS>>(v);
#pragma unroll
                for (int m = 0; m < RL; m++) st(c, j + m * nbpc, v[m]);
            }
        }
    }

    // as run_store_t, but st(i, m, c, p, v) also receives the output slot (i, m)
    // so that callers can keep per-slot accumulators in registers
    template <class TWS, class ST>
    static H3D_D void run_slots_t(cx<T> (&in)[NIN], cx<T> *sm, const TWS &tws, ST &&st)
    {
        stages_to_last_t(in, sm, tws);
        constexpr int NsL = P::Ns(S - 1), nbpc = L / RL;
        const int tid = threadIdx.x;
#pragma unroll
        for (int i = 0; i < NBL; i++) {
            int b = tid + i * NT;
            if (TOTL % NT == 0 || b < TOTL) {
                int c, j;
                LY::template bf<RL>(b, c, j);
                int k = j % NsL;
                cx<T> v[RL];
#pragma unroll
                for (int m = 0; m < RL; m++) {
                    cx<T> x = sm[LY::idx(c, j + m * nbpc)];
                    if (m > 0) x = cmul(x, tws.template get<L, NsL, RL, FWD, S - 1>(i, m, k));
                    v[m] = x;
                }
                dft<T, RL, FWD, kPackSums<T, ROWS>>(v);
#pragma unroll
                for (int m = 0; m < RL; m++) st(i, m, c, j + m * nbpc, v[m]);
            }
        }
    }

    template <class ST>
    static H3D_D void run_store(cx<T> (&in)[NIN], cx<T> *sm, const cx<T> *__restrict__ tw, ST &&st)
    {
        run_store_t(in, sm, GlobalTw<T>{tw}, st);
    }

    // NF independent transforms in lockstep: field f uses the shared-memory
    // buffer sm + f * LY::elems, all fields share one barrier per stage and one
    // twiddle load per butterfly.  Last-stage outputs are left in out[f][...].
    // The caller must __syncthreads() before reusing sm after this returns.
    // stage 0 and the middle stages of NF transforms in lockstep; afterwards
    // buffer f (sm + f * LY::elems) holds the input of transform f's last stage
    template <int NF>
    static H3D_D void run_multi_front(cx<T> (&in)[NF][NIN], cx<T> *sm, const cx<T> *__restrict__ tw)
    {
        constexpr int E = LY::elems;
        const int tid = threadIdx.x;
#pragma unroll
        for (int i = 0; i < NB0; i++) {
            int b = tid + i * NT;
            if (TOT0 % NT == 0 || b < TOT0) {
                int c, j;
                LY::template bf<R0>(b, c, j);
#pragma unroll
                for (int f = 0; f < NF; f++) {
                    dft<T, R0, FWD, kPackSums<T, ROWS>>(in[f] + i * R0);
#pragma unroll
                    for (int m = 0; m < R0; m++) sm[f * E + LY::idx(c, j * R0 + m)] = in[f][i * R0 + m];
                }
            }
        }
        __syncthreads();
        if constexpr (S > 2) mid_multi<NF, 1>(sm, tw);
        if constexpr (S > 3) mid_multi<NF, 2>(sm, tw);
    }

    template <int NF>
    static H3D_D void run_multi(cx<T> (&in)[NF][NIN], cx<T> *sm, cx<T> (&out)[NF][NOUT], const cx<T> *__restrict__ tw)
    {
        constexpr int E = LY::elems;
        const int tid = threadIdx.x;
        run_multi_front<NF>(in, sm, tw);
        constexpr int NsL = P::Ns(S - 1), nbpc = L / RL;
#pragma unroll
        for (int i = 0; i < NBL; i++) {
            int b = tid + i * NT;
            if (TOTL % NT == 0 || b < TOTL) {
                int c, j;
                LY::template bf<RL>(b, c, j);
                const int k = j % NsL;
#pragma unroll
                for (int m = 0; m < RL; m++) {
                    const cx<T> w = m > 0 ? twid<T, FWD>(tw, k * m * (L / (NsL * RL))) : mk<T>(1, 0);
#pragma unroll
                    for (int f = 0; f < NF; f++) {
                        cx<T> x = sm[f * E + LY::idx(c, j + m * nbpc)];
                        out[f][i * RL + m] = m > 0 ? cmul(x, w) : x;
                    }
                }
#pragma unroll
                for (int f = 0; f < NF; f++) dft<T, RL, FWD, kPackSums<T, ROWS>>(out[f] + i * RL);
            }
        }
    }
    template <int NF, int s> static H3D_D void mid_multi(cx<T> *sm, const cx<T> *__restrict__ tw)
    {
        constexpr int E = LY::elems;
        constexpr int R = P::R(s), Ns = P::Ns(s), nbpc = L / R;
        using CN = Cnt<L, TC, NT, R>;
        cx<T> a[NF][CN::NB * R];
        const int tid = threadIdx.x;
#pragma unroll
        for (int i = 0; i < CN::NB; i++) {
            int b = tid + i * NT;
            if (CN::total % NT == 0 || b < CN::total) {
                int c, j;
                LY::template bf<R>(b, c, j);
                const int k = j % Ns;
#pragma unroll
                for (int m = 0; m < R; m++) {
                    const cx<T> w = m > 0 ? twid<T, FWD>(tw, k * m * (L / (Ns * R))) : mk<T>(1, 0);
#pragma unroll
                    for (int f = 0; f < NF; f++) {
                        cx<T> v = sm[f * E + LY::idx(c, j + m * nbpc)];
                        a[f][i * R + m] = m > 0 ? cmul(v, w) : v;
                    }
                }
#pragma unroll
                for (int f = 0; f < NF; f++) dft<T, R, FWD, kPackSums<T, ROWS>>(a[f] + i * R);
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < CN::NB; i++) {
            int b = tid + i * NT;
            if (CN::total % NT == 0 || b < CN::total) {
                int c, j;
                LY::template bf<R>(b, c, j);
                const int k = j % Ns;
                const int base = (j / Ns) * Ns * R + k;
#pragma unroll
                for (int f = 0; f < NF; f++)
#pragma unroll
                    for (int m = 0; m < R; m++) sm[f * E + LY::idx(c, base + m * Ns)] = a[f][i * R + m];
            }
        }
        __syncthreads();
    }

    // the transform with the last-stage outputs left in out[i*RL+m]
    static H3D_D void run(cx<T> (&in)[NIN], cx<T> *sm, cx<T> (&out)[NOUT], const cx<T> *__restrict__ tw)
    {
        const GlobalTw<T> tws{tw};
        stages_to_last_t(in, sm, tws);
        constexpr int NsL = P::Ns(S - 1), nbpc = L / RL;
        const int tid = threadIdx.x;
#pragma unroll
        for (int i = 0; i < NBL; i++) {
            int b = tid + i * NT;
            if (TOTL % NT == 0 || b < TOTL) {
                int c, j;
                LY::template bf<RL>(b, c, j);
                int k = j % NsL;
#pragma unroll
                for (int m = 0; m < RL; m++) {
                    cx<T> x = sm[LY::idx(c, j + m * nbpc)];
                    if (m > 0) x = cmul(x, tws.template get<L, NsL, RL, FWD, S - 1>(i, m, k));
                    out[i * RL + m] = x;
                }
                dft<T, RL, FWD, kPackSums<T, ROWS>>(out + i * RL);
            }
        }
    }
};
