// FFT passes over HBM: strided y/z passes and row (x) passes, plus the fused
// x pass that turns inverse-transformed velocities into forward-transformed
// products without a round trip through HBM.
//
// Replaces xFFT3d (x_fftw.f90:852-1085): the reference's per-plane 2-D r2c,
// y<->z swap, MPI transpose and z-stick c2c become three in-place passes over
// the whole field resident in HBM.
#pragma once
#include <cooperative_groups.h>

#include "fft.cuh"

// ---------------------------------------------------------------------------
// 2/3-rule pruning.  When every mode with some |k_i| > kc = N/3 is zero in the
// state (the reference dealiases at start, dealias_all.f90, and the update
// keeps those modes at zero), the passes of a time step skip what cannot
// change the result: inverse passes read only |k| <= kc and leave whole
// columns or rows of zeros untouched, forward passes store only |k| <= kc, the
// modes the update reads (rhs_velocity.f90:85-142 masks the rest).  Index idx
// of an axis of n points holds the signed wavenumber idx (idx <= n/2) or
// idx - n; n/2 counts as +n/2.
// ---------------------------------------------------------------------------
H3D_HD bool kept(int idx, int n, int kc) { return (idx <= n / 2 ? idx : n - idx) <= kc; }
// outer index y in [0, 2 kc] -> the kept axis index (0..kc, n-kc..n-1)
H3D_HD int kept_index(int y, int n, int kc) { return y <= kc ? y : n - (2 * kc + 1 - y); }

// ---------------------------------------------------------------------------
// strided (y or z) pass:  CTA = TC adjacent kx columns x one outer index,
// transform along an axis of stride `sa` (complex elements).  kl/ks >= 0 prune
// the loads/stores along the transform axis; ko >= 0 maps the outer grid index
// onto the kept indices of the outer axis.
// ---------------------------------------------------------------------------
template <typename T, typename TI, typename TO> struct IOPlain {
    const cx<TI> *src;
    cx<TO> *dst;
    int64_t fs_src, fs_dst;  // field strides
    int64_t sa_src, so_src, sa_dst, so_dst;
    int ncol;
    int n = 0, kl = -1, ks = -1, ko = -1;
    // runs of a batch: nfr > 0 fields per run, run r's fields start rs_src /
    // rs_dst elements after run r-1's; grid index z = r * nfr + f
    int nfr = 0;
    int64_t rs_src = 0, rs_dst = 0;
    H3D_D IOPlain at(int z, int &f) const
    {
        IOPlain b = *this;
        f = z;
        if (nfr > 0) {
            const int r = z / nfr;
            f = z - r * nfr;
            b.src += r * rs_src;
            b.dst += r * rs_dst;
        }
        return b;
    }
    H3D_D int outer(int y) const { return ko >= 0 ? kept_index(y, n, ko) : y; }
    H3D_D cx<T> load(int f, int o, int c, int p) const
    {
        if (c >= ncol || (kl >= 0 && !kept(p, n, kl))) return mk<T>(0, 0);
        return to_cx<T>(src[f * fs_src + p * sa_src + o * so_src + c]);
    }
    H3D_D void store(int f, int o, int c, int p, cx<T> v) const
    {
        if (c < ncol && (ks < 0 || kept(p, n, ks))) dst[f * fs_dst + p * sa_dst + o * so_dst + c] = to_cx<TO>(v);
    }
};

// Spectral pre-operations applied while reading the FP64 state in the first
// inverse (z) pass: column c = kx, outer o = ky index, position p = kz index.
enum PreMode : int {
    PRE_COPY = 0,      // field f of the state
    PRE_SHIFT = 1,     // field f times exp(i (kx+ky+kz) dx/2)   (rhs_velocity.f90:248-257)
    PRE_CURL = 2,      // vorticity component f                 (m_stats.f90:260-274)
    PRE_DLONG = 3,     // du_f/dx_f                              (new: skewness)
    PRE_STRAIN_A = 4,  // S11, S12, S13 for f = 0,1,2            (m_les.f90:1153-1170)
    PRE_STRAIN_B = 5,  // S22, S23, S33 for f = 0,1,2            (m_les.f90:1180-1198)
    PRE_GRAD = 6,      // d phi/dx_f of state field `sfield`     (m_stats.f90:323-326)
    PRE_TRUNC = 7,     // field f with |k|^2 > k2max zeroed       (io_write_4.f90:21-42)
    PRE_CUBE = 8,      // field f with some |k_i| > N/3 zeroed    (m_les.f90:1579-1586)
    PRE_FILT = 9,      // field f times the test filter g         (m_filter_xfftw.f90:81-100)
    PRE_QUART = 10,    // field f with some |k_i| > N/4 zeroed    (rhs_scalars.f90:284-292)
};

// MODE is a compile-time PreMode so that the plain copy carries no per-element
// branching or wavenumber arithmetic
template <typename T, typename TO, int MODE> struct IOSpec {
    const double2 *src;  // state fields, [kz][ky][kx] pitch psrc
    cx<TO> *dst;         // [z][ky][kx] pitch pdst
    int64_t fs_src, fs_dst;
    int n, psrc, pdst, ncol, sfield;
    double dx;     // grid spacing, for PRE_SHIFT
    double k2max;  // truncation radius squared, for PRE_TRUNC
    const double2 *g = nullptr;  // test filter transfer function, for PRE_FILT (pitch psrc)
    int kl = -1, ko = -1;  // 2/3-rule pruning of the kz loads and the ky rows
    int nfr = 0;           // runs of a batch, as IOPlain::at
    int64_t rs_src = 0, rs_dst = 0;
    H3D_D IOSpec at(int z, int &f) const
    {
        IOSpec b = *this;
        f = z;
        if (nfr > 0) {
            const int r = z / nfr;
            f = z - r * nfr;
            b.src += r * rs_src;
            b.dst += r * rs_dst;
        }
        return b;
    }
    H3D_D int outer(int y) const { return ko >= 0 ? kept_index(y, n, ko) : y; }

    H3D_D double2 U(int f, int o, int c, int p) const { return src[f * fs_src + ((int64_t)p * n + o) * psrc + c]; }
    H3D_D cx<T> load(int f, int o, int c, int p) const
    {
        if (c >= ncol || (kl >= 0 && !kept(p, n, kl))) return mk<T>(0, 0);
        if constexpr (MODE == PRE_COPY) return to_cx<T>(U(f, o, c, p));
        const double kx = c, ky = kwave(o, n), kz = kwave(p, n);
        double2 r;
        switch (MODE) {
        case PRE_SHIFT: {
            double2 u = U(f, o, c, p);
            double cs = cos((0.5 * ((kx + ky) + kz)) * dx);
            double sn = sin((0.5 * ((kx + ky) + kz)) * dx);
            r = make_double2(u.x * cs - u.y * sn, u.y * cs + u.x * sn);
            break;
        }
        case PRE_CURL: {
            // x_derivative: (a + ib) k -> (-k b, k a); omega as the reference forms it
            double2 u = U(0, o, c, p), v = U(1, o, c, p), w = U(2, o, c, p);
            if (f == 0) r = make_double2((-(ky * w.y)) - (-(kz * v.y)), (ky * w.x) - (kz * v.x));       // w_y - v_z
            else if (f == 1) r = make_double2((-(kz * u.y)) - (-(kx * w.y)), (kz * u.x) - (kx * w.x));  // u_z - w_x
            else r = make_double2((-(kx * v.y)) - (-(ky * u.y)), (kx * v.x) - (ky * u.x));              // v_x - u_y
            break;
        }
        case PRE_DLONG: {
            double2 u = U(f, o, c, p);
            double k = f == 0 ? kx : f == 1 ? ky : kz;
            r = make_double2(-(k * u.y), k * u.x);
            break;
        }
        case PRE_STRAIN_A: {
            double2 u = U(0, o, c, p);
            if (f == 0) r = make_double2(-kx * u.y, kx * u.x);
            else if (f == 1) { double2 v = U(1, o, c, p); r = make_double2(-0.5 * (ky * u.y + kx * v.y), 0.5 * (ky * u.x + kx * v.x)); }
            else { double2 w = U(2, o, c, p); r = make_double2(-0.5 * (kz * u.y + kx * w.y), 0.5 * (kz * u.x + kx * w.x)); }
            break;
        }
        case PRE_STRAIN_B: {
            double2 v = U(1, o, c, p), w = U(2, o, c, p);
            if (f == 0) r = make_double2(-ky * v.y, ky * v.x);
            else if (f == 1) r = make_double2(-0.5 * (kz * v.y + ky * w.y), 0.5 * (kz * v.x + ky * w.x));
            else r = make_double2(-kz * w.y, kz * w.x);
            break;
        }
        case PRE_GRAD: {
            double2 u = U(sfield, o, c, p);
            double k = f == 0 ? kx : f == 1 ? ky : kz;
            r = make_double2(-(k * u.y), k * u.x);
            break;
        }
        case PRE_TRUNC: {
            const double k2 = kx * kx + ky * ky + kz * kz;
            r = k2 > k2max ? make_double2(0.0, 0.0) : U(f, o, c, p);
            break;
        }
        case PRE_CUBE: {
            const double k3 = (double)(n / 3);
            r = (fabs(kx) > k3 || fabs(ky) > k3 || fabs(kz) > k3) ? make_double2(0.0, 0.0) : U(f, o, c, p);
            break;
        }
        case PRE_QUART: {
            const double k4 = (double)(n / 4);
            r = (fabs(kx) > k4 || fabs(ky) > k4 || fabs(kz) > k4) ? make_double2(0.0, 0.0) : U(f, o, c, p);
            break;
        }
        case PRE_FILT: {
            // filter_xfftw: (a + ib)(c + id) with the transfer function in (c, d)
            const double2 u = U(f, o, c, p), gg = g[((int64_t)p * n + o) * psrc + c];
            r = make_double2(u.x * gg.x - u.y * gg.y, u.y * gg.x + u.x * gg.y);
            break;
        }
        default: r = U(f, o, c, p);
        }
        return to_cx<T>(r);
    }
    H3D_D void store(int f, int o, int c, int p, cx<T> v) const
    {
        if (c < ncol) dst[f * fs_dst + ((int64_t)p * n + o) * pdst + c] = to_cx<TO>(v);
    }
};

// two resident CTAs per SM where two tiles fit in shared memory, so that one
// CTA's loads overlap another's shared-memory stages
template <typename T, int L, int TC, int NT> struct ColMinBlocks {
    static constexpr int value = (NT >= 128 && (size_t)TC * L * sizeof(cx<T>) <= 112 * 1024) ? 2 : 1;
};

template <typename T, int L, int TC, int NT, bool FWD, class IO, int MINB = ColMinBlocks<T, L, TC, NT>::value>
__global__ void __launch_bounds__(NT, MINB) k_colfft(const IO io, const cx<T> *__restrict__ tw)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    using F = ColFFT<T, L, TC, NT, false, FWD, false>;
    int f;
    const IO iob = io.at(blockIdx.z, f);
    const int col0 = blockIdx.x * TC, outer = iob.outer(blockIdx.y);
    cx<T> in[F::NIN];
#pragma unroll
    for (int i = 0; i < F::NB0; i++)
#pragma unroll
        for (int m = 0; m < F::R0; m++) {
            int c, p;
            if (F::in_slot(i, m, c, p)) in[i * F::R0 + m] = iob.load(f, outer, col0 + c, p);
        }
    F::run_store(in, sm, tw, [&](int c, int p, cx<T> v) { iob.store(f, outer, col0 + c, p, v); });
}

// ---------------------------------------------------------------------------
// row (x) passes.  A "column" of the FFT is a PAIR of physical rows (2q, 2q+1)
// packed as z = a + i b; rows are numbered r = z*N + y over the whole field.
//   complex row r: base + r*pitch            (N/2+1 modes used)
//   real row r:    (T*)(base + r*pitch)       (N reals used)
// ---------------------------------------------------------------------------
template <typename T, int L, int TC, int NT, bool REV>
using RowFFT = ColFFT<T, L, TC, NT, true, REV ? false : true, REV>;

// t / d for 0 <= t with t * d < 2^32, by a multiply-high with m = ceil(2^32 / d)
// (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994): the row passes split their flat loop indices
// with a divisor prepared once instead of dividing by a runtime count at every
// iteration
struct DivU32 {
    unsigned m;
    int d;
    H3D_D explicit DivU32(int d_) : m(0xffffffffu / (unsigned)d_ + 1u), d(d_) {}  // d = 1 wraps m to 0
    H3D_D int operator()(int t) const { return m ? (int)__umulhi((unsigned)t, m) : t; }
};

// Hermitian-extended packed spectrum Z[k] = Xa[k] + i Xb[k] of rows A, B at
// k in [0, L); the imaginary parts of kx = 0 and kx = N/2 are ignored, as
// FFTW's c2r does.  Only kx < lim is read (2/3-rule pruning; the rest is zero).
template <typename T, int L, typename TS>
H3D_D cx<T> load_packed(const cx<TS> *__restrict__ A, const cx<TS> *__restrict__ B, int k, int lim = L / 2 + 1)
{
    if (k <= L / 2) {
        if (k >= lim) return mk<T>(0, 0);
        cx<TS> a = A[k], b = B[k];
        if (k == 0 || k == L / 2) { a.y = 0; b.y = 0; }
        return mk<T>((T)(a.x - b.y), (T)(a.y + b.x));
    }
    if (L - k >= lim) return mk<T>(0, 0);
    cx<TS> a = A[L - k], b = B[L - k];
    return mk<T>((T)(a.x + b.y), (T)(-a.y + b.x));
}

// After a forward row transform left Z (natural order) in shared memory: split
// into the half spectra of the two packed rows and store kx < lim of them.
template <typename T, int L, int TC, int NT, typename TS>
H3D_D void store_split(const cx<T> *sm, cx<TS> *__restrict__ base, int64_t pitch, int pair0, int npairs,
                       int lim = L / 2 + 1, T half = (T)0.5)
{
    using LY = Lay<L, TC, true>;
    const int NH = lim < L / 2 + 1 ? lim : L / 2 + 1;
    auto one = [&](int c, int k) {
        cx<T> zk = sm[LY::idx(c, k)], zm = sm[LY::idx(c, k == 0 ? 0 : L - k)];
        cx<TS> xa, xb;
        xa.x = (TS)(half * (zk.x + zm.x));
        xa.y = (TS)(half * (zk.y - zm.y));
        xb.x = (TS)(half * (zk.y + zm.y));
        xb.y = (TS)(-half * (zk.x - zm.x));
        cx<TS> *A = base + (int64_t)(2 * (pair0 + c)) * pitch;
        A[k] = xa;
        A[pitch + k] = xb;
    };
    if constexpr (TC == 1) {  // one pair: no division by the runtime NH
        if (pair0 >= npairs) return;
        for (int k = threadIdx.x; k < NH; k += NT) one(0, k);
    } else {
        const DivU32 dnh(NH);  // t < TC * NH <= 2^15, NH <= 513
        for (int t = threadIdx.x; t < TC * NH; t += NT) {
            int c = dnh(t), k = t - c * NH;
            if (pair0 + c < npairs) one(c, k);
        }
    }
}

// plain c2r (inverse x pass) of one field; writes physical rows in place,
// scaled by norm
template <typename T, int L, int TC, int NT, typename TS>
__global__ void __launch_bounds__(NT) k_xc2r(cx<TS> *base, int64_t fs, int64_t pitch, int npairs, T norm,
                                             const cx<T> *__restrict__ tw, int kx_lim)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    using F = RowFFT<T, L, TC, NT, true>;
    const int pair0 = blockIdx.x * TC;
    cx<TS> *fb = base + blockIdx.z * fs;
    cx<T> in[F::NIN], out[F::NOUT];
#pragma unroll
    for (int i = 0; i < F::NB0; i++)
#pragma unroll
        for (int m = 0; m < F::R0; m++) {
            int c, p;
            if (F::in_slot(i, m, c, p) && pair0 + c < npairs) {
                const cx<TS> *A = fb + (int64_t)(2 * (pair0 + c)) * pitch;
                in[i * F::R0 + m] = load_packed<T, L, TS>(A, A + pitch, p, kx_lim > 0 ? kx_lim : L / 2 + 1);
            } else in[i * F::R0 + m] = mk<T>(0, 0);
        }
    F::run(in, sm, out, tw);
#pragma unroll
    for (int i = 0; i < F::NBL; i++)
#pragma unroll
        for (int m = 0; m < F::RL; m++) {
            int c, p;
            if (F::out_slot(i, m, c, p) && pair0 + c < npairs) {
                TS *A = reinterpret_cast<TS *>(fb + (int64_t)(2 * (pair0 + c)) * pitch);
                A[p] = (TS)(out[i * F::RL + m].x * norm);
                A[2 * pitch + p] = (TS)(out[i * F::RL + m].y * norm);
            }
        }
}

// plain r2c (forward x pass) of one field, in place
template <typename T, int L, int TC, int NT, typename TS>
__global__ void __launch_bounds__(NT) k_xr2c(cx<TS> *base, int64_t fs, int64_t pitch, int npairs,
                                             const cx<T> *__restrict__ tw, int kx_lim)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    using F = RowFFT<T, L, TC, NT, false>;
    const int pair0 = blockIdx.x * TC;
    cx<TS> *fb = base + blockIdx.z * fs;
    cx<T> in[F::NIN], out[F::NOUT];
#pragma unroll
    for (int i = 0; i < F::NB0; i++)
#pragma unroll
        for (int m = 0; m < F::R0; m++) {
            int c, p;
            if (F::in_slot(i, m, c, p) && pair0 + c < npairs) {
                const TS *A = reinterpret_cast<const TS *>(fb + (int64_t)(2 * (pair0 + c)) * pitch);
                in[i * F::R0 + m] = mk<T>((T)A[p], (T)A[2 * pitch + p]);
            } else in[i * F::R0 + m] = mk<T>(0, 0);
        }
    F::run(in, sm, out, tw);
    __syncthreads();
    using LY = typename F::LY;
#pragma unroll
    for (int i = 0; i < F::NBL; i++)
#pragma unroll
        for (int m = 0; m < F::RL; m++) {
            int c, p;
            if (F::out_slot(i, m, c, p)) sm[LY::idx(c, p)] = out[i * F::RL + m];
        }
    __syncthreads();
    store_split<T, L, TC, NT, TS>(sm, fb, pitch, pair0, npairs, kx_lim > 0 ? kx_lim : L / 2 + 1);
}

// ---------------------------------------------------------------------------
// fused x pass:  NIN spectral inputs (after their z and y inverse passes) ->
// c2r -> per-point operator -> NOUT forward r2c outputs, in one kernel.
// One thread-block cluster of NIN CTAs owns a tile of TC row pairs.  CTA r
// inverse-transforms input r and keeps the physical rows in its own shared
// memory; after a cluster barrier every CTA reads the fields it needs from its
// peers' shared memory (distributed shared memory) and forward-transforms the
// outputs o with o % NIN == r.  Inputs are fully consumed before the barrier, so
// outputs may overwrite inputs.
// OP provides NIN, NOUT, NPHYS, NEED_AUX, uses(o, f), cour(in), aux(in) and
// out(o, in, aux).
// ---------------------------------------------------------------------------
struct FusedArgs {
    const void *in[6];   // cx<TS>* of the NIN input fields
    void *out[6];        // cx<TS>* of the NOUT output fields (may alias inputs)
    int64_t pitch;
    int npairs;
    double norm;
    unsigned long long *cmax;  // optional: max over points of OP::cour(in) (bit pattern of a double >= 0)
    double *phys;        // optional: FP64 physical copies of the first OP::NPHYS inputs, [f][row][x]
    int64_t phys_fs, phys_pitch;
    double p0, p1;       // operator parameters
    int kx_lim;          // > 0: only kx < kx_lim is read and stored (2/3-rule pruning)
    int *err;            // optional: set (bit 1) when a bounded wait on the input stage ran out
    int nruns;           // runs of a batch (0 or 1: one run); npairs is per run
    int64_t rstride;     // elements of cx<TS> from one run's work fields to the next run's
};

// tile -> (run, first row pair of the tile) for the staged kernels: the tiles of
// a batch enumerate every run's row pairs, ntr = ceil(npairs / TC) tiles per run
struct TileMap {
    int ntr, nruns;
    H3D_D int total() const { return ntr * nruns; }
    H3D_D void at(int tile, int tc, int &run, int &pair0) const
    {
        run = nruns > 1 ? tile / ntr : 0;
        pair0 = (tile - run * ntr) * tc;
    }
};

template <typename T, int L, int TC, int NT, typename TS, class OP>
__global__ void __cluster_dims__(OP::NIN, 1, 1) __launch_bounds__(NT, 256 / NT)
    k_xfused(const FusedArgs a, const cx<T> *__restrict__ tw)
{
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) unsigned char smraw[];
    // inverse and forward share one plan (and so one set of per-thread twiddles)
    using FI = ColFFT<T, L, TC, NT, true, false, false>;
    using FF = ColFFT<T, L, TC, NT, true, true, false>;
    using LY = typename FF::LY;
    typename FF::CachedTw twc;
    FF::load_twiddles(twc, tw);
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);  // transform work buffer
    cx<T> *ph = sm + LY::elems;                      // this CTA's physical field (a + i b packed)
    cg::cluster_group cl = cg::this_cluster();
    const int r = (int)cl.block_rank();
    const int pair0 = (int)(blockIdx.x / OP::NIN) * TC;
    const T norm = (T)a.norm;
    OP op{(T)a.p0, (T)a.p1};

    // ---- phase 1: input r to physical space, kept in shared memory ----
    {
        cx<T> in[FI::NIN];
        const cx<TS> *fb = reinterpret_cast<const cx<TS> *>(a.in[r]);
#pragma unroll
        for (int i = 0; i < FI::NB0; i++)
#pragma unroll
            for (int m = 0; m < FI::R0; m++) {
                int c, p;
                if (FI::in_slot(i, m, c, p) && pair0 + c < a.npairs) {
                    const cx<TS> *A = fb + (int64_t)(2 * (pair0 + c)) * a.pitch;
                    in[i * FI::R0 + m] = load_packed<T, L, TS>(A, A + a.pitch, p, a.kx_lim > 0 ? a.kx_lim : L / 2 + 1);
                } else in[i * FI::R0 + m] = mk<T>(0, 0);
            }
        FI::run_store_t(in, sm, twc, [&](int c, int p, cx<T> v) {
            // round through the storage type so that every precision sees the
            // same physical values as a separate c2r pass would produce
            const cx<T> x = mk<T>((T)(TS)(v.x * norm), (T)(TS)(v.y * norm));
            ph[LY::idx(c, p)] = x;
            if (a.phys != nullptr && r < OP::NPHYS && pair0 + c < a.npairs) {
                const int64_t row = 2 * (pair0 + c);
                a.phys[r * a.phys_fs + row * a.phys_pitch + p] = (double)x.x;
                a.phys[r * a.phys_fs + (row + 1) * a.phys_pitch + p] = (double)x.y;
            }
        });
    }
    cl.sync();
    const cx<T> *fp[OP::NIN];
#pragma unroll
    for (int f = 0; f < OP::NIN; f++) fp[f] = cl.map_shared_rank(ph, f);

    // ---- Courant maximum (rank 0 scans the whole tile) ----
    if (a.cmax != nullptr && r == 0) {
        double cm = 0.0;
        for (int t = threadIdx.x; t < TC * L; t += NT) {
            const int c = t / L, p = t - c * L;
            if (pair0 + c >= a.npairs) continue;
            T va[OP::NIN], vb[OP::NIN];
#pragma unroll
            for (int f = 0; f < OP::NIN; f++) {
                const cx<T> v = fp[f][LY::idx(c, p)];
                va[f] = v.x;
                vb[f] = v.y;
            }
            cm = fmax(cm, fmax((double)op.cour(va), (double)op.cour(vb)));
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) cm = fmax(cm, __shfl_xor_sync(0xffffffffu, cm, off));
        if ((threadIdx.x & 31) == 0) atomicMax(a.cmax, (unsigned long long)__double_as_longlong(cm));
    }

    // ---- phase 2: outputs o = r, r + NIN, ... ----
#pragma unroll 1
    for (int o = r; o < OP::NOUT; o += OP::NIN) {
        cx<T> in[FF::NIN];
#pragma unroll
        for (int i = 0; i < FF::NB0; i++)
#pragma unroll
            for (int m = 0; m < FF::R0; m++) {
                int c, p;
                const int q = i * FF::R0 + m;
                in[q] = mk<T>(0, 0);
                if (FF::in_slot(i, m, c, p) && pair0 + c < a.npairs) {
                    T va[OP::NIN], vb[OP::NIN];
#pragma unroll
                    for (int f = 0; f < OP::NIN; f++) {
                        if (OP::NEED_AUX || OP::uses(o, f)) {
                            const cx<T> v = fp[f][LY::idx(c, p)];
                            va[f] = v.x;
                            vb[f] = v.y;
                        } else va[f] = vb[f] = (T)0;
                    }
                    T xa = (T)0, xb = (T)0;
                    if (OP::NEED_AUX) { xa = op.aux(va); xb = op.aux(vb); }
                    in[q] = mk<T>(op.out(o, va, xa), op.out(o, vb, xb));
                }
            }
        // each last-stage butterfly reads and writes only its own positions, so
        // its outputs can go straight back into the work buffer
        FF::run_store_t(in, sm, twc, [&](int c, int p, cx<T> v) { sm[LY::idx(c, p)] = v; });
        __syncthreads();
        store_split<T, L, TC, NT, TS>(sm, reinterpret_cast<cx<TS> *>(a.out[o]), a.pitch, pair0, a.npairs,
                                      a.kx_lim > 0 ? a.kx_lim : L / 2 + 1);
        __syncthreads();
    }
    cl.sync();  // peers may still be reading this CTA's physical field
}

// Register-resident variant of the fused x pass (one CTA per tile): the three
// physical inputs stay in registers between the inverse and forward
// transforms, handed over slot for slot because the inverse uses the reversed
// radix plan.  Fewer warps per SM than the cluster variant but no shared-memory
// round trip for the physical fields; the tuner picks between them.
template <typename T, int L, int TC, int NT, typename TS, class OP>
__global__ void __launch_bounds__(NT) k_xfused_reg(const FusedArgs a, const cx<T> *__restrict__ tw)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    using FI = RowFFT<T, L, TC, NT, true>;
    using FF = RowFFT<T, L, TC, NT, false>;
    static_assert(FI::NOUT == FF::NIN, "slot hand-off mismatch");
    constexpr int NP = FI::NOUT;
    const int pair0 = blockIdx.x * TC;
    const T norm = (T)a.norm;
    OP op{(T)a.p0, (T)a.p1};

    cx<T> phys[OP::NIN][NP];
#pragma unroll
    for (int f = 0; f < OP::NIN; f++) {
        cx<T> in[FI::NIN];
        const cx<TS> *fb = reinterpret_cast<const cx<TS> *>(a.in[f]);
#pragma unroll
        for (int i = 0; i < FI::NB0; i++)
#pragma unroll
            for (int m = 0; m < FI::R0; m++) {
                int c, p;
                if (FI::in_slot(i, m, c, p) && pair0 + c < a.npairs) {
                    const cx<TS> *A = fb + (int64_t)(2 * (pair0 + c)) * a.pitch;
                    in[i * FI::R0 + m] = load_packed<T, L, TS>(A, A + a.pitch, p, a.kx_lim > 0 ? a.kx_lim : L / 2 + 1);
                } else in[i * FI::R0 + m] = mk<T>(0, 0);
            }
        // slots of idle butterflies are never written by run(): keep them zero so
        // that the Courant maximum and the products never see stale registers
#pragma unroll
        for (int q = 0; q < NP; q++) phys[f][q] = mk<T>(0, 0);
        FI::run(in, sm, phys[f], tw);
#pragma unroll
        for (int q = 0; q < NP; q++) phys[f][q] = mk<T>(phys[f][q].x * norm, phys[f][q].y * norm);
        __syncthreads();
    }
    // optional physical copies and the Courant maximum
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
                        pb[f * a.phys_fs + r * a.phys_pitch + p] = (double)phys[f][i * FI::RL + m].x;
                        pb[f * a.phys_fs + (r + 1) * a.phys_pitch + p] = (double)phys[f][i * FI::RL + m].y;
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
        // padding slots hold zeros, so they never raise the maximum
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) cm = fmax(cm, __shfl_xor_sync(0xffffffffu, cm, off));
        if ((threadIdx.x & 31) == 0) atomicMax(a.cmax, (unsigned long long)__double_as_longlong(cm));
    }
    // per-point auxiliary (e.g. eddy viscosity)
    cx<T> aux[NP];
#pragma unroll
    for (int q = 0; q < NP; q++) {
        T va[OP::NIN], vb[OP::NIN];
#pragma unroll
        for (int f = 0; f < OP::NIN; f++) { va[f] = phys[f][q].x; vb[f] = phys[f][q].y; }
        aux[q] = mk<T>(op.aux(va), op.aux(vb));
    }
    using LY = typename FF::LY;
#pragma unroll 1
    for (int o = 0; o < OP::NOUT; o++) {
        cx<T> in[FF::NIN], out[FF::NOUT];
#pragma unroll
        for (int q = 0; q < NP; q++) {
            T va[OP::NIN], vb[OP::NIN];
#pragma unroll
            for (int f = 0; f < OP::NIN; f++) { va[f] = phys[f][q].x; vb[f] = phys[f][q].y; }
            in[q] = mk<T>(op.out(o, va, aux[q].x), op.out(o, vb, aux[q].y));
        }
        FF::run(in, sm, out, tw);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < FF::NBL; i++)
#pragma unroll
            for (int m = 0; m < FF::RL; m++) {
                int c, p;
                if (FF::out_slot(i, m, c, p)) sm[LY::idx(c, p)] = out[i * FF::RL + m];
            }
        __syncthreads();
        store_split<T, L, TC, NT, TS>(sm, reinterpret_cast<cx<TS> *>(a.out[o]), a.pitch, pair0, a.npairs,
                                      a.kx_lim > 0 ? a.kx_lim : L / 2 + 1);
        __syncthreads();
    }
}


// Lockstep form of the fused x pass: the NIN inverse transforms advance
// together (one barrier per radix stage for all of them, one twiddle load per
// butterfly) and the NOUT forward transforms in groups of GF, each transform
// with its own shared-memory buffer.  More independent work between barriers
// than k_xfused_reg at the same register budget per transform; the tuner picks.
// MINB > 1 caps the registers so that MINB CTAs share an SM.
template <typename T, int L, int TC, int NT, typename TS, class OP, int GF, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) k_xfused_ms(const FusedArgs a, const cx<T> *__restrict__ tw)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    using FI = RowFFT<T, L, TC, NT, true>;
    using FF = RowFFT<T, L, TC, NT, false>;
    static_assert(FI::NOUT == FF::NIN, "slot hand-off mismatch");
    constexpr int NP = FI::NOUT;
    constexpr int E = Lay<L, TC, true>::elems;
    const int pair0 = blockIdx.x * TC;
    const T norm = (T)a.norm;
    const int lim = a.kx_lim > 0 ? a.kx_lim : L / 2 + 1;
    OP op{(T)a.p0, (T)a.p1};

    cx<T> phys[OP::NIN][NP];
    {
        cx<T> in[OP::NIN][FI::NIN];
#pragma unroll
        for (int f = 0; f < OP::NIN; f++) {
            const cx<TS> *fb = reinterpret_cast<const cx<TS> *>(a.in[f]);
#pragma unroll
            for (int i = 0; i < FI::NB0; i++)
#pragma unroll
                for (int m = 0; m < FI::R0; m++) {
                    int c, p;
                    if (FI::in_slot(i, m, c, p) && pair0 + c < a.npairs) {
                        const cx<TS> *A = fb + (int64_t)(2 * (pair0 + c)) * a.pitch;
                        in[f][i * FI::R0 + m] = load_packed<T, L, TS>(A, A + a.pitch, p, lim);
                    } else in[f][i * FI::R0 + m] = mk<T>(0, 0);
                }
            // idle butterflies never write their slots: keep them zero
#pragma unroll
            for (int q = 0; q < NP; q++) phys[f][q] = mk<T>(0, 0);
        }
        FI::template run_multi<OP::NIN>(in, sm, phys, tw);
    }
#pragma unroll
    for (int f = 0; f < OP::NIN; f++)
#pragma unroll
        for (int q = 0; q < NP; q++) phys[f][q] = mk<T>(phys[f][q].x * norm, phys[f][q].y * norm);
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
                        pb[f * a.phys_fs + r * a.phys_pitch + p] = (double)phys[f][i * FI::RL + m].x;
                        pb[f * a.phys_fs + (r + 1) * a.phys_pitch + p] = (double)phys[f][i * FI::RL + m].y;
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
        if ((threadIdx.x & 31) == 0) atomicMax(a.cmax, (unsigned long long)__double_as_longlong(cm));
    }
    cx<T> aux[NP];
#pragma unroll
    for (int q = 0; q < NP; q++) {
        T va[OP::NIN], vb[OP::NIN];
#pragma unroll
        for (int f = 0; f < OP::NIN; f++) { va[f] = phys[f][q].x; vb[f] = phys[f][q].y; }
        aux[q] = mk<T>(op.aux(va), op.aux(vb));
    }
    using LY = typename FF::LY;
    constexpr int NG = (OP::NOUT + GF - 1) / GF;
#pragma unroll 1
    for (int g = 0; g < NG; g++) {
        cx<T> in[GF][FF::NIN], out[GF][FF::NOUT];
#pragma unroll
        for (int gf = 0; gf < GF; gf++) {
            const int o = g * GF + gf;
#pragma unroll
            for (int q = 0; q < NP; q++) {
                T va[OP::NIN], vb[OP::NIN];
#pragma unroll
                for (int f = 0; f < OP::NIN; f++) { va[f] = phys[f][q].x; vb[f] = phys[f][q].y; }
                in[gf][q] = o < OP::NOUT ? mk<T>(op.out(o, va, aux[q].x), op.out(o, vb, aux[q].y)) : mk<T>(0, 0);
            }
        }
        FF::template run_multi<GF>(in, sm, out, tw);
        __syncthreads();
#pragma unroll
        for (int gf = 0; gf < GF; gf++)
#pragma unroll
            for (int i = 0; i < FF::NBL; i++)
#pragma unroll
                for (int m = 0; m < FF::RL; m++) {
                    int c, p;
                    if (FF::out_slot(i, m, c, p)) sm[gf * E + LY::idx(c, p)] = out[gf][i * FF::RL + m];
                }
        __syncthreads();
#pragma unroll
        for (int gf = 0; gf < GF; gf++) {
            const int o = g * GF + gf;
            if (o < OP::NOUT)
                store_split<T, L, TC, NT, TS>(sm + gf * E, reinterpret_cast<cx<TS> *>(a.out[o]), a.pitch, pair0,
                                              a.npairs, lim);
        }
        __syncthreads();
    }
}

// Staged lockstep form: each CTA walks tiles blockIdx.x, blockIdx.x + gridDim.x,
// ... (grid = the CTAs resident at once).  The kx < lim columns of the next
// tile's input rows are copied into a shared-memory stage with cp.async while
// the current tile is transformed, so the global-load latency that dominates
// k_xfused_ms at its low occupancy overlaps the FFT work.  Stage layout:
// [f][row 0..2 TC)[RS elements], RS = 16-byte chunks per row; rows of a pair
// beyond npairs are neither copied nor read.  Requires 16-byte aligned input
// fields and a pitch that is a multiple of 16 bytes (checked by the host).
H3D_D void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
H3D_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
H3D_D void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <typename TS> struct StageRow {
    static constexpr int PER = 16 / (int)sizeof(cx<TS>);  // elements per 16-byte chunk
    static H3D_HD int chunks(int lim) { return (lim + PER - 1) / PER; }
};

template <typename TS, int NIN, int TC, int NT>
H3D_D void stage_issue(const FusedArgs &a, cx<TS> *st, int pair0, int nch, int64_t roff = 0)
{
    constexpr int PER = StageRow<TS>::PER;
    const int rs = nch * PER;
    if constexpr (TC == 1) {  // one pair: row by row, no division by the runtime nch
        if (pair0 < a.npairs) {
#pragma unroll
            for (int rr = 0; rr < NIN * 2; rr++) {
                const cx<TS> *src = reinterpret_cast<const cx<TS> *>(a.in[rr >> 1]) + roff + (int64_t)(2 * pair0 + (rr & 1)) * a.pitch;
                for (int ch = threadIdx.x; ch < nch; ch += NT) cp_async16(st + rr * rs + ch * PER, src + ch * PER);
            }
        }
    } else {
        const int total = NIN * 2 * TC * nch;
        const DivU32 dch(nch);  // q < total <= 2^18, nch <= 513
        for (int q = threadIdx.x; q < total; q += NT) {
            const int rr = dch(q), ch = q - rr * nch;
            const int r = rr % (2 * TC), f = rr / (2 * TC);
            if (pair0 + r / 2 >= a.npairs) continue;
            const cx<TS> *src = reinterpret_cast<const cx<TS> *>(a.in[f]) + roff + (int64_t)(2 * pair0 + r) * a.pitch + ch * PER;
            cp_async16(st + (f * 2 * TC + r) * rs + ch * PER, src);
        }
    }
    cp_async_commit();
}

template <typename T, int L, int TC, int NT, typename TS, class OP, int GF, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) k_xfused_st(const FusedArgs a, const cx<T> *__restrict__ tw)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    using FI = RowFFT<T, L, TC, NT, true>;
    using FF = RowFFT<T, L, TC, NT, false>;
    static_assert(FI::NOUT == FF::NIN, "slot hand-off mismatch");
    constexpr int NP = FI::NOUT;
    constexpr int E = Lay<L, TC, true>::elems;
    constexpr int NB = OP::NIN > GF ? OP::NIN : GF;
    constexpr size_t SOFF = ((size_t)NB * E * sizeof(cx<T>) + 15) / 16 * 16;  // cp.async wants 16-byte targets
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    cx<TS> *st = reinterpret_cast<cx<TS> *>(smraw + SOFF);
    const T norm = (T)a.norm;
    const int lim = a.kx_lim > 0 ? a.kx_lim : L / 2 + 1;
    const int nch = StageRow<TS>::chunks(lim);
    const int rs = nch * StageRow<TS>::PER;
    const TileMap tm{(a.npairs + TC - 1) / TC, a.nruns > 1 ? a.nruns : 1};
    const int ntiles = tm.total();
    OP op{(T)a.p0, (T)a.p1};
    // each warp's Courant maximum over its tiles, kept in shared memory rather
    // than in a register live across the tile loop; one atomic per warp at the end
    __shared__ double cwarp[NT / 32];
    if ((threadIdx.x & 31) == 0) cwarp[threadIdx.x >> 5] = 0.0;
    if ((int)blockIdx.x < ntiles) {
        int r0, p0;
        tm.at(blockIdx.x, TC, r0, p0);
        stage_issue<TS, OP::NIN, TC, NT>(a, st, p0, nch, r0 * a.rstride);
    }

#pragma unroll 1
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int run, pair0;
        tm.at(tile, TC, run, pair0);
        const int64_t roff = run * a.rstride;
        cx<T> phys[OP::NIN][NP];
        {
            cp_async_wait_all();
            __syncthreads();
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
            __syncthreads();  // the stage is free: prefetch the next tile
            if (tile + (int)gridDim.x < ntiles) {
                int rn, pn;
                tm.at(tile + gridDim.x, TC, rn, pn);
                stage_issue<TS, OP::NIN, TC, NT>(a, st, pn, nch, rn * a.rstride);
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
        using LY = typename FF::LY;
        constexpr int NG = (OP::NOUT + GF - 1) / GF;
        // unrolled: each group's products are fixed at compile time, and an input
        // field that no later group reads (u after uu, uv, uw) is dead during the
        // later transforms; at 512 FP64 this takes the spills from 328 to 16 bytes
#pragma unroll
        for (int g = 0; g < NG; g++) {
            cx<T> in[GF][FF::NIN], out[GF][FF::NOUT];
#pragma unroll
            for (int gf = 0; gf < GF; gf++) {
                const int o = g * GF + gf;
#pragma unroll
                for (int q = 0; q < NP; q++) {
                    T va[OP::NIN], vb[OP::NIN];
#pragma unroll
                    for (int f = 0; f < OP::NIN; f++) { va[f] = phys[f][q].x; vb[f] = phys[f][q].y; }
                    in[gf][q] = o < OP::NOUT ? mk<T>(op.out(o, va, aux[q].x), op.out(o, vb, aux[q].y)) : mk<T>(0, 0);
                }
            }
            FF::template run_multi<GF>(in, sm, out, tw);
            __syncthreads();
#pragma unroll
            for (int gf = 0; gf < GF; gf++)
#pragma unroll
                for (int i = 0; i < FF::NBL; i++)
#pragma unroll
                    for (int m = 0; m < FF::RL; m++) {
                        int c, p;
                        if (FF::out_slot(i, m, c, p)) sm[gf * E + LY::idx(c, p)] = out[gf][i * FF::RL + m];
                    }
            __syncthreads();
#pragma unroll
            for (int gf = 0; gf < GF; gf++) {
                const int o = g * GF + gf;
                if (o < OP::NOUT)
                    store_split<T, L, TC, NT, TS>(sm + gf * E, reinterpret_cast<cx<TS> *>(a.out[o]) + roff, a.pitch, pair0,
                                              a.npairs, lim, OP::QUAD ? (T)0.5 * (T)a.norm * (T)a.norm : (T)0.5);
            }
            __syncthreads();
        }
    }
    cp_async_wait_all();
    if (a.cmax != nullptr && (threadIdx.x & 31) == 0)
        atomicMax(a.cmax, (unsigned long long)__double_as_longlong(cwarp[threadIdx.x >> 5] * (OP::QUAD ? (double)(T)a.norm : 1.0)));
}

// velocity products (rhs_velocity.f90:56-72): uu uv uw vv vw ww; Courant |u|+|v|+|w|
template <typename T> struct OpVel {
    static constexpr int NIN = 3, NOUT = 6, NPHYS = 3;
    static constexpr bool QUAD = true;  // products of degree 2, Courant of degree 1 in the fields
    static constexpr bool NEED_AUX = false;
    static H3D_HD constexpr bool uses(int o, int f)
    {
        return o == 0 ? f == 0 : o == 1 ? f <= 1 : o == 2 ? (f == 0 || f == 2) : o == 3 ? f == 1 : o == 4 ? f >= 1 : f == 2;
    }
    T p0, p1;
    H3D_D T cour(const T *v) const { return fabs(v[0]) + fabs(v[1]) + fabs(v[2]); }
    H3D_D T aux(const T *) const { return (T)0; }
    H3D_D T out(int o, const T *v, T) const
    {
        switch (o) {
        case 0: return v[0] * v[0];
        case 1: return v[0] * v[1];
        case 2: return v[0] * v[2];
        case 3: return v[1] * v[1];
        case 4: return v[1] * v[2];
        default: return v[2] * v[2];
        }
    }
};

// scalar fluxes (rhs_scalars.f90:82-85): phi*u, phi*v, phi*w from (u, v, w, phi)
template <typename T> struct OpScal {
    static constexpr int NIN = 4, NOUT = 3, NPHYS = 0;
    static constexpr bool QUAD = false;
    static constexpr bool NEED_AUX = false;
    static H3D_HD constexpr bool uses(int o, int f) { return f == o || f == 3; }
    T p0, p1;
    H3D_D T cour(const T *v) const { return fabs(v[0]) + fabs(v[1]) + fabs(v[2]); }
    H3D_D T aux(const T *) const { return (T)0; }
    H3D_D T out(int o, const T *v, T) const { return v[3] * v[o]; }
};

// Smagorinsky: inputs S11 S12 S13 S22 S23 S33, aux = nu_t = (Cs Delta)^2 sqrt(2 S:S)
// (m_les.f90:1176-1212), outputs tau_ij = -2 nu_t S_ij (m_les.f90:935,989).
// p0 = (Cs Delta)^2
template <typename T> struct OpSmag {
    static constexpr int NIN = 6, NOUT = 6, NPHYS = 0;
    static constexpr bool QUAD = false;
    static constexpr bool NEED_AUX = true;
    static H3D_HD constexpr bool uses(int o, int f) { return f == o; }
    T p0, p1;
    H3D_D T cour(const T *) const { return (T)0; }
    H3D_D T aux(const T *s) const
    {
        T t = s[0] * s[0];
        t = t + (T)2 * (s[1] * s[1]);
        t = t + (T)2 * (s[2] * s[2]);
        t = t + s[3] * s[3];
        t = t + (T)2 * (s[4] * s[4]);
        t = t + s[5] * s[5];
        return sqrt((T)2 * t) * p0;
    }
    H3D_D T out(int o, const T *s, T nut) const { return ((T)-2 * nut) * s[o]; }
};
