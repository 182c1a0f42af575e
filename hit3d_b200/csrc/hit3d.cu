// C-ABI of the B200 pseudospectral step (declared in include/hit3d_gpu.h):
// device state, transform launchers dispatched on the grid size, the time step
// pipeline, statistics, initial conditions and particles.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <mutex>
#include <set>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/hit3d_gpu.h"
#include "particles.cuh"
#include "ctx.cuh"
#include "passes.cuh"
#include "launch_cfg.cuh"
#include "colpipe.cuh"
#include "spectral.cuh"
#include "fused_update.cuh"

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

int h3d_set_error(cudaError_t e, const char *what, const char *file, int line)
{
    char buf[512];
    snprintf(buf, sizeof buf, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    g_err = buf;
    return -2;
}
int h3d_set_error_msg(int code, const char *msg)
{
    g_err = msg;
    return code;
}
extern "C" const char *hit3d_gpu_last_error(void) { return g_err.c_str(); }

// z pass reading the FP64 state with a spectral pre-operation, writing [z][ky][kx]
template <typename T, int L, int MODE, int CT>
static int zinv_LMC(hit3d_ctx *c, int nf, int sfield, const double2 *src, int64_t src_fs, cx<T> *dst,
                    int64_t dst_fs, int dpitch)
{
    using CF = ColCfgT<T, L, false, CT>;
    using IO = IOSpec<T, T, MODE>;
    IO io;
    io.src = src; io.dst = dst; io.fs_src = src_fs; io.fs_dst = dst_fs;
    io.n = c->n; io.psrc = c->P64; io.pdst = dpitch; io.ncol = c->nh; io.sfield = sfield;
    io.dx = c->dx;
    io.k2max = c->k2max;
    io.g = c->zfilt ? c->zfilt : c->gfilt;
    int rows = c->n;
    if (c->kc_active >= 0) {
        io.kl = io.ko = c->kc_active;
        io.ncol = c->kc_active + 1;
        rows = 2 * c->kc_active + 1;
    }
    int nz = nf;
    if (c->bruns > 0) {  // every run of a batch class: state run stride bru, work run stride brw
        io.nfr = nf;
        io.rs_src = c->bru;
        io.rs_dst = c->brw;
        nz = nf * c->bruns;
    }
    auto k = k_colfft<T, L, CF::TC, CF::NT, false, IO, CF::MINB>;
    H3D_TRY(set_smem(k, CF::SMEM));
    dim3 g((io.ncol + CF::TC - 1) / CF::TC, rows, nz);
    k<<<g, CF::NT, CF::SMEM, c->st>>>(io, twid<T>(c));
    H3D_LAUNCH_CHECK();
    return 0;
}
// the pipelined strided pass (k_colfft_pipe): a grid of resident CTAs walking
// every tile of the pass, with the tile after next in flight
template <typename T, int L, bool FWD, class IO> static int colpipe_launch(hit3d_ctx *c, const IO &io, int ncol, int rows, int nz)
{
    using TI = typename ColIn<IO>::type;
    using CF = ColPipeCfg<T, TI, L>;
    auto k = k_colfft_pipe<T, L, CF::TC, CF::NT, FWD, IO, CF::MINB>;
    H3D_TRY(set_smem(k, CF::SMEM));
    const ColTiles tl{(ncol + CF::TC - 1) / CF::TC, rows};
    const int64_t ntiles = (int64_t)tl.nx * rows * nz;
    if (ntiles > INT32_MAX) return h3d_set_error_msg(-1, "pipelined column pass: too many tiles");
    int64_t grid = (int64_t)c->nsm * CF::MINB;
    grid = grid < ntiles ? grid : ntiles;
    k<<<(unsigned)grid, CF::NT, CF::SMEM, c->st>>>(io, twid<T>(c), tl, (int)ntiles);
    H3D_LAUNCH_CHECK();
    return 0;
}

// the tuned column tile (ctile) applies to the plain copy of grids up to 512;
// ctile 3 takes the pipelined pass at every size
template <typename T, int L, int MODE>
static int zinv_LM(hit3d_ctx *c, int nf, int sfield, const double2 *src, int64_t src_fs, cx<T> *dst,
                   int64_t dst_fs, int dpitch)
{
    if constexpr (MODE == PRE_COPY) {
        if (c->ctile == 3) {
            IOSpec<T, T, PRE_COPY> io;
            io.src = src; io.dst = dst; io.fs_src = src_fs; io.fs_dst = dst_fs;
            io.n = c->n; io.psrc = c->P64; io.pdst = dpitch; io.ncol = c->nh; io.sfield = sfield;
            io.dx = c->dx;
            int rows = c->n;
            if (c->kc_active >= 0) {
                io.kl = io.ko = c->kc_active;
                io.ncol = c->kc_active + 1;
                rows = 2 * c->kc_active + 1;
            }
            int nz = nf;
            if (c->bruns > 0) {
                io.nfr = nf;
                io.rs_src = c->bru;
                io.rs_dst = c->brw;
                nz = nf * c->bruns;
            }
            return colpipe_launch<T, L, false>(c, io, io.ncol, rows, nz);
        }
    }
    if constexpr (L <= 512 && MODE == PRE_COPY) {
        if (c->ctile == 1) return zinv_LMC<T, L, MODE, 1>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
        if (c->ctile == 2) return zinv_LMC<T, L, MODE, 2>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
    }
    return zinv_LMC<T, L, MODE, 0>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
}
template <typename T, int L>
static int zinv_L(hit3d_ctx *c, int nf, int mode, int sfield, const double2 *src, int64_t src_fs, cx<T> *dst,
                  int64_t dst_fs, int dpitch)
{
    switch (mode) {
    case PRE_COPY: return zinv_LM<T, L, PRE_COPY>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
    case PRE_SHIFT: return zinv_LM<T, L, PRE_SHIFT>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
    case PRE_STRAIN_A: return zinv_LM<T, L, PRE_STRAIN_A>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
    case PRE_STRAIN_B: return zinv_LM<T, L, PRE_STRAIN_B>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
    case PRE_GRAD: return zinv_LM<T, L, PRE_GRAD>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
    case PRE_QUART: return zinv_LM<T, L, PRE_QUART>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
    default: break;
    }
    if constexpr (std::is_same<T, double>::value) {
        // statistics pre-operations run in FP64 only
        switch (mode) {
        case PRE_CURL: return zinv_LM<T, L, PRE_CURL>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
        case PRE_DLONG: return zinv_LM<T, L, PRE_DLONG>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
        case PRE_TRUNC: return zinv_LM<T, L, PRE_TRUNC>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
        case PRE_CUBE: return zinv_LM<T, L, PRE_CUBE>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
        case PRE_FILT: return zinv_LM<T, L, PRE_FILT>(c, nf, sfield, src, src_fs, dst, dst_fs, dpitch);
        default: break;
        }
    }
    return h3d_set_error_msg(-1, "unsupported spectral pre-operation");
}
template <typename T>
static int zinv(hit3d_ctx *c, int nf, int mode, int sfield, const double2 *src, int64_t src_fs, cx<T> *dst,
                int64_t dst_fs, int dpitch)
{
#define CALL(L) zinv_L<T, L>(c, nf, mode, sfield, src, src_fs, dst, dst_fs, dpitch)
    H3D_DISPATCH(c->n, CALL)
#undef CALL
}

// in-place strided pass: axis 1 = y (stride pitch, outer z), axis 2 = z (stride n*pitch, outer ky)
template <typename T, int L, bool YPASS, int CT>
static int spass_LAC(hit3d_ctx *c, int axis, bool fwd, cx<T> *base, int64_t fs, int pitch, int nf)
{
    using CF = ColCfgT<T, L, YPASS, CT>;
    IOPlain<T, T, T> io;
    io.src = base; io.dst = base; io.fs_src = fs; io.fs_dst = fs; io.ncol = c->nh;
    if (axis == 1) { io.sa_src = io.sa_dst = pitch; io.so_src = io.so_dst = (int64_t)c->n * pitch; }
    else { io.sa_src = io.sa_dst = (int64_t)c->n * pitch; io.so_src = io.so_dst = pitch; }
    int rows = c->n;
    if (c->kc_active >= 0) {
        // kx <= kc only; inverse passes read |k| <= kc along the axis, forward
        // passes store |k| <= kc; the z pass visits only the kept ky rows
        io.n = c->n;
        io.ncol = c->kc_active + 1;
        if (fwd) io.ks = c->kc_active;
        else io.kl = c->kc_active;
        if (axis == 2) {
            io.ko = c->kc_active;
            rows = 2 * c->kc_active + 1;
        }
    }
    int nz = nf;
    if (c->bruns > 0) {  // every run of a batch class (work fields, run stride brw)
        io.nfr = nf;
        io.rs_src = io.rs_dst = c->brw;
        nz = nf * c->bruns;
    }
    dim3 g((io.ncol + CF::TC - 1) / CF::TC, rows, nz);
    if (fwd) {
        auto k = k_colfft<T, L, CF::TC, CF::NT, true, IOPlain<T, T, T>, CF::MINB>;
        H3D_TRY(set_smem(k, CF::SMEM));
        k<<<g, CF::NT, CF::SMEM, c->st>>>(io, twid<T>(c));
    } else {
        auto k = k_colfft<T, L, CF::TC, CF::NT, false, IOPlain<T, T, T>, CF::MINB>;
        H3D_TRY(set_smem(k, CF::SMEM));
        k<<<g, CF::NT, CF::SMEM, c->st>>>(io, twid<T>(c));
    }
    H3D_LAUNCH_CHECK();
    return 0;
}
template <typename T, int L, bool YPASS>
static int spass_LA(hit3d_ctx *c, int axis, bool fwd, cx<T> *base, int64_t fs, int pitch, int nf)
{
    if (c->ctile == 3) {
        IOPlain<T, T, T> io;
        io.src = base; io.dst = base; io.fs_src = fs; io.fs_dst = fs; io.ncol = c->nh;
        if (axis == 1) { io.sa_src = io.sa_dst = pitch; io.so_src = io.so_dst = (int64_t)c->n * pitch; }
        else { io.sa_src = io.sa_dst = (int64_t)c->n * pitch; io.so_src = io.so_dst = pitch; }
        int rows = c->n;
        if (c->kc_active >= 0) {
            io.n = c->n;
            io.ncol = c->kc_active + 1;
            if (fwd) io.ks = c->kc_active;
            else io.kl = c->kc_active;
            if (axis == 2) {
                io.ko = c->kc_active;
                rows = 2 * c->kc_active + 1;
            }
        }
        int nz = nf;
        if (c->bruns > 0) {
            io.nfr = nf;
            io.rs_src = io.rs_dst = c->brw;
            nz = nf * c->bruns;
        }
        return fwd ? colpipe_launch<T, L, true>(c, io, io.ncol, rows, nz) : colpipe_launch<T, L, false>(c, io, io.ncol, rows, nz);
    }
    if constexpr (L <= 512) {
        if (c->ctile == 1) return spass_LAC<T, L, YPASS, 1>(c, axis, fwd, base, fs, pitch, nf);
        if (c->ctile == 2) return spass_LAC<T, L, YPASS, 2>(c, axis, fwd, base, fs, pitch, nf);
    }
    return spass_LAC<T, L, YPASS, 0>(c, axis, fwd, base, fs, pitch, nf);
}
template <typename T, int L>
static int spass_L(hit3d_ctx *c, int axis, bool fwd, cx<T> *base, int64_t fs, int pitch, int nf)
{
    return axis == 1 ? spass_LA<T, L, true>(c, axis, fwd, base, fs, pitch, nf)
                     : spass_LA<T, L, false>(c, axis, fwd, base, fs, pitch, nf);
}
template <typename T> static int spass(hit3d_ctx *c, int axis, bool fwd, cx<T> *base, int64_t fs, int pitch, int nf)
{
#define CALL(L) spass_L<T, L>(c, axis, fwd, base, fs, pitch, nf)
    H3D_DISPATCH(c->n, CALL)
#undef CALL
}

template <typename T, int L> static int xc2r_L(hit3d_ctx *c, cx<T> *base, int64_t fs, int pitch, int nf)
{
    using RC = RowCfg<T, L>;
    const int npairs = c->n * c->n / 2;
    auto k = k_xc2r<T, L, RC::TC, RC::NT, T>;
    H3D_TRY(set_smem(k, RC::SMEM));
    const double n3 = (double)c->n * c->n * c->n;
    k<<<dim3((npairs + RC::TC - 1) / RC::TC, 1, nf), RC::NT, RC::SMEM, c->st>>>(
        base, fs, pitch, npairs, (T)(1.0 / n3), twid<T>(c), c->kc_active >= 0 ? c->kc_active + 1 : 0);
    H3D_LAUNCH_CHECK();
    return 0;
}
template <typename T> static int xc2r(hit3d_ctx *c, cx<T> *base, int64_t fs, int pitch, int nf)
{
#define CALL(L) xc2r_L<T, L>(c, base, fs, pitch, nf)
    H3D_DISPATCH(c->n, CALL)
#undef CALL
}

template <typename T, int L> static int xr2c_L(hit3d_ctx *c, cx<T> *base, int64_t fs, int pitch, int nf)
{
    using RC = RowCfg<T, L>;
    const int npairs = c->n * c->n / 2;
    auto k = k_xr2c<T, L, RC::TC, RC::NT, T>;
    H3D_TRY(set_smem(k, RC::SMEM));
    k<<<dim3((npairs + RC::TC - 1) / RC::TC, 1, nf), RC::NT, RC::SMEM, c->st>>>(
        base, fs, pitch, npairs, twid<T>(c), c->kc_active >= 0 ? c->kc_active + 1 : 0);
    H3D_LAUNCH_CHECK();
    return 0;
}
template <typename T> static int xr2c(hit3d_ctx *c, cx<T> *base, int64_t fs, int pitch, int nf)
{
#define CALL(L) xr2c_L<T, L>(c, base, fs, pitch, nf)
    H3D_DISPATCH(c->n, CALL)
#undef CALL
}

// the fused x pass (xpass.cuh), instantiated in xpass_f64.cu and xpass_f32.cu
template <typename T, template <class> class OP> int xfused(hit3d_ctx *c, FusedArgs a);
constexpr int kFusedVariants = HIT3D_FUSED_VARIANTS;

static dim3 pw_grid(const hit3d_ctx *c) { return dim3(c->nsm * 4); }
// grid of a grid-stride kernel of 256-thread CTAs that may fit fewer than four
// CTAs per SM: as many CTAs as are resident at once (at most four per SM), so
// that no partial second wave leaves most SMs idle at the end of the pass
static std::mutex g_occ_mu;
static std::vector<std::pair<const void *, int>> g_occ;
template <typename KF> static dim3 pw_grid(const hit3d_ctx *c, KF kernel)
{
    const void *key = reinterpret_cast<const void *>(kernel);
    int per = 0;
    {
        std::lock_guard<std::mutex> lk(g_occ_mu);
        for (auto &e : g_occ)
            if (e.first == key) per = e.second;
        if (per == 0) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, 256, 0) != cudaSuccess) {
                (void)cudaGetLastError();  // not a launch error: fall back to one CTA per SM
                per = 1;
            }
            if (per < 1) per = 1;
            if (per > 4) per = 4;
            g_occ.emplace_back(key, per);
        }
    }
    return dim3(c->nsm * per);
}

// z forward pass of the six velocity products (after their y pass, in P) fused
// with the 2/3-rule update of U and RO and, with zinv, the z inverse of the new
// u, v, w into P[0..2]
template <typename T, int L, bool PRUNED> static int zfwd_update_LP(hit3d_ctx *c, const ZUpdArgs<T> &za)
{
    using CF = ZUpdCfg<T, L>;
    auto k = k_zfwd_update<T, L, CF::TC, CF::NT, CF::NB, CF::MINB, PRUNED>;
    H3D_TRY(set_smem(k, CF::SMEM));
    const int64_t ntiles = (int64_t)((za.ncol + CF::TC - 1) / CF::TC) * za.nrows;
    int64_t grid = (int64_t)c->nsm * CF::MINB;
    grid = grid < ntiles ? grid : ntiles;
    k<<<(unsigned)grid, CF::NT, CF::SMEM, c->st>>>(za, twid<T>(c));
    H3D_LAUNCH_CHECK();
    return 0;
}
template <typename T, int L> static int zfwd_update_L(hit3d_ctx *c, const ZUpdArgs<T> &za)
{
    if (c->kc_active >= 0) {
        if (c->kc_active != L / 3) return h3d_set_error_msg(-1, "fused z pass + update: pruning cutoff is not N/3");
        return zfwd_update_LP<T, L, true>(c, za);
    }
    return zfwd_update_LP<T, L, false>(c, za);
}
template <typename T> static int zfwd_update(hit3d_ctx *c, const StepArgs &a, cx<T> *P, bool zinv)
{
    if (c->bruns > 0) return h3d_set_error_msg(-1, "fused z pass + update: not for batch classes");
    ZUpdArgs<T> za;
    za.a = a;
    za.W = P;
    za.U = c->U;
    za.RO = c->RO;
    za.ncol = c->kc_active >= 0 ? c->kc_active + 1 : c->nh;
    za.nrows = c->kc_active >= 0 ? 2 * c->kc_active + 1 : c->n;
    za.zinv = zinv ? 1 : 0;
#define CALL(L) zfwd_update_L<T, L>(c, za)
    H3D_DISPATCH(c->n, CALL)
#undef CALL
}

// full forward 3-D transform of nf FP64 scratch fields holding physical rows
static int fwd3d64(hit3d_ctx *c, double2 *base, int nf)
{
    H3D_TRY(xr2c<double>(c, base, c->fs64, c->P64, nf));
    H3D_TRY(spass<double>(c, 1, true, base, c->fs64, c->P64, nf));
    H3D_TRY(spass<double>(c, 2, true, base, c->fs64, c->P64, nf));
    return 0;
}
// full inverse of nf spectral FP64 fields in place
static int inv3d64(hit3d_ctx *c, double2 *base, int nf)
{
    H3D_TRY(spass<double>(c, 2, false, base, c->fs64, c->P64, nf));
    H3D_TRY(spass<double>(c, 1, false, base, c->fs64, c->P64, nf));
    H3D_TRY(xc2r<double>(c, base, c->fs64, c->P64, nf));
    return 0;
}
// inverse from the state with a pre-operation into W64[0..nf)
static int inv_from_state(hit3d_ctx *c, int nf, int mode, int sfield, const double2 *src)
{
    H3D_TRY(zinv<double>(c, nf, mode, sfield, src, c->fs64, c->W64, c->fs64, c->P64));
    H3D_TRY(spass<double>(c, 1, false, c->W64, c->fs64, c->P64, nf));
    H3D_TRY(xc2r<double>(c, c->W64, c->fs64, c->P64, nf));
    return 0;
}

// ---------------------------------------------------------------------------
// optional per-stage event markers (hit3d_gpu_step_profile)
// ---------------------------------------------------------------------------
struct Prof {
    static constexpr int MAXM = 64;
    cudaEvent_t ev[MAXM];
    int stage[MAXM];
    int n = 0;
    void mark(cudaStream_t st, int s)
    {
        if (n < MAXM) {
            cudaEventRecord(ev[n], st);
            stage[n] = s;
            n++;
        }
    }
};
#define MARK(s) \
    do {        \
        if (prof) prof->mark(c->st, (s)); \
    } while (0)

// launch shape of k_forcing_energy: kFthreads threads loading the candidate
// modes of a band of up to kFsmall shells, else one thread per shell.  Shells
// beyond the largest a grid has (nint(sqrt(3) N/2) + 1) hold no modes and add
// nothing, so the band is cut there.
struct ForcingLaunch {
    int kfmax, threads;
    size_t smem;
};
static ForcingLaunch forcing_launch(int n, int kfmax)
{
    const int shmax = (int)std::lround(std::sqrt(3.0) * (n / 2)) + 1;
    ForcingLaunch f;
    f.kfmax = kfmax < shmax ? kfmax : shmax;
    f.threads = f.kfmax <= kFsmall ? kFthreads : (f.kfmax + 31) / 32 * 32;
    if (f.threads > 1024) f.threads = 1024;
    f.smem = f.kfmax <= kFsmall ? 0 : sizeof(double) * (size_t)f.kfmax;
    return f;
}

// ---------------------------------------------------------------------------
// one time step
// LES-related transported fields (m_les.f90:111-300): k_sgs for the models with
// an algebraic dissipation (2, 4, 6); k_sgs, (B T_B) and (eps T_eps) with the
// lag model (3, 5, 7)
static int les_nles(int model)
{
    return (model == 2 || model == 4 || model == 6) ? 1 : (model == 3 || model == 5 || model == 7) ? 3
                                                                                                : model == 10 ? 2 : 0;
}
static bool les_dlm(int model) { return model == 2 || model == 3; }
static bool les_dstm(int model) { return model >= 4 && model <= 7; }
// work fields of the Dynamic Structure models past the products (k_dstm_phys layout)
static int dstm_fields(int nles) { return (nles == 3 ? 21 : 20) + 3 * nles; }
static constexpr int kM10Fields = 26;  // work fields of les_model 10 (k_m10_phys layout)
static int filter_transfer(hit3d_ctx *c, int kind, double delta);

// ---------------------------------------------------------------------------
// 2/3-rule pruning for the duration of one step (reset on every exit path)
struct PruneScope {
    hit3d_ctx *c;
    explicit PruneScope(hit3d_ctx *cc) : c(cc)
    {
        c->kc_active = (c->prune_on && c->pruned && c->p.dealias == 0) ? c->n / 3 : -1;
    }
    ~PruneScope() { c->kc_active = -1; }
};

// bring `pruned` up to date with the state (one pass over U and RO, only after
// the state changed); never called while a graph is being recorded
static int ensure_alias_state(hit3d_ctx *c)
{
    if (c->alias_known) return 0;
    c->pruned = 0;
    if (c->p.dealias == 0 && c->prune_on) {
        unsigned long long *d = reinterpret_cast<unsigned long long *>(c->d_red);
        H3D_CHECK(cudaMemsetAsync(d, 0, sizeof(unsigned long long), c->st));
        k_alias_max<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, c->fs64, 3 + c->nsc, c->U, c->RO, d);
        H3D_LAUNCH_CHECK();
        unsigned long long bits = 1;
        H3D_CHECK(cudaMemcpyAsync(&bits, d, sizeof bits, cudaMemcpyDeviceToHost, c->st));
        H3D_CHECK(cudaStreamSynchronize(c->st));
        c->pruned = bits == 0;
    }
    c->alias_known = 1;
    return 0;
}

// zin: W[0..2] already hold the z inverse of this state's velocity (written by
// the previous step's fused z pass + update), so the velocity z inverse is
// skipped; zout: have the fused z pass + update write the next step's.  Both
// need the fused path (chain_ok).
template <typename T>
static int step_once(hit3d_ctx *c, int euler_v, int euler_s, Prof *prof = nullptr, bool zin = false, bool zout = false)
{
    PruneScope prune_scope(c);
    const hit3d_params &p = c->p;
    cx<T> *W = reinterpret_cast<cx<T> *>(c->W);
    const int64_t wfs = c->wfs;
    const int wp = c->wpitch;
    auto Wf = [&](int i) { return W + i * wfs; };
    const int ns = c->int_scalars ? c->nsc : 0;
    const int nprod = 6 + 3 * ns;
    const bool les = p.les_model == 1, les_mlp = p.les_model == HIT3D_LES_LEARNED, dlm = les_dlm(p.les_model);
    const bool lag = p.les_model == 3, dstm = les_dstm(p.les_model), m10 = p.les_model == 10;

    StepArgs a;
    memset(&a, 0, sizeof a);
    a.n = c->n; a.nh = c->nh; a.pitch = c->P64; a.ppitch = wp; a.fs = c->fs64; a.pfs = wfs;
    a.nu = p.nu; a.dt = p.dt; a.euler_v = euler_v; a.euler_s = euler_s;
    a.flow_type = p.flow_type; a.kfmax = p.kfmax; a.famp = p.famp; a.fenergy = c->d_fen; a.nscal = ns;
    a.kc = c->kc_active;  // pruned state: the updates visit only the kept modes
    a.idle = c->idle_passive;
    for (int s = 0; s < p.n_scalars; s++) { a.pe[s] = p.nu / p.sc[s]; a.stype[s] = p.scalar_type[s]; }
    for (int j = 0; j < les_nles(p.les_model); j++) {
        // LES fields: Schmidt number one (m_les.f90:372-391), no mean-gradient source
        a.pe[p.n_scalars + j] = p.nu / 1.0;
        a.stype[p.n_scalars + j] = -1;
    }
    // work fields of the LES models after the nprod products (nps passive scalars):
    // model 1 with scalars: [0,6) strain -> tau, [6, 6+3 nps) scalar gradients -> fluxes
    // model 2: [0,6) strain -> tau, [6] k cube -> k source, [7,10) grad k and
    //          [10, 10+3 nps) scalar gradients -> fluxes
    // model 3: [0,6) strain -> tau, [6] (B T_B) -> k source, [7] (eps T_eps) -> B T_B
    //          source, [8,17) gradients of the three and [17, 17+3 nps) scalar
    //          gradients -> fluxes, [17+3 nps] eps T_eps source
    // then, for 2 and 3, k_sgs truncated (kf) and nu_t (nutf)
    // model 10: as k_m10_phys lays out, scalar gradients at [26, 26+3 nps)
    const int nps = p.n_scalars, kf0 = 3 + p.n_scalars;  // kf0: first LES field of the state
    const int kf = nprod + (lag ? 18 : 10) + 3 * nps, nutf = kf + 1;

    MARK(7);
    if constexpr (std::is_same<T, double>::value) {
        if (dlm) {
            // nu_t from k_sgs truncated to |k| <= kmax, clipped at zero; the clipped
            // field replaces the state when its minimum is negative
            // (les_get_turb_visc_dlm, m_les.f90:1313-1388)
            MARK(6);
            double2 *K = c->U + kf0 * c->fs64;
            c->k2max = (double)c->kmax * (double)c->kmax;
            H3D_TRY(zinv<T>(c, 1, PRE_TRUNC, 0, K, c->fs64, Wf(kf), wfs, wp));
            H3D_TRY(spass<T>(c, 1, false, Wf(kf), wfs, wp, 1));
            H3D_TRY(xc2r<T>(c, Wf(kf), wfs, wp, 1));
            k_phys_partial<<<c->pblocks, 256, 0, c->st>>>(c->n, 2 * (int64_t)wp, 2 * wfs, 1, 2,
                                                          reinterpret_cast<const double *>(Wf(kf)), c->d_part);
            H3D_LAUNCH_CHECK();
            k_phys_final<<<1, 1, 0, c->st>>>(c->pblocks, c->d_part, c->d_kmin);
            H3D_LAUNCH_CHECK();
            k_dlm_nut<<<pw_grid(c), 256, 0, c->st>>>(c->n, 2 * (int64_t)wp, 0.1 * c->dx,
                                                     reinterpret_cast<double *>(Wf(kf)),
                                                     reinterpret_cast<double *>(Wf(nutf)));
            H3D_LAUNCH_CHECK();
            H3D_TRY(xr2c<T>(c, Wf(kf), wfs, wp, 1));
            H3D_TRY(spass<T>(c, 1, true, Wf(kf), wfs, wp, 1));
            H3D_TRY(spass<T>(c, 2, true, Wf(kf), wfs, wp, 1));
            k_dlm_commit<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, c->d_kmin + 2,
                                                        reinterpret_cast<const double2 *>(Wf(kf)), K);
            H3D_LAUNCH_CHECK();
            MARK(7);
        }
    }
    if (p.flow_type == 1) {
        const ForcingLaunch fl = forcing_launch(c->n, p.kfmax);
        k_forcing_energy<<<1, fl.threads, fl.smem, c->st>>>(c->n, c->P64, c->fs64, fl.kfmax, c->U, c->d_fen);
        H3D_LAUNCH_CHECK();
    }
    // reaction sources of type-311 scalars, from this state (phase shift only,
    // rhs_scalars.f90:281-303), in the work fields after the products
    int reac_slot[HIT3D_MAX_SCALARS];
    for (int s = 0; s < HIT3D_MAX_SCALARS; s++) reac_slot[s] = -1;
    if (p.dealias == 1 && ns > 0) {
        int j = 0;
        for (int s = 0; s < p.n_scalars; s++) {
            if (p.scalar_type[s] != 311) continue;
            const int slot = nprod + j++;
            reac_slot[s] = slot;
            H3D_TRY(zinv<T>(c, 1, PRE_QUART, 0, c->U + (3 + s) * c->fs64, c->fs64, Wf(slot), wfs, wp));
            H3D_TRY(spass<T>(c, 1, false, Wf(slot), wfs, wp, 1));
            H3D_TRY(xc2r<T>(c, Wf(slot), wfs, wp, 1));
            k_reaction<T><<<pw_grid(c), 256, 0, c->st>>>(c->n, 2 * (int64_t)wp, p.reac_sc[s], c->U + (3 + s) * c->fs64,
                                                          reinterpret_cast<T *>(Wf(slot)));
            H3D_LAUNCH_CHECK();
            H3D_TRY(xr2c<T>(c, Wf(slot), wfs, wp, 1));
            H3D_TRY(spass<T>(c, 1, true, Wf(slot), wfs, wp, 1));
            H3D_TRY(spass<T>(c, 2, true, Wf(slot), wfs, wp, 1));
        }
    }
    const int npass = p.dealias == 1 ? 2 : 1;
    for (int pass = 0; pass < npass; pass++) {
        const int mode = pass == 0 ? PRE_COPY : PRE_SHIFT;
        MARK(0);
        if (!(zin && pass == 0)) H3D_TRY(zinv<T>(c, 3, mode, 0, c->U, c->fs64, Wf(0), wfs, wp));
        for (int s = 0; s < ns; s++)
            H3D_TRY(zinv<T>(c, 1, mode, 0, c->U + (3 + s) * c->fs64, c->fs64, Wf(6 + 3 * s), wfs, wp));
        MARK(1);
        H3D_TRY(spass<T>(c, 1, false, Wf(0), wfs, wp, 3));
        for (int s = 0; s < ns; s++) H3D_TRY(spass<T>(c, 1, false, Wf(6 + 3 * s), wfs, wp, 1));
        MARK(2);
        if (pass == 0) H3D_CHECK(cudaMemsetAsync(c->d_cmax, 0, sizeof(unsigned long long), c->st));
        for (int s = 0; s < ns; s++) {
            FusedArgs fa;
            memset(&fa, 0, sizeof fa);
            fa.in[0] = Wf(0); fa.in[1] = Wf(1); fa.in[2] = Wf(2); fa.in[3] = Wf(6 + 3 * s);
            fa.out[0] = Wf(6 + 3 * s); fa.out[1] = Wf(7 + 3 * s); fa.out[2] = Wf(8 + 3 * s);
            fa.pitch = wp;
            fa.err = c->d_err;
            H3D_TRY((xfused<T, OpScal>(c, fa)));
        }
        {
            FusedArgs fa;
            memset(&fa, 0, sizeof fa);
            for (int f = 0; f < 3; f++) fa.in[f] = Wf(f);
            for (int o = 0; o < 6; o++) fa.out[o] = Wf(o);
            fa.pitch = wp;
            fa.err = c->d_err;
            if (pass == 0) fa.cmax = c->d_cmax;
            if (pass == 0 && c->np > 0) {
                fa.phys = c->phys;
                fa.phys_fs = (int64_t)c->n * c->n * c->n;
                fa.phys_pitch = c->n;
            }
            H3D_TRY((xfused<T, OpVel>(c, fa)));
        }
        if (pass == 0 && c->np > 0) {
            MARK(7);
            PartArgs pa;
            pa.n = c->n; pa.scheme = c->pscheme; pa.np = c->np; pa.dt = p.dt; pa.dx = c->dx;
            pa.U = c->phys; pa.fs = (int64_t)c->n * c->n * c->n; pa.rp = c->n; pa.xyz = c->d_xyz; pa.uvw = c->d_uvw;
            if (c->pfilt) {
                // the velocity filtered with the particle filter, in physical space
                // (particles_move, m_particles.f90:759-766), in FP64
                c->zfilt = c->pfilt;
                const int rc = zinv<double>(c, 3, PRE_FILT, 0, c->U, c->fs64, c->pbuf, c->fs64, c->P64);
                c->zfilt = nullptr;
                H3D_TRY(rc);
                H3D_TRY(spass<double>(c, 1, false, c->pbuf, c->fs64, c->P64, 3));
                H3D_TRY(xc2r<double>(c, c->pbuf, c->fs64, c->P64, 3));
                pa.U = reinterpret_cast<const double *>(c->pbuf);
                pa.fs = 2 * c->fs64;
                pa.rp = 2 * (int64_t)c->P64;
            }
            k_particles<<<particle_blocks(c->np), 256, 0, c->st>>>(pa);
            H3D_LAUNCH_CHECK();
        }
        MARK(3);
        H3D_TRY(spass<T>(c, 1, true, Wf(0), wfs, wp, nprod));
        MARK(4);
        // without LES, the velocity products' z pass runs inside the update
        // kernel (k_zfwd_update); the scalars' products take the plain z pass
        const bool fuse = c->fuse_update && p.dealias == 0 && p.les_model == 0 && c->bruns == 0;
        if (fuse) {
            if (nprod > 6) H3D_TRY(spass<T>(c, 2, true, Wf(6), wfs, wp, nprod - 6));
        } else {
            H3D_TRY(spass<T>(c, 2, true, Wf(0), wfs, wp, nprod));
        }

        const cx<T> *tau = nullptr;
        if (les && ns > 0) {
            MARK(6);
            // Smagorinsky with passive scalars: stress and the scalars' turbulent
            // fluxes nu_t grad(phi) from the physical fields (m_les.f90:1142-1215,
            // 902-1018, 1028-1091)
            const int t0 = nprod, nf = 6 + 3 * ns;
            H3D_TRY(zinv<T>(c, 3, PRE_STRAIN_A, 0, c->U, c->fs64, Wf(t0), wfs, wp));
            H3D_TRY(zinv<T>(c, 3, PRE_STRAIN_B, 0, c->U, c->fs64, Wf(t0 + 3), wfs, wp));
            for (int s = 0; s < ns; s++)
                H3D_TRY(zinv<T>(c, 3, PRE_GRAD, 3 + s, c->U, c->fs64, Wf(t0 + 6 + 3 * s), wfs, wp));
            H3D_TRY(spass<T>(c, 1, false, Wf(t0), wfs, wp, nf));
            H3D_TRY(xc2r<T>(c, Wf(t0), wfs, wp, nf));
            const double cd = p.c_smag * c->dx;
            k_smag_phys<T><<<pw_grid(c), 256, 0, c->st>>>(c->n, 2 * (int64_t)wp, 2 * wfs, cd * cd,
                                                           reinterpret_cast<T *>(Wf(t0)),
                                                           reinterpret_cast<T *>(Wf(t0 + 6)), 3 * ns);
            H3D_LAUNCH_CHECK();
            H3D_TRY(xr2c<T>(c, Wf(t0), wfs, wp, nf));
            H3D_TRY(spass<T>(c, 1, true, Wf(t0), wfs, wp, nf));
            H3D_TRY(spass<T>(c, 2, true, Wf(t0), wfs, wp, nf));
            tau = Wf(t0);
        } else if (les) {
            MARK(6);
            // Smagorinsky stress from the same state (m_les.f90:1142-1215, 902-1018)
            const int t0 = nprod;
            H3D_TRY(zinv<T>(c, 3, PRE_STRAIN_A, 0, c->U, c->fs64, Wf(t0), wfs, wp));
            H3D_TRY(zinv<T>(c, 3, PRE_STRAIN_B, 0, c->U, c->fs64, Wf(t0 + 3), wfs, wp));
            H3D_TRY(spass<T>(c, 1, false, Wf(t0), wfs, wp, 6));
            FusedArgs fa;
            memset(&fa, 0, sizeof fa);
            for (int f = 0; f < 6; f++) { fa.in[f] = Wf(t0 + f); fa.out[f] = Wf(t0 + f); }
            fa.pitch = wp;
            double cd = p.c_smag * c->dx;
            fa.p0 = cd * cd;
            H3D_TRY((xfused<T, OpSmag>(c, fa)));
            H3D_TRY(spass<T>(c, 1, true, Wf(t0), wfs, wp, 6));
            H3D_TRY(spass<T>(c, 2, true, Wf(t0), wfs, wp, 6));
            tau = Wf(t0);
        }
        const cx<T> *les_src = nullptr, *les_flux = nullptr;
        if constexpr (std::is_same<T, double>::value) {
            if (dstm) {
                // Dynamic Structure Model family (les_models 4-7): test-filtered
                // products (of the forward products above) and velocity, the nine
                // velocity gradients, k_sgs and the LES fields in physical space;
                // one kernel forms tau, the sources and the fluxes
                MARK(6);
                const int t0 = nprod, nl = les_nles(p.les_model);
                const bool lagm = nl == 3;
                const int g0 = lagm ? 21 : 20, nfld = dstm_fields(nl);
                H3D_TRY(zinv<T>(c, 6, PRE_FILT, 0, reinterpret_cast<const double2 *>(Wf(0)), wfs, Wf(t0), wfs, wp));
                H3D_TRY(zinv<T>(c, 3, PRE_FILT, 0, c->U, c->fs64, Wf(t0 + 6), wfs, wp));
                for (int i = 0; i < 3; i++)
                    H3D_TRY(zinv<T>(c, 3, PRE_GRAD, i, c->U, c->fs64, Wf(t0 + 9 + 3 * i), wfs, wp));
                H3D_TRY(zinv<T>(c, 1, PRE_COPY, 0, c->U + kf0 * c->fs64, c->fs64, Wf(t0 + 18), wfs, wp));
                if (lagm) H3D_TRY(zinv<T>(c, 2, PRE_COPY, 0, c->U + (kf0 + 1) * c->fs64, c->fs64, Wf(t0 + 19), wfs, wp));
                else H3D_TRY(zinv<T>(c, 1, PRE_CUBE, 0, c->U + kf0 * c->fs64, c->fs64, Wf(t0 + 19), wfs, wp));
                for (int j = 0; j < nl; j++)
                    H3D_TRY(zinv<T>(c, 3, PRE_GRAD, kf0 + j, c->U, c->fs64, Wf(t0 + g0 + 3 * j), wfs, wp));
                H3D_TRY(spass<T>(c, 1, false, Wf(t0), wfs, wp, nfld));
                H3D_TRY(xc2r<T>(c, Wf(t0), wfs, wp, nfld));
                DstmArgs da;
                da.n = c->n; da.rp = 2 * (int64_t)wp; da.fs = 2 * wfs;
                da.lag = lagm; da.mixed = p.les_model >= 6; da.g0 = g0;
                const double cd = p.c_smag * c->dx;
                da.cs2 = cd * cd;
                da.cmix = p.les_model >= 6 ? p.c_mixed : 1.0;
                da.delta = c->dx;
                da.c_t = p.les_model == 5 ? p.c_t : 1.0;
                k_dstm_phys<<<pw_grid(c), 256, 0, c->st>>>(da, reinterpret_cast<double *>(Wf(t0)), c->d_kmin + 8);
                H3D_LAUNCH_CHECK();
                k_dlm_stats<<<1, 32, 0, c->st>>>((int)pw_grid(c).x, 1.0 / ((double)c->n * c->n * c->n),
                                                 c->U + kf0 * c->fs64, c->d_kmin + 8, c->d_kmin + 4);
                H3D_LAUNCH_CHECK();
                H3D_TRY(xr2c<T>(c, Wf(t0), wfs, wp, 6 + nl));
                H3D_TRY(spass<T>(c, 1, true, Wf(t0), wfs, wp, 6 + nl));
                H3D_TRY(spass<T>(c, 2, true, Wf(t0), wfs, wp, 6 + nl));
                H3D_TRY(xr2c<T>(c, Wf(t0 + g0), wfs, wp, 3 * nl));
                H3D_TRY(spass<T>(c, 1, true, Wf(t0 + g0), wfs, wp, 3 * nl));
                H3D_TRY(spass<T>(c, 2, true, Wf(t0 + g0), wfs, wp, 3 * nl));
                tau = Wf(t0);
            } else if (m10) {
                // les_model 10: the stress of the mixed model from (B T_B) + (eps T_eps),
                // the lag-model sources without k_sgs, the turbulent fluxes
                MARK(6);
                const int t0 = nprod;
                H3D_TRY(zinv<T>(c, 6, PRE_FILT, 0, reinterpret_cast<const double2 *>(Wf(0)), wfs, Wf(t0), wfs, wp));
                H3D_TRY(zinv<T>(c, 3, PRE_FILT, 0, c->U, c->fs64, Wf(t0 + 6), wfs, wp));
                for (int i = 0; i < 3; i++)
                    H3D_TRY(zinv<T>(c, 3, PRE_GRAD, i, c->U, c->fs64, Wf(t0 + 9 + 3 * i), wfs, wp));
                H3D_TRY(zinv<T>(c, 2, PRE_COPY, 0, c->U + kf0 * c->fs64, c->fs64, Wf(t0 + 18), wfs, wp));
                for (int j = 0; j < 2; j++)
                    H3D_TRY(zinv<T>(c, 3, PRE_GRAD, kf0 + j, c->U, c->fs64, Wf(t0 + 20 + 3 * j), wfs, wp));
                for (int s = 0; s < nps; s++)
                    H3D_TRY(zinv<T>(c, 3, PRE_GRAD, 3 + s, c->U, c->fs64, Wf(t0 + kM10Fields + 3 * s), wfs, wp));
                H3D_TRY(spass<T>(c, 1, false, Wf(t0), wfs, wp, kM10Fields + 3 * nps));
                H3D_TRY(xc2r<T>(c, Wf(t0), wfs, wp, kM10Fields + 3 * nps));
                DstmArgs da;
                memset(&da, 0, sizeof da);
                da.n = c->n; da.rp = 2 * (int64_t)wp; da.fs = 2 * wfs;
                const double cd = p.c_smag * c->dx;
                da.cs2 = cd * cd;
                da.cmix = p.c_mixed;
                da.delta = c->dx;
                da.nps = nps;
                k_m10_phys<<<pw_grid(c), 256, 0, c->st>>>(da, reinterpret_cast<double *>(Wf(t0)), c->d_kmin + 8);
                H3D_LAUNCH_CHECK();
                k_dlm_stats<<<1, 32, 0, c->st>>>((int)pw_grid(c).x, 1.0 / ((double)c->n * c->n * c->n),
                                                 c->U + kf0 * c->fs64, c->d_kmin + 8, c->d_kmin + 4,
                                                 c->U + (kf0 + 1) * c->fs64);
                H3D_LAUNCH_CHECK();
                H3D_TRY(xr2c<T>(c, Wf(t0), wfs, wp, 8));
                H3D_TRY(spass<T>(c, 1, true, Wf(t0), wfs, wp, 8));
                H3D_TRY(spass<T>(c, 2, true, Wf(t0), wfs, wp, 8));
                H3D_TRY(xr2c<T>(c, Wf(t0 + 20), wfs, wp, 6 + 3 * nps));
                H3D_TRY(spass<T>(c, 1, true, Wf(t0 + 20), wfs, wp, 6 + 3 * nps));
                H3D_TRY(spass<T>(c, 2, true, Wf(t0 + 20), wfs, wp, 6 + 3 * nps));
                tau = Wf(t0);
            } else if (lag) {
                // dynamic localization model with the lag model for the dissipation
                // (les_model 3; m_les.f90:720-724, 1422-1561, 1629-1684, 1041-1091)
                MARK(6);
                const int t0 = nprod;
                H3D_TRY(zinv<T>(c, 3, PRE_STRAIN_A, 0, c->U, c->fs64, Wf(t0), wfs, wp));
                H3D_TRY(zinv<T>(c, 3, PRE_STRAIN_B, 0, c->U, c->fs64, Wf(t0 + 3), wfs, wp));
                const int ninv = 17 + 3 * nps;
                H3D_TRY(zinv<T>(c, 2, PRE_COPY, 0, c->U + (kf0 + 1) * c->fs64, c->fs64, Wf(t0 + 6), wfs, wp));
                for (int j = 0; j < 3; j++)
                    H3D_TRY(zinv<T>(c, 3, PRE_GRAD, kf0 + j, c->U, c->fs64, Wf(t0 + 8 + 3 * j), wfs, wp));
                for (int s = 0; s < nps; s++)
                    H3D_TRY(zinv<T>(c, 3, PRE_GRAD, 3 + s, c->U, c->fs64, Wf(t0 + 17 + 3 * s), wfs, wp));
                H3D_TRY(spass<T>(c, 1, false, Wf(t0), wfs, wp, ninv));
                H3D_TRY(xc2r<T>(c, Wf(t0), wfs, wp, ninv));
                k_dll_phys<<<pw_grid(c), 256, 0, c->st>>>(
                    c->n, 2 * (int64_t)wp, 2 * wfs, c->dx, 1.0, reinterpret_cast<const double *>(Wf(nutf)),
                    reinterpret_cast<double *>(Wf(t0)), reinterpret_cast<double *>(Wf(t0 + 6)),
                    reinterpret_cast<double *>(Wf(t0 + 7)), reinterpret_cast<double *>(Wf(t0 + 8)), 9 + 3 * nps,
                    reinterpret_cast<double *>(Wf(t0 + ninv)), c->d_kmin + 8);
                H3D_LAUNCH_CHECK();
                k_dlm_stats<<<1, 32, 0, c->st>>>((int)pw_grid(c).x, 1.0 / ((double)c->n * c->n * c->n),
                                                 c->U + kf0 * c->fs64, c->d_kmin + 8, c->d_kmin + 4);
                H3D_LAUNCH_CHECK();
                H3D_TRY(xr2c<T>(c, Wf(t0), wfs, wp, ninv + 1));
                H3D_TRY(spass<T>(c, 1, true, Wf(t0), wfs, wp, ninv + 1));
                H3D_TRY(spass<T>(c, 2, true, Wf(t0), wfs, wp, ninv + 1));
                tau = Wf(t0);
            } else if (dlm) {
                // dynamic localization model: tau = -2 nu_t S for the velocities, and
                // for k_sgs the production 2 nu_t S:S, the dissipation k^(3/2)/Delta
                // and the turbulent fluxes nu_t dk/dx_i (m_les.f90:902-1018,
                // 1422-1621, 1041-1091), all from the physical fields of this state
                MARK(6);
                const int t0 = nprod;
                H3D_TRY(zinv<T>(c, 3, PRE_STRAIN_A, 0, c->U, c->fs64, Wf(t0), wfs, wp));
                H3D_TRY(zinv<T>(c, 3, PRE_STRAIN_B, 0, c->U, c->fs64, Wf(t0 + 3), wfs, wp));
                const int nall = 10 + 3 * nps;
                H3D_TRY(zinv<T>(c, 1, PRE_CUBE, 0, c->U + kf0 * c->fs64, c->fs64, Wf(t0 + 6), wfs, wp));
                H3D_TRY(zinv<T>(c, 3, PRE_GRAD, kf0, c->U, c->fs64, Wf(t0 + 7), wfs, wp));
                for (int s = 0; s < nps; s++)
                    H3D_TRY(zinv<T>(c, 3, PRE_GRAD, 3 + s, c->U, c->fs64, Wf(t0 + 10 + 3 * s), wfs, wp));
                H3D_TRY(spass<T>(c, 1, false, Wf(t0), wfs, wp, nall));
                H3D_TRY(xc2r<T>(c, Wf(t0), wfs, wp, nall));
                k_dlm_phys<<<pw_grid(c), 256, 0, c->st>>>(
                    c->n, 2 * (int64_t)wp, 2 * wfs, c->dx, reinterpret_cast<const double *>(Wf(nutf)),
                    reinterpret_cast<double *>(Wf(t0)), reinterpret_cast<double *>(Wf(t0 + 6)),
                    reinterpret_cast<double *>(Wf(t0 + 7)), 3 + 3 * nps, c->d_kmin + 8);
                H3D_LAUNCH_CHECK();
                k_dlm_stats<<<1, 32, 0, c->st>>>((int)pw_grid(c).x, 1.0 / ((double)c->n * c->n * c->n),
                                                 c->U + kf0 * c->fs64, c->d_kmin + 8, c->d_kmin + 4);
                H3D_LAUNCH_CHECK();
                H3D_TRY(xr2c<T>(c, Wf(t0), wfs, wp, nall));
                H3D_TRY(spass<T>(c, 1, true, Wf(t0), wfs, wp, nall));
                H3D_TRY(spass<T>(c, 2, true, Wf(t0), wfs, wp, nall));
                tau = Wf(t0);
                les_src = Wf(t0 + 6);
                les_flux = Wf(t0 + 7);
            }
        }
        if (les_mlp) {
            MARK(6);
            // learned closure: the nine velocity gradients in physical space, the
            // network per point, the six stresses back to spectral space
            const int t0 = nprod;
            for (int i = 0; i < 3; i++) H3D_TRY(zinv<T>(c, 3, PRE_GRAD, i, c->U, c->fs64, Wf(t0 + 3 * i), wfs, wp));
            H3D_TRY(spass<T>(c, 1, false, Wf(t0), wfs, wp, 9));
            H3D_TRY(xc2r<T>(c, Wf(t0), wfs, wp, 9));
            H3D_TRY(h3d_mlp_apply(c->st, sizeof(T) == 8, (int64_t)c->n * c->n * c->n, c->n, 2 * (int64_t)wp, 2 * wfs,
                                  c->mlp_delta, c->mlp_clip, c->mlp_kernel, c->mlp_wb, Wf(t0), c->d_mlp_err));
            c->nlaunch++;
            H3D_TRY(xr2c<T>(c, Wf(t0), wfs, wp, 6));
            H3D_TRY(spass<T>(c, 1, true, Wf(t0), wfs, wp, 6));
            H3D_TRY(spass<T>(c, 2, true, Wf(t0), wfs, wp, 6));
            tau = Wf(t0);
        }

        MARK(5);
        if (p.dealias == 0) {
            for (int s = 0; s < ns; s++) {
                // sources and turbulent fluxes of the LES fields (layout above)
                // (passive scalars: j < 0, their turbulent or Harlow fluxes only)
                const int j = s - p.n_scalars;
                const cx<T> *src = nullptr, *flux = nullptr;
                if (m10) {
                    if (j >= 0) { src = Wf(nprod + 6 + j); flux = Wf(nprod + 20 + 3 * j); }
                    else flux = Wf(nprod + kM10Fields + 3 * s);
                } else if (dstm && j >= 0) {
                    src = Wf(nprod + 6 + j);
                    flux = Wf(nprod + (les_nles(p.les_model) == 3 ? 21 : 20) + 3 * j);
                } else if (lag) {
                    if (j >= 0) { src = Wf(nprod + (j == 0 ? 6 : j == 1 ? 7 : 17 + 3 * nps)); flux = Wf(nprod + 8 + 3 * j); }
                    else flux = Wf(nprod + 17 + 3 * s);
                } else if (dlm) {
                    if (j == 0) { src = les_src; flux = les_flux; }
                    else flux = Wf(nprod + 10 + 3 * s);
                } else if (les) {
                    flux = Wf(nprod + 6 + 3 * s);
                }
                k_scalar<T><<<pw_grid(c, k_scalar<T>), 256, 0, c->st>>>(a, 0, s, c->dx, Wf(6 + 3 * s), nullptr, c->U,
                                                            c->U + (3 + s) * c->fs64, c->RO + (3 + s) * c->fs64,
                                                            src, flux);
                H3D_LAUNCH_CHECK();
            }
            if (fuse) {
                H3D_TRY(zfwd_update<T>(c, a, Wf(0), zout));
            } else {
                k_update_vel_23<T><<<pw_grid(c, k_update_vel_23<T>), 256, 0, c->st>>>(a, Wf(0), tau, c->U, c->RO);
                H3D_LAUNCH_CHECK();
            }
        } else if (pass == 0) {
            for (int s = 0; s < ns; s++) {
                k_scalar<T><<<pw_grid(c, k_scalar<T>), 256, 0, c->st>>>(a, 1, s, c->dx, Wf(6 + 3 * s), c->SP + s * c->fs64, c->U,
                                                            c->U + (3 + s) * c->fs64, c->RO + (3 + s) * c->fs64);
                H3D_LAUNCH_CHECK();
            }
            k_rhs_vel_ps1<T><<<pw_grid(c, k_rhs_vel_ps1<T>), 256, 0, c->st>>>(a, Wf(0), c->U, c->RP);
            H3D_LAUNCH_CHECK();
        } else {
            for (int s = 0; s < ns; s++) {
                const cx<T> *rs = (s < p.n_scalars && reac_slot[s] >= 0) ? Wf(reac_slot[s]) : nullptr;
                k_scalar<T><<<pw_grid(c, k_scalar<T>), 256, 0, c->st>>>(a, 2, s, c->dx, Wf(6 + 3 * s), c->SP + s * c->fs64, c->U,
                                                            c->U + (3 + s) * c->fs64, c->RO + (3 + s) * c->fs64,
                                                            nullptr, nullptr, rs);
                H3D_LAUNCH_CHECK();
            }
            k_update_vel_ps2<T><<<pw_grid(c, k_update_vel_ps2<T>), 256, 0, c->st>>>(a, c->dx, Wf(0), c->RP, c->U, c->RO);
            H3D_LAUNCH_CHECK();
        }
    }
    MARK(7);
    return 0;
}


// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
static int ctx_alloc(void **p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return h3d_set_error(e, "cudaMalloc", __FILE__, __LINE__);
    return 0;
}

// Context set-up.  ext_U/ext_RO/ext_W (all three or none): state, AB2 history
// and work fields borrowed from a batch's slab instead of allocated here (the
// context does not free them).
static int ctx_init(const hit3d_params *p, hit3d_ctx **out, double2 *ext_U, double2 *ext_RO, void *ext_W);

extern "C" int hit3d_gpu_init(const hit3d_params *p, hit3d_ctx **out)
{
    return ctx_init(p, out, nullptr, nullptr, nullptr);
}

static int ctx_init(const hit3d_params *p, hit3d_ctx **out, double2 *ext_U, double2 *ext_RO, void *ext_W)
{
    if (!p || !out) return h3d_set_error_msg(-1, "hit3d_gpu_init: null argument");
    *out = nullptr;
    if (!size_supported(p->nx)) return h3d_set_error_msg(-3, "hit3d_gpu_init: grid size must be 32, 48, 64, 128, 256, 512 or 1024");
    if (p->n_scalars < 0 || p->n_scalars > HIT3D_MAX_SCALARS) return h3d_set_error_msg(-1, "hit3d_gpu_init: bad n_scalars");
    if (p->dealias != 0 && p->dealias != 1) return h3d_set_error_msg(-1, "hit3d_gpu_init: wrong dealias flag");
    if (p->flow_type == 1 && p->force_type != 1) return h3d_set_error_msg(-1, "hit3d_gpu_init: WRONG FORCE TYPE");
    if (p->flow_type == 1 && p->kfmax < 1) return h3d_set_error_msg(-1, "hit3d_gpu_init: kfmax must be at least 1");
    if (!(p->les_model >= 0 && p->les_model <= 7) && p->les_model != 10 && p->les_model != HIT3D_LES_LEARNED)
        return h3d_set_error_msg(-1, "hit3d_gpu_init: les_model must be 0 (none), 1 (Smagorinsky), 2-3 (dynamic "
                                     "localization), 4-7 (dynamic structure, mixed), 10 (one-equation mixed) or 20 "
                                     "(learned closure)");
    if (les_nles(p->les_model) > 0 && p->precision != 0)
        return h3d_set_error_msg(-1, "hit3d_gpu_init: the LES models with transported fields (les_model 2-7, 10) run "
                                     "with FP64 transforms");
    if (p->les_model == 10 && !(p->c_mixed >= 0.0))
        return h3d_set_error_msg(-1, "hit3d_gpu_init: les_model 10 needs C_mixed >= 0 (c_mixed.in, default 0.5)");
    if (p->les_model == 5 && !(p->c_t > 0.0))
        return h3d_set_error_msg(-1, "hit3d_gpu_init: les_model 5 needs C_T > 0 (the reference reads it from c_t.in)");
    if ((p->les_model == 6 || p->les_model == 7) && !(p->c_mixed > 0.0))
        return h3d_set_error_msg(-1, "hit3d_gpu_init: les_models 6 and 7 need C_mixed > 0 (the reference reads it "
                                     "from c_mixed.in)");
    // passive scalars with LES: turbulent diffusion (les_models 1-3,
    // m_les.f90:1028-1036) or Harlow fluxes (10); the reference stops on
    // scalars with les_models 4-7 (m_les.f90:725-800)
    if (p->n_scalars > 0 && ((p->les_model >= 4 && p->les_model <= 7) || p->les_model == HIT3D_LES_LEARNED))
        return h3d_set_error_msg(-1, "hit3d_gpu_init: passive scalars are not transported with les_model 4-7 or "
                                     "20 (the reference cannot transport scalars with the dynamic structure models)");
    if (p->precision != 0 && p->precision != 1) return h3d_set_error_msg(-1, "hit3d_gpu_init: precision must be 0 or 1");
    for (int s = 0; s < p->n_scalars; s++) {
        // types above 300 carry a reaction; only 311 has one (rhs_scalars.f90:281-303)
        if (p->scalar_type[s] > 300 && p->scalar_type[s] != 311)
            return h3d_set_error_msg(-1, "hit3d_gpu_init: The scalar type has a reaction rate that is not supported yet");
        if (!(p->sc[s] > 0.0)) return h3d_set_error_msg(-1, "hit3d_gpu_init: Schmidt numbers must be > 0");
    }
    H3D_CHECK(cudaSetDevice(p->device));
    hit3d_ctx *c = new hit3d_ctx();
    memset(c, 0, sizeof *c);
    c->rng = Randu();
    c->p = *p;
    if (c->p.dealias == 1 && c->p.les_model) c->p.dealias = 0;  // LES forces the 2/3 rule (m_parameters.f90:416-420)
    c->dev = p->device;
    c->n = p->nx;
    c->nh = c->n / 2 + 1;
    c->P64 = (int)round_up(c->nh, 8);
    c->P32 = (int)round_up(c->nh, 16);
    c->fs64 = (int64_t)c->n * c->n * c->P64;
    c->fs32 = (int64_t)c->n * c->n * c->P32;
    // transported fields beyond velocity: passive scalars, then the LES fields
    c->nsc = p->n_scalars + les_nles(p->les_model);
    c->kmax = c->p.dealias == 0 ? c->n / 3 : (int)floor((double)c->n / 3.0 * sqrt(2.0));
    c->dx = 2.0 * (4.0 * atan(1.0)) / (double)c->n;
    c->int_scalars = c->nsc > 0;
    c->xcfg = 4;  // register-resident fused x pass, the tuner's usual pick
    c->fuse_update = 0;  // the separate z pass + update measured faster so far
    // a clipped k_sgs brings modes beyond N/3 into the state; the LES fields keep
    // the unpruned transforms throughout
    c->prune_on = les_nles(p->les_model) == 0;
    c->kc_active = -1;
    cudaDeviceProp prop;
    H3D_CHECK(cudaGetDeviceProperties(&prop, c->dev));
    c->nsm = prop.multiProcessorCount;
    H3D_CHECK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    int rc = 0;
    const int nf = 3 + c->nsc;
    const size_t f64 = (size_t)c->fs64 * sizeof(double2);
    int nreac = 0;  // type-311 scalars: one work field each for the reaction source (phase shift)
    for (int s = 0; s < p->n_scalars; s++) nreac += (c->p.dealias == 1 && p->scalar_type[s] == 311) ? 1 : 0;
    c->nw = 6 + 3 * c->nsc + nreac +
            (c->p.les_model == 1 ? 6 + 3 * p->n_scalars : c->p.les_model == HIT3D_LES_LEARNED ? 9
                                                                               : c->p.les_model == 2 ? 12 + 3 * p->n_scalars
                                                                               : c->p.les_model == 3 ? 20 + 3 * p->n_scalars
                                                                               : les_dstm(c->p.les_model)
                                                                                   ? dstm_fields(les_nles(c->p.les_model))
                                                                               : c->p.les_model == 10
                                                                                   ? kM10Fields + 3 * p->n_scalars
                                                                                   : 0);
    if (c->p.precision == 0) {
        c->wpitch = c->P64;
        c->wfs = c->fs64;
    } else {
        c->wpitch = c->P32;
        c->wfs = c->fs32;
    }
    const size_t wbytes = (size_t)c->nw * c->wfs * (c->p.precision == 0 ? sizeof(double2) : sizeof(float2));
    if (ext_U) {
        c->U = ext_U;
        c->RO = ext_RO;
        c->W = ext_W;
        c->ext_bufs = 1;
    } else if ((rc = ctx_alloc((void **)&c->U, f64 * nf)) || (rc = ctx_alloc((void **)&c->RO, f64 * nf)) ||
               (rc = ctx_alloc(&c->W, wbytes))) {
        hit3d_gpu_finalize(c);
        return rc;
    }
    if (c->p.dealias == 1) {
        if ((rc = ctx_alloc((void **)&c->RP, f64 * 3)) || (c->nsc && (rc = ctx_alloc((void **)&c->SP, f64 * c->nsc)))) {
            hit3d_gpu_finalize(c);
            return rc;
        }
    }
    if (c->p.precision == 0) c->W64 = reinterpret_cast<double2 *>(c->W);
    else if ((rc = ctx_alloc((void **)&c->W64, f64 * 3))) { hit3d_gpu_finalize(c); return rc; }
    c->pblocks = c->nsm * 2;
    const int kpart = c->kmax > 4 ? c->kmax : 4;
    if ((rc = ctx_alloc((void **)&c->tw64, sizeof(double2) * c->n)) || (rc = ctx_alloc((void **)&c->tw32, sizeof(float2) * c->n)) ||
        (rc = ctx_alloc((void **)&c->d_fen, sizeof(double))) || (rc = ctx_alloc((void **)&c->d_cmax, 2 * sizeof(unsigned long long))) ||
        (rc = ctx_alloc((void **)&c->d_part, sizeof(double) * (size_t)c->pblocks * kpart)) ||
        (rc = ctx_alloc((void **)&c->d_red, sizeof(double) * (size_t)(kpart + 8))) ||
        (rc = ctx_alloc((void **)&c->d_ratio, sizeof(double) * (size_t)kpart)) ||
        (rc = ctx_alloc((void **)&c->stage, sizeof(double2) * (size_t)c->n * c->n * c->nh))) {
        hit3d_gpu_finalize(c);
        return rc;
    }
    c->d_err = reinterpret_cast<int *>(c->d_cmax + 1);
    H3D_CHECK(cudaMemset(c->d_cmax, 0, 2 * sizeof(unsigned long long)));
    // twiddles exp(-2 pi i t/N), computed in long double and rounded once
    std::vector<double2> t64(c->n);
    std::vector<float2> t32(c->n);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int t = 0; t < c->n; t++) {
        long double ang = twopi * (long double)t / (long double)c->n;
        t64[t] = make_double2((double)cosl(ang), (double)(-sinl(ang)));
        t32[t] = make_float2((float)cosl(ang), (float)(-sinl(ang)));
    }
    H3D_CHECK(cudaMemcpy(c->tw64, t64.data(), sizeof(double2) * c->n, cudaMemcpyHostToDevice));
    H3D_CHECK(cudaMemcpy(c->tw32, t32.data(), sizeof(float2) * c->n, cudaMemcpyHostToDevice));
    H3D_CHECK(cudaMemset(c->U, 0, f64 * nf));
    H3D_CHECK(cudaMemset(c->RO, 0, f64 * nf));
    H3D_CHECK(cudaMemset(c->W, 0, wbytes));
    if (les_nles(c->p.les_model) > 0) {
        // [2] the minimum of k_sgs, [4..8) the les.gp means, [8..) block partial sums
        if ((rc = ctx_alloc((void **)&c->d_kmin, sizeof(double) * (8 + 3 * (size_t)pw_grid(c).x)))) {
            hit3d_gpu_finalize(c);
            return rc;
        }
        H3D_CHECK(cudaMemset(c->d_kmin, 0, sizeof(double) * 8));
        // m_les_dlm_k_init (m_les.f90:1394-1413): k_sgs = 0.1 in physical space, so
        // only the (0,0,0) mode, 0.1 N^3 after the unnormalised transform
        // m_les_begin (m_les.f90:430-570): k_sgs = 0.2 for les_model 4, 0.5 for
        // 5-7; with the lag model (B T_B) = (eps T_eps) = 0.5 k_sgs (3), or
        // (B T_B) = k_sgs and (eps T_eps) = 0 (5, 7)
        // les_model 10: (B T_B) = (eps T_eps) = 0.1, no k_sgs field (m_les.f90:592-608)
        const int m = c->p.les_model;
        const double n3 = (double)c->n * (double)c->n * (double)c->n;
        const double2 k0 = make_double2((m <= 3 || m == 10 ? 0.1 : m == 4 ? 0.2 : 0.5) * n3, 0.0);
        const int kf0 = 3 + c->p.n_scalars;  // first LES field of the state
        H3D_CHECK(cudaMemcpy(c->U + kf0 * c->fs64, &k0, sizeof k0, cudaMemcpyHostToDevice));
        if (m == 10) H3D_CHECK(cudaMemcpy(c->U + (kf0 + 1) * c->fs64, &k0, sizeof k0, cudaMemcpyHostToDevice));
        if (les_nles(m) == 3) {
            const double2 b0 = make_double2(m == 3 ? 0.5 * k0.x : k0.x, 0.0);
            const double2 e0 = make_double2(m == 3 ? 0.5 * k0.x : 0.0, 0.0);
            H3D_CHECK(cudaMemcpy(c->U + (kf0 + 1) * c->fs64, &b0, sizeof b0, cudaMemcpyHostToDevice));
            H3D_CHECK(cudaMemcpy(c->U + (kf0 + 2) * c->fs64, &e0, sizeof e0, cudaMemcpyHostToDevice));
        }
        if (les_dstm(m) || m == 10) {
            // the test filter: Gaussian of width 4 dx (m_filter_xfftw.f90:140-150, 197-220)
            if ((rc = ctx_alloc((void **)&c->gfilt, sizeof(double2) * (size_t)c->fs64))) {
                hit3d_gpu_finalize(c);
                return rc;
            }
            if ((rc = filter_transfer(c, 2, 4.0 * c->dx))) {
                hit3d_gpu_finalize(c);
                return rc;
            }
            H3D_CHECK(cudaMemcpyAsync(c->gfilt, c->W64, sizeof(double2) * (size_t)c->fs64, cudaMemcpyDeviceToDevice,
                                      c->st));
            H3D_CHECK(cudaStreamSynchronize(c->st));
        }
    }
    *out = c;
    return 0;
}

extern "C" void hit3d_gpu_finalize(hit3d_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->dev);
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->W64 && c->W64 != c->W) cudaFree(c->W64);
    if (c->ext_bufs) c->U = c->RO = nullptr, c->W = nullptr;  // a batch's slab
    if (c->cs_h2d) {
        cudaStreamSynchronize(c->cs_h2d);
        cudaStreamSynchronize(c->cs_d2h);
        for (int q = 0; q < kCopyStreams - 1; q++) {
            cudaStreamSynchronize(c->cs_up[q]);
            cudaStreamSynchronize(c->cs_dn[q]);
            cudaStreamDestroy(c->cs_up[q]);
            cudaStreamDestroy(c->cs_dn[q]);
            cudaEventDestroy(c->ev_up[q]);
            cudaEventDestroy(c->ev_dn[q]);
        }
        cudaStreamDestroy(c->cs_h2d);
        cudaStreamDestroy(c->cs_d2h);
        cudaEventDestroy(c->ev_in_ready);
        cudaEventDestroy(c->ev_in_free);
        cudaEventDestroy(c->ev_out_ready);
        cudaEventDestroy(c->ev_out_free[0]);
        cudaEventDestroy(c->ev_out_free[1]);
    }
    if (c->sin) cudaFree(c->sin);
    if (c->sout[0]) cudaFree(c->sout[0]);
    if (c->sout[1]) cudaFree(c->sout[1]);
    void *ptrs[] = {c->U, c->RO, c->RP, c->SP, c->W, c->phys, c->tw64, c->tw32, c->d_fen, c->d_part,
                    c->d_red, c->d_ratio, c->d_cmax, c->stage, c->d_xyz, c->d_uvw, c->sgs, c->mlp_wb,
                    c->d_mlp_err, c->d_kmin, c->gfilt, c->pfilt, c->pbuf};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
}

static int transfer_fields(hit3d_ctx *c, double2 *dev, const double *hsrc, double *hdst, int64_t ld1, int nf)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    if (ld1 < c->n + 2) return h3d_set_error_msg(-1, "ld1 must be >= nx+2");
    if (nf < 1 || nf > 3 + c->nsc) return h3d_set_error_msg(-1, "nfields out of range");
    H3D_CHECK(cudaSetDevice(c->dev));
    const size_t width = (size_t)c->nh * sizeof(double2);
    const size_t hp = (size_t)ld1 * sizeof(double);
    const size_t rows = (size_t)c->n * c->n;
    if (hsrc) c->alias_known = 0;
    for (int f = 0; f < nf; f++) {
        double2 *d = dev + f * c->fs64;
        if (hsrc) {
            const double *h = hsrc + (size_t)f * ld1 * rows;
            // ld1 = nx+2 makes a field one contiguous block: one linear copy, which
            // runs at the full host-to-device rate where the pitched copy does not
            if (hp == width)
                H3D_CHECK(cudaMemcpyAsync(c->stage, h, width * rows, cudaMemcpyHostToDevice, c->st));
            else
                H3D_CHECK(cudaMemcpy2DAsync(c->stage, width, h, hp, width, rows, cudaMemcpyHostToDevice, c->st));
            k_ref_to_dev<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, c->stage, d);
            H3D_LAUNCH_CHECK();
        } else {
            double *h = hdst + (size_t)f * ld1 * rows;
            k_dev_to_ref<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, d, c->stage);
            H3D_LAUNCH_CHECK();
            if (hp == width)
                H3D_CHECK(cudaMemcpyAsync(h, c->stage, width * rows, cudaMemcpyDeviceToHost, c->st));
            else
                H3D_CHECK(cudaMemcpy2DAsync(h, hp, c->stage, width, width, rows, cudaMemcpyDeviceToHost, c->st));
        }
    }
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

extern "C" int hit3d_gpu_upload_fields(hit3d_ctx *c, const double *fields, int64_t ld1, int32_t nf)
{
    if (!fields) return h3d_set_error_msg(-1, "null fields");
    return transfer_fields(c, c ? c->U : nullptr, fields, nullptr, ld1, nf);
}
extern "C" int hit3d_gpu_download_fields(hit3d_ctx *c, double *fields, int64_t ld1, int32_t nf)
{
    if (!fields) return h3d_set_error_msg(-1, "null fields");
    return transfer_fields(c, c ? c->U : nullptr, nullptr, fields, ld1, nf);
}
extern "C" int hit3d_gpu_upload_rhs_old(hit3d_ctx *c, const double *r, int64_t ld1, int32_t nf)
{
    if (!r) return h3d_set_error_msg(-1, "null rhs_old");
    return transfer_fields(c, c ? c->RO : nullptr, r, nullptr, ld1, nf);
}
extern "C" int hit3d_gpu_download_rhs_old(hit3d_ctx *c, double *r, int64_t ld1, int32_t nf)
{
    if (!r) return h3d_set_error_msg(-1, "null rhs_old");
    return transfer_fields(c, c ? c->RO : nullptr, nullptr, r, ld1, nf);
}

// streams, staging fields and events of hit3d_gpu_step_host, on first use
static int io_setup(hit3d_ctx *c, int nf)
{
    if (!c->cs_h2d) {
        H3D_CHECK(cudaStreamCreateWithFlags(&c->cs_h2d, cudaStreamNonBlocking));
        H3D_CHECK(cudaStreamCreateWithFlags(&c->cs_d2h, cudaStreamNonBlocking));
        for (int q = 0; q < kCopyStreams - 1; q++) {
            H3D_CHECK(cudaStreamCreateWithFlags(&c->cs_up[q], cudaStreamNonBlocking));
            H3D_CHECK(cudaStreamCreateWithFlags(&c->cs_dn[q], cudaStreamNonBlocking));
            H3D_CHECK(cudaEventCreateWithFlags(&c->ev_up[q], cudaEventDisableTiming));
            H3D_CHECK(cudaEventCreateWithFlags(&c->ev_dn[q], cudaEventDisableTiming));
        }
        H3D_CHECK(cudaEventCreateWithFlags(&c->ev_in_ready, cudaEventDisableTiming));
        H3D_CHECK(cudaEventCreateWithFlags(&c->ev_in_free, cudaEventDisableTiming));
        H3D_CHECK(cudaEventCreateWithFlags(&c->ev_out_ready, cudaEventDisableTiming));
        H3D_CHECK(cudaEventCreateWithFlags(&c->ev_out_free[0], cudaEventDisableTiming));
        H3D_CHECK(cudaEventCreateWithFlags(&c->ev_out_free[1], cudaEventDisableTiming));
    }
    if (c->nstage_io < nf) {
        H3D_CHECK(cudaStreamSynchronize(c->st));
        H3D_CHECK(cudaStreamSynchronize(c->cs_h2d));
        H3D_CHECK(cudaStreamSynchronize(c->cs_d2h));
        for (int q = 0; q < kCopyStreams - 1; q++) {
            H3D_CHECK(cudaStreamSynchronize(c->cs_up[q]));
            H3D_CHECK(cudaStreamSynchronize(c->cs_dn[q]));
        }
        for (double2 **q : {&c->sin, &c->sout[0], &c->sout[1]}) {
            if (*q) cudaFree(*q);
            *q = nullptr;
        }
        c->nstage_io = 0;
        const size_t fe = (size_t)c->n * c->n * c->nh;
        H3D_TRY(ctx_alloc((void **)&c->sin, sizeof(double2) * fe * nf));
        H3D_TRY(ctx_alloc((void **)&c->sout[0], sizeof(double2) * fe * nf));
        H3D_TRY(ctx_alloc((void **)&c->sout[1], sizeof(double2) * fe * nf));
        c->nstage_io = nf;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// restart image in the reference's file layout (restart_io.f90:240-506)
// ---------------------------------------------------------------------------
static constexpr int64_t kRestartHeader = 36;  // 5 x int32 + 2 x float64

static int restart_nles(const hit3d_ctx *c) { return les_nles(c->p.les_model); }

extern "C" int64_t hit3d_gpu_restart_bytes(hit3d_ctx *c, int32_t nums)
{
    if (!c || nums < 0 || nums > c->p.n_scalars) return -1;
    return kRestartHeader + (int64_t)(3 + nums + restart_nles(c)) * c->n * c->n * c->n * 8;
}

extern "C" int hit3d_gpu_restart_pack(hit3d_ctx *c, int32_t nums, double time, double dt, void *image)
{
    if (!c || !image) return h3d_set_error_msg(-1, "hit3d_gpu_restart_pack: null argument");
    if (nums < 0 || nums > c->p.n_scalars)
        return h3d_set_error_msg(-1, "hit3d_gpu_restart_pack: nums must be 0..n_scalars");
    H3D_CHECK(cudaSetDevice(c->dev));
    const int nles = restart_nles(c);
    unsigned char *img = static_cast<unsigned char *>(image);
    const int32_t hdr[5] = {c->n, c->n, c->n, nums, nles};
    memcpy(img, hdr, sizeof hdr);
    memcpy(img + 20, &time, 8);
    memcpy(img + 28, &dt, 8);
    const size_t body = (size_t)c->n * c->n * c->n * 8;
    // variables in file order: velocity, the nums scalars, the LES fields
    const int nvar = 3 + nums + nles;
    for (int v = 0; v < nvar; v++) {
        const int field = v < 3 + nums ? v : 3 + c->p.n_scalars + (v - 3 - nums);
        k_dev_to_restart<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->P64, c->U + field * c->fs64, c->stage);
        H3D_LAUNCH_CHECK();
        H3D_CHECK(cudaMemcpyAsync(img + kRestartHeader + v * body, c->stage, body, cudaMemcpyDeviceToHost, c->st));
    }
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

extern "C" int hit3d_gpu_restart_unpack(hit3d_ctx *c, const void *image, int64_t bytes, double *time, double *dt,
                                        int32_t *nums_file, int32_t *nles_file)
{
    if (!c || !image) return h3d_set_error_msg(-1, "hit3d_gpu_restart_unpack: null argument");
    if (bytes < kRestartHeader) return h3d_set_error_msg(-1, "hit3d_gpu_restart_unpack: truncated header");
    const unsigned char *img = static_cast<const unsigned char *>(image);
    int32_t hdr[5];
    double t = 0.0, d = 0.0;
    memcpy(hdr, img, sizeof hdr);
    memcpy(&t, img + 20, 8);
    memcpy(&d, img + 28, 8);
    if (hdr[0] != c->n || hdr[1] != c->n || hdr[2] != c->n) {
        char buf[160];
        snprintf(buf, sizeof buf, "hit3d_gpu_restart_unpack: Dimensions are different: input file %d^3, restart file %d %d %d",
                 c->n, hdr[0], hdr[1], hdr[2]);
        return h3d_set_error_msg(-1, buf);
    }
    const int nums = hdr[3], nles = hdr[4];
    if (nums < 0 || nles < 0) return h3d_set_error_msg(-1, "hit3d_gpu_restart_unpack: corrupt header (negative counts)");
    const size_t body = (size_t)c->n * c->n * c->n * 8;
    if ((uint64_t)bytes != (uint64_t)kRestartHeader + (uint64_t)(3 + nums + nles) * body)
        return h3d_set_error_msg(-1, "hit3d_gpu_restart_unpack: size does not match the header");
    H3D_CHECK(cudaSetDevice(c->dev));
    const int ns = c->p.n_scalars, nl = restart_nles(c);
    // the context's fields in order; each from the file or zero
    // (restart_io.f90:408-448: extra scalars in the file are dropped, missing
    // ones start from zero for the caller to initialise)
    for (int f = 0; f < 3 + ns + nl; f++) {
        int64_t v = -1;
        if (f < 3) v = f;
        else if (f < 3 + ns) v = (f - 3) < nums ? f : -1;
        else v = (f - 3 - ns) < nles ? 3 + nums + (f - 3 - ns) : -1;
        double2 *dst = c->U + f * c->fs64;
        if (v < 0) {
            H3D_CHECK(cudaMemsetAsync(dst, 0, sizeof(double2) * (size_t)c->fs64, c->st));
            continue;
        }
        H3D_CHECK(cudaMemcpyAsync(c->stage, img + kRestartHeader + v * body, body, cudaMemcpyHostToDevice, c->st));
        k_restart_to_dev<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->P64, c->stage, dst);
        H3D_LAUNCH_CHECK();
    }
    H3D_CHECK(cudaStreamSynchronize(c->st));
    c->alias_known = 0;
    if (time) *time = t;
    if (dt) *dt = d;
    if (nums_file) *nums_file = nums;
    if (nles_file) *nles_file = nles;
    return 0;
}

extern "C" int hit3d_gpu_step(hit3d_ctx *c, int32_t nsteps, int32_t *fov, int32_t *fos, double *courant);

// the boxes of a field's 2/3-rule band in the reference layout (x = bytes of
// kx <= kc, y = kz, z = ky): kept kz and ky each form two runs of indices
struct BandBox {
    int z0, zb, nz, y0, yb, ny;  // reference-layout start, packed start, count (kz, then ky)
};
static int band_boxes(int n, int kc, BandBox *b)
{
    const int lo[2] = {0, n - kc}, pk[2] = {0, kc + 1}, cnt[2] = {kc + 1, kc};
    int q = 0;
    for (int y = 0; y < 2; y++)
        for (int z = 0; z < 2; z++)
            if (cnt[y] > 0 && cnt[z] > 0) b[q++] = BandBox{lo[z], pk[z], cnt[z], lo[y], pk[y], cnt[y]};
    return q;
}
// one field's band between host memory (row pitch hp bytes, n rows per ky slice)
// and the packed band on the device, as up to four strided box copies, which
// go round the streams s[] (rr counts the boxes issued), so that several copy
// engines of the direction share the rows
static cudaError_t band_copy(int n, int kc, double *host, size_t hp, double2 *packed, bool to_device,
                             const cudaStream_t (&s)[kCopyStreams], int &rr)
{
    BandBox b[4];
    const int nbx = band_boxes(n, kc, b), nb = 2 * kc + 1;
    const size_t w = (size_t)(kc + 1) * sizeof(double2);
    for (int q = 0; q < nbx; q++) {
        cudaMemcpy3DParms m;
        memset(&m, 0, sizeof m);
        cudaPitchedPtr hptr = make_cudaPitchedPtr(host, hp, hp, (size_t)n);
        cudaPitchedPtr dptr = make_cudaPitchedPtr(packed, w, w, (size_t)nb);
        const cudaPos hpos = make_cudaPos(0, (size_t)b[q].z0, (size_t)b[q].y0);
        const cudaPos dpos = make_cudaPos(0, (size_t)b[q].zb, (size_t)b[q].yb);
        if (to_device) { m.srcPtr = hptr; m.srcPos = hpos; m.dstPtr = dptr; m.dstPos = dpos; m.kind = cudaMemcpyHostToDevice; }
        else { m.srcPtr = dptr; m.srcPos = dpos; m.dstPtr = hptr; m.dstPos = hpos; m.kind = cudaMemcpyDeviceToHost; }
        m.extent = make_cudaExtent(w, (size_t)b[q].nz, (size_t)b[q].ny);
        cudaError_t e = cudaMemcpy3DAsync(&m, s[rr++ % kCopyStreams]);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

extern "C" int64_t hit3d_gpu_step_host_bytes(hit3d_ctx *c, int32_t nf, int32_t band_only)
{
    if (!c || nf < 1 || nf > 3 + c->nsc) return -1;
    const int kc = c->n / 3;
    return band_only ? (int64_t)nf * (kc + 1) * (2 * kc + 1) * (2 * kc + 1) * 16
                     : (int64_t)nf * c->n * c->n * c->nh * 16;
}

extern "C" int hit3d_gpu_step_host(hit3d_ctx *c, int32_t nio, const double *const *in, double *const *out, int64_t ld1,
                                   int32_t nf, int32_t nsteps, int32_t *fov, int32_t *fos, int32_t band_only)
{
    if (!c || !in || !out || nio < 1 || nsteps < 0) return h3d_set_error_msg(-1, "hit3d_gpu_step_host: bad arguments");
    if (ld1 < c->n + 2) return h3d_set_error_msg(-1, "ld1 must be >= nx+2");
    if (nf < 1 || nf > 3 + c->nsc) return h3d_set_error_msg(-1, "nfields out of range");
    if (band_only && c->p.dealias != 0)
        return h3d_set_error_msg(-1, "hit3d_gpu_step_host: band-only transfers need the 2/3 rule (dealias 0)");
    for (int i = 0; i < nio; i++)
        if (!in[i] || !out[i]) return h3d_set_error_msg(-1, "hit3d_gpu_step_host: null field array");
    H3D_CHECK(cudaSetDevice(c->dev));
    H3D_TRY(io_setup(c, nf));
    const size_t fe = (size_t)c->n * c->n * c->nh;  // complex elements of one reference-layout field
    const size_t width = (size_t)c->nh * sizeof(double2), hp = (size_t)ld1 * sizeof(double);
    const size_t rows = (size_t)c->n * c->n;
    const int kc = c->n / 3;
    // one field as kCopyStreams row ranges, one per copy stream
    auto copy = [&](void *dst, size_t dp, const void *src, size_t sp, cudaMemcpyKind kind,
                    const cudaStream_t (&s)[kCopyStreams]) {
        for (int q = 0; q < kCopyStreams; q++) {
            const size_t r0 = rows * q / kCopyStreams, r1 = rows * (q + 1) / kCopyStreams;
            char *d = static_cast<char *>(dst) + r0 * dp;
            const char *sr = static_cast<const char *>(src) + r0 * sp;
            cudaError_t e = dp == sp && sp == width ? cudaMemcpyAsync(d, sr, width * (r1 - r0), kind, s[q])
                                                    : cudaMemcpy2DAsync(d, dp, sr, sp, width, r1 - r0, kind, s[q]);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    cudaStream_t up[kCopyStreams], down[kCopyStreams];
    up[0] = c->cs_h2d;
    down[0] = c->cs_d2h;
    for (int q = 1; q < kCopyStreams; q++) { up[q] = c->cs_up[q - 1]; down[q] = c->cs_dn[q - 1]; }
    // every copy stream of a direction waits for `start`; the first then waits
    // for the others, so that an event recorded on it covers the whole transfer
    auto fork = [&](const cudaStream_t (&s)[kCopyStreams], cudaEvent_t start) -> int {
        for (int q = 0; q < kCopyStreams; q++) H3D_CHECK(cudaStreamWaitEvent(s[q], start, 0));
        return 0;
    };
    auto join = [&](const cudaStream_t (&s)[kCopyStreams], cudaEvent_t *ev) -> int {
        for (int q = 1; q < kCopyStreams; q++) {
            H3D_CHECK(cudaEventRecord(ev[q - 1], s[q]));
            H3D_CHECK(cudaStreamWaitEvent(s[0], ev[q - 1], 0));
        }
        return 0;
    };
    auto upload = [&](int i) -> int {  // host in[i] -> sin, on the copy-in streams
        H3D_TRY(fork(up, c->ev_in_free));
        int rr = 0;
        for (int f = 0; f < nf; f++) {
            double *h = const_cast<double *>(in[i]) + (size_t)f * ld1 * rows;
            if (band_only) H3D_CHECK(band_copy(c->n, kc, h, hp, c->sin + f * fe, true, up, rr));
            else H3D_CHECK(copy(c->sin + f * fe, width, h, hp, cudaMemcpyHostToDevice, up));
        }
        H3D_TRY(join(up, c->ev_up));
        H3D_CHECK(cudaEventRecord(c->ev_in_ready, c->cs_h2d));
        return 0;
    };
    // the staging buffers start free
    H3D_CHECK(cudaEventRecord(c->ev_in_free, c->st));
    H3D_CHECK(cudaEventRecord(c->ev_out_free[0], c->st));
    H3D_CHECK(cudaEventRecord(c->ev_out_free[1], c->st));
    H3D_TRY(upload(0));
    int32_t ev = fov ? *fov : 0, es = fos ? *fos : 0;
    for (int i = 0; i < nio; i++) {
        // sin -> the state; then sin is free for the next upload, which runs
        // while this state steps and downloads
        H3D_CHECK(cudaStreamWaitEvent(c->st, c->ev_in_ready, 0));
        for (int f = 0; f < nf; f++) {
            if (band_only) k_band_to_dev<<<pw_grid(c), 256, 0, c->st>>>(c->n, kc, c->P64, c->sin + f * fe, c->U + f * c->fs64);
            else k_ref_to_dev<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, c->sin + f * fe, c->U + f * c->fs64);
            H3D_LAUNCH_CHECK();
        }
        H3D_CHECK(cudaEventRecord(c->ev_in_free, c->st));
        if (i + 1 < nio) H3D_TRY(upload(i + 1));
        c->alias_known = 0;
        H3D_TRY(hit3d_gpu_step(c, nsteps, &ev, &es, nullptr));
        // the state -> output set i % 2 once the download two inputs back has
        // left it, then to the host
        const int ob = i & 1;
        double2 *so = c->sout[ob];
        H3D_CHECK(cudaStreamWaitEvent(c->st, c->ev_out_free[ob], 0));
        for (int f = 0; f < nf; f++) {
            if (band_only) k_dev_to_band<<<pw_grid(c), 256, 0, c->st>>>(c->n, kc, c->P64, c->U + f * c->fs64, so + f * fe);
            else k_dev_to_ref<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, c->U + f * c->fs64, so + f * fe);
            H3D_LAUNCH_CHECK();
        }
        H3D_CHECK(cudaEventRecord(c->ev_out_ready, c->st));
        H3D_TRY(fork(down, c->ev_out_ready));
        int rr = 0;
        for (int f = 0; f < nf; f++) {
            double *h = out[i] + (size_t)f * ld1 * rows;
            if (band_only) H3D_CHECK(band_copy(c->n, kc, h, hp, so + f * fe, false, down, rr));
            else H3D_CHECK(copy(h, hp, so + f * fe, width, cudaMemcpyDeviceToHost, down));
        }
        H3D_TRY(join(down, c->ev_dn));
        H3D_CHECK(cudaEventRecord(c->ev_out_free[ob], c->cs_d2h));
    }
    // the compute stream ends after the last download, so that events recorded
    // on it afterwards time the whole call
    H3D_CHECK(cudaStreamWaitEvent(c->st, c->ev_out_free[(nio - 1) & 1], 0));
    H3D_CHECK(cudaStreamSynchronize(c->st));
    if (fov) *fov = ev;
    if (fos) *fos = es;
    return 0;
}

// steps of one call chain the velocity z inverse through the fused z pass +
// update (every step but the first skips it, every step but the last writes
// the next one's); nothing outside a call sees the difference
static bool chain_ok(const hit3d_ctx *c)
{
    return c->fuse_update && c->p.dealias == 0 && c->p.les_model == 0 && c->bruns == 0;
}

extern "C" int hit3d_gpu_step(hit3d_ctx *c, int32_t nsteps, int32_t *fov, int32_t *fos, double *courant)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    if (nsteps < 0) return h3d_set_error_msg(-1, "nsteps < 0");
    if (c->p.les_model == HIT3D_LES_LEARNED && !c->mlp_wb)
        return h3d_set_error_msg(-1, "hit3d_gpu_step: the learned closure (les_model 20) needs weights (hit3d_gpu_les_set_mlp)");
    H3D_CHECK(cudaSetDevice(c->dev));
    H3D_TRY(ensure_alias_state(c));
    int ev = fov ? (*fov != 0) : 0, es = fos ? (*fos != 0) : 0;
    const bool chain = chain_ok(c);
    for (int it = 0; it < nsteps; it++) {
        const bool zin = chain && it > 0, zout = chain && it + 1 < nsteps;
        int rc = c->p.precision == 0 ? step_once<double>(c, ev, es, nullptr, zin, zout)
                                     : step_once<float>(c, ev, es, nullptr, zin, zout);
        if (rc) return rc;
        ev = 0;
        if (c->int_scalars) es = 0;
    }
    if (fov) *fov = ev;
    if (fos) *fos = es;
    if (c->p.les_model == HIT3D_LES_LEARNED && c->mlp_kernel == 1 && nsteps > 0) {
        int herr = 0;
        H3D_CHECK(cudaMemcpyAsync(&herr, c->d_mlp_err, sizeof herr, cudaMemcpyDeviceToHost, c->st));
        H3D_CHECK(cudaStreamSynchronize(c->st));
        if (herr) return h3d_set_error_msg(-5, "hit3d_gpu_step: a tensor-core completion wait of the closure ran out");
    }
    if (nsteps > 0) {
        // the Courant maximum and the error word in one read
        unsigned long long words[2] = {0, 0};
        H3D_CHECK(cudaMemcpyAsync(words, c->d_cmax, sizeof words, cudaMemcpyDeviceToHost, c->st));
        H3D_CHECK(cudaStreamSynchronize(c->st));
        int derr = 0;
        memcpy(&derr, &words[1], sizeof derr);
        if (derr) return h3d_set_error_msg(-5, "hit3d_gpu_step: a fused x pass gave up waiting for its input rows");
        if (courant) {
            double cm;
            memcpy(&cm, &words[0], sizeof cm);
            *courant = cm * c->p.dt / c->dx;
        }
    }
    H3D_CHECK(cudaGetLastError());
    return 0;
}

extern "C" int hit3d_mlp_nparam(void);
extern "C" int hit3d_gpu_les_set_mlp(hit3d_ctx *c, const uint16_t *wb, int64_t nparam, double delta, int32_t clip,
                                     int32_t kernel)
{
    if (!c || !wb) return h3d_set_error_msg(-1, "hit3d_gpu_les_set_mlp: null argument");
    if (kernel != 0 && kernel != 1) return h3d_set_error_msg(-1, "hit3d_gpu_les_set_mlp: kernel must be 0 or 1");
    if (c->p.les_model != HIT3D_LES_LEARNED)
        return h3d_set_error_msg(-1, "hit3d_gpu_les_set_mlp: the context needs les_model 20 (learned closure)");
    if (nparam != hit3d_mlp_nparam()) return h3d_set_error_msg(-1, "hit3d_gpu_les_set_mlp: wrong parameter count");
    if (!(delta > 0.0)) return h3d_set_error_msg(-1, "hit3d_gpu_les_set_mlp: filter width must be positive");
    H3D_CHECK(cudaSetDevice(c->dev));
    if (!c->mlp_wb) H3D_TRY(ctx_alloc(&c->mlp_wb, sizeof(uint16_t) * (size_t)nparam));
    if (!c->d_mlp_err) H3D_TRY(ctx_alloc((void **)&c->d_mlp_err, sizeof(int)));
    H3D_CHECK(cudaMemsetAsync(c->d_mlp_err, 0, sizeof(int), c->st));
    c->mlp_kernel = kernel;
    H3D_CHECK(cudaMemcpyAsync(c->mlp_wb, wb, sizeof(uint16_t) * (size_t)nparam, cudaMemcpyHostToDevice, c->st));
    H3D_CHECK(cudaStreamSynchronize(c->st));
    c->mlp_delta = delta;
    c->mlp_clip = clip != 0;
    return 0;
}

extern "C" void *hit3d_gpu_stream(hit3d_ctx *c) { return c ? (void *)c->st : nullptr; }
extern "C" int64_t hit3d_gpu_launch_count(hit3d_ctx *c) { return c ? c->nlaunch : -1; }

extern "C" int hit3d_gpu_step_profile(hit3d_ctx *c, int32_t nsteps, int32_t *fov, int32_t *fos, double *ms)
{
    if (!c || !ms) return h3d_set_error_msg(-1, "hit3d_gpu_step_profile: null argument");
    H3D_CHECK(cudaSetDevice(c->dev));
    H3D_TRY(ensure_alias_state(c));
    Prof prof;
    for (int i = 0; i < Prof::MAXM; i++) H3D_CHECK(cudaEventCreate(&prof.ev[i]));
    int ev = fov ? (*fov != 0) : 0, es = fos ? (*fos != 0) : 0;
    int rc = 0;
    const bool chain = chain_ok(c);
    for (int it = 0; it < nsteps && rc == 0; it++) {
        prof.n = 0;
        const bool zin = chain && it > 0, zout = chain && it + 1 < nsteps;
        rc = c->p.precision == 0 ? step_once<double>(c, ev, es, &prof, zin, zout)
                                 : step_once<float>(c, ev, es, &prof, zin, zout);
        if (rc) break;
        ev = 0;
        if (c->int_scalars) es = 0;
        cudaError_t e = cudaEventSynchronize(prof.ev[prof.n - 1]);
        if (e != cudaSuccess) { rc = h3d_set_error(e, "cudaEventSynchronize", __FILE__, __LINE__); break; }
        for (int i = 0; i + 1 < prof.n; i++) {
            float t = 0.f;
            cudaEventElapsedTime(&t, prof.ev[i], prof.ev[i + 1]);
            ms[prof.stage[i]] += t;
        }
    }
    for (int i = 0; i < Prof::MAXM; i++) cudaEventDestroy(prof.ev[i]);
    if (rc) return rc;
    if (fov) *fov = ev;
    if (fos) *fos = es;
    return 0;
}

// a pair of timing events, destroyed on every exit path
struct EventPair {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t create()
    {
        cudaError_t e = cudaEventCreate(&e0);
        return e != cudaSuccess ? e : cudaEventCreate(&e1);
    }
    ~EventPair()
    {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
};

// time one fused x pass (velocity products) in the current variant; W is scratch
template <typename T> static int time_fused(hit3d_ctx *c, float *ms)
{
    PruneScope prune_scope(c);  // time the launch shape the step will use
    cx<T> *W = reinterpret_cast<cx<T> *>(c->W);
    FusedArgs fa;
    memset(&fa, 0, sizeof fa);
    for (int f = 0; f < 3; f++) fa.in[f] = W + f * c->wfs;
    for (int o = 0; o < 6; o++) fa.out[o] = W + o * c->wfs;
    fa.pitch = c->wpitch;
    EventPair ev;
    H3D_CHECK(ev.create());
    H3D_TRY((xfused<T, OpVel>(c, fa)));  // warm-up
    H3D_CHECK(cudaEventRecord(ev.e0, c->st));
    for (int r = 0; r < 3; r++) H3D_TRY((xfused<T, OpVel>(c, fa)));
    H3D_CHECK(cudaEventRecord(ev.e1, c->st));
    H3D_CHECK(cudaEventSynchronize(ev.e1));
    H3D_CHECK(cudaEventElapsedTime(ms, ev.e0, ev.e1));
    return 0;
}

extern "C" int hit3d_gpu_autotune(hit3d_ctx *c, int32_t *variant, double *ms_out)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    H3D_CHECK(cudaSetDevice(c->dev));
    H3D_TRY(ensure_alias_state(c));
    int best = 0;
    float bt = 1e30f;
    for (int v = 0; v < kFusedVariants; v++) {
        c->xcfg = v;
        float ms = 0.f;
        int rc = c->p.precision == 0 ? time_fused<double>(c, &ms) : time_fused<float>(c, &ms);
        if (rc) return rc;
        if (ms_out) ms_out[v] = ms / 3.0;
        if (ms < bt) { bt = ms; best = v; }
    }
    c->xcfg = best;
    if (variant) *variant = best;
    return 0;
}

// time the strided passes of one step (z and y inverse of the velocity, y and z
// forward of the six products) in the current column tile; the state is read,
// only the work fields are written
template <typename T> static int time_columns(hit3d_ctx *c, float *ms)
{
    PruneScope prune_scope(c);
    cx<T> *W = reinterpret_cast<cx<T> *>(c->W);
    const int64_t wfs = c->wfs;
    const int wp = c->wpitch;
    auto go = [&]() -> int {
        H3D_TRY(zinv<T>(c, 3, PRE_COPY, 0, c->U, c->fs64, W, wfs, wp));
        H3D_TRY(spass<T>(c, 1, false, W, wfs, wp, 3));
        H3D_TRY(spass<T>(c, 1, true, W, wfs, wp, 6));
        H3D_TRY(spass<T>(c, 2, true, W, wfs, wp, 6));
        return 0;
    };
    EventPair ev;
    H3D_CHECK(ev.create());
    H3D_TRY(go());  // warm-up
    H3D_CHECK(cudaEventRecord(ev.e0, c->st));
    for (int r = 0; r < 3; r++) H3D_TRY(go());
    H3D_CHECK(cudaEventRecord(ev.e1, c->st));
    H3D_CHECK(cudaEventSynchronize(ev.e1));
    H3D_CHECK(cudaEventElapsedTime(ms, ev.e0, ev.e1));
    *ms /= 3.0f;
    return 0;
}

extern "C" int hit3d_gpu_autotune_columns(hit3d_ctx *c, int32_t *tile, double *ms_out)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    H3D_CHECK(cudaSetDevice(c->dev));
    H3D_TRY(ensure_alias_state(c));
    if (c->nw < 6) return h3d_set_error_msg(-1, "hit3d_gpu_autotune_columns: the context has fewer than six work fields");
    int best = 0;
    float bt = 1e30f;
    for (int ct = 0; ct < kColTiles; ct++) {
        if (ms_out) ms_out[ct] = 0.0;
        if (c->n > 512 && ct > 0 && ct < 3) continue;
        c->ctile = ct;
        float ms = 0.f;
        const int rc = c->p.precision == 0 ? time_columns<double>(c, &ms) : time_columns<float>(c, &ms);
        if (rc) {
            c->ctile = 0;
            return rc;
        }
        if (ms_out) ms_out[ct] = ms;
        if (ms < bt) { bt = ms; best = ct; }
    }
    c->ctile = best;
    if (tile) *tile = best;
    return 0;
}

extern "C" int hit3d_gpu_check_finite(hit3d_ctx *c, int64_t *nonfinite)
{
    if (!c || !nonfinite) return h3d_set_error_msg(-1, "hit3d_gpu_check_finite: null argument");
    H3D_CHECK(cudaSetDevice(c->dev));
    unsigned long long *d = reinterpret_cast<unsigned long long *>(c->d_red);
    H3D_CHECK(cudaMemsetAsync(d, 0, sizeof(unsigned long long), c->st));
    const int nf = 3 + c->nsc;
    k_count_nonfinite<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, c->fs64, nf, c->U, d);
    H3D_LAUNCH_CHECK();
    k_count_nonfinite<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, c->fs64, nf, c->RO, d);
    H3D_LAUNCH_CHECK();
    unsigned long long h = 0;
    H3D_CHECK(cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, c->st));
    H3D_CHECK(cudaStreamSynchronize(c->st));
    *nonfinite = (int64_t)h;
    return 0;
}

extern "C" int hit3d_gpu_les_stats(hit3d_ctx *c, double *out4)
{
    if (!c || !out4) return h3d_set_error_msg(-1, "hit3d_gpu_les_stats: null argument");
    if (les_nles(c->p.les_model) == 0)
        return h3d_set_error_msg(-1, "hit3d_gpu_les_stats: les.gp quantities exist for les_models 2-7 and 10 only");
    H3D_CHECK(cudaSetDevice(c->dev));
    H3D_CHECK(cudaMemcpyAsync(out4, c->d_kmin + 4, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->st));
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

extern "C" int hit3d_gpu_set_update_fusion(hit3d_ctx *c, int32_t on)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    c->fuse_update = on != 0;
    return 0;
}

extern "C" int hit3d_gpu_set_pruning(hit3d_ctx *c, int32_t on)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    c->prune_on = on != 0;
    c->alias_known = 0;
    return 0;
}

extern "C" int hit3d_gpu_pruned(hit3d_ctx *c)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    H3D_CHECK(cudaSetDevice(c->dev));
    H3D_TRY(ensure_alias_state(c));
    return c->pruned ? 1 : 0;
}

extern "C" int hit3d_gpu_set_column_tile(hit3d_ctx *c, int32_t t)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    if (t < 0 || t >= kColTiles || (c->n > 512 && t > 0 && t < 3))
        return h3d_set_error_msg(-1, "hit3d_gpu_set_column_tile: no such column tile for this grid");
    c->ctile = t;
    return 0;
}

extern "C" int hit3d_gpu_set_variant(hit3d_ctx *c, int32_t v)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    if (v < 0 || v >= kFusedVariants) return h3d_set_error_msg(-1, "hit3d_gpu_set_variant: no such variant");
    c->xcfg = v;
    return 0;
}

extern "C" int hit3d_gpu_set_dt(hit3d_ctx *c, double dt)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    if (!(dt > 0.0)) return h3d_set_error_msg(-1, "dt must be > 0");
    c->p.dt = dt;
    return 0;
}

extern "C" int hit3d_gpu_set_scalars_active(hit3d_ctx *c, int32_t on)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    // the LES fields are always transported (rhs_scalars.f90:72-74).  While the
    // passive scalars wait for TSCALAR next to LES fields, the reference still
    // advances them, with a RHS of only the mean-gradient source and the LES
    // fluxes (rhs_scalars.f90:28-36, 384-395, main.f90:132-146)
    c->int_scalars = ((on != 0) && c->nsc > 0) || les_nles(c->p.les_model) > 0;
    c->idle_passive = (on == 0 && les_nles(c->p.les_model) > 0) ? c->p.n_scalars : 0;
    return 0;
}

extern "C" int hit3d_gpu_dealias_all(hit3d_ctx *c)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    H3D_CHECK(cudaSetDevice(c->dev));
    // velocity and passive scalars (dealias_all.f90:27), not k_sgs
    k_dealias_all<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, c->fs64, 3 + c->p.n_scalars, c->kmax, c->U);
    H3D_LAUNCH_CHECK();
    H3D_CHECK(cudaStreamSynchronize(c->st));
    c->alias_known = 0;
    return 0;
}

// shell spectrum of nf state fields starting at src -> host es[0..kmax)
static int shell_spectrum(hit3d_ctx *c, const double2 *src, int nf, double *es, double w0 = 0.5)
{
    const int kmax = c->kmax;
    const int nw = 8;
    k_shell_partial<<<c->pblocks, nw * 32, sizeof(double) * nw * kmax, c->st>>>(c->n, c->nh, c->P64, c->fs64, nf, kmax,
                                                                               w0, src, c->d_part);
    H3D_LAUNCH_CHECK();
    k_shell_final<<<(kmax + 127) / 128, 128, 0, c->st>>>(c->pblocks, kmax, c->d_part, c->d_red);
    H3D_LAUNCH_CHECK();
    H3D_CHECK(cudaMemcpyAsync(es, c->d_red, sizeof(double) * kmax, cudaMemcpyDeviceToHost, c->st));
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

// deterministic sums over physical points of W64 fields: returns 4 values
static int phys_sums(hit3d_ctx *c, const double2 *base, int nf, int mode, double *out4)
{
    k_phys_partial<<<c->pblocks, 256, 0, c->st>>>(c->n, 2 * (int64_t)c->P64, 2 * c->fs64, nf, mode,
                                                  reinterpret_cast<const double *>(base), c->d_part);
    H3D_LAUNCH_CHECK();
    k_phys_final<<<1, 1, 0, c->st>>>(c->pblocks, c->d_part, c->d_red);
    H3D_LAUNCH_CHECK();
    H3D_CHECK(cudaMemcpyAsync(out4, c->d_red, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->st));
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

extern "C" int hit3d_gpu_stats(hit3d_ctx *c, double *e_spec, int32_t kmax, double *o)
{
    if (!c || !e_spec || !o) return h3d_set_error_msg(-1, "hit3d_gpu_stats: null argument");
    if (kmax != c->kmax) return h3d_set_error_msg(-1, "hit3d_gpu_stats: kmax does not match the run");
    H3D_CHECK(cudaSetDevice(c->dev));
    const int n = c->n;
    const double fac = 1.0 / ((double)n * n * n);
    double s4[4];
    // enstrophy (m_stats.f90:241-289)
    H3D_TRY(inv_from_state(c, 3, PRE_CURL, 0, c->U));
    H3D_TRY(phys_sums(c, c->W64, 3, 0, s4));
    const double ens = s4[0] * fac;
    // skewness of the longitudinal derivatives
    H3D_TRY(inv_from_state(c, 3, PRE_DLONG, 0, c->U));
    double skew = 0.0;
    for (int f = 0; f < 3; f++) {
        H3D_TRY(phys_sums(c, c->W64 + f * c->fs64, 1, 1, s4));
        double m2 = s4[0] * fac, m3 = s4[1] * fac;
        skew += m3 / pow(m2, 1.5);
    }
    skew /= 3.0;
    // spectrum and derived quantities (m_stats.f90:99-189), host arithmetic in the reference's order
    H3D_TRY(shell_spectrum(c, c->U, 3, e_spec));
    const double nu = c->p.nu, PI = 4.0 * atan(1.0);
    double energy = 0.0;
    for (int k = 0; k < kmax; k++) energy = energy + e_spec[k];
    double eps = 0.0;
    for (int k = 1; k <= kmax; k++) eps = eps + e_spec[k - 1] * (double)(k * k) * 2.0 * nu;
    double eta = pow(nu * nu * nu / eps, 0.25);
    double uvar = 2.0 / 3.0 * energy;
    double sct = 0.0;
    for (int k = 1; k <= kmax; k++) sct = sct + e_spec[k - 1] / (double)k;
    double xl = PI / 2.0 * sct / uvar;
    double lam = sqrt(15.0 * uvar * nu / eps);
    o[0] = energy; o[1] = eps; o[2] = eta; o[3] = eta * (double)kmax; o[4] = uvar; o[5] = xl; o[6] = lam;
    o[7] = uvar * sqrt(15.0 / eps * (1.0 / nu));
    o[8] = sqrt(uvar) * lam / nu;
    o[9] = xl / sqrt(uvar);
    o[10] = ens;
    o[11] = skew;
    return 0;
}

extern "C" int hit3d_gpu_scalar_stats(hit3d_ctx *c, int32_t s, double *spec, int32_t kmax, double *o)
{
    if (!c || !spec || !o) return h3d_set_error_msg(-1, "hit3d_gpu_scalar_stats: null argument");
    if (s < 0 || s >= c->nsc) return h3d_set_error_msg(-1, "hit3d_gpu_scalar_stats: no such scalar");
    if (kmax != c->kmax) return h3d_set_error_msg(-1, "hit3d_gpu_scalar_stats: kmax does not match the run");
    H3D_CHECK(cudaSetDevice(c->dev));
    const int n = c->n;
    const double fac = 1.0 / ((double)n * n * n);
    const double2 *phi = c->U + (3 + s) * c->fs64;
    H3D_TRY(shell_spectrum(c, phi, 1, spec));
    for (int k = 0; k < kmax; k++) spec[k] = 2.0 * spec[k];
    double s4[4];
    H3D_TRY(inv_from_state(c, 3, PRE_GRAD, 3 + s, c->U));
    H3D_TRY(phys_sums(c, c->W64, 3, 0, s4));
    o[0] = 2.0 * (c->p.nu / c->p.sc[s]) * s4[0] * fac;
    H3D_TRY(inv_from_state(c, 1, PRE_COPY, 0, phi));
    H3D_TRY(phys_sums(c, c->W64, 1, 2, s4));
    double m1 = s4[0] * fac, m2 = s4[1] * fac;
    o[1] = m1; o[2] = m2 - m1 * m1; o[3] = s4[2]; o[4] = s4[3];
    return 0;
}

// upload nf host physical arrays (ld1, ny, nz) into W64 rows
static int upload_phys(hit3d_ctx *c, const double *h, int64_t ld1, int nf)
{
    const size_t rows = (size_t)c->n * c->n;
    for (int f = 0; f < nf; f++)
        H3D_CHECK(cudaMemcpy2DAsync(reinterpret_cast<double *>(c->W64 + f * c->fs64), 2 * c->P64 * sizeof(double),
                                    h + (size_t)f * ld1 * rows, ld1 * sizeof(double), c->n * sizeof(double), rows,
                                    cudaMemcpyHostToDevice, c->st));
    return 0;
}

static int target_spectrum(int isp, double peak, double ir_exp, int kmax, std::vector<double> &et);

extern "C" int hit3d_gpu_init_velocity(hit3d_ctx *c, double rn1, int32_t isp, double peak, double ir_exp)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    if (!(isp == -1 || isp == 0 || isp == 1 || isp == 2 || isp == 3))
        return h3d_set_error_msg(-1, "ERROR: WRONG INITIAL SPECTRUM TYPE");
    H3D_CHECK(cudaSetDevice(c->dev));
    const int n = c->n, kmax = c->kmax;
    const size_t ld = (size_t)n + 2, fsz = ld * n * n;
    const double PI = 4.0 * atan(1.0), TWO_PI = 2.0 * PI;
    std::vector<double> g(3 * fsz);
    if (isp == -1) {
        // Taylor-Green (init_velocity.f90:252-293)
        const double dx = 2.0 * PI / (double)n;
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) {
                    double xx = (double)i * dx, yy = (double)j * dx, zz = (double)k * dx;
                    size_t q = i + ld * (j + (size_t)n * k);
                    g[q] = sin(xx) * cos(yy) * cos(zz);
                    g[fsz + q] = -cos(xx) * sin(yy) * cos(zz);
                    g[2 * fsz + q] = 0.0;
                }
        H3D_TRY(upload_phys(c, g.data(), (int64_t)ld, 3));
        H3D_TRY(fwd3d64(c, c->W64, 3));
        H3D_CHECK(cudaMemcpyAsync(c->U, c->W64, sizeof(double2) * 3 * c->fs64, cudaMemcpyDeviceToDevice, c->st));
        H3D_CHECK(cudaStreamSynchronize(c->st));
        return 0;
    }
    // RANDu over six full padded arrays in the reference's order, then Box-Muller
    // (init_velocity.f90:67-113)
    Randu &r = c->rng;
    (void)r.next(-rn1);
    for (size_t q = 0; q < 3 * fsz; q++) g[q] = r.next(rn1);
    for (int f = 0; f < 3; f++)
        for (size_t q = 0; q < fsz; q++) {
            double u2 = r.next(rn1);
            double &u1 = g[f * fsz + q];
            u1 = sqrt(-2.0 * log(u1)) * sin(TWO_PI * u2);
        }
    H3D_TRY(upload_phys(c, g.data(), (int64_t)ld, 3));
    H3D_TRY(fwd3d64(c, c->W64, 3));
    c->alias_known = 0;
    k_init_curl<<<pw_grid(c), 256, 0, c->st>>>(n, c->nh, c->P64, c->fs64, kmax, c->W64, c->U);
    H3D_LAUNCH_CHECK();
    std::vector<double> es(kmax), et, ratio(kmax);
    H3D_TRY(shell_spectrum(c, c->U, 3, es.data()));
    target_spectrum(isp, peak, ir_exp, kmax, et);
    for (int k = 0; k < kmax; k++) ratio[k] = es[k] > 0.0 ? sqrt(et[k] / es[k]) : -1.0;
    H3D_CHECK(cudaMemcpyAsync(c->d_ratio, ratio.data(), sizeof(double) * kmax, cudaMemcpyHostToDevice, c->st));
    c->alias_known = 0;
    k_shell_scale<<<pw_grid(c), 256, 0, c->st>>>(n, c->nh, c->P64, c->fs64, 3, kmax, c->d_ratio, c->U);
    H3D_LAUNCH_CHECK();
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

extern "C" int hit3d_gpu_init_scalar(hit3d_ctx *c, int32_t s, double rn2, double peak)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    if (s < 0 || s >= c->p.n_scalars) return h3d_set_error_msg(-1, "hit3d_gpu_init_scalar: no such passive scalar");
    const int type = c->p.scalar_type[s], ic = type - (type / 100) * 100;
    H3D_CHECK(cudaSetDevice(c->dev));
    const int n = c->n, kmax = c->kmax;
    const size_t ld = (size_t)n + 2, fsz = ld * n * n;
    const double PI = 4.0 * atan(1.0), TWO_PI = 2.0 * PI, dx = 2.0 * PI / (double)n;
    double2 *F = c->U + (3 + s) * c->fs64;
    double2 *G = c->W64;
    c->alias_known = 0;
    if (ic == 0) {
        // init_scalar (init_scalars.f90:60-62): zero
        H3D_CHECK(cudaMemsetAsync(F, 0, sizeof(double2) * (size_t)c->fs64, c->st));
    } else if (ic < 10) {
        // init_scalar_spectrum (init_scalars.f90:84-269): Box-Muller noise from the
        // RANDu stream of RN2 over two full padded arrays, forward transform,
        // shells 1..kmax rescaled to the normalised target spectrum
        if (type != 1 && type != 2 && type != 3)
            return h3d_set_error_msg(-1, "INIT_SCALARS: WRONG INITIAL SPECTRUM TYPE");
        if (!(peak > 0.0)) return h3d_set_error_msg(-1, "hit3d_gpu_init_scalar: peak wavenumber must be > 0");
        std::vector<double> g(2 * fsz);
        Randu &r = c->rng;
        (void)r.next(-rn2);
        for (size_t q = 0; q < 2 * fsz; q++) g[q] = r.next(rn2);
        for (size_t q = 0; q < fsz; q++) g[q] = sqrt(-2.0 * log(g[q])) * sin(TWO_PI * g[fsz + q]);
        H3D_TRY(upload_phys(c, g.data(), (int64_t)ld, 1));
        H3D_TRY(fwd3d64(c, G, 1));
        std::vector<double> es(kmax), et, ratio(kmax);
        H3D_TRY(shell_spectrum(c, G, 1, es.data()));
        // types 1 and 3: the velocity's spectrum 1; type 2: its spectrum 3
        target_spectrum(type == 2 ? 3 : 1, peak, 0.0, kmax, et);
        for (int k = 0; k < kmax; k++) ratio[k] = es[k] > 0.0 ? sqrt(et[k] / es[k]) : -1.0;
        H3D_CHECK(cudaMemcpyAsync(c->d_ratio, ratio.data(), sizeof(double) * kmax, cudaMemcpyHostToDevice, c->st));
        k_shell_scale<<<pw_grid(c), 256, 0, c->st>>>(n, c->nh, c->P64, c->fs64, 1, kmax, c->d_ratio, G);
        H3D_LAUNCH_CHECK();
        if (type == 3) {
            // sign(phi) * 0.9 in physical space, then shells 0 and >= 2 kmax / 3 removed
            H3D_TRY(inv3d64(c, G, 1));
            k_sign09<<<pw_grid(c), 256, 0, c->st>>>(n, 2 * (int64_t)c->P64, reinterpret_cast<double *>(G));
            H3D_LAUNCH_CHECK();
            H3D_TRY(fwd3d64(c, G, 1));
            const int kcut = kmax * 2 / 3;
            for (int k = 0; k < kmax; k++) ratio[k] = (k + 1) < kcut ? 1.0 : -1.0;
            H3D_CHECK(cudaMemcpyAsync(c->d_ratio, ratio.data(), sizeof(double) * kmax, cudaMemcpyHostToDevice, c->st));
            k_shell_scale<<<pw_grid(c), 256, 0, c->st>>>(n, c->nh, c->P64, c->fs64, 1, kmax, c->d_ratio, G);
            H3D_LAUNCH_CHECK();
        }
        H3D_CHECK(cudaMemcpyAsync(F, G, sizeof(double2) * (size_t)c->fs64, cudaMemcpyDeviceToDevice, c->st));
    } else {
        // init_scalar_space (init_scalars.f90:280-345): profiles in physical space
        if (ic != 11 && ic != 12 && ic != 13) return h3d_set_error_msg(-1, "INIT_SCALARS: UNEXPECTED SCALAR TYPE");
        std::vector<double> g(fsz, 0.0);
        if (ic == 11) {
            const double h = std::max(2.0 * dx, TWO_PI / peak);
            for (int k = 0; k < n; k++) {
                const double z = (double)k * dx;
                const double v = tanh((z - PI * 0.5) / h) - tanh((z - PI * 1.5) / h) - 1.0;
                for (int j = 0; j < n; j++)
                    for (int i = 0; i < n; i++) g[i + ld * (j + (size_t)n * k)] = v;
            }
        } else if (ic == 12) {
            const double h = std::max(8.0 * dx, PI / 8.0);
            for (int i = 0; i < n; i++) {
                const double x = (double)i * dx;
                const double v = tanh((x - PI * 0.25) / h) - tanh((x - PI * 0.75) / h) + tanh((x - PI * 1.25) / h) -
                                 tanh((x - PI * 1.75) / h) - 1.0;
                for (size_t r = 0; r < (size_t)n * n; r++) g[i + ld * r] = v;
            }
        } else {
            const double pk = std::min(peak, (double)(n / 8));
            for (int i = 0; i < n; i++) {
                const double v = sin(pk * dx * (double)i);
                for (size_t r = 0; r < (size_t)n * n; r++) g[i + ld * r] = v;
            }
        }
        H3D_TRY(upload_phys(c, g.data(), (int64_t)ld, 1));
        H3D_TRY(fwd3d64(c, G, 1));
        H3D_CHECK(cudaMemcpyAsync(F, G, sizeof(double2) * (size_t)c->fs64, cudaMemcpyDeviceToDevice, c->st));
        if (ic != 13) H3D_CHECK(cudaMemsetAsync(F, 0, sizeof(double2), c->st));  // the mean mode
    }
    // no modes beyond N/3 in any direction (init_scalars.f90:26-33)
    k_dealias_all<<<pw_grid(c), 256, 0, c->st>>>(n, c->nh, c->P64, c->fs64, 1, n / 3, F);
    H3D_LAUNCH_CHECK();
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

extern "C" int hit3d_gpu_particles_filter(hit3d_ctx *c, double delta)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    H3D_CHECK(cudaSetDevice(c->dev));
    if (!(delta > 0.0)) {
        if (c->pfilt) { cudaFree(c->pfilt); c->pfilt = nullptr; }
        if (c->pbuf) { cudaFree(c->pbuf); c->pbuf = nullptr; }
        return 0;
    }
    if (delta < 3.0 * c->dx)
        return h3d_set_error_msg(-1, "hit3d_gpu_particles_filter: particles_filter_size is too small (less than 3*dx)");
    if (!c->pfilt) H3D_TRY(ctx_alloc((void **)&c->pfilt, sizeof(double2) * (size_t)c->fs64));
    if (!c->pbuf) H3D_TRY(ctx_alloc((void **)&c->pbuf, sizeof(double2) * 3 * (size_t)c->fs64));
    // the Gaussian of m_filter_xfftw.f90:197-220 with the particle filter width,
    // made in the FP64 work field and kept
    H3D_TRY(filter_transfer(c, 2, delta));
    H3D_CHECK(cudaMemcpyAsync(c->pfilt, c->W64, sizeof(double2) * (size_t)c->fs64, cudaMemcpyDeviceToDevice, c->st));
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

extern "C" int hit3d_gpu_particles_upload(hit3d_ctx *c, const double *xyzp, const double *uvwp, int64_t np, int32_t scheme)
{
    if (!c || (np > 0 && !xyzp)) return h3d_set_error_msg(-1, "hit3d_gpu_particles_upload: null argument");
    if (scheme != 0 && scheme != 1) return h3d_set_error_msg(-1, "particles_tracking_scheme must be 0 or 1");
    if (np < 0) return h3d_set_error_msg(-1, "np < 0");
    H3D_CHECK(cudaSetDevice(c->dev));
    if (c->d_xyz) { cudaFree(c->d_xyz); c->d_xyz = nullptr; }
    if (c->d_uvw) { cudaFree(c->d_uvw); c->d_uvw = nullptr; }
    c->np = 0;
    if (np == 0) return 0;
    int rc;
    if ((rc = ctx_alloc((void **)&c->d_xyz, sizeof(double) * 3 * np)) || (rc = ctx_alloc((void **)&c->d_uvw, sizeof(double) * 3 * np)))
        return rc;
    if (!c->phys && (rc = ctx_alloc((void **)&c->phys, sizeof(double) * 3 * (size_t)c->n * c->n * c->n))) return rc;
    H3D_CHECK(cudaMemcpy(c->d_xyz, xyzp, sizeof(double) * 3 * np, cudaMemcpyHostToDevice));
    if (uvwp) H3D_CHECK(cudaMemcpy(c->d_uvw, uvwp, sizeof(double) * 3 * np, cudaMemcpyHostToDevice));
    else {
        std::vector<double> m(3 * np, -999.0);
        H3D_CHECK(cudaMemcpy(c->d_uvw, m.data(), sizeof(double) * 3 * np, cudaMemcpyHostToDevice));
    }
    c->np = np;
    c->pscheme = scheme;
    return 0;
}

extern "C" int hit3d_gpu_particles_download(hit3d_ctx *c, double *xyzp, double *uvwp)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    H3D_CHECK(cudaSetDevice(c->dev));
    H3D_CHECK(cudaStreamSynchronize(c->st));
    if (c->np == 0) return 0;
    if (xyzp) H3D_CHECK(cudaMemcpy(xyzp, c->d_xyz, sizeof(double) * 3 * c->np, cudaMemcpyDeviceToHost));
    if (uvwp) H3D_CHECK(cudaMemcpy(uvwp, c->d_uvw, sizeof(double) * 3 * c->np, cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int hit3d_gpu_xfft3d(hit3d_ctx *c, int32_t flag, const double *in, double *out, int64_t ld1)
{
    if (!c || !in || !out) return h3d_set_error_msg(-1, "hit3d_gpu_xfft3d: null argument");
    if (flag != 1 && flag != -1) return h3d_set_error_msg(-1, "hit3d_gpu_xfft3d: flag must be 1 or -1");
    if (ld1 < c->n + 2) return h3d_set_error_msg(-1, "ld1 must be >= nx+2");
    H3D_CHECK(cudaSetDevice(c->dev));
    const size_t rows = (size_t)c->n * c->n;
    const size_t width = (size_t)c->nh * sizeof(double2);
    if (flag == 1) {
        H3D_TRY(upload_phys(c, in, ld1, 1));
        H3D_TRY(fwd3d64(c, c->W64, 1));
        k_dev_to_ref<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, c->W64, c->stage);
        H3D_LAUNCH_CHECK();
        H3D_CHECK(cudaMemcpy2DAsync(out, ld1 * sizeof(double), c->stage, width, width, rows, cudaMemcpyDeviceToHost, c->st));
    } else {
        H3D_CHECK(cudaMemcpy2DAsync(c->stage, width, in, ld1 * sizeof(double), width, rows, cudaMemcpyHostToDevice, c->st));
        k_ref_to_dev<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, c->stage, c->W64);
        H3D_LAUNCH_CHECK();
        H3D_TRY(inv3d64(c, c->W64, 1));
        H3D_CHECK(cudaMemcpy2DAsync(out, ld1 * sizeof(double), reinterpret_cast<double *>(c->W64), 2 * c->P64 * sizeof(double),
                                    c->n * sizeof(double), rows, cudaMemcpyDeviceToHost, c->st));
    }
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

// filter transfer function into the FP64 scratch field W64[0]: kind 2 Gaussian
// (kernel built in physical space and transformed, m_filter_xfftw.f90:197-271),
// kind 4 box of width delta (analytic sinc product)
static int filter_transfer(hit3d_ctx *c, int kind, double delta)
{
    if (kind != 2 && kind != 4) return h3d_set_error_msg(-1, "filter kind must be 2 (Gaussian) or 4 (box)");
    const int n = c->n;
    double2 *G = c->W64;
    if (kind == 2) {
        // Gaussian kernel in physical space, then its transform (m_filter_xfftw.f90:197-220, 259-271)
        if (delta < 3.0 * c->dx) return h3d_set_error_msg(-1, "filter_xfftw_init: delta is too small");
        const size_t ld = (size_t)n + 2;
        std::vector<double> g(ld * n * n, 0.0);
        const double PI = 4.0 * atan(1.0);
        const double c1 = 6.0 / (delta * delta);
        const double sq = sqrt(c1 / PI);
        const double c2 = sq * sq * sq * (c->dx * c->dx * c->dx);
        for (int k = 0; k < n; k++) {
            int dk = k < n - k ? k : n - k;
            double rz = c->dx * (double)dk;
            for (int j = 0; j < n; j++) {
                int dj = j < n - j ? j : n - j;
                double ry = c->dx * (double)dj;
                for (int i = 0; i < n; i++) {
                    int di = i < n - i ? i : n - i;
                    double rx = c->dx * (double)di;
                    rx = rx * rx + ry * ry + rz * rz;
                    double v = c2 * exp(-c1 * rx);
                    if (v < 1.e-20) v = 0.0;
                    g[i + ld * (j + (size_t)n * k)] = v;
                }
            }
        }
        H3D_TRY(upload_phys(c, g.data(), (int64_t)ld, 1));
        H3D_TRY(fwd3d64(c, G, 1));
    } else {
        k_box_transfer<<<pw_grid(c), 256, 0, c->st>>>(n, c->nh, c->P64, delta, G);
        H3D_LAUNCH_CHECK();
    }
    return 0;
}

extern "C" int hit3d_gpu_filter_field(hit3d_ctx *c, int32_t kind, double delta, int32_t field)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    if (field < 0 || field >= 3 + c->nsc) return h3d_set_error_msg(-1, "hit3d_gpu_filter_field: no such field");
    H3D_CHECK(cudaSetDevice(c->dev));
    H3D_TRY(filter_transfer(c, kind, delta));
    c->alias_known = 0;
    k_filter_apply<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, c->P64, c->W64, c->U + field * c->fs64);
    H3D_LAUNCH_CHECK();
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

// download physical rows of nf FP64 fields as compact FP32 [f][z][y][x]
static int download_f32(hit3d_ctx *c, const double2 *base, int nf, float *out, int stride = 1)
{
    const int64_t m = c->n / stride, np = m * m * m;
    float *st = reinterpret_cast<float *>(c->stage);  // n*n*nh double2 >= n^3 floats
    for (int f = 0; f < nf; f++) {
        k_phys_to_f32<<<pw_grid(c), 256, 0, c->st>>>(c->n, 2 * (int64_t)c->P64, stride,
                                                     reinterpret_cast<const double *>(base + f * c->fs64), st);
        H3D_LAUNCH_CHECK();
        H3D_CHECK(cudaMemcpyAsync(out + f * np, st, sizeof(float) * np, cudaMemcpyDeviceToHost, c->st));
        H3D_CHECK(cudaStreamSynchronize(c->st));
    }
    return 0;
}

extern "C" int hit3d_gpu_sgs_samples(hit3d_ctx *c, int32_t kind, double delta, int32_t stride, float *out)
{
    if (!c || !out) return h3d_set_error_msg(-1, "hit3d_gpu_sgs_fields: null argument");
    if (c->p.precision != 0) return h3d_set_error_msg(-1, "hit3d_gpu_sgs_fields: needs a context with FP64 transforms");
    if (stride < 1 || c->n % stride != 0) return h3d_set_error_msg(-1, "hit3d_gpu_sgs_samples: stride must divide nx");
    H3D_CHECK(cudaSetDevice(c->dev));
    const int64_t m = c->n / stride, np = m * m * m;
    if (!c->sgs) H3D_TRY(ctx_alloc((void **)&c->sgs, sizeof(double2) * 6 * (size_t)c->fs64));
    double2 *W = reinterpret_cast<double2 *>(c->W);
    const int64_t fs = c->fs64;
    const int P = c->P64;
    // 1. products of the resolved velocity, transformed forward: W0..5 = (u_i u_j)^
    H3D_TRY(zinv<double>(c, 3, PRE_COPY, 0, c->U, fs, W, fs, P));
    H3D_TRY(spass<double>(c, 1, false, W, fs, P, 3));
    {
        FusedArgs fa;
        memset(&fa, 0, sizeof fa);
        for (int f = 0; f < 3; f++) fa.in[f] = W + f * fs;
        for (int o = 0; o < 6; o++) fa.out[o] = W + o * fs;
        fa.pitch = P;
        H3D_TRY((xfused<double, OpVel>(c, fa)));
    }
    H3D_TRY(spass<double>(c, 1, true, W, fs, P, 6));
    H3D_TRY(spass<double>(c, 2, true, W, fs, P, 6));
    // 2. the filter; W64 is W's first field in FP64 mode, so build G in sgs[5]
    double2 *G = c->sgs + 5 * fs;
    {
        double2 *save = c->W64;
        c->W64 = G;
        int rc = filter_transfer(c, kind, delta);
        c->W64 = save;
        if (rc) return rc;
    }
    // 3. filtered velocity (sgs0..2) and filtered products (W0..5), spectral
    H3D_CHECK(cudaMemcpyAsync(c->sgs, c->U, sizeof(double2) * 3 * fs, cudaMemcpyDeviceToDevice, c->st));
    for (int f = 0; f < 3; f++) {
        k_filter_apply<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, P, G, c->sgs + f * fs);
        H3D_LAUNCH_CHECK();
    }
    for (int f = 0; f < 6; f++) {
        k_filter_apply<<<pw_grid(c), 256, 0, c->st>>>(c->n, c->nh, P, G, W + f * fs);
        H3D_LAUNCH_CHECK();
    }
    // 4. filtered velocity gradients A_ij = d ubar_i / dx_j, nine fields (i-major);
    //    G is no longer needed, so sgs3..5 serve as scratch
    double2 *tmp = c->sgs + 3 * fs;
    for (int i = 0; i < 3; i++) {
        H3D_TRY(zinv<double>(c, 3, PRE_GRAD, i, c->sgs, fs, tmp, fs, P));
        H3D_TRY(spass<double>(c, 1, false, tmp, fs, P, 3));
        H3D_TRY(xc2r<double>(c, tmp, fs, P, 3));
        H3D_TRY(download_f32(c, tmp, 3, out + (9 + 3 * i) * np, stride));
    }
    // 5. physical filtered velocity and products; tau in place of the products
    H3D_TRY(inv3d64(c, c->sgs, 3));
    H3D_TRY(inv3d64(c, W, 6));
    k_sgs_tau<<<pw_grid(c), 256, 0, c->st>>>(c->n, 2 * (int64_t)P, 2 * fs, reinterpret_cast<const double *>(c->sgs),
                                             reinterpret_cast<double *>(W));
    H3D_LAUNCH_CHECK();
    H3D_TRY(download_f32(c, c->sgs, 3, out, stride));
    H3D_TRY(download_f32(c, W, 6, out + 3 * np, stride));
    return 0;
}

extern "C" int hit3d_gpu_sgs_fields(hit3d_ctx *c, int32_t kind, double delta, float *out)
{
    return hit3d_gpu_sgs_samples(c, kind, delta, 1, out);
}

extern "C" int hit3d_gpu_physical_fields(hit3d_ctx *c, int32_t nf, double k2max, double *out, int64_t ld1)
{
    if (!c || !out) return h3d_set_error_msg(-1, "hit3d_gpu_physical_fields: null argument");
    if (ld1 < c->n + 2) return h3d_set_error_msg(-1, "ld1 must be >= nx+2");
    if (nf < 1 || nf > 3 + c->nsc) return h3d_set_error_msg(-1, "hit3d_gpu_physical_fields: nfields out of range");
    H3D_CHECK(cudaSetDevice(c->dev));
    const size_t rows = (size_t)c->n * c->n;
    c->k2max = k2max;
    for (int f0 = 0; f0 < nf; f0 += 3) {
        const int m = nf - f0 < 3 ? nf - f0 : 3;
        H3D_TRY(inv_from_state(c, m, k2max > 0.0 ? PRE_TRUNC : PRE_COPY, 0, c->U + f0 * c->fs64));
        for (int f = 0; f < m; f++)
            H3D_CHECK(cudaMemcpy2DAsync(out + (size_t)(f0 + f) * ld1 * rows, ld1 * sizeof(double),
                                        reinterpret_cast<double *>(c->W64 + f * c->fs64), 2 * c->P64 * sizeof(double),
                                        c->n * sizeof(double), rows, cudaMemcpyDeviceToHost, c->st));
    }
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

// target spectra of init_velocity.f90:193-220 (isp 2 added by this library)
static int target_spectrum(int isp, double peak, double ir_exp, int kmax, std::vector<double> &et)
{
    const double PI = 4.0 * atan(1.0);
    et.assign(kmax, 0.0);
    for (int k = 1; k <= kmax; k++) {
        double wmag = (double)k, ratio_k = wmag / peak;
        if (isp == 0) et[k - 1] = pow(wmag, -5.0 / 3.0);
        else if (isp == 1) et[k - 1] = ratio_k * ratio_k * ratio_k / peak * exp(-3.0 * ratio_k);
        else if (isp == 2) et[k - 1] = pow(wmag, ir_exp) * exp(-2.0 * ratio_k * ratio_k);
        else if (isp == 3) {
            double f = 2.0 * PI * ratio_k, f2 = f * f, d = 1.0 + f2;
            et[k - 1] = (f2 * f2) / (d * d * d);
        } else return -1;
    }
    double tot = 0.0;
    for (int k = 0; k < kmax; k++) tot = tot + et[k];
    for (int k = 0; k < kmax; k++) et[k] = et[k] / tot;
    return 0;
}

extern "C" int hit3d_gpu_velocity_rescale(hit3d_ctx *c, int32_t isp, double peak, double ir_exp)
{
    if (!c) return h3d_set_error_msg(-1, "null context");
    if (isp == -1) return 0;  // Taylor-Green runs are never rescaled (velocity_rescale.f90:24)
    const int n = c->n, kmax = c->kmax;
    std::vector<double> et;
    if (target_spectrum(isp, peak, ir_exp, kmax, et)) return h3d_set_error_msg(-1, "ERROR: WRONG INITIAL SPECTRUM TYPE");
    H3D_CHECK(cudaSetDevice(c->dev));
    // shell energies without the kx = 0 half weight; hits = real entries per shell
    // (velocity_rescale.f90:42-60)
    std::vector<double> es(kmax);
    H3D_TRY(shell_spectrum(c, c->U, 3, es.data(), 1.0));
    std::vector<int64_t> hits(kmax, 0);
    for (int kq = 0; kq < n; kq++) {
        const double ky = kwave(kq, n);
        for (int jq = 0; jq < n; jq++) {
            const double kz = kwave(jq, n);
            for (int kx = 0; kx < n / 2; kx++) {
                const double k2 = (double)kx * kx + ky * ky + kz * kz;
                const int sh = (int)lroundf(sqrtf((float)k2));
                if (sh > 0 && sh <= kmax) hits[sh - 1] += 2;
            }
        }
    }
    const double PI = 4.0 * atan(1.0);
    const double fac = 4.0 / 3.0 * PI / 2.0;
    std::vector<double> ratio(kmax);
    for (int k = 1; k <= kmax; k++) {
        double r1 = (double)k + 0.5, r2 = (double)k - 0.5;
        if (k == 1) r2 = 0.0;
        double e = hits[k - 1] > 0 ? es[k - 1] / (double)hits[k - 1] * fac * (r1 * r1 * r1 - r2 * r2 * r2) : 0.0;
        ratio[k - 1] = e > 0.0 ? sqrt(et[k - 1] / e) : -1.0;
    }
    H3D_CHECK(cudaMemcpyAsync(c->d_ratio, ratio.data(), sizeof(double) * kmax, cudaMemcpyHostToDevice, c->st));
    c->alias_known = 0;
    k_shell_scale<<<pw_grid(c), 256, 0, c->st>>>(n, c->nh, c->P64, c->fs64, 3, kmax, c->d_ratio, c->U);
    H3D_LAUNCH_CHECK();
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

extern "C" int hit3d_gpu_physical_velocity(hit3d_ctx *c, double *out, int64_t ld1)
{
    if (!c || !out) return h3d_set_error_msg(-1, "hit3d_gpu_physical_velocity: null argument");
    if (ld1 < c->n + 2) return h3d_set_error_msg(-1, "ld1 must be >= nx+2");
    H3D_CHECK(cudaSetDevice(c->dev));
    H3D_TRY(inv_from_state(c, 3, PRE_COPY, 0, c->U));
    const size_t rows = (size_t)c->n * c->n;
    for (int f = 0; f < 3; f++)
        H3D_CHECK(cudaMemcpy2DAsync(out + (size_t)f * ld1 * rows, ld1 * sizeof(double),
                                    reinterpret_cast<double *>(c->W64 + f * c->fs64), 2 * c->P64 * sizeof(double),
                                    c->n * sizeof(double), rows, cudaMemcpyDeviceToHost, c->st));
    H3D_CHECK(cudaStreamSynchronize(c->st));
    return 0;
}

// ---------------------------------------------------------------------------
// batched form: many independent runs (uneven sizes, own parameters and seeds)
// advanced together.  After an eager first-order step, chunks of `graph_steps`
// Adams-Bashforth steps of all runs are recorded once into a CUDA graph -- one
// branch per run on its own stream, forked from and joined back into a root
// stream -- and replayed with a single launch per chunk.
// ---------------------------------------------------------------------------
// Runs of a batch that share a grid size, precision and forcing (velocity only,
// 2/3 rule, no LES) form a class: their state, AB2 history and work fields sit
// in one slab (run r at a fixed run stride), and every pass of a step is ONE
// launch over all the class's runs (the run index folded into the grid), with
// each run's viscosity, time step and forcing-band energy in small device
// tables.  Other runs step on their own.
constexpr int kBatchVariants = 7;  // fused x-pass variants 8-14 walk the tiles of several runs

struct BatchClass {
    std::vector<int> runs;
    double2 *U = nullptr, *RO = nullptr;
    void *W = nullptr;
    int64_t ru = 0, rw = 0;  // run strides: state (complex FP64 elements), work fields (transform precision)
    double *tab = nullptr;   // [nu | dt | forcing energy] x runs
    std::vector<double> tab_nu, tab_dt;  // the values uploaded
};

struct hit3d_batch {
    std::vector<hit3d_ctx *> runs;
    std::vector<int> fov, fos;
    std::vector<int> run_class;  // class of each run, -1: stepped on its own
    std::vector<BatchClass> classes;
    int dev = 0;
    cudaStream_t root = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_steps = 0;
    int64_t launches = 0;
    std::vector<double> cap_dt;  // dt, scalar switch and pruning of every run when the graph was recorded
    std::vector<int> cap_scal, cap_prune;
};

static int run_step(hit3d_ctx *c, int ev, int es)
{
    return c->p.precision == 0 ? step_once<double>(c, ev, es) : step_once<float>(c, ev, es);
}

// runs that can join a class, and the key of the class
static bool class_eligible(const hit3d_params &p)
{
    return p.les_model == 0 && p.n_scalars == 0 && p.dealias == 0;
}
static bool same_class(const hit3d_params &a, const hit3d_params &b)
{
    return a.nx == b.nx && a.precision == b.precision && a.flow_type == b.flow_type &&
           (a.flow_type == 0 || (a.kfmax == b.kfmax && a.famp == b.famp));
}

// upload the class's per-run viscosity and time step when they changed
static int class_tables(hit3d_batch *b, BatchClass &k)
{
    const size_t nr = k.runs.size();
    std::vector<double> nu(nr), dt(nr);
    for (size_t i = 0; i < nr; i++) {
        nu[i] = b->runs[k.runs[i]]->p.nu;
        dt[i] = b->runs[k.runs[i]]->p.dt;
    }
    if (nu == k.tab_nu && dt == k.tab_dt) return 0;
    hit3d_ctx *c = b->runs[k.runs[0]];
    H3D_CHECK(cudaMemcpyAsync(k.tab, nu.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, c->st));
    H3D_CHECK(cudaMemcpyAsync(k.tab + nr, dt.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, c->st));
    H3D_CHECK(cudaStreamSynchronize(c->st));
    k.tab_nu = nu;
    k.tab_dt = dt;
    return 0;
}

// every run of the class pruned (state zero beyond N/3): the pruned transforms
static bool class_pruned(hit3d_batch *b, const BatchClass &k)
{
    for (int r : k.runs)
        if (!(b->runs[r]->prune_on && b->runs[r]->pruned)) return false;
    return true;
}

// one step of every run of a class, issued on its first run's stream: forcing
// energy, z and y inverse, fused x pass, y and z forward and the update, each
// one launch over the class (main.f90:124-167 for every run)
// the class fields of the first run's context while a class is issued, reset
// on every exit path
struct ClassScope {
    hit3d_ctx *c;
    ClassScope(hit3d_batch *b, BatchClass &k) : c(b->runs[k.runs[0]])
    {
        c->bruns = (int)k.runs.size();
        c->bru = k.ru;
        c->brw = k.rw;
        c->kc_active = (c->prune_on && class_pruned(b, k)) ? c->n / 3 : -1;
    }
    ~ClassScope()
    {
        c->bruns = 0;
        c->bru = c->brw = 0;
        c->kc_active = -1;
    }
};

template <typename T> static int class_step(hit3d_batch *b, BatchClass &k, int euler)
{
    hit3d_ctx *c = b->runs[k.runs[0]];
    const int nr = (int)k.runs.size();
    const hit3d_params &p = c->p;
    ClassScope scope(b, k);
    cx<T> *W = reinterpret_cast<cx<T> *>(c->W);
    const int64_t wfs = c->wfs;
    const int wp = c->wpitch;
    auto Wf = [&](int i) { return W + i * wfs; };
    double *fen = k.tab + 2 * nr;
    if (p.flow_type == 1) {
        const ForcingLaunch fl = forcing_launch(c->n, p.kfmax);
        k_forcing_energy<<<nr, fl.threads, fl.smem, c->st>>>(c->n, c->P64, c->fs64, fl.kfmax, c->U, fen, k.ru);
        H3D_LAUNCH_CHECK();
    }
    H3D_TRY(zinv<T>(c, 3, PRE_COPY, 0, c->U, c->fs64, Wf(0), wfs, wp));
    H3D_TRY(spass<T>(c, 1, false, Wf(0), wfs, wp, 3));
    {
        FusedArgs fa;
        memset(&fa, 0, sizeof fa);
        for (int f = 0; f < 3; f++) fa.in[f] = Wf(f);
        for (int o = 0; o < 6; o++) fa.out[o] = Wf(o);
        fa.pitch = wp;
        fa.err = c->d_err;
        H3D_TRY((xfused<T, OpVel>(c, fa)));
    }
    H3D_TRY(spass<T>(c, 1, true, Wf(0), wfs, wp, 6));
    H3D_TRY(spass<T>(c, 2, true, Wf(0), wfs, wp, 6));
    StepArgs a;
    memset(&a, 0, sizeof a);
    a.n = c->n; a.nh = c->nh; a.pitch = c->P64; a.ppitch = wp; a.fs = c->fs64; a.pfs = wfs;
    a.nu = p.nu; a.dt = p.dt; a.euler_v = euler; a.euler_s = euler;
    a.flow_type = p.flow_type; a.kfmax = p.kfmax; a.famp = p.famp; a.fenergy = fen;
    a.kc = c->kc_active;
    a.ru = k.ru; a.rp = k.rw; a.nu_r = k.tab; a.dt_r = k.tab + nr;
    // CTAs per run: enough for the run's modes, at most one resident wave in all
    const int64_t nm = (int64_t)(c->kc_active >= 0 ? (int64_t)(c->kc_active + 1) * (2 * c->kc_active + 1) *
                                                         (2 * c->kc_active + 1)
                                                   : (int64_t)c->n * c->n * c->nh);
    int64_t gx = (nm + 255) / 256;
    const int64_t wave = (int64_t)pw_grid(c, k_update_vel_23<T>).x;
    const int64_t cap = wave / nr > 1 ? wave / nr : 1;
    gx = gx < cap ? gx : cap;
    k_update_vel_23<T><<<dim3((unsigned)gx, (unsigned)nr), 256, 0, c->st>>>(a, Wf(0), nullptr, c->U, c->RO);
    H3D_LAUNCH_CHECK();
    return 0;
}
static int class_step_any(hit3d_batch *b, BatchClass &k, int euler)
{
    return b->runs[k.runs[0]]->p.precision == 0 ? class_step<double>(b, k, euler) : class_step<float>(b, k, euler);
}

// the passes of a class step that the tuner's choices affect, on scratch work
// fields only (the state is read, never written): what 0 = the fused x pass,
// 1 = the strided passes (z and y inverse, y and z forward)
template <typename T> static int class_passes(hit3d_batch *b, BatchClass &k, int what)
{
    hit3d_ctx *c = b->runs[k.runs[0]];
    ClassScope scope(b, k);
    cx<T> *W = reinterpret_cast<cx<T> *>(c->W);
    const int64_t wfs = c->wfs;
    const int wp = c->wpitch;
    if (what == 0) {
        FusedArgs fa;
        memset(&fa, 0, sizeof fa);
        for (int f = 0; f < 3; f++) fa.in[f] = W + f * wfs;
        for (int o = 0; o < 6; o++) fa.out[o] = W + o * wfs;
        fa.pitch = wp;
        fa.err = c->d_err;
        return xfused<T, OpVel>(c, fa);
    }
    H3D_TRY(zinv<T>(c, 3, PRE_COPY, 0, c->U, c->fs64, W, wfs, wp));
    H3D_TRY(spass<T>(c, 1, false, W, wfs, wp, 3));
    H3D_TRY(spass<T>(c, 1, true, W, wfs, wp, 6));
    H3D_TRY(spass<T>(c, 2, true, W, wfs, wp, 6));
    return 0;
}
static int class_time(hit3d_batch *b, BatchClass &k, int what, float *ms)
{
    hit3d_ctx *c = b->runs[k.runs[0]];
    auto go = [&]() { return c->p.precision == 0 ? class_passes<double>(b, k, what) : class_passes<float>(b, k, what); };
    EventPair ev;
    H3D_CHECK(ev.create());
    H3D_TRY(go());  // warm-up
    H3D_CHECK(cudaEventRecord(ev.e0, c->st));
    for (int r = 0; r < 3; r++) H3D_TRY(go());
    H3D_CHECK(cudaEventRecord(ev.e1, c->st));
    H3D_CHECK(cudaEventSynchronize(ev.e1));
    H3D_CHECK(cudaEventElapsedTime(ms, ev.e0, ev.e1));
    *ms /= 3.0f;
    return 0;
}

extern "C" int hit3d_batch_nclasses(hit3d_batch *b) { return b ? (int)b->classes.size() : -1; }

extern "C" int hit3d_batch_autotune(hit3d_batch *b, int32_t *choice, double *ms)
{
    if (!b) return h3d_set_error_msg(-1, "hit3d_batch_autotune: null batch");
    H3D_CHECK(cudaSetDevice(b->dev));
    for (hit3d_ctx *cr : b->runs) H3D_TRY(ensure_alias_state(cr));
    for (size_t q = 0; q < b->classes.size(); q++) {
        BatchClass &k = b->classes[q];
        hit3d_ctx *c = b->runs[k.runs[0]];
        double *mq = ms ? ms + q * (kBatchVariants + kColTiles) : nullptr;
        int bv = 13;
        float bt = 1e30f;
        for (int v = 0; v < kBatchVariants; v++) {
            c->xcfg = 8 + v;
            float t = 0.f;
            H3D_TRY(class_time(b, k, 0, &t));
            if (mq) mq[v] = t;
            if (t < bt) { bt = t; bv = 8 + v; }
        }
        c->xcfg = bv;
        int bc = 0;
        bt = 1e30f;
        if (mq)
            for (int ct = 0; ct < kColTiles; ct++) mq[kBatchVariants + ct] = 0.0;
        for (int ct = 0; ct < kColTiles; ct++) {
            if (c->n > 512 && ct > 0 && ct < 3) continue;
            c->ctile = ct;
            float t = 0.f;
            H3D_TRY(class_time(b, k, 1, &t));
            if (mq) mq[kBatchVariants + ct] = t;
            if (t < bt) { bt = t; bc = ct; }
        }
        c->ctile = bc;
        if (choice) { choice[2 * q] = bv; choice[2 * q + 1] = bc; }
    }
    // the recorded graph holds the old launch shapes
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    for (hit3d_ctx *cr : b->runs) H3D_CHECK(cudaStreamSynchronize(cr->st));
    return 0;
}

extern "C" void hit3d_batch_destroy(hit3d_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->dev);
    if (b->root) cudaStreamSynchronize(b->root);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (cudaEvent_t e : b->join) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->root) cudaStreamDestroy(b->root);
    for (hit3d_ctx *c : b->runs) hit3d_gpu_finalize(c);
    for (BatchClass &k : b->classes) {
        if (k.U) cudaFree(k.U);
        if (k.RO) cudaFree(k.RO);
        if (k.W) cudaFree(k.W);
        if (k.tab) cudaFree(k.tab);
    }
    delete b;
}

extern "C" int hit3d_batch_create(const hit3d_params *p, int32_t nruns, hit3d_batch **out)
{
    if (!p || !out || nruns < 1) return h3d_set_error_msg(-1, "hit3d_batch_create: bad arguments");
    *out = nullptr;
    for (int r = 1; r < nruns; r++)
        if (p[r].device != p[0].device) return h3d_set_error_msg(-1, "hit3d_batch_create: all runs must share one device");
    H3D_CHECK(cudaSetDevice(p[0].device));
    hit3d_batch *b = new hit3d_batch();
    b->dev = p[0].device;
    b->run_class.assign(nruns, -1);
    // classes, in order of their first run
    for (int r = 0; r < nruns; r++) {
        if (!class_eligible(p[r]) || b->run_class[r] >= 0) continue;
        BatchClass k;
        for (int q = r; q < nruns; q++)
            if (b->run_class[q] < 0 && class_eligible(p[q]) && same_class(p[r], p[q])) {
                b->run_class[q] = (int)b->classes.size();
                k.runs.push_back(q);
            }
        b->classes.push_back(k);
    }
    b->runs.assign(nruns, nullptr);
    auto fail = [&](int rc) {
        hit3d_batch_destroy(b);
        return rc;
    };
    for (BatchClass &k : b->classes) {
        const hit3d_params &q = p[k.runs[0]];
        const int64_t nh = q.nx / 2 + 1, fs64 = (int64_t)q.nx * q.nx * round_up(nh, 8);
        const int64_t wfs = q.precision == 0 ? fs64 : (int64_t)q.nx * q.nx * round_up(nh, 16);
        const size_t welem = q.precision == 0 ? sizeof(double2) : sizeof(float2);
        const int nr = (int)k.runs.size();
        k.ru = 3 * fs64;
        k.rw = 6 * wfs;
        int rc = 0;
        if ((rc = ctx_alloc((void **)&k.U, sizeof(double2) * (size_t)(k.ru * nr))) ||
            (rc = ctx_alloc((void **)&k.RO, sizeof(double2) * (size_t)(k.ru * nr))) ||
            (rc = ctx_alloc(&k.W, welem * (size_t)(k.rw * nr))) ||
            (rc = ctx_alloc((void **)&k.tab, sizeof(double) * 3 * (size_t)nr)))
            return fail(rc);
        for (int i = 0; i < nr; i++) {
            hit3d_ctx *c = nullptr;
            rc = ctx_init(&p[k.runs[i]], &c, k.U + i * k.ru, k.RO + i * k.ru,
                          static_cast<unsigned char *>(k.W) + welem * (size_t)(i * k.rw));
            if (rc) return fail(rc);
            b->runs[k.runs[i]] = c;
            if (c->nw != 6) return fail(h3d_set_error_msg(-1, "hit3d_batch_create: class work fields mismatch"));
        }
    }
    for (int r = 0; r < nruns; r++) {
        if (b->runs[r]) continue;
        hit3d_ctx *c = nullptr;
        int rc = hit3d_gpu_init(&p[r], &c);
        if (rc) return fail(rc);
        b->runs[r] = c;
    }
    b->fov.assign(nruns, 1);
    b->fos.assign(nruns, 1);
    cudaError_t e = cudaStreamCreateWithFlags(&b->root, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    b->join.resize(nruns, nullptr);
    for (int r = 0; r < nruns && e == cudaSuccess; r++) e = cudaEventCreateWithFlags(&b->join[r], cudaEventDisableTiming);
    if (e != cudaSuccess) return fail(h3d_set_error(e, "hit3d_batch_create", __FILE__, __LINE__));
    *out = b;
    return 0;
}

extern "C" int hit3d_batch_context(hit3d_batch *b, int32_t r, hit3d_ctx **ctx)
{
    if (!b || !ctx || r < 0 || r >= (int)b->runs.size()) return h3d_set_error_msg(-1, "hit3d_batch_context: no such run");
    *ctx = b->runs[r];
    return 0;
}

// the issuing stream of each unit of work: a class's first run, or a lone run
static std::vector<int> batch_units(hit3d_batch *b)
{
    std::vector<int> u;
    for (BatchClass &k : b->classes) u.push_back(k.runs[0]);
    for (size_t r = 0; r < b->runs.size(); r++)
        if (b->run_class[r] < 0) u.push_back((int)r);
    return u;
}

// one Adams-Bashforth step of every run (classes batched), on the units' streams
static int batch_issue(hit3d_batch *b)
{
    for (BatchClass &k : b->classes) H3D_TRY(class_step_any(b, k, 0));
    for (size_t r = 0; r < b->runs.size(); r++)
        if (b->run_class[r] < 0) H3D_TRY(run_step(b->runs[r], 0, 0));
    return 0;
}

// record `steps` Adams-Bashforth steps of every run into one graph
static int batch_capture(hit3d_batch *b, int steps)
{
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    const std::vector<int> units = batch_units(b);
    H3D_CHECK(cudaStreamBeginCapture(b->root, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    for (int s = 0; s < steps && rc == 0; s++) {
        cudaEventRecord(b->fork, b->root);
        for (int r : units) cudaStreamWaitEvent(b->runs[r]->st, b->fork, 0);
        rc = batch_issue(b);
        for (int r : units) {
            cudaEventRecord(b->join[r], b->runs[r]->st);
            cudaStreamWaitEvent(b->root, b->join[r], 0);
        }
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->root, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return h3d_set_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
    b->graph = g;
    H3D_CHECK(cudaGraphInstantiate(&b->exec, g, 0));
    b->graph_steps = steps;
    b->cap_dt.clear();
    b->cap_scal.clear();
    b->cap_prune.clear();
    for (hit3d_ctx *cr : b->runs) {
        b->cap_dt.push_back(cr->p.dt);
        b->cap_scal.push_back(cr->int_scalars);
        b->cap_prune.push_back(cr->prune_on && cr->pruned);
    }
    return 0;
}

extern "C" int hit3d_batch_step(hit3d_batch *b, int32_t nsteps, int32_t graph_steps)
{
    if (!b || nsteps < 0) return h3d_set_error_msg(-1, "hit3d_batch_step: bad arguments");
    for (hit3d_ctx *cr : b->runs)
        if (cr->p.les_model == HIT3D_LES_LEARNED && !cr->mlp_wb)
            return h3d_set_error_msg(-1, "hit3d_batch_step: a run with the learned closure (les_model 20) needs weights "
                                         "(hit3d_gpu_les_set_mlp)");
    if (graph_steps < 1) graph_steps = 1;
    H3D_CHECK(cudaSetDevice(b->dev));
    for (hit3d_ctx *cr : b->runs) H3D_TRY(ensure_alias_state(cr));
    for (BatchClass &k : b->classes) H3D_TRY(class_tables(b, k));
    int left = nsteps;
    // first-order step of runs that need one, outside the graph: a whole class
    // together when all its runs need it, else run by run
    bool any_first = false;
    for (size_t r = 0; r < b->runs.size(); r++) any_first |= b->fov[r] || (b->fos[r] && b->runs[r]->int_scalars);
    if (any_first && left > 0) {
        for (BatchClass &k : b->classes) {
            bool all = true, none = true;
            for (int r : k.runs) {
                all &= b->fov[r] != 0;
                none &= b->fov[r] == 0;
            }
            if (all || none) {
                H3D_TRY(class_step_any(b, k, all ? 1 : 0));
            } else {
                for (int r : k.runs) H3D_TRY(run_step(b->runs[r], b->fov[r], b->fos[r]));
            }
            for (int r : k.runs) b->fov[r] = 0;
        }
        for (size_t r = 0; r < b->runs.size(); r++) {
            if (b->run_class[r] >= 0) continue;
            H3D_TRY(run_step(b->runs[r], b->fov[r], b->fos[r]));
            b->fov[r] = 0;
            if (b->runs[r]->int_scalars) b->fos[r] = 0;
        }
        left--;
    }
    if (left >= graph_steps) {
        bool stale = !b->exec || b->graph_steps != graph_steps || b->cap_dt.size() != b->runs.size();
        for (size_t r = 0; !stale && r < b->runs.size(); r++)
            stale = b->cap_dt[r] != b->runs[r]->p.dt || b->cap_scal[r] != b->runs[r]->int_scalars ||
                    b->cap_prune[r] != (b->runs[r]->prune_on && b->runs[r]->pruned);
        if (stale) {
            for (hit3d_ctx *cr : b->runs) H3D_CHECK(cudaStreamSynchronize(cr->st));
            H3D_TRY(batch_capture(b, graph_steps));
        }
        // order the replay after any eager work on the run streams
        for (size_t r = 0; r < b->runs.size(); r++) {
            H3D_CHECK(cudaEventRecord(b->join[r], b->runs[r]->st));
            H3D_CHECK(cudaStreamWaitEvent(b->root, b->join[r], 0));
        }
        while (left >= graph_steps) {
            H3D_CHECK(cudaGraphLaunch(b->exec, b->root));
            b->launches++;
            left -= graph_steps;
        }
        H3D_CHECK(cudaStreamSynchronize(b->root));
    }
    for (; left > 0; left--) H3D_TRY(batch_issue(b));
    for (hit3d_ctx *cr : b->runs) H3D_CHECK(cudaStreamSynchronize(cr->st));
    // a run with the learned closure on the tensor cores reports a completion
    // wait that ran out, as hit3d_gpu_step does; the fused x passes report a
    // stage wait that ran out in the first run of their class
    for (hit3d_ctx *cr : b->runs) {
        if (cr->p.les_model == HIT3D_LES_LEARNED && cr->mlp_kernel == 1 && nsteps > 0) {
            int herr = 0;
            H3D_CHECK(cudaMemcpy(&herr, cr->d_mlp_err, sizeof herr, cudaMemcpyDeviceToHost));
            if (herr) return h3d_set_error_msg(-5, "hit3d_batch_step: a tensor-core completion wait of the closure ran out");
        }
        int derr = 0;
        H3D_CHECK(cudaMemcpy(&derr, cr->d_err, sizeof derr, cudaMemcpyDeviceToHost));
        if (derr) return h3d_set_error_msg(-5, "hit3d_batch_step: a fused x pass gave up waiting for its input rows");
    }
    return 0;
}

extern "C" int64_t hit3d_batch_graph_launches(hit3d_batch *b) { return b ? b->launches : -1; }
