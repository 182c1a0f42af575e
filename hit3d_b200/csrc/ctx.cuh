// Device state of one simulation (the context behind the C-ABI handle) and the
// launch helpers that every translation unit of the library shares.
#pragma once
#include <cstdint>
#include <cstring>
#include <mutex>
#include <set>
#include <string>
#include <utility>

#include "../../include/hit3d_gpu.h"
#include "common.cuh"
#include "fft.cuh"

// every launch site has the context `c` in scope and counts its kernels
#define H3D_LAUNCH_CHECK()                 \
    do {                                   \
        c->nlaunch++;                      \
        H3D_CHECK(cudaGetLastError());     \
    } while (0)
#define H3D_TRY(x)            \
    do {                      \
        int rc__ = (x);       \
        if (rc__ != 0) return rc__; \
    } while (0)

// Raise a kernel's dynamic shared-memory limit once per kernel and device, so
// that steps recorded into a CUDA graph later make no attribute calls.
template <class K> static int set_smem(K kernel, size_t bytes)
{
    if (bytes <= 48 * 1024) return 0;
    static std::mutex mu;
    static std::set<std::pair<const void *, int>> done;
    int dev = 0;
    H3D_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair((const void *)kernel, dev);
    if (done.count(key)) return 0;
    H3D_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    done.insert(key);
    return 0;
}

#define H3D_DISPATCH(n, CALL)                          \
    switch (n) {                                       \
    case 32: return CALL(32);                          \
    case 48: return CALL(48);                          \
    case 64: return CALL(64);                          \
    case 128: return CALL(128);                        \
    case 256: return CALL(256);                        \
    case 512: return CALL(512);                        \
    case 1024: return CALL(1024);                      \
    default: return h3d_set_error_msg(-3, "unsupported grid size"); \
    }

static bool size_supported(int n)
{
    return n == 32 || n == 48 || n == 64 || n == 128 || n == 256 || n == 512 || n == 1024;
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// RANDu on the host (RANDu.f:12-52), bit-exact with the reference: the
// initial-condition stream stays on the host as the reference generates it.
// ---------------------------------------------------------------------------
namespace {
struct Randu {
    int64_t idum2 = 123456789, iy = 0, iv[32] = {0};
    double next(double idum3)
    {
        const int64_t im1 = 2147483563, im2 = 2147483399, imm1 = im1 - 1;
        const int64_t ia1 = 40014, ia2 = 40692, iq1 = 53668, iq2 = 52774;
        const int64_t ir1 = 12211, ir2 = 3791, ntab = 32, ndiv = 1 + imm1 / ntab;
        const double am = 1.0 / (double)im1, eps = 1.2e-7, rnmx = 1.0 - eps;
        int64_t idum = (int64_t)llround(idum3 / 987.0), k, j;
        if (idum <= 0) {
            idum = (-idum > 1) ? -idum : 1;
            idum2 = idum;
            for (j = ntab + 8; j >= 1; j--) {
                k = idum / iq1;
                idum = ia1 * (idum - k * iq1) - k * ir1;
                if (idum < 0) idum += im1;
                if (j <= ntab) iv[j - 1] = idum;
            }
        }
        k = idum / iq1;
        idum = ia1 * (idum - k * iq1) - k * ir1;
        if (idum < 0) idum += im1;
        k = idum2 / iq2;
        idum2 = ia2 * (idum2 - k * iq2) - k * ir2;
        if (idum2 < 0) idum2 += im2;
        j = 1 + iy / ndiv;
        iy = iv[j - 1] - idum2;
        iv[j - 1] = idum;
        if (iy < 1) iy += imm1;
        double r = am * (double)iy;
        return r < rnmx ? r : rnmx;
    }
};
}  // namespace

constexpr int kCopyStreams = 2;  // copy streams per direction of hit3d_gpu_step_host (4 measured slower)

struct hit3d_ctx {
    hit3d_params p;
    int n, nh, P64, P32, nsc, dev, kmax, nsm;
    int64_t fs64, fs32;
    cudaStream_t st;
    double2 *U, *RO, *RP, *SP;
    void *W;             // work fields in the transform precision
    int nw;
    int64_t wfs;         // complex elements per work field
    int wpitch;
    double2 *W64;        // FP64 scratch (3 fields) for statistics and the transform API
    double2 *sgs;        // FP64 scratch (9 fields) of the subgrid-stress data path, on first use
    double *phys;        // physical u,v,w [3][z][y][x] for particles
    double2 *tw64;
    float2 *tw32;
    double *d_fen, *d_part, *d_red, *d_ratio;
    unsigned long long *d_cmax;  // [0]: Courant maximum (bits of a double >= 0); [1]: the error word d_err
    int *d_err;          // device error word: bit 1 = a fused x pass gave up waiting for its input stage
    double2 *stage;      // one field in the reference layout
    double *d_xyz, *d_uvw;
    int64_t np;
    int pscheme;
    int int_scalars;
    double dx;
    int pblocks;
    int64_t nlaunch;
    int xcfg;            // launch-shape variant of the fused x pass
    int fuse_update;     // 1: z forward pass of the velocity products fused with the update
    int idle_passive;    // passive scalars waiting for TSCALAR while LES fields move
    Randu rng;           // RANDu state, carried from the velocity to the scalar initial
                         // conditions as the reference's module state is (RANDu.f:20-22)
    double k2max;        // truncation radius squared of PRE_TRUNC
    void *mlp_wb;        // bf16 weights of the learned closure (les_model HIT3D_LES_LEARNED)
    double mlp_delta;    // filter width the closure was trained for
    int mlp_clip;        // zero the stress where its dissipation is negative
    int mlp_kernel;      // 0: CUDA cores, 1: tensor cores for the hidden layers
    int *d_mlp_err;      // set by the tensor-core kernel when a completion wait runs out
    double *d_kmin;      // LES with k_sgs: minimum of k_sgs (slot 2), les.gp means, block sums
    double2 *gfilt;      // test filter transfer function of the Dynamic Structure models
    double2 *pfilt;      // particle filter transfer function (particles_filter_size > 0)
    double2 *pbuf;       // 3 FP64 fields: the filtered velocity the particles see
    const double2 *zfilt;  // filter of PRE_FILT when set (else gfilt)
    int prune_on;        // allow 2/3-rule pruning of the step's transforms
    int pruned;          // the state is zero beyond N/3 (checked), so pruning is exact
    int alias_known;     // `pruned` is up to date with the state
    int kc_active;       // >= 0 while a pruned step is being issued: the cutoff N/3
    // pipelined host transfers (hit3d_gpu_step_host), created on first use: copy
    // streams, staging fields in the reference layout and their events
    cudaStream_t cs_h2d, cs_d2h;
    // further copy streams per direction (the copies of one transfer are spread
    // over kCopyStreams streams, so that several copy engines share them) and
    // the events that join them back
    cudaStream_t cs_up[kCopyStreams - 1], cs_dn[kCopyStreams - 1];
    cudaEvent_t ev_up[kCopyStreams - 1], ev_dn[kCopyStreams - 1];
    double2 *sin, *sout[2];  // one input staging set, two output sets used in turn
    int nstage_io;           // fields each staging set holds
    cudaEvent_t ev_in_ready, ev_in_free, ev_out_ready, ev_out_free[2];
    int ext_bufs;        // U, RO and W belong to a batch's slab
    int ctile;           // column-tile shape of the plain strided passes (ColCfgT), grids up to 512
    // while a batch class is being stepped through this context (its first
    // run): the number of runs, and the run strides of the state (complex FP64
    // elements) and of the work fields (elements of the transform precision)
    int bruns;
    int64_t bru, brw;
};

int h3d_mlp_apply(cudaStream_t st, int fp64, int64_t np, int64_t n, int64_t rp, int64_t fs, double delta, int clip,
                  int kernel, const void *wb, void *G, int *err);

static int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

// ---------------------------------------------------------------------------
// transform passes (templated on the compute precision T)
// ---------------------------------------------------------------------------
template <typename T> static const cx<T> *twid(const hit3d_ctx *c);
template <> inline const double2 *twid<double>(const hit3d_ctx *c) { return c->tw64; }
template <> inline const float2 *twid<float>(const hit3d_ctx *c) { return c->tw32; }

