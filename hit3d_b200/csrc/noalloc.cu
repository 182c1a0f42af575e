// hit3d_gpu_xfft3d_static: the forward 3-D transform of one field for callers
// that cannot allocate device memory.
//
// Some hosts cannot call cudaMalloc at the point where they need a transform:
// a code whose device memory is entirely handed out by its own pool allocator
// (so a library allocation would fail or fragment that pool), or a time-critical
// loop that must not risk the device-wide synchronisation cudaMalloc/cudaFree
// can cause.  For them this entry point takes device input and output buffers
// from the caller and keeps its only scratch -- one intermediate field -- in a
// file-scope __device__ array, so it allocates nothing.
//
// Limits and rules:
//   * grid sizes up to N = 128 (the array holds one 65 x 128 x 128 complex
//     field, 17 MB); larger N is rejected with an error;
//   * every GPU that loads this library holds that array until the process exits;
//   * the first call in each CUDA context of a device resolves the array's
//     device address and uploads the twiddle tables (again after a device reset,
//     which creates a new context); make that first call before any stream
//     capture;
//   * all calls share the one array: calls whose work overlaps on the GPU (on
//     different streams, or from different threads) race on it and must be
//     serialised by the caller.  Nothing in the array needs to start at zero:
//     each call first copies its whole input into it;
//   * input and output may be the same buffer, or overlap: the whole input is
//     copied into the array, in stream order, before anything is written to the
//     output.
#include <cmath>
#include <mutex>
#include <vector>

#include <cuda.h>

#include "../../include/hit3d_gpu.h"
#include "launch_cfg.cuh"
#include "passes.cuh"

#define H3D_STATIC_MAX_N 128

static constexpr size_t kScratchElems = (size_t)(H3D_STATIC_MAX_N / 2 + 1) * H3D_STATIC_MAX_N * H3D_STATIC_MAX_N;
// twiddle tables exp(-2 pi i t/N) for N = 32, 48, 64, 128, back to back
static constexpr int kTwOff32 = 0, kTwOff48 = 32, kTwOff64 = 80, kTwOff128 = 144, kTwTotal = 272;

// The scratch field and the twiddles.  In host code these names are host-side
// stand-ins, not device addresses: host code only ever passes the addresses that
// cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) double2 g_fft_scratch[kScratchElems];
static __device__ __align__(256) double2 g_fft_twiddles[kTwTotal];

namespace {

struct DevState {
    bool ready = false;
    unsigned long long ctx_id = 0;  // CUDA context the addresses below belong to
    double2 *scratch = nullptr;     // device address of g_fft_scratch in that context
    double2 *tw = nullptr;          // device address of g_fft_twiddles in that context
};
constexpr int kMaxDevices = 64;
DevState g_dev[kMaxDevices];
std::mutex g_mu;

// unique id of the current CUDA context (driver entry points reached through the
// runtime, so the library needs no link against libcuda); a device reset or a
// re-created primary context gives a new id
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);
int current_ctx_id(unsigned long long *id)
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void *f0 = nullptr, *f1 = nullptr;
        cudaDriverEntryPointQueryResult q0 = cudaDriverEntryPointSymbolNotFound, q1 = cudaDriverEntryPointSymbolNotFound;
        cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f0, 12000, cudaEnableDefault, &q0);
        if (e == cudaSuccess) e = cudaGetDriverEntryPointByVersion("cuCtxGetId", &f1, 12000, cudaEnableDefault, &q1);
        if (e != cudaSuccess) return h3d_set_error(e, "cudaGetDriverEntryPointByVersion", __FILE__, __LINE__);
        if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
            return h3d_set_error_msg(-2, "hit3d_gpu_xfft3d_static: driver lacks cuCtxGetCurrent/cuCtxGetId");
        get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
        get_id = reinterpret_cast<CtxGetIdFn>(f1);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return h3d_set_error_msg(-2, "hit3d_gpu_xfft3d_static: no current CUDA context");
    if (get_id(ctx, id) != CUDA_SUCCESS) return h3d_set_error_msg(-2, "hit3d_gpu_xfft3d_static: cuCtxGetId failed");
    return 0;
}

int tw_offset(int n)
{
    return n == 32 ? kTwOff32 : n == 48 ? kTwOff48 : n == 64 ? kTwOff64 : kTwOff128;
}

// once per device and CUDA context, with that device current
int setup_device(int dev)
{
    std::lock_guard<std::mutex> lk(g_mu);
    DevState &s = g_dev[dev];
    unsigned long long id = 0;
    int rc = current_ctx_id(&id);
    if (rc) return rc;
    if (s.ready && s.ctx_id == id) return 0;
    s.ready = false;
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_fft_scratch);
    if (e != cudaSuccess) return h3d_set_error(e, "cudaGetSymbolAddress(g_fft_scratch)", __FILE__, __LINE__);
    s.scratch = static_cast<double2 *>(p);
    e = cudaGetSymbolAddress(&p, g_fft_twiddles);
    if (e != cudaSuccess) return h3d_set_error(e, "cudaGetSymbolAddress(g_fft_twiddles)", __FILE__, __LINE__);
    s.tw = static_cast<double2 *>(p);
    double2 host[kTwTotal];
    const long double twopi = 6.283185307179586476925286766559005768L;
    const int sizes[4] = {32, 48, 64, 128};
    for (int q = 0; q < 4; q++) {
        const int n = sizes[q], off = tw_offset(n);
        for (int t = 0; t < n; t++) {
            long double a = twopi * (long double)t / (long double)n;
            host[off + t] = make_double2((double)cosl(a), (double)(-sinl(a)));
        }
    }
    e = cudaMemcpyToSymbol(g_fft_twiddles, host, sizeof host);
    if (e != cudaSuccess) return h3d_set_error(e, "cudaMemcpyToSymbol(g_fft_twiddles)", __FILE__, __LINE__);
    s.ctx_id = id;
    s.ready = true;
    return 0;
}

template <int L> int run(const DevState &s, const double *in, double *out, cudaStream_t st)
{
    const int n = L, nh = L / 2 + 1;
    const double2 *tw = s.tw + tw_offset(n);
    double2 *w = s.scratch;
    cudaError_t e = cudaMemcpyAsync(w, in, sizeof(double2) * (size_t)nh * n * n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return h3d_set_error(e, "cudaMemcpyAsync", __FILE__, __LINE__);
    // the launch shapes of the context path's passes (RowCfg, ColCfg), all
    // within the default 48 KB of dynamic shared memory, so no attribute call
    using RC = RowCfg<double, L>;
    using CY = ColCfg<double, L, true>;
    using CZ = ColCfg<double, L, false>;
    static_assert(RC::SMEM <= 48 * 1024 && CY::SMEM <= 48 * 1024 && CZ::SMEM <= 48 * 1024,
                  "static transform: shared memory above the default limit");
    // x: r2c of row pairs, in place (row pitch nh complex = the reference's nx+2 reals)
    {
        const int npairs = n * n / 2;
        k_xr2c<double, L, RC::TC, RC::NT, double><<<(npairs + RC::TC - 1) / RC::TC, RC::NT, RC::SMEM, st>>>(
            w, 0, nh, npairs, tw, 0);
    }
    // y: in place, [z][ky][kx]
    {
        IOPlain<double, double, double> io;
        io.src = w; io.dst = w; io.fs_src = io.fs_dst = 0; io.ncol = nh;
        io.sa_src = io.sa_dst = nh;
        io.so_src = io.so_dst = (int64_t)n * nh;
        dim3 g((nh + CY::TC - 1) / CY::TC, n, 1);
        k_colfft<double, L, CY::TC, CY::NT, true, IOPlain<double, double, double>><<<g, CY::NT, CY::SMEM, st>>>(io, tw);
    }
    // z: out of place into the caller's array, transposed to (kx, kz, ky)
    {
        IOPlain<double, double, double> io;
        io.src = w; io.dst = reinterpret_cast<double2 *>(out); io.fs_src = io.fs_dst = 0; io.ncol = nh;
        io.sa_src = (int64_t)n * nh; io.so_src = nh;   // source [z][ky][kx]: z is the axis, ky the outer index
        io.sa_dst = nh; io.so_dst = (int64_t)n * nh;   // destination [ky][kz][kx]
        dim3 g((nh + CZ::TC - 1) / CZ::TC, n, 1);
        k_colfft<double, L, CZ::TC, CZ::NT, true, IOPlain<double, double, double>><<<g, CZ::NT, CZ::SMEM, st>>>(io, tw);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return h3d_set_error(e, "kernel launch", __FILE__, __LINE__);
    return 0;
}

}  // namespace

extern "C" int hit3d_gpu_xfft3d_static(int32_t n, const double *in, double *out, void *stream)
{
    if (n > H3D_STATIC_MAX_N)
        return h3d_set_error_msg(-3, "hit3d_gpu_xfft3d_static: N exceeds the static scratch limit (N <= 128)");
    if (n != 32 && n != 48 && n != 64 && n != 128)
        return h3d_set_error_msg(-3, "hit3d_gpu_xfft3d_static: grid size must be 32, 48, 64 or 128");
    if (!in || !out) return h3d_set_error_msg(-1, "hit3d_gpu_xfft3d_static: null argument");
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15)
        return h3d_set_error_msg(-1, "hit3d_gpu_xfft3d_static: buffers must be 16-byte aligned");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return h3d_set_error(e, "cudaGetDevice", __FILE__, __LINE__);
    if (dev < 0 || dev >= kMaxDevices) return h3d_set_error_msg(-1, "hit3d_gpu_xfft3d_static: device ordinal too large");
    int rc = setup_device(dev);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (n) {
    case 32: return run<32>(g_dev[dev], in, out, st);
    case 48: return run<48>(g_dev[dev], in, out, st);
    case 64: return run<64>(g_dev[dev], in, out, st);
    default: return run<128>(g_dev[dev], in, out, st);
    }
}
