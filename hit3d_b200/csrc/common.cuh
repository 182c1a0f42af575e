// Common types and helpers for the sm_100a kernels of the pseudospectral step.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define H3D_HD __host__ __device__ __forceinline__
#define H3D_D __device__ __forceinline__

// complex number traits: double -> double2, float -> float2
template <typename T> struct cx_t;
template <> struct cx_t<double> { using type = double2; };
template <> struct cx_t<float> { using type = float2; };
template <typename T> using cx = typename cx_t<T>::type;

template <typename T> H3D_HD cx<T> mk(T x, T y) { cx<T> r; r.x = x; r.y = y; return r; }
H3D_HD double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
H3D_HD double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
H3D_HD float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
H3D_HD float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
H3D_HD double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
H3D_HD float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
H3D_HD double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
H3D_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
H3D_HD double2 conjg(double2 a) { return make_double2(a.x, -a.y); }
H3D_HD float2 conjg(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (fwd) or +i (bwd)
template <bool FWD> H3D_HD double2 mul_mi(double2 a) { return FWD ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x); }
template <bool FWD> H3D_HD float2 mul_mi(float2 a) { return FWD ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x); }

template <typename T> H3D_HD cx<T> to_cx(double2 v) { return mk<T>((T)v.x, (T)v.y); }
template <typename T> H3D_HD cx<T> to_cx(float2 v) { return mk<T>((T)v.x, (T)v.y); }

// Geometry of one field on the device.
//   spectral:  complex [kz][ky][kx], kx in [0, N/2], row pitch P complex
//   physical:  real    [z][y][x],    x in [0, N),   row pitch 2P reals
//   after the x and y forward passes (and before the last inverse pass) a field
//   is complex [z][ky][kx] with the same pitch.
struct Geom {
    int n;       // grid size N (cubic)
    int nh;      // N/2 + 1
    int pitch;   // row pitch in complex elements (>= nh, multiple of 8 for FP64, 16 for FP32)
    int64_t fsz; // complex elements per field = n * n * pitch
};

// signed wavenumber of index i on an axis of length n: i > n/2 maps to i - n,
// so +N/2 stays positive (x_fftw.f90:280-296)
H3D_HD int kwave(int i, int n) { return (2 * i > n) ? i - n : i; }

// nint(sqrt(real(k2,4))): shell index with a float32 square root
// (m_stats.f90:218, m_force.f90:270)
H3D_D int shell32(double k2) { return (int)lroundf(sqrtf((float)k2)); }

#define H3D_CHECK(x)                                                             \
    do {                                                                         \
        cudaError_t e__ = (x);                                                   \
        if (e__ != cudaSuccess) return h3d_set_error(e__, #x, __FILE__, __LINE__); \
    } while (0)

int h3d_set_error(cudaError_t e, const char *what, const char *file, int line);
int h3d_set_error_msg(int code, const char *msg);
