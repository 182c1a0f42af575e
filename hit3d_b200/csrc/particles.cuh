// Lagrangian particle advance (m_particles.f90:815-1230, 1451-1508): trilinear or
// 4-point cubic (CINT) interpolation of the level-n physical velocity, then
// Adams-Bashforth 2 (Euler on the first step) in grid units.  The whole field is
// resident, so the reference's slab halos and migration are periodic wrap-around.
#pragma once
#include "common.cuh"

struct PartArgs {
    int n;
    int scheme;               // 0 trilinear, 1 CINT
    int64_t np;
    double dt, dx;
    const double *U;          // physical u,v,w: [f][z][y][x], row pitch rp, field stride fs
    int64_t fs, rp;
    double *xyz, *uvw;        // (np, 3) each, particle-major as xyzp(3,np)
};

H3D_D void cint_r(double x, double *r)
{
    double s = (x - 1.0) * (x - 2.0);
    r[0] = -x * s;
    r[1] = 3.0 * (x + 1.0) * s;
    s = (x + 1.0) * x;
    r[2] = -3.0 * s * (x - 2.0);
    r[3] = s * (x - 1.0);
}
H3D_D double cint1(double p1, double p2, double p3, double p4, const double *r)
{
    return (r[0] * p1 + r[1] * p2 + r[2] * p3 + r[3] * p4) / 6.0;
}

// Three lanes per particle, one per velocity component, ten particles per warp
// (lanes 30 and 31 idle): each lane gathers its component's stencil (64 points
// for CINT, 8 for trilinear) and advances its own coordinate, with the
// arithmetic of the one-lane-per-particle form component by component.  The
// first-step flag V[0] and every coordinate are read before any lane of the
// particle writes (__syncwarp between).
constexpr int kPartPerWarp = 10;

__global__ void __launch_bounds__(256, 2) k_particles(const PartArgs a)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t p = warp * kPartPerWarp + lane / 3;
    const int c = lane - 3 * (lane / 3);
    const bool active = lane < 3 * kPartPerWarp && p < a.np;
    const int n = a.n;
    double *X = a.xyz + 3 * p, *V = a.uvw + 3 * p;
    double x0 = 0.0, y0 = 0.0, z0 = 0.0, v0 = 0.0, vc = 0.0;
    if (active) {
        x0 = X[0]; y0 = X[1]; z0 = X[2];
        v0 = V[0]; vc = V[c];
    }
    __syncwarp();
    if (!active) return;
    int i = (int)floor(x0), j = (int)floor(y0), k = (int)floor(z0);
    double xp = x0 - (double)i, yp = y0 - (double)j, zp = z0 - (double)k;
    // keep every cell index inside [1, n]: a coordinate that landed exactly on
    // n+1 (fraction 1.0 after a step) would otherwise read past the field
    i = ((i - 1) % n + n) % n + 1;
    j = ((j - 1) % n + n) % n + 1;
    k = ((k - 1) % n + n) % n + 1;
    // 1-based indices of the reference -> 0-based offsets, periodic
    const int64_t rp = a.rp;
    auto idx = [n, rp](int ii, int jj, int kk) -> int64_t {
        return (int64_t)(ii - 1) + rp * ((int64_t)(jj - 1) + (int64_t)n * (int64_t)(kk - 1));
    };
    const double *f = a.U + c * a.fs;
    double up;
    if (a.scheme == 0) {
        double c1 = (1.0 - xp) * (1.0 - yp) * (1.0 - zp);
        double c2 = (xp) * (1.0 - yp) * (1.0 - zp);
        double c3 = (1.0 - xp) * (yp) * (1.0 - zp);
        double c4 = (xp) * (yp) * (1.0 - zp);
        double c5 = (1.0 - xp) * (1.0 - yp) * (zp);
        double c6 = (xp) * (1.0 - yp) * (zp);
        double c7 = (1.0 - xp) * (yp) * (zp);
        double c8 = (xp) * (yp) * (zp);
        int i1 = (i == n) ? 1 : i + 1, j1 = (j == n) ? 1 : j + 1, k1 = (k == n) ? 1 : k + 1;
        double s = c1 * f[idx(i, j, k)] + c2 * f[idx(i1, j, k)] + c3 * f[idx(i, j1, k)] + c4 * f[idx(i1, j1, k)];
        s = s + c5 * f[idx(i, j, k1)] + c6 * f[idx(i1, j, k1)] + c7 * f[idx(i, j1, k1)] + c8 * f[idx(i1, j1, k1)];
        up = s;
    } else {
        double rx[4], ry[4], rz[4];
        cint_r(xp, rx);
        cint_r(yp, ry);
        cint_r(zp, rz);
        int ii[4], jj[4], kk[4];
        for (int q = 0; q < 4; q++) {
            int t = i - 2 + q + 1; if (t < 1) t += n; if (t > n) t -= n; ii[q] = t;
            t = j - 2 + q + 1; if (t < 1) t += n; if (t > n) t -= n; jj[q] = t;
            t = k - 2 + q + 1; if (t < 1) t += n; if (t > n) t -= n; kk[q] = t;
        }
        double t1[4];
        for (int kq = 0; kq < 4; kq++) {
            double t2[4];
            for (int jq = 0; jq < 4; jq++) {
                t2[jq] = cint1(f[idx(ii[0], jj[jq], kk[kq])], f[idx(ii[1], jj[jq], kk[kq])],
                               f[idx(ii[2], jj[jq], kk[kq])], f[idx(ii[3], jj[jq], kk[kq])], rx);
            }
            t1[kq] = cint1(t2[0], t2[1], t2[2], t2[3], ry);
        }
        up = cint1(t1[0], t1[1], t1[2], t1[3], rz);
    }
    const double dx = a.dx, dt = a.dt;
    // this lane's coordinate: fraction and 1-based cell
    double fr = c == 0 ? xp : c == 1 ? yp : zp;
    int cell = c == 0 ? i : c == 1 ? j : k;
    if (v0 == -999.0) fr = fr + dt * up / dx;
    else fr = fr + (1.50 * up - 0.50 * vc) * dt / dx;
    V[c] = up;
    if (c < 2) {
        if (fr > 1.0) { fr = fr - 1.0; cell = cell + 1; if (cell > n) cell = cell - n; }
        if (fr < 0.0) { fr = fr + 1.0; cell = cell - 1; if (cell < 1) cell = cell + n; }
        X[c] = fr + (double)cell;
    } else {
        if (fr > 1.0) { fr = fr - 1.0; cell = cell + 1; }
        if (fr < 0.0) { fr = fr + 1.0; cell = cell - 1; }
        double zn = fr + (double)cell;
        // migration between slabs on one periodic slab (m_particles.f90:1270-1319)
        if (zn >= (double)(n + 1)) zn = zn - (double)n;
        else if (zn < 1.0) zn = zn + (double)n;
        X[2] = zn;
    }
}

// CTAs of 256 threads for np particles (ten per warp)
inline unsigned particle_blocks(int64_t np)
{
    const int64_t warps = (np + kPartPerWarp - 1) / kPartPerWarp;
    return (unsigned)((warps * 32 + 255) / 256);
}
