// The z forward pass of the six velocity products fused with the 2/3-rule
// update (rhs_velocity.f90:85-142, m_force.f90:158-171, main.f90:156-164,
// pressure.f90:13-47).  A CTA owns TC kx columns of one ky row: it transforms
// the six product columns along z one after the other and, as each last-stage
// butterfly comes out, adds k_j P_ij into per-thread accumulators of the three
// RHS components (every transform hands a thread the same output slots).  The
// epilogue then does, for the thread's own modes, what k_update_vel_23 does:
// RHS = -i k_j P_ij - nu k^2 u (zero where ialias > 0), band forcing, AB2 and
// the projection.  The six product spectra are never written to HBM and read
// back, which is the traffic this saves against the separate z pass + update.
#pragma once
#include "fft.cuh"
#include "passes.cuh"
#include "spectral.cuh"

template <typename T, int L> struct ZUpdCfg {
    // 32-byte column segments; 8 output slots per thread
    static constexpr int TC = sizeof(T) == 8 ? 2 : 4;
    static constexpr int NT0 = TC * L / 8;
    static constexpr int NT = NT0 < 32 ? 32 : NT0 > 512 ? 512 : NT0;
    static constexpr int MINB = NT <= 128 ? 3 : 1;
    // transform buffer, then the stage that receives the next product's columns
    static constexpr size_t SOFF = ((size_t)Lay<L, TC, false>::elems * sizeof(cx<T>) + 15) / 16 * 16;
    static constexpr size_t SMEM = SOFF + (size_t)TC * L * sizeof(cx<T>);
};

// copy the TC columns (kx = col0 ...) of product f, row ky, all z, into the
// stage [z][c] with 16-byte cp.async (TC * sizeof(cx<T>) = 32 bytes per z)
template <typename T, int L, int TC, int NT>
H3D_D void zupd_stage(const StepArgs &a, const cx<T> *__restrict__ P, int f, int kyi, int col0, int ncol,
                      cx<T> *st)
{
    constexpr int PER = 16 / (int)sizeof(cx<T>), NCH = TC / PER;
    const cx<T> *src = P + f * a.pfs + (int64_t)kyi * a.ppitch + col0;
    for (int q = threadIdx.x; q < L * NCH; q += NT) {
        const int p = q / NCH, ch = q - p * NCH;
        if (col0 + ch * PER < ncol) cp_async16(st + p * TC + ch * PER, src + (int64_t)p * a.n * a.ppitch + ch * PER);
    }
    cp_async_commit();
}

template <typename T, int L, int TC, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_zfwd_update(const StepArgs a, const cx<T> *__restrict__ P, int ncol,
                                                          double2 *__restrict__ U, double2 *__restrict__ RO,
                                                          const cx<T> *__restrict__ tw)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    cx<T> *st = reinterpret_cast<cx<T> *>(smraw + ZUpdCfg<T, L>::SOFF);
    using F = ColFFT<T, L, TC, NT, false, true, false>;
    const int n = a.n, kc = a.kc;
    const int col0 = blockIdx.x * TC;
    const int kyi = kc >= 0 ? kept_index(blockIdx.y, n, kc) : (int)blockIdx.y;
    const double ky = kwave(kyi, n);
    // acc[c] = k_x P_c1 + k_y P_c2 + k_z P_c3, summed in that order
    double2 acc[3][F::NOUT];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int q = 0; q < F::NOUT; q++) acc[c][q] = make_double2(0.0, 0.0);
    zupd_stage<T, L, TC, NT>(a, P, 0, kyi, col0, ncol, st);
#pragma unroll
    for (int f = 0; f < 6; f++) {
        cx<T> in[F::NIN];
        cp_async_wait_all();
        __syncthreads();  // the stage holds product f; the previous transform has read sm
#pragma unroll
        for (int i = 0; i < F::NB0; i++)
#pragma unroll
            for (int m = 0; m < F::R0; m++) {
                int c, p;
                if (F::in_slot(i, m, c, p)) in[i * F::R0 + m] = col0 + c < ncol ? st[p * TC + c] : mk<T>(0, 0);
            }
        __syncthreads();  // the stage is free: fetch the next product while this one transforms
        if (f < 5) zupd_stage<T, L, TC, NT>(a, P, f + 1, kyi, col0, ncol, st);
        F::run_slots_t(in, sm, GlobalTw<T>{tw}, [&](int i, int m, int c, int p, cx<T> v) {
            const int q = i * F::RL + m;
            const double kx = (double)(col0 + c), kz = (double)kwave(p, n);
            const double vx = (double)v.x, vy = (double)v.y;
            // products uu uv uw vv vw ww
            if (f == 0) { acc[0][q] = make_double2(kx * vx, kx * vy); }
            if (f == 1) {
                acc[0][q] = make_double2(acc[0][q].x + ky * vx, acc[0][q].y + ky * vy);
                acc[1][q] = make_double2(kx * vx, kx * vy);
            }
            if (f == 2) {
                acc[0][q] = make_double2(acc[0][q].x + kz * vx, acc[0][q].y + kz * vy);
                acc[2][q] = make_double2(kx * vx, kx * vy);
            }
            if (f == 3) { acc[1][q] = make_double2(acc[1][q].x + ky * vx, acc[1][q].y + ky * vy); }
            if (f == 4) {
                acc[1][q] = make_double2(acc[1][q].x + kz * vx, acc[1][q].y + kz * vy);
                acc[2][q] = make_double2(acc[2][q].x + ky * vx, acc[2][q].y + ky * vy);
            }
            if (f == 5) { acc[2][q] = make_double2(acc[2][q].x + kz * vx, acc[2][q].y + kz * vy); }
        });
    }
    const double fac = (a.flow_type == 1) ? a.famp / *a.fenergy : 0.0;
    const double rn3 = (double)(n / 3);
#pragma unroll
    for (int i = 0; i < F::NBL; i++)
#pragma unroll
        for (int m = 0; m < F::RL; m++) {
            int c, p;
            if (!F::out_slot(i, m, c, p)) continue;
            const int kx = col0 + c;
            if (kx >= ncol || (kc >= 0 && !kept(p, n, kc))) continue;
            const int q = i * F::RL + m;
            ModeIdx md;
            md.kx = kx; md.kyi = kyi; md.kzi = p;
            md.ax = kx; md.ay = ky; md.az = kwave(p, n);
            md.ialias = (fabs(md.ay) > rn3) + (fabs(md.az) > rn3) + (fabs(md.ax) > rn3);
            const int64_t o = soff(md, n, a.pitch);
            double2 u[3] = {U[o], U[o + a.fs], U[o + 2 * a.fs]};
            double2 r[3];
            if (md.ialias > 0) {
                r[0] = r[1] = r[2] = make_double2(0.0, 0.0);
            } else {
                const double t4 = -a.nu * (md.ax * md.ax + md.ay * md.ay + md.az * md.az);
#pragma unroll
                for (int cc = 0; cc < 3; cc++) {
                    const double2 tt = make_double2(-acc[cc][q].x, -acc[cc][q].y);
                    r[cc] = make_double2(-tt.y + t4 * u[cc].x, tt.x + t4 * u[cc].y);
                }
            }
            if (a.flow_type == 1 && forced(md, n, a.kfmax)) {
#pragma unroll
                for (int cc = 0; cc < 3; cc++) { r[cc].x = r[cc].x + fac * u[cc].x; r[cc].y = r[cc].y + fac * u[cc].y; }
            }
            double2 ro[3] = {RO[o], RO[o + a.fs], RO[o + 2 * a.fs]};
#pragma unroll
            for (int cc = 0; cc < 3; cc++) ab2(u[cc], ro[cc], r[cc], a.dt, a.euler_v);
            project(md, u[0], u[1], u[2]);
#pragma unroll
            for (int cc = 0; cc < 3; cc++) { U[o + cc * a.fs] = u[cc]; RO[o + cc * a.fs] = ro[cc]; }
        }
}
