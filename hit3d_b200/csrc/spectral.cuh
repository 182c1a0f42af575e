// Pointwise spectral kernels of the step: RHS assembly with dealiasing masks,
// band forcing, Adams-Bashforth update and pressure projection fused in one
// pass over the modes; plus forcing energy, dealias, shell spectra, reductions
// and initial-condition shaping.
#pragma once
#include "common.cuh"

struct ModeIdx {
    int kx, kyi, kzi;       // kx in [0, N/2], ky/kz storage indices
    double ax, ay, az;      // signed wavenumbers akx, aky, akz
    int ialias;             // number of |k_i| > N/3 (x_fftw.f90:298-310)
};

H3D_D ModeIdx mode_from(int kx, int kyi, int kzi, int n)
{
    ModeIdx m;
    m.kx = kx;
    m.kyi = kyi;
    m.kzi = kzi;
    m.ax = m.kx;
    m.ay = kwave(m.kyi, n);
    m.az = kwave(m.kzi, n);
    const double rn3 = (double)(n / 3);
    m.ialias = (fabs(m.ay) > rn3) + (fabs(m.az) > rn3) + (fabs(m.ax) > rn3);
    return m;
}
H3D_D ModeIdx mode_of(int64_t t, int n, int nh)
{
    const int64_t r = t / nh;
    return mode_from((int)(t % nh), (int)(r % n), (int)(r / n), n);
}
H3D_D int64_t soff(const ModeIdx &m, int n, int pitch) { return ((int64_t)m.kzi * n + m.kyi) * pitch + m.kx; }

// Mode loops of the 2/3-rule updates.  kc < 0: every mode (index t over
// N x N x (N/2+1)).  kc >= 0 (pruned state: U and RO are zero wherever some
// |k_i| > kc and the update keeps them zero): only the kept modes, t over
// (kc+1) x (2kc+1)^2 with kx fastest, so that masked modes are neither read nor
// written.
H3D_D int64_t mode_count(int n, int nh, int kc)
{
    return kc < 0 ? (int64_t)n * n * nh : (int64_t)(kc + 1) * (2 * kc + 1) * (2 * kc + 1);
}
H3D_D ModeIdx mode_at(int64_t t, int n, int nh, int kc)
{
    if (kc < 0) return mode_of(t, n, nh);
    const int nk = 2 * kc + 1;
    const int kx = (int)(t % (kc + 1));
    const int64_t r = t / (kc + 1);
    const int yc = (int)(r % nk), zc = (int)(r / nk);
    const int kyi = yc <= kc ? yc : n - (nk - yc), kzi = zc <= kc ? zc : n - (nk - zc);
    return mode_of(((int64_t)kzi * n + kyi) * nh + kx, n, nh);
}

// t / d for 0 <= t by a multiply-high with m = ceil(2^64 / d), exact while
// t * d < 2^64 (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994): the per-step mode loops prepare their divisors
// once per thread instead of dividing 64-bit integers at every mode.
struct DivU64 {
    uint64_t m;
    int64_t d;
    H3D_D explicit DivU64(int64_t d_) : m(~0ull / (uint64_t)d_ + 1ull), d(d_) {}  // d = 1 wraps m to 0
    H3D_D int64_t operator()(int64_t t) const { return m ? (int64_t)__umul64hi((uint64_t)t, m) : t; }
};

// mode_at with the divisors prepared: index t of the loop over every mode
// (kc < 0) or over the kept modes (kc >= 0) -> the mode
struct ModeLoop {
    DivU64 dx, dy;
    int n, kc;
    H3D_D ModeLoop(int n_, int nh, int kc_) : dx(kc_ < 0 ? nh : kc_ + 1), dy(kc_ < 0 ? n_ : 2 * kc_ + 1), n(n_), kc(kc_) {}
    H3D_D ModeIdx at(int64_t t) const
    {
        const int64_t r = dx(t), zc = dy(r);
        const int kx = (int)(t - r * dx.d), yc = (int)(r - zc * dy.d);
        int kyi = yc, kzi = (int)zc;
        if (kc >= 0) {
            const int nk = 2 * kc + 1;
            kyi = kyi <= kc ? kyi : n - (nk - kyi);
            kzi = kzi <= kc ? kzi : n - (nk - kzi);
        }
        return mode_from(kx, kyi, kzi, n);
    }
};

// Machiels band forcing: a mode takes part when kx < N/2 (the reference loops
// over real indices 1..nx) and its float32 shell index is in [1, kfmax]
// (m_force.f90:166-209).
H3D_D bool forced(const ModeIdx &m, int n, int kfmax)
{
    if (kfmax <= 0 || m.kx >= n / 2) return false;
    double k2 = m.ax * m.ax + m.ay * m.ay + m.az * m.az;
    if (k2 > (kfmax + 1.0) * (kfmax + 1.0)) return false;
    int sh = shell32(k2);
    return sh > 0 && sh <= kfmax;
}

// pressure projection of one mode (pressure.f90:13-47)
H3D_D void project(const ModeIdx &m, double2 &u, double2 &v, double2 &w)
{
    double kx = m.ax, ky = m.ay, kz = m.az;
    double div2 = kx * u.x + ky * v.x + kz * w.x;
    double div1 = -(kx * u.y + ky * v.y + kz * w.y);
    double l = kx * kx + ky * ky + kz * kz;
    if (l == 0.0) l = 9e20;
    double p1 = -div1 / l, p2 = -div2 / l;
    u.x = u.x + p2 * kx; u.y = u.y - p1 * kx;
    v.x = v.x + p2 * ky; v.y = v.y - p1 * ky;
    w.x = w.x + p2 * kz; w.y = w.y - p1 * kz;
}

// Adams-Bashforth 2 (Euler on the first step) of one mode (main.f90:156-164)
H3D_D void ab2(double2 &f, double2 &ro, double2 r, double dt, bool euler)
{
    if (euler) {
        ro = r;
        f.x = f.x + dt * ro.x;
        f.y = f.y + dt * ro.y;
    } else {
        f.x = f.x + dt * (1.5 * r.x - 0.5 * ro.x);
        f.y = f.y + dt * (1.5 * r.y - 0.5 * ro.y);
        ro = r;
    }
}

template <typename TP> H3D_D double2 ld2(const cx<TP> *p, int64_t i)
{
    cx<TP> v = p[i];
    return make_double2((double)v.x, (double)v.y);
}

struct StepArgs {
    int n, nh, pitch, ppitch;  // state pitch, product pitch
    int64_t fs, pfs;           // state / product field strides (complex elements)
    double nu, dt;
    int euler_v, euler_s;
    int flow_type, kfmax;
    double famp;
    const double *fenergy;     // device: energy in the forcing band
    int nscal;
    double pe[8];
    int stype[8];
    int kc;                    // >= 0: visit only the modes the 2/3 rule keeps (pruned state)
    int idle;                  // passive scalars 0..idle-1 wait for TSCALAR while LES fields move:
                               // no advection or molecular diffusion, only sources and LES fluxes
    // runs of a batch (k_update_vel_23 over gridDim.y runs): run r's state starts
    // r * ru elements after run 0's and its product fields r * rp after; nu_r
    // and dt_r (when set) hold each run's viscosity and time step, and fenergy
    // each run's forcing-band energy
    int64_t ru, rp;
    const double *nu_r, *dt_r;
};

// s = k_x a + k_y b + k_z c rounded in that order (one product, then two fused
// multiply-adds), so that the separate update and the z pass fused with the
// update (which adds the products as their transforms come out) agree exactly
H3D_D double kdot3(double kx, double a, double ky, double b, double kz, double c)
{
    return __fma_rn(kz, c, __fma_rn(ky, b, __dmul_rn(kx, a)));
}

// RHS of one mode with ialias == 0 (rhs_velocity.f90:85-142): -i k_j P_cj - nu k^2 u_c
// from the sums s_c = k_j P_cj
H3D_D void vel23_rhs(const ModeIdx &m, const double2 (&s)[3], const double2 (&u)[3], double nu, double2 (&r)[3])
{
    const double kx = m.ax, ky = m.ay, kz = m.az;
    const double t4 = -nu * (kx * kx + ky * ky + kz * kz);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const double2 tt = make_double2(-s[c].x, -s[c].y);
        r[c] = make_double2(-tt.y + t4 * u[c].x, tt.x + t4 * u[c].y);
    }
}

// 2/3 rule (rhs_velocity.f90:85-142) + forcing + AB2 + pressure.
// P: six product spectra [uu uv uw vv vw ww]; U, RO: velocity state and old RHS
// TAU (optional, Smagorinsky): six subgrid-stress spectra [t11 t12 t13 t22 t23 t33]
// added where ialias == 0 (les_rhsv_turb_visc, m_les.f90:941-1015)
template <typename TP>
__global__ void k_update_vel_23(const StepArgs a, const cx<TP> *__restrict__ P, const cx<TP> *__restrict__ TAU,
                                double2 *__restrict__ U, double2 *__restrict__ RO)
{
    const int64_t nm = mode_count(a.n, a.nh, a.kc);
    const int run = blockIdx.y;
    U += run * a.ru;
    RO += run * a.ru;
    P += run * a.rp;
    const double nu = a.nu_r != nullptr ? a.nu_r[run] : a.nu, dt = a.dt_r != nullptr ? a.dt_r[run] : a.dt;
    const double fac = (a.flow_type == 1) ? a.famp / a.fenergy[run] : 0.0;
    const ModeLoop ml(a.n, a.nh, a.kc);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        ModeIdx m = ml.at(t);
        int64_t o = soff(m, a.n, a.pitch), po = soff(m, a.n, a.ppitch);
        double2 u[3] = {U[o], U[o + a.fs], U[o + 2 * a.fs]};
        double2 r[3];
        if (m.ialias > 0) {
            r[0] = r[1] = r[2] = make_double2(0.0, 0.0);
        } else {
            double2 p11 = ld2<TP>(P, po), p12 = ld2<TP>(P, po + a.pfs), p13 = ld2<TP>(P, po + 2 * a.pfs);
            double2 p22 = ld2<TP>(P, po + 3 * a.pfs), p23 = ld2<TP>(P, po + 4 * a.pfs), p33 = ld2<TP>(P, po + 5 * a.pfs);
            double kx = m.ax, ky = m.ay, kz = m.az;
            const double2 s[3] = {make_double2(kdot3(kx, p11.x, ky, p12.x, kz, p13.x), kdot3(kx, p11.y, ky, p12.y, kz, p13.y)),
                                  make_double2(kdot3(kx, p12.x, ky, p22.x, kz, p23.x), kdot3(kx, p12.y, ky, p22.y, kz, p23.y)),
                                  make_double2(kdot3(kx, p13.x, ky, p23.x, kz, p33.x), kdot3(kx, p13.y, ky, p23.y, kz, p33.y))};
            vel23_rhs(m, s, u, nu, r);
            if (TAU != nullptr) {
                double2 s11 = ld2<TP>(TAU, po), s12 = ld2<TP>(TAU, po + a.pfs), s13 = ld2<TP>(TAU, po + 2 * a.pfs);
                double2 s22 = ld2<TP>(TAU, po + 3 * a.pfs), s23 = ld2<TP>(TAU, po + 4 * a.pfs), s33 = ld2<TP>(TAU, po + 5 * a.pfs);
                r[0].x = r[0].x + kx * s11.y + ky * s12.y + kz * s13.y;
                r[0].y = r[0].y - kx * s11.x - ky * s12.x - kz * s13.x;
                r[1].x = r[1].x + kx * s12.y;
                r[1].y = r[1].y - kx * s12.x;
                r[2].x = r[2].x + kx * s13.y;
                r[2].y = r[2].y - kx * s13.x;
                r[1].x = r[1].x + ky * s22.y + kz * s23.y;
                r[1].y = r[1].y - ky * s22.x - kz * s23.x;
                r[2].x = r[2].x + ky * s23.y + kz * s33.y;
                r[2].y = r[2].y - ky * s23.x - kz * s33.x;
            }
        }
        if (a.flow_type == 1 && forced(m, a.n, a.kfmax)) {
#pragma unroll
            for (int c = 0; c < 3; c++) { r[c].x = r[c].x + fac * u[c].x; r[c].y = r[c].y + fac * u[c].y; }
        }
        double2 ro[3] = {RO[o], RO[o + a.fs], RO[o + 2 * a.fs]};
#pragma unroll
        for (int c = 0; c < 3; c++) ab2(u[c], ro[c], r[c], dt, a.euler_v);
        project(m, u[0], u[1], u[2]);
#pragma unroll
        for (int c = 0; c < 3; c++) { U[o + c * a.fs] = u[c]; RO[o + c * a.fs] = ro[c]; }
    }
}

// phase shift, first half (rhs_velocity.f90:183-232): partial RHS into RP
template <typename TP>
__global__ void k_rhs_vel_ps1(const StepArgs a, const cx<TP> *__restrict__ P, const double2 *__restrict__ U,
                              double2 *__restrict__ RP)
{
    const int64_t nm = (int64_t)a.n * a.n * a.nh;
    const ModeLoop ml(a.n, a.nh, -1);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        ModeIdx m = ml.at(t);
        int64_t o = soff(m, a.n, a.pitch), po = soff(m, a.n, a.ppitch);
        double2 r[3];
        if (m.ialias > 1) {
            r[0] = r[1] = r[2] = make_double2(0.0, 0.0);
        } else {
            double2 u[3] = {U[o], U[o + a.fs], U[o + 2 * a.fs]};
            double2 p11 = ld2<TP>(P, po), p12 = ld2<TP>(P, po + a.pfs), p13 = ld2<TP>(P, po + 2 * a.pfs);
            double2 p22 = ld2<TP>(P, po + 3 * a.pfs), p23 = ld2<TP>(P, po + 4 * a.pfs), p33 = ld2<TP>(P, po + 5 * a.pfs);
            double kx = m.ax, ky = m.ay, kz = m.az;
            double2 t1 = make_double2(-(kx * p11.x + ky * p12.x + kz * p13.x), -(kx * p11.y + ky * p12.y + kz * p13.y));
            double2 t2 = make_double2(-(kx * p12.x + ky * p22.x + kz * p23.x), -(kx * p12.y + ky * p22.y + kz * p23.y));
            double2 t3 = make_double2(-(kx * p13.x + ky * p23.x + kz * p33.x), -(kx * p13.y + ky * p23.y + kz * p33.y));
            double t4 = -a.nu * (kx * kx + ky * ky + kz * kz);
            double2 tt[3] = {t1, t2, t3};
#pragma unroll
            for (int c = 0; c < 3; c++) r[c] = make_double2(-0.5 * tt[c].y + t4 * u[c].x, 0.5 * tt[c].x + t4 * u[c].y);
        }
#pragma unroll
        for (int c = 0; c < 3; c++) RP[o + c * a.fs] = r[c];
    }
}

// shift back by exp(-i k.delta) (rhs_velocity.f90:276-278)
H3D_D double2 shift_back(double2 v, double cs, double sn)
{
    return make_double2(v.x * cs + v.y * sn, v.y * cs - v.x * sn);
}

// phase shift, second half (rhs_velocity.f90:242-408) + forcing + AB2 + pressure.
// Q: six shifted product spectra [u+u+ u+v+ u+w+ v+v+ v+w+ w+w+]
template <typename TP>
__global__ void k_update_vel_ps2(const StepArgs a, double dx, const cx<TP> *__restrict__ Q,
                                 const double2 *__restrict__ RP, double2 *__restrict__ U, double2 *__restrict__ RO)
{
    const int64_t nm = (int64_t)a.n * a.n * a.nh;
    const double fac = (a.flow_type == 1) ? a.famp / *a.fenergy : 0.0;
    const ModeLoop ml(a.n, a.nh, -1);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        ModeIdx m = ml.at(t);
        int64_t o = soff(m, a.n, a.pitch), po = soff(m, a.n, a.ppitch);
        double2 u[3] = {U[o], U[o + a.fs], U[o + 2 * a.fs]};
        double2 r[3];
        double kx = m.ax, ky = m.ay, kz = m.az;
        if (m.ialias < 2) {
            double cs = cos((0.5 * ((kx + ky) + kz)) * dx), sn = sin((0.5 * ((kx + ky) + kz)) * dx);
            r[0] = RP[o]; r[1] = RP[o + a.fs]; r[2] = RP[o + 2 * a.fs];
            double2 A = shift_back(ld2<TP>(Q, po), cs, sn);                // u+u+
            r[0].x = r[0].x + 0.5 * kx * A.y; r[0].y = r[0].y - 0.5 * kx * A.x;
            double2 B = shift_back(ld2<TP>(Q, po + a.pfs), cs, sn);        // u+v+
            r[0].x = r[0].x + 0.5 * ky * B.y; r[0].y = r[0].y - 0.5 * ky * B.x;
            r[1].x = r[1].x + 0.5 * kx * B.y; r[1].y = r[1].y - 0.5 * kx * B.x;
            double2 Cc = shift_back(ld2<TP>(Q, po + 3 * a.pfs), cs, sn);   // v+v+
            r[1].x = r[1].x + 0.5 * ky * Cc.y; r[1].y = r[1].y - 0.5 * ky * Cc.x;
            double2 D4 = shift_back(ld2<TP>(Q, po + 2 * a.pfs), cs, sn);   // u+w+
            double2 D5 = shift_back(ld2<TP>(Q, po + 4 * a.pfs), cs, sn);   // v+w+
            double2 D6 = shift_back(ld2<TP>(Q, po + 5 * a.pfs), cs, sn);   // w+w+
            r[0].x = r[0].x + 0.5 * kz * D4.y; r[0].y = r[0].y - 0.5 * kz * D4.x;
            r[1].x = r[1].x + 0.5 * kz * D5.y; r[1].y = r[1].y - 0.5 * kz * D5.x;
            r[2].x = r[2].x + 0.5 * (kx * D4.y + ky * D5.y + kz * D6.y);
            r[2].y = r[2].y - 0.5 * (kx * D4.x + ky * D5.x + kz * D6.x);
        } else {
            r[0] = r[1] = r[2] = make_double2(0.0, 0.0);
        }
        if (a.flow_type == 1 && forced(m, a.n, a.kfmax)) {
#pragma unroll
            for (int c = 0; c < 3; c++) { r[c].x = r[c].x + fac * u[c].x; r[c].y = r[c].y + fac * u[c].y; }
        }
        double2 ro[3] = {RO[o], RO[o + a.fs], RO[o + 2 * a.fs]};
#pragma unroll
        for (int c = 0; c < 3; c++) ab2(u[c], ro[c], r[c], a.dt, a.euler_v);
        project(m, u[0], u[1], u[2]);
#pragma unroll
        for (int c = 0; c < 3; c++) { U[o + c * a.fs] = u[c]; RO[o + c * a.fs] = ro[c]; }
    }
}

// Scalar RHS + AB2 for scalar s.
//  mode 0 (2/3 rule, rhs_scalars.f90:88-121):     P = fluxes [phi u, phi v, phi w]
//  mode 1 (phase shift, first = unshifted half):  writes SP = 0.5 * flux term (masked)
//  mode 2 (phase shift, final = shifted half):    P = shifted fluxes, adds SP and diffusion
// The uniform-gradient source -u is added over all modes for type 0 scalars
// (rhs_scalars.f90:387-389).
template <typename TP>
// LS, LF (optional, dynamic localization model): spectra of the k_sgs source
// 2 nu_t S:S - k^(3/2)/Delta and of the three fluxes nu_t dk/dx_i, added to the
// RHS where ialias == 0 as LS + i k . LF (m_les.f90:1540-1546, 1609-1615, 1080-1086)
__global__ void k_scalar(const StepArgs a, int mode, int s, double dx, const cx<TP> *__restrict__ P,
                         double2 *__restrict__ SP, const double2 *__restrict__ Uvel, double2 *__restrict__ PHI,
                         double2 *__restrict__ RO, const cx<TP> *__restrict__ LS = nullptr,
                         const cx<TP> *__restrict__ LF = nullptr, const cx<TP> *__restrict__ RS = nullptr)
{
    const int kc = mode == 0 ? a.kc : -1;
    const int64_t nm = mode_count(a.n, a.nh, kc);
    const double pe = a.pe[s];
    const ModeLoop ml(a.n, a.nh, kc);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        ModeIdx m = ml.at(t);
        int64_t o = soff(m, a.n, a.pitch), po = soff(m, a.n, a.ppitch);
        double kx = m.ax, ky = m.ay, kz = m.az;
        // the products are read only where they are used (the 2/3 rule masks the rest)
        double2 pu = make_double2(0.0, 0.0), pv = pu, pw = pu;
        if (mode != 0 || m.ialias == 0) {
            pu = ld2<TP>(P, po);
            pv = ld2<TP>(P, po + a.pfs);
            pw = ld2<TP>(P, po + 2 * a.pfs);
        }
        if (mode == 1) {
            double2 sp = make_double2(0.0, 0.0);
            if (m.ialias < 2) {
                double rt1 = kx * pu.y + ky * pv.y + kz * pw.y;
                double rt2 = kx * pu.x + ky * pv.x + kz * pw.x;
                sp = make_double2(0.5 * rt1, -(0.5 * rt2));
            }
            SP[o] = sp;
            continue;
        }
        double2 phi = PHI[o];
        double2 r;
        double wn2 = kx * kx + ky * ky + kz * kz;
        if (mode == 0) {
            if (m.ialias > 0 || s < a.idle) r = make_double2(0.0, 0.0);
            else {
                double rt1 = kx * pu.y + ky * pv.y + kz * pw.y;
                double rt2 = kx * pu.x + ky * pv.x + kz * pw.x;
                r = make_double2(rt1 - pe * wn2 * phi.x, -rt2 - pe * wn2 * phi.y);
            }
        } else {
            if (m.ialias > 1) r = make_double2(0.0, 0.0);
            else {
                double cs = cos((0.5 * ((kx + ky) + kz)) * dx), sn = sin((0.5 * ((kx + ky) + kz)) * dx);
                double2 a1 = shift_back(pu, cs, sn), a2 = shift_back(pv, cs, sn), a3 = shift_back(pw, cs, sn);
                r = make_double2(+0.5 * (kx * a1.y + ky * a2.y + kz * a3.y), -0.5 * (kx * a1.x + ky * a2.x + kz * a3.x));
                double2 sp = SP[o];
                r.x = r.x + sp.x - pe * wn2 * phi.x;
                r.y = r.y + sp.y - pe * wn2 * phi.y;
            }
        }
        if (RS != nullptr) {  // reaction source, every mode (phase shift, rhs_scalars.f90:300)
            const double2 rs = ld2<TP>(RS, po);
            r.x = r.x + rs.x;
            r.y = r.y + rs.y;
        }
        if (a.stype[s] == 0) {
            double2 u = Uvel[o];
            r.x = r.x - u.x;
            r.y = r.y - u.y;
        }
        // LES: the source LS (LES fields only) and the divergence of the fluxes LF
        if (LF != nullptr && m.ialias == 0) {
            const double2 sv = LS != nullptr ? ld2<TP>(LS, po) : make_double2(0.0, 0.0), f1 = ld2<TP>(LF, po),
                          f2 = ld2<TP>(LF, po + a.pfs), f3 = ld2<TP>(LF, po + 2 * a.pfs);
            r.x = r.x + sv.x - (kx * f1.y + ky * f2.y + kz * f3.y);
            r.y = r.y + sv.y + (kx * f1.x + ky * f2.x + kz * f3.x);
        }
        double2 ro = RO[o];
        ab2(phi, ro, r, a.dt, a.euler_s);
        PHI[o] = phi;
        RO[o] = ro;
    }
}

// Energy in the forcing band (m_force.f90:101-182, summed in the loop order of
// m_force.f90:266-284): E_f = sum over the shells
// 1..kfmax of the shell's (|u|^2 + |v|^2 + |w|^2)/N^6, half weight at kx = 0,
// each mode's real entry and then its imaginary entry added on their own.
// Bands of up to kFsmall shells: the candidate modes |k_i| <= kfmax + 1 in the
// reference's loop order (ky, kz, kx) go in chunks of kFchunk, every thread
// computing the contributions of its candidates (its own loads, all in flight
// at once), and thread 0 adds them, in that order, to the shell sums.  Wider
// bands: thread s of the CTA sums shell s + 1 (and s + 1 + blockDim.x, ...)
// over the same candidates in the same order, and thread 0 adds the shells
// (es, kfmax doubles of dynamic shared memory).  Every shell sum and the final
// sum over the shells in order are rounded alike in both forms, and as one
// thread visiting every candidate in order would round them.  One CTA per run
// of a batch (U advanced by ru per CTA).
constexpr int kFsmall = 16, kFchunk = 1024, kFthreads = 256;
__global__ void k_forcing_energy(int n, int pitch, int64_t fs, int kfmax, const double2 *__restrict__ U,
                                 double *out, int64_t ru = 0)
{
    extern __shared__ double es[];
    U += blockIdx.x * ru;
    out += blockIdx.x;
    const double n3 = (double)n * n * n;
    const double fac = 1.0 / (n3 * n3);
    const int km = kfmax + 1;
    if (kfmax <= kFsmall) {
        __shared__ double fr[kFchunk], fi[kFchunk];
        __shared__ unsigned char fsh[kFchunk];
        // candidate lists: ky and kz storage indices 0..km, n-km..n-1 (all n when
        // they overlap), kx 0..min(km, n/2 - 1)
        const int nk = 2 * km + 1 < n ? 2 * km + 1 : n;
        const int nxc = (km < n / 2 - 1 ? km : n / 2 - 1) + 1;
        const int64_t nc = (int64_t)nk * nk * nxc;
        double e16[kFsmall];
        for (int s = 0; s < kFsmall; s++) e16[s] = 0.0;
        for (int64_t base = 0; base < nc; base += kFchunk) {
            for (int q = threadIdx.x; q < kFchunk; q += blockDim.x) {
                const int64_t t = base + q;
                unsigned char sh8 = 0;
                if (t < nc) {
                    const int kx = (int)(t % nxc);
                    const int64_t r = t / nxc;
                    const int b = (int)(r % nk), a = (int)(r / nk);
                    const int kq = (nk == n || a <= km) ? a : n - (nk - a);
                    const int jq = (nk == n || b <= km) ? b : n - (nk - b);
                    const int ky = kwave(kq, n), kz = kwave(jq, n);
                    const double k2 = (double)kx * kx + (double)ky * ky + (double)kz * kz;
                    const int sh = shell32(k2);
                    if (sh > 0 && sh <= kfmax) {
                        const int64_t o = ((int64_t)jq * n + kq) * pitch + kx;
                        const double2 u = U[o], v = U[fs + o], w = U[2 * fs + o];
                        // real entry then imaginary entry, each added on its own
                        double f2 = __dmul_rn(fac, __dadd_rn(__dadd_rn(__dmul_rn(u.x, u.x), __dmul_rn(v.x, v.x)), __dmul_rn(w.x, w.x)));
                        if (kx == 0) f2 = __dmul_rn(f2, 0.5);
                        fr[q] = f2;
                        f2 = __dmul_rn(fac, __dadd_rn(__dadd_rn(__dmul_rn(u.y, u.y), __dmul_rn(v.y, v.y)), __dmul_rn(w.y, w.y)));
                        if (kx == 0) f2 = __dmul_rn(f2, 0.5);
                        fi[q] = f2;
                        sh8 = (unsigned char)sh;
                    }
                }
                fsh[q] = sh8;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                const int m = nc - base < kFchunk ? (int)(nc - base) : kFchunk;
                for (int q = 0; q < m; q++) {
                    const int sh = fsh[q];
                    if (sh == 0) continue;
                    e16[sh - 1] = __dadd_rn(e16[sh - 1], fr[q]);
                    e16[sh - 1] = __dadd_rn(e16[sh - 1], fi[q]);
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            double e = 0.0;
            for (int s = 0; s < kfmax; s++) e = __dadd_rn(e, e16[s]);
            *out = e;
        }
        return;
    }
    for (int sh0 = threadIdx.x + 1; sh0 <= kfmax; sh0 += blockDim.x) {
        double e = 0.0;
        // storage indices in increasing order whose |wavenumber| <= km: 0..km, n-km..n-1
        for (int kq = 0; kq < n; kq++) {
            if (kq > km && kq < n - km) { kq = n - km - 1; continue; }
            const int ky = kwave(kq, n);
            for (int jq = 0; jq < n; jq++) {
                if (jq > km && jq < n - km) { jq = n - km - 1; continue; }
                const int kz = kwave(jq, n);
                for (int kx = 0; kx <= km && kx < n / 2; kx++) {
                    double k2 = (double)kx * kx + (double)ky * ky + (double)kz * kz;
                    if (shell32(k2) != sh0) continue;
                    const int64_t o = ((int64_t)jq * n + kq) * pitch + kx;
                    double2 u = U[o], v = U[fs + o], w = U[2 * fs + o];
                    // real entry then imaginary entry, each added on its own
                    double f2 = __dmul_rn(fac, __dadd_rn(__dadd_rn(__dmul_rn(u.x, u.x), __dmul_rn(v.x, v.x)), __dmul_rn(w.x, w.x)));
                    if (kx == 0) f2 = __dmul_rn(f2, 0.5);
                    e = __dadd_rn(e, f2);
                    f2 = __dmul_rn(fac, __dadd_rn(__dadd_rn(__dmul_rn(u.y, u.y), __dmul_rn(v.y, v.y)), __dmul_rn(w.y, w.y)));
                    if (kx == 0) f2 = __dmul_rn(f2, 0.5);
                    e = __dadd_rn(e, f2);
                }
            }
        }
        es[sh0 - 1] = e;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double e = 0.0;
    for (int s = 0; s < kfmax; s++) e = __dadd_rn(e, es[s]);
    *out = e;
}

// dealias_all (dealias_all.f90:97-131): zero modes with any |k_i| > kmax
__global__ void k_dealias_all(int n, int nh, int pitch, int64_t fs, int nf, int kmax, double2 *U)
{
    const int64_t nm = (int64_t)n * n * nh;
    const double ak = (double)kmax;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        ModeIdx m = mode_of(t, n, nh);
        if (fabs(m.ax) > ak || fabs(m.ay) > ak || fabs(m.az) > ak) {
            int64_t o = soff(m, n, pitch);
            for (int f = 0; f < nf; f++) U[o + f * fs] = make_double2(0.0, 0.0);
        }
    }
}

// max |component| of nf fields of A and B over the modes the 2/3 rule removes
// (some |k_i| > N/3), as the bit pattern of a non-negative double: zero means
// the transforms of a time step may skip those modes exactly
__global__ void k_alias_max(int n, int nh, int pitch, int64_t fs, int nf, const double2 *__restrict__ A,
                            const double2 *__restrict__ B, unsigned long long *out)
{
    const int64_t nm = (int64_t)n * n * nh;
    double mx = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        ModeIdx m = mode_of(t, n, nh);
        if (m.ialias > 0) {
            const int64_t o = soff(m, n, pitch);
            for (int f = 0; f < nf; f++) {
                const double2 a = A[o + f * fs], b = B[o + f * fs];
                mx = fmax(mx, fmax(fmax(fabs(a.x), fabs(a.y)), fmax(fabs(b.x), fabs(b.y))));
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0 && mx > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(mx));
}

// number of non-finite components among the N^2 (N/2+1) modes of nf fields of
// A (state layout, row pitch `pitch` complex, field stride fs)
__global__ void k_count_nonfinite(int n, int nh, int pitch, int64_t fs, int nf, const double2 *__restrict__ A,
                                  unsigned long long *out)
{
    const int64_t nm = (int64_t)n * n * nh;
    unsigned long long cnt = 0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / nh, o = row * pitch + (t - row * nh);
        for (int f = 0; f < nf; f++) {
            const double2 v = A[o + f * fs];
            cnt += !isfinite(v.x);
            cnt += !isfinite(v.y);
        }
    }
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(out, cnt);
}

// Shell spectrum sum_{shell} fac * |f|^2 (kx = 0 halved, kx = N/2 excluded),
// float32 shell index (m_stats.f90:195-235).  Deterministic: each warp owns a
// private histogram, lane L accumulates the shells congruent to L mod 32 in a
// fixed element order; warps and blocks are combined in index order.
// w0 is the weight of the kx = 0 plane: 0.5 for the statistics (m_stats.f90:222),
// 1 for the decaying-run rescale (velocity_rescale.f90:47-55)
__global__ void k_shell_partial(int n, int nh, int pitch, int64_t fs, int nf, int kmax, double w0,
                                const double2 *__restrict__ U, double *__restrict__ part /* [gridDim.x][kmax] */)
{
    extern __shared__ double hist[];  // [warps][kmax]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < nw * kmax; i += blockDim.x) hist[i] = 0.0;
    __syncthreads();
    const double n3 = (double)n * n * n;
    const double fac = 1.0 / (n3 * n3);
    const int64_t nm = (int64_t)n * n * nh;
    const int64_t per_block = (nm + gridDim.x - 1) / gridDim.x;
    const int64_t b0 = blockIdx.x * per_block, b1 = min(nm, b0 + per_block);
    double *h = hist + warp * kmax;
    for (int64_t base = b0 + warp * 32; base < b1; base += nw * 32) {
        int64_t t = base + lane;
        int sh = -1;
        double e = 0.0;
        if (t < b1) {
            ModeIdx m = mode_of(t, n, nh);
            if (m.kx < n / 2) {
                double k2 = m.ax * m.ax + m.ay * m.ay + m.az * m.az;
                int s = shell32(k2);
                if (s > 0 && s <= kmax) {
                    int64_t o = soff(m, n, pitch);
                    double re = 0.0, im = 0.0;
                    for (int f = 0; f < nf; f++) {
                        double2 v = U[o + f * fs];
                        re = (f == 0) ? v.x * v.x : re + v.x * v.x;
                        im = (f == 0) ? v.y * v.y : im + v.y * v.y;
                    }
                    double e1 = fac * re, e2 = fac * im;
                    if (m.kx == 0) { e1 *= w0; e2 *= w0; }
                    e = e1 + e2;
                    sh = s - 1;
                }
            }
        }
        for (int l = 0; l < 32; l++) {
            int s = __shfl_sync(0xffffffffu, sh, l);
            double v = __shfl_sync(0xffffffffu, e, l);
            if (s >= 0 && (s & 31) == lane) h[s] += v;
        }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < kmax; s += blockDim.x) {
        double acc = 0.0;
        for (int w = 0; w < nw; w++) acc += hist[w * kmax + s];
        part[(int64_t)blockIdx.x * kmax + s] = acc;
    }
}

__global__ void k_shell_final(int nblk, int kmax, const double *__restrict__ part, double *__restrict__ out)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < kmax; s += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int b = 0; b < nblk; b++) acc += part[(int64_t)b * kmax + s];
        out[s] = acc;
    }
}

// Deterministic sums over physical points of the fields:
// mode 0: sum_f x_f^2;  mode 1: x_0^2 and x_0^3 (two sums);  mode 2: x, x^2, min, max of x_0
__global__ void k_phys_partial(int n, int64_t rpitch, int64_t fs, int nf, int mode, const double *__restrict__ X,
                               double *__restrict__ part /* [gridDim.x][4] */)
{
    __shared__ double sh[4][32];
    const int64_t np = (int64_t)n * n * n;
    double s0 = 0.0, s1 = 0.0, mn = 1e300, mx = -1e300;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t row = t / n, x = t - row * n;
        const double *p = X + row * rpitch + x;
        if (mode == 0) {
            double q = 0.0;
            for (int f = 0; f < nf; f++) { double v = p[f * fs]; q = (f == 0) ? v * v : q + v * v; }
            s0 += q;
        } else if (mode == 1) {
            double v = p[0];
            s0 += v * v;
            s1 += v * v * v;
        } else {
            double v = p[0];
            s0 += v;
            s1 += v * v;
            mn = fmin(mn, v);
            mx = fmax(mx, v);
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, off);
        s1 += __shfl_xor_sync(0xffffffffu, s1, off);
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, off));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (l == 0) { sh[0][w] = s0; sh[1][w] = s1; sh[2][w] = mn; sh[3][w] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0, a2 = 1e300, a3 = -1e300;
        for (int i = 0; i < nw; i++) { a0 += sh[0][i]; a1 += sh[1][i]; a2 = fmin(a2, sh[2][i]); a3 = fmax(a3, sh[3][i]); }
        part[blockIdx.x * 4 + 0] = a0; part[blockIdx.x * 4 + 1] = a1;
        part[blockIdx.x * 4 + 2] = a2; part[blockIdx.x * 4 + 3] = a3;
    }
}

__global__ void k_phys_final(int nblk, const double *__restrict__ part, double *__restrict__ out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a0 = 0.0, a1 = 0.0, a2 = 1e300, a3 = -1e300;
    for (int b = 0; b < nblk; b++) {
        a0 += part[b * 4]; a1 += part[b * 4 + 1];
        a2 = fmin(a2, part[b * 4 + 2]); a3 = fmax(a3, part[b * 4 + 3]);
    }
    out[0] = a0; out[1] = a1; out[2] = a2; out[3] = a3;
}

// ---------------------------------------------------------------------------
// dynamic localization model (m_les.f90:1313-1621, 1041-1091)
// ---------------------------------------------------------------------------
// nu_t = C_k Delta sqrt(k) from the truncated k_sgs in physical space, with k
// clipped at zero in place (les_get_turb_visc_dlm, m_les.f90:1313-1388: the
// reference clips only when the minimum is negative, which gives the same
// values).  coef = C_k Delta.
__global__ void k_dlm_nut(int n, int64_t rp, double coef, double *__restrict__ K, double *__restrict__ NUT)
{
    const int64_t np = (int64_t)n * n * n;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / n, o = row * rp + (t - row * n);
        const double k = K[o] > 0.0 ? K[o] : 0.0;
        K[o] = k;
        NUT[o] = coef * sqrt(k);
    }
}

// the clipped k_sgs W replaces the state field when the minimum was negative
__global__ void k_dlm_commit(int n, int nh, int pitch, const double *__restrict__ kmin,
                             const double2 *__restrict__ W, double2 *__restrict__ U)
{
    if (!(*kmin < 0.0)) return;
    const int64_t nm = (int64_t)n * n * nh;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / nh, o = row * pitch + (t - row * nh);
        U[o] = W[o];
    }
}

// physical-space terms, in place, on rows of pitch rp (reals), fields fs reals apart:
//   S[0..6) (S11 S12 S13 S22 S23 S33) -> tau_ij = -2 nu_t S_ij      (m_les.f90:902-1018)
//   KC (k_sgs with the 2/3 rule)      -> 2 nu_t S_ij S_ij - max(KC,0)^1.5 / Delta
//                                                                    (m_les.f90:1422-1621)
//   G[0..3) (dk/dx_i)                 -> nu_t dk/dx_i                (m_les.f90:1041-1091)
// the three sums of a 256-thread block into part[3 blockIdx.x + 0, 1, 2]
H3D_D void block_sums3(double a, double b, double d, double *__restrict__ part)
{
    __shared__ double sh[3][8];
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, off);
        b += __shfl_xor_sync(0xffffffffu, b, off);
        d += __shfl_xor_sync(0xffffffffu, d, off);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = a;
        sh[1][threadIdx.x >> 5] = b;
        sh[2][threadIdx.x >> 5] = d;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += sh[threadIdx.x][w];
        part[3 * blockIdx.x + threadIdx.x] = v;
    }
}

// part[3 b + 0, 1, 2]: block b's sums of the production, of B (zero here) and
// of the dissipation, for the domain means that les.gp reports
// (m_les.f90:1536,1617)
__global__ void __launch_bounds__(256) k_dlm_phys(int n, int64_t rp, int64_t fs, double delta,
                                                  const double *__restrict__ NUT, double *__restrict__ S,
                                                  double *__restrict__ KC, double *__restrict__ G, int ng,
                                                  double *__restrict__ part)
{
    const int64_t np = (int64_t)n * n * n;
    double psum = 0.0, dsum = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / n, o = row * rp + (t - row * n);
        const double nut = NUT[o];
        double sv[6];
#pragma unroll
        for (int c = 0; c < 6; c++) sv[c] = S[o + c * fs];
        double ss = sv[0] * sv[0];
        ss = ss + 2.0 * (sv[1] * sv[1]);
        ss = ss + 2.0 * (sv[2] * sv[2]);
        ss = ss + sv[3] * sv[3];
        ss = ss + 2.0 * (sv[4] * sv[4]);
        ss = ss + sv[5] * sv[5];
        const double kc = KC[o] > 0.0 ? KC[o] : 0.0;
        const double prod = (2.0 * ss) * nut, diss = pow(kc, 1.5) / delta;
        KC[o] = prod - diss;
        psum += prod;
        dsum += diss;
#pragma unroll
        for (int c = 0; c < 6; c++) S[o + c * fs] = (-2.0 * nut) * sv[c];
        for (int d = 0; d < ng; d++) G[o + d * fs] = G[o + d * fs] * nut;
    }
    block_sums3(psum, 0.0, dsum, part);
}

// Dynamic localization model with the lag model for the dissipation
// (les_model 3; m_les.f90:1422-1561, 1629-1684): per point, from nu_t, the six
// strain components S, the physical (B T_B) and (eps T_eps) in BT and ET, and
// the gradients G of k_sgs, (B T_B), (eps T_eps):
//   |S| = sqrt(2 S:S), B = (B T_B) |S|, eps = max(eps T_eps, 0)^1.5 / (Delta C_T^1.5),
//   production Pi = 2 nu_t S:S;
//   sources  k: Pi - eps  -> BT,   B T_B: Pi - B  -> ET,   eps T_eps: B - eps -> S3;
//   tau = -2 nu_t S in S, fluxes nu_t grad in G (nine fields).
// part[3 b + 0, 1, 2]: block sums of Pi, B and eps.
__global__ void __launch_bounds__(256) k_dll_phys(int n, int64_t rp, int64_t fs, double delta, double c_t,
                                                  const double *__restrict__ NUT, double *__restrict__ S,
                                                  double *__restrict__ BT, double *__restrict__ ET,
                                                  double *__restrict__ G, int ng, double *__restrict__ S3,
                                                  double *__restrict__ part)
{
    const int64_t np = (int64_t)n * n * n;
    const double den = delta * pow(c_t, 1.5);
    double psum = 0.0, bsum = 0.0, dsum = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / n, o = row * rp + (t - row * n);
        const double nut = NUT[o];
        double sv[6];
#pragma unroll
        for (int c = 0; c < 6; c++) sv[c] = S[o + c * fs];
        double ss = sv[0] * sv[0];
        ss = ss + 2.0 * (sv[1] * sv[1]);
        ss = ss + 2.0 * (sv[2] * sv[2]);
        ss = ss + sv[3] * sv[3];
        ss = ss + 2.0 * (sv[4] * sv[4]);
        ss = ss + sv[5] * sv[5];
        const double s2 = 2.0 * ss;
        const double prod = s2 * nut;
        const double bb = BT[o] * sqrt(s2);
        const double et = ET[o] > 0.0 ? ET[o] : 0.0;
        const double eps = pow(et, 1.5) / den;
        BT[o] = prod - eps;
        ET[o] = prod - bb;
        S3[o] = bb - eps;
        psum += prod;
        bsum += bb;
        dsum += eps;
#pragma unroll
        for (int c = 0; c < 6; c++) S[o + c * fs] = (-2.0 * nut) * sv[c];
        for (int d = 0; d < ng; d++) G[o + d * fs] = G[o + d * fs] * nut;
    }
    block_sums3(psum, bsum, dsum, part);
}

// Dynamic Structure Model family (les_models 4-7; m_les.f90:1697-1960 with
// 1096-1137, 1422-1621, 1629-1684, 1041-1091), per point of the physical
// fields W (row pitch rp, field stride fs):
//   W[0..6)  test-filtered products (u_i u_j)~ (uu uv uw vv vw ww) -> tau_ij
//   W[6..9)  test-filtered velocity u~_i                            -> sources
//   W[9..18) du_i/dx_j at 9 + 3 i + j
//   W[18]    k_sgs;  W[19] the 2/3-rule k_sgs (algebraic dissipation) or
//   (B T_B);  W[20] (eps T_eps);  W[g0 ..) gradients of the LES fields -> fluxes
// tau_D = 2 max(k, 0) / max(L_kk, 1e-15) L_ij, L_ij = (u_i u_j)~ - u~_i u~_j;
// Pi_D = -tau_ij du_i/dx_j;  nu_t = cmix (c_s dx)^2 sqrt(2 S:S) (cmix = 1 for
// 4, 5, C_mixed for 6, 7); the mixed models add -2 nu_t S to tau and the
// transfer Pi_L = 2 nu_t S:S.  Sources: k: Pi_D + Pi_L - eps;  (B T_B):
// Pi_D + Pi_L - B;  (eps T_eps): B - eps, with eps = max(k~, 0)^1.5 / Delta
// (algebraic, 4 and 6) or max(eps T_eps, 0)^1.5 / (Delta C_T^1.5) and
// B = (B T_B) sqrt(2 S:S) (lag model, 5 and 7).  Fluxes nu_t grad(phi).
struct DstmArgs {
    int n;
    int64_t rp, fs;
    int lag, mixed, g0;
    double cs2, cmix, delta, c_t;
    int nps;  // les_model 10: passive scalars, their gradients at W[26 + 3 s] -> Harlow fluxes
};
__global__ void __launch_bounds__(256) k_dstm_phys(const DstmArgs a, double *__restrict__ W, double *__restrict__ part)
{
    const int64_t np = (int64_t)a.n * a.n * a.n;
    const int nl = a.lag ? 3 : 1;
    const double den = a.delta * (a.lag ? pow(a.c_t, 1.5) : 1.0);
    double psum = 0.0, bsum = 0.0, dsum = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / a.n, o = row * a.rp + (t - row * a.n);
        double g[9], fu[3], fp[6];
#pragma unroll
        for (int q = 0; q < 9; q++) g[q] = W[o + (9 + q) * a.fs];
#pragma unroll
        for (int q = 0; q < 3; q++) fu[q] = W[o + (6 + q) * a.fs];
#pragma unroll
        for (int q = 0; q < 6; q++) fp[q] = W[o + q * a.fs];
        const double kr = W[o + 18 * a.fs];
        // products in the order uu uv uw vv vw ww: (i, j) -> index
        const int pi[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
        double lkk = (fp[0] + fp[3]) + fp[5];
        lkk = lkk - fu[0] * fu[0];
        lkk = lkk - fu[1] * fu[1];
        lkk = lkk - fu[2] * fu[2];
        const double cf = 2.0 * (kr > 0.0 ? kr : 0.0) / (lkk > 1.e-15 ? lkk : 1.e-15);
        double tau[6];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = i; j < 3; j++) tau[pi[i][j]] = (fp[pi[i][j]] - fu[i] * fu[j]) * cf;
        double pid = 0.0;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) pid -= g[3 * i + j] * tau[pi[i][j]];
        double sv[6];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = i; j < 3; j++) sv[pi[i][j]] = 0.5 * (g[3 * i + j] + g[3 * j + i]);
        double ss = sv[0] * sv[0];
        ss = ss + 2.0 * (sv[1] * sv[1]);
        ss = ss + 2.0 * (sv[2] * sv[2]);
        ss = ss + sv[3] * sv[3];
        ss = ss + 2.0 * (sv[4] * sv[4]);
        ss = ss + sv[5] * sv[5];
        const double s2 = 2.0 * ss;
        const double nut = a.cmix * (sqrt(s2) * a.cs2);
        double pil = 0.0;
        if (a.mixed) {
            pil = s2 * nut;
#pragma unroll
            for (int q = 0; q < 6; q++) tau[q] = tau[q] + (-2.0 * nut) * sv[q];
        }
        double eps, bb = 0.0;
        if (a.lag) {
            const double et = W[o + 20 * a.fs];
            bb = W[o + 19 * a.fs] * sqrt(s2);
            eps = pow(et > 0.0 ? et : 0.0, 1.5) / den;
            W[o + 7 * a.fs] = (pid + pil) - bb;
            W[o + 8 * a.fs] = bb - eps;
        } else {
            const double kc = W[o + 19 * a.fs];
            eps = pow(kc > 0.0 ? kc : 0.0, 1.5) / den;
        }
        W[o + 6 * a.fs] = (pid + pil) - eps;
#pragma unroll
        for (int q = 0; q < 6; q++) W[o + q * a.fs] = tau[q];
        for (int q = 0; q < 3 * nl; q++) W[o + (a.g0 + q) * a.fs] = W[o + (a.g0 + q) * a.fs] * nut;
        psum += pid + pil;
        bsum += bb;
        dsum += eps;
    }
    block_sums3(psum, bsum, dsum, part);
}

// les_model 10 (m_les.f90:1223-1307, 2009-2392), per point of W laid out as
// for k_dstm_phys but W[18] (B T_B), W[19] (eps T_eps), W[20..26) their
// gradients: k = (B T_B) + (eps T_eps), c = 2 k / L_kk (0 where L_kk < 1e-10),
// tau_ij = c L_ij - 2 C_mixed nu_t S_ij, Pi = -c L_ij S_ij + C_mixed nu_t^3 /
// (c_s Delta)^4, B = (B T_B) nu_t / (c_s Delta)^2, eps = max(eps T_eps, 0)^1.5 /
// Delta; sources (B T_B): Pi - B -> W[6], (eps T_eps): B - eps -> W[7];
// fluxes nu_t grad -> W[20..26); nu_t = (c_s Delta)^2 sqrt(2 S:S).
__global__ void __launch_bounds__(256) k_m10_phys(const DstmArgs a, double *__restrict__ W, double *__restrict__ part)
{
    const int64_t np = (int64_t)a.n * a.n * a.n;
    const double cd2 = a.cs2, cd4 = a.cs2 * a.cs2;
    double psum = 0.0, bsum = 0.0, dsum = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / a.n, o = row * a.rp + (t - row * a.n);
        double g[9], fu[3], fp[6];
#pragma unroll
        for (int q = 0; q < 9; q++) g[q] = W[o + (9 + q) * a.fs];
#pragma unroll
        for (int q = 0; q < 3; q++) fu[q] = W[o + (6 + q) * a.fs];
#pragma unroll
        for (int q = 0; q < 6; q++) fp[q] = W[o + q * a.fs];
        const double bt = W[o + 18 * a.fs], et = W[o + 19 * a.fs];
        const int pi[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
        double lij[6], sv[6];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = i; j < 3; j++) {
                lij[pi[i][j]] = fp[pi[i][j]] - fu[i] * fu[j];
                sv[pi[i][j]] = 0.5 * (g[3 * i + j] + g[3 * j + i]);
            }
        const double lkk = (lij[0] + lij[3]) + lij[5];
        const double cc = lkk < 1e-10 ? 0.0 : 2.0 * (bt + et) / lkk;
        double ss = sv[0] * sv[0];
        ss = ss + 2.0 * (sv[1] * sv[1]);
        ss = ss + 2.0 * (sv[2] * sv[2]);
        ss = ss + sv[3] * sv[3];
        ss = ss + 2.0 * (sv[4] * sv[4]);
        ss = ss + sv[5] * sv[5];
        const double nut = sqrt(2.0 * ss) * cd2;
        double ls = -lij[0] * sv[0];
        ls = ls - lij[3] * sv[3];
        ls = ls - lij[5] * sv[5];
        ls = ls - 2.0 * lij[1] * sv[1];
        ls = ls - 2.0 * lij[2] * sv[2];
        ls = ls - 2.0 * lij[4] * sv[4];
        const double prod = ls * cc + a.cmix * (nut * nut * nut) / cd4;
        const double bb = bt * (nut / cd2);
        const double eps = pow(et > 0.0 ? et : 0.0, 1.5) / a.delta;
        W[o + 6 * a.fs] = prod - bb;
        W[o + 7 * a.fs] = bb - eps;
        double tau[6];
#pragma unroll
        for (int q = 0; q < 6; q++) {
            tau[q] = cc * lij[q] - a.cmix * 2.0 * nut * sv[q];
            W[o + q * a.fs] = tau[q];
        }
#pragma unroll
        for (int q = 0; q < 6; q++) W[o + (20 + q) * a.fs] = W[o + (20 + q) * a.fs] * nut;
        // Harlow fluxes of the passive scalars (m_les.f90:2191-2270): T tau_ij dphi/dx_j
        // with the time scale T = 1/|S|, |S| = nu_t / (c_s Delta)^2 (T = 0 where |S| < 1e-10)
        const double sm = nut / cd2;
        const double tt = fabs(sm) < 1e-10 ? 0.0 : 1.0 / sm;
        for (int s = 0; s < a.nps; s++) {
            double *gp = W + o + (26 + 3 * s) * a.fs;
            const double g0 = gp[0], g1 = gp[a.fs], g2 = gp[2 * a.fs];
            gp[0] = (tau[0] * g0 + tau[1] * g1 + tau[2] * g2) * tt;
            gp[a.fs] = (tau[1] * g0 + tau[3] * g1 + tau[4] * g2) * tt;
            gp[2 * a.fs] = (tau[2] * g0 + tau[4] * g1 + tau[5] * g2) * tt;
        }
        psum += prod;
        bsum += bb;
        dsum += eps;
    }
    block_sums3(psum, bsum, dsum, part);
}

// Smagorinsky model with passive scalars (les_model 1; m_les.f90:1142-1215,
// 902-1018, 1041-1091): from the six strain components S (physical, in place),
// nu_t = (c_s Delta)^2 sqrt(2 S:S), tau = -2 nu_t S, and the ng scalar gradient
// fields G times nu_t (the turbulent fluxes)
template <typename T>
__global__ void __launch_bounds__(256) k_smag_phys(int n, int64_t rp, int64_t fs, double cs2, T *__restrict__ S,
                                                   T *__restrict__ G, int ng)
{
    const int64_t np = (int64_t)n * n * n;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / n, o = row * rp + (t - row * n);
        double sv[6];
#pragma unroll
        for (int c = 0; c < 6; c++) sv[c] = (double)S[o + c * fs];
        double ss = sv[0] * sv[0];
        ss = ss + 2.0 * (sv[1] * sv[1]);
        ss = ss + 2.0 * (sv[2] * sv[2]);
        ss = ss + sv[3] * sv[3];
        ss = ss + 2.0 * (sv[4] * sv[4]);
        ss = ss + sv[5] * sv[5];
        const double nut = sqrt(2.0 * ss) * cs2;
#pragma unroll
        for (int c = 0; c < 6; c++) S[o + c * fs] = (T)((-2.0 * nut) * sv[c]);
        for (int d = 0; d < ng; d++) G[o + d * fs] = (T)((double)G[o + d * fs] * nut);
    }
}

// out[0..3] = energy, production, B, dissipation of les.gp (m_les.f90:876-892):
// the mean k_sgs from the zero mode K0 (plus K1: (B T_B) + (eps T_eps) for
// les_model 10) of the unnormalised forward transform, and the block sums
// divided by N^3; one warp, fixed summation order
__global__ void k_dlm_stats(int nblk, double inv_n3, const double2 *__restrict__ K0, const double *__restrict__ part,
                            double *__restrict__ out, const double2 *__restrict__ K1 = nullptr)
{
    double p = 0.0, b = 0.0, d = 0.0;
    for (int q = threadIdx.x; q < nblk; q += 32) {
        p += part[3 * q];
        b += part[3 * q + 1];
        d += part[3 * q + 2];
    }
    for (int off = 16; off > 0; off >>= 1) {
        p += __shfl_xor_sync(0xffffffffu, p, off);
        b += __shfl_xor_sync(0xffffffffu, b, off);
        d += __shfl_xor_sync(0xffffffffu, d, off);
    }
    if (threadIdx.x == 0) {
        out[0] = (K1 != nullptr ? K0[0].x + K1[0].x : K0[0].x) * inv_n3;
        out[1] = p * inv_n3;
        out[2] = b * inv_n3;
        out[3] = d * inv_n3;
    }
}

// initial velocity: solenoidal curl of the transformed Gaussian noise G restricted
// to shells 1..kmax with an FP64 shell index (init_velocity.f90:123-149)
__global__ void k_init_curl(int n, int nh, int pitch, int64_t fs, int kmax, const double2 *__restrict__ G,
                            double2 *__restrict__ U)
{
    const int64_t nm = (int64_t)n * n * nh;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        ModeIdx m = mode_of(t, n, nh);
        int64_t o = soff(m, n, pitch);
        double kx = m.ax, ky = m.ay, kz = m.az;
        int sh = (int)llround(sqrt(kx * kx + ky * ky + kz * kz));
        double2 r4 = make_double2(0, 0), r5 = r4, r6 = r4;
        if (sh > 0 && sh <= kmax) {
            double2 g1 = G[o], g2 = G[o + fs], g3 = G[o + 2 * fs];
            r4 = make_double2(-(ky * g3.y - kz * g2.y), ky * g3.x - kz * g2.x);
            r5 = make_double2(-(kz * g1.y - kx * g3.y), kz * g1.x - kx * g3.x);
            r6 = make_double2(-(kx * g2.y - ky * g1.y), kx * g2.x - ky * g1.x);
        }
        U[o] = r4; U[o + fs] = r5; U[o + 2 * fs] = r6;
    }
}

// reaction source of a type-311 scalar (rhs_scalars.f90:281-303), in place on
// the physical band-limited scalar X (row pitch rp): reac (1 - X^2)(X - mean),
// mean the scalar's zero mode K0 over N^3
template <typename T>
__global__ void k_reaction(int n, int64_t rp, double reac, const double2 *__restrict__ K0, T *__restrict__ X)
{
    const int64_t np = (int64_t)n * n * n;
    const double mean = K0[0].x / ((double)n * n * n);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / n, o = row * rp + (t - row * n);
        const double x = (double)X[o];
        X[o] = (T)(reac * (1.0 - x * x) * (x - mean));
    }
}

// physical values of one field (row pitch rp, n per row) -> sign(x) * 0.9
// (init_scalars.f90:242-247; Fortran's sign(1, x) is +1 at x = 0)
__global__ void k_sign09(int n, int64_t rp, double *__restrict__ X)
{
    const int64_t np = (int64_t)n * n * n;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / n, o = row * rp + (t - row * n);
        X[o] = X[o] < 0.0 ? -0.9 : 0.9;
    }
}

// multiply modes of shells 1..kmax by ratio[shell] and zero the rest
// (init_velocity.f90:224-237); ratio[s] < 0 marks an empty shell
__global__ void k_shell_scale(int n, int nh, int pitch, int64_t fs, int nf, int kmax, const double *__restrict__ ratio,
                              double2 *__restrict__ U)
{
    const int64_t nm = (int64_t)n * n * nh;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        ModeIdx m = mode_of(t, n, nh);
        int64_t o = soff(m, n, pitch);
        int sh = shell32(m.ax * m.ax + m.ay * m.ay + m.az * m.az);
        bool keep = sh > 0 && sh <= kmax && ratio[sh - 1] >= 0.0;
        for (int f = 0; f < nf; f++) {
            double2 v = U[o + f * fs];
            if (keep) { double r = ratio[sh - 1]; v.x = v.x * r; v.y = v.y * r; }
            else v = make_double2(0.0, 0.0);
            U[o + f * fs] = v;
        }
    }
}

// spectral filter f <- f * G as a complex product (m_filter_xfftw.f90:92-104);
// G is the transfer function in the device spectral layout
__global__ void k_filter_apply(int n, int nh, int pitch, const double2 *__restrict__ G, double2 *__restrict__ F)
{
    const int64_t nm = (int64_t)n * n * nh;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        ModeIdx m = mode_of(t, n, nh);
        int64_t o = soff(m, n, pitch);
        double2 f = F[o], g = G[o];
        F[o] = make_double2(f.x * g.x - f.y * g.y, f.y * g.x + f.x * g.y);
    }
}

// box filter of width delta: G = prod_a sin(k_a delta/2)/(k_a delta/2), real
__global__ void k_box_transfer(int n, int nh, int pitch, double delta, double2 *__restrict__ G)
{
    const int64_t nm = (int64_t)n * n * nh;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        ModeIdx m = mode_of(t, n, nh);
        double g = 1.0;
        double ks[3] = {m.ax, m.ay, m.az};
        for (int q = 0; q < 3; q++) { double h = 0.5 * ks[q] * delta; g *= (h == 0.0) ? 1.0 : sin(h) / h; }
        G[soff(m, n, pitch)] = make_double2(g, 0.0);
    }
}

// physical rows (pitch rp reals) -> compact FP32 [z][y][x]
// every stride-th point per axis of a physical field (m = n / stride points per axis)
__global__ void k_phys_to_f32(int n, int64_t rp, int stride, const double *__restrict__ src, float *__restrict__ dst)
{
    const int m = n / stride;
    const int64_t np = (int64_t)m * m * m;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / m, x = t - row * m, z = row / m, y = row - z * m;
        dst[t] = (float)src[(z * stride * n + y * stride) * rp + x * stride];
    }
}

// subgrid stress tau_ij = filter(u_i u_j) - filter(u_i) filter(u_j) in physical
// space, in place over the six filtered products P (pitch rp reals, field stride
// fs reals); UB = the three filtered velocities
__global__ void k_sgs_tau(int n, int64_t rp, int64_t fs, const double *__restrict__ UB, double *__restrict__ P)
{
    const int64_t np = (int64_t)n * n * n;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t row = t / n, x = t - row * n;
        const int64_t o = row * rp + x;
        const double u = UB[o], v = UB[fs + o], w = UB[2 * fs + o];
        P[o] -= u * u;
        P[fs + o] -= u * v;
        P[2 * fs + o] -= u * w;
        P[3 * fs + o] -= v * v;
        P[4 * fs + o] -= v * w;
        P[5 * fs + o] -= w * w;
    }
}

// restart body (restart_io.f90:240-334): each variable's Fourier array without
// its last two rows (the kx = N/2 pair), i.e. [ky][kz][kx < N/2] complex; to and
// from the device layout [kz][ky][kx] (pitch P).  The unpacked kx = N/2 modes
// are zero (every dealiasing rule zeroes them).
__global__ void k_dev_to_restart(int n, int pitch, const double2 *__restrict__ D, double2 *__restrict__ R)
{
    const int nk = n / 2;
    const int64_t nm = (int64_t)n * n * nk;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        const int kx = (int)(t % nk);
        const int64_t r = t / nk;
        const int kzi = (int)(r % n), kyi = (int)(r / n);
        R[t] = D[((int64_t)kzi * n + kyi) * pitch + kx];
    }
}
__global__ void k_restart_to_dev(int n, int pitch, const double2 *__restrict__ R, double2 *__restrict__ D)
{
    const int nk = n / 2, nh = nk + 1;
    const int64_t nm = (int64_t)n * n * nh;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        const int kx = (int)(t % nh);
        const int64_t r = t / nh;
        const int kzi = (int)(r % n), kyi = (int)(r / n);
        D[((int64_t)kzi * n + kyi) * pitch + kx] = kx < nk ? R[((int64_t)kyi * n + kzi) * nk + kx] : make_double2(0.0, 0.0);
    }
}

// The 2/3-rule band (every |k_i| <= kc = N/3) packed as [ky'][kz'][kx], ky' and
// kz' in [0, 2 kc] over the kept indices (0..kc, N-kc..N-1), kx in [0, kc]: the
// part of a dealiased state that is not zero by construction.  band -> the
// device layout writes every mode of the field (zero outside the band); the
// device layout -> band reads the band only.
__global__ void k_band_to_dev(int n, int kc, int pitch, const double2 *__restrict__ B, double2 *__restrict__ D)
{
    const int nh = n / 2 + 1, nb = 2 * kc + 1;
    const int64_t nm = (int64_t)n * n * nh;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        const int kx = (int)(t % nh);
        const int64_t r = t / nh;
        const int kyi = (int)(r % n), kzi = (int)(r / n);
        const int yb = kyi <= kc ? kyi : kyi >= n - kc ? kyi - (n - nb) : -1;
        const int zb = kzi <= kc ? kzi : kzi >= n - kc ? kzi - (n - nb) : -1;
        D[r * pitch + kx] =
            (kx <= kc && yb >= 0 && zb >= 0) ? B[((int64_t)yb * nb + zb) * (kc + 1) + kx] : make_double2(0.0, 0.0);
    }
}
__global__ void k_dev_to_band(int n, int kc, int pitch, const double2 *__restrict__ D, double2 *__restrict__ B)
{
    const int nb = 2 * kc + 1;
    const int64_t nm = (int64_t)nb * nb * (kc + 1);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        const int kx = (int)(t % (kc + 1));
        const int64_t r = t / (kc + 1);
        const int zb = (int)(r % nb), yb = (int)(r / nb);
        const int kyi = yb <= kc ? yb : yb + (n - nb), kzi = zb <= kc ? zb : zb + (n - nb);
        B[t] = D[((int64_t)kzi * n + kyi) * pitch + kx];
    }
}

// layout conversion between the reference's (nx+2, ny, nz) Fourier array
// [ky][kz][kx] (pitch nh) and the device layout [kz][ky][kx] (pitch P)
__global__ void k_ref_to_dev(int n, int nh, int pitch, const double2 *__restrict__ R, double2 *__restrict__ D)
{
    const int64_t nm = (int64_t)n * n * nh;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        int kx = (int)(t % nh);
        int64_t r = t / nh;
        int kzi = (int)(r % n), kyi = (int)(r / n);
        D[((int64_t)kzi * n + kyi) * pitch + kx] = R[t];
    }
}
__global__ void k_dev_to_ref(int n, int nh, int pitch, const double2 *__restrict__ D, double2 *__restrict__ R)
{
    const int64_t nm = (int64_t)n * n * nh;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nm; t += (int64_t)gridDim.x * blockDim.x) {
        int kx = (int)(t % nh);
        int64_t r = t / nh;
        int kzi = (int)(r % n), kyi = (int)(r / n);
        R[t] = D[((int64_t)kzi * n + kyi) * pitch + kx];
    }
}
