/*
 * hit3d_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * An FP64 CPU restatement of HIT3DP's pseudospectral timestep, written from the
 * reference Fortran sources, used as the parity checker for the CUDA path.  It is
 * loaded only by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
 * leg; the product library never links or calls it.
 *
 * Parity status: UNPINNED against the reference's own build.  The reference is
 * Fortran + MPI + FFTW3 and none of those toolchains exist on these machines, and
 * the reference ships no golden vectors.  This restatement is pinned only by
 *   - the analytic checks of the reference's (dead) test_rhs_velocity and
 *     test_rhs_scalars routines (rhs_velocity.f90:430-553, rhs_scalars.f90:504-594),
 *   - numpy.fft (pocketfft) for the transform conventions,
 *   - exact integer arithmetic for RANDu.
 *
 * Layout follows the reference exactly: every field is a column-major
 * (nx+2, ny, nz) real*8 array.  Physical space is (x, y, z); Fourier space is
 * (kx re/im interleaved, kz, ky) (x_fftw.f90:321-327).  The forward transform is
 * unnormalised, the inverse multiplies by 1/N^3 (x_fftw.f90:262,1070).
 *
 * Compile with -ffp-contract=off so that a*b+c is never fused, like gfortran -O2
 * on x86-64 without -march flags.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXS 8

/* ------------------------------------------------------------------------- */
/*  RANDu: L'Ecuyer with Bays-Durham shuffle (RANDu.f:12-52).                */
/*  Quirk kept: idum = nint(idum3/987) is recomputed from the caller's seed   */
/*  on every call (RANDu.f:27), so only idum2, iy and iv evolve.             */
/* ------------------------------------------------------------------------- */
typedef struct {
    int64_t idum2, iy, iv[32];
} randu_state;

static int64_t nint_d(double x) { return (int64_t)llround(x); }

void oracle_randu_reset(randu_state *s)
{
    s->idum2 = 123456789;
    s->iy = 0;
    for (int j = 0; j < 32; j++) s->iv[j] = 0;
}

double oracle_randu(randu_state *s, double idum3)
{
    const int64_t im1 = 2147483563, im2 = 2147483399, imm1 = im1 - 1;
    const int64_t ia1 = 40014, ia2 = 40692, iq1 = 53668, iq2 = 52774;
    const int64_t ir1 = 12211, ir2 = 3791, ntab = 32, ndiv = 1 + imm1 / ntab;
    const double am = 1.0 / (double)im1, eps = 1.2e-7, rnmx = 1.0 - eps;
    int64_t idum = nint_d(idum3 / 987.0);
    int64_t k, j;
    if (idum <= 0) {
        idum = (-idum > 1) ? -idum : 1;
        s->idum2 = idum;
        for (j = ntab + 8; j >= 1; j--) {
            k = idum / iq1;
            idum = ia1 * (idum - k * iq1) - k * ir1;
            if (idum < 0) idum += im1;
            if (j <= ntab) s->iv[j - 1] = idum;
        }
    }
    k = idum / iq1;
    idum = ia1 * (idum - k * iq1) - k * ir1;
    if (idum < 0) idum += im1;
    k = s->idum2 / iq2;
    s->idum2 = ia2 * (s->idum2 - k * iq2) - k * ir2;
    if (s->idum2 < 0) s->idum2 += im2;
    j = 1 + s->iy / ndiv;
    s->iy = s->iv[j - 1] - s->idum2;
    s->iv[j - 1] = idum;
    if (s->iy < 1) s->iy += imm1;
    double r = am * (double)s->iy;
    return r < rnmx ? r : rnmx;
}

/* Fill out[0..count) with the stream that begins with random(-seed) and
 * continues with random(seed), discarding the first value (init_velocity.f90:70-71). */
void oracle_randu_stream(double seed, int64_t count, double *out)
{
    randu_state s;
    oracle_randu_reset(&s);
    (void)oracle_randu(&s, -seed);
    for (int64_t i = 0; i < count; i++) out[i] = oracle_randu(&s, seed);
}

/* ------------------------------------------------------------------------- */
/*  1-D complex FFT, mixed radix 2/3/4/5, Stockham autosort.                  */
/*  Stands in for FFTW3's DFFTW_EXECUTE (x_fftw.f90:211-256).  Twiddles are  */
/*  computed in long double and rounded once.                                 */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n, nf, fac[40];
    double *tw; /* tw[2t], tw[2t+1] = cos(2 pi t/n), -sin(2 pi t/n) */
} fftplan;

static void plan_init(fftplan *p, int n)
{
    p->n = n;
    p->nf = 0;
    int m = n;
    while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
    while (m % 3 == 0) { p->fac[p->nf++] = 3; m /= 3; }
    while (m % 5 == 0) { p->fac[p->nf++] = 5; m /= 5; }
    if (m != 1) { fprintf(stderr, "oracle: unsupported FFT length %d\n", n); abort(); }
    p->tw = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int t = 0; t < n; t++) {
        long double a = twopi * (long double)t / (long double)n;
        p->tw[2 * t] = (double)cosl(a);
        p->tw[2 * t + 1] = (double)(-sinl(a));
    }
}

static void plan_free(fftplan *p) { free(p->tw); p->tw = NULL; }

/* x: interleaved complex of length n; y: scratch of the same size.
 * sign = -1 forward (e^{-i...}), +1 backward, both unnormalised. */
static void fft1d(const fftplan *p, double *x, double *y, int sign)
{
    const int n = p->n;
    double *src = x, *dst = y;
    int Ns = 1;
    for (int s = 0; s < p->nf; s++) {
        const int R = p->fac[s], m = n / R, step = n / (Ns * R);
        for (int j = 0; j < m; j++) {
            const int k = j % Ns;
            double ar[5], ai[5];
            for (int r = 0; r < R; r++) {
                double xr = src[2 * (j + r * m)], xi = src[2 * (j + r * m) + 1];
                int t = (r * k * step) % n;
                double wr = p->tw[2 * t], wi = p->tw[2 * t + 1];
                if (sign > 0) wi = -wi;
                ar[r] = xr * wr - xi * wi;
                ai[r] = xr * wi + xi * wr;
            }
            double br[5], bi[5];
            if (R == 2) {
                br[0] = ar[0] + ar[1]; bi[0] = ai[0] + ai[1];
                br[1] = ar[0] - ar[1]; bi[1] = ai[0] - ai[1];
            } else if (R == 4) {
                double s0r = ar[0] + ar[2], s0i = ai[0] + ai[2];
                double d0r = ar[0] - ar[2], d0i = ai[0] - ai[2];
                double s1r = ar[1] + ar[3], s1i = ai[1] + ai[3];
                double d1r = ar[1] - ar[3], d1i = ai[1] - ai[3];
                /* multiply d1 by -i*sign... forward: -i, backward: +i */
                double er, ei;
                if (sign < 0) { er = d1i; ei = -d1r; } else { er = -d1i; ei = d1r; }
                br[0] = s0r + s1r; bi[0] = s0i + s1i;
                br[2] = s0r - s1r; bi[2] = s0i - s1i;
                br[1] = d0r + er;  bi[1] = d0i + ei;
                br[3] = d0r - er;  bi[3] = d0i - ei;
            } else {
                /* direct DFT for radix 3 and 5 */
                for (int q = 0; q < R; q++) {
                    double sr = 0.0, si = 0.0;
                    for (int r = 0; r < R; r++) {
                        int t = ((q * r) % R) * (n / R);
                        double wr = p->tw[2 * t], wi = p->tw[2 * t + 1];
                        if (sign > 0) wi = -wi;
                        sr += ar[r] * wr - ai[r] * wi;
                        si += ar[r] * wi + ai[r] * wr;
                    }
                    br[q] = sr; bi[q] = si;
                }
            }
            const int base = (j / Ns) * Ns * R + k;
            for (int q = 0; q < R; q++) {
                dst[2 * (base + q * Ns)] = br[q];
                dst[2 * (base + q * Ns) + 1] = bi[q];
            }
        }
        double *t = src; src = dst; dst = t;
        Ns *= R;
    }
    if (src != x) memcpy(x, src, sizeof(double) * 2 * (size_t)n);
}

/* exported for the transform conventions test */
void oracle_fft1d(int n, double *x, int sign)
{
    fftplan p;
    plan_init(&p, n);
    double *y = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    fft1d(&p, x, y, sign);
    free(y);
    plan_free(&p);
}

/* ------------------------------------------------------------------------- */
/*  Oracle state: module globals of m_fields / m_work / x_fftw / m_force.    */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n, nscal, nles, dealias, flow_type, force_type, kfmax, kmax, les_model, nwrk;
    int isp_type;
    double nu, dt, famp, dx, c_smag, les_delta, peak_wavenum, ir_exp;
    double pe[MAXS + 1];
    int scalar_type[MAXS];
    size_t fsz;               /* (n+2)*n*n */
    double *fields, *rhs_old, *wrk, *turb_visc;
    double *akx, *aky, *akz;
    signed char *ialias;
    int nfn, *fn_i, *fn_j, *fn_k;  /* forced nodes */
    fftplan plan;
    double courant, time;
    double les_stat[4];       /* les.gp: mean k_sgs, production, B, dissipation */
    randu_state rs;           /* RANDu module state (RANDu.f:20-22), kept between initial conditions */
    double reac[MAXS];        /* reaction rates reac_sc of the scalars (rhs_scalars.f90:281-303) */
    double c_t, c_mixed;      /* lag-model scale (c_t.in) and mixed-model fraction (c_mixed.in) */
    double *gfilt;            /* test filter transfer function (DSTM models) */
    double *vsrc;             /* vel_source_les: 3 fields (DSTM models) */
    double *tauij;            /* tauij: 6 fields, strain then stress (les_model 10) */
    int fov, fos, int_scalars;
    double *scratch;          /* per-thread FFT scratch: nthreads * 4n doubles */
    int nthreads;
} oracle_t;

#define IX(o, i, j, k) ((size_t)(i) + (size_t)((o)->n + 2) * ((size_t)(j) + (size_t)(o)->n * (size_t)(k)))
#define F(o, m) ((o)->fields + (size_t)(m) * (o)->fsz)
#define W(o, m) ((o)->wrk + (size_t)(m) * (o)->fsz)
#define RO(o, m) ((o)->rhs_old + (size_t)(m) * (o)->fsz)

static int nint_shell32(double k2)
{
    /* nint(sqrt(real(k2,4))) -- float32 sqrt (m_stats.f90:218, m_force.f90:270) */
    float f = (float)k2;
    float s = sqrtf(f);
    return (int)lroundf(s);
}

static int nint_shell64(double k2)
{
    /* nint(sqrt(k2)) in FP64 (init_velocity.f90:127) */
    return (int)llround(sqrt(k2));
}

static int tid(void)
{
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}

/* x_fftw_init tables (x_fftw.f90:261-310) */
static void tables_init(oracle_t *o)
{
    int n = o->n;
    o->akx = (double *)calloc(n + 2, sizeof(double));
    o->aky = (double *)calloc(n, sizeof(double));
    o->akz = (double *)calloc(n, sizeof(double));
    for (int i = 0; i < n + 2; i += 2) { o->akx[i] = (double)(i / 2); o->akx[i + 1] = o->akx[i]; }
    for (int k = 0; k < n; k++) { double a = (double)k; if (a > 0.5 * n) a -= n; o->aky[k] = a; }
    for (int j = 0; j < n; j++) { double a = (double)j; if (a > 0.5 * n) a -= n; o->akz[j] = a; }
    o->ialias = (signed char *)calloc(o->fsz, 1);
    double rnx3 = (double)(n / 3);
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 2; i++) {
                int c = 0;
                if (fabs(o->aky[k]) > rnx3) c++;
                if (fabs(o->akz[j]) > rnx3) c++;
                if (fabs(o->akx[i]) > rnx3) c++;
                o->ialias[IX(o, i, j, k)] = (signed char)c;
            }
}

/* ------------------------------------------------------------------------- */
/*  3-D transforms on one (nx+2,ny,nz) array (x_fftw.f90:852-1085)           */
/* ------------------------------------------------------------------------- */
static void swap_yz(oracle_t *o, double *a)
{
    int n = o->n;
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < n; k++)
        for (int j = k + 1; j < n; j++)
            for (int i = 0; i < n + 2; i++) {
                double t = a[IX(o, i, j, k)];
                a[IX(o, i, j, k)] = a[IX(o, i, k, j)];
                a[IX(o, i, k, j)] = t;
            }
}

/* complex FFT along dim 2 (index j) for every kx and every k */
static void c2c_dim2(oracle_t *o, double *a, int sign)
{
    int n = o->n, nh = n / 2 + 1;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; k++) {
        double *buf = o->scratch + (size_t)tid() * 4 * n;
        double *y = buf + 2 * n;
        for (int ix = 0; ix < nh; ix++) {
            for (int j = 0; j < n; j++) {
                buf[2 * j] = a[IX(o, 2 * ix, j, k)];
                buf[2 * j + 1] = a[IX(o, 2 * ix + 1, j, k)];
            }
            fft1d(&o->plan, buf, y, sign);
            for (int j = 0; j < n; j++) {
                a[IX(o, 2 * ix, j, k)] = buf[2 * j];
                a[IX(o, 2 * ix + 1, j, k)] = buf[2 * j + 1];
            }
        }
    }
}

/* r2c along x for every (j,k): two real rows per complex transform */
static void r2c_x(oracle_t *o, double *a)
{
    int n = o->n;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; k++) {
        double *z = o->scratch + (size_t)tid() * 4 * n;
        double *y = z + 2 * n;
        for (int j = 0; j < n; j += 2) {
            double *ra = a + IX(o, 0, j, k), *rb = a + IX(o, 0, j + 1, k);
            for (int t = 0; t < n; t++) { z[2 * t] = ra[t]; z[2 * t + 1] = rb[t]; }
            fft1d(&o->plan, z, y, -1);
            for (int kx = 0; kx <= n / 2; kx++) {
                int m = (n - kx) % n;
                double zr = z[2 * kx], zi = z[2 * kx + 1];
                double mr = z[2 * m], mi = -z[2 * m + 1];
                ra[2 * kx] = 0.5 * (zr + mr);
                ra[2 * kx + 1] = 0.5 * (zi + mi);
                rb[2 * kx] = 0.5 * (zi - mi);
                rb[2 * kx + 1] = -0.5 * (zr - mr);
            }
        }
    }
}

/* c2r along x for every (j,k), times norm; imaginary parts of kx=0 and kx=N/2
 * are ignored, as in FFTW's c2r. */
static void c2r_x(oracle_t *o, double *a, double norm)
{
    int n = o->n;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; k++) {
        double *z = o->scratch + (size_t)tid() * 4 * n;
        double *y = z + 2 * n;
        for (int j = 0; j < n; j += 2) {
            double *ra = a + IX(o, 0, j, k), *rb = a + IX(o, 0, j + 1, k);
            for (int kx = 0; kx <= n / 2; kx++) {
                double xar = ra[2 * kx], xai = ra[2 * kx + 1];
                double xbr = rb[2 * kx], xbi = rb[2 * kx + 1];
                if (kx == 0 || kx == n / 2) { xai = 0.0; xbi = 0.0; }
                z[2 * kx] = xar - xbi;
                z[2 * kx + 1] = xai + xbr;
                if (kx > 0 && kx < n / 2) {
                    z[2 * (n - kx)] = xar + xbi;
                    z[2 * (n - kx) + 1] = -xai + xbr;
                }
            }
            fft1d(&o->plan, z, y, +1);
            for (int t = 0; t < n; t++) { ra[t] = norm * z[2 * t]; rb[t] = norm * z[2 * t + 1]; }
        }
    }
}

static void xfft3d(oracle_t *o, int flag, double *a)
{
    int n = o->n;
    if (flag == 1) {
        r2c_x(o, a);
        /* c2c along y within each z-plane: layout (kx, ky, z) */
        c2c_dim2(o, a, -1);
        swap_yz(o, a);
        c2c_dim2(o, a, -1);
    } else {
        c2c_dim2(o, a, +1);
        swap_yz(o, a);
        c2c_dim2(o, a, +1);
        c2r_x(o, a, 1.0 / ((double)n * (double)n * (double)n));
    }
}

void oracle_fft3d(oracle_t *o, int flag, double *a) { xfft3d(o, flag, a); }

/* ------------------------------------------------------------------------- */
/*  create / destroy                                                          */
/* ------------------------------------------------------------------------- */
void oracle_filter_g(oracle_t *o, int kind, double delta, double *g);
void oracle_apply_filter(oracle_t *o, const double *g, double *a);

oracle_t *oracle_create(int n, int nscal, int dealias, int flow_type, int force_type, int kfmax,
                        double nu, double dt, double famp, int les_model, double c_smag,
                        const double *sc, const int *scalar_type)
{
    if (nscal > MAXS) return NULL;
    oracle_t *o = (oracle_t *)calloc(1, sizeof(oracle_t));
    o->n = n; o->nscal = nscal; o->dealias = dealias; o->flow_type = flow_type;
    o->force_type = force_type; o->kfmax = kfmax; o->nu = nu; o->dt = dt; o->famp = famp;
    o->les_model = les_model; o->c_smag = c_smag;
    o->dx = 2.0 * (4.0 * atan(1.0)) / (double)n;
    o->les_delta = o->dx;
    /* LES-related transported quantities: k_sgs for the DLM (m_les.f90:111-123);
     * k_sgs, (B T_B), (eps T_eps) with the lag model (m_les.f90:124-137); all
     * with Schmidt number one (m_les.f90:372-391) */
    o->nles = (les_model == 2 || les_model == 4 || les_model == 6) ? 1
            : (les_model == 3 || les_model == 5 || les_model == 7) ? 3 : les_model == 10 ? 2 : 0;
    o->c_t = 1.0;
    o->c_mixed = 0.0;
    oracle_randu_reset(&o->rs);
    /* passive scalars go with les_models 0-3 and 10 (m_les.f90:725-800 stops on 4-7) */
    if (nscal > 0 && les_model >= 4 && les_model <= 7) { free(o); return NULL; }
    /* kmax (m_parameters.f90:123-131) */
    if (dealias == 0) o->kmax = n / 3;
    else o->kmax = (int)floor((double)n / 3.0 * sqrt(2.0));
    for (int s = 0; s < nscal; s++) { o->pe[s] = nu / sc[s]; o->scalar_type[s] = scalar_type[s]; }
    for (int j = 0; j < o->nles; j++) o->pe[nscal + j] = nu / 1.0;
    o->fsz = (size_t)(n + 2) * n * n;
    o->nwrk = 7;
    if (6 + nscal + o->nles > o->nwrk) o->nwrk = 6 + nscal + o->nles;
    if (dealias == 1 && 3 + nscal + o->nles + 6 > o->nwrk) o->nwrk = 3 + nscal + o->nles + 6;
    /* the DSTM models use four work arrays past the LES fields (m_work.f90) */
    if (les_model >= 4 && 3 + nscal + o->nles + 5 > o->nwrk) o->nwrk = 3 + nscal + o->nles + 5;
    o->fields = (double *)calloc(o->fsz * (3 + nscal + o->nles), sizeof(double));
    o->rhs_old = (double *)calloc(o->fsz * (3 + nscal + o->nles), sizeof(double));
    o->wrk = (double *)calloc(o->fsz * o->nwrk, sizeof(double));
    if (les_model) o->turb_visc = (double *)calloc(o->fsz, sizeof(double));
    if (!o->fields || !o->rhs_old || !o->wrk) return NULL;
    tables_init(o);
    plan_init(&o->plan, n);
#ifdef _OPENMP
    o->nthreads = omp_get_max_threads();
#else
    o->nthreads = 1;
#endif
    o->scratch = (double *)malloc(sizeof(double) * 4 * (size_t)n * o->nthreads);
    /* forced node list (m_force.f90:13-97), loop order k, j, i over i<nx */
    if (flow_type == 1) {
        int cnt = 0;
        for (int pass = 0; pass < 2; pass++) {
            int m = 0;
            for (int k = 0; k < n; k++)
                for (int j = 0; j < n; j++)
                    for (int i = 0; i < n; i++) {
                        double k2 = o->akx[i] * o->akx[i] + o->aky[k] * o->aky[k] + o->akz[j] * o->akz[j];
                        int sh = nint_shell32(k2);
                        if (sh > 0 && sh <= kfmax) {
                            if (pass == 1) { o->fn_i[m] = i; o->fn_j[m] = j; o->fn_k[m] = k; }
                            m++;
                        }
                    }
            if (pass == 0) {
                cnt = m;
                o->fn_i = (int *)malloc(sizeof(int) * (cnt + 1));
                o->fn_j = (int *)malloc(sizeof(int) * (cnt + 1));
                o->fn_k = (int *)malloc(sizeof(int) * (cnt + 1));
            }
        }
        o->nfn = cnt;
    }
    o->fov = 1; o->fos = 1; o->int_scalars = nscal > 0;
    /* m_les_dlm_k_init (m_les.f90:1394-1413): k_sgs = 0.1 in physical space,
     * i.e. only the (0,0,0) mode, 0.1 N^3 after the unnormalised transform */
    if (o->nles) F(o, 3 + nscal)[0] = 0.1 * (double)n * (double)n * (double)n;
    /* lag model: (B T_B) = (eps T_eps) = 0.5 k_sgs (m_les.f90:474-479) */
    if (les_model == 3) F(o, 4 + nscal)[0] = F(o, 5 + nscal)[0] = 0.5 * F(o, 3 + nscal)[0];
    /* DSTM models (m_les_begin, m_les.f90:485-570): k_sgs = 0.2 (4) or 0.5
     * (5-7); with the lag model (B T_B) = k_sgs and (eps T_eps) = 0; the test
     * filter is the Gaussian of width 4 dx (m_filter_xfftw.f90:140-150) */
    if (les_model >= 4 && les_model <= 7) {
        const double n3 = (double)n * (double)n * (double)n;
        F(o, 3 + nscal)[0] = (les_model == 4 ? 0.2 : 0.5) * n3;
        if (o->nles == 3) { F(o, 4 + nscal)[0] = F(o, 3 + nscal)[0]; F(o, 5 + nscal)[0] = 0.0; }
        o->gfilt = (double *)calloc(o->fsz, sizeof(double));
        o->vsrc = (double *)calloc(3 * o->fsz, sizeof(double));
        oracle_filter_g(o, 2, 4.0 * o->dx, o->gfilt);
    }
    /* les_model 10 (m_les.f90:592-608): (B T_B) = (eps T_eps) = 0.1, no k_sgs */
    if (les_model == 10) {
        const double n3 = (double)n * (double)n * (double)n;
        F(o, 3 + nscal)[0] = 0.1 * n3;
        F(o, 4 + nscal)[0] = 0.1 * n3;
        o->gfilt = (double *)calloc(o->fsz, sizeof(double));
        o->tauij = (double *)calloc(6 * o->fsz, sizeof(double));
        oracle_filter_g(o, 2, 4.0 * o->dx, o->gfilt);
    }
    return o;
}

void oracle_destroy(oracle_t *o)
{
    if (!o) return;
    free(o->fields); free(o->rhs_old); free(o->wrk); free(o->turb_visc);
    free(o->akx); free(o->aky); free(o->akz); free(o->ialias);
    free(o->fn_i); free(o->fn_j); free(o->fn_k); free(o->scratch);
    free(o->gfilt); free(o->vsrc); free(o->tauij);
    plan_free(&o->plan);
    free(o);
}

double *oracle_fields(oracle_t *o) { return o->fields; }
double *oracle_rhs_old(oracle_t *o) { return o->rhs_old; }
double *oracle_wrk(oracle_t *o) { return o->wrk; }
int oracle_nwrk(oracle_t *o) { return o->nwrk; }

/* restart_read_parallel (restart_io.f90:341-506), one task: the 36-byte header
 * (nx, ny, nz, nums, nles as int32, TIME and DT as float64), a dimension check,
 * then rows 1..nx of every variable into fields(1:nx, :, :, n) for the velocity
 * and min(nums, n_scalars) scalars, and the LES variables from after the file's
 * nums scalars.  Rows nx+1, nx+2 and fields the file lacks are zeroed (the
 * reference initialises added scalars afterwards; the caller does that here).
 * Returns 0, or -1 (no file / short read), -2 (dimensions differ). */
int oracle_read_restart(oracle_t *o, const char *path, double *time, double *dt, int *nums_file, int *nles_file)
{
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    int32_t h[5];
    double td[2];
    if (fread(h, 4, 5, f) != 5 || fread(td, 8, 2, f) != 2) { fclose(f); return -1; }
    const int n = o->n;
    if (h[0] != n || h[1] != n || h[2] != n) { fclose(f); return -2; }
    const int nums1 = h[3], nles1 = h[4];
    const size_t fsz = o->fsz, per = (size_t)n * n * n;
    double *tmp = (double *)malloc(sizeof(double) * per);
    if (!tmp) { fclose(f); return -1; }
    memset(o->fields, 0, sizeof(double) * fsz * (size_t)(3 + o->nscal + o->nles));
    const int nread = 3 + (o->nscal < nums1 ? o->nscal : nums1);
    int rc = 0;
    for (int v = 0; v < nread + o->nles && rc == 0; v++) {
        int field, var;
        if (v < nread) { field = v; var = v; }
        else {
            const int j = v - nread;
            if (j >= nles1) break;
            field = 3 + o->nscal + j;
            var = 3 + nums1 + j;
        }
        if (fseek(f, 36 + (long)var * (long)(per * 8), SEEK_SET) != 0 || fread(tmp, 8, per, f) != per) { rc = -1; break; }
        double *dst = o->fields + (size_t)field * fsz;
        for (size_t row = 0; row < (size_t)n * n; row++)
            memcpy(dst + row * (size_t)(n + 2), tmp + row * (size_t)n, sizeof(double) * (size_t)n);
    }
    free(tmp);
    fclose(f);
    if (rc == 0) {
        if (time) *time = td[0];
        if (dt) *dt = td[1];
        if (nums_file) *nums_file = nums1;
        if (nles_file) *nles_file = nles1;
    }
    return rc;
}
void oracle_set_reaction(oracle_t *o, int s, double rate) { o->reac[s] = rate; }
/* C_T of les_model 5 (c_t.in) and C_mixed of les_models 6, 7 (c_mixed.in) */
void oracle_set_les_constants(oracle_t *o, double c_t, double c_mixed) { o->c_t = c_t; o->c_mixed = c_mixed; }
int oracle_kmax(oracle_t *o) { return o->kmax; }
int oracle_nforced(oracle_t *o) { return o->nfn; }
double oracle_courant(oracle_t *o) { return o->courant; }
void oracle_set_dt(oracle_t *o, double dt) { o->dt = dt; }
void oracle_set_flags(oracle_t *o, int fov, int fos, int int_scalars)
{
    o->fov = fov; o->fos = fos; o->int_scalars = int_scalars;
}
void oracle_get_flags(oracle_t *o, int *flags) { flags[0] = o->fov; flags[1] = o->fos; flags[2] = o->int_scalars; }

/* ------------------------------------------------------------------------- */
/*  dealias_all (dealias_all.f90:97-131)                                     */
/* ------------------------------------------------------------------------- */
void oracle_dealias_all(oracle_t *o)
{
    int n = o->n;
    double akmax = (double)o->kmax;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 2; i++)
                if (fabs(o->akx[i]) > akmax || fabs(o->aky[k]) > akmax || fabs(o->akz[j]) > akmax)
                    for (int m = 0; m < 3 + o->nscal; m++) F(o, m)[IX(o, i, j, k)] = 0.0;
}

/* ------------------------------------------------------------------------- */
/*  Smagorinsky turbulent viscosity (m_les.f90:1142-1215)                    */
/* ------------------------------------------------------------------------- */
static void strain_first(oracle_t *o, int second)
{
    int n = o->n;
    double *u = F(o, 0), *v = F(o, 1), *w = F(o, 2);
    double *w4 = W(o, 4), *w5 = W(o, 5), *w6 = W(o, 6);
    const double half = 0.5;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 1; i += 2) {
                size_t a = IX(o, i, j, k), b = a + 1;
                double kx0 = o->akx[i], kx1 = o->akx[i + 1], ky = o->aky[k], kz = o->akz[j];
                if (!second) {
                    w4[a] = -kx1 * u[b];
                    w4[b] = kx0 * u[a];
                    w5[a] = -half * (ky * u[b] + kx1 * v[b]);
                    w5[b] = half * (ky * u[a] + kx0 * v[a]);
                    w6[a] = -half * (kz * u[b] + kx1 * w[b]);
                    w6[b] = half * (kz * u[a] + kx0 * w[a]);
                } else {
                    w4[a] = -ky * v[b];
                    w4[b] = ky * v[a];
                    w5[a] = -half * (kz * v[b] + ky * w[b]);
                    w5[b] = half * (kz * v[a] + ky * w[a]);
                    w6[a] = -kz * w[b];
                    w6[b] = kz * w[a];
                }
            }
}

static void les_get_turb_visc_smag(oracle_t *o)
{
    int n = o->n;
    double *tv = o->turb_visc;
    strain_first(o, 0);
    for (int m = 4; m <= 6; m++) xfft3d(o, -1, W(o, m));
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                size_t a = IX(o, i, j, k);
                double s4 = W(o, 4)[a], s5 = W(o, 5)[a], s6 = W(o, 6)[a];
                double t = s4 * s4;
                t = t + 2.0 * (s5 * s5);
                t = t + 2.0 * (s6 * s6);
                tv[a] = t;
            }
    strain_first(o, 1);
    for (int m = 4; m <= 6; m++) xfft3d(o, -1, W(o, m));
    double cd = o->c_smag * o->les_delta;
    cd = cd * cd;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                size_t a = IX(o, i, j, k);
                double s4 = W(o, 4)[a], s5 = W(o, 5)[a], s6 = W(o, 6)[a];
                double t = tv[a] + s4 * s4;
                t = t + 2.0 * (s5 * s5);
                t = t + s6 * s6;
                t = sqrt(2.0 * t);
                tv[a] = t * cd;
            }
}

/* les_rhsv_turb_visc (m_les.f90:902-1018) followed by the ialias mask of
 * les_rhs_velocity (m_les.f90:682-690) */
static void derivative(oracle_t *o, const double *src, char axis, double *dst);
static void les_rhs_velocity(oracle_t *o)
{
    int n = o->n;
    double *tv = o->turb_visc;
    /* les_rhs_velocity (m_les.f90:635-676): the DSTM velocity sources (4-7),
     * the eddy-viscosity stress (1-3, 6, 7) */
    if (o->les_model >= 4 && o->les_model <= 7)
        for (int m = 0; m < 3; m++) {
            double *r = W(o, 1 + m), *vs = o->vsrc + (size_t)m * o->fsz;
            for (size_t q = 0; q < o->fsz; q++) r[q] = r[q] + vs[q];
        }
    if (o->les_model == 10) {
        /* les_add_vel_source_from_tauij (m_les.f90:2344-2392) */
        const size_t fsz = o->fsz;
        const int comp[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
        const char dirs[3] = {'x', 'y', 'z'};
        for (int q = 0; q < 6; q++) xfft3d(o, 1, o->tauij + (size_t)q * fsz);
        double *d = W(o, 3 + o->nscal + o->nles + 1);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                derivative(o, o->tauij + (size_t)comp[i][j] * fsz, dirs[j], d);
                double *r = W(o, 1 + i);
                for (size_t q = 0; q < fsz; q++) r[q] = r[q] - d[q];
            }
    }
    const int eddy = o->les_model <= 3 || o->les_model == 6 || o->les_model == 7;
    for (int pass = 0; pass < (eddy ? 2 : 0); pass++) {
        strain_first(o, pass);
        for (int m = 4; m <= 6; m++) {
            double *a = W(o, m);
            xfft3d(o, -1, a);
            for (int k = 0; k < n; k++)
                for (int j = 0; j < n; j++)
                    for (int i = 0; i < n; i++) {
                        size_t q = IX(o, i, j, k);
                        a[q] = -2.0 * tv[q] * a[q];
                    }
            xfft3d(o, 1, a);
        }
        double *r1 = W(o, 1), *r2 = W(o, 2), *r3 = W(o, 3);
        double *w4 = W(o, 4), *w5 = W(o, 5), *w6 = W(o, 6);
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n + 1; i += 2) {
                    size_t a = IX(o, i, j, k), b = a + 1;
                    if (o->ialias[a] != 0) continue;
                    double kx0 = o->akx[i], kx1 = o->akx[i + 1], ky = o->aky[k], kz = o->akz[j];
                    if (pass == 0) {
                        r1[a] = r1[a] + kx1 * w4[b] + ky * w5[b] + kz * w6[b];
                        r1[b] = r1[b] - kx0 * w4[a] - ky * w5[a] - kz * w6[a];
                        r2[a] = r2[a] + kx1 * w5[b];
                        r2[b] = r2[b] - kx0 * w5[a];
                        r3[a] = r3[a] + kx1 * w6[b];
                        r3[b] = r3[b] - kx0 * w6[a];
                    } else {
                        r2[a] = r2[a] + ky * w4[b] + kz * w5[b];
                        r2[b] = r2[b] - ky * w4[a] - kz * w5[a];
                        r3[a] = r3[a] + ky * w5[b] + kz * w6[b];
                        r3[b] = r3[b] - ky * w5[a] - kz * w6[a];
                    }
                }
    }
    for (size_t q = 0; q < o->fsz; q++)
        if (o->ialias[q] != 0) { W(o, 1)[q] = 0.0; W(o, 2)[q] = 0.0; W(o, 3)[q] = 0.0; }
}

/* ------------------------------------------------------------------------- */
/*  Dynamic localization model (les_model 2)                                  */
/* ------------------------------------------------------------------------- */
static void copy_field(oracle_t *o, double *dst, const double *src);

/* les_get_turb_visc_dlm (m_les.f90:1313-1388): nu_t = C_k Delta sqrt(k_sgs)
 * from k_sgs truncated to |k|^2 <= kmax^2; if k_sgs < 0 anywhere, the clipped
 * field replaces the state. */
static void les_get_turb_visc_dlm(oracle_t *o)
{
    int n = o->n, nk = 3 + o->nscal;
    const double C_k = 0.1;
    double *w0 = W(o, 0), *tv = o->turb_visc;
    copy_field(o, w0, F(o, nk));
    const double rkmax2 = (double)(o->kmax * o->kmax);
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 2; i++) {
                double wmag2 = o->akx[i] * o->akx[i] + o->aky[k] * o->aky[k] + o->akz[j] * o->akz[j];
                if (wmag2 > rkmax2) w0[IX(o, i, j, k)] = 0.0;
            }
    xfft3d(o, -1, w0);
    double mn = w0[0];
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                double v = w0[IX(o, i, j, k)];
                if (v < mn) mn = v;
            }
    if (mn < 0.0)
        for (size_t q = 0; q < o->fsz; q++) w0[q] = w0[q] > 0.0 ? w0[q] : 0.0;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                size_t a = IX(o, i, j, k);
                tv[a] = C_k * o->les_delta * sqrt(w0[a]);
            }
    if (mn < 0.0) {
        xfft3d(o, 1, w0);
        copy_field(o, F(o, nk), w0);
    }
}

/* m_les_k_src_dlm (m_les.f90:1422-1561): production 2 nu_t S_ij S_ij of
 * k_sgs, added to its RHS where ialias == 0.  The strain components are taken
 * where ialias == 0 and zero elsewhere.  (The reference zeroes its two work
 * arrays only before the first of the three passes, so from the second pass on
 * their aliased entries still hold the previous pass's physical values; that
 * content depends on what the transform library leaves in the row padding and
 * cannot be reproduced.  Every pass starts from zero here.) */
static void strain_pair(oracle_t *o, int pass, double *s1, double *s2)
{
    int n = o->n;
    double *u = F(o, 0), *v = F(o, 1), *w = F(o, 2);
    const double half = 0.5;
    memset(s1, 0, sizeof(double) * o->fsz);
    memset(s2, 0, sizeof(double) * o->fsz);
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 1; i += 2) {
                size_t a = IX(o, i, j, k), b = a + 1;
                if (o->ialias[a] != 0) continue;
                double kx0 = o->akx[i], kx1 = o->akx[i + 1], ky = o->aky[k], kz = o->akz[j];
                if (pass == 0) {
                    s1[a] = -kx1 * u[b];  s1[b] = kx0 * u[a];                         /* S11 */
                    s2[a] = -half * (ky * u[b] + kx1 * v[b]);                         /* S12 */
                    s2[b] = half * (ky * u[a] + kx0 * v[a]);
                } else if (pass == 1) {
                    s1[a] = -half * (kz * u[b] + kx1 * w[b]);                         /* S13 */
                    s1[b] = half * (kz * u[a] + kx0 * w[a]);
                    s2[a] = -ky * v[b];  s2[b] = ky * v[a];                           /* S22 */
                } else {
                    s1[a] = -half * (kz * v[b] + ky * w[b]);                          /* S23 */
                    s1[b] = half * (kz * v[a] + ky * w[a]);
                    s2[a] = -kz * w[b];  s2[b] = kz * w[a];                           /* S33 */
                }
            }
}

static void les_k_src_dlm(oracle_t *o)
{
    int n1 = 3 + o->nscal + o->nles + 1, n2 = n1 + 1, kn = 3 + o->nscal + 1;
    double *w0 = W(o, 0), *a1 = W(o, n1), *a2 = W(o, n2), *tv = o->turb_visc;
    memset(w0, 0, sizeof(double) * o->fsz);
    for (int pass = 0; pass < 3; pass++) {
        strain_pair(o, pass, a1, a2);
        xfft3d(o, -1, a1);
        xfft3d(o, -1, a2);
        /* S11^2 + 2 S12^2, then 2 S13^2 + S22^2, then 2 S23^2 + S33^2 */
        const double c1 = pass == 0 ? 1.0 : 2.0, c2 = pass == 0 ? 2.0 : 1.0;
        for (size_t q = 0; q < o->fsz; q++) {
            double t = w0[q];
            t = t + (pass == 0 ? a1[q] * a1[q] : c1 * (a1[q] * a1[q]));
            t = t + (pass == 0 ? c2 * (a2[q] * a2[q]) : a2[q] * a2[q]);
            w0[q] = t;
        }
    }
    for (size_t q = 0; q < o->fsz; q++) w0[q] = 2.0 * w0[q];
    /* with les_model 5 only |S|^2 in wrk0 is wanted (m_les.f90:1508-1510) */
    if (o->les_model == 5) return;
    int n = o->n;
    for (size_t q = 0; q < o->fsz; q++) a1[q] = w0[q];
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                size_t a = IX(o, i, j, k);
                a1[a] = a1[a] * tv[a];
            }
    xfft3d(o, 1, a1);
    /* saved for les.gp (m_les.f90:1536): the zero mode over N^3 */
    o->les_stat[1] += a1[0] / ((double)n * n * n);
    double *r = W(o, kn);
    for (size_t q = 0; q < o->fsz; q++)
        if (o->ialias[q] == 0) r[q] = r[q] + a1[q];
    /* with the lag model the transfer term is also a source for (B T_B)
     * (m_les.f90:1547-1557) */
    if (o->les_model == 3 || o->les_model == 7) {
        double *rb = W(o, kn + 1);
        for (size_t q = 0; q < o->fsz; q++)
            if (o->ialias[q] == 0) rb[q] = rb[q] + a1[q];
    }
}

/* m_les_lag_model_sources (m_les.f90:1629-1684): B = (B T_B) |S| with
 * |S|^2 = 2 S_ij S_ij left in wrk0 by les_k_src_dlm, eps = max(eps T_eps, 0)^1.5
 * / (Delta C_T^1.5); where ialias == 0 the RHS of k_sgs loses eps, that of
 * (B T_B) loses B and that of (eps T_eps) gains B - eps. */
static void les_lag_model_sources(oracle_t *o)
{
    /* C_T = 1 (m_les.f90:43-44) unless les_model 5 read c_t.in (m_les.f90:195-207) */
    const double C_T = o->les_model == 5 ? o->c_t : 1.0;
    int n = o->n, nk = 3 + o->nscal + 1, n1 = 3 + o->nscal + o->nles + 1, n2 = n1 + 1;
    double *w0 = W(o, 0), *b = W(o, n1), *e = W(o, n2);
    copy_field(o, b, F(o, nk));            /* (B T_B): field nk+1 in the 1-based count */
    xfft3d(o, -1, b);
    for (size_t q = 0; q < o->fsz; q++) b[q] = b[q] * sqrt(w0[q]);
    xfft3d(o, 1, b);
    copy_field(o, e, F(o, nk + 1));        /* (eps T_eps) */
    xfft3d(o, -1, e);
    for (size_t q = 0; q < o->fsz; q++) {
        double v = e[q] > 0.0 ? e[q] : 0.0;
        e[q] = pow(v, 1.5) / (o->les_delta * pow(C_T, 1.5));
    }
    xfft3d(o, 1, e);
    o->les_stat[2] += b[0] / ((double)n * n * n);
    o->les_stat[3] += e[0] / ((double)n * n * n);
    double *rk = W(o, nk), *rb = W(o, nk + 1), *re = W(o, nk + 2);
    for (size_t q = 0; q < o->fsz; q++)
        if (o->ialias[q] == 0) {
            rk[q] = rk[q] - e[q];
            rb[q] = rb[q] - b[q];
            re[q] = re[q] + b[q] - e[q];
        }
}

/* m_les_k_diss_algebraic (m_les.f90:1567-1621): dissipation k^(3/2)/Delta of
 * the dealiased, clipped k_sgs, subtracted where ialias == 0 */
static void les_k_diss_algebraic(oracle_t *o)
{
    int n = o->n, kn = 3 + o->nscal + 1;
    double *w0 = W(o, 0);
    copy_field(o, w0, F(o, kn - 1));
    for (size_t q = 0; q < o->fsz; q++)
        if (o->ialias[q] > 0) w0[q] = 0.0;
    xfft3d(o, -1, w0);
    for (size_t q = 0; q < o->fsz; q++) {
        double v = w0[q] > 0.0 ? w0[q] : 0.0;
        w0[q] = pow(v, 1.5) / o->les_delta;
    }
    xfft3d(o, 1, w0);
    o->les_stat[3] += w0[0] / ((double)n * n * n);    /* m_les.f90:1617 */
    double *r = W(o, kn);
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                size_t a = IX(o, i, j, k);
                if (o->ialias[a] == 0) r[a] = r[a] - w0[a];
            }
}

static void derivative(oracle_t *o, const double *src, char axis, double *dst);

/* m_les_dstm_vel_k_sources (m_les.f90:1697-1960), the Dynamic Structure Model:
 * tau_ij = 2 k_sgs / L_kk * L_ij with L_ij = (u_i u_j)~ - u~_i u~_j (~: the test
 * filter), max(k_sgs, 0) and max(L_kk, 1e-15); velocity sources -d tau_ij/dx_j
 * and the k_sgs source -tau_ij du_i/dx_j (also a source for (B T_B) with
 * les_models 5 and 7), all added where ialias == 0.  The reference's
 * diagnostic outputs of this routine (units 698, 699 and the k., L., F.,
 * tau.., pi. real*4 dumps) are left out. */
static void les_dstm_vel_k_sources(oracle_t *o)
{
    const int n = o->n, ns = o->nscal, nl = o->nles;
    const int nk = 3 + ns + 1;              /* 1-based field number of k_sgs */
    const int n2 = 3 + ns + nl + 1, n3 = n2 + 1, n4 = n2 + 2, n5 = n2 + 3;
    const double n3d = (double)n * n * n;
    double *w1 = W(o, 0), *a2 = W(o, n2), *a3 = W(o, n3), *a4 = W(o, n4), *a5 = W(o, n5);
    const size_t fsz = o->fsz;
    const char dirs[3] = {'x', 'y', 'z'};
    /* k_sgs in physical space */
    copy_field(o, w1, F(o, nk - 1));
    xfft3d(o, -1, w1);
    /* L_kk = (u_k u_k)~ - u~_k u~_k */
    copy_field(o, a3, F(o, 0)); copy_field(o, a4, F(o, 1)); copy_field(o, a5, F(o, 2));
    xfft3d(o, -1, a3); xfft3d(o, -1, a4); xfft3d(o, -1, a5);
    for (size_t q = 0; q < fsz; q++) a2[q] = a3[q] * a3[q] + a4[q] * a4[q] + a5[q] * a5[q];
    xfft3d(o, 1, a2);
    oracle_apply_filter(o, o->gfilt, a2);
    xfft3d(o, -1, a2);
    copy_field(o, a3, F(o, 0)); copy_field(o, a4, F(o, 1)); copy_field(o, a5, F(o, 2));
    oracle_apply_filter(o, o->gfilt, a3); oracle_apply_filter(o, o->gfilt, a4); oracle_apply_filter(o, o->gfilt, a5);
    xfft3d(o, -1, a3); xfft3d(o, -1, a4); xfft3d(o, -1, a5);
    for (size_t q = 0; q < fsz; q++) a2[q] = a2[q] - a3[q] * a3[q] - a4[q] * a4[q] - a5[q] * a5[q];
    /* the coefficient 2 k / L_kk */
    for (size_t q = 0; q < fsz; q++) {
        double kk = w1[q] > 0.0 ? w1[q] : 0.0, lk = a2[q] > 1.e-15 ? a2[q] : 1.e-15;
        w1[q] = 2.0 * kk / lk;
    }
    memset(o->vsrc, 0, sizeof(double) * 3 * fsz);
    double *rk = W(o, nk), *rb = W(o, nk + 1);
    const int to_b = o->les_model == 5 || o->les_model == 7;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            copy_field(o, a2, F(o, i)); copy_field(o, a3, F(o, j));
            copy_field(o, a4, F(o, i)); copy_field(o, a5, F(o, j));
            xfft3d(o, -1, a2); xfft3d(o, -1, a3);
            oracle_apply_filter(o, o->gfilt, a4); oracle_apply_filter(o, o->gfilt, a5);
            xfft3d(o, -1, a4); xfft3d(o, -1, a5);
            for (size_t q = 0; q < fsz; q++) a2[q] = a2[q] * a3[q];
            xfft3d(o, 1, a2);
            oracle_apply_filter(o, o->gfilt, a2);
            xfft3d(o, -1, a2);
            for (size_t q = 0; q < fsz; q++) {
                double t = a2[q] - a4[q] * a5[q];
                a2[q] = t * w1[q];                  /* tau_ij in physical space */
            }
            copy_field(o, a3, F(o, i));
            derivative(o, a3, dirs[j], a3);
            xfft3d(o, -1, a3);
            for (size_t q = 0; q < fsz; q++) a5[q] = -a3[q] * a2[q];
            xfft3d(o, 1, a2);
            xfft3d(o, 1, a5);
            for (size_t q = 0; q < fsz; q++) a3[q] = -a2[q];
            derivative(o, a3, dirs[j], a3);
            double *vs = o->vsrc + (size_t)i * fsz;
            for (size_t q = 0; q < fsz; q++)
                if (o->ialias[q] == 0) {
                    vs[q] = vs[q] + a3[q];
                    rk[q] = rk[q] + a5[q];
                    if (to_b) rb[q] = rb[q] + a5[q];
                }
            o->les_stat[1] += a5[0] / n3d;
        }
}

/* m_les_rhss_turb_visc1 (m_les.f90:1041-1091): sum_i d/dx_i (nu_t d phi/dx_i)
 * added to the RHS of field m where ialias == 0 */
static void les_rhss_turb_visc1(oracle_t *o, int m)
{
    int n = o->n;
    int t1 = 3 + o->nscal + o->nles + 1, t2 = t1 + 1;
    double *w0 = W(o, 0), *a1 = W(o, t1), *a2 = W(o, t2), *tv = o->turb_visc;
    copy_field(o, a1, F(o, m - 1));
    memset(w0, 0, sizeof(double) * o->fsz);
    const char dirs[3] = {'x', 'y', 'z'};
    for (int d = 0; d < 3; d++) {
        derivative(o, a1, dirs[d], a2);
        xfft3d(o, -1, a2);
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) {
                    size_t a = IX(o, i, j, k);
                    a2[a] = a2[a] * tv[a];
                }
        xfft3d(o, 1, a2);
        derivative(o, a2, dirs[d], a2);
        for (size_t q = 0; q < o->fsz; q++) w0[q] = w0[q] + a2[q];
    }
    double *r = W(o, m);
    for (size_t q = 0; q < o->fsz; q++)
        if (o->ialias[q] == 0) r[q] = r[q] + w0[q];
}

/* ------------------------------------------------------------------------- */
/*  rhs_scalars (rhs_scalars.f90:1-402)                                      */
/* ------------------------------------------------------------------------- */
static void phase_factors(oracle_t *o)
{
    int n = o->n;
    double *w0 = W(o, 0);
    const double half = 0.5;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 1; i += 2) {
                size_t a = IX(o, i, j, k);
                w0[a] = cos(half * (o->akx[i] + o->aky[k] + o->akz[j]) * o->dx);
                w0[a + 1] = sin(half * (o->akx[i + 1] + o->aky[k] + o->akz[j]) * o->dx);
            }
}

static void copy_field(oracle_t *o, double *dst, const double *src) { memcpy(dst, src, sizeof(double) * o->fsz); }

static void mul3(oracle_t *o, double *dst, const double *a, const double *b)
{
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < o->fsz; q++) dst[q] = a[q] * b[q];
}

static void les_dstm_vel_k_sources(oracle_t *o);
static void les_get_turb_visc(oracle_t *o)
{
    /* les_get_turb_visc (m_les.f90:1096-1137) */
    const int m = o->les_model;
    if (m == 1 || m == 4 || m == 5) les_get_turb_visc_smag(o);
    if (m == 2 || m == 3) les_get_turb_visc_dlm(o);
    if (m == 6 || m == 7) {
        les_get_turb_visc_smag(o);
        for (size_t q = 0; q < o->fsz; q++) o->turb_visc[q] = o->c_mixed * o->turb_visc[q];
    }
    if (m == 10) {
        /* les_get_turb_visc_smag_save_sij (m_les.f90:1223-1307): the same
         * viscosity, the physical strain S11 S12 S13 S22 S23 S33 kept in tauij */
        les_get_turb_visc_smag(o);
        const size_t fsz = o->fsz;
        for (int pass = 0; pass < 2; pass++) {
            strain_first(o, pass);
            for (int q = 0; q < 3; q++) {
                xfft3d(o, -1, W(o, 4 + q));
                memcpy(o->tauij + (size_t)(3 * pass + q) * fsz, W(o, 4 + q), sizeof(double) * fsz);
            }
        }
    }
}

/* m_les_get_tauij_dstm_source_BT (m_les.f90:2009-2179), les_model 10: with
 * k = (B T_B) + (eps T_eps), L_ij = (u_i u_j)~ - u~_i u~_j and c = 2 k / L_kk
 * (0 where L_kk < 1e-10): tau_ij = c L_ij - 2 C_mixed nu_t S_ij, kept in tauij
 * in physical space, and the (B T_B) source Pi = -c L_ij S_ij + C_mixed
 * nu_t^3 / (c_s Delta)^4 (masked with the rest of the LES RHS afterwards). */
static void les_tauij_dstm_source_bt(oracle_t *o)
{
    const int ns = o->nscal, nl = o->nles;
    const int n2i = 3 + ns + nl + 1;
    const size_t fsz = o->fsz;
    double *w1 = W(o, 0), *a2 = W(o, n2i), *a3 = W(o, n2i + 1), *a4 = W(o, n2i + 2), *a5 = W(o, n2i + 3);
    double *L[3] = {w1, a2, a3}, *tv = o->turb_visc, *ta = o->tauij;
    for (int i = 0; i < 3; i++) {
        copy_field(o, a4, F(o, i));
        xfft3d(o, -1, a4);
        for (size_t q = 0; q < fsz; q++) a4[q] = a4[q] * a4[q];
        xfft3d(o, 1, a4);
        oracle_apply_filter(o, o->gfilt, a4);
        xfft3d(o, -1, a4);
        copy_field(o, a5, F(o, i));
        oracle_apply_filter(o, o->gfilt, a5);
        xfft3d(o, -1, a5);
        for (size_t q = 0; q < fsz; q++) L[i][q] = a4[q] - a5[q] * a5[q];
    }
    for (size_t q = 0; q < fsz; q++) a4[q] = w1[q] + a2[q] + a3[q];
    for (size_t q = 0; q < fsz; q++) a5[q] = F(o, 3 + ns)[q] + F(o, 4 + ns)[q];
    xfft3d(o, -1, a5);
    for (int k = 0; k < o->n; k++)
        for (int j = 0; j < o->n; j++)
            for (int i = 0; i < o->n; i++) {
                size_t q = IX(o, i, j, k);
                a4[q] = a4[q] < 1e-10 ? 0.0 : 2.0 * a5[q] / a4[q];
            }
    for (size_t q = 0; q < fsz; q++)
        a5[q] = -w1[q] * ta[q] - a2[q] * ta[3 * fsz + q] - a3[q] * ta[5 * fsz + q];
    const int diag[3] = {0, 3, 5};
    for (int d = 0; d < 3; d++)
        for (int k = 0; k < o->n; k++)
            for (int j = 0; j < o->n; j++)
                for (int i = 0; i < o->n; i++) {
                    size_t q = IX(o, i, j, k);
                    double *t = ta + (size_t)diag[d] * fsz;
                    t[q] = a4[q] * L[d][q] - o->c_mixed * 2.0 * tv[q] * t[q];
                }
    int nn = 0;
    for (int i = 0; i < 3; i++)
        for (int j = i; j < 3; j++, nn++) {
            if (i == j) continue;
            copy_field(o, w1, F(o, i)); copy_field(o, a2, F(o, j));
            xfft3d(o, -1, w1); xfft3d(o, -1, a2);
            for (size_t q = 0; q < fsz; q++) w1[q] = w1[q] * a2[q];
            xfft3d(o, 1, w1);
            oracle_apply_filter(o, o->gfilt, w1);
            xfft3d(o, -1, w1);
            copy_field(o, a2, F(o, i)); copy_field(o, a3, F(o, j));
            oracle_apply_filter(o, o->gfilt, a2); oracle_apply_filter(o, o->gfilt, a3);
            xfft3d(o, -1, a2); xfft3d(o, -1, a3);
            double *t = ta + (size_t)nn * fsz;
            for (size_t q = 0; q < fsz; q++) {
                w1[q] = w1[q] - a2[q] * a3[q];
                a5[q] = a5[q] - 2.0 * w1[q] * t[q];
            }
            for (int k = 0; k < o->n; k++)
                for (int jj = 0; jj < o->n; jj++)
                    for (int ii = 0; ii < o->n; ii++) {
                        size_t q = IX(o, ii, jj, k);
                        t[q] = a4[q] * w1[q] - o->c_mixed * 2.0 * tv[q] * t[q];
                    }
        }
    const double cd = o->c_smag * o->les_delta, cd4 = cd * cd * cd * cd;
    for (size_t q = 0; q < fsz; q++) a5[q] = a5[q] * a4[q];
    for (int k = 0; k < o->n; k++)
        for (int j = 0; j < o->n; j++)
            for (int i = 0; i < o->n; i++) {
                size_t q = IX(o, i, j, k);
                a5[q] = a5[q] + o->c_mixed * (tv[q] * tv[q] * tv[q]) / cd4;
            }
    xfft3d(o, 1, a5);
    double *rb = W(o, 3 + ns + 1);
    for (size_t q = 0; q < fsz; q++) rb[q] = rb[q] + a5[q];
    o->les_stat[1] = a5[0] / ((double)o->n * o->n * o->n);
}

/* m_les_rhss_sgs_flux_harlow (m_les.f90:2191-2270): for each passive scalar
 * the RHS gains d/dx_i (T tau_ij dphi/dx_j), tau_ij the physical stress left in
 * tauij, T = (c_s Delta)^2 / nu_t (0 where nu_t / (c_s Delta)^2 < 1e-10). */
static void les_rhss_sgs_flux_harlow(oracle_t *o)
{
    const int ns = o->nscal, nl = o->nles, n = o->n;
    const size_t fsz = o->fsz;
    double *w1 = W(o, 0), *a2 = W(o, 3 + ns + nl + 1), *a3 = W(o, 3 + ns + nl + 2), *a4 = W(o, 3 + ns + nl + 3),
           *a5 = W(o, 3 + ns + nl + 4), *tv = o->turb_visc, *ta = o->tauij;
    const double cd = o->c_smag * o->les_delta;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                size_t q = IX(o, i, j, k);
                double v = tv[q] / (cd * cd);
                a5[q] = fabs(v) < 1e-10 ? 0.0 : 1.0 / v;
            }
    const int row[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    const char dirs[3] = {'x', 'y', 'z'};
    for (int s = 1; s <= ns; s++) {
        copy_field(o, w1, F(o, 2 + s));
        derivative(o, w1, 'z', a3);
        derivative(o, w1, 'y', a2);
        derivative(o, w1, 'x', w1);
        xfft3d(o, -1, w1); xfft3d(o, -1, a2); xfft3d(o, -1, a3);
        double *r = W(o, 3 + s);
        for (int c = 0; c < 3; c++) {
            const double *t0 = ta + (size_t)row[c][0] * fsz, *t1 = ta + (size_t)row[c][1] * fsz,
                         *t2 = ta + (size_t)row[c][2] * fsz;
            for (size_t q = 0; q < fsz; q++) a4[q] = t0[q] * w1[q] + t1[q] * a2[q] + t2[q] * a3[q];
            for (size_t q = 0; q < fsz; q++) a4[q] = a4[q] * a5[q];
            xfft3d(o, 1, a4);
            derivative(o, a4, dirs[c], a4);
            for (size_t q = 0; q < fsz; q++) r[q] = r[q] + a4[q];
        }
    }
}

/* m_les_lag_model_sources_no_k (m_les.f90:2282-2338): B = (B T_B) |S| with
 * |S| = nu_t / (c_s Delta)^2, eps = max(eps T_eps, 0)^1.5 / (Delta C_T^1.5),
 * C_T = 1; (B T_B) loses B, (eps T_eps) gains B - eps. */
static void les_lag_model_sources_no_k(oracle_t *o)
{
    const int ns = o->nscal, nl = o->nles, n = o->n;
    const size_t fsz = o->fsz;
    double *w1 = W(o, 0), *a2 = W(o, 3 + ns + nl + 1), *a5 = W(o, 3 + ns + nl + 4), *tv = o->turb_visc;
    const double cd = o->c_smag * o->les_delta, C_T = 1.0;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                size_t q = IX(o, i, j, k);
                a5[q] = tv[q] / (cd * cd);
            }
    copy_field(o, w1, F(o, 3 + ns));
    xfft3d(o, -1, w1);
    for (size_t q = 0; q < fsz; q++) w1[q] = w1[q] * a5[q];
    xfft3d(o, 1, w1);
    copy_field(o, a2, F(o, 4 + ns));
    xfft3d(o, -1, a2);
    for (size_t q = 0; q < fsz; q++) {
        double v = a2[q] > 0.0 ? a2[q] : 0.0;
        a2[q] = pow(v, 1.5) / (o->les_delta * pow(C_T, 1.5));
    }
    xfft3d(o, 1, a2);
    double *rb = W(o, 3 + ns + 1), *re = W(o, 3 + ns + 2);
    for (size_t q = 0; q < fsz; q++) {
        rb[q] = rb[q] - w1[q];
        re[q] = re[q] + w1[q] - a2[q];
    }
    o->les_stat[2] = w1[0] / ((double)n * n * n);
    o->les_stat[3] = a2[0] / ((double)n * n * n);
}

static void oracle_rhs_scalars(oracle_t *o)
{
    int n = o->n, ns = o->nscal, nl = o->nles;
    if (o->les_model) les_get_turb_visc(o);
    if (!o->int_scalars && nl == 0) {
        for (int m = 0; m < 3; m++) { copy_field(o, W(o, 1 + m), F(o, m)); xfft3d(o, -1, W(o, 1 + m)); }
        return;
    }
    for (int m = 4; m <= 3 + ns + nl; m++) memset(W(o, m), 0, sizeof(double) * o->fsz);
    if (o->dealias == 0) {
        for (int m = 0; m < 3; m++) { copy_field(o, W(o, 1 + m), F(o, m)); xfft3d(o, -1, W(o, 1 + m)); }
        /* passive scalars only once they are switched on; LES quantities always
         * (rhs_scalars.f90:72-74) */
        for (int s = o->int_scalars ? 1 : ns + 1; s <= ns + nl; s++) {
            copy_field(o, W(o, 0), F(o, 2 + s));
            xfft3d(o, -1, W(o, 0));
            for (int c = 1; c <= 3; c++) {
                mul3(o, W(o, s + 2 + c), W(o, 0), W(o, c));
                xfft3d(o, 1, W(o, s + 2 + c));
            }
            double *r = W(o, 3 + s), *p2 = W(o, 4 + s), *p3 = W(o, 5 + s), *phi = F(o, 2 + s);
            double pe = o->pe[s - 1];
#pragma omp parallel for schedule(static)
            for (int k = 0; k < n; k++)
                for (int j = 0; j < n; j++)
                    for (int i = 0; i < n + 1; i += 2) {
                        size_t a = IX(o, i, j, k), b = a + 1;
                        if (o->ialias[a] > 0) { r[a] = 0.0; r[b] = 0.0; continue; }
                        double rt1 = o->akx[i + 1] * r[b] + o->aky[k] * p2[b] + o->akz[j] * p3[b];
                        double rt2 = o->akx[i] * r[a] + o->aky[k] * p2[a] + o->akz[j] * p3[a];
                        double wn2 = o->akx[i] * o->akx[i] + o->aky[k] * o->aky[k] + o->akz[j] * o->akz[j];
                        r[a] = rt1 - pe * wn2 * phi[a];
                        r[b] = -rt2 - pe * wn2 * phi[b];
                    }
        }
    } else {
        phase_factors(o);
        double *w0 = W(o, 0);
        for (int m = 1; m <= 3 + ns; m++) {
            double *d = W(o, m), *f = F(o, m - 1);
#pragma omp parallel for schedule(static)
            for (int k = 0; k < n; k++)
                for (int j = 0; j < n; j++)
                    for (int i = 0; i < n + 1; i += 2) {
                        size_t a = IX(o, i, j, k), b = a + 1;
                        d[a] = f[a] * w0[a] - f[b] * w0[b];
                        d[b] = f[b] * w0[a] + f[a] * w0[b];
                    }
            xfft3d(o, -1, d);
        }
        int n1 = ns + 4, n2 = ns + 5;
        for (int m = 4; m <= 3 + ns; m++) {
            mul3(o, W(o, n1), W(o, m), W(o, 1));
            mul3(o, W(o, n2), W(o, m), W(o, 2));
            mul3(o, W(o, m), W(o, m), W(o, 3));
            xfft3d(o, 1, W(o, n1));
            xfft3d(o, 1, W(o, n2));
            xfft3d(o, 1, W(o, m));
            double *A = W(o, n1), *B = W(o, n2), *C = W(o, m);
#pragma omp parallel for schedule(static)
            for (int k = 0; k < n; k++)
                for (int j = 0; j < n; j++)
                    for (int i = 0; i < n + 1; i += 2) {
                        size_t a = IX(o, i, j, k), b = a + 1;
                        if (o->ialias[a] > 1) { C[a] = 0.0; C[b] = 0.0; continue; }
                        double r11 = A[a] * w0[a] + A[b] * w0[b];
                        double r12 = A[b] * w0[a] - A[a] * w0[b];
                        double r21 = B[a] * w0[a] + B[b] * w0[b];
                        double r22 = B[b] * w0[a] - B[a] * w0[b];
                        double r31 = C[a] * w0[a] + C[b] * w0[b];
                        double r32 = C[b] * w0[a] - C[a] * w0[b];
                        C[a] = +0.5 * (o->akx[i + 1] * r12 + o->aky[k] * r22 + o->akz[j] * r32);
                        C[b] = -0.5 * (o->akx[i] * r11 + o->aky[k] * r21 + o->akz[j] * r31);
                    }
        }
        for (int m = 0; m < 3; m++) { copy_field(o, W(o, 1 + m), F(o, m)); xfft3d(o, -1, W(o, 1 + m)); }
        for (int m = 4; m <= 3 + ns; m++) {
            copy_field(o, W(o, 0), F(o, m - 1));
            xfft3d(o, -1, W(o, 0));
            mul3(o, W(o, n1), W(o, 0), W(o, 1));
            mul3(o, W(o, n2), W(o, 0), W(o, 2));
            mul3(o, W(o, 0), W(o, 0), W(o, 3));
            xfft3d(o, 1, W(o, n1));
            xfft3d(o, 1, W(o, n2));
            xfft3d(o, 1, W(o, 0));
            double *A = W(o, n1), *B = W(o, n2), *C = W(o, 0), *r = W(o, m), *phi = F(o, m - 1);
            double pe = o->pe[m - 4];
#pragma omp parallel for schedule(static)
            for (int k = 0; k < n; k++)
                for (int j = 0; j < n; j++)
                    for (int i = 0; i < n + 1; i += 2) {
                        size_t a = IX(o, i, j, k), b = a + 1;
                        if (o->ialias[a] < 2) {
                            double rt1 = o->akx[i + 1] * A[b] + o->aky[k] * B[b] + o->akz[j] * C[b];
                            double rt2 = o->akx[i] * A[a] + o->aky[k] * B[a] + o->akz[j] * C[a];
                            double wn2 = o->akx[i] * o->akx[i] + o->aky[k] * o->aky[k] + o->akz[j] * o->akz[j];
                            r[a] = r[a] + 0.5 * rt1 - pe * wn2 * phi[a];
                            r[b] = r[b] - 0.5 * rt2 - pe * wn2 * phi[b];
                        }
                    }
        }
        /* reaction rates (rhs_scalars.f90:281-303), phase shift only: type 311 gains
         * reac (1 - phi~^2)(phi~ - <phi>), phi~ the scalar without the modes of
         * some |k_i| > N/4, <phi> its mean; other types above 300 stop the run */
        for (int s = 1; s <= o->nscal; s++) {
            if (o->scalar_type[s - 1] <= 300) continue;
            double *w1 = W(o, 3 + ns + nl + 4), *w2 = W(o, 3 + ns + nl + 5);
            copy_field(o, w1, F(o, 2 + s));
            for (int k = 0; k < n; k++)
                for (int j = 0; j < n; j++)
                    for (int i = 0; i < n + 1; i += 2) {
                        size_t a = IX(o, i, j, k);
                        if (fabs(o->akx[i]) > n / 4 || fabs(o->aky[k]) > n / 4 || fabs(o->akz[j]) > n / 4)
                            w1[a] = w1[a + 1] = 0.0;
                    }
            xfft3d(o, -1, w1);
            const double mean = F(o, 2 + s)[0] / ((double)n * n * n);
            for (size_t q = 0; q < o->fsz; q++) w2[q] = o->reac[s - 1] * (1.0 - w1[q] * w1[q]) * (w1[q] - mean);
            xfft3d(o, 1, w2);
            double *r = W(o, 3 + s);
            for (size_t q = 0; q < o->fsz; q++) r[q] = r[q] + w2[q];
        }
    }
    /* uniform mean-gradient source for type-0 scalars (rhs_scalars.f90:387-389) */
    for (int s = 1; s <= ns; s++)
        if (o->scalar_type[s - 1] == 0) {
            double *r = W(o, s + 3), *u = F(o, 0);
            for (size_t q = 0; q < o->fsz; q++) r[q] = r[q] - u[q];
        }
    /* les_rhs_scalars, DLM branch (m_les.f90:714-719) */
    /* les_rhs_scalars (m_les.f90:700-858); les.gp sums restart every step */
    if (o->les_model) {
        /* energy: k_sgs, or (B T_B) + (eps T_eps) for les_model 10 (m_les.f90:880-884) */
        if (nl > 0)
            o->les_stat[0] = (F(o, 3 + ns)[0] + (o->les_model == 10 ? F(o, 4 + ns)[0] : 0.0)) /
                             ((double)o->n * o->n * o->n);
        o->les_stat[1] = o->les_stat[2] = o->les_stat[3] = 0.0;
        switch (o->les_model) {
        case 2: les_k_src_dlm(o); les_k_diss_algebraic(o); break;
        case 3: les_k_src_dlm(o); les_lag_model_sources(o); break;
        case 4: les_dstm_vel_k_sources(o); les_k_diss_algebraic(o); break;
        case 5: les_dstm_vel_k_sources(o); les_k_src_dlm(o); les_lag_model_sources(o); break;
        case 6: les_dstm_vel_k_sources(o); les_k_src_dlm(o); break;
        case 7: les_dstm_vel_k_sources(o); les_k_src_dlm(o); les_lag_model_sources(o); break;
        case 10:
            les_rhss_turb_visc1(o, 4 + ns);
            les_rhss_turb_visc1(o, 5 + ns);
            les_tauij_dstm_source_bt(o);
            if (ns > 0) les_rhss_sgs_flux_harlow(o);
            les_lag_model_sources_no_k(o);
            break;
        }
        if (o->les_model != 10)
            for (int m = 4; m <= 3 + ns + nl; m++) les_rhss_turb_visc1(o, m);
        if (o->les_model == 6) les_k_diss_algebraic(o);
        /* no aliasing in the scalar RHSs (m_les.f90:860-870) */
        for (int m = 4; m <= 3 + ns + nl; m++) {
            double *r = W(o, m);
            for (size_t q = 0; q < o->fsz; q++)
                if (o->ialias[q] != 0) r[q] = 0.0;
        }
    }
}

/* ------------------------------------------------------------------------- */
/*  rhs_velocity (rhs_velocity.f90:1-419)                                    */
/* ------------------------------------------------------------------------- */
static void shift_back(oracle_t *o, double *a)
{
    int n = o->n;
    double *w0 = W(o, 0);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 1; i += 2) {
                size_t p = IX(o, i, j, k), q = p + 1;
                double rt = a[p] * w0[p] + a[q] * w0[q];
                a[q] = a[q] * w0[p] - a[p] * w0[q];
                a[p] = rt;
            }
}

static void shift_fwd(oracle_t *o, double *d, const double *f)
{
    int n = o->n;
    double *w0 = W(o, 0);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 1; i += 2) {
                size_t a = IX(o, i, j, k), b = a + 1;
                d[a] = f[a] * w0[a] - f[b] * w0[b];
                d[b] = f[b] * w0[a] + f[a] * w0[b];
            }
}

static void oracle_rhs_velocity(oracle_t *o)
{
    int n = o->n;
    double *w1 = W(o, 1), *w2 = W(o, 2), *w3 = W(o, 3), *w4 = W(o, 4), *w5 = W(o, 5), *w6 = W(o, 6);
    /* Courant number (rhs_velocity.f90:31-38) */
    double cmax = 0.0;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                size_t a = IX(o, i, j, k);
                double c = fabs(w1[a]) + fabs(w2[a]) + fabs(w3[a]);
                if (c > cmax) cmax = c;
            }
    o->courant = cmax * o->dt / o->dx;

    /* six products (both branches compute them identically) */
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                size_t a = IX(o, i, j, k);
                double u = w1[a], v = w2[a], w = w3[a];
                double t1 = u * u, t2 = u * v, t3 = u * w, t4 = v * v, t5 = v * w, t6 = w * w;
                w1[a] = t1; w2[a] = t2; w3[a] = t3; w4[a] = t4; w5[a] = t5; w6[a] = t6;
            }
    for (int m = 1; m <= 6; m++) xfft3d(o, 1, W(o, m));
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 2; i++) {
                size_t a = IX(o, i, j, k);
                double kx = o->akx[i], ky = o->aky[k], kz = o->akz[j];
                double t1 = -(kx * w1[a] + ky * w2[a] + kz * w3[a]);
                double t2 = -(kx * w2[a] + ky * w4[a] + kz * w5[a]);
                double t3 = -(kx * w3[a] + ky * w5[a] + kz * w6[a]);
                double t4 = -o->nu * (kx * kx + ky * ky + kz * kz);
                w1[a] = t1; w2[a] = t2; w3[a] = t3; w4[a] = t4;
            }
    double *fu[3] = {F(o, 0), F(o, 1), F(o, 2)};
    double *wr[3] = {w1, w2, w3};
    if (o->dealias == 0) {
#pragma omp parallel for schedule(static)
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n + 1; i += 2) {
                    size_t a = IX(o, i, j, k), b = a + 1;
                    if (o->ialias[a] > 0) {
                        for (int c = 0; c < 3; c++) { wr[c][a] = 0.0; wr[c][b] = 0.0; }
                    } else {
                        for (int c = 0; c < 3; c++) {
                            double rt = -wr[c][b] + w4[a] * fu[c][a];
                            wr[c][b] = wr[c][a] + w4[b] * fu[c][b];
                            wr[c][a] = rt;
                        }
                    }
                }
    } else {
        memset(W(o, 0), 0, sizeof(double) * o->fsz);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n + 1; i += 2) {
                    size_t a = IX(o, i, j, k), b = a + 1;
                    if (o->ialias[a] > 1) {
                        for (int c = 0; c < 3; c++) { wr[c][a] = 0.0; wr[c][b] = 0.0; }
                    } else {
                        for (int c = 0; c < 3; c++) {
                            double rt = -0.5 * wr[c][b] + w4[a] * fu[c][a];
                            wr[c][b] = 0.5 * wr[c][a] + w4[b] * fu[c][b];
                            wr[c][a] = rt;
                        }
                    }
                }
        phase_factors(o);
        shift_fwd(o, w4, fu[0]);
        shift_fwd(o, w5, fu[1]);
        xfft3d(o, -1, w4);
        xfft3d(o, -1, w5);
        /* (u+)(u+) */
        mul3(o, w6, w4, w4);
        xfft3d(o, 1, w6);
        shift_back(o, w6);
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n + 1; i += 2) {
                    size_t a = IX(o, i, j, k), b = a + 1;
                    w1[a] = w1[a] + 0.5 * o->akx[i + 1] * w6[b];
                    w1[b] = w1[b] - 0.5 * o->akx[i] * w6[a];
                }
        /* (u+)(v+) */
        mul3(o, w6, w4, w5);
        xfft3d(o, 1, w6);
        shift_back(o, w6);
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n + 1; i += 2) {
                    size_t a = IX(o, i, j, k), b = a + 1;
                    w1[a] = w1[a] + 0.5 * o->aky[k] * w6[b];
                    w1[b] = w1[b] - 0.5 * o->aky[k] * w6[a];
                    w2[a] = w2[a] + 0.5 * o->akx[i + 1] * w6[b];
                    w2[b] = w2[b] - 0.5 * o->akx[i] * w6[a];
                }
        /* (v+)(v+) */
        mul3(o, w6, w5, w5);
        xfft3d(o, 1, w6);
        shift_back(o, w6);
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n + 1; i += 2) {
                    size_t a = IX(o, i, j, k), b = a + 1;
                    w2[a] = w2[a] + 0.5 * o->aky[k] * w6[b];
                    w2[b] = w2[b] - 0.5 * o->aky[k] * w6[a];
                }
        /* w+ */
        shift_fwd(o, w6, fu[2]);
        xfft3d(o, -1, w6);
        mul3(o, w4, w4, w6);
        mul3(o, w5, w5, w6);
        mul3(o, w6, w6, w6);
        xfft3d(o, 1, w4);
        xfft3d(o, 1, w5);
        xfft3d(o, 1, w6);
        shift_back(o, w4);
        shift_back(o, w5);
        shift_back(o, w6);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n + 1; i += 2) {
                    size_t a = IX(o, i, j, k), b = a + 1;
                    double kx0 = o->akx[i], kx1 = o->akx[i + 1], ky = o->aky[k], kz = o->akz[j];
                    if (o->ialias[a] < 2) {
                        w1[a] = w1[a] + 0.5 * kz * w4[b];
                        w1[b] = w1[b] - 0.5 * kz * w4[a];
                        w2[a] = w2[a] + 0.5 * kz * w5[b];
                        w2[b] = w2[b] - 0.5 * kz * w5[a];
                        w3[a] = w3[a] + 0.5 * (kx1 * w4[b] + ky * w5[b] + kz * w6[b]);
                        w3[b] = w3[b] - 0.5 * (kx0 * w4[a] + ky * w5[a] + kz * w6[a]);
                    } else {
                        w1[a] = 0.0; w1[b] = 0.0; w2[a] = 0.0; w2[b] = 0.0; w3[a] = 0.0; w3[b] = 0.0;
                    }
                }
    }
    if (o->les_model) les_rhs_velocity(o);
}

/* ------------------------------------------------------------------------- */
/*  force_velocity (m_force.f90:101-182)                                     */
/* ------------------------------------------------------------------------- */
static double forcing_energy(oracle_t *o)
{
    int n = o->n;
    double fac = 1.0 / (((double)n * n * n) * ((double)n * n * n));
    /* one sum per shell 1..kfmax (any kfmax the input gives, m_parameters.f90:308) */
    double *es = (double *)calloc((size_t)(o->kfmax > 0 ? o->kfmax : 1), sizeof(double));
    double *u = F(o, 0), *v = F(o, 1), *w = F(o, 2);
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                double k2 = o->akx[i] * o->akx[i] + o->aky[k] * o->aky[k] + o->akz[j] * o->akz[j];
                int sh = nint_shell32(k2);
                if (sh > 0 && sh <= o->kfmax) {
                    size_t a = IX(o, i, j, k);
                    double f2 = fac * (u[a] * u[a] + v[a] * v[a] + w[a] * w[a]);
                    if (o->akx[i] == 0.0) f2 = f2 * 0.5;
                    es[sh - 1] = es[sh - 1] + f2;
                }
            }
    double e = 0.0;
    for (int s = 0; s < o->kfmax; s++) e = e + es[s];
    free(es);
    return e;
}

double oracle_forcing_energy(oracle_t *o) { return forcing_energy(o); }

static void force_velocity(oracle_t *o)
{
    double energy = forcing_energy(o);
    double fac = o->famp / energy;
    for (int m = 0; m < o->nfn; m++) {
        size_t a = IX(o, o->fn_i[m], o->fn_j[m], o->fn_k[m]);
        for (int c = 0; c < 3; c++) W(o, 1 + c)[a] = W(o, 1 + c)[a] + fac * F(o, c)[a];
    }
}

/* ------------------------------------------------------------------------- */
/*  pressure (pressure.f90:1-51)                                             */
/* ------------------------------------------------------------------------- */
static void pressure(oracle_t *o)
{
    int n = o->n;
    double *u = F(o, 0), *v = F(o, 1), *w = F(o, 2);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 1; i += 2) {
                size_t a = IX(o, i, j, k), b = a + 1;
                double kx0 = o->akx[i], kx1 = o->akx[i + 1], ky = o->aky[k], kz = o->akz[j];
                double div2 = kx0 * u[a] + ky * v[a] + kz * w[a];
                double div1 = -(kx1 * u[b] + ky * v[b] + kz * w[b]);
                double l1 = kx0 * kx0 + ky * ky + kz * kz;
                double l2 = kx1 * kx1 + ky * ky + kz * kz;
                if (l1 == 0.0) l1 = 9e20;
                if (l2 == 0.0) l2 = 9e20;
                double p1 = -div1 / l1, p2 = -div2 / l2;
                u[a] = u[a] + p2 * kx1; u[b] = u[b] - p1 * kx0;
                v[a] = v[a] + p2 * ky;  v[b] = v[b] - p1 * ky;
                w[a] = w[a] + p2 * kz;  w[b] = w[b] - p1 * kz;
            }
}

void oracle_pressure(oracle_t *o) { pressure(o); }

/* ------------------------------------------------------------------------- */
/*  one timestep of the hydro task (main.f90:124-170)                        */
/* ------------------------------------------------------------------------- */
void oracle_step(oracle_t *o, int nsteps)
{
    for (int it = 0; it < nsteps; it++) {
        oracle_rhs_scalars(o);
        if (o->int_scalars || o->nles > 0) {
            int nlo = 3, nhi = 3 + o->nscal + o->nles;
            double dt = o->dt;
            for (int m = nlo; m < nhi; m++) {
                double *f = F(o, m), *r = RO(o, m), *w = W(o, m + 1);
                if (o->fos) {
                    for (size_t q = 0; q < o->fsz; q++) { r[q] = w[q]; f[q] = f[q] + dt * r[q]; }
                } else {
                    for (size_t q = 0; q < o->fsz; q++) {
                        f[q] = f[q] + dt * (1.5 * w[q] - 0.5 * r[q]);
                        r[q] = w[q];
                    }
                }
            }
            o->fos = 0;
        }
        oracle_rhs_velocity(o);
        if (o->flow_type == 1) force_velocity(o);
        double dt = o->dt;
        for (int m = 0; m < 3; m++) {
            double *f = F(o, m), *r = RO(o, m), *w = W(o, m + 1);
            if (o->fov) {
#pragma omp parallel for schedule(static)
                for (size_t q = 0; q < o->fsz; q++) { r[q] = w[q]; f[q] = f[q] + dt * r[q]; }
            } else {
#pragma omp parallel for schedule(static)
                for (size_t q = 0; q < o->fsz; q++) {
                    f[q] = f[q] + dt * (1.5 * w[q] - 0.5 * r[q]);
                    r[q] = w[q];
                }
            }
        }
        o->fov = 0;
        pressure(o);
        o->time += o->dt;
    }
}

/* RHS only (no update): rhs_scalars + rhs_velocity + forcing; results in wrk1..3+ns */
void oracle_rhs(oracle_t *o)
{
    oracle_rhs_scalars(o);
    /* rhs_velocity reuses wrk4..; save scalar RHS first */
    int ns = (o->int_scalars ? o->nscal : 0) + o->nles;
    double *save = NULL;
    if (ns) {
        save = (double *)malloc(sizeof(double) * o->fsz * ns);
        memcpy(save, W(o, 4), sizeof(double) * o->fsz * ns);
    }
    oracle_rhs_velocity(o);
    if (o->flow_type == 1) force_velocity(o);
    if (ns) { memcpy(W(o, 4), save, sizeof(double) * o->fsz * ns); free(save); }
}

/* ------------------------------------------------------------------------- */
/*  statistics (m_stats.f90:99-440) + velocity-derivative skewness (new)     */
/*  out[0..kmax) = e_spec; out[kmax..] = energy, eps_v, eta, etakmax, uvar,  */
/*  x_length, lambda, re_lambda, re_lambda1, tau_e, enstrophy, skewness      */
/* ------------------------------------------------------------------------- */
static void derivative(oracle_t *o, const double *src, char axis, double *dst)
{
    /* x_derivative (x_fftw.f90:637-682); src and dst may be the same array */
    int n = o->n;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 2; i++) {
                size_t a = IX(o, i, j, k);
                double kk = axis == 'x' ? o->akx[i] : axis == 'y' ? o->aky[k] : o->akz[j];
                dst[a] = kk * src[a];
            }
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 1; i += 2) {
                size_t a = IX(o, i, j, k);
                double rt = -dst[a + 1];
                dst[a + 1] = dst[a];
                dst[a] = rt;
            }
}

void oracle_energy_spectrum(oracle_t *o, int field0, int ncomp, double *es)
{
    int n = o->n;
    double fac = 1.0 / (((double)n * n * n) * ((double)n * n * n));
    for (int s = 0; s < o->kmax; s++) es[s] = 0.0;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                double k2 = o->akx[i] * o->akx[i] + o->aky[k] * o->aky[k] + o->akz[j] * o->akz[j];
                int sh = nint_shell32(k2);
                if (sh > 0 && sh <= o->kmax) {
                    size_t a = IX(o, i, j, k);
                    double sq = 0.0;
                    for (int c = 0; c < ncomp; c++) {
                        double x = F(o, field0 + c)[a];
                        sq = (c == 0) ? x * x : sq + x * x;
                    }
                    double f2 = fac * sq;
                    if (o->akx[i] == 0.0) f2 = 0.5 * f2;
                    es[sh - 1] = es[sh - 1] + f2;
                }
            }
}

void oracle_stats(oracle_t *o, double *out)
{
    int n = o->n, kmax = o->kmax;
    double PI = 4.0 * atan(1.0);
    double *es = out;
    double fac = 1.0 / ((double)n * n * n);
    /* enstrophy (m_stats.f90:241-289) */
    for (int m = 0; m < 3; m++) copy_field(o, W(o, 1 + m), F(o, m));
    derivative(o, W(o, 3), 'y', W(o, 6));
    derivative(o, W(o, 3), 'x', W(o, 5));
    derivative(o, W(o, 2), 'z', W(o, 4));
    derivative(o, W(o, 2), 'x', W(o, 3));
    derivative(o, W(o, 1), 'z', W(o, 2));
    derivative(o, W(o, 1), 'y', W(o, 1));
    for (size_t q = 0; q < o->fsz; q++) {
        W(o, 3)[q] = W(o, 3)[q] - W(o, 1)[q];
        W(o, 2)[q] = W(o, 2)[q] - W(o, 5)[q];
        W(o, 1)[q] = W(o, 6)[q] - W(o, 4)[q];
    }
    for (int m = 1; m <= 3; m++) xfft3d(o, -1, W(o, m));
    double ens = 0.0;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                size_t a = IX(o, i, j, k);
                double x = W(o, 1)[a] * W(o, 1)[a] + W(o, 2)[a] * W(o, 2)[a] + W(o, 3)[a] * W(o, 3)[a];
                ens += x;
            }
    ens = ens * fac;
    /* skewness of the longitudinal derivatives (new statistic) */
    double skew = 0.0;
    for (int c = 0; c < 3; c++) {
        derivative(o, F(o, c), c == 0 ? 'x' : c == 1 ? 'y' : 'z', W(o, 1));
        xfft3d(o, -1, W(o, 1));
        double m2 = 0.0, m3 = 0.0;
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) {
                    double d = W(o, 1)[IX(o, i, j, k)];
                    m2 += d * d;
                    m3 += d * d * d;
                }
        m2 *= fac; m3 *= fac;
        skew += m3 / pow(m2, 1.5);
    }
    skew /= 3.0;
    /* spectrum and derived quantities (m_stats.f90:99-189) */
    oracle_energy_spectrum(o, 0, 3, es);
    double energy = 0.0;
    for (int k = 0; k < kmax; k++) energy = energy + es[k];
    double eps = 0.0;
    for (int k = 1; k <= kmax; k++) eps = eps + es[k - 1] * (double)(k * k) * 2.0 * o->nu;
    double eta = pow(o->nu * o->nu * o->nu / eps, 0.25);
    double etakmax = eta * (double)kmax;
    double uvar = 2.0 / 3.0 * energy;
    double sct = 0.0;
    for (int k = 1; k <= kmax; k++) sct = sct + es[k - 1] / (double)k;
    double xl = PI / 2.0 * sct / uvar;
    double lam = sqrt(15.0 * uvar * o->nu / eps);
    double rel = uvar * sqrt(15.0 / eps * (1.0 / o->nu));
    double rel1 = sqrt(uvar) * lam / o->nu;
    double taue = xl / sqrt(uvar);
    double *d = out + kmax;
    d[0] = energy; d[1] = eps; d[2] = eta; d[3] = etakmax; d[4] = uvar; d[5] = xl;
    d[6] = lam; d[7] = rel; d[8] = rel1; d[9] = taue; d[10] = ens; d[11] = skew;
}

/* scalar statistics (m_stats.f90:295-440): per scalar out[s*(kmax+5)+..] =
 * spectrum (x2), dissipation, mean, variance, min, max */
void oracle_scalar_stats(oracle_t *o, double *out)
{
    int n = o->n, kmax = o->kmax;
    double fac = 1.0 / ((double)n * n * n);
    for (int s = 0; s < o->nscal; s++) {
        double *d = out + (size_t)s * (kmax + 5);
        oracle_energy_spectrum(o, 3 + s, 1, d);
        for (int k = 0; k < kmax; k++) d[k] = 2.0 * d[k];
        copy_field(o, W(o, 0), F(o, 3 + s));
        derivative(o, W(o, 0), 'x', W(o, 1));
        derivative(o, W(o, 0), 'y', W(o, 2));
        derivative(o, W(o, 0), 'z', W(o, 3));
        for (int m = 1; m <= 3; m++) xfft3d(o, -1, W(o, m));
        double q = 0.0;
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) {
                    size_t a = IX(o, i, j, k);
                    q += W(o, 1)[a] * W(o, 1)[a] + W(o, 2)[a] * W(o, 2)[a] + W(o, 3)[a] * W(o, 3)[a];
                }
        d[kmax] = 2.0 * o->pe[s] * q * fac;
        xfft3d(o, -1, W(o, 0));
        double m1 = 0.0, m2 = 0.0, mn = 1e300, mx = -1e300;
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) {
                    double x = W(o, 0)[IX(o, i, j, k)];
                    m1 += x; m2 += x * x;
                    if (x < mn) mn = x;
                    if (x > mx) mx = x;
                }
        m1 *= fac; m2 *= fac;
        d[kmax + 1] = m1; d[kmax + 2] = m2 - m1 * m1; d[kmax + 3] = mn; d[kmax + 4] = mx;
    }
}

/* ------------------------------------------------------------------------- */
/*  initial velocity (init_velocity.f90:1-246); isp 0, 1, 3 as the reference */
/*  and isp 2 = k^ir_exp * exp(-2 (k/k_p)^2), a spectrum the reference lacks */
/* ------------------------------------------------------------------------- */
int oracle_init_velocity(oracle_t *o, double rn1, int isp_type, double peak_wavenum, double ir_exp)
{
    int n = o->n, kmax = o->kmax;
    double PI = 4.0 * atan(1.0), TWO_PI = 2.0 * PI;
    if (isp_type == -1) {
        /* Taylor-Green (init_velocity.f90:252-293) */
        double dx = 2.0 * PI / (double)n;
        for (int k = 0; k < n; k++) {
            double zz = (double)k * dx;
            for (int j = 0; j < n; j++) {
                double yy = (double)j * dx;
                for (int i = 0; i < n; i++) {
                    double xx = (double)i * dx;
                    size_t a = IX(o, i, j, k);
                    W(o, 1)[a] = sin(xx) * cos(yy) * cos(zz);
                    W(o, 2)[a] = -cos(xx) * sin(yy) * cos(zz);
                    W(o, 3)[a] = 0.0;
                }
            }
        }
        for (int m = 1; m <= 3; m++) { xfft3d(o, 1, W(o, m)); copy_field(o, F(o, m - 1), W(o, m)); }
        return 0;
    }
    /* random numbers over the full padded arrays, wrk1..6 in order */
    randu_state *st = &o->rs;
    (void)oracle_randu(st, -rn1);
    for (int m = 1; m <= 6; m++) {
        double *w = W(o, m);
        for (size_t q = 0; q < o->fsz; q++) w[q] = oracle_randu(st, rn1);
    }
    for (int m = 1; m <= 3; m++) {
        double *a = W(o, m), *b = W(o, m + 3);
        for (size_t q = 0; q < o->fsz; q++) a[q] = sqrt(-2.0 * log(a[q])) * sin(TWO_PI * b[q]);
    }
    for (int m = 1; m <= 3; m++) xfft3d(o, 1, W(o, m));
    double *w1 = W(o, 1), *w2 = W(o, 2), *w3 = W(o, 3), *w4 = W(o, 4), *w5 = W(o, 5), *w6 = W(o, 6);
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 1; i += 2) {
                size_t a = IX(o, i, j, k), b = a + 1;
                double kx0 = o->akx[i], kx1 = o->akx[i + 1], ky = o->aky[k], kz = o->akz[j];
                int sh = nint_shell64(kx0 * kx0 + ky * ky + kz * kz);
                if (sh > 0 && sh <= kmax) {
                    w4[a] = -(ky * w3[b] - kz * w2[b]);
                    w4[b] = ky * w3[a] - kz * w2[a];
                    w5[a] = -(kz * w1[b] - kx1 * w3[b]);
                    w5[b] = kz * w1[a] - kx0 * w3[a];
                    w6[a] = -(kx1 * w2[b] - ky * w1[b]);
                    w6[b] = kx0 * w2[a] - ky * w1[a];
                } else {
                    w4[a] = w4[b] = w5[a] = w5[b] = w6[a] = w6[b] = 0.0;
                }
            }
    for (int m = 0; m < 3; m++) copy_field(o, F(o, m), W(o, 4 + m));
    double *es = (double *)calloc(kmax + 1, sizeof(double));
    double *et = (double *)calloc(kmax + 1, sizeof(double));
    oracle_energy_spectrum(o, 0, 3, es);
    for (int k = 1; k <= kmax; k++) {
        double wmag = (double)k, ratio = wmag / peak_wavenum;
        if (isp_type == 0) et[k - 1] = pow(wmag, -5.0 / 3.0);
        else if (isp_type == 1) et[k - 1] = ratio * ratio * ratio / peak_wavenum * exp(-3.0 * ratio);
        else if (isp_type == 2) et[k - 1] = pow(wmag, ir_exp) * exp(-2.0 * ratio * ratio);
        else if (isp_type == 3) {
            double f = 2.0 * PI * ratio;
            double f2 = f * f, d = 1.0 + f2;
            et[k - 1] = (f2 * f2) / (d * d * d);
        } else { free(es); free(et); return -1; }
    }
    double tot = 0.0;
    for (int k = 0; k < kmax; k++) tot = tot + et[k];
    for (int k = 0; k < kmax; k++) et[k] = et[k] / tot;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 2; i++) {
                double k2 = o->akx[i] * o->akx[i] + o->aky[k] * o->aky[k] + o->akz[j] * o->akz[j];
                int sh = nint_shell32(k2);
                size_t a = IX(o, i, j, k);
                if (sh > 0 && sh <= kmax && es[sh - 1] > 0.0) {
                    double r = sqrt(et[sh - 1] / es[sh - 1]);
                    for (int c = 0; c < 3; c++) F(o, c)[a] = F(o, c)[a] * r;
                } else {
                    for (int c = 0; c < 3; c++) F(o, c)[a] = 0.0;
                }
            }
    free(es); free(et);
    return 0;
}

/* init_scalar (init_scalars.f90:41-345) for passive scalar s (0-based):
 * type 0 zero; 1, 2, 3 Box-Muller noise from the RANDu stream of RN2 over
 * wrk1, wrk2, shaped to the normalised spectrum (3: then sign * 0.9 with
 * shells 0 and >= 2 kmax / 3 removed); 11, 12, 13 physical profiles.  The
 * modes with ialias > 0 are zeroed afterwards, as init_scalars does. */
int oracle_init_scalar(oracle_t *o, int s, double rn2, double peak)
{
    int n = o->n, kmax = o->kmax, type = o->scalar_type[s], ic = type - (type / 100) * 100;
    double PI = 4.0 * atan(1.0), TWO_PI = 2.0 * PI, dx = 2.0 * PI / (double)n;
    double *f = F(o, 3 + s), *w0 = W(o, 0), *w1 = W(o, 1), *w2 = W(o, 2), *w3 = W(o, 3);
    if (ic == 0) {
        memset(f, 0, sizeof(double) * o->fsz);
    } else if (ic < 10) {
        if (type != 1 && type != 2 && type != 3) return -1;
        (void)oracle_randu(&o->rs, -rn2);
        for (size_t q = 0; q < o->fsz; q++) w1[q] = oracle_randu(&o->rs, rn2);
        for (size_t q = 0; q < o->fsz; q++) w2[q] = oracle_randu(&o->rs, rn2);
        for (size_t q = 0; q < o->fsz; q++) w3[q] = sqrt(-2.0 * log(w1[q])) * sin(TWO_PI * w2[q]);
        xfft3d(o, 1, w3);
        copy_field(o, f, w3);
        double *es = (double *)calloc(kmax + 1, sizeof(double)), *et = (double *)calloc(kmax + 1, sizeof(double));
        oracle_energy_spectrum(o, 3 + s, 1, es);
        for (int k = 1; k <= kmax; k++) {
            double wmag = (double)k, ratio = wmag / peak;
            if (type == 1 || type == 3) et[k - 1] = ratio * ratio * ratio / peak * exp(-3.0 * ratio);
            else {
                double ff = 2.0 * PI * ratio, f2 = ff * ff, d = 1.0 + f2;
                et[k - 1] = (f2 * f2) / (d * d * d);
            }
        }
        double tot = 0.0;
        for (int k = 0; k < kmax; k++) tot = tot + et[k];
        for (int k = 0; k < kmax; k++) et[k] = et[k] / tot;
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n + 2; i++) {
                    double k2 = o->akx[i] * o->akx[i] + o->aky[k] * o->aky[k] + o->akz[j] * o->akz[j];
                    int sh = nint_shell32(k2);
                    size_t a = IX(o, i, j, k);
                    f[a] = (sh > 0 && sh <= kmax && es[sh - 1] > 0.0) ? w3[a] * sqrt(et[sh - 1] / es[sh - 1]) : 0.0;
                }
        free(es); free(et);
        if (type == 3) {
            copy_field(o, w0, f);
            xfft3d(o, -1, w0);
            for (size_t q = 0; q < o->fsz; q++) w0[q] = w0[q] < 0.0 ? -0.9 : 0.9;
            xfft3d(o, 1, w0);
            for (int k = 0; k < n; k++)
                for (int j = 0; j < n; j++)
                    for (int i = 0; i < n + 2; i++) {
                        double k2 = o->akx[i] * o->akx[i] + o->aky[k] * o->aky[k] + o->akz[j] * o->akz[j];
                        int sh = nint_shell32(k2);
                        if (sh == 0 || sh >= kmax * 2 / 3) w0[IX(o, i, j, k)] = 0.0;
                    }
            copy_field(o, f, w0);
        }
    } else {
        if (ic != 11 && ic != 12 && ic != 13) return -1;
        memset(w0, 0, sizeof(double) * o->fsz);
        double h11 = fmax(2.0 * dx, TWO_PI / peak), h12 = fmax(8.0 * dx, PI / 8.0);
        double pk = fmin(peak, (double)(n / 8));
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) {
                    double z = (double)k * dx, x = (double)i * dx, v;
                    if (ic == 11) v = tanh((z - PI * 0.5) / h11) - tanh((z - PI * 1.5) / h11) - 1.0;
                    else if (ic == 12)
                        v = tanh((x - PI * 0.25) / h12) - tanh((x - PI * 0.75) / h12) + tanh((x - PI * 1.25) / h12) -
                            tanh((x - PI * 1.75) / h12) - 1.0;
                    else v = sin(pk * dx * (double)i);
                    w0[IX(o, i, j, k)] = v;
                }
        xfft3d(o, 1, w0);
        copy_field(o, f, w0);
        if (ic != 13) f[0] = 0.0;
    }
    for (size_t q = 0; q < o->fsz; q++)
        if (o->ialias[q] > 0) f[q] = 0.0;
    return 0;
}

/* ------------------------------------------------------------------------- */
/*  velocity_rescale (velocity_rescale.f90:1-159): shell energies without the */
/*  kx=0 half weight, averaged by hits and scaled by the shell volume, then   */
/*  the velocity is rescaled to the target spectrum                           */
/* ------------------------------------------------------------------------- */
int oracle_velocity_rescale(oracle_t *o, int isp_type, double peak_wavenum, double ir_exp)
{
    int n = o->n, kmax = o->kmax;
    double PI = 4.0 * atan(1.0);
    if (isp_type == -1) return 0;
    double fac = 1.0 / (((double)n * n * n) * ((double)n * n * n));
    double *es = (double *)calloc(kmax, sizeof(double));
    double *et = (double *)calloc(kmax, sizeof(double));
    int64_t *hits = (int64_t *)calloc(kmax, sizeof(int64_t));
    double *u = F(o, 0), *v = F(o, 1), *w = F(o, 2);
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                double k2 = o->akx[i] * o->akx[i] + o->aky[k] * o->aky[k] + o->akz[j] * o->akz[j];
                int sh = nint_shell32(k2);
                if (sh > 0 && sh <= kmax) {
                    size_t a = IX(o, i, j, k);
                    hits[sh - 1] += 1;
                    es[sh - 1] = es[sh - 1] + fac * (u[a] * u[a] + v[a] * v[a] + w[a] * w[a]);
                }
            }
    double fv = 4.0 / 3.0 * PI / 2.0;
    for (int k = 1; k <= kmax; k++) {
        double r1 = (double)k + 0.5, r2 = (double)k - 0.5;
        if (k == 1) r2 = 0.0;
        if (hits[k - 1] > 0) es[k - 1] = es[k - 1] / (double)hits[k - 1] * fv * (r1 * r1 * r1 - r2 * r2 * r2);
        else es[k - 1] = 0.0;
    }
    for (int k = 1; k <= kmax; k++) {
        double wmag = (double)k, ratio = wmag / peak_wavenum;
        if (isp_type == 0) et[k - 1] = pow(wmag, -5.0 / 3.0);
        else if (isp_type == 1) et[k - 1] = ratio * ratio * ratio / peak_wavenum * exp(-3.0 * ratio);
        else if (isp_type == 2) et[k - 1] = pow(wmag, ir_exp) * exp(-2.0 * ratio * ratio);
        else if (isp_type == 3) {
            double f = 2.0 * PI * ratio, f2 = f * f, d = 1.0 + f2;
            et[k - 1] = (f2 * f2) / (d * d * d);
        } else { free(es); free(et); free(hits); return -1; }
    }
    double tot = 0.0;
    for (int k = 0; k < kmax; k++) tot = tot + et[k];
    for (int k = 0; k < kmax; k++) et[k] = et[k] / tot;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 2; i++) {
                double k2 = o->akx[i] * o->akx[i] + o->aky[k] * o->aky[k] + o->akz[j] * o->akz[j];
                int sh = nint_shell32(k2);
                size_t a = IX(o, i, j, k);
                if (sh > 0 && sh <= kmax && es[sh - 1] > 0.0) {
                    double r = sqrt(et[sh - 1] / es[sh - 1]);
                    for (int c = 0; c < 3; c++) F(o, c)[a] = F(o, c)[a] * r;
                } else {
                    for (int c = 0; c < 3; c++) F(o, c)[a] = 0.0;
                }
            }
    free(es); free(et); free(hits);
    return 0;
}

/* ------------------------------------------------------------------------- */
/*  particles (m_particles.f90:815-1230, 1451-1508) on one periodic slab     */
/*  uphys: three (nx+2,ny,nz) physical velocity arrays; xyzp/uvwp: 3*np,     */
/*  particle-major like the reference's (3,np) arrays.                       */
/* ------------------------------------------------------------------------- */
static double cint1(double p1, double p2, double p3, double p4, const double *r)
{
    return (r[0] * p1 + r[1] * p2 + r[2] * p3 + r[3] * p4) / 6.0;
}

static void cint_r(double x, double *r)
{
    double s = (x - 1.0) * (x - 2.0);
    r[0] = -x * s;
    r[1] = 3.0 * (x + 1.0) * s;
    s = (x + 1.0) * x;
    r[2] = -3.0 * s * (x - 2.0);
    r[3] = s * (x - 1.0);
}

static double cint_3d(const double a[4][4][4] /* [k][j][i] */, double x, double y, double z)
{
    double r[4], t2[4][4], t1[4];
    cint_r(x, r);
    for (int k = 0; k < 4; k++)
        for (int j = 0; j < 4; j++) t2[k][j] = cint1(a[k][j][0], a[k][j][1], a[k][j][2], a[k][j][3], r);
    cint_r(y, r);
    for (int k = 0; k < 4; k++) t1[k] = cint1(t2[k][0], t2[k][1], t2[k][2], t2[k][3], r);
    cint_r(z, r);
    return cint1(t1[0], t1[1], t1[2], t1[3], r);
}

void oracle_particles_step(int n, double dt, const double *uphys, int64_t np, double *xyzp, double *uvwp,
                           int scheme)
{
    size_t fsz = (size_t)(n + 2) * n * n;
    double PI = 4.0 * atan(1.0);
    double dx = 2.0 * PI / (double)n, dy = dx, dz = dx;
    const double *U[3] = {uphys, uphys + fsz, uphys + 2 * fsz};
#define PIX(i, j, k) ((size_t)((i) - 1) + (size_t)(n + 2) * ((size_t)((j) - 1) + (size_t)n * (size_t)((k) - 1)))
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < np; p++) {
        double *X = xyzp + 3 * p, *V = uvwp + 3 * p;
        int i = (int)floor(X[0]), j = (int)floor(X[1]), k = (int)floor(X[2]);
        double xp = X[0] - (double)i, yp = X[1] - (double)j, zp = X[2] - (double)k;
        double up[3];
        if (scheme == 0) {
            double c1 = (1.0 - xp) * (1.0 - yp) * (1.0 - zp);
            double c2 = (xp) * (1.0 - yp) * (1.0 - zp);
            double c3 = (1.0 - xp) * (yp) * (1.0 - zp);
            double c4 = (xp) * (yp) * (1.0 - zp);
            double c5 = (1.0 - xp) * (1.0 - yp) * (zp);
            double c6 = (xp) * (1.0 - yp) * (zp);
            double c7 = (1.0 - xp) * (yp) * (zp);
            double c8 = (xp) * (yp) * (zp);
            int i1 = (i == n) ? 1 : i + 1;
            int j1 = (j == n) ? 1 : j + 1;
            int k1 = (k == n) ? 1 : k + 1;
            for (int c = 0; c < 3; c++) {
                const double *f = U[c];
                double s = c1 * f[PIX(i, j, k)] + c2 * f[PIX(i1, j, k)] + c3 * f[PIX(i, j1, k)] + c4 * f[PIX(i1, j1, k)];
                s = s + c5 * f[PIX(i, j, k1)] + c6 * f[PIX(i1, j, k1)] + c7 * f[PIX(i, j1, k1)] + c8 * f[PIX(i1, j1, k1)];
                up[c] = s;
            }
        } else {
            double loc[3][4][4][4];
            for (int kk = 0; kk < 4; kk++) {
                int k1 = k - 2 + kk + 1;
                if (k1 < 1) k1 += n;
                if (k1 > n) k1 -= n;
                for (int jj = 0; jj < 4; jj++) {
                    int j1 = j - 2 + jj + 1;
                    if (j1 < 1) j1 += n;
                    if (j1 > n) j1 -= n;
                    for (int ii = 0; ii < 4; ii++) {
                        int i1 = i - 2 + ii + 1;
                        if (i1 < 1) i1 += n;
                        if (i1 > n) i1 -= n;
                        for (int c = 0; c < 3; c++) loc[c][kk][jj][ii] = U[c][PIX(i1, j1, k1)];
                    }
                }
            }
            for (int c = 0; c < 3; c++) up[c] = cint_3d(loc[c], xp, yp, zp);
        }
        if (V[0] == -999.0) {
            xp = xp + dt * up[0] / dx;
            yp = yp + dt * up[1] / dy;
            zp = zp + dt * up[2] / dz;
        } else {
            xp = xp + (1.50 * up[0] - 0.50 * V[0]) * dt / dx;
            yp = yp + (1.50 * up[1] - 0.50 * V[1]) * dt / dy;
            zp = zp + (1.50 * up[2] - 0.50 * V[2]) * dt / dz;
        }
        V[0] = up[0]; V[1] = up[1]; V[2] = up[2];
        if (xp > 1.0) { xp = xp - 1.0; i = i + 1; if (i > n) i = i - n; }
        if (xp < 0.0) { xp = xp + 1.0; i = i - 1; if (i < 1) i = i + n; }
        if (yp > 1.0) { yp = yp - 1.0; j = j + 1; if (j > n) j = j - n; }
        if (yp < 0.0) { yp = yp + 1.0; j = j - 1; if (j < 1) j = j + n; }
        if (zp > 1.0) { zp = zp - 1.0; k = k + 1; }
        if (zp < 0.0) { zp = zp + 1.0; k = k - 1; }
        X[0] = xp + (double)i;
        X[1] = yp + (double)j;
        X[2] = zp + (double)k;
        /* slab migration on a single periodic slab (m_particles.f90:1270-1319) */
        if (X[2] >= (double)(n + 1)) X[2] = X[2] - (double)n;
        else if (X[2] < 1.0) X[2] = X[2] + (double)n;
    }
#undef PIX
}

/* lattice initialisation (m_particles.f90:220-262, 314-319): returns nptot */
int64_t oracle_particles_lattice(int n, int64_t nptot_in, double *xyzp /* may be NULL */)
{
    int64_t npt = (int64_t)((double)nptot_in > 0 ? pow((double)nptot_in, 1.0 / 3.0) : 0);
    if (nptot_in - npt * npt * npt >= (npt + 1) * (npt + 1) * (npt + 1) - nptot_in) npt = npt + 1;
    int64_t nptot = npt * npt * npt;
    if (!xyzp) return nptot;
    double PI = 4.0 * atan(1.0);
    double sctmp = 2.0 * PI / (double)npt;
    int64_t m = 0;
    for (int64_t k = 1; k <= npt; k++)
        for (int64_t j = 1; j <= npt; j++)
            for (int64_t i = 1; i <= npt; i++) {
                xyzp[3 * m + 0] = ((double)(i - 1) + 0.5) * sctmp;
                xyzp[3 * m + 1] = ((double)(j - 1) + 0.5) * sctmp;
                xyzp[3 * m + 2] = ((double)(k - 1) + 0.5) * sctmp;
                m++;
            }
    for (int64_t p = 0; p < nptot * 3; p++) {
        double x = xyzp[p];
        if (x >= 2.0 * PI || x < 0.0) xyzp[p] = x - 2.0 * PI * floor(x / (2.0 * PI));
    }
    for (int64_t p = 0; p < nptot; p++) {
        xyzp[3 * p + 0] = xyzp[3 * p + 0] / (2.0 * PI / (double)n) + 1.0;
        xyzp[3 * p + 1] = xyzp[3 * p + 1] / (2.0 * PI / (double)n) + 1.0;
        xyzp[3 * p + 2] = xyzp[3 * p + 2] / (2.0 * PI / (double)n) + 1.0;
    }
    return nptot;
}

/* ------------------------------------------------------------------------- */
/*  filters (m_filter_xfftw.f90:121-286) and subgrid stress                  */
/*  kind 2 = Gaussian (reference), kind 4 = box (new).  Returns filter_g in  */
/*  the Fourier layout of one (nx+2,ny,nz) array.                            */
/* ------------------------------------------------------------------------- */
void oracle_filter_g(oracle_t *o, int kind, double delta, double *g)
{
    int n = o->n;
    double PI = 4.0 * atan(1.0), dx = o->dx;
    memset(g, 0, sizeof(double) * o->fsz);
    if (kind == 2) {
        double c1 = 6.0 / (delta * delta);
        double sq = sqrt(c1 / PI);
        double c2 = sq * sq * sq * (dx * dx * dx);
        for (int k = 0; k < n; k++) {
            int dk = k < n - k ? k : n - k;
            double rz = dx * (double)dk;
            for (int j = 0; j < n; j++) {
                int dj = j < n - j ? j : n - j;
                double ry = dx * (double)dj;
                for (int i = 0; i < n; i++) {
                    int di = i < n - i ? i : n - i;
                    double rx = dx * (double)di;
                    rx = rx * rx + ry * ry + rz * rz;
                    double v = c2 * exp(-c1 * rx);
                    if (v < 1.e-20) v = 0.0;
                    g[IX(o, i, j, k)] = v;
                }
            }
        }
        xfft3d(o, 1, g);
    } else {
        /* box filter of width delta: spectral transfer function
         * prod_a sin(k_a delta/2)/(k_a delta/2), real, stored in the re slots */
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n + 1; i += 2) {
                    double h = 1.0;
                    double ks[3] = {o->akx[i], o->aky[k], o->akz[j]};
                    for (int a = 0; a < 3; a++) {
                        double t = 0.5 * ks[a] * delta;
                        h *= (t == 0.0) ? 1.0 : sin(t) / t;
                    }
                    g[IX(o, i, j, k)] = h;
                    g[IX(o, i, j, k) + 1] = 0.0;
                }
    }
}

void oracle_apply_filter(oracle_t *o, const double *g, double *a)
{
    int n = o->n;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n + 1; i += 2) {
                size_t p = IX(o, i, j, k);
                double x = a[p], y = a[p + 1], c = g[p], d = g[p + 1];
                a[p] = x * c - y * d;
                a[p + 1] = y * c + x * d;
            }
}

int oracle_n(oracle_t *o) { return o->n; }
void oracle_les_stats(oracle_t *o, double *out)
{
    for (int q = 0; q < 4; q++) out[q] = o->les_stat[q];
}
size_t oracle_fsz(oracle_t *o) { return o->fsz; }
double oracle_time(oracle_t *o) { return o->time; }
void oracle_set_time(oracle_t *o, double t) { o->time = t; }
double *oracle_turb_visc(oracle_t *o) { return o->turb_visc; }
