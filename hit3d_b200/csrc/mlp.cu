// C-ABI of the learned subgrid closure (declared in include/hit3d_gpu.h): a
// network handle with its training data on one device, the training step
// (forward, backward, weight gradients, Adam) and inference.  No reference
// counterpart; the Smagorinsky model (m_les.f90:1142-1215) is the fallback.
#include <cmath>
#include <cstring>
#include <mutex>
#include <set>
#include <vector>

#include "../../include/hit3d_gpu.h"
#include "mlp_tc.cuh"

#define M_TRY(x)                    \
    do {                            \
        int rc__ = (x);             \
        if (rc__ != 0) return rc__; \
    } while (0)

struct hit3d_mlp {
    int dev;
    cudaStream_t st;
    float *w, *m, *v, *g;  // fp32 master parameters, Adam moments, gradient
    __nv_bfloat16 *wb;     // the bf16 weights the kernels read
    int64_t t;             // Adam steps taken
    float *A, *tau;        // dataset [9][P] and [6][P]
    int64_t P;
    double delta, inv_norm, inv_norm_p;
    // minibatch scratch for up to cap points
    int64_t cap;
    float *z, *x, *d, *d4, *lossp, *part, *losses;
    int32_t *idx;
    int64_t loss_cap;
};

static int mlp_smem(const void *k)
{
    static std::mutex mu;
    static std::set<std::pair<const void *, int>> done;
    int dev = 0;
    H3D_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair(k, dev);
    if (done.count(key)) return 0;
    H3D_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_SMEM));
    done.insert(key);
    return 0;
}

static void mfree(void *p)
{
    if (p) cudaFree(p);
}

extern "C" int hit3d_mlp_nparam(void) { return MLP_NPARAM; }

// Glorot-uniform hidden weights from a splitmix64 stream, the output layer
// scaled by 0.1, zero biases
static void init_weights(uint64_t seed, std::vector<float> &w)
{
    w.assign(MLP_NPARAM, 0.0f);
    uint64_t s = seed;
    auto uni = [&]() { s = splitmix64(s); return (double)(s >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0; };
    struct L { int off, nin, nout; double scale; } ls[4] = {
        {MLP_W1, MLP_IN, MLP_H, 1.0}, {MLP_W2, MLP_H, MLP_H, 1.0}, {MLP_W3, MLP_H, MLP_H, 1.0}, {MLP_W4, MLP_H, MLP_OUT, 0.1}};
    for (auto &l : ls) {
        const double a = l.scale * std::sqrt(6.0 / (l.nin + l.nout));
        for (int q = 0; q < l.nin * l.nout; q++) w[l.off + q] = (float)(a * uni());
    }
}

static int upload_params(hit3d_mlp *m, const float *w)
{
    H3D_CHECK(cudaMemcpyAsync(m->w, w, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice, m->st));
    k_to_bf16<<<(MLP_NPARAM + 255) / 256, 256, 0, m->st>>>(MLP_NPARAM, m->w, m->wb);
    H3D_CHECK(cudaGetLastError());
    H3D_CHECK(cudaMemsetAsync(m->m, 0, sizeof(float) * MLP_NPARAM, m->st));
    H3D_CHECK(cudaMemsetAsync(m->v, 0, sizeof(float) * MLP_NPARAM, m->st));
    H3D_CHECK(cudaStreamSynchronize(m->st));
    m->t = 0;
    return 0;
}

extern "C" int hit3d_mlp_create(int32_t device, uint64_t seed, hit3d_mlp **out)
{
    if (!out) return h3d_set_error_msg(-1, "hit3d_mlp_create: null argument");
    *out = nullptr;
    H3D_CHECK(cudaSetDevice(device));
    hit3d_mlp *m = new hit3d_mlp();
    m->dev = device;
    int rc = 0;
    auto fail = [&](int r) { hit3d_mlp_destroy(m); return r; };
    if (cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess)
        return fail(h3d_set_error_msg(-2, "hit3d_mlp_create: stream creation failed"));
    for (float **p : {&m->w, &m->m, &m->v, &m->g})
        if (cudaMalloc(p, sizeof(float) * MLP_NPARAM) != cudaSuccess)
            return fail(h3d_set_error_msg(-4, "hit3d_mlp_create: out of device memory"));
    if (cudaMalloc(&m->wb, sizeof(__nv_bfloat16) * MLP_NPARAM) != cudaSuccess)
        return fail(h3d_set_error_msg(-4, "hit3d_mlp_create: out of device memory"));
    std::vector<float> w;
    init_weights(seed, w);
    if ((rc = upload_params(m, w.data())) != 0) return fail(rc);
    *out = m;
    return 0;
}

extern "C" int hit3d_mlp_destroy(hit3d_mlp *m)
{
    if (!m) return 0;
    cudaSetDevice(m->dev);
    if (m->st) cudaStreamSynchronize(m->st);
    for (void *p : {(void *)m->w, (void *)m->m, (void *)m->v, (void *)m->g, (void *)m->wb, (void *)m->A, (void *)m->tau,
                    (void *)m->z, (void *)m->x, (void *)m->d, (void *)m->d4, (void *)m->lossp, (void *)m->part,
                    (void *)m->losses, (void *)m->idx})
        mfree(p);
    if (m->st) cudaStreamDestroy(m->st);
    delete m;
    return 0;
}

extern "C" int hit3d_mlp_set_params(hit3d_mlp *m, const float *w)
{
    if (!m || !w) return h3d_set_error_msg(-1, "hit3d_mlp_set_params: null argument");
    H3D_CHECK(cudaSetDevice(m->dev));
    return upload_params(m, w);
}

extern "C" int hit3d_mlp_get_params(hit3d_mlp *m, float *w)
{
    if (!m || !w) return h3d_set_error_msg(-1, "hit3d_mlp_get_params: null argument");
    H3D_CHECK(cudaSetDevice(m->dev));
    H3D_CHECK(cudaMemcpyAsync(w, m->w, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, m->st));
    H3D_CHECK(cudaStreamSynchronize(m->st));
    return 0;
}

extern "C" int hit3d_mlp_get_bf16(hit3d_mlp *m, uint16_t *wb)
{
    if (!m || !wb) return h3d_set_error_msg(-1, "hit3d_mlp_get_bf16: null argument");
    H3D_CHECK(cudaSetDevice(m->dev));
    H3D_CHECK(cudaMemcpyAsync(wb, m->wb, sizeof(uint16_t) * MLP_NPARAM, cudaMemcpyDeviceToHost, m->st));
    H3D_CHECK(cudaStreamSynchronize(m->st));
    return 0;
}

// the dataset: gradients A [9][P] and stresses tau [6][P] (host, fp32); the
// stresses are stored deviatoric, the loss normalisations computed in FP64
extern "C" int hit3d_mlp_set_data(hit3d_mlp *m, const float *A, const float *tau, int64_t P, double delta)
{
    if (!m || !A || !tau) return h3d_set_error_msg(-1, "hit3d_mlp_set_data: null argument");
    if (P <= 0 || P > INT32_MAX) return h3d_set_error_msg(-1, "hit3d_mlp_set_data: point count out of range");
    if (!(delta > 0.0)) return h3d_set_error_msg(-1, "hit3d_mlp_set_data: filter width must be positive");
    H3D_CHECK(cudaSetDevice(m->dev));
    std::vector<float> td((size_t)6 * P);
    double sn = 0.0, sp = 0.0;
    for (int64_t q = 0; q < P; q++) {
        const double tr = ((double)tau[q] + tau[3 * P + q] + tau[5 * P + q]) / 3.0;
        float t6[6];
        for (int c = 0; c < 6; c++) t6[c] = (float)(tau[c * P + q] - ((c == 0 || c == 3 || c == 5) ? tr : 0.0));
        // strain from A (11, 12, 13, 22, 23, 33)
        const int ii[6] = {0, 0, 0, 1, 1, 2}, jj[6] = {0, 1, 2, 1, 2, 2};
        double n2 = 0.0, pi = 0.0;
        for (int c = 0; c < 6; c++) {
            const double s = 0.5 * ((double)A[(3 * ii[c] + jj[c]) * P + q] + A[(3 * jj[c] + ii[c]) * P + q]);
            n2 += frob_w(c) * (double)t6[c] * t6[c];
            pi -= frob_w(c) * (double)t6[c] * s;
            td[c * P + q] = t6[c];
        }
        sn += n2;
        sp += pi * pi;
    }
    mfree(m->A);
    mfree(m->tau);
    m->A = m->tau = nullptr;
    if (cudaMalloc(&m->A, sizeof(float) * 9 * P) != cudaSuccess || cudaMalloc(&m->tau, sizeof(float) * 6 * P) != cudaSuccess)
        return h3d_set_error_msg(-4, "hit3d_mlp_set_data: out of device memory");
    H3D_CHECK(cudaMemcpyAsync(m->A, A, sizeof(float) * 9 * P, cudaMemcpyHostToDevice, m->st));
    H3D_CHECK(cudaMemcpyAsync(m->tau, td.data(), sizeof(float) * 6 * P, cudaMemcpyHostToDevice, m->st));
    H3D_CHECK(cudaStreamSynchronize(m->st));
    m->P = P;
    m->delta = delta;
    m->inv_norm = sn > 0 ? (double)P / sn : 1.0;
    m->inv_norm_p = sp > 0 ? (double)P / sp : 1.0;
    return 0;
}

extern "C" int hit3d_mlp_norms(hit3d_mlp *m, double *out2)
{
    if (!m || !out2) return h3d_set_error_msg(-1, "hit3d_mlp_norms: null argument");
    out2[0] = m->inv_norm;
    out2[1] = m->inv_norm_p;
    return 0;
}

static int ensure_cap(hit3d_mlp *m, int64_t np)
{
    if (np <= m->cap) return 0;
    for (void *p : {(void *)m->z, (void *)m->x, (void *)m->d, (void *)m->d4, (void *)m->lossp, (void *)m->part,
                    (void *)m->idx})
        mfree(p);
    m->z = m->x = m->d = m->d4 = m->lossp = m->part = nullptr;
    m->idx = nullptr;
    m->cap = 0;
    const int64_t nb = (np + MLP_NT - 1) / MLP_NT, nc = (np + WG_C - 1) / WG_C;
    bool ok = cudaMalloc(&m->z, sizeof(float) * 3 * MLP_H * np) == cudaSuccess &&
              cudaMalloc(&m->d, sizeof(float) * 3 * MLP_H * np) == cudaSuccess &&
              cudaMalloc(&m->x, sizeof(float) * MLP_IN * np) == cudaSuccess &&
              cudaMalloc(&m->d4, sizeof(float) * MLP_OUT * np) == cudaSuccess &&
              cudaMalloc(&m->lossp, sizeof(float) * nb) == cudaSuccess &&
              cudaMalloc(&m->part, sizeof(float) * MLP_NPARAM * nc) == cudaSuccess &&
              cudaMalloc(&m->idx, sizeof(int32_t) * np) == cudaSuccess;
    if (!ok) return h3d_set_error_msg(-4, "hit3d_mlp: out of device memory for the minibatch");
    m->cap = np;
    return 0;
}

static MlpBatch batch_args(hit3d_mlp *m, int64_t np, double lam)
{
    MlpBatch b;
    b.np = np; b.idx = m->idx; b.A = m->A; b.tau = m->tau; b.P = m->P;
    b.delta = (float)m->delta; b.inv_norm = (float)m->inv_norm; b.inv_norm_p = (float)m->inv_norm_p; b.lam = (float)lam;
    b.z = m->z; b.x = m->x; b.d = m->d; b.d4 = m->d4; b.loss = m->lossp;
    return b;
}

// loss (into dev_loss) and gradient (into m->g) of the minibatch in m->idx
static int loss_grad(hit3d_mlp *m, int64_t np, double lam, float *dev_loss)
{
    M_TRY(mlp_smem((const void *)k_mlp_fwd));
    M_TRY(mlp_smem((const void *)k_mlp_bwd));
    const MlpBatch b = batch_args(m, np, lam);
    const int nb = (int)((np + MLP_NT - 1) / MLP_NT), nc = (int)((np + WG_C - 1) / WG_C);
    k_mlp_fwd<<<nb, MLP_NT, MLP_SMEM, m->st>>>(b, m->wb);
    H3D_CHECK(cudaGetLastError());
    k_sum_partials<<<1, 32, 0, m->st>>>(nb, m->lossp, dev_loss);
    H3D_CHECK(cudaGetLastError());
    k_mlp_bwd<<<nb, MLP_NT, MLP_SMEM, m->st>>>(b, m->wb);
    H3D_CHECK(cudaGetLastError());
    k_mlp_wgrad_part<<<dim3(nc, 4), 256, 0, m->st>>>(b, m->part);
    H3D_CHECK(cudaGetLastError());
    k_mlp_wgrad_sum<<<(MLP_NPARAM + 255) / 256, 256, 0, m->st>>>(nc, m->part, m->g);
    H3D_CHECK(cudaGetLastError());
    return 0;
}

extern "C" int hit3d_mlp_loss_grad(hit3d_mlp *m, const int32_t *idx, int64_t np, double lam, float *loss, float *grad)
{
    if (!m || !idx || !loss || !grad) return h3d_set_error_msg(-1, "hit3d_mlp_loss_grad: null argument");
    if (!m->A) return h3d_set_error_msg(-1, "hit3d_mlp_loss_grad: no data (call hit3d_mlp_set_data)");
    if (np <= 0) return h3d_set_error_msg(-1, "hit3d_mlp_loss_grad: empty minibatch");
    for (int64_t p = 0; p < np; p++)
        if (idx[p] < 0 || idx[p] >= m->P) return h3d_set_error_msg(-1, "hit3d_mlp_loss_grad: index out of range");
    H3D_CHECK(cudaSetDevice(m->dev));
    M_TRY(ensure_cap(m, np));
    if (m->loss_cap < 1) {
        if (cudaMalloc(&m->losses, sizeof(float)) != cudaSuccess) return h3d_set_error_msg(-4, "hit3d_mlp: out of memory");
        m->loss_cap = 1;
    }
    H3D_CHECK(cudaMemcpyAsync(m->idx, idx, sizeof(int32_t) * np, cudaMemcpyHostToDevice, m->st));
    M_TRY(loss_grad(m, np, lam, m->losses));
    H3D_CHECK(cudaMemcpyAsync(loss, m->losses, sizeof(float), cudaMemcpyDeviceToHost, m->st));
    H3D_CHECK(cudaMemcpyAsync(grad, m->g, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, m->st));
    H3D_CHECK(cudaStreamSynchronize(m->st));
    return 0;
}

extern "C" int hit3d_mlp_train(hit3d_mlp *m, int32_t nsteps, int64_t batch, double lr, double lam, uint64_t seed,
                               float *losses)
{
    if (!m) return h3d_set_error_msg(-1, "hit3d_mlp_train: null argument");
    if (!m->A) return h3d_set_error_msg(-1, "hit3d_mlp_train: no data (call hit3d_mlp_set_data)");
    if (nsteps < 0 || batch <= 0 || batch > INT32_MAX) return h3d_set_error_msg(-1, "hit3d_mlp_train: bad step count or batch");
    H3D_CHECK(cudaSetDevice(m->dev));
    M_TRY(ensure_cap(m, batch));
    if (m->loss_cap < nsteps) {
        mfree(m->losses);
        m->losses = nullptr;
        m->loss_cap = 0;
        if (cudaMalloc(&m->losses, sizeof(float) * (nsteps > 0 ? nsteps : 1)) != cudaSuccess)
            return h3d_set_error_msg(-4, "hit3d_mlp_train: out of device memory");
        m->loss_cap = nsteps;
    }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int s = 0; s < nsteps; s++) {
        k_sample_idx<<<(unsigned)((batch + 255) / 256), 256, 0, m->st>>>(batch, m->P, splitmix64(seed + 0x632be59bd9b4e019ull * (uint64_t)(m->t + 1)), m->idx);
        H3D_CHECK(cudaGetLastError());
        M_TRY(loss_grad(m, batch, lam, m->losses + s));
        m->t++;
        const float c1 = (float)(1.0 - std::pow((double)b1, (double)m->t)), c2 = (float)(1.0 - std::pow((double)b2, (double)m->t));
        k_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, m->st>>>(MLP_NPARAM, (float)lr, b1, b2, eps, c1, c2, m->g, m->w, m->m,
                                                             m->v, m->wb);
        H3D_CHECK(cudaGetLastError());
    }
    if (losses && nsteps > 0)
        H3D_CHECK(cudaMemcpyAsync(losses, m->losses, sizeof(float) * nsteps, cudaMemcpyDeviceToHost, m->st));
    H3D_CHECK(cudaStreamSynchronize(m->st));
    return 0;
}

static int sm_count()
{
    static int cache[64] = {0};
    int dev = 0;
    H3D_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) H3D_CHECK(cudaDeviceGetAttribute(&cache[dev], cudaDevAttrMultiProcessorCount, dev));
    return cache[dev];
}

// one launch of the inference kernel on fields in device memory (used by the
// LES step as well): kernel 0 = fp32 activations on the CUDA cores, 1 = hidden
// layers on the tensor cores (bf16 activations); err receives 1 if a
// tensor-core completion wait ran out
int h3d_mlp_apply(cudaStream_t st, int fp64, int64_t np, int64_t n, int64_t rp, int64_t fs, double delta, int clip,
                  int kernel, const void *wb, void *G, int *err)
{
    if ((np + MLP_NT - 1) / MLP_NT > INT32_MAX) return h3d_set_error_msg(-1, "h3d_mlp_apply: too many points");
    const __nv_bfloat16 *w = static_cast<const __nv_bfloat16 *>(wb);
    if (kernel == 1) {
        if (!err) return h3d_set_error_msg(-1, "h3d_mlp_apply: the tensor-core kernel needs an error flag");
        const int64_t ntile = (np + TC_TILE - 1) / TC_TILE;
        const int nsm = sm_count();
        if (nsm <= 0) return nsm;
        const int nblk = (int)std::min<int64_t>(ntile, (int64_t)nsm * 4);
        if (fp64)
            k_mlp_apply_tc<double><<<nblk, TC_TILE, TC_SMEM, st>>>(np, n, rp, fs, (float)delta, clip, w, (double *)G, err);
        else
            k_mlp_apply_tc<float><<<nblk, TC_TILE, TC_SMEM, st>>>(np, n, rp, fs, (float)delta, clip, w, (float *)G, err);
        H3D_CHECK(cudaGetLastError());
        return 0;
    }
    if (kernel != 0) return h3d_set_error_msg(-1, "h3d_mlp_apply: kernel must be 0 or 1");
    const int nblk = (int)((np + MLP_NT - 1) / MLP_NT);
    if (fp64) {
        M_TRY(mlp_smem((const void *)k_mlp_apply<double>));
        k_mlp_apply<double><<<nblk, MLP_NT, MLP_SMEM, st>>>(np, n, rp, fs, (float)delta, clip, w, (double *)G);
    } else {
        M_TRY(mlp_smem((const void *)k_mlp_apply<float>));
        k_mlp_apply<float><<<nblk, MLP_NT, MLP_SMEM, st>>>(np, n, rp, fs, (float)delta, clip, w, (float *)G);
    }
    H3D_CHECK(cudaGetLastError());
    return 0;
}

extern "C" int hit3d_mlp_predict(hit3d_mlp *m, const float *A, int64_t np, double delta, int32_t clip, int32_t kernel,
                                 float *tau)
{
    if (!m || !A || !tau) return h3d_set_error_msg(-1, "hit3d_mlp_predict: null argument");
    if (np <= 0) return h3d_set_error_msg(-1, "hit3d_mlp_predict: empty input");
    if (kernel != 0 && kernel != 1) return h3d_set_error_msg(-1, "hit3d_mlp_predict: kernel must be 0 or 1");
    H3D_CHECK(cudaSetDevice(m->dev));
    float *G = nullptr;
    int *err = nullptr;
    if (cudaMalloc(&G, sizeof(float) * 9 * np) != cudaSuccess || cudaMalloc(&err, sizeof(int)) != cudaSuccess) {
        mfree(G);
        return h3d_set_error_msg(-4, "hit3d_mlp_predict: out of device memory");
    }
    int rc = 0, herr = 0;
    if (cudaMemsetAsync(err, 0, sizeof(int), m->st) != cudaSuccess ||
        cudaMemcpyAsync(G, A, sizeof(float) * 9 * np, cudaMemcpyHostToDevice, m->st) != cudaSuccess)
        rc = h3d_set_error_msg(-2, "hit3d_mlp_predict: upload failed");
    if (!rc) rc = h3d_mlp_apply(m->st, 0, np, np, np, np, delta, clip, kernel, m->wb, G, err);
    if (!rc && (cudaMemcpyAsync(tau, G, sizeof(float) * 6 * np, cudaMemcpyDeviceToHost, m->st) != cudaSuccess ||
                cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, m->st) != cudaSuccess))
        rc = h3d_set_error_msg(-2, "hit3d_mlp_predict: download failed");
    if (!rc && cudaStreamSynchronize(m->st) != cudaSuccess) rc = h3d_set_error_msg(-2, "hit3d_mlp_predict: kernel failed");
    if (!rc && herr) rc = h3d_set_error_msg(-5, "hit3d_mlp_predict: a tensor-core completion wait ran out");
    cudaFree(G);
    cudaFree(err);
    return rc;
}
