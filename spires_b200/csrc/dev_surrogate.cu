// dev_surrogate.cu -- the learned surrogate of the hyper-parameter search.
//
// An MLP 10 -> 128 -> 128 -> 2 with GELU (erf form) that maps a candidate's
// features (hyper-parameters plus its low-fidelity loss) to the mean and the
// log-variance of its full-fidelity log-NRMSE. Trained on the device with
// the Gaussian negative log-likelihood
//     loss = mean_s 0.5 * (v_s + (y_s - m_s)^2 * exp(-v_s))
// by Adam, all in FP32; inference can round weights and activations to BF16
// (FP32 accumulation).
//
// Every product is one of three tiled FP32 GEMM forms on 32x32 tiles staged
// in shared memory:
//     NT: C[i][j] = sum_k A[i][k] B[j][k]   (activations x weights^T)
//     NN: C[i][j] = sum_k A[i][k] B[k][j]   (output gradients x weights)
//     TN: C[i][j] = sum_k A[k][i] B[k][j]   (weight gradients over the batch)
// with fused epilogues (bias, GELU and its pre-activation store, gradient
// scaling by GELU'). The network is 18k parameters and the batches are a few
// thousand rows, so these are latency-sized launches; the layer shapes do
// not fill a tensor-core tile schedule worth its setup.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "sp_alloc.h"
#include "sp_dev.h"
#include "sp_dev_internal.h"

namespace {

constexpr int kIn = 10, kHid = 128, kOut = 2;
constexpr int kP1 = kHid * kIn, kP1b = kHid, kP2 = kHid * kHid, kP2b = kHid, kP3 = kOut * kHid,
              kP3b = kOut;
constexpr int kParams = kP1 + kP1b + kP2 + kP2b + kP3 + kP3b;
// parameter offsets: W1 [128][10], b1, W2 [128][128], b2, W3 [2][128], b3
constexpr int oW1 = 0, ob1 = oW1 + kP1, oW2 = ob1 + kP1b, ob2 = oW2 + kP2, oW3 = ob2 + kP2b,
              ob3 = oW3 + kP3;

constexpr int TILE = 32;

enum Epi : int { EPI_NONE = 0, EPI_BIAS = 1, EPI_BIAS_GELU = 2, EPI_GELU_GRAD = 3 };

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float x)
{
    // d/dx x Phi(x) = Phi(x) + x phi(x)
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

__device__ __forceinline__ float to_bf16(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Generic tiled GEMM. FORM 0 = NT, 1 = NN, 2 = TN (see the file comment).
// C is M x N (ldc); A, B as the form reads them. Epilogues:
//   EPI_BIAS       C = acc + bias[j]
//   EPI_BIAS_GELU  Z = acc + bias[j] (stored to Zout), C = gelu(Z)
//   EPI_GELU_GRAD  C = acc * gelu'(Zin[i][j])
// bf16: round both operands to BF16 as they are staged (inference only).
template <int FORM>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const float *__restrict__ A,
                                              int lda, const float *__restrict__ B, int ldb,
                                              float *__restrict__ C, int ldc,
                                              const float *__restrict__ bias, int epi,
                                              float *__restrict__ Zout, const float *__restrict__ Zin,
                                              int ldz, int bf16, int round_out)
{
    __shared__ float sA[TILE][TILE + 1];
    __shared__ float sB[TILE][TILE + 1];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
    const int i0 = blockIdx.y * TILE, j0 = blockIdx.x * TILE;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};  // rows ty, ty+8, ty+16, ty+24 of the tile; column tx
    for (int k0 = 0; k0 < K; k0 += TILE) {
        for (int r = ty; r < TILE; r += 8) {
            // sA[r][c] = A(i0 + r, k0 + c); sB[c][r'] holds B(k0 + c, j0 + r')
            const int c = tx;
            float a = 0.f, bv = 0.f;
            const int ia = i0 + r, ka = k0 + c;
            if (ia < M && ka < K)
                a = (FORM == 2) ? A[(size_t)ka * lda + ia] : A[(size_t)ia * lda + ka];
            const int jb = j0 + r, kb = k0 + c;
            if (jb < N && kb < K)
                bv = (FORM == 0) ? B[(size_t)jb * ldb + kb] : B[(size_t)kb * ldb + jb];
            if (bf16) {
                a = to_bf16(a);
                bv = to_bf16(bv);
            }
            sA[r][c] = a;
            sB[r][c] = bv;  // sB[j][k]
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < TILE; ++k) {
            const float bk = sB[tx][k];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                acc[q] = fmaf(sA[ty + 8 * q][k], bk, acc[q]);
        }
        __syncthreads();
    }
    const int j = j0 + tx;
    if (j >= N)
        return;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int i = i0 + ty + 8 * q;
        if (i >= M)
            continue;
        float v = acc[q];
        if (epi == EPI_BIAS || epi == EPI_BIAS_GELU)
            v += bias[j];
        if (epi == EPI_BIAS_GELU) {
            if (Zout)
                Zout[(size_t)i * ldz + j] = v;
            v = gelu(v);
        } else if (epi == EPI_GELU_GRAD) {
            v *= gelu_grad(Zin[(size_t)i * ldz + j]);
        }
        if (round_out)
            v = to_bf16(v);
        C[(size_t)i * ldc + j] = v;
    }
}

// dL/d(out) of the Gaussian NLL for rows [0, B), scaled by 1/B; also the
// per-row loss terms.
__global__ void k_nll_grad(const float *__restrict__ out, const float *__restrict__ y, int B,
                           float *__restrict__ dout, float *__restrict__ row_loss)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= B)
        return;
    const float m = out[2 * s], v = out[2 * s + 1];
    const float r = y[s] - m, iv = expf(-v);
    const float inv = 1.0f / (float)B;
    dout[2 * s] = -r * iv * inv;
    dout[2 * s + 1] = 0.5f * (1.0f - r * r * iv) * inv;
    row_loss[s] = 0.5f * (v + r * r * iv);
}

// Column sums (bias gradients): g[j] = sum_s D[s][j], fixed order per column.
__global__ void k_colsum(const float *__restrict__ D, int B, int N, float *__restrict__ g)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N)
        return;
    float a = 0.f;
    for (int s = 0; s < B; ++s)
        a += D[(size_t)s * N + j];
    g[j] = a;
}

// loss = sum of row terms / B (one block, fixed tree)
__global__ void k_mean(const float *__restrict__ x, int B, float *out)
{
    __shared__ float part[256];
    float a = 0.f;
    for (int s = threadIdx.x; s < B; s += 256)
        a += x[s];
    part[threadIdx.x] = a;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *out = part[0] / (float)B;
}

// Adam (Kingma & Ba 2015) with bias correction; step t >= 1.
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m1,
                       float *__restrict__ m2, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    p[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// PCG32 (O'Neill 2014) for the seeded initialisation and batch shuffles.
struct Pcg {
    uint64_t s;
    uint32_t next()
    {
        const uint64_t old = s;
        s = old * 6364136223846793005ull + 1442695040888963407ull;
        const uint32_t xs = (uint32_t)(((old >> 18) ^ old) >> 27);
        const uint32_t rot = (uint32_t)(old >> 59);
        return (xs >> rot) | (xs << ((32u - rot) & 31u));
    }
    float uniform() { return (float)(next() >> 8) * (1.0f / 16777216.0f); }
};

}  // namespace

struct sp_mlp {
    cudaStream_t stream = nullptr;
    float *p = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    int cap = 0;  // rows the work buffers hold
    float *X = nullptr, *y = nullptr, *Z1 = nullptr, *H1 = nullptr, *Z2 = nullptr, *H2 = nullptr,
          *O = nullptr, *dO = nullptr, *dH2 = nullptr, *dH1 = nullptr, *rl = nullptr,
          *loss = nullptr, *pb = nullptr;
    long long t = 0;        // Adam steps taken
    long long launches = 0; // kernels launched
};

#define MK(x)                                                                      \
    do {                                                                           \
        cudaError_t e_ = (x);                                                      \
        if (e_ != cudaSuccess) {                                                   \
            sp_dev_note_error(#x, e_);                                             \
            return (e_ == cudaErrorMemoryAllocation) ? SP_EALLOC : SP_EINTERNAL;   \
        }                                                                          \
    } while (0)

static void mlp_free_work(sp_mlp *m)
{
    float *bufs[] = {m->X, m->y, m->Z1, m->H1, m->Z2, m->H2, m->O, m->dO, m->dH2, m->dH1, m->rl};
    for (float *b : bufs)
        if (b)
            sp_cuda_free(b);
    m->X = m->y = m->Z1 = m->H1 = m->Z2 = m->H2 = m->O = m->dO = m->dH2 = m->dH1 = m->rl =
        nullptr;
    m->cap = 0;
}

static int mlp_reserve(sp_mlp *m, int rows)
{
    if (rows <= m->cap)
        return SP_OK;
    mlp_free_work(m);
    const size_t r = (size_t)rows;
    MK(sp_cuda_malloc(&m->X, r * kIn * 4));
    MK(sp_cuda_malloc(&m->y, r * 4));
    MK(sp_cuda_malloc(&m->Z1, r * kHid * 4));
    MK(sp_cuda_malloc(&m->H1, r * kHid * 4));
    MK(sp_cuda_malloc(&m->Z2, r * kHid * 4));
    MK(sp_cuda_malloc(&m->H2, r * kHid * 4));
    MK(sp_cuda_malloc(&m->O, r * kOut * 4));
    MK(sp_cuda_malloc(&m->dO, r * kOut * 4));
    MK(sp_cuda_malloc(&m->dH2, r * kHid * 4));
    MK(sp_cuda_malloc(&m->dH1, r * kHid * 4));
    MK(sp_cuda_malloc(&m->rl, r * 4));
    m->cap = rows;
    return SP_OK;
}

template <int FORM>
static void gemm(sp_mlp *m, int M, int N, int K, const float *A, int lda, const float *B, int ldb,
                 float *C, int ldc, const float *bias, int epi, float *Zout, const float *Zin,
                 int ldz, int bf16, int round_out)
{
    dim3 grid((N + TILE - 1) / TILE, (M + TILE - 1) / TILE);
    k_gemm<FORM><<<grid, 256, 0, m->stream>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, epi, Zout,
                                               Zin, ldz, bf16, round_out);
    m->launches++;
}

// forward over rows [0, B) of m->X (params P), outputs in m->O
static void forward(sp_mlp *m, const float *P, int B, int bf16)
{
    gemm<0>(m, B, kHid, kIn, m->X, kIn, P + oW1, kIn, m->H1, kHid, P + ob1, EPI_BIAS_GELU, m->Z1,
            nullptr, kHid, bf16, bf16);
    gemm<0>(m, B, kHid, kHid, m->H1, kHid, P + oW2, kHid, m->H2, kHid, P + ob2, EPI_BIAS_GELU,
            m->Z2, nullptr, kHid, bf16, bf16);
    gemm<0>(m, B, kOut, kHid, m->H2, kHid, P + oW3, kHid, m->O, kOut, P + ob3, EPI_BIAS, nullptr,
            nullptr, 0, bf16, 0);
}

// loss and gradient (into m->g) for rows [0, B) of m->X / m->y
static void backward(sp_mlp *m, int B)
{
    const float *P = m->p;
    float *G = m->g;
    k_nll_grad<<<(B + 255) / 256, 256, 0, m->stream>>>(m->O, m->y, B, m->dO, m->rl);
    k_mean<<<1, 256, 0, m->stream>>>(m->rl, B, m->loss);
    m->launches += 2;
    // layer 3
    gemm<2>(m, kOut, kHid, B, m->dO, kOut, m->H2, kHid, G + oW3, kHid, nullptr, EPI_NONE, nullptr,
            nullptr, 0, 0, 0);
    k_colsum<<<1, 32, 0, m->stream>>>(m->dO, B, kOut, G + ob3);
    // dZ2 = (dO W3) * gelu'(Z2)
    gemm<1>(m, B, kHid, kOut, m->dO, kOut, P + oW3, kHid, m->dH2, kHid, nullptr, EPI_GELU_GRAD,
            nullptr, m->Z2, kHid, 0, 0);
    // layer 2
    gemm<2>(m, kHid, kHid, B, m->dH2, kHid, m->H1, kHid, G + oW2, kHid, nullptr, EPI_NONE, nullptr,
            nullptr, 0, 0, 0);
    k_colsum<<<1, kHid, 0, m->stream>>>(m->dH2, B, kHid, G + ob2);
    // dZ1 = (dZ2 W2) * gelu'(Z1)
    gemm<1>(m, B, kHid, kHid, m->dH2, kHid, P + oW2, kHid, m->dH1, kHid, nullptr, EPI_GELU_GRAD,
            nullptr, m->Z1, kHid, 0, 0);
    // layer 1
    gemm<2>(m, kHid, kIn, B, m->dH1, kHid, m->X, kIn, G + oW1, kIn, nullptr, EPI_NONE, nullptr,
            nullptr, 0, 0, 0);
    k_colsum<<<1, kHid, 0, m->stream>>>(m->dH1, B, kHid, G + ob1);
    m->launches += 3;
}

extern "C" int sp_mlp_num_params(void) { return kParams; }

extern "C" void sp_mlp_destroy(sp_mlp *m)
{
    if (!m)
        return;
    if (m->stream)
        cudaStreamSynchronize(m->stream);
    mlp_free_work(m);
    float *bufs[] = {m->p, m->g, m->m1, m->m2, m->loss, m->pb};
    for (float *b : bufs)
        if (b)
            sp_cuda_free(b);
    if (m->stream)
        cudaStreamDestroy(m->stream);
    delete m;
}

// Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases from PCG32.
extern "C" int sp_mlp_create(uint64_t seed, sp_mlp **out)
{
    *out = nullptr;
    sp_mlp *m = new sp_mlp();
    int rc = SP_OK;
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
        sp_cuda_malloc(&m->p, kParams * 4) != cudaSuccess || sp_cuda_malloc(&m->g, kParams * 4) != cudaSuccess ||
        sp_cuda_malloc(&m->m1, kParams * 4) != cudaSuccess ||
        sp_cuda_malloc(&m->m2, kParams * 4) != cudaSuccess || sp_cuda_malloc(&m->loss, 4) != cudaSuccess ||
        sp_cuda_malloc(&m->pb, kParams * 4) != cudaSuccess)
        rc = SP_EALLOC;
    if (!rc) {
        std::vector<float> h(kParams);
        Pcg r{seed * 2862933555777941757ull + 3037000493ull};
        auto fill = [&](int off, int cnt, int fan_in) {
            const float a = 1.0f / sqrtf((float)fan_in);
            for (int k = 0; k < cnt; ++k)
                h[off + k] = (2.0f * r.uniform() - 1.0f) * a;
        };
        fill(oW1, kP1, kIn);
        fill(ob1, kP1b, kIn);
        fill(oW2, kP2, kHid);
        fill(ob2, kP2b, kHid);
        fill(oW3, kP3, kHid);
        fill(ob3, kP3b, kHid);
        if (cudaMemcpy(m->p, h.data(), kParams * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(m->m1, 0, kParams * 4) != cudaSuccess ||
            cudaMemset(m->m2, 0, kParams * 4) != cudaSuccess)
            rc = SP_EINTERNAL;
    }
    if (rc) {
        cudaGetLastError();
        sp_mlp_destroy(m);
        return rc;
    }
    *out = m;
    return SP_OK;
}

extern "C" int sp_mlp_get_params(sp_mlp *m, float *h)
{
    MK(cudaMemcpy(h, m->p, kParams * 4, cudaMemcpyDeviceToHost));
    return SP_OK;
}

extern "C" int sp_mlp_set_params(sp_mlp *m, const float *h)
{
    MK(cudaMemcpy(m->p, h, kParams * 4, cudaMemcpyHostToDevice));
    MK(cudaMemset(m->m1, 0, kParams * 4));
    MK(cudaMemset(m->m2, 0, kParams * 4));
    m->t = 0;
    return SP_OK;
}

// Loss and gradient of the NLL over n host rows (FP32, no parameter change).
extern "C" int sp_mlp_loss_grad(sp_mlp *m, const float *X, const float *y, int n, float *loss,
                                float *grad)
{
    if (n <= 0)
        return SP_EINVAL;
    int rc = mlp_reserve(m, n);
    if (rc)
        return rc;
    MK(cudaMemcpyAsync(m->X, X, (size_t)n * kIn * 4, cudaMemcpyHostToDevice, m->stream));
    MK(cudaMemcpyAsync(m->y, y, (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    forward(m, m->p, n, 0);
    backward(m, n);
    MK(cudaGetLastError());
    MK(cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->stream));
    if (grad)
        MK(cudaMemcpyAsync(grad, m->g, kParams * 4, cudaMemcpyDeviceToHost, m->stream));
    MK(cudaStreamSynchronize(m->stream));
    return SP_OK;
}

// Adam on minibatches of a shuffled copy of the n rows, for `epochs` passes.
// The rows are uploaded once; each step gathers its minibatch on the host
// order (a permutation of row indices) into the front of the work buffers.
extern "C" int sp_mlp_train(sp_mlp *m, const float *X, const float *y, int n, int epochs,
                            int batch, float lr, uint64_t seed, float *final_loss)
{
    if (n <= 0 || epochs < 0 || batch <= 0)
        return SP_EINVAL;
    if (batch > n)
        batch = n;
    int rc = mlp_reserve(m, batch);
    if (rc)
        return rc;
    const size_t steps_per_epoch = (size_t)((n + batch - 1) / batch);
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i)
        perm[i] = i;
    std::vector<float> xb((size_t)batch * kIn), yb(batch);
    float *hx = nullptr, *hy = nullptr;
    MK(cudaMallocHost(&hx, steps_per_epoch * (size_t)batch * kIn * 4));
    MK(cudaMallocHost(&hy, steps_per_epoch * (size_t)batch * 4));
    Pcg r{seed ^ 0x5DEECE66Dull};
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs && !rc; ++ep) {
        // Fisher-Yates shuffle of the row order
        for (int i = n - 1; i > 0; --i) {
            const int j = (int)(r.next() % (uint32_t)(i + 1));
            const int t = perm[i];
            perm[i] = perm[j];
            perm[j] = t;
        }
        for (size_t st = 0; st < steps_per_epoch; ++st) {
            const int s0 = (int)(st * batch);
            const int B = (s0 + batch <= n) ? batch : n - s0;
            float *px = hx + st * (size_t)batch * kIn, *py = hy + st * (size_t)batch;
            for (int k = 0; k < B; ++k) {
                memcpy(px + (size_t)k * kIn, X + (size_t)perm[s0 + k] * kIn, kIn * 4);
                py[k] = y[perm[s0 + k]];
            }
            if (cudaMemcpyAsync(m->X, px, (size_t)B * kIn * 4, cudaMemcpyHostToDevice,
                                m->stream) != cudaSuccess ||
                cudaMemcpyAsync(m->y, py, (size_t)B * 4, cudaMemcpyHostToDevice, m->stream) !=
                    cudaSuccess) {
                rc = SP_EINTERNAL;
                break;
            }
            forward(m, m->p, B, 0);
            backward(m, B);
            m->t++;
            const float c1 = 1.0f - powf(b1, (float)m->t), c2 = 1.0f - powf(b2, (float)m->t);
            k_adam<<<(kParams + 255) / 256, 256, 0, m->stream>>>(m->p, m->g, m->m1, m->m2, kParams,
                                                                 lr, b1, b2, eps, c1, c2);
            m->launches++;
        }
        // the pinned staging of this epoch is reused by the next one
        if (cudaStreamSynchronize(m->stream) != cudaSuccess)
            rc = SP_EINTERNAL;
    }
    if (!rc && final_loss &&
        cudaMemcpy(final_loss, m->loss, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = SP_EINTERNAL;
    cudaStreamSynchronize(m->stream);
    cudaFreeHost(hx);
    cudaFreeHost(hy);
    if (cudaGetLastError() != cudaSuccess)
        rc = SP_EINTERNAL;
    return rc;
}

// Predicted (mean, log-variance) for n host rows; bf16 = 1 runs the BF16
// inference path (weights and activations rounded to BF16, products and sums
// in FP32 on the CUDA cores: a 10 -> 128 -> 128 -> 2 network is too small for
// tensor-core tiles to pay).
extern "C" int sp_mlp_predict(sp_mlp *m, const float *X, int n, int bf16, float *mean,
                              float *logvar)
{
    if (n <= 0)
        return SP_EINVAL;
    int rc = mlp_reserve(m, n);
    if (rc)
        return rc;
    MK(cudaMemcpyAsync(m->X, X, (size_t)n * kIn * 4, cudaMemcpyHostToDevice, m->stream));
    forward(m, m->p, n, bf16);
    MK(cudaGetLastError());
    std::vector<float> o((size_t)n * kOut);
    MK(cudaMemcpyAsync(o.data(), m->O, (size_t)n * kOut * 4, cudaMemcpyDeviceToHost, m->stream));
    MK(cudaStreamSynchronize(m->stream));
    for (int s = 0; s < n; ++s) {
        if (mean)
            mean[s] = o[2 * s];
        if (logvar)
            logvar[s] = o[2 * s + 1];
    }
    return SP_OK;
}

extern "C" long long sp_mlp_launches(const sp_mlp *m) { return m->launches; }
