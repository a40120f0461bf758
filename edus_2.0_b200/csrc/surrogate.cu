// Learned HSEX surrogate: a multilayer perceptron trained on the GPU by its
// own forward and backward kernels (no reference counterpart).
//
// Network: n_in -> H -> H -> H -> n_out, GELU after each hidden layer, linear
// output.  Weights are kept in FP32 (the optimiser's master copy) and in BF16
// (what the tensor cores multiply); activations are FP32 and are rounded to
// BF16 as the operand of the next product; every product accumulates in FP32
// (mma.sync.m16n8k16.f32.bf16.bf16.f32).  Loss: mean squared error over the
// batch and the outputs.  Optimiser: Adam.
//
// Layouts: a batch of B samples is row-major [B][features]; a weight matrix is
// row-major [in][out].  All batch buffers passed to the entry points are
// device pointers.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/edus_gpu.h"

namespace {

constexpr int kLayers = 4;  // three hidden layers and the output layer

// ---------------------------------------------------------------------------
// C[M][N] (+)= op(A)[M][K] op(B)[K][N], FP32 accumulate.  A(i, k) =
// A[i * a_rs + k * a_cs], B(k, j) = B[k * b_rs + j * b_cs] (BF16), so a
// transposed operand is only a change of strides.  Tiles of 64 x 64 with K
// steps of 16, four warps of 32 x 32 (2 x 4 m16n8 fragments).  Out-of-range
// rows, columns and K are read as zero and not written.
constexpr int TM = 64, TN = 64, TKK = 16;

__device__ __forceinline__ unsigned pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    const unsigned short l = *reinterpret_cast<unsigned short*>(&lo);
    const unsigned short h = *reinterpret_cast<unsigned short*>(&hi);
    return (unsigned)l | ((unsigned)h << 16);
}

__global__ void __launch_bounds__(128) gemm_bf16_kernel(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                       long long a_rs, long long a_cs,
                                                       const __nv_bfloat16* __restrict__ B, long long b_rs,
                                                       long long b_cs, float* __restrict__ C, int ldc,
                                                       const float* __restrict__ bias, int accumulate) {
    __shared__ __nv_bfloat16 As[TM][TKK + 8];  // [row][k], padded
    __shared__ __nv_bfloat16 Bs[TN][TKK + 8];  // [col][k], padded
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int g = lane >> 2, tg = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int k0 = 0; k0 < K; k0 += TKK) {
        for (int e = threadIdx.x; e < TM * TKK; e += blockDim.x) {
            const int r = e / TKK, k = e - (e / TKK) * TKK;
            const int gi = m0 + r, gk = k0 + k;
            As[r][k] = (gi < M && gk < K) ? A[gi * a_rs + gk * a_cs] : zero;
        }
        for (int e = threadIdx.x; e < TN * TKK; e += blockDim.x) {
            const int c = e / TKK, k = e - (e / TKK) * TKK;
            const int gj = n0 + c, gk = k0 + k;
            Bs[c][k] = (gj < N && gk < K) ? B[gk * b_rs + gj * b_cs] : zero;
        }
        __syncthreads();
        unsigned af[2][4], bfr[4][2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = wm + i * 16 + g;
            af[i][0] = pack_bf16(As[r][tg * 2], As[r][tg * 2 + 1]);
            af[i][1] = pack_bf16(As[r + 8][tg * 2], As[r + 8][tg * 2 + 1]);
            af[i][2] = pack_bf16(As[r][tg * 2 + 8], As[r][tg * 2 + 9]);
            af[i][3] = pack_bf16(As[r + 8][tg * 2 + 8], As[r + 8][tg * 2 + 9]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = wn + j * 8 + g;
            bfr[j][0] = pack_bf16(Bs[c][tg * 2], Bs[c][tg * 2 + 1]);
            bfr[j][1] = pack_bf16(Bs[c][tg * 2 + 8], Bs[c][tg * 2 + 9]);
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                    "{%0,%1,%2,%3};\n"
                    : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
                    : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]), "r"(bfr[j][0]), "r"(bfr[j][1]));
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int row = m0 + wm + i * 16 + g + (r >= 2 ? 8 : 0);
                const int col = n0 + wn + j * 8 + tg * 2 + (r & 1);
                if (row < M && col < N) {
                    float v = acc[i][j][r];
                    if (bias) v += bias[col];
                    float* dst = C + (long long)row * ldc + col;
                    *dst = accumulate ? *dst + v : v;
                }
            }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

// a = GELU(z) (FP32) and its BF16 copy
__global__ void gelu_kernel(const float* __restrict__ z, float* __restrict__ a, __nv_bfloat16* __restrict__ ab,
                            long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float v = gelu(z[i]);
        a[i] = v;
        ab[i] = __float2bfloat16(v);
    }
}
__global__ void to_bf16_kernel(const float* __restrict__ x, __nv_bfloat16* __restrict__ xb, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        xb[i] = __float2bfloat16(x[i]);
}
// dz = da * GELU'(z), and its BF16 copy
__global__ void gelu_back_kernel(const float* __restrict__ da, const float* __restrict__ z, float* __restrict__ dz,
                                 __nv_bfloat16* __restrict__ dzb, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float v = da[i] * gelu_grad(z[i]);
        dz[i] = v;
        dzb[i] = __float2bfloat16(v);
    }
}
// dy = 2 (y - t) / n_total, and the loss (mean of squares; one atomic per block)
__global__ void mse_kernel(const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ dy,
                           __nv_bfloat16* __restrict__ dyb, long long n, float scale, float* __restrict__ loss) {
    __shared__ float red[256];
    float s = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float d = y[i] - t[i];
        s += d * d;
        const float g = 2.f * d * scale;
        dy[i] = g;
        dyb[i] = __float2bfloat16(g);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0] * scale);
}
// db[j] = sum_i dz[i][j]
__global__ void colsum_kernel(const float* __restrict__ dz, float* __restrict__ db, int rows, int cols) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    float s = 0.f;
    for (int i = 0; i < rows; ++i) s += dz[(long long)i * cols + j];
    db[j] = s;
}
// Adam on the FP32 master weights, refreshing their BF16 copy
__global__ void adam_kernel(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, long long n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        wb[i] = __float2bfloat16(wi);
    }
}

int grid1(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 8); }

}  // namespace

struct edus_mlp {
    int dims[kLayers + 1] = {0};  // n_in, H, H, H, n_out
    int device = 0;
    std::string err;
    long long nparams = 0;
    float* params = nullptr;      // FP32 master: W0 b0 W1 b1 W2 b2 W3 b3
    float* grads = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    __nv_bfloat16* wbf = nullptr;  // BF16 copy (same offsets as params)
    long long woff[kLayers] = {0}, boff[kLayers] = {0};
    int step = 0;
    // activations for a batch of up to `cap` samples
    int cap = 0;
    float* z[kLayers] = {nullptr};  // pre-activations [B][dims[l+1]]
    float* a[kLayers] = {nullptr};  // GELU of the hidden pre-activations
    __nv_bfloat16* ab[kLayers + 1] = {nullptr};  // BF16 operands: ab[0] = x, ab[l] = a[l-1]
    float* da = nullptr;
    float* dz = nullptr;
    __nv_bfloat16* dzb = nullptr;
    float* loss = nullptr;
    cudaStream_t stream = nullptr;
};

namespace {

thread_local std::string g_mlp_create_error;

int mfail(edus_mlp* m, int code, const std::string& msg) {
    if (m) m->err = msg;
    else g_mlp_create_error = msg;
    return code;
}
#define MCU(m, call)                                                                                              \
    do {                                                                                                          \
        cudaError_t e_ = (call);                                                                                  \
        if (e_ != cudaSuccess) return mfail(m, EDUS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void gemm(edus_mlp* mm, int M, int N, int K, const __nv_bfloat16* A, long long a_rs, long long a_cs,
          const __nv_bfloat16* B, long long b_rs, long long b_cs, float* C, int ldc, const float* bias) {
    dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
    gemm_bf16_kernel<<<grid, 128, 0, mm->stream>>>(M, N, K, A, a_rs, a_cs, B, b_rs, b_cs, C, ldc, bias, 0);
}

int ensure_cap(edus_mlp* m, int B) {
    if (B <= m->cap) return EDUS_OK;
    for (int l = 0; l < kLayers; ++l) {
        cudaFree(m->z[l]);
        cudaFree(m->a[l]);
        m->z[l] = m->a[l] = nullptr;
    }
    for (int l = 0; l <= kLayers; ++l) {
        cudaFree(m->ab[l]);
        m->ab[l] = nullptr;
    }
    cudaFree(m->da);
    cudaFree(m->dz);
    cudaFree(m->dzb);
    m->da = m->dz = nullptr;
    m->dzb = nullptr;
    m->cap = 0;
    int wmax = 0;
    for (int l = 0; l <= kLayers; ++l) wmax = std::max(wmax, m->dims[l]);
    for (int l = 0; l < kLayers; ++l) {
        MCU(m, cudaMalloc((void**)&m->z[l], (size_t)B * m->dims[l + 1] * sizeof(float)));
        MCU(m, cudaMalloc((void**)&m->a[l], (size_t)B * m->dims[l + 1] * sizeof(float)));
    }
    for (int l = 0; l <= kLayers; ++l)
        MCU(m, cudaMalloc((void**)&m->ab[l], (size_t)B * m->dims[l] * sizeof(__nv_bfloat16)));
    MCU(m, cudaMalloc((void**)&m->da, (size_t)B * wmax * sizeof(float)));
    MCU(m, cudaMalloc((void**)&m->dz, (size_t)B * wmax * sizeof(float)));
    MCU(m, cudaMalloc((void**)&m->dzb, (size_t)B * wmax * sizeof(__nv_bfloat16)));
    m->cap = B;
    return EDUS_OK;
}

// forward pass of B samples x (device FP32 [B][n_in]); output in z[kLayers-1]
void forward(edus_mlp* m, int B, const float* x) {
    to_bf16_kernel<<<grid1((long long)B * m->dims[0]), 256, 0, m->stream>>>(x, m->ab[0], (long long)B * m->dims[0]);
    for (int l = 0; l < kLayers; ++l) {
        const int in = m->dims[l], out = m->dims[l + 1];
        gemm(m, B, out, in, m->ab[l], in, 1, m->wbf + m->woff[l], out, 1, m->z[l], out, m->params + m->boff[l]);
        if (l < kLayers - 1)
            gelu_kernel<<<grid1((long long)B * out), 256, 0, m->stream>>>(m->z[l], m->a[l], m->ab[l + 1],
                                                                          (long long)B * out);
    }
}

// gradients of the mean squared error into m->grads (the loss into m->loss)
void backward(edus_mlp* m, int B, const float* target) {
    const int nout = m->dims[kLayers];
    const long long n = (long long)B * nout;
    cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream);
    mse_kernel<<<grid1(n), 256, 0, m->stream>>>(m->z[kLayers - 1], target, m->dz, m->dzb, n, 1.f / (float)n, m->loss);
    for (int l = kLayers - 1; l >= 0; --l) {
        const int in = m->dims[l], out = m->dims[l + 1];
        // dW = a_{l-1}^T dz : [in][B] x [B][out]
        gemm(m, in, out, B, m->ab[l], 1, in, m->dzb, out, 1, m->grads + m->woff[l], out, nullptr);
        colsum_kernel<<<(out + 127) / 128, 128, 0, m->stream>>>(m->dz, m->grads + m->boff[l], B, out);
        if (l == 0) break;
        // da_{l-1} = dz W^T : [B][out] x [out][in]
        gemm(m, B, in, out, m->dzb, out, 1, m->wbf + m->woff[l], 1, out, m->da, in, nullptr);
        gelu_back_kernel<<<grid1((long long)B * in), 256, 0, m->stream>>>(m->da, m->z[l - 1], m->dz, m->dzb,
                                                                          (long long)B * in);
    }
}

}  // namespace

extern "C" {

int edus_mlp_create(int n_in, int n_hidden, int n_out, unsigned long long seed, int device, edus_mlp** out) {
    if (!out || n_in < 1 || n_hidden < 1 || n_out < 1) return mfail(nullptr, EDUS_ERR_ARG, "bad MLP sizes");
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return mfail(nullptr, EDUS_ERR_CUDA, "cudaSetDevice failed");
    edus_mlp* m = new edus_mlp();
    m->device = device;
    m->dims[0] = n_in;
    for (int l = 1; l < kLayers; ++l) m->dims[l] = n_hidden;
    m->dims[kLayers] = n_out;
    long long off = 0;
    for (int l = 0; l < kLayers; ++l) {
        m->woff[l] = off;
        off += (long long)m->dims[l] * m->dims[l + 1];
        m->boff[l] = off;
        off += m->dims[l + 1];
    }
    m->nparams = off;
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc((void**)&m->params, off * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&m->grads, off * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&m->m, off * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&m->v, off * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&m->wbf, off * sizeof(__nv_bfloat16)) != cudaSuccess ||
        cudaMalloc((void**)&m->loss, sizeof(float)) != cudaSuccess) {
        edus_mlp_destroy(m);
        return mfail(nullptr, EDUS_ERR_NOMEM, "MLP device allocation failed");
    }
    // uniform initialisation scaled by the fan-in (seeded LCG), zero biases
    std::vector<float> p(off, 0.f);
    unsigned long long s = seed * 6364136223846793005ULL + 1442695040888963407ULL;
    auto uni = [&]() {
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        return ((s >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
    };
    for (int l = 0; l < kLayers; ++l) {
        const double a = std::sqrt(3.0 / m->dims[l]) * (l < kLayers - 1 ? std::sqrt(2.0) : 1.0);
        for (long long i = 0; i < (long long)m->dims[l] * m->dims[l + 1]; ++i) p[m->woff[l] + i] = (float)(a * uni());
    }
    const int rc = edus_mlp_set_params(m, p.data());
    if (rc) {
        g_mlp_create_error = m->err;
        edus_mlp_destroy(m);
        return rc;
    }
    *out = m;
    return EDUS_OK;
}

int edus_mlp_destroy(edus_mlp* m) {
    if (!m) return EDUS_OK;
    if (m->stream) cudaStreamSynchronize(m->stream);
    cudaFree(m->params);
    cudaFree(m->grads);
    cudaFree(m->m);
    cudaFree(m->v);
    cudaFree(m->wbf);
    cudaFree(m->loss);
    for (int l = 0; l < kLayers; ++l) {
        cudaFree(m->z[l]);
        cudaFree(m->a[l]);
    }
    for (int l = 0; l <= kLayers; ++l) cudaFree(m->ab[l]);
    cudaFree(m->da);
    cudaFree(m->dz);
    cudaFree(m->dzb);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return EDUS_OK;
}

const char* edus_mlp_last_error(const edus_mlp* m) { return m ? m->err.c_str() : g_mlp_create_error.c_str(); }

long long edus_mlp_param_count(const edus_mlp* m) { return m ? m->nparams : 0; }

int edus_mlp_set_params(edus_mlp* m, const float* host) {
    if (!m || !host) return EDUS_ERR_ARG;
    MCU(m, cudaSetDevice(m->device));
    MCU(m, cudaMemcpyAsync(m->params, host, m->nparams * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    to_bf16_kernel<<<grid1(m->nparams), 256, 0, m->stream>>>(m->params, m->wbf, m->nparams);
    MCU(m, cudaMemsetAsync(m->m, 0, m->nparams * sizeof(float), m->stream));
    MCU(m, cudaMemsetAsync(m->v, 0, m->nparams * sizeof(float), m->stream));
    m->step = 0;
    MCU(m, cudaStreamSynchronize(m->stream));
    return EDUS_OK;
}

int edus_mlp_get_params(edus_mlp* m, float* host) {
    if (!m || !host) return EDUS_ERR_ARG;
    MCU(m, cudaSetDevice(m->device));
    MCU(m, cudaMemcpyAsync(host, m->params, m->nparams * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCU(m, cudaStreamSynchronize(m->stream));
    return EDUS_OK;
}

int edus_mlp_forward(edus_mlp* m, int batch, const float* x, float* y) {
    if (!m || !x || !y || batch < 1) return EDUS_ERR_ARG;
    MCU(m, cudaSetDevice(m->device));
    int rc;
    if ((rc = ensure_cap(m, batch))) return rc;
    forward(m, batch, x);
    MCU(m, cudaMemcpyAsync(y, m->z[kLayers - 1], (size_t)batch * m->dims[kLayers] * sizeof(float),
                           cudaMemcpyDeviceToDevice, m->stream));
    MCU(m, cudaGetLastError());
    MCU(m, cudaStreamSynchronize(m->stream));
    return EDUS_OK;
}

int edus_mlp_gradients(edus_mlp* m, int batch, const float* x, const float* target, float* grads_host,
                       float* loss_host) {
    if (!m || !x || !target || batch < 1) return EDUS_ERR_ARG;
    MCU(m, cudaSetDevice(m->device));
    int rc;
    if ((rc = ensure_cap(m, batch))) return rc;
    forward(m, batch, x);
    backward(m, batch, target);
    MCU(m, cudaGetLastError());
    if (grads_host)
        MCU(m, cudaMemcpyAsync(grads_host, m->grads, m->nparams * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    if (loss_host) MCU(m, cudaMemcpyAsync(loss_host, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCU(m, cudaStreamSynchronize(m->stream));
    return EDUS_OK;
}

int edus_mlp_train_step(edus_mlp* m, int batch, const float* x, const float* target, float lr, float* loss_host) {
    if (!m || !x || !target || batch < 1 || !(lr > 0.f)) return EDUS_ERR_ARG;
    MCU(m, cudaSetDevice(m->device));
    int rc;
    if ((rc = ensure_cap(m, batch))) return rc;
    forward(m, batch, x);
    backward(m, batch, target);
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    adam_kernel<<<grid1(m->nparams), 256, 0, m->stream>>>(m->params, m->wbf, m->grads, m->m, m->v, m->nparams, lr, b1,
                                                          b2, 1e-8f, c1, c2);
    MCU(m, cudaGetLastError());
    if (loss_host) {
        MCU(m, cudaMemcpyAsync(loss_host, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
        MCU(m, cudaStreamSynchronize(m->stream));
    }
    return EDUS_OK;
}

}  // extern "C"
