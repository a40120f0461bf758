// Learned HSEX surrogate: a multilayer perceptron trained on the GPU by its
// own forward and backward kernels (no reference counterpart).
//
// Network: n_in -> H -> H -> H -> n_out, GELU after each hidden layer, linear
// output.  Weights are kept in FP32 (the optimiser's master copy) and in BF16
// (what the tensor cores multiply); activations are FP32 and are rounded to
// BF16 as the operand of the next product; every product accumulates in FP32
// in tensor memory (tcgen05.mma kind::f16, 128 x 128 tiles).  Loss: mean squared error over the
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
// C[M][N] (+)= op(A)[M][K] op(B)[K][N] on the 5th-generation tensor cores
// (tcgen05.mma kind::f16, BF16 operands, FP32 accumulator in tensor memory).
// A(i, k) = A[i * a_rs + k * a_cs], B(k, j) = B[k * b_rs + j * b_cs] (BF16), so
// a transposed operand is only a change of strides.
//
// A CTA of 4 warps owns a 128 x 128 tile of C, accumulated in 128 TMEM columns
// (lane = row, column = output column).  K runs in chunks of 64: the 128 threads
// gather A's 128 x 64 and B's 64 x 128 chunk from global memory (strided,
// out-of-range rows, columns and K read as zero) into shared memory in the
// K-major, non-swizzled layout of the tensor-core operand descriptors: 8 rows x
// 16 bytes per core matrix, core matrices of one 8-row group contiguous along K
// (leading byte offset 128 B), 8-row groups 1024 B apart (stride byte offset).
// One thread issues the chunk's four 128 x 128 x 16 MMAs and commits them to an
// mbarrier, which every thread waits on (bounded) before the next chunk
// overwrites the operands.  Epilogue: each warp reads its 32 TMEM lanes
// (tcgen05.ld 32x32b, 8 columns at a time), adds the bias, writes C.
constexpr int UM = 128, UN = 128, UK = 64;
constexpr int TM = UM, TN = UN;
// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N, M
constexpr unsigned kUmmaIdesc =
    (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(UN >> 3) << 17) | ((unsigned)(UM >> 4) << 24);

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// shared-memory operand descriptor (K-major, no swizzle, descriptor version 1)
__device__ __forceinline__ unsigned long long umma_desc(const void* p) {
    return (unsigned long long)((smem_addr(p) >> 4) & 0x3FFFu) | ((unsigned long long)(128u >> 4) << 16) |
           ((unsigned long long)(1024u >> 4) << 32) | (1ull << 46);
}

// element offset of (row r, k) of a 64-wide K chunk in the core-matrix layout
__device__ __forceinline__ int umma_off(int r, int k) { return (r >> 3) * 512 + (k >> 3) * 64 + (r & 7) * 8 + (k & 7); }

__device__ __forceinline__ bool mbar_wait_parity(unsigned long long* bar, unsigned parity, int limit) {
    for (int i = 0; i < limit; ++i) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__global__ void __launch_bounds__(128) gemm_bf16_kernel(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                       long long a_rs, long long a_cs,
                                                       const __nv_bfloat16* __restrict__ B, long long b_rs,
                                                       long long b_cs, float* __restrict__ C, int ldc,
                                                       const float* __restrict__ bias, int accumulate,
                                                       int* __restrict__ status) {
    __shared__ __align__(1024) __nv_bfloat16 As[UM * UK];  // 16 KB
    __shared__ __align__(1024) __nv_bfloat16 Bs[UN * UK];  // 16 KB
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ unsigned tmem_slot;
    const int m0 = blockIdx.y * UM, n0 = blockIdx.x * UN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(&tmem_slot)),
                     "r"(UN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(&mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const unsigned tmem = tmem_slot;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    unsigned phase = 0;
    bool ok = true;
    for (int k0 = 0; k0 < K; k0 += UK) {
        for (int e = threadIdx.x; e < UM * UK; e += blockDim.x) {
            const int r = e / UK, k = e - (e / UK) * UK;
            const int gi = m0 + r, gk = k0 + k;
            As[umma_off(r, k)] = (gi < M && gk < K) ? A[gi * a_rs + gk * a_cs] : zero;
        }
        for (int e = threadIdx.x; e < UN * UK; e += blockDim.x) {
            const int c = e / UK, k = e - (e / UK) * UK;
            const int gj = n0 + c, gk = k0 + k;
            Bs[umma_off(c, k)] = (gj < N && gk < K) ? B[gk * b_rs + gj * b_cs] : zero;
        }
        // the operands were written by the generic proxy; the tensor core reads them by the async proxy
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
            for (int st = 0; st < UK / 16; ++st) {
                const unsigned long long da = umma_desc(As + st * 128);  // two core matrices = 16 of K
                const unsigned long long db = umma_desc(Bs + st * 128);
                const unsigned accum = (k0 > 0 || st > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(kUmmaIdesc), "r"(accum)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_addr(&mbar))
                         : "memory");
        }
        // the MMAs have read the operands (and written TMEM) once the phase completes
        if (!mbar_wait_parity(&mbar, phase, 1 << 24)) {
            // give up: report, wait (bounded again) for the MMAs in flight, skip the rest
            ok = false;
            mbar_wait_parity(&mbar, phase, 1 << 24);
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        if (__syncthreads_or(!ok)) {
            ok = false;
            break;
        }
    }
    if (!ok && threadIdx.x == 0 && status) atomicOr(status, 1);
    // epilogue: TMEM lanes 32 warp .. 32 warp + 31 are this warp's rows
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < (ok ? UN : 0); c0 += 8) {
        unsigned v[8];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
            : "r"(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (row < M) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int col = n0 + c0 + j;
                if (col < N) {
                    float x = __uint_as_float(v[j]);
                    if (bias) x += bias[col];
                    float* dst = C + (long long)row * ldc + col;
                    *dst = accumulate ? *dst + x : x;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(UN) : "memory");
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
    int* status = nullptr;  // set when a GEMM's bounded wait for its tensor-core MMAs ran out
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

// After a synchronisation: report (and clear) a GEMM wait that ran out.
int mlp_status(edus_mlp* m) {
    int v = 0;
    MCU(m, cudaMemcpy(&v, m->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (v) {
        MCU(m, cudaMemset(m->status, 0, sizeof(int)));
        return mfail(m, EDUS_ERR_TIMEOUT, "a bounded wait for the tensor-core MMAs of a GEMM ran out");
    }
    return EDUS_OK;
}

void gemm(edus_mlp* mm, int M, int N, int K, const __nv_bfloat16* A, long long a_rs, long long a_cs,
          const __nv_bfloat16* B, long long b_rs, long long b_cs, float* C, int ldc, const float* bias) {
    dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
    gemm_bf16_kernel<<<grid, 128, 0, mm->stream>>>(M, N, K, A, a_rs, a_cs, B, b_rs, b_cs, C, ldc, bias, 0,
                                                   mm->status);
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
        cudaMalloc((void**)&m->loss, sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&m->status, sizeof(int)) != cudaSuccess ||
        cudaMemset(m->status, 0, sizeof(int)) != cudaSuccess) {
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
    cudaFree(m->status);
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
    return mlp_status(m);
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
    return mlp_status(m);
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
        return mlp_status(m);
    }
    return EDUS_OK;
}

}  // extern "C"
