// Training and evaluation kernels of the learned eddy-viscosity closure (lbm_closure.cuh).
//
// The network is tiny (1441 trained parameters) and the samples many, so training is a stream
// over samples: each block keeps the parameters in shared memory, runs forward and backward for
// one sample per thread, parks the per-sample vectors the weight gradient needs in shared memory,
// and then accumulates the outer products of a chunk of samples into per-thread gradient
// entries.  Block partial gradients are summed in a fixed order by a second kernel (FP64), so the
// gradient is deterministic.  Adam updates the parameters in place.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "../../include/lbm_b200.h"
#include "lbm_closure.cuh"
#include "lbm_dispatch.h"

using namespace lbm;

struct LbmMlp {
    int device;
    int max_blocks;
    float* partial;      // [max_blocks][MLP_TRAINED]
    double* loss_part;   // [max_blocks]
};

namespace {

constexpr int CHUNK = 128;                              // samples per block iteration (= threads)
constexpr int REC = MLP_IN + 4 * MLP_H + 1;             // x, h1, dz1, h2, dz2, dy per sample
static_assert(REC == 139, "per-sample record");

// Features from the per-sample state (SoA [10][n]: Pxx Pyy Pzz Pxy Pxz Pyz rho ux uy uz).
__global__ void __launch_bounds__(256) k_closure_features(const float* __restrict__ state, long long n,
                                                         float* __restrict__ feats) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        float v[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) v[k] = state[k * n + s];
        float x[MLP_IN];
        closure_features<float>(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9], x);
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) feats[k * n + s] = x[k];
    }
}

// Evaluation: one sample per thread, first-layer activations parked in shared memory (the same
// summation order as closure_nu_t).
__global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ params, const float* __restrict__ feats,
                                                    long long n, float* __restrict__ nu) {
    __shared__ float w[MLP_PARAMS];
    __shared__ float hs[MLP_H][128 + 1];
    for (int i = threadIdx.x; i < MLP_PARAMS; i += blockDim.x) w[i] = params[i];
    __syncthreads();
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        float x[MLP_IN];
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) x[k] = feats[k * n + s];
#pragma unroll 1
        for (int k = 0; k < MLP_H; ++k) {
            float z = w[MLP_B1 + k];
#pragma unroll
            for (int i = 0; i < MLP_IN; ++i) z += x[i] * w[MLP_W1 + i * MLP_H + k];
            hs[k][threadIdx.x] = mlp_silu<float>(z);
        }
        float y = w[MLP_B3];
#pragma unroll 1
        for (int k = 0; k < MLP_H; ++k) {
            float z = w[MLP_B2 + k];
#pragma unroll 8
            for (int j = 0; j < MLP_H; ++j) z += hs[j][threadIdx.x] * w[MLP_W2 + j * MLP_H + k];
            y += mlp_silu<float>(z) * w[MLP_W3 + k];
        }
        nu[s] = w[MLP_SCALE] * mlp_softplus<float>(y);
    }
}

// Forward + backward of one chunk of samples per iteration; gradient entries accumulated per
// thread over the block's chunks (entry e = threadIdx.x + k * CHUNK).
__global__ void __launch_bounds__(CHUNK) k_mlp_grad_partial(const float* __restrict__ params,
                                                           const float* __restrict__ feats,
                                                           const float* __restrict__ target,
                                                           const float* __restrict__ weight, long long n,
                                                           float inv_wsum, float* __restrict__ partial,
                                                           double* __restrict__ loss_part) {
    extern __shared__ float sm[];
    float* w = sm;                         // MLP_PARAMS
    float* rec = sm + MLP_PARAMS + 2;      // CHUNK * REC (offset keeps 8-byte alignment)
    for (int i = threadIdx.x; i < MLP_PARAMS; i += blockDim.x) w[i] = params[i];
    constexpr int PER = (MLP_TRAINED + CHUNK - 1) / CHUNK;
    float acc[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) acc[k] = 0.f;
    double loss = 0.0;
    const float scale = params[MLP_SCALE];
    __syncthreads();
    const long long nchunks = (n + CHUNK - 1) / CHUNK;
    for (long long c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const long long s = c * CHUNK + threadIdx.x;
        float* r = rec + threadIdx.x * REC;
        float* rx = r;
        float* rh1 = r + MLP_IN;
        float* rdz1 = rh1 + MLP_H;
        float* rh2 = rdz1 + MLP_H;
        float* rdz2 = rh2 + MLP_H;
        float* rdy = rdz2 + MLP_H;
        if (s < n) {
            float x[MLP_IN];
#pragma unroll
            for (int k = 0; k < MLP_IN; ++k) x[k] = rx[k] = feats[k * n + s];
            float z1[MLP_H];
#pragma unroll
            for (int k = 0; k < MLP_H; ++k) {
                float z = w[MLP_B1 + k];
#pragma unroll
                for (int i = 0; i < MLP_IN; ++i) z += x[i] * w[MLP_W1 + i * MLP_H + k];
                z1[k] = z;
                rh1[k] = mlp_silu<float>(z);
            }
            float y = w[MLP_B3];
            for (int k = 0; k < MLP_H; ++k) {
                float z = w[MLP_B2 + k];
#pragma unroll 8
                for (int j = 0; j < MLP_H; ++j) z += rh1[j] * w[MLP_W2 + j * MLP_H + k];
                rdz2[k] = z;                                   // z2, turned into dz2 below
                const float h2 = mlp_silu<float>(z);
                rh2[k] = h2;
                y += h2 * w[MLP_W3 + k];
            }
            const float nu = scale * mlp_softplus<float>(y);
            const float wt = weight ? weight[s] : 1.f;
            const float res = nu - target[s];
            loss += (double)wt * res * res * inv_wsum;
            const float dy = 2.f * wt * res * inv_wsum * scale * (y > 20.f ? 1.f : mlp_sigmoid<float>(y));
            rdy[0] = dy;
            for (int k = 0; k < MLP_H; ++k) {
                const float z = rdz2[k];
                const float sg = mlp_sigmoid<float>(z);
                rdz2[k] = dy * w[MLP_W3 + k] * sg * (1.f + z * (1.f - sg));
            }
#pragma unroll
            for (int j = 0; j < MLP_H; ++j) {
                float d = 0.f;
#pragma unroll 8
                for (int k = 0; k < MLP_H; ++k) d += rdz2[k] * w[MLP_W2 + j * MLP_H + k];
                const float z = z1[j];
                const float sg = mlp_sigmoid<float>(z);
                rdz1[j] = d * sg * (1.f + z * (1.f - sg));
            }
        } else {
            for (int k = 0; k < REC; ++k) r[k] = 0.f;
        }
        __syncthreads();
        // weight gradient entries of this thread, summed over the chunk
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int e = threadIdx.x + k * CHUNK;
            if (e >= MLP_TRAINED) break;
            int ao, bo;       // record offsets of the two factors (ao < 0: factor 1)
            if (e < MLP_B1) { ao = e / MLP_H; bo = MLP_IN + MLP_H + e % MLP_H; }                    // x_i dz1_k
            else if (e < MLP_W2) { ao = -1; bo = MLP_IN + MLP_H + (e - MLP_B1); }                  // dz1_k
            else if (e < MLP_B2) { const int q = e - MLP_W2; ao = MLP_IN + q / MLP_H; bo = MLP_IN + 3 * MLP_H + q % MLP_H; }
            else if (e < MLP_W3) { ao = -1; bo = MLP_IN + 3 * MLP_H + (e - MLP_B2); }              // dz2_k
            else if (e < MLP_B3) { ao = MLP_IN + 2 * MLP_H + (e - MLP_W3); bo = MLP_IN + 4 * MLP_H; }  // h2_k dy
            else { ao = -1; bo = MLP_IN + 4 * MLP_H; }                                             // dy
            float g = 0.f;
            if (ao >= 0) {
                for (int t = 0; t < CHUNK; ++t) g += rec[t * REC + ao] * rec[t * REC + bo];
            } else {
                for (int t = 0; t < CHUNK; ++t) g += rec[t * REC + bo];
            }
            acc[k] += g;
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = threadIdx.x + k * CHUNK;
        if (e < MLP_TRAINED) partial[(long long)blockIdx.x * MLP_TRAINED + e] = acc[k];
    }
    // block loss: fixed-order tree in shared memory
    __shared__ double red[CHUNK];
    red[threadIdx.x] = loss;
    __syncthreads();
    for (int h = CHUNK / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_part[blockIdx.x] = red[0];
}

__global__ void k_mlp_grad_finish(const float* __restrict__ partial, const double* __restrict__ loss_part,
                                  int blocks, float* __restrict__ grad, double* __restrict__ loss) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < MLP_TRAINED) {
        double s = 0.0;
        for (int b = 0; b < blocks; ++b) s += partial[(long long)b * MLP_TRAINED + e];
        grad[e] = (float)s;
    } else if (e == MLP_TRAINED) {
        grad[e] = 0.f;                    // the output scale is not trained
        if (loss) {
            double s = 0.0;
            for (int b = 0; b < blocks; ++b) s += loss_part[b];
            *loss = s;
        }
    }
}

__global__ void k_mlp_adam(const float* __restrict__ grad, float* __restrict__ params, float* __restrict__ m,
                           float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= MLP_TRAINED) return;
    const float g = grad[e];
    const float mm = b1 * m[e] + (1.f - b1) * g;
    const float vv = b2 * v[e] + (1.f - b2) * g * g;
    m[e] = mm;
    v[e] = vv;
    params[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

int device_ptr_ok(const void* p, bool nullable) {
    if (p == nullptr) return nullable ? 0 : 1;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) ? 0 : 1;
}

int grid_for(long long n, int threads) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long b = (n + threads - 1) / threads;
    const long long cap = (long long)sms * 8;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

extern "C" {

int lbm_closure_features(const float* state, int64_t n, float* feats, void* stream) {
    if (n < 1) return abi_fail(LBM_E_INVALID, "n must be positive");
    if (device_ptr_ok(state, false) || device_ptr_ok(feats, false))
        return abi_fail(LBM_E_INVALID, "state and feats must be device pointers");
    k_closure_features<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(state, n, feats);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LBM_OK : abi_fail(LBM_E_CUDA, "closure features: %s", cudaGetErrorString(e));
}

int lbm_mlp_forward(const float* params, const float* feats, int64_t n, float* nu, void* stream) {
    if (n < 1) return abi_fail(LBM_E_INVALID, "n must be positive");
    if (device_ptr_ok(params, false) || device_ptr_ok(feats, false) || device_ptr_ok(nu, false))
        return abi_fail(LBM_E_INVALID, "params, feats and nu must be device pointers");
    k_mlp_forward<<<grid_for(n, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(params, feats, n, nu);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LBM_OK : abi_fail(LBM_E_CUDA, "mlp forward: %s", cudaGetErrorString(e));
}

int lbm_mlp_create(int max_blocks, LbmMlp** out) {
    if (out == nullptr || max_blocks < 1) return abi_fail(LBM_E_INVALID, "out must not be NULL, max_blocks >= 1");
    *out = nullptr;
    LbmMlp* m = new LbmMlp();
    cudaGetDevice(&m->device);
    m->max_blocks = max_blocks;
    m->partial = nullptr;
    m->loss_part = nullptr;
    cudaError_t e = cudaMalloc(&m->partial, sizeof(float) * MLP_TRAINED * (size_t)max_blocks);
    if (e == cudaSuccess) e = cudaMalloc(&m->loss_part, sizeof(double) * (size_t)max_blocks);
    if (e == cudaSuccess) {
        const int smem = (MLP_PARAMS + 2 + CHUNK * REC) * (int)sizeof(float);
        e = cudaFuncSetAttribute(k_mlp_grad_partial, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    }
    if (e != cudaSuccess) {
        cudaFree(m->partial);
        cudaFree(m->loss_part);
        delete m;
        return abi_fail(LBM_E_CUDA, "lbm_mlp_create: %s", cudaGetErrorString(e));
    }
    *out = m;
    return LBM_OK;
}

int lbm_mlp_destroy(LbmMlp* m) {
    if (m == nullptr) return LBM_OK;
    cudaFree(m->partial);
    cudaFree(m->loss_part);
    delete m;
    return LBM_OK;
}

int lbm_mlp_loss_grad(LbmMlp* m, const float* params, const float* feats, const float* target, const float* weight,
                      int64_t n, double inv_wsum, float* grad, double* loss, void* stream) {
    if (m == nullptr) return abi_fail(LBM_E_INVALID, "trainer is NULL");
    if (n < 1) return abi_fail(LBM_E_INVALID, "n must be positive");
    if (device_ptr_ok(params, false) || device_ptr_ok(feats, false) || device_ptr_ok(target, false) ||
        device_ptr_ok(weight, true) || device_ptr_ok(grad, false) || device_ptr_ok(loss, true))
        return abi_fail(LBM_E_INVALID, "params, feats, target, weight, grad and loss must be device pointers");
    const long long chunks = (n + CHUNK - 1) / CHUNK;
    const int blocks = (int)(chunks < m->max_blocks ? chunks : m->max_blocks);
    const int smem = (MLP_PARAMS + 2 + CHUNK * REC) * (int)sizeof(float);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_mlp_grad_partial<<<blocks, CHUNK, smem, s>>>(params, feats, target, weight, n, (float)inv_wsum, m->partial,
                                                   m->loss_part);
    k_mlp_grad_finish<<<(MLP_PARAMS + 255) / 256, 256, 0, s>>>(m->partial, m->loss_part, blocks, grad, loss);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LBM_OK : abi_fail(LBM_E_CUDA, "mlp loss/grad: %s", cudaGetErrorString(e));
}

int lbm_mlp_adam(const float* grad, float* params, float* m1, float* m2, double lr, double beta1, double beta2,
                 double eps, int step, void* stream) {
    if (step < 1) return abi_fail(LBM_E_INVALID, "Adam steps count from 1");
    if (device_ptr_ok(grad, false) || device_ptr_ok(params, false) || device_ptr_ok(m1, false) ||
        device_ptr_ok(m2, false))
        return abi_fail(LBM_E_INVALID, "grad, params and the moment buffers must be device pointers");
    const float c1 = (float)(1.0 - pow(beta1, step)), c2 = (float)(1.0 - pow(beta2, step));
    k_mlp_adam<<<(MLP_TRAINED + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        grad, params, m1, m2, (float)lr, (float)beta1, (float)beta2, (float)eps, c1, c2);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LBM_OK : abi_fail(LBM_E_CUDA, "mlp adam: %s", cudaGetErrorString(e));
}

}  // extern "C"
