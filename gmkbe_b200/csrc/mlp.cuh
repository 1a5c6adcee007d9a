// Subtree-size model for the learned schedule: a 16-64-64-1 perceptron with
// ReLU hidden layers, FP16 weights and inputs, FP32 accumulation, trained on
// the GPU by the kernels below (forward, backward, Adam).  Target: log1p of a
// root task's search-tree nodes.  The model only orders the roots (largest
// predicted first); it never prunes, so the result set does not depend on it.
//
// Parameter layout (FP32 master copy and FP16 working copy alike):
//   W1[64][16] b1[64] W2[64][64] b2[64] W3[64] b3
// Features per root x (root_features_kernel), each log1p-scaled:
//   0 k, 1 depth (0 for a root task), 2 deg x, 3 |V| - deg x,
//   4 candidate U count (ids > x), 5 exclusion count (ids < x),
//   6 sum deg y over N(x) (2-hop size with repeats), 7 max deg y, 8 min deg y,
//   9 mean deg y, 10 |V|, 11 |U|, 12 sum over y of |N(y) above x|,
//   13 sum over y of |N(y) below x|, 14 #y with deg y <= k + 1,
//   15 log2 bucket of deg x.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>

#include "enum_core.cuh"

namespace gmk {
namespace mlp {

constexpr int F = 16;
constexpr int H = 64;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + H * F;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + H;
constexpr int NP = OFF_B3 + 1;   // 5313 parameters
constexpr int kBlock = 128;

// One warp per root: the 16 features of root task x.
__global__ void root_features_kernel(GraphView g, uint32_t k, __half* out) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t x = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (x >= g.nl) return;
    const uint32_t d = degree(g, (uint32_t)x);
    const uint32_t* row = g.adj + g.off[x];
    unsigned long long sum = 0, above = 0, below = 0, small = 0, words = 0;
    uint32_t mx = 0, mn = 0xFFFFFFFFu;
    for (uint32_t i = lane; i < d; i += 32) {
        const uint32_t y = row[i];
        const uint32_t dy = degree(g, y);
        sum += dy;
        mx = dy > mx ? dy : mx;
        mn = dy < mn ? dy : mn;
        small += dy <= k + 1 ? 1u : 0u;
        const uint32_t a = count_above(g, y, (uint32_t)x, &words);
        above += a;
        below += dy - a - 1;   // y's neighbours below x (x itself excluded)
    }
    for (int o = 16; o; o >>= 1) {
        sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
        above += __shfl_xor_sync(0xFFFFFFFFu, above, o);
        below += __shfl_xor_sync(0xFFFFFFFFu, below, o);
        small += __shfl_xor_sync(0xFFFFFFFFu, small, o);
        const uint32_t a = __shfl_xor_sync(0xFFFFFFFFu, mx, o);
        const uint32_t b = __shfl_xor_sync(0xFFFFFFFFu, mn, o);
        mx = a > mx ? a : mx;
        mn = b < mn ? b : mn;
    }
    if (lane != 0) return;
    const uint32_t nv = g.n - g.nl;
    float f[F];
    f[0] = (float)k;
    f[1] = 0.f;
    f[2] = (float)d;
    f[3] = (float)(nv - d);
    f[4] = (float)(g.nl - 1 - x);
    f[5] = (float)x;
    f[6] = (float)sum;
    f[7] = (float)mx;
    f[8] = d ? (float)mn : 0.f;
    f[9] = d ? (float)sum / (float)d : 0.f;
    f[10] = (float)nv;
    f[11] = (float)g.nl;
    f[12] = (float)above;
    f[13] = (float)below;
    f[14] = (float)small;
    f[15] = (float)(32 - __clz(d | 1u));
    for (int i = 0; i < F; ++i) out[x * F + i] = __float2half_rn(log1pf(f[i]));
}

__device__ __forceinline__ void stage_weights(const __half* w, __half* sw) {
    for (int i = threadIdx.x; i < NP; i += blockDim.x) sw[i] = w[i];
    __syncthreads();
}

// Forward pass, one thread per sample.  act (optional): h1, h2 per sample
// (2H floats) for the backward pass.
__global__ void __launch_bounds__(kBlock) forward_kernel(const __half* w, const __half* x,
                                                         uint32_t n, float* act, float* out) {
    __shared__ __half sw[NP];
    stage_weights(w, sw);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float xin[F];
    for (int f = 0; f < F; ++f) xin[f] = __half2float(x[(uint64_t)i * F + f]);
    float h1[H];
    for (int j = 0; j < H; ++j) {
        float a = __half2float(sw[OFF_B1 + j]);
        for (int f = 0; f < F; ++f) a = fmaf(__half2float(sw[OFF_W1 + j * F + f]), xin[f], a);
        h1[j] = a > 0.f ? a : 0.f;
    }
    float o = __half2float(sw[OFF_B3]);
    for (int j = 0; j < H; ++j) {
        float a = __half2float(sw[OFF_B2 + j]);
        for (int q = 0; q < H; ++q) a = fmaf(__half2float(sw[OFF_W2 + j * H + q]), h1[q], a);
        const float h2 = a > 0.f ? a : 0.f;
        if (act) act[(uint64_t)i * 2 * H + H + j] = h2;
        o = fmaf(__half2float(sw[OFF_W3 + j]), h2, o);
    }
    if (act)
        for (int j = 0; j < H; ++j) act[(uint64_t)i * 2 * H + j] = h1[j];
    out[i] = o;
}

// Backward pass of the mean squared error, one thread per sample; weight
// gradients are summed per block in shared memory, then added to grad.
__global__ void __launch_bounds__(kBlock) backward_kernel(const __half* w, const __half* x,
                                                          const float* y, const float* act,
                                                          const float* out, uint32_t n,
                                                          float* grad, float* loss) {
    __shared__ __half sw[NP];
    __shared__ float sg[NP];
    for (int p = threadIdx.x; p < NP; p += blockDim.x) sg[p] = 0.f;
    stage_weights(w, sw);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const float* h1 = act + (uint64_t)i * 2 * H;
        const float* h2 = h1 + H;
        const float e = out[i] - y[i];
        atomicAdd(loss, e * e / (float)n);
        const float dout = 2.f * e / (float)n;
        atomicAdd(&sg[OFF_B3], dout);
        float dh2[H];
        for (int j = 0; j < H; ++j) {
            const float a = h2[j];
            atomicAdd(&sg[OFF_W3 + j], dout * a);
            dh2[j] = a > 0.f ? dout * __half2float(sw[OFF_W3 + j]) : 0.f;
            if (dh2[j] != 0.f) atomicAdd(&sg[OFF_B2 + j], dh2[j]);
        }
        float xin[F];
        for (int f = 0; f < F; ++f) xin[f] = __half2float(x[(uint64_t)i * F + f]);
        for (int q = 0; q < H; ++q) {
            const float a = h1[q];
            float s = 0.f;
            for (int j = 0; j < H; ++j) {
                if (dh2[j] == 0.f) continue;
                if (a != 0.f) atomicAdd(&sg[OFF_W2 + j * H + q], dh2[j] * a);
                s = fmaf(__half2float(sw[OFF_W2 + j * H + q]), dh2[j], s);
            }
            const float dh1 = a > 0.f ? s : 0.f;
            if (dh1 != 0.f) {
                atomicAdd(&sg[OFF_B1 + q], dh1);
                for (int f = 0; f < F; ++f) atomicAdd(&sg[OFF_W1 + q * F + f], dh1 * xin[f]);
            }
        }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < NP; p += blockDim.x)
        if (sg[p] != 0.f) atomicAdd(&grad[p], sg[p]);
}

// Adam step on the FP32 master weights; refreshes the FP16 copy.
__global__ void adam_kernel(float* master, __half* w, const float* grad, float* m, float* v,
                            float lr, float b1, float b2, float eps, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    const float g = grad[p];
    const float mm = b1 * m[p] + (1.f - b1) * g;
    const float vv = b2 * v[p] + (1.f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    const float upd = lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    master[p] -= upd;
    w[p] = __float2half_rn(master[p]);
}

__global__ void to_half_kernel(const float* master, __half* w) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < NP) w[p] = __float2half_rn(master[p]);
}

__global__ void float_to_half_kernel(const float* in, __half* out, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __float2half_rn(in[i]);
}

}  // namespace mlp
}  // namespace gmk
