// cnn.cuh — periodic 3x3 convolutional network of the learned subgrid closure.
//
// Network: L layers of 3x3 convolutions with periodic padding; layer 0 maps the 3 input
// channels (filtered vorticity, u, w) to C channels, layers 1..L-2 map C -> C, the last maps
// C -> 1 (the subgrid forcing); GELU(x) = x Phi(x) after every layer but the last.
// Activations are [B][C][H][W] float; weights [Co][Ci][3][3] then bias [Co], layer after
// layer, in one flat parameter vector.  Forward, backward (data and weight gradients) and Adam
// are hand-written kernels; all reductions are in fixed order (deterministic).
#pragma once
#include <cuda_runtime.h>

namespace dns2d {
namespace cnn {

constexpr int TILE = 16;  // output tile edge (pixels)
constexpr int COT = 8;    // output channels per CTA

// y[b][co][y][x] = bias[co] + sum_ci sum_{ky,kx} w[co][ci][ky][kx] x[b][ci][(y+ky-1)%H][(x+kx-1)%W]
// grid (ceil(W/16), ceil(H/16), B * ceil(Co/8)), block 16 x 16.
__global__ void k_conv3x3(const float *__restrict__ x, const float *__restrict__ w, const float *__restrict__ bias,
                          float *__restrict__ y, int B, int Ci, int Co, int H, int W)
{
    extern __shared__ float sm[];
    float *tin = sm;                             // [Ci][18][18]
    float *tw = sm + (size_t)Ci * (TILE + 2) * (TILE + 2);  // [COT][Ci][9]
    const int ncot = (Co + COT - 1) / COT;
    const int b = blockIdx.z / ncot, cot = blockIdx.z % ncot;
    const int x0 = blockIdx.x * TILE, y0 = blockIdx.y * TILE;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TILE + tx;
    const float *xb = x + (size_t)b * Ci * H * W;
    for (int e = tid; e < Ci * (TILE + 2) * (TILE + 2); e += TILE * TILE) {
        const int ci = e / ((TILE + 2) * (TILE + 2));
        const int r = e % ((TILE + 2) * (TILE + 2));
        const int yy = (y0 + r / (TILE + 2) - 1 + H) % H;
        const int xx = (x0 + r % (TILE + 2) - 1 + W) % W;
        tin[e] = xb[((size_t)ci * H + yy) * W + xx];
    }
    for (int e = tid; e < COT * Ci * 9; e += TILE * TILE) {
        const int c = e / (Ci * 9);
        const int co = cot * COT + c;
        tw[e] = (co < Co) ? w[(size_t)co * Ci * 9 + e % (Ci * 9)] : 0.0f;
    }
    __syncthreads();
    float acc[COT];
#pragma unroll
    for (int c = 0; c < COT; ++c) {
        const int co = cot * COT + c;
        acc[c] = (co < Co) ? bias[co] : 0.0f;
    }
    for (int ci = 0; ci < Ci; ++ci) {
        const float *t = tin + (size_t)ci * (TILE + 2) * (TILE + 2);
        float v[9];
#pragma unroll
        for (int ky = 0; ky < 3; ++ky)
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) v[ky * 3 + kx] = t[(ty + ky) * (TILE + 2) + tx + kx];
#pragma unroll
        for (int c = 0; c < COT; ++c) {
            const float *wc = tw + ((size_t)c * Ci + ci) * 9;
#pragma unroll
            for (int k = 0; k < 9; ++k) acc[c] = fmaf(wc[k], v[k], acc[c]);
        }
    }
    const int ox = x0 + tx, oy = y0 + ty;
    if (ox < W && oy < H) {
#pragma unroll
        for (int c = 0; c < COT; ++c) {
            const int co = cot * COT + c;
            if (co < Co) y[(((size_t)b * Co + co) * H + oy) * W + ox] = acc[c];
        }
    }
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z)
{
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__global__ void k_gelu(const float *__restrict__ z, float *__restrict__ a, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        a[i] = gelu(z[i]);
}

// da -> dz = da * GELU'(z), in place on da
__global__ void k_gelu_back(const float *__restrict__ z, float *__restrict__ g, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        g[i] *= gelu_grad(z[i]);
}

// weights of the data-gradient convolution: wt[ci][co][ky][kx] = w[co][ci][2-ky][2-kx]
__global__ void k_flip_weights(const float *__restrict__ w, float *__restrict__ wt, int Ci, int Co)
{
    const int n = Ci * Co * 9;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int ci = e / (Co * 9), r = e % (Co * 9), co = r / 9, k = r % 9;
        wt[e] = w[((size_t)co * Ci + ci) * 9 + (8 - k)];
    }
}

// dw[co][ci][ky][kx] = sum_{b,y,x} dy[b][co][y][x] x[b][ci][y+ky-1][x+kx-1], db[co] = sum dy
// grid (Ci, Co), block 256; fixed-order block reduction.
__global__ void k_conv3x3_wgrad(const float *__restrict__ x, const float *__restrict__ dy, float *__restrict__ dw,
                                float *__restrict__ db, int B, int Ci, int Co, int H, int W)
{
    __shared__ float red[10][256];
    const int ci = blockIdx.x, co = blockIdx.y;
    float acc[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) acc[k] = 0.0f;
    const size_t npix = (size_t)B * H * W;
    for (size_t p = threadIdx.x; p < npix; p += blockDim.x) {
        const int b = (int)(p / ((size_t)H * W));
        const int r = (int)(p % ((size_t)H * W));
        const int yy = r / W, xx = r % W;
        const float g = dy[(((size_t)b * Co + co) * H + yy) * W + xx];
        const float *xc = x + ((size_t)b * Ci + ci) * H * W;
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
            const int sy = (yy + ky - 1 + H) % H;
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
                const int sx = (xx + kx - 1 + W) % W;
                acc[ky * 3 + kx] = fmaf(g, xc[(size_t)sy * W + sx], acc[ky * 3 + kx]);
            }
        }
        acc[9] += g;
    }
#pragma unroll
    for (int k = 0; k < 10; ++k) red[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
#pragma unroll
            for (int k = 0; k < 10; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < 9) dw[((size_t)co * Ci + ci) * 9 + threadIdx.x] = red[threadIdx.x][0];
    if (threadIdx.x == 9 && ci == 0) db[co] = red[9][0];
}

// mean squared error over n values and its gradient 2 (p - t) / n; per-block partial losses
__global__ void k_mse(const float *__restrict__ pred, const float *__restrict__ tgt, float *__restrict__ grad,
                      double *__restrict__ part, size_t n)
{
    __shared__ double red[256];
    double acc = 0.0;
    const float sc = 2.0f / (float)n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float d = pred[i] - tgt[i];
        grad[i] = sc * d;
        acc += (double)d * d;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Adam (bias-corrected) on the flat parameter vector
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

}  // namespace cnn
}  // namespace dns2d
