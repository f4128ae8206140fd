// hbg_surrogate.cu -- the learned part of the mixed form: an MLP surrogate of the regular part of the
// infinite-depth wave term of the Green function, trained on the device by this file's own forward
// and backward kernels on samples of the library's own table and series evaluation, and evaluated on
// the 5th-generation tensor cores (tcgen05.mma kind::f16, BF16 operands, FP32 accumulators in TMEM).
//
// What it learns.  For X = K R in [0, 100) and Y = -K (z + zeta) in [0, 50) the wave term is
// (green_inf.rs:316-368)
//     F  = S + g,   S = -2 e^-Y J0(X) (log(Y + R0) + gamma - log 2),   R0 = sqrt(X^2 + Y^2),
// S holding the logarithmic singularity at R0 = 0 in closed form.  The network maps the inputs
// (u, v, w) = (2 log1p(X) / log 101 - 1, 2 log1p(Y) / log 51 - 1, 0) to six outputs: g, dg/dX, dg/dY
// (the regular real part and its radial and vertical derivatives) and I, dI/dX, dI/dY (the imaginary
// part -2 pi e^-Y J0(X) and its derivatives), each standardized by its mean and spread over the
// training set.  The third input stays 0: the term replaced is the same function at every depth (in
// finite depth it enters the kernel as F(K R, K v3), green_fin.rs:1051-1071, the depth-dependent parts
// being the per-frequency tiles), so a K h input would carry nothing.  Architecture 3 -> 128 -> 128 ->
// 128 -> 128 -> 6, SiLU, weights rounded to BF16 in the forward pass (FP32 master copy and Adam
// moments), activations rounded to BF16 between layers, FP32 accumulation.  Outside the domain the
// table/series evaluation is used.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "hbg_tc.cuh"

#include <cmath>
#include <vector>

namespace hbg {

constexpr int SG_IN = 3, SG_H = 128, SG_OUT = 6;
// parameter layout (FP32): W0 [H][IN], b0 [H], W1..W3 [H][H], b1..b3 [H], W4 [OUT][H], b4 [OUT]
constexpr int SG_OFF_W0 = 0, SG_OFF_B0 = SG_OFF_W0 + SG_H * SG_IN;
constexpr int SG_OFF_W1 = SG_OFF_B0 + SG_H;
constexpr int SG_LAYER_HH = SG_H * SG_H + SG_H;  // W and b of a hidden layer
constexpr int SG_OFF_W4 = SG_OFF_W1 + 3 * SG_LAYER_HH, SG_OFF_B4 = SG_OFF_W4 + SG_OUT * SG_H;
constexpr int SG_PARAMS = SG_OFF_B4 + SG_OUT;  // 50,822
// the trained domain: X = K R in [0, 100), Y = -K (z + zeta) in [0, 50)
constexpr double SG_XMAX = 100.0, SG_YMAX = 50.0;
static_assert(SURROGATE_FLOATS == SG_PARAMS + 2 * SG_OUT, "parameters then means and spreads");

__host__ __device__ inline int sg_off_w(int l) { return l == 0 ? SG_OFF_W0 : l < 4 ? SG_OFF_W1 + (l - 1) * SG_LAYER_HH : SG_OFF_W4; }
__host__ __device__ inline int sg_off_b(int l) {
    return l == 0 ? SG_OFF_B0 : l < 4 ? SG_OFF_W1 + (l - 1) * SG_LAYER_HH + SG_H * SG_H : SG_OFF_B4;
}
__host__ __device__ inline int sg_fan_in(int l) { return l == 0 ? SG_IN : SG_H; }
__host__ __device__ inline int sg_fan_out(int l) { return l == 4 ? SG_OUT : SG_H; }

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }
__device__ __forceinline__ float silu_d(float z) {
    const float s = 1.f / (1.f + __expf(-z));
    return s * (1.f + z * (1.f - s));
}

__device__ __forceinline__ void sg_inputs(double X, double Y, float* in) {
    in[0] = (float)(2.0 * log1p(X) / log1p(SG_XMAX) - 1.0);
    in[1] = (float)(2.0 * log1p(Y) / log1p(SG_YMAX) - 1.0);
    in[2] = 0.f;  // the replaced term has no depth dependence (see the header)
}

// The six targets at (X, Y) from the table evaluation (FP64).
__device__ void sg_targets(double X, double Y, double* t) {
    const Wave w = wave_kernel<false>(X, Y);
    double j0, j1;
    bessel_j01<false>(X, j0, j1);
    const double eY = exp(-Y), R0 = sqrt(X * X + Y * Y);
    const double lg = log(Y + R0) + (GAMMA - LOG2);
    const double S = -2.0 * eY * j0 * lg;
    const double SX = 2.0 * eY * j1 * lg - 2.0 * eY * j0 * X / (R0 * (Y + R0));
    const double SY = 2.0 * eY * j0 * lg - 2.0 * eY * j0 / R0;
    t[0] = w.F - S;
    t[1] = w.FX - SX;
    t[2] = w.FY - SY;
    t[3] = w.I;
    t[4] = w.IX;
    t[5] = w.IY;
}

// Radical inverse in base b (Halton sequence), index i >= 1.
__device__ __forceinline__ double halton(uint64_t i, int b) {
    double f = 1.0, r = 0.0;
    while (i > 0) {
        f /= b;
        r += f * (double)(i % b);
        i /= b;
    }
    return r;
}

// Samples i0 + 1 .. i0 + n of the 2-D Halton sequence, log-spaced over the domain:
// X = 101^u - 1, Y = 51^v - 1; inputs [n][3] (FP32) and FP64 targets [n][6].
__global__ void k_sg_samples(int n, uint64_t i0, float* __restrict__ in, double* __restrict__ tg,
                             double* __restrict__ xy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t h = i0 + (uint64_t)i + 1;
    const double X = expm1(halton(h, 2) * log1p(SG_XMAX)), Y = expm1(halton(h, 3) * log1p(SG_YMAX));
    sg_inputs(X, Y, in + 3 * (size_t)i);
    sg_targets(X, Y, tg + 6 * (size_t)i);
    if (xy) {
        xy[2 * (size_t)i] = X;
        xy[2 * (size_t)i + 1] = Y;
    }
}

// Targets at given points (FP64), for evaluation against the network.
__global__ void k_sg_table(int n, const double* __restrict__ xy, double* __restrict__ tg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    sg_targets(xy[2 * (size_t)i], xy[2 * (size_t)i + 1], tg + 6 * (size_t)i);
}

__global__ void k_sg_inputs(int n, const double* __restrict__ xy, float* __restrict__ in) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    sg_inputs(xy[2 * (size_t)i], xy[2 * (size_t)i + 1], in + 3 * (size_t)i);
}

// ---------------------------------------------------------------- training kernels (SIMT, FP32)
// C[m][n] (+)= sum_k A(m, k) B(k, n) with general strides: A(m, k) = A[m sam + k sak],
// B(k, n) = B[k sbk + n sbn], C[m ldc + n]; 64 x 64 tiles, 16-deep k chunks in shared memory,
// 4 x 4 outputs a thread.  beta 0 overwrites, 1 accumulates.
__global__ void __launch_bounds__(256) k_sg_gemm(int M, int N, int K, const float* __restrict__ A, int sam, int sak,
                                                 const float* __restrict__ B, int sbk, int sbn, float* __restrict__ C,
                                                 int ldc, int beta) {
    __shared__ float As[16][64 + 4], Bs[16][64 + 4];
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int t = threadIdx.x; t < 16 * 64; t += 256) {
            const int kk = t / 64, mm = t % 64;
            const int m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < M && k < K) ? A[(size_t)m * sam + (size_t)k * sak] : 0.f;
            const int n = n0 + mm;
            Bs[kk][mm] = (n < N && k < K) ? B[(size_t)k * sbk + (size_t)n * sbn] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                a[i] = As[kk][ty * 4 + i];
                b[i] = Bs[kk][tx * 4 + i];
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] += a[i] * b[j];
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
            if (m < M && n < N) {
                float* c = C + (size_t)m * ldc + n;
                *c = beta ? *c + acc[i][j] : acc[i][j];
            }
        }
}

static void sg_gemm(int M, int N, int K, const float* A, int sam, int sak, const float* B, int sbk, int sbn, float* C,
                    int ldc, int beta, cudaStream_t s) {
    dim3 g((N + 63) / 64, (M + 63) / 64);
    k_sg_gemm<<<g, 256, 0, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, beta);
}

// Z [B][n] += bias; H = bf16(silu(Z)) (act) or H = Z (the output layer).
__global__ void k_sg_bias_act(int Bn, int n, const float* __restrict__ bias, float* __restrict__ Z,
                              float* __restrict__ H, int act) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)Bn * n) return;
    const float z = Z[t] + bias[t % n];
    Z[t] = z;
    H[t] = act ? bf16r(silu(z)) : z;
}

__global__ void k_sg_round(int n, const float* __restrict__ a, float* __restrict__ b) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) b[t] = bf16r(a[t]);
}

// dOut = 2 (Out - T) / (B OUT); loss partial sums (sum of squares) per block into part[blockIdx.x].
__global__ void k_sg_loss(int Bn, const float* __restrict__ out, const float* __restrict__ tg,
                          float* __restrict__ dout, float* __restrict__ part) {
    __shared__ float sh[256];
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    float e = 0.f;
    if (t < (size_t)Bn * SG_OUT) {
        const float d = out[t] - tg[t];
        dout[t] = 2.f * d / (float)(Bn * SG_OUT);
        e = d * d;
    }
    sh[threadIdx.x] = e;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// dZ = dH * silu'(Z)
__global__ void k_sg_dact(size_t n, const float* __restrict__ Z, float* __restrict__ dH) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) dH[t] *= silu_d(Z[t]);
}

// db[j] = sum over the batch of dZ[b][j] (one thread per j, fixed order).
__global__ void k_sg_colsum(int Bn, int n, const float* __restrict__ dZ, float* __restrict__ db) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    float s = 0.f;
    for (int b = 0; b < Bn; b++) s += dZ[(size_t)b * n + j];
    db[j] = s;
}

__global__ void k_sg_adam(int n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, float lr, float b1, float b2, float c1, float c2) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float gt = g[t];
    const float mt = b1 * m[t] + (1.f - b1) * gt, vt = b2 * v[t] + (1.f - b2) * gt * gt;
    m[t] = mt;
    v[t] = vt;
    p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + 1e-8f);
}

// Training state on the device: master parameters, their BF16-rounded copy, gradients, moments and
// the activations of one batch.
struct SgTrainer {
    int Bn = 0;
    float *p = nullptr, *pr = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    float *Z[5] = {}, *H[5] = {}, *dH = nullptr, *dH2 = nullptr, *part = nullptr;
    std::vector<void*> owned;
    bool alloc(int batch) {
        Bn = batch;
        auto get = [&](size_t bytes) -> float* {
            void* q = nullptr;
            if (cudaMalloc(&q, bytes) != cudaSuccess) return nullptr;
            owned.push_back(q);  // only successful allocations are counted
            return static_cast<float*>(q);
        };
        p = get(SG_PARAMS * 4);
        pr = get(SG_PARAMS * 4);
        g = get(SG_PARAMS * 4);
        m = get(SG_PARAMS * 4);
        v = get(SG_PARAMS * 4);
        for (int l = 0; l < 5; l++) {
            Z[l] = get((size_t)Bn * SG_H * 4);
            H[l] = get((size_t)Bn * SG_H * 4);
        }
        dH = get((size_t)Bn * SG_H * 4);
        dH2 = get((size_t)Bn * SG_H * 4);
        part = get(((size_t)Bn * SG_OUT + 255) / 256 * 4);
        return owned.size() == 18;
    }
    ~SgTrainer() {
        for (void* q : owned) cudaFree(q);
    }
    // forward of inputs X0 [Bn][3] (already BF16-rounded) with the rounded parameters pr
    void forward(const float* X0, int n, cudaStream_t s) {
        const float* in = X0;
        for (int l = 0; l < 5; l++) {
            const int fi = sg_fan_in(l), fo = sg_fan_out(l);
            // Z = in W^T : A = in (n x fi), B(k, j) = W[j][k]
            sg_gemm(n, fo, fi, in, fi, 1, pr + sg_off_w(l), 1, fi, Z[l], fo, 0, s);
            k_sg_bias_act<<<(unsigned)(((size_t)n * fo + 255) / 256), 256, 0, s>>>(n, fo, pr + sg_off_b(l), Z[l], H[l],
                                                                                  l < 4);
            in = H[l];
        }
    }
    // gradients of the mean squared error against targets T [n][6] into g; loss partials in part
    void backward(const float* X0, const float* T, int n, cudaStream_t s) {
        const int nb = (int)(((size_t)n * SG_OUT + 255) / 256);
        k_sg_loss<<<nb, 256, 0, s>>>(n, H[4], T, dH, part);
        float* d = dH;   // dZ of the current layer [n][fo]
        float* o = dH2;  // dH of the layer below
        for (int l = 4; l >= 0; l--) {
            const int fi = sg_fan_in(l), fo = sg_fan_out(l);
            const float* in = l > 0 ? H[l - 1] : X0;
            // dW = dZ^T in : (fo x fi) = sum_b dZ[b][j] in[b][k]
            sg_gemm(fo, fi, n, d, 1, fo, in, fi, 1, g + sg_off_w(l), fi, 0, s);
            k_sg_colsum<<<(fo + 127) / 128, 128, 0, s>>>(n, fo, d, g + sg_off_b(l));
            if (l > 0) {
                // dH_below = dZ W : (n x fi) = sum_j dZ[b][j] W[j][k]
                sg_gemm(n, fi, fo, d, fo, 1, pr + sg_off_w(l), fi, 1, o, fi, 0, s);
                k_sg_dact<<<(unsigned)(((size_t)n * fi + 255) / 256), 256, 0, s>>>((size_t)n * fi, Z[l - 1], o);
                float* t = d;
                d = o;
                o = t;
            }
        }
    }
};

// ---------------------------------------------------------------- inference on the tensor cores
// 5th-generation tensor cores: a CTA of 256 threads evaluates 256 samples a pass as two 128-row tiles.
// Layer 0 (3 -> 128) on the CUDA cores; each hidden layer is, per tile, eight tcgen05.mma of
// kind::f16 (BF16 operands, M 128, N 128, K 16) from shared memory into a TMEM accumulator (FP32);
// thread r of a tile reads its row back (tcgen05.ld), adds the bias, applies SiLU, rounds to BF16
// and writes the row into the shared A tile of the next layer; the output layer is one more MMA
// (N 16, six used).  Operands are K-major in the 128-byte swizzle layout: rows of 128 bytes (64
// BF16 of K), 16-byte units XOR-ed with the row index mod 8, two K halves 16 KB apart per tile.
//
// The packed weight image, copied whole into each persistent CTA's shared memory: W1..W3 as B
// operands [128 rows j][K 128] (32 KB each), W4 [16 rows, 6 used][K 128] (4 KB), then FP32: W0
// [128][3], biases b0..b3 [4][128] and b4 [8] (BF16-rounded values), output means and spreads [12].
constexpr int SG_TILE_BYTES = SG_H * SG_H * 2;  // one 128 x 128 BF16 operand
constexpr size_t SG_IMG_W4 = 3 * (size_t)SG_TILE_BYTES;
constexpr size_t SG_IMG_F = SG_IMG_W4 + 16 * SG_H * 2;
constexpr int SG_F_W0 = 0, SG_F_B = SG_H * SG_IN, SG_F_N = SG_F_B + 4 * SG_H + 8;
constexpr size_t SG_IMG_BYTES = (SG_IMG_F + (size_t)(SG_F_N + 2 * SG_OUT) * 4 + 1023) / 1024 * 1024;
// dynamic shared memory of a network CTA: alignment slack, the image, two A tiles, the mbarrier
constexpr size_t SG_TC_SMEM = 1024 + SG_IMG_BYTES + 2 * (size_t)SG_TILE_BYTES + 16;
constexpr uint32_t SG_TMEM_COLS = 512;  // accumulators: tiles at columns 0 and 128, outputs at 256 and 288

// byte offset of element (row, k) in a K-major 128-byte-swizzled operand of `rows` rows, K = 128
__host__ __device__ constexpr size_t sg_sw_off(int rows, int row, int k) {
    return (size_t)(k / 64) * rows * 128 + (size_t)row * 128 + (size_t)((((k % 64) / 8) ^ (row & 7)) * 16) + (k % 8) * 2;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
}

__host__ __device__ constexpr uint32_t sg_idesc_bf16(int M, int N) {
    return (1u << 4)      // D format F32
           | (1u << 7)    // A format BF16
           | (1u << 10)   // B format BF16
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__global__ void k_sg_pack(const float* __restrict__ params, const float* __restrict__ norm, uint8_t* __restrict__ img) {
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    for (int t = t0; t < 3 * SG_H * SG_H; t += st) {
        const int l = t / (SG_H * SG_H), j = (t / SG_H) % SG_H, k = t % SG_H;
        *reinterpret_cast<__nv_bfloat16*>(img + (size_t)l * SG_TILE_BYTES + sg_sw_off(SG_H, j, k)) =
            __float2bfloat16_rn(params[sg_off_w(l + 1) + j * SG_H + k]);
    }
    for (int t = t0; t < 16 * SG_H; t += st) {
        const int j = t / SG_H, k = t % SG_H;
        *reinterpret_cast<__nv_bfloat16*>(img + SG_IMG_W4 + sg_sw_off(16, j, k)) =
            __float2bfloat16_rn(j < SG_OUT ? params[SG_OFF_W4 + j * SG_H + k] : 0.f);
    }
    float* f = reinterpret_cast<float*>(img + SG_IMG_F);
    for (int t = t0; t < SG_H * SG_IN; t += st) f[SG_F_W0 + t] = bf16r(params[SG_OFF_W0 + t]);
    for (int t = t0; t < 4 * SG_H + 8; t += st)
        f[SG_F_B + t] = bf16r(t < 4 * SG_H ? params[sg_off_b(t / SG_H) + t % SG_H]
                                           : (t - 4 * SG_H < SG_OUT ? params[SG_OFF_B4 + t - 4 * SG_H] : 0.f));
    for (int t = t0; t < 2 * SG_OUT; t += st) f[SG_F_N + t] = norm[t];
}

// The shared-memory side of a network CTA: the image, the two A tiles, the MMA barrier and TMEM.
struct SgTc {
    const uint8_t* img;
    uint8_t* A;
    uint64_t* bar;
    uint32_t tmem;
    uint32_t phase;
};

// The CTA's setup (every thread): the image copied in, the barrier, TMEM allocated (warp 0).
__device__ __forceinline__ SgTc sg_tc_setup(uint8_t* raw, const uint8_t* __restrict__ img_g, uint32_t* tslot) {
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    const uint4* src = reinterpret_cast<const uint4*>(img_g);
    uint4* dst = reinterpret_cast<uint4*>(base);
    for (int t = tid; t < (int)(SG_IMG_BYTES / 16); t += nt) dst[t] = src[t];
    SgTc c;
    c.img = base;
    c.A = base + SG_IMG_BYTES;
    c.bar = reinterpret_cast<uint64_t*>(c.A + 2 * SG_TILE_BYTES);
    c.phase = 0;
    if (tid == 0) {
        tc::mbar_init(c.bar, 1);
        tc::fence_barrier_init();
    }
    if (tid < 32) tc::tmem_alloc(tslot, SG_TMEM_COLS);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    c.tmem = *tslot;
    return c;
}

// Every MMA complete (bounded), then TMEM freed: the CTA's teardown (every thread).
__device__ __forceinline__ void sg_tc_teardown(SgTc& c, int* err) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid == 0) {
        tc::mma_commit(c.bar);
        if (!tc::mbar_wait(c.bar, c.phase) && err) atomicExch(err, 9);
    }
    tc::tc_fence_before();
    __syncthreads();
    if (tid < 32) tc::tmem_dealloc(c.tmem, SG_TMEM_COLS);
}

// Row `row` of A tile `m` (128 BF16 values h[0..127] given as 64 packed pairs) into shared memory.
__device__ __forceinline__ void sg_put_row(uint8_t* tile, int row, const uint32_t* h2) {
#pragma unroll
    for (int u = 0; u < 16; u++) {  // 16-byte units of 8 values: K = 8 u .. 8 u + 7
        const int k = 8 * u;
        *reinterpret_cast<uint4*>(tile + sg_sw_off(SG_H, row, k)) =
            make_uint4(h2[4 * u], h2[4 * u + 1], h2[4 * u + 2], h2[4 * u + 3]);
    }
}

__device__ __forceinline__ float silu_fast(float z) { return __fdividef(z, 1.f + __expf(-z)); }

// One pass of the network for the CTA's 256 threads (thread t: tile t / 128, row t % 128; the warps
// of a tile are the four TMEM lane quarters): inputs (u, v) of the thread's sample, out6 its six
// de-standardized outputs.  Every thread of the CTA calls it.  false when an MMA wait timed out.
__device__ bool sg_tc_forward(SgTc& c, float u, float v, float* out6) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int m = tid >> 7, row = tid & 127, quad = (tid >> 5) & 3;
    uint8_t* tile = c.A + (size_t)m * SG_TILE_BYTES;
    const float* f = reinterpret_cast<const float*>(c.img + SG_IMG_F);
    const float* W0 = f + SG_F_W0;
    const float* bias = f + SG_F_B;
    bool ok = true;
    // layer 0 on the CUDA cores (inputs rounded to BF16 as in training; w = 0)
    {
        const float ub = bf16r(u), vb = bf16r(v);
        uint32_t h2[64];
#pragma unroll
        for (int j2 = 0; j2 < 64; j2++) {
            const int j = 2 * j2;
            const float z0 = fmaf(W0[3 * j], ub, fmaf(W0[3 * j + 1], vb, bias[j]));
            const float z1 = fmaf(W0[3 * j + 3], ub, fmaf(W0[3 * j + 4], vb, bias[j + 1]));
            h2[j2] = pack_bf16(silu_fast(z0), silu_fast(z1));
        }
        sg_put_row(tile, row, h2);
    }
    const uint32_t taccum = c.tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)m * SG_H;
    for (int l = 1; l <= 4; l++) {
        tc::fence_proxy_async_smem();  // the A rows written by this thread, visible to the tensor core
        __syncthreads();
        if (tid == 0) {
            tc::tc_fence_after();
            const bool last = l == 4;
            const uint32_t idesc = last ? sg_idesc_bf16(128, 16) : sg_idesc_bf16(128, SG_H);
            const uint8_t* B = last ? c.img + SG_IMG_W4 : c.img + (size_t)(l - 1) * SG_TILE_BYTES;
            const int brows = last ? 16 : SG_H;
            for (int mm = 0; mm < 2; mm++) {
                const uint32_t a0 = tc::smem_u32(c.A + (size_t)mm * SG_TILE_BYTES), b0 = tc::smem_u32(B);
                const uint32_t d = c.tmem + (last ? 256u + 32u * mm : (uint32_t)mm * SG_H);
#pragma unroll
                for (int kk = 0; kk < SG_H / 16; kk++) {
                    const uint32_t ko = (uint32_t)(kk / 4) * 128u * 128u + (uint32_t)(kk % 4) * 32u;
                    const uint32_t kb = (uint32_t)(kk / 4) * (uint32_t)brows * 128u + (uint32_t)(kk % 4) * 32u;
                    tc::mma_f16(d, tc::desc_kmajor_sw128(a0 + ko), tc::desc_kmajor_sw128(b0 + kb), idesc, kk > 0);
                }
            }
            tc::mma_commit(c.bar);
        }
        const bool done = tc::mbar_wait(c.bar, c.phase);
        c.phase ^= 1u;
        ok = ok && done;
        tc::tc_fence_after();
        if (l < 4) {  // bias, SiLU, BF16: the next layer's A row
            const float* b = bias + l * SG_H;
            uint32_t h2[64];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float acc[32];
                tc::tmem_ld32(taccum + 32 * q, acc);
#pragma unroll
                for (int e = 0; e < 16; e++)
                    h2[16 * q + e] = pack_bf16(silu_fast(acc[2 * e] + b[32 * q + 2 * e]),
                                               silu_fast(acc[2 * e + 1] + b[32 * q + 2 * e + 1]));
            }
            tc::tc_fence_before();
            sg_put_row(tile, row, h2);
        } else {
            float acc[32];
            tc::tmem_ld32(c.tmem + ((uint32_t)(quad * 32) << 16) + 256u + 32u * m, acc);
            const float* nm = f + SG_F_N;
#pragma unroll
            for (int q = 0; q < SG_OUT; q++) out6[q] = nm[q] + nm[SG_OUT + q] * (acc[q] + bias[4 * SG_H + q]);
            tc::tc_fence_before();
        }
    }
    __syncthreads();  // every accumulator read before a later pass's MMAs overwrite TMEM
    return ok;
}

// out [n][6] (FP32, de-standardized) from inputs [n][3]: persistent CTAs of 256 threads, 256 samples
// a pass.  err (may be null) set to 9 if an MMA wait timed out.
__global__ void __launch_bounds__(256, 1) k_sg_infer_tc(int n, const uint8_t* __restrict__ img_g,
                                                        const float* __restrict__ in, float* __restrict__ out,
                                                        int* __restrict__ err) {
    extern __shared__ uint8_t sg_raw[];
    __shared__ uint32_t tslot;
    SgTc c = sg_tc_setup(sg_raw, img_g, &tslot);
    const int tid = threadIdx.x;
    bool ok = true;
    for (int s0 = blockIdx.x * 256; s0 < n; s0 += gridDim.x * 256) {
        const int i = s0 + tid;
        const float u = i < n ? in[3 * (size_t)i] : 0.f, v = i < n ? in[3 * (size_t)i + 1] : 0.f;
        float o[SG_OUT];
        ok = sg_tc_forward(c, u, v, o) && ok;
        if (i < n)
#pragma unroll
            for (int q = 0; q < SG_OUT; q++) out[(size_t)i * SG_OUT + q] = o[q];
    }
    if (!ok && err) atomicExch(err, 9);
    sg_tc_teardown(c, err);
}

// The wave term from the network's outputs: the logarithmic part in closed form (J0, J1 from the
// 1-D table below X = 30, the Hankel asymptotics above), the regular part and the imaginary part from the network, FY by the identity
// FY = -F - 2 / R0.
__device__ inline Wave sg_wave(double X, double Y, const float* o) {
    double j0, j1;
    bessel_j01<false>(X, j0, j1);
    const double eY = exp(-Y), R0 = sqrt(X * X + Y * Y);
    const double lg = log(Y + R0) + (GAMMA - LOG2);
    Wave w;
    w.F = -2.0 * eY * j0 * lg + (double)o[0];
    w.FX = 2.0 * eY * j1 * lg - 2.0 * eY * j0 * X / (R0 * (Y + R0)) + (double)o[1];
    w.FY = -w.F - 2.0 / R0;
    w.I = o[3];
    w.IX = o[4];
    w.IY = o[5];
    w.c = eY * j0;
    return w;
}

// The mixed-form assembly with the network as the wave term inside its domain (X < 100, Y < 50,
// R0 > 0; the tables and series outside): persistent CTAs (the weight image loaded once per CTA, TMEM
// held for the launch), work items (tile pair, frequency) taken round-robin; the per-item work is
// k_assemble's, the network run for the CTA's 256 pairs of each row group at once.
template <bool FINITE>
__global__ void __launch_bounds__(256, 1) k_assemble_sg(PanelsView pv, const double* __restrict__ st,
                                                       const FreqInfo* __restrict__ fi, const FdParams* __restrict__ fdp,
                                                       const float* __restrict__ tiles, const double* __restrict__ fpt,
                                                       OutF32 out, int F, const uint8_t* __restrict__ img_g,
                                                       unsigned long long* __restrict__ counts, int* __restrict__ err) {
    extern __shared__ uint8_t sg_raw[];
    __shared__ double sT[4][32][33];
    __shared__ uint32_t tslot;
    if (pv.invalid()) return;  // invalid panels: the solve reports them
    SgTc c = sg_tc_setup(sg_raw, img_g, &tslot);
    bool ok = true;
    const int N = pv.N;
    const int nt = (N + 31) / 32, ntp = nt * (nt + 1) / 2;
    const size_t NN = (size_t)N * N;
    const int tx = threadIdx.x, ty = threadIdx.y;
    unsigned long long used = 0;
    for (int item = blockIdx.x; item < ntp * F; item += gridDim.x) {
        const int f = item / ntp;
        int idx = item % ntp, kb = 0;
        while (idx >= nt - kb) {
            idx -= nt - kb;
            kb++;
        }
        const int nb = kb + idx;
        const int K0 = kb * 32, N0 = nb * 32;
        const FreqInfo info = fi[f];
        const double K = info.K, logc = info.logc;
        __syncthreads();  // sT of the previous item written out
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int n = N0 + tx, k = K0 + ty + 8 * i;
            if (n < N && k < N)
#pragma unroll
                for (int q = 0; q < 4; q++) sT[q][ty + 8 * i][tx] = __ldg(st + q * NN + (size_t)n + (size_t)k * N);
        }
        __syncthreads();
        const int k = K0 + tx;
        const int kc = min(k, N - 1);
        double xk[3], nk[3], ak;
        for (int d = 0; d < 3; d++) {
            xk[d] = pv.at(P_C + d, kc);
            nk[d] = pv.at(P_N + d, kc);
        }
        ak = pv.at(P_AREA, kc);
        const int kindk = pv.kind[kc];
        const FdParams* fd = FINITE ? fdp + f : nullptr;
        const float* T1 = FINITE ? tiles + (size_t)f * (T1F_SIZE + T2F_SIZE) : nullptr;
        const float* T2 = FINITE ? T1 + T1F_SIZE : nullptr;
        const double* fp = FINITE ? fpt + (size_t)f * FP_PLANES * N : nullptr;
#pragma unroll 1
        for (int i = 0; i < 4; i++) {
            const int nl = ty + 8 * i, n = N0 + nl;
            const bool live = k < N && n < N && (kb != nb || k <= n);
            const int ncl = min(n, N - 1);
            double xn[3], nn3[3];
            for (int d = 0; d < 3; d++) {
                xn[d] = pv.at(P_C + d, ncl);
                nn3[d] = pv.at(P_N + d, ncl);
            }
            const double an = pv.at(P_AREA, ncl);
            const int kindn = pv.kind[ncl];
            double dx = xk[0] - xn[0], dy = xk[1] - xn[1];
            double R = sqrt(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
            const double X = K * R, Y = -K * (xk[2] + xn[2]);
            const bool inb = live && X < SG_XMAX && Y < SG_YMAX && (X > 0.0 || Y > 0.0);
            float o6[SG_OUT] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (__syncthreads_or(inb)) {  // the CTA's 256 pairs through the network at once
                float in3[3];
                sg_inputs(X, Y, in3);
                ok = sg_tc_forward(c, in3[0], in3[1], o6) && ok;
            }
            if (!live) continue;
            used += inb;
            Kern w;
            if (FINITE) {
                if (inb) {
                    const Wave sw = sg_wave(X, Y, o6);
                    w = finite_kernel<true, float, true>(*fd, T1, T2, R, xk[2], xn[2], fp + k, fp + n, N, &sw);
                } else {
                    w = finite_kernel<true>(*fd, T1, T2, R, xk[2], xn[2], fp + k, fp + n, N);
                }
            } else {
                w = inb ? wave_kern(K, sg_wave(X, Y, o6)) : pair_kernel_inf<true>(K, R, xk[2], xn[2]);
            }
            size_t o1 = (size_t)k + (size_t)n * N;
            double2 s1, d1;
            apply_kernel(__ldg(st + o1), __ldg(st + NN + o1), __ldg(st + 2 * NN + o1), __ldg(st + 3 * NN + o1), an,
                         nn3[0], nn3[1], nn3[2], kindn, xk, xn, K, logc, w, R, false, s1, d1);
            out.put(f, k, n, s1, make_double2((k == n ? free_term(kindk) : 0.0) - d1.x, -d1.y));
            if (n != k) {
                double2 s2, d2;
                apply_kernel(sT[0][tx][nl], sT[1][tx][nl], sT[2][tx][nl], sT[3][tx][nl], ak, nk[0], nk[1], nk[2],
                             kindk, xn, xk, K, logc, w, R, true, s2, d2);
                sT[0][tx][nl] = s2.x;
                sT[1][tx][nl] = s2.y;
                sT[2][tx][nl] = -d2.x;
                sT[3][tx][nl] = -d2.y;
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int n = N0 + tx, kl = ty + 8 * i, kk = K0 + kl;
            if (n < N && kk < N && (kb != nb || n > kk))
                out.put(f, n, kk, make_double2(sT[0][kl][tx], sT[1][kl][tx]), make_double2(sT[2][kl][tx], sT[3][kl][tx]));
        }
    }
    // pairs whose wave term came from the network
    for (int o = 16; o > 0; o >>= 1) used += __shfl_xor_sync(0xffffffffu, used, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(counts, used);
    if (!ok) atomicExch(err, 9);
    sg_tc_teardown(c, err);
}

void launch_sg_pack(const float* params_norm, uint8_t* img, cudaStream_t s) {
    k_sg_pack<<<64, 256, 0, s>>>(params_norm, params_norm + SG_PARAMS, img);
}

size_t sg_image_bytes() { return SG_IMG_BYTES; }

void launch_assemble_f32_sg(const PanelsView& pv, const double* st, int F, const FreqInfo* fi, const FdParams* fd,
                            const float* tiles, const double* fpt, bool finite, float* S, float* A, int Np,
                            const uint8_t* img, unsigned long long* counts, int* err, cudaStream_t s) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    OutF32 o{S, A, 2 * (size_t)Np * Np, Np};
    if (finite) {
        cudaFuncSetAttribute(k_assemble_sg<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SG_TC_SMEM);
        k_assemble_sg<true><<<nsm, dim3(32, 8), SG_TC_SMEM, s>>>(pv, st, fi, fd, tiles, fpt, o, F, img, counts, err);
    } else {
        cudaFuncSetAttribute(k_assemble_sg<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SG_TC_SMEM);
        k_assemble_sg<false><<<nsm, dim3(32, 8), SG_TC_SMEM, s>>>(pv, st, fi, fd, tiles, fpt, o, F, img, counts, err);
    }
}

// ---------------------------------------------------------------- host side
static uint64_t sg_lcg(uint64_t& st) {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return st >> 11;
}

// Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights from a seeded LCG, zero biases.
static void sg_init(std::vector<float>& p, uint64_t seed) {
    p.assign(SG_PARAMS, 0.f);
    uint64_t st = seed * 2654435761ull + 12345;
    for (int l = 0; l < 5; l++) {
        const int fi = sg_fan_in(l), fo = sg_fan_out(l);
        const float a = (l == 0 ? 2.0f : 1.0f) * std::sqrt(3.0f / fi);
        for (int i = 0; i < fo * fi; i++)
            p[sg_off_w(l) + i] = a * (2.0f * (float)((double)sg_lcg(st) / 9007199254740992.0) - 1.0f);
    }
}

__global__ void k_sg_standardize(size_t n, const double* __restrict__ t, const double* __restrict__ mean,
                                 const double* __restrict__ spread, float* __restrict__ o) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n * SG_OUT) {
        const int c = (int)(i % SG_OUT);
        o[i] = (float)((t[i] - mean[c]) / spread[c]);
    }
}

struct DevArr {
    void* p = nullptr;
    ~DevArr() {
        if (p) cudaFree(p);
    }
    template <class T>
    T* alloc(size_t n) {
        if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) p = nullptr;
        return static_cast<T*>(p);
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

int surrogate_train(int64_t n_train, int batch, int steps, double lr0, uint64_t seed, int64_t n_val, float* params_out,
                    float* norm_out, double* report, const char** msg) {
    if (n_train < batch || batch < 64 || steps < 1 || n_val < 16) {
        *msg = "surrogate training: need n_train >= batch >= 64, steps >= 1, n_val >= 16";
        return HB_ERR_VALUE;
    }
    cudaStream_t s = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    DevArr din, dtg, dtf, dmean, dspread, dvin, dvtg, dvout, dnorm;
    float* in = din.alloc<float>((size_t)n_train * 3);
    double* tg = dtg.alloc<double>((size_t)n_train * SG_OUT);
    float* tf = dtf.alloc<float>((size_t)n_train * SG_OUT);
    double* mean = dmean.alloc<double>(SG_OUT);
    double* spread = dspread.alloc<double>(SG_OUT);
    float* vin = dvin.alloc<float>((size_t)n_val * 3);
    double* vtg = dvtg.alloc<double>((size_t)n_val * SG_OUT);
    float* vout = dvout.alloc<float>((size_t)n_val * SG_OUT);
    float* dn = dnorm.alloc<float>(2 * SG_OUT);
    SgTrainer tr;
    if (!in || !tg || !tf || !mean || !spread || !vin || !vtg || !vout || !dn || !tr.alloc(batch)) {
        *msg = "surrogate training: device allocation failed";
        return HB_ERR_INTERNAL;
    }
    // samples of the table evaluation: training set, then a disjoint validation set
    k_sg_samples<<<(unsigned)((n_train + 255) / 256), 256, 0, s>>>((int)n_train, 0, in, tg, nullptr);
    k_sg_samples<<<(unsigned)((n_val + 255) / 256), 256, 0, s>>>((int)n_val, (uint64_t)n_train, vin, vtg, nullptr);
    k_sg_round<<<(unsigned)((n_train * 3 + 255) / 256), 256, 0, s>>>((int)(n_train * 3), in, in);
    // standardization from the first 65536 samples (host)
    const int ns = (int)std::min<int64_t>(n_train, 65536);
    std::vector<double> ht((size_t)ns * SG_OUT);
    cudaMemcpyAsync(ht.data(), tg, ht.size() * 8, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    double hm[SG_OUT], hs[SG_OUT];
    for (int c = 0; c < SG_OUT; c++) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i < ns; i++) a += ht[(size_t)i * SG_OUT + c];
        a /= ns;
        for (int i = 0; i < ns; i++) b += (ht[(size_t)i * SG_OUT + c] - a) * (ht[(size_t)i * SG_OUT + c] - a);
        hm[c] = a;
        hs[c] = std::sqrt(b / ns) + 1e-30;
    }
    cudaMemcpyAsync(mean, hm, sizeof hm, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(spread, hs, sizeof hs, cudaMemcpyHostToDevice, s);
    k_sg_standardize<<<(unsigned)((n_train * SG_OUT + 255) / 256), 256, 0, s>>>((size_t)n_train, tg, mean, spread, tf);
    std::vector<float> hp;
    sg_init(hp, seed);
    cudaMemcpyAsync(tr.p, hp.data(), SG_PARAMS * 4, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(tr.m, 0, SG_PARAMS * 4, s);
    cudaMemsetAsync(tr.v, 0, SG_PARAMS * 4, s);
    const int nbp = (SG_PARAMS + 255) / 256;
    const int nparts = (int)(((size_t)batch * SG_OUT + 255) / 256);
    std::vector<float> hpart(nparts);
    double loss_first = -1.0, loss_last = -1.0;
    const int64_t nbatches = n_train / batch;
    for (int st = 0; st < steps; st++) {
        const int64_t b0 = (st % nbatches) * batch;
        k_sg_round<<<nbp, 256, 0, s>>>(SG_PARAMS, tr.p, tr.pr);
        tr.forward(in + 3 * b0, batch, s);
        tr.backward(in + 3 * b0, tf + SG_OUT * b0, batch, s);
        const double t = st + 1;
        const float lr = (float)(lr0 * 0.5 * (1.0 + std::cos(3.141592653589793 * st / steps)));
        k_sg_adam<<<nbp, 256, 0, s>>>(SG_PARAMS, tr.p, tr.g, tr.m, tr.v, lr, 0.9f, 0.999f,
                                      (float)(1.0 - std::pow(0.9, t)), (float)(1.0 - std::pow(0.999, t)));
        if (st == 0 || st == steps - 1) {
            cudaMemcpyAsync(hpart.data(), tr.part, nparts * 4, cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            double a = 0.0;
            for (float v : hpart) a += v;
            (st == 0 ? loss_first : loss_last) = a / ((double)batch * SG_OUT);
        }
    }
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float train_ms = 0.f;
    cudaEventElapsedTime(&train_ms, e0, e1);
    // validation through the tensor-core inference kernel
    float hn[2 * SG_OUT];
    for (int c = 0; c < SG_OUT; c++) {
        hn[c] = (float)hm[c];
        hn[SG_OUT + c] = (float)hs[c];
    }
    cudaMemcpyAsync(dn, hn, sizeof hn, cudaMemcpyHostToDevice, s);
    DevArr dimg, derr;
    uint8_t* img = dimg.alloc<uint8_t>(SG_IMG_BYTES);
    int* ierr = derr.alloc<int>(1);
    if (!img || !ierr) {
        *msg = "surrogate training: device allocation failed";
        return HB_ERR_INTERNAL;
    }
    cudaMemsetAsync(ierr, 0, sizeof(int), s);
    k_sg_pack<<<64, 256, 0, s>>>(tr.p, dn, img);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_sg_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SG_TC_SMEM);
    k_sg_infer_tc<<<nsm, 256, SG_TC_SMEM, s>>>((int)n_val, img, vin, vout, ierr);
    int herr = 0;
    cudaMemcpyAsync(&herr, ierr, sizeof(int), cudaMemcpyDeviceToHost, s);
    std::vector<float> ho((size_t)n_val * SG_OUT);
    std::vector<double> hv((size_t)n_val * SG_OUT);
    cudaMemcpyAsync(ho.data(), vout, ho.size() * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hv.data(), vtg, hv.size() * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(params_out, tr.p, SG_PARAMS * 4, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cudaGetLastError() != cudaSuccess || herr != 0) {
        *msg = herr ? "surrogate training: a tensor-core wait of the validation timed out" : "CUDA error in surrogate training";
        return HB_ERR_INTERNAL;
    }
    for (int c = 0; c < 2 * SG_OUT; c++) norm_out[c] = hn[c];
    // report: [0] first loss, [1] last loss, [2] train ms, [3..8] validation rms error / spread,
    // [9..14] max |error| / max |target| per output
    report[0] = loss_first;
    report[1] = loss_last;
    report[2] = train_ms;
    for (int c = 0; c < SG_OUT; c++) {
        double se = 0.0, me = 0.0, mt = 0.0;
        for (int64_t i = 0; i < n_val; i++) {
            const double d = (double)ho[(size_t)i * SG_OUT + c] - hv[(size_t)i * SG_OUT + c];
            se += d * d;
            me = std::max(me, std::fabs(d));
            mt = std::max(mt, std::fabs(hv[(size_t)i * SG_OUT + c]));
        }
        report[3 + c] = std::sqrt(se / n_val) / hs[c];
        report[9 + c] = me / std::max(mt, 1e-300);
    }
    return 0;
}

// Gradients of the training loss at given parameters for given (standardized) samples: the
// training kernels' forward and backward, exposed for their check against a CPU computation.
int surrogate_grad(const float* params, int n, const float* inputs, const float* targets, float* grads, double* loss,
                   const char** msg) {
    if (n < 1) {
        *msg = "n must be positive";
        return HB_ERR_VALUE;
    }
    SgTrainer tr;
    DevArr din, dtf;
    float* in = din.alloc<float>((size_t)n * 3);
    float* tf = dtf.alloc<float>((size_t)n * SG_OUT);
    if (!in || !tf || !tr.alloc(n)) {
        *msg = "device allocation failed";
        return HB_ERR_INTERNAL;
    }
    cudaStream_t s = 0;
    cudaMemcpy(in, inputs, (size_t)n * 12, cudaMemcpyHostToDevice);
    cudaMemcpy(tf, targets, (size_t)n * SG_OUT * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(tr.p, params, SG_PARAMS * 4, cudaMemcpyHostToDevice);
    k_sg_round<<<(n * 3 + 255) / 256, 256, 0, s>>>(n * 3, in, in);
    k_sg_round<<<(SG_PARAMS + 255) / 256, 256, 0, s>>>(SG_PARAMS, tr.p, tr.pr);
    tr.forward(in, n, s);
    tr.backward(in, tf, n, s);
    const int nparts = (int)(((size_t)n * SG_OUT + 255) / 256);
    std::vector<float> hpart(nparts);
    cudaMemcpy(hpart.data(), tr.part, nparts * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(grads, tr.g, SG_PARAMS * 4, cudaMemcpyDeviceToHost);
    if (cudaGetLastError() != cudaSuccess) {
        *msg = "CUDA error in the surrogate gradient";
        return HB_ERR_INTERNAL;
    }
    double a = 0.0;
    for (float v : hpart) a += v;
    *loss = a / ((double)n * SG_OUT);
    return 0;
}

// Network and table at the same points: out_net / out_table [n][6] (either may be NULL), and the
// device time of each evaluation over all n points (points resident on the device, one warm-up).
int surrogate_eval(const float* params, const float* norm, int n, const double* xy, double* out_net,
                   double* out_table, double* ms2, const char** msg) {
    DevArr dxy, din, dout, dtg, dp, dn;
    double* x = dxy.alloc<double>((size_t)n * 2);
    float* in = din.alloc<float>((size_t)n * 3);
    float* o = dout.alloc<float>((size_t)n * SG_OUT);
    double* tg = dtg.alloc<double>((size_t)n * SG_OUT);
    float* p = dp.alloc<float>(SG_PARAMS);
    float* nm = dn.alloc<float>(2 * SG_OUT);
    if (!x || !in || !o || !tg || !p || !nm) {
        *msg = "device allocation failed";
        return HB_ERR_INTERNAL;
    }
    cudaMemcpy(x, xy, (size_t)n * 16, cudaMemcpyHostToDevice);
    cudaMemcpy(p, params, SG_PARAMS * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(nm, norm, 2 * SG_OUT * 4, cudaMemcpyHostToDevice);
    DevArr dimg, derr;
    uint8_t* img = dimg.alloc<uint8_t>(SG_IMG_BYTES);
    int* ierr = derr.alloc<int>(1);
    if (!img || !ierr) {
        *msg = "device allocation failed";
        return HB_ERR_INTERNAL;
    }
    cudaMemset(ierr, 0, sizeof(int));
    k_sg_pack<<<64, 256>>>(p, nm, img);
    cudaFuncSetAttribute(k_sg_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SG_TC_SMEM);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto timed = [&](auto launch) {
        launch();
        cudaEventRecord(e0);
        launch();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return (double)ms;
    };
    const unsigned nb = (unsigned)((n + 255) / 256);
    // the network's time includes forming its inputs from (X, Y)
    ms2[0] = timed([&] {
        k_sg_inputs<<<nb, 256>>>(n, x, in);
        k_sg_infer_tc<<<nsm, 256, SG_TC_SMEM>>>(n, img, in, o, ierr);
    });
    ms2[1] = timed([&] { k_sg_table<<<nb, 256>>>(n, x, tg); });
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (out_net) {
        std::vector<float> h((size_t)n * SG_OUT);
        cudaMemcpy(h.data(), o, h.size() * 4, cudaMemcpyDeviceToHost);
        for (size_t i = 0; i < h.size(); i++) out_net[i] = h[i];
    }
    if (out_table) cudaMemcpy(out_table, tg, (size_t)n * SG_OUT * 8, cudaMemcpyDeviceToHost);
    int herr = 0;
    cudaMemcpy(&herr, ierr, sizeof(int), cudaMemcpyDeviceToHost);
    if (cudaGetLastError() != cudaSuccess || herr != 0) {
        *msg = herr ? "a tensor-core wait of the surrogate evaluation timed out" : "CUDA error in the surrogate evaluation";
        return HB_ERR_INTERNAL;
    }
    return 0;
}

}  // namespace hbg
