// hbg_surrogate.cu -- the learned part of the mixed form: an MLP surrogate of the regular part of the
// infinite-depth wave term of the Green function, trained on the device by this file's own forward
// and backward kernels on samples of the library's own table evaluation, and evaluated on the
// tensor cores (mma.sync BF16, FP32 accumulation).
//
// What it learns.  In the table region X = K R, Y = -K (z + zeta) in [0, 30)^2 the wave term is
// (green_inf.rs:316-368, identity form)
//     F  = S + g,   S = -2 e^-Y J0(X) (log(Y + R0) + gamma - log 2),   R0 = sqrt(X^2 + Y^2),
// S holding the logarithmic singularity at R0 = 0 in closed form.  The network maps the inputs
// (u, v, w) = (2 log1p(X) / log 31 - 1, 2 log1p(Y) / log 31 - 1, 1 / (K h)) -- w = 0 for infinite
// depth -- to six outputs: g, dg/dX, dg/dY (the regular real part and its radial and vertical
// derivatives) and I, dI/dX, dI/dY (the imaginary part -2 pi e^-Y J0(X) and its derivatives), each
// standardized by its mean and spread over the training set.  Architecture 3 -> 128 -> 128 -> 128
// -> 128 -> 6, SiLU, weights rounded to BF16 in the forward pass (FP32 master copy and Adam
// moments), activations rounded to BF16 between layers, FP32 accumulation.  Outside [0, 30)^2 the
// table/series evaluation is used.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

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
constexpr double SG_XMAX = 30.0;
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
    const double L = log(1.0 + SG_XMAX);
    in[0] = (float)(2.0 * log1p(X) / L - 1.0);
    in[1] = (float)(2.0 * log1p(Y) / L - 1.0);
    in[2] = 0.f;  // 1 / (K h): infinite depth
}

// The six targets at (X, Y) from the table evaluation (FP64).
__device__ void sg_targets(double X, double Y, double* t) {
    const Wave w = wave_kernel<false>(X, Y);
    double f[4];
    table1d(X, f);
    const double j0 = f[0], j1 = f[1], eY = exp(-Y), R0 = sqrt(X * X + Y * Y);
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

// Samples i0 + 1 .. i0 + n of the 2-D Halton sequence, log-spaced over [0, 30)^2:
// X = (31^u - 1), Y = (31^v - 1); inputs [n][3] (FP32) and FP64 targets [n][6].
__global__ void k_sg_samples(int n, uint64_t i0, float* __restrict__ in, double* __restrict__ tg,
                             double* __restrict__ xy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t h = i0 + (uint64_t)i + 1;
    const double L = log(1.0 + SG_XMAX);
    const double X = expm1(halton(h, 2) * L), Y = expm1(halton(h, 3) * L);
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
// A warp evaluates 16 samples per pass: each layer is a 16 x 128 by 128 x 128 product of
// mma.sync m16n8k16 BF16 tiles; the FP32 accumulator fragments of one layer become, after bias,
// SiLU and rounding, the BF16 A fragments of the next without leaving registers.  Weights in
// shared memory as BF16 rows padded to 136 entries (conflict-free B fragment reads).
constexpr int SG_LD = SG_H + 8;
constexpr size_t SG_SMEM = (size_t)(SG_H * 16 + 3 * SG_H * SG_LD + 8 * SG_LD) * 2 + (size_t)(4 * SG_H + 8) * 4;

__device__ __forceinline__ void mma_bf16_16816(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// out [n][6] (FP32, de-standardized by mean/spread norm[0..5], norm[6..11]) from inputs [n][3].
__global__ void __launch_bounds__(256) k_sg_infer(int n, const float* __restrict__ params, const float* __restrict__ norm,
                                                  const float* __restrict__ in, float* __restrict__ out) {
    extern __shared__ __align__(16) uint8_t sg_smem[];
    __nv_bfloat16* w0 = reinterpret_cast<__nv_bfloat16*>(sg_smem);  // [H][16] (k padded)
    __nv_bfloat16* wh = w0 + SG_H * 16;                              // 3 x [H][SG_LD]
    __nv_bfloat16* w4 = wh + 3 * SG_H * SG_LD;                       // [8][SG_LD] (rows 6, 7 zero)
    float* bias = reinterpret_cast<float*>(w4 + 8 * SG_LD);          // b0..b3 [4][H], b4 [8]
    for (int t = threadIdx.x; t < SG_H * 16; t += blockDim.x) {
        const int j = t / 16, k = t % 16;
        w0[t] = __float2bfloat16_rn(k < SG_IN ? params[SG_OFF_W0 + j * SG_IN + k] : 0.f);
    }
    for (int t = threadIdx.x; t < 3 * SG_H * SG_LD; t += blockDim.x) {
        const int l = t / (SG_H * SG_LD), r = t % (SG_H * SG_LD), j = r / SG_LD, k = r % SG_LD;
        wh[t] = __float2bfloat16_rn(k < SG_H ? params[sg_off_w(l + 1) + j * SG_H + k] : 0.f);
    }
    for (int t = threadIdx.x; t < 8 * SG_LD; t += blockDim.x) {
        const int j = t / SG_LD, k = t % SG_LD;
        w4[t] = __float2bfloat16_rn(j < SG_OUT && k < SG_H ? params[SG_OFF_W4 + j * SG_H + k] : 0.f);
    }
    for (int t = threadIdx.x; t < 4 * SG_H + 8; t += blockDim.x)
        bias[t] = bf16r(t < 4 * SG_H ? params[sg_off_b(t / SG_H) + t % SG_H]
                                     : (t - 4 * SG_H < SG_OUT ? params[SG_OFF_B4 + t - 4 * SG_H] : 0.f));
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
    const int warps = gridDim.x * (blockDim.x >> 5), wid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t* w0u = reinterpret_cast<const uint32_t*>(w0);
    const uint32_t* whu = reinterpret_cast<const uint32_t*>(wh);
    const uint32_t* w4u = reinterpret_cast<const uint32_t*>(w4);
    for (int s0 = wid * 16; s0 < n; s0 += warps * 16) {
        // layer 0: A = [u v w 0 ...] (k padded to 16)
        uint32_t a[8][4];
        {
            const int r0 = s0 + g, r1 = s0 + g + 8;
            float x0 = 0.f, x1 = 0.f, y0 = 0.f, y1 = 0.f;
            if (tq < 2) {
                const int c = 2 * tq;
                if (r0 < n) {
                    x0 = in[3 * (size_t)r0 + c];
                    y0 = c + 1 < SG_IN ? in[3 * (size_t)r0 + c + 1] : 0.f;
                }
                if (r1 < n) {
                    x1 = in[3 * (size_t)r1 + c];
                    y1 = c + 1 < SG_IN ? in[3 * (size_t)r1 + c + 1] : 0.f;
                }
            }
            uint32_t a0[4] = {pack_bf16(x0, y0), pack_bf16(x1, y1), 0u, 0u};
            float acc[16][4];
#pragma unroll
            for (int nt = 0; nt < 16; nt++) {
                acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
                const int j = nt * 8 + g;
                mma_bf16_16816(acc[nt], a0, w0u[(j * 16 + 2 * tq) / 2], w0u[(j * 16 + 2 * tq + 8) / 2]);
            }
#pragma unroll
            for (int kt = 0; kt < 8; kt++) {
                const int c0 = (2 * kt) * 8 + 2 * tq, c1 = (2 * kt + 1) * 8 + 2 * tq;
                const float* b = bias;
                a[kt][0] = pack_bf16(silu(acc[2 * kt][0] + b[c0]), silu(acc[2 * kt][1] + b[c0 + 1]));
                a[kt][1] = pack_bf16(silu(acc[2 * kt][2] + b[c0]), silu(acc[2 * kt][3] + b[c0 + 1]));
                a[kt][2] = pack_bf16(silu(acc[2 * kt + 1][0] + b[c1]), silu(acc[2 * kt + 1][1] + b[c1 + 1]));
                a[kt][3] = pack_bf16(silu(acc[2 * kt + 1][2] + b[c1]), silu(acc[2 * kt + 1][3] + b[c1 + 1]));
            }
        }
        // hidden layers 1..3
#pragma unroll 1
        for (int l = 0; l < 3; l++) {
            const uint32_t* W = whu + (size_t)l * SG_H * SG_LD / 2;
            float acc[16][4];
#pragma unroll
            for (int nt = 0; nt < 16; nt++) {
                acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
                const int j = nt * 8 + g;
#pragma unroll
                for (int kt = 0; kt < 8; kt++)
                    mma_bf16_16816(acc[nt], a[kt], W[(j * SG_LD + kt * 16 + 2 * tq) / 2],
                                   W[(j * SG_LD + kt * 16 + 2 * tq + 8) / 2]);
            }
            const float* b = bias + (l + 1) * SG_H;
#pragma unroll
            for (int kt = 0; kt < 8; kt++) {
                const int c0 = (2 * kt) * 8 + 2 * tq, c1 = (2 * kt + 1) * 8 + 2 * tq;
                a[kt][0] = pack_bf16(silu(acc[2 * kt][0] + b[c0]), silu(acc[2 * kt][1] + b[c0 + 1]));
                a[kt][1] = pack_bf16(silu(acc[2 * kt][2] + b[c0]), silu(acc[2 * kt][3] + b[c0 + 1]));
                a[kt][2] = pack_bf16(silu(acc[2 * kt + 1][0] + b[c1]), silu(acc[2 * kt + 1][1] + b[c1 + 1]));
                a[kt][3] = pack_bf16(silu(acc[2 * kt + 1][2] + b[c1]), silu(acc[2 * kt + 1][3] + b[c1 + 1]));
            }
        }
        // output layer: one n-tile of 8 (6 used)
        float o[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kt = 0; kt < 8; kt++)
            mma_bf16_16816(o, a[kt], w4u[(g * SG_LD + kt * 16 + 2 * tq) / 2], w4u[(g * SG_LD + kt * 16 + 2 * tq + 8) / 2]);
        const float* b4 = bias + 4 * SG_H;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int r = s0 + g + (q >= 2 ? 8 : 0), c = 2 * tq + (q & 1);
            if (r < n && c < SG_OUT) out[(size_t)r * SG_OUT + c] = norm[c] + norm[SG_OUT + c] * (o[q] + b4[c]);
        }
    }
}

// ---------------------------------------------------------------- the network inside the assembly
// The packed weight image (global memory, copied whole into each persistent CTA's shared memory):
// w0 [H][16] BF16 (k padded), w1..w3 [H][SG_LD] BF16, w4 [8][SG_LD] BF16 (rows 6, 7 zero), biases
// FP32 [4 H + 8] (BF16-rounded values), output means and spreads FP32 [12].
constexpr size_t SG_IMG_WH = (size_t)SG_H * 16 * 2;
constexpr size_t SG_IMG_W4 = SG_IMG_WH + (size_t)3 * SG_H * SG_LD * 2;
constexpr size_t SG_IMG_B = SG_IMG_W4 + (size_t)8 * SG_LD * 2;
constexpr size_t SG_IMG_N = SG_IMG_B + (size_t)(4 * SG_H + 8) * 4;
constexpr size_t SG_IMG_BYTES = (SG_IMG_N + 2 * SG_OUT * 4 + 15) / 16 * 16;
static_assert(SG_IMG_B % 16 == 0, "biases at a 16-byte boundary");

__global__ void k_sg_pack(const float* __restrict__ params, const float* __restrict__ norm, uint8_t* __restrict__ img) {
    __nv_bfloat16* w0 = reinterpret_cast<__nv_bfloat16*>(img);
    __nv_bfloat16* wh = reinterpret_cast<__nv_bfloat16*>(img + SG_IMG_WH);
    __nv_bfloat16* w4 = reinterpret_cast<__nv_bfloat16*>(img + SG_IMG_W4);
    float* bias = reinterpret_cast<float*>(img + SG_IMG_B);
    float* nm = reinterpret_cast<float*>(img + SG_IMG_N);
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    for (int t = t0; t < SG_H * 16; t += st) {
        const int j = t / 16, k = t % 16;
        w0[t] = __float2bfloat16_rn(k < SG_IN ? params[SG_OFF_W0 + j * SG_IN + k] : 0.f);
    }
    for (int t = t0; t < 3 * SG_H * SG_LD; t += st) {
        const int l = t / (SG_H * SG_LD), r = t % (SG_H * SG_LD), j = r / SG_LD, k = r % SG_LD;
        wh[t] = __float2bfloat16_rn(k < SG_H ? params[sg_off_w(l + 1) + j * SG_H + k] : 0.f);
    }
    for (int t = t0; t < 8 * SG_LD; t += st) {
        const int j = t / SG_LD, k = t % SG_LD;
        w4[t] = __float2bfloat16_rn(j < SG_OUT && k < SG_H ? params[SG_OFF_W4 + j * SG_H + k] : 0.f);
    }
    for (int t = t0; t < 4 * SG_H + 8; t += st)
        bias[t] = bf16r(t < 4 * SG_H ? params[sg_off_b(t / SG_H) + t % SG_H]
                                     : (t - 4 * SG_H < SG_OUT ? params[SG_OFF_B4 + t - 4 * SG_H] : 0.f));
    for (int t = t0; t < 2 * SG_OUT; t += st) nm[t] = norm[t];
}

// One forward pass for the 32 lanes of a warp (each lane's inputs u, v; w = 0), lanes 0-15 and
// 16-31 as two m16 tiles of mma.sync m16n8k16 BF16; out6 = the de-standardized outputs of the
// lane's own sample.  Every lane of the warp must call it.
__device__ __forceinline__ void sg_warp_mlp(const uint8_t* img, float u, float v, float* out6) {
    const uint32_t* w0u = reinterpret_cast<const uint32_t*>(img);
    const uint32_t* whu = reinterpret_cast<const uint32_t*>(img + SG_IMG_WH);
    const uint32_t* w4u = reinterpret_cast<const uint32_t*>(img + SG_IMG_W4);
    const float* bias = reinterpret_cast<const float*>(img + SG_IMG_B);
    const float* nm = reinterpret_cast<const float*>(img + SG_IMG_N);
    const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
#pragma unroll 1
    for (int mt = 0; mt < 2; mt++) {
        const float u0 = __shfl_sync(0xffffffffu, u, mt * 16 + g), v0 = __shfl_sync(0xffffffffu, v, mt * 16 + g);
        const float u1 = __shfl_sync(0xffffffffu, u, mt * 16 + g + 8), v1 = __shfl_sync(0xffffffffu, v, mt * 16 + g + 8);
        uint32_t a[8][4];
        {
            const uint32_t a0[4] = {tq == 0 ? pack_bf16(u0, v0) : 0u, tq == 0 ? pack_bf16(u1, v1) : 0u, 0u, 0u};
            float acc[16][4];
#pragma unroll
            for (int nt = 0; nt < 16; nt++) {
                acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
                const int j = nt * 8 + g;
                mma_bf16_16816(acc[nt], a0, w0u[(j * 16 + 2 * tq) / 2], w0u[(j * 16 + 2 * tq + 8) / 2]);
            }
#pragma unroll
            for (int kt = 0; kt < 8; kt++) {
                const int c0 = (2 * kt) * 8 + 2 * tq, c1 = (2 * kt + 1) * 8 + 2 * tq;
                a[kt][0] = pack_bf16(silu(acc[2 * kt][0] + bias[c0]), silu(acc[2 * kt][1] + bias[c0 + 1]));
                a[kt][1] = pack_bf16(silu(acc[2 * kt][2] + bias[c0]), silu(acc[2 * kt][3] + bias[c0 + 1]));
                a[kt][2] = pack_bf16(silu(acc[2 * kt + 1][0] + bias[c1]), silu(acc[2 * kt + 1][1] + bias[c1 + 1]));
                a[kt][3] = pack_bf16(silu(acc[2 * kt + 1][2] + bias[c1]), silu(acc[2 * kt + 1][3] + bias[c1 + 1]));
            }
        }
#pragma unroll 1
        for (int l = 0; l < 3; l++) {
            const uint32_t* W = whu + (size_t)l * SG_H * SG_LD / 2;
            float acc[16][4];
#pragma unroll
            for (int nt = 0; nt < 16; nt++) {
                acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
                const int j = nt * 8 + g;
#pragma unroll
                for (int kt = 0; kt < 8; kt++)
                    mma_bf16_16816(acc[nt], a[kt], W[(j * SG_LD + kt * 16 + 2 * tq) / 2],
                                   W[(j * SG_LD + kt * 16 + 2 * tq + 8) / 2]);
            }
            const float* b = bias + (l + 1) * SG_H;
#pragma unroll
            for (int kt = 0; kt < 8; kt++) {
                const int c0 = (2 * kt) * 8 + 2 * tq, c1 = (2 * kt + 1) * 8 + 2 * tq;
                a[kt][0] = pack_bf16(silu(acc[2 * kt][0] + b[c0]), silu(acc[2 * kt][1] + b[c0 + 1]));
                a[kt][1] = pack_bf16(silu(acc[2 * kt][2] + b[c0]), silu(acc[2 * kt][3] + b[c0 + 1]));
                a[kt][2] = pack_bf16(silu(acc[2 * kt + 1][0] + b[c1]), silu(acc[2 * kt + 1][1] + b[c1 + 1]));
                a[kt][3] = pack_bf16(silu(acc[2 * kt + 1][2] + b[c1]), silu(acc[2 * kt + 1][3] + b[c1 + 1]));
            }
        }
        float o[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kt = 0; kt < 8; kt++)
            mma_bf16_16816(o, a[kt], w4u[(g * SG_LD + kt * 16 + 2 * tq) / 2], w4u[(g * SG_LD + kt * 16 + 2 * tq + 8) / 2]);
        // row r of the tile (lane mt * 16 + r) holds column c at lane 4 (r % 8) + c / 2, register
        // (c % 2) + 2 (r / 8)
        const int r = lane - mt * 16;
#pragma unroll
        for (int c = 0; c < SG_OUT; c++) {
            const int src = 4 * (r & 7) + c / 2;
            const float lo = __shfl_sync(0xffffffffu, o[c & 1], src & 31);
            const float hi = __shfl_sync(0xffffffffu, o[2 + (c & 1)], src & 31);
            if (r >= 0 && r < 16) out6[c] = nm[c] + nm[SG_OUT + c] * ((r < 8 ? lo : hi) + bias[4 * SG_H + c]);
        }
    }
}

// The wave term from the network's outputs: the logarithmic part in closed form (J0, J1 from the
// 1-D table), the regular part and the imaginary part from the network, FY by the identity
// FY = -F - 2 / R0.
__device__ inline Wave sg_wave(double X, double Y, const float* o) {
    double f[4];
    table1d(X, f);
    const double j0 = f[0], j1 = f[1], eY = exp(-Y), R0 = sqrt(X * X + Y * Y);
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

// The mixed-form assembly with the network as the wave term inside its domain (X, Y < 30, R0 > 0;
// the tables outside): persistent CTAs (the weight image is loaded once per CTA), work items
// (tile pair, frequency) taken round-robin; the per-item work is k_assemble's.
template <bool FINITE>
__global__ void __launch_bounds__(256, 1) k_assemble_sg(PanelsView pv, const double* __restrict__ st,
                                                       const FreqInfo* __restrict__ fi, const FdParams* __restrict__ fdp,
                                                       const float* __restrict__ tiles, const double* __restrict__ fpt,
                                                       OutF32 out, int F, const uint8_t* __restrict__ img_g,
                                                       unsigned long long* __restrict__ counts) {
    extern __shared__ __align__(16) uint8_t img[];
    __shared__ double sT[4][32][33];
    if (pv.invalid()) return;  // invalid panels: the solve reports them
    {
        const uint4* src = reinterpret_cast<const uint4*>(img_g);
        uint4* dst = reinterpret_cast<uint4*>(img);
        for (int t = threadIdx.y * 32 + threadIdx.x; t < (int)(SG_IMG_BYTES / 16); t += 256) dst[t] = src[t];
    }
    __syncthreads();
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
            const bool inb = live && X < SG_XMAX && Y < SG_XMAX && (X > 0.0 || Y > 0.0);
            float o6[SG_OUT] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            __syncwarp();
            if (__any_sync(0xffffffffu, inb)) {
                float in3[3];
                sg_inputs(X, Y, in3);
                sg_warp_mlp(img, in3[0], in3[1], o6);
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
}

void launch_sg_pack(const float* params_norm, uint8_t* img, cudaStream_t s) {
    k_sg_pack<<<64, 256, 0, s>>>(params_norm, params_norm + SG_PARAMS, img);
}

size_t sg_image_bytes() { return SG_IMG_BYTES; }

void launch_assemble_f32_sg(const PanelsView& pv, const double* st, int F, const FreqInfo* fi, const FdParams* fd,
                            const float* tiles, const double* fpt, bool finite, float* S, float* A, int Np,
                            const uint8_t* img, unsigned long long* counts, cudaStream_t s) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    OutF32 o{S, A, 2 * (size_t)Np * Np, Np};
    if (finite) {
        cudaFuncSetAttribute(k_assemble_sg<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SG_IMG_BYTES);
        k_assemble_sg<true><<<nsm, dim3(32, 8), SG_IMG_BYTES, s>>>(pv, st, fi, fd, tiles, fpt, o, F, img, counts);
    } else {
        cudaFuncSetAttribute(k_assemble_sg<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SG_IMG_BYTES);
        k_assemble_sg<false><<<nsm, dim3(32, 8), SG_IMG_BYTES, s>>>(pv, st, fi, fd, tiles, fpt, o, F, img, counts);
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
    cudaFuncSetAttribute(k_sg_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SG_SMEM);
    k_sg_infer<<<148, 256, SG_SMEM, s>>>((int)n_val, tr.p, dn, vin, vout);
    std::vector<float> ho((size_t)n_val * SG_OUT);
    std::vector<double> hv((size_t)n_val * SG_OUT);
    cudaMemcpyAsync(ho.data(), vout, ho.size() * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hv.data(), vtg, hv.size() * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(params_out, tr.p, SG_PARAMS * 4, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cudaGetLastError() != cudaSuccess) {
        *msg = "CUDA error in surrogate training";
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
    cudaFuncSetAttribute(k_sg_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SG_SMEM);
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
        k_sg_infer<<<2 * nsm, 256, SG_SMEM>>>(n, p, nm, in, o);
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
    if (cudaGetLastError() != cudaSuccess) {
        *msg = "CUDA error in the surrogate evaluation";
        return HB_ERR_INTERNAL;
    }
    return 0;
}

}  // namespace hbg
