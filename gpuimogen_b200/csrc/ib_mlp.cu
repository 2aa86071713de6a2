// ib_mlp.cu -- training kernels of the drag-decay MLP (FP32) and its exact training targets.
//
// The network (16 inputs, 3 x 64 ReLU, 1 linear output; parameter layout IB_MLP_OFF_* in
// imogen_b200.h) is trained on the GPU with these kernels: one CTA takes a tile of 64 samples,
// runs the forward pass with every activation in shared memory, back-propagates the mean squared
// error and writes that tile's gradient to its own row of a workspace; a second kernel sums the
// rows in a fixed order (so the gradient is deterministic), and an Adam kernel updates the FP32
// master parameters.  Inference in the drag step runs the same network in BF16 on the tensor
// cores (ib_drag_learned.cu).
#include "ib_drag.cuh"
#include "ib_internal.cuh"

namespace ib {

constexpr int MT = 64;    // samples per tile
constexpr int MTH = 256;  // threads per tile CTA
constexpr int H = IB_MLP_HID, IN = IB_MLP_IN;

struct MlpSmem {
    float W1[H][IN], W1T[IN][H], W2[H][H], W2T[H][H], W3[H][H], W3T[H][H];
    float b1[H], b2[H], b3[H], w4[H];
    float X[MT][IN], H1[MT][H], H2[MT][H], H3[MT][H], G1[MT][H], G2[MT][H];
    float y[MT], dy[MT];
};

__device__ void mlp_load_params(MlpSmem &s, const float *p)
{
    for (int i = threadIdx.x; i < H * IN; i += blockDim.x) {
        const int j = i / IN, k = i % IN;
        s.W1[j][k] = s.W1T[k][j] = p[IB_MLP_OFF_W1 + i];
    }
    for (int i = threadIdx.x; i < H * H; i += blockDim.x) {
        const int j = i / H, k = i % H;
        s.W2[j][k] = s.W2T[k][j] = p[IB_MLP_OFF_W2 + i];
        s.W3[j][k] = s.W3T[k][j] = p[IB_MLP_OFF_W3 + i];
    }
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        s.b1[i] = p[IB_MLP_OFF_B1 + i];
        s.b2[i] = p[IB_MLP_OFF_B2 + i];
        s.b3[i] = p[IB_MLP_OFF_B3 + i];
        s.w4[i] = p[IB_MLP_OFF_W4 + i];
    }
}

// out[r][j] = relu(b[j] + sum_k in[r][k] WT[k][j]) for rows r < rows; thread = (j, row group)
template <int K>
__device__ __forceinline__ void dense_relu(const float (*in)[K], const float (*WT)[H], const float *b, float (*out)[H],
                                           int rows)
{
    const int j = threadIdx.x % H, r0 = threadIdx.x / H, rstep = MTH / H;
    for (int r = r0; r < MT; r += rstep) {
        float acc = b[j];
#pragma unroll 16
        for (int k = 0; k < K; k++) acc = fmaf(in[r][k], WT[k][j], acc);
        out[r][j] = (r < rows && acc > 0.f) ? acc : 0.f;
    }
}

// Forward pass of one tile into shared memory; y[r] for r < rows.
__device__ void mlp_tile_forward(MlpSmem &s, const float *x, int64_t base, int rows, float b4)
{
    for (int i = threadIdx.x; i < MT * IN; i += blockDim.x) {
        const int r = i / IN, k = i % IN;
        s.X[r][k] = (r < rows) ? x[(base + r) * IN + k] : 0.f;
    }
    __syncthreads();
    dense_relu<IN>(s.X, s.W1T, s.b1, s.H1, rows);
    __syncthreads();
    dense_relu<H>(s.H1, s.W2T, s.b2, s.H2, rows);
    __syncthreads();
    dense_relu<H>(s.H2, s.W3T, s.b3, s.H3, rows);
    __syncthreads();
    // y[r] = b4 + w4 . H3[r]: one warp per row group, lanes over units
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = warp; r < MT; r += MTH / 32) {
        float acc = s.H3[r][lane] * s.w4[lane] + s.H3[r][lane + 32] * s.w4[lane + 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) s.y[r] = acc + b4;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(MTH) mlp_forward_kernel(const float *__restrict__ p, const float *__restrict__ x,
                                                           int64_t n, float *__restrict__ y)
{
    extern __shared__ __align__(16) unsigned char mlp_smem_raw[];
    MlpSmem &s = *reinterpret_cast<MlpSmem *>(mlp_smem_raw);
    mlp_load_params(s, p);
    const float b4 = p[IB_MLP_OFF_B4];
    __syncthreads();
    const int64_t ntiles = (n + MT - 1) / MT;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t base = tile * MT;
        const int rows = (int)((n - base < (int64_t)MT) ? (n - base) : (int64_t)MT);
        mlp_tile_forward(s, x, base, rows, b4);
        for (int r = threadIdx.x; r < rows; r += blockDim.x) y[base + r] = s.y[r];
        __syncthreads();
    }
}

// dW[j][k] += sum_r G[r][j] In[r][k] (thread = (k, j group)), db[j] += sum_r G[r][j]
template <int K>
__device__ __forceinline__ void dense_grad(const float (*G)[H], const float (*In)[K], float *gW, float *gb)
{
    for (int i = threadIdx.x; i < H * K; i += blockDim.x) {
        const int j = i / K, k = i % K;
        float acc = 0.f;
        for (int r = 0; r < MT; r++) acc = fmaf(G[r][j], In[r][k], acc);
        gW[i] = acc;
    }
    for (int j = threadIdx.x; j < H; j += blockDim.x) {
        float acc = 0.f;
        for (int r = 0; r < MT; r++) acc += G[r][j];
        gb[j] = acc;
    }
}

// Gout[r][k] = (sum_j Gin[r][j] W[j][k]) * (A[r][k] > 0)   (back through a ReLU layer)
__device__ __forceinline__ void dense_back(const float (*Gin)[H], const float (*W)[H], const float (*A)[H],
                                           float (*Gout)[H])
{
    const int k = threadIdx.x % H, r0 = threadIdx.x / H, rstep = MTH / H;
    for (int r = r0; r < MT; r += rstep) {
        float acc = 0.f;
#pragma unroll 16
        for (int j = 0; j < H; j++) acc = fmaf(Gin[r][j], W[j][k], acc);
        Gout[r][k] = (A[r][k] > 0.f) ? acc : 0.f;
    }
}

// One tile: forward, loss, backward; the tile's gradient goes to partial[tile][*], its summed
// squared error to partial[tile][IB_MLP_NPARAM].
__global__ void __launch_bounds__(MTH) mlp_grad_kernel(const float *__restrict__ p, const float *__restrict__ x,
                                                        const float *__restrict__ target, int64_t n,
                                                        float *__restrict__ partial, int64_t stride)
{
    extern __shared__ __align__(16) unsigned char mlp_smem_raw[];
    MlpSmem &s = *reinterpret_cast<MlpSmem *>(mlp_smem_raw);
    mlp_load_params(s, p);
    const float b4 = p[IB_MLP_OFF_B4];
    __syncthreads();
    const int64_t ntiles = (n + MT - 1) / MT;
    const float inv_n = 1.0f / (float)n;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t base = tile * MT;
        const int rows = (int)((n - base < (int64_t)MT) ? (n - base) : (int64_t)MT);
        float *gp = partial + tile * stride;
        mlp_tile_forward(s, x, base, rows, b4);
        for (int r = threadIdx.x; r < MT; r += blockDim.x) {
            const float e = (r < rows) ? s.y[r] - target[base + r] : 0.f;
            s.dy[r] = 2.f * e * inv_n;
            s.y[r] = e * e;
        }
        __syncthreads();
        // output layer: dw4[j] = sum_r dy[r] H3[r][j], db4 = sum_r dy[r], G1 = dy w4 (H3 > 0)
        for (int i = threadIdx.x; i < H * MT; i += blockDim.x) {
            const int r = i / H, j = i % H;
            s.G1[r][j] = (s.H3[r][j] > 0.f) ? s.dy[r] * s.w4[j] : 0.f;
        }
        if (threadIdx.x < H) {
            const int j = threadIdx.x;
            float acc = 0.f;
            for (int r = 0; r < MT; r++) acc = fmaf(s.dy[r], s.H3[r][j], acc);
            gp[IB_MLP_OFF_W4 + j] = acc;
        } else if (threadIdx.x == H) {
            float acc = 0.f, l = 0.f;
            for (int r = 0; r < MT; r++) {
                acc += s.dy[r];
                l += s.y[r];
            }
            gp[IB_MLP_OFF_B4] = acc;
            gp[IB_MLP_NPARAM] = l;
        }
        __syncthreads();
        dense_grad<H>(s.G1, s.H2, gp + IB_MLP_OFF_W3, gp + IB_MLP_OFF_B3);
        dense_back(s.G1, s.W3, s.H2, s.G2);
        __syncthreads();
        dense_grad<H>(s.G2, s.H1, gp + IB_MLP_OFF_W2, gp + IB_MLP_OFF_B2);
        dense_back(s.G2, s.W2, s.H1, s.G1);
        __syncthreads();
        dense_grad<IN>(s.G1, s.X, gp + IB_MLP_OFF_W1, gp + IB_MLP_OFF_B1);
        __syncthreads();
    }
}

// grad[i] = sum over tiles of partial[tile][i] in tile order; loss = sum of tile losses / n
__global__ void mlp_reduce_kernel(const float *__restrict__ partial, int64_t ntiles, int64_t stride,
                                  float *__restrict__ grad, float *__restrict__ loss, float inv_n)
{
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i > IB_MLP_NPARAM) return;
    float acc = 0.f;
    for (int64_t t = 0; t < ntiles; t++) acc += partial[t * stride + i];
    if (i < IB_MLP_NPARAM) grad[i] = acc;
    else if (loss) *loss = acc * inv_n;
}

__global__ void mlp_adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                                float *__restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                                float c2)
{
    for (int64_t i = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; i < n; i += (int64_t)blockDim.x * gridDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// Exact LogTrap2 decay exponent s = t k_eff for raw features (rho_g, rho_d, |dv|, u, dt)
__global__ void drag_decay_kernel(const double *__restrict__ f, int64_t n, DragParams d, double *__restrict__ s)
{
    for (int64_t i = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; i < n; i += (int64_t)blockDim.x * gridDim.x) {
        const double g0 = f[5 * i], d0 = f[5 * i + 1], t0 = f[5 * i + 2], t1 = f[5 * i + 3], t = f[5 * i + 4];
        s[i] = t * logtrap_keff<2>(d, g0, d0, t0, t1, t);
    }
}

static int mlp_smem_attr(const void *fn)
{
    static int done_fwd = 0, done_grad = 0;
    int &done = (fn == (const void *)mlp_forward_kernel) ? done_fwd : done_grad;
    if (done) return IB_SUCCESSFUL;
    int rc = check_cuda(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem)));
    if (rc == IB_SUCCESSFUL) done = 1;
    return rc;
}

}  // namespace ib

using namespace ib;

extern "C" int64_t ib_mlpWorkspaceFloats(int64_t n)
{
    if (n < 1) return 0;
    const int64_t stride = ((int64_t)IB_MLP_NPARAM + 1 + 7) / 8 * 8;
    return ((n + MT - 1) / MT) * stride;
}

extern "C" int ib_mlpLossGrad(const float *params, const float *x, const float *target, int64_t n, float *grad,
                              float *loss_out, float *partial, void *stream)
{
    if (!params || !x || !target || !grad || !partial) return IB_ERROR_NULL_POINTER;
    if (n < 1) return IB_ERROR_INVALID_ARGS;
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    if ((rc = mlp_smem_attr((const void *)mlp_grad_kernel))) return rc;
    const int64_t ntiles = (n + MT - 1) / MT;
    const int64_t stride = ((int64_t)IB_MLP_NPARAM + 1 + 7) / 8 * 8;
    const int grid = (int)std::min<int64_t>(ntiles, (int64_t)num_sms());
    mlp_grad_kernel<<<grid, MTH, sizeof(MlpSmem), st>>>(params, x, target, n, partial, stride);
    if ((rc = check_launch())) return rc;
    mlp_reduce_kernel<<<(IB_MLP_NPARAM + 1 + 255) / 256, 256, 0, st>>>(partial, ntiles, stride, grad, loss_out,
                                                                      1.0f / (float)n);
    return check_launch();
}

extern "C" int ib_mlpForward(const float *params, const float *x, int64_t n, float *y, void *stream)
{
    if (!params || !x || !y) return IB_ERROR_NULL_POINTER;
    if (n < 1) return IB_ERROR_INVALID_ARGS;
    int rc;
    if ((rc = mlp_smem_attr((const void *)mlp_forward_kernel))) return rc;
    const int64_t ntiles = (n + MT - 1) / MT;
    const int grid = (int)std::min<int64_t>(ntiles, (int64_t)num_sms());
    mlp_forward_kernel<<<grid, MTH, sizeof(MlpSmem), (cudaStream_t)stream>>>(params, x, n, y);
    return check_launch();
}

extern "C" int ib_mlpAdam(float *params, const float *grad, float *m, float *v, int64_t nparam, float lr, float beta1,
                          float beta2, float eps, int step, void *stream)
{
    if (!params || !grad || !m || !v) return IB_ERROR_NULL_POINTER;
    if (nparam < 1 || step < 1) return IB_ERROR_INVALID_ARGS;
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    mlp_adam_kernel<<<(unsigned)std::min<int64_t>((nparam + 255) / 256, 1024), 256, 0, (cudaStream_t)stream>>>(
        params, grad, m, v, nparam, lr, beta1, beta2, eps, c1, c2);
    return check_launch();
}

extern "C" int ib_dragDecayExact(const double *features, int64_t n, const ib_thermo *tg, const ib_thermo *td,
                                 double *s_out, void *stream)
{
    if (!features || !tg || !td || !s_out) return IB_ERROR_NULL_POINTER;
    if (n < 1) return IB_ERROR_INVALID_ARGS;
    const DragParams d = drag_constants(tg, td);
    const int nb = (int)std::min<int64_t>((n + 255) / 256, (int64_t)16 * num_sms());
    drag_decay_kernel<<<nb, 256, 0, (cudaStream_t)stream>>>(features, n, d, s_out);
    return check_launch();
}
