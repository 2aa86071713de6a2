// ib_drag_learned.cu -- the drag-decay MLP on the 5th-generation tensor cores, and the learned
// two-fluid drag step with the exact LogTrap2 integrator as fallback.
//
// One CTA = 128 threads = one tile of 128 cells = the M of one tcgen05.mma (cta_group::1,
// kind::f16, BF16 x BF16 -> FP32).  The three weight matrices sit in shared memory as BF16 in
// the no-swizzle K-major core-matrix layout (ib_tcgen05.cuh); each thread writes its cell's
// feature row, thread 0 issues the MMAs of a layer (K = 16 for the first, 4 x K = 16 for the
// others) into 64 tensor-memory columns and commits them to an mbarrier, and every thread reads
// its own accumulator row back (tcgen05.ld 32x32b), adds the bias in FP32, applies ReLU and
// writes the BF16 row of the next layer's A operand.  The 64 -> 1 output layer is a dot product in FP32.
// The update of the cell then runs in FP64 exactly as the exact integrator's (ib_drag.cuh), with
// the predicted decay exponent in place of the integrated one.
#include "ib_drag.cuh"
#include "ib_internal.cuh"
#include "ib_tcgen05.cuh"

namespace ib {

constexpr int LT = 128;  // cells per tile, threads per CTA, MMA M
constexpr int NH = IB_MLP_HID;
constexpr int KH = NH;  // hidden-layer K: the 64 activations (4 MMAs of K = 16)

// Shared memory of one CTA.  The first layer's bias rides inside its MMA: input columns 14 and 15
// of A0 hold the constant 1 and the matching weight columns the bias split into a BF16 high part
// and a BF16 remainder (about 16 significant bits together; K = 16 is the smallest MMA anyway).
// The hidden layers' biases are added in FP32 when the accumulators are read back (a bias block
// in K would cost a fifth MMA per layer).
struct LearnedSmem {
    alignas(128) unsigned char W1[NH * 16 * 2];
    alignas(128) unsigned char W2[NH * KH * 2];
    alignas(128) unsigned char W3[NH * KH * 2];
    // A0 (the first layer's [128 x 16] input) lives in the first 4 KB of A1: it is written at the
    // start of a tile, after the previous tile's last MMA has read A1, and dead once the first
    // layer's MMA has completed, before A1 is written
    alignas(128) unsigned char A1[LT * KH * 2];
    float b2[NH], b3[NH];
    double stage[9][LT];  // drag mode: the next tile's gas and dust values, fetched behind the MMAs
    float w4[NH];
    float b4;
    uint32_t tmem;
    alignas(8) uint64_t bar;
};

struct LearnedArgs {
    const float *params;
    float fshift[5], fscale[5], oshift, oscale, lo[5], hi[5];
    const float *xin;  // mode 0: n x 16 features (columns 14 and 15 are ignored)
    float *yout;       // mode 0: n outputs
    double *gas, *dust;
    int64_t S;
    DragParams d;
    double dt;
    unsigned long long *fallbacks;
    int64_t n;
    unsigned int *err;
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&h);
}

// two FP32 lanes at once (packed f32x2 arithmetic of sm_100)
__device__ __forceinline__ float2 add2(float2 a, float2 b)
{
    unsigned long long x = *reinterpret_cast<unsigned long long *>(&a), y = *reinterpret_cast<unsigned long long *>(&b), z;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(z) : "l"(x), "l"(y));
    return *reinterpret_cast<float2 *>(&z);
}

__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
    unsigned long long x = *reinterpret_cast<unsigned long long *>(&a), y = *reinterpret_cast<unsigned long long *>(&b),
                       z = *reinterpret_cast<unsigned long long *>(&c);
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(z) : "l"(x), "l"(y));
    return *reinterpret_cast<float2 *>(&z);
}

// relu(lo), relu(hi) -> BF16x2 in one conversion (lo in the low half)
__device__ __forceinline__ uint32_t relu_bf16x2(float lo, float hi)
{
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

__device__ __forceinline__ void store_bf16x8(unsigned char *dst, const float *v)
{
    uint4 u;
    u.x = pack_bf16x2(v[0], v[1]);
    u.y = pack_bf16x2(v[2], v[3]);
    u.z = pack_bf16x2(v[4], v[5]);
    u.w = pack_bf16x2(v[6], v[7]);
    *reinterpret_cast<uint4 *>(dst) = u;
}

__device__ __forceinline__ void put_bf16(unsigned char *base, uint32_t off, float v)
{
    *reinterpret_cast<__nv_bfloat16 *>(base + off) = __float2bfloat16_rn(v);
}

// Weight matrix [64 out][K] -> BF16 core-matrix layout; with a bias, split into columns bcol and
// bcol + 1
__device__ void load_weights(unsigned char *W, const float *src, int kin, int K, int bcol, const float *bias)
{
    for (int i = threadIdx.x; i < NH * K; i += blockDim.x) {
        const int j = i / K, k = i % K;
        float v = 0.f;
        if (k < kin) v = src[j * kin + k];
        if (bias && (k == bcol || k == bcol + 1)) {
            const float b = bias[j];
            const float hi = __bfloat162float(__float2bfloat16_rn(b));
            v = (k == bcol) ? hi : b - hi;
        }
        put_bf16(W, core_offset(j, k, K), v);
    }
}

// this thread's accumulator row (16 columns at a time) + bias (none for the first layer, whose
// bias is inside its MMA) -> ReLU -> BF16 row r of A1
__device__ __forceinline__ void hidden_to_a1(unsigned char *A1, int r, uint32_t taddr, const float *bias)
{
#pragma unroll
    for (int c = 0; c < NH; c += 16) {
        float h[16];
        tmem_ld16(taddr + c, h);
        tmem_wait_ld();
        if (bias) {
#pragma unroll
            for (int j = 0; j < 16; j += 2) {
                const float2 r = add2(make_float2(h[j], h[j + 1]), *reinterpret_cast<const float2 *>(bias + c + j));
                h[j] = r.x;
                h[j + 1] = r.y;
            }
        }
        uint4 u0, u1;
        u0.x = relu_bf16x2(h[0], h[1]);
        u0.y = relu_bf16x2(h[2], h[3]);
        u0.z = relu_bf16x2(h[4], h[5]);
        u0.w = relu_bf16x2(h[6], h[7]);
        u1.x = relu_bf16x2(h[8], h[9]);
        u1.y = relu_bf16x2(h[10], h[11]);
        u1.z = relu_bf16x2(h[12], h[13]);
        u1.w = relu_bf16x2(h[14], h[15]);
        *reinterpret_cast<uint4 *>(A1 + core_offset(r, c, KH)) = u0;
        *reinterpret_cast<uint4 *>(A1 + core_offset(r, c + 8, KH)) = u1;
    }
}

// All threads: make this thread's shared-memory writes visible to the tensor cores and order its
// tensor-memory accesses, then a CTA barrier that also agrees on `ok`.
__device__ __forceinline__ bool tc_sync(bool ok)
{
    fence_proxy_async_smem();
    tc_fence_before();
    ok = __syncthreads_and(ok);
    tc_fence_after();
    return ok;
}

// Learned-path update: the exact integrator's momentum exchange and gas heating (drag_apply) with
// decay factor exp(-s), written with one reciprocal per density instead of per-axis divisions.
__device__ __forceinline__ void drag_apply_learned(double *g, double *ds, int64_t S, double g0, double gE,
                                                   const double gm[3], double d0, const double dm[3],
                                                   const double dvv[3], double rdi, double decay)
{
    const double rsum = 1.0 / (g0 + d0);
    const double mu = g0 * d0 * rsum;
    double pd = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double vstick = (gm[k] + dm[k]) * rsum;
        const double dvt = dvv[k] * decay;
        const double q = d0 * vstick - dvt * mu;
        g[(2 + k) * S] = g0 * vstick + dvt * mu;
        ds[(2 + k) * S] = q;
        pd += q * q - dm[k] * dm[k];
    }
    g[S] = gE - .5 * pd * rdi;
}

// Drag mode: start copying the nine gas/dust values of cell i into this thread's column of the
// stage (asynchronous copies, waited for by the same thread before it reads them).
__device__ __forceinline__ void stage_cell(LearnedSmem &s, const LearnedArgs &a, int64_t i)
{
    const int tid = threadIdx.x;
    const double *src[9] = {a.gas + i, a.gas + i + a.S, a.gas + i + 2 * a.S, a.gas + i + 3 * a.S,
                            a.gas + i + 4 * a.S, a.dust + i, a.dust + i + 2 * a.S, a.dust + i + 3 * a.S,
                            a.dust + i + 4 * a.S};
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&s.stage[k][tid]);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src[k]) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <int MODE>
__global__ void __launch_bounds__(LT, 5) mlp_tc_kernel(LearnedArgs a)
{
    extern __shared__ __align__(1024) unsigned char learned_smem_raw[];
    LearnedSmem &s = *reinterpret_cast<LearnedSmem *>(learned_smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    const float *p = a.params;
    load_weights(s.W1, p + IB_MLP_OFF_W1, 16, 16, 14, p + IB_MLP_OFF_B1);
    load_weights(s.W2, p + IB_MLP_OFF_W2, NH, KH, -1, nullptr);
    load_weights(s.W3, p + IB_MLP_OFF_W3, NH, KH, -1, nullptr);
    for (int i = tid; i < NH; i += LT) {
        s.w4[i] = p[IB_MLP_OFF_W4 + i];
        s.b2[i] = p[IB_MLP_OFF_B2 + i];
        s.b3[i] = p[IB_MLP_OFF_B3 + i];
    }
    if (tid == 0) {
        s.b4 = p[IB_MLP_OFF_B4];
        mbar_init(&s.bar, 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(&s.tmem, NH);
    tc_sync(true);
    const uint32_t tmem = s.tmem;
    const uint32_t my_row = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t id = idesc_bf16_f32(LT, NH);
    unsigned char *const A0 = s.A1;
    const uint64_t dA0 = smem_desc(A0, 128, 256), dW1 = smem_desc(s.W1, 128, 256);
    uint32_t phase = 0;
    bool ok = true;
    const int64_t ntiles = (a.n + LT - 1) / LT;
    if (MODE == 1 && (int64_t)blockIdx.x * LT + tid < a.n) stage_cell(s, a, (int64_t)blockIdx.x * LT + tid);

    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t i = tile * LT + tid;
        const bool live = i < a.n;
        // ---- features: columns 0..13 (drag: 0..4), 14 and 15 = 1 for the bias ----
        float f[16];
#pragma unroll
        for (int k = 0; k < 16; k++) f[k] = 0.f;
        bool indom = live;
        double g0 = 1, gE = 0, d0 = 1, gm[3] = {0, 0, 0}, dm[3] = {0, 0, 0}, dvv[3] = {0, 0, 0}, rdi = 1, magdv = 0;
        if (MODE == 0) {
            if (live)
                for (int k = 0; k < 14; k++) f[k] = a.xin[i * IB_MLP_IN + k];
        } else if (live) {
            stage_wait();
            g0 = s.stage[0][tid]; gE = s.stage[1][tid];
            d0 = s.stage[5][tid];
#pragma unroll
            for (int k = 0; k < 3; k++) { gm[k] = s.stage[2 + k][tid]; dm[k] = s.stage[6 + k][tid]; }
            // the next tile's values stream in behind this tile's MMAs and update
            const int64_t inext = i + (int64_t)gridDim.x * LT;
            if (inext < a.n) stage_cell(s, a, inext);
            const double rgi = 1.0 / g0;
            rdi = 1.0 / d0;
            double dvsq = 0, momsq = 0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                dvv[k] = gm[k] * rgi - dm[k] * rdi;
                dvsq += dvv[k] * dvv[k];
                momsq += gm[k] * gm[k];
            }
            magdv = sqrt(dvsq);
            const double u = (gE - .5 * momsq * rgi) * rgi;
            const float raw[5] = {logf((float)g0), logf((float)d0), logf((float)magdv), logf((float)u),
                                  logf((float)a.dt)};
#pragma unroll
            for (int k = 0; k < 5; k++) {
                indom = indom && (raw[k] >= a.lo[k]) && (raw[k] <= a.hi[k]);
                f[k] = (raw[k] - a.fshift[k]) * a.fscale[k];
            }
            if (!indom || magdv < 1e-9) {
#pragma unroll
                for (int k = 0; k < 5; k++) f[k] = 0.f;
            }
        }
        f[14] = 1.f;
        f[15] = 1.f;
        store_bf16x8(A0 + core_offset(tid, 0, 16), f);
        store_bf16x8(A0 + core_offset(tid, 8, 16), f + 8);
        ok = tc_sync(ok);
        if (!ok) break;
        // ---- layer 1: [128 x 16] x [16 -> 64], bias in columns 14-15 ----
        if (tid == 0) {
            tc_mma_bf16(tmem, dA0, dW1, id, 0);
            tc_commit(&s.bar);
        }
        ok = mbar_wait(&s.bar, phase);
        phase ^= 1;
        tc_fence_after();
        hidden_to_a1(s.A1, tid, my_row, nullptr);
        ok = tc_sync(ok);
        if (!ok) break;
        // ---- layers 2 and 3: [128 x 64] x [64 -> 64] as 4 MMAs of K = 16 ----
        for (int layer = 0; layer < 2; layer++) {
            const unsigned char *W = layer ? s.W3 : s.W2;
            if (tid == 0) {
#pragma unroll
                for (int kk = 0; kk < KH / 16; kk++)
                    tc_mma_bf16(tmem, smem_desc(s.A1 + kk * 256, 128, KH * 16), smem_desc(W + kk * 256, 128, KH * 16),
                                id, kk > 0);
                tc_commit(&s.bar);
            }
            ok = mbar_wait(&s.bar, phase);
            phase ^= 1;
            tc_fence_after();
            if (layer == 0) {
                hidden_to_a1(s.A1, tid, my_row, s.b2);
                ok = tc_sync(ok);
                if (!ok) break;
            }
        }
        if (!ok) break;
        // ---- output: y = b4 + w4 . relu(h3) (FP32, straight from tensor memory) ----
        float2 y2 = make_float2(0.f, 0.f);  // even and odd hidden units
#pragma unroll
        for (int c = 0; c < NH; c += 16) {
            float h[16];
            tmem_ld16(my_row + c, h);
            tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < 16; j += 2) {
                float2 z = add2(make_float2(h[j], h[j + 1]), *reinterpret_cast<const float2 *>(s.b3 + c + j));
                z.x = fmaxf(z.x, 0.f);
                z.y = fmaxf(z.y, 0.f);
                y2 = fma2(*reinterpret_cast<const float2 *>(s.w4 + c + j), z, y2);
            }
        }
        const float y = s.b4 + (y2.x + y2.y);
        if (MODE == 0) {
            if (live) a.yout[i] = y;
        } else {
            bool fb = false;
            if (live) {
                double decay = 1.0;
                if (magdv < 1e-9) {
                    fb = true;  // the exact integrator's no-drag cut: let it handle the cell
                } else if (indom) {
                    // FP32 exponentials: their 1e-7 relative error is far below the network's
                    const float sp = expf(a.oshift + a.oscale * y);
                    if (isfinite(sp)) decay = (double)expf(-sp);
                    else fb = true;
                } else {
                    fb = true;
                }
                double *g = a.gas + i, *ds = a.dust + i;
                if (fb) {
                    const double g2 = gm[0], g3 = gm[1], g4 = gm[2], d2 = dm[0], d3 = dm[1], d4 = dm[2];
                    double t0, t1;
                    drag_features(g0, gE, g2, g3, g4, d0, d2, d3, d4, t0, t1);
                    const double k = logtrap_keff<2>(a.d, g0, d0, t0, t1, a.dt);
                    drag_apply(g, ds, a.S, g0, gE, g2, g3, g4, d0, d2, d3, d4, a.dt, k);
                } else {
                    drag_apply_learned(g, ds, a.S, g0, gE, gm, d0, dm, dvv, rdi, decay);
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, fb && magdv >= 1e-9);
            if ((tid & 31) == 0 && m && a.fallbacks) atomicAdd(a.fallbacks, (unsigned long long)__popc(m));
        }
        // every thread's tensor-memory reads are done before the next tile's MMAs overwrite them
        tc_fence_before();
    }
    if (MODE == 1) stage_wait();  // no copy into shared memory outlives the CTA (early exit)
    if (!ok && tid == 0) {
        atomicOr(a.err, 2u);
        mbar_wait(&s.bar, phase ^ 1);  // one more bounded wait for a late MMA before freeing its columns
    }
    tc_sync(true);
    if (warp == 0) tmem_dealloc(tmem, NH);
}

static void fill_model(LearnedArgs &a, const ib_drag_model *m)
{
    a.params = m->params;
    for (int k = 0; k < 5; k++) {
        a.fshift[k] = m->feature_shift[k];
        a.fscale[k] = m->feature_scale[k];
        a.lo[k] = m->domain_lo[k];
        a.hi[k] = m->domain_hi[k];
    }
    a.oshift = m->out_shift;
    a.oscale = m->out_scale;
}

template <int MODE>
static int launch_mlp_tc(const LearnedArgs &a, cudaStream_t st)
{
    auto kern = mlp_tc_kernel<MODE>;
    const size_t shm = sizeof(LearnedSmem);
    static bool attr = false;
    int rc;
    if (!attr) {
        if ((rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm))))
            return rc;
        if ((rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100))))
            return rc;
        attr = true;
    }
    // A CTA walks its tiles to the end, so the grid is what fits at once: counted here from the
    // registers and shared memory (the occupancy query reports 1 for this kernel), at most 8
    // (8 x 64 tensor-memory columns are all 512 of an SM).
    static int per_sm = 0;
    if (per_sm == 0) {
        cudaFuncAttributes fa;
        int dev = 0, smem_sm = 0, resv = 0;
        if ((rc = check_cuda(cudaFuncGetAttributes(&fa, kern)))) return rc;
        if ((rc = check_cuda(cudaGetDevice(&dev)))) return rc;
        if ((rc = check_cuda(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev))))
            return rc;
        if ((rc = check_cuda(cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev)))) return rc;
        const int regs = (fa.numRegs + 7) / 8 * 8;
        const int by_regs = 65536 / std::max(1, regs * LT);
        const int by_smem = smem_sm / (int)(shm + fa.sharedSizeBytes + resv);
        per_sm = std::max(1, std::min(std::min(by_regs, by_smem), 8));
    }
    const int64_t ntiles = (a.n + LT - 1) / LT;
    const unsigned grid = (unsigned)std::min<int64_t>(ntiles, (int64_t)per_sm * num_sms());
    kern<<<grid, LT, shm, st>>>(a);
    return check_launch();
}

}  // namespace ib

using namespace ib;

extern "C" int ib_mlpInferTC(const float *params, const float *x, int64_t n, float *y, void *stream)
{
    if (!params || !x || !y) return IB_ERROR_NULL_POINTER;
    if (n < 1) return IB_ERROR_INVALID_ARGS;
    LearnedArgs a = {};
    a.params = params;
    a.xin = x;
    a.yout = y;
    a.n = n;
    a.err = scratch().wait_flag();
    if (!a.err) return IB_ERROR_NOMEM;
    return launch_mlp_tc<0>(a, (cudaStream_t)stream);
}

extern "C" int ib_cudaSource2FluidDragLearned(ib_fluid *gas, ib_fluid *dust, const ib_thermo *tg, const ib_thermo *td,
                                              const ib_drag_model *model, double dt,
                                              unsigned long long *fallback_count, void *stream)
{
    if (!gas || !dust || !tg || !td || !model || !model->params || !gas->q || !dust->q) return IB_ERROR_NULL_POINTER;
    if (gas->grid.nx != dust->grid.nx || gas->grid.ny != dust->grid.ny || gas->grid.nz != dust->grid.nz ||
        gas->grid.slab_pitch != dust->grid.slab_pitch)
        return IB_ERROR_INVALID_ARGS;
    const int64_t n = (int64_t)gas->grid.nx * gas->grid.ny * gas->grid.nz;
    if (n < 1 || gas->grid.slab_pitch < n) return IB_ERROR_INVALID_ARGS;
    LearnedArgs a = {};
    fill_model(a, model);
    a.gas = gas->q;
    a.dust = dust->q;
    a.S = gas->grid.slab_pitch;
    a.d = drag_constants(tg, td);
    a.dt = dt;
    a.fallbacks = fallback_count;
    a.n = n;
    a.err = scratch().wait_flag();
    if (!a.err) return IB_ERROR_NOMEM;
    return launch_mlp_tc<1>(a, (cudaStream_t)stream);
}
