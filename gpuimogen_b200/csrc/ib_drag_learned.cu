// ib_drag_learned.cu -- the drag-decay MLP on the 5th-generation tensor cores, and the learned
// two-fluid drag step with the exact LogTrap2 integrator as fallback.
//
// One CTA = 128 threads = one tile of 128 cells = the M of one tcgen05.mma (cta_group::1,
// kind::f16, BF16 x BF16 -> FP32).  The three weight matrices sit in shared memory as BF16 in
// the no-swizzle K-major core-matrix layout (ib_tcgen05.cuh); each thread writes its cell's
// feature row, thread 0 issues the MMAs of a layer (K = 16 for the first, 4 x K = 16 for the
// others) into 64 tensor-memory columns and commits them to an mbarrier, and every thread reads
// its own accumulator row back (tcgen05.ld 32x32b), adds the bias, applies ReLU and writes the
// BF16 row of the next layer's A operand.  The 64 -> 1 output layer is a dot product in FP32.
// The update of the cell then runs in FP64 exactly as the exact integrator's (ib_drag.cuh), with
// the predicted decay exponent in place of the integrated one.
#include "ib_drag.cuh"
#include "ib_internal.cuh"
#include "ib_tcgen05.cuh"

namespace ib {

constexpr int LT = 128;  // cells per tile, threads per CTA, MMA M
constexpr int NH = IB_MLP_HID;

struct LearnedSmem {
    alignas(128) unsigned char W1[NH * 16 * 2];
    alignas(128) unsigned char W2[NH * NH * 2];
    alignas(128) unsigned char W3[NH * NH * 2];
    alignas(128) unsigned char A0[LT * 16 * 2];
    alignas(128) unsigned char A1[LT * NH * 2];
    float b1[NH], b2[NH], b3[NH], w4[NH];
    float b4;
    uint32_t tmem;
    alignas(8) uint64_t bar;
};

struct LearnedArgs {
    const float *params;
    float fshift[5], fscale[5], oshift, oscale, lo[5], hi[5];
    const float *xin;  // mode 0: n x 16 features
    float *yout;       // mode 0: n outputs
    double *gas, *dust;
    int64_t S;
    DragParams d;
    double dt;
    unsigned long long *fallbacks;
    int64_t n;
    unsigned int *err;
};

__device__ __forceinline__ void store_bf16x8(unsigned char *dst, const float *v)
{
    uint4 u;
    __nv_bfloat162 h0 = __floats2bfloat162_rn(v[0], v[1]), h1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 h2 = __floats2bfloat162_rn(v[4], v[5]), h3 = __floats2bfloat162_rn(v[6], v[7]);
    u.x = *reinterpret_cast<uint32_t *>(&h0);
    u.y = *reinterpret_cast<uint32_t *>(&h1);
    u.z = *reinterpret_cast<uint32_t *>(&h2);
    u.w = *reinterpret_cast<uint32_t *>(&h3);
    *reinterpret_cast<uint4 *>(dst) = u;
}

// bias + ReLU of this thread's 64 accumulators -> BF16 row r of A1 (K = 64)
__device__ __forceinline__ void hidden_to_a1(unsigned char *A1, int r, float *h, const float *b)
{
#pragma unroll
    for (int g = 0; g < 8; g++) {
        float v[8];
#pragma unroll
        for (int e = 0; e < 8; e++) v[e] = fmaxf(h[8 * g + e] + b[8 * g + e], 0.f);
        store_bf16x8(A1 + core_offset(r, 8 * g, NH), v);
    }
}

__device__ __forceinline__ void tmem_row64(uint32_t taddr, float *h)
{
    tmem_ld16(taddr, h);
    tmem_ld16(taddr + 16, h + 16);
    tmem_ld16(taddr + 32, h + 32);
    tmem_ld16(taddr + 48, h + 48);
    tmem_wait_ld();
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

template <int MODE>
__global__ void __launch_bounds__(LT, 4) mlp_tc_kernel(LearnedArgs a)
{
    extern __shared__ __align__(1024) unsigned char learned_smem_raw[];
    LearnedSmem &s = *reinterpret_cast<LearnedSmem *>(learned_smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    const float *p = a.params;
    for (int i = tid; i < NH * 16; i += LT) {
        const int j = i / 16, k = i % 16;
        *reinterpret_cast<__nv_bfloat16 *>(s.W1 + core_offset(j, k, 16)) = __float2bfloat16_rn(p[IB_MLP_OFF_W1 + i]);
    }
    for (int i = tid; i < NH * NH; i += LT) {
        const int j = i / NH, k = i % NH;
        *reinterpret_cast<__nv_bfloat16 *>(s.W2 + core_offset(j, k, NH)) = __float2bfloat16_rn(p[IB_MLP_OFF_W2 + i]);
        *reinterpret_cast<__nv_bfloat16 *>(s.W3 + core_offset(j, k, NH)) = __float2bfloat16_rn(p[IB_MLP_OFF_W3 + i]);
    }
    for (int i = tid; i < NH; i += LT) {
        s.b1[i] = p[IB_MLP_OFF_B1 + i];
        s.b2[i] = p[IB_MLP_OFF_B2 + i];
        s.b3[i] = p[IB_MLP_OFF_B3 + i];
        s.w4[i] = p[IB_MLP_OFF_W4 + i];
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
    uint32_t phase = 0;
    bool ok = true;
    const int64_t ntiles = (a.n + LT - 1) / LT;
    float h[NH];

    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t i = tile * LT + tid;
        const bool live = i < a.n;
        // ---- features ----
        float f[16];
#pragma unroll
        for (int k = 0; k < 16; k++) f[k] = 0.f;
        bool indom = live;
        double g0 = 1, gE = 0, g2 = 0, g3 = 0, g4 = 0, d0 = 1, d2 = 0, d3 = 0, d4 = 0, magdv = 0, u = 0;
        if (MODE == 0) {
            if (live)
                for (int k = 0; k < IB_MLP_IN; k++) f[k] = a.xin[i * IB_MLP_IN + k];
        } else if (live) {
            double *g = a.gas + i, *ds = a.dust + i;
            g0 = g[0]; gE = g[a.S]; g2 = g[2 * a.S]; g3 = g[3 * a.S]; g4 = g[4 * a.S];
            d0 = ds[0]; d2 = ds[2 * a.S]; d3 = ds[3 * a.S]; d4 = ds[4 * a.S];
            drag_features(g0, gE, g2, g3, g4, d0, d2, d3, d4, magdv, u);
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
        store_bf16x8(s.A0 + core_offset(tid, 0, 16), f);
        store_bf16x8(s.A0 + core_offset(tid, 8, 16), f + 8);
        ok = tc_sync(ok);
        if (!ok) break;
        // ---- layer 1: [128 x 16] x [16 -> 64] ----
        if (tid == 0) {
            tc_mma_bf16(tmem, smem_desc(s.A0, 128, 256), smem_desc(s.W1, 128, 256), id, 0);
            tc_commit(&s.bar);
        }
        ok = mbar_wait(&s.bar, phase);
        phase ^= 1;
        tc_fence_after();
        tmem_row64(my_row, h);
        hidden_to_a1(s.A1, tid, h, s.b1);
        ok = tc_sync(ok);
        if (!ok) break;
        // ---- layers 2 and 3: [128 x 64] x [64 -> 64] as 4 MMAs of K = 16 ----
        for (int layer = 0; layer < 2; layer++) {
            const unsigned char *W = layer ? s.W3 : s.W2;
            if (tid == 0) {
#pragma unroll
                for (int kk = 0; kk < 4; kk++)
                    tc_mma_bf16(tmem, smem_desc(s.A1 + kk * 256, 128, 1024), smem_desc(W + kk * 256, 128, 1024), id,
                                kk > 0);
                tc_commit(&s.bar);
            }
            ok = mbar_wait(&s.bar, phase);
            phase ^= 1;
            tc_fence_after();
            tmem_row64(my_row, h);
            if (layer == 0) hidden_to_a1(s.A1, tid, h, s.b2);
            ok = tc_sync(ok);
            if (!ok) break;
        }
        if (!ok) break;
        // ---- output: y = b4 + w4 . relu(h + b3) ----
        float y = s.b4;
#pragma unroll
        for (int j = 0; j < NH; j++) y = fmaf(s.w4[j], fmaxf(h[j] + s.b3[j], 0.f), y);
        if (MODE == 0) {
            if (live) a.yout[i] = y;
        } else {
            double k_use = 0.0, t_use = 1.0;
            bool fb = false;
            if (live) {
                if (magdv < 1e-9) {
                    k_use = 0.0;  // the exact integrator's no-drag cut
                } else if (indom) {
                    const float sp = expf(a.oshift + a.oscale * y);
                    if (isfinite(sp)) k_use = (double)sp;
                    else fb = true;
                } else {
                    fb = true;
                }
                if (fb) {
                    k_use = logtrap_keff<2>(a.d, g0, d0, magdv, u, a.dt);
                    t_use = a.dt;
                }
                drag_apply(a.gas + i, a.dust + i, a.S, g0, gE, g2, g3, g4, d0, d2, d3, d4, t_use, k_use);
            }
            const unsigned m = __ballot_sync(0xffffffffu, fb);
            if ((tid & 31) == 0 && m && a.fallbacks) atomicAdd(a.fallbacks, (unsigned long long)__popc(m));
        }
    }
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
    int per_sm = 0;
    if ((rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, LT, shm)))) return rc;
    // 4 CTAs of 128 threads fit by registers and shared memory; 8 x 64 tensor-memory columns are
    // all 512 of an SM.  CTAs never wait on each other, so a grid above residency only queues.
    per_sm = std::max(4, std::min(per_sm, 8));
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
