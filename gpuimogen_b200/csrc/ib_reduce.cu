// ib_reduce.cu -- soundspeed, CFL timestep reduction and freezeAndPtot.
//
// The reference computes the CFL limit in three steps: a soundspeed pass that writes c_s
// (gpuclass/cudaSoundspeed.cu:178-193), a reduction kernel that reads the fluid and c_s and
// leaves at most 128 block minima in pinned host memory (cflTimestep.cu:276-377), then a host
// loop, MPI_Allreduce and the HLL/HLLC halving (:204-237).  Here the fused variant computes c_s
// inline, reduces with warp shuffles, and the last block to finish folds the block minima and
// applies the halving on the device, so the timestep can stay on the GPU.
#include <cstdio>
#include <mutex>

#include <cuda.h>

#include "ib_cfl.cuh"
#include "ib_internal.cuh"

namespace ib {

__global__ void soundspeed_kernel(const double *__restrict__ q, int64_t slab, int64_t n, double gg1,
                                  double *__restrict__ cs)
{
    for (int64_t x = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; x < n; x += (int64_t)blockDim.x * gridDim.x) {
        cs[x] = soundspeed_cell(q[x], q[x + slab], q[x + 2 * slab], q[x + 3 * slab], q[x + 4 * slab], gg1);
    }
}

// The cells one pass of the CFL loop reads: U cells a grid stride apart, every load issued before
// the arithmetic, so that a thread keeps U cells' loads in flight (the minimum does not depend on
// the order in which the cells are visited).
constexpr int kCflUnroll = 2;

template <int SIM, bool XJ, bool FUSED, bool CYL = false>
__global__ void __launch_bounds__(256) cfl_kernel(const double *__restrict__ q, const double *__restrict__ cs_in,
                                                  int64_t slab, int64_t n, double gg1, double hmin, double hx,
                                                  double hy, double hz, int halve, double *__restrict__ partial,
                                                  unsigned int *__restrict__ counter, double *__restrict__ tau_out,
                                                  int nx = 1, double rin = 0.0)
{
    double tmin = 1e37;
    const int64_t stride = (int64_t)blockDim.x * gridDim.x;
    constexpr bool NEED_E = FUSED, NEED_PY = FUSED || SIM > 1 || XJ, NEED_PZ = FUSED || SIM > 2 || XJ;
    int64_t x0 = threadIdx.x + (int64_t)blockIdx.x * blockDim.x;
    for (; x0 < n; x0 += kCflUnroll * stride) {
        double rho[kCflUnroll], E[kCflUnroll], px[kCflUnroll], py[kCflUnroll], pz[kCflUnroll], cs[kCflUnroll];
#pragma unroll
        for (int u = 0; u < kCflUnroll; u++) {
            const int64_t x = x0 + u * stride;
            const bool in = (u == 0) || x < n;
            rho[u] = in ? q[x] : 1.0;
            px[u] = in ? q[x + 2 * slab] : 0.0;
            E[u] = (NEED_E && in) ? q[x + slab] : 0.0;
            py[u] = (NEED_PY && in) ? q[x + 3 * slab] : 0.0;
            pz[u] = (NEED_PZ && in) ? q[x + 4 * slab] : 0.0;
            if constexpr (!FUSED) cs[u] = in ? cs_in[x] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kCflUnroll; u++) {
            const int64_t x = x0 + u * stride;
            if (u > 0 && x >= n) break;
            if constexpr (FUSED) cs[u] = soundspeed_cell(rho[u], E[u], px[u], py[u], pz[u], gg1);
            // the cell's own velocity terms: a sweep dimension the grid lacks contributes nothing
            const double vy = (SIM > 1 || XJ) ? py[u] : 0.0, vz = (SIM > 2 || XJ) ? pz[u] : 0.0;
            if constexpr (CYL)
                tmin = min_keep(tmin, cfl_cell_cyl<SIM, XJ>(rho[u], px[u], vy, vz, cs[u], hmin, hx, hy, hz, rin,
                                                            (int)(x % nx)));
            else
                tmin = min_keep(tmin, cfl_cell<SIM, XJ>(rho[u], px[u], vy, vz, cs[u], hmin, hx, hy, hz));
        }
    }
    // warp then block reduction
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tmin = min_keep(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
    __shared__ double wmin[8];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) wmin[wid] = tmin;
    __syncthreads();
    if (wid == 0) {
        tmin = (lane < (int)(blockDim.x >> 5)) ? wmin[lane] : 1e37;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tmin = min_keep(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
        if (lane == 0) {
            partial[blockIdx.x] = tmin;
            __threadfence();
            unsigned int done = atomicAdd(counter, 1u);
            last = (done == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (last) {
        // final fold of the block minima by the last block (reads see all blocks' writes after
        // their fences and the counter)
        __threadfence();
        double m = 1e37;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) m = min_keep(m, ((volatile double *)partial)[b]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = min_keep(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) wmin[wid] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            double r = 1e38;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) r = (wmin[w] < r) ? wmin[w] : r;
            if (halve) r = r / 2;  // HLL/HLLC (cflTimestep.cu:232-237)
            *tau_out = r;
            *counter = 0u;  // ready for the next call on this stream
        }
    }
}

// Blocks of the allocating CFL launch: as many as are resident at once (the loop strides over the
// cells, so a second wave would only add a tail), at most one per 256 cells.
template <int S, bool X, bool F, bool C>
static int cfl_grid(int64_t n)
{
    static const int per_sm = [] {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, cfl_kernel<S, X, F, C>, 256, 0) != cudaSuccess || b < 1)
            b = 4;
        return b;
    }();
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)per_sm * num_sms()));
}

int launch_cfl(const double *q, const double *cs, int64_t slab, const int grid[3], const ib_geometry *geo,
               int method, double gamma, double *tau_dev, cudaStream_t st)
{
    int sim = 1;
    if (geo->global_rez[1] > 1) sim = 2;
    if (geo->global_rez[2] > 1) sim = 3;
    const bool cyl = (geo->shape == IB_GEOMETRY_CYLINDRICAL);
    // the reference's kernel table (cflTimestep.cu:175-193): square 1-D Xin-Jin takes the HLLC
    // form (case 12), cylindrical 1-D Xin-Jin the Xin-Jin form (case 15)
    const bool xj = (method == IB_METHOD_XINJIN) && (sim > 1 || cyl);
    double hmin = geo->h[0];
    if (cyl) {
        if (sim == 3) hmin = (hmin < geo->h[2]) ? hmin : geo->h[2];  // dr, dz (cflTimestep.cu:301-304)
    } else {
        if (sim > 1 && geo->h[1] < hmin) hmin = geo->h[1];
        if (sim > 2 && geo->h[2] < hmin) hmin = geo->h[2];
    }
    int64_t n = (int64_t)grid[0] * grid[1] * grid[2];
    Scratch &sc = scratch();
    unsigned int *counter = sc.cfl_counter();
    if (!counter) return IB_ERROR_NOMEM;
    int halve = (method == IB_METHOD_HLL || method == IB_METHOD_HLLC) ? 1 : 0;
    double gg1 = gamma * (gamma - 1);
    bool fused = (cs == nullptr);
#define IB_CFL_LAUNCH_C(S, X, F, C)                                                                          \
    do {                                                                                                     \
        const int nb = cfl_grid<S, X, F, C>(n);                                                              \
        double *partial = sc.cfl_partial(nb);                                                                \
        if (!partial) return IB_ERROR_NOMEM;                                                                 \
        cfl_kernel<S, X, F, C><<<nb, 256, 0, st>>>(q, cs, slab, n, gg1, hmin, geo->h[0], geo->h[1], geo->h[2],  \
                                                   halve, partial, counter, tau_dev, grid[0], geo->r_inner);    \
    } while (0)
#define IB_CFL_LAUNCH(S, X, F) IB_CFL_LAUNCH_C(S, X, F, false)
    if (cyl && fused) {
        if (xj) {
            if (sim == 1) IB_CFL_LAUNCH_C(1, true, true, true);
            else if (sim == 2) IB_CFL_LAUNCH_C(2, true, true, true);
            else IB_CFL_LAUNCH_C(3, true, true, true);
        }
        else if (sim == 1) IB_CFL_LAUNCH_C(1, false, true, true);
        else if (sim == 2) IB_CFL_LAUNCH_C(2, false, true, true);
        else IB_CFL_LAUNCH_C(3, false, true, true);
    } else if (cyl) {
        if (xj) {
            if (sim == 1) IB_CFL_LAUNCH_C(1, true, false, true);
            else if (sim == 2) IB_CFL_LAUNCH_C(2, true, false, true);
            else IB_CFL_LAUNCH_C(3, true, false, true);
        }
        else if (sim == 1) IB_CFL_LAUNCH_C(1, false, false, true);
        else if (sim == 2) IB_CFL_LAUNCH_C(2, false, false, true);
        else IB_CFL_LAUNCH_C(3, false, false, true);
    } else if (fused) {
        if (xj) { if (sim == 2) IB_CFL_LAUNCH(2, true, true); else IB_CFL_LAUNCH(3, true, true); }
        else if (sim == 1) IB_CFL_LAUNCH(1, false, true);
        else if (sim == 2) IB_CFL_LAUNCH(2, false, true);
        else IB_CFL_LAUNCH(3, false, true);
    } else {
        if (xj) { if (sim == 2) IB_CFL_LAUNCH(2, true, false); else IB_CFL_LAUNCH(3, true, false); }
        else if (sim == 1) IB_CFL_LAUNCH(1, false, false);
        else if (sim == 2) IB_CFL_LAUNCH(2, false, false);
        else IB_CFL_LAUNCH(3, false, false);
    }
#undef IB_CFL_LAUNCH
#undef IB_CFL_LAUNCH_C
    return check_launch();
}

int launch_soundspeed(const double *q, int64_t slab, int64_t n, double gamma, double *cs, cudaStream_t st)
{
    int nb = (int)std::min<int64_t>((n + 255) / 256, (int64_t)8 * num_sms());
    if (nb < 1) nb = 1;
    soundspeed_kernel<<<nb, 256, 0, st>>>(q, slab, n, gamma * (gamma - 1), cs);
    return check_launch();
}

// ------------------------------------------------------------------------------------------
// freezeAndPtot, hydro (cukern_FreezeSpeed_hydro, freezeAndPtot.cu:229-290): one warp-multiple
// block per x row.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) freeze_ptot_kernel(double *__restrict__ q, int64_t slab, int nx, double gam,
                                                          double gm1, double cs0sq, double *__restrict__ ptot,
                                                          double *__restrict__ freeze)
{
    const int64_t row = blockIdx.x;
    double *rho = q + row * nx, *E = rho + slab, *px = rho + 2 * slab, *py = rho + 3 * slab, *pz = rho + 4 * slab;
    double *pt = ptot + row * nx;
    double CsMax = 0.0;
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
        double rhoinv = 1.0 / rho[x];
        double psqhf = .5 * (px[x] * px[x] + py[x] * py[x] + pz[x] * pz[x]);
        double P = gm1 * (E[x] - psqhf * rhoinv);
        if (gam * P * rhoinv < cs0sq) {
            P = cs0sq / (gam * rhoinv);
            E[x] = psqhf * rhoinv + P / gm1;
        }
        pt[x] = P;
        double Cs = sqrt(gam * P * rhoinv) + fabs(px[x] * rhoinv);
        if (Cs > CsMax) CsMax = Cs;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double v = __shfl_xor_sync(0xffffffffu, CsMax, o);
        if (v > CsMax) CsMax = v;
    }
    __shared__ double wm[4];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = CsMax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = wm[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) if (wm[w] > m) m = wm[w];
        freeze[row] = m;
    }
}

int launch_freeze_ptot(double *q, int64_t slab, const int grid[3], double gamma, double cs_min, double *ptot,
                       double *freeze, cudaStream_t st)
{
    int64_t rows = (int64_t)grid[1] * grid[2];
    if (rows <= 0) return IB_SUCCESSFUL;
    freeze_ptot_kernel<<<(unsigned)rows, 128, 0, st>>>(q, slab, grid[0], gamma, gamma - 1.0, cs_min * cs_min, ptot,
                                                      freeze);
    return check_launch();
}

}  // namespace ib

// ------------------------------------------------------------------------------------------
// CFL timestep without any device allocation (ib_cflTimestepNoAlloc)
//
// The ordinary CFL entry points keep their per-block minima in scratch memory that the library
// obtains from cudaMalloc on first use.  Some callers cannot let the library allocate: a host
// application that has reserved the GPU's memory for its own pool (so an extra cudaMalloc may
// fail), or a time-critical loop that must not pay for the device-wide synchronisation that
// cudaMalloc and cudaFree can cause.  This variant runs the same reduction kernel with its
// scratch in a fixed array compiled into the library instead.
//
// The array is a file-scope device variable, so every GPU that loads the library carries it
// (a little over 64 KB) until the process exits.  All calls on a device share it and it keeps
// whatever the last call left there: the completion counter is cleared at the start of every
// call, and two calls that overlap on the GPU (for example on two streams) would race on it.
// ------------------------------------------------------------------------------------------
namespace ib {

constexpr int kNoAllocMaxBlocks = 8192;  // one partial minimum per reduction block
// largest grid this entry point accepts (the documented limit; the kernel itself strides over
// any number of cells with at most kNoAllocMaxBlocks blocks)
constexpr int64_t kNoAllocMaxCells = (int64_t)134217728;

// [0, 256): completion counter (first 4 bytes); [256, 256 + 8*8192): partial minima
static __device__ __align__(256) unsigned char g_cfl_noalloc_scratch[256 + sizeof(double) * kNoAllocMaxBlocks];

// Device address of the array, looked up with the device current and cached per device and
// context: after a cudaDeviceReset, or under a context the caller made current through the
// driver API, the module may be loaded at another address, so a new context looks it up again.
// Host code must not hand the symbol itself to a kernel: in host code it names a host-side
// stand-in.
typedef CUresult (*PFN_ctx_get_current)(CUcontext *);
struct NoAllocSlot {
    CUcontext ctx = nullptr;
    unsigned char *addr = nullptr;
};
static NoAllocSlot g_noalloc_slot[64];
static std::mutex g_noalloc_mu;

static CUcontext current_context()
{
    static PFN_ctx_get_current fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_ctx_get_current>(p);
        cudaGetLastError();
        return (PFN_ctx_get_current) nullptr;
    }();
    CUcontext c = nullptr;
    if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
    return c;
}

static int noalloc_scratch(unsigned char **out)
{
    int dev = 0;
    int rc = check_cuda(cudaGetDevice(&dev));
    if (rc) return rc;
    if (dev < 0 || dev >= 64) return IB_ERROR_INVALID_ARGS;
    // no context current yet on this thread (a first call): cudaGetSymbolAddress makes the
    // device's primary context current, and the slot records that context afterwards
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    NoAllocSlot &s = g_noalloc_slot[dev];
    CUcontext ctx = current_context();
    if (!s.addr || !ctx || ctx != s.ctx) {
        void *p = nullptr;
        rc = check_cuda(cudaGetSymbolAddress(&p, g_cfl_noalloc_scratch));
        if (rc) return rc;
        s.addr = static_cast<unsigned char *>(p);
        s.ctx = current_context();
    }
    *out = s.addr;
    return IB_SUCCESSFUL;
}

}  // namespace ib

extern "C" int ib_cflTimestepNoAlloc(const ib_fluid *fluid, double gamma, const ib_geometry *geo, int method,
                                     double *tau_device, void *stream)
{
    using namespace ib;
    if (!fluid || !geo || !fluid->q || !tau_device) return IB_ERROR_NULL_POINTER;
    const ib_grid &g = fluid->grid;
    if (g.nx < 1 || g.ny < 1 || g.nz < 1) return IB_ERROR_INVALID_ARGS;
    const int64_t n = (int64_t)g.nx * g.ny * g.nz;
    if (g.slab_pitch < n) return IB_ERROR_INVALID_ARGS;
    if (n > kNoAllocMaxCells) {
        fprintf(stderr, "ib_cflTimestepNoAlloc: %lld cells exceed the fixed scratch limit of %lld cells\n",
                (long long)n, (long long)kNoAllocMaxCells);
        return IB_ERROR_INVALID_ARGS;
    }
    if (method < IB_METHOD_HLL || method > IB_METHOD_XINJIN) return IB_ERROR_INVALID_ARGS;
    if (geo->shape != 0) return IB_ERROR_NOIMPLEMENT;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned char *base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc) return rc;
    unsigned int *counter = reinterpret_cast<unsigned int *>(base);
    double *partial = reinterpret_cast<double *>(base + 256);
    if ((rc = check_cuda(cudaMemsetAsync(counter, 0, sizeof(unsigned int), st)))) return rc;

    int sim = 1;
    if (geo->global_rez[1] > 1) sim = 2;
    if (geo->global_rez[2] > 1) sim = 3;
    const bool xj = (method == IB_METHOD_XINJIN) && (sim > 1);
    double hmin = geo->h[0];
    if (sim > 1 && geo->h[1] < hmin) hmin = geo->h[1];
    if (sim > 2 && geo->h[2] < hmin) hmin = geo->h[2];
    // as many blocks as launch_cfl uses (the kernel strides over the cells), within the array
    const int nb = (int)std::max<int64_t>(
        1, std::min<int64_t>((n + 255) / 256, std::min<int64_t>((int64_t)4 * num_sms(), kNoAllocMaxBlocks)));
    const int halve = (method == IB_METHOD_HLL || method == IB_METHOD_HLLC) ? 1 : 0;
    const double gg1 = gamma * (gamma - 1);
    const int64_t slab = g.slab_pitch;
    const double *q = fluid->q;
#define IB_NOALLOC_CFL(S, X)                                                                             \
    cfl_kernel<S, X, true><<<nb, 256, 0, st>>>(q, nullptr, slab, n, gg1, hmin, geo->h[0], geo->h[1], geo->h[2], \
                                               halve, partial, counter, tau_device)
    if (xj) { if (sim == 2) IB_NOALLOC_CFL(2, true); else IB_NOALLOC_CFL(3, true); }
    else if (sim == 1) IB_NOALLOC_CFL(1, false);
    else if (sim == 2) IB_NOALLOC_CFL(2, false);
    else IB_NOALLOC_CFL(3, false);
#undef IB_NOALLOC_CFL
    return check_launch();
}
