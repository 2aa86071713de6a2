// ib_ensemble.cu -- batched ensemble of independent 1-D problems in one persistent launch.
//
// Each problem is what the reference runs as a one-dimensional fluid: per iteration the CFL
// timestep (cflTimestep.cu:107-252; in 1-D the HLL template, |p_x| only, halved for HLL/HLLC),
// dt = CFL * tau with the last-step clip (TimeManager.m:124-186), then the forward and the
// backward fluid step, each the 1-D shortcut of performFluidUpdate_3D (flux.cu:52-68): one x
// sweep followed by the boundary fill, and t += 2 dt with Kahan compensation
// (TimeManager.m:270-277).  Here a CTA takes a problem from a device work counter and runs it to
// its end without leaving the kernel; the problem's cells stay in L2 between sweeps (one
// problem is at most a few hundred KB), so the launch reads and writes HBM about once per cell.
// The per-cell arithmetic is the library's sweep (tile_sweep), CFL and boundary code, so every
// problem's result equals running it alone through the library's 1-D entry points.
#include "ib_bc.cuh"
#include "ib_cfl.cuh"
#include "ib_internal.cuh"
#include "ib_sweep.cuh"

namespace ib {

struct EnsArgs {
    double *q;
    int64_t S;
    const int64_t *off;
    const double *h;
    const int32_t *order;
    double *t_out;
    int32_t *it_out;
    unsigned int *counter;
    int32_t np;
    int32_t bc0, bc1;
    int32_t itermax;
    int32_t target;    // chunk length to aim for
    int32_t lcap;      // largest chunk the shared memory holds
    double gg1;        // gamma (gamma - 1), soundspeed
    double cfl, t_end;
    int32_t halve;
};

// Boundary fill of one 1-D problem after a sweep (setFluidBoundary along x), both sides in order.
__device__ __forceinline__ void ens_boundary(double *qb, int64_t S, int n, int bc0, int bc1)
{
    for (int side = 0; side < 2; side++) {
        const int mode = side ? bc1 : bc0;
        if (mode == IB_BC_OUTFLOW) {
            outflow_x(qb, S, 1, n, side, 1, 4);
        } else if (mode == IB_BC_MIRROR || mode == IB_BC_CONST || mode == IB_BC_LINEAR) {
            for (int k = 0; k < 5; k++) sas_x(qb + k * S, 1, n, mode, side, k == 2, 4);
        }
    }
}

// Chunk length for a pencil of n cells: as in the tile launcher, every chunk >= 8 cells.
__device__ __forceinline__ int ens_chunk(int n, int target)
{
    int nc = max(1, (n + target - 1) / target);
    int Lc = (n + nc - 1) / nc;
    while (nc > 1 && (Lc < 8 || n - (nc - 1) * Lc < 8)) {
        nc--;
        Lc = (n + nc - 1) / nc;
    }
    return Lc;
}

template <int METHOD, int SLOPE, typename FT, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) ensemble_kernel(EnsArgs a, FluidConsts<FT> c)
{
    extern __shared__ __align__(16) double tsm[];
    __shared__ int64_t colbase[1];
    __shared__ bool colok[1];
    __shared__ int s_prob;
    __shared__ double s_red[NT / 32];
    __shared__ double s_dt;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) {
        colbase[0] = 0;
        colok[0] = true;
    }
    for (;;) {
        if (tid == 0) {
            const unsigned k = atomicAdd(a.counter, 1u);
            s_prob = (k < (unsigned)a.np) ? (a.order ? a.order[k] : (int)k) : -1;
        }
        __syncthreads();
        const int p = s_prob;
        if (p < 0) break;
        const int64_t off = a.off[p];
        const int64_t nn = a.off[p + 1] - off;
        const double h = a.h[p];
        const int n = (int)nn;
        const int Lc = (nn >= 9 && nn < (1 << 30)) ? ens_chunk(n, a.target) : 0;
        if (Lc == 0 || Lc > a.lcap || p >= a.np) {
            if (tid == 0 && p < a.np) {
                a.t_out[p] = 0.0;
                a.it_out[p] = -1;  // not run: fewer than 9 cells or a chunk beyond the tile
            }
            __syncthreads();
            continue;
        }
        double *qb = a.q + off;
        double t = 0.0, kc = 0.0;
        int it = 0;
        while (it < a.itermax && t < a.t_end * (1 - 1e-14)) {
            // tau: NaN-ignoring minimum of the signal-crossing times, halved for HLL/HLLC
            double tmin = 1e37;
            for (int x = tid; x < n; x += NT) {
                const double rho = qb[x], px = qb[x + 2 * a.S];
                const double cs = soundspeed_cell(rho, qb[x + a.S], px, qb[x + 3 * a.S], qb[x + 4 * a.S], a.gg1);
                tmin = min_keep(tmin, cfl_cell<1, false>(rho, px, 0.0, 0.0, cs, h, h, h, h));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) tmin = min_keep(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
            if (lane == 0) s_red[wid] = tmin;
            __syncthreads();
            if (tid == 0) {
                double r = 1e38;
                for (int w = 0; w < NT / 32; w++) r = (s_red[w] < r) ? s_red[w] : r;
                if (a.halve) r = r / 2;
                double dt = __dmul_rn(a.cfl, r);
                if (__dadd_rn(t, __dmul_rn(2.0, dt)) > a.t_end) dt = __dmul_rn(.5, __dadd_rn(a.t_end, -t));
                s_dt = dt;
            }
            __syncthreads();
            const double dt = s_dt;
            const double lambda = dt / h;
            for (int half = 0; half < 2; half++) {
                tile_sweep<METHOD, SLOPE, FT, 1, 1>(qb, a.S, colbase, colok, 1, n, Lc, lambda, c, tsm);
                if (tid == 0) ens_boundary(qb, a.S, n, a.bc0, a.bc1);
                __syncthreads();
            }
            const double y = __dadd_rn(__dmul_rn(2.0, dt), -kc);
            const double tn = __dadd_rn(t, y);
            kc = __dadd_rn(__dadd_rn(tn, -t), -y);
            t = tn;
            it++;
        }
        if (tid == 0) {
            a.t_out[p] = t;
            a.it_out[p] = it;
        }
        __syncthreads();
    }
}

// Shared memory of one CTA: the tile of a chunk of up to lcap cells.
template <typename FT>
static size_t ens_smem(int lcap)
{
    return tile_smem_bytes<1>(lcap, sizeof(FT));
}

template <int METHOD, int SLOPE, typename FT, int NT>
static int launch_ens_nt(const EnsArgs &a0, const FluidConsts<FT> &c, int ctas_per_sm, cudaStream_t st)
{
    EnsArgs a = a0;
    auto kern = ensemble_kernel<METHOD, SLOPE, FT, NT>;
    const size_t shm = ens_smem<FT>(a.lcap);
    static int attr_bytes = 0;
    int rc;
    if ((int)shm > attr_bytes) {
        if ((rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm))))
            return rc;
        attr_bytes = (int)shm;
    }
    int per_sm = 0;
    if ((rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, shm)))) return rc;
    if (per_sm < 1) return IB_ERROR_INVALID_ARGS;
    if (ctas_per_sm > 0 && ctas_per_sm < per_sm) per_sm = ctas_per_sm;
    const int64_t grid = std::min<int64_t>((int64_t)per_sm * num_sms(), a.np);
    if ((rc = check_cuda(cudaMemsetAsync(a.counter, 0, sizeof(unsigned int), st)))) return rc;
    kern<<<(unsigned)grid, NT, shm, st>>>(a, c);
    return check_launch();
}

template <int METHOD, int SLOPE, typename FT>
static int launch_ens(const EnsArgs &a, const FluidConsts<FT> &c, int threads, int ctas_per_sm, cudaStream_t st)
{
    switch (threads) {
    case 128: return launch_ens_nt<METHOD, SLOPE, FT, 128>(a, c, ctas_per_sm, st);
    case 256: return launch_ens_nt<METHOD, SLOPE, FT, 256>(a, c, ctas_per_sm, st);
    case 512: return launch_ens_nt<METHOD, SLOPE, FT, 512>(a, c, ctas_per_sm, st);
    default: return IB_ERROR_INVALID_ARGS;
    }
}

template <int METHOD, typename FT>
static int launch_ens_slope(int slope, const EnsArgs &a, const FluidConsts<FT> &c, int threads, int cps,
                            cudaStream_t st)
{
    if (slope == IB_SLOPE_MC) return launch_ens<METHOD, IB_SLOPE_MC, FT>(a, c, threads, cps, st);
    if (slope == IB_SLOPE_OSPRE) return launch_ens<METHOD, IB_SLOPE_OSPRE, FT>(a, c, threads, cps, st);
    return IB_ERROR_NOIMPLEMENT;
}

}  // namespace ib

using namespace ib;

extern "C" int ib_riemannEnsemble(const ib_ensemble *e, const ib_fluid_thermo *thermo, int method, double cfl,
                                  double t_end, int32_t itermax, const ib_numerics *num,
                                  const ib_ensemble_tuning *tuning, void *stream)
{
    if (!e || !thermo) return IB_ERROR_NULL_POINTER;
    if (!e->q || !e->offsets || !e->h || !e->t_out || !e->iters_out) return IB_ERROR_NULL_POINTER;
    if (e->nproblems < 1 || e->slab_pitch < 1) return IB_ERROR_INVALID_ARGS;
    if (method != IB_METHOD_HLL && method != IB_METHOD_HLLC) return IB_ERROR_NOIMPLEMENT;
    if (!(cfl > 0) || !(t_end >= 0) || !(t_end < 1e300)) return IB_ERROR_INVALID_ARGS;
    for (int s = 0; s < 2; s++) {
        const int m = e->bc[s];
        if (m != IB_BC_CIRCULAR && m != IB_BC_MIRROR && m != IB_BC_CONST && m != IB_BC_LINEAR && m != IB_BC_OUTFLOW)
            return IB_ERROR_INVALID_ARGS;
    }
    const double gamma = thermo->gamma;
    if (!(gamma > 1)) return IB_ERROR_INVALID_ARGS;
    if (thermo->c_isothermal != -1) return IB_ERROR_NOIMPLEMENT;
    const int slope = num ? num->slope_limiter : IB_SLOPE_OSPRE;
    const int prec = num ? num->precision : IB_PREC_FP64;
    int threads = 256, chunk = 0, cps = 0;
    if (tuning) {
        if (tuning->threads) threads = tuning->threads;
        chunk = tuning->chunk;
        cps = tuning->ctas_per_sm;
    }
    if (threads != 128 && threads != 256 && threads != 512) return IB_ERROR_INVALID_ARGS;
    if (chunk == 0) chunk = threads - 8;
    if (chunk < 120 || chunk > threads - 8 || cps < 0) return IB_ERROR_INVALID_ARGS;
    EnsArgs a;
    a.q = e->q;
    a.S = e->slab_pitch;
    a.off = e->offsets;
    a.h = e->h;
    a.order = e->order;
    a.t_out = e->t_out;
    a.it_out = e->iters_out;
    a.counter = scratch().ensemble_counter();
    if (!a.counter) return IB_ERROR_NOMEM;
    a.np = e->nproblems;
    a.bc0 = e->bc[0];
    a.bc1 = e->bc[1];
    a.itermax = (itermax > 0) ? itermax : 0x7fffffff;
    a.target = chunk;
    a.lcap = chunk + 8;
    a.gg1 = gamma * (gamma - 1);
    a.cfl = cfl;
    a.t_end = t_end;
    a.halve = 1;
    cudaStream_t st = (cudaStream_t)stream;
    const double rho_min = thermo->rho_min;
    if (method == IB_METHOD_HLLC) {
        if (prec == IB_PREC_FP32_FLUX)
            return launch_ens_slope<IB_METHOD_HLLC, float>(slope, a, make_consts<float>(gamma, rho_min, -1), threads,
                                                          cps, st);
        if (prec != IB_PREC_FP64) return IB_ERROR_INVALID_ARGS;
        return launch_ens_slope<IB_METHOD_HLLC, double>(slope, a, make_consts<double>(gamma, rho_min, -1), threads,
                                                       cps, st);
    }
    if (prec != IB_PREC_FP64) return IB_ERROR_NOIMPLEMENT;
    return launch_ens_slope<IB_METHOD_HLL, double>(slope, a, make_consts<double>(gamma, rho_min, -1), threads, cps,
                                                  st);
}
