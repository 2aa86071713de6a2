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
// The per-cell arithmetic is the library's sweep arithmetic (stage_prims / stage_faces /
// stage_flux in ens_sweep), CFL and boundary code, so every problem's result equals running it
// alone through the library's 1-D entry points.
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
    int32_t lcap;      // tile rows (chunk + 8 halo cells) the shared memory planes hold, <= threads
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

// Number of chunks for a problem of n cells: chunk ch covers cells [ch n / nc, (ch + 1) n / nc), so
// no chunk is longer than the target and, as the in-place rules need, none is shorter than 8 cells.
// Every output cell is the same function of the 9 original cells around it whatever the chunks.
__device__ __forceinline__ int ens_nchunks(int n, int target)
{
    int nc = max(1, (n + target - 1) / target);
    while (nc > 1 && n / nc < 8) nc--;
    return nc;
}

// One x sweep of a problem of n cells in nc chunks (ens_nchunks; the longest chunk + 8 <= lcap <= NT):
// the tile sweep's in-place rules (each chunk loads its cells and 4 halo cells a side of the original
// state; the last four outputs of a chunk wait in `pend` until the next chunk has loaded them, the
// first chunk's first four in `first` until the last chunk has read them through the periodic
// wrap) with the row kernel's phases: tile row i of a chunk is thread i, which keeps that cell's
// state in registers through both stages; two shared-memory planes of FT swap roles between the
// stages, so a chunk takes seven barriers.  The arithmetic is the library's sweep arithmetic
// (stage_prims / stage_faces / stage_flux), so the results are those of the tile sweep.
template <int METHOD, int SLOPE, typename FT, int NT>
__device__ __forceinline__ void ens_sweep(double *qb, int64_t S, int n, int nchunks, double lambda,
                                          const FluidConsts<FT> &c, FT *SA, FT *SB, int TR, double *pend,
                                          double *first)
{
    const int i = threadIdx.x;
    const bool single = (nchunks == 1);
    for (int ch = 0; ch < nchunks; ch++) {
        const int cb = (int)((int64_t)ch * n / nchunks);
        const int len = (int)((int64_t)(ch + 1) * n / nchunks) - cb;
        const int tr = len + 8;
        double u0[5], u1[5];
        V5<FT> keep;
        if (i < tr) {
            const int cell = mod_n(cb - 4 + i, n);
#pragma unroll
            for (int k = 0; k < 5; k++) u0[k] = qb[(int64_t)k * S + cell];
        }
        __syncthreads();  // this chunk has loaded the original state of its halo
        if (ch > 0 && i < 4) {
#pragma unroll
            for (int k = 0; k < 5; k++) qb[(int64_t)k * S + cb - 4 + i] = pend[k * 4 + i];
        }
        // ---- stage A: prims and fluxes in SA, left faces in SB ----
        if (i < tr) {
            V5<FT> w = stage_prims<METHOD, 1, FT>(u0, c);  // HLL floors u0
#pragma unroll
            for (int k = 0; k < 5; k++) SA[k * TR + i] = w.a[k];
        }
        __syncthreads();
        if (i >= 1 && i <= tr - 2) {
            V5<FT> w, dl, dr, L;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                w.a[k] = SA[k * TR + i];
                dl.a[k] = w.a[k] - SA[k * TR + i - 1];
                dr.a[k] = SA[k * TR + i + 1] - w.a[k];
            }
            stage_faces<METHOD, SLOPE, FT>(c, w, dl, dr, L, keep);
#pragma unroll
            for (int k = 0; k < 5; k++) SB[k * TR + i] = L.a[k];
        }
        __syncthreads();
        if (i >= 1 && i <= tr - 3) {
            V5<FT> Lr;
#pragma unroll
            for (int k = 0; k < 5; k++) Lr.a[k] = SB[k * TR + i + 1];
            keep = stage_flux<METHOD, FT>(c, keep, Lr);
#pragma unroll
            for (int k = 0; k < 5; k++) SA[k * TR + i] = keep.a[k];
        }
        __syncthreads();
        if (i >= 2 && i <= tr - 3) {
#pragma unroll
            for (int k = 0; k < 5; k++) u1[k] = u0[k] - lambda * ((double)keep.a[k] - (double)SA[k * TR + i - 1]);
        }
        // ---- stage B: prims and fluxes in SB, left faces in SA (no barrier: stage A's last
        // phase read SA only) ----
        if (i >= 2 && i <= tr - 3) {
            V5<FT> w = stage_prims<METHOD, 1, FT>(u1, c);  // HLL floors u1
#pragma unroll
            for (int k = 0; k < 5; k++) {
                SB[k * TR + i] = w.a[k];
                u0[k] = u1[k] + u0[k];  // the output's (u1 + u0), rounded as it is there first
            }
        }
        __syncthreads();
        if (i >= 3 && i <= tr - 4) {
            V5<FT> w, dl, dr, L;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                w.a[k] = SB[k * TR + i];
                dl.a[k] = w.a[k] - SB[k * TR + i - 1];
                dr.a[k] = SB[k * TR + i + 1] - w.a[k];
            }
            stage_faces<METHOD, SLOPE, FT>(c, w, dl, dr, L, keep);
#pragma unroll
            for (int k = 0; k < 5; k++) SA[k * TR + i] = L.a[k];
        }
        __syncthreads();
        if (i >= 3 && i <= tr - 5) {
            V5<FT> Lr;
#pragma unroll
            for (int k = 0; k < 5; k++) Lr.a[k] = SA[k * TR + i + 1];
            keep = stage_flux<METHOD, FT>(c, keep, Lr);
#pragma unroll
            for (int k = 0; k < 5; k++) SB[k * TR + i] = keep.a[k];
        }
        __syncthreads();
        if (i >= 4 && i <= tr - 5) {
            const int m = i - 4;  // output cell cb + m
            double out[5];
#pragma unroll
            for (int k = 0; k < 5; k++)
                out[k] = .5 * (u0[k] - lambda * ((double)keep.a[k] - (double)SB[k * TR + i - 1]));
            if (!single && ch == 0 && m < 4) {
#pragma unroll
                for (int k = 0; k < 5; k++) first[k * 4 + m] = out[k];
            } else if (!single && m >= len - 4) {
#pragma unroll
                for (int k = 0; k < 5; k++) pend[k * 4 + m - (len - 4)] = out[k];
            } else {
#pragma unroll
                for (int k = 0; k < 5; k++) qb[(int64_t)k * S + cb + m] = out[k];
            }
        }
        // the next chunk's first barrier separates these reads of SB and writes of pend from its
        // stage A
    }
    __syncthreads();
    if (!single && i < 4) {
#pragma unroll
        for (int k = 0; k < 5; k++) {
            qb[(int64_t)k * S + n - 4 + i] = pend[k * 4 + i];
            qb[(int64_t)k * S + i] = first[k * 4 + i];
        }
    }
    __syncthreads();
}

// Three CTAs of 256 threads per SM (80 registers) rather than four: at 64 registers a thread's
// state of two stages spills; 512-thread CTAs keep two per SM, one would idle half the SM.
template <int METHOD, int SLOPE, typename FT, int NT>
__global__ void __launch_bounds__(NT, NT == 512 ? 2 : 768 / NT) ensemble_kernel(EnsArgs a, FluidConsts<FT> c)
{
    extern __shared__ __align__(16) double tsm[];
    __shared__ int s_prob;
    __shared__ double s_red[NT / 32];
    __shared__ double s_dt;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double *pend = tsm;        // [5][4]
    double *first = tsm + 20;  // [5][4]
    FT *SA = reinterpret_cast<FT *>(tsm + 40);  // [5][lcap]
    FT *SB = SA + 5 * a.lcap;
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
        const int nc = (nn >= 9 && nn < (1 << 30)) ? ens_nchunks(n, a.target) : 0;
        if (nc == 0 || (n + nc - 1) / nc + 8 > a.lcap || p >= a.np) {
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
                ens_sweep<METHOD, SLOPE, FT, NT>(qb, a.S, n, nc, lambda, c, SA, SB, a.lcap, pend, first);
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

// Shared memory of one CTA: the pending and first outputs, two planes of a chunk of up to lcap
// tile rows.
template <typename FT>
static size_t ens_smem(int lcap)
{
    return sizeof(double) * 40 + sizeof(FT) * 10 * (size_t)lcap;
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
    if (per_sm < 1 || a.lcap > NT) return IB_ERROR_INVALID_ARGS;
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
