// ib_xinjin.cu -- Xin-Jin relaxing TVD sweep (cukern_XinJinHydro_step, gpuclass/cudaFluidStep.cu:2427-2654)
// with the per-row freezing speed of cukern_PressureFreezeSolverHydro (:2867-2941).
//
// The reference needs the maximum of |v|+c_s over the whole swept row before each stage, so it
// runs freeze / predictor / freeze / corrector as four kernels with a host reduction in
// between (MGA_globalReduceDimension, cudaCommon.cu:919-1004).  Here one CTA owns one pencil:
// it stages the pencil in shared memory, reduces the freezing speed in-block, and runs both
// stages, so a sweep is one launch with one read and one write of the state.
#include "ib_internal.cuh"

namespace ib {

__device__ __forceinline__ double block_max_keep(double v, double *red)
{
    // maximum ignoring NaN candidates, as the reference's `(a > b) ? a : b` tree
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = (w > v) ? w : v;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < nw; w++) m = (red[w] > m) ? red[w] : m;
    return m;
}

// Uses memory slab 2 (px) as the transported momentum whatever the sweep direction, as the
// reference's freeze kernel does.
__device__ __forceinline__ double freeze_cell(const double *U, int n, int i, double gamma, double gm1)
{
    double invrho = 1.0 / U[i];
    double psq = U[3 * n + i];
    double px = U[4 * n + i];
    psq = psq * psq + px * px;
    px = U[2 * n + i];
    psq += px * px;
    double P = (U[n + i] - .5 * psq * invrho) * gm1;
    return fabs(px) * invrho + sqrt(gamma * P * invrho);
}

template <int FLIM>
__global__ void __launch_bounds__(256) xj_pencil_kernel(double *q, int64_t slab, int nx, int ny, int nz, int dir,
                                                        double lambda, double gamma, double minmass, double mintemp)
{
    extern __shared__ __align__(16) double sm[];
    const int n = (dir == 1) ? nx : (dir == 2 ? ny : nz);
    double *U0 = sm;            // [5][n] fluid
    double *U1 = U0 + 5 * n;    // [5][n] prediction, then corrected output
    double *Lb = U1 + 5 * n;    // [n] left-going flux of the current component
    double *Rb = Lb + n;        // [n] right-going
    double *dLb = Rb + n;       // [n]
    double *dRb = dLb + n;      // [n]
    double *Pv = dRb + n;       // [n] pressure
    double *Vx = Pv + n;        // [n] normal velocity
    __shared__ double red[32];

    const int64_t p = blockIdx.x;
    int64_t base, stride;
    if (dir == 1) { base = p * nx; stride = 1; }
    else if (dir == 2) { base = (p % nx) + (int64_t)nx * ny * (p / nx); stride = nx; }
    else { base = p; stride = (int64_t)nx * ny; }
    const int nslot = 1 + dir;
    const double gm1 = gamma - 1.0;

    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int k = 0; k < 5; k++) U0[k * n + i] = q[k * slab + base + i * stride];
    __syncthreads();

    for (int stage = 0; stage < 2; stage++) {
        const double *Qin = (stage == 0) ? U0 : U1;
        const double lam = (stage == 0) ? 0.25 * lambda : 0.5 * lambda;
        // freezing speed of the row
        double cm = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double v = freeze_cell(Qin, n, i, gamma, gm1);
            cm = (v > cm) ? v : cm;
        }
        const double Cf = block_max_keep(cm, red);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double q0 = Qin[i], q1 = Qin[n + i], q2 = Qin[2 * n + i], q3 = Qin[3 * n + i], q4 = Qin[4 * n + i];
            Pv[i] = gm1 * (q1 - .5 * (q4 * q4 + q3 * q3 + q2 * q2) / q0);
            Vx[i] = Qin[nslot * n + i] / q0;
        }
        // proposed values, one component at a time; kept in registers per thread (<= 8 cells)
        double prop[5][8];
        __syncthreads();
        for (int k = 0; k < 5; k++) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                double qk = Qin[k * n + i], w;
                if (k == 0) w = Qin[nslot * n + i];
                else if (k == 1) w = Vx[i] * (qk + Pv[i]);
                else if (k == nslot) w = Vx[i] * qk + Pv[i];
                else w = Vx[i] * qk;
                Lb[i] = (Cf * qk - w);
                Rb[i] = (Cf * qk + w);
            }
            __syncthreads();
            if (stage == 1) {
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    int il = (i == 0) ? n - 1 : i - 1;
                    dLb[i] = 0.5 * (Lb[i] - Lb[il]);
                    dRb[i] = 0.5 * (Rb[i] - Rb[il]);
                }
                __syncthreads();
                double nl[8], nr[8];
                int m = 0;
                for (int i = threadIdx.x; i < n; i += blockDim.x, m++) {
                    int ir = (i == n - 1) ? 0 : i + 1;
                    nl[m] = Lb[i] - flux_limit<FLIM>(dLb[i], dLb[ir]);
                    nr[m] = Rb[i] + flux_limit<FLIM>(dRb[i], dRb[ir]);
                }
                __syncthreads();
                m = 0;
                for (int i = threadIdx.x; i < n; i += blockDim.x, m++) { Lb[i] = nl[m]; Rb[i] = nr[m]; }
                __syncthreads();
            }
            int m = 0;
            for (int i = threadIdx.x; i < n; i += blockDim.x, m++) {
                int il = (i == 0) ? n - 1 : i - 1, ir = (i == n - 1) ? 0 : i + 1;
                double b = (stage == 0) ? Qin[k * n + i] : U0[k * n + i];
                prop[k][m] = b - lam * (Rb[i] - Rb[il] - Lb[ir] + Lb[i]);
            }
            __syncthreads();
        }
        // floors (cudaFluidStep.cu:2620-2629) and store
        int m = 0;
        for (int i = threadIdx.x; i < n; i += blockDim.x, m++) {
            double p0 = prop[0][m], p1 = prop[1][m], p2 = prop[2][m], p3 = prop[3][m], p4 = prop[4][m];
            p0 = (p0 < minmass) ? minmass : p0;
            double w = .5 * (p2 * p2 + p3 * p3 + p4 * p4) / p0;
            if ((p1 - w) < p0 * mintemp) p1 = w + p0 * mintemp;
            U1[i] = p0; U1[n + i] = p1; U1[2 * n + i] = p2; U1[3 * n + i] = p3; U1[4 * n + i] = p4;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int k = 0; k < 5; k++) q[k * slab + base + i * stride] = U1[k * n + i];
}

int launch_xj_sweep(int flim, int dir, double *q, int64_t slab, const int grid[3], double lambda, double gamma,
                    double rho_min, cudaStream_t st)
{
    const int n = grid[dir - 1];
    const int64_t N = (int64_t)grid[0] * grid[1] * grid[2];
    if (n > 2048) return IB_ERROR_NOIMPLEMENT;  // per-thread proposal registers cover 8 cells x 256 threads
    const size_t shm = (size_t)16 * n * sizeof(double);
    const size_t shm_cap = 227 * 1024 - 1024;  // opt-in limit minus the kernel's static shared memory
    if (shm > shm_cap) return IB_ERROR_NOIMPLEMENT;
    const int64_t np = N / n;
    const double mintemp = 1e-5 / (gamma - 1);
    int nt = std::min(256, ((n + 31) / 32) * 32);
    if ((n + nt - 1) / nt > 8) nt = 256;
#define IB_XJ(F)                                                                                              \
    do {                                                                                                      \
        static bool attr_set = false;                                                                         \
        if (!attr_set) {                                                                                      \
            int rc_ = check_cuda(cudaFuncSetAttribute(xj_pencil_kernel<F>,                                    \
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm_cap)); \
            if (rc_) return rc_;                                                                              \
            attr_set = true;                                                                                  \
        }                                                                                                     \
        xj_pencil_kernel<F><<<(unsigned)np, nt, shm, st>>>(q, slab, grid[0], grid[1], grid[2], dir, lambda, gamma, \
                                                           rho_min, mintemp);                                 \
    } while (0)
    switch (flim) {
    case IB_FLUX_OSPRE: IB_XJ(IB_FLUX_OSPRE); break;
    case IB_FLUX_VANLEER: IB_XJ(IB_FLUX_VANLEER); break;
    case IB_FLUX_MINMOD: IB_XJ(IB_FLUX_MINMOD); break;
    case IB_FLUX_SUPERBEE: IB_XJ(IB_FLUX_SUPERBEE); break;
    default: IB_XJ(IB_FLUX_ZERO); break;
    }
#undef IB_XJ
    return check_launch();
}

}  // namespace ib
