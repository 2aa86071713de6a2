// ib_drag.cu -- two-fluid gas-dust drag source (gpuclass/cudaSource2FluidDrag.cu).
//
// The reference's default LogTrap2 path runs two kernels over a 3-slab temporary: one writes
// [|dv|, e_int/rho] (cukern_prepareForERK_h0, :1883-1908), the other integrates the drag
// (cukern_LogTrapSolve, :1531-1686) launched with at most 32 blocks of 96 threads (:730-757).
// Here one kernel does both per cell with the temporaries in registers, over a full-GPU grid:
// 10 doubles read and 7 written per cell.
#include "ib_drag.cuh"
#include "ib_internal.cuh"

namespace ib {

template <int ORDER>
__global__ void __launch_bounds__(256) logtrap_kernel(double *__restrict__ gas, double *__restrict__ dust, int64_t S,
                                                      int64_t n, DragParams d, double t)
{
    for (int64_t x = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; x < n; x += (int64_t)blockDim.x * gridDim.x) {
        double *g = gas + x, *ds = dust + x;
        const double g0 = g[0], gE = g[S], g2 = g[2 * S], g3 = g[3 * S], g4 = g[4 * S];
        const double d0 = ds[0], d2 = ds[2 * S], d3 = ds[3 * S], d4 = ds[4 * S];
        double t0, t1;
        drag_features(g0, gE, g2, g3, g4, d0, d2, d3, d4, t0, t1);
        const double k = logtrap_keff<ORDER>(d, g0, d0, t0, t1, t);
        drag_apply(g, ds, S, g0, gE, g2, g3, g4, d0, d2, d3, d4, t, k);
    }
}

int launch_drag(double *gas, double *dust, int64_t slab, int64_t n, const double dp[11], double dt, int method,
                cudaStream_t st)
{
    DragParams d{dp[0], dp[1], dp[2], dp[3], dp[4], dp[5], dp[6]};
    if (n <= 0) return IB_SUCCESSFUL;
    int nb = (int)std::min<int64_t>((n + 255) / 256, (int64_t)16 * num_sms());
    if (method == IB_DRAG_LOGTRAP2) logtrap_kernel<2><<<nb, 256, 0, st>>>(gas, dust, slab, n, d, dt);
    else if (method == IB_DRAG_LOGTRAP3) logtrap_kernel<3><<<nb, 256, 0, st>>>(gas, dust, slab, n, d, dt);
    else return IB_ERROR_NOIMPLEMENT;
    return check_launch();
}

}  // namespace ib
