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

// solveDragEMP (cudaSource2FluidDrag.cu:305-370) / solveDragRK4 (:372-475) on the scalar
// relative speed, then cukern_applyFinalDeltaV; cells with |dv| < 1e-9 are left unchanged (the
// reference divides by |dv| there).
template <bool RK4>
__global__ void __launch_bounds__(256) rk_drag_kernel(double *__restrict__ gas, double *__restrict__ dust, int64_t S,
                                                      int64_t n, DragParams d, double dt)
{
    for (int64_t x = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; x < n; x += (int64_t)blockDim.x * gridDim.x) {
        double *g = gas + x, *ds = dust + x;
        double w0, u0, f, acc, stage, wf;
        drag_initial_dv(g, ds, S, w0, u0);
        if (w0 < 1e-9) continue;
        const double rA = g[0], rB = ds[0];
        f = drag_accel<true>(d, rA, rB, w0, u0, w0);
        if (!RK4) {
            stage = w0 + (.5 * dt) * f;
            acc = 0 * f;
            f = drag_accel<false>(d, rA, rB, w0, u0, stage);
            wf = w0 + dt * (acc + 1.0 * f);
        } else {
            stage = w0 + (0.5 * dt) * f;
            acc = 1.0 * f;
            f = drag_accel<false>(d, rA, rB, w0, u0, stage);
            stage = w0 + (0.5 * dt) * f;
            acc += 2.0 * f;
            f = drag_accel<false>(d, rA, rB, w0, u0, stage);
            stage = w0 + (1.0 * dt) * f;
            acc += 2.0 * f;
            f = drag_accel<false>(d, rA, rB, w0, u0, stage);
            wf = w0 + (dt / 6.0) * (acc + 1.0 * f);
        }
        drag_apply_final_dv(g, ds, S, wf);
    }
}

// solveDragETDRK1 (cudaSource2FluidDrag.cu:477-560, no pressure-gradient term): exponential
// Euler with the drag rate at t = 0; cells with |dv| < 1e-9 (k = 0) are left unchanged (the
// reference evaluates 0/0 there).
__global__ void __launch_bounds__(256) etdrk1_kernel(double *__restrict__ gas, double *__restrict__ dust, int64_t S,
                                                     int64_t n, DragParams d, double t)
{
    for (int64_t x = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; x < n; x += (int64_t)blockDim.x * gridDim.x) {
        double *g = gas + x, *ds = dust + x;
        const double g0 = g[0], gE = g[S], g2 = g[2 * S], g3 = g[3 * S], g4 = g[4 * S];
        const double d0 = ds[0], d2 = ds[2 * S], d3 = ds[3 * S], d4 = ds[4 * S];
        double t0, t1;
        bool skip;
        drag_features(g0, gE, g2, g3, g4, d0, d2, d3, d4, t0, t1);
        const double k = drag_k(d, g0, d0, t0, t1, skip);
        if (skip) continue;
        drag_apply_etdrk1(g, ds, S, t, k);
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
    else if (method == IB_DRAG_EMP) rk_drag_kernel<false><<<nb, 256, 0, st>>>(gas, dust, slab, n, d, dt);
    else if (method == IB_DRAG_RK4) rk_drag_kernel<true><<<nb, 256, 0, st>>>(gas, dust, slab, n, d, dt);
    else if (method == IB_DRAG_ETDRK1) etdrk1_kernel<<<nb, 256, 0, st>>>(gas, dust, slab, n, d, dt);
    else return IB_ERROR_NOIMPLEMENT;  // ETDRK2 needs the finite-difference pressure gradient
    return check_launch();
}

}  // namespace ib
