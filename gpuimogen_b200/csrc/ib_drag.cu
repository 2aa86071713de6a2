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
                                                      int64_t n, DragParams d, DevScalar dts)
{
    if (dts.off()) return;  // a device timestep of 0: after the end time
    const double t = dts.get();
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
                                                      int64_t n, DragParams d, DevScalar dts)
{
    if (dts.off()) return;
    const double dt = dts.get();
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
                                                     int64_t n, DragParams d, DevScalar dts)
{
    if (dts.off()) return;
    const double t = dts.get();
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

// solveDragETDRK2 (cudaSource2FluidDrag.cu:575-690), exponential midpoint, in two kernels: the
// gas internal energy density e_int = E - p^2/2rho (gas2press, :1870-1873) goes to a scratch slab,
// then one thread per cell takes its periodic central differences (the pressure gradient of
// prepareForExpMethod with spaceOrder 2, :1728-1866), the drag rate k0, the driven half step of
// cukern_ExpMidpoint_partA (:1247-1312), the rate k1 there and the update of
// cukern_ExpMidpoint_partB (:1325-1420), all in registers.  findMidGradP2 (:2395-2520) rewrites
// only gradient slabs that no later kernel reads, so it is not run.  Cells where k0 or k1 is zero
// (|dv| < 1e-9) are left unchanged; the reference evaluates 0/0 there.
__global__ void __launch_bounds__(256) eint_kernel(const double *__restrict__ gas, int64_t S, int64_t n,
                                                   double *__restrict__ P)
{
    for (int64_t x = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; x < n; x += (int64_t)blockDim.x * gridDim.x) {
        const double g0 = gas[x], gE = gas[S + x], g2 = gas[2 * S + x], g3 = gas[3 * S + x], g4 = gas[4 * S + x];
        P[x] = (gE - .5 * (g2 * g2 + g3 * g3 + g4 * g4) / g0);
    }
}

struct Etd2Grid {
    int nx, ny, nz;
    int layout;                // 0: 3-D, 1: x-y plane (nz = 1), 2: x-z plane (ny = 1 < nz)
    double lamx, lamy, lamz;   // (gamma - 1) / (2 h)
    double gm1;
};

__global__ void __launch_bounds__(256) etdrk2_kernel(double *__restrict__ gas, double *__restrict__ dust, int64_t S,
                                                     const double *__restrict__ P, Etd2Grid G, DragParams d,
                                                     DevScalar dts)
{
    if (dts.off()) return;
    const double t = dts.get();
    const int64_t chunks = (G.nx + blockDim.x - 1) / blockDim.x;
    const int64_t work = chunks * G.ny * G.nz;
    for (int64_t w = blockIdx.x; w < work; w += gridDim.x) {
        const int64_t row = w / chunks;
        const int x = (int)(w - row * chunks) * (int)blockDim.x + (int)threadIdx.x;
        if (x >= G.nx) continue;
        const int y = (int)(row % G.ny), z = (int)(row / G.ny);
        const int xm = (x == 0) ? G.nx - 1 : x - 1, xp = (x == G.nx - 1) ? 0 : x + 1;
        const int ym = (y == 0) ? G.ny - 1 : y - 1, yp = (y == G.ny - 1) ? 0 : y + 1;
        const int zm = (z == 0) ? G.nz - 1 : z - 1, zp = (z == G.nz - 1) ? 0 : z + 1;
        const int64_t nx = G.nx, plane = (int64_t)G.nx * G.ny;
        const int64_t i = row * nx + x;
        double *g = gas + i, *ds = dust + i;
        const double g0 = g[0], g2 = g[2 * S], g3 = g[3 * S], g4 = g[4 * S];
        const double d0 = ds[0], d2 = ds[2 * S], d3 = ds[3 * S], d4 = ds[4 * S];
        double Gr[3], dvx, dvy, dvz, dvsq;
        Gr[0] = G.lamx * (P[row * nx + xp] - P[row * nx + xm]);
        dvx = (g2) / g0 - d2 / d0;
        dvy = (g3) / g0 - d3 / d0;
        dvz = (g4) / g0 - d4 / d0;
        if (G.layout == 0) {
            Gr[1] = G.lamy * (P[z * plane + yp * nx + x] - P[z * plane + ym * nx + x]);
            Gr[2] = G.lamz * (P[zp * plane + y * nx + x] - P[zm * plane + y * nx + x]);
            dvsq = dvx * dvx;
            dvsq += dvy * dvy;
            dvsq += dvz * dvz;
        } else if (G.layout == 2) {
            Gr[1] = 0.0;
            Gr[2] = G.lamz * (P[zp * nx + x] - P[zm * nx + x]);
            dvsq = dvy * dvy;
            dvsq += dvx * dvx;
            dvsq += dvz * dvz;
        } else {
            Gr[1] = G.lamy * (P[yp * nx + x] - P[ym * nx + x]);
            Gr[2] = 0.0;
            dvsq = dvz * dvz;
            dvsq += dvx * dvx;
            dvsq += dvy * dvy;
        }
        double t0 = sqrt(dvsq), t1 = P[i] / g0;
        bool skip;
        double k = drag_k(d, g0, d0, t0, t1, skip);
        if (skip) continue;
        // partA: driven decay of each component over t with rate k0
        const double rhoginv = 1.0 / g0;
        const double mom[3] = {g2, g3, g4};
        double duint = 0;
        dvsq = 0;
#pragma unroll
        for (int ax = 0; ax < 3; ax++) {
            double a0 = Gr[ax], dv_i;
            if (ax == 0) dv_i = (g2 + t * a0) * rhoginv - d2 / d0;
            else dv_i = (mom[ax]) * rhoginv - d3 / d0;  // the reference reads the dust y momentum for z too
            a0 *= rhoginv / k;
            const double dv_t = a0 + (dv_i - a0) * exp(-t * k);
            const double q = k * a0 * a0 * t - 2 * a0 * (dv_i - a0) * expm1(-k * t) -
                             (dv_i - a0) * (dv_i - a0) * expm1(-2 * k * t);
            if (ax == 0) { dvsq = dv_t * dv_t; duint = q; }
            else { dvsq += dv_t * dv_t; duint += q; }
        }
        t0 = sqrt(dvsq);
        t1 += G.gm1 * duint * rhoginv;
        k = drag_k(d, g0, d0, t0, t1, skip);
        if (skip) continue;
        // partB: dv -> dv exp(-t k1) about the centre-of-mass velocity
        drag_apply_etdrk1(g, ds, S, t, k);
    }
}

int launch_drag(double *gas, double *dust, int64_t slab, const int grid[3], const double h[3], const double dp[11],
                DevScalar dt, int method, cudaStream_t st)
{
    DragParams d{dp[0], dp[1], dp[2], dp[3], dp[4], dp[5], dp[6]};
    const int64_t n = (int64_t)grid[0] * grid[1] * grid[2];
    if (n <= 0) return IB_SUCCESSFUL;
    int nb = (int)std::min<int64_t>((n + 255) / 256, (int64_t)16 * num_sms());
    if (method == IB_DRAG_LOGTRAP2) logtrap_kernel<2><<<nb, 256, 0, st>>>(gas, dust, slab, n, d, dt);
    else if (method == IB_DRAG_LOGTRAP3) logtrap_kernel<3><<<nb, 256, 0, st>>>(gas, dust, slab, n, d, dt);
    else if (method == IB_DRAG_EMP) rk_drag_kernel<false><<<nb, 256, 0, st>>>(gas, dust, slab, n, d, dt);
    else if (method == IB_DRAG_RK4) rk_drag_kernel<true><<<nb, 256, 0, st>>>(gas, dust, slab, n, d, dt);
    else if (method == IB_DRAG_ETDRK1) etdrk1_kernel<<<nb, 256, 0, st>>>(gas, dust, slab, n, d, dt);
    else if (method == IB_DRAG_ETDRK2) {
        if (!h) return IB_ERROR_NULL_POINTER;
        double *P = scratch().bytes((size_t)n * sizeof(double));
        if (!P) return IB_ERROR_NOMEM;
        eint_kernel<<<nb, 256, 0, st>>>(gas, slab, n, P);
        int rc = check_launch();
        if (rc) return rc;
        Etd2Grid G;
        G.nx = grid[0]; G.ny = grid[1]; G.nz = grid[2];
        G.layout = (G.nz > 1 && G.ny > 1) ? 0 : (G.nz > 1 ? 2 : 1);
        // prepareForExpMethod (cudaSource2FluidDrag.cu:1737-1741): scaling gamma - 1 over 2 h
        G.lamx = dp[8] / (2.0 * h[0]);
        G.lamy = dp[8] / (2.0 * h[1]);
        G.lamz = dp[8] / (2.0 * h[2]);
        G.gm1 = dp[8];
        const int64_t work = ((int64_t)(G.nx + 255) / 256) * G.ny * G.nz;
        const int nb2 = (int)std::min<int64_t>(work, (int64_t)16 * num_sms());
        etdrk2_kernel<<<nb2, 256, 0, st>>>(gas, dust, slab, P, G, d, dt);
    } else return IB_ERROR_NOIMPLEMENT;
    return check_launch();
}

}  // namespace ib
