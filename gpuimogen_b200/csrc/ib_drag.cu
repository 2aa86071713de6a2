// ib_drag.cu -- two-fluid gas-dust drag source (gpuclass/cudaSource2FluidDrag.cu).
//
// The reference's default LogTrap2 path runs two kernels over a 3-slab temporary: one writes
// [|dv|, e_int/rho] (cukern_prepareForERK_h0, :1883-1908), the other integrates the drag
// (cukern_LogTrapSolve, :1531-1686) launched with at most 32 blocks of 96 threads (:730-757).
// Here one kernel does both per cell with the temporaries in registers, over a full-GPU grid:
// 10 doubles read and 7 written per cell.
#include "ib_internal.cuh"

namespace ib {

struct DragParams {
    double visc0, viscpow, lampow, alpha, beta, delta, epsilon;
};

// allregimeCdrag (cudaSource2FluidDrag.cu:819-833)
__device__ __forceinline__ double allregime_cdrag(double Re, double Kn)
{
    double cunningham = 1 + Kn * (1.142 + 1 * 0.558 * exp(-0.999 / Kn));
    double C_drag = (3 / Re + .45 * pow(Re, -.319) + .0509 * Re / (8710 + Re)) / cunningham;
    return C_drag;
}

// cukern_GasDustDrag_GeneralLinearCore with srcBlock 0 (cudaSource2FluidDrag.cu:836-890)
__device__ __forceinline__ double drag_k(const DragParams &d, double rhoA, double rhoB, double magdv, double u, bool &skip)
{
    if (magdv < 1e-9) { skip = true; return 0; }
    skip = false;
    double Tn = d.alpha * u;
    double Re = d.delta * rhoA * magdv * pow(Tn, d.viscpow);
    double Kn = d.beta * pow(Tn, d.lampow) / rhoA;
    double Cd_hat = allregime_cdrag(Re, Kn);
    return Cd_hat * magdv * (rhoA + rhoB) * d.epsilon;
}

template <int ORDER>
__global__ void __launch_bounds__(256) logtrap_kernel(double *__restrict__ gas, double *__restrict__ dust, int64_t S,
                                                      int64_t n, DragParams d, double t)
{
    for (int64_t x = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; x < n; x += (int64_t)blockDim.x * gridDim.x) {
        double *g = gas + x, *ds = dust + x;
        const double g0 = g[0], gE = g[S], g2 = g[2 * S], g3 = g[3 * S], g4 = g[4 * S];
        const double d0 = ds[0], d2 = ds[2 * S], d3 = ds[3 * S], d4 = ds[4 * S];
        double dv, dvsq, press, t0, t1, t2;
        double mu, k, dv_i, dv_t, duint, rhoginv, pdustsq, vstick, qq;
        bool skip;
        // prepare: [|dv|, u] (cukern_prepareForERK_h0)
        dv = (g2) / g0 - d2 / d0;
        dvsq = dv * dv;
        dv = (g3) / g0 - d3 / d0;
        dvsq += dv * dv;
        dv = (g4) / g0 - d4 / d0;
        dvsq += dv * dv;
        press = (gE - .5 * (g2 * g2 + g3 * g3 + g4 * g4) / g0);
        t0 = sqrt(dvsq);
        t1 = press / g0;
        // LogTrap (cukern_LogTrapSolve)
        mu = d0 / (g0 + d0);
        k = drag_k(d, g0, d0, t0, t1, skip);
        t2 = skip ? 0 : k;
        k = t2;
        dv_i = t0;
        dv_t = dv_i * exp(-t * k);
        dvsq = dv_t * dv_t;
        duint = -.5 * dv_i * dv_i * mu * expm1(-2 * k * t);
        t0 = sqrt(dvsq);
        t1 += duint;
        k = drag_k(d, g0, d0, t0, t1, skip);
        if (!skip) t2 += k;
        if (ORDER == 3) {
            t1 -= duint;
            k = .25 * (t2);
            dv_t = dv_i * exp(-t * k);
            dvsq = dv_t * dv_t;
            duint = -0.5 * dv_i * dv_i * mu * expm1(-2 * k * t);
            t0 = sqrt(dvsq);
            t1 += duint;
            k = drag_k(d, g0, d0, t0, t1, skip);
            t0 = skip ? 0 : k;
            k = (0.16666666666666666667 * t2 + 0.66666666666666666667 * t0);
        } else {
            k = .5 * t2;
        }
        mu = mu * g0;
        rhoginv = 1.0 / g0;

        pdustsq = -d2 * d2;
        vstick = (g2 + d2) / (g0 + d0);
        dv_i = (g2) * rhoginv - d2 / d0;
        dv_t = dv_i * exp(-t * k);
        g[2 * S] = g0 * vstick + dv_t * mu;
        ds[2 * S] = qq = d0 * vstick - dv_t * mu;
        pdustsq += qq * qq;

        pdustsq -= d3 * d3;
        vstick = (g3 + d3) / (g0 + d0);
        dv_i = (g3) * rhoginv - d3 / d0;
        dv_t = dv_i * exp(-t * k);
        g[3 * S] = g0 * vstick + dv_t * mu;
        ds[3 * S] = qq = d0 * vstick - dv_t * mu;
        pdustsq += qq * qq;

        pdustsq -= d4 * d4;
        vstick = (g4 + d4) / (g0 + d0);
        dv_i = (g4) * rhoginv - d4 / d0;
        dv_t = dv_i * exp(-t * k);
        g[4 * S] = g0 * vstick + dv_t * mu;
        ds[4 * S] = qq = d0 * vstick - dv_t * mu;
        pdustsq += qq * qq;

        g[S] = gE - .5 * pdustsq / d0;
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
