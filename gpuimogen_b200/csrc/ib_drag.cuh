// ib_drag.cuh -- drag law and LogTrap update shared by the exact and the learned drag kernels
// (gpuclass/cudaSource2FluidDrag.cu).
#pragma once

#include <cmath>

#include "ib_common.cuh"

namespace ib {

struct DragParams {
    double visc0, viscpow, lampow, alpha, beta, delta, epsilon;
};

// x^y.  The strict build calls pow as the reference does; the product build uses
// exp(y log x) for positive finite x (one log shared by the two powers of the temperature in the
// drag law), within a few ulp of pow for the drag law's exponents and arguments.
struct PowBase {
    double x, lx;
    bool fast;
};
__device__ __forceinline__ PowBase pow_base(double x)
{
#ifdef IB_STRICT_ARITH
    return PowBase{x, 0.0, false};
#else
    const bool fast = x > 0.0 && x < 1e300;
    return PowBase{x, fast ? log(x) : 0.0, fast};
#endif
}
__device__ __forceinline__ double pow_of(const PowBase &b, double y)
{
    return b.fast ? exp(y * b.lx) : pow(b.x, y);
}

// allregimeCdrag (cudaSource2FluidDrag.cu:819-833)
__device__ __forceinline__ double allregime_cdrag(double Re, double Kn)
{
    double cunningham = 1 + Kn * (1.142 + 1 * 0.558 * exp(-0.999 / Kn));
    double C_drag = (3 / Re + .45 * pow_of(pow_base(Re), -.319) + .0509 * Re / (8710 + Re)) / cunningham;
    return C_drag;
}

// cukern_GasDustDrag_GeneralLinearCore with srcBlock 0 (cudaSource2FluidDrag.cu:836-890)
__device__ __forceinline__ double drag_k(const DragParams &d, double rhoA, double rhoB, double magdv, double u, bool &skip)
{
    if (magdv < 1e-9) { skip = true; return 0; }
    skip = false;
    double Tn = d.alpha * u;
    const PowBase bT = pow_base(Tn);
    double Re = d.delta * rhoA * magdv * pow_of(bT, d.viscpow);
    double Kn = d.beta * pow_of(bT, d.lampow) / rhoA;
    double Cd_hat = allregime_cdrag(Re, Kn);
    return Cd_hat * magdv * (rhoA + rhoB) * d.epsilon;
}

// LogTrap effective rate k_eff of one cell from rho_gas g0, rho_dust d0, |dv| t0 and specific
// internal energy t1 (cukern_LogTrapSolve, cudaSource2FluidDrag.cu:1531-1660); the update then
// scales dv by exp(-t k_eff).
template <int ORDER>
__device__ __forceinline__ double logtrap_keff(const DragParams &d, double g0, double d0, double t0, double t1, double t)
{
    double mu, k, dv_i, dv_t, dvsq, duint, t2;
    bool skip;
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
    return k;
}

// Relative-velocity features of one cell: |dv| and the gas specific internal energy
// (cukern_prepareForERK_h0, cudaSource2FluidDrag.cu:1883-1908).
__device__ __forceinline__ void drag_features(double g0, double gE, double g2, double g3, double g4, double d0, double d2,
                                              double d3, double d4, double &magdv, double &u)
{
    double dv, dvsq, press;
#ifdef IB_STRICT_ARITH
    dv = (g2) / g0 - d2 / d0;
    dvsq = dv * dv;
    dv = (g3) / g0 - d3 / d0;
    dvsq += dv * dv;
    dv = (g4) / g0 - d4 / d0;
    dvsq += dv * dv;
    press = (gE - .5 * (g2 * g2 + g3 * g3 + g4 * g4) / g0);
    magdv = sqrt(dvsq);
    u = press / g0;
#else  // the two density reciprocals once instead of eight divisions
    const double ig = 1.0 / g0, id = 1.0 / d0;
    dv = g2 * ig - d2 * id;
    dvsq = dv * dv;
    dv = g3 * ig - d3 * id;
    dvsq += dv * dv;
    dv = g4 * ig - d4 * id;
    dvsq += dv * dv;
    press = (gE - .5 * (g2 * g2 + g3 * g3 + g4 * g4) * ig);
    magdv = sqrt(dvsq);
    u = press * ig;
#endif
}

// Momentum exchange about the centre-of-mass velocity with dv -> dv exp(-t k), gas energy
// absorbing the dust's kinetic-energy change (cudaSource2FluidDrag.cu:1660-1686).
__device__ __forceinline__ void drag_apply(double *g, double *ds, int64_t S, double g0, double gE, double g2, double g3,
                                           double g4, double d0, double d2, double d3, double d4, double t, double k)
{
    double mu, rhoginv, pdustsq, vstick, dv_i, dv_t, qq;
    // the reference evaluates exp(-t k) once per axis with the same argument; once is the same value
    const double decay = exp(-t * k);
#ifdef IB_STRICT_ARITH
    mu = d0 / (g0 + d0);
    mu = mu * g0;
    rhoginv = 1.0 / g0;
    auto over_sum = [&](double x) { return x / (g0 + d0); };
    auto over_d0 = [&](double x) { return x / d0; };
#else  // three reciprocals instead of nine divisions
    const double isum = 1.0 / (g0 + d0), rhodinv = 1.0 / d0;
    mu = d0 * isum;
    mu = mu * g0;
    rhoginv = 1.0 / g0;
    auto over_sum = [&](double x) { return x * isum; };
    auto over_d0 = [&](double x) { return x * rhodinv; };
#endif

    pdustsq = -d2 * d2;
    vstick = over_sum(g2 + d2);
    dv_i = (g2) * rhoginv - over_d0(d2);
    dv_t = dv_i * decay;
    g[2 * S] = g0 * vstick + dv_t * mu;
    ds[2 * S] = qq = d0 * vstick - dv_t * mu;
    pdustsq += qq * qq;

    pdustsq -= d3 * d3;
    vstick = over_sum(g3 + d3);
    dv_i = (g3) * rhoginv - over_d0(d3);
    dv_t = dv_i * decay;
    g[3 * S] = g0 * vstick + dv_t * mu;
    ds[3 * S] = qq = d0 * vstick - dv_t * mu;
    pdustsq += qq * qq;

    pdustsq -= d4 * d4;
    vstick = over_sum(g4 + d4);
    dv_i = (g4) * rhoginv - over_d0(d4);
    dv_t = dv_i * decay;
    g[4 * S] = g0 * vstick + dv_t * mu;
    ds[4 * S] = qq = d0 * vstick - dv_t * mu;
    pdustsq += qq * qq;

#ifdef IB_STRICT_ARITH
    g[S] = gE - .5 * pdustsq / d0;
#else
    g[S] = gE - .5 * pdustsq * rhodinv;
#endif
}

// cukern_GasDustDrag_GeneralAccel (cudaSource2FluidDrag.cu:898-931): -d|dv|/dt at |dv| = w; the
// gas is credited with the relative kinetic energy dissipated since w0 unless INI.
template <bool INI>
__device__ __forceinline__ double drag_accel(const DragParams &d, double rhoA, double rhoB, double w0, double u0, double w)
{
    double u;
    if (INI) u = u0;
    else u = u0 + .5 * rhoB * (w0 * w0 - w * w) / (rhoA + rhoB);
    const double Tn = d.alpha * u;
    const PowBase bT = pow_base(Tn);
    const double Re = d.delta * rhoA * w * pow_of(bT, d.viscpow);
    const double Kn = d.beta * pow_of(bT, d.lampow) / rhoA;
    const double Cd_hat = allregime_cdrag(Re, Kn);
    return -(Cd_hat * w * w * (rhoA + rhoB) * d.epsilon);
}

// cukern_findInitialDeltaV (cudaSource2FluidDrag.cu:1014-1050): w0 = |dv|, u0 = e_int / rho_gas
__device__ __forceinline__ void drag_initial_dv(const double *g, const double *ds, int64_t S, double &w0, double &u0)
{
    double u, q, dvsq, rhoginv, rhodinv, momsq;
    rhoginv = 1 / g[0];
    rhodinv = 1 / ds[0];
    q = g[2 * S];
    u = q * rhoginv - ds[2 * S] * rhodinv;
    momsq = q * q;
    dvsq = u * u;
    q = g[3 * S];
    u = q * rhoginv - ds[3 * S] * rhodinv;
    momsq += q * q;
    dvsq += u * u;
    q = g[4 * S];
    u = q * rhoginv - ds[4 * S] * rhodinv;
    momsq += q * q;
    dvsq += u * u;
    w0 = sqrt(dvsq);
    u0 = (g[S] - .5 * momsq * rhoginv) * rhoginv;
}

// cukern_applyFinalDeltaV (cudaSource2FluidDrag.cu:1160-1229)
__device__ __forceinline__ void drag_apply_final_dv(double *g, double *ds, int64_t S, double wf)
{
    double vstick[3], dvhat[3], a, b, c, p1, p2, dustmom, dustmomfin;
    const double rhog = g[0], rhod = ds[0];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        p1 = g[(2 + k) * S];
        p2 = ds[(2 + k) * S];
        vstick[k] = (p1 + p2) / (rhog + rhod);
        dvhat[k] = p1 / rhog - p2 / rhod;
    }
    a = wf / sqrt(dvhat[0] * dvhat[0] + dvhat[1] * dvhat[1] + dvhat[2] * dvhat[2]);
    dvhat[0] *= a;
    dvhat[1] *= a;
    dvhat[2] *= a;
    b = rhog * rhod / (rhog + rhod);
    dustmom = ds[2 * S] * ds[2 * S];
    g[2 * S] = rhog * vstick[0] + dvhat[0] * b;
    ds[2 * S] = c = rhod * vstick[0] - dvhat[0] * b;
    dustmomfin = c * c;
    dustmom += ds[3 * S] * ds[3 * S];
    g[3 * S] = rhog * vstick[1] + dvhat[1] * b;
    ds[3 * S] = c = rhod * vstick[1] - dvhat[1] * b;
    dustmomfin += c * c;
    dustmom += ds[4 * S] * ds[4 * S];
    g[4 * S] = rhog * vstick[2] + dvhat[2] * b;
    ds[4 * S] = c = rhod * vstick[2] - dvhat[2] * b;
    dustmomfin += c * c;
    g[S] += .5 * (dustmom - dustmomfin) / ds[0];
    ds[S] = .5 * dustmomfin / ds[0] + 1e-4 * ds[0];
}

// cukern_ETDRK1 without the pressure-gradient term (cudaSource2FluidDrag.cu:1426-1510) with the
// drag rate k at t = 0; k > 0.
__device__ __forceinline__ void drag_apply_etdrk1(double *gas, double *dust, int64_t S, double t, double k)
{
    double rhoginv, mu, pdustsq, vstick, dv_i, dv_t, q, dpdt;
    rhoginv = 1.0 / gas[0];
    mu = gas[0] * dust[0] / (gas[0] + dust[0]);
    pdustsq = 0;
#pragma unroll
    for (int ax = 2; ax <= 4; ax++) {
        pdustsq -= dust[ax * S] * dust[ax * S];
        vstick = (gas[ax * S] + dust[ax * S]) / (gas[0] + dust[0]);
        dpdt = 0;
        dv_i = (gas[ax * S]) * rhoginv - dust[ax * S] / dust[0];
        dpdt *= mu * rhoginv;
        dv_t = dpdt / k + (dv_i - dpdt / k) * exp(-t * k);
        gas[ax * S] = gas[0] * vstick + dv_t * mu;
        dust[ax * S] = q = dust[0] * vstick - dv_t * mu;
        pdustsq += q * q;
    }
    gas[S] -= .5 * pdustsq / dust[0];
}

// Drag constants dragparams[0..6] (cudaSource2FluidDrag.cu:196-218).
inline DragParams drag_constants(const ib_thermo *tg, const ib_thermo *td)
{
    const double gam = tg->gamma;
    const double ddust = sqrt(td->sigma0 / 3.141592653589793);
    DragParams d;
    d.visc0 = tg->mu0;
    d.viscpow = -tg->mu_t_index;
    d.lampow = tg->sigma_t_index;
    d.alpha = tg->mass * (gam - 1.0) / (298.15 * tg->k_bolt);
    d.beta = sqrt(2.0) * tg->mass / (tg->sigma0 * ddust);
    d.delta = ddust / tg->mu0;
    d.epsilon = td->sigma0 / (1.0 * td->mass);
    return d;
}

}  // namespace ib
