// ib_cfl.cuh -- per-cell soundspeed and CFL signal-crossing time, shared by the reduction
// kernels and the fused ensemble kernel.
#pragma once

#include "ib_common.cuh"

namespace ib {

// c_s^2 = gamma(gamma-1)(E - p^2/2rho)/rho, clamped at 0 (cudaSoundspeed.cu:184-191)
__device__ __forceinline__ double soundspeed_cell(double rho, double E, double px, double py, double pz, double gg1)
{
    double rhoinv = 1 / rho;
    double csq = gg1 * (E - .5 * (px * px + py * py + pz * pz) * rhoinv) * rhoinv;
    if (csq < 0.0) csq = 0.0;
    return sqrt(csq);
}

// Signal-crossing time of one cell (cflTimestep.cu:254-340).  sim = spatial dimension.
template <int SIM, bool XJ>
__device__ __forceinline__ double cfl_cell(double rho, double px, double py, double pz, double cs, double hmin,
                                           double hx, double hy, double hz)
{
    double u;
    if constexpr (!XJ) {
        double p;
        if constexpr (SIM == 1) {
            p = fabs(px);
        } else {
            double pp = px * px;
            pp = pp + py * py;
            if constexpr (SIM > 2) pp = pp + pz * pz;
            p = sqrt(pp);
        }
        u = p / rho + cs;
        u = hmin / u;
    } else {
        double v;
        u = hx / (fabs(px) / rho + cs);
        v = hy / (fabs(py) / rho + cs);
        u = (u < v) ? u : v;
        if constexpr (SIM > 2) {
            v = hz / (fabs(pz) / rho + cs);
            u = (u < v) ? u : v;
        }
    }
    return u;
}

// The same in cylindrical geometry (cflTimestep.cu:301-333): hx = dr, hy = dtheta, rc = the cell's
// radius r_inner + i dr; hmin = dr (min(dr, dz) in 3-D).  HLL/HLLC take min(rc dtheta, hmin) over
// the speed |p|/rho + c_s; Xin-Jin takes the r and z crossing times and rc dtheta over |v_theta| + c_s.
template <int SIM, bool XJ>
__device__ __forceinline__ double cfl_cell_cyl(double rho, double px, double py, double pz, double cs, double hmin,
                                               double hx, double hy, double hz, double rin, int i)
{
    double u;
    if constexpr (!XJ) {
        double p;
        if constexpr (SIM == 1) {
            p = fabs(px);
        } else {
            double pp = px * px;
            pp = pp + py * py;
            if constexpr (SIM > 2) pp = pp + pz * pz;
            p = sqrt(pp);
        }
        u = p / rho + cs;
        double w = (rin + i * hx) * hy;
        w = (w < hmin) ? w : hmin;
        u = w / u;
    } else {
        double v;
        u = hx / (fabs(px) / rho + cs);
        if constexpr (SIM > 1) {
            v = (rin + i * hx) * hy / (fabs(py) / rho + cs);
            u = (u < v) ? u : v;
        }
        if constexpr (SIM > 2) {
            v = hz / (fabs(pz) / rho + cs);
            u = (u < v) ? u : v;
        }
    }
    return u;
}

// NaN-ignoring minimum, as the reference's ternaries: a NaN candidate never replaces the running value
__device__ __forceinline__ double min_keep(double cur, double cand) { return (cand < cur) ? cand : cur; }

}  // namespace ib
