// ib_common.cuh -- shared device arithmetic of the fluid-step kernels.
//
// Every expression keeps the evaluation order of the reference kernels
// (imogenproject/gpuImogen gpuclass/cudaFluidStep.cu, limiter_functions.h) so that the
// library's strict build (-fmad=false) reproduces the reference arithmetic operation for
// operation; the default build lets nvcc contract multiply-adds.
//
// Memory layout of one fluid: five slabs [rho, E, px, py, pz] of nx*ny*nz doubles each,
// x fastest, slab pitch a multiple of 32 doubles (256 B).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/imogen_b200.h"

namespace ib {

// ------------------------------------------------------------------------------------------
// A timestep-derived factor (a sweep's lambda = dt / h, a source step's dt) given either by value
// or, for loops that keep their timestep on the device (a captured CUDA graph replayed
// iteration after iteration), as (*p * mul) / div read by the kernel itself.  The device form
// performs the division the host would (dt / h), so both give the same bits.  A device
// timestep of exactly 0 marks an iteration after the end time: kernels then return at once.
// ------------------------------------------------------------------------------------------
struct DevScalar {
    double v;
    const double *p;
    double mul, div;
    static DevScalar of(double x) { return DevScalar{x, nullptr, 1.0, 1.0}; }
    static DevScalar device(const double *dtp, double mul, double div) { return DevScalar{0.0, dtp, mul, div}; }
    __device__ __forceinline__ double get() const { return p ? (*p * mul) / div : v; }
    __device__ __forceinline__ bool off() const { return p && *p == 0.0; }
};

// ------------------------------------------------------------------------------------------
// Per-sweep thermodynamic constants (cudaFluidStep.cu:289-311), passed by value.
// ------------------------------------------------------------------------------------------
template <typename FT>
struct FluidConsts {
    FT gamma, gm1, govergm1;
    FT isotemp, isotempsq;
    double minmass, mintemp;  // floors stay FP64
};

template <typename FT>
inline FluidConsts<FT> make_consts(double gamma, double rho_min, double c_iso)
{
    FluidConsts<FT> c;
    c.gamma = (FT)gamma;
    c.gm1 = (FT)(gamma - 1.0);
    c.govergm1 = (FT)(gamma / (gamma - 1.0));
    c.isotemp = (FT)c_iso;
    c.isotempsq = (FT)(c_iso * c_iso);
    c.minmass = rho_min;
    c.mintemp = 1e-5 / (gamma - 1);  // cudaFluidStep.cu:298
    return c;
}

// ------------------------------------------------------------------------------------------
// Limiters (limiter_functions.h:11-119).  Slope limiters return half the limited difference.
// ------------------------------------------------------------------------------------------
template <typename FT>
__device__ __forceinline__ FT flux_minmod(FT A, FT B)
{
    if (A * B < 0) return (FT)0.0;
    if (fabs(A) > fabs(B)) return B;
    return A;
}

template <int SLOPE, typename FT>
__device__ __forceinline__ FT slope_limit(FT A, FT B)
{
    if constexpr (SLOPE == IB_SLOPE_OSPRE) {  // limiter_functions.h:87-95
        FT R = A * B;
        if (R > 0) {
            FT S = A + B;
            return (FT).75 * R * S / (S * S - R);
        }
        return (FT)0.0;
    } else if constexpr (SLOPE == IB_SLOPE_MC) {  // limiter_functions.h:105-115
        if (A * B <= 0) return (FT)0;
#ifdef IB_STRICT_ARITH
        FT R = B / A;
        FT S = (FT).25 + (FT).25 * R;
        S = (S < R) ? S : R;
        S = (S < 1) ? S : (FT)1.0;
        return S * A;
#else
        // min(.25(1+R), R, 1) * A with R = B/A, without the division: for A and B of one sign
        // it is the smaller in magnitude of .25(A+B), B and A
        FT S = (FT).25 * (A + B);
        if (A > 0) {
            S = (S < B) ? S : B;
            return (S < A) ? S : A;
        }
        S = (S > B) ? S : B;
        return (S > A) ? S : A;
#endif
    } else if constexpr (SLOPE == IB_SLOPE_VANLEER) {  // limiter_functions.h:54-61
        FT r = A * B;
        if (r > (FT)0.0) return r / (A + B);
        return (FT)0;
    } else if constexpr (SLOPE == IB_SLOPE_MINMOD) {  // limiter_functions.h:71-77
        // the FP64 reference returns this limiter through a float
        if (A * B < 0) return (FT)0.0;
        if (fabs(A) > fabs(B)) return (FT)(float)((FT).5 * B);
        return (FT)(float)((FT).5 * A);
    } else if constexpr (SLOPE == IB_SLOPE_SUPERBEE) {  // limiter_functions.h:80-86
        if (A * B < 0) return (FT)0.0;
        if (B < A) return flux_minmod<FT>(A, 2 * B);
        return (FT).5 * flux_minmod<FT>(2 * A, B);
    } else if constexpr (SLOPE == IB_SLOPE_VANALBADA) {  // limiter_functions.h:97-102
        FT R = A * B;
        if (R < 0) return (FT)0;
        return (FT).5 * R * (A + B) / (A * A + B * B);
    } else {
        return (FT)0.0;
    }
}

template <int FLIM>
__device__ __forceinline__ double flux_limit(double A, double B)
{
    if constexpr (FLIM == IB_FLUX_OSPRE) {  // limiter_functions.h:36-42
        double r = A * B;
        if (r <= 0.0) return 0.0;
        return 1.5 * r * (A + B) / (A * A + r + B * B);
    } else if constexpr (FLIM == IB_FLUX_VANLEER) {  // limiter_functions.h:11-19
        double r = 2.0 * A * B;
        if (r > 0.0) return r / (A + B);
        return 0;
    } else if constexpr (FLIM == IB_FLUX_MINMOD) {
        return flux_minmod<double>(A, B);
    } else if constexpr (FLIM == IB_FLUX_SUPERBEE) {  // limiter_functions.h:28-34
        if (A * B < 0) return 0.0;
        if (B < A) return flux_minmod<double>(A, 2 * B);
        return flux_minmod<double>(2 * A, B);
    } else {
        return 0.0;
    }
}

template <typename FT>
__device__ __forceinline__ FT dsqrt(FT x) { return sqrt(x); }
template <>
__device__ __forceinline__ float dsqrt<float>(float x) { return sqrtf(x); }

// ------------------------------------------------------------------------------------------
// Einfeldt wave-speed bounds (cudaFluidStep.cu:1728-1755, isothermal 1780-1799)
// ------------------------------------------------------------------------------------------
// irL, irR: 1/rhoL and 1/rhoR as the product build forms them (the HLLC star flux reuses them)
template <typename FT>
__device__ __forceinline__ void einfeldt(const FluidConsts<FT> &c, FT rhoL, FT vL, FT PL, FT rhoR,
                                         FT vR, FT PR, FT dvsq, FT &sl, FT &sr, FT &irL, FT &irR)
{
#ifdef IB_STRICT_ARITH
    FT csql = c.gamma * PL / rhoL;
    FT csqr = c.gamma * PR / rhoR;
    FT Fa = dsqrt<FT>(rhoR / rhoL);
    irL = (FT)1.0 / rhoL;  // unused by the strict star flux, which divides as the reference does
    irR = (FT)1.0 / rhoR;
#else
    irL = (FT)1.0 / rhoL;
    irR = (FT)1.0 / rhoR;
    FT csql = c.gamma * PL * irL;
    FT csqr = c.gamma * PR * irR;
    FT Fa = dsqrt<FT>(rhoR * irL);
#endif
    FT Fb = (FT)1.0 / ((FT)1.0 + Fa);
    FT Croe = ((csql + Fa * csqr) + (FT).5 * c.gm1 * dvsq * Fa * Fb) * Fb;
    FT Vroe = (vL + Fa * vR) * Fb;
    Croe = Vroe - dsqrt<FT>(Croe);
    sl = vL - dsqrt<FT>(csql);
    sr = vR + dsqrt<FT>(csqr);
    sl = (Croe < sl) ? Croe : sl;
    Croe = 2 * Vroe - Croe;
    sr = (Croe > sr) ? Croe : sr;
}

template <typename FT>
__device__ __forceinline__ void einfeldt(const FluidConsts<FT> &c, FT rhoL, FT vL, FT PL, FT rhoR,
                                         FT vR, FT PR, FT dvsq, FT &sl, FT &sr)
{
    FT irL, irR;
    einfeldt<FT>(c, rhoL, vL, PL, rhoR, vR, PR, dvsq, sl, sr, irL, irR);
}

template <typename FT>
__device__ __forceinline__ void einfeldt_iso(FT rhoL, FT vL, FT rhoR, FT vR, FT cs, FT &sl, FT &sr)
{
    FT Fa = dsqrt<FT>(rhoR / rhoL);
    FT Fb = (FT)1.0 / ((FT)1.0 + Fa);
    FT Vroe = (vL + Fa * vR) * Fb;
    cs = Vroe - cs;
    sl = vL - cs;
    sr = vR + cs;
    sl = (cs < sl) ? cs : sl;
    cs = 2 * Vroe - cs;
    sr = (cs > sr) ? cs : sr;
}

// Five-component states.  For HLLC: prims = [rho, e_int, v_n, v_t1, v_t2], edges carry
// [rho, P, v_n, v_t1, v_t2]; fluxes = [rho, E, p_n, p_t1, p_t2].
template <typename FT>
struct V5 {
    FT a[5];
};

// Conserved -> HLLC primitives (cudaFluidStep.cu:1200-1237).  u: [rho, E, p_n, p_t1, p_t2].
template <typename FT>
__device__ __forceinline__ V5<FT> hllc_prims(FT A, FT B, FT C, FT D, FT E)
{
    FT F = (FT)1.0 / A;
    B -= (FT).5 * (C * C + D * D + E * E) * F;
    C *= F;
    D *= F;
    E *= F;
    V5<FT> w;
    w.a[0] = A; w.a[1] = B; w.a[2] = C; w.a[3] = D; w.a[4] = E;
    return w;
}

// Limited faces of one cell from its primitive value and its two backward differences.
// L/R faces: rho, P = gm1*(e -/+ s), v.  (cudaFluidStep.cu:1287-1310)
template <int SLOPE, typename FT>
__device__ __forceinline__ void hllc_faces(const FluidConsts<FT> &c, const V5<FT> &w,
                                           const V5<FT> &dl, const V5<FT> &dr, V5<FT> &L, V5<FT> &R)
{
#pragma unroll
    for (int k = 0; k < 5; k++) {
        FT s = slope_limit<SLOPE, FT>(dl.a[k], dr.a[k]);
        if (k == 1) {
            L.a[1] = c.gm1 * (w.a[1] - s);
            R.a[1] = c.gm1 * (w.a[1] + s);
        } else {
            L.a[k] = w.a[k] - s;
            R.a[k] = w.a[k] + s;
        }
    }
}

// HLLC flux through the face between the right face state of the left cell (l) and the left
// face state of the right cell (r).  (cudaFluidStep.cu:1318-1432)
template <typename FT>
__device__ __forceinline__ V5<FT> hllc_flux(const FluidConsts<FT> &c, const V5<FT> &l, const V5<FT> &r)
{
    const FT rhoL = l.a[0], PL = l.a[1], vxL = l.a[2], vyL = l.a[3], vzL = l.a[4];
    const FT rhoR = r.a[0], PR = r.a[1], vxR = r.a[2], vyR = r.a[3], vzR = r.a[4];
    FT A, B, C, D, E, F, G, H;
    C = vxL - vxR;
    D = vyL - vyR;
    E = vzL - vzR;
    C = C * C + D * D + E * E;
    FT sl, sr, irL, irR;
    einfeldt<FT>(c, rhoL, vxL, PL, rhoR, vxR, PR, C, sl, sr, irL, irR);
    C = sl;
    D = sr;
    A = rhoL * (C - vxL);
    B = rhoR * (D - vxR);
    E = (B * vxR - PR - A * vxL + PL) / (B - A);  // Batten et al. eq. 34

    V5<FT> f;
    if (E > 0) {
        if (C > 0) {  // left state
            A = rhoL; B = vxL; C = vyL; D = vzL;
            E = (FT).5 * (B * B + C * C + D * D) * A;
            F = PL;
            A *= B;
            C *= A;
            D *= A;
            G = A * B + F;
            B *= (E + c.govergm1 * F);
            f.a[0] = A; f.a[1] = B; f.a[2] = G; f.a[3] = C; f.a[4] = D;
        } else {  // left star state
            A = rhoL; B = vxL;
            D = A * (C - B) / (C - E);
            F = vyL; H = vzL;
            G = (FT).5 * (B * B + F * F + H * H);
            A = D * E;
            F *= A;
            H *= A;
            C *= (E - B);
            B = PL + D * (C + E * B);
#ifdef IB_STRICT_ARITH
            G = D * E * (c.govergm1 * PL / rhoL + G + C);
#else
            G = D * E * (c.govergm1 * PL * irL + G + C);
#endif
            f.a[0] = A; f.a[1] = G; f.a[2] = B; f.a[3] = F; f.a[4] = H;
        }
    } else {
        if (D > 0) {  // right star state
            A = rhoR; B = vxR;
            C = A * (D - B) / (D - E);
            F = vyR; H = vzR;
            G = (FT).5 * (B * B + F * F + H * H);
            A = C * E;
            F *= A;
            H *= A;
            D *= (E - B);
            B = PR + C * (D + E * B);
#ifdef IB_STRICT_ARITH
            G = C * E * (c.govergm1 * PR / rhoR + G + D);
#else
            G = C * E * (c.govergm1 * PR * irR + G + D);
#endif
            f.a[0] = A; f.a[1] = G; f.a[2] = B; f.a[3] = F; f.a[4] = H;
        } else {  // right state
            A = rhoR; B = vxR; C = vyR; D = vzR;
            E = (FT).5 * (B * B + C * C + D * D) * A;
            F = PR;
            A *= B;
            C *= A;
            D *= A;
            G = A * B + F;
            B *= (E + c.govergm1 * F);
            f.a[0] = A; f.a[1] = B; f.a[2] = G; f.a[3] = C; f.a[4] = D;
        }
    }
    return f;
}

// Slab offsets (in slabs) of the local components [rho, E, p_n, p_t1, p_t2] for a sweep along
// direction dir; HLLC (cudaFluidStep.cu:1200-1219) and HLL (1864-1882) differ for z.
template <int DIR>
struct HllcSlots {
    static constexpr int n = (DIR == 1) ? 2 : ((DIR == 2) ? 3 : 4);
    static constexpr int t1 = (DIR == 1) ? 3 : ((DIR == 2) ? 2 : 3);
    static constexpr int t2 = (DIR == 1) ? 4 : ((DIR == 2) ? 4 : 2);
};
template <int DIR>
struct HllSlots {
    static constexpr int n = (DIR == 1) ? 2 : ((DIR == 2) ? 3 : 4);
    static constexpr int t1 = (DIR == 1) ? 3 : ((DIR == 2) ? 2 : 2);
    static constexpr int t2 = (DIR == 1) ? 4 : ((DIR == 2) ? 4 : 3);
};

__device__ __forceinline__ int wrapi(int i, int n) { return (i < 0) ? i + n : ((i >= n) ? i - n : i); }

// Pencil addressing: pencil index p of a sweep along dir -> offset of its first cell.
struct PencilMap {
    int nx, ny, nz;
    int dir;
    __device__ __forceinline__ int64_t base(int64_t p) const
    {
        if (dir == 1) return p * nx;
        if (dir == 2) {
            int64_t x = p % nx, z = p / nx;
            return x + (int64_t)nx * ny * z;
        }
        return p;
    }
    __device__ __forceinline__ int64_t stride() const
    {
        return dir == 1 ? 1 : (dir == 2 ? (int64_t)nx : (int64_t)nx * ny);
    }
    __device__ __forceinline__ int length() const { return dir == 1 ? nx : (dir == 2 ? ny : nz); }
};

}  // namespace ib
