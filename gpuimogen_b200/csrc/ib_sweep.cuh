// ib_sweep.cuh -- fused SSPRK2 directional sweep kernels (HLLC, HLL) without transposes.
//
// The reference runs each sweep as two kernels (stage A into a 6-slab temporary, stage B
// back into the fluid) along memory x, after transposing the arrays so that the swept axis is
// fastest (gpuclass/flux.cu:46-49, cudaArrayRotateB.cu).  Each stage's value at cell i depends
// only on cells i-2..i+2 of the row, periodically wrapped (cudaFluidStep.cu:1157-1162), so here
// both stages run in one kernel straight on the XYZ arrays:
//
//  * row kernel (x sweeps, rows up to 1024 cells): one CTA holds one whole periodic row, one
//    thread per cell (or two), neighbours exchanged through two shared-memory planes;
//    coalesced loads and stores, no halo recomputation.
//  * pipeline kernels (y and z sweeps of pencils up to 512 cells): persistent CTAs walk blocks
//    of adjacent whole pencils that arrive by TMA, double-buffered, and leave by TMA store.
//  * chunked pipeline (pencils above 512 cells): chunks with 4 halo rows per side, the halos
//    copied to a side buffer first so every chunk is an independent job.
//  * tile kernel (whatever the TMA rules exclude: odd nx, long odd rows): a CTA walks four
//    neighbouring pencils in chunks staged in shared memory.
#pragma once

#include <type_traits>

#include "ib_common.cuh"
#include "ib_tma.cuh"
#include "ib_cyl.cuh"

namespace ib {

// ------------------------------------------------------------------------------------------
// Stage helpers shared by both kernels
// ------------------------------------------------------------------------------------------
template <typename FT>
__device__ __forceinline__ V5<FT> v5_sub(const V5<FT> &a, const V5<FT> &b)
{
    V5<FT> r;
#pragma unroll
    for (int k = 0; k < 5; k++) r.a[k] = a.a[k] - b.a[k];
    return r;
}

// HLL primitives: [rho, v_n, P, v_t1, v_t2] with P taken from the floored pressure
// (cudaFluidStep.cu:1864-1888)
template <typename FT>
__device__ __forceinline__ V5<FT> hll_prims(FT rho, FT pn, FT P, FT pt1, FT pt2)
{
    V5<FT> w;
    w.a[0] = rho;
    w.a[1] = pn / rho;
    w.a[2] = P;
    w.a[3] = pt1 / rho;
    w.a[4] = pt2 / rho;
    return w;
}

template <int SLOPE, typename FT>
__device__ __forceinline__ void hll_faces(const V5<FT> &w, const V5<FT> &dl, const V5<FT> &dr,
                                          V5<FT> &L, V5<FT> &R)
{
#pragma unroll
    for (int k = 0; k < 5; k++) {
        FT s = slope_limit<SLOPE, FT>(dl.a[k], dr.a[k]);
        R.a[k] = w.a[k] + s;
        L.a[k] = w.a[k] - s;
    }
}

// HLL flux (cudaFluidStep.cu:2057-2198).  le = right face of the left cell, re = left face of
// the right cell, both [rho, v_n, P, v_t1, v_t2].  Output [rho, E, p_n, p_t1, p_t2].
template <typename FT>
__device__ __forceinline__ V5<FT> hll_flux(const FluidConsts<FT> &c, const V5<FT> &le, const V5<FT> &re)
{
    const FT Ale = le.a[0], Ble = le.a[1], Cle = le.a[2], Dle = le.a[3], Ele = le.a[4];
    const FT Are = re.a[0], Bre = re.a[1], Cre = re.a[2], Dre = re.a[3], Ere = re.a[4];
    FT Utilde = (Bre - Ble), Sleft = (Dre - Dle), Sright = (Ere - Ele);
    FT sl, sr;
    const bool iso = !(c.isotemp == (FT)-1);
    if (!iso) {
        einfeldt<FT>(c, Ale, Ble, Cle, Are, Bre, Cre, Utilde * Utilde + Sleft * Sleft + Sright * Sright, sl, sr);
    } else {
        // the isothermal bound receives c_iso^2 where a speed is expected (cudaFluidStep.cu:2131)
        einfeldt_iso<FT>(Ale, Ble, Are, Bre, c.isotempsq, sl, sr);
    }
    Sleft = sl;
    Sright = sr;
    FT Atilde = 1 / (Sright - Sleft);
    FT Fa = Ale * Ble;
    FT Fb = Are * Bre;
    V5<FT> f;
    int mode = 1;
    if (Sleft >= 0) mode = 0;
    if (Sright <= 0) mode = 2;
    if (mode == 0) {
        f.a[0] = Fa;
        if (!iso) {
            f.a[1] = Ble * (c.govergm1 * Cle + (FT).5 * Ale * (Ble * Ble + Dle * Dle + Ele * Ele));
            f.a[2] = Fa * Ble + Cle;
        } else {
            f.a[1] = Ble * (Cle + (FT).5 * Ale * (Ble * Ble + Dle * Dle + Ele * Ele));
            f.a[2] = Fa * Ble + c.isotempsq * Ale;
        }
        f.a[3] = Fa * Dle;
        f.a[4] = Fa * Ele;
    } else if (mode == 1) {
        f.a[0] = (Sright * (Ble - Sleft) * Ale - Sleft * (Bre - Sright) * Are) * Atilde;
        if (!iso) {
            f.a[2] = (Sright * (Ble - Sleft) * Fa - Sleft * (Bre - Sright) * Fb + Sright * Cle - Sleft * Cre) * Atilde;
        } else {
            f.a[2] = (Sright * (Ble - Sleft) * Fa - Sleft * (Bre - Sright) * Fb +
                      c.isotempsq * (Sright * Ale - Sleft * Are)) * Atilde;
        }
        f.a[3] = (Sright * (Ble - Sleft) * Ale * Dle - Sleft * (Bre - Sright) * Are * Dre) * Atilde;
        f.a[4] = (Sright * (Ble - Sleft) * Ale * Ele - Sleft * (Bre - Sright) * Are * Ere) * Atilde;
        if (!iso) {
            Fa = (FT).5 * Ale * (Ble * Ble + Dle * Dle + Ele * Ele);
            Fb = (FT).5 * Are * (Bre * Bre + Dre * Dre + Ere * Ere);
            FT e = (Sright * (Ble - Sleft) * Fa - Sleft * (Bre - Sright) * Fb);
            f.a[1] = (e + (c.govergm1 * (Sright * Cle * Ble - Sleft * Cre * Bre) + Sleft * Sright * (Cre - Cle) / c.gm1)) * Atilde;
        } else {
            // isothermal energy flux lacks the 1/(S_R-S_L) factor (cudaFluidStep.cu:2178-2182)
            Fa = (FT).5 * Ale * (Ble * Ble + Dle * Dle + Ele * Ele) + Cle;
            Fb = (FT).5 * Are * (Bre * Bre + Dre * Dre + Ere * Ere) + Cre;
            f.a[1] = (Sright * (Ble - Sleft) * Fa - Sleft * (Bre - Sright) * Fb);
        }
    } else {
        f.a[0] = Fb;
        if (!iso) {
            f.a[1] = Bre * (c.govergm1 * Cre + (FT).5 * Are * (Bre * Bre + Dre * Dre + Ere * Ere));
            f.a[2] = Fb * Bre + Cre;
        } else {
            f.a[1] = Bre * (Cre + (FT).5 * Are * (Bre * Bre + Dre * Dre + Ere * Ere));
            f.a[2] = Fb * Bre + c.isotemp * Are;  // c_iso, not c_iso^2 (cudaFluidStep.cu:2191)
        }
        f.a[3] = Fb * Dre;
        f.a[4] = Fb * Ere;
    }
    return f;
}

// HLL pressure solver with floors (cukern_PressureSolverHydro, cudaFluidStep.cu:2813-2864) on a
// conserved state in local order u = [rho, E, p_n, p_t1, p_t2]; mom[m] = local index of memory
// slab 2+m (the reference sums px, py, pz in slab order).  Returns P, modifies u.
template <int DIR>
__device__ __forceinline__ double hll_pressure(double u[5], double minmass, double mintemp, double gm1)
{
    // local index of memory slabs 2,3,4 under HllSlots<DIR>
    constexpr int m2 = (HllSlots<DIR>::n == 2) ? 2 : ((HllSlots<DIR>::t1 == 2) ? 3 : 4);
    constexpr int m3 = (HllSlots<DIR>::n == 3) ? 2 : ((HllSlots<DIR>::t1 == 3) ? 3 : 4);
    constexpr int m4 = (HllSlots<DIR>::n == 4) ? 2 : ((HllSlots<DIR>::t1 == 4) ? 3 : 4);
    double rho = u[0], E, z, momsq, P;
    if (rho < minmass) {
        P = minmass / rho;
        rho = u[0] = minmass;
        E = u[1] = P * u[1];
        z = u[m2] = P * u[m2];
        momsq = z * z;
        z = u[m3] = P * u[m3];
        momsq += z * z;
        z = u[m4] = P * u[m4];
        momsq += z * z;
    } else {
        E = u[1];
        z = u[m2];
        momsq = z * z;
        z = u[m3];
        momsq += z * z;
        z = u[m4];
        momsq += z * z;
    }
    P = E - .5 * momsq / rho;
    if (P < rho * mintemp) {
        P = mintemp * rho;
        u[1] = (.5 * momsq / rho) + P;
    }
    return P * gm1;
}

// Local component k of a sweep along DIR -> memory slab
template <int METHOD, int DIR>
__device__ __forceinline__ constexpr int slot_of(int k)
{
    if (k < 2) return k;
    if constexpr (METHOD == IB_METHOD_HLLC) {
        return k == 2 ? HllcSlots<DIR>::n : (k == 3 ? HllcSlots<DIR>::t1 : HllcSlots<DIR>::t2);
    } else {
        return k == 2 ? HllSlots<DIR>::n : (k == 3 ? HllSlots<DIR>::t1 : HllSlots<DIR>::t2);
    }
}

// Per-cell stage "prims" for either method.  For HLL the floors are applied to u first.
template <int METHOD, int DIR, typename FT>
__device__ __forceinline__ V5<FT> stage_prims(double u[5], const FluidConsts<FT> &c)
{
    if constexpr (METHOD == IB_METHOD_HLLC) {
        return hllc_prims<FT>((FT)u[0], (FT)u[1], (FT)u[2], (FT)u[3], (FT)u[4]);
    } else {
        double P = hll_pressure<DIR>(u, c.minmass, c.mintemp, (double)c.gm1);
        return hll_prims<FT>((FT)u[0], (FT)u[2], (FT)P, (FT)u[3], (FT)u[4]);
    }
}

template <int METHOD, int SLOPE, typename FT>
__device__ __forceinline__ void stage_faces(const FluidConsts<FT> &c, const V5<FT> &w, const V5<FT> &dl,
                                            const V5<FT> &dr, V5<FT> &L, V5<FT> &R)
{
    if constexpr (METHOD == IB_METHOD_HLLC) hllc_faces<SLOPE, FT>(c, w, dl, dr, L, R);
    else hll_faces<SLOPE, FT>(w, dl, dr, L, R);
}

template <int METHOD, typename FT>
__device__ __forceinline__ V5<FT> stage_flux(const FluidConsts<FT> &c, const V5<FT> &l, const V5<FT> &r)
{
    if constexpr (METHOD == IB_METHOD_HLLC) return hllc_flux<FT>(c, l, r);
    else return hll_flux<FT>(c, l, r);
}

// lambda times the flux difference of one cell in cylindrical geometry, component by component
// (local order rho, E, p_n, p_t1, p_t2; p_n = p_r in a radial sweep).  fR / fL: fluxes through the
// cell's outer / inner face.  Radial: rc = the cell centre radius; HLLC weights the faces by
// (rc +- dr/2) / rc and subtracts dr / (2 rc) times the cell's two face pressures from p_r's
// difference (cudaFluidStep.cu:1164-1171, 1488-1495); HLL folds lambda into those factors and
// subtracts the stage input's pressure (adiabatic) or rho c_iso^2 with rho the predicted density
// (isothermal) times lambda dr / rc (1837-1842, 2270-2290, 2371-2391).  CYL_THETA_DIV divides by
// the pencil radius; CYL_THETA_LAM gets lambda already divided by it.
template <int METHOD, int GEO>
__device__ __forceinline__ double cyl_dflux(int k, double fR, double fL, double lam, double rc, double dr,
                                            double rpen, double psum, double p_hll, double rho1,
                                            const FluidConsts<double> &c)
{
    // The product build multiplies by one reciprocal of the radius where the reference divides
    // (one division per cell or pencil instead of three or five); the strict build divides.
    if constexpr (GEO == CYL_RADIAL) {
#ifndef IB_STRICT_ARITH
        const double ri = 1.0 / rc;
#endif
        if constexpr (METHOD == IB_METHOD_HLLC) {
#ifdef IB_STRICT_ARITH
            const double cA = (rc - .5 * dr) / (rc);
            const double cB = (rc + .5 * dr) / (rc);
            const double cC = 0.5 * dr / rc;
#else
            const double cA = (rc - .5 * dr) * ri;
            const double cB = (rc + .5 * dr) * ri;
            const double cC = 0.5 * dr * ri;
#endif
            double d = cB * fR - cA * fL;
            if (k == 2) d = d - cC * psum;
            return lam * d;
        } else {
#ifdef IB_STRICT_ARITH
            const double cA = lam * (rc - .5 * dr) / (rc);
            const double cB = lam * (rc + .5 * dr) / (rc);
            const double cC = lam * dr / rc;
#else
            const double cA = lam * (rc - .5 * dr) * ri;
            const double cB = lam * (rc + .5 * dr) * ri;
            const double cC = lam * dr * ri;
#endif
            double d = cB * fR - cA * fL;
            if (k == 2) {
                if (c.isotemp == -1) d = d - p_hll * cC;
                else d = d - rho1 * c.isotempsq * cC;
            }
            return d;
        }
    } else if constexpr (GEO == CYL_THETA_DIV) {
#ifdef IB_STRICT_ARITH
        return lam * (fR - fL) / rpen;
#else
        return lam * (fR - fL) * (1.0 / rpen);
#endif
    } else {
        return lam * (fR - fL);
    }
}

struct SweepArgs {
    double *q;
    int64_t slab;
    int nx, ny, nz;
    DevScalar lambda;
    double crin, cdr;  // radial sweeps (GEO == CYL_RADIAL): radius of cell 0's centre, radial cell size
};

// ------------------------------------------------------------------------------------------
// Row kernel: one CTA per x row (nx <= CPT*blockDim.x), periodic in shared memory.
// Dynamic shared memory: 2 planes x 5 components x nx elements of FT; with row_ssum, 5 x nx
// doubles more hold u1 + u0 of the SSPRK average through the second stage, so that neither state
// stays in registers there (fewer spills at 64 registers; slower for the 512-cell rows and two
// cells per thread, which keep them in registers).
// ------------------------------------------------------------------------------------------
#ifndef IB_ROW_MINB
#define IB_ROW_MINB 2
#endif
template <int CPT, int NFIX>
__host__ __device__ constexpr bool row_ssum() { return CPT == 1 && NFIX != 512; }

// NS: sweeps applied in a row (1, or 2 for the two same-axis sweeps in the middle of an iteration).
// GEO == CYL_RADIAL: the radial sweep of cylindrical geometry (x = r), whose update weights the
// faces by their radii and adds the geometric pressure term to p_r (cyl_dflux); one cell per
// thread, FP64, one sweep.
// PADN (rows of a run-time length only): stride of the shared-memory planes fixed at PADN cells,
// so that the phases address them at constant offsets; 0 = the row length.
template <int METHOD, int SLOPE, typename FT, int CPT, int NFIX = 0, int NS = 1, int GEO = CYL_NONE, int PADN = 0>
__global__ void __launch_bounds__(512, (CPT == 1) ? IB_ROW_MINB : 1) sweep_row_kernel(SweepArgs a, FluidConsts<FT> c)
{
    static_assert(PADN == 0 || (NFIX == 0 && CPT == 1), "a fixed plane stride for rows of a run-time length");
    static_assert(GEO == CYL_NONE || (GEO == CYL_RADIAL && row_ssum<CPT, NFIX>() && NS == 1 &&
                                      std::is_same<FT, double>::value),
                  "radial rows: one cell per thread with the SSPRK sum in shared memory, one FP64 sweep");
    // its own name: every declaration of one extern shared array must agree on the alignment, and
    // the TMA kernels' smem_raw is 1024-byte aligned
    extern __shared__ __align__(16) unsigned char row_smem_raw[];
    const int n = NFIX ? NFIX : a.nx;  // NFIX: the row length fixed at compile time
    const int NP = PADN ? PADN : n;    // stride of the planes
    FT *SA = reinterpret_cast<FT *>(row_smem_raw);
    FT *SB = SA + 5 * NP;
    double *SS = reinterpret_cast<double *>(row_smem_raw + (size_t)10 * NP * sizeof(FT));
    const int64_t row = blockIdx.x;
    double *q = a.q + row * n;
    const int64_t S = a.slab;
    if (a.lambda.off()) return;  // a device timestep of 0: after the end time
    const double lambda = a.lambda.get();

    double u0[CPT][5], u1[CPT][5];
    V5<FT> keep[CPT];  // right faces, later fluxes
    bool act[CPT];
    // radial rows: the stage's face pressure sum (HLLC) or its input's pressure (HLL)
    double psum = 0.0, php = 0.0;
#pragma unroll
    for (int m = 0; m < CPT; m++) {
        int i = threadIdx.x + m * blockDim.x;
        act[m] = i < n;
#pragma unroll
        for (int k = 0; k < 5; k++) u0[m][k] = act[m] ? q[(int64_t)slot_of<METHOD, 1>(k) * S + i] : 1.0;
    }

#pragma unroll
    for (int sw = 0; sw < NS; sw++) {
    if (NS > 1 && sw > 0) {
        // the next sweep starts from this one's result (the planes alternate: no barrier)
#pragma unroll
        for (int m = 0; m < CPT; m++)
#pragma unroll
            for (int k = 0; k < 5; k++) u0[m][k] = u1[m][k];
    }
#pragma unroll
    for (int stage = 0; stage < 2; stage++) {
        double (*u)[5] = (stage == 0) ? u0 : u1;
        // the planes swap roles between the stages, so neither stage rewrites the plane the
        // other's last phase reads and no barrier separates them
        FT *PX = (stage == 0) ? SA : SB;  // primitives, then fluxes
        FT *PY = (stage == 0) ? SB : SA;  // left faces
        // (a) primitives -> PX
#pragma unroll
        for (int m = 0; m < CPT; m++) {
            int i = threadIdx.x + m * blockDim.x;
            if (act[m]) {
                V5<FT> w = stage_prims<METHOD, 1, FT>(u[m], c);
#pragma unroll
                for (int k = 0; k < 5; k++) PX[k * NP + i] = w.a[k];
                if (GEO == CYL_RADIAL && METHOD == IB_METHOD_HLL) php = (double)w.a[2];
                if (row_ssum<CPT, NFIX>() && stage == 1) {  // after the prims: HLL floors u1 in place
#pragma unroll
                    for (int k = 0; k < 5; k++) SS[k * NP + i] = u1[m][k] + u0[m][k];
                }
            }
        }
        __syncthreads();
        // (b) limited faces; left faces -> PY, right faces kept
#pragma unroll
        for (int m = 0; m < CPT; m++) {
            int i = threadIdx.x + m * blockDim.x;
            if (act[m]) {
                int il = (i == 0) ? n - 1 : i - 1, ir = (i == n - 1) ? 0 : i + 1;
                V5<FT> w, dl, dr, L;
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    w.a[k] = PX[k * NP + i];
                    dl.a[k] = w.a[k] - PX[k * NP + il];
                    dr.a[k] = PX[k * NP + ir] - w.a[k];
                }
                stage_faces<METHOD, SLOPE, FT>(c, w, dl, dr, L, keep[m]);
#pragma unroll
                for (int k = 0; k < 5; k++) PY[k * NP + i] = L.a[k];
                if (GEO == CYL_RADIAL && METHOD == IB_METHOD_HLLC) psum = (double)L.a[1] + (double)keep[m].a[1];
            }
        }
        __syncthreads();
        // (c) flux through face i+1/2 -> PX
#pragma unroll
        for (int m = 0; m < CPT; m++) {
            int i = threadIdx.x + m * blockDim.x;
            if (act[m]) {
                int ir = (i == n - 1) ? 0 : i + 1;
                V5<FT> Lr;
#pragma unroll
                for (int k = 0; k < 5; k++) Lr.a[k] = PY[k * NP + ir];
                keep[m] = stage_flux<METHOD, FT>(c, keep[m], Lr);
#pragma unroll
                for (int k = 0; k < 5; k++) PX[k * NP + i] = keep[m].a[k];
            }
        }
        __syncthreads();
        // (d) conservative update
#pragma unroll
        for (int m = 0; m < CPT; m++) {
            int i = threadIdx.x + m * blockDim.x;
            if (act[m]) {
                int il = (i == 0) ? n - 1 : i - 1;
                if constexpr (GEO == CYL_RADIAL) {
                    const double rc = a.crin + i * a.cdr;
                    // the isothermal HLL term's density: the new prediction (stage 0), the stage's
                    // own floored input (stage 1)
                    const double rho_in = u1[m][0];
#pragma unroll
                    for (int k = 0; k < 5; k++) {
                        const double rho1 = (stage == 0) ? (k == 0 ? 0.0 : u1[m][0]) : rho_in;
                        const double d = cyl_dflux<METHOD, GEO>(k, (double)keep[m].a[k], (double)PX[k * NP + il], lambda,
                                                                rc, a.cdr, 0.0, psum, php, rho1, c);
                        if (stage == 0) u1[m][k] = u0[m][k] - d;
                        else u1[m][k] = .5 * (SS[k * NP + i] - d);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 5; k++) {
                        double df = (double)keep[m].a[k] - (double)PX[k * NP + il];
                        if (stage == 0) u1[m][k] = u0[m][k] - lambda * df;
                        else if (row_ssum<CPT, NFIX>()) u1[m][k] = .5 * (SS[k * NP + i] - lambda * df);
                        else u1[m][k] = .5 * (u1[m][k] + u0[m][k] - lambda * df);
                    }
                }
            }
        }
    }
    }
#pragma unroll
    for (int m = 0; m < CPT; m++) {
        int i = threadIdx.x + m * blockDim.x;
        if (act[m]) {
#pragma unroll
            for (int k = 0; k < 5; k++) q[(int64_t)slot_of<METHOD, 1>(k) * S + i] = u1[m][k];
        }
    }
}

// ------------------------------------------------------------------------------------------
// TMA-fed pencil pipeline: a persistent CTA walks pencil blocks b = blockIdx.x, +gridDim.x, ...
// Each block is W adjacent whole pencils (x: one row, W = 1).  Thread 0 keeps two TMA loads
// in flight (double-buffered U0 tiles, one mbarrier each), so the next block's 5 slabs arrive
// while this one is computed; results leave through a TMA store from a third tile.  The tile
// layout is the TMA box's: [memory slab k][cell i][column] with the column fastest.  The
// arithmetic per cell is the row kernel's.
// Dynamic shared memory: 3 tiles of 5*W*n doubles (each rounded to 128 B) + 2 planes of
// 5*W*n elements of FT.
// ------------------------------------------------------------------------------------------
struct PipeArgs {
    int n;              // pencil length
    int npw;            // pencil blocks per line of x (nx / W; 1 for x sweeps)
    int bh;             // rows per TMA box along the pencil (n, or n / 2 for pencils above 256)
    int nh;             // boxes per pencil and slab (1 or 2)
    int64_t nblocks;    // pencil blocks in the grid
    DevScalar lambda;
    unsigned int *err;  // set to 1 when a TMA wait ran out
    uint32_t spin;      // poll limit of the tile waits
};

__host__ __device__ __forceinline__ size_t pipe_tile_bytes(int n, int W)
{
    return ((size_t)40 * n * W + 127) / 128 * 128;
}

// The tile of block b is one TMA box.  x sweeps: rank 3 (x, row, slab), box (n, 1, 5).  y/z sweeps:
// rank 5 (x, row within half, half, other axis, slab), box (W, bh, nh, 1, 5), so pencils of up to
// 512 cells arrive in one copy laid out [slab][cell][column].
template <int DIR>
__device__ __forceinline__ void pipe_load(double *dst, const CUtensorMap *tm, int64_t b, const PipeArgs &a, int W,
                                          uint64_t *bar)
{
    if (DIR == 1) tma_load_3d(dst, tm, 0, (int)b, 0, bar);
    else tma_load_5d(dst, tm, (int)(b % a.npw) * W, 0, 0, (int)(b / a.npw), 0, bar);
}

template <int DIR>
__device__ __forceinline__ void pipe_store(const CUtensorMap *tm, const double *src, int64_t b, const PipeArgs &a,
                                           int W)
{
    if (DIR == 1) tma_store_3d(tm, src, 0, (int)b, 0);
    else tma_store_5d(tm, src, (int)(b % a.npw) * W, 0, 0, (int)(b / a.npw), 0);
}

// NS: sweeps applied to each block in a row (1 or 2)
template <int METHOD, int SLOPE, typename FT, int DIR, int W, int CPT, int NFIX = 0, int NS = 1>
__global__ void __launch_bounds__(512, (CPT == 1) ? 2 : 1)
    sweep_pipe_kernel(const __grid_constant__ CUtensorMap tm, PipeArgs a, FluidConsts<FT> c)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[2];
    const int n = NFIX ? NFIX : a.n;  // NFIX: the pencil length fixed at compile time
    const int NW = n * W;
    const size_t tb = pipe_tile_bytes(n, W);
    // input tile t (computed, not an indexed array, which would live in local memory)
    auto Ub = [&](int t) { return reinterpret_cast<double *>(smem_raw + t * tb); };
    double *O = reinterpret_cast<double *>(smem_raw + 2 * tb);
    FT *PA = reinterpret_cast<FT *>(smem_raw + 3 * tb);
    FT *PB = PA + 5 * NW;
    const uint32_t tile_tx = (uint32_t)(40 * NW);
    // u1 + u0 through the second stage in the output tile rather than registers: fewer spills for
    // the FP64 one-cell-per-thread blocks (64 registers); the others are faster without it
    constexpr bool SSUM = (CPT == 1) && (sizeof(FT) == 8);
    constexpr int s0 = slot_of<METHOD, DIR>(0), s1 = slot_of<METHOD, DIR>(1), s2 = slot_of<METHOD, DIR>(2),
                  s3 = slot_of<METHOD, DIR>(3), s4 = slot_of<METHOD, DIR>(4);
    const int slots[5] = {s0, s1, s2, s3, s4};
    const int col = (W == 1) ? 0 : (int)(threadIdx.x % W);
    const int rows_per_pass = blockDim.x / W;
    int ci[CPT], il[CPT], ir[CPT];
    bool act[CPT];
#pragma unroll
    for (int m = 0; m < CPT; m++) {
        ci[m] = (int)(threadIdx.x / W) + m * rows_per_pass;
        act[m] = ci[m] < n;
        il[m] = (ci[m] == 0) ? n - 1 : ci[m] - 1;
        ir[m] = (ci[m] == n - 1) ? 0 : ci[m] + 1;
    }
    auto SI = [&](int k, int j) { return (k * n + j) * W + col; };
    if (a.lambda.off()) return;  // a device timestep of 0: after the end time
    const double lambda = a.lambda.get();
    const int64_t step = gridDim.x;
    const bool leader = threadIdx.x == 0;

    if (leader) {
        prefetch_tmap(&tm);
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    bool issued0 = false, issued1 = false;  // leader's bookkeeping of loads in flight
    if (leader) {
        const int64_t b0 = blockIdx.x, b1 = blockIdx.x + step;
        if (b0 < a.nblocks) {
            mbar_arrive_expect_tx(&full[0], tile_tx);
            pipe_load<DIR>(Ub(0), &tm, b0, a, W, &full[0]);
            issued0 = true;
        }
        if (b1 < a.nblocks) {
            mbar_arrive_expect_tx(&full[1], tile_tx);
            pipe_load<DIR>(Ub(1), &tm, b1, a, W, &full[1]);
            issued1 = true;
        }
    }
    uint32_t phase0 = 0, phase1 = 0;
    int it = 0;
    for (int64_t b = blockIdx.x; b < a.nblocks; b += step, it++) {
        const int t = it & 1;
        double *Ut = Ub(t);
        const uint32_t par = t ? phase1 : phase0;
        const bool ok = mbar_wait_cta(&full[t], par, a.spin);  // uniform across the CTA
        if (t) phase1 ^= 1; else phase0 ^= 1;
        if (!ok) {
            // a tile never arrived: report, drain what is still in flight, leave
            if (leader) {
                atomicOr(a.err, 1u);
                mbar_wait(&full[t], par);  // give the late tile one more bounded wait
                if (t == 0 && issued1) mbar_wait(&full[1], phase1);
                if (t == 1 && issued0) mbar_wait(&full[0], phase0);
                bulk_wait_all();
            }
            return;
        }
        double u0[CPT][5], u1[CPT][5];
#pragma unroll
        for (int m = 0; m < CPT; m++)
#pragma unroll
            for (int k = 0; k < 5; k++) u0[m][k] = act[m] ? Ut[SI(slots[k], ci[m])] : 1.0;
        V5<FT> keep[CPT];
#pragma unroll
        for (int sw = 0; sw < NS; sw++) {
        if (NS > 1 && sw > 0) {
            // the next sweep starts from this one's result in the output tile (each thread reads
            // the cells it wrote)
#pragma unroll
            for (int m = 0; m < CPT; m++)
#pragma unroll
                for (int k = 0; k < 5; k++) u0[m][k] = act[m] ? O[SI(slots[k], ci[m])] : 1.0;
        }
#pragma unroll
        for (int stage = 0; stage < 2; stage++) {
            double (*u)[5] = (stage == 0) ? u0 : u1;
            // the planes swap roles between the stages: neither stage rewrites the plane that the
            // other's last phase reads, so no barrier separates them
            FT *X = (stage == 0) ? PA : PB;  // primitives, then fluxes
            FT *Y = (stage == 0) ? PB : PA;  // left faces
#pragma unroll
            for (int m = 0; m < CPT; m++) {
                if (act[m]) {
                    V5<FT> w = stage_prims<METHOD, DIR, FT>(u[m], c);
#pragma unroll
                    for (int k = 0; k < 5; k++) X[SI(k, ci[m])] = w.a[k];
                    if (SSUM && stage == 1) {
                        // u1 + u0 of the SSPRK average goes to this block's output tile, so
                        // neither state stays in registers through the second stage (after the
                        // prims: the HLL pressure pass floors u1 in place)
#pragma unroll
                        for (int k = 0; k < 5; k++) O[SI(slots[k], ci[m])] = u1[m][k] + u0[m][k];
                    }
                }
            }
            __syncthreads();
            if (stage == 0 && sw == 0 && leader) {
                // every thread has read tile t: prefetch the block after next into it
                const int64_t bn = b + 2 * step;
                if (bn < a.nblocks) {
                    fence_proxy_async_smem();
                    mbar_arrive_expect_tx(&full[t], tile_tx);
                    pipe_load<DIR>(Ut, &tm, bn, a, W, &full[t]);
                } else {
                    if (t == 0) issued0 = false; else issued1 = false;
                }
            }
#pragma unroll
            for (int m = 0; m < CPT; m++) {
                if (act[m]) {
                    V5<FT> w, dl, dr, L;
#pragma unroll
                    for (int k = 0; k < 5; k++) {
                        w.a[k] = X[SI(k, ci[m])];
                        dl.a[k] = w.a[k] - X[SI(k, il[m])];
                        dr.a[k] = X[SI(k, ir[m])] - w.a[k];
                    }
                    stage_faces<METHOD, SLOPE, FT>(c, w, dl, dr, L, keep[m]);
#pragma unroll
                    for (int k = 0; k < 5; k++) Y[SI(k, ci[m])] = L.a[k];
                }
            }
            __syncthreads();
#pragma unroll
            for (int m = 0; m < CPT; m++) {
                if (act[m]) {
                    V5<FT> Lr;
#pragma unroll
                    for (int k = 0; k < 5; k++) Lr.a[k] = Y[SI(k, ir[m])];
                    keep[m] = stage_flux<METHOD, FT>(c, keep[m], Lr);
#pragma unroll
                    for (int k = 0; k < 5; k++) X[SI(k, ci[m])] = keep[m].a[k];
                }
            }
            // the previous block's store must have read O before stage 1 writes it
            if (stage == 0 && sw == 0 && leader) bulk_wait_read_all();
            __syncthreads();
#pragma unroll
            for (int m = 0; m < CPT; m++) {
                if (act[m]) {
#pragma unroll
                    for (int k = 0; k < 5; k++) {
                        double df = (double)keep[m].a[k] - (double)X[SI(k, il[m])];
                        if (stage == 0) u1[m][k] = u0[m][k] - lambda * df;
                        else if (SSUM) {
                            double &o = O[SI(slots[k], ci[m])];
                            o = .5 * (o - lambda * df);
                        } else {
                            O[SI(slots[k], ci[m])] = .5 * (u1[m][k] + u0[m][k] - lambda * df);
                        }
                    }
                }
            }
        }
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (leader) {
            pipe_store<DIR>(&tm, O, b, a, W);
            bulk_commit();
        }
    }
    if (leader) bulk_wait_all();
}

// ------------------------------------------------------------------------------------------
// Pencil-pair kernel (y and z sweeps, pencils up to 256 cells or of 512, x even): the row kernel's
// layout applied to a TMA box.  One CTA per block of two adjacent pencils, n threads (one cell
// each, as the x row kernel), four CTAs per SM (two of 512 threads for 512-cell pencils); thread
// 0 loads the block's 5-slab box (2 x n x 5
// doubles, 16-byte rows) with one TMA copy, the CTA sweeps the two pencils one after the other
// through the row kernel's phases (two shared-memory planes that swap roles between the stages,
// the SSPRK sum u1 + u0 in a third), writes each pencil's result over its own column of the box
// and leaves by one TMA store.  No persistent pipeline: the other CTAs on the SM hide a block's
// load, as they hide the row kernel's.
// Dynamic shared memory: the box (pipe_tile_bytes(n, WC)), 2 planes of 5 NP elements of FT and
// 5 NP doubles for the SSPRK sum (NP: the pencil length, or PADN).
// ------------------------------------------------------------------------------------------
// n: pencil length (the box), np: stride of the planes (the pencil length, or PADN)
__host__ __device__ __forceinline__ size_t pair_smem_bytes(int n, int ftsize, int wc, int np)
{
    return pipe_tile_bytes(n, wc) + (size_t)10 * np * ftsize + (size_t)40 * np;
}

// WC: pencils per box (2; 4 for z sweeps of x-y planes above 1 MB, whose 16-byte rows a plane
// apart the memory system serves poorly: 32-byte rows, three CTAs per SM)
// GEO == CYL_THETA_DIV / CYL_THETA_LAM: the theta sweep of cylindrical geometry (y = theta), the
// flux difference divided by the pencil's radius or lambda divided by it first (cyl_dflux); the
// radius of the pencil at radial index x and z index z is theta_radius(cyl, x, z).  FP64, one sweep.
// PADN (pencils of a run-time length only): stride of the shared-memory planes fixed at PADN
// cells, so that the phases address them at constant offsets (HLLC FP64, pencils of 129-255 cells:
// fewer spills); 0 = the pencil length.
template <int METHOD, int SLOPE, typename FT, int DIR, int NFIX = 0, int NS = 1, int WC = 2, int GEO = CYL_NONE,
          int PADN = 0>
__global__ void __launch_bounds__(NFIX == 512 ? 512 : 256, NFIX == 512 ? 2 : (WC == 4 ? 3 : 4))
    sweep_pair_kernel(const __grid_constant__ CUtensorMap tm, PipeArgs a, FluidConsts<FT> c, CylPencil cyl)
{
    static_assert(GEO == CYL_NONE || ((GEO == CYL_THETA_DIV || GEO == CYL_THETA_LAM) && DIR == 2 && NS == 1 &&
                                      std::is_same<FT, double>::value),
                  "theta pencils: y sweeps, one FP64 sweep");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full;
    const int n = NFIX ? NFIX : a.n;
    // stride of the shared-memory planes
    const int NP = NFIX ? NFIX : (PADN ? PADN : n);
    double *T = reinterpret_cast<double *>(smem_raw);  // the box: [slab][cell][column]
    FT *SA = reinterpret_cast<FT *>(smem_raw + pipe_tile_bytes(n, WC));
    FT *SB = SA + 5 * NP;
    double *SS = reinterpret_cast<double *>(SB + 5 * NP);
    constexpr int s0 = slot_of<METHOD, DIR>(0), s1 = slot_of<METHOD, DIR>(1), s2 = slot_of<METHOD, DIR>(2),
                  s3 = slot_of<METHOD, DIR>(3), s4 = slot_of<METHOD, DIR>(4);
    const int slots[5] = {s0, s1, s2, s3, s4};
    const int64_t b = blockIdx.x;
    const int i = threadIdx.x;
    const bool act = i < n;
    const int il = (i == 0) ? n - 1 : i - 1, ir = (i == n - 1) ? 0 : i + 1;
    if (a.lambda.off()) return;  // a device timestep of 0: after the end time
    const double lambda = a.lambda.get();
    const bool leader = threadIdx.x == 0;
    // the box's TMA copy needs a 128-byte aligned destination: a CTA whose tile is not aligned
    // leaves its block undone and sets bit 2 of the wait flag instead of issuing the copy
    if (smem_u32(T) & 127u) {
        if (leader) atomicOr(a.err, 2u);
        return;
    }
    if (leader) {
        mbar_init(&full, 1);
        fence_mbar_init();
        mbar_arrive_expect_tx(&full, (uint32_t)(40 * WC * n));
        pipe_load<DIR>(T, &tm, b, a, WC, &full);
    }
    const bool ok = mbar_wait_cta(&full, 0, a.spin);  // uniform across the CTA
    if (!ok) {
        if (leader) {
            atomicOr(a.err, 1u);
            mbar_wait(&full, 0);  // one more bounded wait for the late box
        }
        return;
    }
#pragma unroll 1
    for (int col = 0; col < WC; col++) {
        auto TI = [&](int k) { return (k * n + i) * WC + col; };
        double u0[5], u1[5];
        V5<FT> keep;
        double rp = 0.0, lam = lambda;  // theta pencils: the pencil's radius and the lambda it takes
        if constexpr (GEO != CYL_NONE) {
            rp = theta_radius(cyl, (int)(b % a.npw) * WC + col, (int)(b / a.npw));
            if (GEO == CYL_THETA_LAM) lam = lambda / rp;
        }
#pragma unroll
        for (int k = 0; k < 5; k++) u0[k] = act ? T[TI(slots[k])] : 1.0;
#pragma unroll
        for (int sw = 0; sw < NS; sw++) {
            if (NS > 1 && sw > 0) {
#pragma unroll
                for (int k = 0; k < 5; k++) u0[k] = u1[k];
            }
#pragma unroll
            for (int stage = 0; stage < 2; stage++) {
                double *u = (stage == 0) ? u0 : u1;
                FT *PX = (stage == 0) ? SA : SB;  // primitives, then fluxes
                FT *PY = (stage == 0) ? SB : SA;  // left faces
                if (act) {
                    V5<FT> w = stage_prims<METHOD, DIR, FT>(u, c);
#pragma unroll
                    for (int k = 0; k < 5; k++) PX[k * NP + i] = w.a[k];
                    if (stage == 1) {
#pragma unroll
                        for (int k = 0; k < 5; k++) SS[k * NP + i] = u1[k] + u0[k];
                    }
                }
                __syncthreads();
                if (act) {
                    V5<FT> w, dl, dr, L;
#pragma unroll
                    for (int k = 0; k < 5; k++) {
                        w.a[k] = PX[k * NP + i];
                        dl.a[k] = w.a[k] - PX[k * NP + il];
                        dr.a[k] = PX[k * NP + ir] - w.a[k];
                    }
                    stage_faces<METHOD, SLOPE, FT>(c, w, dl, dr, L, keep);
#pragma unroll
                    for (int k = 0; k < 5; k++) PY[k * NP + i] = L.a[k];
                }
                __syncthreads();
                if (act) {
                    V5<FT> Lr;
#pragma unroll
                    for (int k = 0; k < 5; k++) Lr.a[k] = PY[k * NP + ir];
                    keep = stage_flux<METHOD, FT>(c, keep, Lr);
#pragma unroll
                    for (int k = 0; k < 5; k++) PX[k * NP + i] = keep.a[k];
                }
                __syncthreads();
                if (act) {
#pragma unroll
                    for (int k = 0; k < 5; k++) {
                        if constexpr (GEO == CYL_NONE) {
                            double df = (double)keep.a[k] - (double)PX[k * NP + il];
                            if (stage == 0) u1[k] = u0[k] - lambda * df;
                            else u1[k] = .5 * (SS[k * NP + i] - lambda * df);
                        } else {
                            const double d = cyl_dflux<METHOD, GEO>(k, (double)keep.a[k], (double)PX[k * NP + il], lam,
                                                                    0.0, 0.0, rp, 0.0, 0.0, 0.0, c);
                            if (stage == 0) u1[k] = u0[k] - d;
                            else u1[k] = .5 * (SS[k * NP + i] - d);
                        }
                    }
                }
            }
        }
        // this pencil's result over its own column of the box (its inputs were read above)
        if (act) {
#pragma unroll
            for (int k = 0; k < 5; k++) T[TI(slots[k])] = u1[k];
        }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (leader) {
        pipe_store<DIR>(&tm, T, b, a, WC);
        bulk_commit();
        bulk_wait_all();
    }
}

// Wide-block variant for z sweeps of large x-y planes.  A block is WL = G*W adjacent columns of
// whole pencils (64-byte box rows for WL = 8: z rows sit a plane apart, megabytes, and narrow
// rows there waste most of each memory access), computed in G groups of W columns through
// shared-memory planes sized for one group.  Results overwrite the tile in place and leave by one
// TMA store, so two tiles fit: the refill of a tile is issued after the store from it has read
// it, one block ahead (block b + grid is requested while block b is computed).
template <int METHOD, int SLOPE, typename FT, int DIR, int W, int G, int CPT, int NFIX = 0, int NS = 1>
__global__ void __launch_bounds__(512, 1)
    sweep_pipe_wide_kernel(const __grid_constant__ CUtensorMap tm, PipeArgs a, FluidConsts<FT> c)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[2];
    constexpr int WL = W * G;
    const int n = NFIX ? NFIX : a.n;
    const size_t tb = pipe_tile_bytes(n, WL);
    auto Ub = [&](int t) { return reinterpret_cast<double *>(smem_raw + t * tb); };
    FT *SA = reinterpret_cast<FT *>(smem_raw + 2 * tb);
    FT *SB = SA + 5 * n * W;
    const uint32_t tile_tx = (uint32_t)(40 * n * WL);
    constexpr int s0 = slot_of<METHOD, DIR>(0), s1 = slot_of<METHOD, DIR>(1), s2 = slot_of<METHOD, DIR>(2),
                  s3 = slot_of<METHOD, DIR>(3), s4 = slot_of<METHOD, DIR>(4);
    const int slots[5] = {s0, s1, s2, s3, s4};
    const int col = (int)(threadIdx.x % W);
    const int rows_per_pass = blockDim.x / W;
    int ci[CPT], il[CPT], ir[CPT];
    bool act[CPT];
#pragma unroll
    for (int m = 0; m < CPT; m++) {
        ci[m] = (int)(threadIdx.x / W) + m * rows_per_pass;
        act[m] = ci[m] < n;
        il[m] = (ci[m] == 0) ? n - 1 : ci[m] - 1;
        ir[m] = (ci[m] == n - 1) ? 0 : ci[m] + 1;
    }
    auto SI = [&](int k, int j) { return (k * n + j) * W + col; };
    if (a.lambda.off()) return;  // a device timestep of 0: after the end time
    const double lambda = a.lambda.get();
    const int64_t step = gridDim.x;
    const bool leader = threadIdx.x == 0;

    if (leader) {
        prefetch_tmap(&tm);
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    // bit t: a load into tile t is in flight (leader's bookkeeping) / parity to wait for on t
    uint32_t issued = 0, phase = 0;
    if (leader) {
        for (int t = 0; t < 2; t++) {
            const int64_t bt = blockIdx.x + t * step;
            if (bt < a.nblocks) {
                mbar_arrive_expect_tx(&full[t], tile_tx);
                pipe_load<DIR>(Ub(t), &tm, bt, a, WL, &full[t]);
                issued |= 1u << t;
            }
        }
    }
    int it = 0;
    for (int64_t b = blockIdx.x; b < a.nblocks; b += step, it++) {
        const int t = it & 1;
        double *Ut = Ub(t);
        const bool ok = mbar_wait_cta(&full[t], (phase >> t) & 1, a.spin);  // uniform across the CTA
        if (!ok) {
            if (leader) {
                atomicOr(a.err, 1u);
                mbar_wait(&full[t], (phase >> t) & 1);  // one more bounded wait for the late tile
                if ((issued >> (t ^ 1)) & 1) mbar_wait(&full[t ^ 1], (phase >> (t ^ 1)) & 1);
                bulk_wait_all();
            }
            return;
        }
        phase ^= 1u << t;
        issued &= ~(1u << t);
#pragma unroll 1
        for (int g = 0; g < G; g++) {
            const int tc = g * W + col;  // column within the tile
            auto TI = [&](int k, int j) { return (k * n + j) * WL + tc; };
            double u0[CPT][5], u1[CPT][5];
#pragma unroll
            for (int m = 0; m < CPT; m++)
#pragma unroll
                for (int k = 0; k < 5; k++) u0[m][k] = act[m] ? Ut[TI(slots[k], ci[m])] : 1.0;
            V5<FT> keep[CPT];
#pragma unroll
            for (int sw = 0; sw < NS; sw++) {
            if (NS > 1 && sw > 0) {
                // the previous sweep's result, in place in the tile (each thread's own cells);
                // the loop below ends with a barrier, so the planes are free
#pragma unroll
                for (int m = 0; m < CPT; m++)
#pragma unroll
                    for (int k = 0; k < 5; k++) u0[m][k] = act[m] ? Ut[TI(slots[k], ci[m])] : 1.0;
            }
#pragma unroll
            for (int stage = 0; stage < 2; stage++) {
                double (*u)[5] = (stage == 0) ? u0 : u1;
#pragma unroll
                for (int m = 0; m < CPT; m++) {
                    if (act[m]) {
                        V5<FT> w = stage_prims<METHOD, DIR, FT>(u[m], c);
#pragma unroll
                        for (int k = 0; k < 5; k++) SA[SI(k, ci[m])] = w.a[k];
                    }
                }
                __syncthreads();
                if (stage == 0 && sw == 0 && g == 0 && it > 0 && leader) {
                    // the other tile's block has been stored: once that store has read it,
                    // request the next block into it
                    bulk_wait_read_all();
                    const int64_t bn = b + step;
                    if (bn < a.nblocks) {
                        mbar_arrive_expect_tx(&full[t ^ 1], tile_tx);
                        pipe_load<DIR>(Ub(t ^ 1), &tm, bn, a, WL, &full[t ^ 1]);
                        issued |= 1u << (t ^ 1);
                    }
                }
#pragma unroll
                for (int m = 0; m < CPT; m++) {
                    if (act[m]) {
                        V5<FT> w, dl, dr, L;
#pragma unroll
                        for (int k = 0; k < 5; k++) {
                            w.a[k] = SA[SI(k, ci[m])];
                            dl.a[k] = w.a[k] - SA[SI(k, il[m])];
                            dr.a[k] = SA[SI(k, ir[m])] - w.a[k];
                        }
                        stage_faces<METHOD, SLOPE, FT>(c, w, dl, dr, L, keep[m]);
#pragma unroll
                        for (int k = 0; k < 5; k++) SB[SI(k, ci[m])] = L.a[k];
                    }
                }
                __syncthreads();
#pragma unroll
                for (int m = 0; m < CPT; m++) {
                    if (act[m]) {
                        V5<FT> Lr;
#pragma unroll
                        for (int k = 0; k < 5; k++) Lr.a[k] = SB[SI(k, ir[m])];
                        keep[m] = stage_flux<METHOD, FT>(c, keep[m], Lr);
#pragma unroll
                        for (int k = 0; k < 5; k++) SA[SI(k, ci[m])] = keep[m].a[k];
                    }
                }
                __syncthreads();
#pragma unroll
                for (int m = 0; m < CPT; m++) {
                    if (act[m]) {
#pragma unroll
                        for (int k = 0; k < 5; k++) {
                            double df = (double)keep[m].a[k] - (double)SA[SI(k, il[m])];
                            if (stage == 0) u1[m][k] = u0[m][k] - lambda * df;
                            // each thread rewrites only the cells it read
                            else Ut[TI(slots[k], ci[m])] = .5 * (u1[m][k] + u0[m][k] - lambda * df);
                        }
                    }
                }
                __syncthreads();  // the planes are rewritten next (stage 1, the next sweep or group)
            }
            }
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (leader) {
            pipe_store<DIR>(&tm, Ut, b, a, WL);
            bulk_commit();
        }
    }
    if (leader) bulk_wait_all();
}

// ------------------------------------------------------------------------------------------
// Chunked pipeline for pencils longer than 512 cells.  A pencil is cut into C chunks of L cells
// (the last one shorter); a job is one chunk of a block of W adjacent pencils, computed on R = L + 8
// rows: the chunk plus 4 rows of halo on each side (both SSPRK stages are recomputed on the halo).
// x rows: W = 1, L = 248; y/z pencils: W = 4, L = 120 (32-byte box rows: 16-byte rows at the large
// strides of long pencils are served poorly).
//   * Independent jobs: before the sweep, chunk_halo_kernel copies every job's 8 halo rows (the
//     4 before its chunk and the 4 after, periodic) to a side buffer, contiguous per job, and a job
//     takes its halo from there.  No job reads what another writes, so the jobs of one pencil run
//     on any CTAs in any order and the persistent grid deals them out evenly.
//   * A job's L chunk rows arrive as one TMA box (rows past the pencil's end are filled and idle)
//     and its halo block as one untiled bulk copy, on the same mbarrier; the loads of the next two
//     jobs are in flight while one is computed (double-buffered, bounded waits).  Outputs are
//     plain stores from registers.
// Dynamic shared memory: 2 tiles of 40*L*W bytes and 2 halo blocks of 320*W bytes (each rounded to
// 128), the SSPRK sum u1 + u0 through the second stage (40*R*W bytes: neither state stays in
// registers there), then 2 planes of 5*R*W elements of FT.
// ------------------------------------------------------------------------------------------
struct ChunkArgs {
    double *q;
    const double *side;  // halo rows of every job: [group * C + chunk][slab][8 rows][W]
    int64_t slab;        // doubles between slabs
    int64_t rs;          // doubles between consecutive cells of a pencil
    int64_t os;          // doubles between consecutive pencils along the other axis (rows for x)
    int n;               // pencil length (> 512)
    int C;               // chunks per pencil: ceil(n / L)
    int npw;             // pencil blocks per line of x (nx / W; 1 for x sweeps)
    int64_t ngroups;     // pencil blocks in the grid
    DevScalar lambda;
    unsigned int *err;   // set to 1 when a TMA wait ran out
    uint32_t spin;       // poll limit of the tile waits
};

__host__ __device__ constexpr size_t chunk_smem_bytes(int W, int R, int ftsize)
{
    return 2 * (((size_t)40 * (R - 8) * W + 127) / 128 * 128) + 2 * (((size_t)320 * W + 127) / 128 * 128) +
           (size_t)40 * R * W + (size_t)10 * R * W * ftsize;
}

// First cell of pencil block grp, column col.
__device__ __forceinline__ int64_t chunk_base(const ChunkArgs &a, int DIR, int W, int64_t grp, int col)
{
    if (DIR == 1) return grp * a.os;
    return (grp % a.npw) * W + col + (grp / a.npw) * a.os;
}

// Side buffer: for every job (pencil block grp, chunk cc), rows c0-4 .. c0-1 and cend .. cend+3
// (mod n) of the 5 slabs, c0 = cc*L, cend = min(c0 + L, n).  One thread per value.
template <int DIR, int W>
__global__ void __launch_bounds__(256) chunk_halo_kernel(ChunkArgs a, int L, double *side)
{
    const int64_t total = a.ngroups * a.C * 5 * 8 * W;
    for (int64_t t = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; t < total; t += (int64_t)blockDim.x * gridDim.x) {
        const int col = (int)(t % W);
        const int rr = (int)((t / W) % 8);
        const int k = (int)((t / (8 * W)) % 5);
        const int64_t job = t / (40 * W);  // grp * C + cc
        const int cc = (int)(job % a.C);
        const int64_t grp = job / a.C;
        const int c0 = cc * L, cend = (c0 + L < a.n) ? c0 + L : a.n;
        int row = (rr < 4) ? c0 - 4 + rr : cend + (rr - 4);
        if (row < 0) row += a.n;
        else if (row >= a.n) row -= a.n;
        side[t] = a.q[chunk_base(a, DIR, W, grp, col) + k * a.slab + (int64_t)row * a.rs];
    }
}

template <int DIR>
__device__ __forceinline__ void chunk_load(double *dst, const CUtensorMap *tm, int64_t grp, int g0, const ChunkArgs &a,
                                           int W, uint64_t *bar)
{
    if (DIR == 1) tma_load_3d(dst, tm, g0, (int)grp, 0, bar);
    else tma_load_4d(dst, tm, (int)(grp % a.npw) * W, g0, (int)(grp / a.npw), 0, bar);
}

template <int METHOD, int SLOPE, typename FT, int DIR, int W, int R>
__global__ void __launch_bounds__(512, 2)
    sweep_chunk_kernel(const __grid_constant__ CUtensorMap tm, ChunkArgs a, FluidConsts<FT> c)
{
    constexpr int L = R - 8;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[2];
    constexpr size_t tb = ((size_t)40 * L * W + 127) / 128 * 128;
    constexpr size_t hb = ((size_t)320 * W + 127) / 128 * 128;
    // tile and halo block of buffer b (computed, not indexed arrays, which would live in local memory)
    auto Ub = [&](int b) { return reinterpret_cast<double *>(smem_raw + b * tb); };
    auto Hb = [&](int b) { return reinterpret_cast<double *>(smem_raw + 2 * tb + b * hb); };
    double *SS = reinterpret_cast<double *>(smem_raw + 2 * tb + 2 * hb);
    FT *SA = reinterpret_cast<FT *>(smem_raw + 2 * tb + 2 * hb + (size_t)40 * R * W);
    FT *SB = SA + 5 * R * W;
    constexpr uint32_t tile_tx = 40u * L * W + 320u * W;
    constexpr int s0 = slot_of<METHOD, DIR>(0), s1 = slot_of<METHOD, DIR>(1), s2 = slot_of<METHOD, DIR>(2),
                  s3 = slot_of<METHOD, DIR>(3), s4 = slot_of<METHOD, DIR>(4);
    const int slots[5] = {s0, s1, s2, s3, s4};
    const int col = (W == 1) ? 0 : (int)(threadIdx.x % W);
    const int r = (int)(threadIdx.x / W);  // row of this thread in the job; blockDim.x = W * R
    const int il = (r > 0) ? r - 1 : 0, ir = (r < R - 1) ? r + 1 : R - 1;  // edge rows: unused results
    auto SI = [&](int k, int j) { return (k * R + j) * W + col; };
    const int n = a.n, C = a.C;
    if (a.lambda.off()) return;  // a device timestep of 0: after the end time
    const double lambda = a.lambda.get();
    const bool leader = threadIdx.x == 0;
    const int64_t njobs_all = a.ngroups * C;
    const int64_t step = gridDim.x;

    if (leader) {
        prefetch_tmap(&tm);
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int64_t j, int buf) {  // leader only
        mbar_arrive_expect_tx(&full[buf], tile_tx);
        chunk_load<DIR>(Ub(buf), &tm, j / C, (int)(j % C) * L, a, W, &full[buf]);
        bulk_load(Hb(buf), a.side + j * 40 * W, 320u * W, &full[buf]);
    };
    // bit b: a load into buffer b is in flight (leader's bookkeeping) / parity to wait for on b
    uint32_t issued = 0, phase = 0;
    if (leader) {
        for (int t = 0; t < 2; t++) {
            const int64_t jt = blockIdx.x + t * step;
            if (jt < njobs_all) { issue(jt, t); issued |= 1u << t; }
        }
    }
    int it = 0;
    for (int64_t j = blockIdx.x; j < njobs_all; j += step, it++) {
        const int buf = it & 1;
        const int64_t grp = j / C;
        const int cc = (int)(j % C);
        const int c0 = cc * L;                    // first cell of the chunk
        const int cend = (c0 + L < n) ? c0 + L : n;
        const bool ok = mbar_wait_cta(&full[buf], (phase >> buf) & 1, a.spin);
        if (!ok) {
            if (leader) {
                atomicOr(a.err, 1u);
                mbar_wait(&full[buf], (phase >> buf) & 1);  // one more bounded wait for the late tile
                if ((issued >> (buf ^ 1)) & 1) mbar_wait(&full[buf ^ 1], (phase >> (buf ^ 1)) & 1);
            }
            return;
        }
        phase ^= 1u << buf;
        issued &= ~(1u << buf);
        // this thread's cell g = c0 - 4 + r: left halo (side buffer, boundary cc), chunk (tile),
        // right halo (side buffer, boundary cc + 1 mod C), or idle
        const int g = c0 - 4 + r;
        const bool act = g < cend + 4;
        double u0[5], u1[5];
        if (g >= c0 && g < cend) {
            const double *Ut = Ub(buf);
#pragma unroll
            for (int k = 0; k < 5; k++) u0[k] = Ut[(slots[k] * L + (g - c0)) * W + col];
        } else if (act) {
            const int rr = (g < c0) ? r : 4 + (g - cend);
            const double *H = Hb(buf);
#pragma unroll
            for (int k = 0; k < 5; k++) u0[k] = H[(slots[k] * 8 + rr) * W + col];
        } else {
#pragma unroll
            for (int k = 0; k < 5; k++) u0[k] = 1.0;
        }
        V5<FT> keep;
#pragma unroll
        for (int stage = 0; stage < 2; stage++) {
            double *u = (stage == 0) ? u0 : u1;
            {
                V5<FT> w = stage_prims<METHOD, DIR, FT>(u, c);
#pragma unroll
                for (int k = 0; k < 5; k++) SA[SI(k, r)] = w.a[k];
                if (stage == 1) {  // after the prims: HLL floors u1 in place
#pragma unroll
                    for (int k = 0; k < 5; k++) SS[SI(k, r)] = u1[k] + u0[k];
                }
            }
            __syncthreads();
            if (stage == 0 && leader) {
                // every thread has read tile buf: request the job after next into it
                const int64_t jn = j + 2 * step;
                if (jn < njobs_all) {
                    fence_proxy_async_smem();
                    issue(jn, buf);
                    issued |= 1u << buf;
                }
            }
            {
                V5<FT> w, dl, dr, Lf;
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    w.a[k] = SA[SI(k, r)];
                    dl.a[k] = w.a[k] - SA[SI(k, il)];
                    dr.a[k] = SA[SI(k, ir)] - w.a[k];
                }
                stage_faces<METHOD, SLOPE, FT>(c, w, dl, dr, Lf, keep);
#pragma unroll
                for (int k = 0; k < 5; k++) SB[SI(k, r)] = Lf.a[k];
            }
            __syncthreads();
            {
                V5<FT> Lr;
#pragma unroll
                for (int k = 0; k < 5; k++) Lr.a[k] = SB[SI(k, ir)];
                keep = stage_flux<METHOD, FT>(c, keep, Lr);
#pragma unroll
                for (int k = 0; k < 5; k++) SA[SI(k, r)] = keep.a[k];
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < 5; k++) {
                double df = (double)keep.a[k] - (double)SA[SI(k, il)];
                if (stage == 0) u1[k] = u0[k] - lambda * df;
                else u1[k] = .5 * (SS[SI(k, r)] - lambda * df);
            }
            __syncthreads();  // the planes are rewritten next
        }
        if (g >= c0 && g < cend) {
            double *base = a.q + chunk_base(a, DIR, W, grp, col);
#pragma unroll
            for (int k = 0; k < 5; k++) base[slots[k] * a.slab + (int64_t)g * a.rs] = u1[k];
        }
    }
}

// The HLL corrector adds (fluid after the floors of the predictor's pressure pass) and
// (predicted state after its own floors): u0 above already holds the floored fluid because
// stage_prims floors u in place, and u1 holds the floored prediction.  Both match the
// reference, whose pressure passes write the floors back to memory before each stage.

__device__ __forceinline__ int mod_n(int j, int n)
{
    int r = j % n;
    return r < 0 ? r + n : r;
}

// ------------------------------------------------------------------------------------------
// Tile-march kernel (y and z sweeps, long x rows).  One CTA owns W neighbouring pencils and
// walks them in chunks of Lc cells.  A chunk stages U0 for cells [cb-4, cb+Lc+4) in shared
// memory, runs stage A over [cb-2, cb+Lc+2) and stage B over [cb, cb+Lc), one tile cell per
// thread per phase, neighbours through shared-memory planes.  In-place safety: the next
// chunk re-reads the last four outputs of this one, so they are written only after that
// chunk's load; the last chunk re-reads cells 0..3 (periodic wrap), so the first chunk's first
// four outputs are written at the very end.
// Shared memory (doubles unless FT is float): U0t[5][TR][W], U1t[5][TR1][W] (double),
// PA,PB,PC[5][TR][W] (FT), pending[5][4][W], first[5][4][W] (double); TR = Lc+8, TR1 = Lc+4.
// ------------------------------------------------------------------------------------------
struct TileArgs {
    double *q;
    int64_t slab;
    int nx, ny, nz;
    int n;            // pencil length
    int64_t npencil;
    int Lc;           // chunk length
    DevScalar lambda;
    CylPencil cyl;    // cylindrical sweeps (GEO != CYL_NONE): radial rin, dr or the theta radius rule
};

// GEO == CYL_RADIAL adds one double per tile row and column: the HLL stage input's pressure
template <int W, int GEO = CYL_NONE>
__host__ __device__ __forceinline__ size_t tile_smem_bytes(int Lc, size_t ft)
{
    const size_t TR = Lc + 8, TR1 = Lc + 4;
    return sizeof(double) * (5 * TR * W + 5 * TR1 * W + 2 * 5 * 4 * W) + ft * 3 * 5 * TR * W +
           (GEO == CYL_RADIAL ? sizeof(double) * TR * W : 0);
}

// One sweep of W pencils by one CTA.  colbase[c] = offset of pencil c's first cell, colok[c] =
// whether pencil c exists, stride = distance between consecutive cells of a pencil, n = pencil
// length, S = slab pitch.  tsm = dynamic shared memory of tile_smem_bytes<W>(Lc).  Must be
// called by all threads of the CTA.
template <int METHOD, int SLOPE, typename FT, int DIR, int W, int GEO = CYL_NONE>
__device__ __forceinline__ void tile_sweep(double *qbase, int64_t S, const int64_t *colbase, const bool *colok,
                                           int64_t stride, int n, int Lc, double lambda, const FluidConsts<FT> &c,
                                           double *tsm, const double *colr = nullptr, double crin = 0.0,
                                           double cdr = 0.0)
{
    static_assert(GEO == CYL_NONE || std::is_same<FT, double>::value, "cylindrical sweeps are FP64");
    static_assert(GEO != CYL_RADIAL || DIR == 1, "radial sweeps run along x");
    const int TR = Lc + 8, TR1 = Lc + 4;
    double *U0t = tsm;                       // [5][TR][W]
    double *U1t = U0t + 5 * TR * W;          // [5][TR1][W]
    double *pend = U1t + 5 * TR1 * W;        // [5][4][W]
    double *first = pend + 5 * 4 * W;        // [5][4][W]
    FT *PA = reinterpret_cast<FT *>(first + 5 * 4 * W);  // [5][TR][W]
    FT *PB = PA + 5 * TR * W;
    FT *PC = PB + 5 * TR * W;
    double *PP = reinterpret_cast<double *>(PC + 5 * TR * W);  // [TR][W], GEO == CYL_RADIAL only
    constexpr int s0 = slot_of<METHOD, DIR>(0), s1 = slot_of<METHOD, DIR>(1), s2 = slot_of<METHOD, DIR>(2),
                  s3 = slot_of<METHOD, DIR>(3), s4 = slot_of<METHOD, DIR>(4);
    const int slots[5] = {s0, s1, s2, s3, s4};
    auto IDX = [&](int k, int r, int col, int R) { return (k * R + r) * W + col; };

    const int nchunks = (n + Lc - 1) / Lc;
    const bool single = (nchunks == 1);

    for (int ch = 0; ch < nchunks; ch++) {
        const int cb = ch * Lc;
        const int len = min(Lc, n - cb);          // outputs of this chunk
        const int tr = len + 8, tr1 = len + 4;    // tile rows in use
        // ---- load U0 for cells [cb-4, cb+len+4) ----
        for (int it = threadIdx.x; it < tr * W; it += blockDim.x) {
            const int r = it / W, col = it - r * W;
            const int cell = mod_n(cb - 4 + r, n);
            const double *src = qbase + colbase[col] + (int64_t)cell * stride;
#pragma unroll
            for (int k = 0; k < 5; k++) U0t[IDX(k, r, col, TR)] = src[slots[k] * S];
        }
        __syncthreads();
        // the previous chunk's last four outputs can go now that this chunk has read them
        if (ch > 0) {
            for (int it = threadIdx.x; it < 4 * W; it += blockDim.x) {
                const int r = it / W, col = it - r * W;
                if (!colok[col]) continue;
                double *dst = qbase + colbase[col] + (int64_t)(cb - 4 + r) * stride;
#pragma unroll
                for (int k = 0; k < 5; k++) dst[slots[k] * S] = pend[IDX(k, r, col, 4)];
            }
        }
        // ---- stage A ----
        for (int it = threadIdx.x; it < tr * W; it += blockDim.x) {      // prims (floors U0 for HLL)
            const int r = it / W, col = it - r * W;
            double u[5];
#pragma unroll
            for (int k = 0; k < 5; k++) u[k] = U0t[IDX(k, r, col, TR)];
            V5<FT> w = stage_prims<METHOD, DIR, FT>(u, c);
            if (METHOD == IB_METHOD_HLL) {
#pragma unroll
                for (int k = 0; k < 5; k++) U0t[IDX(k, r, col, TR)] = u[k];
                if constexpr (GEO == CYL_RADIAL) PP[r * W + col] = (double)w.a[2];  // the solver's P
            }
#pragma unroll
            for (int k = 0; k < 5; k++) PA[IDX(k, r, col, TR)] = w.a[k];
        }
        __syncthreads();
        for (int it = threadIdx.x + W; it < (tr - 1) * W; it += blockDim.x) {  // faces, rows 1..tr-2
            const int r = it / W, col = it - r * W;
            V5<FT> w, dl, dr, L, R;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                w.a[k] = PA[IDX(k, r, col, TR)];
                dl.a[k] = w.a[k] - PA[IDX(k, r - 1, col, TR)];
                dr.a[k] = PA[IDX(k, r + 1, col, TR)] - w.a[k];
            }
            stage_faces<METHOD, SLOPE, FT>(c, w, dl, dr, L, R);
#pragma unroll
            for (int k = 0; k < 5; k++) { PB[IDX(k, r, col, TR)] = L.a[k]; PC[IDX(k, r, col, TR)] = R.a[k]; }
        }
        __syncthreads();
        for (int it = threadIdx.x + W; it < (tr - 2) * W; it += blockDim.x) {  // fluxes through r+1/2, r = 1..tr-3
            const int r = it / W, col = it - r * W;
            V5<FT> Lr, Rl;
#pragma unroll
            for (int k = 0; k < 5; k++) { Rl.a[k] = PC[IDX(k, r, col, TR)]; Lr.a[k] = PB[IDX(k, r + 1, col, TR)]; }
            V5<FT> f = stage_flux<METHOD, FT>(c, Rl, Lr);
#pragma unroll
            for (int k = 0; k < 5; k++) PA[IDX(k, r, col, TR)] = f.a[k];
        }
        __syncthreads();
        for (int it = threadIdx.x; it < tr1 * W; it += blockDim.x) {  // U1 for tile rows 2..tr-3
            const int r1 = it / W, col = it - r1 * W, r = r1 + 2;
            if constexpr (GEO == CYL_NONE) {
#pragma unroll
                for (int k = 0; k < 5; k++)
                    U1t[IDX(k, r1, col, TR1)] = U0t[IDX(k, r, col, TR)] -
                                                lambda * ((double)PA[IDX(k, r, col, TR)] - (double)PA[IDX(k, r - 1, col, TR)]);
            } else {
                const double rc = (GEO == CYL_RADIAL) ? crin + mod_n(cb - 2 + r1, n) * cdr : 0.0;
                const double rp = (GEO == CYL_RADIAL) ? 0.0 : colr[col];
                const double lam = (GEO == CYL_THETA_LAM) ? lambda / rp : lambda;
                const double psum = (GEO == CYL_RADIAL && METHOD == IB_METHOD_HLLC)
                                        ? (double)PB[IDX(1, r, col, TR)] + (double)PC[IDX(1, r, col, TR)] : 0.0;
                const double php = (GEO == CYL_RADIAL && METHOD == IB_METHOD_HLL) ? PP[r * W + col] : 0.0;
#pragma unroll
                for (int k = 0; k < 5; k++)
                    U1t[IDX(k, r1, col, TR1)] =
                        U0t[IDX(k, r, col, TR)] -
                        cyl_dflux<METHOD, GEO>(k, (double)PA[IDX(k, r, col, TR)], (double)PA[IDX(k, r - 1, col, TR)], lam,
                                               rc, cdr, rp, psum, php, U1t[IDX(0, r1, col, TR1)], c);
            }
        }
        __syncthreads();
        // ---- stage B (rows of U1t; U1t row r1 is cell cb-2+r1) ----
        for (int it = threadIdx.x; it < tr1 * W; it += blockDim.x) {
            const int r1 = it / W, col = it - r1 * W;
            double u[5];
#pragma unroll
            for (int k = 0; k < 5; k++) u[k] = U1t[IDX(k, r1, col, TR1)];
            V5<FT> w = stage_prims<METHOD, DIR, FT>(u, c);
            if (METHOD == IB_METHOD_HLL) {
#pragma unroll
                for (int k = 0; k < 5; k++) U1t[IDX(k, r1, col, TR1)] = u[k];
                if constexpr (GEO == CYL_RADIAL) PP[r1 * W + col] = (double)w.a[2];
            }
#pragma unroll
            for (int k = 0; k < 5; k++) PA[IDX(k, r1, col, TR)] = w.a[k];
        }
        __syncthreads();
        for (int it = threadIdx.x + W; it < (tr1 - 1) * W; it += blockDim.x) {
            const int r = it / W, col = it - r * W;
            V5<FT> w, dl, dr, L, R;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                w.a[k] = PA[IDX(k, r, col, TR)];
                dl.a[k] = w.a[k] - PA[IDX(k, r - 1, col, TR)];
                dr.a[k] = PA[IDX(k, r + 1, col, TR)] - w.a[k];
            }
            stage_faces<METHOD, SLOPE, FT>(c, w, dl, dr, L, R);
#pragma unroll
            for (int k = 0; k < 5; k++) { PB[IDX(k, r, col, TR)] = L.a[k]; PC[IDX(k, r, col, TR)] = R.a[k]; }
        }
        __syncthreads();
        for (int it = threadIdx.x + W; it < (tr1 - 2) * W; it += blockDim.x) {
            const int r = it / W, col = it - r * W;
            V5<FT> Lr, Rl;
#pragma unroll
            for (int k = 0; k < 5; k++) { Rl.a[k] = PC[IDX(k, r, col, TR)]; Lr.a[k] = PB[IDX(k, r + 1, col, TR)]; }
            V5<FT> f = stage_flux<METHOD, FT>(c, Rl, Lr);
#pragma unroll
            for (int k = 0; k < 5; k++) PA[IDX(k, r, col, TR)] = f.a[k];
        }
        __syncthreads();
        for (int it = threadIdx.x; it < len * W; it += blockDim.x) {  // outputs: U1t rows 2..len+1
            const int m = it / W, col = it - m * W, r1 = m + 2;
            double out[5];
            if constexpr (GEO == CYL_NONE) {
#pragma unroll
                for (int k = 0; k < 5; k++)
                    out[k] = .5 * (U1t[IDX(k, r1, col, TR1)] + U0t[IDX(k, r1 + 2, col, TR)] -
                                   lambda * ((double)PA[IDX(k, r1, col, TR)] - (double)PA[IDX(k, r1 - 1, col, TR)]));
            } else {
                const double rc = (GEO == CYL_RADIAL) ? crin + (cb + m) * cdr : 0.0;
                const double rp = (GEO == CYL_RADIAL) ? 0.0 : colr[col];
                const double lam = (GEO == CYL_THETA_LAM) ? lambda / rp : lambda;
                const double psum = (GEO == CYL_RADIAL && METHOD == IB_METHOD_HLLC)
                                        ? (double)PB[IDX(1, r1, col, TR)] + (double)PC[IDX(1, r1, col, TR)] : 0.0;
                const double php = (GEO == CYL_RADIAL && METHOD == IB_METHOD_HLL) ? PP[r1 * W + col] : 0.0;
                const double rho1 = U1t[IDX(0, r1, col, TR1)];
#pragma unroll
                for (int k = 0; k < 5; k++)
                    out[k] = .5 * (U1t[IDX(k, r1, col, TR1)] + U0t[IDX(k, r1 + 2, col, TR)] -
                                   cyl_dflux<METHOD, GEO>(k, (double)PA[IDX(k, r1, col, TR)],
                                                          (double)PA[IDX(k, r1 - 1, col, TR)], lam, rc, cdr, rp, psum,
                                                          php, rho1, c));
            }
            const int cell = cb + m;
            if (!single && ch == 0 && m < 4) {
#pragma unroll
                for (int k = 0; k < 5; k++) first[IDX(k, m, col, 4)] = out[k];
            } else if (!single && m >= len - 4) {
                const int pr = m - (len - 4);
#pragma unroll
                for (int k = 0; k < 5; k++) pend[IDX(k, pr, col, 4)] = out[k];
            } else if (colok[col]) {
                double *dst = qbase + colbase[col] + (int64_t)cell * stride;
#pragma unroll
                for (int k = 0; k < 5; k++) dst[slots[k] * S] = out[k];
            }
        }
        __syncthreads();
    }
    if (!single) {
        const int cbl = (nchunks - 1) * Lc, lenl = n - cbl;
        for (int it = threadIdx.x; it < 4 * W; it += blockDim.x) {
            const int r = it / W, col = it - r * W;
            if (!colok[col]) continue;
            double *dl = qbase + colbase[col] + (int64_t)(cbl + lenl - 4 + r) * stride;
            double *df = qbase + colbase[col] + (int64_t)r * stride;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                dl[slots[k] * S] = pend[IDX(k, r, col, 4)];
                df[slots[k] * S] = first[IDX(k, r, col, 4)];
            }
        }
    }
    __syncthreads();
}

template <int METHOD, int SLOPE, typename FT, int DIR, int W, int GEO = CYL_NONE>
__global__ void __launch_bounds__(256, 4) sweep_tile_kernel(TileArgs a, FluidConsts<FT> c)
{
    extern __shared__ __align__(16) double tsm[];
    __shared__ int64_t colbase[W];
    __shared__ bool colok[W];
    __shared__ double colr[W];
    if (a.lambda.off()) return;  // a device timestep of 0: after the end time
    int64_t stride;
    if (DIR == 1) stride = 1;
    else if (DIR == 2) stride = a.nx;
    else stride = (int64_t)a.nx * a.ny;
    if (threadIdx.x < W) {
        int64_t p = (int64_t)blockIdx.x * W + threadIdx.x;
        colok[threadIdx.x] = p < a.npencil;
        if (p >= a.npencil) p = 0;
        int64_t b;
        if (DIR == 1) b = p * a.nx;
        else if (DIR == 2) b = (p % a.nx) + (int64_t)a.nx * a.ny * (p / a.nx);
        else b = p;
        colbase[threadIdx.x] = b;
        // theta pencils (DIR 2): radial index p mod nx, z index p / nx
        if (GEO == CYL_THETA_DIV || GEO == CYL_THETA_LAM)
            colr[threadIdx.x] = theta_radius(a.cyl, (int)(p % a.nx), (int)(p / a.nx));
    }
    __syncthreads();
    tile_sweep<METHOD, SLOPE, FT, DIR, W, GEO>(a.q, a.slab, colbase, colok, stride, a.n, a.Lc, a.lambda.get(), c, tsm,
                                               colr, a.cyl.rin, a.cyl.dr);
}

}  // namespace ib
