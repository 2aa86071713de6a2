// ib_xinjin.cu -- Xin-Jin relaxing TVD sweep (cukern_XinJinHydro_step, gpuclass/cudaFluidStep.cu:2427-2654)
// with the per-row freezing speed of cukern_PressureFreezeSolverHydro (:2867-2941).
//
// The reference needs the maximum of |v|+c_s over the whole swept row before each stage, so it
// runs freeze / predictor / freeze / corrector as four kernels with a host reduction in
// between (MGA_globalReduceDimension, cudaCommon.cu:919-1004).  Here one CTA owns one pencil (or
// 2 to 4 adjacent y/z pencils): it keeps them in registers, reduces each freezing speed in-block,
// and runs both stages, so a sweep is one launch with one read and one write of the state.
#include <cstdlib>

#include "ib_internal.cuh"

namespace ib {

// Maximum over the pencil of column `col` (W interleaved pencils per block), ignoring NaN
// candidates as the reference's `(a > b) ? a : b` tree does.
template <int W>
__device__ __forceinline__ double block_max_keep(double v, double *red, int col)
{
#pragma unroll
    for (int o = 16; o >= W; o >>= 1) {
        double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = (w > v) ? w : v;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane < W) red[wid * W + lane] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < nw; w++) m = (red[w * W + col] > m) ? red[w * W + col] : m;
    return m;
}

// Freezing speed |v| + c_s of one cell.  Uses memory slab 2 (px) as the transported momentum
// whatever the sweep direction, as the reference's freeze kernel does.
__device__ __forceinline__ double freeze_cell(const double (&X)[5], double invrho, double gamma, double gm1)
{
    double psq = X[3];
    double px = X[4];
    psq = psq * psq + px * px;
    px = X[2];
    psq += px * px;
    double P = (X[1] - .5 * psq * invrho) * gm1;
    return fabs(px) * invrho + sqrt(gamma * P * invrho);
}

// The left- and right-going limited fluxes of one component, flux_limit<FLIM>(A1, B1) and
// flux_limit<FLIM>(A2, B2).  Product build, Ospre and van Leer: their two divisions share one
// (1/(d1 d2) times d2 and d1) when d1, d2 and d1 d2 are all normal numbers, so that neither
// reciprocal can overflow; otherwise (subnormal denominators of momenta near 1e-154, where a
// reciprocal of infinity times an underflowed zero numerator would give NaN) each divides on
// its own, as the strict build always does.
template <int FLIM>
__device__ __forceinline__ void flux_limit_pair(double A1, double B1, double A2, double B2, double &o1, double &o2)
{
#ifndef IB_STRICT_ARITH
    if constexpr (FLIM == IB_FLUX_OSPRE || FLIM == IB_FLUX_VANLEER) {
        double n1, d1, n2, d2;
        bool p1, p2;
        if constexpr (FLIM == IB_FLUX_OSPRE) {  // 1.5 r (A + B) / (A^2 + r + B^2), 0 where r <= 0
            const double r1 = A1 * B1, r2 = A2 * B2;
            p1 = !(r1 <= 0.0);
            p2 = !(r2 <= 0.0);
            n1 = 1.5 * r1 * (A1 + B1);
            d1 = A1 * A1 + r1 + B1 * B1;
            n2 = 1.5 * r2 * (A2 + B2);
            d2 = A2 * A2 + r2 + B2 * B2;
        } else {  // 2AB / (A + B) where 2AB > 0
            const double r1 = 2.0 * A1 * B1, r2 = 2.0 * A2 * B2;
            p1 = r1 > 0.0;
            p2 = r2 > 0.0;
            n1 = r1;
            d1 = A1 + B1;
            n2 = r2;
            d2 = A2 + B2;
        }
        d1 = p1 ? d1 : 1.0;
        d2 = p2 ? d2 : 1.0;
        const double pd = d1 * d2;
        constexpr double kMinNormal = 2.2250738585072014e-308, kMax = 1.7976931348623157e308;
        if (fabs(d1) >= kMinNormal && fabs(d2) >= kMinNormal && fabs(pd) >= kMinNormal && fabs(pd) <= kMax) {
            const double rr = 1.0 / pd;
            o1 = p1 ? n1 * (d2 * rr) : 0.0;
            o2 = p2 ? n2 * (d1 * rr) : 0.0;
        } else {
            o1 = p1 ? n1 / d1 : 0.0;
            o2 = p2 ? n2 / d2 : 0.0;
        }
        return;
    }
#endif
    o1 = flux_limit<FLIM>(A1, B1);
    o2 = flux_limit<FLIM>(A2, B2);
}

// W adjacent pencils per block (W = 1 for x rows; y/z pencils take W = 2 or 4 when nx allows it,
// so that the loads of a warp cover 16- or 32-byte runs of x instead of single doubles a row or a
// plane apart).  Thread t works on column t % W and cells t / W + m * S (m < CPT,
// S = blockDim / W); a cell's five conserved variables stay in registers through both stages and
// only the relaxation fluxes L = C q - F, R = C q + F pass through shared memory ([5][n][W]
// each), so a stage costs the freezing-speed reduction and one (predictor) or three (corrector)
// barriers.  RELOAD (x rows): the corrector re-reads its base state from memory, coalesced and
// L2-resident, rather than keep it in registers; fewer spills made x 0.85 -> 0.82 ms at 256^3 and
// 0.30 -> 0.27 ms at 2048^2, while the strided y/z loads measured slower that way.
//
// Cylindrical geometry (GEO, ib_cyl.cuh): radial x sweeps weight the relaxation fluxes by the face
// radii and add 2 dr / r_c times the stage input's pressure to p_r, the factor 2 compensating the
// halved lambda (cudaFluidStep.cu:2463-2470, 2576-2581, 2603-2607); theta y sweeps divide the
// update by the pencil radius or lambda by it first (2478-2480, 2582-2585, 2608-2611).
template <int FLIM, int W, int CPT, bool RELOAD, int GEO = CYL_NONE>
__global__ void __launch_bounds__(1024) xj_pencil_kernel(double *q, int64_t slab, int nx, int ny, int nz, int dir,
                                                         DevScalar lam_in, double gamma, double minmass, double mintemp,
                                                         CylPencil cyl)
{
    if (lam_in.off()) return;  // a device timestep of 0: after the end time
    const double lambda = lam_in.get();
    extern __shared__ __align__(16) double sm[];
    __shared__ double red[32 * W];
    const int n = (dir == 1) ? nx : (dir == 2 ? ny : nz);
    const int NW = n * W;
    double *Lb = sm;            // [5][n][W]
    double *Rb = Lb + 5 * NW;   // [5][n][W]

    const int col = (W == 1) ? 0 : (int)(threadIdx.x % W);
    const int r0 = (int)(threadIdx.x / W), S = (int)(blockDim.x / W);
    auto IX = [&](int k, int i) { return (k * n + i) * W + col; };
    const int64_t p = (int64_t)blockIdx.x * W + col;  // this column's pencil
    int64_t base, stride;
    if (dir == 1) { base = p * nx; stride = 1; }
    else if (dir == 2) { base = (p % nx) + (int64_t)nx * ny * (p / nx); stride = nx; }
    else { base = p; stride = (int64_t)nx * ny; }
    const int nslot = 1 + dir;
    const double gm1 = gamma - 1.0;
    // theta pencils: the radius of this column's pencil (radial index p mod nx, z index p / nx)
    const double rpen = (GEO == CYL_THETA_DIV || GEO == CYL_THETA_LAM)
                            ? theta_radius(cyl, (int)(p % nx), (int)(p / nx)) : 1.0;
    double pcell[GEO == CYL_RADIAL ? CPT : 1];  // radial: each cell's stage-input pressure

    double u0[CPT][5], u1[CPT][5];
    // 1 / density of each cell's current stage input: the product build computes it once per stage
    // (for the freezing speed, the pressure and the velocity) and takes the corrector's from the
    // predictor's floor; the strict build divides where the reference does
#ifndef IB_STRICT_ARITH
    double rinv[CPT];
#endif
#pragma unroll
    for (int m = 0; m < CPT; m++) {
        const int i = r0 + m * S;
#pragma unroll
        for (int k = 0; k < 5; k++) u0[m][k] = (i < n) ? q[k * slab + base + i * stride] : 1.0;
    }

#pragma unroll
    for (int stage = 0; stage < 2; stage++) {
        const double lam = (stage == 0) ? 0.25 * lambda : 0.5 * lambda;
        // freezing speed of the pencil (cudaFluidStep.cu:2867-2941 + the global max)
        double cm = 0.0;
#pragma unroll
        for (int m = 0; m < CPT; m++) {
            if (r0 + m * S < n) {
                const double(&X)[5] = (stage == 0) ? u0[m] : u1[m];
#ifdef IB_STRICT_ARITH
                const double v = freeze_cell(X, 1.0 / X[0], gamma, gm1);
#else
                if (stage == 0) rinv[m] = 1.0 / X[0];
                const double v = freeze_cell(X, rinv[m], gamma, gm1);
#endif
                cm = (v > cm) ? v : cm;
            }
        }
        const double Cf = block_max_keep<W>(cm, red, col);
        // relaxation fluxes of every component (cudaFluidStep.cu:2470-2520)
#pragma unroll
        for (int m = 0; m < CPT; m++) {
            const int i = r0 + m * S;
            if (i < n) {
                const double *Q = (stage == 0) ? u0[m] : u1[m];
                const double q1 = Q[1], q2 = Q[2], q3 = Q[3], q4 = Q[4];
#ifdef IB_STRICT_ARITH
                const double Pv = gm1 * (q1 - .5 * (q4 * q4 + q3 * q3 + q2 * q2) / Q[0]);
                const double Vx = Q[nslot] / Q[0];
#else
                const double ir = rinv[m];
                const double Pv = gm1 * (q1 - .5 * (q4 * q4 + q3 * q3 + q2 * q2) * ir);
                const double Vx = Q[nslot] * ir;
#endif
                if constexpr (GEO == CYL_RADIAL) pcell[m] = Pv;
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    const double qk = Q[k];
                    double w;
                    if (k == 0) w = Q[nslot];
                    else if (k == 1) w = Vx * (qk + Pv);
                    else if (k == nslot) w = Vx * qk + Pv;
                    else w = Vx * qk;
                    Lb[IX(k, i)] = (Cf * qk - w);
                    Rb[IX(k, i)] = (Cf * qk + w);
                }
            }
        }
        __syncthreads();
        if (stage == 1) {
            // limited second-order fluxes (cudaFluidStep.cu:2560-2600), written back in place
            double nl[CPT][5], nr[CPT][5];
#pragma unroll
            for (int m = 0; m < CPT; m++) {
                const int i = r0 + m * S;
                if (i < n) {
                    const int il = (i == 0) ? n - 1 : i - 1, ir = (i == n - 1) ? 0 : i + 1;
#pragma unroll
                    for (int k = 0; k < 5; k++) {
                        const double Lm = Lb[IX(k, il)], L0 = Lb[IX(k, i)], Lp = Lb[IX(k, ir)];
                        const double Rm = Rb[IX(k, il)], R0 = Rb[IX(k, i)], Rp = Rb[IX(k, ir)];
                        const double dL0 = 0.5 * (L0 - Lm), dLp = 0.5 * (Lp - L0);
                        const double dR0 = 0.5 * (R0 - Rm), dRp = 0.5 * (Rp - R0);
                        double limL, limR;
                        flux_limit_pair<FLIM>(dL0, dLp, dR0, dRp, limL, limR);
                        nl[m][k] = L0 - limL;
                        nr[m][k] = R0 + limR;
                    }
                }
            }
            __syncthreads();
#pragma unroll
            for (int m = 0; m < CPT; m++) {
                const int i = r0 + m * S;
                if (i < n) {
#pragma unroll
                    for (int k = 0; k < 5; k++) { Lb[IX(k, i)] = nl[m][k]; Rb[IX(k, i)] = nr[m][k]; }
                }
            }
            __syncthreads();
        }
        // update and floors (cudaFluidStep.cu:2610-2629)
#pragma unroll
        for (int m = 0; m < CPT; m++) {
            const int i = r0 + m * S;
            if (i < n) {
                const int il = (i == 0) ? n - 1 : i - 1, ir = (i == n - 1) ? 0 : i + 1;
                double pr[5];
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    // the block's own pencils are unchanged in memory until the final store
                    const double b = (RELOAD && stage == 1) ? q[k * slab + base + i * stride] : u0[m][k];
                    if constexpr (GEO == CYL_NONE) {
                        pr[k] = b - lam * (Rb[IX(k, i)] - Rb[IX(k, il)] - Lb[IX(k, ir)] + Lb[IX(k, i)]);
                    } else if constexpr (GEO == CYL_THETA_DIV) {
#ifdef IB_STRICT_ARITH
                        pr[k] = b - lam * (Rb[IX(k, i)] - Rb[IX(k, il)] - Lb[IX(k, ir)] + Lb[IX(k, i)]) / rpen;
#else
                        // the product build multiplies by the radius' reciprocal (one division)
                        pr[k] = b - lam * (Rb[IX(k, i)] - Rb[IX(k, il)] - Lb[IX(k, ir)] + Lb[IX(k, i)]) * (1.0 / rpen);
#endif
                    } else if constexpr (GEO == CYL_THETA_LAM) {
                        const double lr = lam / rpen;
                        pr[k] = b - lr * (Rb[IX(k, i)] - Rb[IX(k, il)] - Lb[IX(k, ir)] + Lb[IX(k, i)]);
                    } else {
                        const double rc = cyl.rin + i * cyl.dr;
#ifdef IB_STRICT_ARITH
                        const double cA = (rc - .5 * cyl.dr) / (rc);
                        const double cB = (rc + .5 * cyl.dr) / (rc);
                        const double cC = 2.0 * cyl.dr / rc;
#else
                        const double ri = 1.0 / rc;  // the product build: one division per cell
                        const double cA = (rc - .5 * cyl.dr) * ri;
                        const double cB = (rc + .5 * cyl.dr) * ri;
                        const double cC = 2.0 * cyl.dr * ri;
#endif
                        pr[k] = b - lam * (cB * Rb[IX(k, i)] - cA * Rb[IX(k, il)] - cB * Lb[IX(k, ir)] + cA * Lb[IX(k, i)]);
                        if (k == 2) pr[k] += lam * cC * pcell[m];
                    }
                }
                double p0 = pr[0], p1 = pr[1];
                const double p2 = pr[2], p3 = pr[3], p4 = pr[4];
                p0 = (p0 < minmass) ? minmass : p0;
#ifdef IB_STRICT_ARITH
                double w = .5 * (p2 * p2 + p3 * p3 + p4 * p4) / p0;
#else
                rinv[m] = 1.0 / p0;
                double w = .5 * (p2 * p2 + p3 * p3 + p4 * p4) * rinv[m];
#endif
                if ((p1 - w) < p0 * mintemp) p1 = w + p0 * mintemp;
                u1[m][0] = p0; u1[m][1] = p1; u1[m][2] = p2; u1[m][3] = p3; u1[m][4] = p4;
            }
        }
    }
#pragma unroll
    for (int m = 0; m < CPT; m++) {
        const int i = r0 + m * S;
        if (i < n) {
#pragma unroll
            for (int k = 0; k < 5; k++) q[k * slab + base + i * stride] = u1[m][k];
        }
    }
}

// y/z sweeps of pencils of up to 256 cells, or of 512: the pencil-pair kernel's structure.  One TMA
// box of WC adjacent pencils (the box [slab][cell][column] with the column fastest, 16-byte rows for
// WC = 2) per CTA of one thread per cell; the CTA sweeps the pencils one after the other through
// xj_pencil_kernel's arithmetic (one column, one cell per thread: the freezing-speed reduction over
// the block, the relaxation fluxes through shared memory), writes each result over its own column
// of the box and leaves by one TMA store.  No strided loads from global memory (xj_pencil_kernel's
// y/z loads are single doubles or 16-byte pieces a row apart) and four CTAs per SM at 256 cells.
// Every tile wait is bounded (a.spin); one that runs out sets the error flag and leaves.
struct XjPairArgs {
    int n, npw;
    DevScalar lambda;
    double gamma, minmass, mintemp;
    unsigned int *err;
    uint32_t spin;
    CylPencil cyl;  // cylindrical theta pencils (GEO): the radius rule
};

__host__ __device__ __forceinline__ size_t xj_box_bytes(int n, int wc) { return ((size_t)40 * n * wc + 127) / 128 * 128; }

// GEO == CYL_THETA_DIV / CYL_THETA_LAM: cylindrical theta pencils (y), the update's flux
// difference divided by the pencil's radius or the stage's lambda divided by it, as in
// xj_pencil_kernel.
// PADN (pencils of a run-time length only): stride of the flux planes fixed at PADN cells, so
// that the phases address them at constant offsets; 0 = the pencil length.
template <int FLIM, int DIR, int NFIX, int WC, int GEO = CYL_NONE, int PADN = 0>
__global__ void __launch_bounds__(NFIX == 512 ? 512 : 256, NFIX == 512 ? 2 : 4)
    xj_pair_kernel(const __grid_constant__ CUtensorMap tm, XjPairArgs a)
{
    static_assert(GEO == CYL_NONE || ((GEO == CYL_THETA_DIV || GEO == CYL_THETA_LAM) && DIR == 2),
                  "theta pencils run along y");
    static_assert(DIR != 1 || (WC == 1 && GEO == CYL_NONE), "x rows: one row per box, square geometry");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full;
    __shared__ double red[32];
    const int n = NFIX ? NFIX : a.n;
    const int NP = NFIX ? NFIX : (PADN ? PADN : n);  // stride of the flux planes
    double *T = reinterpret_cast<double *>(smem_raw);                        // [5][n][WC]
    double *Lb = reinterpret_cast<double *>(smem_raw + xj_box_bytes(n, WC));  // [5][NP]
    double *Rb = Lb + 5 * NP;                                                 // [5][NP]
    const int i = threadIdx.x;
    const bool act = i < n;
    const int il = (i == 0) ? n - 1 : i - 1, ir = (i == n - 1) ? 0 : i + 1;
    constexpr int nslot = 1 + DIR;
    const double gm1 = a.gamma - 1.0;
    const int64_t b = blockIdx.x;
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
        if constexpr (DIR == 1) tma_load_3d(T, &tm, 0, (int)b, 0, &full);
        else tma_load_5d(T, &tm, (int)(b % a.npw) * WC, 0, 0, (int)(b / a.npw), 0, &full);
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
#ifndef IB_STRICT_ARITH
        double rinv = 1.0;
#endif
        const double rpen = (GEO != CYL_NONE) ? theta_radius(a.cyl, (int)(b % a.npw) * WC + col, (int)(b / a.npw)) : 1.0;
#pragma unroll
        for (int k = 0; k < 5; k++) u0[k] = act ? T[TI(k)] : 1.0;
#pragma unroll
        for (int stage = 0; stage < 2; stage++) {
            const double lam = (stage == 0) ? 0.25 * lambda : 0.5 * lambda;
            const double(&X)[5] = (stage == 0) ? u0 : u1;
            // a NaN freezing speed (negative pressure) never wins, as in the reference's max
            double cm = 0.0;
            if (act) {
#ifdef IB_STRICT_ARITH
                const double v = freeze_cell(X, 1.0 / X[0], a.gamma, gm1);
#else
                if (stage == 0) rinv = 1.0 / X[0];
                const double v = freeze_cell(X, rinv, a.gamma, gm1);
#endif
                cm = (v > cm) ? v : cm;
            }
            const double Cf = block_max_keep<1>(cm, red, 0);
            if (act) {
                const double q1 = X[1], q2 = X[2], q3 = X[3], q4 = X[4];
#ifdef IB_STRICT_ARITH
                const double Pv = gm1 * (q1 - .5 * (q4 * q4 + q3 * q3 + q2 * q2) / X[0]);
                const double Vx = X[nslot] / X[0];
#else
                const double Pv = gm1 * (q1 - .5 * (q4 * q4 + q3 * q3 + q2 * q2) * rinv);
                const double Vx = X[nslot] * rinv;
#endif
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    const double qk = X[k];
                    double w;
                    if (k == 0) w = X[nslot];
                    else if (k == 1) w = Vx * (qk + Pv);
                    else if (k == nslot) w = Vx * qk + Pv;
                    else w = Vx * qk;
                    Lb[k * NP + i] = (Cf * qk - w);
                    Rb[k * NP + i] = (Cf * qk + w);
                }
            }
            __syncthreads();
            if (stage == 1) {
                double nl[5], nr[5];
                if (act) {
#pragma unroll
                    for (int k = 0; k < 5; k++) {
                        const double Lm = Lb[k * NP + il], L0 = Lb[k * NP + i], Lp = Lb[k * NP + ir];
                        const double Rm = Rb[k * NP + il], R0 = Rb[k * NP + i], Rp = Rb[k * NP + ir];
                        const double dL0 = 0.5 * (L0 - Lm), dLp = 0.5 * (Lp - L0);
                        const double dR0 = 0.5 * (R0 - Rm), dRp = 0.5 * (Rp - R0);
                        double limL, limR;
                        flux_limit_pair<FLIM>(dL0, dLp, dR0, dRp, limL, limR);
                        nl[k] = L0 - limL;
                        nr[k] = R0 + limR;
                    }
                }
                __syncthreads();
                if (act) {
#pragma unroll
                    for (int k = 0; k < 5; k++) { Lb[k * NP + i] = nl[k]; Rb[k * NP + i] = nr[k]; }
                }
                __syncthreads();
            }
            if (act) {
                double pr[5];
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    if constexpr (GEO == CYL_NONE) {
                        pr[k] = u0[k] - lam * (Rb[k * NP + i] - Rb[k * NP + il] - Lb[k * NP + ir] + Lb[k * NP + i]);
                    } else if constexpr (GEO == CYL_THETA_DIV) {
#ifdef IB_STRICT_ARITH
                        pr[k] = u0[k] - lam * (Rb[k * NP + i] - Rb[k * NP + il] - Lb[k * NP + ir] + Lb[k * NP + i]) / rpen;
#else
                        pr[k] = u0[k] - lam * (Rb[k * NP + i] - Rb[k * NP + il] - Lb[k * NP + ir] + Lb[k * NP + i]) *
                                            (1.0 / rpen);
#endif
                    } else {
                        const double lr = lam / rpen;
                        pr[k] = u0[k] - lr * (Rb[k * NP + i] - Rb[k * NP + il] - Lb[k * NP + ir] + Lb[k * NP + i]);
                    }
                }
                double p0 = pr[0], p1 = pr[1];
                const double p2 = pr[2], p3 = pr[3], p4 = pr[4];
                p0 = (p0 < a.minmass) ? a.minmass : p0;
#ifdef IB_STRICT_ARITH
                double w = .5 * (p2 * p2 + p3 * p3 + p4 * p4) / p0;
#else
                rinv = 1.0 / p0;
                double w = .5 * (p2 * p2 + p3 * p3 + p4 * p4) * rinv;
#endif
                if ((p1 - w) < p0 * a.mintemp) p1 = w + p0 * a.mintemp;
                u1[0] = p0; u1[1] = p1; u1[2] = p2; u1[3] = p3; u1[4] = p4;
            }
        }
        // this pencil's result over its own column of the box (its inputs were read above)
        if (act) {
#pragma unroll
            for (int k = 0; k < 5; k++) T[TI(k)] = u1[k];
        }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (leader) {
        if constexpr (DIR == 1) tma_store_3d(&tm, T, 0, (int)b, 0);
        else tma_store_5d(&tm, T, (int)(b % a.npw) * WC, 0, 0, (int)(b / a.npw), 0);
        bulk_commit();
        bulk_wait_all();
    }
}

// Returns IB_ERROR_NOIMPLEMENT (the caller falls back to xj_pencil_kernel) where TMA's rules or
// the kernel's sizes do not hold: nx a multiple of WC, 16-byte aligned base and slab pitch, pencils
// of up to 256 cells or of 512.
template <int FLIM, int DIR, int NFIX, int WC, int GEO = CYL_NONE, int PADN = 0>
static int launch_xj_pair(double *q, int64_t slab, const int grid[3], DevScalar lambda, double gamma, double rho_min,
                          double mintemp, cudaStream_t st, CylPencil cyl = CylPencil{0.0, 0.0, 0, 0})
{
    const int nx = grid[0], ny = grid[1], nz = grid[2];
    const int n = grid[DIR - 1];
    if ((NFIX && n != NFIX) || (!NFIX && n > 256) || n < 3 || (nx % WC) || (PADN && n > PADN))
        return IB_ERROR_NOIMPLEMENT;
    if (((uintptr_t)q & 15) || (slab * 8) % 16) return IB_ERROR_NOIMPLEMENT;
    CUtensorMap tm;
    int npw;
    int64_t nblocks;
    int rc;
    if constexpr (DIR == 1) {
        // x rows: a box of one whole row and 5 slabs (rows of up to 256 cells, an even number, so
        // that the row pitch is a multiple of 16 bytes)
        if (n > 256 || (nx & 1)) return IB_ERROR_NOIMPLEMENT;
        npw = 1;
        nblocks = (int64_t)ny * nz;
        if (nblocks >= (int64_t)1 << 31) return IB_ERROR_NOIMPLEMENT;
        uint64_t dims[3] = {(uint64_t)nx, (uint64_t)nblocks, 5};
        uint64_t strides[2] = {(uint64_t)nx * 8, (uint64_t)slab * 8};
        uint32_t box[3] = {(uint32_t)nx, 1, 5};
        rc = encode_tmap_f64(&tm, q, 3, dims, strides, box);
    } else {
        const uint64_t other = (DIR == 2) ? nz : ny;
        const uint64_t rs = (DIR == 2) ? (uint64_t)nx * 8 : (uint64_t)nx * ny * 8;  // along the pencil
        const uint64_t os = (DIR == 2) ? (uint64_t)nx * ny * 8 : (uint64_t)nx * 8;  // across pencils
        // TMA boxes are at most 256 rows: a 512-cell pencil comes as two rows of 256
        const int bh = (n > 256) ? n / 2 : n, nh = (n > 256) ? 2 : 1;
        uint64_t dims[5] = {(uint64_t)nx, (uint64_t)bh, (uint64_t)nh, other, 5};
        uint64_t strides[4] = {rs, rs * bh, os, (uint64_t)slab * 8};
        uint32_t box[5] = {WC, (uint32_t)bh, (uint32_t)nh, 1, 5};
        npw = nx / WC;
        nblocks = (int64_t)npw * other;
        if (nblocks >= (int64_t)1 << 31) return IB_ERROR_NOIMPLEMENT;
        rc = encode_tmap_f64(&tm, q, 5, dims, strides, box);
    }
    if (rc) return rc;
    unsigned int *err = scratch().wait_flag();
    if (!err) return IB_ERROR_NOMEM;
    const int nt = (n + 31) / 32 * 32;
    const size_t shm = xj_box_bytes(n, WC) + (size_t)80 * (NFIX ? NFIX : (PADN ? PADN : n));
    static int attr_bytes = 0;
    if ((int)shm > attr_bytes) {
        rc = check_cuda(cudaFuncSetAttribute(xj_pair_kernel<FLIM, DIR, NFIX, WC, GEO, PADN>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        if (rc) return rc;
        attr_bytes = (int)shm;
    }
    XjPairArgs a{n, npw, lambda, gamma, rho_min, mintemp, err, tile_wait_limit(), cyl};
    xj_pair_kernel<FLIM, DIR, NFIX, WC, GEO, PADN><<<(unsigned)nblocks, nt, shm, st>>>(tm, a);
    return check_launch();
}

// Cylindrical theta pencils (y) of up to 256 cells in the pencil-box kernel
template <int FLIM>
static int launch_xj_pair_theta(int geo, double *q, int64_t slab, const int grid[3], DevScalar lambda, double gamma,
                                double rho_min, double mintemp, cudaStream_t st, const CylPencil &cyl)
{
    const int n = grid[1];
    if (geo == CYL_THETA_DIV) {
        if (n == 256)
            return launch_xj_pair<FLIM, 2, 256, 2, CYL_THETA_DIV>(q, slab, grid, lambda, gamma, rho_min, mintemp, st, cyl);
        return launch_xj_pair<FLIM, 2, 0, 2, CYL_THETA_DIV>(q, slab, grid, lambda, gamma, rho_min, mintemp, st, cyl);
    }
    if (n == 256)
        return launch_xj_pair<FLIM, 2, 256, 2, CYL_THETA_LAM>(q, slab, grid, lambda, gamma, rho_min, mintemp, st, cyl);
    return launch_xj_pair<FLIM, 2, 0, 2, CYL_THETA_LAM>(q, slab, grid, lambda, gamma, rho_min, mintemp, st, cyl);
}

template <int FLIM>
static int launch_xj_pair_dir(int dir, double *q, int64_t slab, const int grid[3], DevScalar lambda, double gamma,
                              double rho_min, double mintemp, cudaStream_t st)
{
    const int n = grid[dir - 1];
    // pencils of 65-127 and 129-255 cells: flux planes of a fixed 128- or 256-cell stride (96^3 y/z
    // 0.048 -> 0.046 ms, 112^3 0.076 -> 0.071, 160^3 0.206 -> 0.194, 192^3 0.351 -> 0.331; a 256-cell
    // stride for pencils of 128 or fewer measured slower, the larger planes costing CTAs per SM)
    if (dir == 1) {  // x rows of up to 256 cells, one row per box
        if (n == 256) return launch_xj_pair<FLIM, 1, 256, 1>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
        if (n > 128)
            return launch_xj_pair<FLIM, 1, 0, 1, CYL_NONE, 256>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
        if (n > 64 && n < 128)
            return launch_xj_pair<FLIM, 1, 0, 1, CYL_NONE, 128>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
        return launch_xj_pair<FLIM, 1, 0, 1>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
    }
    if (dir == 2) {
        if (n == 512) return launch_xj_pair<FLIM, 2, 512, 2>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
        if (n == 256) return launch_xj_pair<FLIM, 2, 256, 2>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
        if (n > 128)
            return launch_xj_pair<FLIM, 2, 0, 2, CYL_NONE, 256>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
        if (n > 64 && n < 128)
            return launch_xj_pair<FLIM, 2, 0, 2, CYL_NONE, 128>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
        return launch_xj_pair<FLIM, 2, 0, 2>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
    }
    if (n == 512) return launch_xj_pair<FLIM, 3, 512, 2>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
    if (n == 256) return launch_xj_pair<FLIM, 3, 256, 2>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
    if (n > 128) return launch_xj_pair<FLIM, 3, 0, 2, CYL_NONE, 256>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
    if (n > 64 && n < 128)
        return launch_xj_pair<FLIM, 3, 0, 2, CYL_NONE, 128>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
    return launch_xj_pair<FLIM, 3, 0, 2>(q, slab, grid, lambda, gamma, rho_min, mintemp, st);
}

int launch_xj_sweep(int flim, int dir, double *q, int64_t slab, const int grid[3], DevScalar lambda, double gamma,
                    double rho_min, cudaStream_t st, const CylSweep *cyl)
{
    const int geo = cyl ? cyl->kind : CYL_NONE;
    const CylPencil cp = cyl ? cyl->pencil : CylPencil{0.0, 0.0, 0, 0};
    if ((geo == CYL_RADIAL && dir != 1) || ((geo == CYL_THETA_DIV || geo == CYL_THETA_LAM) && dir != 2))
        return IB_ERROR_INVALID_ARGS;
    // square grids: TMA pencil boxes for y/z pencils and x rows (IMOGEN_B200_XJPAIR=0: the pencil kernel)
    static const bool xj_pair = [] {
        const char *e = getenv("IMOGEN_B200_XJPAIR");
        return !(e && e[0] == '0');
    }();
    const bool long_pencils = grid[dir - 1] >= pair_min_cells();
    if (xj_pair && long_pencils && geo == CYL_NONE) {
        const double mt = 1e-5 / (gamma - 1);
        int rc;
        switch (flim) {
        case IB_FLUX_OSPRE: rc = launch_xj_pair_dir<IB_FLUX_OSPRE>(dir, q, slab, grid, lambda, gamma, rho_min, mt, st); break;
        case IB_FLUX_VANLEER: rc = launch_xj_pair_dir<IB_FLUX_VANLEER>(dir, q, slab, grid, lambda, gamma, rho_min, mt, st); break;
        case IB_FLUX_MINMOD: rc = launch_xj_pair_dir<IB_FLUX_MINMOD>(dir, q, slab, grid, lambda, gamma, rho_min, mt, st); break;
        case IB_FLUX_SUPERBEE: rc = launch_xj_pair_dir<IB_FLUX_SUPERBEE>(dir, q, slab, grid, lambda, gamma, rho_min, mt, st); break;
        default: rc = launch_xj_pair_dir<IB_FLUX_ZERO>(dir, q, slab, grid, lambda, gamma, rho_min, mt, st); break;
        }
        if (rc != IB_ERROR_NOIMPLEMENT) return rc;
    }
    if (xj_pair && long_pencils && dir == 2 && (geo == CYL_THETA_DIV || geo == CYL_THETA_LAM)) {
        const double mt = 1e-5 / (gamma - 1);
        int rc;
        switch (flim) {
        case IB_FLUX_OSPRE: rc = launch_xj_pair_theta<IB_FLUX_OSPRE>(geo, q, slab, grid, lambda, gamma, rho_min, mt, st, cp); break;
        case IB_FLUX_VANLEER: rc = launch_xj_pair_theta<IB_FLUX_VANLEER>(geo, q, slab, grid, lambda, gamma, rho_min, mt, st, cp); break;
        case IB_FLUX_MINMOD: rc = launch_xj_pair_theta<IB_FLUX_MINMOD>(geo, q, slab, grid, lambda, gamma, rho_min, mt, st, cp); break;
        case IB_FLUX_SUPERBEE: rc = launch_xj_pair_theta<IB_FLUX_SUPERBEE>(geo, q, slab, grid, lambda, gamma, rho_min, mt, st, cp); break;
        default: rc = launch_xj_pair_theta<IB_FLUX_ZERO>(geo, q, slab, grid, lambda, gamma, rho_min, mt, st, cp); break;
        }
        if (rc != IB_ERROR_NOIMPLEMENT) return rc;
    }
    const int n = grid[dir - 1];
    const int64_t N = (int64_t)grid[0] * grid[1] * grid[2];
    if (n > 2048) return IB_ERROR_NOIMPLEMENT;  // 1024 threads x 2 cells per pencil block
    const int64_t np = N / n;
    const double mintemp = 1e-5 / (gamma - 1);
    // y/z pencils: W adjacent pencils per block when nx allows it (IMOGEN_B200_XJW caps W)
    static const int xjw = [] {
        const char *e = getenv("IMOGEN_B200_XJW");
        return (e && e[0] >= '1' && e[0] <= '4') ? e[0] - '0' : 4;
    }();
    // Blocks of at most 512 threads run two or more per SM and measured faster than 1024-thread
    // blocks of wider runs (256^3: y 1.33 ms at W = 2 against 1.39 at W = 4; 128^3: W = 4 0.146 ms,
    // W = 8 0.171); W = 2 in a 1024-thread block still beats W = 1 (512 x 512 x 64, y: 1.55 / 1.78).
    int W = 1;
    if (dir > 1 && geo == CYL_NONE) {  // cylindrical theta sweeps: one pencil per block
        for (int w = 4; w >= 2; w >>= 1)
            if (w <= xjw && grid[0] % w == 0 && n * w <= 512) { W = w; break; }
        // pencils of 257-512 cells: 4 pencils of 2 cells a thread (full 32-byte runs) rather than 2
        // of one cell, both 1024 threads (512 x 512 x 64, y: 1.53 -> 1.32 ms; at 256 or fewer cells
        // the 2-cell form measured slower: 256^3 y 1.31 -> 1.37)
        if (W == 1 && xjw >= 4 && grid[0] % 4 == 0 && n * 4 <= 2048) W = 4;
        else if (W == 1 && xjw >= 2 && grid[0] % 2 == 0 && n * 2 <= 1024) W = 2;
    }
    const int CPT = (n * W > 1024) ? 2 : 1;
    const int rows = (n + CPT - 1) / CPT;
    const int nt = ((rows * W + 31) / 32) * 32;
    const size_t shm = (size_t)10 * n * W * sizeof(double);
    const size_t shm_cap = 227 * 1024 - 2048;  // opt-in limit minus the kernel's static shared memory
    if (shm > shm_cap) return IB_ERROR_NOIMPLEMENT;
    const unsigned nblk = (unsigned)(np / W);
#define IB_XJ_G(F, WW, CC, RR, GG)                                                                            \
    do {                                                                                                      \
        static bool attr_set = false;                                                                         \
        if (!attr_set) {                                                                                      \
            int rc_ = check_cuda(cudaFuncSetAttribute(xj_pencil_kernel<F, WW, CC, RR, GG>,                    \
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm_cap)); \
            if (rc_) return rc_;                                                                              \
            attr_set = true;                                                                                  \
        }                                                                                                     \
        xj_pencil_kernel<F, WW, CC, RR, GG><<<nblk, nt, shm, st>>>(q, slab, grid[0], grid[1], grid[2], dir,   \
                                                                   lambda, gamma, rho_min, mintemp, cp);      \
    } while (0)
#define IB_XJ(F, WW, CC, RR) IB_XJ_G(F, WW, CC, RR, CYL_NONE)
#define IB_XJ_W(F)                                                                    \
    do {                                                                              \
        if (geo == CYL_RADIAL) {                                                      \
            if (CPT == 2) IB_XJ_G(F, 1, 2, true, CYL_RADIAL);                         \
            else IB_XJ_G(F, 1, 1, true, CYL_RADIAL);                                  \
        } else if (geo == CYL_THETA_DIV) {                                            \
            if (CPT == 2) IB_XJ_G(F, 1, 2, false, CYL_THETA_DIV);                     \
            else IB_XJ_G(F, 1, 1, false, CYL_THETA_DIV);                              \
        } else if (geo == CYL_THETA_LAM) {                                            \
            if (CPT == 2) IB_XJ_G(F, 1, 2, false, CYL_THETA_LAM);                     \
            else IB_XJ_G(F, 1, 1, false, CYL_THETA_LAM);                              \
        } else if (W == 4 && CPT == 2) IB_XJ(F, 4, 2, true);                          \
        else if (W == 4) IB_XJ(F, 4, 1, false);                                       \
        else if (W == 2) IB_XJ(F, 2, 1, false);                                       \
        else if (CPT == 2 && dir == 1) IB_XJ(F, 1, 2, true);                          \
        else if (CPT == 2) IB_XJ(F, 1, 2, false);                                     \
        else if (dir == 1) IB_XJ(F, 1, 1, true);                                      \
        else IB_XJ(F, 1, 1, false);                                                   \
    } while (0)
    switch (flim) {
    case IB_FLUX_OSPRE: IB_XJ_W(IB_FLUX_OSPRE); break;
    case IB_FLUX_VANLEER: IB_XJ_W(IB_FLUX_VANLEER); break;
    case IB_FLUX_MINMOD: IB_XJ_W(IB_FLUX_MINMOD); break;
    case IB_FLUX_SUPERBEE: IB_XJ_W(IB_FLUX_SUPERBEE); break;
    default: IB_XJ_W(IB_FLUX_ZERO); break;
    }
#undef IB_XJ_W
#undef IB_XJ
#undef IB_XJ_G
    return check_launch();
}

}  // namespace ib
