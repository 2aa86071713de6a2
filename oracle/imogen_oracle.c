/*
 * imogen_oracle.c -- CPU oracle (test infrastructure) for the Imogen fluid-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY: called by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline as the checker; never by the product library.
 *
 * Every function restates the arithmetic of one reference kernel (imogenproject/gpuImogen,
 * paths relative to that project) in the reference's own evaluation order, so that with
 * -ffp-contract=off the results are the same IEEE operations the reference performs (the
 * reference kernels are SIMT FP64; their per-thread expressions are reproduced here per cell).
 * The transposes the reference performs between sweeps (cudaArrayRotateB.cu) only move data,
 * so the oracle sweeps each pencil in place with the matching stride instead.
 *
 * Pinned: tests/test_golden_cpu.py checks this oracle bit for bit against golden vectors made by
 * the reference's own kernels compiled with -fmad=false (tests/golden/make_golden.py,
 * oracle/ref_harness/) for HLL, HLLC and Xin-Jin fluid steps, the CFL timestep and the LogTrap
 * drag integrators.
 */
#include "imogen_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_OK 0
#define OR_ERR_INVALID 1
#define OR_ERR_NOIMPL 2

/* ------------------------------------------------------------------------------------------
 * Limiters (gpuclass/limiter_functions.h:11-119).  Slope limiters return HALF the limited
 * difference (projection from cell centre to face).
 * ---------------------------------------------------------------------------------------- */
static double slope_ospre(double A, double B)          /* limiter_functions.h:87-95 */
{
    double R = A * B;
    if (R > 0) {
        double S = A + B;
        return .75 * R * S / (S * S - R);
    }
    return 0.0;
}

static double slope_mc(double A, double B)             /* limiter_functions.h:105-115 */
{
    if (A * B <= 0) return 0;
    double R = B / A;
    double S = .25 + .25 * R;
    S = (S < R) ? S : R;
    S = (S < 1) ? S : 1.0;
    return S * A;
}

static double slope_vanleer(double A, double B)        /* limiter_functions.h:54-61 */
{
    double r = A * B;
    if (r > 0.0) return r / (A + B);
    return 0;
}

static double slope_minmod(double A, double B)         /* limiter_functions.h:71-77 */
{
    /* the FP64 build declares this limiter with a float return type: the half slope is
     * rounded to single precision on return */
    if (A * B < 0) return 0.0;
    if (fabs(A) > fabs(B)) return (double)(float)(.5 * B);
    return (double)(float)(.5 * A);
}

static double flux_minmod(double A, double B)          /* limiter_functions.h:21-26 */
{
    if (A * B < 0) return 0.0;
    if (fabs(A) > fabs(B)) return B;
    return A;
}

static double slope_superbee(double A, double B)       /* limiter_functions.h:80-86 */
{
    if (A * B < 0) return 0.0;
    if (B < A) return flux_minmod(A, 2 * B);
    return .5 * flux_minmod(2 * A, B);
}

static double slope_vanalbada(double A, double B)      /* limiter_functions.h:97-102 */
{
    double R = A * B;
    if (R < 0) return 0;
    return .5 * R * (A + B) / (A * A + B * B);
}

static double slope_apply(int which, double A, double B)
{
    switch (which) {
    case OR_SLOPE_OSPRE: return slope_ospre(A, B);
    case OR_SLOPE_MC: return slope_mc(A, B);
    case OR_SLOPE_VANLEER: return slope_vanleer(A, B);
    case OR_SLOPE_MINMOD: return slope_minmod(A, B);
    case OR_SLOPE_SUPERBEE: return slope_superbee(A, B);
    case OR_SLOPE_VANALBADA: return slope_vanalbada(A, B);
    default: return 0.0;
    }
}

static double flux_ospre(double A, double B)           /* limiter_functions.h:36-42 */
{
    double r = A * B;
    if (r <= 0.0) return 0.0;
    return 1.5 * r * (A + B) / (A * A + r + B * B);
}

static double flux_vanleer(double A, double B)         /* limiter_functions.h:11-19 */
{
    double r = 2.0 * A * B;
    if (r > 0.0) return r / (A + B);
    return 0;
}

static double flux_superbee(double A, double B)        /* limiter_functions.h:28-34 */
{
    if (A * B < 0) return 0.0;
    if (B < A) return flux_minmod(A, 2 * B);
    return flux_minmod(2 * A, B);
}

static double flux_apply(int which, double A, double B)
{
    switch (which) {
    case OR_FLUX_OSPRE: return flux_ospre(A, B);
    case OR_FLUX_VANLEER: return flux_vanleer(A, B);
    case OR_FLUX_MINMOD: return flux_minmod(A, B);
    case OR_FLUX_SUPERBEE: return flux_superbee(A, B);
    default: return 0.0;
    }
}

/* ------------------------------------------------------------------------------------------
 * Constants uploaded per sweep (cudaFluidStep.cu:289-311)
 * ---------------------------------------------------------------------------------------- */
typedef struct {
    double gamma, gm1, minmass, mintemp, govergm1, isotemp, isotempsq;
} fconst;

static fconst make_consts(const or_step *p)
{
    fconst c;
    c.gamma = p->gamma;
    c.gm1 = p->gamma - 1.0;
    c.minmass = p->rho_min;
    c.mintemp = 1e-5 / (p->gamma - 1);       /* cudaFluidStep.cu:298 */
    c.govergm1 = p->gamma / (p->gamma - 1.0);
    c.isotemp = p->c_iso;
    c.isotempsq = p->c_iso * p->c_iso;
    return c;
}

typedef struct { double vl, vr; } bounds2;

/* computeEinfeldtBounds (cudaFluidStep.cu:1728-1755) */
static bounds2 einfeldt(const fconst *c, double rhoL, double vL, double PL, double rhoR,
                        double vR, double PR, double dvsq)
{
    double csql = c->gamma * PL / rhoL;
    double csqr = c->gamma * PR / rhoR;
    double Fa = sqrt(rhoR / rhoL);
    double Fb = 1.0 / (1.0 + Fa);
    double Croe = ((csql + Fa * csqr) + .5 * c->gm1 * dvsq * Fa * Fb) * Fb;
    bounds2 sb;
    double Vroe = (vL + Fa * vR) * Fb;
    Croe = Vroe - sqrt(Croe);
    sb.vl = vL - sqrt(csql);
    sb.vr = vR + sqrt(csqr);
    sb.vl = (Croe < sb.vl) ? Croe : sb.vl;
    Croe = 2 * Vroe - Croe;
    sb.vr = (Croe > sb.vr) ? Croe : sb.vr;
    return sb;
}

/* computeEinfeldtBounds_isothermal (cudaFluidStep.cu:1780-1799) */
static bounds2 einfeldt_iso(double rhoL, double vL, double rhoR, double vR, double cs)
{
    double Fa = sqrt(rhoR / rhoL);
    double Fb = 1.0 / (1.0 + Fa);
    bounds2 sb;
    double Vroe = (vL + Fa * vR) * Fb;
    cs = Vroe - cs;
    sb.vl = vL - cs;
    sb.vr = vR + cs;
    sb.vl = (cs < sb.vl) ? cs : sb.vl;
    cs = 2 * Vroe - cs;
    sb.vr = (cs > sb.vr) ? cs : sb.vr;
    return sb;
}

/* Row buffers: a pencil is gathered into local order [rho, E, p_normal, p_t1, p_t2]. */
typedef struct {
    int n;
    double *u[5];    /* conserved, local order */
    double *w[5];    /* scratch */
    double *edge[10];
    double *flux[5];
    double *tmp[5];
} rowbuf;

static void rowbuf_alloc(rowbuf *r, int n)
{
    int k;
    double *blk = (double *)malloc(sizeof(double) * (size_t)n * 30);
    r->n = n;
    for (k = 0; k < 5; k++) r->u[k] = blk + (size_t)n * k;
    for (k = 0; k < 5; k++) r->w[k] = blk + (size_t)n * (5 + k);
    for (k = 0; k < 10; k++) r->edge[k] = blk + (size_t)n * (10 + k);
    for (k = 0; k < 5; k++) r->flux[k] = blk + (size_t)n * (20 + k);
    for (k = 0; k < 5; k++) r->tmp[k] = blk + (size_t)n * (25 + k);
}

static void rowbuf_free(rowbuf *r) { free(r->u[0]); }

static inline int wrap(int i, int n) { return (i < 0) ? i + n : ((i >= n) ? i - n : i); }

/* Cylindrical geometry of one pencil.  kind: 0 square (or the z sweep), 1 radial sweep (the
 * face-area factors and the geometric pressure term), 2 theta sweep with the flux difference
 * divided by r (FLUX_THETA_213), 3 theta sweep with lambda divided by r first (FLUX_THETA_231).
 * Radial cell i has its centre at rin + i dr; r is a theta pencil's radius. */
typedef struct {
    int kind;
    double rin, dr;
    double r;
} rowgeo;

static const rowgeo ROWGEO_SQUARE = {0, 0.0, 0.0, 0.0};

/* Radius the reference's theta kernels compute for the pencil at radial index j (layout
 * theta,r,z): thread row ty = j mod 4 starts at ty dr + rin and every pass of the block's row
 * loop adds 4 dr (YBLOCKS = 4; cudaFluidStep.cu:848-850, 1112-1116, 1844-1846, 2462-2464). */
static double theta_radius_213(int j, double rin, double dr)
{
    double r = (double)(j % 4) * dr + rin;
    int m;
    for (m = 0; m < j / 4; m++) r = r + 4.0 * dr;
    return r;
}

/* ------------------------------------------------------------------------------------------
 * HLLC, 2nd order MUSCL (cukern_HLLC_2ndorder, cudaFluidStep.cu:1124-1463), one stage.
 * in[5]: conserved state of the row (local order).  flux[k][i] = flux through face i+1/2.
 * ---------------------------------------------------------------------------------------- */
static void hllc_row_flux(rowbuf *r, double *const in[5], const fconst *c, int slope)
{
    int n = r->n, i, k;
    /* primitive variables: rho, e_int, vx, vy, vz (cudaFluidStep.cu:1200-1237) */
    for (i = 0; i < n; i++) {
        double A = in[0][i], B = in[1][i], C = in[2][i], D = in[3][i], E = in[4][i];
        double F = 1.0 / A;
        B -= .5 * (C * C + D * D + E * E) * F;
        C *= F;
        D *= F;
        E *= F;
        r->w[0][i] = A; r->w[1][i] = B; r->w[2][i] = C; r->w[3][i] = D; r->w[4][i] = E;
    }
    /* backward difference, limited half slope, face states (cudaFluidStep.cu:1287-1310) */
    for (k = 0; k < 5; k++) {
        double *v = r->w[k];
        for (i = 0; i < n; i++) {
            double dl = v[i] - v[wrap(i - 1, n)];
            double dr = v[wrap(i + 1, n)] - v[i];
            double s = slope_apply(slope, dl, dr);
            if (k == 1) {
                r->edge[2][i] = c->gm1 * (v[i] - s);  /* pressure, left face  (BOS2) */
                r->edge[3][i] = c->gm1 * (v[i] + s);  /* pressure, right face (BOS3) */
            } else {
                r->edge[2 * k][i] = v[i] - s;
                r->edge[2 * k + 1][i] = v[i] + s;
            }
        }
    }
    /* Riemann problem at face i+1/2 between cell i (right face) and i+1 (left face) */
    for (i = 0; i < n; i++) {
        int ir = wrap(i + 1, n);
        double rhoL = r->edge[1][i], PL = r->edge[3][i], vxL = r->edge[5][i];
        double vyL = r->edge[7][i], vzL = r->edge[9][i];
        double rhoR = r->edge[0][ir], PR = r->edge[2][ir], vxR = r->edge[4][ir];
        double vyR = r->edge[6][ir], vzR = r->edge[8][ir];
        double A, B, C, D, E, F, G, H;
        int mode;
        double fr, fe, fpx, fpy, fpz;

        C = vxL - vxR;
        D = vyL - vyR;
        E = vzL - vzR;
        C = C * C + D * D + E * E;
        bounds2 sb = einfeldt(c, rhoL, vxL, PL, rhoR, vxR, PR, C);
        C = sb.vl;
        D = sb.vr;
        A = vxL;
        B = vxR;
        A = rhoL * (C - A);
        B = rhoR * (D - B);
        E = (B * vxR - PR - A * vxL + PL) / (B - A);  /* Batten et al. eq. 34 */

        if (E > 0) mode = (C > 0) ? 0 : 2;
        else mode = (D > 0) ? 3 : 1;

        switch (mode) {
        case 0:
            A = rhoL; B = vxL; C = vyL; D = vzL;
            E = .5 * (B * B + C * C + D * D) * A;
            F = PL;
            A *= B;
            C *= A;
            D *= A;
            G = A * B + F;
            B *= (E + c->govergm1 * F);
            fr = A; fe = B; fpx = G; fpy = C; fpz = D;
            break;
        case 2:
            A = rhoL; B = vxL;
            D = A * (C - B) / (C - E);
            F = vyL; H = vzL;
            G = .5 * (B * B + F * F + H * H);
            A = D * E;
            F *= A;
            H *= A;
            C *= (E - B);
            B = PL + D * (C + E * B);
            G = D * E * (c->govergm1 * PL / rhoL + G + C);
            fr = A; fe = G; fpx = B; fpy = F; fpz = H;
            break;
        case 3:
            A = rhoR; B = vxR;
            C = A * (D - B) / (D - E);
            F = vyR; H = vzR;
            G = .5 * (B * B + F * F + H * H);
            A = C * E;
            F *= A;
            H *= A;
            D *= (E - B);
            B = PR + C * (D + E * B);
            G = C * E * (c->govergm1 * PR / rhoR + G + D);
            fr = A; fe = G; fpx = B; fpy = F; fpz = H;
            break;
        default: /* case 1 */
            A = rhoR; B = vxR; C = vyR; D = vzR;
            E = .5 * (B * B + C * C + D * D) * A;
            F = PR;
            A *= B;
            C *= A;
            D *= A;
            G = A * B + F;
            B *= (E + c->govergm1 * F);
            fr = A; fe = B; fpx = G; fpy = C; fpz = D;
            break;
        }
        r->flux[0][i] = fr; r->flux[1][i] = fe; r->flux[2][i] = fpx;
        r->flux[3][i] = fpy; r->flux[4][i] = fpz;
    }
}

/* lambda times the flux difference of cell i, component k, after hllc_row_flux.  Radial
 * sweeps weight the faces by their radii and add the cell's mean face pressure to the radial
 * momentum (cylgeomA/B/C, cudaFluidStep.cu:1164-1171, 1488-1495); theta sweeps divide by r
 * (1499-1505) or use lambda / r (1506-1512). */
static double hllc_dflux(const rowbuf *r, const rowgeo *G, double lam, int k, int i)
{
    const int il = wrap(i - 1, r->n);
    const double fr = r->flux[k][i], fl = r->flux[k][il];
    if (G->kind == 1) {
        double R = G->rin + i * G->dr;
        double cA = (R - .5 * G->dr) / (R);
        double cB = (R + .5 * G->dr) / (R);
        double cC = 0.5 * G->dr / R;
        double d = cB * fr - cA * fl;
        if (k == 2) d = d - cC * (r->edge[2][i] + r->edge[3][i]);
        return lam * d;
    }
    if (G->kind == 2) return lam * (fr - fl) / G->r;
    return lam * (fr - fl);
}

/* SSPRK2 with HLLC (cudaFluidStep.cu:1510-1559 stage A, 1560-1600 stage B) */
static void hllc_row_sweep(rowbuf *r, const fconst *c, int slope, double lambda, const rowgeo *G)
{
    int n = r->n, i, k;
    double lam = lambda;
    if (G->kind == 3) lam /= G->r;
    hllc_row_flux(r, r->u, c, slope);
    for (k = 0; k < 5; k++)
        for (i = 0; i < n; i++)
            r->tmp[k][i] = r->u[k][i] - hllc_dflux(r, G, lam, k, i);
    hllc_row_flux(r, r->tmp, c, slope);
    for (k = 0; k < 5; k++)
        for (i = 0; i < n; i++)
            r->u[k][i] = .5 * (r->tmp[k][i] + r->u[k][i] - hllc_dflux(r, G, lam, k, i));
}

/* ------------------------------------------------------------------------------------------
 * HLL (cukern_HLL_step, cudaFluidStep.cu:1801-2422) and its pressure solver
 * (cukern_PressureSolverHydro, cudaFluidStep.cu:2813-2864).
 * ---------------------------------------------------------------------------------------- */
/* Floors rho and e_int of state s in place (local row order is fine: the solver is
 * symmetric in the momenta) and returns the gas pressure into P.  The reference sums the
 * squared momenta in memory-slab order px, py, pz; mom_order gives which local index holds
 * slab 2, 3, 4. */
static void hll_pressure_row(double *const s[5], double *P, int n, const fconst *c,
                             const int mom_order[3])
{
    int i;
    for (i = 0; i < n; i++) {
        double rho = s[0][i], E, z, momsq, p;
        if (rho < c->minmass) {
            p = c->minmass / rho;
            rho = s[0][i] = c->minmass;
            E = s[1][i] = p * s[1][i];
            z = s[mom_order[0]][i] = p * s[mom_order[0]][i];
            momsq = z * z;
            z = s[mom_order[1]][i] = p * s[mom_order[1]][i];
            momsq += z * z;
            z = s[mom_order[2]][i] = p * s[mom_order[2]][i];
            momsq += z * z;
        } else {
            E = s[1][i];
            z = s[mom_order[0]][i];
            momsq = z * z;
            z = s[mom_order[1]][i];
            momsq += z * z;
            z = s[mom_order[2]][i];
            momsq += z * z;
        }
        p = E - .5 * momsq / rho;
        if (p < rho * c->mintemp) {
            p = c->mintemp * rho;
            s[1][i] = (.5 * momsq / rho) + p;
            P[i] = p * c->gm1;
        } else {
            P[i] = p * c->gm1;
        }
    }
}

static void hll_row_flux(rowbuf *r, double *const in[5], const double *P, const fconst *c,
                         int slope)
{
    int n = r->n, i, k;
    /* primitives rho, v_n, P, v_t1, v_t2 -> w[0..4] (cudaFluidStep.cu:1864-1888) */
    for (i = 0; i < n; i++) {
        double Ale = in[0][i];
        r->w[0][i] = Ale;
        r->w[1][i] = in[2][i] / Ale;
        r->w[2][i] = P[i];
        r->w[3][i] = in[3][i] / Ale;
        r->w[4][i] = in[4][i] / Ale;
    }
    /* slopes, left/right faces (cudaFluidStep.cu:1935-1959) */
    for (k = 0; k < 5; k++) {
        double *v = r->w[k];
        for (i = 0; i < n; i++) {
            double bd = v[i] - v[wrap(i - 1, n)];
            double bdr = v[wrap(i + 1, n)] - v[i];
            double Fa = slope_apply(slope, bd, bdr);
            r->edge[2 * k + 1][i] = v[i] + Fa;  /* right face */
            r->edge[2 * k][i] = v[i] - Fa;      /* left face  */
        }
    }
    for (i = 0; i < n; i++) {
        int ir = wrap(i + 1, n);
        /* Xle = right face of cell i, Xre = left face of cell i+1 (cudaFluidStep.cu:2049-2055) */
        double Ale = r->edge[1][i], Ble = r->edge[3][i], Cle = r->edge[5][i];
        double Dle = r->edge[7][i], Ele = r->edge[9][i];
        double Are = r->edge[0][ir], Bre = r->edge[2][ir], Cre = r->edge[4][ir];
        double Dre = r->edge[6][ir], Ere = r->edge[8][ir];
        double Utilde = (Bre - Ble), Sleft = (Dre - Dle), Sright = (Ere - Ele);
        double Atilde, Fa, Fb;
        double f0, f1, f2, f3, f4;
        bounds2 sb;
        int mode;
        if (c->isotemp == -1) {
            sb = einfeldt(c, Ale, Ble, Cle, Are, Bre, Cre,
                          Utilde * Utilde + Sleft * Sleft + Sright * Sright);
        } else {
            /* the isothermal bound is handed c_iso^2 where a speed is expected
             * (cudaFluidStep.cu:2131) */
            sb = einfeldt_iso(Ale, Ble, Are, Bre, c->isotempsq);
        }
        Sleft = sb.vl;
        Sright = sb.vr;
        Atilde = 1 / (Sright - Sleft);
        Fa = Ale * Ble;
        Fb = Are * Bre;
        mode = 1;
        if (Sleft >= 0) mode = 0;
        if (Sright <= 0) mode = 2;
        switch (mode) {
        case 0:
            f0 = Fa;
            if (c->isotemp == -1) {
                f1 = Ble * (c->govergm1 * Cle + .5 * Ale * (Ble * Ble + Dle * Dle + Ele * Ele));
                f2 = Fa * Ble + Cle;
            } else {
                f1 = Ble * (Cle + .5 * Ale * (Ble * Ble + Dle * Dle + Ele * Ele));
                f2 = Fa * Ble + c->isotempsq * Ale;
            }
            f3 = Fa * Dle;
            f4 = Fa * Ele;
            break;
        case 1:
            f0 = (Sright * (Ble - Sleft) * Ale - Sleft * (Bre - Sright) * Are) * Atilde;
            if (c->isotemp == -1) {
                f2 = (Sright * (Ble - Sleft) * Fa - Sleft * (Bre - Sright) * Fb + Sright * Cle -
                      Sleft * Cre) * Atilde;
            } else {
                f2 = (Sright * (Ble - Sleft) * Fa - Sleft * (Bre - Sright) * Fb +
                      c->isotempsq * (Sright * Ale - Sleft * Are)) * Atilde;
            }
            f3 = (Sright * (Ble - Sleft) * Ale * Dle - Sleft * (Bre - Sright) * Are * Dre) * Atilde;
            f4 = (Sright * (Ble - Sleft) * Ale * Ele - Sleft * (Bre - Sright) * Are * Ere) * Atilde;
            if (c->isotemp == -1) {
                Fa = .5 * Ale * (Ble * Ble + Dle * Dle + Ele * Ele);
                Fb = .5 * Are * (Bre * Bre + Dre * Dre + Ere * Ere);
                f1 = (Sright * (Ble - Sleft) * Fa - Sleft * (Bre - Sright) * Fb);
                f1 = (f1 + (c->govergm1 * (Sright * Cle * Ble - Sleft * Cre * Bre) +
                            Sleft * Sright * (Cre - Cle) / c->gm1)) * Atilde;
            } else {
                /* isothermal energy flux is left without the 1/(S_R-S_L) factor
                 * (cudaFluidStep.cu:2178-2182) */
                Fa = .5 * Ale * (Ble * Ble + Dle * Dle + Ele * Ele) + Cle;
                Fb = .5 * Are * (Bre * Bre + Dre * Dre + Ere * Ere) + Cre;
                f1 = (Sright * (Ble - Sleft) * Fa - Sleft * (Bre - Sright) * Fb);
            }
            break;
        default:
            f0 = Fb;
            if (c->isotemp == -1) {
                f1 = Bre * (c->govergm1 * Cre + .5 * Are * (Bre * Bre + Dre * Dre + Ere * Ere));
                f2 = Fb * Bre + Cre;
            } else {
                f1 = Bre * (Cre + .5 * Are * (Bre * Bre + Dre * Dre + Ere * Ere));
                /* c_iso, not c_iso^2 (cudaFluidStep.cu:2191) */
                f2 = Fb * Bre + c->isotemp * Are;
            }
            f3 = Fb * Dre;
            f4 = Fb * Ere;
            break;
        }
        r->flux[0][i] = f0; r->flux[1][i] = f1; r->flux[2][i] = f2;
        r->flux[3][i] = f3; r->flux[4][i] = f4;
    }
}

/* The flux difference of cell i, component k, after hll_row_flux, as the HLL kernel subtracts
 * it.  Radial sweeps take the radius factors with lambda folded in (cudaFluidStep.cu:1837-1842)
 * and add the geometric pressure term to the radial momentum: the stage input's pressure from
 * the pressure solver, or for an isothermal fluid rho c^2 with rho the density of the predicted
 * state (Qstore[0], which the predictor has just written; 2270-2290, 2371-2391).  Theta sweeps
 * divide by r or use lambda / r (2293-2305, 2255-2268). */
static double hll_dflux(const rowbuf *r, const rowgeo *G, const fconst *c, double lam, const double *P,
                        double *const U1[5], int k, int i)
{
    const int il = wrap(i - 1, r->n);
    const double fr = r->flux[k][i], fl = r->flux[k][il];
    if (G->kind == 1) {
        double Fa = G->rin + i * G->dr;
        double cA = lam * (Fa - .5 * G->dr) / (Fa);
        double cB = lam * (Fa + .5 * G->dr) / (Fa);
        double cC = lam * G->dr / Fa;
        double d = cB * fr - cA * fl;
        if (k == 2) {
            if (c->isotemp == -1) d = d - P[i] * cC;
            else d = d - U1[0][i] * c->isotempsq * cC;
        }
        return d;
    }
    if (G->kind == 2) return lam * (fr - fl) / G->r;
    return lam * (fr - fl);
}

static void hll_row_sweep(rowbuf *r, const fconst *c, int slope, double lambda,
                          const int mom_order[3], const rowgeo *G)
{
    int n = r->n, i, k;
    double *Pcopy = (double *)malloc(sizeof(double) * (size_t)n);
    double *U1[5];
    double *blk = (double *)malloc(sizeof(double) * (size_t)n * 5);
    double lam = lambda;
    if (G->kind == 3) lam /= G->r;
    for (k = 0; k < 5; k++) U1[k] = blk + (size_t)n * k;
    /* pressure + floors on the fluid, predictor (PCswitch RK_PREDICT, SSPRK); the density
     * (k = 0) is written first, as the isothermal radial term reads it */
    hll_pressure_row(r->u, Pcopy, n, c, mom_order);
    hll_row_flux(r, r->u, Pcopy, c, slope);
    for (k = 0; k < 5; k++)
        for (i = 0; i < n; i++)
            U1[k][i] = r->u[k][i] - hll_dflux(r, G, c, lam, Pcopy, U1, k, i);
    /* pressure + floors on the predicted state, corrector */
    hll_pressure_row(U1, Pcopy, n, c, mom_order);
    hll_row_flux(r, U1, Pcopy, c, slope);
    for (k = 0; k < 5; k++)
        for (i = 0; i < n; i++)
            r->u[k][i] = .5 * (r->u[k][i] + U1[k][i] - hll_dflux(r, G, c, lam, Pcopy, U1, k, i));
    free(blk);
    free(Pcopy);
}

/* ------------------------------------------------------------------------------------------
 * Xin-Jin relaxing TVD (cukern_XinJinHydro_step, cudaFluidStep.cu:2427-2654) with the
 * per-row freezing speed of cukern_PressureFreezeSolverHydro (cudaFluidStep.cu:2867-2941).
 * The XJ kernel works in memory slab order; `nslot` is the slab of the normal momentum.
 * mem[k] = local index that holds memory slab k.
 * ---------------------------------------------------------------------------------------- */
static double xj_freeze(double *const s[5], int n, const fconst *c, const int mem[5])
{
    /* Uses memory slab 2 (p_x) as the normal momentum whatever the sweep direction, as the
     * reference kernel does.  Max of |px|/rho + c_s over the row, NaNs never win. */
    int i;
    double cmax = 0.0;
    for (i = 0; i < n; i++) {
        double invrho = 1.0 / s[mem[0]][i];
        double psq = s[mem[3]][i];
        double px = s[mem[4]][i];
        double P, locCf;
        psq = psq * psq + px * px;
        px = s[mem[2]][i];
        psq += px * px;
        P = (s[mem[1]][i] - .5 * psq * invrho) * c->gm1;
        locCf = fabs(px) * invrho + sqrt(c->gamma * P * invrho);
        cmax = (locCf > cmax) ? locCf : cmax;
    }
    return cmax;
}

static void xj_stage(double *const Qin[5], double *const Qbase[5], double *const Qout[5],
                     int n, const fconst *c, double Cf, double lambda, int corrector,
                     int nslot, int flim, rowbuf *r, const rowgeo *G)
{
    /* Qin: state the fluxes are built from; Qbase: state that is updated (corrector) */
    int i, k;
    double *P = r->tmp[0], *vx = r->tmp[1];
    double *L = r->w[0], *R = r->w[1], *dL = r->w[2], *dR = r->w[3];
    double *prop[5];
    for (k = 0; k < 5; k++) prop[k] = r->edge[k];
    for (i = 0; i < n; i++) {
        double q0 = Qin[0][i], q1 = Qin[1][i], q2 = Qin[2][i], q3 = Qin[3][i], q4 = Qin[4][i];
        P[i] = c->gm1 * (q1 - .5 * (q4 * q4 + q3 * q3 + q2 * q2) / q0);
        vx[i] = Qin[nslot][i] / q0;
    }
    for (k = 0; k < 5; k++) {
        for (i = 0; i < n; i++) {
            double w;
            double *q = Qin[k];
            if (k == 0) w = Qin[nslot][i];
            else if (k == 1) w = vx[i] * (q[i] + P[i]);
            else if (k == nslot) w = vx[i] * q[i] + P[i];
            else w = vx[i] * q[i];
            L[i] = (Cf * q[i] - w);   /* left-going  */
            R[i] = (Cf * q[i] + w);   /* right-going */
        }
        if (corrector) {
            for (i = 0; i < n; i++) {
                dL[i] = 0.5 * (L[i] - L[wrap(i - 1, n)]);
                dR[i] = 0.5 * (R[i] - R[wrap(i - 1, n)]);
            }
            /* limited corrections use the unmodified backward differences of the
             * neighbour, so compute into scratch first */
            for (i = 0; i < n; i++) {
                r->edge[5][i] = L[i] - flux_apply(flim, dL[i], dL[wrap(i + 1, n)]);
                r->edge[6][i] = R[i] + flux_apply(flim, dR[i], dR[wrap(i + 1, n)]);
            }
            for (i = 0; i < n; i++) { L[i] = r->edge[5][i]; R[i] = r->edge[6][i]; }
        }
        for (i = 0; i < n; i++) {
            int il = wrap(i - 1, n), ir = wrap(i + 1, n);
            double base = corrector ? Qbase[k][i] : Qin[k][i];
            if (G->kind == 1) {
                /* radial: face radii, and 2 dr / r times the cell pressure on p_r, the 2
                 * undoing the halved lambda (cudaFluidStep.cu:2463-2470, 2576-2581, 2603-2607) */
                double Rc = G->rin + i * G->dr;
                double cA = (Rc - .5 * G->dr) / (Rc);
                double cB = (Rc + .5 * G->dr) / (Rc);
                double cC = 2.0 * G->dr / Rc;
                prop[k][i] = base - lambda * (cB * R[i] - cA * R[il] - cB * L[ir] + cA * L[i]);
                if (k == 2) prop[k][i] += lambda * cC * P[i];
            } else if (G->kind == 2) {
                prop[k][i] = base - lambda * (R[i] - R[il] - L[ir] + L[i]) / G->r;
            } else {
                prop[k][i] = base - lambda * (R[i] - R[il] - L[ir] + L[i]);
            }
        }
    }
    for (i = 0; i < n; i++) {
        double p0 = prop[0][i], p1 = prop[1][i], p2 = prop[2][i], p3 = prop[3][i], p4 = prop[4][i];
        double w;
        p0 = (p0 < c->minmass) ? c->minmass : p0;
        w = .5 * (p2 * p2 + p3 * p3 + p4 * p4) / p0;
        if ((p1 - w) < p0 * c->mintemp) p1 = w + p0 * c->mintemp;
        Qout[0][i] = p0; Qout[1][i] = p1; Qout[2][i] = p2; Qout[3][i] = p3; Qout[4][i] = p4;
    }
}

static void xj_row_sweep(rowbuf *r, const fconst *c, int flim, double lambda, int dir, const rowgeo *G)
{
    /* r->u holds the row in memory slab order for XJ; the theta form with lambda / r divides
     * each stage's lambda (0.25 and 0.5 of the sweep's) by r (cudaFluidStep.cu:2478-2480) */
    int n = r->n, k;
    int mem[5] = {0, 1, 2, 3, 4};
    int nslot = 1 + dir;
    double *U1[5];
    double *blk = (double *)malloc(sizeof(double) * (size_t)n * 5);
    double Cf, la = 0.25 * lambda, lb = 0.5 * lambda;
    if (G->kind == 3) {
        la /= G->r;
        lb /= G->r;
    }
    for (k = 0; k < 5; k++) U1[k] = blk + (size_t)n * k;
    Cf = xj_freeze(r->u, n, c, mem);
    xj_stage(r->u, r->u, U1, n, c, Cf, la, 0, nslot, flim, r, G);
    Cf = xj_freeze(U1, n, c, mem);
    xj_stage(U1, r->u, r->u, n, c, Cf, lb, 1, nslot, flim, r, G);
    free(blk);
}

/* ------------------------------------------------------------------------------------------
 * Sweep driver: gather each pencil along dir, run the row scheme, scatter back.
 * ---------------------------------------------------------------------------------------- */
static void pencil_geometry(const or_grid *g, int dir, int *n, long *stride, long *npencil)
{
    long N = (long)g->nx * g->ny * g->nz;
    if (dir == 1) { *n = g->nx; *stride = 1; }
    else if (dir == 2) { *n = g->ny; *stride = g->nx; }
    else { *n = g->nz; *stride = (long)g->nx * g->ny; }
    *npencil = N / *n;
}

static long pencil_base(const or_grid *g, int dir, long p)
{
    if (dir == 1) return p * g->nx;
    if (dir == 2) {
        long x = p % g->nx, z = p / g->nx;
        return x + (long)g->nx * g->ny * z;
    }
    return p;  /* dir 3: pencils indexed by x + nx*y */
}

/* Geometry of pencil pp of a sweep along dir (see rowgeo).  Theta pencils: with
 * OR_CYL_GEOMETRIC_RADIUS r = r_inner + i h[0] (i = radial index); otherwise the radius the
 * reference's kernels compute, whose radial step is the sweep direction's cell size h[1]
 * (gamHost[9], cudaFluidStep.cu:305-307, 340).  Layout theta,r,z: theta_radius_213 of the radial
 * index, or of the z index when nx = 1 < nz (the launch then treats z as the second dimension,
 * cudaFluidStep.cu:325-329).  Layout theta,z,r: i h[1] + r_inner from the block index, which is
 * always 0 when nz = 1 (the same reshaping), so every such pencil gets r_inner. */
static rowgeo pencil_rowgeo(const or_grid *g, const or_step *p, int dir, long pp)
{
    rowgeo G = ROWGEO_SQUARE;
    if (p->geometry != OR_GEO_CYLINDRICAL || dir == 3) return G;
    if (dir == 1) {
        G.kind = 1;
        G.rin = p->r_inner;
        G.dr = p->h[0];
        return G;
    }
    {
        const int i = (int)(pp % g->nx), kz = (int)(pp / g->nx);
        G.kind = (p->theta_form == OR_THETA_231) ? 3 : 2;
        if (p->cyl_flags & OR_CYL_GEOMETRIC_RADIUS) G.r = p->r_inner + i * p->h[0];
        else if (p->theta_form == OR_THETA_231) G.r = (g->nz == 1 ? 0 : i) * p->h[1] + p->r_inner;
        else G.r = theta_radius_213((g->nx == 1 && g->nz > 1) ? kz : i, p->r_inner, p->h[1]);
    }
    return G;
}

int or_theta_form(int sweep_dir, int step_number)
{
    const int sweep = (step_number + 3 * (sweep_dir > 0)) % 6;
    return (sweep == 0 || sweep == 5) ? OR_THETA_231 : OR_THETA_213;
}

int or_fluid_sweep(double *q, const or_grid *g, const or_step *p, int dir)
{
    int n;
    long stride, npencil;
    fconst c;
    double lambda;
    /* slab order that becomes local [rho, E, p_n, p_t1, p_t2] (cudaFluidStep.cu:1200-1219 for
     * HLLC, 1864-1882 for HLL); XJ keeps memory order */
    static const int hllc_map[3][5] = {{0, 1, 2, 3, 4}, {0, 1, 3, 2, 4}, {0, 1, 4, 3, 2}};
    static const int hll_map[3][5] = {{0, 1, 2, 3, 4}, {0, 1, 3, 2, 4}, {0, 1, 4, 2, 3}};
    const int *map;
    int mom_order[3];
    if (dir < 1 || dir > 3) return OR_ERR_INVALID;
    if (p->method < 1 || p->method > 3) return OR_ERR_INVALID;
    pencil_geometry(g, dir, &n, &stride, &npencil);
    if (n < 3) return OR_OK;  /* cudaFluidStep.cu:313 */
    c = make_consts(p);
    lambda = p->dt / p->h[dir - 1];
    map = (p->method == 2) ? hllc_map[dir - 1] : ((p->method == 1) ? hll_map[dir - 1] : hllc_map[0]);
    if (p->method == 3) map = hllc_map[0];
    {
        /* local index holding memory slabs 2, 3, 4 (pressure solver sums px, py, pz) */
        int k, m;
        for (m = 0; m < 3; m++)
            for (k = 0; k < 5; k++)
                if (map[k] == 2 + m) mom_order[m] = k;
    }

#pragma omp parallel
    {
        rowbuf r;
        long pp;
        rowbuf_alloc(&r, n);
#pragma omp for schedule(static)
        for (pp = 0; pp < npencil; pp++) {
            long b = pencil_base(g, dir, pp);
            int i, k;
            for (k = 0; k < 5; k++) {
                const double *s = q + (long)map[k] * g->slab + b;
                for (i = 0; i < n; i++) r.u[k][i] = s[(long)i * stride];
            }
            rowgeo G = pencil_rowgeo(g, p, dir, pp);
            if (p->method == 2) hllc_row_sweep(&r, &c, p->slope_limiter, lambda, &G);
            else if (p->method == 1) hll_row_sweep(&r, &c, p->slope_limiter, lambda, mom_order, &G);
            else xj_row_sweep(&r, &c, p->flux_limiter, lambda, dir, &G);
            for (k = 0; k < 5; k++) {
                double *s = q + (long)map[k] * g->slab + b;
                for (i = 0; i < n; i++) s[(long)i * stride] = r.u[k][i];
            }
        }
        rowbuf_free(&r);
    }
    return OR_OK;
}

/* ------------------------------------------------------------------------------------------
 * Boundary conditions along a pencil with the X-kernel semantics of cudaStatics.cu (used
 * inside the fluid step, where the swept direction is the fastest memory direction).
 * v[k] points at the first cell of the pencil in slab k; s = stride along the pencil.
 * ---------------------------------------------------------------------------------------- */
#define PV(k, i) v[k][(long)(i) * s]

static void bc_pencil_sas(double *v, long s, int n, int mode, int side, int anti, int depth)
{
    /* cukern_{x}{minus,plus}{Symmetrize,Antisymmetrize}, extrapolate{FlatConst,Linear}
     * (cudaStatics.cu:1305-1400).  MIRROR_OFFSET = 1. */
    int t;
    double f[4];
    if (mode == OR_BC_MIRROR) {
        for (t = 0; t < depth; t++) {
            if (side == 0) {
                double a = v[(long)(depth + 1 + t) * s];
                v[(long)(depth - 1 - t) * s] = anti ? -a : a;
            } else {
                double a = v[(long)(n - depth - 2 - t) * s];
                v[(long)(n - depth + t) * s] = anti ? -a : a;
            }
        }
    } else if (mode == OR_BC_CONST) {
        if (side == 0) {
            double a = v[(long)depth * s];
            for (t = 0; t < depth; t++) v[(long)t * s] = a;
        } else {
            double a = v[(long)(n - depth - 1) * s];
            for (t = 0; t < depth; t++) v[(long)(n - depth + t) * s] = a;
        }
    } else if (mode == OR_BC_LINEAR) {
        if (side == 0) {
            /* phi[t] = phi[depth] + (depth - t)*(phi[depth] - phi[depth+1]) */
            for (t = 0; t < 4; t++) f[t] = v[(long)(t + depth) * s];
            for (t = 0; t < depth; t++) v[(long)t * s] = v[(long)depth * s] + (double)(depth - t) * (f[0] - f[1]);
        } else {
            /* base = n-depth-1; phi[base+t+2] = f1 + (t+1)(f1-f0).  The reference also writes
             * one cell past the end of the pencil (t = depth-1); that write is dropped. */
            long b = n - depth - 1;
            for (t = 0; t < 4; t++) f[t] = v[(b + t) * s];
            for (t = 0; t < depth; t++) {
                long dst = b + t + 2;
                if (dst < n) v[dst * s] = f[1] + (double)(t + 1) * (f[1] - f[0]);
            }
        }
    }
}

/* cukern_SetOutflowX (cudaStatics.cu:462-545) along one pencil of all five slabs.
 * nd = physical normal direction (1..3).  restFrmSpeed: 1.05 on the - side, -1.198-.0047 i
 * on the + side (cudaStatics.cu:379-384).
 * The reference's - side kernel indexes from depth cells before the pencil start (it writes
 * the depth cells preceding the row and reads cell 0); this restatement applies the
 * evident intent, reading cell `depth` and writing cells 0..depth-1 like the + side. */
static void bc_pencil_outflow(double *v[5], long s, int n, int side, int nd, int depth)
{
    int t, k;
    long src = (side == 1) ? (n - 1 - depth) : depth;
    double a = v[1 + nd][src * s];
    int direct = side ? 1 : -1;
    if (a * direct > 0) {
        for (k = 0; k < 5; k++) {
            double val = v[k][src * s];
            for (t = 0; t < depth; t++) {
                long dst = side ? (src + 1 + t) : t;
                v[k][dst * s] = val;
            }
        }
    } else {
        double rho = v[0][src * s];
        double E0 = v[1][src * s];
        double p1x = v[2][src * s], p1y = v[3][src * s], p1z = v[4][src * s];
        for (t = 0; t < depth; t++) {
            long dst = side ? (src + 1 + t) : t;
            int ridx = side ? (depth + t) : t;
            double rf = side ? (-1.198 - .0047 * t) : 1.05;
            double E = E0, p1, p2;
            (void)ridx;
            v[0][dst * s] = rho;
            p1 = p1x; p2 = rho * 0.0;
            v[2][dst * s] = p2;
            E += .5 * (p2 - p1) * (p2 + p1) / rho;
            p1 = p1y; p2 = (nd == 1) ? rho * rf : rho * (p1y / rho);
            v[3][dst * s] = p2;
            E += .5 * (p2 - p1) * (p2 + p1) / rho;
            p1 = p1z; p2 = rho * 0.0;
            v[4][dst * s] = p2;
            E += .5 * (p2 - p1) * (p2 + p1) / rho;
            v[1][dst * s] = E;
        }
    }
}

int or_fluid_boundary(double *q, const or_grid *g, const int32_t bc[6], int dir, int depth)
{
    int n, side;
    long stride, npencil;
    if (dir < 1 || dir > 3) return OR_ERR_INVALID;
    pencil_geometry(g, dir, &n, &stride, &npencil);
    for (side = 0; side < 2; side++) {
        int mode = bc[2 * (dir - 1) + side];
        long pp;
        if (mode == OR_BC_CIRCULAR || mode == OR_BC_STATIONARY) continue;
        if (mode == OR_BC_WALL || mode == OR_BC_FREEBALANCE) return OR_ERR_NOIMPL;
        for (pp = 0; pp < npencil; pp++) {
            long b = pencil_base(g, dir, pp);
            double *v[5];
            int k;
            for (k = 0; k < 5; k++) v[k] = q + (long)k * g->slab + b;
            if (mode == OR_BC_OUTFLOW) {
                bc_pencil_outflow(v, stride, n, side, dir, depth);
            } else {
                for (k = 0; k < 5; k++) {
                    int anti = (k >= 2) && (k - 1 == dir);  /* vectorComponent == direction */
                    bc_pencil_sas(v[k], stride, n, mode, side, anti, depth);
                }
            }
        }
    }
    return OR_OK;
}

/* ------------------------------------------------------------------------------------------
 * performFluidUpdate_3D (flux.cu:27-165)
 * ---------------------------------------------------------------------------------------- */
int or_fluid_step_3d(double *q, const or_grid *g, const or_step *p0, const int32_t bc[6],
                     int sweep_dir, int step_number)
{
    static const int fluxcall[3][6] = {{1, 2, 1, 2, 3, 3}, {3, 1, 2, 3, 1, 2}, {2, 3, 3, 1, 2, 1}};
    int sweep = (step_number + 3 * (sweep_dir > 0)) % 6;
    int nstep, rc;
    int ext[3];
    or_step pst = *p0;
    const or_step *p = &pst;
    pst.theta_form = or_theta_form(sweep_dir, step_number);
    ext[0] = g->nx; ext[1] = g->ny; ext[2] = g->nz;
    if (g->ny == 1 && g->nz == 1) {
        rc = or_fluid_sweep(q, g, p, 1);
        if (rc) return rc;
        return or_fluid_boundary(q, g, bc, 1, 4);
    }
    for (nstep = 0; nstep < 3; nstep++) {
        int d = fluxcall[nstep][sweep];
        if (ext[d - 1] > 3) {
            rc = or_fluid_sweep(q, g, p, d);
            if (rc) return rc;
            rc = or_fluid_boundary(q, g, bc, d, 4);
            if (rc) return rc;
        }
    }
    return OR_OK;
}

/* ------------------------------------------------------------------------------------------
 * Soundspeed and CFL
 * ---------------------------------------------------------------------------------------- */
void or_soundspeed(const double *q, const or_grid *g, double gamma, double *cs)
{
    long N = (long)g->nx * g->ny * g->nz, x;
    double gg1 = gamma * (gamma - 1);
    const double *rho = q, *E = q + g->slab, *px = q + 2 * g->slab, *py = q + 3 * g->slab,
                 *pz = q + 4 * g->slab;
#pragma omp parallel for schedule(static)
    for (x = 0; x < N; x++) {
        double rhoinv = 1 / rho[x];
        double csq = gg1 * (E[x] - .5 * (px[x] * px[x] + py[x] * py[x] + pz[x] * pz[x]) * rhoinv) * rhoinv;
        if (csq < 0.0) csq = 0.0;
        cs[x] = sqrt(csq);
    }
}

double or_cfl_timestep(const double *q, const double *cs, const or_grid *g, const double h[3],
                       const int32_t global_rez[3], int method)
{
    return or_cfl_timestep_geo(q, cs, g, h, global_rez, method, OR_GEO_SQUARE, 0.0);
}

double or_cfl_timestep_geo(const double *q, const double *cs, const or_grid *g, const double h[3],
                           const int32_t global_rez[3], int method, int geometry, double r_inner)
{
    long N = (long)g->nx * g->ny * g->nz, x;
    int spacedim = 0, sim;
    int algo_xj;
    double tmin = 1e38;
    const double *rho = q, *px = q + 2 * g->slab, *py = q + 3 * g->slab, *pz = q + 4 * g->slab;
    double hmin;
    if (global_rez[1] > 1) spacedim = 1;
    if (global_rez[2] > 1) spacedim = 2;
    sim = spacedim + 1;
    /* ctype table (cflTimestep.cu:175-193): square 1-D Xin-Jin uses the HLLC kernel (case 12), the
     * cylindrical one the Xin-Jin kernel (case 15) */
    algo_xj = (method == 3) && (sim > 1 || geometry == OR_GEO_CYLINDRICAL);
    hmin = h[0];
    if (geometry == OR_GEO_CYLINDRICAL) {
        /* dr, and dz in 3-D; the theta extent is taken per cell (cflTimestep.cu:301-304) */
        if (sim == 3) hmin = (hmin < h[2]) ? hmin : h[2];
    } else {
        if (sim > 1 && h[1] < hmin) hmin = h[1];
        if (sim > 2 && h[2] < hmin) hmin = h[2];
    }
#pragma omp parallel for reduction(min : tmin) schedule(static)
    for (x = 0; x < N; x++) {
        double u, v;
        if (!algo_xj) {
            double p;
            if (sim == 1) {
                p = fabs(px[x]);
            } else {
                double pp = px[x], qq;
                pp = pp * pp;
                qq = py[x];
                pp = pp + qq * qq;
                if (sim > 2) {
                    qq = pz[x];
                    pp = pp + qq * qq;
                }
                p = sqrt(pp);
            }
            u = p / rho[x] + cs[x];
            if (geometry == OR_GEO_CYLINDRICAL) {
                /* r dtheta of this cell's radius (cflTimestep.cu:316-320) */
                double w = (r_inner + (x % g->nx) * h[0]) * h[1];
                w = (w < hmin) ? w : hmin;
                u = w / u;
            } else {
                u = hmin / u;
            }
        } else {
            double r = rho[x];
            u = h[0] / (fabs(px[x]) / r + cs[x]);
            if (sim > 1) {
                if (geometry == OR_GEO_CYLINDRICAL)
                    v = (r_inner + (x % g->nx) * h[0]) * h[1] / (fabs(py[x]) / r + cs[x]);
                else
                    v = h[1] / (fabs(py[x]) / r + cs[x]);
                u = (u < v) ? u : v;
            }
            if (sim > 2) {
                v = h[2] / (fabs(pz[x]) / r + cs[x]);
                u = (u < v) ? u : v;
            }
        }
        if (u < tmin) tmin = u;   /* NaN never wins, as in the reference's ternary min */
    }
    if (tmin > 1e37) tmin = 1e37;  /* per-thread initial value in the kernel */
    if (method == 1 || method == 2) tmin = tmin / 2;
    return tmin;
}

/* ------------------------------------------------------------------------------------------
 * Cylindrical geometric source terms (cukern_SourceCylindricalTerms,
 * cudaSourceCylindricalTerms.cu:119-222).  Per cell: v_r' = v_theta^2 / r, v_theta' = -v_r
 * v_theta / r over dt by the two-stage Gauss-Legendre collocation method (the Butcher table of
 * the fourth-order Gauss-Legendre method, with the reference's own decimal constants) and two
 * fixed-point passes.  The stage updates are restated as the reference writes them, including
 * the sign of the second stage's term in the first v_theta update and the second v_theta
 * update's use of the old v_r of stage B in both terms; the kinetic-energy change goes into
 * internal energy except that a non-positive pressure is reset.  Runs on the XYZ layout.
 * ---------------------------------------------------------------------------------------- */
#define GL4_A11 .25
#define GL4_A12 -0.038675134594812865529
#define GL4_A21 0.53867513459481286553
#define GL4_A22 .25

void or_cyl_source(double *q, const or_grid *g, double dt, double dr, double r_inner)
{
    const long nx = g->nx, N = (long)g->nx * g->ny * g->nz;
    const long S = g->slab;
    long x;
#pragma omp parallel for schedule(static)
    for (x = 0; x < N; x++) {
        double *base = q + x;
        double r = r_inner + (int)(x % nx) * dr;
        double rho, u, v, w, E, newP, vrA, vphiA, vrB, vphiB, diffmom, diffmomB, scratch;
        int it;
        rho = base[0];
        u = base[2 * S] / rho;
        v = base[3 * S] / rho;
        diffmom = dt * v / r;
        vrA = u + GL4_A11 * v * diffmom;
        vphiA = v - GL4_A11 * u * diffmom;
        vrB = u + GL4_A12 * v * diffmom;
        vphiB = v - GL4_A12 * u * diffmom;
        for (it = 0; it < 2; it++) {
            diffmom = dt * vphiA / r;
            diffmomB = dt * vphiB / r;
            scratch = vrA;
            vrA = u + GL4_A11 * vphiA * diffmom + GL4_A12 * vphiB * diffmomB;
            vphiA = v - GL4_A11 * scratch * diffmom + GL4_A12 * vrB * diffmomB;
            diffmom = dt * vphiA / r;
            scratch = vrB;
            vrB = u + GL4_A21 * vphiA * diffmom + GL4_A22 * vphiB * diffmomB;
            vphiB = v - GL4_A21 * scratch * diffmom + GL4_A22 * scratch * diffmomB;
        }
        u = rho * (u + .5 * dt * (vphiA * vphiA + vphiB * vphiB) / r);
        v = rho * (v - .5 * dt * (vphiA * vrA + vphiB * vrB) / r);
        E = base[S];
        w = base[4 * S];
        newP = E - .5 * (u * u + v * v + w * w) / rho;
        if (newP <= 0.0) base[S] = .5 * (u * u + v * v + w * w) / rho + .00001 * rho;
        base[2 * S] = u;
        base[3 * S] = v;
    }
}

/* ------------------------------------------------------------------------------------------
 * freezeAndPtot (hydro)
 * ---------------------------------------------------------------------------------------- */
void or_freeze_and_ptot(double *q, const or_grid *g, double gamma, double cs_min,
                        double *ptot, double *freeze)
{
    long rows = (long)g->ny * g->nz, r;
    double gm1 = gamma - 1.0, cs0sq = cs_min * cs_min;
#pragma omp parallel for schedule(static)
    for (r = 0; r < rows; r++) {
        long x0 = r * g->nx, x;
        double CsMax = 0.0;
        double *rho = q, *E = q + g->slab, *px = q + 2 * g->slab, *py = q + 3 * g->slab,
               *pz = q + 4 * g->slab;
        for (x = x0; x < x0 + g->nx; x++) {
            double rhoinv = 1.0 / rho[x];
            double psqhf = .5 * (px[x] * px[x] + py[x] * py[x] + pz[x] * pz[x]);
            double P = gm1 * (E[x] - psqhf * rhoinv);
            double Cs;
            if (gamma * P * rhoinv < cs0sq) {
                P = cs0sq / (gamma * rhoinv);
                E[x] = psqhf * rhoinv + P / gm1;
            }
            ptot[x] = P;
            Cs = sqrt(gamma * P * rhoinv) + fabs(px[x] * rhoinv);
            if (Cs > CsMax) CsMax = Cs;
        }
        freeze[r] = CsMax;
    }
}

/* ------------------------------------------------------------------------------------------
 * Per-array boundary conditions in XYZ storage (cudaStatics mex semantics)
 * ---------------------------------------------------------------------------------------- */
int or_array_boundary(double *phi, const or_grid *g, int bc_mode, int dir, int side,
                      int vec_component, int depth)
{
    int n;
    long stride, npencil, pp;
    int anti = (vec_component == dir);
    if (dir < 1 || dir > 3 || side < 0 || side > 1) return OR_ERR_INVALID;
    if (bc_mode == OR_BC_CIRCULAR || bc_mode == OR_BC_STATIONARY) return OR_OK;
    if (bc_mode == OR_BC_WALL || bc_mode == OR_BC_FREEBALANCE) return OR_ERR_NOIMPL;
    if (bc_mode == OR_BC_OUTFLOW) return OR_OK;  /* handled by the fluid-level entry */
    if (bc_mode == OR_BC_LINEAR && dir != 1) return OR_ERR_NOIMPL;  /* cudaStatics.cu:1187-1220 */
    pencil_geometry(g, dir, &n, &stride, &npencil);
    for (pp = 0; pp < npencil; pp++) {
        double *v = phi + pencil_base(g, dir, pp);
        long s = stride;
        int q;
        if (dir == 1 || bc_mode == OR_BC_LINEAR) {
            bc_pencil_sas(v, s, n, bc_mode, side, anti, depth);
            continue;
        }
        if (bc_mode == OR_BC_MIRROR) {
            for (q = 0; q < depth; q++) {
                double a;
                if (side == 0) {
                    /* y: 2*depth-1+MIRROR_OFFSET-q; z: 2*depth+MIRROR_OFFSET-q
                     * (cudaStatics.cu:1413-1421 vs 1471-1481) */
                    int src = (dir == 2) ? (2 * depth - q) : (2 * depth + 1 - q);
                    a = v[(long)src * s];
                    v[(long)q * s] = anti ? -a : a;
                } else {
                    a = v[(long)(n - 1 - 2 * depth + q) * s];
                    v[(long)(n - 1 - q) * s] = anti ? -a : a;
                }
            }
        } else if (bc_mode == OR_BC_CONST) {
            if (side == 0) {
                double f = v[(long)depth * s];
                for (q = 0; q < depth; q++) v[(long)q * s] = f;
            } else {
                /* y/z + side copies cell n-depth (cudaStatics.cu:1443-1448, 1524-1531) */
                double f = v[(long)(n - depth) * s];
                for (q = 0; q < depth; q++) v[(long)(n - 1 - q) * s] = f;
            }
        }
    }
    return OR_OK;
}

void or_statics_fade(double *phi, const double *statics, int64_t n, int64_t pitch)
{
    int64_t i;
    for (i = 0; i < n; i++) {
        long xaddr = (long)statics[i];
        double f0 = statics[i + pitch];
        double c = statics[i + 2 * pitch];
        if (c != 1.0) {
            double wval = f0 * c + (1.0 - c) * phi[xaddr];
            if (isnan(wval)) wval = f0 * c;
            phi[xaddr] = wval;
        } else {
            phi[xaddr] = f0;
        }
    }
}

/* ------------------------------------------------------------------------------------------
 * Two-fluid drag (cudaSource2FluidDrag.cu)
 * thermo: [gamma, mass, mu0, muTindex, sigma0, sigmaTindex, kBolt, Cisothermal]
 * ---------------------------------------------------------------------------------------- */
void or_drag_params(const double tg[8], const double td[8], double dt, double out[11])
{
    /* cudaSource2FluidDrag.cu:196-218 */
    double gam = tg[0];
    double nu0 = tg[2], nupow = tg[3], lampow = tg[5];
    double ddust = sqrt(td[4] / 3.141592653589793);
    double mgas = tg[1], mdust = td[1];
    out[0] = nu0;
    out[1] = -nupow;
    out[2] = lampow;
    out[3] = mgas * (gam - 1.0) / (298.15 * tg[6]);
    out[4] = sqrt(2.0) * mgas / (tg[4] * ddust);
    out[5] = ddust / nu0;
    out[6] = td[4] / (1.0 * mdust);
    out[7] = dt;
    out[8] = (gam - 1.0);
    out[9] = .25 * td[4] / mdust;
    out[10] = 16 * (gam - 1.0) / 3.0;
}

/* allregimeCdrag (cudaSource2FluidDrag.cu:819-833) */
static double allregime_cdrag(double Re, double Kn)
{
    double cunningham = 1 + Kn * (1.142 + 1 * 0.558 * exp(-0.999 / Kn));
    double C_drag = (3 / Re + .45 * pow(Re, -.319) + .0509 * Re / (8710 + Re)) / cunningham;
    return C_drag;
}

/* cukern_GasDustDrag_GeneralLinearCore with srcBlock = 0 (cudaSource2FluidDrag.cu:836-890):
 * returns k for |dv| = magdv and specific internal energy u; sets *skip when |dv| < 1e-9 */
static double drag_k(const double dp[11], double rhoA, double rhoB, double magdv, double u, int *skip)
{
    double Tn, Re, Kn, Cd_hat;
    if (magdv < 1e-9) { *skip = 1; return 0; }
    *skip = 0;
    Tn = dp[3] * u;
    Re = dp[5] * rhoA * magdv * pow(Tn, dp[1]);
    Kn = dp[4] * pow(Tn, dp[2]) / rhoA;
    Cd_hat = allregime_cdrag(Re, Kn);
    return Cd_hat * magdv * (rhoA + rhoB) * dp[6];
}

/* cukern_prepareForERK_h0 (cudaSource2FluidDrag.cu:1883-1908) + cukern_LogTrapSolve
 * (cudaSource2FluidDrag.cu:1531-1686) for one cell; gas/dust point at the cell in slab 0. */
static void logtrap_cell(double *gas, double *dust, long S, const double dp[11], double t, int order)
{
    double dv, dvsq, press, t0, t1, t2;
    double mu, k, dv_i, dv_t, duint, rhoginv, pdustsq, vstick, q;
    int skip;
    /* prepare: [|dv|, u] */
    dv = (gas[2 * S]) / gas[0] - dust[2 * S] / dust[0];
    dvsq = dv * dv;
    dv = (gas[3 * S]) / gas[0] - dust[3 * S] / dust[0];
    dvsq += dv * dv;
    dv = (gas[4 * S]) / gas[0] - dust[4 * S] / dust[0];
    dvsq += dv * dv;
    press = (gas[S] - .5 * (gas[2 * S] * gas[2 * S] + gas[3 * S] * gas[3 * S] + gas[4 * S] * gas[4 * S]) / gas[0]);
    t0 = sqrt(dvsq);         /* tmp slab 0 */
    t1 = press / gas[0];     /* tmp slab 1 */
    t2 = 0;                  /* tmp slab 2 */

    mu = dust[0] / (gas[0] + dust[0]);
    k = drag_k(dp, gas[0], dust[0], t0, t1, &skip);
    t2 = skip ? 0 : k;       /* resetAccumulator */
    k = t2;
    dv_i = t0;
    dv_t = dv_i * exp(-t * k);
    dvsq = dv_t * dv_t;
    duint = -.5 * dv_i * dv_i * mu * expm1(-2 * k * t);
    t0 = sqrt(dvsq);
    t1 += duint;
    k = drag_k(dp, gas[0], dust[0], t0, t1, &skip);
    if (!skip) t2 += k;      /* accumulate */
    if (order == 3) {
        t1 -= duint;
        k = .25 * (t2);
        dv_t = dv_i * exp(-t * k);
        dvsq = dv_t * dv_t;
        duint = -0.5 * dv_i * dv_i * mu * expm1(-2 * k * t);
        t0 = sqrt(dvsq);
        t1 += duint;
        k = drag_k(dp, gas[0], dust[0], t0, t1, &skip);
        t0 = skip ? 0 : k;   /* written into slab 0 with reset */
        k = (0.16666666666666666667 * t2 + 0.66666666666666666667 * t0);
    } else {
        k = .5 * t2;
    }
    mu = mu * gas[0];
    rhoginv = 1.0 / gas[0];

    pdustsq = -dust[2 * S] * dust[2 * S];
    vstick = (gas[2 * S] + dust[2 * S]) / (gas[0] + dust[0]);
    dv_i = (gas[2 * S]) * rhoginv - dust[2 * S] / dust[0];
    dv_t = dv_i * exp(-t * k);
    gas[2 * S] = gas[0] * vstick + dv_t * mu;
    dust[2 * S] = q = dust[0] * vstick - dv_t * mu;
    pdustsq += q * q;

    pdustsq -= dust[3 * S] * dust[3 * S];
    vstick = (gas[3 * S] + dust[3 * S]) / (gas[0] + dust[0]);
    dv_i = (gas[3 * S]) * rhoginv - dust[3 * S] / dust[0];
    dv_t = dv_i * exp(-t * k);
    gas[3 * S] = gas[0] * vstick + dv_t * mu;
    dust[3 * S] = q = dust[0] * vstick - dv_t * mu;
    pdustsq += q * q;

    pdustsq -= dust[4 * S] * dust[4 * S];
    vstick = (gas[4 * S] + dust[4 * S]) / (gas[0] + dust[0]);
    dv_i = (gas[4 * S]) * rhoginv - dust[4 * S] / dust[0];
    dv_t = dv_i * exp(-t * k);
    gas[4 * S] = gas[0] * vstick + dv_t * mu;
    dust[4 * S] = q = dust[0] * vstick - dv_t * mu;
    pdustsq += q * q;

    gas[S] -= .5 * pdustsq / dust[0];
}

void or_drag_logtrap_cells(double *gas, double *dust, int64_t n, int64_t slab,
                           const double dp[11], double dt, int order)
{
    int64_t i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < n; i++) logtrap_cell(gas + i, dust + i, slab, dp, dt, order);
}

/* cukern_GasDustDrag_GeneralAccel (cudaSource2FluidDrag.cu:898-931): -d|dv|/dt at |dv| = w.
 * ini = 1 uses the initial specific internal energy u0 as is (ONLY_DV_INI); otherwise the gas
 * is credited with the relative kinetic energy dissipated since w0. */
static double drag_accel(const double dp[11], double rhoA, double rhoB, double w0, double u0, double w, int ini)
{
    double u, Tn, Re, Kn, Cd_hat, accel;
    if (ini) u = u0;
    else u = u0 + .5 * rhoB * (w0 * w0 - w * w) / (rhoA + rhoB);
    Tn = dp[3] * u;
    Re = dp[5] * rhoA * w * pow(Tn, dp[1]);
    Kn = dp[4] * pow(Tn, dp[2]) / rhoA;
    Cd_hat = allregime_cdrag(Re, Kn);
    accel = Cd_hat * w * w * (rhoA + rhoB) * dp[6];
    return -accel;
}

/* cukern_findInitialDeltaV (cudaSource2FluidDrag.cu:1014-1050): w0 = |dv|, u0 = e_int / rho_gas */
static void initial_dv(const double *g, const double *d, long S, double *w0, double *u0)
{
    double u, q, dvsq, rhoginv, rhodinv, momsq;
    rhoginv = 1 / g[0];
    rhodinv = 1 / d[0];
    q = g[2 * S];
    u = q * rhoginv - d[2 * S] * rhodinv;
    momsq = q * q;
    dvsq = u * u;
    q = g[3 * S];
    u = q * rhoginv - d[3 * S] * rhodinv;
    momsq += q * q;
    dvsq += u * u;
    q = g[4 * S];
    u = q * rhoginv - d[4 * S] * rhodinv;
    momsq += q * q;
    dvsq += u * u;
    *w0 = sqrt(dvsq);
    *u0 = (g[S] - .5 * momsq * rhoginv) * rhoginv;
}

/* cukern_applyFinalDeltaV (cudaSource2FluidDrag.cu:1160-1229): relative velocity rescaled to
 * magnitude wf about the centre-of-mass velocity, gas energy credited with the dust's kinetic
 * energy loss, dust energy reset to p^2/2rho + 1e-4 rho. */
static void apply_final_dv(double *g, double *d, long S, double wf)
{
    double vstick[3], dvhat[3], rhog, rhod, a, b, c, p1, p2, dustmom, dustmomfin;
    int k;
    rhog = g[0];
    rhod = d[0];
    for (k = 0; k < 3; k++) {
        p1 = g[(2 + k) * S];
        p2 = d[(2 + k) * S];
        vstick[k] = (p1 + p2) / (rhog + rhod);
        dvhat[k] = p1 / rhog - p2 / rhod;
    }
    a = wf / sqrt(dvhat[0] * dvhat[0] + dvhat[1] * dvhat[1] + dvhat[2] * dvhat[2]);
    dvhat[0] *= a;
    dvhat[1] *= a;
    dvhat[2] *= a;
    b = rhog * rhod / (rhog + rhod);
    dustmom = d[2 * S] * d[2 * S];
    g[2 * S] = rhog * vstick[0] + dvhat[0] * b;
    d[2 * S] = c = rhod * vstick[0] - dvhat[0] * b;
    dustmomfin = c * c;
    dustmom += d[3 * S] * d[3 * S];
    g[3 * S] = rhog * vstick[1] + dvhat[1] * b;
    d[3 * S] = c = rhod * vstick[1] - dvhat[1] * b;
    dustmomfin += c * c;
    dustmom += d[4 * S] * d[4 * S];
    g[4 * S] = rhog * vstick[2] + dvhat[2] * b;
    d[4 * S] = c = rhod * vstick[2] - dvhat[2] * b;
    dustmomfin += c * c;
    g[S] += .5 * (dustmom - dustmomfin) / d[0];
    d[S] = .5 * dustmomfin / d[0] + 1e-4 * d[0];
}

/* solveDragEMP (cudaSource2FluidDrag.cu:305-370) and solveDragRK4 (:372-475) on one cell: the
 * scalar ODE d|dv|/dt = -accel(|dv|) by the explicit midpoint or the classic RK4 tableau, stage
 * by stage as the reference's kernels store them (tmp slab 0 = w0, 2 = accumulator, 3 = f,
 * 4 = stage), then the final update.  Cells with |dv| < 1e-9 are left unchanged (the reference
 * divides by |dv| there and writes NaN). */
static void rk_cell(double *g, double *d, long S, const double dp[11], double dt, int rk4)
{
    double w0, u0, f, acc, stage, wf;
    initial_dv(g, d, S, &w0, &u0);
    if (w0 < 1e-9) return;
    f = drag_accel(dp, g[0], d[0], w0, u0, w0, 1);
    if (!rk4) {
        stage = w0 + .5 * dt * f;
        acc = 0 * f;
        f = drag_accel(dp, g[0], d[0], w0, u0, stage, 0);
        wf = w0 + dt * (acc + 1.0 * f);
    } else {
        stage = w0 + 0.5 * dt * f;
        acc = 1.0 * f;
        f = drag_accel(dp, g[0], d[0], w0, u0, stage, 0);
        stage = w0 + 0.5 * dt * f;
        acc += 2.0 * f;
        f = drag_accel(dp, g[0], d[0], w0, u0, stage, 0);
        stage = w0 + 1.0 * dt * f;
        acc += 2.0 * f;
        f = drag_accel(dp, g[0], d[0], w0, u0, stage, 0);
        wf = w0 + (dt / 6.0) * (acc + 1.0 * f);
    }
    apply_final_dv(g, d, S, wf);
}

/* solveDragETDRK1 without the pressure-gradient term (cudaSource2FluidDrag.cu:477-560, kernel
 * cukern_ETDRK1 :1426-1510): exponential Euler with the drag rate at t = 0.  Cells with
 * |dv| < 1e-9 (k = 0) are left unchanged (the reference evaluates 0/0 there). */
static void etdrk1_cell(double *gas, double *dust, long S, const double dp[11], double t)
{
    double dv, dvsq, press, t0, t1, k, rhoginv, mu, pdustsq, vstick, dv_i, dv_t, q, dpdt;
    int skip, ax;
    dv = (gas[2 * S]) / gas[0] - dust[2 * S] / dust[0];
    dvsq = dv * dv;
    dv = (gas[3 * S]) / gas[0] - dust[3 * S] / dust[0];
    dvsq += dv * dv;
    dv = (gas[4 * S]) / gas[0] - dust[4 * S] / dust[0];
    dvsq += dv * dv;
    press = (gas[S] - .5 * (gas[2 * S] * gas[2 * S] + gas[3 * S] * gas[3 * S] + gas[4 * S] * gas[4 * S]) / gas[0]);
    t0 = sqrt(dvsq);
    t1 = press / gas[0];
    k = drag_k(dp, gas[0], dust[0], t0, t1, &skip);
    if (skip) return;
    rhoginv = 1.0 / gas[0];
    mu = gas[0] * dust[0] / (gas[0] + dust[0]);
    pdustsq = 0;
    for (ax = 2; ax <= 4; ax++) {
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

/* solveDragETDRK2 (cudaSource2FluidDrag.cu:575-690), exponential midpoint, as the reference
 * compiles it (ACCOUNT_GRADP and EXPO_DOTR undefined, :56-63):
 *   prepareForExpMethod, spaceOrder 2 (:1728-1866): per cell [|dv|, e_int/rho, G_x, G_y, G_z] with
 *     G the periodic central difference (gamma-1)/(2h) (e_int(+1) - e_int(-1)) of the gas internal
 *     energy density e_int = E - p^2/2rho (gas2press :1870-1873).  Three layouts: 3-D
 *     (cukern_prepareForERK3D_h2 :1913-2000, |dv|^2 summed x, y, z), x-y (nz = 1,
 *     cukern_prepareForERK2D_h2 :2123-2180, summed z, x, y, G_z = 0) and x-z (ny = 1 < nz,
 *     cukern_prepareForERKRZ_h2 :2238-2290, summed y, x, z, G_y = 0);
 *   k0 = GeneralLinearCore (:836-890) of (|dv|, e_int/rho);
 *   cukern_ExpMidpoint_partA (:1247-1312) with t = dt: per axis a = G rho^-1 / k0,
 *     dv(t) = a + (dv - a) exp(-k0 t) (the x axis adds t G to the gas momentum first; the z axis
 *     reads the dust y momentum, both as the reference does), the new |dv| and e_int/rho plus the
 *     drag heating;
 *   k1 = GeneralLinearCore of those; cukern_ExpMidpoint_partB (:1325-1420) with t = dt and no
 *     pressure-gradient term: dv <- dv exp(-k1 t) about the centre-of-mass velocity, gas E loses
 *     the dust kinetic-energy gain.
 * findMidGradP2 (:2395-2520) rewrites only the gradient slabs, which no later kernel reads, so it
 * is not restated.  Cells where k0 or k1 is zero (|dv| < 1e-9) are left unchanged: the reference
 * evaluates 0/0 there. */
static int drag_etdrk2(double *gas, double *dust, const or_grid *g, const double dp[11], double t,
                       const double h[3])
{
    const long nx = g->nx, ny = g->ny, nz = g->nz, S = g->slab, N = nx * ny * nz;
    const int three_d = nz > 1 && ny > 1, xz = nz > 1 && ny == 1;
    const double lamx = dp[8] / (2.0 * h[0]), lamy = dp[8] / (2.0 * h[1]), lamz = dp[8] / (2.0 * h[2]);
    double *P = (double *)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
    long i;
    if (!P) return OR_ERR_INVALID;
#pragma omp parallel for schedule(static)
    for (i = 0; i < N; i++)
        P[i] = (gas[S + i] - .5 * (gas[2 * S + i] * gas[2 * S + i] + gas[3 * S + i] * gas[3 * S + i] +
                                   gas[4 * S + i] * gas[4 * S + i]) / gas[i]);
#pragma omp parallel for schedule(static)
    for (i = 0; i < N; i++) {
        const long x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
        const long xm = (x + nx - 1) % nx, xp = (x + 1) % nx;
        const long ym = (y + ny - 1) % ny, yp = (y + 1) % ny;
        const long zm = (z + nz - 1) % nz, zp = (z + 1) % nz;
        double *gs = gas + i, *ds = dust + i;
        double dvx, dvy, dvz, dvsq, G[3], t0, t1, k, rhoginv, a0, dv_i, dv_t, duint, mu, pdustsq, vstick, dpdt,
            q;
        int skip, ax;
        G[0] = lamx * (P[z * nx * ny + y * nx + xp] - P[z * nx * ny + y * nx + xm]);
        dvx = (gs[2 * S]) / gs[0] - ds[2 * S] / ds[0];
        dvy = (gs[3 * S]) / gs[0] - ds[3 * S] / ds[0];
        dvz = (gs[4 * S]) / gs[0] - ds[4 * S] / ds[0];
        if (three_d) {
            G[1] = lamy * (P[z * nx * ny + yp * nx + x] - P[z * nx * ny + ym * nx + x]);
            G[2] = lamz * (P[zp * nx * ny + y * nx + x] - P[zm * nx * ny + y * nx + x]);
            dvsq = dvx * dvx;
            dvsq += dvy * dvy;
            dvsq += dvz * dvz;
        } else if (xz) {
            G[1] = 0.0;
            G[2] = lamz * (P[zp * nx + x] - P[zm * nx + x]);
            dvsq = dvy * dvy;
            dvsq += dvx * dvx;
            dvsq += dvz * dvz;
        } else {
            G[1] = lamy * (P[yp * nx + x] - P[ym * nx + x]);
            G[2] = 0.0;
            dvsq = dvz * dvz;
            dvsq += dvx * dvx;
            dvsq += dvy * dvy;
        }
        t0 = sqrt(dvsq);
        t1 = P[i] / gs[0];
        k = drag_k(dp, gs[0], ds[0], t0, t1, &skip);
        if (skip) continue;
        /* partA */
        rhoginv = 1.0 / gs[0];
        dvsq = 0;
        duint = 0;
        for (ax = 0; ax < 3; ax++) {
            a0 = G[ax];
            if (ax == 0) dv_i = (gs[2 * S] + t * a0) * rhoginv - ds[2 * S] / ds[0];
            else dv_i = (gs[(2 + ax) * S]) * rhoginv - ds[3 * S] / ds[0];
            a0 *= rhoginv / k;
            dv_t = a0 + (dv_i - a0) * exp(-t * k);
            if (ax == 0) dvsq = dv_t * dv_t;
            else dvsq += dv_t * dv_t;
            q = k * a0 * a0 * t - 2 * a0 * (dv_i - a0) * expm1(-k * t) - (dv_i - a0) * (dv_i - a0) * expm1(-2 * k * t);
            if (ax == 0) duint = q;
            else duint += q;
        }
        t0 = sqrt(dvsq);
        t1 += dp[8] * duint * rhoginv;
        k = drag_k(dp, gs[0], ds[0], t0, t1, &skip);
        if (skip) continue;
        /* partB */
        mu = gs[0] * ds[0] / (gs[0] + ds[0]);
        pdustsq = 0;
        for (ax = 2; ax <= 4; ax++) {
            if (ax == 2) pdustsq = -ds[2 * S] * ds[2 * S];
            else pdustsq -= ds[ax * S] * ds[ax * S];
            vstick = (gs[ax * S] + ds[ax * S]) / (gs[0] + ds[0]);
            dpdt = 0;
            dv_i = (gs[ax * S]) * rhoginv - ds[ax * S] / ds[0];
            dpdt *= mu * rhoginv;
            dv_t = dpdt / k + (dv_i - dpdt / k) * exp(-t * k);
            gs[ax * S] = gs[0] * vstick + dv_t * mu;
            ds[ax * S] = q = ds[0] * vstick - dv_t * mu;
            pdustsq += q * q;
        }
        gs[S] -= .5 * pdustsq / ds[0];
    }
    free(P);
    return OR_OK;
}

int or_drag_2fluid(double *gas, double *dust, const or_grid *g, const double tg[8],
                   const double td[8], double dt, int method, const double *h)
{
    double dp[11];
    long N = (long)g->nx * g->ny * g->nz;
    or_drag_params(tg, td, dt, dp);
    long i;
    if (method == 4 || method == 5) {
        or_drag_logtrap_cells(gas, dust, N, g->slab, dp, dt, method == 4 ? 2 : 3);
        return OR_OK;
    }
    if (method == 0 || method == 1) {
#pragma omp parallel for schedule(static)
        for (i = 0; i < N; i++) rk_cell(gas + i, dust + i, g->slab, dp, dt, method == 1);
        return OR_OK;
    }
    if (method == 2) {
#pragma omp parallel for schedule(static)
        for (i = 0; i < N; i++) etdrk1_cell(gas + i, dust + i, g->slab, dp, dt);
        return OR_OK;
    }
    if (method == 3) {
        if (!h) return OR_ERR_INVALID;
        return drag_etdrk2(gas, dust, g, dp, dt, h);
    }
    return OR_ERR_NOIMPL;
}
