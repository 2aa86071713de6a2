/*
 * imogen_oracle.h -- CPU oracle for the Imogen fluid-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64 restatement of the arithmetic of the
 * reference's GPU kernels (imogenproject/gpuImogen, gpuclass/), used by the test suite,
 * by __graft_entry__.smoke() and by bench.py's CPU baseline leg as the checker.  The product
 * path (gpuimogen_b200) never calls it.
 *
 * Build flags matter: it must be compiled with -ffp-contract=off so that every a*b+c is two
 * roundings, exactly as written in the reference source.  Under that rule the library's
 * "strict" build (nvcc -fmad=false) reproduces these results bit for bit.
 *
 * Memory layout (same as the library): one fluid = 5 slabs [rho, E, px, py, pz], each slab
 * nx*ny*nz doubles with x fastest, slabs `slab` doubles apart (slab >= nx*ny*nz).
 */
#ifndef IMOGEN_ORACLE_H
#define IMOGEN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t nx, ny, nz;
    int32_t pad_;
    int64_t slab;          /* doubles between consecutive slabs */
} or_grid;

/* Runtime physics switches for one fluid sweep (gpuclass/cudaFluidStep.cu:289-311). */
typedef struct {
    double dt;
    double h[3];           /* cell size per physical direction */
    double gamma;          /* already replaced by 2 for isothermal fluids by the caller */
    double rho_min;
    double c_iso;          /* -1 = adiabatic */
    int32_t method;        /* 1 HLL, 2 HLLC, 3 Xin-Jin */
    int32_t slope_limiter; /* OR_SLOPE_* (HLL / HLLC reconstruction) */
    int32_t flux_limiter;  /* OR_FLUX_*  (Xin-Jin TVD correction) */
    int32_t geometry;      /* OR_GEO_SQUARE or OR_GEO_CYLINDRICAL (x = r, y = theta, z = z) */
    double r_inner;        /* cylindrical: radius of the centre of radial cell 0 (pInnerRadius) */
    int32_t theta_form;    /* cylindrical theta sweeps: OR_THETA_213 or OR_THETA_231 */
    int32_t cyl_flags;     /* OR_CYL_GEOMETRIC_RADIUS: theta sweeps take r = r_inner + i*h[0] */
} or_step;

enum { OR_GEO_SQUARE = 0, OR_GEO_CYLINDRICAL = 1 };
/* The reference permutes memory so that the swept direction is fastest; for a theta sweep the
 * radial direction is then either the second (layout theta,r,z: FLUX_THETA_213, the flux
 * difference is divided by r) or the third (theta,z,r: FLUX_THETA_231, lambda is divided by r
 * first), which rounds differently (cudaFluidStep.cu:264-278, 848-855, 1085-1106).  Which one a
 * sweep of a fluid step gets follows from the sweep index (or_theta_form). */
enum { OR_THETA_213 = 0, OR_THETA_231 = 1 };
enum { OR_CYL_GEOMETRIC_RADIUS = 1 };

enum { OR_SLOPE_OSPRE = 0, OR_SLOPE_MC = 1, OR_SLOPE_VANLEER = 2, OR_SLOPE_MINMOD = 3,
       OR_SLOPE_SUPERBEE = 4, OR_SLOPE_VANALBADA = 5, OR_SLOPE_ZERO = 6 };
enum { OR_FLUX_OSPRE = 0, OR_FLUX_VANLEER = 1, OR_FLUX_MINMOD = 2, OR_FLUX_SUPERBEE = 3,
       OR_FLUX_ZERO = 4 };

/* BCModeTypes (gpuclass/cudaCommon.h:49) */
enum { OR_BC_CIRCULAR = 0, OR_BC_MIRROR = 1, OR_BC_WALL = 2, OR_BC_STATIONARY = 3,
       OR_BC_CONST = 4, OR_BC_LINEAR = 5, OR_BC_OUTFLOW = 6, OR_BC_FREEBALANCE = 7 };

/* One directional SSPRK2 sweep of a single fluid along physical direction dir (1,2,3),
 * periodic in the sweep direction (performFluidUpdate_1D, cudaFluidStep.cu:233-663). */
int or_fluid_sweep(double *q, const or_grid *g, const or_step *p, int dir);

/* Boundary fill of one fluid after a sweep along dir, as setFluidBoundary
 * (cudaStatics.cu:112-197) does it inside the fluid step: the array is then laid out with the
 * swept direction fastest, so only the X-direction kernels run, along direction dir.
 * bc[6] = [-X,+X,-Y,+Y,-Z,+Z].  depth = halo size (4). */
int or_fluid_boundary(double *q, const or_grid *g, const int32_t bc[6], int dir, int depth);

/* Full 3-sweep Strang-ordered fluid update (performFluidUpdate_3D, flux.cu:27-165):
 * sweep_dir = +1 forward / -1 backward, step_number = iteration count. */
int or_fluid_step_3d(double *q, const or_grid *g, const or_step *p, const int32_t bc[6],
                     int sweep_dir, int step_number);

/* c_s = sqrt(max(0, gamma(gamma-1) e/rho)) (cudaSoundspeed.cu:178-193). */
void or_soundspeed(const double *q, const or_grid *g, double gamma, double *cs);

/* tau = CFL-limited time (already halved for HLL/HLLC) (cflTimestep.cu:107-377);
 * global_rez gives the dimensionality, h the cell sizes. */
double or_cfl_timestep(const double *q, const double *cs, const or_grid *g, const double h[3],
                       const int32_t global_rez[3], int method);

/* The same in cylindrical geometry (geometry = OR_GEO_CYLINDRICAL): the theta extent of a cell
 * is (r_inner + i h[0]) h[1] for radial index i (cflTimestep.cu:301-333). */
double or_cfl_timestep_geo(const double *q, const double *cs, const or_grid *g, const double h[3],
                           const int32_t global_rez[3], int method, int geometry, double r_inner);

/* Geometric source terms of cylindrical coordinates over dt (cukern_SourceCylindricalTerms,
 * cudaSourceCylindricalTerms.cu:119-222): the centrifugal and Coriolis exchange between p_r and
 * p_theta, integrated by a two-stage Gauss-Legendre step with two fixed-point iterations, with
 * the reference's stage arithmetic as written; dr = h[0]. */
void or_cyl_source(double *q, const or_grid *g, double dt, double dr, double r_inner);

/* The theta form a theta sweep of a fluid step gets (sweep index (step_number + 3 [sweep_dir >
 * 0]) mod 6, flux.cu:46-49, through the permutations of cudaArrayRotateB.cu:580-643). */
int or_theta_form(int sweep_dir, int step_number);

/* freezeAndPtot hydro (freezeAndPtot.cu:32-147, 229-290): writes Ptot[N], freeze[ny*nz]
 * and floors E in place where c_s < cs_min. */
void or_freeze_and_ptot(double *q, const or_grid *g, double gamma, double cs_min,
                        double *ptot, double *freeze);

/* Per-array boundary condition as the cudaStatics mex applies it to an array stored in
 * XYZ order (cudaStatics.cu:85-104, 199-286, 1086-1532): memory direction = dir.
 * vec_component = 0 scalar, 1..3 vector component (mirror antisymmetry). side 0 = -, 1 = +. */
int or_array_boundary(double *phi, const or_grid *g, int bc_mode, int dir, int side,
                      int vec_component, int depth);

/* Statics fade list (cukern_applySpecial_fade, cudaStatics.cu:1240-1266). */
void or_statics_fade(double *phi, const double *statics, int64_t n, int64_t pitch);

/* Two-fluid drag (cudaSource2FluidDrag.cu).  thermo arrays: [gamma, mass, mu0, muTindex,
 * sigma0, sigmaTindex, kBolt, Cisothermal].  method 0 EMP, 1 RK4, 2 ETDRK1, 3 ETDRK2,
 * 4 LogTrap2, 5 LogTrap3.  h = cell sizes [hx, hy, hz], read by ETDRK2 only (its pressure
 * gradient); may be NULL for the other methods. */
int or_drag_2fluid(double *gas, double *dust, const or_grid *g, const double thermo_gas[8],
                   const double thermo_dust[8], double dt, int method, const double *h);

/* Drag constants the reference uploads (cudaSource2FluidDrag.cu:203-218). */
void or_drag_params(const double thermo_gas[8], const double thermo_dust[8], double dt,
                    double out[11]);

/* Exact LogTrap drag for a batch of independent cells given in SoA form; used by tests and
 * by the learned-drag training-set generator. */
void or_drag_logtrap_cells(double *gas, double *dust, int64_t n, int64_t slab,
                           const double dp[11], double dt, int order);

#ifdef __cplusplus
}
#endif
#endif
