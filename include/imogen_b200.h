/*
 * imogen_b200.h -- C ABI of the B200-native Imogen fluid-step library (libimogen_b200.so).
 *
 * One entry point per mex function of the reference's fluid-step hot path
 * (imogenproject/gpuImogen, gpuclass/), with the same argument meaning and in-place
 * semantics, expressed with plain pointers and POD structs so that a thin mex / ctypes / cgo
 * shim can bind them.  All array pointers are DEVICE pointers unless stated otherwise; the
 * caller owns every buffer it passes.  Every call is ordered on the given CUDA stream
 * (NULL = legacy default stream) and only returns to the host early where it must produce a
 * host value (the CFL timestep).  Return value: IB_SUCCESSFUL (0) or one of the reference's
 * error codes (gpuclass/imogenChecks.h:11-24); no entry point calls exit().
 *
 * Layout of a fluid: one allocation of five slabs [rho, E, px, py, pz]; each slab holds
 * nx*ny*nz doubles, x fastest, and slabs are `slab_pitch` doubles apart (a multiple of 32,
 * i.e. 256 B, as MGA_allocSlab pads them, gpuclass/cudaCommon.cu:339-370).  Arrays always stay
 * in XYZ order: the library sweeps y and z in place instead of transposing
 * (gpuclass/cudaArrayRotateB.cu is not needed).
 */
#ifndef IMOGEN_B200_H
#define IMOGEN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define IB_API __attribute__((visibility("default")))
#else
#define IB_API
#endif

/* Status codes (gpuclass/imogenChecks.h:11-24) */
#define IB_SUCCESSFUL 0
#define IB_ERROR_INVALID_ARGS -100
#define IB_ERROR_CRASH -101
#define IB_ERROR_NULL_POINTER -102
#define IB_ERROR_NOIMPLEMENT -105
#define IB_ERROR_NOMEM -106
#define IB_ERROR_CUDA -1000

/* Fluid methods (gpuclass/cudaFluidStep.h:6-8) */
#define IB_METHOD_HLL 1
#define IB_METHOD_HLLC 2
#define IB_METHOD_XINJIN 3

/* Slope limiters for HLL/HLLC reconstruction (gpuclass/limiter_functions.h:54-119).
 * The reference selects one at compile time (SLOPEFUNC, cudaFluidStep.cu:129-135; default
 * Ospre); here it is a runtime choice. */
#define IB_SLOPE_OSPRE 0
#define IB_SLOPE_MC 1
#define IB_SLOPE_VANLEER 2
#define IB_SLOPE_MINMOD 3
#define IB_SLOPE_SUPERBEE 4
#define IB_SLOPE_VANALBADA 5
#define IB_SLOPE_ZERO 6

/* Flux limiters for the Xin-Jin TVD correction (limiter_functions.h:11-45; LIMITERFUNC,
 * cudaFluidStep.cu:122-127, default Ospre). */
#define IB_FLUX_OSPRE 0
#define IB_FLUX_VANLEER 1
#define IB_FLUX_MINMOD 2
#define IB_FLUX_SUPERBEE 3
#define IB_FLUX_ZERO 4

/* Flux precision: FP64 everywhere, or HLLC/limiter arithmetic in FP32 with FP64 conserved
 * accumulation (the reference's FLOATFLUX compile option, cudaFluidStep.cu:118-122). */
#define IB_PREC_FP64 0
#define IB_PREC_FP32_FLUX 1

/* Boundary modes, BCModeTypes (gpuclass/cudaCommon.h:49); order [-X, +X, -Y, +Y, -Z, +Z]. */
#define IB_BC_CIRCULAR 0
#define IB_BC_MIRROR 1
#define IB_BC_WALL 2
#define IB_BC_STATIONARY 3
#define IB_BC_CONST 4
#define IB_BC_LINEAR 5
#define IB_BC_OUTFLOW 6
#define IB_BC_FREEBALANCE 7

/* Drag integrators (cudaSource2FluidDrag.cu:226-245) */
#define IB_DRAG_EMP 0
#define IB_DRAG_RK4 1
#define IB_DRAG_ETDRK1 2
#define IB_DRAG_ETDRK2 3
#define IB_DRAG_LOGTRAP2 4
#define IB_DRAG_LOGTRAP3 5

typedef struct ib_grid {
    int32_t nx, ny, nz;
    int32_t reserved;
    int64_t slab_pitch; /* doubles between slabs, multiple of 32, >= nx*ny*nz */
} ib_grid;

/* Statics ("fade") list of one array: device array [3][pitch] of
 * [linear index; value; coefficient] (cudaStatics.cu:1240-1266). */
typedef struct ib_statics {
    const double *data;
    int64_t count;
    int64_t pitch;
} ib_statics;

/* One fluid: the FluidManager canister (mass/ener/mom, cudaCommonML.cu:400-432) with its
 * boundary data (BCSettings, cudaCommon.h:51-58) and halo depth (4, run/starterRun.m:60-67). */
typedef struct ib_fluid {
    double *q;
    ib_grid grid;
    int32_t bc[6];
    int32_t halo;
    int32_t reserved;
    ib_statics statics[5];
} ib_fluid;

/* Per-fluid thermodynamics used by the fluid step (fluid.thermoDetails, fluid.MINMASS;
 * flux_ML_iface.cu:117-143). c_isothermal = -1 for an adiabatic fluid. */
typedef struct ib_fluid_thermo {
    double gamma;
    double rho_min;
    double c_isothermal;
} ib_fluid_thermo;

/* Geometry (GeometryParams, cudaCommon.h; accessMatlabGeometryClass, cudaCommonML.cu:453-481).
 * shape: IB_GEOMETRY_SQUARE (h = dx, dy, dz) or IB_GEOMETRY_CYLINDRICAL (x = r, y = theta,
 * z = z; h = dr, dtheta, dz; r_inner = radius of the centre of radial cell 0, pInnerRadius,
 * GeometryManager.m:300-311).  global_rez gives the dimensionality for the CFL
 * (globalDomainRez, cflTimestep.cu:85-87).  The RZ layout (ny = 1) of the reference's
 * RZCYLINDRICAL is not a separate shape here: a cylindrical grid with ny = 1 sweeps r and z. */
enum { IB_GEOMETRY_SQUARE = 0, IB_GEOMETRY_CYLINDRICAL = 1 };
typedef struct ib_geometry {
    double h[3];
    double r_inner;
    int32_t shape;
    int32_t global_rez[3];
} ib_geometry;

/* Numerical switches that the reference fixes at compile time; NULL = reference defaults
 * (Ospre slope limiter, Ospre flux limiter, FP64, the reference's cylindrical arithmetic).
 * flags: IB_FLAG_CYL_GEOMETRIC_RADIUS makes cylindrical theta sweeps use the cell centre radius
 * r_inner + i dr; without it they compute the radius as the reference's kernels do, with the theta
 * cell size as the radial step (cudaFluidStep.cu:305-307, 340, 848-855) and, for the sweeps whose
 * memory layout is theta,z,r on a 2-D grid, r_inner for every radius. */
enum { IB_FLAG_CYL_GEOMETRIC_RADIUS = 1 };
typedef struct ib_numerics {
    int32_t slope_limiter;
    int32_t flux_limiter;
    int32_t precision;
    int32_t flags;
} ib_numerics;

/* Microphysics of one fluid for the drag source (ThermoDetails, cudaCommon.h;
 * accessMatlabThermoDetails, cudaCommonML.cu:434-451). */
typedef struct ib_thermo {
    double gamma, mass, mu0, mu_t_index, sigma0, sigma_t_index, k_bolt, c_isothermal;
} ib_thermo;

/* Smallest legal slab pitch (doubles) for an nx*ny*nz array: numel rounded up to 32. */
IB_API int64_t ib_slab_pitch(int32_t nx, int32_t ny, int32_t nz);

/* ---------------------------------------------------------------------------------------------
 * The reference's GPU tags (for the mex glue).  A Matlab GPU array crosses into a mex function as
 * an int64 vector (cudaCommon.h:184-196):
 *   [dim0, dim1, dim2, numSlabs, halo, partitionDir, nGPUs, exteriorHalo, permtag,
 *    circularBits, vectorComponent, (deviceID, devicePtr) x nGPUs]
 * These calls decode tags into the structs of this header.  Host only: no device is touched.
 * ------------------------------------------------------------------------------------------- */
#define IB_GPU_TAG_LENGTH 11
#define IB_GPU_TAG_DIM0 0
#define IB_GPU_TAG_DIM1 1
#define IB_GPU_TAG_DIM2 2
#define IB_GPU_TAG_DIMSLAB 3
#define IB_GPU_TAG_HALO 4
#define IB_GPU_TAG_PARTDIR 5
#define IB_GPU_TAG_NGPUS 6
#define IB_GPU_TAG_EXTERIORHALO 7
#define IB_GPU_TAG_PERMTAG 8
#define IB_GPU_TAG_CIRCULARBITS 9
#define IB_GPU_TAG_VECTOR_COMPONENT 10
#define IB_GPU_TAG_MAX_GPUS 4 /* MAX_GPUS_USED, cudaCommon.h:11 */

/* Replaces decodeMatlabBCs (gpuclass/cudaCommonML.cu:203-232): the IB_BC_* mode of one of the
 * bcModes strings "circ", "const", "linear", "mirror", "bcstatic", "wall", "outflow",
 * "freebalance"; IB_ERROR_INVALID_ARGS for any other string. */
IB_API int ib_bcModeFromString(const char *name);

/* Replaces deserializeTagToMGArray (gpuclass/cudaCommon.cu:117-170) for one array, with the
 * checks of sanityCheckTag (cudaCommonML.cu:109-198): the device pointer, the extents and slab
 * pitch (numel * 8 bytes rounded up to 256, in doubles), and optionally the vector component and
 * the halo-sharing bits.  This library runs one GPU with arrays in XYZ order: a tag with
 * nGPUs > 1 or a permtag other than 1 (or 0, unset) returns IB_ERROR_NOIMPLEMENT; a malformed tag
 * IB_ERROR_INVALID_ARGS. */
IB_API int ib_arrayFromGpuTag(const int64_t *tag, int32_t taglen, double **ptr, ib_grid *grid,
                              int32_t *vector_component, int32_t *circular_bits);

/* Replaces MGA_accessFluidCanister (gpuclass/cudaCommonML.cu:400-432): the tags of a fluid's
 * mass, ener, mom(1), mom(2), mom(3) arrays into one ib_fluid.  The five must be slabs of one
 * allocation at the pitch MGA_allocSlab gives them (cudaCommon.cu:339-370; otherwise
 * IB_ERROR_NOIMPLEMENT), with equal extents, device and halo-sharing bits and vector components
 * 0, 0, 1, 2, 3.  bc_modes: the six IB_BC_* modes [-X, +X, -Y, +Y, -Z, +Z] decoded from the
 * arrays' boundaryData.bcModes (ib_bcModeFromString); a face whose circularBits bit is set must
 * be IB_BC_CIRCULAR.  With bc_modes NULL every face must have its bit set and is circular.  The
 * boundary depth is 4 (run/starterRun.m:60-67); statics lists are left empty. */
IB_API int ib_fluidFromGpuTags(const int64_t *const tags[5], const int32_t taglen[5], const int32_t *bc_modes,
                               ib_fluid *out);

/* Human-readable name of a status code. */
IB_API const char *ib_status_string(int status);

/* Last CUDA error seen by the library (cudaError_t value), 0 if none. */
IB_API int ib_last_cuda_error(void);

/* Number of kernels this process has launched through the library (all devices). */
IB_API long long ib_launch_count(void);

/* Health of the TMA-fed sweep kernels on the current device (no reference counterpart: the
 * reference has no asynchronous copies).  Their waits for a tile are bounded; a wait that runs
 * out makes the kernel leave early and sets a flag, which this call reads (synchronising with
 * the device): 0 = no wait ran out, bit 1 = one did and the state of that sweep is invalid,
 * bit 2 = a pencil-pair kernel found its shared-memory tile unaligned for the TMA copy and left
 * its block undone, < 0 = status code.  clear != 0 resets the flag. */
IB_API int ib_device_wait_status(int clear);

/* For failure-detection tests (no reference counterpart): how many times the TMA-fed sweep
 * kernels poll for each tile before their wait gives up, for launches after this call from any
 * thread; polls < 0 restores the default (2^26 polls, seconds).  A wait that gives up makes the
 * kernel wait (with the default limit) for the copies it has in flight, leave without finishing
 * its sweep and set the flag ib_device_wait_status reads; with polls = 0 every tile wait gives up
 * at once, so a test can exercise that path without any fault. */
IB_API int ib_setTileWaitLimit(long long polls);

/* Replaces the cudaFluidStep mex (gpuclass/cudaFluidStep.cu:161-227): one SSPRK2 directional
 * sweep of one fluid, in place, without boundary fill.
 * params = [dt, purehydro, gamma, rho_min, method (1 HLL | 2 HLLC | 3 XJ), direction (1..3)
 *           (, c_isothermal (, theta_layout))], nparams 6, 7 or 8; c_isothermal != -1 makes the
 * fluid isothermal and gamma := 2.  In cylindrical geometry direction 1 is r and 2 theta; the
 * reference takes a theta sweep's form from the arrays' memory permutation, which this API's
 * XYZ-ordered arrays do not carry: theta_layout 0 (default) = the form of layout theta,r,z
 * (FLUX_THETA_213), 1 = theta,z,r (FLUX_THETA_231).  Cylindrical sweeps are FP64 only. */
IB_API int ib_cudaFluidStep(ib_fluid *fluid, const ib_geometry *geo, const double *params, int nparams,
                     const ib_numerics *num, void *stream);

/* Replaces the fluidstep mex (gpuclass/flux_ML_iface.cu:37-160 -> performFluidUpdate_3D,
 * flux.cu:27-165): the three Strang-ordered sweeps plus boundary fill after each, for every
 * fluid in turn.  params = [dt, purehydro, sweep direction (+1 | -1), iteration, method]. */
IB_API int ib_fluidstep(ib_fluid *fluids, const ib_fluid_thermo *thermo, int nfluids,
                 const ib_geometry *geo, const double *params, int nparams,
                 const ib_numerics *num, void *stream);

/* Two-fluid drag as the source term of a complete timestep: fluids[0] is the gas, fluids[1] the
 * dust; method is one of IB_DRAG_* (ib_cudaSource2FluidDrag). */
typedef struct ib_drag_source {
    ib_thermo thermo_gas;
    ib_thermo thermo_dust;
    int32_t method;
    int32_t reserved;
} ib_drag_source;

/* Replaces performCompleteTimestep (gpuclass/flux_multi.cu:174-272), the fluid part of the
 * flux_multi mex and of imogenCore's main loop (gpuimogen_core.cu:954-1054): source half step,
 * forward fluid step of every fluid, full source step, backward fluid step, source half step.
 * params = [dt, purehydro, iteration, method].  The source is the two-fluid drag when drag is
 * not NULL (nfluids must then be 2); with drag == NULL there is none (the reference's srcType 0)
 * and each fluid runs its forward and backward step back to back.  The backward step's sweep
 * order is the forward one's reversed, so the forward step's last sweep and the backward step's
 * first are along the same axis with the same dt; when the boundary fill between them has
 * nothing to do (both faces of that axis periodic, no statics) the two run as one double-sweep
 * launch (HLL/HLLC), which gives the same result as ib_fluidstep(+1) then ib_fluidstep(-1). */
IB_API int ib_completeTimestep(ib_fluid *fluids, const ib_fluid_thermo *thermo, int nfluids,
                               const ib_geometry *geo, const double *params, int nparams,
                               const ib_numerics *num, const ib_drag_source *drag, void *stream);

/* ---------------------------------------------------------------------------------------------
 * The main loop with its timestep on the device (no reference counterpart: the reference reads
 * tau back to the host every iteration, TimeManager.m:124-186).  A loop that keeps dt on the
 * device can capture a whole iteration -- CFL of every fluid, ib_timeUpdate,
 * ib_completeTimestepDeviceDt, ib_timeAdvance -- in a CUDA graph and replay it without host
 * reads between iterations (one graph per iteration index modulo 6, which fixes the sweep
 * order).  After the end time dt is 0 and every kernel that reads it returns at once, so
 * iterations replayed past the end change nothing.
 * ------------------------------------------------------------------------------------------- */
typedef struct ib_time_state {  /* device memory */
    double tau[4];      /* CFL time of each fluid, written by ib_cflTimestepFused(..., tau_device = &tau[k]) */
    double dt;          /* this iteration's timestep; 0 once time has reached tmax */
    double time;        /* simulated time */
    double kahan;       /* compensation of the time sum */
    double cfl;         /* CFL number */
    double tmax;        /* end time (INFINITY: none) */
    int64_t iteration;  /* iterations taken */
    int32_t nfluids;    /* tau entries in use, 1..4 */
    int32_t status;     /* 1 once a non-finite CFL time stopped the loop (dt stays 0) */
} ib_time_state;

/* TimeManager.update (time/TimeManager.m:124-186) on the device: dt = cfl * min(tau[0..nfluids)),
 * clipped so that time + 2 dt <= tmax; dt = 0 once time >= tmax (1 - 1e-14) or status != 0. */
IB_API int ib_timeUpdate(ib_time_state *ts, void *stream);

/* TimeManager.step (:270-277) on the device: iteration += 1 and time += 2 dt (compensated), when
 * dt > 0. */
IB_API int ib_timeAdvance(ib_time_state *ts, void *stream);

/* ib_completeTimestep with the timestep read from device memory (*dt_device) by every kernel
 * (lambda = *dt_device / h in the sweeps, computed as the host form computes it, so both give
 * the same bits); params = [purehydro, iteration, method].  No host value depends on dt, so the
 * call can be captured in a CUDA graph after a first, uncaptured call of the same shape has set
 * up the library's scratch memory and kernel attributes. */
IB_API int ib_completeTimestepDeviceDt(ib_fluid *fluids, const ib_fluid_thermo *thermo, int nfluids,
                                       const ib_geometry *geo, const double *dt_device, const double *params,
                                       int nparams, const ib_numerics *num, const ib_drag_source *drag,
                                       void *stream);

/* Replaces the cudaSoundspeed mex for hydro (gpuclass/cudaSoundspeed.cu:54-105,
 * calculateSoundspeed :107-150): cs_out[N] = sqrt(max(0, gamma(gamma-1) e_int / rho)). */
IB_API int ib_cudaSoundspeed(const ib_fluid *fluid, double gamma, double *cs_out, void *stream);

/* Replaces the cflTimestep mex (gpuclass/cflTimestep.cu:64-103 -> computeLocalCFLTimestep
 * :107-252): *tau_host = min over cells of the signal-crossing time, halved for HLL/HLLC.
 * cs is the soundspeed array from ib_cudaSoundspeed.  Synchronises the stream.  The kernel
 * stores tau into pinned, mapped host memory (allocated once per device), so the read-back is
 * not queued behind device-to-host copies the caller has running on other streams. */
IB_API int ib_cflTimestep(const ib_fluid *fluid, const double *cs, const ib_geometry *geo, int method,
                   double *tau_host, void *stream);

/* Same value as ib_cudaSoundspeed + ib_cflTimestep in one pass over the fluid (no soundspeed
 * array).  If tau_device is not NULL the result is also left there and the call does not
 * synchronise (tau_host may then be NULL). */
IB_API int ib_cflTimestepFused(const ib_fluid *fluid, double gamma, const ib_geometry *geo, int method,
                        double *tau_host, double *tau_device, void *stream);

/* No counterpart in the reference.  The same timestep as ib_cflTimestepFused, for callers that
 * cannot let the library allocate device memory: an application that has reserved the GPU's
 * memory for its own allocator, or a loop that must not pay for the device-wide
 * synchronisation cudaMalloc/cudaFree can cause.  The reduction's scratch is a fixed array built
 * into the library (about 64 KB on every GPU that loads it, kept until exit), so the call
 * allocates nothing; the result goes to *tau_device (caller-owned device memory) and the call
 * does not synchronise.  Limit: at most 134,217,728 cells; larger grids return
 * IB_ERROR_INVALID_ARGS.  The first call on a device (and the first under each new context, e.g.
 * after cudaDeviceReset) looks up the array's device address, so make that first call outside
 * any stream capture.  All calls on a
 * device share the array (its counter is cleared at the start of each call): calls that overlap
 * on the GPU, e.g. on two streams, race. */
IB_API int ib_cflTimestepNoAlloc(const ib_fluid *fluid, double gamma, const ib_geometry *geo, int method,
                                 double *tau_device, void *stream);

/* Replaces the freezeAndPtot mex for hydro (gpuclass/freezeAndPtot.cu:32-147, kernel
 * :229-290): ptot[N] = gas pressure (raising E where c_s < cs_min), freeze[ny*nz] = max over
 * each x row of |px|/rho + c_s. */
IB_API int ib_freezeAndPtot(ib_fluid *fluid, double gamma, int purehydro, double cs_min, double *ptot,
                     double *freeze, void *stream);

/* Replaces the cudaStatics mex = setBoundaryConditions (gpuclass/cudaStatics.cu:85-104 ->
 * setArrayBoundaryConditions :199-286) for one array stored in XYZ order: applies its statics
 * and its boundary modes on both faces of `direction`.  vector_component: 0 scalar, 1..3 the
 * momentum component the array holds (mirror parity).  For outflow the array must be the
 * density slab of a fluid (the reference's numSlabs == 0 check, :255-259); the whole fluid
 * whose density slab starts at phi is then updated (slab_pitch from grid). */
IB_API int ib_cudaStatics(double *phi, const ib_grid *grid, const int32_t bc[6], int halo,
                   int vector_component, const ib_statics *statics, int direction, void *stream);

/* Boundary fill of a whole fluid as the fluid step performs it after a sweep along
 * `direction` (setFluidBoundary, gpuclass/cudaStatics.cu:112-197). */
IB_API int ib_setFluidBoundary(ib_fluid *fluid, int direction, void *stream);

/* Replaces the cudaSource2FluidDrag mex (gpuclass/cudaSource2FluidDrag.cu:125-181 ->
 * sourcefunction_2FluidDrag :189-246): gas-dust drag over dt, in place.
 * params = [dt, method (IB_DRAG_*)].  geo is read by ETDRK2 only (its pressure gradient uses the
 * cell sizes h, periodic central differences); it may be NULL for the other methods.  ETDRK2 uses
 * the library's scratch memory (one slab). */
IB_API int ib_cudaSource2FluidDrag(ib_fluid *gas, ib_fluid *dust, const ib_thermo *thermo_gas,
                            const ib_thermo *thermo_dust, const ib_geometry *geo,
                            const double *params, int nparams, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Batched ensemble of independent 1-D problems (no single reference counterpart: each problem
 * is what the reference runs as a 1-D fluid, the main loop of imogen.m:115-139 with
 * TimeManager.m:124-186,270-277 deciding dt, performFluidUpdate_3D's 1-D shortcut
 * flux.cu:52-68 for each half step and cflTimestep.cu:107-252 for tau).  Every problem runs on
 * its own clock to its own end, all in one kernel launch.
 * ------------------------------------------------------------------------------------------- */
typedef struct ib_ensemble {
    double *q;                /* device: 5 slabs [rho, E, px, py, pz] of slab_pitch doubles; problem p
                                 occupies cells offsets[p] .. offsets[p+1]-1 of every slab */
    int64_t slab_pitch;
    const int64_t *offsets;   /* device, nproblems + 1 entries, increasing, each problem >= 9 cells */
    const double *h;          /* device, cell width of each problem */
    const int32_t *order;     /* device, order in which CTAs pick problems (a permutation of
                                 0..nproblems-1, e.g. longest first), or NULL for 0, 1, ... */
    double *t_out;            /* device, simulated time each problem reached */
    int32_t *iters_out;       /* device, iterations each problem took */
    int32_t nproblems;
    int32_t bc[2];            /* -x and +x boundary modes (IB_BC_*), halo depth 4 */
    int32_t reserved;
} ib_ensemble;

/* Launch shape of the ensemble kernel (what the autotuner chooses); NULL or zeros = defaults
 * (256 threads, chunk 248 cells, as many CTAs per SM as fit). */
typedef struct ib_ensemble_tuning {
    int32_t threads;          /* 128, 256 or 512 */
    int32_t chunk;            /* cells per shared-memory chunk, 8 .. threads - 8 */
    int32_t ctas_per_sm;      /* 0 = occupancy limit */
    int32_t reserved;
} ib_ensemble_tuning;

/* Runs every problem of the ensemble to t_end (or itermax iterations) with the HLL or HLLC
 * method (1 or 2): per iteration tau = CFL reduction over the problem, dt = cfl * tau clipped so
 * that t + 2 dt <= t_end, forward and backward SSPRK2 sweep each followed by the boundary fill,
 * t += 2 dt (compensated).  num selects slope limiter (Ospre or MC) and precision (FP64 or the
 * FP32-flux form for HLLC).  One persistent launch: CTAs take problems from a device work
 * counter; the call does not synchronise and can be captured in a CUDA graph after a first
 * call outside capture (the first call allocates the counter). */
IB_API int ib_riemannEnsemble(const ib_ensemble *e, const ib_fluid_thermo *thermo, int method, double cfl,
                              double t_end, int32_t itermax, const ib_numerics *num,
                              const ib_ensemble_tuning *tuning, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Learned drag (no reference counterpart: it stands in for the LogTrap2 integrator of
 * cudaSource2FluidDrag.cu:709-795 and keeps that integrator as fallback and as the measure of
 * its error).
 *
 * The LogTrap2 update of a cell is fixed by one number, the decay exponent s = dt * k_eff of
 * the gas-dust relative velocity (dv -> dv * exp(-s) about the centre-of-mass velocity, the gas
 * absorbing the kinetic energy lost).  A small MLP predicts log s from five features:
 *   x = ((log rho_gas, log rho_dust, log |dv|, log u, log dt) - feature_shift) * feature_scale,
 *   u = specific internal energy of the gas (temperature), padded with zeros to 16 inputs
 *   (inputs 14 and 15 are reserved: the tensor-core inference feeds the first-layer bias
 *   through them, so they must stay zero in training data);
 *   3 hidden layers of 64 ReLU units, linear output y, log s = out_shift + out_scale * y.
 * Parameters are one FP32 vector laid out as below (FP32 master copy for training; inference
 * runs in BF16 on the tensor cores with FP32 accumulation).
 * ------------------------------------------------------------------------------------------- */
#define IB_MLP_IN 16
#define IB_MLP_HID 64
#define IB_MLP_OFF_W1 0       /* [64][16] */
#define IB_MLP_OFF_B1 1024    /* [64] */
#define IB_MLP_OFF_W2 1088    /* [64][64], row = output unit */
#define IB_MLP_OFF_B2 5184
#define IB_MLP_OFF_W3 5248
#define IB_MLP_OFF_B3 9344
#define IB_MLP_OFF_W4 9408    /* [64] */
#define IB_MLP_OFF_B4 9472    /* [1] */
#define IB_MLP_NPARAM 9473

/* Training kernels (FP32).  x: n x 16 row-major features, target: n values of the normalised
 * log s.  ib_mlpLossGrad computes the mean squared error over the n samples and its gradient
 * with respect to every parameter (grad: IB_MLP_NPARAM floats; partial: device workspace of
 * ib_mlpWorkspaceFloats(n) floats); loss_out (device, 1 float) may be NULL.  ib_mlpForward writes
 * the n outputs y.  ib_mlpAdam takes one Adam step (m, v: moment buffers, step >= 1). */
IB_API int64_t ib_mlpWorkspaceFloats(int64_t n);
IB_API int ib_mlpLossGrad(const float *params, const float *x, const float *target, int64_t n, float *grad,
                          float *loss_out, float *partial, void *stream);
IB_API int ib_mlpForward(const float *params, const float *x, int64_t n, float *y, void *stream);
IB_API int ib_mlpAdam(float *params, const float *grad, float *m, float *v, int64_t nparam, float lr, float beta1,
                      float beta2, float eps, int step, void *stream);

/* The same network on the tensor cores (tcgen05, BF16 weights and activations, FP32
 * accumulation, biases as BF16 high + low parts): y[i] for n rows of normalised features
 * x (n x 16; columns 14 and 15 are ignored). */
IB_API int ib_mlpInferTC(const float *params, const float *x, int64_t n, float *y, void *stream);

/* Exact training targets: for n samples with features f = (rho_gas, rho_dust, |dv|, u, dt)
 * (device, n x 5 doubles, the raw values) the LogTrap2 decay exponent s = dt * k_eff of
 * cudaSource2FluidDrag.cu:1531-1686 with the drag constants of thermo_gas/thermo_dust; s = 0 where
 * |dv| < 1e-9 (the reference's no-drag cut). */
IB_API int ib_dragDecayExact(const double *features, int64_t n, const ib_thermo *thermo_gas,
                             const ib_thermo *thermo_dust, double *s_out, void *stream);

/* Model handed to the learned drag step: params (device, IB_MLP_NPARAM FP32; converted to BF16
 * per call) and the normalisation. domain_lo/hi bound the five raw log-features the model was
 * trained on; cells outside take the exact path. */
typedef struct ib_drag_model {
    const float *params;
    float feature_shift[5], feature_scale[5];
    float out_shift, out_scale;
    float domain_lo[5], domain_hi[5];
} ib_drag_model;

/* Two-fluid drag over dt with the learned decay (same in-place update and argument meaning as
 * ib_cudaSource2FluidDrag with method LogTrap2): per cell the MLP runs on the tensor cores
 * (tcgen05, BF16 x BF16 -> FP32 in tensor memory) and the exact FP64 LogTrap2 takes over where
 * the cell fails the check: features outside the trained domain, or a predicted decay that is
 * not finite.  fallback_count (device, one unsigned long long, added to; may be NULL) counts
 * those cells. */
IB_API int ib_cudaSource2FluidDragLearned(ib_fluid *gas, ib_fluid *dust, const ib_thermo *thermo_gas,
                                          const ib_thermo *thermo_dust, const ib_drag_model *model, double dt,
                                          unsigned long long *fallback_count, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* IMOGEN_B200_H */
