// harness.cu -- host driver for the reference's own GPU code (test infrastructure).
//
// Links against the reference's gpuclass sources compiled from where they lie (see Makefile):
// sets up single-GPU MGArrays the way the reference's standalone driver does
// (generateDummyFluid, gpuclass/gpuimogen_core.cu:602-690: one 5-slab holder, slab k offset by
// k*slabPitch, numSlabs = -k), then calls the reference's own entry points:
//   performFluidUpdate_1D (cudaFluidStep.cu:233) in the sweep order of performFluidUpdate_3D
//   (flux.cu:27), flipArrayIndices (cudaArrayRotateB.cu:103), computeLocalCFLTimestep (cflTimestep.cu:107),
//   calculateSoundspeed (cudaSoundspeed.cu:107), sourcefunction_2FluidDrag
//   (cudaSource2FluidDrag.cu:189) and setFluidBoundary (boundaryConds.cu).
// The outputs become golden vectors for the tests (tests/golden/make_golden.py).
#include <csignal>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <execinfo.h>
#include <unistd.h>

#include "cudaCommon.h"
#include "cudaArrayRotateB.h"
#include "cudaFluidStep.h"
#include "cflTimestep.h"
#include "cudaSoundspeed.h"
#include "cudaSource2FluidDrag.h"
#include "cudaStatics.h"
#include "cudaSourceCylindricalTerms.h"

// One rank: the reference's halo exchange returns at once when its topology has a single rank
// in the exchange direction (cudaHaloExchange.cu:157-158); its source pulls in HDF5, so this
// stand-in does the same.
int exchange_MPI_Halos(MGArray *phi, int nArrays, ParallelTopology *topo, int xchgDir)
{
    (void)phi; (void)nArrays; (void)topo; (void)xchgDir;
    return SUCCESSFUL;
}

// The reference reports errors with printf; a fully buffered stdout would lose them if the
// process aborts, so stdout is made unbuffered and an abort prints the native call stack.
static void on_abort(int sig)
{
    void *frames[64];
    int n = backtrace(frames, 64);
    const char msg[] = "ref harness: abort, native stack:\n";
    write(2, msg, sizeof(msg) - 1);
    backtrace_symbols_fd(frames, n, 2);
    signal(sig, SIG_DFL);
    raise(sig);
}

__attribute__((constructor)) static void harness_init()
{
    setvbuf(stdout, NULL, _IONBF, 0);
    signal(SIGABRT, on_abort);
}

static int trace_on()
{
    static int t = -1;
    if (t < 0) { const char *e = getenv("IMOGEN_REF_TRACE"); t = (e && e[0] == '1') ? 1 : 0; }
    return t;
}
#define TRACE(...) do { if (trace_on()) { fprintf(stderr, __VA_ARGS__); fputc('\n', stderr); } } while (0)

static void make_topology(ParallelTopology *t)
{
    memset(t, 0, sizeof(*t));
    t->ndim = 3;
    t->comm = 0;
    for (int i = 0; i < 3; i++) { t->nproc[i] = 1; t->coord[i] = 0; t->dimcomm[i] = 0; }
    for (int i = 0; i < 8; i++) t->cudaStreamPtrs[i] = 0;
}

static GeometryParams make_geometry(int nx, int ny, int nz, const double h[3])
{
    GeometryParams g;
    memset(&g, 0, sizeof(g));
    g.shape = SQUARE;
    for (int i = 0; i < 3; i++) g.h[i] = h[i];
    g.globalRez[0] = nx; g.globalRez[1] = ny; g.globalRez[2] = nz;
    g.localRez[0] = nx; g.localRez[1] = ny; g.localRez[2] = nz;
    return g;
}

// Allocates a 5-slab holder and fills fl[0..4] (MGA_allocSlab, cudaCommon.cu:339-370)
static int make_fluid(MGArray *holder, MGArray fl[5], int nx, int ny, int nz, const int bc[6], int halo)
{
    MGArray sk;
    memset(&sk, 0, sizeof(sk));
    sk.dim[0] = nx; sk.dim[1] = ny; sk.dim[2] = nz;
    sk.numel = (int64_t)nx * ny * nz;
    sk.numSlabs = 1;
    sk.haloSize = halo;
    sk.partitionDir = PARTITION_X;
    sk.addExteriorHalo = 0;
    sk.currentPermutation[0] = 1; sk.currentPermutation[1] = 2; sk.currentPermutation[2] = 3;
    sk.permtag = MGA_numsToPermtag(&sk.currentPermutation[0]);
    sk.nGPUs = 1;
    sk.deviceID[0] = 0;
    sk.partNumel[0] = (int)sk.numel;
    int64_t bytes = sk.numel * (int64_t)sizeof(double);
    int64_t pitch = ((bytes + 255) / 256) * 256;
    sk.slabPitch[0] = pitch;
    for (int i = 0; i < 6; i++) sk.boundaryConditions.mode[i] = (BCModeTypes)bc[i];
    sk.vectorComponent = 0;
    int rc = MGA_allocSlab(&sk, holder, 5);
    if (rc != SUCCESSFUL) return rc;
    for (int k = 0; k < 5; k++) {
        fl[k] = *holder;
        fl[k].numSlabs = -k;
        fl[k].devicePtr[0] = holder->devicePtr[0] + k * (holder->slabPitch[0] / sizeof(double));
        fl[k].vectorComponent = (k >= 2) ? k - 1 : 0;
    }
    return SUCCESSFUL;
}

static void upload(MGArray *holder, const double *hq, int64_t hslab, int64_t n)
{
    for (int k = 0; k < 5; k++)
        cudaMemcpy(holder->devicePtr[0] + k * (holder->slabPitch[0] / 8), hq + k * hslab, n * 8, cudaMemcpyHostToDevice);
}

static void download(MGArray *holder, double *hq, int64_t hslab, int64_t n)
{
    for (int k = 0; k < 5; k++)
        cudaMemcpy(hq + k * hslab, holder->devicePtr[0] + k * (holder->slabPitch[0] / 8), n * 8, cudaMemcpyDeviceToHost);
}

static FluidMethods to_method(int m)
{
    return m == 1 ? METHOD_HLL : (m == 2 ? METHOD_HLLC : METHOD_XINJIN);
}

static int cfl_tau(MGArray fl[5], GeometryParams *geo, double gamma, int method, double *tau)
{
    MGArray cs;
    int rc = MGA_allocSlab(&fl[0], &cs, 1);
    TRACE("cs alloc rc %d", rc);
    if (rc != SUCCESSFUL) return rc;
    rc = calculateSoundspeed(&fl[0], NULL, &cs, gamma);
    TRACE("soundspeed rc %d", rc);
    if (rc != SUCCESSFUL) return rc;
    double rez[3] = {(double)geo->globalRez[0], (double)geo->globalRez[1], (double)geo->globalRez[2]};
    rc = computeLocalCFLTimestep(&fl[0], &cs, geo, method, rez, tau);
    MGA_delete(&cs);
    return rc;
}

// The 3-D fluid step: the sweep order and index permutations of performFluidUpdate_3D
// (flux.cu:27-156), each 1-D step, boundary fill and permutation done by the reference's own
// functions.  flux.cu itself is not linked: its standalone stream accessor getGPUTypeStreams
// (flux.cu:16-23) has no return statement, which g++ compiles to a function that runs on into
// whatever code follows it, so performFluidUpdate_3D crashes when built with g++ for NOMATLAB.
// The accessor's effect (two streams, taken from the topology) is reproduced here.
static int fluid_update_3d(MGArray *fluid, ParallelTopology *topo, FluidStepParams fsp)
{
    const int sweep = (fsp.stepNumber + 3 * (fsp.stepDirection > 0)) % 6;
    FluidStepParams sp = fsp;
    int rc;
    if (fluid->dim[1] == 1 && fluid->dim[2] == 1) {
        sp.stepDirection = 1;
        rc = performFluidUpdate_1D(fluid, sp, topo, (MGArray *)NULL);
        if (rc != SUCCESSFUL) return rc;
        rc = setFluidBoundary(fluid, &fsp.geometry, 1);
        if (rc != SUCCESSFUL) return rc;
        return exchange_MPI_Halos(fluid, 5, topo, 1);
    }
    static const int preperm[6] = {0, 2, 0, 2, 3, 3};
    static const int fluxcall[3][6] = {{1, 2, 1, 2, 3, 3}, {3, 1, 2, 3, 1, 2}, {2, 3, 3, 1, 2, 1}};
    static const int permcall[3][6] = {{3, 2, 2, 3, 3, 2}, {2, 3, 3, 5, 2, 6}, {6, 3, 5, 0, 2, 0}};
    cudaStream_t *streams = &topo->cudaStreamPtrs[0];
    MGArray tmp;
    memset(&tmp, 0, sizeof(tmp));
    tmp.nGPUs = -1;  // "not allocated": performFluidUpdate_1D allocates it on first use
    rc = preperm[sweep] ? flipArrayIndices(fluid, (MGArray **)NULL, 5, preperm[sweep], streams, (MGArray *)NULL)
                        : SUCCESSFUL;
    for (int n = 0; n < 3 && rc == SUCCESSFUL; n++) {
        const int dir = fluxcall[n][sweep];
        if (fluid->dim[0] > 3) {
            sp.stepDirection = dir;
            // Xin-Jin sweeps get NULL, so the reference allocates their temporary itself: its
            // Xin-Jin branch sets the kernels' scratch pointers (wStepValues, a local array,
            // cudaFluidStep.cu:315) only when it allocates the temporary (:362-371), so with a
            // temporary that an earlier sweep or transpose already allocated the pressure/freeze
            // and Xin-Jin kernels would get uninitialised pointers (performFluidUpdate_3D,
            // flux.cu, passes one temporary to every sweep of a step)
            rc = performFluidUpdate_1D(fluid, sp, topo, sp.stepMethod == METHOD_XINJIN ? (MGArray *)NULL : &tmp);
            if (rc == SUCCESSFUL) rc = setFluidBoundary(fluid, &fsp.geometry, dir);
            if (rc == SUCCESSFUL) rc = exchange_MPI_Halos(fluid, 5, topo, dir);
        }
        if (rc == SUCCESSFUL && permcall[n][sweep])
            rc = flipArrayIndices(fluid, (MGArray **)NULL, 5, permcall[n][sweep], streams, &tmp);
    }
    if (tmp.nGPUs != -1) {
        int rd = MGA_delete(&tmp);
        if (rc == SUCCESSFUL) rc = rd;
    }
    return rc;
}

extern "C" {

// Runs `niter` main-loop iterations (CFL, forward fluid step, backward fluid step) of one fluid
// with the reference's code.  hq: host (5, hslab) doubles, in/out.  dts_out[niter] receives dt.
int ref_run(double *hq, int nx, int ny, int nz, int64_t hslab, double gamma, double rho_min, double c_iso,
            int method, const double *h, const int *bc, double cfl, int niter, double *dts_out)
{
    MGArray holder, fl[5];
    TRACE("ref_run %dx%dx%d method %d", nx, ny, nz, method);
    int rc = make_fluid(&holder, fl, nx, ny, nz, bc, 4);
    TRACE("make_fluid rc %d", rc);
    if (rc != SUCCESSFUL) return rc;
    const int64_t n = (int64_t)nx * ny * nz;
    upload(&holder, hq, hslab, n);
    ParallelTopology topo;
    make_topology(&topo);
    GeometryParams geo = make_geometry(nx, ny, nz, h);
    FluidStepParams fsp;
    memset(&fsp, 0, sizeof(fsp));
    fsp.onlyHydro = 1;
    fsp.thermoGamma = (c_iso != -1) ? 2.0 : gamma;  // flux_ML_iface.cu:140-143
    fsp.Cisothermal = c_iso;
    fsp.minimumRho = rho_min;
    fsp.stepMethod = to_method(method);
    fsp.geometry = geo;
    for (int it = 0; it < niter && rc == SUCCESSFUL; it++) {
        double tau = 0;
        rc = cfl_tau(fl, &geo, gamma, method, &tau);
        TRACE("it %d cfl rc %d tau %g", it, rc, tau);
        if (rc != SUCCESSFUL) break;
        fsp.dt = cfl * tau;
        fsp.stepNumber = it;
        dts_out[it] = fsp.dt;
        fsp.stepDirection = 1;
        rc = fluid_update_3d(&fl[0], &topo, fsp);
        TRACE("it %d forward rc %d", it, rc);
        if (rc != SUCCESSFUL) break;
        fsp.stepDirection = -1;
        rc = fluid_update_3d(&fl[0], &topo, fsp);
        TRACE("it %d backward rc %d", it, rc);
    }
    cudaDeviceSynchronize();
    download(&holder, hq, hslab, n);
    MGA_delete(&holder);
    return rc;
}

// CFL timestep of one fluid (cudaSoundspeed + cflTimestep mex pair)
int ref_cfl(const double *hq, int nx, int ny, int nz, int64_t hslab, double gamma, int method, const double *h,
            double *tau_out)
{
    MGArray holder, fl[5];
    const int bc[6] = {0, 0, 0, 0, 0, 0};
    int rc = make_fluid(&holder, fl, nx, ny, nz, bc, 4);
    if (rc != SUCCESSFUL) return rc;
    upload(&holder, hq, hslab, (int64_t)nx * ny * nz);
    GeometryParams geo = make_geometry(nx, ny, nz, h);
    rc = cfl_tau(fl, &geo, gamma, method, tau_out);
    MGA_delete(&holder);
    return rc;
}

// Two-fluid drag over dt with the reference's integrator `method` (0..5)
int ref_drag(double *hgas, double *hdust, int nx, int ny, int nz, int64_t hslab, const double *tg, const double *td,
             double dt, int method)
{
    MGArray hg, hd, g[5], d[5];
    const int bc[6] = {0, 0, 0, 0, 0, 0};
    int rc = make_fluid(&hg, g, nx, ny, nz, bc, 4);
    if (rc != SUCCESSFUL) return rc;
    rc = make_fluid(&hd, d, nx, ny, nz, bc, 4);
    if (rc != SUCCESSFUL) return rc;
    const int64_t n = (int64_t)nx * ny * nz;
    upload(&hg, hgas, hslab, n);
    upload(&hd, hdust, hslab, n);
    ThermoDetails a, b;
    memset(&a, 0, sizeof(a));
    memset(&b, 0, sizeof(b));
    a.gamma = tg[0]; a.m = tg[1]; a.mu0 = tg[2]; a.muTindex = tg[3]; a.sigma0 = tg[4]; a.sigmaTindex = tg[5];
    a.kBolt = tg[6]; a.Cisothermal = tg[7];
    b.gamma = td[0]; b.m = td[1]; b.mu0 = td[2]; b.muTindex = td[3]; b.sigma0 = td[4]; b.sigmaTindex = td[5];
    b.kBolt = td[6]; b.Cisothermal = td[7];
    double h[3] = {1.0 / nx, 1.0 / ny, 1.0 / nz};
    GeometryParams geo = make_geometry(nx, ny, nz, h);
    rc = sourcefunction_2FluidDrag(&g[0], &d[0], &geo, &a, &b, dt, method);
    cudaDeviceSynchronize();
    download(&hg, hgas, hslab, n);
    download(&hd, hdust, hslab, n);
    MGA_delete(&hg);
    MGA_delete(&hd);
    return rc;
}

// Times `niter` iterations of the reference's own fluid loop on the device (ms, CUDA events)
int ref_time(double *hq, int nx, int ny, int nz, int64_t hslab, double gamma, int method, const double *h,
             double cfl, int nwarm, int niter, double *ms_out)
{
    MGArray holder, fl[5];
    const int bc[6] = {0, 0, 0, 0, 0, 0};
    int rc = make_fluid(&holder, fl, nx, ny, nz, bc, 4);
    if (rc != SUCCESSFUL) return rc;
    upload(&holder, hq, hslab, (int64_t)nx * ny * nz);
    ParallelTopology topo;
    make_topology(&topo);
    GeometryParams geo = make_geometry(nx, ny, nz, h);
    FluidStepParams fsp;
    memset(&fsp, 0, sizeof(fsp));
    fsp.onlyHydro = 1;
    fsp.thermoGamma = gamma;
    fsp.Cisothermal = -1;
    fsp.minimumRho = 1e-5;
    fsp.stepMethod = to_method(method);
    fsp.geometry = geo;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int it = 0; it < nwarm + niter && rc == SUCCESSFUL; it++) {
        if (it == nwarm) {
            cudaDeviceSynchronize();
            cudaEventRecord(e0, 0);
        }
        double tau = 0;
        rc = cfl_tau(fl, &geo, gamma, method, &tau);
        fsp.dt = cfl * tau;
        fsp.stepNumber = it;
        fsp.stepDirection = 1;
        if (rc == SUCCESSFUL) rc = fluid_update_3d(&fl[0], &topo, fsp);
        fsp.stepDirection = -1;
        if (rc == SUCCESSFUL) rc = fluid_update_3d(&fl[0], &topo, fsp);
    }
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    *ms_out = ms;
    MGA_delete(&holder);
    return rc;
}

// ---- cylindrical geometry (x = r, y = theta, z = z) ----

static GeometryParams make_cyl_geometry(int nx, int ny, int nz, const double h[3], double r_inner)
{
    GeometryParams g = make_geometry(nx, ny, nz, h);
    g.shape = CYLINDRICAL;
    g.Rinner = r_inner;
    return g;
}

// One cylindrical sweep along dir with the reference's performFluidUpdate_1D.  A theta sweep
// (dir 2) runs on the array permuted so that theta is fastest: form 0 = layout theta,r,z
// (exchange X and Y, code 2), form 1 = theta,z,r (rotate left, code 5); the array is permuted
// back afterwards.  No boundary fill.
int ref_sweep_cyl(double *hq, int nx, int ny, int nz, int64_t hslab, double gamma, double rho_min, double c_iso,
                  int method, const double *h, double r_inner, int dir, int form, double dt)
{
    MGArray holder, fl[5];
    const int bc[6] = {0, 0, 0, 0, 0, 0};
    int rc = make_fluid(&holder, fl, nx, ny, nz, bc, 4);
    if (rc != SUCCESSFUL) return rc;
    const int64_t n = (int64_t)nx * ny * nz;
    upload(&holder, hq, hslab, n);
    ParallelTopology topo;
    make_topology(&topo);
    cudaStream_t *streams = &topo.cudaStreamPtrs[0];
    FluidStepParams fsp;
    memset(&fsp, 0, sizeof(fsp));
    fsp.onlyHydro = 1;
    fsp.thermoGamma = (c_iso != -1) ? 2.0 : gamma;
    fsp.Cisothermal = c_iso;
    fsp.minimumRho = rho_min;
    fsp.stepMethod = to_method(method);
    fsp.geometry = make_cyl_geometry(nx, ny, nz, h, r_inner);
    fsp.dt = dt;
    fsp.stepDirection = dir;
    const int pre = (dir == 2) ? (form == 0 ? 2 : 5) : 0;
    const int post = (dir == 2) ? (form == 0 ? 2 : 6) : 0;
    if (pre) rc = flipArrayIndices(&fl[0], (MGArray **)NULL, 5, pre, streams, (MGArray *)NULL);
    if (rc == SUCCESSFUL) rc = performFluidUpdate_1D(&fl[0], fsp, &topo, (MGArray *)NULL);
    if (rc == SUCCESSFUL && post) rc = flipArrayIndices(&fl[0], (MGArray **)NULL, 5, post, streams, (MGArray *)NULL);
    cudaDeviceSynchronize();
    download(&holder, hq, hslab, n);
    MGA_delete(&holder);
    return rc;
}

// The cylindrical source over dt on an XYZ-ordered fluid (sourcefunction_CylindricalTerms)
int ref_cyl_source(double *hq, int nx, int ny, int nz, int64_t hslab, const double *h, double r_inner, double dt)
{
    MGArray holder, fl[5];
    const int bc[6] = {0, 0, 0, 0, 0, 0};
    int rc = make_fluid(&holder, fl, nx, ny, nz, bc, 4);
    if (rc != SUCCESSFUL) return rc;
    const int64_t n = (int64_t)nx * ny * nz;
    upload(&holder, hq, hslab, n);
    double hh[3] = {h[0], h[1], h[2]};
    rc = sourcefunction_CylindricalTerms(&fl[0], dt, &hh[0], r_inner);
    cudaDeviceSynchronize();
    download(&holder, hq, hslab, n);
    MGA_delete(&holder);
    return rc;
}

// CFL timestep in cylindrical geometry
int ref_cfl_cyl(const double *hq, int nx, int ny, int nz, int64_t hslab, double gamma, int method, const double *h,
                double r_inner, double *tau_out)
{
    MGArray holder, fl[5];
    const int bc[6] = {0, 0, 0, 0, 0, 0};
    int rc = make_fluid(&holder, fl, nx, ny, nz, bc, 4);
    if (rc != SUCCESSFUL) return rc;
    upload(&holder, hq, hslab, (int64_t)nx * ny * nz);
    GeometryParams geo = make_cyl_geometry(nx, ny, nz, h, r_inner);
    rc = cfl_tau(fl, &geo, gamma, method, tau_out);
    MGA_delete(&holder);
    return rc;
}

// One-fluid main loop in cylindrical geometry, as performCompleteTimestep runs it with the
// cylinder-only source (srcType 1, flux_multi.cu:161-250; srcC___, sourceStep.cu:498-518):
// CFL, source dt/2, forward step, source dt, backward step, source dt/2, each source followed by
// the boundary fill of directions 1, 2, 3 (setAllBoundaryConditions, sourceStep.cu:276-291).
int ref_run_cyl(double *hq, int nx, int ny, int nz, int64_t hslab, double gamma, double rho_min, double c_iso,
                int method, const double *h, double r_inner, const int *bc, double cfl, int niter, double *dts_out)
{
    MGArray holder, fl[5];
    int rc = make_fluid(&holder, fl, nx, ny, nz, bc, 4);
    if (rc != SUCCESSFUL) return rc;
    const int64_t n = (int64_t)nx * ny * nz;
    upload(&holder, hq, hslab, n);
    ParallelTopology topo;
    make_topology(&topo);
    GeometryParams geo = make_cyl_geometry(nx, ny, nz, h, r_inner);
    FluidStepParams fsp;
    memset(&fsp, 0, sizeof(fsp));
    fsp.onlyHydro = 1;
    fsp.thermoGamma = (c_iso != -1) ? 2.0 : gamma;
    fsp.Cisothermal = c_iso;
    fsp.minimumRho = rho_min;
    fsp.stepMethod = to_method(method);
    fsp.geometry = geo;
    auto source = [&](double dt) {
        int r = sourcefunction_CylindricalTerms(&fl[0], dt, &geo.h[0], geo.Rinner);
        for (int d = 1; d <= 3 && r == SUCCESSFUL; d++) r = setFluidBoundary(&fl[0], &geo, d);
        return r;
    };
    for (int it = 0; it < niter && rc == SUCCESSFUL; it++) {
        double tau = 0;
        rc = cfl_tau(fl, &geo, gamma, method, &tau);
        if (rc != SUCCESSFUL) break;
        fsp.dt = cfl * tau;
        fsp.stepNumber = it;
        dts_out[it] = fsp.dt;
        rc = source(0.5 * fsp.dt);
        fsp.stepDirection = 1;
        if (rc == SUCCESSFUL) rc = fluid_update_3d(&fl[0], &topo, fsp);
        if (rc == SUCCESSFUL) rc = source(fsp.dt);
        fsp.stepDirection = -1;
        if (rc == SUCCESSFUL) rc = fluid_update_3d(&fl[0], &topo, fsp);
        if (rc == SUCCESSFUL) rc = source(0.5 * fsp.dt);
    }
    cudaDeviceSynchronize();
    download(&holder, hq, hslab, n);
    MGA_delete(&holder);
    return rc;
}

}  // extern "C"
