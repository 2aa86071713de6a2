// ib_capi.cu -- extern "C" entry points (include/imogen_b200.h) and host orchestration.
//
// Host logic restated from the reference's mex glue and orchestration:
//   ib_cudaFluidStep       <- cudaFluidStep.cu:161-227 + performFluidUpdate_1D :233-663
//   ib_fluidstep           <- flux_ML_iface.cu:37-160 + performFluidUpdate_3D flux.cu:27-165
//   ib_cflTimestep(Fused)  <- cflTimestep.cu:64-252, cudaSoundspeed.cu:54-150
//   ib_freezeAndPtot       <- freezeAndPtot.cu:32-147
//   ib_cudaStatics         <- cudaStatics.cu:85-104, 199-350
//   ib_setFluidBoundary    <- cudaStatics.cu:112-197
//   ib_cudaSource2FluidDrag<- cudaSource2FluidDrag.cu:125-246
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>

#include "ib_internal.cuh"
#include "ib_sweep_launch.cuh"

namespace ib {

static thread_local int g_last_cuda_error = 0;

int check_cuda(cudaError_t e)
{
    if (e != cudaSuccess) {
        g_last_cuda_error = (int)e;
        return (e == cudaErrorMemoryAllocation) ? IB_ERROR_NOMEM : IB_ERROR_CUDA;
    }
    return IB_SUCCESSFUL;
}

static std::atomic<long long> g_launches{0};

int check_launch()
{
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return check_cuda(cudaGetLastError());
}

int num_sms()
{
    static int cache[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (cache[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cache[dev] = v;
    }
    return cache[dev];
}

static std::atomic<long long> g_tile_wait_limit{-1};

int pair_min_cells()
{
    static const int v = [] {
        const char *e = getenv("IMOGEN_B200_PAIRMIN");
        return e ? atoi(e) : 64;
    }();
    return v;
}

uint32_t tile_wait_limit()
{
    const long long v = g_tile_wait_limit.load(std::memory_order_relaxed);
    return v < 0 ? (uint32_t)IB_TMA_SPIN_LIMIT : (uint32_t)v;
}

static std::mutex g_scratch_mu;

Scratch &scratch()
{
    static Scratch per_dev[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    return per_dev[dev];
}

double *Scratch::cfl_partial(int nblocks)
{
    std::lock_guard<std::mutex> g(g_scratch_mu);
    if (nblocks > partial_n_) {
        if (partial_) cudaFree(partial_);
        partial_ = nullptr;
        partial_n_ = 0;
        // room for every grid the CFL launch sizes (at most 8 resident 256-thread blocks per SM),
        // so the array is never replaced under a CUDA graph that captured its address
        const int cap = std::max(nblocks, 8 * num_sms());
        if (cudaMalloc(&partial_, sizeof(double) * cap) != cudaSuccess) return nullptr;
        partial_n_ = cap;
    }
    return partial_;
}

unsigned int *Scratch::cfl_counter()
{
    std::lock_guard<std::mutex> g(g_scratch_mu);
    if (!counter_) {
        if (cudaMalloc(&counter_, sizeof(unsigned int)) != cudaSuccess) { counter_ = nullptr; return nullptr; }
        if (cudaMemset(counter_, 0, sizeof(unsigned int)) != cudaSuccess) return nullptr;
    }
    return counter_;
}

// The CFL kernel's last block writes the timestep straight into pinned, mapped host memory, so
// reading it back needs no copy-engine transfer: a device-to-host copy would queue behind any
// large download the caller has running on another stream (a 671 MB state read-out held each
// timestep read for ~13 ms) while the kernel's store does not.
double *Scratch::cfl_tau()
{
    std::lock_guard<std::mutex> g(g_scratch_mu);
    if (!tau_) {
        void *h = nullptr, *d = nullptr;
        if (cudaHostAlloc(&h, sizeof(double), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess)
            return nullptr;
        if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
            cudaFreeHost(h);
            return nullptr;
        }
        tau_host_ = static_cast<double *>(h);
        tau_ = static_cast<double *>(d);
    }
    return tau_;
}

volatile double *Scratch::cfl_tau_host() { return tau_host_; }

unsigned int *Scratch::wait_flag()
{
    std::lock_guard<std::mutex> g(g_scratch_mu);
    if (!wait_flag_) {
        if (cudaMalloc(&wait_flag_, sizeof(unsigned int)) != cudaSuccess) { wait_flag_ = nullptr; return nullptr; }
        if (cudaMemset(wait_flag_, 0, sizeof(unsigned int)) != cudaSuccess) return nullptr;
    }
    return wait_flag_;
}

unsigned int *Scratch::ensemble_counter()
{
    std::lock_guard<std::mutex> g(g_scratch_mu);
    if (!ens_counter_) {
        if (cudaMalloc(&ens_counter_, sizeof(unsigned int)) != cudaSuccess) { ens_counter_ = nullptr; return nullptr; }
    }
    return ens_counter_;
}

double *Scratch::bytes(size_t nbytes)
{
    std::lock_guard<std::mutex> g(g_scratch_mu);
    if (nbytes > gen_n_) {
        if (gen_) cudaFree(gen_);
        gen_ = nullptr;
        gen_n_ = 0;
        if (cudaMalloc(&gen_, nbytes) != cudaSuccess) return nullptr;
        gen_n_ = nbytes;
    }
    return gen_;
}

int launch_sweep(int method, int slope, int precision, int dir, double *q, int64_t slab, const int grid[3],
                 DevScalar lambda, double gamma, double rho_min, double c_iso, cudaStream_t st, int nsweep)
{
    if (method == IB_METHOD_HLLC) {
        if (precision == IB_PREC_FP32_FLUX)
            return launch_hllc32(slope, dir, q, slab, grid, lambda, gamma, rho_min, c_iso, st, nsweep);
        return launch_hllc64(slope, dir, q, slab, grid, lambda, gamma, rho_min, c_iso, st, nsweep);
    }
    if (method == IB_METHOD_HLL)
        return launch_hll64(slope, dir, q, slab, grid, lambda, gamma, rho_min, c_iso, st, nsweep);
    return IB_ERROR_INVALID_ARGS;
}

// ---------------------------------------------------------------------------------------------
// Validation helpers
// ---------------------------------------------------------------------------------------------
static int validate_grid(const ib_grid &g)
{
    if (g.nx < 1 || g.ny < 1 || g.nz < 1) return IB_ERROR_INVALID_ARGS;
    int64_t n = (int64_t)g.nx * g.ny * g.nz;
    if (g.slab_pitch < n) return IB_ERROR_INVALID_ARGS;
    if (n > ((int64_t)1 << 31)) return IB_ERROR_INVALID_ARGS;  // 32-bit cell indices in the reductions
    return IB_SUCCESSFUL;
}

static int validate_fluid(const ib_fluid *f)
{
    if (!f || !f->q) return IB_ERROR_NULL_POINTER;
    int rc = validate_grid(f->grid);
    if (rc) return rc;
    for (int i = 0; i < 6; i++)
        if (f->bc[i] < IB_BC_CIRCULAR || f->bc[i] > IB_BC_FREEBALANCE) return IB_ERROR_INVALID_ARGS;
    if (f->halo < 1 || f->halo > 8) return IB_ERROR_INVALID_ARGS;
    return IB_SUCCESSFUL;
}

struct Numerics {
    int slope = IB_SLOPE_OSPRE, flim = IB_FLUX_OSPRE, prec = IB_PREC_FP64, flags = 0;
};

static int get_numerics(const ib_numerics *num, Numerics &n)
{
    if (num) {
        n.slope = num->slope_limiter;
        n.flim = num->flux_limiter;
        n.prec = num->precision;
        n.flags = num->flags;
    }
    if (n.slope < IB_SLOPE_OSPRE || n.slope > IB_SLOPE_ZERO) return IB_ERROR_INVALID_ARGS;
    if (n.flim < IB_FLUX_OSPRE || n.flim > IB_FLUX_ZERO) return IB_ERROR_INVALID_ARGS;
    if (n.prec != IB_PREC_FP64 && n.prec != IB_PREC_FP32_FLUX) return IB_ERROR_INVALID_ARGS;
    if (n.flags & ~IB_FLAG_CYL_GEOMETRIC_RADIUS) return IB_ERROR_INVALID_ARGS;
    return IB_SUCCESSFUL;
}

static bool geometry_ok(const ib_geometry *geo)
{
    return geo->shape == IB_GEOMETRY_SQUARE || geo->shape == IB_GEOMETRY_CYLINDRICAL;
}

// The cylindrical form of a sweep along dir (cudaFluidStep.cu:264-278): x = r, y = theta (z
// sweeps are plain).  theta_layout: 0 = the reference's memory layout theta,r,z (FLUX_THETA_213),
// 1 = theta,z,r (FLUX_THETA_231).  The theta radius rule (ib_cyl.cuh): the cell centre radius
// with IB_FLAG_CYL_GEOMETRIC_RADIUS, else the reference's arithmetic with the theta cell size as
// its radial step, whose launch treats the radial axis as the second one when a theta,z,r grid
// has nz = 1 (block index, and so the radius term, 0) and the z axis as the second one when a
// theta,r,z grid has nx = 1 < nz (cudaFluidStep.cu:325-329).
static CylSweep cyl_sweep(const ib_geometry *geo, const ib_grid &g, int dir, int theta_layout, const Numerics &nm)
{
    CylSweep cs{CYL_NONE, CylPencil{0.0, 0.0, 0, 0}};
    if (geo->shape != IB_GEOMETRY_CYLINDRICAL || dir == 3) return cs;
    if (dir == 1) {
        cs.kind = CYL_RADIAL;
        cs.pencil = CylPencil{geo->r_inner, geo->h[0], RMODE_GEOMETRIC, 0};
        return cs;
    }
    cs.kind = theta_layout ? CYL_THETA_LAM : CYL_THETA_DIV;
    if (nm.flags & IB_FLAG_CYL_GEOMETRIC_RADIUS)
        cs.pencil = CylPencil{geo->r_inner, geo->h[0], RMODE_GEOMETRIC, 0};
    else if (theta_layout)
        cs.pencil = CylPencil{geo->r_inner, geo->h[1], g.nz == 1 ? RMODE_INNER : RMODE_INDEX, 0};
    else
        cs.pencil = CylPencil{geo->r_inner, geo->h[1], RMODE_ACC4, (g.nx == 1 && g.nz > 1) ? 1 : 0};
    return cs;
}

// Which theta layout the theta sweep of a fluid step has in the reference: the permutations of
// performFluidUpdate_3D (flux.cu:46-49, cudaArrayRotateB.cu:580-643) leave r third in memory for
// sweep indices 0 and 5, second for the others.
static int theta_layout_of(int sweep_dir, int step_number)
{
    const int sweep = (step_number + 3 * (sweep_dir > 0)) % 6;
    return (sweep == 0 || sweep == 5) ? 1 : 0;
}

// The timestep of a call: a host value, or the address of a device value that the kernels read
// themselves (loops that keep dt on the device and replay a captured graph).
struct StepDt {
    double dt;
    const double *dtp;
    // a sweep's lambda = dt / h (the same division in either form)
    DevScalar lambda(double h) const { return dtp ? DevScalar::device(dtp, 1.0, h) : DevScalar::of(dt / h); }
    // frac * dt for a source step (frac 1 or 1/2: exact in either form)
    DevScalar part(double frac) const { return dtp ? DevScalar::device(dtp, frac, 1.0) : DevScalar::of(frac * dt); }
};

// One directional update (performFluidUpdate_1D); gamma already 2 for isothermal fluids.  With
// nsweep = 2 the same update is applied twice in a row (HLL/HLLC: one launch where the kernel
// allows it; Xin-Jin: two launches).
static int fluid_update_1d(ib_fluid *f, const ib_geometry *geo, int method, int dir, const StepDt &dt, double gamma,
                           double rho_min, double c_iso, const Numerics &nm, cudaStream_t st, int nsweep = 1,
                           int theta_layout = 0)
{
    const int grid[3] = {f->grid.nx, f->grid.ny, f->grid.nz};
    if (grid[dir - 1] < 3) return IB_SUCCESSFUL;  // cudaFluidStep.cu:313
    const DevScalar lambda = dt.lambda(geo->h[dir - 1]);
    const CylSweep cs = cyl_sweep(geo, f->grid, dir, theta_layout, nm);
    if (method == IB_METHOD_XINJIN) {
        for (int k = 0; k < nsweep; k++) {
            int rc = launch_xj_sweep(nm.flim, dir, f->q, f->grid.slab_pitch, grid, lambda, gamma, rho_min, st,
                                     cs.kind != CYL_NONE ? &cs : nullptr);
            if (rc) return rc;
        }
        return IB_SUCCESSFUL;
    }
    if (cs.kind != CYL_NONE) {
        if (nm.prec != IB_PREC_FP64) return IB_ERROR_NOIMPLEMENT;  // cylindrical sweeps are FP64
        for (int k = 0; k < nsweep; k++) {
            int rc = launch_sweep_cyl(method, nm.slope, f->q, f->grid.slab_pitch, grid, lambda, gamma, rho_min, c_iso,
                                      st, cs);
            if (rc) return rc;
        }
        return IB_SUCCESSFUL;
    }
    return launch_sweep(method, nm.slope, nm.prec, dir, f->q, f->grid.slab_pitch, grid, lambda, gamma, rho_min, c_iso,
                        st, nsweep);
}

static bool has_statics(const ib_fluid *f)
{
    for (int k = 0; k < 5; k++)
        if (f->statics[k].data && f->statics[k].count > 0) return true;
    return false;
}

// setFluidBoundary (cudaStatics.cu:112-197): statics of the density array, then per side the
// statics of every array followed by that side's condition.
static int fluid_boundary(ib_fluid *f, int dir, cudaStream_t st)
{
    const int grid[3] = {f->grid.nx, f->grid.ny, f->grid.nz};
    const int64_t S = f->grid.slab_pitch;
    int rc;
    if (!has_statics(f)) return launch_fluid_boundary(f->q, S, grid, f->bc, f->halo, dir, st);
    const int64_t numel = (int64_t)grid[0] * grid[1] * grid[2];
    if ((rc = launch_statics(f->q, &f->statics[0], numel, st))) return rc;
    for (int side = 0; side < 2; side++) {
        for (int k = 0; k < 5; k++)
            if ((rc = launch_statics(f->q + k * S, &f->statics[k], numel, st))) return rc;
        int32_t bc1[6];
        memcpy(bc1, f->bc, sizeof(bc1));
        bc1[2 * (dir - 1) + (1 - side)] = IB_BC_CIRCULAR;
        if ((rc = launch_fluid_boundary(f->q, S, grid, bc1, f->halo, dir, st))) return rc;
    }
    return IB_SUCCESSFUL;
}

// The sweep directions of one fluid step (performFluidUpdate_3D, flux.cu:27-165): sweep index
// (iteration + 3 [direction > 0]) mod 6 selects a row of the ordering table (flux.cu:46-49).  The
// backward step's order is the forward one's reversed, so the last sweep of the forward step and
// the first of the backward step are along the same axis.
static void sweep_order(int step_number, int sweep_dir, int out[3])
{
    static const int fluxcall[3][6] = {{1, 2, 1, 2, 3, 3}, {3, 1, 2, 3, 1, 2}, {2, 3, 3, 1, 2, 1}};
    const int sweep = (step_number + 3 * (sweep_dir > 0)) % 6;
    for (int n = 0; n < 3; n++) out[n] = fluxcall[n][(sweep + 6) % 6];
}

struct FluidParams {
    double gamma, rho_min, c_iso;
};

static FluidParams fluid_params(const ib_fluid_thermo &t)
{
    FluidParams p{t.gamma, t.rho_min, t.c_isothermal};
    if (p.c_iso != -1) p.gamma = 2;  // flux_ML_iface.cu:140-143
    return p;
}

// One sweep of a fluid step and the boundary fill after it (flux.cu:102-110).
static int sweep_and_fill(ib_fluid *f, const ib_geometry *geo, int method, int d, const StepDt &dt, const FluidParams &fp,
                          const Numerics &nm, cudaStream_t st, int nsweep = 1, int theta_layout = 0)
{
    const int ext[3] = {f->grid.nx, f->grid.ny, f->grid.nz};
    if (ext[d - 1] <= 3) return IB_SUCCESSFUL;
    int rc = fluid_update_1d(f, geo, method, d, dt, fp.gamma, fp.rho_min, fp.c_iso, nm, st, nsweep, theta_layout);
    if (rc) return rc;
    return fluid_boundary(f, d, st);
}

// One fluid step (forward or backward) of one fluid, all three sweeps; 1-D grids take the
// shortcut of flux.cu:35-68 (one x sweep).
static int fluid_step_one(ib_fluid *f, const ib_geometry *geo, int method, const StepDt &dt, const FluidParams &fp,
                          const Numerics &nm, int sweep_dir, int step_number, cudaStream_t st)
{
    const int ext[3] = {f->grid.nx, f->grid.ny, f->grid.nz};
    if (ext[1] == 1 && ext[2] == 1) {
        int rc = fluid_update_1d(f, geo, method, 1, dt, fp.gamma, fp.rho_min, fp.c_iso, nm, st);
        if (rc) return rc;
        return fluid_boundary(f, 1, st);
    }
    int order[3];
    sweep_order(step_number, sweep_dir, order);
    const int layout = theta_layout_of(sweep_dir, step_number);
    for (int n = 0; n < 3; n++) {
        int rc = sweep_and_fill(f, geo, method, order[n], dt, fp, nm, st, 1, layout);
        if (rc) return rc;
    }
    return IB_SUCCESSFUL;
}

// Forward then backward fluid step of one fluid with nothing in between.  The forward step's
// last sweep and the backward step's first are along the same axis d with the same dt; when the
// boundary fill between them does nothing (both faces of d periodic, no statics) they are one
// double-sweep launch: the same updates in the same order, so the result is identical.
static int fluid_fwd_bwd(ib_fluid *f, const ib_geometry *geo, int method, const StepDt &dt, const FluidParams &fp,
                         const Numerics &nm, int step_number, cudaStream_t st)
{
    const int ext[3] = {f->grid.nx, f->grid.ny, f->grid.nz};
    const bool one_d = ext[1] == 1 && ext[2] == 1;
    int fwd[3], bwd[3];
    if (one_d) {
        fwd[0] = fwd[1] = fwd[2] = 1;
    } else {
        sweep_order(step_number, 1, fwd);
        sweep_order(step_number, -1, bwd);
    }
    const int d = one_d ? 1 : fwd[2];
    // (cylindrical: the two steps' theta sweeps can differ in form, so they stay apart)
    const bool fuse = (one_d || bwd[0] == d) && ext[d - 1] > 3 && f->bc[2 * (d - 1)] == IB_BC_CIRCULAR &&
                      f->bc[2 * (d - 1) + 1] == IB_BC_CIRCULAR && !has_statics(f) &&
                      geo->shape == IB_GEOMETRY_SQUARE;
    if (!fuse) {
        int rc = fluid_step_one(f, geo, method, dt, fp, nm, 1, step_number, st);
        if (rc) return rc;
        return fluid_step_one(f, geo, method, dt, fp, nm, -1, step_number, st);
    }
    int rc;
    if (!one_d)
        for (int n = 0; n < 2; n++)
            if ((rc = sweep_and_fill(f, geo, method, fwd[n], dt, fp, nm, st))) return rc;
    if ((rc = sweep_and_fill(f, geo, method, d, dt, fp, nm, st, 2))) return rc;
    if (!one_d)
        for (int n = 1; n < 3; n++)
            if ((rc = sweep_and_fill(f, geo, method, bwd[n], dt, fp, nm, st))) return rc;
    return IB_SUCCESSFUL;
}

// Two-fluid drag over dt (sourcefunction_2FluidDrag, cudaSource2FluidDrag.cu:189-246): the drag
// constants of the two fluids' microphysics, then the integrator's kernel(s).
static int drag_source(ib_fluid *gas, ib_fluid *dust, const ib_thermo *tg, const ib_thermo *td,
                       const ib_geometry *geo, DevScalar dt, int method, cudaStream_t st)
{
    int rc;
    if (!gas || !dust || !tg || !td || !gas->q || !dust->q) return IB_ERROR_NULL_POINTER;
    if ((rc = validate_grid(gas->grid))) return rc;
    if (gas->grid.nx != dust->grid.nx || gas->grid.ny != dust->grid.ny || gas->grid.nz != dust->grid.nz ||
        gas->grid.slab_pitch != dust->grid.slab_pitch)
        return IB_ERROR_INVALID_ARGS;
    if (method < IB_DRAG_EMP || method > IB_DRAG_LOGTRAP3) return IB_ERROR_INVALID_ARGS;
    // drag constants (cudaSource2FluidDrag.cu:196-218; dragparams[7] = dt goes to the kernels
    // separately)
    double dp[11];
    const double gam = tg->gamma;
    const double ddust = sqrt(td->sigma0 / 3.141592653589793);
    dp[0] = tg->mu0;
    dp[1] = -tg->mu_t_index;
    dp[2] = tg->sigma_t_index;
    dp[3] = tg->mass * (gam - 1.0) / (298.15 * tg->k_bolt);
    dp[4] = sqrt(2.0) * tg->mass / (tg->sigma0 * ddust);
    dp[5] = ddust / tg->mu0;
    dp[6] = td->sigma0 / (1.0 * td->mass);
    dp[7] = 0.0;
    dp[8] = (gam - 1.0);
    dp[9] = .25 * td->sigma0 / td->mass;
    dp[10] = 16 * (gam - 1.0) / 3.0;
    const int grid[3] = {gas->grid.nx, gas->grid.ny, gas->grid.nz};
    if (method == IB_DRAG_ETDRK2) {
        // the pressure gradient needs the cell sizes (prepareForExpMethod, cudaSource2FluidDrag.cu:1728-1741)
        if (!geo) return IB_ERROR_NULL_POINTER;
        if (geo->shape != 0) return IB_ERROR_NOIMPLEMENT;  // cylindrical gradients: out of scope
    }
    return launch_drag(gas->q, dust->q, gas->grid.slab_pitch, grid, geo ? geo->h : nullptr, dp, dt, method, st);
}

// performCompleteTimestep (flux_multi.cu:174-272); params = [purehydro, iteration, method].
static int complete_timestep(ib_fluid *fluids, const ib_fluid_thermo *thermo, int nfluids, const ib_geometry *geo,
                             const StepDt &dt, const double *params, const ib_numerics *num,
                             const ib_drag_source *drag, cudaStream_t st)
{
    int rc;
    if (!fluids || !thermo || !geo) return IB_ERROR_NULL_POINTER;
    if (nfluids < 1) return IB_ERROR_INVALID_ARGS;
    Numerics nm;
    if ((rc = get_numerics(num, nm))) return rc;
    if (!geometry_ok(geo)) return IB_ERROR_NOIMPLEMENT;
    const bool cyl = geo->shape == IB_GEOMETRY_CYLINDRICAL;
    const int purehydro = (int)params[0];
    const int step_number = (int)params[1];
    const int method = (int)params[2];
    if (purehydro != 1) return IB_ERROR_NOIMPLEMENT;
    if (method < IB_METHOD_HLL || method > IB_METHOD_XINJIN) return IB_ERROR_INVALID_ARGS;
    if (drag && nfluids != 2) return IB_ERROR_INVALID_ARGS;  // gas and dust
    for (int fi = 0; fi < nfluids; fi++)
        if ((rc = validate_fluid(&fluids[fi]))) return rc;
    if (!drag && !cyl) {
        // no source between the two fluid steps (srcType 0, flux_multi.cu:161-163): the fluids
        // are independent, each runs forward then backward
        for (int fi = 0; fi < nfluids; fi++)
            if ((rc = fluid_fwd_bwd(&fluids[fi], geo, method, dt, fluid_params(thermo[fi]), nm, step_number, st)))
                return rc;
        return IB_SUCCESSFUL;
    }
    // Sources (flux_multi.cu:174-272): source dt/2, forward, source dt, backward, source dt/2, the
    // source being the two-fluid drag (srcType 8, src___D), the cylindrical terms of every fluid
    // (1, srcC___) or both split as cylinder dt/2, drag, cylinder dt/2 (9, srcC__D;
    // sourceStep.cu:200-226, 300-329, 498-562).  The cylinder sources end with
    // setAllBoundaryConditions (sourceStep.cu:276-291), which fills fluid 0's boundaries in
    // directions 1, 2, 3 once per fluid: its loop indexes fluids[0].  Directions of 3 cells or
    // fewer are left alone, as inside the fluid step.
    const int grid[3] = {fluids[0].grid.nx, fluids[0].grid.ny, fluids[0].grid.nz};
    auto cyl_terms = [&](double frac) -> int {
        for (int fi = 0; fi < nfluids; fi++) {
            const int g3[3] = {fluids[fi].grid.nx, fluids[fi].grid.ny, fluids[fi].grid.nz};
            int r = launch_cyl_source(fluids[fi].q, fluids[fi].grid.slab_pitch, g3, geo->h[0], geo->r_inner,
                                      dt.part(frac), st);
            if (r) return r;
        }
        return IB_SUCCESSFUL;
    };
    auto all_boundaries = [&]() -> int {
        for (int fi = 0; fi < nfluids; fi++)
            for (int d = 1; d <= 3; d++) {
                if (grid[d - 1] <= 3) continue;
                int r = fluid_boundary(&fluids[0], d, st);
                if (r) return r;
            }
        return IB_SUCCESSFUL;
    };
    auto source = [&](double frac) -> int {
        int r;
        if (cyl) {
            if ((r = cyl_terms(drag ? 0.5 * frac : frac))) return r;
            if (drag && (r = drag_source(&fluids[0], &fluids[1], &drag->thermo_gas, &drag->thermo_dust, geo,
                                         dt.part(frac), drag->method, st)))
                return r;
            if (drag && (r = cyl_terms(0.5 * frac))) return r;
            return all_boundaries();
        }
        return drag_source(&fluids[0], &fluids[1], &drag->thermo_gas, &drag->thermo_dust, geo, dt.part(frac),
                           drag->method, st);
    };
    if ((rc = source(0.5))) return rc;
    for (int fi = 0; fi < nfluids; fi++)
        if ((rc = fluid_step_one(&fluids[fi], geo, method, dt, fluid_params(thermo[fi]), nm, 1, step_number, st)))
            return rc;
    if ((rc = source(1.0))) return rc;
    for (int fi = 0; fi < nfluids; fi++)
        if ((rc = fluid_step_one(&fluids[fi], geo, method, dt, fluid_params(thermo[fi]), nm, -1, step_number, st)))
            return rc;
    return source(0.5);
}

}  // namespace ib

using namespace ib;

// =============================================================================================
// C ABI
// =============================================================================================
extern "C" {

int64_t ib_slab_pitch(int32_t nx, int32_t ny, int32_t nz)
{
    int64_t n = (int64_t)nx * ny * nz;
    return ((n + 31) / 32) * 32;
}

const char *ib_status_string(int status)
{
    switch (status) {
    case IB_SUCCESSFUL: return "SUCCESSFUL";
    case IB_ERROR_INVALID_ARGS: return "ERROR_INVALID_ARGS";
    case IB_ERROR_CRASH: return "ERROR_CRASH";
    case IB_ERROR_NULL_POINTER: return "ERROR_NULL_POINTER";
    case IB_ERROR_NOIMPLEMENT: return "ERROR_NOIMPLEMENT";
    case IB_ERROR_NOMEM: return "ERROR_NOMEM";
    case IB_ERROR_CUDA: return "ERROR_CUDA";
    default: return "UNKNOWN";
    }
}

int ib_last_cuda_error(void) { return g_last_cuda_error; }

long long ib_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int ib_setTileWaitLimit(long long polls)
{
    g_tile_wait_limit.store(polls < 0 ? -1 : std::min<long long>(polls, IB_TMA_SPIN_LIMIT), std::memory_order_relaxed);
    return IB_SUCCESSFUL;
}

int ib_device_wait_status(int clear)
{
    unsigned int *f = ib::scratch().wait_flag();
    if (!f) return IB_ERROR_NOMEM;
    unsigned int v = 0;
    int rc = ib::check_cuda(cudaMemcpy(&v, f, sizeof(v), cudaMemcpyDeviceToHost));
    if (rc) return rc;
    if (clear && v) {
        rc = ib::check_cuda(cudaMemset(f, 0, sizeof(unsigned int)));
        if (rc) return rc;
    }
    return (int)v;
}

int ib_cudaFluidStep(ib_fluid *fluid, const ib_geometry *geo, const double *params, int nparams,
                     const ib_numerics *num, void *stream)
{
    int rc;
    if (!geo || !params) return IB_ERROR_NULL_POINTER;
    if ((rc = validate_fluid(fluid))) return rc;
    if (nparams < 6 || nparams > 8) return IB_ERROR_INVALID_ARGS;
    Numerics nm;
    if ((rc = get_numerics(num, nm))) return rc;
    if (!geometry_ok(geo)) return IB_ERROR_NOIMPLEMENT;
    const double dt = params[0];
    const int purehydro = (int)params[1];
    double gamma = params[2];
    const double rho_min = params[3];
    const int method = (int)params[4];
    const int dir = (int)params[5];
    double c_iso = -1;
    if (nparams == 7 || (nparams == 8 && params[6] != -1)) {  // 8 parameters: -1 = adiabatic
        c_iso = params[6];
        gamma = 2;
    }
    const int theta_layout = (nparams == 8) ? (int)params[7] : 0;
    if (theta_layout != 0 && theta_layout != 1) return IB_ERROR_INVALID_ARGS;
    if (purehydro != 1) return IB_ERROR_NOIMPLEMENT;  // the MHD sweeps are dead in the reference
    if (method < IB_METHOD_HLL || method > IB_METHOD_XINJIN || dir < 1 || dir > 3) return IB_ERROR_INVALID_ARGS;
    return fluid_update_1d(fluid, geo, method, dir, StepDt{dt, nullptr}, gamma, rho_min, c_iso, nm,
                           (cudaStream_t)stream, 1, theta_layout);
}

int ib_fluidstep(ib_fluid *fluids, const ib_fluid_thermo *thermo, int nfluids, const ib_geometry *geo,
                 const double *params, int nparams, const ib_numerics *num, void *stream)
{
    int rc;
    if (!fluids || !thermo || !geo || !params) return IB_ERROR_NULL_POINTER;
    if (nparams != 5 || nfluids < 1) return IB_ERROR_INVALID_ARGS;
    Numerics nm;
    if ((rc = get_numerics(num, nm))) return rc;
    if (!geometry_ok(geo)) return IB_ERROR_NOIMPLEMENT;
    const StepDt dt{params[0], nullptr};
    const int purehydro = (int)params[1];
    const int sweep_dir = (int)params[2];
    const int step_number = (int)params[3];
    const int method = (int)params[4];
    if (purehydro != 1) return IB_ERROR_NOIMPLEMENT;
    if (method < IB_METHOD_HLL || method > IB_METHOD_XINJIN) return IB_ERROR_INVALID_ARGS;
    cudaStream_t st = (cudaStream_t)stream;
    for (int fi = 0; fi < nfluids; fi++) {
        if ((rc = validate_fluid(&fluids[fi]))) return rc;
        if ((rc = fluid_step_one(&fluids[fi], geo, method, dt, fluid_params(thermo[fi]), nm, sweep_dir, step_number,
                                 st)))
            return rc;
    }
    return IB_SUCCESSFUL;
}

int ib_completeTimestep(ib_fluid *fluids, const ib_fluid_thermo *thermo, int nfluids, const ib_geometry *geo,
                        const double *params, int nparams, const ib_numerics *num, const ib_drag_source *drag,
                        void *stream)
{
    if (!params) return IB_ERROR_NULL_POINTER;
    if (nparams != 4) return IB_ERROR_INVALID_ARGS;
    return complete_timestep(fluids, thermo, nfluids, geo, StepDt{params[0], nullptr}, params + 1, num, drag,
                             (cudaStream_t)stream);
}

int ib_completeTimestepDeviceDt(ib_fluid *fluids, const ib_fluid_thermo *thermo, int nfluids,
                                const ib_geometry *geo, const double *dt_device, const double *params, int nparams,
                                const ib_numerics *num, const ib_drag_source *drag, void *stream)
{
    if (!params || !dt_device) return IB_ERROR_NULL_POINTER;
    if (nparams != 3) return IB_ERROR_INVALID_ARGS;
    return complete_timestep(fluids, thermo, nfluids, geo, StepDt{0.0, dt_device}, params, num, drag,
                             (cudaStream_t)stream);
}

int ib_cudaSoundspeed(const ib_fluid *fluid, double gamma, double *cs_out, void *stream)
{
    int rc;
    if (!fluid || !cs_out) return IB_ERROR_NULL_POINTER;
    if ((rc = validate_grid(fluid->grid))) return rc;
    if (!fluid->q) return IB_ERROR_NULL_POINTER;
    const int64_t n = (int64_t)fluid->grid.nx * fluid->grid.ny * fluid->grid.nz;
    return launch_soundspeed(fluid->q, fluid->grid.slab_pitch, n, gamma, cs_out, (cudaStream_t)stream);
}

static int cfl_common(const ib_fluid *fluid, const double *cs, double gamma, const ib_geometry *geo, int method,
                      double *tau_host, double *tau_device, void *stream)
{
    int rc;
    if (!fluid || !geo || !fluid->q) return IB_ERROR_NULL_POINTER;
    if ((rc = validate_grid(fluid->grid))) return rc;
    if (method < IB_METHOD_HLL || method > IB_METHOD_XINJIN) return IB_ERROR_INVALID_ARGS;
    if (!geometry_ok(geo)) return IB_ERROR_NOIMPLEMENT;
    if (!tau_host && !tau_device) return IB_ERROR_NULL_POINTER;
    cudaStream_t st = (cudaStream_t)stream;
    double *tau = tau_device ? tau_device : scratch().cfl_tau();
    if (!tau) return IB_ERROR_NOMEM;
    const int grid[3] = {fluid->grid.nx, fluid->grid.ny, fluid->grid.nz};
    if ((rc = launch_cfl(fluid->q, cs, fluid->grid.slab_pitch, grid, geo, method, gamma, tau, st))) return rc;
    if (tau_host && tau_device) {
        if ((rc = check_cuda(cudaMemcpyAsync(tau_host, tau, sizeof(double), cudaMemcpyDeviceToHost, st)))) return rc;
        if ((rc = check_cuda(cudaStreamSynchronize(st)))) return rc;
    } else if (tau_host) {  // host-mapped slot: the kernel's store is visible once the stream is done
        if ((rc = check_cuda(cudaStreamSynchronize(st)))) return rc;
        *tau_host = *scratch().cfl_tau_host();
    }
    return IB_SUCCESSFUL;
}

int ib_cflTimestep(const ib_fluid *fluid, const double *cs, const ib_geometry *geo, int method, double *tau_host,
                   void *stream)
{
    if (!cs || !tau_host) return IB_ERROR_NULL_POINTER;
    return cfl_common(fluid, cs, 0.0, geo, method, tau_host, nullptr, stream);
}

int ib_cflTimestepFused(const ib_fluid *fluid, double gamma, const ib_geometry *geo, int method, double *tau_host,
                        double *tau_device, void *stream)
{
    return cfl_common(fluid, nullptr, gamma, geo, method, tau_host, tau_device, stream);
}

int ib_freezeAndPtot(ib_fluid *fluid, double gamma, int purehydro, double cs_min, double *ptot, double *freeze,
                     void *stream)
{
    int rc;
    if (!fluid || !fluid->q || !ptot || !freeze) return IB_ERROR_NULL_POINTER;
    if ((rc = validate_grid(fluid->grid))) return rc;
    if (purehydro != 1) return IB_ERROR_NOIMPLEMENT;
    const int grid[3] = {fluid->grid.nx, fluid->grid.ny, fluid->grid.nz};
    return launch_freeze_ptot(fluid->q, fluid->grid.slab_pitch, grid, gamma, cs_min, ptot, freeze,
                              (cudaStream_t)stream);
}

int ib_cudaStatics(double *phi, const ib_grid *grid, const int32_t bc[6], int halo, int vector_component,
                   const ib_statics *statics, int direction, void *stream)
{
    int rc;
    if (!phi || !grid || !bc) return IB_ERROR_NULL_POINTER;
    if ((rc = validate_grid(*grid))) return rc;
    if (direction < 1 || direction > 3 || halo < 1 || halo > 8) return IB_ERROR_INVALID_ARGS;
    if (vector_component < 0 || vector_component > 3) return IB_ERROR_INVALID_ARGS;
    cudaStream_t st = (cudaStream_t)stream;
    const int g3[3] = {grid->nx, grid->ny, grid->nz};
    for (int side = 0; side < 2; side++) {
        if ((rc = launch_statics(phi, statics, (int64_t)grid->nx * grid->ny * grid->nz, st))) return rc;
        const int mode = bc[2 * (direction - 1) + side];
        if (mode == IB_BC_OUTFLOW) {
            int32_t bc1[6] = {IB_BC_CIRCULAR, IB_BC_CIRCULAR, IB_BC_CIRCULAR,
                              IB_BC_CIRCULAR, IB_BC_CIRCULAR, IB_BC_CIRCULAR};
            bc1[2 * (direction - 1) + side] = IB_BC_OUTFLOW;
            rc = launch_fluid_boundary(phi, grid->slab_pitch, g3, bc1, halo, direction, st);
        } else {
            rc = launch_array_boundary(phi, g3, mode, direction, side, vector_component, halo, st);
        }
        if (rc) return rc;
    }
    return IB_SUCCESSFUL;
}

int ib_setFluidBoundary(ib_fluid *fluid, int direction, void *stream)
{
    int rc;
    if ((rc = validate_fluid(fluid))) return rc;
    if (direction < 1 || direction > 3) return IB_ERROR_INVALID_ARGS;
    return fluid_boundary(fluid, direction, (cudaStream_t)stream);
}

int ib_cudaSource2FluidDrag(ib_fluid *gas, ib_fluid *dust, const ib_thermo *tg, const ib_thermo *td,
                            const ib_geometry *geo, const double *params, int nparams, void *stream)
{
    if (!params) return IB_ERROR_NULL_POINTER;
    if (nparams != 2) return IB_ERROR_INVALID_ARGS;  // cudaSource2FluidDrag.cu:157-163
    return drag_source(gas, dust, tg, td, geo, DevScalar::of(params[0]), (int)params[1], (cudaStream_t)stream);
}

}  // extern "C"
