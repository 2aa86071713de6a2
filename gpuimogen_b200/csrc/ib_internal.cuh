// ib_internal.cuh -- host-side plumbing shared by the library's translation units.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "ib_common.cuh"
#include "ib_tma.cuh"
#include "ib_cyl.cuh"

namespace ib {

// Records the last CUDA error and maps it to the library's status codes.
int check_cuda(cudaError_t e);
int check_launch();
int num_sms();
// Poll limit of the TMA-fed kernels' tile waits (IB_TMA_SPIN_LIMIT unless ib_setTileWaitLimit set one).
uint32_t tile_wait_limit();
// Shortest y/z pencil (cells) the pencil-box kernels take: a CTA of theirs has one thread per cell
// and runs its pencils one after the other, so shorter pencils go to kernels that pack several
// pencils into a block (IMOGEN_B200_PAIRMIN overrides).
int pair_min_cells();

// Reusable per-device scratch: grown on demand, never shrunk, freed at process exit.  The
// reference allocates and frees a 6-slab temporary per call (cudaFluidStep.cu:508-513); the
// fused sweeps here need none beyond the chunked pipeline's halo side buffer; the others
// are the reductions, the ETDRK2 drag's internal-energy slab, the wait flags and the ensemble's
// work counter.
class Scratch {
public:
    double *cfl_partial(int nblocks);
    unsigned int *cfl_counter();
    double *cfl_tau();        // device address of the host-mapped timestep slot
    volatile double *cfl_tau_host();  // the same slot as the host sees it (after cfl_tau())
    double *bytes(size_t nbytes);  // general scratch (reused between calls on the device)
    unsigned int *wait_flag();     // set by a kernel whose bounded wait ran out (zeroed once)
    unsigned int *ensemble_counter();  // work counter of the ensemble kernel

private:
    double *partial_ = nullptr;
    int partial_n_ = 0;
    unsigned int *counter_ = nullptr;
    double *tau_ = nullptr;       // device pointer into tau_host_
    double *tau_host_ = nullptr;  // pinned, mapped host memory
    double *gen_ = nullptr;
    size_t gen_n_ = 0;
    unsigned int *wait_flag_ = nullptr;
    unsigned int *ens_counter_ = nullptr;
};
Scratch &scratch();

// Launchers (return IB_* status)
int launch_sweep(int method, int slope, int precision, int dir, double *q, int64_t slab, const int grid[3],
                 DevScalar lambda, double gamma, double rho_min, double c_iso, cudaStream_t st, int nsweep = 1);
int launch_xj_sweep(int flim, int dir, double *q, int64_t slab, const int grid[3], DevScalar lambda, double gamma,
                    double rho_min, cudaStream_t st, const CylSweep *cyl = nullptr);
// cylindrical geometry: HLL/HLLC radial (x) and theta (y) sweeps; the source terms over dt
int launch_sweep_cyl(int method, int slope, double *q, int64_t slab, const int grid[3], DevScalar lambda,
                     double gamma, double rho_min, double c_iso, cudaStream_t st, const CylSweep &cs);
int launch_cyl_source(double *q, int64_t slab, const int grid[3], double dr, double r_inner, DevScalar dt,
                      cudaStream_t st);
int launch_cfl(const double *q, const double *cs, int64_t slab, const int grid[3], const ib_geometry *geo,
               int method, double gamma, double *tau_dev, cudaStream_t st);
int launch_soundspeed(const double *q, int64_t slab, int64_t n, double gamma, double *cs, cudaStream_t st);
int launch_freeze_ptot(double *q, int64_t slab, const int grid[3], double gamma, double cs_min, double *ptot,
                       double *freeze, cudaStream_t st);
int launch_fluid_boundary(double *q, int64_t slab, const int grid[3], const int32_t bc[6], int halo, int dir,
                          cudaStream_t st);
int launch_array_boundary(double *phi, const int grid[3], int mode, int dir, int side, int vec_component, int halo,
                          cudaStream_t st);
int launch_statics(double *phi, const ib_statics *st_list, int64_t numel, cudaStream_t st);
int launch_drag(double *gas, double *dust, int64_t slab, const int grid[3], const double h[3], const double dp[11],
                DevScalar dt, int method, cudaStream_t st);

}  // namespace ib
