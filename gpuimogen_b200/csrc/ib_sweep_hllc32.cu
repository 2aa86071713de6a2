// ib_sweep_hllc32.cu -- instantiates the fused sweep kernels for method IB_METHOD_HLLC with float flux arithmetic.
#include "ib_sweep_launch.cuh"

namespace ib {
int launch_hllc32(int slope, int dir, double *q, int64_t slab, const int grid[3], DevScalar lambda, double gamma,
              double rho_min, double c_iso, cudaStream_t st, int nsweep)
{
    return launch_sweep_slope<IB_METHOD_HLLC, float>(slope, dir, q, slab, grid, lambda, gamma, rho_min, c_iso, st, nsweep);
}
}  // namespace ib
