// ib_sweep_cyl.cu -- instantiates the cylindrical-geometry sweeps (HLL and HLLC, FP64) with the
// geometry's update (ib_cyl.cuh): radial x sweeps in the row kernel (rows up to 512 cells) and
// theta y sweeps in the pencil-pair kernel (pencils up to 256 cells, x even), the tile kernel
// for other shapes.
#include "ib_sweep_launch.cuh"

namespace ib {
int launch_sweep_cyl(int method, int slope, double *q, int64_t slab, const int grid[3], DevScalar lambda,
                     double gamma, double rho_min, double c_iso, cudaStream_t st, const CylSweep &cs)
{
    if (method == IB_METHOD_HLLC)
        return launch_sweep_cyl_slope<IB_METHOD_HLLC>(slope, q, slab, grid, lambda, gamma, rho_min, c_iso, st, cs);
    if (method == IB_METHOD_HLL)
        return launch_sweep_cyl_slope<IB_METHOD_HLL>(slope, q, slab, grid, lambda, gamma, rho_min, c_iso, st, cs);
    return IB_ERROR_INVALID_ARGS;
}
}  // namespace ib
