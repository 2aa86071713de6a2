// ib_boundary.cu -- boundary fill and statics (gpuclass/cudaStatics.cu).
//
// Inside the fluid step the reference fills the boundary right after each sweep, while the
// arrays are transposed so that the swept axis is fastest; it therefore always runs the
// X-direction kernels (setFluidBoundary -> setBoundarySAS / setOutflowCondition with
// memory direction 1, cudaStatics.cu:112-197, 1305-1400, 462-545).  launch_fluid_boundary
// applies those same X-kernel rules along the physical pencils of the swept direction of the
// XYZ-ordered arrays.  The cudaStatics mex on an XYZ array instead uses the kernels of the
// array's memory direction (cudaStatics.cu:1404-1532), reproduced by launch_array_boundary.
#include "ib_bc.cuh"
#include "ib_internal.cuh"

namespace ib {

struct PencilIdx {
    int nx, ny, nz, dir;
    __device__ __forceinline__ void get(int64_t p, int64_t &base, int64_t &stride, int &n) const
    {
        if (dir == 1) { base = p * nx; stride = 1; n = nx; }
        else if (dir == 2) { base = (p % nx) + (int64_t)nx * ny * (p / nx); stride = nx; n = ny; }
        else { base = p; stride = (int64_t)nx * ny; n = nz; }
    }
};

__global__ void fluid_boundary_kernel(double *q, int64_t S, PencilIdx pi, int64_t npencil, int mode0, int mode1,
                                      int depth)
{
    const int64_t p = threadIdx.x + (int64_t)blockIdx.x * blockDim.x;
    if (p >= npencil) return;
    int64_t base, s;
    int n;
    pi.get(p, base, s, n);
    double *v0 = q + base;
    for (int side = 0; side < 2; side++) {
        const int mode = side ? mode1 : mode0;
        if (mode == IB_BC_OUTFLOW) {
            outflow_x(v0, S, s, n, side, pi.dir, depth);
        } else if (mode == IB_BC_MIRROR || mode == IB_BC_CONST || mode == IB_BC_LINEAR) {
            for (int k = 0; k < 5; k++) sas_x(v0 + k * S, s, n, mode, side, (k >= 2) && (k - 1 == pi.dir), depth);
        }
    }
}

static bool mode_ok(int m)
{
    return m == IB_BC_CIRCULAR || m == IB_BC_STATIONARY || m == IB_BC_MIRROR || m == IB_BC_CONST ||
           m == IB_BC_LINEAR || m == IB_BC_OUTFLOW;
}

int launch_fluid_boundary(double *q, int64_t slab, const int grid[3], const int32_t bc[6], int halo, int dir,
                          cudaStream_t st)
{
    const int m0 = bc[2 * (dir - 1)], m1 = bc[2 * (dir - 1) + 1];
    if (m0 == IB_BC_WALL || m1 == IB_BC_WALL || m0 == IB_BC_FREEBALANCE || m1 == IB_BC_FREEBALANCE)
        return IB_ERROR_NOIMPLEMENT;
    if (!mode_ok(m0) || !mode_ok(m1)) return IB_ERROR_INVALID_ARGS;
    const bool any = !((m0 == IB_BC_CIRCULAR || m0 == IB_BC_STATIONARY) && (m1 == IB_BC_CIRCULAR || m1 == IB_BC_STATIONARY));
    if (!any) return IB_SUCCESSFUL;
    const int n = grid[dir - 1];
    if (n < 2 * halo + 1) return IB_ERROR_INVALID_ARGS;
    const int64_t N = (int64_t)grid[0] * grid[1] * grid[2];
    const int64_t np = N / n;
    PencilIdx pi{grid[0], grid[1], grid[2], dir};
    fluid_boundary_kernel<<<(unsigned)((np + 127) / 128), 128, 0, st>>>(q, slab, pi, np, m0, m1, halo);
    return check_launch();
}

// Per-array rules in memory direction dir for XYZ storage (cudaStatics mex)
__global__ void array_boundary_kernel(double *phi, PencilIdx pi, int64_t npencil, int mode, int side, bool anti,
                                      int depth)
{
    const int64_t p = threadIdx.x + (int64_t)blockIdx.x * blockDim.x;
    if (p >= npencil) return;
    int64_t base, s;
    int n;
    pi.get(p, base, s, n);
    double *v = phi + base;
    if (pi.dir == 1 || mode == IB_BC_LINEAR) {
        sas_x(v, s, n, mode, side, anti, depth);
        return;
    }
    if (mode == IB_BC_MIRROR) {
        for (int q = 0; q < depth; q++) {
            double a;
            if (side == 0) {
                // y: 2*depth-1+MIRROR_OFFSET-q (cudaStatics.cu:1413-1421); z: 2*depth+MIRROR_OFFSET-q (1471-1481)
                int src = (pi.dir == 2) ? (2 * depth - q) : (2 * depth + 1 - q);
                a = v[(int64_t)src * s];
                v[(int64_t)q * s] = anti ? -a : a;
            } else {
                a = v[(int64_t)(n - 1 - 2 * depth + q) * s];
                v[(int64_t)(n - 1 - q) * s] = anti ? -a : a;
            }
        }
    } else if (mode == IB_BC_CONST) {
        if (side == 0) {
            double f = v[(int64_t)depth * s];
            for (int q = 0; q < depth; q++) v[(int64_t)q * s] = f;
        } else {
            // the y and z + side kernels copy cell n-depth (cudaStatics.cu:1443-1448, 1524-1531)
            double f = v[(int64_t)(n - depth) * s];
            for (int q = 0; q < depth; q++) v[(int64_t)(n - 1 - q) * s] = f;
        }
    }
}

int launch_array_boundary(double *phi, const int grid[3], int mode, int dir, int side, int vec_component, int halo,
                          cudaStream_t st)
{
    if (mode == IB_BC_CIRCULAR || mode == IB_BC_STATIONARY) return IB_SUCCESSFUL;
    if (mode == IB_BC_WALL || mode == IB_BC_FREEBALANCE) return IB_ERROR_NOIMPLEMENT;
    if (mode == IB_BC_LINEAR && dir != 1) return IB_ERROR_NOIMPLEMENT;  // cudaStatics.cu:1187-1220
    if (!(mode == IB_BC_MIRROR || mode == IB_BC_CONST || mode == IB_BC_LINEAR)) return IB_ERROR_INVALID_ARGS;
    const int n = grid[dir - 1];
    if (n < 2 * halo + 2) return IB_ERROR_INVALID_ARGS;  // the z mirror reads cell 2*halo+1
    const int64_t N = (int64_t)grid[0] * grid[1] * grid[2];
    const int64_t np = N / n;
    PencilIdx pi{grid[0], grid[1], grid[2], dir};
    array_boundary_kernel<<<(unsigned)((np + 127) / 128), 128, 0, st>>>(phi, pi, np, mode, side, vec_component == dir,
                                                                        halo);
    return check_launch();
}

// cukern_applySpecial_fade (cudaStatics.cu:1240-1266)
__global__ void statics_kernel(double *phi, const double *statics, int64_t count, int64_t pitch, int64_t numel)
{
    const int64_t i = threadIdx.x + (int64_t)blockIdx.x * blockDim.x;
    if (i >= count) return;
    const double xd = statics[i];
    if (!(xd >= 0.0 && xd < (double)numel)) return;  // indices outside the array are ignored
    const int64_t xaddr = (int64_t)xd;
    const double f0 = statics[i + pitch];
    const double c = statics[i + 2 * pitch];
    if (c != 1.0) {
        double wval = f0 * c + (1.0 - c) * phi[xaddr];
        if (isnan(wval)) wval = f0 * c;
        phi[xaddr] = wval;
    } else {
        phi[xaddr] = f0;
    }
}

int launch_statics(double *phi, const ib_statics *sl, int64_t numel, cudaStream_t st)
{
    if (sl == nullptr || sl->data == nullptr || sl->count <= 0) return IB_SUCCESSFUL;
    if (sl->pitch < sl->count) return IB_ERROR_INVALID_ARGS;
    statics_kernel<<<(unsigned)((sl->count + 127) / 128), 128, 0, st>>>(phi, sl->data, sl->count, sl->pitch, numel);
    return check_launch();
}

}  // namespace ib
