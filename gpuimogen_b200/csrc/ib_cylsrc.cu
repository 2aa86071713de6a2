// ib_cylsrc.cu -- geometric source terms of cylindrical coordinates (x = r, y = theta, z = z):
// cukern_SourceCylindricalTerms, gpuclass/cudaSourceCylindricalTerms.cu:119-222.
//
// Per cell, v_r' = v_theta^2 / r and v_theta' = -v_r v_theta / r over dt, integrated by the
// two-stage Gauss-Legendre collocation method (fourth order; the reference's own decimal values of
// its Butcher table, cudaSourceCylindricalTerms.cu:107-114, so that results agree bit for bit)
// with an explicit first guess and two fixed-point passes.  The stage updates follow the reference
// as written: the first v_theta update adds the second stage's term where the method subtracts it,
// and the second v_theta update uses the old stage-B v_r in both of its terms.  The change of
// kinetic energy is left in the internal energy (total energy unchanged) unless the pressure would
// become non-positive, where E is reset to the new kinetic energy plus 1e-5 rho.
//
// One thread per cell: a grid-stride loop over the arrays in XYZ order, 5 loads and at most 3
// stores of 8 bytes per cell (HBM-bound; it runs once per source step).
#include "ib_internal.cuh"

namespace ib {

namespace {
constexpr double kGL11 = .25;
constexpr double kGL12 = -0.038675134594812865529;
constexpr double kGL21 = 0.53867513459481286553;
constexpr double kGL22 = .25;
}  // namespace

__global__ void __launch_bounds__(256) cyl_source_kernel(double *__restrict__ q, int64_t slab, int nx, int64_t n,
                                                         double rin, double dr, DevScalar dts)
{
    if (dts.off()) return;  // a device timestep of 0: after the end time
    const double dt = dts.get();
    for (int64_t x = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; x < n; x += (int64_t)blockDim.x * gridDim.x) {
        double *base = q + x;
        const double r = rin + (int)(x % nx) * dr;
        const double rho = base[0];
        double u = base[2 * slab] / rho;  // v_r
        double v = base[3 * slab] / rho;  // v_theta
        double diffmom = dt * v / r;
        double vrA = u + kGL11 * v * diffmom;
        double vphiA = v - kGL11 * u * diffmom;
        double vrB = u + kGL12 * v * diffmom;
        double vphiB = v - kGL12 * u * diffmom;
#pragma unroll
        for (int it = 0; it < 2; it++) {
            diffmom = dt * vphiA / r;
            const double diffmomB = dt * vphiB / r;
            double scratch = vrA;
            vrA = u + kGL11 * vphiA * diffmom + kGL12 * vphiB * diffmomB;
            vphiA = v - kGL11 * scratch * diffmom + kGL12 * vrB * diffmomB;
            diffmom = dt * vphiA / r;
            scratch = vrB;
            vrB = u + kGL21 * vphiA * diffmom + kGL22 * vphiB * diffmomB;
            vphiB = v - kGL21 * scratch * diffmom + kGL22 * scratch * diffmomB;
        }
        u = rho * (u + .5 * dt * (vphiA * vphiA + vphiB * vphiB) / r);
        v = rho * (v - .5 * dt * (vphiA * vrA + vphiB * vrB) / r);
        const double E = base[slab];
        const double w = base[4 * slab];
        const double newP = E - .5 * (u * u + v * v + w * w) / rho;
        if (newP <= 0.0) base[slab] = .5 * (u * u + v * v + w * w) / rho + .00001 * rho;
        base[2 * slab] = u;
        base[3 * slab] = v;
    }
}

int launch_cyl_source(double *q, int64_t slab, const int grid[3], double dr, double r_inner, DevScalar dt,
                      cudaStream_t st)
{
    const int64_t n = (int64_t)grid[0] * grid[1] * grid[2];
    if (n <= 0) return IB_SUCCESSFUL;
    int nb = (int)std::min<int64_t>((n + 255) / 256, (int64_t)8 * num_sms());
    if (nb < 1) nb = 1;
    cyl_source_kernel<<<nb, 256, 0, st>>>(q, slab, grid[0], n, r_inner, dr, dt);
    return check_launch();
}

}  // namespace ib
