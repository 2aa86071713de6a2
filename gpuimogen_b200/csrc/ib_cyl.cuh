// ib_cyl.cuh -- cylindrical geometry of the sweeps (x = r, y = theta, z = z), shared by the
// HLL/HLLC tile kernel and the Xin-Jin pencil kernel.
//
// The reference selects the geometry per sweep (cudaFluidStep.cu:264-278): an x sweep becomes
// FLUX_RADIAL, whose update weights the two faces by their radii and adds a geometric pressure
// term to p_r; a y sweep becomes FLUX_THETA_213 or FLUX_THETA_231 by where its memory
// permutation put r, dividing the flux difference by r (213) or lambda by r before use (231);
// z sweeps are plain.  The radius a theta kernel computes is restated by theta_radius (see there).
#pragma once

#include "ib_common.cuh"

namespace ib {

// kernel template values of the geometry
enum { CYL_NONE = 0, CYL_RADIAL = 1, CYL_THETA_DIV = 2, CYL_THETA_LAM = 3 };

// How a theta pencil's radius is computed, from its radial index i (or z index kz):
//   RMODE_GEOMETRIC  rin + i dr                       (dr = h[0]: the cell centre radius)
//   RMODE_ACC4       (i mod 4) dr + rin, plus 4 dr once per pass of the kernel's 4-row loop
//                    (layout theta,r,z: cudaFluidStep.cu:848-850, 1112-1116, 1844-1846, 2462-2464)
//   RMODE_INDEX      i dr + rin                       (layout theta,z,r: the block index, 852-855)
//   RMODE_INNER      rin                              (layout theta,z,r on a 2-D grid, where the
//                    launch treats the radial axis as the second one and the block index is 0)
// The reference's modes take dr = h[1], the theta cell size (gamHost[9] = h[stepDirection-1],
// cudaFluidStep.cu:305-307); jz: the z index replaces i (layout theta,r,z with nx = 1 < nz).
enum { RMODE_GEOMETRIC = 0, RMODE_ACC4 = 1, RMODE_INDEX = 2, RMODE_INNER = 3 };

struct CylPencil {
    double rin, dr;
    int rmode, jz;
};

__device__ __forceinline__ double theta_radius(const CylPencil &g, int i, int kz)
{
    const int j = g.jz ? kz : i;
    switch (g.rmode) {
    case RMODE_GEOMETRIC: return g.rin + j * g.dr;
    case RMODE_ACC4: {
        double r = (j % 4) * g.dr + g.rin;
        for (int m = 0; m < j / 4; m++) r = r + 4.0 * g.dr;
        return r;
    }
    case RMODE_INDEX: return j * g.dr + g.rin;
    default: return g.rin;
    }
}

// Host description of one cylindrical sweep (x = r, y = theta)
struct CylSweep {
    int kind;          // CYL_*
    CylPencil pencil;  // theta: radius rule; radial: rin, dr = h[0]
};

}  // namespace ib
