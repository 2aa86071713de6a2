// ib_bc.cuh -- per-pencil boundary rules shared by the boundary kernels and the fused
// ensemble kernel (X-kernel semantics of gpuclass/cudaStatics.cu along any pencil).
#pragma once

#include "ib_common.cuh"

namespace ib {

// X-kernel semantics for one slab along one pencil (cudaStatics.cu:1305-1400); MIRROR_OFFSET = 1
__device__ __forceinline__ void sas_x(double *v, int64_t s, int n, int mode, int side, bool anti, int depth)
{
    if (mode == IB_BC_MIRROR) {
        for (int t = 0; t < depth; t++) {
            if (side == 0) {
                double a = v[(int64_t)(depth + 1 + t) * s];
                v[(int64_t)(depth - 1 - t) * s] = anti ? -a : a;
            } else {
                double a = v[(int64_t)(n - depth - 2 - t) * s];
                v[(int64_t)(n - depth + t) * s] = anti ? -a : a;
            }
        }
    } else if (mode == IB_BC_CONST) {
        if (side == 0) {
            double a = v[(int64_t)depth * s];
            for (int t = 0; t < depth; t++) v[(int64_t)t * s] = a;
        } else {
            double a = v[(int64_t)(n - depth - 1) * s];
            for (int t = 0; t < depth; t++) v[(int64_t)(n - depth + t) * s] = a;
        }
    } else if (mode == IB_BC_LINEAR) {
        double f[4];
        if (side == 0) {
            for (int t = 0; t < 4; t++) f[t] = v[(int64_t)(t + depth) * s];
            for (int t = 0; t < depth; t++) v[(int64_t)t * s] = v[(int64_t)depth * s] + (double)(depth - t) * (f[0] - f[1]);
        } else {
            // the reference also writes one cell past the end of the pencil; that write is dropped
            int64_t b = n - depth - 1;
            for (int t = 0; t < 4; t++) f[t] = v[(b + t) * s];
            for (int t = 0; t < depth; t++) {
                int64_t dst = b + t + 2;
                if (dst < n) v[dst * s] = f[1] + (double)(t + 1) * (f[1] - f[0]);
            }
        }
    }
}

// cukern_SetOutflowX (cudaStatics.cu:462-545) on the five slabs of one pencil.  The - side
// follows the evident intent (read cell `depth`, write cells 0..depth-1): the reference's - side
// kernel starts depth cells before the row and so writes outside it.
__device__ __forceinline__ void outflow_x(double *v0, int64_t S, int64_t s, int n, int side, int nd, int depth)
{
    const int64_t src = (side == 1) ? (n - 1 - depth) : depth;
    const double a = v0[(1 + nd) * S + src * s];
    const int direct = side ? 1 : -1;
    if (a * direct > 0) {
        for (int k = 0; k < 5; k++) {
            double val = v0[k * S + src * s];
            for (int t = 0; t < depth; t++) {
                int64_t dst = side ? (src + 1 + t) : t;
                v0[k * S + dst * s] = val;
            }
        }
    } else {
        const double rho = v0[src * s], E0 = v0[S + src * s];
        const double p1x = v0[2 * S + src * s], p1y = v0[3 * S + src * s], p1z = v0[4 * S + src * s];
        for (int t = 0; t < depth; t++) {
            int64_t dst = side ? (src + 1 + t) : t;
            double rf = side ? (-1.198 - .0047 * t) : 1.05;  // restFrmSpeed (cudaStatics.cu:379-384)
            double E = E0, p1, p2;
            v0[dst * s] = rho;
            p1 = p1x; p2 = rho * 0.0;
            v0[2 * S + dst * s] = p2;
            E += .5 * (p2 - p1) * (p2 + p1) / rho;
            p1 = p1y; p2 = (nd == 1) ? rho * rf : rho * (p1y / rho);
            v0[3 * S + dst * s] = p2;
            E += .5 * (p2 - p1) * (p2 + p1) / rho;
            p1 = p1z; p2 = rho * 0.0;
            v0[4 * S + dst * s] = p2;
            E += .5 * (p2 - p1) * (p2 + p1) / rho;
            v0[S + dst * s] = E;
        }
    }
}

}  // namespace ib
