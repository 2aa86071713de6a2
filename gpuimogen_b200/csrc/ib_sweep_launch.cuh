// ib_sweep_launch.cuh -- host launch logic for the fused sweep kernels of one (method, flux type).
#pragma once

#include "ib_internal.cuh"
#include "ib_sweep.cuh"

#include <cstdlib>
#include <type_traits>

namespace ib {

// Tile-march launch: W pencils per CTA, chunks of ~TARGET cells, every chunk >= 8 cells.
template <int METHOD, int SLOPE, typename FT, int DIR, int W, int GEO = CYL_NONE>
int launch_tile_dw(double *q, int64_t slab, const int grid[3], DevScalar lambda, const FluidConsts<FT> &c,
                   cudaStream_t st, int target, CylPencil cyl = CylPencil{0.0, 0.0, 0, 0})
{
    const int n = grid[DIR - 1];
    const int64_t npencil = (int64_t)grid[0] * grid[1] * grid[2] / n;
    // every phase of a chunk must fit in one pass of the CTA's threads: (Lc+8)*W <= 256
    const int lc_max = 256 / W - 8;
    if (target > lc_max) target = lc_max;
    int nc = std::max(1, (n + target - 1) / target);
    int Lc = (n + nc - 1) / nc;
    while (nc > 1 && (Lc < 8 || n - (nc - 1) * Lc < 8)) {
        nc--;
        Lc = (n + nc - 1) / nc;
    }
    if (Lc > lc_max) return IB_ERROR_NOIMPLEMENT;  // pencil too short to split into valid chunks
    TileArgs a{q, slab, grid[0], grid[1], grid[2], n, npencil, Lc, lambda, cyl};
    const size_t shm = tile_smem_bytes<W, GEO>(Lc, sizeof(FT));
    static int attr_bytes = 0;
    // opt in whenever the size grows: without it the limit is 48 KB including the static
    // shared memory and the 1 KB the driver reserves per block (48640 B at 256-cell pencils fails)
    if ((int)shm > attr_bytes) {
        int rc = check_cuda(cudaFuncSetAttribute(sweep_tile_kernel<METHOD, SLOPE, FT, DIR, W, GEO>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        if (rc) return rc;
        attr_bytes = (int)shm;
    }
    const unsigned nblk = (unsigned)((npencil + W - 1) / W);
    sweep_tile_kernel<METHOD, SLOPE, FT, DIR, W, GEO><<<nblk, 256, shm, st>>>(a, c);
    return check_launch();
}

// TMA-fed persistent pipeline (sweep_pipe_kernel): W whole pencils of length n <= 512 per
// block, W*n <= CPT*512 threads' cells.  Returns IB_ERROR_NOIMPLEMENT (caller falls back) when
// the grid does not meet TMA's rules: x even (16-byte strides and box rows), W dividing nx,
// pencils above 256 cells even (two box rows of n/2).
//
// G > 1 selects sweep_pipe_wide_kernel: blocks of W*G columns (one TMA box), computed W at a time,
// results stored from the input tile; pencils up to 256 cells, y/z sweeps only.
template <int METHOD, int SLOPE, typename FT, int DIR, int W, int CPT, int NFIX = 0, int G = 1>
int launch_pipe(double *q, int64_t slab, const int grid[3], DevScalar lambda, const FluidConsts<FT> &c, cudaStream_t st,
                int nsweep)
{
    const int nx = grid[0], ny = grid[1], nz = grid[2];
    const int n = grid[DIR - 1];
    constexpr int WL = W * G;  // columns per block (and per TMA box)
    if (n > 512 || (n > 256 && (n & 1)) || W * n > CPT * 512 || (nx & 1) || nx % WL) return IB_ERROR_NOIMPLEMENT;
    if (DIR == 1 && n > 256) return IB_ERROR_NOIMPLEMENT;
    if (G > 1 && (DIR == 1 || n > 256)) return IB_ERROR_NOIMPLEMENT;
    if (((uintptr_t)q & 15) || (slab * 8) % 16) return IB_ERROR_NOIMPLEMENT;
    const int bh = (n > 256) ? n / 2 : n, nh = (n > 256) ? 2 : 1;
    CUtensorMap tm;
    uint64_t dims[5], strides[4];
    uint32_t box[5];
    int rank;
    int64_t nblocks;
    const int npw = (DIR == 1) ? 1 : nx / WL;
    if (DIR == 1) {
        rank = 3;
        dims[0] = nx; dims[1] = (uint64_t)ny * nz; dims[2] = 5;
        strides[0] = (uint64_t)nx * 8; strides[1] = (uint64_t)slab * 8;
        box[0] = nx; box[1] = 1; box[2] = 5;
        nblocks = (int64_t)ny * nz;
    } else {
        rank = 5;
        const uint64_t other = (DIR == 2) ? nz : ny;
        const uint64_t rs = (DIR == 2) ? (uint64_t)nx * 8 : (uint64_t)nx * ny * 8;   // along the pencil
        const uint64_t os = (DIR == 2) ? (uint64_t)nx * ny * 8 : (uint64_t)nx * 8;   // across pencils
        dims[0] = nx; dims[1] = bh; dims[2] = nh; dims[3] = other; dims[4] = 5;
        strides[0] = rs; strides[1] = rs * bh; strides[2] = os; strides[3] = (uint64_t)slab * 8;
        box[0] = WL; box[1] = bh; box[2] = nh; box[3] = 1; box[4] = 5;
        nblocks = (int64_t)npw * other;
    }
    if (nblocks >= (int64_t)1 << 31) return IB_ERROR_NOIMPLEMENT;
    int rc = encode_tmap_f64(&tm, q, rank, dims, strides, box);
    if (rc) return rc;
    unsigned int *err = scratch().wait_flag();
    if (!err) return IB_ERROR_NOMEM;
    const int nt = ((W * n + CPT - 1) / CPT + 31) / 32 * 32;  // a multiple of 32, hence of W
    if (nt > 512) return IB_ERROR_NOIMPLEMENT;
    const size_t shm = (G == 1 ? 3 * pipe_tile_bytes(n, W) : 2 * pipe_tile_bytes(n, WL)) +
                       (size_t)10 * W * n * sizeof(FT);
    if (NFIX && n != NFIX) return IB_ERROR_NOIMPLEMENT;
    if (shm > 227 * 1024) return IB_ERROR_NOIMPLEMENT;
    const int ns = (nsweep == 2) ? 2 : 1;
    auto kern = [ns] {
        if constexpr (G == 1)
            return ns == 2 ? &sweep_pipe_kernel<METHOD, SLOPE, FT, DIR, W, CPT, NFIX, 2>
                           : &sweep_pipe_kernel<METHOD, SLOPE, FT, DIR, W, CPT, NFIX, 1>;
        else
            return ns == 2 ? &sweep_pipe_wide_kernel<METHOD, SLOPE, FT, DIR, W, G, CPT, NFIX, 2>
                           : &sweep_pipe_wide_kernel<METHOD, SLOPE, FT, DIR, W, G, CPT, NFIX, 1>;
    }();
    static int attr_bytes[2] = {0, 0};
    if ((int)shm > attr_bytes[ns - 1]) {
        rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        if (rc) return rc;
        attr_bytes[ns - 1] = (int)shm;
    }
    int per_sm = 0;
    rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, shm));
    if (rc) return rc;
    if (per_sm < 1) return IB_ERROR_NOIMPLEMENT;
    const int64_t want = (int64_t)per_sm * num_sms();
    const unsigned nblk = (unsigned)std::min<int64_t>(want, nblocks);
    PipeArgs a{n, npw, bh, nh, nblocks, lambda, err, tile_wait_limit()};
    kern<<<nblk, nt, shm, st>>>(tm, a, c);
    return check_launch();
}

// Pencil-pair kernel (sweep_pair_kernel): y/z pencils of at most 256 cells or of 512 (the box
// arrives as two rows of 256), x even; one CTA per block of two adjacent pencils.  Returns
// IB_ERROR_NOIMPLEMENT (caller falls back) otherwise.  GEO: cylindrical theta pencils (y, one
// sweep), with their radius rule in cyl.
template <int METHOD, int SLOPE, typename FT, int DIR, int NFIX = 0, int WC = 2, int GEO = CYL_NONE, int PADN = 0>
int launch_pair(double *q, int64_t slab, const int grid[3], DevScalar lambda, const FluidConsts<FT> &c, cudaStream_t st,
                int nsweep, CylPencil cyl = CylPencil{0.0, 0.0, 0, 0})
{
    static_assert(PADN == 0 || NFIX == 0, "a fixed plane stride for pencils of a run-time length");
    static_assert(GEO == CYL_NONE || DIR == 2, "theta pencils run along y");
    if (GEO != CYL_NONE && nsweep != 1) return IB_ERROR_NOIMPLEMENT;
    static_assert(DIR != 1, "x rows take the row kernel");
    static_assert(WC == 2 || (WC == 4 && NFIX != 512), "boxes of 2 pencils, or 4 of at most 256 cells");
    const int nx = grid[0], ny = grid[1], nz = grid[2];
    const int n = grid[DIR - 1];
    if ((n > 256 && !(NFIX == 512 && n == 512)) || (nx % WC)) return IB_ERROR_NOIMPLEMENT;
    if (NFIX && n != NFIX) return IB_ERROR_NOIMPLEMENT;
    if (((uintptr_t)q & 15) || (slab * 8) % 16) return IB_ERROR_NOIMPLEMENT;
    const uint64_t other = (DIR == 2) ? nz : ny;
    const uint64_t rs = (DIR == 2) ? (uint64_t)nx * 8 : (uint64_t)nx * ny * 8;   // along the pencil
    const uint64_t os = (DIR == 2) ? (uint64_t)nx * ny * 8 : (uint64_t)nx * 8;   // across pencils
    // TMA boxes are at most 256 rows: a 512-cell pencil comes as two rows of 256 (half, row)
    const int bh = (n > 256) ? n / 2 : n, nh = (n > 256) ? 2 : 1;
    uint64_t dims[5] = {(uint64_t)nx, (uint64_t)bh, (uint64_t)nh, other, 5};
    uint64_t strides[4] = {rs, rs * bh, os, (uint64_t)slab * 8};
    uint32_t box[5] = {WC, (uint32_t)bh, (uint32_t)nh, 1, 5};
    const int npw = nx / WC;
    const int64_t nblocks = (int64_t)npw * other;
    if (nblocks >= (int64_t)1 << 31) return IB_ERROR_NOIMPLEMENT;
    CUtensorMap tm;
    int rc = encode_tmap_f64(&tm, q, 5, dims, strides, box);
    if (rc) return rc;
    unsigned int *err = scratch().wait_flag();
    if (!err) return IB_ERROR_NOMEM;
    const int nt = (n + 31) / 32 * 32;
    if (PADN && n > PADN) return IB_ERROR_NOIMPLEMENT;
    const size_t shm = pair_smem_bytes(n, (int)sizeof(FT), WC, NFIX ? NFIX : (PADN ? PADN : n));
    const int ns = (nsweep == 2) ? 2 : 1;
    auto kern = &sweep_pair_kernel<METHOD, SLOPE, FT, DIR, NFIX, 1, WC, GEO, PADN>;
    if constexpr (GEO == CYL_NONE) {
        if (ns == 2) kern = &sweep_pair_kernel<METHOD, SLOPE, FT, DIR, NFIX, 2, WC, CYL_NONE, PADN>;
    }
    static int attr_bytes[2] = {0, 0};
    if ((int)shm > attr_bytes[ns - 1]) {
        rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        if (rc) return rc;
        attr_bytes[ns - 1] = (int)shm;
    }
    PipeArgs a{n, npw, bh, nh, nblocks, lambda, err, tile_wait_limit()};
    kern<<<(unsigned)nblocks, nt, shm, st>>>(tm, a, c, cyl);
    return check_launch();
}

// Radial rows (cylindrical x sweeps) of at most 512 cells: the row kernel with the radial update,
// one CTA per row.  Returns IB_ERROR_NOIMPLEMENT (caller falls back) for longer rows.
template <int METHOD, int SLOPE>
int launch_row_radial(double *q, int64_t slab, const int grid[3], DevScalar lambda, const FluidConsts<double> &c,
                      cudaStream_t st, const CylPencil &cyl)
{
    const int nx = grid[0];
    if (nx > 512) return IB_ERROR_NOIMPLEMENT;
    SweepArgs a{q, slab, grid[0], grid[1], grid[2], lambda, cyl.rin, cyl.dr};
    const int64_t rows = (int64_t)grid[1] * grid[2];
    const int nt = ((nx + 31) / 32) * 32;
    const size_t shm = (size_t)10 * nx * sizeof(double) + (size_t)40 * nx;  // two planes, the SSPRK sum
    if (nx == 256) {  // the length at compile time (constant plane offsets, fewer spills); 30 KB
        sweep_row_kernel<METHOD, SLOPE, double, 1, 256, 1, CYL_RADIAL><<<(unsigned)rows, nt, shm, st>>>(a, c);
        return check_launch();
    }
    auto kern = sweep_row_kernel<METHOD, SLOPE, double, 1, 0, 1, CYL_RADIAL>;
    static int attr_bytes = 0;
    if ((int)shm > attr_bytes) {
        int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        if (rc) return rc;
        attr_bytes = (int)shm;
    }
    kern<<<(unsigned)rows, nt, shm, st>>>(a, c);
    return check_launch();
}

// Chunked TMA pipeline (sweep_chunk_kernel) for pencils of more than 512 cells: W = 1, R = 256
// (x rows) or W = 4, R = 128 (y/z pencils), after chunk_halo_kernel has copied the rows around the
// chunk boundaries to scratch memory.  Returns IB_ERROR_NOIMPLEMENT (caller falls back) when the
// grid does not meet TMA's rules: x rows of even length; y/z with W dividing nx.
template <int METHOD, int SLOPE, typename FT, int DIR, int W, int R>
int launch_chunk(double *q, int64_t slab, const int grid[3], DevScalar lambda, const FluidConsts<FT> &c, cudaStream_t st)
{
    constexpr int L = R - 8;
    const int nx = grid[0], ny = grid[1], nz = grid[2];
    const int n = grid[DIR - 1];
    if (n <= 512) return IB_ERROR_NOIMPLEMENT;
    if (DIR == 1 && (n & 1)) return IB_ERROR_NOIMPLEMENT;
    if (DIR != 1 && ((nx & 1) || nx % W)) return IB_ERROR_NOIMPLEMENT;
    if (((uintptr_t)q & 15) || (slab * 8) % 16) return IB_ERROR_NOIMPLEMENT;
    CUtensorMap tm;
    uint64_t dims[4], strides[3];
    uint32_t box[4];
    int rank;
    ChunkArgs a;
    a.q = q;
    a.slab = slab;
    a.n = n;
    a.C = (n + L - 1) / L;
    a.lambda = lambda;
    if (DIR == 1) {
        rank = 3;
        dims[0] = nx; dims[1] = (uint64_t)ny * nz; dims[2] = 5;
        strides[0] = (uint64_t)nx * 8; strides[1] = (uint64_t)slab * 8;
        box[0] = L; box[1] = 1; box[2] = 5;
        a.rs = 1; a.os = nx; a.npw = 1;
        a.ngroups = (int64_t)ny * nz;
    } else {
        rank = 4;
        const uint64_t other = (DIR == 2) ? nz : ny;
        a.rs = (DIR == 2) ? (int64_t)nx : (int64_t)nx * ny;
        a.os = (DIR == 2) ? (int64_t)nx * ny : (int64_t)nx;
        dims[0] = nx; dims[1] = n; dims[2] = other; dims[3] = 5;
        strides[0] = (uint64_t)a.rs * 8; strides[1] = (uint64_t)a.os * 8; strides[2] = (uint64_t)slab * 8;
        box[0] = W; box[1] = L; box[2] = 1; box[3] = 5;
        a.npw = nx / W;
        a.ngroups = (int64_t)a.npw * other;
    }
    if (a.ngroups >= ((int64_t)1 << 31) / a.C) return IB_ERROR_NOIMPLEMENT;
    int rc = encode_tmap_f64(&tm, q, rank, dims, strides, box);
    if (rc) return rc;
    a.err = scratch().wait_flag();
    if (!a.err) return IB_ERROR_NOMEM;
    a.spin = tile_wait_limit();
    // halo rows of every chunk boundary, copied before the sweep overwrites them
    const int64_t nside = a.ngroups * a.C * 40 * W;
    double *side = scratch().bytes((size_t)nside * sizeof(double));
    if (!side) return IB_ERROR_NOMEM;
    a.side = side;
    {
        const int hb = (int)std::min<int64_t>((nside + 255) / 256, (int64_t)8 * num_sms());
        chunk_halo_kernel<DIR, W><<<hb, 256, 0, st>>>(a, L, side);
        rc = check_launch();
        if (rc) return rc;
    }
    const int nt = W * R;
    const size_t shm = chunk_smem_bytes(W, R, (int)sizeof(FT));
    auto kern = sweep_chunk_kernel<METHOD, SLOPE, FT, DIR, W, R>;
    static int attr_bytes = 0;
    if ((int)shm > attr_bytes) {
        rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        if (rc) return rc;
        attr_bytes = (int)shm;
    }
    int per_sm = 0;
    rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, shm));
    if (rc) return rc;
    if (per_sm < 1) return IB_ERROR_NOIMPLEMENT;
    const int64_t njobs = a.ngroups * a.C;
    const unsigned nblk = (unsigned)std::min<int64_t>((int64_t)per_sm * num_sms(), njobs);
    kern<<<nblk, nt, shm, st>>>(tm, a, c);
    return check_launch();
}

template <int METHOD, int SLOPE, typename FT>
int launch_tile_t(int dir, double *q, int64_t slab, const int grid[3], DevScalar lambda, const FluidConsts<FT> &c,
                  cudaStream_t st)
{
    if (dir == 1) return launch_tile_dw<METHOD, SLOPE, FT, 1, 1>(q, slab, grid, lambda, c, st, 248);
    if (dir == 2) return launch_tile_dw<METHOD, SLOPE, FT, 2, 4>(q, slab, grid, lambda, c, st, 56);
    return launch_tile_dw<METHOD, SLOPE, FT, 3, 4>(q, slab, grid, lambda, c, st, 56);
}

// One sweep along dir, or nsweep = 2 sweeps in a row with the same lambda (the two same-axis
// sweeps in the middle of an iteration).  The row and pipeline kernels apply both to a block
// while it is on chip; the chunked pipeline and the tile kernel are launched once per sweep.
template <int METHOD, int SLOPE, typename FT>
int launch_sweep_t(int dir, double *q, int64_t slab, const int grid[3], DevScalar lambda, const FluidConsts<FT> &c,
                   cudaStream_t st, int nsweep = 1)
{
    const int nx = grid[0], ny = grid[1], nz = grid[2];
    const int n = grid[dir - 1];
    const int64_t N = (int64_t)nx * ny * nz;
    if (n <= 0 || N <= 0) return IB_SUCCESSFUL;

    static const bool use_pipe = [] {
        const char *e = getenv("IMOGEN_B200_PIPE");  // 0 = the non-TMA kernels only
        return !(e && e[0] == '0');
    }();
    // x rows load contiguously and the row kernel below is faster for them; y and z pencils
    // go through the TMA-fed pipeline (IMOGEN_B200_PIPE=x also sends x rows there)
    static const int pipe_x = [] {
        const char *e = getenv("IMOGEN_B200_PIPE");
        return (e && e[0] == 'x') ? 1 : 0;
    }();
    if (use_pipe && n <= 512 && (dir > 1 || pipe_x)) {
        int rc = IB_ERROR_NOIMPLEMENT;
        // z pencils of large x-y planes: blocks 4 columns wide (32-byte rows), which the memory
        // system serves far better than 16-byte rows at megabyte strides
        const bool wide = (dir == 3) && ((int64_t)nx * ny * 8 > (1 << 20));
        // y/z pencils of up to 256 cells and of 512 take the pencil-pair kernel (one 2-pencil box
        // per 256-thread CTA, four CTAs per SM: 256^3 FP64 y 0.93 -> 0.76 ms, FP32 flux
        // 0.52 -> 0.44 ms; 512-cell y pencils 4.01 -> 3.60 ms at 512 x 512 x 256) rather than the
        // persistent pipeline, which remains for other lengths when the pair kernel declines
        // (pencils shorter than pair_min_cells() leave most of a pencil-pair CTA idle: pipeline)
        const bool pair = n >= pair_min_cells();
        constexpr bool pair512 = true;
        // z of x-y planes above 1 MB, FP64: 4-pencil boxes through the pencil-pair kernel (512 x 512
        // x 256: z 3.96 -> 3.58 ms); FP32 flux keeps its 8-column wide blocks (2.43 ms against 2.77
        // for the 4-pencil boxes)
        const bool wide4 = sizeof(FT) == 8 && pair;
        static const int wide8 = [] {
            const char *e = getenv("IMOGEN_B200_WIDE8");  // 0 = 4-column blocks for wide z planes
            return (e && e[0] == '0') ? 0 : 1;
        }();
        if (dir == 1) {
            if (n <= 256) rc = launch_pipe<METHOD, SLOPE, FT, 1, 1, 1>(q, slab, grid, lambda, c, st, nsweep);
        } else if (n == 256 && !wide) {
            if (pair) {
                if (dir == 2) rc = launch_pair<METHOD, SLOPE, FT, 2, 256>(q, slab, grid, lambda, c, st, nsweep);
                else rc = launch_pair<METHOD, SLOPE, FT, 3, 256>(q, slab, grid, lambda, c, st, nsweep);
            } else if (dir == 2) rc = launch_pipe<METHOD, SLOPE, FT, 2, 2, 1, 256>(q, slab, grid, lambda, c, st, nsweep);
            else rc = launch_pipe<METHOD, SLOPE, FT, 3, 2, 1, 256>(q, slab, grid, lambda, c, st, nsweep);
        } else if (n == 128 && !wide) {
            if (pair) {
                if (dir == 2) rc = launch_pair<METHOD, SLOPE, FT, 2, 128>(q, slab, grid, lambda, c, st, nsweep);
                else rc = launch_pair<METHOD, SLOPE, FT, 3, 128>(q, slab, grid, lambda, c, st, nsweep);
            } else if (dir == 2) rc = launch_pipe<METHOD, SLOPE, FT, 2, 2, 1, 128>(q, slab, grid, lambda, c, st, nsweep);
            else rc = launch_pipe<METHOD, SLOPE, FT, 3, 2, 1, 128>(q, slab, grid, lambda, c, st, nsweep);
        } else if (n <= 256 && !wide) {
            if (pair) {
                // Pencils of 65-127 cells (HLLC, FP32 flux too; HLL FP64) and of 129-255 (HLLC):
                // planes of a fixed 128- or 256-cell stride (HLLC FP64 96^3 y/z 0.061 -> 0.053 ms,
                // 160^3 0.254 -> 0.225, 192^3 0.436 -> 0.387; FP32 flux 192^3 0.225 -> 0.199; HLL
                // 112^3 0.104 -> 0.102).  HLL's 129-255-cell pencils measured 4-5 % slower with it,
                // and so did a 256-cell stride for pencils of 128 or fewer: the larger planes cost
                // CTAs per SM.
                constexpr bool padded128 =
                    METHOD == IB_METHOD_HLLC || (METHOD == IB_METHOD_HLL && sizeof(FT) == 8);
                constexpr bool padded = METHOD == IB_METHOD_HLLC;
                if (padded128 && n > 64 && n < 128) {
                    if (dir == 2) rc = launch_pair<METHOD, SLOPE, FT, 2, 0, 2, CYL_NONE, padded128 ? 128 : 0>(
                                      q, slab, grid, lambda, c, st, nsweep);
                    else rc = launch_pair<METHOD, SLOPE, FT, 3, 0, 2, CYL_NONE, padded128 ? 128 : 0>(
                             q, slab, grid, lambda, c, st, nsweep);
                } else if (padded && n > 128) {
                    if (dir == 2) rc = launch_pair<METHOD, SLOPE, FT, 2, 0, 2, CYL_NONE, padded ? 256 : 0>(
                                      q, slab, grid, lambda, c, st, nsweep);
                    else rc = launch_pair<METHOD, SLOPE, FT, 3, 0, 2, CYL_NONE, padded ? 256 : 0>(q, slab, grid, lambda,
                                                                                                c, st, nsweep);
                } else if (dir == 2) rc = launch_pair<METHOD, SLOPE, FT, 2>(q, slab, grid, lambda, c, st, nsweep);
                else rc = launch_pair<METHOD, SLOPE, FT, 3>(q, slab, grid, lambda, c, st, nsweep);
            }
            if (rc == IB_ERROR_NOIMPLEMENT) {
                if (dir == 2) rc = launch_pipe<METHOD, SLOPE, FT, 2, 2, 1>(q, slab, grid, lambda, c, st, nsweep);
                else rc = launch_pipe<METHOD, SLOPE, FT, 3, 2, 1>(q, slab, grid, lambda, c, st, nsweep);
            }
        } else if (n == 256) {
            // z of x-y planes above 1 MB: FP64 takes 4-pencil boxes (32-byte rows) through the
            // pencil-pair kernel; the FP32 flux takes 8-column wide blocks (64-byte rows) computed 4
            // columns at a time (3.48 -> 2.52 ms at 512 x 512 x 256); the 4-column pipeline blocks
            // remain where neither applies.
            if (wide4) rc = launch_pair<METHOD, SLOPE, FT, 3, 256, 4>(q, slab, grid, lambda, c, st, nsweep);
            if constexpr (sizeof(FT) == 4) {
                if (rc == IB_ERROR_NOIMPLEMENT && wide8 == 1)
                    rc = launch_pipe<METHOD, SLOPE, FT, 3, 4, 2, 256, 2>(q, slab, grid, lambda, c, st, nsweep);
            }
            if (rc == IB_ERROR_NOIMPLEMENT) rc = launch_pipe<METHOD, SLOPE, FT, 3, 4, 2, 256>(q, slab, grid, lambda, c, st, nsweep);
        } else if (n <= 256) {
            if (wide4) rc = launch_pair<METHOD, SLOPE, FT, 3, 0, 4>(q, slab, grid, lambda, c, st, nsweep);
            if constexpr (sizeof(FT) == 4) {
                if (rc == IB_ERROR_NOIMPLEMENT && wide8 == 1)
                    rc = launch_pipe<METHOD, SLOPE, FT, 3, 4, 2, 0, 2>(q, slab, grid, lambda, c, st, nsweep);
            }
            if (rc == IB_ERROR_NOIMPLEMENT) rc = launch_pipe<METHOD, SLOPE, FT, 3, 4, 2>(q, slab, grid, lambda, c, st, nsweep);
        } else if (n == 512) {
            if (pair512) {
                if (dir == 2) rc = launch_pair<METHOD, SLOPE, FT, 2, 512>(q, slab, grid, lambda, c, st, nsweep);
                else rc = launch_pair<METHOD, SLOPE, FT, 3, 512>(q, slab, grid, lambda, c, st, nsweep);
            }
            if (rc == IB_ERROR_NOIMPLEMENT) {
                if (dir == 2) rc = launch_pipe<METHOD, SLOPE, FT, 2, 2, 2, 512>(q, slab, grid, lambda, c, st, nsweep);
                else rc = launch_pipe<METHOD, SLOPE, FT, 3, 2, 2, 512>(q, slab, grid, lambda, c, st, nsweep);
            }
        } else {
            if (dir == 2) rc = launch_pipe<METHOD, SLOPE, FT, 2, 2, 2>(q, slab, grid, lambda, c, st, nsweep);
            else rc = launch_pipe<METHOD, SLOPE, FT, 3, 2, 2>(q, slab, grid, lambda, c, st, nsweep);
        }
        if (rc != IB_ERROR_NOIMPLEMENT) return rc;
    }

    // pencils above 512 cells: chunked TMA pipeline (x rows above 1024 cells; y and z above 512)
    static const int use_chunk = [] {
        const char *e = getenv("IMOGEN_B200_CHUNK");  // 0 = the tile kernel for long pencils
        return (e && e[0] == '0') ? 0 : 1;
    }();
    if (use_pipe && use_chunk && n > 512 && (dir > 1 || nx > 1024)) {
        int rc;
        if (nsweep > 1) {
            rc = launch_sweep_t<METHOD, SLOPE, FT>(dir, q, slab, grid, lambda, c, st, 1);
            if (rc) return rc;
            return launch_sweep_t<METHOD, SLOPE, FT>(dir, q, slab, grid, lambda, c, st, nsweep - 1);
        }
        if (dir == 1) rc = launch_chunk<METHOD, SLOPE, FT, 1, 1, 256>(q, slab, grid, lambda, c, st);
        else if (dir == 2) rc = launch_chunk<METHOD, SLOPE, FT, 2, 4, 128>(q, slab, grid, lambda, c, st);
        else rc = launch_chunk<METHOD, SLOPE, FT, 3, 4, 128>(q, slab, grid, lambda, c, st);
        if (rc != IB_ERROR_NOIMPLEMENT) return rc;
    }

    if (dir == 1 && nx <= 1024) {
        // one CTA per row, one or two cells per thread
        SweepArgs a{q, slab, nx, ny, nz, lambda};
        const int64_t rows = (int64_t)ny * nz;
        static const int xcpt = [] {
            const char *e = getenv("IMOGEN_B200_XCPT");  // 2 = two cells per thread for all rows
            return (e && e[0] == '2') ? 2 : 1;
        }();
        const int cpt = (nx <= 512 && xcpt == 1) ? 1 : 2;
        // the planes, plus the SSPRK sum where row_ssum holds (one cell per thread, rows but 512)
        const size_t shm = (size_t)10 * nx * sizeof(FT) + ((cpt == 1 && nx != 512) ? (size_t)40 * nx : 0);
        // rows above 384 FP64 cells need more than the default 48 KB of shared memory
        auto opt_in = [](auto kern, size_t bytes) {
            return check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        };
        auto launch_rows = [&](auto ns_tag) -> int {
            constexpr int NS = decltype(ns_tag)::value;
            if (cpt == 1) {
                int nt = ((nx + 31) / 32) * 32;
                const size_t max1 = (size_t)10 * 512 * sizeof(FT) + (size_t)40 * 512;
                // common row lengths get the length at compile time (cheaper shared-memory indexing)
                if (nx == 256) {
                    sweep_row_kernel<METHOD, SLOPE, FT, 1, 256, NS><<<(unsigned)rows, nt, shm, st>>>(a, c);
                } else if (nx == 512) {
                    static const int rc0 = opt_in(sweep_row_kernel<METHOD, SLOPE, FT, 1, 512, NS>, max1);
                    if (rc0) return rc0;
                    sweep_row_kernel<METHOD, SLOPE, FT, 1, 512, NS><<<(unsigned)rows, nt, shm, st>>>(a, c);
                } else if (nx == 128) {
                    sweep_row_kernel<METHOD, SLOPE, FT, 1, 128, NS><<<(unsigned)rows, nt, shm, st>>>(a, c);
                } else if ((METHOD == IB_METHOD_HLLC || (METHOD == IB_METHOD_HLL && sizeof(FT) == 8)) && nx > 64 &&
                           nx < 128) {
                    // planes of a fixed 128- or 256-cell stride: constant offsets in the phases,
                    // fewer spills (HLLC 96^3 x 0.049 -> 0.046 ms, 160^3 0.204 -> 0.190; HLL 4-5 %)
                    const size_t shm_p = (size_t)10 * 128 * sizeof(FT) + (size_t)40 * 128;
                    sweep_row_kernel<METHOD, SLOPE, FT, 1, 0, NS, CYL_NONE, 128><<<(unsigned)rows, nt, shm_p, st>>>(a, c);
                } else if (METHOD == IB_METHOD_HLLC && nx > 256 && nx < 512) {
                    // HLLC rows of 257-511 cells: planes of a fixed 512-cell stride (384 cells: x
                    // 0.209 -> 0.195 ms at 384 x 96 x 96, FP32 flux 0.111 -> 0.106; registers already
                    // limit these CTAs to two per SM, so the larger planes cost none)
                    const size_t shm_p = (size_t)10 * 512 * sizeof(FT) + (size_t)40 * 512;
                    static const int rcp = opt_in(sweep_row_kernel<METHOD, SLOPE, FT, 1, 0, NS, CYL_NONE, 512>, shm_p);
                    if (rcp) return rcp;
                    sweep_row_kernel<METHOD, SLOPE, FT, 1, 0, NS, CYL_NONE, 512><<<(unsigned)rows, nt, shm_p, st>>>(a, c);
                } else if ((METHOD == IB_METHOD_HLLC || (METHOD == IB_METHOD_HLL && sizeof(FT) == 8)) && nx > 128 &&
                           nx < 256) {
                    const size_t shm_p = (size_t)10 * 256 * sizeof(FT) + (size_t)40 * 256;
                    sweep_row_kernel<METHOD, SLOPE, FT, 1, 0, NS, CYL_NONE, 256><<<(unsigned)rows, nt, shm_p, st>>>(a, c);
                } else {
                    static const int rc1 = opt_in(sweep_row_kernel<METHOD, SLOPE, FT, 1, 0, NS>, max1);
                    if (rc1) return rc1;
                    sweep_row_kernel<METHOD, SLOPE, FT, 1, 0, NS><<<(unsigned)rows, nt, shm, st>>>(a, c);
                }
            } else {
                int nt = (((nx + 1) / 2 + 31) / 32) * 32;
                static const int rc2 =
                    opt_in(sweep_row_kernel<METHOD, SLOPE, FT, 2, 0, NS>, (size_t)10 * 1024 * sizeof(FT));
                if (rc2) return rc2;
                sweep_row_kernel<METHOD, SLOPE, FT, 2, 0, NS><<<(unsigned)rows, nt, shm, st>>>(a, c);
            }
            return IB_SUCCESSFUL;
        };
        int rc = (nsweep == 2) ? launch_rows(std::integral_constant<int, 2>{})
                               : launch_rows(std::integral_constant<int, 1>{});
        if (rc) return rc;
        return check_launch();
    }

    for (int k = 0; k < nsweep; k++) {
        int rc = launch_tile_t<METHOD, SLOPE, FT>(dir, q, slab, grid, lambda, c, st);
        if (rc) return rc;
    }
    return IB_SUCCESSFUL;
}

template <int METHOD, typename FT>
int launch_sweep_slope(int slope, int dir, double *q, int64_t slab, const int grid[3], DevScalar lambda, double gamma,
                       double rho_min, double c_iso, cudaStream_t st, int nsweep)
{
    FluidConsts<FT> c = make_consts<FT>(gamma, rho_min, c_iso);
    switch (slope) {
    case IB_SLOPE_OSPRE: return launch_sweep_t<METHOD, IB_SLOPE_OSPRE, FT>(dir, q, slab, grid, lambda, c, st, nsweep);
    case IB_SLOPE_MC: return launch_sweep_t<METHOD, IB_SLOPE_MC, FT>(dir, q, slab, grid, lambda, c, st, nsweep);
    case IB_SLOPE_VANLEER: return launch_sweep_t<METHOD, IB_SLOPE_VANLEER, FT>(dir, q, slab, grid, lambda, c, st, nsweep);
    case IB_SLOPE_MINMOD: return launch_sweep_t<METHOD, IB_SLOPE_MINMOD, FT>(dir, q, slab, grid, lambda, c, st, nsweep);
    case IB_SLOPE_SUPERBEE: return launch_sweep_t<METHOD, IB_SLOPE_SUPERBEE, FT>(dir, q, slab, grid, lambda, c, st, nsweep);
    case IB_SLOPE_VANALBADA: return launch_sweep_t<METHOD, IB_SLOPE_VANALBADA, FT>(dir, q, slab, grid, lambda, c, st, nsweep);
    case IB_SLOPE_ZERO: return launch_sweep_t<METHOD, IB_SLOPE_ZERO, FT>(dir, q, slab, grid, lambda, c, st, nsweep);
    default: return IB_ERROR_INVALID_ARGS;
    }
}

// Cylindrical sweeps, FP64: radial x rows of up to 512 cells in the row kernel and theta y pencils
// of up to 256 cells (x even) in the pencil-pair kernel, each with the geometry's update; other
// shapes in the tile kernel with the same update
template <int METHOD, int SLOPE>
int launch_sweep_cyl_t(double *q, int64_t slab, const int grid[3], DevScalar lambda, const FluidConsts<double> &c,
                       cudaStream_t st, const CylSweep &cs)
{
    static const bool fast_env = [] {
        const char *e = getenv("IMOGEN_B200_CYLFAST");  // 0 = the tile kernel for every cylindrical sweep
        return !(e && e[0] == '0');
    }();
    // theta pencils shorter than pair_min_cells() take the tile kernel (several pencils a CTA)
    const bool fast = fast_env && (cs.kind == CYL_RADIAL || grid[1] >= pair_min_cells());
    int rc = IB_ERROR_NOIMPLEMENT;
    switch (cs.kind) {
    case CYL_RADIAL:
        if (fast) rc = launch_row_radial<METHOD, SLOPE>(q, slab, grid, lambda, c, st, cs.pencil);
        if (rc != IB_ERROR_NOIMPLEMENT) return rc;
        return launch_tile_dw<METHOD, SLOPE, double, 1, 1, CYL_RADIAL>(q, slab, grid, lambda, c, st, 248, cs.pencil);
    case CYL_THETA_DIV:
        // 256-cell pencils get the length at compile time (fewer registers for indexing, no spills)
        if (fast && grid[1] == 256)
            rc = launch_pair<METHOD, SLOPE, double, 2, 256, 2, CYL_THETA_DIV>(q, slab, grid, lambda, c, st, 1, cs.pencil);
        else if (fast)
            rc = launch_pair<METHOD, SLOPE, double, 2, 0, 2, CYL_THETA_DIV>(q, slab, grid, lambda, c, st, 1, cs.pencil);
        if (rc != IB_ERROR_NOIMPLEMENT) return rc;
        return launch_tile_dw<METHOD, SLOPE, double, 2, 4, CYL_THETA_DIV>(q, slab, grid, lambda, c, st, 56, cs.pencil);
    case CYL_THETA_LAM:
        if (fast && grid[1] == 256)
            rc = launch_pair<METHOD, SLOPE, double, 2, 256, 2, CYL_THETA_LAM>(q, slab, grid, lambda, c, st, 1, cs.pencil);
        else if (fast)
            rc = launch_pair<METHOD, SLOPE, double, 2, 0, 2, CYL_THETA_LAM>(q, slab, grid, lambda, c, st, 1, cs.pencil);
        if (rc != IB_ERROR_NOIMPLEMENT) return rc;
        return launch_tile_dw<METHOD, SLOPE, double, 2, 4, CYL_THETA_LAM>(q, slab, grid, lambda, c, st, 56, cs.pencil);
    default: return IB_ERROR_INVALID_ARGS;
    }
}

template <int METHOD>
int launch_sweep_cyl_slope(int slope, double *q, int64_t slab, const int grid[3], DevScalar lambda, double gamma,
                           double rho_min, double c_iso, cudaStream_t st, const CylSweep &cs)
{
    FluidConsts<double> c = make_consts<double>(gamma, rho_min, c_iso);
    switch (slope) {
    case IB_SLOPE_OSPRE: return launch_sweep_cyl_t<METHOD, IB_SLOPE_OSPRE>(q, slab, grid, lambda, c, st, cs);
    case IB_SLOPE_MC: return launch_sweep_cyl_t<METHOD, IB_SLOPE_MC>(q, slab, grid, lambda, c, st, cs);
    case IB_SLOPE_VANLEER: return launch_sweep_cyl_t<METHOD, IB_SLOPE_VANLEER>(q, slab, grid, lambda, c, st, cs);
    case IB_SLOPE_MINMOD: return launch_sweep_cyl_t<METHOD, IB_SLOPE_MINMOD>(q, slab, grid, lambda, c, st, cs);
    case IB_SLOPE_SUPERBEE: return launch_sweep_cyl_t<METHOD, IB_SLOPE_SUPERBEE>(q, slab, grid, lambda, c, st, cs);
    case IB_SLOPE_VANALBADA: return launch_sweep_cyl_t<METHOD, IB_SLOPE_VANALBADA>(q, slab, grid, lambda, c, st, cs);
    case IB_SLOPE_ZERO: return launch_sweep_cyl_t<METHOD, IB_SLOPE_ZERO>(q, slab, grid, lambda, c, st, cs);
    default: return IB_ERROR_INVALID_ARGS;
    }
}

int launch_hllc64(int slope, int dir, double *q, int64_t slab, const int grid[3], DevScalar lambda, double gamma,
                  double rho_min, double c_iso, cudaStream_t st, int nsweep);
int launch_hllc32(int slope, int dir, double *q, int64_t slab, const int grid[3], DevScalar lambda, double gamma,
                  double rho_min, double c_iso, cudaStream_t st, int nsweep);
int launch_hll64(int slope, int dir, double *q, int64_t slab, const int grid[3], DevScalar lambda, double gamma,
                 double rho_min, double c_iso, cudaStream_t st, int nsweep);

}  // namespace ib
