// ib_tags.cu -- host-side decoding of the reference's GPU tags into the library's structs.
//
// A Matlab GPU array of the reference (GPU_Type / ImogenArray) crosses into a mex function as an
// int64 vector, its "GPU tag" (cudaCommon.h:184-196):
//   [dim0, dim1, dim2, numSlabs, halo, partitionDir, nGPUs, exteriorHalo, permtag,
//    circularBits, vectorComponent, (deviceID, devicePtr) x nGPUs]
// deserializeTagToMGArray (cudaCommon.cu:117-170) unpacks it; sanityCheckTag
// (cudaCommonML.cu:109-198) rejects malformed ones; a fluid is the FluidManager canister's five
// arrays mass, ener, mom(1..3) (MGA_accessFluidCanister, cudaCommonML.cu:400-432), slabs of one
// allocation laid out by MGA_allocSlab (cudaCommon.cu:339-370); boundary modes come from the
// arrays' boundaryData.bcModes strings (decodeMatlabBCs, cudaCommonML.cu:203-232).
//
// Only what this library runs is accepted: one GPU (nGPUs == 1), arrays in XYZ order (permtag 1,
// or 0, which the reference lets through as unset), and the five slabs of a fluid at a common
// pitch in one allocation.  Everything else returns a status code; nothing here touches the GPU.
#include <cstdint>
#include <cstring>

#include "../../include/imogen_b200.h"

namespace {

// sanityCheckTag (cudaCommonML.cu:109-198) for a non-null array
int check_tag(const int64_t *t, int32_t len)
{
    if (!t) return IB_ERROR_NULL_POINTER;
    if (len < IB_GPU_TAG_LENGTH) return IB_ERROR_INVALID_ARGS;
    const int64_t nx = t[IB_GPU_TAG_DIM0], ny = t[IB_GPU_TAG_DIM1], nz = t[IB_GPU_TAG_DIM2];
    if (nx < 0 || ny < 0 || nz < 0) return IB_ERROR_INVALID_ARGS;
    const int64_t ndev = t[IB_GPU_TAG_NGPUS];
    if (ndev < 1 || ndev > IB_GPU_TAG_MAX_GPUS) return IB_ERROR_INVALID_ARGS;
    if (t[IB_GPU_TAG_HALO] < 0) return IB_ERROR_INVALID_ARGS;
    const int64_t perm = t[IB_GPU_TAG_PERMTAG];
    if (perm < 0 || perm > 6) return IB_ERROR_INVALID_ARGS;
    const int64_t circ = t[IB_GPU_TAG_CIRCULARBITS];
    if (circ < 0 || circ > 63) return IB_ERROR_INVALID_ARGS;
    const int64_t vec = t[IB_GPU_TAG_VECTOR_COMPONENT];
    if (vec < 0 || vec > 3) return IB_ERROR_INVALID_ARGS;
    const int64_t pdir = t[IB_GPU_TAG_PARTDIR];
    if (pdir < 1 || pdir > 3) return IB_ERROR_INVALID_ARGS;
    if (len != IB_GPU_TAG_LENGTH + 2 * ndev) return IB_ERROR_INVALID_ARGS;
    for (int64_t j = 0; j < ndev; j++) {
        const int64_t dev = t[IB_GPU_TAG_LENGTH + 2 * j];
        if (dev < 0 || dev >= IB_GPU_TAG_MAX_GPUS) return IB_ERROR_INVALID_ARGS;
    }
    // what this library runs: one GPU, XYZ memory order, a non-empty array
    if (ndev != 1) return IB_ERROR_NOIMPLEMENT;
    if (perm != 0 && perm != 1) return IB_ERROR_NOIMPLEMENT;
    if (nx < 1 || ny < 1 || nz < 1) return IB_ERROR_INVALID_ARGS;
    if (nx > INT32_MAX || ny > INT32_MAX || nz > INT32_MAX) return IB_ERROR_INVALID_ARGS;
    if (t[IB_GPU_TAG_LENGTH + 1] == 0) return IB_ERROR_NULL_POINTER;
    return IB_SUCCESSFUL;
}

// One slab's pitch in doubles: numel * 8 bytes rounded up to 256 (MGA_allocSlab via
// deserializeTagToMGArray's slabPitch, cudaCommon.cu:147-148)
int64_t tag_pitch(const int64_t *t)
{
    const int64_t n = t[IB_GPU_TAG_DIM0] * t[IB_GPU_TAG_DIM1] * t[IB_GPU_TAG_DIM2];
    return (n * 8 + 255) / 256 * 256 / 8;
}

// The MPI halo-sharing bit of each face, [-X, +X, -Y, +Y, -Z, +Z] (MGA_BOUNDARY_*, cudaCommon.h:206-211)
bool circular_bit(int64_t bits, int face) { return (bits >> face) & 1; }

}  // namespace

extern "C" {

int ib_bcModeFromString(const char *name)
{
    // decodeMatlabBCs (cudaCommonML.cu:219-226)
    if (!name) return IB_ERROR_NULL_POINTER;
    if (!strcmp(name, "circ")) return IB_BC_CIRCULAR;
    if (!strcmp(name, "const")) return IB_BC_CONST;
    if (!strcmp(name, "linear")) return IB_BC_LINEAR;
    if (!strcmp(name, "mirror")) return IB_BC_MIRROR;
    if (!strcmp(name, "bcstatic")) return IB_BC_STATIONARY;
    if (!strcmp(name, "wall")) return IB_BC_WALL;
    if (!strcmp(name, "outflow")) return IB_BC_OUTFLOW;
    if (!strcmp(name, "freebalance")) return IB_BC_FREEBALANCE;
    return IB_ERROR_INVALID_ARGS;
}

int ib_arrayFromGpuTag(const int64_t *tag, int32_t taglen, double **ptr, ib_grid *grid, int32_t *vector_component,
                       int32_t *circular_bits)
{
    if (!ptr || !grid) return IB_ERROR_NULL_POINTER;
    int rc = check_tag(tag, taglen);
    if (rc) return rc;
    *ptr = reinterpret_cast<double *>(static_cast<uintptr_t>(tag[IB_GPU_TAG_LENGTH + 1]));
    grid->nx = (int32_t)tag[IB_GPU_TAG_DIM0];
    grid->ny = (int32_t)tag[IB_GPU_TAG_DIM1];
    grid->nz = (int32_t)tag[IB_GPU_TAG_DIM2];
    grid->reserved = 0;
    grid->slab_pitch = tag_pitch(tag);
    if (vector_component) *vector_component = (int32_t)tag[IB_GPU_TAG_VECTOR_COMPONENT];
    if (circular_bits) *circular_bits = (int32_t)tag[IB_GPU_TAG_CIRCULARBITS];
    return IB_SUCCESSFUL;
}

int ib_fluidFromGpuTags(const int64_t *const tags[5], const int32_t taglen[5], const int32_t *bc_modes,
                        ib_fluid *out)
{
    if (!tags || !taglen || !out) return IB_ERROR_NULL_POINTER;
    int64_t base = 0, pitch = 0, circ = 0, dev = 0;
    for (int k = 0; k < 5; k++) {
        int rc = check_tag(tags[k], taglen[k]);
        if (rc) return rc;
        const int64_t *t = tags[k];
        // mass and ener are scalars, mom(1..3) the x, y, z components (cudaCommonML.cu:427-429)
        const int64_t want_vec = (k < 2) ? 0 : k - 1;
        if (t[IB_GPU_TAG_VECTOR_COMPONENT] != want_vec) return IB_ERROR_INVALID_ARGS;
        if (k == 0) {
            base = t[IB_GPU_TAG_LENGTH + 1];
            pitch = tag_pitch(t);
            circ = t[IB_GPU_TAG_CIRCULARBITS];
            dev = t[IB_GPU_TAG_LENGTH];
            continue;
        }
        for (int d = 0; d < 3; d++)
            if (t[d] != tags[0][d]) return IB_ERROR_INVALID_ARGS;
        if (t[IB_GPU_TAG_LENGTH] != dev) return IB_ERROR_INVALID_ARGS;
        if (t[IB_GPU_TAG_CIRCULARBITS] != circ) return IB_ERROR_INVALID_ARGS;
        // slab k of the fluid's allocation (MGA_allocSlab, cudaCommon.cu:339-370)
        if (t[IB_GPU_TAG_LENGTH + 1] != base + k * pitch * 8) return IB_ERROR_NOIMPLEMENT;
    }
    if (base % 16) return IB_ERROR_NOIMPLEMENT;  // MGA allocations are 256-byte aligned
    ib_fluid f;
    memset(&f, 0, sizeof(f));
    f.q = reinterpret_cast<double *>(static_cast<uintptr_t>(base));
    f.grid.nx = (int32_t)tags[0][IB_GPU_TAG_DIM0];
    f.grid.ny = (int32_t)tags[0][IB_GPU_TAG_DIM1];
    f.grid.nz = (int32_t)tags[0][IB_GPU_TAG_DIM2];
    f.grid.slab_pitch = pitch;
    f.halo = 4;  // the boundary depth the reference's BC kernels use (run/starterRun.m:60-67)
    for (int face = 0; face < 6; face++) {
        int mode;
        if (bc_modes) {
            mode = bc_modes[face];
            if (mode < IB_BC_CIRCULAR || mode > IB_BC_FREEBALANCE) return IB_ERROR_INVALID_ARGS;
            // a face that shares its halo circularly cannot have another boundary mode
            if (circular_bit(circ, face) && mode != IB_BC_CIRCULAR) return IB_ERROR_INVALID_ARGS;
        } else {
            // no bcModes: every face must be marked circular by the tag
            if (!circular_bit(circ, face)) return IB_ERROR_INVALID_ARGS;
            mode = IB_BC_CIRCULAR;
        }
        f.bc[face] = mode;
    }
    *out = f;
    return IB_SUCCESSFUL;
}

}  // extern "C"
