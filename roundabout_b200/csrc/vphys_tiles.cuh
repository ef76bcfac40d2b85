// vphys_tiles.cuh -- the face-tile geometry of the TMA-staged momentum solve,
// as host/device functions without device intrinsics, so the CPU tests
// compile this header as plain C++ and check that every shared-memory index
// the kernel forms from it stays inside its block.
#pragma once

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#endif

namespace vphys {

// Tile shape of the TMA-staged momentum solve: consumer warps per CTA, faces
// per tile, cells per block row (the tile's cells from an even start).
constexpr int MT_WARPS = 4;
constexpr int MT_TW = 32 * MT_WARPS;
constexpr int MT_BW = MT_TW + 4;

// ---- face tiles of the momentum solve --------------------------------------
// A tile is TW consecutive faces of one family in the flattened face index:
// u faces f = i + (nx+1) j (i in [0, nx], j in [0, ny)), v faces f = i + nx j
// (i in [0, nx), j in [0, ny]).  The cells either side of every face of a tile
// come from level blocks of the cell fields whose first element is rounded
// down to an even index (a tiled TMA copy of 8-byte elements must start on a
// 16-byte boundary); `box` is the number of cells such a block holds.
struct FaceTile {
    long long xa, xb;   // first cell index of block A / block B (even; xb only for v tiles)
    long long xw;       // first face index of the tile (the velocity block)
};
// For face `f` of a tile: which block (0: A, 1: B) and which offset inside it
// hold the left/lower and the right/upper cell.
struct FaceCells {
    int bl, ol, br, orr;
    long long cl, cr;   // the cells' flattened indices (the clamping of the reference)
};

__host__ __device__ __forceinline__ long long floor_even(long long x) { return x - (x & 1); }

__host__ __device__ __forceinline__ FaceTile face_tile(bool xf, long long f0, int nx)
{
    FaceTile t;
    t.xw = f0;
    if (xf) {
        const long long j0 = f0 / (nx + 1), i0 = f0 - j0 * (nx + 1);
        const long long cl0 = (i0 > 0 ? i0 - 1 : 0) + (long long)nx * j0;
        t.xa = floor_even(cl0);
        t.xb = t.xa;
    } else {
        t.xa = floor_even(f0 - nx);   // row j-1 of the tile's faces (negative rows are never read)
        t.xb = floor_even(f0);        // row j
    }
    return t;
}

__host__ __device__ __forceinline__ FaceCells face_cells(bool xf, long long f, int nx, int ny, const FaceTile &t)
{
    FaceCells c;
    if (xf) {
        const long long j = f / (nx + 1), i = f - j * (nx + 1);
        const long long il = i - 1 > 0 ? i - 1 : 0, ir = i < nx - 1 ? i : nx - 1;
        c.cl = il + (long long)nx * j;
        c.cr = ir + (long long)nx * j;
        c.bl = 0;
        c.br = 0;
        c.ol = (int)(c.cl - t.xa);
        c.orr = (int)(c.cr - t.xa);
    } else {
        const long long j = f / nx, i = f - j * nx;
        const long long jb = j - 1 > 0 ? j - 1 : 0, ja = j < ny - 1 ? j : ny - 1;
        c.cl = i + (long long)nx * jb;
        c.cr = i + (long long)nx * ja;
        // block A holds row j-1 of the tile's faces, block B row j; a clamped
        // cell is read from the block that holds its row
        c.bl = (jb == j - 1) ? 0 : 1;
        c.ol = (int)(c.cl - (c.bl ? t.xb : t.xa));
        c.br = (ja == j) ? 1 : 0;
        c.orr = (int)(c.cr - (c.br ? t.xb : t.xa));
    }
    return c;
}

}  // namespace vphys
