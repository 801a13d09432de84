// layout.cuh -- where a lattice lives in device memory.
//
// Populations are structure-of-arrays: nine planes, one per direction.  A plane has ly+2
// rows (Y = 0..ly+1, the ghost rows included) of `pitch` elements; node (X, Y) with
// X = 0..lx+1 sits at element Y*pitch + X + xoff - 1, so the first interior column X = 1
// starts a 128-byte line and x is the contiguous, coalesced axis (the reference's node
// array is y-contiguous, lb.c:98-100).  The tag plane uses the same element index with one
// byte per node.
//
// Slots of boundary nodes whose source lies outside the lattice ("stale" slots: the
// reference never streams into them, lb.c:258-267, so they keep the second buffer's old
// content) are kept in a side store: two parities x nine directions x `nper` perimeter
// nodes.  pidx() numbers the perimeter: row Y=1, row Y=ly, then column X=1 and column X=lx
// without their corners.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lbgpu {

struct Geo {
    int lx, ly;
    int xoff;        // element offset of column X = 1 inside a row
    int nb;          // boundary table length, max(lx, ly) + 2
    int nper;        // perimeter side-store stride, 2*lx + 2*ly
    long long pitch; // elements per row
    long long plane; // elements per direction plane, (ly + 2) * pitch
    // 16-bit storage only: the per-row shift table (device), or null.  Stored values are then
    // relative to S_i(Y) = f_eq_i(1, (u_s(Y), 0)) of the row that consumes them instead of to
    // w_i.  Layout, all float, Y = 0..ly+1: u_s[Y]; base[Y][9] = S_i(Y); rebase[Y][9] =
    // S_i(Y) - S_i(Y + c_iy) (0 where c_iy = 0 or Y + c_iy is outside 0..ly+1); rows[Y] = 1 where
    // some rebase[Y][i] is not zero, else 0 (a profile constant over bands of rows needs the
    // rebase only on the rows at a band's edge).
    const float *shift_u;
    // 16-bit storage only: stochastic rounding keys (codec.cuh) of the launch's collision and,
    // for the two-step sweep, of the second one; 0 rounds to nearest.
    unsigned rs_key, rs_key2;
    __host__ __device__ __forceinline__ const float *shift_base(int Y) const { return shift_u + (ly + 2) + 9 * Y; }
    __host__ __device__ __forceinline__ const float *shift_rebase(int Y) const
    {
        return shift_u + 10 * (ly + 2) + 9 * Y;
    }
    __host__ __device__ __forceinline__ bool shift_rebased(int Y) const { return shift_u[19 * (ly + 2) + Y] != 0.0f; }

    __host__ __device__ __forceinline__ long long idx(int X, int Y) const
    {
        return (long long)Y * pitch + (long long)(X + xoff - 1);
    }
    __host__ __device__ __forceinline__ bool interior(int X, int Y) const
    {
        return X >= 1 && X <= lx && Y >= 1 && Y <= ly;
    }
    __host__ __device__ __forceinline__ bool perimeter(int X, int Y) const
    {
        return X == 1 || X == lx || Y == 1 || Y == ly;
    }
    __host__ __device__ __forceinline__ int pidx(int X, int Y) const
    {
        if (Y == 1) return X - 1;
        if (Y == ly) return lx + X - 1;
        if (X == 1) return 2 * lx + Y - 2;
        return 2 * lx + ly + Y - 2;
    }
    // Ghost-ring numbering: row Y=0, row Y=ly+1 (X = 0..lx+1), then columns X=0 and
    // X=lx+1 for Y = 1..ly; nghost() entries.
    __host__ __device__ __forceinline__ int nghost() const { return 2 * (lx + 2) + 2 * ly; }
    __host__ __device__ __forceinline__ int gidx(int X, int Y) const
    {
        if (Y == 0) return X;
        if (Y == ly + 1) return lx + 2 + X;
        if (X == 0) return 2 * (lx + 2) + Y - 1;
        return 2 * (lx + 2) + ly + Y - 1;
    }
};

// Build the geometry of an lx x ly lattice whose elements are `elem_bytes` wide.
inline Geo make_geo(int lx, int ly, int elem_bytes)
{
    Geo g;
    const int align = 128 / elem_bytes;  // elements per 128-byte line
    g.lx = lx;
    g.ly = ly;
    g.xoff = align;
    g.pitch = ((long long)(align + lx + 1) + align - 1) / align * align;
    g.plane = (long long)(ly + 2) * g.pitch;
    g.nb = (lx > ly ? lx : ly) + 2;
    g.nper = 2 * lx + 2 * ly;
    g.shift_u = nullptr;
    g.rs_key = 0;
    g.rs_key2 = 0;
    return g;
}

}  // namespace lbgpu
