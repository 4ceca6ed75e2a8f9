// geom.cuh — device layout of every field of the solver context.
//
// All 3-D fields share ONE padded box so that a kernel computes one linear index per cell
// and reaches every field with it.  The box covers the widest halo the reference declares
// (u(0:nx+2, 0:ny+1, 0:nz+1), v(.., 0:ny+2, ..), w(.., .., 0:nz+2); 0_modules.f90:92-94):
//     i in [0, nx+2], j in [0, ny+2], k in [0, nz+2]
//     idx(i,j,k) = BASE + (i-1) + px*j + pxy*k,   px = round_up(nx+3, 16), pxy = px*(ny+3)
// so that the first interior element i = 1 of every row is 128-byte aligned (BASE = 16
// elements, px a multiple of 16) and the i = 0 ghost sits in the previous row's padding.
// Cell fields (1..nx) and face fields (1..nx+1) use the same box; their ghosts are unused.
// WENO ghosts beyond the halo (-2..0, n+1..n+3) are never stored: they are computed on the
// fly from interior values, exactly as weno1 builds them (14_level_set.f90:530-570).
#pragma once
#include <cstdint>

namespace suli {

constexpr int kBase = 16;

struct Geo {
    int nx, ny, nz;
    int px;          // row pitch (elements)
    int py;          // rows per plane = ny + 3
    long long pxy;   // plane pitch = px * py
    long long n;     // allocation length (elements)

    __host__ __device__ inline long long idx(int i, int j, int k) const {
        return (long long)kBase + (i - 1) + (long long)px * j + pxy * k;
    }
    // the same index in 32-bit arithmetic (a field holds fewer than 2^31 elements; suli_create
    // refuses larger grids)
    __host__ __device__ inline int idx32(int i, int j, int k) const {
        return kBase + (i - 1) + px * j + (int)pxy * k;
    }
};

inline Geo make_geo(int nx, int ny, int nz) {
    Geo g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.px = ((nx + 3 + 15) / 16) * 16;
    g.py = ny + 3;
    g.pxy = (long long)g.px * g.py;
    long long last = (long long)kBase + g.pxy * (nz + 3);
    g.n = ((last + 63) / 64) * 64;
    return g;
}

// Boundary conditions resolved for device code.
struct BC {
    int x0, xf, y0, yf, z0, zf;   // ccx0..cczf
    int perx, pery, perz;         // periodic flags as the reference tests them
    int wrapf;                    // suli_params.periodic_faces: end faces of a periodic axis averaged across the wrap
};

// Neighbour index maps of the Poisson operator's ghost copies (9_grad.f90:99-116):
// periodic -> wrap, otherwise Neumann copy of the adjacent interior value.
__host__ __device__ inline int map_lo(int i, int n, int per) { return (i < 1) ? (per ? n : 1) : i; }
__host__ __device__ inline int map_hi(int i, int n, int per) { return (i > n) ? (per ? 1 : n) : i; }
__host__ __device__ inline int map_any(int i, int n, int per) {
    return (i < 1) ? (per ? n : 1) : ((i > n) ? (per ? 1 : n) : i);
}

// Neighbour offsets of cell (i,j,k) in a box; a Neumann face maps to the cell itself.
struct Nb {
    int xm, xp, ym, yp, zm, zp;
};
__host__ __device__ inline Nb neighbours(const Geo& G, const BC& bc, int i, int j, int k) {
    Nb o;
    const int px = G.px, pxy = (int)G.pxy;
    o.xm = (i > 1) ? -1 : (bc.perx ? G.nx - 1 : 0);
    o.xp = (i < G.nx) ? 1 : (bc.perx ? -(G.nx - 1) : 0);
    o.ym = (j > 1) ? -px : (bc.pery ? (G.ny - 1) * px : 0);
    o.yp = (j < G.ny) ? px : (bc.pery ? -(G.ny - 1) * px : 0);
    o.zm = (k > 1) ? -pxy : (bc.perz ? (G.nz - 1) * pxy : 0);
    o.zp = (k < G.nz) ? pxy : (bc.perz ? -(G.nz - 1) * pxy : 0);
    return o;
}

}  // namespace suli
