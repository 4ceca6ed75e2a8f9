// obstacle.cuh — bottom obstacles (obst_t != 0): the column operations of contorno.
//
// The masks of obstaculo (3_contorno.f90:494-762) give, for each column, the k up to which
// the velocity components are zeroed: ku(0:nx+2, 0:ny+1), kv(0:nx+1, 0:ny+2),
// kw(0:nx+1, 0:ny+1), Fortran order.  suli_set_obstacle keeps ku, kv in [-1, nz] and kw in
// [-1, nz+1], so every k touched below (0 .. mask + 1) lies inside the halo of geom.cuh.
#pragma once
#include "geom.cuh"

namespace suli {

struct ObstMasks {
    const int *ku, *kv, *kw;
};

// contorno(1/2), 3_contorno.f90:266-294, for column (i, j), 0 <= i <= nx+2, 0 <= j <= ny+2:
// zero u, v, w from k = 0 up to the column's mask, then capture the first value above it into
// ub, vb, wb for the wall friction of convdiff; u's column i = nx+2 and v's row j = ny+2 are
// only zeroed.  Columns are independent: each reads and writes only its own (i, j).
__host__ __device__ inline void obst_columns(const Geo& G, const ObstMasks& M, double* u, double* v, double* w,
                                             double* ub, double* vb, double* wb, int i, int j) {
    const int nx = G.nx, ny = G.ny, lu = nx + 3, lv = nx + 2;
    if (i <= nx + 1 && j <= ny + 1) {
        const int a = M.ku[i + lu * j], b = M.kv[i + lv * j], d = M.kw[i + lv * j];
        for (int k = 0; k <= a; ++k) u[G.idx32(i, j, k)] = 0.;
        for (int k = 0; k <= b; ++k) v[G.idx32(i, j, k)] = 0.;
        for (int k = 0; k <= d; ++k) w[G.idx32(i, j, k)] = 0.;
        ub[G.idx32(i, j, a + 1)] = u[G.idx32(i, j, a + 1)];
        vb[G.idx32(i, j, b + 1)] = v[G.idx32(i, j, b + 1)];
        wb[G.idx32(i, j, d + 1)] = w[G.idx32(i, j, d + 1)];
    }
    if (i == nx + 2 && j <= ny + 1) {
        const int a = M.ku[i + lu * j];
        for (int k = 0; k <= a; ++k) u[G.idx32(i, j, k)] = 0.;
    }
    if (j == ny + 2 && i <= nx + 1) {
        const int b = M.kv[i + lv * j];
        for (int k = 0; k <= b; ++k) v[G.idx32(i, j, k)] = 0.;
    }
}

// contorno(3), 3_contorno.f90:445-481: the level set at cell (i, j, k) inside the obstacle
// (1 <= k <= kw(i,j) - 1) from the fluid neighbours at the same height, or from the cell
// above at the obstacle's top.  Writes *out and returns true when the reference assigns the
// cell.  A neighbour outside 1..nx, 1..ny is never read (the reference reads ls outside its
// bounds there): its fluid test is false.  Every cell read is outside all obstacle columns at
// that height, or above the own column's top, so no cell read is rewritten: the cells can be
// updated in place in any order.
__host__ __device__ inline bool obst_ls_value(const Geo& G, const int* kw, const double* ls, int i, int j, int k,
                                              double* out) {
    const int nx = G.nx, ny = G.ny, nz = G.nz, lw = nx + 2;
    auto K = [&](int ii, int jj) { return kw[ii + lw * jj]; };
    auto fluid = [&](int ii, int jj) { return ii >= 1 && ii <= nx && jj >= 1 && jj <= ny && K(ii, jj) < k; };
    auto solid = [&](int ii, int jj) { return K(ii, jj) >= k; };
    auto L = [&](int ii, int jj, int kk) { return ls[G.idx32(ii, jj, kk)]; };
    if (fluid(i - 1, j) && fluid(i, j - 1)) { *out = (L(i - 1, j, k) + L(i, j - 1, k)) * 0.5; return true; }
    if (fluid(i + 1, j) && fluid(i, j - 1)) { *out = (L(i + 1, j, k) + L(i, j - 1, k)) * 0.5; return true; }
    if (fluid(i + 1, j) && fluid(i, j + 1)) { *out = (L(i + 1, j, k) + L(i, j + 1, k)) * 0.5; return true; }
    if (fluid(i - 1, j) && fluid(i, j + 1)) { *out = (L(i - 1, j, k) + L(i, j + 1, k)) * 0.5; return true; }
    if (fluid(i - 1, j) && solid(i, j - 1) && solid(i, j + 1)) { *out = L(i - 1, j, k); return true; }
    if (fluid(i, j - 1) && solid(i - 1, j) && solid(i + 1, j)) { *out = L(i, j - 1, k); return true; }
    if (fluid(i + 1, j) && solid(i, j - 1) && solid(i, j + 1)) { *out = L(i + 1, j, k); return true; }
    if (fluid(i, j + 1) && solid(i - 1, j) && solid(i + 1, j)) { *out = L(i, j + 1, k); return true; }
    if (k == K(i, j) - 1 && k < nz) { *out = L(i, j, k + 1); return true; }
    return false;
}

}  // namespace suli
