// k_fp64.cu — FP64 kernels of the SuLi-IC hot path for sm_100a.
//
// Every expression keeps the reference's order of operations except that divisions by a
// constant or a shared divisor are done as one reciprocal and multiplications (cell sizes,
// WENO weights, normals, the Jacobi-scaled coefficients), and FMA contraction is on: FP64
// division and sqrt are multi-instruction sequences that bound these stencils, not memory.
// Results differ from a literal CPU evaluation by rounding only (a few ulp per value); the
// parity tests bound the difference per field.  Reductions are
// deterministic: fixed warp-shuffle trees per block and a fixed-order sum of the block
// partials done by the last block to finish (no floating-point atomics).
#include <cuda_runtime.h>
#include <cmath>
#include "advect.cuh"
#include "ctx.cuh"
#include "obstacle.cuh"
#include "pdl.cuh"
#include "reduce.cuh"
#include "weno.cuh"

namespace suli {

#define FIDX(a, i, j, k) (a)[G.idx32((i), (j), (k))]

// ------------------------------------------------------------------------------------
// small helpers of 8_derivadas.f90
// ------------------------------------------------------------------------------------
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
// Fortran MAX(x,0.) / MIN(x,0.)
template <typename R>
__device__ __forceinline__ R pmax(R a, R b) { return a > b ? a : b; }
template <typename R>
__device__ __forceinline__ R pmin(R a, R b) { return a < b ? a : b; }
// read a stored FP64 value in the compute type R of the kernel
#define RLD(a, i, j, k) R(FIDX((a), (i), (j), (k)))

struct Thread3 {
    int i, j, k;
};
__device__ __forceinline__ Thread3 tid3(int i0, int j0, int k0) {
    Thread3 t;
    t.i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
    t.j = j0 + blockIdx.y * blockDim.y + threadIdx.y;
    t.k = k0 + blockIdx.z * blockDim.z + threadIdx.z;
    return t;
}
static inline dim3 grid3(int ni, int nj, int nk, dim3 b) {
    return dim3((ni + b.x - 1) / b.x, (nj + b.y - 1) / b.y, (nk + b.z - 1) / b.z);
}
static const dim3 kBlk(32, 8, 1);

template <typename R>
struct Weno3 {
    R dpx, dnx, dpy, dny, dpz, dnz;
};
// der_weno at one cell (14_level_set.f90:343-384) of a cell field f, in compute type R.
// rx, ry, rz: 1/dx, 1/dy, 1/dz in R
template <typename R>
__device__ __forceinline__ Weno3<R> der_weno_at(const Geo& G, const double* __restrict__ f, int i, int j, int k,
                                                int ihx, int ihy, int ihz, R rx, R ry, R rz) {
    Weno3<R> W;
    R P[7];
    pencil7<R>([&](int q) { return R(FIDX(f, q, j, k)); }, i, G.nx, ihx, P);
    weno_pair<R>(P, rx, W.dpx, W.dnx);
    pencil7<R>([&](int q) { return R(FIDX(f, i, q, k)); }, j, G.ny, ihy, P);
    weno_pair<R>(P, ry, W.dpy, W.dny);
    pencil7<R>([&](int q) { return R(FIDX(f, i, j, q)); }, k, G.nz, ihz, P);
    weno_pair<R>(P, rz, W.dpz, W.dnz);
    return W;
}
template <typename R>
__device__ __forceinline__ R larger(R a, R b) { return (fabs(a) > fabs(b)) ? a : b; }
// a / b in the compute type: IEEE in FP64; in the mixed path's FP32 arithmetic the hardware
// reciprocal (__fdividef, 2 ulp), since an IEEE FP32 division costs as much as the rest of a
// stencil term (every divisor here is a density, a norm or a sum of squares, far below 2^126)
template <typename R>
__device__ __forceinline__ R rdiv(R a, R b) {
    if constexpr (sizeof(R) == 8) return a / b;
    else return __fdividef(a, b);
}

struct LsConst {
    int ihx, ihy, ihz, ihn;
    double dx, dy, dz, dx1;
    double ad;          // alpha1*dx1
    double pi;
    double rho1, rho2, mi1, mi2;
    int t_hs;           // 0 linear mix of rho and mu in H, 1 geometric (14_level_set.f90:696-703)
    double mu1s, mu2s;  // mi_f1 * 10000, mi_f2 * 10000
    double rx, ry, rz;  // 1/dx, 1/dy, 1/dz (the WENO divided differences)
    float frx, fry, frz;   // the same reciprocals formed in FP32 (1.f / float(dx)), for R = float
    template <typename R>
    __device__ __forceinline__ R rcp(int d) const {
        if constexpr (sizeof(R) == 8) return R(d == 0 ? rx : (d == 1 ? ry : rz));
        else return R(d == 0 ? frx : (d == 1 ? fry : frz));
    }
};

// ------------------------------------------------------------------------------------
// level set: mod_ls1 part A + heaviside + volume (14_level_set.f90:612-722, 743-759)
// ------------------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_lsprops(Geo G, LsConst L, const double* __restrict__ ls,
                                                 double* mod_ls, double* nrmx, double* nrmy, double* nrmz,
                                                 double* hs, double* hsx, double* hsy, double* hsz, double* rho,
                                                 double* ls_nu, int do_mod, int do_hs, int do_vol,
                                                 double* partial, unsigned int* counter, double* out) {
    const Thread3 t = tid3(1, 1, 1);
    const bool in = (t.i <= G.nx && t.j <= G.ny && t.k <= G.nz);
    double vol = 0.0;
    if (in) {
        const long long c = G.idx(t.i, t.j, t.k);
        const Weno3<R> W = der_weno_at<R>(G, ls, t.i, t.j, t.k, L.ihx, L.ihy, L.ihz, L.rcp<R>(0), L.rcp<R>(1), L.rcp<R>(2));
        const R ar = larger(W.dpx, W.dnx), br = larger(W.dpy, W.dny), cr = larger(W.dpz, W.dnz);
        if (do_mod) {
            const R m = sqrt(ar * ar + br * br + cr * cr);
            mod_ls[c] = (double)m;
            if (m == R(0)) { nrmx[c] = 0.; nrmy[c] = 0.; nrmz[c] = 0.; }
            else { const R im = rdiv<R>(R(1), m); nrmx[c] = (double)(ar * im); nrmy[c] = (double)(br * im); nrmz[c] = (double)(cr * im); }
        }
        const double a = (double)ar, b = (double)br, cc = (double)cr;   // the Heaviside stays FP64
        if (do_hs) {
            const double l = ls[c];
            double h;
            if (l < -L.ad) {
                h = 0.; hsx[c] = 0.; hsy[c] = 0.; hsz[c] = 0.;
            } else if (l > L.ad) {
                h = 1.; hsx[c] = 0.; hsy[c] = 0.; hsz[c] = 0.;
            } else {
                h = 0.5 * (1. + l / L.ad + 1. / L.pi * sin(L.pi * l / L.ad));
                const double cs = cos(L.pi * l / L.ad);
                hsx[c] = 0.5 * a * (1. + cs) / L.ad;
                hsy[c] = 0.5 * b * (1. + cs) / L.ad;
                hsz[c] = 0.5 * cc * (1. + cs) / L.ad;
            }
            hs[c] = h;
            if (L.t_hs == 0) {
                rho[c] = L.rho1 * (1. - h) + L.rho2 * h;
                ls_nu[c] = L.mi1 * (1. - h) + L.mi2 * h;
            } else {
                rho[c] = pow(L.rho1, 1. - h) + pow(L.rho2, h) - 1.;
                ls_nu[c] = (pow(L.mu1s, 1. - h) + pow(L.mu2s, h) - 1.) / 10000.;
            }
            if (do_vol) vol = (1. - (1. - h)) * L.dx * L.dy * L.dz;
        }
    }
    if (do_vol) {
        double ta, tb;
        if (reduce2_last(vol, 0.0, partial, counter, ta, tb) && flat_tid() == 0) out[0] = ta;
    }
}

// mod_ls1 part B: curvature from the WENO derivatives of the normal (14_level_set.f90:761-803)
template <typename R>
__global__ void __launch_bounds__(256) k_curv(Geo G, LsConst L, const double* __restrict__ nx_,
                                              const double* __restrict__ ny_, const double* __restrict__ nz_,
                                              double* ddx, double* ddy, double* ddz, double* kurv) {
    const Thread3 t = tid3(1, 1, 1);
    if (t.i > G.nx || t.j > G.ny || t.k > G.nz) return;
    R P[7], dp, dn;
    pencil7<R>([&](int q) { return R(FIDX(nx_, q, t.j, t.k)); }, t.i, G.nx, L.ihn, P);
    weno_pair<R>(P, L.rcp<R>(0), dp, dn);
    const R ax = (fabs(dn) > fabs(dp)) ? dn : dp;
    pencil7<R>([&](int q) { return R(FIDX(ny_, t.i, q, t.k)); }, t.j, G.ny, L.ihn, P);
    weno_pair<R>(P, L.rcp<R>(1), dp, dn);
    const R ay = (fabs(dn) > fabs(dp)) ? dn : dp;
    pencil7<R>([&](int q) { return R(FIDX(nz_, t.i, t.j, q)); }, t.k, G.nz, L.ihn, P);
    weno_pair<R>(P, L.rcp<R>(2), dp, dn);
    const R az = (fabs(dn) > fabs(dp)) ? dn : dp;
    const long long c = G.idx(t.i, t.j, t.k);
    ddx[c] = (double)ax; ddy[c] = (double)ay; ddz[c] = (double)az;
    kurv[c] = (double)(ax + ay + az);
}

// conv_weno + intt_ls: one TVD-RK3 stage of level-set transport (14_level_set.f90:287-341)
template <typename R>
__global__ void __launch_bounds__(256) k_ls_advect(Geo G, LsConst L, const double* __restrict__ cur,
                                                   const double* phi0, double* out,
                                                   const double* __restrict__ u, const double* __restrict__ v,
                                                   const double* __restrict__ w, double a, double b, double gd) {
    const Thread3 t = tid3(1, 1, 1);
    if (t.i > G.nx || t.j > G.ny || t.k > G.nz) return;
    const int i = t.i, j = t.j, k = t.k;
    const Weno3<R> W = der_weno_at<R>(G, cur, i, j, k, L.ihx, L.ihy, L.ihz, L.rcp<R>(0), L.rcp<R>(1), L.rcp<R>(2));
    const R ua = (RLD(u, i, j, k) + RLD(u, i + 1, j, k)) * R(0.5);
    const R va = (RLD(v, i, j, k) + RLD(v, i, j + 1, k)) * R(0.5);
    const R wa = (RLD(w, i, j, k) + RLD(w, i, j, k + 1)) * R(0.5);
    const R apos = pmax(ua, R(0)), aneg = pmin(ua, R(0));
    const R bpos = pmax(va, R(0)), bneg = pmin(va, R(0));
    const R cpos = pmax(wa, R(0)), cneg = pmin(wa, R(0));
    const R sy7 = -(apos * W.dnx + aneg * W.dpx + bpos * W.dny + bneg * W.dpy + cpos * W.dnz + cneg * W.dpz);
    const long long c = G.idx(i, j, k);
    const double p0 = phi0[c];
    const double gxv = cur[c];
    out[c] = a * p0 + b * gxv + gd * (double)sy7;   // the stage combination in FP64
}

// reinic_weno selection (14_level_set.f90:406-431)
template <typename R>
__device__ __forceinline__ R reinit_mod(R l, const Weno3<R>& W) {
    const R cst = R(0.00000001);
    R a, b, c;
    if (l > R(0)) {
        a = pmax(pmax(W.dnx, cst), -pmin(W.dpx, cst));
        b = pmax(pmax(W.dny, cst), -pmin(W.dpy, cst));
        c = pmax(pmax(W.dnz, cst), -pmin(W.dpz, cst));
    } else {
        a = pmax(pmax(W.dpx, cst), -pmin(W.dnx, cst));
        b = pmax(pmax(W.dpy, cst), -pmin(W.dny, cst));
        c = pmax(pmax(W.dpz, cst), -pmin(W.dnz, cst));
    }
    return sqrt(a * a + b * b + c * c);
}

template <typename R>
__global__ void __launch_bounds__(256) k_reinit_funcs(Geo G, LsConst L, const double* __restrict__ ls,
                                                      double* funcs) {
    const Thread3 t = tid3(1, 1, 1);
    if (t.i > G.nx || t.j > G.ny || t.k > G.nz) return;
    const Weno3<R> W = der_weno_at<R>(G, ls, t.i, t.j, t.k, L.ihx, L.ihy, L.ihz, L.rcp<R>(0), L.rcp<R>(1), L.rcp<R>(2));
    const long long c = G.idx(t.i, t.j, t.k);
    const R l = R(ls[c]);
    const R m = reinit_mod(l, W);
    const R dx1 = R(L.dx1);
    funcs[c] = (double)rdiv<R>(l, sqrt(l * l + m * m * dx1 * dx1));
}

template <typename R>
__global__ void __launch_bounds__(256) k_reinit_stage(Geo G, LsConst L, const double* __restrict__ cur,
                                                      const double* phi0, double* out,
                                                      const double* __restrict__ funcs, double a, double b,
                                                      double gd) {
    const Thread3 t = tid3(1, 1, 1);
    if (t.i > G.nx || t.j > G.ny || t.k > G.nz) return;
    const Weno3<R> W = der_weno_at<R>(G, cur, t.i, t.j, t.k, L.ihx, L.ihy, L.ihz, L.rcp<R>(0), L.rcp<R>(1), L.rcp<R>(2));
    const long long c = G.idx(t.i, t.j, t.k);
    const double l = cur[c];
    const R m = reinit_mod(R(l), W);
    const R sy7 = R(funcs[c]) * (R(1) - m);
    const double p0 = phi0[c];
    out[c] = a * p0 + b * l + gd * (double)sy7;   // the stage combination in FP64
}

// signed band error of the reinitialisation (14_level_set.f90:492-503): sum and count
__global__ void __launch_bounds__(256) k_reinit_err(Geo G, const double* __restrict__ after,
                                                    const double* __restrict__ before, double band,
                                                    double* partial, unsigned int* counter, double* out) {
    const Thread3 t = tid3(1, 1, 1);
    double s = 0.0, n = 0.0;
    if (t.i <= G.nx && t.j <= G.ny && t.k <= G.nz) {
        const long long c = G.idx(t.i, t.j, t.k);
        const double l = after[c];
        if (fabs(l) <= band) { s = l - before[c]; n = 1.0; }
    }
    double ta, tb;
    if (reduce2_last(s, n, partial, counter, ta, tb) && flat_tid() == 0) { out[0] = ta; out[1] = tb; }
}

// ls = ls + ls_m over the cells (14_level_set.f90:196-202)
__global__ void k_ls_shift(Geo G, double* ls, double shift) {
    const Thread3 t = tid3(1, 1, 1);
    if (t.i > G.nx || t.j > G.ny || t.k > G.nz) return;
    const long long c = G.idx(t.i, t.j, t.k);
    ls[c] = ls[c] + shift;
}

// volume correction step (14_level_set.f90:259-265)
__global__ void k_volfix(Geo G, double* ls, const double* __restrict__ mod_ls, double dt1fac, double vol_ini) {
    const Thread3 t = tid3(1, 1, 1);
    if (t.i > G.nx || t.j > G.ny || t.k > G.nz) return;
    const long long c = G.idx(t.i, t.j, t.k);
    ls[c] = ls[c] - dt1fac * mod_ls[c] / vol_ini;
}

// ------------------------------------------------------------------------------------
// visco (5_viscosidade.f90:12-219), m_turb 0 / 1 (m_turb 2: k_facenu_dir below)
// ------------------------------------------------------------------------------------
struct ViscConst {
    double dx, dy, dz, cdel, csmag;   // cdel = (dx*dy*dz)**(2/3) computed on the host
};
// A thread owns KZ cells of a column (i, j, k0 .. k0 + KZ - 1); the loads of the unrolled loop
// share their addresses between neighbouring cells (a plane's values serve the cell below and
// the one above), so a cell costs about 21 distinct loads instead of 36 and all are issued
// together.  KZ > 1 is used only when nz is a multiple of KZ.
template <typename R, int KZ>
__global__ void __launch_bounds__(256) k_nut(Geo G, ViscConst V, const double* __restrict__ u,
                                             const double* __restrict__ v, const double* __restrict__ w,
                                             const double* __restrict__ rho, double* __restrict__ nut) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k0 = blockIdx.z * KZ + 1;
    if (i > G.nx || j > G.ny || k0 > G.nz) return;
    const int px = G.px, pxy = (int)G.pxy;
    int cp[KZ + 3];   // index of (i, j, k0 - 1 + q)
#pragma unroll
    for (int q = 0; q < KZ + 3; ++q) cp[q] = G.idx32(i, j, k0 - 1) + q * pxy;
    const R itdx = R(1. / (2. * V.dx)), itdy = R(1. / (2. * V.dy)), itdz = R(1. / (2. * V.dz));
#pragma unroll
    for (int m = 0; m < KZ; ++m) {
// a field value at (i + di, j + dj, k + dk) of cell k = k0 + m
#define AT(a, di, dj, dk) R((a)[cp[m + 1 + (dk)] + (di) + (dj) * px])
        // derivax/y/z of the staggered fields, then interp?_fc to the cell centre
        const R dudx = ((AT(u, 1, 0, 0) - AT(u, -1, 0, 0)) * itdx + (AT(u, 2, 0, 0) - AT(u, 0, 0, 0)) * itdx) * R(0.5);
        const R dudy = ((AT(u, 0, 1, 0) - AT(u, 0, -1, 0)) * itdy + (AT(u, 1, 1, 0) - AT(u, 1, -1, 0)) * itdy) * R(0.5);
        const R dudz = ((AT(u, 0, 0, 1) - AT(u, 0, 0, -1)) * itdz + (AT(u, 1, 0, 1) - AT(u, 1, 0, -1)) * itdz) * R(0.5);
        const R dvdx = ((AT(v, 1, 0, 0) - AT(v, -1, 0, 0)) * itdx + (AT(v, 1, 1, 0) - AT(v, -1, 1, 0)) * itdx) * R(0.5);
        const R dvdy = ((AT(v, 0, 1, 0) - AT(v, 0, -1, 0)) * itdy + (AT(v, 0, 2, 0) - AT(v, 0, 0, 0)) * itdy) * R(0.5);
        const R dvdz = ((AT(v, 0, 0, 1) - AT(v, 0, 0, -1)) * itdz + (AT(v, 0, 1, 1) - AT(v, 0, 1, -1)) * itdz) * R(0.5);
        const R dwdx = ((AT(w, 1, 0, 0) - AT(w, -1, 0, 0)) * itdx + (AT(w, 1, 0, 1) - AT(w, -1, 0, 1)) * itdx) * R(0.5);
        const R dwdy = ((AT(w, 0, 1, 0) - AT(w, 0, -1, 0)) * itdy + (AT(w, 0, 1, 1) - AT(w, 0, -1, 1)) * itdy) * R(0.5);
        const R dwdz = ((AT(w, 0, 0, 1) - AT(w, 0, 0, -1)) * itdz + (AT(w, 0, 0, 2) - AT(w, 0, 0, 0)) * itdz) * R(0.5);
#undef AT
        const R p1 = dudx + R(0.5) * (dudy + dvdx + dudz + dwdx);
        const R p2 = dvdy + R(0.5) * (dvdx + dudy + dvdz + dwdy);
        const R p3 = dwdz + R(0.5) * (dwdy + dvdz + dudz + dwdx);
        const int c = cp[m + 1];
        nut[c] = (double)(R(V.cdel * V.csmag * V.csmag) * sqrt(R(2.) * (p1 + p2 + p3) * (p1 + p2 + p3)) * R(rho[c]));
    }
}

// xnut/ynut/znut = face(ls_nu) + face(nut) with the end-face copy of interp?_cf
__global__ void __launch_bounds__(256) k_facenu(Geo G, int m_turb, const double* __restrict__ ls_nu,
                                                const double* __restrict__ nut, double* xnut, double* ynut,
                                                double* znut) {
    const Thread3 t = tid3(1, 1, 1);
    const int i = t.i, j = t.j, k = t.k, nx = G.nx, ny = G.ny, nz = G.nz;
    if (i > nx + 1 || j > ny + 1 || k > nz + 1) return;
    if (j <= ny && k <= nz) {
        const int ic = clampi(i, 2, nx);
        const double lx = (FIDX(ls_nu, ic, j, k) + FIDX(ls_nu, ic - 1, j, k)) * 0.5;
        const double xa = m_turb ? (FIDX(nut, ic, j, k) + FIDX(nut, ic - 1, j, k)) * 0.5 : 0.;
        FIDX(xnut, i, j, k) = lx + xa;
    }
    if (i <= nx && k <= nz) {
        const int jc = clampi(j, 2, ny);
        const double ly = (FIDX(ls_nu, i, jc, k) + FIDX(ls_nu, i, jc - 1, k)) * 0.5;
        const double ya = m_turb ? (FIDX(nut, i, jc, k) + FIDX(nut, i, jc - 1, k)) * 0.5 : 0.;
        FIDX(ynut, i, j, k) = ly + ya;
    }
    if (i <= nx && j <= ny) {
        const int kc = clampi(k, 2, nz);
        const double lz = (FIDX(ls_nu, i, j, kc) + FIDX(ls_nu, i, j, kc - 1)) * 0.5;
        const double za = m_turb ? (FIDX(nut, i, j, kc) + FIDX(nut, i, j, kc - 1)) * 0.5 : 0.;
        FIDX(znut, i, j, k) = lz + za;
    }
}

// m_turb = 2, directional Smagorinsky (5_viscosidade.f90:58-61, 104-164): each face's eddy
// viscosity from the strain of its own velocity component, without the density factor:
//   xnut_a = dx*dx*Cs*Cs*sqrt(2 p1 p1),  p1 = du/dx + (du/dy + dv/dx + du/dz + dw/dx)/2,
// with dv/dx, dw/dx averaged face -> edge (interpx_cf, end copy) -> u-face (interpy_fc /
// interpz_fc), and likewise for ynut_a, znut_a.  nut is not written.  Then
// xnut = face(ls_nu) + xnut_a as in k_facenu.
struct ViscDirConst {
    double itdx, itdy, itdz;   // 1/(2 dx), 1/(2 dy), 1/(2 dz)
    double cx, cy, cz;         // dx*dx*Cs*Cs, dy*dy*Cs*Cs, dz*dz*Cs*Cs in the reference's order
};
template <typename R>
__global__ void __launch_bounds__(256) k_facenu_dir(Geo G, ViscDirConst V, const double* __restrict__ u,
                                                    const double* __restrict__ v, const double* __restrict__ w,
                                                    const double* __restrict__ ls_nu, double* xnut, double* ynut,
                                                    double* znut) {
    const Thread3 t = tid3(1, 1, 1);
    const int i = t.i, j = t.j, k = t.k, nx = G.nx, ny = G.ny, nz = G.nz;
    if (i > nx + 1 || j > ny + 1 || k > nz + 1) return;
    const int px = G.px, pxy = (int)G.pxy, c0 = G.idx32(i, j, k);
    const R itdx = R(V.itdx), itdy = R(V.itdy), itdz = R(V.itdz);
#define AT(a, di, dj, dk) R((a)[c0 + (di) + (dj) * px + (dk) * pxy])
    // centred derivatives (derivax/y/z, 8_derivadas.f90:1-68) at an offset from this face
#define DX(a, di, dj, dk) ((AT(a, (di) + 1, dj, dk) - AT(a, (di) - 1, dj, dk)) * itdx)
#define DY(a, di, dj, dk) ((AT(a, di, (dj) + 1, dk) - AT(a, di, (dj) - 1, dk)) * itdy)
#define DZ(a, di, dj, dk) ((AT(a, di, dj, (dk) + 1) - AT(a, di, dj, (dk) - 1)) * itdz)
    if (j <= ny && k <= nz) {   // u-faces i = 1..nx+1
        const int ic = clampi(i, 2, nx), o1 = ic - i, o0 = ic - 1 - i;
        const R dvdx_x = ((DX(v, o1, 0, 0) + DX(v, o0, 0, 0)) * R(0.5) + (DX(v, o1, 1, 0) + DX(v, o0, 1, 0)) * R(0.5)) * R(0.5);
        const R dwdx_x = ((DX(w, o1, 0, 0) + DX(w, o0, 0, 0)) * R(0.5) + (DX(w, o1, 0, 1) + DX(w, o0, 0, 1)) * R(0.5)) * R(0.5);
        const R p1 = DX(u, 0, 0, 0) + R(0.5) * (DY(u, 0, 0, 0) + dvdx_x + DZ(u, 0, 0, 0) + dwdx_x);
        const R xa = R(V.cx) * sqrt(R(2.) * p1 * p1);
        const double lx = (ls_nu[c0 + o1] + ls_nu[c0 + o0]) * 0.5;
        xnut[c0] = lx + (double)xa;
    }
    if (i <= nx && k <= nz) {   // v-faces j = 1..ny+1
        const int jc = clampi(j, 2, ny), q1 = jc - j, q0 = jc - 1 - j;
        const R dudy_y = ((DY(u, 0, q1, 0) + DY(u, 0, q0, 0)) * R(0.5) + (DY(u, 1, q1, 0) + DY(u, 1, q0, 0)) * R(0.5)) * R(0.5);
        const R dwdy_y = ((DY(w, 0, q1, 0) + DY(w, 0, q0, 0)) * R(0.5) + (DY(w, 0, q1, 1) + DY(w, 0, q0, 1)) * R(0.5)) * R(0.5);
        const R p1 = DY(v, 0, 0, 0) + R(0.5) * (DX(v, 0, 0, 0) + dudy_y + DZ(v, 0, 0, 0) + dwdy_y);
        const R ya = R(V.cy) * sqrt(R(2.) * p1 * p1);
        const double ly = (ls_nu[c0 + q1 * px] + ls_nu[c0 + q0 * px]) * 0.5;
        ynut[c0] = ly + (double)ya;
    }
    if (i <= nx && j <= ny) {   // w-faces k = 1..nz+1
        const int kc = clampi(k, 2, nz), r1 = kc - k, r0 = kc - 1 - k;
        const R dvdz_z = ((DZ(v, 0, 0, r1) + DZ(v, 0, 0, r0)) * R(0.5) + (DZ(v, 0, 1, r1) + DZ(v, 0, 1, r0)) * R(0.5)) * R(0.5);
        const R dudz_z = ((DZ(u, 0, 0, r1) + DZ(u, 0, 0, r0)) * R(0.5) + (DZ(u, 1, 0, r1) + DZ(u, 1, 0, r0)) * R(0.5)) * R(0.5);
        const R p1 = DZ(w, 0, 0, 0) + R(0.5) * (DY(w, 0, 0, 0) + dvdz_z + dudz_z + DX(w, 0, 0, 0));
        const R za = R(V.cz) * sqrt(R(2.) * p1 * p1);
        const double lz = (ls_nu[c0 + r1 * pxy] + ls_nu[c0 + r0 * pxy]) * 0.5;
        znut[c0] = lz + (double)za;
    }
#undef DZ
#undef DY
#undef DX
#undef AT
}

// ------------------------------------------------------------------------------------
// convdiff + classico (6_convdiff.f90:14-189, 7_advectivo.f90:3-290)
// ------------------------------------------------------------------------------------
struct CDConst {
    double idx, idy, idz, gx, gz, sigma, cz;   // reciprocal cell sizes; cz = gz/(chezy*chezy)
    int tf;                                  // tf_u/v/w are non-zero
    int cap_z2, cap_y2, cap_yn;              // planes where ub/vb/wb are captured (3_contorno.f90:247-264)
    int obst;                                // obstacles: captured above each column, friction read everywhere
};
struct CDFields {
    const double *u, *v, *w, *rho, *hsx, *hsy, *hsz, *kurv, *nut, *xnut, *ynut, *znut, *ub, *vb, *wb;
    const double *tfu, *tfv, *tfw;
    double *Fu, *Fv, *Fw;
};

// the reference subtracts (gz/C^2)|ub| u at every face (6_convdiff.f90:156,168,183); ub is zero
// except where contorno captured it, so only those faces are read
__device__ __forceinline__ bool on_cap(const CDConst& C, int j, int k, int ny) {
    return C.obst || (C.cap_z2 && k == 2) || (C.cap_y2 && j == 2) || (C.cap_yn && j == ny);
}

// classico der = 2 (centred, 7_advectivo.f90:115-170) and der = 3 (second-order upwind,
// :174-285) for one velocity component a at its face c: along direction d (element stride
// s[d]) the face sits at m[d] of the component's n[d] points, vel[d] is the advecting
// velocity, ih[d] = 1/h.  Terms summed in direction order, as the reference does.
template <typename R, int DER>
__device__ __forceinline__ R classico_hi(const double* __restrict__ a, int c, const int s[3], const int m[3],
                                         const int n[3], const R vel[3], const R ih[3]) {
    R acc = R(0.);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const R ap = R(a[c + s[d]]), am = R(a[c - s[d]]);
        R term;
        if constexpr (DER == 2) {
            term = vel[d] * ((ap - am) * (R(0.5) * ih[d]));   // derivax/y/z (8_derivadas.f90:1-68)
        } else {
            const R a0 = R(a[c]);
            // the points two away, where the one-sided formulas use them (else this face):
            // every load stays inside the component's halo
            const R amm = R(a[c - (m[d] > 1 ? 2 * s[d] : 0)]);
            const R app = R(a[c + (m[d] < n[d] ? 2 * s[d] : 0)]);
            // derivax/y/zu2n (:194-290): backward one-sided, centred on the first point
            const R dn = m[d] > 1 ? R(0.5) * (amm - R(4.) * am + R(3.) * a0) * ih[d]
                                  : R(0.5) * (ap - am) * ih[d];
            // derivax/y/zu2p (:83-179): forward one-sided, centred on the last point
            const R dp = m[d] < n[d] ? R(0.5) * (-app + R(4.) * ap - R(3.) * a0) * ih[d]
                                     : R(0.5) * (ap - am) * ih[d];
            term = pmax(vel[d], R(0.)) * dn + pmin(vel[d], R(0.)) * dp;
        }
        acc = d == 0 ? term : acc + term;
    }
    return acc;
}

// DER: classico's scheme (adv_type = 1); ADV: 2 rotacional, 3 antissim (advect.cuh; der = 1)
template <typename R, int DER, int ADV>
__global__ void __launch_bounds__(256) k_convdiff(Geo G, CDConst C, CDFields F) {
    const Thread3 t = tid3(1, 1, 1);
    const int i = t.i, j = t.j, k = t.k, nx = G.nx, ny = G.ny, nz = G.nz;
    if (i > nx + 1 || j > ny + 1 || k > nz + 1) return;
    const R idx = R(C.idx), idy = R(C.idy), idz = R(C.idz);   // 1/dx, 1/dy, 1/dz
    // every load is the face's own index plus a constant offset (32-bit): a field value at
    // (i + di, j + dj, k + dk), read in the compute type R
    const int px = G.px, pxy = (int)G.pxy, c0 = (int)G.idx(i, j, k);
#define AT(a, di, dj, dk) R((a)[c0 + (di) + (dj) * px + (dk) * pxy])
    const double* __restrict__ u = F.u;
    const double* __restrict__ v = F.v;
    const double* __restrict__ w = F.w;
    // ---- Fu on u-faces (i = 1..nx+1, j = 1..ny, k = 1..nz)
    if (j <= ny && k <= nz) {
        const R uc = AT(u, 0, 0, 0);
        const int ic = clampi(i, 2, nx);
        R uint_;
        if constexpr (ADV != 1) {
            uint_ = split_form_u<R, ADV>(FaceTaps<R>{c0, px, pxy}, u, v, w, i, j, k, nx, idx, idy, idz);
        } else if constexpr (DER == 1) {
            const R bma4 = (AT(v, 0, 0, 0) + AT(v, -1, 0, 0) + AT(v, 0, 1, 0) + AT(v, -1, 1, 0)) * R(0.25);
            const R dma4 = (AT(w, 0, 0, 0) + AT(w, -1, 0, 0) + AT(w, 0, 0, 1) + AT(w, -1, 0, 1)) * R(0.25);
            R a1 = pmax(uc, R(0.)), a2 = pmin(uc, R(0.));
            const R dudx = a1 * (uc - AT(u, -1, 0, 0)) * idx + a2 * (AT(u, 1, 0, 0) - uc) * idx;
            a1 = pmax(bma4, R(0.)); a2 = pmin(bma4, R(0.));
            const R dudy = a1 * (uc - AT(u, 0, -1, 0)) * idy + a2 * (AT(u, 0, 1, 0) - uc) * idy;
            a1 = pmax(dma4, R(0.)); a2 = pmin(dma4, R(0.));
            const R dudz = a1 * (uc - AT(u, 0, 0, -1)) * idz + a2 * (AT(u, 0, 0, 1) - uc) * idz;
            uint_ = dudx + dudy + dudz;
        } else {
            // transverse velocities face -> centre (interp?_fc) -> u-face (interpx_cf, end copy)
            const int o1 = ic - i, o0 = ic - 1 - i;
            const R bma = ((AT(v, o1, 0, 0) + AT(v, o1, 1, 0)) * R(0.5) + (AT(v, o0, 0, 0) + AT(v, o0, 1, 0)) * R(0.5)) * R(0.5);
            const R dma = ((AT(w, o1, 0, 0) + AT(w, o1, 0, 1)) * R(0.5) + (AT(w, o0, 0, 0) + AT(w, o0, 0, 1)) * R(0.5)) * R(0.5);
            const int s[3] = {1, px, pxy}, m[3] = {i, j, k}, n[3] = {nx + 1, ny, nz};
            const R vel[3] = {uc, bma, dma}, ih[3] = {idx, idy, idz};
            uint_ = classico_hi<R, DER>(u, c0, s, m, n, vel, ih);
        }
        const R rhox = (AT(F.rho, (ic) - i, 0, 0) + AT(F.rho, (ic - 1) - i, 0, 0)) * R(0.5);
        const R tx1 = rdiv<R>(AT(F.hsx, (ic) - i, 0, 0) * AT(F.kurv, (ic) - i, 0, 0), AT(F.rho, (ic) - i, 0, 0));
        const R tx0 = rdiv<R>(AT(F.hsx, (ic - 1) - i, 0, 0) * AT(F.kurv, (ic - 1) - i, 0, 0), AT(F.rho, (ic - 1) - i, 0, 0));
        const R dhsdx = (tx1 + tx0) * R(0.5);
        const R ama_i = AT(F.nut, (clampi(i, 1, nx)) - i, 0, 0) * idx;
        const R ama_m = AT(F.nut, (clampi(i - 1, 1, nx)) - i, 0, 0) * idx;
        const int jp = clampi(j + 1, 2, ny), jm = clampi(j, 2, ny);
        const R bma_p = ((AT(F.xnut, 0, (jp) - j, 0) + AT(F.xnut, 0, (jp - 1) - j, 0)) * R(0.5)) * idy;
        const R bma_m = ((AT(F.xnut, 0, (jm) - j, 0) + AT(F.xnut, 0, (jm - 1) - j, 0)) * R(0.5)) * idy;
        const int kp = clampi(k + 1, 2, nz), km = clampi(k, 2, nz);
        const R dma_p = ((AT(F.xnut, 0, 0, (kp) - k) + AT(F.xnut, 0, 0, (kp - 1) - k)) * R(0.5)) * idz;
        const R dma_m = ((AT(F.xnut, 0, 0, (km) - k) + AT(F.xnut, 0, 0, (km - 1) - k)) * R(0.5)) * idz;
        const R Gv = (ama_i * R(2.) * (AT(u, 1, 0, 0) - uc) - ama_m * R(2.) * (uc - AT(u, -1, 0, 0))) * idx +
                          bma_p * ((AT(u, 0, 1, 0) - uc) * idy + (AT(v, 0, 1, 0) - AT(v, -1, 1, 0)) * idx) -
                          bma_m * ((uc - AT(u, 0, -1, 0)) * idy + (AT(v, 0, 0, 0) - AT(v, -1, 0, 0)) * idx) +
                          dma_p * ((AT(u, 0, 0, 1) - uc) * idz + (AT(w, 0, 0, 1) - AT(w, -1, 0, 1)) * idx) -
                          dma_m * ((uc - AT(u, 0, 0, -1)) * idz + (AT(w, 0, 0, 0) - AT(w, -1, 0, 0)) * idx);
        R r = -uint_ + rdiv<R>(Gv, rhox) + R(C.gx) - R(C.sigma) * dhsdx;
        if (C.tf) r = r + AT(F.tfu, 0, 0, 0);
        if (on_cap(C, j, k, ny)) { const R b = AT(F.ub, 0, 0, 0); r = r - R(C.cz) * sqrt(b * b) * uc; }
        F.Fu[c0] = (double)r;
    }
    // ---- Fv on v-faces (i = 1..nx, j = 1..ny+1, k = 1..nz)
    if (i <= nx && k <= nz) {
        const R vc = AT(v, 0, 0, 0);
        const int jc = clampi(j, 2, ny);
        R vint;
        if constexpr (ADV != 1) {
            vint = split_form_v<R, ADV>(FaceTaps<R>{c0, px, pxy}, u, v, w, i, j, k, ny, idx, idy, idz);
        } else if constexpr (DER == 1) {
            const R amb4 = (AT(u, 0, 0, 0) + AT(u, 1, 0, 0) + AT(u, 0, -1, 0) + AT(u, 1, -1, 0)) * R(0.25);
            const R dmb4 = (AT(w, 0, 0, 0) + AT(w, 0, -1, 0) + AT(w, 0, 0, 1) + AT(w, 0, -1, 1)) * R(0.25);
            R a1 = pmax(amb4, R(0.)), a2 = pmin(amb4, R(0.));
            const R dvdx = a1 * (vc - AT(v, -1, 0, 0)) * idx + a2 * (AT(v, 1, 0, 0) - vc) * idx;
            a1 = pmax(vc, R(0.)); a2 = pmin(vc, R(0.));
            const R dvdy = a1 * (vc - AT(v, 0, -1, 0)) * idy + a2 * (AT(v, 0, 1, 0) - vc) * idy;
            a1 = pmax(dmb4, R(0.)); a2 = pmin(dmb4, R(0.));
            const R dvdz = a1 * (vc - AT(v, 0, 0, -1)) * idz + a2 * (AT(v, 0, 0, 1) - vc) * idz;
            vint = dvdx + dvdy + dvdz;
        } else {
            const int q1 = jc - j, q0 = jc - 1 - j;
            const R amb = ((AT(u, 0, q1, 0) + AT(u, 1, q1, 0)) * R(0.5) + (AT(u, 0, q0, 0) + AT(u, 1, q0, 0)) * R(0.5)) * R(0.5);
            const R dmb = ((AT(w, 0, q1, 0) + AT(w, 0, q1, 1)) * R(0.5) + (AT(w, 0, q0, 0) + AT(w, 0, q0, 1)) * R(0.5)) * R(0.5);
            const int s[3] = {1, px, pxy}, m[3] = {i, j, k}, n[3] = {nx, ny + 1, nz};
            const R vel[3] = {amb, vc, dmb}, ih[3] = {idx, idy, idz};
            vint = classico_hi<R, DER>(v, c0, s, m, n, vel, ih);
        }
        const R rhoy = (AT(F.rho, 0, (jc) - j, 0) + AT(F.rho, 0, (jc - 1) - j, 0)) * R(0.5);
        const R ty1 = rdiv<R>(AT(F.hsy, 0, (jc) - j, 0) * AT(F.kurv, 0, (jc) - j, 0), AT(F.rho, 0, (jc) - j, 0));
        const R ty0 = rdiv<R>(AT(F.hsy, 0, (jc - 1) - j, 0) * AT(F.kurv, 0, (jc - 1) - j, 0), AT(F.rho, 0, (jc - 1) - j, 0));
        const R dhsdy = (ty1 + ty0) * R(0.5);
        const int ip = clampi(i + 1, 2, nx), im = clampi(i, 2, nx);
        const R amb_p = ((AT(F.ynut, (ip) - i, 0, 0) + AT(F.ynut, (ip - 1) - i, 0, 0)) * R(0.5)) * idx;
        const R amb_m = ((AT(F.ynut, (im) - i, 0, 0) + AT(F.ynut, (im - 1) - i, 0, 0)) * R(0.5)) * idx;
        const R bmb_j = AT(F.nut, 0, (clampi(j, 1, ny)) - j, 0) * idy;
        const R bmb_m = AT(F.nut, 0, (clampi(j - 1, 1, ny)) - j, 0) * idy;
        const int kp = clampi(k + 1, 2, nz), km = clampi(k, 2, nz);
        const R dmb_p = ((AT(F.ynut, 0, 0, (kp) - k) + AT(F.ynut, 0, 0, (kp - 1) - k)) * R(0.5)) * idz;
        const R dmb_m = ((AT(F.ynut, 0, 0, (km) - k) + AT(F.ynut, 0, 0, (km - 1) - k)) * R(0.5)) * idz;
        const R Gv = amb_p * ((AT(v, 1, 0, 0) - vc) * idx + (AT(u, 1, 0, 0) - AT(u, 1, -1, 0)) * idy) -
                          amb_m * ((vc - AT(v, -1, 0, 0)) * idx + (AT(u, 0, 0, 0) - AT(u, 0, -1, 0)) * idy) +
                          (bmb_j * R(2.) * (AT(v, 0, 1, 0) - vc) - bmb_m * R(2.) * (vc - AT(v, 0, -1, 0))) * idy +
                          dmb_p * ((AT(v, 0, 0, 1) - vc) * idz + (AT(w, 0, 0, 1) - AT(w, 0, -1, 1)) * idy) -
                          dmb_m * ((vc - AT(v, 0, 0, -1)) * idz + (AT(w, 0, 0, 0) - AT(w, 0, -1, 0)) * idy);
        R r = -vint + rdiv<R>(Gv, rhoy) - R(C.sigma) * dhsdy;
        if (C.tf) r = r + AT(F.tfv, 0, 0, 0);
        if (on_cap(C, j, k, ny)) { const R b = AT(F.vb, 0, 0, 0); r = r - R(C.cz) * sqrt(b * b) * vc; }
        F.Fv[c0] = (double)r;
    }
    // ---- Fw on w-faces (i = 1..nx, j = 1..ny, k = 1..nz+1)
    if (i <= nx && j <= ny) {
        const R wc = AT(w, 0, 0, 0);
        const int kc = clampi(k, 2, nz);
        R wint;
        if constexpr (ADV != 1) {
            wint = split_form_w<R, ADV>(FaceTaps<R>{c0, px, pxy}, u, v, w, i, j, k, nz, idx, idy, idz);
        } else if constexpr (DER == 1) {
            const R amd4 = (AT(u, 0, 0, 0) + AT(u, 1, 0, 0) + AT(u, 0, 0, -1) + AT(u, 1, 0, -1)) * R(0.25);
            const R bmd4 = (AT(v, 0, 0, 0) + AT(v, 0, 1, 0) + AT(v, 0, 0, -1) + AT(v, 0, 1, -1)) * R(0.25);
            R a1 = pmax(amd4, R(0.)), a2 = pmin(amd4, R(0.));
            const R dwdx = a1 * (wc - AT(w, -1, 0, 0)) * idx + a2 * (AT(w, 1, 0, 0) - wc) * idx;
            a1 = pmax(bmd4, R(0.)); a2 = pmin(bmd4, R(0.));
            const R dwdy = a1 * (wc - AT(w, 0, -1, 0)) * idy + a2 * (AT(w, 0, 1, 0) - wc) * idy;
            a1 = pmax(wc, R(0.)); a2 = pmin(wc, R(0.));
            const R dwdz = a1 * (wc - AT(w, 0, 0, -1)) * idz + a2 * (AT(w, 0, 0, 1) - wc) * idz;
            wint = dwdx + dwdy + dwdz;
        } else {
            const int r1 = kc - k, r0 = kc - 1 - k;
            const R amd = ((AT(u, 0, 0, r1) + AT(u, 1, 0, r1)) * R(0.5) + (AT(u, 0, 0, r0) + AT(u, 1, 0, r0)) * R(0.5)) * R(0.5);
            const R bmd = ((AT(v, 0, 0, r1) + AT(v, 0, 1, r1)) * R(0.5) + (AT(v, 0, 0, r0) + AT(v, 0, 1, r0)) * R(0.5)) * R(0.5);
            const int s[3] = {1, px, pxy}, m[3] = {i, j, k}, n[3] = {nx, ny, nz + 1};
            const R vel[3] = {amd, bmd, wc}, ih[3] = {idx, idy, idz};
            wint = classico_hi<R, DER>(w, c0, s, m, n, vel, ih);
        }
        const R rhoz = (AT(F.rho, 0, 0, (kc) - k) + AT(F.rho, 0, 0, (kc - 1) - k)) * R(0.5);
        const R tz1 = rdiv<R>(AT(F.hsz, 0, 0, (kc) - k) * AT(F.kurv, 0, 0, (kc) - k), AT(F.rho, 0, 0, (kc) - k));
        const R tz0 = rdiv<R>(AT(F.hsz, 0, 0, (kc - 1) - k) * AT(F.kurv, 0, 0, (kc - 1) - k), AT(F.rho, 0, 0, (kc - 1) - k));
        const R dhsdz = (tz1 + tz0) * R(0.5);
        const int ip = clampi(i + 1, 2, nx), im = clampi(i, 2, nx);
        const R amd_p = ((AT(F.znut, (ip) - i, 0, 0) + AT(F.znut, (ip - 1) - i, 0, 0)) * R(0.5)) * idx;
        const R amd_m = ((AT(F.znut, (im) - i, 0, 0) + AT(F.znut, (im - 1) - i, 0, 0)) * R(0.5)) * idx;
        const int jp = clampi(j + 1, 2, ny), jm = clampi(j, 2, ny);
        const R bmd_p = ((AT(F.znut, 0, (jp) - j, 0) + AT(F.znut, 0, (jp - 1) - j, 0)) * R(0.5)) * idy;
        const R bmd_m = ((AT(F.znut, 0, (jm) - j, 0) + AT(F.znut, 0, (jm - 1) - j, 0)) * R(0.5)) * idy;
        const R dmd_k = AT(F.nut, 0, 0, (clampi(k, 1, nz)) - k) * idz;
        const R dmd_m = AT(F.nut, 0, 0, (clampi(k - 1, 1, nz)) - k) * idz;
        const R Gv = amd_p * ((AT(w, 1, 0, 0) - wc) * idx + (AT(u, 1, 0, 0) - AT(u, 1, 0, -1)) * idz) -
                          amd_m * ((wc - AT(w, -1, 0, 0)) * idx + (AT(u, 0, 0, 0) - AT(u, 0, 0, -1)) * idz) +
                          bmd_p * ((AT(w, 0, 1, 0) - wc) * idy + (AT(v, 0, 1, 0) - AT(v, 0, 1, -1)) * idz) -
                          bmd_m * ((wc - AT(w, 0, -1, 0)) * idy + (AT(v, 0, 0, 0) - AT(v, 0, 0, -1)) * idz) +
                          (dmd_k * R(2.) * (AT(w, 0, 0, 1) - wc) - dmd_m * R(2.) * (wc - AT(w, 0, 0, -1))) * idz;
        R r = -wint + rdiv<R>(Gv, rhoz) - R(C.gz) - R(C.sigma) * dhsdz;
        if (C.tf) r = r + AT(F.tfw, 0, 0, 0);
        if (on_cap(C, j, k, ny)) { const R b = AT(F.wb, 0, 0, 0); r = r - R(C.cz) * sqrt(b * b) * wc; }
        F.Fw[c0] = (double)r;
    }
#undef AT
}

// ------------------------------------------------------------------------------------
// tempo (11_diversos.f90:10-230)
// ------------------------------------------------------------------------------------
struct TempoArgs {
    double* a[3]; const double* F[3]; double* a0[3]; double* f0[3]; double* f1[3];
    int tm, tt, it;
    double dt;
};
__global__ void __launch_bounds__(256) k_tempo(Geo G, TempoArgs T) {
    const Thread3 t = tid3(1, 1, 1);
    const int i = t.i, j = t.j, k = t.k;
    if (i > G.nx + 1 || j > G.ny + 1 || k > G.nz + 1) return;
    const bool valid[3] = {j <= G.ny && k <= G.nz, i <= G.nx && k <= G.nz, i <= G.nx && j <= G.ny};
    const long long c = G.idx(i, j, k);
    const double dt = T.dt;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        if (!valid[m]) continue;
        double* A = T.a[m];
        const double Fv = T.F[m][c];
        if (T.tm == 0 || (T.tm == 3 && T.it == 1)) {
            A[c] = A[c] + dt * Fv;
            if (T.tm == 3) T.f0[m][c] = Fv;
        } else if (T.tm == 1) {
            if (T.tt == 1) { const double aux1 = dt; T.a0[m][c] = A[c]; A[c] = A[c] + aux1 * Fv; }
            else if (T.tt == 2) { const double aux1 = dt; A[c] = T.a0[m][c] + aux1 * Fv; }
        } else if (T.tm == 2) {
            if (T.tt == 1) {
                const double aux1 = dt;
                T.a0[m][c] = A[c]; T.f0[m][c] = Fv; A[c] = A[c] + aux1 * Fv;
            } else if (T.tt == 2) {
                const double aux1 = 2. * dt;
                T.f1[m][c] = Fv; A[c] = T.a0[m][c] - dt * T.f0[m][c] + aux1 * Fv;
            } else if (T.tt == 3) {
                const double aux1 = dt / 6.;
                A[c] = T.a0[m][c] + aux1 * (T.f0[m][c] + 4. * T.f1[m][c] + Fv);
            }
        } else if (T.tm == 3) {
            A[c] = A[c] + dt * 0.5 * (3 * Fv - T.f0[m][c]);
            T.f0[m][c] = Fv;
        }
    }
}

// ------------------------------------------------------------------------------------
// contorno (3_contorno.f90:10-492), phases in the reference's order.  prd_corr returns
// zeros (:899-919), so its "+ dpd?" terms vanish.  ccz0 = cczf = 0 is the periodic-z
// extension mirroring the periodic-x rows.
// ------------------------------------------------------------------------------------
struct BCArgs {
    double *u, *v, *w, *ub, *vb, *wb, *prd1;
    Planes pl;
    int nlock;
    int obst;   // obstacle columns replace the wall-friction capture of the walls
};
// pressure ghosts: composition of the x, y, z copies (:37-54) = value at the mapped index.  One
// thread per ghost cell of the halo surface: the two x layers (all j, k), the two y layers
// (interior i, all k), the two z layers (interior i, j); reads touch only interior cells.
__global__ void k_prd_ghosts(Geo G, BC bc, double* prd1) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const long long nxf = 2LL * (ny + 2) * (nz + 2), nyf = 2LL * nx * (nz + 2), nzf = 2LL * nx * ny;
    int i, j, k;
    if (q < nxf) {
        const long long r = q >> 1;
        i = (q & 1) ? nx + 1 : 0; j = (int)(r % (ny + 2)); k = (int)(r / (ny + 2));
    } else if (q < nxf + nyf) {
        const long long r = (q - nxf) >> 1;
        j = ((q - nxf) & 1) ? ny + 1 : 0; i = 1 + (int)(r % nx); k = (int)(r / nx);
    } else if (q < nxf + nyf + nzf) {
        const long long r = (q - nxf - nyf) >> 1;
        k = ((q - nxf - nyf) & 1) ? nz + 1 : 0; i = 1 + (int)(r % nx); j = 1 + (int)(r / nx);
    } else {
        return;
    }
    const int mi = map_any(i, nx, bc.perx), mj = map_any(j, ny, bc.pery), mk = map_any(k, nz, bc.perz);
    FIDX(prd1, i, j, k) = FIDX(prd1, mi, mj, mk);
}

// y walls (:58-114), thread per (i,k)
__global__ void k_bc_y(Geo G, BC bc, BCArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = G.nx, ny = G.ny, nz = G.nz, ny1 = ny + 1;
    const bool per = (bc.y0 == 0 && bc.yf == 0);
    const int lu = nx + 3, lv = nx + 2;   // leading dims of byx*, byy*/byz* planes
    // u: i in 0..nx+2, k in 0..nz+1
    if (i <= nx + 2 && k <= nz + 1) {
        double* u = A.u;
        if (per) FIDX(u, i, 0, k) = FIDX(u, i, ny, k);
        if (bc.y0 == 1) FIDX(u, i, 0, k) = FIDX(u, i, 1, k);
        if (bc.y0 == 2) FIDX(u, i, 0, k) = -FIDX(u, i, 1, k);
        if (bc.y0 == 3) FIDX(u, i, 0, k) = A.pl.byx0[i + lu * k];
        if (per) FIDX(u, i, ny + 1, k) = FIDX(u, i, 1, k);
        if (bc.yf == 1) FIDX(u, i, ny + 1, k) = FIDX(u, i, ny, k);
        if (bc.yf == 2) FIDX(u, i, ny + 1, k) = -FIDX(u, i, ny, k);
        if (bc.yf == 3) FIDX(u, i, ny + 1, k) = A.pl.byxf[i + lu * k];
    }
    // v: i in 0..nx+1, k in 0..nz+1
    if (i <= nx + 1 && k <= nz + 1) {
        double* v = A.v;
        if (per) { FIDX(v, i, 0, k) = FIDX(v, i, ny1 - 1, k); FIDX(v, i, 1, k) = FIDX(v, i, ny1, k); }
        if (bc.y0 == 1) FIDX(v, i, 0, k) = -FIDX(v, i, 2, k);
        if (bc.y0 == 2) FIDX(v, i, 0, k) = FIDX(v, i, 2, k);
        if (bc.y0 == 3) FIDX(v, i, 0, k) = A.pl.byy0[i + lv * k];
        if (per) FIDX(v, i, ny1 + 1, k) = FIDX(v, i, 2, k);
        if (bc.yf == 1) FIDX(v, i, ny1 + 1, k) = -FIDX(v, i, ny1 - 1, k);
        if (bc.yf == 2) FIDX(v, i, ny1 + 1, k) = FIDX(v, i, ny1 - 1, k);
        if (bc.yf == 3) FIDX(v, i, ny1 + 1, k) = A.pl.byyf1[i + lv * k];
    }
    // w: i in 0..nx+1, k in 0..nz+2
    if (i <= nx + 1 && k <= nz + 2) {
        double* w = A.w;
        if (per) FIDX(w, i, 0, k) = FIDX(w, i, ny, k);
        if (bc.y0 == 1) FIDX(w, i, 0, k) = FIDX(w, i, 1, k);
        if (bc.y0 == 2) FIDX(w, i, 0, k) = -FIDX(w, i, 1, k);
        if (bc.y0 == 3) FIDX(w, i, 0, k) = A.pl.byz0[i + lv * k];
        if (per) FIDX(w, i, ny + 1, k) = FIDX(w, i, 1, k);
        if (bc.yf == 1) FIDX(w, i, ny + 1, k) = FIDX(w, i, ny, k);
        if (bc.yf == 2) FIDX(w, i, ny + 1, k) = -FIDX(w, i, ny, k);
        if (bc.yf == 3) FIDX(w, i, ny + 1, k) = A.pl.byzf[i + lv * k];
    }
}

// x walls (:116-197), thread per (j,k)
__global__ void k_bc_x(Geo G, BC bc, BCArgs A) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = G.nx, ny = G.ny, nz = G.nz, nx1 = nx + 1;
    const bool per = (bc.x0 == 0 && bc.xf == 0);
    const int ly = ny + 2, lyv = ny + 3;   // leading dims of bxx*/bxz* and bxy* planes
    if (j <= ny + 1 && k <= nz + 1) {   // u
        double* u = A.u;
        if (per) FIDX(u, 0, j, k) = FIDX(u, nx1 - 1, j, k);
        if (bc.x0 == 1) FIDX(u, 0, j, k) = -FIDX(u, 2, j, k);
        if (bc.x0 == 2) FIDX(u, 0, j, k) = FIDX(u, 2, j, k);
        if (bc.x0 == 3) FIDX(u, 0, j, k) = A.pl.bxx0[j + ly * k];
        if (per) FIDX(u, nx1 + 1, j, k) = FIDX(u, 2, j, k);
        if (bc.xf == 1) FIDX(u, nx1 + 1, j, k) = -FIDX(u, nx1 - 1, j, k);
        if (bc.xf == 2) FIDX(u, nx1 + 1, j, k) = FIDX(u, nx1 - 1, j, k);
        if (bc.xf == 3) FIDX(u, nx1 + 1, j, k) = A.pl.bxxf1[j + ly * k];
        if (bc.xf == 4) FIDX(u, nx1 + 1, j, k) = FIDX(u, nx1, j, k);
    }
    if (j <= ny + 2 && k <= nz + 1) {   // v
        double* v = A.v;
        if (per) FIDX(v, 0, j, k) = FIDX(v, nx, j, k);
        if (bc.x0 == 1) FIDX(v, 0, j, k) = FIDX(v, 1, j, k);
        if (bc.x0 == 2) FIDX(v, 0, j, k) = -FIDX(v, 1, j, k);
        if (bc.x0 == 3 || bc.x0 == 4) FIDX(v, 0, j, k) = A.pl.bxy0[j + lyv * k];
        if (per) FIDX(v, nx + 1, j, k) = FIDX(v, 1, j, k);
        if (bc.xf == 1) FIDX(v, nx + 1, j, k) = FIDX(v, nx, j, k);
        if (bc.xf == 2) FIDX(v, nx + 1, j, k) = -FIDX(v, nx, j, k);
        if (bc.xf == 3) FIDX(v, nx + 1, j, k) = A.pl.bxyf[j + lyv * k];
        if (bc.xf == 4) FIDX(v, nx + 1, j, k) = FIDX(v, nx, j, k);
    }
    if (j <= ny + 1 && k <= nz + 2) {   // w
        double* w = A.w;
        if (per) FIDX(w, 0, j, k) = FIDX(w, nx, j, k);
        if (bc.x0 == 1) FIDX(w, 0, j, k) = FIDX(w, 1, j, k);
        if (bc.x0 == 2) FIDX(w, 0, j, k) = -FIDX(w, 1, j, k);
        if (bc.x0 == 3) FIDX(w, 0, j, k) = A.pl.bxz0[j + ly * k];
        if (bc.x0 == 4) FIDX(w, 0, j, k) = FIDX(w, 1, j, k);
        if (per) FIDX(w, nx + 1, j, k) = FIDX(w, 1, j, k);
        if (bc.xf == 1) FIDX(w, nx + 1, j, k) = FIDX(w, nx, j, k);
        if (bc.xf == 2) FIDX(w, nx + 1, j, k) = -FIDX(w, nx, j, k);
        if (bc.xf == 3) FIDX(w, nx + 1, j, k) = A.pl.bxzf[j + ly * k];
        if (bc.xf == 4) FIDX(w, nx + 1, j, k) = FIDX(w, nx, j, k);
    }
}

// z walls (:199-241) and the wall-friction capture (:247-264), thread per (i,j)
__global__ void k_bc_z(Geo G, BC bc, BCArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = G.nx, ny = G.ny, nz = G.nz, nz1 = nz + 1;
    const bool per = (bc.z0 == 0 && bc.zf == 0);
    const int lu = nx + 3, lv = nx + 2;
    if (i <= nx + 2 && j <= ny + 1) {   // u
        double* u = A.u;
        if (per) FIDX(u, i, j, 0) = FIDX(u, i, j, nz);
        if (bc.z0 == 1) FIDX(u, i, j, 0) = FIDX(u, i, j, 1);
        if (bc.z0 == 2) FIDX(u, i, j, 0) = -FIDX(u, i, j, 1);
        if (bc.z0 == 3) FIDX(u, i, j, 0) = A.pl.bzx0[i + lu * j];
        if (per) FIDX(u, i, j, nz + 1) = FIDX(u, i, j, 1);
        if (bc.zf == 1) FIDX(u, i, j, nz + 1) = FIDX(u, i, j, nz);
        if (bc.zf == 2) FIDX(u, i, j, nz + 1) = -FIDX(u, i, j, nz);
        if (bc.zf == 3) FIDX(u, i, j, nz + 1) = A.pl.bzxf[i + lu * j];
    }
    if (i <= nx + 1 && j <= ny + 2) {   // v
        double* v = A.v;
        if (per) FIDX(v, i, j, 0) = FIDX(v, i, j, nz);
        if (bc.z0 == 1) FIDX(v, i, j, 0) = FIDX(v, i, j, 1);
        if (bc.z0 == 2) FIDX(v, i, j, 0) = -FIDX(v, i, j, 1);
        if (bc.z0 == 3) FIDX(v, i, j, 0) = A.pl.bzy0[i + lv * j];
        if (per) FIDX(v, i, j, nz + 1) = FIDX(v, i, j, 1);
        if (bc.zf == 1) FIDX(v, i, j, nz + 1) = FIDX(v, i, j, nz);
        if (bc.zf == 2) FIDX(v, i, j, nz + 1) = -FIDX(v, i, j, nz);
        if (bc.zf == 3) FIDX(v, i, j, nz + 1) = A.pl.bzyf[i + lv * j];
    }
    if (i <= nx + 1 && j <= ny + 1) {   // w
        double* w = A.w;
        if (per) FIDX(w, i, j, 0) = FIDX(w, i, j, nz1 - 1);
        if (bc.z0 == 1) FIDX(w, i, j, 0) = -FIDX(w, i, j, 2);
        if (bc.z0 == 2) FIDX(w, i, j, 0) = FIDX(w, i, j, 2);
        if (bc.z0 == 3) FIDX(w, i, j, 0) = A.pl.bzz0[i + lv * j];
        if (per) FIDX(w, i, j, nz1 + 1) = FIDX(w, i, j, 2);
        if (bc.zf == 1) FIDX(w, i, j, nz1 + 1) = -FIDX(w, i, j, nz1 - 1);
        if (bc.zf == 2) FIDX(w, i, j, nz1 + 1) = FIDX(w, i, j, nz1 - 1);
        if (bc.zf == 3) FIDX(w, i, j, nz1 + 1) = A.pl.bzzf1[i + lv * j];
    }
    // capture of the k = 2 plane: each thread copies within its own (i,j) column, after its z writes
    if (bc.z0 == 2 && !A.obst) {
        if (i <= nx + 2 && j <= ny + 1) FIDX(A.ub, i, j, 2) = FIDX(A.u, i, j, 2);
        if (i <= nx + 1 && j <= ny + 2) FIDX(A.vb, i, j, 2) = FIDX(A.v, i, j, 2);
        if (i <= nx + 1 && j <= ny + 1) FIDX(A.wb, i, j, 2) = FIDX(A.w, i, j, 2);
    }
}

// capture of the j = 2 and j = ny planes (:254-264), after the z phase, thread per (i,k)
__global__ void k_bc_capture_y(Geo G, BC bc, BCArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    for (int side = 0; side < 2; ++side) {
        if (side == 0 && bc.y0 != 2) continue;
        if (side == 1 && bc.yf != 2) continue;
        const int j = (side == 0) ? 2 : ny;
        if (i <= nx + 2 && k <= nz + 1) FIDX(A.ub, i, j, k) = FIDX(A.u, i, j, k);
        if (i <= nx + 1 && k <= nz + 1) FIDX(A.vb, i, j, k) = FIDX(A.v, i, j, k);
        if (i <= nx + 1 && k <= nz + 2) FIDX(A.wb, i, j, k) = FIDX(A.w, i, j, k);
    }
}

// obstacle columns (:266-294) in place of the capture, thread per (i, j), 0..nx+2 x 0..ny+2
__global__ void k_bc_obst(Geo G, ObstMasks M, BCArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > G.nx + 2 || j > G.ny + 2) return;
    obst_columns(G, M, A.u, A.v, A.w, A.ub, A.vb, A.wb, i, j);
}

// contorno(3): level set inside the obstacle (:445-481), thread per column (i, j)
__global__ void k_ls_obst(Geo G, const int* __restrict__ kw, double* ls) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > G.nx || j > G.ny) return;
    const int top = kw[i + (G.nx + 2) * j] - 1;
    for (int k = 1; k <= top; ++k) {
        double val;
        if (obst_ls_value(G, kw, ls, i, j, k, &val)) ls[G.idx32(i, j, k)] = val;
    }
}

// boundary_waves (3_contorno.f90:952-1082).  The reference rounds the whole level set through
// a single-precision copy on every call (thread per cell), then writes the inflow planes and
// the level set of column i = 1 from the wave (thread per (j, k), 0..ny+1 x 0..nz+2; k = nz+2
// is the top row of bxz0, which the reference leaves unset: 0 here).
__global__ void k_ls_round_float(Geo G, double* ls) {
    const Thread3 t = tid3(1, 1, 1);
    if (t.i > G.nx || t.j > G.ny || t.k > G.nz) return;
    const int c = G.idx32(t.i, t.j, t.k);
    ls[c] = (double)(float)ls[c];
}
__global__ void k_waves(Geo G, WaveCoef W, double dx, double dz, double time, double* ls, double* bxx0, double* bxx1,
                        double* bxz0) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    const int ny = G.ny, nz = G.nz, row = ny + 2;
    if (j > ny + 1 || k > nz + 2) return;
    if (k == nz + 2) { bxz0[j + row * k] = 0.; return; }
    const WavePoint P0 = wave_point(W, 0, k, dx, dz, time), P1 = wave_point(W, 1, k, dx, dz, time);
    bxx0[j + row * k] = P0.u;
    bxz0[j + row * k] = P0.w;
    bxx1[j + row * k] = P1.u;
    if (j >= 1 && j <= ny && k >= 1 && k <= nz) ls[G.idx32(1, j, k)] = (double)P1.ls;
}

// nlock = 2: boundary-normal velocities, y then x then z (:297-441)
__global__ void k_bc_ny(Geo G, BC bc, BCArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = G.nx, ny = G.ny, nz = G.nz, ny1 = ny + 1, lv = nx + 2;
    if (i > nx + 1 || k > nz + 1) return;
    double* v = A.v;
    const bool per = (bc.y0 == 0 && bc.yf == 0);
    if (per) FIDX(v, i, 1, k) = FIDX(v, i, ny1, k);
    if (bc.y0 == 1 || bc.y0 == 2) FIDX(v, i, 1, k) = 0.;
    if (bc.y0 == 3) FIDX(v, i, 1, k) = A.pl.byy1[i + lv * k];
    if (per) FIDX(v, i, ny1, k) = FIDX(v, i, 1, k);
    if (bc.yf == 1 || bc.yf == 2) FIDX(v, i, ny1, k) = 0.;
    if (bc.yf == 3) FIDX(v, i, ny1, k) = A.pl.byyf[i + lv * k];
}
__global__ void k_bc_nx(Geo G, BC bc, BCArgs A) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = G.nx, ny = G.ny, nz = G.nz, nx1 = nx + 1, ly = ny + 2;
    const bool per = (bc.x0 == 0 && bc.xf == 0);
    if (j <= ny + 1 && k <= nz + 1) {
        double* u = A.u;
        if (per) FIDX(u, 1, j, k) = FIDX(u, nx1, j, k);
        if (bc.x0 == 1 || bc.x0 == 2) FIDX(u, 1, j, k) = 0.;
        if (bc.x0 == 3) FIDX(u, 1, j, k) = A.pl.bxx1[j + ly * k];
        if (per) FIDX(u, nx1, j, k) = FIDX(u, 1, j, k);
        if (bc.xf == 1) FIDX(u, nx1, j, k) = 0.;
        if (bc.xf == 2) { FIDX(u, nx1, j, k) = 0.; FIDX(u, nx1 + 1, j, k) = FIDX(u, nx1 - 1, j, k); }
        if (bc.xf == 3) FIDX(u, nx1, j, k) = A.pl.bxxf[j + ly * k];
        if (bc.xf == 4) FIDX(u, nx1, j, k) = FIDX(u, nx1 - 1, j, k);
    }
    if (bc.xf == 2) {
        if (j <= ny + 2 && k <= nz + 1) FIDX(A.v, nx + 1, j, k) = -FIDX(A.v, nx, j, k);
        if (j <= ny + 1 && k <= nz + 2) FIDX(A.w, nx + 1, j, k) = -FIDX(A.w, nx, j, k);
    }
}
__global__ void k_bc_nz(Geo G, BC bc, BCArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = G.nx, ny = G.ny, nz = G.nz, nz1 = nz + 1, lv = nx + 2;
    if (i > nx + 1 || j > ny + 1) return;
    double* w = A.w;
    const bool per = (bc.z0 == 0 && bc.zf == 0);
    if (per) FIDX(w, i, j, 1) = FIDX(w, i, j, nz1);
    if (bc.z0 == 1 || bc.z0 == 2) FIDX(w, i, j, 1) = 0.;
    if (bc.z0 == 3) FIDX(w, i, j, 1) = A.pl.bzz1[i + lv * j];
    if (per) FIDX(w, i, j, nz1) = FIDX(w, i, j, 1);
    if (bc.zf == 1 || bc.zf == 2) FIDX(w, i, j, nz1) = 0.;
    if (bc.zf == 3) FIDX(w, i, j, nz1) = A.pl.bzzf[i + lv * j];
}

// outflow_fix = 1 (an extension, after contorno(2) with ccxf = 4): one block sums the net
// volume flux through the boundary planes (the sum of graddin's right-hand side over the cells,
// telescoped), then shifts the outflow faces u(nx+1, j, k) above the obstacle mask ku(nx+1, j)
// by one uniform value so that the net flux vanishes.  Fixed-order tree sums (deterministic).
constexpr int kFixThreads = 1024;
__global__ void __launch_bounds__(kFixThreads) k_outflow_fix(Geo G, BCArgs A, const int* __restrict__ ku, double dx,
                                                            double dy, double dz) {
    __shared__ double s_delta;
    const int nx = G.nx, ny = G.ny, nz = G.nz, tid = threadIdx.x;
    double fx = 0., fy = 0., fz = 0., open = 0.;
    for (int q = tid; q < ny * nz; q += kFixThreads) {
        const int j = 1 + q % ny, k = 1 + q / ny;
        fx += FIDX(A.u, nx + 1, j, k) - FIDX(A.u, 1, j, k);
        open += (!ku || k > ku[(nx + 1) + (nx + 3) * j]) ? 1. : 0.;
    }
    for (int q = tid; q < nx * nz; q += kFixThreads) {
        const int i = 1 + q % nx, k = 1 + q / nx;
        fy += FIDX(A.v, i, ny + 1, k) - FIDX(A.v, i, 1, k);
    }
    for (int q = tid; q < nx * ny; q += kFixThreads) {
        const int i = 1 + q % nx, j = 1 + q / nx;
        fz += FIDX(A.w, i, j, nz + 1) - FIDX(A.w, i, j, 1);
    }
    fx = block_sum(fx);
    fy = block_sum(fy);
    fz = block_sum(fz);
    open = block_sum(open);
    if (tid == 0) {
        const double net = fx * (dy * dz) + fy * (dx * dz) + fz * (dx * dy);
        s_delta = (open > 0.) ? -net / (open * (dy * dz)) : 0.;
    }
    __syncthreads();
    const double delta = s_delta;
    for (int q = tid; q < ny * nz; q += kFixThreads) {
        const int j = 1 + q % ny, k = 1 + q / ny;
        if (!ku || k > ku[(nx + 1) + (nx + 3) * j]) FIDX(A.u, nx + 1, j, k) += delta;
    }
}

// ------------------------------------------------------------------------------------
// graddin (9_grad.f90:10-278)
// ------------------------------------------------------------------------------------
struct CGConst {
    double cx, cy, cz;     // dt/(dx*dx) ...
    double dx, dy, dz;
    double rdx, rdy, rdz;  // 1/dx, 1/dy, 1/dz
    double tol;            // cg_tol
    double div_tol;        // div_tol (0: off)
    double ncell;          // nx*ny*nz
    int mode, maxit;
};
// face density of graddin and posdin: the centre average with the reference's clamped end faces,
// or (periodic_faces = 1 on a periodic axis) the average across the wrap at both end faces
__device__ __forceinline__ double rho_face_x(const Geo& G, const BC& bc, const double* rho, int f, int j, int k) {
    if (bc.wrapf && bc.perx && (f == 1 || f == G.nx + 1)) return (FIDX(rho, 1, j, k) + FIDX(rho, G.nx, j, k)) * 0.5;
    const int fc = clampi(f, 2, G.nx);
    return (FIDX(rho, fc, j, k) + FIDX(rho, fc - 1, j, k)) * 0.5;
}
__device__ __forceinline__ double rho_face_y(const Geo& G, const BC& bc, const double* rho, int i, int f, int k) {
    if (bc.wrapf && bc.pery && (f == 1 || f == G.ny + 1)) return (FIDX(rho, i, 1, k) + FIDX(rho, i, G.ny, k)) * 0.5;
    const int fc = clampi(f, 2, G.ny);
    return (FIDX(rho, i, fc, k) + FIDX(rho, i, fc - 1, k)) * 0.5;
}
__device__ __forceinline__ double rho_face_z(const Geo& G, const BC& bc, const double* rho, int i, int j, int f) {
    if (bc.wrapf && bc.perz && (f == 1 || f == G.nz + 1)) return (FIDX(rho, i, j, 1) + FIDX(rho, i, j, G.nz)) * 0.5;
    const int fc = clampi(f, 2, G.nz);
    return (FIDX(rho, i, j, fc) + FIDX(rho, i, j, fc - 1)) * 0.5;
}

// Set-up of the scaled system in three passes, so that each face conductance is divided once:
// faces -> diagonal, e and b -> scaled coefficients and first residual.  The face values, their
// sums and the scaled coefficients are the same expressions, in the same order, as forming
// every face where it is used.

// minus-face conductances of every cell, the reference's c/((rho_a + rho_b)/2) with the clamped
// end faces (:46-87): sx(i) = face between i-1 and i (at i = 1 the face of i = 2)
__global__ void __launch_bounds__(256) k_cg_faces(Geo G, BC bc, CGConst K, const double* __restrict__ rho, double* sx,
                                                  double* sy, double* sz) {
    const Thread3 t = tid3(1, 1, 1);
    const int i = t.i, j = t.j, k = t.k;
    if (i > G.nx || j > G.ny || k > G.nz) return;
    const long long c = G.idx(i, j, k);
    sx[c] = K.cx / rho_face_x(G, bc, rho, i, j, k);
    sy[c] = K.cy / rho_face_y(G, bc, rho, i, j, k);
    sz[c] = K.cz / rho_face_z(G, bc, rho, i, j, k);
}

// the plus face of a cell: the next cell's minus face, or at the last cell the same clamped face
// (with periodic_faces on a periodic axis: the first cell's minus face, the same face of the box)
struct PlusFaces {
    double xp, yp, zp;
};
__device__ __forceinline__ PlusFaces plus_faces(const Geo& G, const BC& bc, int i, int j, int k, long long c,
                                                const double* sx, const double* sy, const double* sz) {
    const bool wx = bc.wrapf && bc.perx, wy = bc.wrapf && bc.pery, wz = bc.wrapf && bc.perz;
    return PlusFaces{(i < G.nx) ? sx[c + 1] : sx[c - (wx ? G.nx - 1 : 0)],
                     (j < G.ny) ? sy[c + G.px] : sy[c - (wy ? (long long)(G.ny - 1) * G.px : 0)],
                     (k < G.nz) ? sz[c + G.pxy] : sz[c - (wz ? (long long)(G.nz - 1) * G.pxy : 0)]};
}

// diagonal d, scaled unknown e = prd1*sqrt(d), scaled right-hand side b = q/sqrt(d) (:46-87, :118-124)
__global__ void __launch_bounds__(256) k_cg_diag(Geo G, BC bc, CGConst K, const double* __restrict__ sx,
                                                 const double* __restrict__ sy, const double* __restrict__ sz,
                                                 const double* __restrict__ u, const double* __restrict__ v,
                                                 const double* __restrict__ w, const double* __restrict__ prd1,
                                                 double* d, double* e, double* b, double* sdo, double* isdo) {
    const Thread3 t = tid3(1, 1, 1);
    const int i = t.i, j = t.j, k = t.k;
    if (i > G.nx || j > G.ny || k > G.nz) return;
    const long long c = G.idx(i, j, k);
    const PlusFaces P = plus_faces(G, bc, i, j, k, c, sx, sy, sz);
    const double dv = P.xp + sx[c] + P.yp + sy[c] + P.zp + sz[c];
    const double q = (FIDX(u, i, j, k) - FIDX(u, i + 1, j, k)) * K.rdx + (FIDX(v, i, j, k) - FIDX(v, i, j + 1, k)) * K.rdy +
                     (FIDX(w, i, j, k) - FIDX(w, i, j, k + 1)) * K.rdz;
    const double sd = sqrt(dv);
    const double isd = 1.0 / sd;
    d[c] = dv;
    e[c] = prd1[c] * sd;
    b[c] = q * isd;
    sdo[c] = sd;
    isdo[c] = isd;
}

// scaled face coefficients s/sqrt(d_c d_nb) = s * (1/sqrt(d_c)) * (1/sqrt(d_nb)) and the first
// residual (:126-151); reduction of r.r and b.b
constexpr int kCoefZ = 4;
__global__ void __launch_bounds__(256, 4) k_cg_coef(Geo G, BC bc, CGConst K, const double* __restrict__ sx,
                                                    const double* __restrict__ sy, const double* __restrict__ sz,
                                                    const double* __restrict__ sd, const double* __restrict__ isd,
                                                    const double* __restrict__ e, const double* __restrict__ b,
                                                    const double* __restrict__ prd1, double* ax, double* ay,
                                                    double* az, double* r, CGState* st, double* partial,
                                                    unsigned int* counter) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    double rr = 0.0, bbv = 0.0;
    // a thread owns kCoefZ cells of a column: 4x fewer blocks than one cell a thread, whose
    // partials the grid reduction (one counter) would otherwise take in turn
#pragma unroll
    for (int m = 0; m < kCoefZ; ++m) {
    const int k = blockIdx.z * kCoefZ + 1 + m;
    if (i <= nx && j <= ny && k <= nz) {
        const int c = (int)G.idx(i, j, k);
        const int px = G.px, pxy = (int)G.pxy;
        const Nb o = neighbours(G, bc, i, j, k);   // ghost-mapped neighbours (periodic wrap / Neumann self)
        const double ic = isd[c];
        const PlusFaces P = plus_faces(G, bc, i, j, k, c, sx, sy, sz);
        const double sxp = P.xp, syp = P.yp, szp = P.zp;
        const double app = sxp * ic * isd[c + o.xp];
        const double anp = sx[c] * ic * isd[c + o.xm];
        const double bpp = syp * ic * isd[c + o.yp];
        const double bnp = sy[c] * ic * isd[c + o.ym];
        const double cpp = szp * ic * isd[c + o.zp];
        const double cnp = sz[c] * ic * isd[c + o.zm];
        ax[c] = anp; ay[c] = bnp; az[c] = cnp;
        if (i == nx) ax[c + 1] = app;
        if (j == ny) ay[c + px] = bpp;
        if (k == nz) az[c + pxy] = cpp;
        // e at a neighbour: interior value, or the halo value prd1(ghost)*sqrt(d(mapped ghost))
        auto ee = [&](bool ghost, int cg, int off) { return ghost ? prd1[cg] * sd[c + off] : e[c + off]; };
        const double bv = b[c];
        const double rv = e[c] - app * ee(i == nx, c + 1, o.xp) - anp * ee(i == 1, c - 1, o.xm) -
                          bpp * ee(j == ny, c + px, o.yp) - bnp * ee(j == 1, c - px, o.ym) -
                          cpp * ee(k == nz, c + pxy, o.zp) - cnp * ee(k == 1, c - pxy, o.zm) - bv;
        r[c] = rv;
        rr += rv * rv;
        bbv += bv * bv;
    }
    }
    double trr, tbb;
    if (reduce2_last(rr, bbv, partial, counter, trr, tbb) && flat_tid() == 0) {
        st->rr = trr;
        st->rr_start = trr;
        st->bb = tbb;
        st->thr = (K.mode == 0) ? K.tol / K.ncell : K.tol * K.tol * tbb;
        st->alpha = 0.; st->beta = 0.; st->pq = 0.;
        st->iters = 0;
        st->maxit = K.maxit;
        st->mode = K.mode;
        st->status = 0;
        st->div_tol = K.div_tol;
        st->rmax = 0.;
        const bool go = (fabs(trr) > st->thr) && (K.maxit > 0);
        st->done = go ? 0 : 1;
        if (!isfinite(trr)) { st->status = SULI_ERR_NAN; st->done = 1; }
    }
}

// CG kernel A: p = r + beta*p_old (also at the neighbours), q = A~p, reduction of p.q (:192-205).
// One thread owns a column of kCGZA cells: the z neighbours of its cells are shared in
// registers and every global load of the column is independent (issued back to back), which
// is what keeps enough bytes in flight; x/y neighbours come through L1.  32-bit offsets.
constexpr int kTX = 32, kTY = 8, kCGZA = 4, kCGZB = 8;
__global__ void __launch_bounds__(kTX * kTY) k_cg_spmv(Geo G, BC bc, const double* __restrict__ r,
                                                       const double* __restrict__ p_old, double* __restrict__ p_new,
                                                       double* __restrict__ q, const double* __restrict__ ax,
                                                       const double* __restrict__ ay, const double* __restrict__ az,
                                                       CGState* st, double* partial, unsigned int* counter) {
    pdl_wait();
    if (st->done) return;
    const double beta = st->beta;
    const int nx = G.nx, ny = G.ny, nz = G.nz, px = G.px, pxy = (int)G.pxy;
    const int i = blockIdx.x * kTX + threadIdx.x + 1, j = blockIdx.y * kTY + threadIdx.y + 1;
    const int k0 = blockIdx.z * kCGZA + 1;
    double dot = 0.;
    if (i <= nx && j <= ny) {
        // neighbour offsets with the ghost maps of 9_grad.f90:99-116 (periodic wrap or Neumann copy)
        const int oxm = (i > 1) ? -1 : (bc.perx ? nx - 1 : 0);
        const int oxp = (i < nx) ? 1 : (bc.perx ? -(nx - 1) : 0);
        const int oym = (j > 1) ? -px : (bc.pery ? (ny - 1) * px : 0);
        const int oyp = (j < ny) ? px : (bc.pery ? -(ny - 1) * px : 0);
        const int c0 = kBase + (i - 1) + px * j;
        double col[kCGZA + 2];   // p at k0-1 .. k0+kCGZA
#pragma unroll
        for (int m = 0; m < kCGZA + 2; ++m) {
            const int k = map_any(k0 - 1 + m, nz, bc.perz);
            const int c = c0 + pxy * k;
            col[m] = r[c] + beta * p_old[c];
        }
#pragma unroll
        for (int m = 0; m < kCGZA; ++m) {
            const int k = k0 + m;
            if (k > nz) break;
            const int c = c0 + pxy * k;
            const double pxp = r[c + oxp] + beta * p_old[c + oxp];
            const double pxm = r[c + oxm] + beta * p_old[c + oxm];
            const double pyp = r[c + oyp] + beta * p_old[c + oyp];
            const double pym = r[c + oym] + beta * p_old[c + oym];
            const double pc = col[m + 1];
            const double qv = pc - pxp * ax[c + 1] - pxm * ax[c] - pyp * ay[c + px] - pym * ay[c] -
                              col[m + 2] * az[c + pxy] - col[m] * az[c];
            q[c] = qv;
            p_new[c] = pc;
            dot += pc * qv;
        }
    }
    double tpq, tdum;
    if (reduce2_last(dot, 0.0, partial, counter, tpq, tdum) && flat_tid() == 0) {
        st->rr_start = st->rr;
        st->pq = tpq;
        st->alpha = st->rr / tpq;
        if (!isfinite(st->alpha)) { st->status = SULI_ERR_NAN; st->done = 1; }
    }
}

// CG kernel A with two x cells a thread: every field row is read as 16-byte pairs (a warp moves
// 512 contiguous bytes a load), the pair's inner x neighbours come from the pair itself and only
// its two outer x neighbours are scalar loads.  Per cell the same expression as k_cg_spmv; only
// the p.q partial sums are grouped differently.  Needs nx even.
__global__ void __launch_bounds__(kTX * kTY) k_cg_spmv2(Geo G, BC bc, const double* __restrict__ r,
                                                        const double* __restrict__ p_old, double* __restrict__ p_new,
                                                        double* __restrict__ q, const double* __restrict__ ax,
                                                        const double* __restrict__ ay, const double* __restrict__ az,
                                                        CGState* st, double* partial, unsigned int* counter) {
    pdl_wait();
    if (st->done) return;
    const double beta = st->beta;
    const int nx = G.nx, ny = G.ny, nz = G.nz, px = G.px, pxy = (int)G.pxy;
    const int i0 = 2 * (blockIdx.x * kTX + threadIdx.x) + 1, j = blockIdx.y * kTY + threadIdx.y + 1;
    const int k0 = blockIdx.z * kCGZA + 1;
    double dot = 0.;
    if (i0 <= nx && j <= ny) {
        const int oxm = (i0 > 1) ? -1 : (bc.perx ? nx - 1 : 0);            // of cell i0
        const int oxp = (i0 + 1 < nx) ? 1 : (bc.perx ? -(nx - 1) : 0);     // of cell i0 + 1
        const int oym = (j > 1) ? -px : (bc.pery ? (ny - 1) * px : 0);
        const int oyp = (j < ny) ? px : (bc.pery ? -(ny - 1) * px : 0);
        const int c0 = kBase + (i0 - 1) + px * j;
        auto ld2 = [](const double* a, int c) { return *reinterpret_cast<const double2*>(a + c); };
        auto pn2 = [&](int c) {
            const double2 a = ld2(r, c), b = ld2(p_old, c);
            return make_double2(a.x + beta * b.x, a.y + beta * b.y);
        };
        double2 col[kCGZA + 2];   // p of the pair at k0-1 .. k0+kCGZA
#pragma unroll
        for (int m = 0; m < kCGZA + 2; ++m) col[m] = pn2(c0 + pxy * map_any(k0 - 1 + m, nz, bc.perz));
#pragma unroll
        for (int m = 0; m < kCGZA; ++m) {
            const int k = k0 + m;
            if (k > nz) break;
            const int c = c0 + pxy * k;
            const double pxm = r[c + oxm] + beta * p_old[c + oxm];                 // left of cell i0
            const double pxp = r[c + 1 + oxp] + beta * p_old[c + 1 + oxp];         // right of cell i0 + 1
            const double2 pym = pn2(c + oym), pyp = pn2(c + oyp);
            const double2 pc = col[m + 1], pzm = col[m], pzp = col[m + 2];
            const double2 axc = ld2(ax, c), ayc = ld2(ay, c), ayp = ld2(ay, c + px), azc = ld2(az, c),
                          azp = ld2(az, c + pxy);
            const double ax2 = ax[c + 2];
            const double q0 = pc.x - pc.y * axc.y - pxm * axc.x - pyp.x * ayp.x - pym.x * ayc.x - pzp.x * azp.x -
                              pzm.x * azc.x;
            const double q1 = pc.y - pxp * ax2 - pc.x * axc.y - pyp.y * ayp.y - pym.y * ayc.y - pzp.y * azp.y -
                              pzm.y * azc.y;
            *reinterpret_cast<double2*>(q + c) = make_double2(q0, q1);
            *reinterpret_cast<double2*>(p_new + c) = pc;
            dot += pc.x * q0;
            dot += pc.y * q1;
        }
    }
    double tpq, tdum;
    if (reduce2_last(dot, 0.0, partial, counter, tpq, tdum) && flat_tid() == 0) {
        st->rr_start = st->rr;
        st->pq = tpq;
        st->alpha = st->rr / tpq;
        if (!isfinite(st->alpha)) { st->status = SULI_ERR_NAN; st->done = 1; }
    }
}

// CG kernel B: e -= alpha p, r -= alpha q, reduction of r.r, beta and the stopping test (:210-221, :175)
__global__ void __launch_bounds__(kTX * kTY) k_cg_update(Geo G, double* __restrict__ e, double* __restrict__ r,
                                                         const double* __restrict__ p, const double* __restrict__ q,
                                                         CGState* st, double* partial, unsigned int* counter) {
    pdl_wait();
    if (st->done) return;
    const double alpha = st->alpha;
    const int i = blockIdx.x * kTX + threadIdx.x + 1, j = blockIdx.y * kTY + threadIdx.y + 1;
    const int k0 = blockIdx.z * kCGZB + 1;
    const int pxy = (int)G.pxy;
    double rr = 0.;
    if (i <= G.nx && j <= G.ny) {
        const int c0 = kBase + (i - 1) + G.px * j;
        const int k1 = min(k0 + kCGZB - 1, G.nz);
        for (int k = k0; k <= k1; ++k) {
            const int c = c0 + pxy * k;
            e[c] = e[c] - alpha * p[c];
            const double rn = r[c] - alpha * q[c];
            r[c] = rn;
            rr += rn * rn;
        }
    }
    double trr, tdum;
    if (reduce2_last(rr, 0.0, partial, counter, trr, tdum) && flat_tid() == 0) {
        const double rr_old = st->rr;
        st->rr = trr;
        st->beta = trr / rr_old;
        st->iters = st->iters + 1;
        bool go;
        if (st->mode == 0) go = fabs(st->rr_start) > st->thr;
        else go = trr > st->thr;
        if (st->iters >= st->maxit) { go = false; st->status = SULI_WARN_CG_MAXIT; }
        if (!isfinite(trr)) { go = false; st->status = SULI_ERR_NAN; }
        st->done = go ? 0 : 1;
    }
}

// Divergence test of a finished CG solve (div_tol > 0): max |sqrt(d) r~| over the cells is the
// max |div u| that posdin leaves with this pressure (the unscaled residual of the face-flux
// balance).  Above div_tol, the stopping threshold on r~.r~ is lowered by (div_tol/max)^2 / 2
// (at least 4x) and the solve resumes; the host relaunches the iteration loop.
__global__ void __launch_bounds__(256) k_cg_divcheck(Geo G, const double* __restrict__ sd,
                                                     const double* __restrict__ r, CGState* st, double* partial,
                                                     unsigned int* counter) {
    if (!st->done || st->status != 0 || !(st->div_tol > 0.)) return;
    const Thread3 t = tid3(1, 1, 1);
    double m = 0.;
    if (t.i <= G.nx && t.j <= G.ny && t.k <= G.nz) {
        const long long c = G.idx(t.i, t.j, t.k);
        m = fabs(sd[c] * r[c]);
        if (isnan(m)) m = INFINITY;
    }
    double ta, tb, tm;
    if (reduce3_last(0., 0., m, partial, counter, ta, tb, tm) && flat_tid() == 0) {
        st->rmax = tm;
        if (tm > st->div_tol && st->iters < st->maxit && isfinite(tm)) {
            const double f = 0.5 * (st->div_tol / tm) * (st->div_tol / tm);
            st->thr = st->thr * fmin(0.25, f);
            st->done = 0;
        }
    }
}

// loop condition of the CG iteration graph: repeat until the state says done
__global__ void k_cg_cond(cudaGraphConditionalHandle h, const CGState* st) {
    pdl_wait();
    cudaGraphSetConditional(h, st->done ? 0u : 1u);
}

// de-normalisation over the halo box (:268-274)
__global__ void k_cg_final(Geo G, BC bc, const double* __restrict__ sdv, const double* __restrict__ e,
                           double* prd1, const CGState* st) {
    const Thread3 t = tid3(0, 0, 0);
    const int i = t.i, j = t.j, k = t.k, nx = G.nx, ny = G.ny, nz = G.nz;
    if (i > nx + 1 || j > ny + 1 || k > nz + 1) return;
    const int mi = map_any(i, nx, bc.perx), mj = map_any(j, ny, bc.pery), mk = map_any(k, nz, bc.perz);
    const bool gh = (mi != i || mj != j || mk != k);
    const double sd = FIDX(sdv, mi, mj, mk);   // sqrt(d), stored by the set-up
    if (!gh) {
        FIDX(prd1, i, j, k) = FIDX(e, i, j, k) / sd;
    } else if (st->iters == 0) {
        FIDX(prd1, i, j, k) = (FIDX(prd1, i, j, k) * sd) / sd;
    } else {
        FIDX(prd1, i, j, k) = FIDX(e, mi, mj, mk) / sd;
    }
}

// ------------------------------------------------------------------------------------
// posdin (10_pos.f90:1-96) and est (4_plot.f90:500-525)
// ------------------------------------------------------------------------------------
// A thread owns a column of kPosZ faces (i, j, k0 .. k0 + kPosZ - 1) and walks it in z, so the
// plane below (prd1 and rho at k - 1) was read by the same thread a step earlier and comes from
// L1 instead of being fetched again from DRAM by another block.
constexpr int kPosZ = 8;
__global__ void __launch_bounds__(256) k_posdin(Geo G, BC bc, double aux1, double aux2, double aux3,
                                                const double* __restrict__ rho, const double* __restrict__ prd1,
                                                double* __restrict__ u, double* __restrict__ v,
                                                double* __restrict__ w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k0 = blockIdx.z * kPosZ + 1;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    if (i > nx + 1 || j > ny + 1) return;
    const int k1 = min(k0 + kPosZ - 1, nz + 1);
    for (int k = k0; k <= k1; ++k) {
        if (j <= ny && k <= nz) {
            const double rhox = rho_face_x(G, bc, rho, i, j, k);
            FIDX(u, i, j, k) = FIDX(u, i, j, k) - aux1 * (FIDX(prd1, i, j, k) - FIDX(prd1, i - 1, j, k)) / rhox;
        }
        if (i <= nx && k <= nz) {
            const double rhoy = rho_face_y(G, bc, rho, i, j, k);
            FIDX(v, i, j, k) = FIDX(v, i, j, k) - aux2 * (FIDX(prd1, i, j, k) - FIDX(prd1, i, j - 1, k)) / rhoy;
        }
        if (i <= nx && j <= ny) {
            const double rhoz = rho_face_z(G, bc, rho, i, j, k);
            FIDX(w, i, j, k) = FIDX(w, i, j, k) - aux3 * (FIDX(prd1, i, j, k) - FIDX(prd1, i, j, k - 1)) / rhoz;
        }
    }
}

// A thread walks kEstChunks chunks of kEstZ cells of a column.  Each chunk's loop is unrolled and
// loads from clamped plane indices, so its loads are issued together; planes past nz are left
// out of the maximum.  The w face above a cell is the face below the next one.  The differences
// are multiplied by the cell sizes' reciprocals, formed on the host (as in every FP64 kernel
// here, a division by a constant is one reciprocal and multiplications).
constexpr int kEstZ = 4, kEstChunks = 4;
__global__ void __launch_bounds__(256) k_est(Geo G, double rdx, double rdy, double rdz, const double* __restrict__ u,
                                             const double* __restrict__ v, const double* __restrict__ w,
                                             double* partial, unsigned int* counter, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    double m = 0.;
    if (i <= G.nx && j <= G.ny) {
        for (int ch = 0; ch < kEstChunks; ++ch) {
            const int k0 = (blockIdx.z * kEstChunks + ch) * kEstZ + 1;
            if (k0 > G.nz) break;
            double wz[kEstZ + 1];
#pragma unroll
            for (int q = 0; q <= kEstZ; ++q) wz[q] = FIDX(w, i, j, min(k0 + q, G.nz + 1));
#pragma unroll
            for (int q = 0; q < kEstZ; ++q) {
                const int k = min(k0 + q, G.nz);
                const double dv = (FIDX(u, i + 1, j, k) - FIDX(u, i, j, k)) * rdx + (FIDX(v, i, j + 1, k) - FIDX(v, i, j, k)) * rdy +
                                  (wz[q + 1] - wz[q]) * rdz;
                if (k0 + q <= G.nz) m = isnan(dv) ? INFINITY : fmax(m, fabs(dv));
            }
        }
    }
    double ta, tb;
    if (reduce2_last(m, 0.0, partial, counter, ta, tb, true) && flat_tid() == 0) out[0] = ta;
}

__global__ void k_fill(double* a, long long n, double v) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) a[q] = v;
}

// ------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------
static LsConst ls_const(const suli_ctx* c) {
    LsConst L;
    L.ihx = (c->P.ccx0 == 0) ? 0 : 2;
    L.ihy = (c->P.ccy0 == 0) ? 0 : 2;
    L.ihz = (c->P.ccz0 == 0) ? 0 : 1;
    L.ihn = L.ihz;   // der_weno leaves ihs at its z value (14_level_set.f90:377, 717)
    L.dx = c->P.dx; L.dy = c->P.dy; L.dz = c->P.dz;
    L.rx = 1. / L.dx; L.ry = 1. / L.dy; L.rz = 1. / L.dz;
    L.frx = 1.f / (float)L.dx; L.fry = 1.f / (float)L.dy; L.frz = 1.f / (float)L.dz;
    L.dx1 = fmax(L.dx, fmax(L.dy, L.dz));
    L.ad = c->P.alpha1 * L.dx1;
    L.pi = acos(-1.0);
    L.rho1 = c->P.rho_f1; L.rho2 = c->P.rho_f2; L.mi1 = c->P.mi_f1; L.mi2 = c->P.mi_f2;
    L.t_hs = c->P.t_hs;
    L.mu1s = c->P.mi_f1 * 10000.; L.mu2s = c->P.mi_f2 * 10000.;
    return L;
}
static dim3 cells_grid(const Geo& g) { return grid3(g.nx, g.ny, g.nz, kBlk); }
static dim3 faces_grid(const Geo& g) { return grid3(g.nx + 1, g.ny + 1, g.nz + 1, kBlk); }

// stencil arithmetic in FP32 for the mixed-precision path (precision 1), FP64 otherwise; the
// fields stay FP64 either way
#define LAUNCH_R(kern, grid, block, ...)                                                   \
    do {                                                                                   \
        if (c->P.precision == 1) kern<float><<<(grid), (block), 0, c->stream>>>(__VA_ARGS__);  \
        else kern<double><<<(grid), (block), 0, c->stream>>>(__VA_ARGS__);                 \
    } while (0)

void launch_lsprops(suli_ctx* c, const double* ls, bool do_mod, bool do_hs, bool do_vol) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_LSPROPS, 1);
    LAUNCH_R(k_lsprops, cells_grid(G), kBlk,
        G, ls_const(c), ls, c->f[SULI_F_MOD_LS], c->nrmx, c->nrmy, c->nrmz, c->f[SULI_F_HS], c->f[SULI_F_HSX],
        c->f[SULI_F_HSY], c->f[SULI_F_HSZ], c->f[SULI_F_RHO], c->f[SULI_F_LS_NU], do_mod, do_hs, do_vol,
        c->red_partial, c->red_counter, c->red_out);
}
void launch_curv(suli_ctx* c) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_CURV, 1);
    LAUNCH_R(k_curv, cells_grid(G), kBlk, G, ls_const(c), c->nrmx, c->nrmy, c->nrmz, c->f[SULI_F_DDLSDX],
                                                   c->f[SULI_F_DDLSDY], c->f[SULI_F_DDLSDZ], c->f[SULI_F_KURV]);
}
void launch_ls_advect(suli_ctx* c, const double* cur, const double* phi0, double* out, double a, double b, double gd) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_LS_ADVECT, 1);
    LAUNCH_R(k_ls_advect, cells_grid(G), kBlk, G, ls_const(c), cur, phi0, out, c->f[SULI_F_U], c->f[SULI_F_V],
                                                        c->f[SULI_F_W], a, b, gd);
}
void launch_reinit_funcs(suli_ctx* c) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_REINIT, 1);
    LAUNCH_R(k_reinit_funcs, cells_grid(G), kBlk, G, ls_const(c), c->f[SULI_F_LS], c->funcs);
}
void launch_reinit_stage(suli_ctx* c, const double* cur, const double* phi0, double* out, double a, double b, double gd) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_REINIT, 1);
    LAUNCH_R(k_reinit_stage, cells_grid(G), kBlk, G, ls_const(c), cur, phi0, out, c->funcs, a, b, gd);
}
void launch_reinit_err(suli_ctx* c, const double* after, const double* before, double band) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_REINIT, 1);
    k_reinit_err<<<cells_grid(G), kBlk, 0, c->stream>>>(G, after, before, band, c->red_partial, c->red_counter,
                                                         c->red_out);
}
void launch_ls_shift(suli_ctx* c, double shift) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_VOLFIX, 1);
    k_ls_shift<<<cells_grid(G), kBlk, 0, c->stream>>>(G, c->f[SULI_F_LS], shift);
}
void launch_volfix(suli_ctx* c, double dt1fac) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_VOLFIX, 1);
    k_volfix<<<cells_grid(G), kBlk, 0, c->stream>>>(G, c->f[SULI_F_LS], c->f[SULI_F_MOD_LS], dt1fac, c->vol_ini);
}
constexpr int kNutZ = 4;   // cells of a column per thread in k_nut
void launch_visco(suli_ctx* c) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_VISCO, c->P.m_turb == 1 ? 2 : 1);
    if (c->P.m_turb == 2) {
        ViscDirConst V;
        const double cs = c->P.csmag;
        V.itdx = 1. / (2. * c->P.dx); V.itdy = 1. / (2. * c->P.dy); V.itdz = 1. / (2. * c->P.dz);
        V.cx = c->P.dx * c->P.dx * cs * cs; V.cy = c->P.dy * c->P.dy * cs * cs; V.cz = c->P.dz * c->P.dz * cs * cs;
        if (c->P.precision == 1)
            k_facenu_dir<float><<<faces_grid(G), kBlk, 0, c->stream>>>(G, V, c->f[SULI_F_U], c->f[SULI_F_V],
                                                                     c->f[SULI_F_W], c->f[SULI_F_LS_NU],
                                                                     c->f[SULI_F_XNUT], c->f[SULI_F_YNUT],
                                                                     c->f[SULI_F_ZNUT]);
        else
            k_facenu_dir<double><<<faces_grid(G), kBlk, 0, c->stream>>>(G, V, c->f[SULI_F_U], c->f[SULI_F_V],
                                                                      c->f[SULI_F_W], c->f[SULI_F_LS_NU],
                                                                      c->f[SULI_F_XNUT], c->f[SULI_F_YNUT],
                                                                      c->f[SULI_F_ZNUT]);
        return;
    }
    if (c->P.m_turb == 1) {
        ViscConst V;
        V.dx = c->P.dx; V.dy = c->P.dy; V.dz = c->P.dz; V.csmag = c->P.csmag;
        V.cdel = pow(c->P.dx * c->P.dy * c->P.dz, 2. / 3.);
        const bool col = G.nz % kNutZ == 0;
        const dim3 gn = grid3(G.nx, G.ny, col ? G.nz / kNutZ : G.nz, kBlk);
        const double *u = c->f[SULI_F_U], *v = c->f[SULI_F_V], *w = c->f[SULI_F_W], *rho = c->f[SULI_F_RHO];
        double* nut = c->f[SULI_F_NUT];
        if (c->P.precision == 1) {   // FP32 arithmetic over the FP64 state
            if (col) k_nut<float, kNutZ><<<gn, kBlk, 0, c->stream>>>(G, V, u, v, w, rho, nut);
            else k_nut<float, 1><<<gn, kBlk, 0, c->stream>>>(G, V, u, v, w, rho, nut);
        } else {
            if (col) k_nut<double, kNutZ><<<gn, kBlk, 0, c->stream>>>(G, V, u, v, w, rho, nut);
            else k_nut<double, 1><<<gn, kBlk, 0, c->stream>>>(G, V, u, v, w, rho, nut);
        }
    }
    k_facenu<<<faces_grid(G), kBlk, 0, c->stream>>>(G, c->P.m_turb, c->f[SULI_F_LS_NU], c->f[SULI_F_NUT],
                                                     c->f[SULI_F_XNUT], c->f[SULI_F_YNUT], c->f[SULI_F_ZNUT]);
}
template <typename R>
static void convdiff_der(suli_ctx* c, const CDConst& C, const CDFields& F) {
    const Geo& G = c->g;
    if (c->P.adv_type == 2) {
        k_convdiff<R, 1, 2><<<faces_grid(G), kBlk, 0, c->stream>>>(G, C, F);
        return;
    }
    if (c->P.adv_type == 3) {
        k_convdiff<R, 1, 3><<<faces_grid(G), kBlk, 0, c->stream>>>(G, C, F);
        return;
    }
    switch (c->P.der) {
    case 2: k_convdiff<R, 2, 1><<<faces_grid(G), kBlk, 0, c->stream>>>(G, C, F); break;
    case 3: k_convdiff<R, 3, 1><<<faces_grid(G), kBlk, 0, c->stream>>>(G, C, F); break;
    default: k_convdiff<R, 1, 1><<<faces_grid(G), kBlk, 0, c->stream>>>(G, C, F); break;
    }
}
void launch_convdiff(suli_ctx* c) {
    const Geo& G = c->g;
    CDConst C;
    C.idx = 1. / c->P.dx; C.idy = 1. / c->P.dy; C.idz = 1. / c->P.dz;
    C.gx = c->P.gx; C.gz = c->P.gz; C.sigma = c->P.sigma;
    C.cz = c->P.gz / (c->P.chezy * c->P.chezy);
    C.tf = c->tf_active ? 1 : 0;
    C.cap_z2 = (c->P.ccz0 == 2); C.cap_y2 = (c->P.ccy0 == 2); C.cap_yn = (c->P.ccyf == 2);
    C.obst = (c->P.obst_t != 0);
    CDFields F;
    F.u = c->f[SULI_F_U]; F.v = c->f[SULI_F_V]; F.w = c->f[SULI_F_W]; F.rho = c->f[SULI_F_RHO];
    F.hsx = c->f[SULI_F_HSX]; F.hsy = c->f[SULI_F_HSY]; F.hsz = c->f[SULI_F_HSZ]; F.kurv = c->f[SULI_F_KURV];
    F.nut = c->f[SULI_F_NUT]; F.xnut = c->f[SULI_F_XNUT]; F.ynut = c->f[SULI_F_YNUT]; F.znut = c->f[SULI_F_ZNUT];
    F.ub = c->f[SULI_F_UB]; F.vb = c->f[SULI_F_VB]; F.wb = c->f[SULI_F_WB];
    F.tfu = c->f[SULI_F_TF_U]; F.tfv = c->f[SULI_F_TF_V]; F.tfw = c->f[SULI_F_TF_W];
    F.Fu = c->f[SULI_F_FU]; F.Fv = c->f[SULI_F_FV]; F.Fw = c->f[SULI_F_FW];
    ProfScope ps(c, SULI_K_CONVDIFF, 1);
    cudaMemcpyAsync(c->f[SULI_F_PRD0], c->f[SULI_F_PRD1], G.n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    if (c->P.precision == 1)   // FP32 arithmetic over the FP64 state
        convdiff_der<float>(c, C, F);
    else
        convdiff_der<double>(c, C, F);
}
void launch_tempo(suli_ctx* c, int tt, int it) {
    const Geo& G = c->g;
    TempoArgs T;
    T.a[0] = c->f[SULI_F_U]; T.a[1] = c->f[SULI_F_V]; T.a[2] = c->f[SULI_F_W];
    T.F[0] = c->f[SULI_F_FU]; T.F[1] = c->f[SULI_F_FV]; T.F[2] = c->f[SULI_F_FW];
    T.a0[0] = c->f[SULI_F_U0]; T.a0[1] = c->f[SULI_F_V0]; T.a0[2] = c->f[SULI_F_W0];
    T.f0[0] = c->f[SULI_F_FU0]; T.f0[1] = c->f[SULI_F_FV0]; T.f0[2] = c->f[SULI_F_FW0];
    T.f1[0] = c->f[SULI_F_FU1]; T.f1[1] = c->f[SULI_F_FV1]; T.f1[2] = c->f[SULI_F_FW1];
    T.tm = c->P.t_tempo; T.tt = tt; T.it = it; T.dt = c->dt;
    ProfScope ps(c, SULI_K_TEMPO, 1);
    k_tempo<<<faces_grid(G), kBlk, 0, c->stream>>>(G, T);
}
void launch_boundary_waves(suli_ctx* c) {
    const Geo& G = c->g;
    const dim3 b2(32, 8);
    ProfScope ps(c, SULI_K_CONTORNO, 2);
    k_ls_round_float<<<cells_grid(G), kBlk, 0, c->stream>>>(G, c->f[SULI_F_LS]);
    cudaMemsetAsync(c->f[SULI_F_BXY0], 0, c->plane_elems[SULI_F_BXY0] * sizeof(double), c->stream);   // v1 never set
    k_waves<<<grid3(G.ny + 2, G.nz + 3, 1, b2), b2, 0, c->stream>>>(G, c->wave, c->P.dx, c->P.dz, c->t, c->f[SULI_F_LS],
                                                                     c->f[SULI_F_BXX0], c->f[SULI_F_BXX1], c->f[SULI_F_BXZ0]);
}
void launch_contorno(suli_ctx* c, int nlock) {
    const Geo& G = c->g;
    const bool obst = (c->P.obst_t != 0);
    const dim3 b2(32, 8);
    if (nlock == 3) {   // acts only with obstacles (3_contorno.f90:445-487)
        if (!obst) return;
        {
            ProfScope ps(c, SULI_K_CONTORNO, 1);
            k_ls_obst<<<grid3(G.nx, G.ny, 1, b2), b2, 0, c->stream>>>(G, c->obst_kw, c->f[SULI_F_LS]);
        }
        launch_lsprops(c, c->f[SULI_F_LS], false, true, false);   // heaviside()
        return;
    }
    if (nlock != 1 && nlock != 2) return;
    BCArgs A;
    A.u = c->f[SULI_F_U]; A.v = c->f[SULI_F_V]; A.w = c->f[SULI_F_W];
    A.ub = c->f[SULI_F_UB]; A.vb = c->f[SULI_F_VB]; A.wb = c->f[SULI_F_WB];
    A.prd1 = c->f[SULI_F_PRD1];
    A.pl = c->planes();
    A.nlock = nlock;
    A.obst = obst ? 1 : 0;
    const bool capy = !obst && (c->bc.y0 == 2 || c->bc.yf == 2);
    ProfScope ps(c, SULI_K_CONTORNO, (nlock == 2 ? 7 + (c->P.outflow_fix == 1 && c->bc.xf == 4 ? 1 : 0) : 4) +
                                         (capy || obst ? 1 : 0));
    {
        const long long ng = 2LL * (G.ny + 2) * (G.nz + 2) + 2LL * G.nx * (G.nz + 2) + 2LL * G.nx * G.ny;
        k_prd_ghosts<<<(unsigned)((ng + 255) / 256), 256, 0, c->stream>>>(G, c->bc, A.prd1);
    }
    k_bc_y<<<grid3(G.nx + 3, G.nz + 3, 1, b2), b2, 0, c->stream>>>(G, c->bc, A);
    k_bc_x<<<grid3(G.ny + 3, G.nz + 3, 1, b2), b2, 0, c->stream>>>(G, c->bc, A);
    k_bc_z<<<grid3(G.nx + 3, G.ny + 3, 1, b2), b2, 0, c->stream>>>(G, c->bc, A);
    if (capy) k_bc_capture_y<<<grid3(G.nx + 3, G.nz + 3, 1, b2), b2, 0, c->stream>>>(G, c->bc, A);
    if (obst) {
        const ObstMasks M{c->obst_ku, c->obst_kv, c->obst_kw};
        k_bc_obst<<<grid3(G.nx + 3, G.ny + 3, 1, b2), b2, 0, c->stream>>>(G, M, A);
    }
    if (nlock == 2) {
        k_bc_ny<<<grid3(G.nx + 2, G.nz + 2, 1, b2), b2, 0, c->stream>>>(G, c->bc, A);
        k_bc_nx<<<grid3(G.ny + 3, G.nz + 3, 1, b2), b2, 0, c->stream>>>(G, c->bc, A);
        k_bc_nz<<<grid3(G.nx + 2, G.ny + 2, 1, b2), b2, 0, c->stream>>>(G, c->bc, A);
        if (c->P.outflow_fix == 1 && c->bc.xf == 4)
            k_outflow_fix<<<1, kFixThreads, 0, c->stream>>>(G, A, obst ? c->obst_ku : nullptr, c->P.dx, c->P.dy,
                                                            c->P.dz);
    }
}
static CGConst cg_const(const suli_ctx* c) {
    CGConst K;
    K.cx = c->dt / (c->P.dx * c->P.dx);
    K.cy = c->dt / (c->P.dy * c->P.dy);
    K.cz = c->dt / (c->P.dz * c->P.dz);
    K.dx = c->P.dx; K.dy = c->P.dy; K.dz = c->P.dz;
    K.rdx = 1. / K.dx; K.rdy = 1. / K.dy; K.rdz = 1. / K.dz;
    K.tol = c->P.cg_tol;
    K.div_tol = c->P.div_tol;
    K.ncell = (double)(c->P.nx * c->P.ny * c->P.nz);
    K.mode = c->P.cg_stop;
    K.maxit = c->P.cg_maxit;
    return K;
}
void launch_cg_setup(suli_ctx* c) {
    const Geo& G = c->g;
    const CGConst K = cg_const(c);
    ProfScope ps(c, SULI_K_CG_SETUP, 3);
    // face scratch: the CG direction and product vectors, written again before the iterations read them
    double *sx = c->cg_pa, *sy = c->cg_pb, *sz = c->cg_q;
    k_cg_faces<<<cells_grid(G), kBlk, 0, c->stream>>>(G, c->bc, K, c->f[SULI_F_RHO], sx, sy, sz);
    k_cg_diag<<<cells_grid(G), kBlk, 0, c->stream>>>(G, c->bc, K, sx, sy, sz, c->f[SULI_F_U], c->f[SULI_F_V], c->f[SULI_F_W],
                                                      c->f[SULI_F_PRD1], c->cg_d, c->cg_e, c->cg_b, c->cg_sd, c->cg_isd);
    k_cg_coef<<<grid3(G.nx, G.ny, (G.nz + kCoefZ - 1) / kCoefZ, kBlk), kBlk, 0, c->stream>>>(G, c->bc, K, sx, sy, sz, c->cg_sd, c->cg_isd, c->cg_e, c->cg_b,
                                                      c->f[SULI_F_PRD1], c->cg_ax, c->cg_ay, c->cg_az, c->cg_r, c->cg,
                                                      c->red_partial, c->red_counter);
}
void launch_cg_iter(suli_ctx* c, const double* p_old, double* p_new) {
    const Geo& G = c->g;
    const dim3 b(kTX, kTY, 1);
    const dim3 ga((G.nx + kTX - 1) / kTX, (G.ny + kTY - 1) / kTY, (G.nz + kCGZA - 1) / kCGZA);
    const dim3 gb((G.nx + kTX - 1) / kTX, (G.ny + kTY - 1) / kTY, (G.nz + kCGZB - 1) / kCGZB);
    {
        ProfScope ps(c, SULI_K_CG_SPMV, 1);
        if (G.nx % 2 == 0) {
            const dim3 g2((G.nx / 2 + kTX - 1) / kTX, (G.ny + kTY - 1) / kTY, (G.nz + kCGZA - 1) / kCGZA);
            pdl_launch(k_cg_spmv2, g2, b, c->stream, G, c->bc, (const double*)c->cg_r, p_old, p_new, c->cg_q,
                       (const double*)c->cg_ax, (const double*)c->cg_ay, (const double*)c->cg_az, c->cg,
                       c->red_partial, c->red_counter);
        } else {
            pdl_launch(k_cg_spmv, ga, b, c->stream, G, c->bc, (const double*)c->cg_r, p_old, p_new, c->cg_q,
                       (const double*)c->cg_ax, (const double*)c->cg_ay, (const double*)c->cg_az, c->cg,
                       c->red_partial, c->red_counter);
        }
    }
    ProfScope ps(c, SULI_K_CG_UPDATE, 1);
    pdl_launch(k_cg_update, gb, b, c->stream, G, c->cg_e, c->cg_r, (const double*)p_new, (const double*)c->cg_q, c->cg,
               c->red_partial, c->red_counter);
}
void launch_cg_cond(suli_ctx* c, cudaGraphConditionalHandle h) { pdl_launch(k_cg_cond, 1, 1, c->stream, h, c->cg); }
void launch_cg_divcheck(suli_ctx* c) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_CG_FINAL, 1);
    k_cg_divcheck<<<cells_grid(G), kBlk, 0, c->stream>>>(G, c->cg_sd, c->cg_r, c->cg, c->red_partial, c->red_counter);
}
void launch_cg_final(suli_ctx* c, const double* e) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_CG_FINAL, 1);
    k_cg_final<<<grid3(G.nx + 2, G.ny + 2, G.nz + 2, kBlk), kBlk, 0, c->stream>>>(G, c->bc, c->cg_sd, e,
                                                                                   c->f[SULI_F_PRD1], c->cg);
}
void launch_posdin(suli_ctx* c) {
    const Geo& G = c->g;
    const double aux1 = c->dt / c->P.dx, aux2 = c->dt / c->P.dy, aux3 = c->dt / c->P.dz;
    ProfScope ps(c, SULI_K_POSDIN, 1);
    k_posdin<<<grid3(G.nx + 1, G.ny + 1, (G.nz + 1 + kPosZ - 1) / kPosZ, kBlk), kBlk, 0, c->stream>>>(G, c->bc, aux1, aux2, aux3, c->f[SULI_F_RHO], c->f[SULI_F_PRD1],
                                                     c->f[SULI_F_U], c->f[SULI_F_V], c->f[SULI_F_W]);
    cudaMemcpyAsync(c->f[SULI_F_PRD], c->f[SULI_F_PRD1], G.n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
}
void launch_est(suli_ctx* c) {
    const Geo& G = c->g;
    ProfScope ps(c, SULI_K_EST, 1);
    k_est<<<grid3(G.nx, G.ny, (G.nz + kEstZ * kEstChunks - 1) / (kEstZ * kEstChunks), kBlk), kBlk, 0, c->stream>>>(G, 1. / c->P.dx, 1. / c->P.dy, 1. / c->P.dz, c->f[SULI_F_U],
                                                  c->f[SULI_F_V], c->f[SULI_F_W], c->red_partial, c->red_counter,
                                                  c->red_out);
}
void launch_fill(suli_ctx* c, double* a, double v) {
    const long long n = (long long)c->g.n;
    k_fill<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(a, n, v);
}

}  // namespace suli
