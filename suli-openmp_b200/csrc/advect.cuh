// advect.cuh — the flux-split advective forms of 6_convdiff.f90:72-79 other than classico,
// per face: rotacional (adv_type = 2, 7_advectivo.f90:293-457) and antissim (adv_type = 3,
// :460-653).  The reference builds both on first-order upwinding only (der = 1).
//
// Along one direction, with the advecting velocity c split as c+ = max(c, 0), c- = min(c, 0)
// and the advected component a at the points m-1, m, m+1:
//   rotacional:  ((c+ a)(m) - (c+ a)(m-1))/h + ((c- a)(m+1) - (c- a)(m))/h
//   antissim:    half of that, plus half of the advective upwind difference
//                c+(m) (a(m) - a(m-1))/h + c-(m) (a(m+1) - a(m))/h.
// The transverse advecting velocities are classico's four-point averages at each point.
// The reference keeps c+ and c- in arrays whose end planes it fills separately; each value
// is read here from the point the reference reads it from:
//   * antissim copies plane 1 into plane 0 (:521-522, 571-572, 618-619), so c+ below the
//     first point is c+ at the first point, and copies the last face into the plane past a
//     component's own last face (:524, 574, 621), so c- there is c- at the last face;
//   * rotacional computes every plane from the velocities; above the top w-face it sets c+
//     where c- is meant (:433), leaving c- there unset in the reference, and c- = min(w, 0)
//     of that ghost is used (it enters only Fw on the top face, which the boundary fill
//     overwrites).
// Every read stays inside the padded box of geom.cuh for faces i <= nx+1, j <= ny+1,
// k <= nz+1.
#pragma once
#include "geom.cuh"

namespace suli {

// reads of the padded-box fields around one face, converted to the compute type R
template <typename R>
struct FaceTaps {
    int c0, px, pxy;
    __host__ __device__ __forceinline__ R operator()(const double* a, int di, int dj, int dk) const {
        return R(a[c0 + di + dj * px + dk * pxy]);
    }
};

template <typename R>
__host__ __device__ __forceinline__ R split_pos(R c) { return c > R(0.) ? c : R(0.); }
template <typename R>
__host__ __device__ __forceinline__ R split_neg(R c) { return c < R(0.) ? c : R(0.); }

// one direction's term: a at m-1, m, m+1; c at the point read for c+(m-1), at m, and at the
// point read for c-(m+1); ih = 1/h
template <typename R, int ADV>
__host__ __device__ __forceinline__ R split_term(R am, R a0, R ap, R cm, R c0, R cp, R ih) {
    const R Pm = split_pos(cm), P0 = split_pos(c0), N0 = split_neg(c0), Np = split_neg(cp);
    const R f = (P0 * a0 - Pm * am) * ih + (Np * ap - N0 * a0) * ih;
    if constexpr (ADV == 2) {
        return f;
    } else {
        return (f + P0 * (a0 - am) * ih + N0 * (ap - a0) * ih) * R(0.5);
    }
}

// offset of the point read for c+(m-1): antissim's copied plane 0 reads plane 1
template <int ADV>
__host__ __device__ __forceinline__ int split_lo(int m) { return (ADV == 3 && m == 1) ? 0 : -1; }
// offset of the point read for c-(m+1) along a component's own direction, n = its last face
template <int ADV>
__host__ __device__ __forceinline__ int split_hi(int m, int n) { return (ADV == 3 && m == n) ? 0 : 1; }

// u-face (i, j, k), 1 <= i <= nx+1
template <typename R, int ADV>
__host__ __device__ __forceinline__ R split_form_u(const FaceTaps<R>& T, const double* u, const double* v,
                                                   const double* w, int i, int j, int k, int nx, R idx, R idy,
                                                   R idz) {
    // v and w averaged to the u-face shifted by (0, dj, dk)
    auto bma = [&](int dj) { return (T(v, 0, dj, 0) + T(v, -1, dj, 0) + T(v, 0, dj + 1, 0) + T(v, -1, dj + 1, 0)) * R(0.25); };
    auto dma = [&](int dk) { return (T(w, 0, 0, dk) + T(w, -1, 0, dk) + T(w, 0, 0, dk + 1) + T(w, -1, 0, dk + 1)) * R(0.25); };
    const R um = T(u, -1, 0, 0), u0 = T(u, 0, 0, 0), up = T(u, 1, 0, 0);
    const R tx = split_term<R, ADV>(um, u0, up, T(u, split_lo<ADV>(i), 0, 0), u0,
                                    T(u, split_hi<ADV>(i, nx + 1), 0, 0), idx);
    const R ty = split_term<R, ADV>(T(u, 0, -1, 0), u0, T(u, 0, 1, 0), bma(split_lo<ADV>(j)), bma(0), bma(1), idy);
    const R tz = split_term<R, ADV>(T(u, 0, 0, -1), u0, T(u, 0, 0, 1), dma(split_lo<ADV>(k)), dma(0), dma(1), idz);
    return tx + ty + tz;
}

// v-face (i, j, k), 1 <= j <= ny+1
template <typename R, int ADV>
__host__ __device__ __forceinline__ R split_form_v(const FaceTaps<R>& T, const double* u, const double* v,
                                                   const double* w, int i, int j, int k, int ny, R idx, R idy,
                                                   R idz) {
    auto amb = [&](int di) { return (T(u, di, 0, 0) + T(u, di + 1, 0, 0) + T(u, di, -1, 0) + T(u, di + 1, -1, 0)) * R(0.25); };
    auto dmb = [&](int dk) { return (T(w, 0, 0, dk) + T(w, 0, -1, dk) + T(w, 0, 0, dk + 1) + T(w, 0, -1, dk + 1)) * R(0.25); };
    const R v0 = T(v, 0, 0, 0);
    const R tx = split_term<R, ADV>(T(v, -1, 0, 0), v0, T(v, 1, 0, 0), amb(split_lo<ADV>(i)), amb(0), amb(1), idx);
    const R ty = split_term<R, ADV>(T(v, 0, -1, 0), v0, T(v, 0, 1, 0), T(v, 0, split_lo<ADV>(j), 0), v0,
                                    T(v, 0, split_hi<ADV>(j, ny + 1), 0), idy);
    const R tz = split_term<R, ADV>(T(v, 0, 0, -1), v0, T(v, 0, 0, 1), dmb(split_lo<ADV>(k)), dmb(0), dmb(1), idz);
    return tx + ty + tz;
}

// w-face (i, j, k), 1 <= k <= nz+1
template <typename R, int ADV>
__host__ __device__ __forceinline__ R split_form_w(const FaceTaps<R>& T, const double* u, const double* v,
                                                   const double* w, int i, int j, int k, int nz, R idx, R idy,
                                                   R idz) {
    auto amd = [&](int di) { return (T(u, di, 0, 0) + T(u, di + 1, 0, 0) + T(u, di, 0, -1) + T(u, di + 1, 0, -1)) * R(0.25); };
    auto bmd = [&](int dj) { return (T(v, 0, dj, 0) + T(v, 0, dj + 1, 0) + T(v, 0, dj, -1) + T(v, 0, dj + 1, -1)) * R(0.25); };
    const R w0 = T(w, 0, 0, 0);
    const R tx = split_term<R, ADV>(T(w, -1, 0, 0), w0, T(w, 1, 0, 0), amd(split_lo<ADV>(i)), amd(0), amd(1), idx);
    const R ty = split_term<R, ADV>(T(w, 0, -1, 0), w0, T(w, 0, 1, 0), bmd(split_lo<ADV>(j)), bmd(0), bmd(1), idy);
    const R tz = split_term<R, ADV>(T(w, 0, 0, -1), w0, T(w, 0, 0, 1), T(w, 0, 0, split_lo<ADV>(k)), w0,
                                    T(w, 0, 0, split_hi<ADV>(k, nz + 1)), idz);
    return tx + ty + tz;
}

}  // namespace suli
