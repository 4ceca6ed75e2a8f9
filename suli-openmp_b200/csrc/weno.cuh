// weno.cuh — fifth-order WENO one-sided derivatives (Jiang–Shu) of a cell field along one
// axis, as the reference's pencil routine weno1 computes them (14_level_set.f90:511-610),
// re-expressed per cell so that a thread needs only the seven values phi(i-3..i+3).
//
// Ghost values outside 1..n are rebuilt from interior values with the pencil routine's own
// rules (ihs, :530-570): 0 periodic with phi(0) = phi(n-1) (the reference's offset),
// 1 one-sided extrapolation (1/5 rows at the low end, 1/11 rows at the high end),
// 2 the 1/11 "zero derivative" rows at both ends.  The arithmetic is the reference's with its
// divisions rearranged: the reciprocal of h formed once on the host, and in FP64 the nonlinear
// weights w_k/q_k^2 / sum_m w_m/q_m^2 formed over a common denominator (one division per side).
#pragma once

namespace suli {

// Fetch phi(m) of a pencil at position m in [i-3, i+3], applying the ghost rules.
// `at(m)` returns the stored interior value for m in 1..n.
template <typename T, typename F>
__device__ __forceinline__ void pencil7(F at, int i, int n, int ihs, T P[7]) {
    if (i >= 4 && i <= n - 3) {
#pragma unroll
        for (int m = 0; m < 7; ++m) P[m] = at(i - 3 + m);
        return;
    }
    // boundary neighbourhood: build the ghosts the reference builds for the whole pencil
    T g_lo[3], g_hi[3];   // g_lo[0] = phi(0), g_lo[1] = phi(-1), g_lo[2] = phi(-2); g_hi[0] = phi(n+1) ...
    if (ihs == 0) {
        g_lo[0] = at(n - 1); g_lo[1] = at(n - 2); g_lo[2] = at(n - 3);
        g_hi[0] = at(2); g_hi[1] = at(3); g_hi[2] = at(4);
    } else {
        const T p1 = at(1), p2 = at(2), p3 = at(3);
        const T qn = at(n), qn1 = at(n - 1), qn2 = at(n - 2);
        if (ihs == 1) {
            g_lo[0] = T(1. / 5.) * (T(12.) * p1 - T(9.) * p2 + T(2.) * p3);
            g_lo[1] = T(1. / 5.) * (T(12.) * g_lo[0] - T(9.) * p1 + T(2.) * p2);
            g_lo[2] = T(1. / 5.) * (T(12.) * g_lo[1] - T(9.) * g_lo[0] + T(2.) * p1);
        } else {
            g_lo[0] = T(1. / 11.) * (T(18.) * p1 - T(9.) * p2 + T(2.) * p3);
            g_lo[1] = T(1. / 11.) * (T(18.) * g_lo[0] - T(9.) * p1 + T(2.) * p2);
            g_lo[2] = T(1. / 11.) * (T(18.) * g_lo[1] - T(9.) * g_lo[0] + T(2.) * p1);
        }
        g_hi[0] = T(1. / 11.) * (T(18.) * qn - T(9.) * qn1 + T(2.) * qn2);
        g_hi[1] = T(1. / 11.) * (T(18.) * g_hi[0] - T(9.) * qn + T(2.) * qn1);
        g_hi[2] = T(1. / 11.) * (T(18.) * g_hi[1] - T(9.) * g_hi[0] + T(2.) * qn);
    }
#pragma unroll
    for (int m = 0; m < 7; ++m) {
        const int q = i - 3 + m;
        T val;
        if (q < 1) val = g_lo[-q];
        else if (q > n) val = g_hi[q - n - 1];
        else val = at(q);
        P[m] = val;
    }
}

// omega_k = (w_k/q_k^2) / sum_m (w_m/q_m^2), q_k = eps + is_k.  FP64: over the common
// denominator q_1^2 q_2^2 q_3^2 (q >= eps = 1e-8, so the products stay far inside the FP64
// range); FP32 (the mixed path's arithmetic, where that product can underflow): the three
// quotients and one reciprocal of their sum, each with the hardware reciprocal (__fdividef, 2
// ulp; q^2 stays far below the 2^126 where it would flush), since IEEE FP32 divisions were a
// third of the WENO kernels' instructions.
template <typename T>
__device__ __forceinline__ void nonlinear_weights(T is1, T is2, T is3, T eps, T w1, T w2, T w3, T& o1, T& o2,
                                                  T& o3) {
    const T a = (eps + is1) * (eps + is1), b = (eps + is2) * (eps + is2), c = (eps + is3) * (eps + is3);
    if constexpr (sizeof(T) == 8) {
        const T n1 = w1 * (b * c), n2 = w2 * (a * c), n3 = w3 * (a * b);
        const T inv = T(1) / (n1 + n2 + n3);
        o1 = n1 * inv; o2 = n2 * inv; o3 = n3 * inv;
    } else {
        const T al1 = __fdividef(w1, a), al2 = __fdividef(w2, b), al3 = __fdividef(w3, c);
        const T inv = __fdividef(T(1), al1 + al2 + al3);
        o1 = al1 * inv; o2 = al2 * inv; o3 = al3 * inv;
    }
}

// One-sided derivatives from the seven values P[0..6] = phi(i-3..i+3) and ih = 1/h (formed
// once on the host, in the compute type): dp = phi_x^+ (dphidxp, right-biased), dn = phi_x^-
// (dphidxn, left-biased).
template <typename T>
__device__ __forceinline__ void weno_pair(const T P[7], T ih, T& dp, T& dn) {
    // D[m] = (phi(i-2+m) - phi(i-3+m))/h; up(i-4..i) = D1..D5, un(i..i+4) = D0..D4
    T D[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) D[m] = (P[m + 1] - P[m]) * ih;
    const T aux1 = T(13. / 12.), aux2 = T(1. / 4.), aux3 = T(1. / 6.), aux6 = T(0.00000001);
    const T w1 = T(0.1), w2 = T(0.6), w3 = T(0.3);
    // right-biased: up(i)=D5, up(i-1)=D4, up(i-2)=D3, up(i-3)=D2, up(i-4)=D1
    {
        const T u0 = D[5], u1 = D[4], u2 = D[3], u3 = D[2], u4 = D[1];
        T a, b;
        a = u0 - 2 * u1 + u2; b = u0 - 4 * u1 + 3 * u2;
        const T is1 = aux1 * a * a + aux2 * b * b;
        a = u1 - 2 * u2 + u3; b = u1 - u3;
        const T is2 = aux1 * a * a + aux2 * b * b;
        a = u2 - 2 * u3 + u4; b = 3 * u2 - 4 * u3 + u4;
        const T is3 = aux1 * a * a + aux2 * b * b;
        T o1, o2, o3;
        nonlinear_weights(is1, is2, is3, aux6, w1, w2, w3, o1, o2, o3);
        dp = aux3 * (o1 * (2 * u0 - 7 * u1 + 11 * u2) + o2 * (-u1 + 5 * u2 + 2 * u3) +
                     o3 * (2 * u2 + 5 * u3 - u4));
    }
    // left-biased: un(i)=D0, un(i+1)=D1, un(i+2)=D2, un(i+3)=D3, un(i+4)=D4
    {
        const T v0 = D[0], v1 = D[1], v2 = D[2], v3 = D[3], v4 = D[4];
        T a, b;
        a = v0 - 2 * v1 + v2; b = v0 - 4 * v1 + 3 * v2;
        const T is1 = aux1 * a * a + aux2 * b * b;
        a = v1 - 2 * v2 + v3; b = v1 - v3;
        const T is2 = aux1 * a * a + aux2 * b * b;
        a = v2 - 2 * v3 + v4; b = 3 * v2 - 4 * v3 + v4;
        const T is3 = aux1 * a * a + aux2 * b * b;
        T o1, o2, o3;
        nonlinear_weights(is1, is2, is3, aux6, w1, w2, w3, o1, o2, o3);
        dn = aux3 * (o1 * (2 * v0 - 7 * v1 + 11 * v2) + o2 * (-v1 + 5 * v2 + 2 * v3) +
                     o3 * (2 * v2 + 5 * v3 - v4));
    }
}

}  // namespace suli
