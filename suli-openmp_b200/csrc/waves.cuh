// waves.cuh — wave inflow at x = 0: wave_t = 1 Stokes I, 2 Stokes II, 5 Stokes V.
//
// wave_coefficients() is waves_coef (3_contorno.f90:1084-1205), run once on the host: the
// wavelength from the dispersion relation (fixed-point iteration for Stokes I/II; for Stokes V
// a scan of 10000 wavelengths for the one where the two conditions on the parameter lamb
// agree), then the Stokes V elevation and velocity amplitudes.  wave_point() is the per-point
// part of boundary_waves (:952-1082): elevation h_f(i), the distance h_f(i) - kp(k) rounded to
// single precision (the reference keeps it in a real(4) array), and u, w where that distance
// is not negative.
#pragma once
#include <cmath>

namespace suli {

struct WaveCoef {
    int type = 0;
    double a_w = 0, p_w = 0, h0_f = 0, l0_w = 0, l_w = 0, c_w = 0, f_w = 0, n_w = 0;
    double aeta[6] = {0, 0, 0, 0, 0, 0}, avel[6] = {0, 0, 0, 0, 0, 0};   // [1..5]
    double tanh_h = 0, sinh_h = 0;                                      // tanh, sinh of n_w h0_f
};

inline WaveCoef wave_coefficients(int wave_t, double gz) {
    WaveCoef W;
    const double pi = std::acos(-1.);
    W.type = wave_t;
    W.a_w = 0.03; W.p_w = 2.5; W.h0_f = 1.;     // amplitude, period, still depth
    W.l0_w = gz * W.p_w * W.p_w / (2. * pi);
    if (wave_t <= 2) {
        W.l_w = gz * W.p_w * W.p_w / (2. * pi);
        for (int i = 1; i <= 1000; ++i) W.l_w = gz * W.p_w * W.p_w / (2. * pi) * std::tanh(2. * pi * W.h0_f / W.l_w);
    } else {
        auto pw = [](double x, double e) { return std::pow(x, e); };
        double s = 0, c = 0, b33 = 0, b35 = 0, b55 = 0, c1 = 0, c2 = 0;
        auto coefs = [&](double lw) {
            s = std::sinh(2. * pi * W.h0_f / lw);
            c = std::cosh(2. * pi * W.h0_f / lw);
            b33 = 3. * (8. * pw(c, 6.) + 1.) / (64. * pw(s, 6.));
            b35 = (88128. * pw(c, 14.) - 208224. * pw(c, 12) + 70848. * pw(c, 10.) + 54000. * pw(c, 8.) - 21816. * pw(c, 6.) +
                   6264. * pw(c, 4.) - 54. * c * c - 81.) / (12288. * pw(s, 12.) * (6. * c * c - 1.));
            b55 = (192000. * pw(c, 16.) - 262720. * pw(c, 14.) + 83680. * pw(c, 12) + 20160. * pw(c, 10.) - 7280. * pw(c, 8.) +
                   7160. * pw(c, 6.) - 1800. * pw(c, 4.) - 1050. * c * c + 225.) /
                  (12288 * pw(s, 10.) * (6. * c * c - 1.) * (8. * pw(c, 4.) - 11. * c * c + 3.));
            c1 = (8. * pw(c, 4.) - 8. * c * c + 9.) / (8. * pw(s, 4.));
            c2 = (3840. * pw(c, 12.) - 4096. * pw(c, 10.) + 2592. * pw(c, 8.) - 1008. * pw(c, 6.) + 5944. * pw(c, 4.) -
                  1830. * c * c + 147.) / (512. * pw(s, 10.) * (6. * c * c - 1.));
        };
        double erro0 = 999., lamb = 0.;
        const int nxii = 10000;
        for (int ii = 1; ii <= nxii; ++ii) {
            double lamb1 = 0., lamb2 = 0.;
            const double l_w1 = W.l0_w * 0.5 + W.l0_w * ((double)ii / nxii) * 2.5;
            coefs(l_w1);
            for (int i = 1; i <= 10000; ++i) lamb1 = pi * W.a_w * 2. / l_w1 - pw(lamb1, 3.) * b33 - pw(lamb1, 5.) * (b35 + b55);
            for (int i = 1; i <= 10000; ++i)
                lamb2 = std::sqrt((l_w1 / (W.l0_w * std::tanh(2. * pi * W.h0_f / l_w1)) - 1.) / (c1 + pw(lamb2, 2.) * c2));
            const double erro = std::fabs(lamb1 - lamb2);
            if (erro < erro0) { erro0 = erro; lamb = lamb1; W.l_w = l_w1; }
        }
        const double n_w = 2. * pi / W.l_w, p_w = W.p_w;
        coefs(W.l_w);
        const double a11 = 1. / s;
        const double a13 = -c * c * (5. * c * c + 1.) / (8. * pw(s, 5.));
        const double a15 = -(1184. * pw(c, 10.) - 1440. * pw(c, 8.) - 1992. * pw(c, 6.) + 2641. * pw(c, 4.) - 249. * pw(c, 2.) + 18.) /
                           (1536. * pw(s, 11.));
        const double a22 = 3. / (8. * pw(s, 4.));
        const double a24 = (192. * pw(c, 8.) - 424. * pw(c, 6.) - 312. * pw(c, 4.) + 480. * c * c - 17.) / (768. * pw(s, 10.));
        const double a33 = (13. - 4. * c * c) / (64. * pw(s, 7.));
        const double a35 = (512. * pw(c, 12.) + 4224. * pw(c, 10.) - 6800. * pw(c, 8.) - 12808. * pw(c, 6.) + 16704. * pw(c, 4.) -
                            3154. * c * c + 107.) / (4096. * pw(s, 13.) * (6. * c * c - 1.));
        const double a44 = (80. * pw(c, 6.) - 816. * pw(c, 4.) + 1338. * c * c - 197.) / (1536. * pw(s, 10.) * (6. * c * c - 1.));
        const double a55 = -(2880. * pw(c, 10.) - 72480. * pw(c, 8.) + 324000. * pw(c, 6.) - 432000. * pw(c, 4.) + 163470. * c * c -
                             16245.) / (61440. * pw(s, 11.) * (6. * c * c - 1.) * (8. * pw(c, 4.) - 11. * c * c + 3.));
        const double b22 = c * (2. * c * c + 1.) / (4. * pw(s, 3.));
        const double b24 = c * (272. * pw(c, 8.) - 504. * pw(c, 6.) - 192. * pw(c, 4.) + 322 * c * c + 21.) / (384. * pw(s, 9.));
        const double b44 = c * (768. * pw(c, 10.) - 448. * pw(c, 8.) - 48. * pw(c, 6.) + 48. * pw(c, 4.) + 106. * c * c - 21.) /
                           (384. * pw(s, 9.) * (6. * c * c - 1.));
        W.aeta[1] = lamb / n_w;
        W.aeta[2] = (lamb * lamb * b22 + pw(lamb, 4.) * b24) / n_w;
        W.aeta[3] = (pw(lamb, 3.) * b33 + pw(lamb, 5.) * b35) / n_w;
        W.aeta[4] = pw(lamb, 4.) * b44 / n_w;
        W.aeta[5] = pw(lamb, 5.) * b55 / n_w;
        W.avel[1] = 1. * 2. * pi / (p_w * n_w) * (lamb * a11 + pw(lamb, 3.) * a13 + pw(lamb, 5.) * a15);
        W.avel[2] = 2. * 2. * pi / (p_w * n_w) * (pw(lamb, 2.) * a22 + pw(lamb, 4.) * a24);
        W.avel[3] = 3. * 2. * pi / (p_w * n_w) * (pw(lamb, 3.) * a33 + pw(lamb, 5.) * a35);
        W.avel[4] = 4. * 2. * pi / (p_w * n_w) * (pw(lamb, 4.) * a44);
        W.avel[5] = 5. * 2. * pi / (p_w * n_w) * (pw(lamb, 5.) * a55);
    }
    W.c_w = W.l_w / W.p_w;
    W.f_w = 2. * pi / W.p_w;
    W.n_w = 2. * pi / W.l_w;
    W.tanh_h = std::tanh(W.n_w * W.h0_f);
    W.sinh_h = std::sinh(W.n_w * W.h0_f);
    return W;
}

struct WavePoint {
    float ls;       // h_f(i) - kp(k) in single precision
    double u, w;    // u at the face (i, k), w at the face below the cell centre (i, k)
};

// boundary_waves at column i (0 or 1) and height index k (0..nz+1), time t
__host__ __device__ inline WavePoint wave_point(const WaveCoef& W, int i, int k, double dx, double dz, double t) {
    const double kp = (k - 0.5) * dz;
    const double n_w = W.n_w, f_w = W.f_w, a_w = W.a_w, h0_f = W.h0_f, shh = W.sinh_h, th = W.tanh_h;
    const double aux2 = n_w * dx * (i - 0.5) - f_w * t;   // phase of eta and w
    const double aux3 = n_w * dx * (i - 1.) - f_w * t;    // phase of u
    double hf;
    if (W.type == 1) {
        hf = h0_f + a_w * cos(aux2);
    } else if (W.type == 2) {
        hf = h0_f + a_w * cos(aux2) + n_w * a_w * a_w * (3. - th * th) / (4. * th * th * th) * cos(2. * aux2);
    } else {
        hf = h0_f + W.aeta[1] * cos(aux2) + W.aeta[2] * cos(2. * aux2) + W.aeta[3] * cos(3. * aux2) +
             W.aeta[4] * cos(4. * aux2) + W.aeta[5] * cos(5. * aux2);
    }
    WavePoint P;
    P.ls = (float)(hf - kp);
    P.u = 0.;
    P.w = 0.;
    if (P.ls >= 0.f) {
        if (W.type == 1) {
            P.u = a_w * f_w * cosh(n_w * kp) / shh * cos(aux3);
            P.w = a_w * f_w * sinh(n_w * (kp - 0.5 * dz)) / shh * sin(aux2);
        } else if (W.type == 2) {
            const double sh4 = pow(shh, 4.);
            P.u = a_w * f_w * cosh(n_w * kp) / shh * cos(aux3) + 3. / 4. * a_w * a_w * f_w * n_w * cosh(2. * n_w * kp) / sh4 * cos(2 * aux3);
            P.w = a_w * f_w * sinh(n_w * (kp - 0.5 * dz)) / shh * sin(aux2) +
                  3. / 4. * a_w * a_w * f_w * n_w * sinh(2. * n_w * (kp - 0.5 * dz)) / sh4 * sin(2. * aux3);
        } else {
            const double aux4 = n_w * kp, aux5 = n_w * (kp - 0.5 * dz);
            P.u = W.avel[1] * cosh(aux4) * cos(aux3) + W.avel[2] * cosh(2 * aux4) * cos(2 * aux3) +
                  W.avel[3] * cosh(3 * aux4) * cos(3 * aux3) + W.avel[4] * cosh(4 * aux4) * cos(4 * aux3) +
                  W.avel[5] * cosh(5 * aux4) * cos(5 * aux3);
            P.w = W.avel[1] * sinh(aux5) * sin(aux2) + W.avel[2] * sinh(2 * aux5) * sin(2 * aux2) +
                  W.avel[3] * sinh(3 * aux5) * sin(3 * aux2) + W.avel[4] * sinh(4 * aux5) * sin(4 * aux2) +
                  W.avel[5] * sinh(5 * aux5) * sin(5 * aux2);
        }
    }
    return P;
}

}  // namespace suli
