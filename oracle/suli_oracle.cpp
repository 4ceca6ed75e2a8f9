/*
 * suli_oracle.cpp — CPU restatement (FP64) of the SuLi-IC per-time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The product path
 * (libsuli_gpu.so) never links or calls it.
 *
 * PARITY UNPINNED: the reference (lacia-udesc/SuLi-OpenMP, SuLi-IC/) is Fortran 90 and no
 * Fortran compiler exists where this was written, so the reference could not be run to
 * produce golden outputs, and it ships no tests or expected values.  This restatement
 * follows the reference routine by routine (citations below, paths relative to SuLi-IC/),
 * keeping its array extents, loop order, expression order and quirks, and is checked by
 * analytic known answers in tests/ (manufactured fields, exactness of the stencils on
 * polynomials, invariants).
 *
 * Floating point: every literal of the reference is double (-fdefault-real-8,
 * Makefile:7).  Build with -O2 -ffp-contract=off (no FMA contraction, no fast-math) so the
 * order of operations written here is the order executed.  Built twice: serially (the
 * checker: reductions in the reference's serial order) and with -fopenmp (the timed CPU
 * baseline; parallel reductions, labelled as such).
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/suli_gpu.h"

#ifdef _OPENMP
#define OMP_FOR _Pragma("omp parallel for collapse(2) schedule(static)")
#else
#define OMP_FOR
#endif

namespace {

/* Fortran array with inclusive bounds lo..hi in each dimension, column-major. */
struct Arr {
    int lo[3] = {0, 0, 0}, hi[3] = {-1, -1, -1};
    long s1 = 0, s2 = 0;
    std::vector<double> a;
    void init(int l0, int h0, int l1, int h1, int l2, int h2) {
        lo[0] = l0; hi[0] = h0; lo[1] = l1; hi[1] = h1; lo[2] = l2; hi[2] = h2;
        s1 = h0 - l0 + 1; s2 = s1 * (h1 - l1 + 1);
        a.assign((size_t)(s2 * (h2 - l2 + 1)), 0.0);
    }
    inline double& operator()(int i, int j, int k) {
        return a[(size_t)((i - lo[0]) + s1 * (j - lo[1]) + s2 * (k - lo[2]))];
    }
    inline double operator()(int i, int j, int k) const {
        return a[(size_t)((i - lo[0]) + s1 * (j - lo[1]) + s2 * (k - lo[2]))];
    }
    size_t size() const { return a.size(); }
};

/* Fortran MAX/MIN on two doubles (gfortran: a > b ? a : b for MAX). */
static inline double fmax2(double a, double b) { return a > b ? a : b; }
static inline double fmin2(double a, double b) { return a < b ? a : b; }

struct Oracle {
    suli_params P;
    int nx, ny, nz, nx1, ny1, nz1;
    double dx, dy, dz, dx1, pi;
    /* scalars of disc / ls_param */
    double dt, t, dt1, vol_ini, vol_ins;
    int ntt;
    double a_dt[3];
    double adtl[3], bdtl[3], gdtl[3];
    /* fields (0_modules.f90) */
    Arr u, v, w, ub, vb, wb, prd1, prd0, prd, rho, ls_nu;
    Arr Fu, u0, fu0, fu1, Fv, v0, fv0, fv1, Fw, w0, fw0, fw1;
    Arr nut, xnut, ynut, znut;
    Arr ls, mod_ls, kurv, hs, ddlsdx, ddlsdy, ddlsdz, hsx, hsy, hsz;
    Arr tf_u, tf_v, tf_w;
    Arr bxx0, bxx1, bxy0, bxz0, bxxf, bxxf1, bxyf, bxzf;
    Arr byx0, byy0, byy1, byz0, byxf, byyf, byyf1, byzf;
    Arr bzx0, bzy0, bzz0, bzz1, bzxf, bzyf, bzzf, bzzf1;
    /* obstacle masks (0_modules.f90:76-79): ku(0:nx1+1,0:ny+1), kv(0:nx+1,0:ny1+1),
       kw(0:nx+1,0:ny+1), the k up to which a column's velocity is zeroed */
    std::vector<int> ku, kv, kw;
    bool has_obstacle = false;
    int KU(int i, int j) const { return ku[(size_t)i + (size_t)(nx + 3) * j]; }
    int KV(int i, int j) const { return kv[(size_t)i + (size_t)(nx + 2) * j]; }
    int KW(int i, int j) const { return kw[(size_t)i + (size_t)(nx + 2) * j]; }
    void contorno_obstacle();
    void level_set_obstacle();
    void outflow_fix();
    void wrap_faces(Arr& rx, Arr& ry, Arr& rz) const;
    /* wave inflow (module wave_c, 0_modules.f90:164-174) */
    double p_w = 0, n_w = 0, c_w = 0, l_w = 0, a_w = 0, f_w = 0, h0_f = 0, l0_w = 0;
    double avel[6] = {0}, aeta[6] = {0};   /* avel1..5, aeta1..5 at [1..5] */
    std::vector<double> kp;                /* kp(0:nz+1) */
    void waves_coef();
    void boundary_waves();
    /* statistics of the last calls */
    int last_cg_iters = 0;
    double last_cg_resid = 0.0;
    double last_cg_rmax = 0.0;
    int last_reinit_iters = 0;
    int last_volfix_iters = 0;

    Arr* field(int id);
    void alloc();

    /* routines */
    void weno1(double* dp, double* dn, int n, double h, const double* phi0, int ihs) const;
    void der_weno(const Arr& f, Arr& ta1, Arr& tb1, Arr& tc1, Arr& td1, Arr& te1, Arr& tf1, int& ihs) const;
    void conv_weno(Arr& sy7);
    void intt_ls(const Arr& hx, Arr& gx, Arr& ta1, int itrl, Arr& ls1);
    void reinic_weno();
    void heaviside();
    void mod_ls1();
    double volume() const;
    void level_set();
    void visco();
    void classico(Arr& uint_, Arr& vint, Arr& wint);
    void rotacional(Arr& uint_, Arr& vint, Arr& wint);
    void antissim(Arr& uint_, Arr& vint, Arr& wint);
    void convdiff();
    void tempo(int tt, int it);
    void contorno(int nlock);
    int graddin();
    void posdin();
    double est() const;
    void cell(Arr& a) { a.init(1, nx, 1, ny, 1, nz); }
};

void Oracle::alloc() {
    nx = P.nx; ny = P.ny; nz = P.nz; nx1 = nx + 1; ny1 = ny + 1; nz1 = nz + 1;
    dx = P.dx; dy = P.dy; dz = P.dz;
    dx1 = std::max(dx, std::max(dy, dz));       /* 0_modules.f90:197 */
    pi = std::acos(-1.0);                        /* 0_modules.f90:4 */
    u.init(0, nx1 + 1, 0, ny + 1, 0, nz + 1);    /* 0_modules.f90:92 */
    v.init(0, nx + 1, 0, ny1 + 1, 0, nz + 1);    /* :93 */
    w.init(0, nx + 1, 0, ny + 1, 0, nz1 + 1);    /* :94 */
    ub.init(0, nx1 + 1, 0, ny + 1, 0, nz + 1);   /* :71-73 */
    vb.init(0, nx + 1, 0, ny1 + 1, 0, nz + 1);
    wb.init(0, nx + 1, 0, ny + 1, 0, nz1 + 1);
    prd1.init(0, nx + 1, 0, ny + 1, 0, nz + 1);  /* :121 */
    prd0.init(0, nx + 1, 0, ny + 1, 0, nz + 1);
    prd.init(0, nx + 1, 0, ny + 1, 0, nz + 1);
    cell(rho); cell(ls_nu);
    Fu.init(1, nx1, 1, ny, 1, nz); u0 = Fu; fu0 = Fu; fu1 = Fu;   /* :131-133 */
    Fv.init(1, nx, 1, ny1, 1, nz); v0 = Fv; fv0 = Fv; fv1 = Fv;
    Fw.init(1, nx, 1, ny, 1, nz1); w0 = Fw; fw0 = Fw; fw1 = Fw;
    cell(nut); xnut = Fu; ynut = Fv; znut = Fw;                   /* :182-185 */
    cell(ls); cell(mod_ls); cell(kurv); cell(hs); cell(ddlsdx); cell(ddlsdy); cell(ddlsdz);
    cell(hsx); cell(hsy); cell(hsz);
    tf_u = Fu; tf_v = Fv; tf_w = Fw;
    bxx0.init(0, ny + 1, 0, nz + 1, 0, 0); bxx1 = bxx0; bxxf = bxx0; bxxf1 = bxx0;   /* :96-118 */
    bxy0.init(0, ny1 + 1, 0, nz + 1, 0, 0); bxyf = bxy0;
    bxz0.init(0, ny + 1, 0, nz1 + 1, 0, 0); bxzf = bxz0;
    byx0.init(0, nx1 + 1, 0, nz + 1, 0, 0); byxf = byx0;
    byy0.init(0, nx + 1, 0, nz + 1, 0, 0); byy1 = byy0; byyf = byy0; byyf1 = byy0;
    byz0.init(0, nx + 1, 0, nz1 + 1, 0, 0); byzf = byz0;
    bzx0.init(0, nx1 + 1, 0, ny + 1, 0, 0); bzxf = bzx0;
    bzy0.init(0, nx + 1, 0, ny1 + 1, 0, 0); bzyf = bzy0;
    bzz0.init(0, nx + 1, 0, ny + 1, 0, 0); bzz1 = bzz0; bzzf = bzz0; bzzf1 = bzz0;
    /* TVD-RK3 coefficients, 14_level_set.f90:34-44 */
    adtl[0] = 1.;      bdtl[0] = 0.;      gdtl[0] = 1.;
    adtl[1] = 3. / 4.; bdtl[1] = 1. / 4.; gdtl[1] = 1. / 4.;
    adtl[2] = 1. / 3.; bdtl[2] = 2. / 3.; gdtl[2] = 2. / 3.;
    dt = P.dt; t = 0.; dt1 = P.dt1; vol_ini = 0.; vol_ins = 0.;
    ntt = 1; a_dt[0] = a_dt[1] = a_dt[2] = P.dt;
}

Arr* Oracle::field(int id) {
    switch (id) {
    case SULI_F_U: return &u; case SULI_F_V: return &v; case SULI_F_W: return &w;
    case SULI_F_PRD1: return &prd1; case SULI_F_PRD0: return &prd0; case SULI_F_PRD: return &prd;
    case SULI_F_RHO: return &rho; case SULI_F_LS_NU: return &ls_nu;
    case SULI_F_FU: return &Fu; case SULI_F_U0: return &u0; case SULI_F_FU0: return &fu0; case SULI_F_FU1: return &fu1;
    case SULI_F_FV: return &Fv; case SULI_F_V0: return &v0; case SULI_F_FV0: return &fv0; case SULI_F_FV1: return &fv1;
    case SULI_F_FW: return &Fw; case SULI_F_W0: return &w0; case SULI_F_FW0: return &fw0; case SULI_F_FW1: return &fw1;
    case SULI_F_NUT: return &nut; case SULI_F_XNUT: return &xnut; case SULI_F_YNUT: return &ynut; case SULI_F_ZNUT: return &znut;
    case SULI_F_LS: return &ls; case SULI_F_MOD_LS: return &mod_ls; case SULI_F_KURV: return &kurv; case SULI_F_HS: return &hs;
    case SULI_F_DDLSDX: return &ddlsdx; case SULI_F_DDLSDY: return &ddlsdy; case SULI_F_DDLSDZ: return &ddlsdz;
    case SULI_F_HSX: return &hsx; case SULI_F_HSY: return &hsy; case SULI_F_HSZ: return &hsz;
    case SULI_F_UB: return &ub; case SULI_F_VB: return &vb; case SULI_F_WB: return &wb;
    case SULI_F_TF_U: return &tf_u; case SULI_F_TF_V: return &tf_v; case SULI_F_TF_W: return &tf_w;
    case SULI_F_BXX0: return &bxx0; case SULI_F_BXX1: return &bxx1; case SULI_F_BXY0: return &bxy0; case SULI_F_BXZ0: return &bxz0;
    case SULI_F_BXXF: return &bxxf; case SULI_F_BXXF1: return &bxxf1; case SULI_F_BXYF: return &bxyf; case SULI_F_BXZF: return &bxzf;
    case SULI_F_BYX0: return &byx0; case SULI_F_BYY0: return &byy0; case SULI_F_BYY1: return &byy1; case SULI_F_BYZ0: return &byz0;
    case SULI_F_BYXF: return &byxf; case SULI_F_BYYF: return &byyf; case SULI_F_BYYF1: return &byyf1; case SULI_F_BYZF: return &byzf;
    case SULI_F_BZX0: return &bzx0; case SULI_F_BZY0: return &bzy0; case SULI_F_BZZ0: return &bzz0; case SULI_F_BZZ1: return &bzz1;
    case SULI_F_BZXF: return &bzxf; case SULI_F_BZYF: return &bzyf; case SULI_F_BZZF: return &bzzf; case SULI_F_BZZF1: return &bzzf1;
    default: return nullptr;
    }
}

/* ---------------------------------------------------------------------------------------
 * weno1 — 14_level_set.f90:511-610.  phi0[0..n-1] = phi0(1..n); outputs dp = dphidxp
 * (right-biased, phi_x^+) and dn = dphidxn (left-biased, phi_x^-).  Ghosts by ihs:
 * 0 periodic with the reference's off-by-one (phi(0) = phi(n-1), :533-540), 1 one-sided
 * extrapolation with the asymmetric 1/5 and 1/11 rows (:548-556), 2 "zero derivative"
 * extrapolation (:564-569).
 * ------------------------------------------------------------------------------------- */
void Oracle::weno1(double* dp, double* dn, int n, double h, const double* phi0, int ihs) const {
    std::vector<double> ph((size_t)n + 6), upv((size_t)n + 4), unv((size_t)n + 4);
    auto P_ = [&](int i) -> double& { return ph[(size_t)(i + 2)]; };     /* phi1(-2:n+3) */
    auto UP = [&](int i) -> double& { return upv[(size_t)(i + 3)]; };    /* up(-3:n)     */
    auto UN = [&](int i) -> double& { return unv[(size_t)(i - 1)]; };    /* un(1:n+4)    */
    const double aux1 = 13. / 12., aux2 = 1. / 4., aux3 = 1. / 6.;
    const double auxx[3] = {0.1, 0.6, 0.3};
    const double aux6 = 0.00000001;
    for (int i = 1; i <= n; ++i) P_(i) = phi0[i - 1];
    if (ihs == 0) {
        P_(0) = P_(n - 1); P_(-1) = P_(n - 2); P_(-2) = P_(n - 3);
        P_(n + 1) = P_(2); P_(n + 2) = P_(3); P_(n + 3) = P_(4);
    } else if (ihs == 1) {
        P_(0)  = 1. / 5. * (12. * P_(1)  - 9. * P_(2) + 2. * P_(3));
        P_(-1) = 1. / 5. * (12. * P_(0)  - 9. * P_(1) + 2. * P_(2));
        P_(-2) = 1. / 5. * (12. * P_(-1) - 9. * P_(0) + 2. * P_(1));
        P_(n + 1) = 1. / 11. * (18. * P_(n)     - 9. * P_(n - 1) + 2. * P_(n - 2));
        P_(n + 2) = 1. / 11. * (18. * P_(n + 1) - 9. * P_(n)     + 2. * P_(n - 1));
        P_(n + 3) = 1. / 11. * (18. * P_(n + 2) - 9. * P_(n + 1) + 2. * P_(n));
    } else if (ihs == 2) {
        P_(0)  = 1. / 11. * (18. * P_(1)  - 9. * P_(2) + 2. * P_(3));
        P_(-1) = 1. / 11. * (18. * P_(0)  - 9. * P_(1) + 2. * P_(2));
        P_(-2) = 1. / 11. * (18. * P_(-1) - 9. * P_(0) + 2. * P_(1));
        P_(n + 1) = 1. / 11. * (18. * P_(n)     - 9. * P_(n - 1) + 2. * P_(n - 2));
        P_(n + 2) = 1. / 11. * (18. * P_(n + 1) - 9. * P_(n)     + 2. * P_(n - 1));
        P_(n + 3) = 1. / 11. * (18. * P_(n + 2) - 9. * P_(n + 1) + 2. * P_(n));
    }
    for (int i = -3; i <= n; ++i) UP(i) = (P_(i + 3) - P_(i + 2)) / h;
    for (int i = 1; i <= n + 4; ++i) UN(i) = (P_(i - 2) - P_(i - 3)) / h;
    for (int i = 1; i <= n; ++i) {
        double isup[3], isun[3], alpup[3], alpun[3];
        double a, b;
        a = UP(i) - 2 * UP(i - 1) + UP(i - 2); b = UP(i) - 4 * UP(i - 1) + 3 * UP(i - 2);
        isup[0] = aux1 * a * a + aux2 * b * b;
        a = UN(i) - 2 * UN(i + 1) + UN(i + 2); b = UN(i) - 4 * UN(i + 1) + 3 * UN(i + 2);
        isun[0] = aux1 * a * a + aux2 * b * b;
        a = UP(i - 1) - 2 * UP(i - 2) + UP(i - 3); b = UP(i - 1) - UP(i - 3);
        isup[1] = aux1 * a * a + aux2 * b * b;
        a = UN(i + 1) - 2 * UN(i + 2) + UN(i + 3); b = UN(i + 1) - UN(i + 3);
        isun[1] = aux1 * a * a + aux2 * b * b;
        a = UP(i - 2) - 2 * UP(i - 3) + UP(i - 4); b = 3 * UP(i - 2) - 4 * UP(i - 3) + UP(i - 4);
        isup[2] = aux1 * a * a + aux2 * b * b;
        a = UN(i + 2) - 2 * UN(i + 3) + UN(i + 4); b = 3 * UN(i + 2) - 4 * UN(i + 3) + UN(i + 4);
        isun[2] = aux1 * a * a + aux2 * b * b;
        for (int kk = 0; kk < 3; ++kk) {
            alpup[kk] = auxx[kk] / ((aux6 + isup[kk]) * (aux6 + isup[kk]));
            alpun[kk] = auxx[kk] / ((aux6 + isun[kk]) * (aux6 + isun[kk]));
        }
        const double sp = alpup[0] + alpup[1] + alpup[2];
        const double sn = alpun[0] + alpun[1] + alpun[2];
        const double op0 = alpup[0] / sp, op1 = alpup[1] / sp, op2 = alpup[2] / sp;
        const double on0 = alpun[0] / sn, on1 = alpun[1] / sn, on2 = alpun[2] / sn;
        dp[i - 1] = aux3 * (op0 * (2 * UP(i) - 7 * UP(i - 1) + 11 * UP(i - 2)) +
                            op1 * (-UP(i - 1) + 5 * UP(i - 2) + 2 * UP(i - 3)) +
                            op2 * (2 * UP(i - 2) + 5 * UP(i - 3) - UP(i - 4)));
        dn[i - 1] = aux3 * (on0 * (2 * UN(i) - 7 * UN(i + 1) + 11 * UN(i + 2)) +
                            on1 * (-UN(i + 1) + 5 * UN(i + 2) + 2 * UN(i + 3)) +
                            on2 * (2 * UN(i + 2) + 5 * UN(i + 3) - UN(i + 4)));
    }
}

/* der_weno — 14_level_set.f90:343-384.  ihs is an in/out argument: it leaves set to 1,
 * which the callers' later weno1 calls inherit (the mod_ls1 quirk, :717, :763-777).
 * x: periodic if ccx0 = 0 else ihs 2; y likewise with ccy0; z: always 1 (periodic z is an
 * extension of this build, used only when ccz0 = 0). */
void Oracle::der_weno(const Arr& f, Arr& ta1, Arr& tb1, Arr& tc1, Arr& td1, Arr& te1, Arr& tf1,
                      int& ihs) const {
    const int ihx = (P.ccx0 == 0) ? 0 : 2;
    const int ihy = (P.ccy0 == 0) ? 0 : 2;
    const int ihz = (P.ccz0 == 0) ? 0 : 1;
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        std::vector<double> pin((size_t)std::max(nx, std::max(ny, nz))), pp(pin.size()), pn(pin.size());
#ifdef _OPENMP
#pragma omp for collapse(2) schedule(static)
#endif
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j) {
                for (int i = 1; i <= nx; ++i) pin[i - 1] = f(i, j, k);
                weno1(pp.data(), pn.data(), nx, dx, pin.data(), ihx);
                for (int i = 1; i <= nx; ++i) { ta1(i, j, k) = pp[i - 1]; td1(i, j, k) = pn[i - 1]; }
            }
#ifdef _OPENMP
#pragma omp for collapse(2) schedule(static)
#endif
        for (int k = 1; k <= nz; ++k)
            for (int i = 1; i <= nx; ++i) {
                for (int j = 1; j <= ny; ++j) pin[j - 1] = f(i, j, k);
                weno1(pp.data(), pn.data(), ny, dy, pin.data(), ihy);
                for (int j = 1; j <= ny; ++j) { tb1(i, j, k) = pp[j - 1]; te1(i, j, k) = pn[j - 1]; }
            }
#ifdef _OPENMP
#pragma omp for collapse(2) schedule(static)
#endif
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                for (int k = 1; k <= nz; ++k) pin[k - 1] = f(i, j, k);
                weno1(pp.data(), pn.data(), nz, dz, pin.data(), ihz);
                for (int k = 1; k <= nz; ++k) { tc1(i, j, k) = pp[k - 1]; tf1(i, j, k) = pn[k - 1]; }
            }
    }
    ihs = (P.ccz0 == 0) ? 0 : 1;
}

/* conv_weno — 14_level_set.f90:308-341: sy7 = -(u.grad ls) with upwind WENO derivatives
 * and cell-centred velocity averages. */
void Oracle::conv_weno(Arr& sy7) {
    Arr ta1, tb1, tc1, td1, te1, tf1;
    cell(ta1); cell(tb1); cell(tc1); cell(td1); cell(te1); cell(tf1);
    int ihs = 0;
    der_weno(ls, ta1, tb1, tc1, td1, te1, tf1, ihs);
    OMP_FOR
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double apos = fmax2((u(i, j, k) + u(i + 1, j, k)) * 0.5, 0.);
                const double aneg = fmin2((u(i, j, k) + u(i + 1, j, k)) * 0.5, 0.);
                const double bpos = fmax2((v(i, j, k) + v(i, j + 1, k)) * 0.5, 0.);
                const double bneg = fmin2((v(i, j, k) + v(i, j + 1, k)) * 0.5, 0.);
                const double cpos = fmax2((w(i, j, k) + w(i, j, k + 1)) * 0.5, 0.);
                const double cneg = fmin2((w(i, j, k) + w(i, j, k + 1)) * 0.5, 0.);
                sy7(i, j, k) = -(apos * td1(i, j, k) + aneg * ta1(i, j, k) + bpos * te1(i, j, k) +
                                 bneg * tb1(i, j, k) + cpos * tf1(i, j, k) + cneg * tc1(i, j, k));
            }
}

/* intt_ls — 14_level_set.f90:287-306: TVD-RK3 stage, ls1 = a*ta1 + b*gx + g*dt1*hx. */
void Oracle::intt_ls(const Arr& hx, Arr& gx, Arr& ta1, int itrl, Arr& ls1) {
    const double a = adtl[itrl - 1], b = bdtl[itrl - 1], g = gdtl[itrl - 1];
    const bool first = (a == 1.);
    OMP_FOR
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                if (first) ta1(i, j, k) = ls1(i, j, k);
                gx(i, j, k) = ls1(i, j, k);
                ls1(i, j, k) = a * ta1(i, j, k) + b * gx(i, j, k) + g * dt1 * hx(i, j, k);
            }
}

/* Godunov-type one-sided selection of reinic_weno, 14_level_set.f90:406-431. */
static inline void reinit_select(double lsv, double& ta, double& tb, double& tc,
                                 double td, double te, double tf) {
    const double c = 0.00000001;
    if (lsv > 0.) {
        ta = fmax2(fmax2(td, c), -fmin2(ta, c));
        tb = fmax2(fmax2(te, c), -fmin2(tb, c));
        tc = fmax2(fmax2(tf, c), -fmin2(tc, c));
    } else {
        ta = fmax2(fmax2(ta, c), -fmin2(td, c));
        tb = fmax2(fmax2(tb, c), -fmin2(te, c));
        tc = fmax2(fmax2(tc, c), -fmin2(tf, c));
    }
}

/* reinic_weno — 14_level_set.f90:386-509. */
void Oracle::reinic_weno() {
    Arr ta1, tb1, tc1, td1, te1, tf1, func_s, sy7, gx, ta1s, lsaux;
    cell(ta1); cell(tb1); cell(tc1); cell(td1); cell(te1); cell(tf1);
    cell(func_s); cell(sy7); cell(gx); cell(ta1s); cell(lsaux);
    int ihs = 0;
    der_weno(ls, ta1, tb1, tc1, td1, te1, tf1, ihs);
    OMP_FOR
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                double a = ta1(i, j, k), b = tb1(i, j, k), c = tc1(i, j, k);
                reinit_select(ls(i, j, k), a, b, c, td1(i, j, k), te1(i, j, k), tf1(i, j, k));
                const double m = std::sqrt(a * a + b * b + c * c);
                const double l = ls(i, j, k);
                func_s(i, j, k) = l / std::sqrt(l * l + m * m * dx1 * dx1);
            }
    int il = 0;
    double error = 999.;
    while (error > dt1 * dx1 * dx1) {
        il = il + 1;
        for (int itrl = 1; itrl <= 3; ++itrl) {
            der_weno(ls, ta1, tb1, tc1, td1, te1, tf1, ihs);
            OMP_FOR
            for (int k = 1; k <= nz; ++k)
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i) {
                        double a = ta1(i, j, k), b = tb1(i, j, k), c = tc1(i, j, k);
                        reinit_select(ls(i, j, k), a, b, c, td1(i, j, k), te1(i, j, k), tf1(i, j, k));
                        const double m = std::sqrt(a * a + b * b + c * c);
                        sy7(i, j, k) = func_s(i, j, k) * (1. - m);
                        lsaux(i, j, k) = ls(i, j, k);
                    }
            intt_ls(sy7, gx, ta1s, itrl, ls);
        }
        if (il == P.reinit_maxit) {
            error = 0.;
        } else if (il < 1) {
            error = 999.;
        } else {
            /* signed mean change over the band |ls| <= 2*alpha1*dx1 (:492-503), summed in the
               reference's serial order as (error + ls) - lsaux */
            error = 0.;
            long nr = 0;
            const double band = 2. * P.alpha1 * dx1;
            for (int k = 1; k <= nz; ++k)
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i)
                        if (std::fabs(ls(i, j, k)) <= band) {
                            error = error + ls(i, j, k) - lsaux(i, j, k);
                            nr = nr + 1;
                        }
            error = error / (double)nr;   /* nr = 0 gives NaN and ends the loop, as in Fortran */
        }
    }
    last_reinit_iters = il;
}

/* heaviside — 14_level_set.f90:612-707 (t_hs = 0 and 1). */
void Oracle::heaviside() {
    Arr ta1, tb1, tc1, td1, te1, tf1;
    cell(ta1); cell(tb1); cell(tc1); cell(td1); cell(te1); cell(tf1);
    int ihs = 0;
    der_weno(ls, ta1, tb1, tc1, td1, te1, tf1, ihs);
    const double ad = P.alpha1 * dx1;
    OMP_FOR
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double gxv = (std::fabs(ta1(i, j, k)) > std::fabs(td1(i, j, k))) ? ta1(i, j, k) : td1(i, j, k);
                const double gyv = (std::fabs(tb1(i, j, k)) > std::fabs(te1(i, j, k))) ? tb1(i, j, k) : te1(i, j, k);
                const double gzv = (std::fabs(tc1(i, j, k)) > std::fabs(tf1(i, j, k))) ? tc1(i, j, k) : tf1(i, j, k);
                const double l = ls(i, j, k);
                double h;
                if (l < -P.alpha1 * dx1) {
                    h = 0.; hsx(i, j, k) = 0.; hsy(i, j, k) = 0.; hsz(i, j, k) = 0.;
                } else if (l > P.alpha1 * dx1) {
                    h = 1.; hsx(i, j, k) = 0.; hsy(i, j, k) = 0.; hsz(i, j, k) = 0.;
                } else {
                    h = 0.5 * (1. + l / ad + 1. / pi * std::sin(pi * l / ad));
                    const double cs = std::cos(pi * l / ad);
                    hsx(i, j, k) = 0.5 * gxv * (1. + cs) / ad;
                    hsy(i, j, k) = 0.5 * gyv * (1. + cs) / ad;
                    hsz(i, j, k) = 0.5 * gzv * (1. + cs) / ad;
                }
                hs(i, j, k) = h;
                if (P.t_hs == 0) {
                    rho(i, j, k) = P.rho_f1 * (1. - h) + P.rho_f2 * h;
                    ls_nu(i, j, k) = P.mi_f1 * (1. - h) + P.mi_f2 * h;
                } else {                                /* :700-701, aux1 = mi_f1*10000 (:656-657) */
                    rho(i, j, k) = std::pow(P.rho_f1, 1. - h) + std::pow(P.rho_f2, h) - 1.;
                    ls_nu(i, j, k) = (std::pow(P.mi_f1 * 10000., 1. - h) + std::pow(P.mi_f2 * 10000., h) - 1.) / 10000.;
                }
            }
}

/* mod_ls1 — 14_level_set.f90:709-805: |grad ls| and curvature from the WENO derivative of
 * the unit normal (normals' WENO uses ihs = 1 in every direction, inherited from der_weno). */
void Oracle::mod_ls1() {
    Arr ta1, tb1, tc1, td1, te1, tf1, nxa, nya, nza;
    cell(ta1); cell(tb1); cell(tc1); cell(td1); cell(te1); cell(tf1); cell(nxa); cell(nya); cell(nza);
    int ihs = 0;
    der_weno(ls, ta1, tb1, tc1, td1, te1, tf1, ihs);
    OMP_FOR
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double a = (std::fabs(ta1(i, j, k)) > std::fabs(td1(i, j, k))) ? ta1(i, j, k) : td1(i, j, k);
                const double b = (std::fabs(tb1(i, j, k)) > std::fabs(te1(i, j, k))) ? tb1(i, j, k) : te1(i, j, k);
                const double c = (std::fabs(tc1(i, j, k)) > std::fabs(tf1(i, j, k))) ? tc1(i, j, k) : tf1(i, j, k);
                const double m = std::sqrt(a * a + b * b + c * c);
                mod_ls(i, j, k) = m;
                if (m == 0) { nxa(i, j, k) = 0.; nya(i, j, k) = 0.; nza(i, j, k) = 0.; }
                else { nxa(i, j, k) = a / m; nya(i, j, k) = b / m; nza(i, j, k) = c / m; }
            }
    /* WENO of the normal components with the inherited ihs in all three directions */
    const int ihn = ihs;
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        std::vector<double> pin((size_t)std::max(nx, std::max(ny, nz))), pp(pin.size()), pn(pin.size());
#ifdef _OPENMP
#pragma omp for collapse(2) schedule(static)
#endif
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j) {
                for (int i = 1; i <= nx; ++i) pin[i - 1] = nxa(i, j, k);
                weno1(pp.data(), pn.data(), nx, dx, pin.data(), ihn);
                for (int i = 1; i <= nx; ++i) { ta1(i, j, k) = pp[i - 1]; td1(i, j, k) = pn[i - 1]; }
            }
#ifdef _OPENMP
#pragma omp for collapse(2) schedule(static)
#endif
        for (int k = 1; k <= nz; ++k)
            for (int i = 1; i <= nx; ++i) {
                for (int j = 1; j <= ny; ++j) pin[j - 1] = nya(i, j, k);
                weno1(pp.data(), pn.data(), ny, dy, pin.data(), ihn);
                for (int j = 1; j <= ny; ++j) { tb1(i, j, k) = pp[j - 1]; te1(i, j, k) = pn[j - 1]; }
            }
#ifdef _OPENMP
#pragma omp for collapse(2) schedule(static)
#endif
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                for (int k = 1; k <= nz; ++k) pin[k - 1] = nza(i, j, k);
                weno1(pp.data(), pn.data(), nz, dz, pin.data(), ihn);
                for (int k = 1; k <= nz; ++k) { tc1(i, j, k) = pp[k - 1]; tf1(i, j, k) = pn[k - 1]; }
            }
    }
    OMP_FOR
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                ddlsdx(i, j, k) = (std::fabs(td1(i, j, k)) > std::fabs(ta1(i, j, k))) ? td1(i, j, k) : ta1(i, j, k);
                ddlsdy(i, j, k) = (std::fabs(te1(i, j, k)) > std::fabs(tb1(i, j, k))) ? te1(i, j, k) : tb1(i, j, k);
                ddlsdz(i, j, k) = (std::fabs(tf1(i, j, k)) > std::fabs(tc1(i, j, k))) ? tf1(i, j, k) : tc1(i, j, k);
                kurv(i, j, k) = ddlsdx(i, j, k) + ddlsdy(i, j, k) + ddlsdz(i, j, k);
            }
}

/* vol = sum (1-(1-hs)) dx dy dz in serial order — 14_level_set.f90:208-215, 246-253. */
double Oracle::volume() const {
    double vol = 0.;
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
                vol = vol + (1. - (1. - hs(i, j, k))) * dx * dy * dz;
    return vol;
}

/* level_set — 14_level_set.f90:221-285.  The volume-correction loop has no cap in the
 * reference; here it stops after 1000 passes (documented difference, never reached in
 * the test cases). */
void Oracle::level_set() {
    Arr sy7, gx, ta1;
    cell(sy7); cell(gx); cell(ta1);
    const double dtaux = dt1;
    dt1 = dt;
    for (int itrl = 1; itrl <= 3; ++itrl) {
        conv_weno(sy7);
        intt_ls(sy7, gx, ta1, itrl, ls);
    }
    dt1 = dtaux;
    reinic_weno();
    mod_ls1();
    heaviside();
    vol_ins = volume();
    last_volfix_iters = 0;
    while (std::fabs(vol_ins - vol_ini) / vol_ins > P.vol_tol && last_volfix_iters < 1000) {
        const double fac = (vol_ins - vol_ini);
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i)
                    ls(i, j, k) = ls(i, j, k) - dt1 * fac * mod_ls(i, j, k) / vol_ini;
        mod_ls1();
        heaviside();
        vol_ins = volume();
        ++last_volfix_iters;
    }
    mod_ls1();
    heaviside();
}

/* ---------------------------------------------------------------------------------------
 * 8_derivadas.f90 helpers: centre -> face interpolation with end-face copy
 * (interp?_cf, :304-327, :353-380, :406-434).  `src` has extents (1..dimx,1..dimy,1..dimz).
 * ------------------------------------------------------------------------------------- */
static void interpx_cf(const Arr& a, int dimx, int dimy, int dimz, Arr& out) {
    out.init(1, dimx + 1, 1, dimy, 1, dimz);
    for (int k = 1; k <= dimz; ++k)
        for (int j = 1; j <= dimy; ++j) {
            for (int i = 2; i <= dimx; ++i) out(i, j, k) = (a(i, j, k) + a(i - 1, j, k)) * 0.5;
            out(1, j, k) = out(2, j, k);
            out(dimx + 1, j, k) = out(dimx, j, k);
        }
}
static void interpy_cf(const Arr& a, int dimx, int dimy, int dimz, Arr& out) {
    out.init(1, dimx, 1, dimy + 1, 1, dimz);
    for (int k = 1; k <= dimz; ++k)
        for (int j = 2; j <= dimy; ++j)
            for (int i = 1; i <= dimx; ++i) out(i, j, k) = (a(i, j, k) + a(i, j - 1, k)) * 0.5;
    for (int k = 1; k <= dimz; ++k)
        for (int i = 1; i <= dimx; ++i) {
            out(i, 1, k) = out(i, 2, k);
            out(i, dimy + 1, k) = out(i, dimy, k);
        }
}
static void interpz_cf(const Arr& a, int dimx, int dimy, int dimz, Arr& out) {
    out.init(1, dimx, 1, dimy, 1, dimz + 1);
    for (int k = 2; k <= dimz; ++k)
        for (int j = 1; j <= dimy; ++j)
            for (int i = 1; i <= dimx; ++i) out(i, j, k) = (a(i, j, k) + a(i, j, k - 1)) * 0.5;
    for (int j = 1; j <= dimy; ++j)
        for (int i = 1; i <= dimx; ++i) {
            out(i, j, 1) = out(i, j, 2);
            out(i, j, dimz + 1) = out(i, j, dimz);
        }
}

/* face -> centre averages interp?_fc (8_derivadas.f90:331-349, 384-402, 438-455) along
 * direction d (0 x, 1 y, 2 z): out has one point fewer than n[] along d. */
static void interp_fc(const Arr& a, int d, const int n[3], Arr& out) {
    const int ex = d == 0, ey = d == 1, ez = d == 2;
    out.init(1, n[0] - ex, 1, n[1] - ey, 1, n[2] - ez);
    for (int k = 1; k <= n[2] - ez; ++k)
        for (int j = 1; j <= n[1] - ey; ++j)
            for (int i = 1; i <= n[0] - ex; ++i) out(i, j, k) = (a(i, j, k) + a(i + ex, j + ey, k + ez)) * 0.5;
}

/* Derivatives of 8_derivadas.f90 along direction d of a field with one halo layer, over the
 * points (1..n[0], 1..n[1], 1..n[2]):
 *   deriva     centred (derivax/y/z, :1-68);
 *   deriva_u2p second-order forward one-sided, centred on the last point (derivax/y/zu2p, :83-179);
 *   deriva_u2n second-order backward one-sided, centred on the first point (derivax/y/zu2n,
 *              :194-290). */
static void deriva(const Arr& a, int d, const int n[3], double h, Arr& out) {
    const int ex = d == 0, ey = d == 1, ez = d == 2;
    out.init(1, n[0], 1, n[1], 1, n[2]);
    for (int k = 1; k <= n[2]; ++k)
        for (int j = 1; j <= n[1]; ++j)
            for (int i = 1; i <= n[0]; ++i)
                out(i, j, k) = (a(i + ex, j + ey, k + ez) - a(i - ex, j - ey, k - ez)) / (2. * h);
}
static void deriva_u2p(const Arr& a, int d, const int n[3], double h, Arr& out) {
    const int ex = d == 0, ey = d == 1, ez = d == 2;
    out.init(1, n[0], 1, n[1], 1, n[2]);
    for (int k = 1; k <= n[2]; ++k)
        for (int j = 1; j <= n[1]; ++j)
            for (int i = 1; i <= n[0]; ++i) {
                const int m = d == 0 ? i : (d == 1 ? j : k);
                if (m < n[d])
                    out(i, j, k) = 0.5 * (-a(i + 2 * ex, j + 2 * ey, k + 2 * ez) + 4. * a(i + ex, j + ey, k + ez) -
                                          3. * a(i, j, k)) / h;
                else
                    out(i, j, k) = 0.5 * (a(i + ex, j + ey, k + ez) - a(i - ex, j - ey, k - ez)) / h;
            }
}
static void deriva_u2n(const Arr& a, int d, const int n[3], double h, Arr& out) {
    const int ex = d == 0, ey = d == 1, ez = d == 2;
    out.init(1, n[0], 1, n[1], 1, n[2]);
    for (int k = 1; k <= n[2]; ++k)
        for (int j = 1; j <= n[1]; ++j)
            for (int i = 1; i <= n[0]; ++i) {
                const int m = d == 0 ? i : (d == 1 ? j : k);
                if (m > 1)
                    out(i, j, k) = 0.5 * (a(i - 2 * ex, j - 2 * ey, k - 2 * ez) - 4. * a(i - ex, j - ey, k - ez) +
                                          3. * a(i, j, k)) / h;
                else
                    out(i, j, k) = 0.5 * (a(i + ex, j + ey, k + ez) - a(i - ex, j - ey, k - ez)) / h;
            }
}

/* visco — 5_viscosidade.f90:12-219 (m_turb 0, 1 and 2). */
void Oracle::visco() {
    Arr xa, ya, za;
    xa.init(1, nx1, 1, ny, 1, nz); ya.init(1, nx, 1, ny1, 1, nz); za.init(1, nx, 1, ny, 1, nz1);
    if (P.m_turb == 2) {
        /* directional Smagorinsky (:58-61, 104-164): each face's eddy viscosity from the strain
           of its own velocity component, without the density factor; the cross derivatives go
           face -> edge (interp?_cf, end copy) -> face (interp?_fc).  nut is not written. */
        const int du[3] = {nx1, ny, nz}, dv[3] = {nx, ny1, nz}, dw[3] = {nx, ny, nz1};
        Arr dudx_i, dudy_i, dudz_i, dvdx_i, dvdy_i, dvdz_i, dwdx_i, dwdy_i, dwdz_i;
        deriva(u, 0, du, dx, dudx_i); deriva(v, 0, dv, dx, dvdx_i); deriva(w, 0, dw, dx, dwdx_i);
        deriva(u, 1, du, dy, dudy_i); deriva(v, 1, dv, dy, dvdy_i); deriva(w, 1, dw, dy, dwdy_i);
        deriva(u, 2, du, dz, dudz_i); deriva(v, 2, dv, dz, dvdz_i); deriva(w, 2, dw, dz, dwdz_i);
        const int exy[3] = {nx1, ny1, nz}, exz[3] = {nx1, ny, nz1}, eyz[3] = {nx, ny1, nz1};
        Arr t, dvdx_x, dwdx_x, dudy_y, dwdy_y, dudz_z, dvdz_z;
        interpx_cf(dvdx_i, nx, ny1, nz, t);  interp_fc(t, 1, exy, dvdx_x);
        interpx_cf(dwdx_i, nx, ny, nz1, t);  interp_fc(t, 2, exz, dwdx_x);
        interpy_cf(dudy_i, nx1, ny, nz, t);  interp_fc(t, 0, exy, dudy_y);
        interpy_cf(dwdy_i, nx, ny, nz1, t);  interp_fc(t, 2, eyz, dwdy_y);
        interpz_cf(dudz_i, nx1, ny, nz, t);  interp_fc(t, 0, exz, dudz_z);
        interpz_cf(dvdz_i, nx, ny1, nz, t);  interp_fc(t, 1, eyz, dvdz_z);
        const double cs = P.csmag;
        for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx1; ++i) {
            const double p1 = dudx_i(i, j, k) + 0.5 * (dudy_i(i, j, k) + dvdx_x(i, j, k) + dudz_i(i, j, k) + dwdx_x(i, j, k));
            xa(i, j, k) = dx * dx * cs * cs * std::sqrt(2. * p1 * p1);
        }
        for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny1; ++j) for (int i = 1; i <= nx; ++i) {
            const double p1 = dvdy_i(i, j, k) + 0.5 * (dvdx_i(i, j, k) + dudy_y(i, j, k) + dvdz_i(i, j, k) + dwdy_y(i, j, k));
            ya(i, j, k) = dy * dy * cs * cs * std::sqrt(2. * p1 * p1);
        }
        for (int k = 1; k <= nz1; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
            const double p1 = dwdz_i(i, j, k) + 0.5 * (dwdy_i(i, j, k) + dvdz_z(i, j, k) + dudz_z(i, j, k) + dwdx_i(i, j, k));
            za(i, j, k) = dz * dz * cs * cs * std::sqrt(2. * p1 * p1);
        }
    } else if (P.m_turb == 1) {
        /* centred derivatives on the staggered grids (derivax/y/z, 8_derivadas.f90:1-68)
           then face -> centre averages (interp?_fc); fused per cell here, same arithmetic */
        const double cdel = std::pow(dx * dy * dz, 2. / 3.);
        OMP_FOR
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    auto dudx_i = [&](int ii, int jj, int kk) { return (u(ii + 1, jj, kk) - u(ii - 1, jj, kk)) / (2. * dx); };
                    auto dudy_i = [&](int ii, int jj, int kk) { return (u(ii, jj + 1, kk) - u(ii, jj - 1, kk)) / (2. * dy); };
                    auto dudz_i = [&](int ii, int jj, int kk) { return (u(ii, jj, kk + 1) - u(ii, jj, kk - 1)) / (2. * dz); };
                    auto dvdx_i = [&](int ii, int jj, int kk) { return (v(ii + 1, jj, kk) - v(ii - 1, jj, kk)) / (2. * dx); };
                    auto dvdy_i = [&](int ii, int jj, int kk) { return (v(ii, jj + 1, kk) - v(ii, jj - 1, kk)) / (2. * dy); };
                    auto dvdz_i = [&](int ii, int jj, int kk) { return (v(ii, jj, kk + 1) - v(ii, jj, kk - 1)) / (2. * dz); };
                    auto dwdx_i = [&](int ii, int jj, int kk) { return (w(ii + 1, jj, kk) - w(ii - 1, jj, kk)) / (2. * dx); };
                    auto dwdy_i = [&](int ii, int jj, int kk) { return (w(ii, jj + 1, kk) - w(ii, jj - 1, kk)) / (2. * dy); };
                    auto dwdz_i = [&](int ii, int jj, int kk) { return (w(ii, jj, kk + 1) - w(ii, jj, kk - 1)) / (2. * dz); };
                    const double dudx = (dudx_i(i, j, k) + dudx_i(i + 1, j, k)) * 0.5;
                    const double dudy = (dudy_i(i, j, k) + dudy_i(i + 1, j, k)) * 0.5;
                    const double dudz = (dudz_i(i, j, k) + dudz_i(i + 1, j, k)) * 0.5;
                    const double dvdx = (dvdx_i(i, j, k) + dvdx_i(i, j + 1, k)) * 0.5;
                    const double dvdy = (dvdy_i(i, j, k) + dvdy_i(i, j + 1, k)) * 0.5;
                    const double dvdz = (dvdz_i(i, j, k) + dvdz_i(i, j + 1, k)) * 0.5;
                    const double dwdx = (dwdx_i(i, j, k) + dwdx_i(i, j, k + 1)) * 0.5;
                    const double dwdy = (dwdy_i(i, j, k) + dwdy_i(i, j, k + 1)) * 0.5;
                    const double dwdz = (dwdz_i(i, j, k) + dwdz_i(i, j, k + 1)) * 0.5;
                    const double p1 = dudx + 0.5 * (dudy + dvdx + dudz + dwdx);
                    const double p2 = dvdy + 0.5 * (dvdx + dudy + dvdz + dwdy);
                    const double p3 = dwdz + 0.5 * (dwdy + dvdz + dudz + dwdx);
                    nut(i, j, k) = cdel * P.csmag * P.csmag * std::sqrt(2. * (p1 + p2 + p3) * (p1 + p2 + p3)) * rho(i, j, k);
                }
        interpx_cf(nut, nx, ny, nz, xa);
        interpy_cf(nut, nx, ny, nz, ya);
        interpz_cf(nut, nx, ny, nz, za);
    } else if (P.m_turb != 0) {
        std::fprintf(stderr, "oracle: m_turb=%d not restated\n", P.m_turb);
        std::abort();
    }
    Arr lx, ly, lz;
    interpx_cf(ls_nu, nx, ny, nz, lx);
    interpy_cf(ls_nu, nx, ny, nz, ly);
    interpz_cf(ls_nu, nx, ny, nz, lz);
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx1; ++i)
        xnut(i, j, k) = lx(i, j, k) + xa(i, j, k);
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny1; ++j) for (int i = 1; i <= nx; ++i)
        ynut(i, j, k) = ly(i, j, k) + ya(i, j, k);
    for (int k = 1; k <= nz1; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        znut(i, j, k) = lz(i, j, k) + za(i, j, k);
}

/* classico, der = 2 (centred, 7_advectivo.f90:115-170) and der = 3 (second-order upwind,
 * :174-285) for one velocity component `a` on its faces (extents n[]): vel[d] is the velocity
 * that advects it along direction d (the component itself along its own direction). */
static void classico_hi(int der, const Arr& a, const int n[3], const Arr* const vel[3], const double h[3], Arr& out) {
    Arr D[3], Dn[3], Dp[3];
    for (int d = 0; d < 3; ++d) {
        if (der == 2) {
            deriva(a, d, n, h[d], D[d]);
        } else {
            deriva_u2n(a, d, n, h[d], Dn[d]);
            deriva_u2p(a, d, n, h[d], Dp[d]);
        }
    }
    for (int k = 1; k <= n[2]; ++k)
        for (int j = 1; j <= n[1]; ++j)
            for (int i = 1; i <= n[0]; ++i) {
                double s = 0.;
                for (int d = 0; d < 3; ++d) {
                    const double c = (*vel[d])(i, j, k);
                    const double term = der == 2 ? c * D[d](i, j, k)
                                                 : fmax2(c, 0.) * Dn[d](i, j, k) + fmin2(c, 0.) * Dp[d](i, j, k);
                    s = d == 0 ? term : s + term;
                }
                out(i, j, k) = s;
            }
}

/* classico — 7_advectivo.f90:3-290.  der = 1 first-order upwind with 4-point transverse
 * averages (:33-113); der = 2, 3 average the transverse velocities face -> centre
 * (interp?_fc) -> face (interp?_cf, end faces copied). */
void Oracle::classico(Arr& uint_, Arr& vint, Arr& wint) {
    if (P.der == 2 || P.der == 3) {
        const int du[3] = {nx1, ny, nz}, dv[3] = {nx, ny1, nz}, dw[3] = {nx, ny, nz1};
        Arr t, bma, dma, amb, dmb, amd, bmd;
        interp_fc(v, 1, dv, t); interpx_cf(t, nx, ny, nz, bma);   /* :134-135 (:178-179) */
        interp_fc(w, 2, dw, t); interpx_cf(t, nx, ny, nz, dma);
        interp_fc(u, 0, du, t); interpy_cf(t, nx, ny, nz, amb);
        interp_fc(w, 2, dw, t); interpy_cf(t, nx, ny, nz, dmb);
        interp_fc(u, 0, du, t); interpz_cf(t, nx, ny, nz, amd);
        interp_fc(v, 1, dv, t); interpz_cf(t, nx, ny, nz, bmd);
        const double h[3] = {dx, dy, dz};
        const Arr* const vu[3] = {&u, &bma, &dma};
        const Arr* const vv[3] = {&amb, &v, &dmb};
        const Arr* const vw[3] = {&amd, &bmd, &w};
        classico_hi(P.der, u, du, vu, h, uint_);
        classico_hi(P.der, v, dv, vv, h, vint);
        classico_hi(P.der, w, dw, vw, h, wint);
        return;
    }
    if (P.der != 1) { std::fprintf(stderr, "oracle: der=%d not restated\n", P.der); std::abort(); }
    OMP_FOR
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx1; ++i) {
                const double bma = (v(i, j, k) + v(i - 1, j, k) + v(i, j + 1, k) + v(i - 1, j + 1, k)) * 0.25;
                const double dma = (w(i, j, k) + w(i - 1, j, k) + w(i, j, k + 1) + w(i - 1, j, k + 1)) * 0.25;
                double a1 = fmax2(u(i, j, k), 0.), a2 = fmin2(u(i, j, k), 0.);
                const double dudx = a1 * (u(i, j, k) - u(i - 1, j, k)) / dx + a2 * (u(i + 1, j, k) - u(i, j, k)) / dx;
                a1 = fmax2(bma, 0.); a2 = fmin2(bma, 0.);
                const double dudy = a1 * (u(i, j, k) - u(i, j - 1, k)) / dy + a2 * (u(i, j + 1, k) - u(i, j, k)) / dy;
                a1 = fmax2(dma, 0.); a2 = fmin2(dma, 0.);
                const double dudz = a1 * (u(i, j, k) - u(i, j, k - 1)) / dz + a2 * (u(i, j, k + 1) - u(i, j, k)) / dz;
                uint_(i, j, k) = dudx + dudy + dudz;
            }
    OMP_FOR
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny1; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double amb = (u(i, j, k) + u(i + 1, j, k) + u(i, j - 1, k) + u(i + 1, j - 1, k)) * 0.25;
                const double dmb = (w(i, j, k) + w(i, j - 1, k) + w(i, j, k + 1) + w(i, j - 1, k + 1)) * 0.25;
                double a1 = fmax2(amb, 0.), a2 = fmin2(amb, 0.);
                const double dvdx = a1 * (v(i, j, k) - v(i - 1, j, k)) / dx + a2 * (v(i + 1, j, k) - v(i, j, k)) / dx;
                a1 = fmax2(v(i, j, k), 0.); a2 = fmin2(v(i, j, k), 0.);
                const double dvdy = a1 * (v(i, j, k) - v(i, j - 1, k)) / dy + a2 * (v(i, j + 1, k) - v(i, j, k)) / dy;
                a1 = fmax2(dmb, 0.); a2 = fmin2(dmb, 0.);
                const double dvdz = a1 * (v(i, j, k) - v(i, j, k - 1)) / dz + a2 * (v(i, j, k + 1) - v(i, j, k)) / dz;
                vint(i, j, k) = dvdx + dvdy + dvdz;
            }
    OMP_FOR
    for (int k = 1; k <= nz1; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double amd = (u(i, j, k) + u(i + 1, j, k) + u(i, j, k - 1) + u(i + 1, j, k - 1)) * 0.25;
                const double bmd = (v(i, j, k) + v(i, j + 1, k) + v(i, j, k - 1) + v(i, j + 1, k - 1)) * 0.25;
                double a1 = fmax2(amd, 0.), a2 = fmin2(amd, 0.);
                const double dwdx = a1 * (w(i, j, k) - w(i - 1, j, k)) / dx + a2 * (w(i + 1, j, k) - w(i, j, k)) / dx;
                a1 = fmax2(bmd, 0.); a2 = fmin2(bmd, 0.);
                const double dwdy = a1 * (w(i, j, k) - w(i, j - 1, k)) / dy + a2 * (w(i, j + 1, k) - w(i, j, k)) / dy;
                a1 = fmax2(w(i, j, k), 0.); a2 = fmin2(w(i, j, k), 0.);
                const double dwdz = a1 * (w(i, j, k) - w(i, j, k - 1)) / dz + a2 * (w(i, j, k + 1) - w(i, j, k)) / dz;
                wint(i, j, k) = dwdx + dwdy + dwdz;
            }
}

/* The velocity splits c+ = max(c, 0), c- = min(c, 0) of rotacional and antissim, held in
 * arrays of extents (0:nx1+1, 0:ny1+1, 0:nz1+1) shared by the three components. */
struct Splits {
    Arr ap, an, bp, bn, dp, dn;
    Splits(int nx1, int ny1, int nz1) {
        for (Arr* a : {&ap, &an, &bp, &bn, &dp, &dn}) a->init(0, nx1 + 1, 0, ny1 + 1, 0, nz1 + 1);
    }
    void set(int i, int j, int k, double a, double b, double d) {
        ap(i, j, k) = fmax2(a, 0.); an(i, j, k) = fmin2(a, 0.);
        bp(i, j, k) = fmax2(b, 0.); bn(i, j, k) = fmin2(b, 0.);
        dp(i, j, k) = fmax2(d, 0.); dn(i, j, k) = fmin2(d, 0.);
    }
};

/* rotacional — 7_advectivo.f90:293-457 (der = 1; the reference stops for any other scheme):
 * first-order upwind differences of the fluxes c+ a and c- a.  The reference's w part sets
 * dp where dn is meant one plane above the top w-face (:433), leaving dn there unset (its
 * value is indeterminate); here it is min(w, 0) of that ghost, as the u and v parts do at
 * their ends.  It enters only Fw on the top face, which the boundary fill overwrites. */
void Oracle::rotacional(Arr& uint_, Arr& vint, Arr& wint) {
    if (P.der != 1) { std::fprintf(stderr, "oracle: rotacional needs der = 1\n"); std::abort(); }
    Splits S(nx1, ny1, nz1);
    Arr &ap = S.ap, &an = S.an, &bp = S.bp, &bn = S.bn, &dp = S.dp, &dn = S.dn;
    /* u (:335-370) */
    for (int k = 0; k <= nz + 1; ++k)
        for (int j = 0; j <= ny + 1; ++j)
            for (int i = 1; i <= nx + 1; ++i) {
                const double bma = (v(i, j, k) + v(i - 1, j, k) + v(i, j + 1, k) + v(i - 1, j + 1, k)) * 0.25;
                const double dma = (w(i, j, k) + w(i - 1, j, k) + w(i, j, k + 1) + w(i - 1, j, k + 1)) * 0.25;
                S.set(i, j, k, u(i, j, k), bma, dma);
            }
    for (int k = 0; k <= nz + 1; ++k)
        for (int j = 0; j <= ny + 1; ++j) {
            ap(0, j, k) = fmax2(u(0, j, k), 0.);
            an(nx1 + 1, j, k) = fmin2(u(nx1 + 1, j, k), 0.);
        }
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx1; ++i) {
                const double dudx = (ap(i, j, k) * u(i, j, k) - ap(i - 1, j, k) * u(i - 1, j, k)) / dx +
                                    (an(i + 1, j, k) * u(i + 1, j, k) - an(i, j, k) * u(i, j, k)) / dx;
                const double dudy = (bp(i, j, k) * u(i, j, k) - bp(i, j - 1, k) * u(i, j - 1, k)) / dy +
                                    (bn(i, j + 1, k) * u(i, j + 1, k) - bn(i, j, k) * u(i, j, k)) / dy;
                const double dudz = (dp(i, j, k) * u(i, j, k) - dp(i, j, k - 1) * u(i, j, k - 1)) / dz +
                                    (dn(i, j, k + 1) * u(i, j, k + 1) - dn(i, j, k) * u(i, j, k)) / dz;
                uint_(i, j, k) = dudx + dudy + dudz;
            }
    /* v (:373-409) */
    for (int k = 0; k <= nz + 1; ++k)
        for (int j = 1; j <= ny + 1; ++j)
            for (int i = 0; i <= nx + 1; ++i) {
                const double amb = (u(i, j, k) + u(i + 1, j, k) + u(i, j - 1, k) + u(i + 1, j - 1, k)) * 0.25;
                const double dmb = (w(i, j, k) + w(i, j - 1, k) + w(i, j, k + 1) + w(i, j - 1, k + 1)) * 0.25;
                S.set(i, j, k, amb, v(i, j, k), dmb);
            }
    for (int k = 0; k <= nz + 1; ++k)
        for (int i = 0; i <= nx + 1; ++i) {
            bp(i, 0, k) = fmax2(v(i, 0, k), 0.);
            bn(i, ny1 + 1, k) = fmin2(v(i, ny1 + 1, k), 0.);
        }
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny1; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double dvdx = (ap(i, j, k) * v(i, j, k) - ap(i - 1, j, k) * v(i - 1, j, k)) / dx +
                                    (an(i + 1, j, k) * v(i + 1, j, k) - an(i, j, k) * v(i, j, k)) / dx;
                const double dvdy = (bp(i, j, k) * v(i, j, k) - bp(i, j - 1, k) * v(i, j - 1, k)) / dy +
                                    (bn(i, j + 1, k) * v(i, j + 1, k) - bn(i, j, k) * v(i, j, k)) / dy;
                const double dvdz = (dp(i, j, k) * v(i, j, k) - dp(i, j, k - 1) * v(i, j, k - 1)) / dz +
                                    (dn(i, j, k + 1) * v(i, j, k + 1) - dn(i, j, k) * v(i, j, k)) / dz;
                vint(i, j, k) = dvdx + dvdy + dvdz;
            }
    /* w (:412-446) */
    for (int k = 1; k <= nz + 1; ++k)
        for (int j = 0; j <= ny + 1; ++j)
            for (int i = 0; i <= nx + 1; ++i) {
                const double amd = (u(i, j, k) + u(i + 1, j, k) + u(i, j, k - 1) + u(i + 1, j, k - 1)) * 0.25;
                const double bmd = (v(i, j, k) + v(i, j + 1, k) + v(i, j, k - 1) + v(i, j + 1, k - 1)) * 0.25;
                S.set(i, j, k, amd, bmd, w(i, j, k));
            }
    for (int j = 0; j <= ny + 1; ++j)
        for (int i = 0; i <= nx + 1; ++i) {
            dp(i, j, 0) = fmax2(w(i, j, 0), 0.);
            dn(i, j, nz1 + 1) = fmin2(w(i, j, nz1 + 1), 0.);
        }
    for (int k = 1; k <= nz1; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double dwdx = (ap(i, j, k) * w(i, j, k) - ap(i - 1, j, k) * w(i - 1, j, k)) / dx +
                                    (an(i + 1, j, k) * w(i + 1, j, k) - an(i, j, k) * w(i, j, k)) / dx;
                const double dwdy = (bp(i, j, k) * w(i, j, k) - bp(i, j - 1, k) * w(i, j - 1, k)) / dy +
                                    (bn(i, j + 1, k) * w(i, j + 1, k) - bn(i, j, k) * w(i, j, k)) / dy;
                const double dwdz = (dp(i, j, k) * w(i, j, k) - dp(i, j, k - 1) * w(i, j, k - 1)) / dz +
                                    (dn(i, j, k + 1) * w(i, j, k + 1) - dn(i, j, k) * w(i, j, k)) / dz;
                wint(i, j, k) = dwdx + dwdy + dwdz;
            }
}

/* antissim — 7_advectivo.f90:460-653 (der = 1 only): the mean of the flux-difference form of
 * rotacional and the advective upwind form, with the split arrays' end planes filled by
 * copies of their neighbours (:521-524, 571-574, 618-621). */
void Oracle::antissim(Arr& uint_, Arr& vint, Arr& wint) {
    if (P.der != 1) { std::fprintf(stderr, "oracle: antissim needs der = 1\n"); std::abort(); }
    Splits S(nx1, ny1, nz1);
    Arr &ap = S.ap, &an = S.an, &bp = S.bp, &bn = S.bn, &dp = S.dp, &dn = S.dn;
    /* the copies ap(0,:,:) = ap(1,:,:), bp(:,0,:) = bp(:,1,:), dp(:,:,0) = dp(:,:,1) */
    auto low_copies = [&]() {
        for (int k = 0; k <= nz1 + 1; ++k)
            for (int j = 0; j <= ny1 + 1; ++j) ap(0, j, k) = ap(1, j, k);
        for (int k = 0; k <= nz1 + 1; ++k)
            for (int i = 0; i <= nx1 + 1; ++i) bp(i, 0, k) = bp(i, 1, k);
        for (int j = 0; j <= ny1 + 1; ++j)
            for (int i = 0; i <= nx1 + 1; ++i) dp(i, j, 0) = dp(i, j, 1);
    };
    /* one direction of one component: F at m-1, m, m+1, the splits P, N at m-1, m, m+1 */
    auto term = [](double Fm, double F0, double Fp, double Pm, double P0, double N0, double Np, double h) {
        return ((P0 * F0 - Pm * Fm) / h + (Np * Fp - N0 * F0) / h + P0 * (F0 - Fm) / h + N0 * (Fp - F0) / h) * 0.5;
    };
    /* u (:503-545) */
    for (int k = 1; k <= nz + 1; ++k)
        for (int j = 1; j <= ny + 1; ++j)
            for (int i = 1; i <= nx + 1; ++i) {
                const double bma = (v(i, j, k) + v(i - 1, j, k) + v(i, j + 1, k) + v(i - 1, j + 1, k)) * 0.25;
                const double dma = (w(i, j, k) + w(i - 1, j, k) + w(i, j, k + 1) + w(i - 1, j, k + 1)) * 0.25;
                S.set(i, j, k, u(i, j, k), bma, dma);
            }
    low_copies();
    for (int k = 0; k <= nz1 + 1; ++k)
        for (int j = 0; j <= ny1 + 1; ++j) an(nx1 + 1, j, k) = an(nx1, j, k);
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx1; ++i) {
                const double dudx = term(u(i - 1, j, k), u(i, j, k), u(i + 1, j, k), ap(i - 1, j, k), ap(i, j, k),
                                         an(i, j, k), an(i + 1, j, k), dx);
                const double dudy = term(u(i, j - 1, k), u(i, j, k), u(i, j + 1, k), bp(i, j - 1, k), bp(i, j, k),
                                         bn(i, j, k), bn(i, j + 1, k), dy);
                const double dudz = term(u(i, j, k - 1), u(i, j, k), u(i, j, k + 1), dp(i, j, k - 1), dp(i, j, k),
                                         dn(i, j, k), dn(i, j, k + 1), dz);
                uint_(i, j, k) = dudx + dudy + dudz;
            }
    /* v (:549-595) */
    for (int k = 1; k <= nz + 1; ++k)
        for (int j = 1; j <= ny + 1; ++j)
            for (int i = 1; i <= nx + 1; ++i) {
                const double amb = (u(i, j, k) + u(i + 1, j, k) + u(i, j - 1, k) + u(i + 1, j - 1, k)) * 0.25;
                const double dmb = (w(i, j, k) + w(i, j - 1, k) + w(i, j, k + 1) + w(i, j - 1, k + 1)) * 0.25;
                S.set(i, j, k, amb, v(i, j, k), dmb);
            }
    low_copies();
    for (int k = 0; k <= nz1 + 1; ++k)
        for (int i = 0; i <= nx1 + 1; ++i) bn(i, ny1 + 1, k) = bn(i, ny1, k);
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny1; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double dvdx = term(v(i - 1, j, k), v(i, j, k), v(i + 1, j, k), ap(i - 1, j, k), ap(i, j, k),
                                         an(i, j, k), an(i + 1, j, k), dx);
                const double dvdy = term(v(i, j - 1, k), v(i, j, k), v(i, j + 1, k), bp(i, j - 1, k), bp(i, j, k),
                                         bn(i, j, k), bn(i, j + 1, k), dy);
                const double dvdz = term(v(i, j, k - 1), v(i, j, k), v(i, j, k + 1), dp(i, j, k - 1), dp(i, j, k),
                                         dn(i, j, k), dn(i, j, k + 1), dz);
                vint(i, j, k) = dvdx + dvdy + dvdz;
            }
    /* w (:598-640) */
    for (int k = 1; k <= nz + 1; ++k)
        for (int j = 1; j <= ny + 1; ++j)
            for (int i = 1; i <= nx + 1; ++i) {
                const double amd = (u(i, j, k) + u(i + 1, j, k) + u(i, j, k - 1) + u(i + 1, j, k - 1)) * 0.25;
                const double bmd = (v(i, j, k) + v(i, j + 1, k) + v(i, j, k - 1) + v(i, j + 1, k - 1)) * 0.25;
                S.set(i, j, k, amd, bmd, w(i, j, k));
            }
    low_copies();
    for (int j = 0; j <= ny1 + 1; ++j)
        for (int i = 0; i <= nx1 + 1; ++i) dn(i, j, nz1 + 1) = dn(i, j, nz1);
    for (int k = 1; k <= nz1; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double dwdx = term(w(i - 1, j, k), w(i, j, k), w(i + 1, j, k), ap(i - 1, j, k), ap(i, j, k),
                                         an(i, j, k), an(i + 1, j, k), dx);
                const double dwdy = term(w(i, j - 1, k), w(i, j, k), w(i, j + 1, k), bp(i, j - 1, k), bp(i, j, k),
                                         bn(i, j, k), bn(i, j + 1, k), dy);
                const double dwdz = term(w(i, j, k - 1), w(i, j, k), w(i, j, k + 1), dp(i, j, k - 1), dp(i, j, k),
                                         dn(i, j, k), dn(i, j, k + 1), dz);
                wint(i, j, k) = dwdx + dwdy + dwdz;
            }
}

/* convdiff — 6_convdiff.f90:14-189.  The sponge term -(w-0)*epis_z with epis_z = 0
 * (:65, call commented out at :86) is omitted; it changes at most the sign of a zero. */
void Oracle::convdiff() {
    prd0.a = prd1.a;                                    /* :62 */
    Arr uint_, vint, wint;
    uint_.init(1, nx1, 1, ny, 1, nz); vint.init(1, nx, 1, ny1, 1, nz); wint.init(1, nx, 1, ny, 1, nz1);
    if (P.adv_type == 2)                                /* :72-79 */
        rotacional(uint_, vint, wint);
    else if (P.adv_type == 3)
        antissim(uint_, vint, wint);
    else
        classico(uint_, vint, wint);
    Arr rhox, rhoy, rhoz, dhsdx, dhsdy, dhsdz, tx, ty, tz;
    interpx_cf(rho, nx, ny, nz, rhox);
    interpy_cf(rho, nx, ny, nz, rhoy);
    interpz_cf(rho, nx, ny, nz, rhoz);
    cell(tx); cell(ty); cell(tz);
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
        tx(i, j, k) = hsx(i, j, k) * kurv(i, j, k) / rho(i, j, k);
        ty(i, j, k) = hsy(i, j, k) * kurv(i, j, k) / rho(i, j, k);
        tz(i, j, k) = hsz(i, j, k) * kurv(i, j, k) / rho(i, j, k);
    }
    interpx_cf(tx, nx, ny, nz, dhsdx);
    interpy_cf(ty, nx, ny, nz, dhsdy);
    interpz_cf(tz, nx, ny, nz, dhsdz);
    Arr bma, dma, amb, dmb, amd, bmd, ama, bmb, dmd;
    interpy_cf(xnut, nx1, ny, nz, bma);     /* (nx1,ny1,nz) */
    interpz_cf(xnut, nx1, ny, nz, dma);     /* (nx1,ny,nz1) */
    interpx_cf(ynut, nx, ny1, nz, amb);     /* (nx1,ny1,nz) */
    interpz_cf(ynut, nx, ny1, nz, dmb);     /* (nx,ny1,nz1) */
    interpx_cf(znut, nx, ny, nz1, amd);     /* (nx1,ny,nz1) */
    interpy_cf(znut, nx, ny, nz1, bmd);     /* (nx,ny1,nz1) */
    ama.init(0, nx1, 1, ny, 1, nz); bmb.init(1, nx, 0, ny1, 1, nz); dmd.init(1, nx, 1, ny, 0, nz1);
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
        ama(i, j, k) = nut(i, j, k) / dx;
        bmb(i, j, k) = nut(i, j, k) / dy;
        dmd(i, j, k) = nut(i, j, k) / dz;
    }
    for (auto& x : bma.a) x = x / dy;
    for (auto& x : dma.a) x = x / dz;
    for (auto& x : amb.a) x = x / dx;
    for (auto& x : dmb.a) x = x / dz;
    for (auto& x : amd.a) x = x / dx;
    for (auto& x : bmd.a) x = x / dy;
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) { ama(0, j, k) = ama(1, j, k); ama(nx1, j, k) = ama(nx, j, k); }
    for (int k = 1; k <= nz; ++k) for (int i = 1; i <= nx; ++i) { bmb(i, 0, k) = bmb(i, 1, k); bmb(i, ny1, k) = bmb(i, ny, k); }
    for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) { dmd(i, j, 0) = dmd(i, j, 1); dmd(i, j, nz1) = dmd(i, j, nz); }
    const double cz = P.gz / (P.chezy * P.chezy);
    const double sg = P.sigma;
    OMP_FOR
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx1; ++i) {
                const double G = (ama(i, j, k) * 2. * (u(i + 1, j, k) - u(i, j, k)) -
                                  ama(i - 1, j, k) * 2. * (u(i, j, k) - u(i - 1, j, k))) / dx +
                                 bma(i, j + 1, k) * ((u(i, j + 1, k) - u(i, j, k)) / dy + (v(i, j + 1, k) - v(i - 1, j + 1, k)) / dx) -
                                 bma(i, j, k) * ((u(i, j, k) - u(i, j - 1, k)) / dy + (v(i, j, k) - v(i - 1, j, k)) / dx) +
                                 dma(i, j, k + 1) * ((u(i, j, k + 1) - u(i, j, k)) / dz + (w(i, j, k + 1) - w(i - 1, j, k + 1)) / dx) -
                                 dma(i, j, k) * ((u(i, j, k) - u(i, j, k - 1)) / dz + (w(i, j, k) - w(i - 1, j, k)) / dx);
                Fu(i, j, k) = -uint_(i, j, k) + G / rhox(i, j, k) + P.gx - sg * dhsdx(i, j, k) + tf_u(i, j, k) -
                              cz * std::sqrt(ub(i, j, k) * ub(i, j, k)) * u(i, j, k);
            }
    OMP_FOR
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny1; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double G = amb(i + 1, j, k) * ((v(i + 1, j, k) - v(i, j, k)) / dx + (u(i + 1, j, k) - u(i + 1, j - 1, k)) / dy) -
                                 amb(i, j, k) * ((v(i, j, k) - v(i - 1, j, k)) / dx + (u(i, j, k) - u(i, j - 1, k)) / dy) +
                                 (bmb(i, j, k) * 2. * (v(i, j + 1, k) - v(i, j, k)) -
                                  bmb(i, j - 1, k) * 2. * (v(i, j, k) - v(i, j - 1, k))) / dy +
                                 dmb(i, j, k + 1) * ((v(i, j, k + 1) - v(i, j, k)) / dz + (w(i, j, k + 1) - w(i, j - 1, k + 1)) / dy) -
                                 dmb(i, j, k) * ((v(i, j, k) - v(i, j, k - 1)) / dz + (w(i, j, k) - w(i, j - 1, k)) / dy);
                Fv(i, j, k) = -vint(i, j, k) + G / rhoy(i, j, k) - sg * dhsdy(i, j, k) + tf_v(i, j, k) -
                              cz * std::sqrt(vb(i, j, k) * vb(i, j, k)) * v(i, j, k);
            }
    OMP_FOR
    for (int k = 1; k <= nz1; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double G = amd(i + 1, j, k) * ((w(i + 1, j, k) - w(i, j, k)) / dx + (u(i + 1, j, k) - u(i + 1, j, k - 1)) / dz) -
                                 amd(i, j, k) * ((w(i, j, k) - w(i - 1, j, k)) / dx + (u(i, j, k) - u(i, j, k - 1)) / dz) +
                                 bmd(i, j + 1, k) * ((w(i, j + 1, k) - w(i, j, k)) / dy + (v(i, j + 1, k) - v(i, j + 1, k - 1)) / dz) -
                                 bmd(i, j, k) * ((w(i, j, k) - w(i, j - 1, k)) / dy + (v(i, j, k) - v(i, j, k - 1)) / dz) +
                                 (dmd(i, j, k) * 2. * (w(i, j, k + 1) - w(i, j, k)) -
                                  dmd(i, j, k - 1) * 2. * (w(i, j, k) - w(i, j, k - 1))) / dz;
                Fw(i, j, k) = -wint(i, j, k) + G / rhoz(i, j, k) - P.gz - sg * dhsdz(i, j, k) + tf_w(i, j, k) -
                              cz * std::sqrt(wb(i, j, k) * wb(i, j, k)) * w(i, j, k);
            }
}

/* tempo — 11_diversos.f90:10-230. */
void Oracle::tempo(int tt, int it) {
    const int tm = P.t_tempo;
    auto loop3 = [&](Arr& a, Arr& F, Arr& a0, Arr& f0, Arr& f1, int ex, int ey, int ez) {
        for (int k = 1; k <= nz + ez; ++k)
            for (int j = 1; j <= ny + ey; ++j)
                for (int i = 1; i <= nx + ex; ++i) {
                    if (tm == 0 || (tm == 3 && it == 1)) {
                        a(i, j, k) = a(i, j, k) + dt * F(i, j, k);
                    } else if (tm == 1) {
                        if (tt == 1) { const double aux1 = dt; a0(i, j, k) = a(i, j, k); a(i, j, k) = a(i, j, k) + aux1 * F(i, j, k); }
                        else if (tt == 2) { const double aux1 = dt; a(i, j, k) = a0(i, j, k) + aux1 * F(i, j, k); }
                    } else if (tm == 2) {
                        if (tt == 1) {
                            const double aux1 = dt;
                            a0(i, j, k) = a(i, j, k); f0(i, j, k) = F(i, j, k); a(i, j, k) = a(i, j, k) + aux1 * F(i, j, k);
                        } else if (tt == 2) {
                            const double aux1 = 2. * dt;
                            f1(i, j, k) = F(i, j, k); a(i, j, k) = a0(i, j, k) - dt * f0(i, j, k) + aux1 * F(i, j, k);
                        } else if (tt == 3) {
                            const double aux1 = dt / 6.;
                            a(i, j, k) = a0(i, j, k) + aux1 * (f0(i, j, k) + 4. * f1(i, j, k) + F(i, j, k));
                        }
                    } else if (tm == 3 && it != 1) {
                        a(i, j, k) = a(i, j, k) + dt * 0.5 * (3 * F(i, j, k) - f0(i, j, k));
                        f0(i, j, k) = F(i, j, k);
                    }
                }
        if (tm == 3 && it == 1) f0.a = F.a;
    };
    loop3(u, Fu, u0, fu0, fu1, 1, 0, 0);
    loop3(v, Fv, v0, fv0, fv1, 0, 1, 0);
    loop3(w, Fw, w0, fw0, fw1, 0, 0, 1);
}

/* contorno — 3_contorno.f90:10-492 (obst_t = 0, mms_t = 0).  prd_corr (:872-950) returns
 * zeros, so the "+ dpdx" terms vanish.  ccz0 = cczf = 0 (periodic z) is an extension that
 * mirrors the reference's periodic-x rows. */
/* Obstacle columns of contorno(1/2) (3_contorno.f90:266-294): velocities zeroed from k = 0 up
 * to the column's mask, and the first value above it captured for the wall friction. */
void Oracle::contorno_obstacle() {
    if (!has_obstacle) { std::fprintf(stderr, "oracle: obst_t != 0 without masks\n"); std::abort(); }
    for (int j = 0; j <= ny + 1; ++j)
        for (int i = 0; i <= nx + 1; ++i) {
            for (int k = 0; k <= KU(i, j); ++k) u(i, j, k) = 0.;
            for (int k = 0; k <= KV(i, j); ++k) v(i, j, k) = 0.;
            for (int k = 0; k <= KW(i, j); ++k) w(i, j, k) = 0.;
            ub(i, j, KU(i, j) + 1) = u(i, j, KU(i, j) + 1);
            vb(i, j, KV(i, j) + 1) = v(i, j, KV(i, j) + 1);
            wb(i, j, KW(i, j) + 1) = w(i, j, KW(i, j) + 1);
        }
    for (int j = 0; j <= ny + 1; ++j)
        for (int k = 0; k <= KU(nx1 + 1, j); ++k) u(nx1 + 1, j, k) = 0.;
    for (int i = 0; i <= nx + 1; ++i)
        for (int k = 0; k <= KV(i, ny1 + 1); ++k) v(i, ny1 + 1, k) = 0.;
}

/* Option periodic_faces = 1 (an extension; the reference has no counterpart): on a periodic axis
 * the two end faces of interp?_cf, which are one face of the periodic box, both take the average
 * across the wrap, (rho(1) + rho(n)) * 0.5, in place of the copies of their neighbour faces
 * (8_derivadas.f90:318-323).  graddin's scaled operator is then symmetric where the density
 * varies across the periodic boundary, and posdin moves both copies of that face alike. */
void Oracle::wrap_faces(Arr& rx, Arr& ry, Arr& rz) const {
    if (P.periodic_faces != 1) return;
    if (P.ccx0 == 0)
        for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j)
            rx(1, j, k) = rx(nx1, j, k) = (rho(1, j, k) + rho(nx, j, k)) * 0.5;
    if (P.ccy0 == 0)
        for (int k = 1; k <= nz; ++k) for (int i = 1; i <= nx; ++i)
            ry(i, 1, k) = ry(i, ny1, k) = (rho(i, 1, k) + rho(i, ny, k)) * 0.5;
    if (P.ccz0 == 0)
        for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
            rz(i, j, 1) = rz(i, j, nz1) = (rho(i, j, 1) + rho(i, j, nz)) * 0.5;
}

/* Option outflow_fix = 1 (an extension; the reference has no counterpart): after
 * contorno(2) has copied the outflow plane (ccxf = 4, 3_contorno.f90:193-197, 362-409), shift
 * u(nx+1,j,k) by one uniform delta over the outflow faces above the obstacle mask so that the
 * net volume flux through the boundary is zero.  graddin's all-Neumann system (9_grad.f90:96-116)
 * is then consistent: the sum of its right-hand side over the cells, which telescopes to the
 * net boundary flux, vanishes.  Sums in the order written here (j fastest, then k). */
void Oracle::outflow_fix() {
    double fx = 0., fy = 0., fz = 0.;
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) fx = fx + (u(nx1, j, k) - u(1, j, k));
    for (int k = 1; k <= nz; ++k) for (int i = 1; i <= nx; ++i) fy = fy + (v(i, ny1, k) - v(i, 1, k));
    for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) fz = fz + (w(i, j, nz1) - w(i, j, 1));
    const double net = fx * (dy * dz) + fy * (dx * dz) + fz * (dx * dy);
    long long open = 0;
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) open += (!has_obstacle || k > KU(nx1, j)) ? 1 : 0;
    if (open == 0) return;
    const double delta = -net / ((double)open * (dy * dz));
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            if (!has_obstacle || k > KU(nx1, j)) u(nx1, j, k) = u(nx1, j, k) + delta;
}

/* contorno(3) (3_contorno.f90:445-481): the level set inside the obstacle (k < kw) taken
 * from the neighbouring fluid cells at the same height, or from the cell above at the
 * obstacle's top.  A neighbour outside 1..nx, 1..ny is never read: the reference reads ls
 * outside its bounds there, and here that neighbour's "fluid" test is false.  A cell whose
 * fluid neighbours are read is itself never rewritten (its own mask is below k), so the
 * loop order does not matter. */
void Oracle::level_set_obstacle() {
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i)
            for (int k = 1; k <= KW(i, j) - 1; ++k) {
                auto fluid = [&](int ii, int jj) { return ii >= 1 && ii <= nx && jj >= 1 && jj <= ny && KW(ii, jj) < k; };
                auto solid = [&](int ii, int jj) { return KW(ii, jj) >= k; };
                if (fluid(i - 1, j) && fluid(i, j - 1))
                    ls(i, j, k) = (ls(i - 1, j, k) + ls(i, j - 1, k)) * 0.5;
                else if (fluid(i + 1, j) && fluid(i, j - 1))
                    ls(i, j, k) = (ls(i + 1, j, k) + ls(i, j - 1, k)) * 0.5;
                else if (fluid(i + 1, j) && fluid(i, j + 1))
                    ls(i, j, k) = (ls(i + 1, j, k) + ls(i, j + 1, k)) * 0.5;
                else if (fluid(i - 1, j) && fluid(i, j + 1))
                    ls(i, j, k) = (ls(i - 1, j, k) + ls(i, j + 1, k)) * 0.5;
                else if (fluid(i - 1, j) && solid(i, j - 1) && solid(i, j + 1))
                    ls(i, j, k) = ls(i - 1, j, k);
                else if (fluid(i, j - 1) && solid(i - 1, j) && solid(i + 1, j))
                    ls(i, j, k) = ls(i, j - 1, k);
                else if (fluid(i + 1, j) && solid(i, j - 1) && solid(i, j + 1))
                    ls(i, j, k) = ls(i + 1, j, k);
                else if (fluid(i, j + 1) && solid(i - 1, j) && solid(i + 1, j))
                    ls(i, j, k) = ls(i, j + 1, k);
                else if (k == KW(i, j) - 1 && k < nz)
                    ls(i, j, k) = ls(i, j, k + 1);
            }
}

/* waves_coef — 3_contorno.f90:1084-1205: Stokes I/II wavelength by fixed-point iteration of
 * the dispersion relation; Stokes V by scanning wavelengths for the two conditions on lamb. */
void Oracle::waves_coef() {
    const double pi = std::acos(-1.), gz = P.gz;
    kp.assign(nz + 2, 0.);
    for (int k = 0; k <= nz + 1; ++k) kp[k] = (k - 0.5) * dz;
    a_w = 0.03; p_w = 2.5; h0_f = 1.;
    l0_w = gz * p_w * p_w / (2. * pi);
    if (P.wave_t <= 2) {
        l_w = gz * p_w * p_w / (2. * pi);
        for (int i = 1; i <= 1000; ++i) l_w = gz * p_w * p_w / (2. * pi) * std::tanh(2. * pi * h0_f / l_w);
        c_w = l_w / p_w; f_w = 2. * pi / p_w; n_w = 2. * pi / l_w;
        return;
    }
    /* wave_t == 5 */
    auto pw = [](double x, double e) { return std::pow(x, e); };
    double erro0 = 999., lamb = 0.;
    const int nxii = 10000;
    double s, c, b33, b35, b55, c1, c2;
    auto coefs = [&](double lw) {
        s = std::sinh(2. * pi * h0_f / lw);
        c = std::cosh(2. * pi * h0_f / lw);
        b33 = 3. * (8. * pw(c, 6.) + 1.) / (64. * pw(s, 6.));
        b35 = (88128. * pw(c, 14.) - 208224. * pw(c, 12) + 70848. * pw(c, 10.) + 54000. * pw(c, 8.) - 21816. * pw(c, 6.) +
               6264. * pw(c, 4.) - 54. * c * c - 81.) / (12288. * pw(s, 12.) * (6. * c * c - 1.));
        b55 = (192000. * pw(c, 16.) - 262720. * pw(c, 14.) + 83680. * pw(c, 12) + 20160. * pw(c, 10.) - 7280. * pw(c, 8.) +
               7160. * pw(c, 6.) - 1800. * pw(c, 4.) - 1050. * c * c + 225.) /
              (12288 * pw(s, 10.) * (6. * c * c - 1.) * (8. * pw(c, 4.) - 11. * c * c + 3.));
        c1 = (8. * pw(c, 4.) - 8. * c * c + 9.) / (8. * pw(s, 4.));
        c2 = (3840. * pw(c, 12.) - 4096. * pw(c, 10.) + 2592. * pw(c, 8.) - 1008. * pw(c, 6.) + 5944. * pw(c, 4.) - 1830. * c * c +
              147.) / (512. * pw(s, 10.) * (6. * c * c - 1.));
    };
    for (int ii = 1; ii <= nxii; ++ii) {
        double lamb1 = 0., lamb2 = 0.;
        const double l_w1 = l0_w * 0.5 + l0_w * ((double)ii / nxii) * 2.5;
        coefs(l_w1);
        for (int i = 1; i <= 10000; ++i) lamb1 = pi * a_w * 2. / l_w1 - pw(lamb1, 3.) * b33 - pw(lamb1, 5.) * (b35 + b55);
        for (int i = 1; i <= 10000; ++i)
            lamb2 = std::sqrt((l_w1 / (l0_w * std::tanh(2. * pi * h0_f / l_w1)) - 1.) / (c1 + pw(lamb2, 2.) * c2));
        const double erro = std::fabs(lamb1 - lamb2);
        if (erro < erro0) { erro0 = erro; lamb = lamb1; l_w = l_w1; }
    }
    c_w = l_w / p_w; f_w = 2. * pi / p_w; n_w = 2. * pi / l_w;
    coefs(l_w);
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
    const double a55 = -(2880. * pw(c, 10.) - 72480. * pw(c, 8.) + 324000. * pw(c, 6.) - 432000. * pw(c, 4.) + 163470. * c * c - 16245.) /
                       (61440. * pw(s, 11.) * (6. * c * c - 1.) * (8. * pw(c, 4.) - 11. * c * c + 3.));
    const double b22 = c * (2. * c * c + 1.) / (4. * pw(s, 3.));
    const double b24 = c * (272. * pw(c, 8.) - 504. * pw(c, 6.) - 192. * pw(c, 4.) + 322 * c * c + 21.) / (384. * pw(s, 9.));
    const double b44 = c * (768. * pw(c, 10.) - 448. * pw(c, 8.) - 48. * pw(c, 6.) + 48. * pw(c, 4.) + 106. * c * c - 21.) /
                       (384. * pw(s, 9.) * (6. * c * c - 1.));
    aeta[1] = lamb / n_w;
    aeta[2] = (lamb * lamb * b22 + pw(lamb, 4.) * b24) / n_w;
    aeta[3] = (pw(lamb, 3.) * b33 + pw(lamb, 5.) * b35) / n_w;
    aeta[4] = pw(lamb, 4.) * b44 / n_w;
    aeta[5] = pw(lamb, 5.) * b55 / n_w;
    avel[1] = 1. * 2. * pi / (p_w * n_w) * (lamb * a11 + pw(lamb, 3.) * a13 + pw(lamb, 5.) * a15);
    avel[2] = 2. * 2. * pi / (p_w * n_w) * (pw(lamb, 2.) * a22 + pw(lamb, 4.) * a24);
    avel[3] = 3. * 2. * pi / (p_w * n_w) * (pw(lamb, 3.) * a33 + pw(lamb, 5.) * a35);
    avel[4] = 4. * 2. * pi / (p_w * n_w) * (pw(lamb, 4.) * a44);
    avel[5] = 5. * 2. * pi / (p_w * n_w) * (pw(lamb, 5.) * a55);
}

/* boundary_waves — 3_contorno.f90:952-1082: the wave's elevation, u and w at the inflow
 * columns i = 0, 1 at time t.  The reference works on a single-precision copy ls1 of the
 * level set and copies all of it back, so every call rounds ls to float32; the inflow column
 * i = 1 takes the elevation's distance h_f(1) - kp(k).  Of the planes it writes, bxy0 comes
 * from an array v1 that is never set and the top row of bxz0 from an unset w1(0,:,nz+2):
 * both are 0 here. */
void Oracle::boundary_waves() {
    if (kp.empty()) waves_coef();
    const int W = P.wave_t;
    const double tanhh = std::tanh(n_w * h0_f), shh = std::sinh(n_w * h0_f);
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) ls(i, j, k) = (double)(float)ls(i, j, k);
    for (auto& x : bxy0.a) x = 0.;
    for (int j = 0; j <= ny + 1; ++j) bxz0(j, nz1 + 1, 0) = 0.;
    for (int k = 0; k <= nz + 1; ++k)
        for (int j = 0; j <= ny + 1; ++j)
            for (int i = 0; i <= 1; ++i) {
                double hf, u1, w1;
                const double aux2 = n_w * dx * (i - 0.5) - f_w * t, aux3 = n_w * dx * (i - 1.) - f_w * t;
                if (W == 1) {
                    hf = h0_f + a_w * std::cos(n_w * dx * (i - 0.5) - f_w * t);
                } else if (W == 2) {
                    hf = h0_f + a_w * std::cos(aux2) + n_w * a_w * a_w * (3. - tanhh * tanhh) / (4. * tanhh * tanhh * tanhh) * std::cos(2. * aux2);
                } else {
                    hf = h0_f + aeta[1] * std::cos(aux2) + aeta[2] * std::cos(2. * aux2) + aeta[3] * std::cos(3. * aux2) +
                         aeta[4] * std::cos(4. * aux2) + aeta[5] * std::cos(5. * aux2);
                }
                const float ls1 = (float)(hf - kp[k]);
                if (ls1 >= 0.f) {
                    if (W == 1) {
                        u1 = a_w * f_w * std::cosh(n_w * kp[k]) / shh * std::cos(n_w * dx * (i - 1.) - f_w * t);
                        w1 = a_w * f_w * std::sinh(n_w * (kp[k] - 0.5 * dz)) / shh * std::sin(n_w * dx * (i - 0.5) - f_w * t);
                    } else if (W == 2) {
                        u1 = a_w * f_w * std::cosh(n_w * kp[k]) / shh * std::cos(aux3) +
                             3. / 4. * a_w * a_w * f_w * n_w * std::cosh(2. * n_w * kp[k]) / std::pow(shh, 4.) * std::cos(2 * aux3);
                        w1 = a_w * f_w * std::sinh(n_w * (kp[k] - 0.5 * dz)) / shh * std::sin(aux2) +
                             3. / 4. * a_w * a_w * f_w * n_w * std::sinh(2. * n_w * (kp[k] - 0.5 * dz)) / std::pow(shh, 4.) *
                                 std::sin(2. * aux3);
                    } else {
                        const double aux4 = n_w * kp[k], aux5 = n_w * (kp[k] - 0.5 * dz);
                        u1 = avel[1] * std::cosh(aux4) * std::cos(aux3) + avel[2] * std::cosh(2 * aux4) * std::cos(2 * aux3) +
                             avel[3] * std::cosh(3 * aux4) * std::cos(3 * aux3) + avel[4] * std::cosh(4 * aux4) * std::cos(4 * aux3) +
                             avel[5] * std::cosh(5 * aux4) * std::cos(5 * aux3);
                        w1 = avel[1] * std::sinh(aux5) * std::sin(aux2) + avel[2] * std::sinh(2 * aux5) * std::sin(2 * aux2) +
                             avel[3] * std::sinh(3 * aux5) * std::sin(3 * aux2) + avel[4] * std::sinh(4 * aux5) * std::sin(4 * aux2) +
                             avel[5] * std::sinh(5 * aux5) * std::sin(5 * aux2);
                    }
                } else {
                    u1 = 0.; w1 = 0.;
                }
                if (i == 0) { bxx0(j, k, 0) = u1; bxz0(j, k, 0) = w1; }
                else {
                    bxx1(j, k, 0) = u1;
                    if (j >= 1 && j <= ny && k >= 1 && k <= nz) ls(1, j, k) = (double)ls1;
                }
            }
}

void Oracle::contorno(int nlock) {
    const int X0 = P.ccx0, XF = P.ccxf, Y0 = P.ccy0, YF = P.ccyf, Z0 = P.ccz0, ZF = P.cczf;
    const int I1 = nx1 + 1, J1 = ny1 + 1, K1 = nz1 + 1;   /* u/v/w outer ghost index */
    auto X_all = [&](Arr& a, auto fn) { for (int k = a.lo[2]; k <= a.hi[2]; ++k) for (int j = a.lo[1]; j <= a.hi[1]; ++j) fn(j, k); };
    auto Y_all = [&](Arr& a, auto fn) { for (int k = a.lo[2]; k <= a.hi[2]; ++k) for (int i = a.lo[0]; i <= a.hi[0]; ++i) fn(i, k); };
    auto Z_all = [&](Arr& a, auto fn) { for (int j = a.lo[1]; j <= a.hi[1]; ++j) for (int i = a.lo[0]; i <= a.hi[0]; ++i) fn(i, j); };
    if (nlock == 1 || nlock == 2) {
        /* pressure ghosts (:37-54) */
        if (X0 == 0 && XF == 0) X_all(prd1, [&](int j, int k) { prd1(0, j, k) = prd1(nx, j, k); prd1(nx + 1, j, k) = prd1(1, j, k); });
        else X_all(prd1, [&](int j, int k) { prd1(0, j, k) = prd1(1, j, k); prd1(nx + 1, j, k) = prd1(nx, j, k); });
        if (Y0 == 0 && YF == 0) Y_all(prd1, [&](int i, int k) { prd1(i, 0, k) = prd1(i, ny, k); prd1(i, ny + 1, k) = prd1(i, 1, k); });
        else Y_all(prd1, [&](int i, int k) { prd1(i, 0, k) = prd1(i, 1, k); prd1(i, ny + 1, k) = prd1(i, ny, k); });
        if (Z0 == 0 && ZF == 0) Z_all(prd1, [&](int i, int j) { prd1(i, j, 0) = prd1(i, j, nz); prd1(i, j, nz + 1) = prd1(i, j, 1); });
        else Z_all(prd1, [&](int i, int j) { prd1(i, j, 0) = prd1(i, j, 1); prd1(i, j, nz + 1) = prd1(i, j, nz); });
        /* y = 0 wall (:58-85) */
        if (Y0 == 0 && YF == 0) {
            Y_all(u, [&](int i, int k) { u(i, 0, k) = u(i, ny, k); });
            Y_all(v, [&](int i, int k) { v(i, 0, k) = v(i, ny1 - 1, k); v(i, 1, k) = v(i, ny1, k); });
            Y_all(w, [&](int i, int k) { w(i, 0, k) = w(i, ny, k); });
        }
        if (Y0 == 1) { Y_all(u, [&](int i, int k) { u(i, 0, k) = u(i, 1, k); }); Y_all(v, [&](int i, int k) { v(i, 0, k) = -v(i, 2, k); }); Y_all(w, [&](int i, int k) { w(i, 0, k) = w(i, 1, k); }); }
        if (Y0 == 2) { Y_all(u, [&](int i, int k) { u(i, 0, k) = -u(i, 1, k); }); Y_all(v, [&](int i, int k) { v(i, 0, k) = v(i, 2, k); }); Y_all(w, [&](int i, int k) { w(i, 0, k) = -w(i, 1, k); }); }
        if (Y0 == 3) { Y_all(u, [&](int i, int k) { u(i, 0, k) = byx0(i, k, 0); }); Y_all(v, [&](int i, int k) { v(i, 0, k) = byy0(i, k, 0); }); Y_all(w, [&](int i, int k) { w(i, 0, k) = byz0(i, k, 0); }); }
        /* y = yf wall (:87-114) */
        if (Y0 == 0 && YF == 0) {
            Y_all(u, [&](int i, int k) { u(i, ny + 1, k) = u(i, 1, k); });
            Y_all(v, [&](int i, int k) { v(i, J1, k) = v(i, 2, k); });
            Y_all(w, [&](int i, int k) { w(i, ny + 1, k) = w(i, 1, k); });
        }
        if (YF == 1) { Y_all(u, [&](int i, int k) { u(i, ny + 1, k) = u(i, ny, k); }); Y_all(v, [&](int i, int k) { v(i, J1, k) = -v(i, ny1 - 1, k); }); Y_all(w, [&](int i, int k) { w(i, ny + 1, k) = w(i, ny, k); }); }
        if (YF == 2) { Y_all(u, [&](int i, int k) { u(i, ny + 1, k) = -u(i, ny, k); }); Y_all(v, [&](int i, int k) { v(i, J1, k) = v(i, ny1 - 1, k); }); Y_all(w, [&](int i, int k) { w(i, ny + 1, k) = -w(i, ny, k); }); }
        if (YF == 3) { Y_all(u, [&](int i, int k) { u(i, ny + 1, k) = byxf(i, k, 0); }); Y_all(v, [&](int i, int k) { v(i, J1, k) = byyf1(i, k, 0); }); Y_all(w, [&](int i, int k) { w(i, ny + 1, k) = byzf(i, k, 0); }); }
        /* x = 0 wall (:116-161) */
        if (X0 == 0 && XF == 0) {
            X_all(u, [&](int j, int k) { u(0, j, k) = u(nx1 - 1, j, k); });
            X_all(v, [&](int j, int k) { v(0, j, k) = v(nx, j, k); });
            X_all(w, [&](int j, int k) { w(0, j, k) = w(nx, j, k); });
        }
        if (X0 == 1) { X_all(u, [&](int j, int k) { u(0, j, k) = -u(2, j, k); }); X_all(v, [&](int j, int k) { v(0, j, k) = v(1, j, k); }); X_all(w, [&](int j, int k) { w(0, j, k) = w(1, j, k); }); }
        if (X0 == 2) { X_all(u, [&](int j, int k) { u(0, j, k) = u(2, j, k); }); X_all(v, [&](int j, int k) { v(0, j, k) = -v(1, j, k); }); X_all(w, [&](int j, int k) { w(0, j, k) = -w(1, j, k); }); }
        if (X0 == 3) { X_all(u, [&](int j, int k) { u(0, j, k) = bxx0(j, k, 0); }); X_all(v, [&](int j, int k) { v(0, j, k) = bxy0(j, k, 0); }); X_all(w, [&](int j, int k) { w(0, j, k) = bxz0(j, k, 0); }); }
        if (X0 == 4) { X_all(v, [&](int j, int k) { v(0, j, k) = bxy0(j, k, 0); }); X_all(w, [&](int j, int k) { w(0, j, k) = w(1, j, k); }); }
        /* x = xf wall (:163-197) */
        if (X0 == 0 && XF == 0) {
            X_all(u, [&](int j, int k) { u(I1, j, k) = u(2, j, k); });
            X_all(v, [&](int j, int k) { v(nx + 1, j, k) = v(1, j, k); });
            X_all(w, [&](int j, int k) { w(nx + 1, j, k) = w(1, j, k); });
        }
        if (XF == 1) { X_all(u, [&](int j, int k) { u(I1, j, k) = -u(nx1 - 1, j, k); }); X_all(v, [&](int j, int k) { v(nx + 1, j, k) = v(nx, j, k); }); X_all(w, [&](int j, int k) { w(nx + 1, j, k) = w(nx, j, k); }); }
        if (XF == 2) { X_all(u, [&](int j, int k) { u(I1, j, k) = u(nx1 - 1, j, k); }); X_all(v, [&](int j, int k) { v(nx + 1, j, k) = -v(nx, j, k); }); X_all(w, [&](int j, int k) { w(nx + 1, j, k) = -w(nx, j, k); }); }
        if (XF == 3) { X_all(u, [&](int j, int k) { u(I1, j, k) = bxxf1(j, k, 0); }); X_all(v, [&](int j, int k) { v(nx + 1, j, k) = bxyf(j, k, 0); }); X_all(w, [&](int j, int k) { w(nx + 1, j, k) = bxzf(j, k, 0); }); }
        if (XF == 4) { X_all(u, [&](int j, int k) { u(I1, j, k) = u(nx1, j, k); }); X_all(v, [&](int j, int k) { v(nx + 1, j, k) = v(nx, j, k); }); X_all(w, [&](int j, int k) { w(nx + 1, j, k) = w(nx, j, k); }); }
        /* z = 0 wall (:199-219) */
        if (Z0 == 0 && ZF == 0) {
            Z_all(u, [&](int i, int j) { u(i, j, 0) = u(i, j, nz); });
            Z_all(v, [&](int i, int j) { v(i, j, 0) = v(i, j, nz); });
            Z_all(w, [&](int i, int j) { w(i, j, 0) = w(i, j, nz1 - 1); });
        }
        if (Z0 == 1) { Z_all(u, [&](int i, int j) { u(i, j, 0) = u(i, j, 1); }); Z_all(v, [&](int i, int j) { v(i, j, 0) = v(i, j, 1); }); Z_all(w, [&](int i, int j) { w(i, j, 0) = -w(i, j, 2); }); }
        if (Z0 == 2) { Z_all(u, [&](int i, int j) { u(i, j, 0) = -u(i, j, 1); }); Z_all(v, [&](int i, int j) { v(i, j, 0) = -v(i, j, 1); }); Z_all(w, [&](int i, int j) { w(i, j, 0) = w(i, j, 2); }); }
        if (Z0 == 3) { Z_all(u, [&](int i, int j) { u(i, j, 0) = bzx0(i, j, 0); }); Z_all(v, [&](int i, int j) { v(i, j, 0) = bzy0(i, j, 0); }); Z_all(w, [&](int i, int j) { w(i, j, 0) = bzz0(i, j, 0); }); }
        /* z = zf (:221-241) */
        if (Z0 == 0 && ZF == 0) {
            Z_all(u, [&](int i, int j) { u(i, j, nz + 1) = u(i, j, 1); });
            Z_all(v, [&](int i, int j) { v(i, j, nz + 1) = v(i, j, 1); });
            Z_all(w, [&](int i, int j) { w(i, j, K1) = w(i, j, 2); });
        }
        if (ZF == 1) { Z_all(u, [&](int i, int j) { u(i, j, nz + 1) = u(i, j, nz); }); Z_all(v, [&](int i, int j) { v(i, j, nz + 1) = v(i, j, nz); }); Z_all(w, [&](int i, int j) { w(i, j, K1) = -w(i, j, nz1 - 1); }); }
        if (ZF == 2) { Z_all(u, [&](int i, int j) { u(i, j, nz + 1) = -u(i, j, nz); }); Z_all(v, [&](int i, int j) { v(i, j, nz + 1) = -v(i, j, nz); }); Z_all(w, [&](int i, int j) { w(i, j, K1) = w(i, j, nz1 - 1); }); }
        if (ZF == 3) { Z_all(u, [&](int i, int j) { u(i, j, nz + 1) = bzxf(i, j, 0); }); Z_all(v, [&](int i, int j) { v(i, j, nz + 1) = bzyf(i, j, 0); }); Z_all(w, [&](int i, int j) { w(i, j, K1) = bzzf1(i, j, 0); }); }
        /* wall-friction capture (:247-264), or the obstacle columns (:266-294) */
        if (P.obst_t != 0) {
            contorno_obstacle();
        } else {
            if (Z0 == 2) {
                Z_all(u, [&](int i, int j) { ub(i, j, 2) = u(i, j, 2); });
                Z_all(v, [&](int i, int j) { vb(i, j, 2) = v(i, j, 2); });
                Z_all(w, [&](int i, int j) { wb(i, j, 2) = w(i, j, 2); });
            }
            if (Y0 == 2) {
                Y_all(u, [&](int i, int k) { ub(i, 2, k) = u(i, 2, k); });
                Y_all(v, [&](int i, int k) { vb(i, 2, k) = v(i, 2, k); });
                Y_all(w, [&](int i, int k) { wb(i, 2, k) = w(i, 2, k); });
            }
            if (YF == 2) {
                Y_all(u, [&](int i, int k) { ub(i, ny1 - 1, k) = u(i, ny1 - 1, k); });
                Y_all(v, [&](int i, int k) { vb(i, ny1 - 1, k) = v(i, ny1 - 1, k); });
                Y_all(w, [&](int i, int k) { wb(i, ny1 - 1, k) = w(i, ny1 - 1, k); });
            }
        }
    }
    if (nlock == 3 && P.obst_t != 0) {                  /* :445-487 */
        level_set_obstacle();
        heaviside();
    }
    if (nlock == 2) {
        /* boundary-normal velocities (:297-441) */
        if (Y0 == 0 && YF == 0) Y_all(v, [&](int i, int k) { v(i, 1, k) = v(i, ny1, k); });
        if (Y0 == 1 || Y0 == 2) Y_all(v, [&](int i, int k) { v(i, 1, k) = 0.; });
        if (Y0 == 3) Y_all(v, [&](int i, int k) { v(i, 1, k) = byy1(i, k, 0); });
        if (Y0 == 0 && YF == 0) Y_all(v, [&](int i, int k) { v(i, ny1, k) = v(i, 1, k); });
        if (YF == 1 || YF == 2) Y_all(v, [&](int i, int k) { v(i, ny1, k) = 0.; });
        if (YF == 3) Y_all(v, [&](int i, int k) { v(i, ny1, k) = byyf(i, k, 0); });
        if (X0 == 0 && XF == 0) X_all(u, [&](int j, int k) { u(1, j, k) = u(nx1, j, k); });
        if (X0 == 1 || X0 == 2) X_all(u, [&](int j, int k) { u(1, j, k) = 0.; });
        if (X0 == 3) X_all(u, [&](int j, int k) { u(1, j, k) = bxx1(j, k, 0); });
        if (X0 == 0 && XF == 0) X_all(u, [&](int j, int k) { u(nx1, j, k) = u(1, j, k); });
        if (XF == 1) X_all(u, [&](int j, int k) { u(nx1, j, k) = 0.; });
        if (XF == 2) {
            X_all(u, [&](int j, int k) { u(nx1, j, k) = 0.; });
            X_all(u, [&](int j, int k) { u(I1, j, k) = u(nx1 - 1, j, k); });
            X_all(v, [&](int j, int k) { v(nx + 1, j, k) = -v(nx, j, k); });
            X_all(w, [&](int j, int k) { w(nx + 1, j, k) = -w(nx, j, k); });
        }
        if (XF == 3) X_all(u, [&](int j, int k) { u(nx1, j, k) = bxxf(j, k, 0); });
        if (XF == 4) X_all(u, [&](int j, int k) { u(nx1, j, k) = u(nx1 - 1, j, k); });
        if (Z0 == 0 && ZF == 0) Z_all(w, [&](int i, int j) { w(i, j, 1) = w(i, j, nz1); });
        if (Z0 == 1 || Z0 == 2) Z_all(w, [&](int i, int j) { w(i, j, 1) = 0.; });
        if (Z0 == 3) Z_all(w, [&](int i, int j) { w(i, j, 1) = bzz1(i, j, 0); });
        if (Z0 == 0 && ZF == 0) Z_all(w, [&](int i, int j) { w(i, j, nz1) = w(i, j, 1); });
        if (ZF == 1 || ZF == 2) Z_all(w, [&](int i, int j) { w(i, j, nz1) = 0.; });
        if (ZF == 3) Z_all(w, [&](int i, int j) { w(i, j, nz1) = bzzf(i, j, 0); });
        if (P.outflow_fix == 1 && XF == 4) outflow_fix();
    }
    /* nlock = 3 acts only with obstacles (obst_t != 0, :445-487): nothing to do here. */
}

/* graddin — 9_grad.f90:10-278: Jacobi-scaled conjugate gradient on the variable-density
 * pressure equation, warm-started from prd1.  Returns the iteration count. */
int Oracle::graddin() {
    const double N = (double)nx * ny * nz;
    Arr rhox, rhoy, rhoz, si, sj, sk;
    interpx_cf(rho, nx, ny, nz, rhox);
    interpy_cf(rho, nx, ny, nz, rhoy);
    interpz_cf(rho, nx, ny, nz, rhoz);
    wrap_faces(rhox, rhoy, rhoz);
    si.init(1, nx1, 1, ny, 1, nz); sj.init(1, nx, 1, ny1, 1, nz); sk.init(1, nx, 1, ny, 1, nz1);
    const double cx = dt / (dx * dx), cy = dt / (dy * dy), cz = dt / (dz * dz);
    for (auto& x : si.a) x = cx;
    for (auto& x : sj.a) x = cy;
    for (auto& x : sk.a) x = cz;
    for (size_t n = 0; n < si.size(); ++n) si.a[n] = si.a[n] / rhox.a[n];
    for (size_t n = 0; n < sj.size(); ++n) sj.a[n] = sj.a[n] / rhoy.a[n];
    for (size_t n = 0; n < sk.size(); ++n) sk.a[n] = sk.a[n] / rhoz.a[n];
    Arr d, e, r, p, q, ap, an, bp, bn, cp, cn, mp;
    d.init(0, nx1, 0, ny1, 0, nz1); e = d; r = d; p = d; mp = d;
    cell(q); cell(ap); cell(an); cell(bp); cell(bn); cell(cp); cell(cn);
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
        d(i, j, k) = si(i + 1, j, k) + si(i, j, k) + sj(i, j + 1, k) + sj(i, j, k) + sk(i, j, k + 1) + sk(i, j, k);
        q(i, j, k) = (u(i, j, k) - u(i + 1, j, k)) / dx + (v(i, j, k) - v(i, j + 1, k)) / dy + (w(i, j, k) - w(i, j, k + 1)) / dz;
    }
    const bool perx = (P.ccx0 == 0), pery = (P.ccy0 == 0), perz = (P.ccz0 == 0);
    auto ghosts = [&](Arr& a) {      /* :99-116, :153-170, :234-262 */
        for (int k = 0; k <= nz1; ++k) for (int j = 0; j <= ny1; ++j) {
            if (perx) { a(0, j, k) = a(nx, j, k); a(nx1, j, k) = a(1, j, k); }
            else { a(0, j, k) = a(1, j, k); a(nx1, j, k) = a(nx, j, k); }
        }
        for (int k = 0; k <= nz1; ++k) for (int i = 0; i <= nx1; ++i) {
            if (pery) { a(i, 0, k) = a(i, ny, k); a(i, ny1, k) = a(i, 1, k); }
            else { a(i, 0, k) = a(i, 1, k); a(i, ny1, k) = a(i, ny, k); }
        }
        for (int j = 0; j <= ny1; ++j) for (int i = 0; i <= nx1; ++i) {
            if (perz) { a(i, j, 0) = a(i, j, nz); a(i, j, nz1) = a(i, j, 1); }
            else { a(i, j, 0) = a(i, j, 1); a(i, j, nz1) = a(i, j, nz); }
        }
    };
    ghosts(d);
    for (int k = 0; k <= nz1; ++k) for (int j = 0; j <= ny1; ++j) for (int i = 0; i <= nx1; ++i)
        e(i, j, k) = prd1(i, j, k) * std::sqrt(d(i, j, k));
    double alfamupr = 0.;
    double bb = 0.;
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
        ap(i, j, k) = si(i + 1, j, k) / std::sqrt(d(i, j, k) * d(i + 1, j, k));
        an(i, j, k) = si(i, j, k) / std::sqrt(d(i, j, k) * d(i - 1, j, k));
        bp(i, j, k) = sj(i, j + 1, k) / std::sqrt(d(i, j, k) * d(i, j + 1, k));
        bn(i, j, k) = sj(i, j, k) / std::sqrt(d(i, j, k) * d(i, j - 1, k));
        cp(i, j, k) = sk(i, j, k + 1) / std::sqrt(d(i, j, k) * d(i, j, k + 1));
        cn(i, j, k) = sk(i, j, k) / std::sqrt(d(i, j, k) * d(i, j, k - 1));
        const double b = q(i, j, k) / std::sqrt(d(i, j, k));
        r(i, j, k) = e(i, j, k) - ap(i, j, k) * e(i + 1, j, k) - an(i, j, k) * e(i - 1, j, k)
                   - bp(i, j, k) * e(i, j + 1, k) - bn(i, j, k) * e(i, j - 1, k)
                   - cp(i, j, k) * e(i, j, k + 1) - cn(i, j, k) * e(i, j, k - 1) - b;
        alfamupr = alfamupr + r(i, j, k) * r(i, j, k);
        bb = bb + b * b;
    }
    ghosts(r);
    p.a = r.a;
    int cont = 0;
    double rr = alfamupr;
    double thr = (P.cg_stop == 0) ? P.cg_tol / N : P.cg_tol * P.cg_tol * bb;
    auto keep_going = [&]() {
        if (cont >= P.cg_maxit) return false;
        return (P.cg_stop == 0) ? (std::fabs(alfamupr) > thr) : (rr > thr);
    };
    /* div_tol > 0 (an extension): once the residual test holds, max |sqrt(d) r~| (the largest
       |div u| posdin leaves) must be within div_tol too; otherwise the threshold is lowered by
       (div_tol/max)^2 / 2, at least 4x, and the iterations resume. */
    for (;;) {
    while (keep_going()) {
        cont = cont + 1;
        double amu = 0., adi = 0., bmu = 0.;
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : amu, adi)
#endif
        for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
            mp(i, j, k) = p(i, j, k) - p(i + 1, j, k) * ap(i, j, k) - p(i - 1, j, k) * an(i, j, k)
                        - p(i, j + 1, k) * bp(i, j, k) - p(i, j - 1, k) * bn(i, j, k)
                        - p(i, j, k + 1) * cp(i, j, k) - p(i, j, k - 1) * cn(i, j, k);
            amu = amu + r(i, j, k) * r(i, j, k);
            adi = adi + p(i, j, k) * mp(i, j, k);
        }
        alfamupr = amu;
        const double alfa = amu / adi;
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : bmu)
#endif
        for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
            e(i, j, k) = e(i, j, k) - alfa * p(i, j, k);
            r(i, j, k) = r(i, j, k) - alfa * mp(i, j, k);
            bmu = bmu + r(i, j, k) * r(i, j, k);
        }
        const double beta = bmu / amu;
        OMP_FOR
        for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
            p(i, j, k) = r(i, j, k) + beta * p(i, j, k);
        ghosts(e);
        ghosts(p);
        rr = bmu;
    }
    if (!(P.div_tol > 0.) || cont >= P.cg_maxit) break;
    double m = 0.;
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        m = std::max(m, std::fabs(std::sqrt(d(i, j, k)) * r(i, j, k)));
    last_cg_rmax = m;
    if (!(m > P.div_tol)) break;
    thr = thr * std::min(0.25, 0.5 * (P.div_tol / m) * (P.div_tol / m));
    }
    /* de-normalisation over the whole halo box (:268-274) */
    for (int k = 0; k <= nz + 1; ++k) for (int j = 0; j <= ny + 1; ++j) for (int i = 0; i <= nx + 1; ++i)
        prd1(i, j, k) = e(i, j, k) / std::sqrt(d(i, j, k));
    last_cg_iters = cont;
    last_cg_resid = (bb > 0.) ? std::sqrt(rr / bb) : 0.;
    return cont;
}

/* posdin — 10_pos.f90:1-96. */
void Oracle::posdin() {
    const double aux1 = dt / dx, aux2 = dt / dy;
    Arr rhox, rhoy, rhoz;
    interpx_cf(rho, nx, ny, nz, rhox);
    interpy_cf(rho, nx, ny, nz, rhoy);
    interpz_cf(rho, nx, ny, nz, rhoz);
    wrap_faces(rhox, rhoy, rhoz);
    for (int k = 1; k <= nz; ++k) {
        for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx1; ++i)
            u(i, j, k) = u(i, j, k) - aux1 * (prd1(i, j, k) - prd1(i - 1, j, k)) / rhox(i, j, k);
        for (int j = 1; j <= ny1; ++j) for (int i = 1; i <= nx; ++i)
            v(i, j, k) = v(i, j, k) - aux2 * (prd1(i, j, k) - prd1(i, j - 1, k)) / rhoy(i, j, k);
    }
    for (int k = 1; k <= nz1; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        w(i, j, k) = w(i, j, k) - dt / dz * (prd1(i, j, k) - prd1(i, j, k - 1)) / rhoz(i, j, k);
    prd.a = prd1.a;
}

/* est — 4_plot.f90:500-525: max |div u|. */
double Oracle::est() const {
    double m = 0.;
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
        const double dv = (u(i + 1, j, k) - u(i, j, k)) / dx + (v(i, j + 1, k) - v(i, j, k)) / dy + (w(i, j, k + 1) - w(i, j, k)) / dz;
        m = std::max(m, std::fabs(dv));
    }
    return m;
}

}  /* namespace */

/* ======================================================================================
 * C API used by tests/ and bench.py (ctypes).
 * ==================================================================================== */
extern "C" {

int orc_field_extent(const suli_params* p, int f, int lo[3], int hi[3]) {
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    auto set = [&](int a, int b, int c, int d, int e, int g) { lo[0] = a; hi[0] = b; lo[1] = c; hi[1] = d; lo[2] = e; hi[2] = g; return 0; };
    switch (f) {
    case SULI_F_U: case SULI_F_UB: return set(0, nx + 2, 0, ny + 1, 0, nz + 1);
    case SULI_F_V: case SULI_F_VB: return set(0, nx + 1, 0, ny + 2, 0, nz + 1);
    case SULI_F_W: case SULI_F_WB: return set(0, nx + 1, 0, ny + 1, 0, nz + 2);
    case SULI_F_PRD1: case SULI_F_PRD0: case SULI_F_PRD: return set(0, nx + 1, 0, ny + 1, 0, nz + 1);
    case SULI_F_RHO: case SULI_F_LS_NU: case SULI_F_NUT: case SULI_F_LS: case SULI_F_MOD_LS: case SULI_F_KURV:
    case SULI_F_HS: case SULI_F_DDLSDX: case SULI_F_DDLSDY: case SULI_F_DDLSDZ: case SULI_F_HSX: case SULI_F_HSY: case SULI_F_HSZ:
        return set(1, nx, 1, ny, 1, nz);
    case SULI_F_FU: case SULI_F_U0: case SULI_F_FU0: case SULI_F_FU1: case SULI_F_XNUT: case SULI_F_TF_U:
        return set(1, nx + 1, 1, ny, 1, nz);
    case SULI_F_FV: case SULI_F_V0: case SULI_F_FV0: case SULI_F_FV1: case SULI_F_YNUT: case SULI_F_TF_V:
        return set(1, nx, 1, ny + 1, 1, nz);
    case SULI_F_FW: case SULI_F_W0: case SULI_F_FW0: case SULI_F_FW1: case SULI_F_ZNUT: case SULI_F_TF_W:
        return set(1, nx, 1, ny, 1, nz + 1);
    case SULI_F_BXX0: case SULI_F_BXX1: case SULI_F_BXXF: case SULI_F_BXXF1: return set(0, ny + 1, 0, nz + 1, 0, 0);
    case SULI_F_BXY0: case SULI_F_BXYF: return set(0, ny + 2, 0, nz + 1, 0, 0);
    case SULI_F_BXZ0: case SULI_F_BXZF: return set(0, ny + 1, 0, nz + 2, 0, 0);
    case SULI_F_BYX0: case SULI_F_BYXF: return set(0, nx + 2, 0, nz + 1, 0, 0);
    case SULI_F_BYY0: case SULI_F_BYY1: case SULI_F_BYYF: case SULI_F_BYYF1: return set(0, nx + 1, 0, nz + 1, 0, 0);
    case SULI_F_BYZ0: case SULI_F_BYZF: return set(0, nx + 1, 0, nz + 2, 0, 0);
    case SULI_F_BZX0: case SULI_F_BZXF: return set(0, nx + 2, 0, ny + 1, 0, 0);
    case SULI_F_BZY0: case SULI_F_BZYF: return set(0, nx + 1, 0, ny + 2, 0, 0);
    case SULI_F_BZZ0: case SULI_F_BZZ1: case SULI_F_BZZF: case SULI_F_BZZF1: return set(0, nx + 1, 0, ny + 1, 0, 0);
    default: return -1;
    }
}

void* orc_create(const suli_params* p) {
    if (!p || p->nx < 4 || p->ny < 4 || p->nz < 4) return nullptr;
    Oracle* o = new Oracle();
    o->P = *p;
    o->alloc();
    return o;
}
void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }

int orc_upload(void* h, int f, const double* src) {
    Oracle* o = static_cast<Oracle*>(h);
    Arr* a = o->field(f);
    if (!a) return -1;
    std::memcpy(a->a.data(), src, a->size() * sizeof(double));
    return 0;
}
int orc_download(void* h, int f, double* dst) {
    Oracle* o = static_cast<Oracle*>(h);
    Arr* a = o->field(f);
    if (!a) return -1;
    std::memcpy(dst, a->a.data(), a->size() * sizeof(double));
    return 0;
}
int orc_set_scalar(void* h, int id, double val) {
    Oracle* o = static_cast<Oracle*>(h);
    switch (id) {
    case SULI_S_DT: o->dt = val; return 0;
    case SULI_S_VOL_INI: o->vol_ini = val; return 0;
    case SULI_S_VOL_INS: o->vol_ins = val; return 0;
    case SULI_S_DT1: o->dt1 = val; return 0;
    case SULI_S_T: o->t = val; return 0;
    case SULI_S_NTT: o->ntt = (int)val; return 0;
    case SULI_S_A_DT1: o->a_dt[0] = val; return 0;
    case SULI_S_A_DT2: o->a_dt[1] = val; return 0;
    case SULI_S_A_DT3: o->a_dt[2] = val; return 0;
    default: return -1;
    }
}
int orc_get_scalar(void* h, int id, double* val) {
    if (id == SULI_S_FALLBACKS) { *val = 0.; return 0; }   /* the restatement solves in FP64 only */
    Oracle* o = static_cast<Oracle*>(h);
    switch (id) {
    case SULI_S_DT: *val = o->dt; return 0;
    case SULI_S_VOL_INI: *val = o->vol_ini; return 0;
    case SULI_S_VOL_INS: *val = o->vol_ins; return 0;
    case SULI_S_DT1: *val = o->dt1; return 0;
    case SULI_S_T: *val = o->t; return 0;
    case SULI_S_NTT: *val = o->ntt; return 0;
    case SULI_S_A_DT1: *val = o->a_dt[0]; return 0;
    case SULI_S_A_DT2: *val = o->a_dt[1]; return 0;
    case SULI_S_A_DT3: *val = o->a_dt[2]; return 0;
    default: return -1;
    }
}

/* iniciais without presets — 2_iniciais.f90:36-46 and the RK table :85-104. */
int orc_iniciais(void* h, double u_init) {
    Oracle* o = static_cast<Oracle*>(h);
    o->t = 0.;
    std::fill(o->u.a.begin(), o->u.a.end(), u_init);
    std::fill(o->v.a.begin(), o->v.a.end(), 0.);
    std::fill(o->w.a.begin(), o->w.a.end(), 0.);
    std::fill(o->prd0.a.begin(), o->prd0.a.end(), 0.);
    std::fill(o->prd1.a.begin(), o->prd1.a.end(), 0.);
    std::fill(o->ub.a.begin(), o->ub.a.end(), 0.);
    std::fill(o->vb.a.begin(), o->vb.a.end(), 0.);
    std::fill(o->wb.a.begin(), o->wb.a.end(), 0.);
    if (o->P.wave_t > 0) {                               /* 2_iniciais.f90:52-66 */
        o->waves_coef();
    } else {
    std::fill(o->bxx0.a.begin(), o->bxx0.a.end(), u_init);
    std::fill(o->bxx1.a.begin(), o->bxx1.a.end(), u_init);
    if (o->P.obst_t != 0) {
        /* 2_iniciais.f90:60-65: bxx1(:,0:ku(1,j)) = 0 for every j, i.e. whole rows of the
           plane up to each column's mask (the reference's index order, kept) */
        if (!o->has_obstacle) { std::fprintf(stderr, "oracle: obst_t != 0 without masks\n"); std::abort(); }
        for (int j = 0; j <= o->ny + 1; ++j)
            for (int jj = 0; jj <= o->ny + 1; ++jj) {
                for (int k = 0; k <= o->KU(1, j); ++k) o->bxx1(jj, k, 0) = 0.;
                for (int k = 0; k <= o->KU(0, j); ++k) o->bxx0(jj, k, 0) = 0.;
            }
    }
    }
    const int tm = o->P.t_tempo;
    const double dt = o->P.dt;
    o->dt = dt;
    if (tm == 0 || tm == 3) { o->ntt = 1; o->a_dt[0] = o->a_dt[1] = o->a_dt[2] = 1.0 * dt; }
    else if (tm == 1) { o->ntt = 2; o->a_dt[0] = 0.5 * dt; o->a_dt[1] = 1.0 * dt; o->a_dt[2] = 1.0 * dt; }
    else { o->ntt = 3; o->a_dt[0] = 0.5 * dt; o->a_dt[1] = 1.0 * dt; o->a_dt[2] = 1.0 * dt; }
    return 0;
}
int orc_level_set_ini(void* h) {
    Oracle* o = static_cast<Oracle*>(h);
    if (o->P.t_hs != 0) {                              /* 14_level_set.f90:47-51, 196-202 */
        const double ls_m = 0.481803535 * o->dx1 * o->P.alpha1;
        for (int k = 1; k <= o->nz; ++k)
            for (int j = 1; j <= o->ny; ++j)
                for (int i = 1; i <= o->nx; ++i) o->ls(i, j, k) = o->ls(i, j, k) + ls_m;
    }
    o->heaviside();
    o->vol_ini = o->volume();
    o->mod_ls1();
    return 0;
}
int orc_level_set(void* h, double* vol_ins) {
    Oracle* o = static_cast<Oracle*>(h);
    o->level_set();
    if (vol_ins) *vol_ins = o->vol_ins;
    return 0;
}
int orc_heaviside(void* h) { static_cast<Oracle*>(h)->heaviside(); return 0; }
int orc_mod_ls1(void* h) { static_cast<Oracle*>(h)->mod_ls1(); return 0; }
int orc_volume(void* h, double* vol) { *vol = static_cast<Oracle*>(h)->volume(); return 0; }
int orc_der_weno(void* h, int field, double* out6) {
    /* six WENO derivatives of a cell field (ta1,tb1,tc1,td1,te1,tf1 stacked), for tests */
    Oracle* o = static_cast<Oracle*>(h);
    Arr* src = o->field(field);
    if (!src) return -1;
    Arr t[6];
    for (auto& a : t) o->cell(a);
    int ihs = 0;
    o->der_weno(*src, t[0], t[1], t[2], t[3], t[4], t[5], ihs);
    const size_t n = t[0].size();
    for (int m = 0; m < 6; ++m) std::memcpy(out6 + m * n, t[m].a.data(), n * sizeof(double));
    return 0;
}
int orc_reinic_weno(void* h, int* iters) {
    Oracle* o = static_cast<Oracle*>(h);
    o->reinic_weno();
    if (iters) *iters = o->last_reinit_iters;
    return 0;
}
int orc_visco(void* h) { static_cast<Oracle*>(h)->visco(); return 0; }
int orc_convdiff(void* h) { static_cast<Oracle*>(h)->convdiff(); return 0; }
int orc_tempo(void* h, int tt, int it) { static_cast<Oracle*>(h)->tempo(tt, it); return 0; }
int orc_contorno(void* h, int nlock) { static_cast<Oracle*>(h)->contorno(nlock); return 0; }
int orc_graddin(void* h, int* iters, double* resid) {
    Oracle* o = static_cast<Oracle*>(h);
    const int it = o->graddin();
    if (iters) *iters = it;
    if (resid) *resid = o->last_cg_resid;
    return (it >= o->P.cg_maxit) ? SULI_WARN_CG_MAXIT : 0;
}
int orc_posdin(void* h) { static_cast<Oracle*>(h)->posdin(); return 0; }
int orc_est(void* h, double* m) { *m = static_cast<Oracle*>(h)->est(); return 0; }
int orc_set_dt(void* h, double dt) { static_cast<Oracle*>(h)->dt = dt; return 0; }

/* One time step — 1_principal.f90:64-108 (mms_t = 0, no plot/restart IO), then est(). */
int orc_step(void* h, int it, suli_step_stats* st) {
    Oracle* o = static_cast<Oracle*>(h);
    int status = 0;
    o->t = it * o->dt;
    o->level_set();
    o->contorno(3);
    for (int tt = 1; tt <= o->ntt; ++tt) {
        o->dt = o->a_dt[tt - 1];
        o->visco();
        o->convdiff();
        o->tempo(tt, it);
        if (o->P.wave_t > 0) o->boundary_waves();      /* 1_principal.f90:84 */
        o->contorno(2);
        const int n = o->graddin();
        if (n >= o->P.cg_maxit) status = SULI_WARN_CG_MAXIT;
        if (st) { st->cg_iters[tt - 1] = n; st->cg_resid[tt - 1] = o->last_cg_resid; }
        o->posdin();
        o->contorno(1);
    }
    if (st) {
        st->vol_ins = o->vol_ins;
        st->max_div = o->est();
        st->status = status;
    }
    return status;
}
int orc_last_reinit_iters(void* h) { return static_cast<Oracle*>(h)->last_reinit_iters; }
int orc_boundary_waves(void* h) {
    Oracle* o = static_cast<Oracle*>(h);
    if (o->P.wave_t != 1 && o->P.wave_t != 2 && o->P.wave_t != 5) return SULI_ERR_ARG;
    o->boundary_waves();
    return 0;
}
/* the masks of obstaculo (3_contorno.f90:741-760), Fortran order, checked like
   suli_set_obstacle: ku, kv in [-1, nz], kw in [-1, nz+1] */
int orc_set_obstacle(void* h, const int* ku, const int* kv, const int* kw) {
    Oracle* o = static_cast<Oracle*>(h);
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    const size_t nu = (size_t)(nx + 3) * (ny + 2), nv = (size_t)(nx + 2) * (ny + 3), nw = (size_t)(nx + 2) * (ny + 2);
    for (size_t q = 0; q < nu; ++q) if (ku[q] < -1 || ku[q] > nz) return SULI_ERR_ARG;
    for (size_t q = 0; q < nv; ++q) if (kv[q] < -1 || kv[q] > nz) return SULI_ERR_ARG;
    for (size_t q = 0; q < nw; ++q) if (kw[q] < -1 || kw[q] > nz + 1) return SULI_ERR_ARG;
    o->ku.assign(ku, ku + nu);
    o->kv.assign(kv, kv + nv);
    o->kw.assign(kw, kw + nw);
    o->has_obstacle = true;
    return 0;
}
int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  /* extern "C" */
