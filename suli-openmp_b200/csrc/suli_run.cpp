// suli_run — a native host program that runs SuLi-IC's time loop on one GPU through the C-ABI
// of libsuli_gpu.so (include/suli_gpu.h), the way the reference's PROGRAM PNH runs it on the
// host (1_principal.f90:46-108).
//
// Set-up as the reference's: iniciais (2_iniciais.f90:36-46, 85-104), the level-set preset,
// level_set_ini (14_level_set.f90:196-217), contorno(1) and contorno(3).  Then, for
// it = 1..steps, one of three equivalent step forms:
//   mode=loop  the reference's loop body, one entry point per subroutine: level_set,
//              [contorno(3)], and for every RK stage tt: dt = a_dt(tt), visco, convdiff,
//              tempo(tt, it), [boundary_waves], contorno(2), graddin, posdin, contorno(1);
//              then est (1_principal.f90:64-108);
//   mode=step  suli_step, the same calls inside the library;
//   mode=host  suli_step_host with u, v, w, prd1 and ls kept in host arrays between steps.
// All three give the same fields.
//
// Usage: suli_run [key=value ...]
//   case=dam_break|sloshing  nx= ny= nz= dx=  steps=  print=  mode=loop|step|host
//   precision=0|1  cg_tol=  div_tol=  device=  dump=<prefix>  preset=<file>
// `dump` writes u, v, w, prd1 and ls after the last step as raw float64 in the module arrays'
// Fortran order and extents (<prefix>_u.bin, ...).  `preset` writes the case's time step and
// level-set preset (one float64, then ls over the cells in Fortran order) and stops before
// the library is asked for a device.
//
// Exit status: 0 on success, 1 on a usage error, 2 when the library returns an error (its
// message is printed; without a GPU that is SULI_ERR_NODEVICE from suli_create).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "suli_gpu.h"

namespace {

struct Config {
    std::string kase = "dam_break", mode = "loop", dump, preset;
    int nx = 64, ny = 32, nz = 48, steps = 10, print = 1, precision = 0, device = 0;
    double dx = 0.01, cg_tol = 1e-10, div_tol = 0.0;
};

const char* code_name(int rc) {
    switch (rc) {
    case SULI_OK: return "SULI_OK";
    case SULI_WARN_CG_MAXIT: return "SULI_WARN_CG_MAXIT";
    case SULI_ERR_ARG: return "SULI_ERR_ARG";
    case SULI_ERR_CUDA: return "SULI_ERR_CUDA";
    case SULI_ERR_NAN: return "SULI_ERR_NAN";
    case SULI_ERR_UNSUPPORTED: return "SULI_ERR_UNSUPPORTED";
    case SULI_ERR_NOMEM: return "SULI_ERR_NOMEM";
    case SULI_ERR_NODEVICE: return "SULI_ERR_NODEVICE";
    case SULI_ERR_SIZE: return "SULI_ERR_SIZE";
    default: return "unknown status";
    }
}

bool parse(int argc, char** argv, Config& c) {
    for (int a = 1; a < argc; ++a) {
        const char* eq = std::strchr(argv[a], '=');
        if (!eq) return false;
        const std::string k(argv[a], eq - argv[a]), v(eq + 1);
        if (v.empty()) return false;
        if (k == "case") c.kase = v;
        else if (k == "mode") c.mode = v;
        else if (k == "dump") c.dump = v;
        else if (k == "preset") c.preset = v;
        else if (k == "nx") c.nx = std::atoi(v.c_str());
        else if (k == "ny") c.ny = std::atoi(v.c_str());
        else if (k == "nz") c.nz = std::atoi(v.c_str());
        else if (k == "steps") c.steps = std::atoi(v.c_str());
        else if (k == "print") c.print = std::atoi(v.c_str());
        else if (k == "precision") c.precision = std::atoi(v.c_str());
        else if (k == "device") c.device = std::atoi(v.c_str());
        else if (k == "dx") c.dx = std::atof(v.c_str());
        else if (k == "cg_tol") c.cg_tol = std::atof(v.c_str());
        else if (k == "div_tol") c.div_tol = std::atof(v.c_str());
        else return false;
    }
    return (c.kase == "dam_break" || c.kase == "sloshing") &&
           (c.mode == "loop" || c.mode == "step" || c.mode == "host") && c.nx > 0 && c.ny > 0 && c.nz > 0 &&
           c.steps >= 0 && c.print >= 1 && (c.precision == 0 || c.precision == 1) && c.dx > 0 && c.cg_tol > 0 &&
           c.div_tol >= 0;
}

// Water and air as the benchmark cases state them, closed no-slip box with a free-slip lid,
// Smagorinsky Cs = 0.1, RK3, relative-residual Poisson test; dt from a CFL number with the
// gravity-wave speed sqrt(g * depth), fixed over the run.
suli_params case_params(const Config& c, double& depth) {
    suli_params p;
    suli_params_default(&p);
    p.nx = c.nx; p.ny = c.ny; p.nz = c.nz;
    p.dx = p.dy = p.dz = c.dx;
    p.ccx0 = p.ccxf = 2;
    p.ccy0 = p.ccyf = 2;
    p.ccz0 = 2; p.cczf = 1;
    p.rho_f1 = 1.2; p.mi_f1 = 1.8e-5;
    p.rho_f2 = 1000.0; p.mi_f2 = 1e-3;
    p.gx = 0.0; p.gz = 9.81;
    p.m_turb = 1; p.csmag = 0.1;
    p.t_tempo = 2;
    p.cg_stop = 1; p.cg_maxit = 20000;
    p.dt1 = 0.1 * c.dx;
    p.cg_tol = c.cg_tol;
    p.div_tol = c.div_tol;
    p.precision = c.precision;
    if (c.precision == 1) { p.inner_tol = 1e-3; p.refine_maxit = 30; }
    if (c.kase == "dam_break") {
        depth = 0.30;
        p.dt = 0.2 * c.dx / std::sqrt(9.81 * depth);
    } else {
        depth = 0.32;
        p.dt = 0.25 * c.dx / std::sqrt(9.81 * depth);
    }
    return p;
}

// The level-set preset over the cells (1..nx, 1..ny, 1..nz), Fortran order, positive in
// water (14_level_set.f90:26-29): the dam break's water box of 0.25 x 0.30 m (scaled with the
// grid) against the x = 0 wall, or the sloshing tank's surface depth + 0.02 cos(pi x/Lx)
// cos(pi y/Ly).
std::vector<double> ls_preset(const Config& c) {
    std::vector<double> ls((size_t)c.nx * c.ny * c.nz);
    const double lx = c.nx * c.dx, ly = c.ny * c.dx;
    const double a = 0.25 * (c.nx * c.dx / 0.64), h = 0.30 * (c.nz * c.dx / 0.48);
    const double depth = 0.32 * (c.nz * c.dx / 0.64);
    const double pi = std::acos(-1.0);
    size_t q = 0;
    for (int k = 1; k <= c.nz; ++k)
        for (int j = 1; j <= c.ny; ++j)
            for (int i = 1; i <= c.nx; ++i, ++q) {
                const double x = (i - 0.5) * c.dx, y = (j - 0.5) * c.dx, z = (k - 0.5) * c.dx;
                if (c.kase == "dam_break") {
                    if (x <= a && z <= h) {
                        ls[q] = std::fmin(a - x, h - z);
                    } else {
                        const double ox = std::fmax(x - a, 0.0), oz = std::fmax(z - h, 0.0);
                        ls[q] = -std::sqrt(ox * ox + oz * oz);
                    }
                } else {
                    ls[q] = depth + 0.02 * std::cos(pi * x / lx) * std::cos(pi * y / ly) - z;
                }
            }
    return ls;
}

size_t field_size(const suli_params& p, int f) {
    int lo[3], hi[3];
    if (suli_field_extent(&p, f, lo, hi) != SULI_OK) return 0;
    return (size_t)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
}

struct Run {
    suli_ctx* ctx = nullptr;
    ~Run() { suli_destroy(ctx); }
    // a library error ends the run with its message
    bool ok(int rc, const char* what) const {
        if (rc >= 0) return true;
        std::fprintf(stderr, "suli_run: %s failed: %s (%d): %s\n", what, code_name(rc), rc,
                     ctx ? suli_last_error(ctx) : "no context");
        return false;
    }
};

// The reference's loop body (1_principal.f90:64-108) through the per-subroutine entry points.
int step_loop(Run& R, const suli_params& p, int it, suli_step_stats& st) {
    suli_ctx* c = R.ctx;
    double dt = 0.0, ntt = 0.0, a_dt[3] = {0.0, 0.0, 0.0};
    if (!R.ok(suli_get_scalar(c, SULI_S_DT, &dt), "get dt")) return -1;
    if (!R.ok(suli_set_scalar(c, SULI_S_T, it * dt), "set t")) return -1;
    if (!R.ok(suli_get_scalar(c, SULI_S_NTT, &ntt), "get ntt")) return -1;
    for (int q = 0; q < 3; ++q)
        if (!R.ok(suli_get_scalar(c, SULI_S_A_DT1 + q, &a_dt[q]), "get a_dt")) return -1;
    double vol = 0.0;
    if (!R.ok(suli_level_set(c, &vol), "level_set")) return -1;
    if (p.obst_t != 0 && !R.ok(suli_contorno(c, 3), "contorno(3)")) return -1;
    int status = SULI_OK;
    for (int tt = 1; tt <= (int)ntt; ++tt) {
        if (!R.ok(suli_set_dt(c, a_dt[tt - 1]), "set_dt")) return -1;
        if (!R.ok(suli_visco(c), "visco")) return -1;
        if (!R.ok(suli_convdiff(c), "convdiff")) return -1;
        if (!R.ok(suli_tempo(c, tt, it), "tempo")) return -1;
        if (p.wave_t != 0 && !R.ok(suli_boundary_waves(c), "boundary_waves")) return -1;
        if (!R.ok(suli_contorno(c, 2), "contorno(2)")) return -1;
        int n = 0;
        double res = 0.0;
        const int rg = suli_graddin(c, &n, &res);
        if (!R.ok(rg, "graddin")) return -1;
        if (rg > 0) status = rg;   // the reference prints "pulou pressão" and goes on (9_grad.f90:178)
        st.cg_iters[tt - 1] = n;
        st.cg_resid[tt - 1] = res;
        if (!R.ok(suli_posdin(c), "posdin")) return -1;
        if (!R.ok(suli_contorno(c, 1), "contorno(1)")) return -1;
    }
    for (int tt = (int)ntt; tt < 3; ++tt) { st.cg_iters[tt] = 0; st.cg_resid[tt] = 0.0; }
    if (!R.ok(suli_est(c, &st.max_div), "est")) return -1;
    if (!R.ok(suli_get_scalar(c, SULI_S_VOL_INS, &st.vol_ins), "get vol_ins")) return -1;
    st.status = status;
    return status;
}

bool dump_fields(Run& R, const suli_params& p, const std::string& prefix) {
    const int fields[5] = {SULI_F_U, SULI_F_V, SULI_F_W, SULI_F_PRD1, SULI_F_LS};
    const char* names[5] = {"u", "v", "w", "prd1", "ls"};
    for (int q = 0; q < 5; ++q) {
        std::vector<double> a(field_size(p, fields[q]));
        if (!R.ok(suli_download(R.ctx, fields[q], a.data()), "download")) return false;
        const std::string path = prefix + "_" + names[q] + ".bin";
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f || std::fwrite(a.data(), sizeof(double), a.size(), f) != a.size()) {
            std::fprintf(stderr, "suli_run: cannot write %s\n", path.c_str());
            if (f) std::fclose(f);
            return false;
        }
        std::fclose(f);
    }
    return true;
}

}  // namespace

int main(int argc, char** argv) {
    Config cfg;
    if (!parse(argc, argv, cfg)) {
        std::fprintf(stderr,
                     "usage: suli_run [case=dam_break|sloshing] [nx= ny= nz= dx=] [steps=] [print=] "
                     "[mode=loop|step|host] [precision=0|1] [cg_tol=] [div_tol=] [device=] [dump=prefix] "
                     "[preset=file]\n");
        return 1;
    }
    double depth = 0.0;
    const suli_params p = case_params(cfg, depth);
    if (!cfg.preset.empty()) {
        const std::vector<double> ls = ls_preset(cfg);
        FILE* f = std::fopen(cfg.preset.c_str(), "wb");
        const bool ok = f && std::fwrite(&p.dt, sizeof(double), 1, f) == 1 &&
                        std::fwrite(ls.data(), sizeof(double), ls.size(), f) == ls.size();
        if (f) std::fclose(f);
        if (!ok) {
            std::fprintf(stderr, "suli_run: cannot write %s\n", cfg.preset.c_str());
            return 1;
        }
        return 0;
    }
    Run R;
    if (!R.ok(suli_create(&p, cfg.device, &R.ctx), "suli_create")) return 2;
    // set-up (1_principal.f90:46-62): iniciais, the preset, level_set_ini, contorno(1), contorno(3)
    if (!R.ok(suli_iniciais(R.ctx, 0.0), "iniciais")) return 2;
    const std::vector<double> ls0 = ls_preset(cfg);
    if (!R.ok(suli_upload(R.ctx, SULI_F_LS, ls0.data()), "upload ls")) return 2;
    if (!R.ok(suli_level_set_ini(R.ctx), "level_set_ini")) return 2;
    if (!R.ok(suli_contorno(R.ctx, 1), "contorno(1)")) return 2;
    if (!R.ok(suli_contorno(R.ctx, 3), "contorno(3)")) return 2;
    // mode=host: the state lives in these arrays between steps
    const int hf[5] = {SULI_F_U, SULI_F_V, SULI_F_W, SULI_F_PRD1, SULI_F_LS};
    std::vector<std::vector<double>> host;
    const double* hin[5] = {nullptr};
    double* hout[5] = {nullptr};
    if (cfg.mode == "host") {
        host.resize(5);
        for (int q = 0; q < 5; ++q) {
            host[q].resize(field_size(p, hf[q]));
            if (!R.ok(suli_download(R.ctx, hf[q], host[q].data()), "download")) return 2;
            hin[q] = host[q].data();
            hout[q] = host[q].data();
        }
    }
    std::printf("suli_run: case %s %dx%dx%d dx=%g dt=%g mode %s precision %d\n", cfg.kase.c_str(), p.nx, p.ny,
                p.nz, p.dx, p.dt, cfg.mode.c_str(), p.precision);
    for (int it = 1; it <= cfg.steps; ++it) {
        suli_step_stats st;
        std::memset(&st, 0, sizeof(st));
        int rc;
        if (cfg.mode == "loop") {
            rc = step_loop(R, p, it, st);
            if (rc < 0) return 2;
        } else if (cfg.mode == "step") {
            rc = suli_step(R.ctx, it, &st);
            if (!R.ok(rc, "suli_step")) return 2;
        } else {
            rc = suli_step_host(R.ctx, it, 5, hf, hin, 5, hf, hout, &st);
            if (!R.ok(rc, "suli_step_host")) return 2;
        }
        if (it % cfg.print == 0 || it == cfg.steps)
            std::printf("it %6d  t %.6e  cg %d %d %d  resid %.3e  max|div u| %.3e  vol %.12e%s\n", it, it * p.dt,
                        st.cg_iters[0], st.cg_iters[1], st.cg_iters[2],
                        std::fmax(st.cg_resid[0], std::fmax(st.cg_resid[1], st.cg_resid[2])), st.max_div, st.vol_ins,
                        rc > 0 ? "  (Poisson iteration cap)" : "");
    }
    if (!cfg.dump.empty() && !dump_fields(R, p, cfg.dump)) return 2;
    return 0;
}
