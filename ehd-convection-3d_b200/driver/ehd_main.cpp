// ehd_main.cpp -- command-line driver of the EHD step, the host program the
// reference's main() (main.cu:23-314) is, on top of the C ABI (include/ehd.h).
//
// The reference fixes everything at compile time (LBM.h:30-86); here the same
// quantities are options.  The loop keeps main.cu's structure and output
// files: data.dat (Tecplot zones, main.cu:167-168, 210-212, 268), the "<t>.dat"
// uz files for DMD every --dmd-every steps (main.cu:213-224), umax.dat
// (record_umax, main.cu:236), the "Current = " line (main.cu:227-231), the
// performance report (main.cu:242-266) and data_end.dat (main.cu:275-277).
//
//   ehd_sim [--nx 122] [--ny 122] [--nz 101] [--lx L] [--ly L]
//           [--T t --M m --C c --Fe fe | --nu .. --K .. --charge0 .. --diffu ..]
//           [--lambda-f 1/12] [--lambda-g 1e-6] [--uw 0] [--exf 0]
//           [--steps 1000] [--save-every N] [--current-every 1000] [--dmd-every 50000]
//           [--precision fp64|fp32|fp16|bf16] [--restart] [--hydrostatic NSTEPS]
//           [--seed 0] [--amp 1e-3] [--checkpoint PATH] [--resume PATH] [--no-output]
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ehd.h"

namespace {

struct Options {
    int nx = 122, ny = 122, nz = 101;
    double lx = -1, ly = -1;
    double T = -1, M = -1, C = -1, Fe = -1;
    double nu = 0.0251004, K = 2.5e-5, charge0 = 10.0, diffu = 6.25e-5;
    double lambda_f = 1.0 / 12.0, lambda_g = 1.0e-6, uw = 0.0, exf = 0.0;
    long long steps = 1000, save_every = 0, current_every = 1000, dmd_every = 50000;
    int precision = EHD_PREC_FP64;
    bool restart = false, no_output = false;
    long long hydrostatic = -1;
    unsigned long long seed = 0;
    double amp = 1e-3;
    std::string checkpoint, resume;
};

int die(const char *what) {
    std::fprintf(stderr, "ehd_sim: %s: %s\n", what, ehd_last_error());
    return 1;
}

bool parse(int argc, char **argv, Options &o) {
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&](double &d) {
            if (i + 1 >= argc) return false;
            d = std::atof(argv[++i]);
            return true;
        };
        auto ival = [&](long long &v) {
            if (i + 1 >= argc) return false;
            v = std::atoll(argv[++i]);
            return true;
        };
        double d;
        long long v;
        if (a == "--nx" && ival(v)) o.nx = (int)v;
        else if (a == "--ny" && ival(v)) o.ny = (int)v;
        else if (a == "--nz" && ival(v)) o.nz = (int)v;
        else if (a == "--lx" && val(d)) o.lx = d;
        else if (a == "--ly" && val(d)) o.ly = d;
        else if (a == "--T" && val(d)) o.T = d;
        else if (a == "--M" && val(d)) o.M = d;
        else if (a == "--C" && val(d)) o.C = d;
        else if (a == "--Fe" && val(d)) o.Fe = d;
        else if (a == "--nu" && val(d)) o.nu = d;
        else if (a == "--K" && val(d)) o.K = d;
        else if (a == "--charge0" && val(d)) o.charge0 = d;
        else if (a == "--diffu" && val(d)) o.diffu = d;
        else if (a == "--lambda-f" && val(d)) o.lambda_f = d;
        else if (a == "--lambda-g" && val(d)) o.lambda_g = d;
        else if (a == "--uw" && val(d)) o.uw = d;
        else if (a == "--exf" && val(d)) o.exf = d;
        else if (a == "--steps" && ival(v)) o.steps = v;
        else if (a == "--save-every" && ival(v)) o.save_every = v;
        else if (a == "--current-every" && ival(v)) o.current_every = v;
        else if (a == "--dmd-every" && ival(v)) o.dmd_every = v;
        else if (a == "--hydrostatic" && ival(v)) o.hydrostatic = v;
        else if (a == "--seed" && ival(v)) o.seed = (unsigned long long)v;
        else if (a == "--amp" && val(d)) o.amp = d;
        else if (a == "--restart") o.restart = true;
        else if (a == "--no-output") o.no_output = true;
        else if (a == "--checkpoint" && i + 1 < argc) o.checkpoint = argv[++i];
        else if (a == "--resume" && i + 1 < argc) o.resume = argv[++i];
        else if (a == "--precision" && i + 1 < argc) {
            const std::string p = argv[++i];
            o.precision = p == "fp32" ? EHD_PREC_FP32
                        : p == "fp16" ? EHD_PREC_FP16
                        : p == "bf16" ? EHD_PREC_BF16 : EHD_PREC_FP64;
        } else {
            std::fprintf(stderr, "ehd_sim: unknown or incomplete option %s\n", a.c_str());
            return false;
        }
    }
    return true;
}

// umax of the current fields as record_umax (LBM.cu:1673-1713) reports it
double umax_of(ehd_ctx *ctx) {
    ehd_diag d;
    return ehd_diagnostics(ctx, &d) == EHD_OK ? d.umax : NAN;
}

}  // namespace

int main(int argc, char **argv) {
    Options o;
    if (!parse(argc, argv, o)) return 2;
    ehd_params P{};
    P.nx = o.nx;
    P.ny = o.ny;
    P.nz = o.nz;
    P.lz = 1.0;
    P.dz = P.lz / (o.nz - 1);
    P.lx = o.lx > 0 ? o.lx : o.nx * P.dz;  // LBM.h:40-45: dx = dy = dz
    P.ly = o.ly > 0 ? o.ly : o.ny * P.dz;
    P.dx = P.lx / o.nx;
    P.dy = P.ly / o.ny;
    P.cfl = 0.01;
    P.dt = P.cfl * P.dz;
    P.rho0 = 1600.0;
    P.voltage = 1.0e4;
    P.eps = 1.0e-4;
    P.nu = o.nu;
    P.K = o.K;
    P.charge0 = o.charge0;
    P.diffu = o.diffu;
    P.uw = o.uw;
    P.exf = o.exf;
    P.lambda_f = o.lambda_f;
    P.lambda_g = o.lambda_g;
    if (o.T > 0 && ehd_params_from_groups(&P, o.T, o.M, o.C, o.Fe) != EHD_OK) return die("parameters");
    double T, M, C, Fe;
    ehd_groups_from_params(&P, &T, &M, &C, &Fe);  // compute_parameters, LBM.cu:1356-1379
    std::printf("Simulating 3D electrohydrodynamics vortices\n");
    std::printf("      domain size: %dx%dx%d\n", P.nx, P.ny, P.nz);
    std::printf("                T: %g\n                M: %g\n                C: %g\n"
                "               Fe: %g\n",
                T, M, C, Fe);
    std::printf("            uwall: %g\n   External force: %g\n        timesteps: %lld\n\n",
                P.uw, P.exf, o.steps);

    ehd_config cfg{};
    cfg.precision = o.precision;
    ehd_ctx *ctx = nullptr;
    if (ehd_create(&P, &cfg, &ctx) != EHD_OK) return die("create");
    double i0 = 0.0;
    if (!o.resume.empty()) {
        if (ehd_restore(ctx, o.resume.c_str()) != EHD_OK) return die("resume");
    } else if (o.restart) {
        if (ehd_read_data_end(ctx, "data_end.dat") != EHD_OK) return die("read data_end.dat");
    } else if (o.hydrostatic >= 0) {
        // the column's own state broadcast over the plane, plus seeded noise
        ehd_config c64{};
        c64.precision = EHD_PREC_FP64;
        ehd_ctx *col = nullptr;
        if (ehd_hydrostatic_column(&P, &c64, (int)o.hydrostatic, &col, &i0) != EHD_OK)
            return die("hydrostatic column");
        const int rc = ehd_set_state_from_column(ctx, col, o.seed, o.amp);
        ehd_destroy(col);
        if (rc != EHD_OK) return die("state from column");
        ehd_set_reference_current(ctx, i0);
    } else if (ehd_initialize(ctx) != EHD_OK) {
        return die("initialize");
    }
    if (!o.no_output && ehd_write_tecplot(ctx, "data.dat", 1) != EHD_OK) return die("data.dat");
    FILE *fumax = o.no_output ? nullptr : std::fopen("umax.dat", "w");

    const auto t0 = std::chrono::steady_clock::now();
    ehd_diag d{};
    for (long long i = 0; i < o.steps; ++i) {
        if (ehd_step(ctx, 1) != EHD_OK) return die("step");
        if (o.save_every > 0 && i % o.save_every == 1 && !o.no_output)
            if (ehd_write_tecplot(ctx, "data.dat", 0) != EHD_OK) return die("data.dat");
        if (o.dmd_every > 0 && i % o.dmd_every == 1 && !o.no_output) {
            ehd_diag dd{};
            if (ehd_diagnostics(ctx, &dd) != EHD_OK) return die("diagnostics");
            std::printf("Iteration: %lld, physical time: %g.\n", i, dd.time);
            char name[128];
            std::snprintf(name, sizeof(name), "%g.dat", dd.time);
            if (ehd_write_dmd(ctx, name) != EHD_OK) return die("DMD file");
        }
        if (o.current_every > 0 && i % o.current_every == 1) {
            if (ehd_diagnostics(ctx, &d) != EHD_OK) return die("diagnostics");
            if (i0 != 0.0) std::printf("Current = %g  Nu_e = %g\n", d.current, d.nu_e);
            else std::printf("Current = %g\n", d.current);
            if (fumax) std::fprintf(fumax, "%10.6f %10.6f\n", d.time, d.umax);
            if (d.nonfinite) {
                std::fprintf(stderr, "ehd_sim: non-finite field at step %lld\n", i);
                return 3;
            }
        }
    }
    if (ehd_synchronize(ctx) != EHD_OK) return die("synchronize");
    const double runtime =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const double speed = (double)o.steps * (double)P.nx * P.ny * P.nz / (1e6 * runtime);
    std::printf(" ----- performance information -----\n");
    std::printf("               timesteps: %lld\n", o.steps);
    std::printf("           clock runtime: %.3f (s)\n", runtime);
    std::printf("                   speed: %.2f (Mlups)\n", speed);
    if (!o.no_output) {
        if (ehd_write_tecplot(ctx, "data.dat", 0) != EHD_OK) return die("data.dat");
        if (fumax) std::fprintf(fumax, "%10.6f %10.6f\n", d.time, umax_of(ctx));
        if (ehd_write_data_end(ctx, "data_end.dat") != EHD_OK) return die("data_end.dat");
    }
    if (fumax) std::fclose(fumax);
    if (!o.checkpoint.empty() && ehd_checkpoint(ctx, o.checkpoint.c_str()) != EHD_OK)
        return die("checkpoint");
    ehd_destroy(ctx);
    return 0;
}
