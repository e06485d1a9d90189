// gks_dns: the reference's run driver (weno/src/Main.cpp:10-49 and Evolve,
// update.cpp:41-173) on one B200 through the gks_b200 C ABI.
//
// Same inputs (InitialConditions/params, Init000 in the case directory), same
// banner, same statistics line per step, same one-time field dump at t >= t0,
// same loop (dt from the CFL condition once at the start, step while
// t <= tmax = 7 t0).  The state stays on the device between steps; the halo
// exchange of the reference is the periodic wrap inside the kernels.
//
// usage: gks_dns [options]
//   --case DIR         case directory (default .)
//   --precision P      fp64 (default) | mixed
//   --cfl C            CFL number (default 0.02, param.h:17)
//   --tmax T           stop time in eddy turnover times t0 (default 7, param.h:62)
//   --steps N          stop after N steps instead
//   --dt-every-step    recompute dt every step (the reference computes it once)
//   --fix-zsweep       z-sweep transverse slopes along the rotated axes
//   --direct-energy    WENO on rho E (the reference GPU kernel's choice)
//   --gpu-prandtl      no 1/Pr factor in the slope solve (the reference GPU kernel)
//   --visc-power E     mu = mu0 (T/T0)^E instead of Sutherland's law
//   --stats-every N    statistics line every N steps (default 1)
//   --no-field         skip the Results/Field dump
//   --reinit PATH      write the final state in the Init layout to PATH
//                      (the reference's WriteReInit targets InitialCondition/, a typo)
//   --particles        track the particles of InitialConditions/unirand (numparticles
//                      from particleCount): every step, their properties from the
//                      current state (generateSplines + getParticleProp) and a move by
//                      dt (Particle::track) before the field's step, and at every
//                      statistics line a line "particles t/t0 TKE SijSij SKEWu SKEWw N"
//                      (GetParticleStats).  The reference defines this tracker
//                      (update.cpp:1082-1303) but its Evolve never calls it.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "gks_driver_io.h"

namespace {

struct Options {
    std::string casedir = ".";
    int precision = GKS_FP64;
    double cfl = 0.02;
    double tmax_t0 = 7.0;
    long steps = -1;
    bool dt_every_step = false;
    int flags = 0;
    bool gpu_prandtl = false;
    int visc_law = GKS_VISC_SUTHERLAND;
    double visc_exp = 0.76;
    int stats_every = 1;
    bool field = true;
    std::string reinit;
    bool particles = false;
};

int usage(const char *msg)
{
    fprintf(stderr, "gks_dns: %s (see the header of gks_dns.cpp for options)\n", msg);
    return 2;
}

bool parse(int argc, char **argv, Options &o, std::string &err)
{
    for (int a = 1; a < argc; ++a) {
        const std::string s = argv[a];
        auto next = [&](const char *name) -> const char * {
            if (a + 1 >= argc) {
                err = std::string("missing value for ") + name;
                return nullptr;
            }
            return argv[++a];
        };
        const char *v = nullptr;
        if (s == "--case") { if (!(v = next("--case"))) return false; o.casedir = v; }
        else if (s == "--precision") {
            if (!(v = next("--precision"))) return false;
            if (!strcmp(v, "fp64")) o.precision = GKS_FP64;
            else if (!strcmp(v, "mixed")) o.precision = GKS_MIXED;
            else { err = "precision must be fp64 or mixed"; return false; }
        }
        else if (s == "--cfl") { if (!(v = next("--cfl"))) return false; o.cfl = atof(v); }
        else if (s == "--tmax") { if (!(v = next("--tmax"))) return false; o.tmax_t0 = atof(v); }
        else if (s == "--steps") { if (!(v = next("--steps"))) return false; o.steps = atol(v); }
        else if (s == "--dt-every-step") o.dt_every_step = true;
        else if (s == "--fix-zsweep") o.flags |= GKS_FIX_ZSWEEP;
        else if (s == "--direct-energy") o.flags |= GKS_DIRECT_ENERGY;
        else if (s == "--gpu-prandtl") o.gpu_prandtl = true;
        else if (s == "--visc-power") { if (!(v = next("--visc-power"))) return false; o.visc_law = GKS_VISC_POWER; o.visc_exp = atof(v); }
        else if (s == "--stats-every") { if (!(v = next("--stats-every"))) return false; o.stats_every = atoi(v); }
        else if (s == "--no-field") o.field = false;
        else if (s == "--reinit") { if (!(v = next("--reinit"))) return false; o.reinit = v; }
        else if (s == "--particles") o.particles = true;
        else { err = "unknown option " + s; return false; }
    }
    if (!(o.cfl > 0) || o.stats_every < 1) {
        err = "cfl must be positive and --stats-every at least 1";
        return false;
    }
    return true;
}

int die(gks_ctx *ctx, int rc, const char *what)
{
    fprintf(stderr, "gks_dns: %s failed (%d): %s\n", what, rc, gks_last_error(ctx));
    gks_destroy(ctx);
    return 1;
}

} // namespace

int main(int argc, char **argv)
{
    Options o;
    std::string err;
    if (!parse(argc, argv, o, err)) return usage(err.c_str());

    gksdrv::RunParams p;
    if (!(err = gksdrv::read_params(o.casedir, p)).empty()) return usage(err.c_str());
    gksdrv::Field W;
    if (!(err = gksdrv::read_init(o.casedir, p, W)).empty()) return usage(err.c_str());
    std::vector<double> xyz[3]; // initial particle positions x0, y0, z0
    if (o.particles && !(err = gksdrv::read_unirand(o.casedir, p, xyz)).empty()) return usage(err.c_str());

    const double prandtl = 0.7; // param.h:16
    gksdrv::print_params(p, o.cfl, prandtl);

    gks_phys ph{};
    ph.nc = p.nc;
    ph.K = p.K();
    ph.visc_law = o.visc_law;
    ph.gam = p.gam;
    ph.gas_r = p.R;
    ph.T0 = p.T0();
    ph.mu0 = p.mu0;
    ph.visc_exp = o.visc_exp;
    ph.pr_factor = o.gpu_prandtl ? 1.0 : 1 / prandtl; // GPUupdate.cu:839 / GKMflux.cpp:289
    ph.p0 = p.p0;
    ph.den0 = p.rho0;
    ph.Mt = p.Mt;
    ph.t0 = p.t0;

    gks_ctx *ctx = nullptr;
    int rc = gks_create(&ctx, 1, &ph, o.precision, o.flags);
    if (rc) {
        fprintf(stderr, "gks_dns: gks_create failed (%d); is a CUDA device available?\n", rc);
        return 1;
    }
    if ((rc = gks_upload(ctx, 0, W.ptr))) return die(ctx, rc, "upload");
    if ((rc = gks_check(ctx))) return die(ctx, rc, "initial state check");
    double dt = 0;
    if ((rc = gks_timestep(ctx, 0, o.cfl, &dt))) return die(ctx, rc, "timestep");
    if (o.particles) { // locateParticles (update.cpp:1269-1292) on one rank
        if ((rc = gks_particles_locate(ctx, 0, p.particles, xyz[0].data(), xyz[1].data(), xyz[2].data())))
            return die(ctx, rc, "particles_locate");
    }
    auto particle_line = [&](double t_over_t0) -> int {
        gks_particle_stats_out ps;
        const int r = gks_particles_stats(ctx, 0, &ps);
        if (!r)
            printf("particles %.6f %.15e %.15e %.15e %.15e %lld\n", t_over_t0, ps.tke, ps.sijsij, ps.skew_u, ps.skew_w,
                   ps.count);
        return r;
    };

    const double tmax = o.tmax_t0 * p.t0;
    double t = 0;
    int iter = 1;
    bool dumped = false;
    long step = 0;
    gks_stats_out st;
    double step_seconds = 0;
    auto done = [&]() { return o.steps >= 0 ? step >= o.steps : !(t <= tmax); };
    while (!done()) {
        if (step % o.stats_every == 0) {
            if ((rc = gks_stats(ctx, 0, &st))) return die(ctx, rc, "stats");
            gksdrv::print_stats_line(t / p.t0, st);
        }
        if (o.field && t >= p.t0 && !dumped) { // update.cpp:126-129
            if ((rc = gks_download(ctx, 0, W.ptr))) return die(ctx, rc, "download");
            if (!(err = gksdrv::write_field(o.casedir + "/Results/Field", 0, iter, p, W)).empty())
                fprintf(stderr, "gks_dns: %s\n", err.c_str());
            dumped = true;
        }
        if (o.particles) {
            if ((rc = gks_particles_props(ctx, 0))) return die(ctx, rc, "particles_props");
            if (step % o.stats_every == 0 && (rc = particle_line(t / p.t0))) return die(ctx, rc, "particles_stats");
            if ((rc = gks_particles_track(ctx, 0, dt))) return die(ctx, rc, "particles_track");
        }
        const auto a = std::chrono::steady_clock::now();
        if ((rc = gks_step(ctx, 1))) return die(ctx, rc, "step");
        if ((rc = gks_sync(ctx))) return die(ctx, rc, "step");
        step_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
        if (o.dt_every_step && (rc = gks_timestep(ctx, 0, o.cfl, &dt))) return die(ctx, rc, "timestep");
        t += dt;
        ++iter;
        ++step;
    }
    if ((rc = gks_stats(ctx, 0, &st))) return die(ctx, rc, "stats");
    gksdrv::print_stats_line(t / p.t0, st);
    if (o.particles) {
        if ((rc = gks_particles_props(ctx, 0))) return die(ctx, rc, "particles_props");
        if ((rc = particle_line(t / p.t0))) return die(ctx, rc, "particles_stats");
    }
    if (!o.reinit.empty()) {
        if ((rc = gks_download(ctx, 0, W.ptr))) return die(ctx, rc, "download");
        if (!(err = gksdrv::write_reinit(o.reinit, p, W)).empty()) fprintf(stderr, "gks_dns: %s\n", err.c_str());
    }
    const double cells = (double)p.nc * p.nc * p.nc;
    fprintf(stderr, "gks_dns: %ld steps, %.3f s in steps, %.4e cell-updates/s\n", step, step_seconds,
            step_seconds > 0 ? cells * step / step_seconds : 0.0);
    gks_destroy(ctx);
    return 0;
}
