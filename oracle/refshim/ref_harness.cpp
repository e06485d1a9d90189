/*
 * Harness around the reference's own CPU hot path (weno/src/update.cpp built
 * with -DUseCPU, GKMflux.cpp, FlowField.cpp, param.cpp), compiled from the
 * reference sources where they lie into oracle/_ref/ref_harness.
 *
 * TEST INFRASTRUCTURE ONLY: it produces golden vectors and the CPU timing
 * baseline.  Nothing in the product library links it.
 *
 * The reference's main (weno/src/Main.cpp:10-49) hard-codes a 4x4x4 process
 * grid and runs to t = 7 t0 through Evolve (update.cpp:41-173); this harness
 * replaces only that driver: a single rank owning the periodic block (or, for
 * timing, a y-slab of it), then the same calls Evolve makes per step:
 * generateSplines + PrintStats (update.cpp:122-124), evolveEulerian
 * (update.cpp:131-133), HaloTransfer (update.cpp:139-141), t += dt.
 *
 * Modes
 *   run  <casedir> <outdir> <nsteps> <cfl> <stats 0|1> <dumps a,b,..> [field 0|1]
 *        Reads <casedir>/InitialConditions/{params,Init000}.  cfl <= 0 keeps
 *        the reference's own dt (cfl macro 0.02, param.h:17); cfl > 0 sets
 *        dt = cfl*dx/maxVAL with maxVAL from the reference's timestep().
 *        Writes W_<step>.bin (5 padded arrays), stats.bin (per stats call:
 *        t/t0 TKE Diss SKEWu SKEWv SKEWw KURTu KURTv KURTw), meta.txt.  With
 *        field 1, the reference's writeField (update.cpp:1305-1319) dumps the
 *        primitives once, at the first step with t >= t0, where Evolve does
 *        (update.cpp:126-129), into <casedir>/Results/Field/Field_0_<iter>.
 *   time <casedir> <nsteps> <slabs> <cfl> [warmup] [slab]
 *        Times evolveEulerian + HaloTransfer on y-slab <slab> (default 0) of a
 *        <slabs>x1x1 process grid, read from InitialConditions/Init<slab>00
 *        as the reference's Initialize_DHIT reads a rank's block
 *        (FlowField.cpp:73-75), after [warmup] untimed steps; prints one
 *        JSON line.  The single-rank MPI stand-in wraps the slab's own halo,
 *        so a slab's step does the work of a rank of that grid.
 *   weno <in> <out>   ApplyWENO (update.cpp:502-625) on packed stencils.
 *   flux <in> <out>   flux (GKMflux.cpp:11-215) on packed interface states.
 *
 * Built with -DUseGPU (oracle/_ref/ref_gpu_harness) the same driver runs the
 * reference's own GPU path instead: update.cpp with -DUseGPU, GPUupdate.cu and
 * GPUAlloc.cu compiled for sm_100a with the reference makefile's nvcc flags
 * (weno/makefileGPU:27-31, arch changed).  evolveEulerian(W, dev) (update.cpp:
 * 179-183) then calls evolve (GPUupdate.cu:65-196), which copies the padded
 * field to the device, runs derivs/flip/flux/update kernels and copies it back.
 * Modes run and time only.
 */
#include <mpi.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <sys/stat.h>
#include <unistd.h>

#include "FlowField.h"
#include "GKMflux.h"
#include "param.h"
#include "update.h"
#ifdef UseGPU
#include <cuda_runtime.h>
#endif

/* File-scope globals of weno/src/update.cpp:7-33 read and written here. */
extern ptype dt, t, maxVAL;
extern int iter;
extern ptype TKE, Diss, SKEWu, SKEWv, SKEWw, KURTu, KURTv, KURTw;

namespace {

struct Halo {
    /* send / receive buffers of the six faces; sizes as in Evolve, update.cpp:75-90
     * (names avoid the reference's single-letter macros, e.g. R in param.h:18) */
    std::vector<double> sW, rW, sE, rE, sS, rS, sN, rN, sB, rB, sF, rF;
    void alloc()
    {
        const size_t lr = (size_t)nt_segy * nt_segz * 3 * 5;
        const size_t ns = (size_t)nt_segx * nt_segz * 3 * 5;
        const size_t fb = (size_t)nt_segx * nt_segy * 3 * 5;
        sW.resize(lr); rW.resize(lr); sE.resize(lr); rE.resize(lr);
        sS.resize(ns); rS.resize(ns); sN.resize(ns); rN.resize(ns);
        sB.resize(fb); rB.resize(fb); sF.resize(fb); rF.resize(fb);
    }
    void exchange(ptype *W[5])
    {
        HaloTransfer(W, sW.data(), rW.data(), sE.data(), rE.data(), sS.data(), rS.data(), sN.data(),
                     rN.data(), sB.data(), rB.data(), sF.data(), rF.data());
    }
};

/* One step of the reference's hot path, as Evolve calls it (update.cpp:131-137). */
struct Stepper {
#ifdef UseGPU
    DevAlloc *dev = nullptr;
    void init()
    {
        dev = new DevAlloc(); /* GPUAlloc.cu:3-17: 50 unchecked cudaMallocs */
        ptype *all[] = {dev->d_W0, dev->d_W1, dev->d_W2, dev->d_W3, dev->d_W4, dev->d_F0x, dev->d_F1x,
                        dev->d_F2x, dev->d_F3x, dev->d_F4x, dev->d_F0y, dev->d_F1y, dev->d_F2y, dev->d_F3y,
                        dev->d_F4y, dev->d_F0z, dev->d_F1z, dev->d_F2z, dev->d_F3z, dev->d_F4z, dev->d_DW0xl,
                        dev->d_DW1xl, dev->d_DW2xl, dev->d_DW3xl, dev->d_DW4xl, dev->d_DW0yl, dev->d_DW1yl,
                        dev->d_DW2yl, dev->d_DW3yl, dev->d_DW4yl, dev->d_DW0zl, dev->d_DW1zl, dev->d_DW2zl,
                        dev->d_DW3zl, dev->d_DW4zl, dev->d_DW0xr, dev->d_DW1xr, dev->d_DW2xr, dev->d_DW3xr,
                        dev->d_DW4xr, dev->d_DW0yr, dev->d_DW1yr, dev->d_DW2yr, dev->d_DW3yr, dev->d_DW4yr,
                        dev->d_DW0zr, dev->d_DW1zr, dev->d_DW2zr, dev->d_DW3zr, dev->d_DW4zr};
        /* refuse to launch anything on a failed allocation */
        const cudaError_t e = cudaGetLastError();
        for (ptype *a : all)
            if (a == nullptr || e != cudaSuccess) {
                fprintf(stderr, "DevAlloc failed: %s\n", cudaGetErrorString(e));
                exit(3);
            }
    }
    void step(ptype *W[5])
    {
        evolveEulerian(W, dev);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            fprintf(stderr, "reference GPU step failed: %s\n", cudaGetErrorString(e));
            exit(3);
        }
    }
#else
    ptype *Fx[5], *Fy[5], *Fz[5];
    void init()
    {
        for (int q = 0; q < 5; ++q) {
            Fx[q] = new ptype[Nt_seg]();
            Fy[q] = new ptype[Nt_seg]();
            Fz[q] = new ptype[Nt_seg]();
        }
    }
    void step(ptype *W[5]) { evolveEulerian(W, Fx, Fy, Fz); }
#endif
};

void setup_block(int slabs, int slab = 0)
{
    nprocs = 1;
    procDim[0] = slabs;
    procDim[1] = 1;
    procDim[2] = 1;
    procId[0] = slab;
    procId[1] = procId[2] = 0;
    myrank_3d = 0;
    GetParams();
    segment();
}

void write_padded(const std::string &path, ptype *W[5])
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) { perror(path.c_str()); exit(2); }
    for (int q = 0; q < 5; ++q) fwrite(W[q], sizeof(double), (size_t)Nt_seg, f);
    fclose(f);
}

std::vector<int> parse_list(const char *s)
{
    std::vector<int> v;
    std::string str(s);
    size_t p = 0;
    while (p < str.size()) {
        size_t q = str.find(',', p);
        if (q == std::string::npos) q = str.size();
        if (q > p) v.push_back(atoi(str.substr(p, q - p).c_str()));
        p = q + 1;
    }
    return v;
}

int mode_run(int argc, char **argv)
{
    if (argc < 8) { fprintf(stderr, "run <casedir> <outdir> <nsteps> <cfl> <stats> <dumps>\n"); return 2; }
    const std::string outdir = argv[3];
    const int nsteps = atoi(argv[4]);
    const double cfl_run = atof(argv[5]);
    const int do_stats = atoi(argv[6]);
    const std::vector<int> dumps = parse_list(argv[7]);
    const int do_field = argc > 8 ? atoi(argv[8]) : 0;
    if (chdir(argv[2]) != 0) { perror("chdir"); return 2; }

    setup_block(1);
    ptype *W[5];
    for (int q = 0; q < 5; ++q) W[q] = new ptype[Nt_seg]();
    Stepper stepper;
    stepper.init();
    ptype *den = new ptype[Nt_seg], *u = new ptype[Nt_seg], *v = new ptype[Nt_seg],
          *w = new ptype[Nt_seg], *p = new ptype[Nt_seg];
    UBspline_3d_d *splinep[5];
    Halo halo;
    halo.alloc();

    Initialize_DHIT(W);
    halo.exchange(W);
    timestep(W);
    const double dt_reference = dt;
    if (cfl_run > 0) dt = cfl_run * dx / maxVAL;
    t = 0;
    iter = 1;

    FILE *fs = fopen((outdir + "/stats.bin").c_str(), "wb");
    auto stats = [&]() {
        generateSplines(W, splinep, den, u, v, w, p);
        PrintStats(W, splinep);
        for (int q = 0; q < 5; ++q) destroy_Bspline(splinep[q]);
        const double rec[9] = {t / t0, TKE, Diss, SKEWu, SKEWv, SKEWw, KURTu, KURTv, KURTw};
        fwrite(rec, sizeof(double), 9, fs);
    };
    auto dump = [&](int s) {
        for (int d : dumps)
            if (d == s) write_padded(outdir + "/W_" + std::to_string(s) + ".bin", W);
    };

    int field_done = 0;
    auto field = [&]() { // Evolve's one-time dump, update.cpp:126-129
        if (!do_field || field_done || !(t >= t0)) return;
        mkdir("Results", 0755);
        mkdir("Results/Field", 0755);
        generateSplines(W, splinep, den, u, v, w, p);
        writeField(den, u, v, w, p);
        for (int q = 0; q < 5; ++q) destroy_Bspline(splinep[q]);
        field_done = 1;
    };

    for (int s = 0; s < nsteps; ++s) {
        if (do_stats) stats();
        field();
        dump(s);
        stepper.step(W);
        halo.exchange(W);
        t += dt;
        iter++;
    }
    if (do_stats) stats();
    dump(nsteps);
    fclose(fs);

    FILE *fm = fopen((outdir + "/meta.txt").c_str(), "w");
    fprintf(fm, "nc %d\nnt %d\ndx %.17g\ndt %.17g\ndt_reference %.17g\nmaxVAL %.17g\n", nc, nt, dx, dt,
            dt_reference, maxVAL);
    fprintf(fm, "gam %.17g\nK %d\nT0 %.17g\nmu0 %.17g\nden0 %.17g\np0 %.17g\nMt %.17g\nRe %.17g\nt0 %.17g\n",
            gam, K, T0, mu0, den0, p0, Mt, Re, t0);
    fclose(fm);
    return 0;
}

int mode_time(int argc, char **argv)
{
    if (argc < 6) { fprintf(stderr, "time <casedir> <nsteps> <slabs> <cfl> [warmup] [slab]\n"); return 2; }
    const int nsteps = atoi(argv[3]);
    const int slabs = atoi(argv[4]);
    const double cfl_run = atof(argv[5]);
    const int warmup = argc > 6 ? atoi(argv[6]) : 0;
    const int slab = argc > 7 ? atoi(argv[7]) : 0;
    if (slab < 0 || slab >= slabs) { fprintf(stderr, "slab out of range\n"); return 2; }
    if (chdir(argv[2]) != 0) { perror("chdir"); return 2; }
    setup_block(slabs, slab);
    ptype *W[5];
    for (int q = 0; q < 5; ++q) W[q] = new ptype[Nt_seg]();
    Stepper stepper;
    stepper.init();
    Halo halo;
    halo.alloc();
    Initialize_DHIT(W);
    halo.exchange(W);
    timestep(W);
    if (cfl_run > 0) dt = cfl_run * dx / maxVAL;
    for (int s = 0; s < warmup; ++s) {
        stepper.step(W);
        halo.exchange(W);
    }
    double tot = 0, tstep = 0;
    for (int s = 0; s < nsteps; ++s) {
        auto a = std::chrono::steady_clock::now();
        stepper.step(W);
        auto m = std::chrono::steady_clock::now();
        halo.exchange(W);
        auto b = std::chrono::steady_clock::now();
        tot += std::chrono::duration<double>(b - a).count();
        tstep += std::chrono::duration<double>(m - a).count();
    }
    /* seconds: step + halo exchange; step_seconds: evolveEulerian alone (on the GPU
     * path: evolve, i.e. its host<->device copies and kernels) */
    printf("{\"cells\": %d, \"nc\": %d, \"slab\": [%d, %d, %d], \"slab_index\": %d, \"steps\": %d, "
           "\"seconds\": %.9g, \"step_seconds\": %.9g, \"cell_updates_per_s\": %.9g}\n",
           Nc_seg, nc, nc_segy, nc_segx, nc_segz, slab, nsteps, tot, tstep, (double)Nc_seg * nsteps / tot);
    return 0;
}

std::vector<double> read_blob(const char *path, int &n, std::vector<double> &hdr, int nhdr)
{
    FILE *f = fopen(path, "rb");
    if (!f) { perror(path); exit(2); }
    int32_t nn;
    if (fread(&nn, 4, 1, f) != 1) exit(2);
    n = nn;
    hdr.resize(nhdr);
    if (nhdr && fread(hdr.data(), 8, nhdr, f) != (size_t)nhdr) exit(2);
    std::vector<double> rest;
    double x;
    while (fread(&x, 8, 1, f) == 1) rest.push_back(x);
    fclose(f);
    return rest;
}

#ifdef UseCPU
int mode_weno(int argc, char **argv)
{
    if (argc < 4) return 2;
    int n;
    std::vector<double> hdr;
    std::vector<double> in = read_blob(argv[2], n, hdr, 1);
    gam = hdr[0];
    if ((int)in.size() != n * 30) { fprintf(stderr, "weno: bad input size\n"); return 2; }
    std::vector<double> out((size_t)n * 10);
    for (int c = 0; c < n; ++c) {
        double s[6][5];
        for (int a = 0; a < 6; ++a)
            for (int q = 0; q < 5; ++q) s[a][q] = in[(size_t)c * 30 + a * 5 + q];
        double wl[5], wr[5];
        ApplyWENO(s[0], s[1], s[2], s[3], s[4], s[5], wl, wr);
        for (int q = 0; q < 5; ++q) {
            out[(size_t)c * 10 + q] = wl[q];
            out[(size_t)c * 10 + 5 + q] = wr[q];
        }
    }
    FILE *f = fopen(argv[3], "wb");
    fwrite(out.data(), 8, out.size(), f);
    fclose(f);
    return 0;
}

int mode_flux(int argc, char **argv)
{
    if (argc < 4) return 2;
    int n;
    std::vector<double> hdr;
    std::vector<double> in = read_blob(argv[2], n, hdr, 2);
    gam = hdr[0];
    K = (int)hdr[1];
    if ((int)in.size() != n * 53) { fprintf(stderr, "flux: bad input size\n"); return 2; }
    std::vector<double> out((size_t)n * 5);
    for (int c = 0; c < n; ++c) {
        double v[10][5];
        const double *r = &in[(size_t)c * 53];
        for (int a = 0; a < 10; ++a)
            for (int q = 0; q < 5; ++q) v[a][q] = r[a * 5 + q];
        double F[5];
        flux(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9], r[50], r[51], r[52], F);
        for (int q = 0; q < 5; ++q) out[(size_t)c * 5 + q] = F[q];
    }
    FILE *f = fopen(argv[3], "wb");
    fwrite(out.data(), 8, out.size(), f);
    fclose(f);
    return 0;
}
#endif

} // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: ref_harness run|time|weno|flux ...\n");
        return 2;
    }
    const std::string mode = argv[1];
    if (mode == "run") return mode_run(argc, argv);
    if (mode == "time") return mode_time(argc, argv);
#ifdef UseCPU
    if (mode == "weno") return mode_weno(argc, argv);
    if (mode == "flux") return mode_flux(argc, argv);
#endif
    fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
}
