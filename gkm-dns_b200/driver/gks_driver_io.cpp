// Reference-compatible inputs, outputs and printing (formats in gks_driver_io.h).
#include "gks_driver_io.h"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sys/stat.h>

namespace gksdrv {

double RunParams::dx() const { return 2.0 * (std::atan(1.0) * 4.0) / nc; }

void Field::alloc(int n)
{
    nc = n;
    const size_t N = nt() * nt() * nt();
    for (int q = 0; q < 5; ++q) {
        w[q].assign(N, 0.0);
        ptr[q] = w[q].data();
    }
}

std::string read_params(const std::string &casedir, RunParams &p)
{
    const std::string path = casedir + "/InitialConditions/params";
    std::ifstream in(path, std::ios::binary);
    if (!in) return "cannot open " + path;
    int n = 0;
    double v[7];
    in.read((char *)&n, sizeof(int));
    in.read((char *)v, sizeof(v));
    if (!in) return path + " is shorter than 4 + 7*8 bytes";
    if (n < 4) return path + ": grid size must be at least 4";
    p.nc = n;
    p.gam = v[0];
    p.rho0 = v[1];
    p.Mt = v[2];
    p.Re = v[3];
    p.mu0 = v[4];
    p.p0 = v[5];
    p.t0 = v[6];
    if (!(p.gam > 1.0) || !(p.rho0 > 0) || !(p.p0 > 0) || !(p.t0 > 0) || !(p.mu0 >= 0))
        return path + ": non-physical constants";
    std::ifstream pc(casedir + "/InitialConditions/particleCount", std::ios::binary);
    if (pc) pc.read((char *)&p.particles, sizeof(int));
    return "";
}

std::string read_unirand(const std::string &casedir, const RunParams &p, std::vector<double> xyz[3])
{
    const std::string path = casedir + "/InitialConditions/unirand";
    if (p.particles < 1) return casedir + "/InitialConditions/particleCount holds no particles";
    std::ifstream in(path, std::ios::binary);
    if (!in) return "cannot open " + path;
    for (int q = 0; q < 3; ++q) {
        xyz[q].resize(p.particles);
        in.read((char *)xyz[q].data(), p.particles * sizeof(double));
        if (!in) return path + " is shorter than 3 * numparticles doubles";
    }
    return "";
}

std::string read_init(const std::string &casedir, const RunParams &p, Field &W)
{
    const std::string path = casedir + "/InitialConditions/Init000";
    std::ifstream in(path, std::ios::binary);
    if (!in) return "cannot open " + path;
    const size_t nc = p.nc, Nc = nc * nc * nc;
    std::vector<double> prim[5];
    for (int q = 0; q < 5; ++q) {
        prim[q].resize(Nc);
        in.read((char *)prim[q].data(), Nc * sizeof(double));
        if (!in) return path + " is shorter than 5*nc^3 doubles";
    }
    W.alloc(p.nc);
    const int n = p.nc;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < n; ++k) {
                const size_t J = (size_t)k * n * n + (size_t)i * n + j; // FlowField.cpp:95
                const double u = prim[0][J], v = prim[1][J], w = prim[2][J], d = prim[3][J], pr = prim[4][J];
                const double vsq = (u * u + v * v + w * w);
                const size_t I = W.idx(j + 3, i + 3, k + 3);
                W.w[0][I] = d; // FlowField.cpp:97-102
                W.w[1][I] = u * d;
                W.w[2][I] = v * d;
                W.w[3][I] = w * d;
                W.w[4][I] = d * (pr / (d * (p.gam - 1.0)) + 0.5 * vsq);
            }
    return "";
}

std::string write_reinit(const std::string &path, const RunParams &p, const Field &W)
{
    // WriteReInit (update.cpp:1352-1391): primitives u, v, w, rho, p in the Init layout
    const int n = p.nc;
    const size_t Nc = (size_t)n * n * n;
    std::vector<double> out[5];
    for (auto &o : out) o.resize(Nc);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < n; ++k) {
                const size_t I = W.idx(j + 3, i + 3, k + 3);
                const size_t J = (size_t)k * n * n + (size_t)i * n + j;
                const double d = W.w[0][I];
                const double u = W.w[1][I] / d, v = W.w[2][I] / d, w = W.w[3][I] / d;
                const double vsq = (u * u + v * v + w * w);
                out[0][J] = u;
                out[1][J] = v;
                out[2][J] = w;
                out[3][J] = d;
                out[4][J] = (d * (p.gam - 1)) * (W.w[4][I] / d - 0.5 * vsq);
            }
    std::ofstream f(path, std::ios::binary);
    if (!f) return "cannot write " + path;
    for (auto &o : out) f.write((const char *)o.data(), Nc * sizeof(double));
    return f ? "" : "short write to " + path;
}

static void mkdirs(const std::string &dir)
{
    std::string acc;
    for (size_t i = 0; i <= dir.size(); ++i) {
        if (i == dir.size() || dir[i] == '/') {
            if (!acc.empty()) mkdir(acc.c_str(), 0755);
        }
        if (i < dir.size()) acc += dir[i];
    }
}

std::string write_field(const std::string &dir, int rank, int iter, const RunParams &p, const Field &W)
{
    mkdirs(dir);
    char name[256];
    snprintf(name, sizeof(name), "%s/Field_%i_%i", dir.c_str(), rank, iter);
    FILE *f = fopen(name, "w");
    if (!f) return std::string("cannot write ") + name;
    const int n = p.nc;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < n; ++k) {
                const size_t I = W.idx(j + 3, i + 3, k + 3);
                const double d = W.w[0][I];
                const double u = W.w[1][I] / d, v = W.w[2][I] / d, w = W.w[3][I] / d;
                const double vsq = u * u + v * v + w * w;
                const double pr = (d * (p.gam - 1)) * (W.w[4][I] / d - 0.5 * vsq);
                fprintf(f, "%d %d %d %.15e %.15e %.15e %.15e %.15e\n", i, j, k, d, u, v, w, pr);
            }
    fclose(f);
    return "";
}

void print_params(const RunParams &p, double cfl, double prandtl)
{
    // PrintParams, FlowField.cpp:305-334 (one block: nc_seg = nc, 1 x 1 x 1)
    using std::cout;
    using std::endl;
    cout << endl << "GKM DNS DHIT" << endl;
    cout << "Initializing Field ....." << endl;
    cout << "______________________________" << endl << endl;
    cout << "nc            =  " << p.nc << endl;
    cout << "nc_segy       =  " << p.nc << endl;
    cout << "nc_segx       =  " << p.nc << endl;
    cout << "nc_segz       =  " << p.nc << endl;
    cout << "T0            =  " << p.T0() << endl;
    cout << "Mt            =  " << p.Mt << endl;
    cout << "Re            =  " << p.Re << endl;
    cout << "dx            =  " << p.dx() << endl;
    cout << "eddy time     =  " << p.t0 << endl;
    cout << "p0            =  " << p.p0 << endl;
    cout << "den0          =  " << p.rho0 << endl;
    cout << "gam           =  " << p.gam << endl;
    cout << "mu0           =  " << p.mu0 << endl;
    cout << "K             =  " << p.K() << endl;
    cout << "CFL           =  " << cfl << endl;
    cout << "Prandtl No.   =  " << prandtl << endl;
    cout << "numParticles  =  " << p.particles << endl;
    cout << "nprocs    =  " << 1 << " x " << 1 << " x " << 1 << endl;
    cout << endl << "Field Initialized ! " << endl;
    cout << "______________________________" << endl;
    cout << endl << "TIME              TKE" << endl;
    cout << "______________________________" << endl << endl;
}

void print_stats_line(double t_over_t0, const gks_stats_out &s)
{
    // update.cpp:657, 779-780
    std::cout.precision(8);
    std::cout << std::scientific << t_over_t0 << "  " << s.tke << "  " << s.diss << "  " << s.skew[0] << "  "
              << s.skew[1] << "  " << s.skew[2] << "  " << s.kurt[0] << "  " << s.kurt[1] << "  " << s.kurt[2]
              << "  " << s.prms << "  " << s.trms << "  "
              << "  " << s.vrms << std::endl;
}

} // namespace gksdrv
