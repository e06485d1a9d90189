// File formats and printing of the reference's driver, kept byte-compatible:
//   InitialConditions/params          int n; double gam, rho0, Mt, Re, mu0, p0, t0   (FlowField.cpp:15-50)
//   InitialConditions/particleCount   int                                             (FlowField.cpp:53-56)
//   InitialConditions/Init000         u, v, w, rho, p; nc^3 doubles each, MATLAB order
//                                     J = k*ny*nx + i*ny + j                          (FlowField.cpp:59-112)
//   Results/Field/Field_<rank>_<iter> text dump of primitives                         (update.cpp:1305-1319)
//   stdout                            parameter banner (FlowField.cpp:305-334) and one
//                                     statistics line per step (update.cpp:778-781)
#pragma once

#include <string>
#include <vector>

#include "gks_b200.h"

namespace gksdrv {

struct RunParams {
    int nc = 0;
    int particles = 0;
    double gam = 0, rho0 = 0, Mt = 0, Re = 0, mu0 = 0, p0 = 0, t0 = 0;
    double R = 287.0;                                     // param.h:18
    int K() const { return int((5.0 - 3.0 * gam) / (gam - 1.0)); } // FlowField.cpp:41
    double T0() const { return p0 / (R * rho0); }          // FlowField.cpp:46
    double dx() const;                                      // FlowField.cpp:45
};

// Padded conservative field: 5 arrays of (nc+6)^3 doubles, the reference's W.
struct Field {
    int nc = 0;
    std::vector<double> w[5];
    double *ptr[5];
    void alloc(int n);
    size_t nt() const { return (size_t)nc + 6; }
    size_t idx(int j, int i, int k) const { return ((size_t)j * nt() + i) * nt() + k; }
};

// Returns an empty string on success, else the error message.
std::string read_params(const std::string &casedir, RunParams &p);
std::string read_init(const std::string &casedir, const RunParams &p, Field &W);
// InitialConditions/unirand: x0, y0, z0 of p.particles doubles each (locateParticles, update.cpp:1278-1284).
std::string read_unirand(const std::string &casedir, const RunParams &p, std::vector<double> xyz[3]);
std::string write_reinit(const std::string &path, const RunParams &p, const Field &W);
std::string write_field(const std::string &dir, int rank, int iter, const RunParams &p, const Field &W);

void print_params(const RunParams &p, double cfl, double prandtl);
void print_stats_line(double t_over_t0, const gks_stats_out &s);

} // namespace gksdrv
