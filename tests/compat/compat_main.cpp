// Exercises gks_compat.h the way the reference's update.cpp would: the
// globals of weno/src/param.h (declared here with the reference's names and
// types), a DevAlloc built once, evolve(W, dev, dt) once per step.
//   compat_main <in.bin> <out.bin> <nc> <dt> <steps> <gam> <mu0> <p0> <den0> <Mt> <t0> [<ranks> <rank>]
// in/out: 5 padded arrays of (nc+6)^3 doubles, or with ranks > 1 rank's
// padded y-slab block of (nc/ranks + 6) (nc+6)^2 doubles each (procDim =
// {ranks, 1, 1}: one rank of the reference's y decomposition).
#include <cstdio>
#include <cstdlib>
#include <vector>

typedef double ptype;  // param.h:22
#define R 287.0        // param.h:18
int nc_segx, nc_segy, nc_segz, K, procDim[3], Nt_seg, sta[3];
ptype T0, mu0, den0, p0, Mt, gam, t0;

#include "gks_compat.h"

int main(int argc, char **argv)
{
    if (argc < 12) return 2;
    const int nc = atoi(argv[3]);
    const double dt = atof(argv[4]);
    const int steps = atoi(argv[5]);
    gam = atof(argv[6]);
    mu0 = atof(argv[7]);
    p0 = atof(argv[8]);
    den0 = atof(argv[9]);
    Mt = atof(argv[10]);
    t0 = atof(argv[11]);
    const int ranks = argc > 13 ? atoi(argv[12]) : 1, rank = argc > 13 ? atoi(argv[13]) : 0;
    procDim[0] = ranks;
    procDim[1] = procDim[2] = 1;
    nc_segy = nc / ranks; // FlowField.cpp:22-24
    nc_segx = nc_segz = nc;
    sta[0] = rank * nc_segy; // segment(), FlowField.cpp:282-284
    sta[1] = sta[2] = 0;
    K = int((5.0 - 3.0 * gam) / (gam - 1.0)); // FlowField.cpp:41
    T0 = p0 / (R * den0);                     // FlowField.cpp:46
    const size_t nt = nc + 6, N = (size_t)(nc_segy + 6) * nt * nt;
    Nt_seg = (int)N; // FlowField.cpp:27-30
    std::vector<double> buf(5 * N);
    FILE *f = fopen(argv[1], "rb");
    if (!f || fread(buf.data(), sizeof(double), 5 * N, f) != 5 * N) return 3;
    fclose(f);
    ptype *W[5];
    for (int q = 0; q < 5; ++q) W[q] = buf.data() + q * N;
    DevAlloc *dev = new DevAlloc();
    for (int s = 0; s < steps; ++s) evolve(W, dev, dt);
    delete dev;
    f = fopen(argv[2], "wb");
    fwrite(buf.data(), sizeof(double), 5 * N, f);
    fclose(f);
    return 0;
}
