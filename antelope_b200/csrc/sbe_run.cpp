// sbe_run: command-line drop-in for the reference executable (exec_hhg_mpi,
// built from src/GeneralModel/antelope.cpp).  Like the reference it reads
// ./inputParam.cfg (or the path given as the first argument) and writes
// outlaserdata.dat, laserParameters.dat, interband_dipole_full_evol.dat,
// intraband_current_full_evol.dat, occupation__full__evol.dat and
// coherence__full__evol.dat into the working directory (or --out DIR).
//
//   sbe_run [cfg] [--out DIR] [--precision fp64|mixed] [--device N] [--graph]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/sbe.h"

int main(int argc, char **argv)
{
    std::string cfg = "inputParam.cfg", out = ".";
    sbe_opts o;
    sbe_opts_default(&o);
    for (int i = 1; i < argc; ++i) {
        const char *a = argv[i];
        if (!std::strcmp(a, "--out") && i + 1 < argc) out = argv[++i];
        else if (!std::strcmp(a, "--precision") && i + 1 < argc) {
            const char *p = argv[++i];
            o.precision = !std::strcmp(p, "mixed") ? 1 : 0;
        } else if (!std::strcmp(a, "--device") && i + 1 < argc) o.device = std::atoi(argv[++i]);
        else if (!std::strcmp(a, "--graph")) o.use_graph = 1;
        else if (!std::strcmp(a, "-h") || !std::strcmp(a, "--help")) {
            std::printf("usage: sbe_run [inputParam.cfg] [--out DIR] [--precision fp64|mixed] [--device N] [--graph]\n");
            return 0;
        } else cfg = a;
    }
    sbe_problem *p = nullptr;
    sbe_status st = sbe_problem_from_cfg(cfg.c_str(), &p);
    if (st != SBE_OK) {
        std::fprintf(stderr, "%s\n", sbe_last_error_message());
        return EXIT_FAILURE;
    }
    sbe_dims d;
    sbe_problem_dims(p, &d);
    if (d.gauge == 0 && d.model == 0)
        std::printf("Note: gauge LengthWannier (the reference's default when 'gauge' is absent).\n");
    std::printf("k-grid %d x %d x %d = %d points, Nt = %d, dt = %g, bands = %d\n", d.Nk[0], d.Nk[1], d.Nk[2],
                d.ntotal, d.Nt, d.dt, d.nband);
    sbe_problem_destroy(p);
    st = sbe_run_cfg(cfg.c_str(), out.c_str(), &o);
    if (st != SBE_OK) {
        std::fprintf(stderr, "%s\n", sbe_last_error_message());
        return EXIT_FAILURE;
    }
    std::printf("\n\nWriting output-data\n\n");
    return 0;
}
