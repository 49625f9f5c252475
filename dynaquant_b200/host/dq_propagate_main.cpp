// dq_propagate — command-line driver: `dq_propagate <infile> [--device N]`,
// the counterpart of the reference's `propagate <infile>` (propagate.cu:29-60):
// parses the input file, runs it on one GPU and writes the output files
// into its outfolder.  Relative paths in the file are taken from the current
// directory, as the reference opens them.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/dq_host.h"

int main(int argc, char** argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: %s <infile> [--device N]\n", argv[0]);
        return 2;
    }
    int device = 0;
    for (int i = 2; i + 1 < argc; ++i)
        if (!strcmp(argv[i], "--device")) device = atoi(argv[i + 1]);
    dq_infile in;
    char err[1024] = {0};
    if (dq_infile_parse(argv[1], &in, err, sizeof err) != DQ_OK) {
        fprintf(stderr, "%s\n", err);
        return 1;
    }
    printf("hamfile %s, dt %g fs, totalsteps %d, runs %d, m %d, outfolder %s\n", in.hamfile, in.dt, in.totalsteps,
           in.ensembleavgmode == DQ_ENS_AVG_NONE ? 1 : in.ensembleruns, in.m, in.outfolder);
    const auto t0 = std::chrono::steady_clock::now();
    const dq_status st = dq_infile_run(&in, nullptr, device, err, sizeof err);
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (st != DQ_OK) {
        fprintf(stderr, "run failed (%d): %s\n", st, err);
        return 1;
    }
    printf("done in %.3f s\n", s);
    return 0;
}
