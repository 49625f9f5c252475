/* dq_host.h — the C++ host of the propagator behind a C ABI: the reference's
 * `key = value` input file, its data files, and the run driver that sets up a
 * dq_ctx from them and writes the reference's output files.
 *
 * Reference interfaces replaced (DynaQuant):
 *   dq_infile_parse  systemClass::parseInFile (systemClass.cu:184-735) with
 *                    stringSplit/stringTrim (cppUtility.cpp:82-106)
 *   dq_infile_run    main's set-up and ensemble loop (propagate.cu:29-298):
 *                    readInHam (sparseMatrixClasses.cu:75-230), prepForKA /
 *                    prepForHsr / prepForZZReal (systemClass.cu:912-1207),
 *                    the initial state (systemClass.cu:1329-1481), spectra
 *                    directions (spectraClass.cu:300-496) and the files of
 *                    popPrintClass, statePrintClass, spectraClass and
 *                    calcInvPatricRatio (invParticRat.dat).
 */
#ifndef DQ_HOST_H
#define DQ_HOST_H

#include "dq.h"

#ifdef __cplusplus
extern "C" {
#endif

#define DQ_HOST_PATH_MAX 1024

/* ensembleavgmode (systemClass.h ENS_AVG_MODE_*) */
enum { DQ_ENS_AVG_NONE = 0, DQ_ENS_AVG_FIRST = 1, DQ_ENS_AVG_CONTINUATION = 2 };
/* simtype (SIM_TYPE_*) */
enum {
    DQ_SIM_CONST_HAM = 0,
    DQ_SIM_HSR = 1,
    DQ_SIM_KUBO_ANDERSON = 2,
    DQ_SIM_ZZ_REAL_NOISE = 3,
    DQ_SIM_ZZ_COMPLEX_NOISE = 4
};
/* propmode (PROP_MODE_*) */
enum { DQ_PROP_LANCZOS = 0, DQ_PROP_TAYLOR_LANCZOS = 1 };

/* Every key of the reference's input file, with the reference's defaults
 * (systemClass.cu:30-80), plus this build's own keys, which the reference
 * would skip as unknown.  Strings are stored as read (relative paths are
 * resolved by dq_infile_run against its base directory). */
typedef struct dq_infile {
    double dt;
    int totalsteps;
    int ensembleavgmode;
    int ensembleruns;
    int m;
    int ka_substeps;
    int absorbspec;
    int cdspec;
    int lineshapedress;
    double gausswidth;
    int dostatelooping;
    int stepsperloop;
    int writeoutpops;
    int printallpops;
    int writebinarypops;
    int printpop[10];     /* -1 = unset */
    int print_partic;
    int writeoutstates;   /* write states every this many steps (<= 0: never) */
    int initstate;
    int initfromfile;
    int propmode;
    int simtype;
    int staticdis;
    double sigmastatdis;
    double temperature;
    int debug_diags;
    int tk_p;
    int tk_m_aux;
    char hamfile[DQ_HOST_PATH_MAX];
    char statefile[DQ_HOST_PATH_MAX];
    char outfile[DQ_HOST_PATH_MAX];
    char tkmatfile[DQ_HOST_PATH_MAX];
    char outfolder[DQ_HOST_PATH_MAX];
    char hsr_stddevfile[DQ_HOST_PATH_MAX];
    char ka_paramsfile[DQ_HOST_PATH_MAX];
    char zz_specd_file[DQ_HOST_PATH_MAX];
    char dipolefile[DQ_HOST_PATH_MAX];
    char posfile[DQ_HOST_PATH_MAX];
    char initstatefile[DQ_HOST_PATH_MAX];
    /* this build's keys (no reference counterpart) */
    int precision;        /* `precision = PREC_FP64 | PREC_MIXED` (default FP64, as the reference) */
    unsigned long long seed;   /* `seed`: the Philox key of every random draw (default 0) */
    int pop_every;        /* `pop_every`: population records every this many steps (default 1) */
    /* bookkeeping of the parse */
    int n_assignments;    /* lines with '=' whose key had no '!' */
    int n_unknown;        /* of those, keys the parser does not know (skipped, as the reference does) */
} dq_infile;

/* The reference's defaults (and 0 / empty for what it leaves unset). */
DQ_API void dq_infile_defaults(dq_infile *in);

/* Parses an input file the way systemClass::parseInFile does: every line that
 * contains '=' is split at its first '=', the key is what precedes it and the
 * value starts two characters after it (stringSplit); both are trimmed of
 * leading/trailing tabs and then spaces (stringTrim); a key that contains '!'
 * is skipped, unknown keys are skipped, numbers are read with atoi/atof (so a
 * trailing "! comment" after a number is ignored), and a 0/1 flag with any
 * other value, or an unknown enumeration name, fails with DQ_ERR_ARG like the
 * reference's "must be 0 or 1. Aborting.".  One deviation: a line ending in
 * '=' (where the reference's substr would throw) gives an empty value.
 * Needs no GPU.  errbuf (may be NULL) receives a message on failure. */
DQ_API dq_status dq_infile_parse(const char *path, dq_infile *out, char *errbuf, int errbuf_len);

/* One line as dq_infile_parse reads it: returns 1 and the trimmed key and
 * value for an assignment, 0 for a line without '=', 2 for a key containing
 * '!' (skipped).  The line-level step of parseInFile (systemClass.cu:239-250,
 * cppUtility.cpp:82-106). */
DQ_API int dq_infile_split_line(const char *line, char *key, int key_len, char *value, int value_len);

/* Runs the simulation an input file describes, on CUDA device `device`:
 * reads hamfile (and the noise, spectral-density, dipole, position and
 * initial-state files the keys name; relative paths against base_dir, NULL =
 * the current directory, as the reference opens them), creates one context per
 * initial condition (1, or the 3 polarisation directions of absorbspec /
 * cdspec), propagates its `ensembleruns` runs (1 with ENS_AVG_MODE_NONE) as one
 * batched ensemble for `totalsteps` steps (Lanczos, or Taylor-Krylov with
 * propmode = PROP_MODE_TAYLOR_LANCZOS), and writes into outfolder (created if
 * missing) what the keys ask for: pops.dat (writeoutpops with printallpops;
 * text or binary; ENS_AVG_MODE_CONTINUATION adds to an existing file),
 * _states_<t>.dat every writeoutstates steps, invParticRat.dat (print_partic),
 * and the absorption / CD correlation and spectrum files per direction and
 * their mean.  Runs are independent trajectories keyed by `seed`, so the
 * reference's wall-clock seeding is not reproduced. */
DQ_API dq_status dq_infile_run(const dq_infile *in, const char *base_dir, int device, char *errbuf, int errbuf_len);

#ifdef __cplusplus
}
#endif
#endif /* DQ_HOST_H */
