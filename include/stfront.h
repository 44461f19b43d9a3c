/*
 * stfront.h -- the `structure` front end over the GPU sweep engine
 * (libstfront.so; the command-line program stgpu_structure uses the same
 * code).
 *
 * It keeps the reference program's user-facing formats so it can replace it:
 *   - parameters: the mainparams / extraparams files ("#define KEY value"
 *     lines, src/params.c:43-330 GetParams, ReadFile, SetValue) and the
 *     command-line flags -m -e -s -i -o -K -L -N -D (src/params.c:87-145);
 *   - data: the genotype file (src/datain.c:65-333 ReadData: marker names,
 *     map distances, per-individual label / population / popflag / location /
 *     phenotype / extra columns, one or PLOIDY rows per individual), recoded
 *     as src/datain.c:824-904 CountAlleles does;
 *   - results: the OUTFILE_f file (src/output.c:1354-1423 OutPutResults and
 *     the printers it calls) and OUTFILE_q when PRINTQHAT=1
 *     (src/output.c:914-953 PrintQFile).
 *
 * The reference reads these into process globals and exits on any error;
 * here a run is an opaque handle, every call returns a status (0 or a
 * negative code) and stf_last_error() gives the message.
 */
#ifndef STFRONT_H
#define STFRONT_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct stf_run stf_run;

enum stf_status { STF_OK = 0, STF_ERR_ARG = -1, STF_ERR_PARAMS = -2, STF_ERR_DATA = -3,
                  STF_ERR_IO = -4, STF_ERR_UNSUPPORTED = -5 };

/* Parameters from the files and flags (argv as given to the program;
 * argv[0] is the program name).  Files are found as the reference finds
 * them: -m / -e arguments, else mainparams / extraparams in the working
 * directory.                                                               */
int stf_open(int argc, char **argv, stf_run **out);
int stf_close(stf_run *r);
const char *stf_last_error(const stf_run *r);

/* Parameter values by their mainparams/extraparams names (integer, real or
 * string keys, e.g. "MAXPOPS", "ALPHA", "DATAFILE"); 0 if known.           */
int stf_param_int(const stf_run *r, const char *key, int *value);
int stf_param_double(const stf_run *r, const char *key, double *value);
int stf_param_str(const stf_run *r, const char *key, char *buf, size_t n);
/* Sets an integer parameter (e.g. SEED to the seed a run actually used,
 * as src/ran.c:114-126 Randomize does before it is printed).             */
int stf_set_param_int(stf_run *r, const char *key, int value);

/* Reads DATAFILE and recodes alleles (CountAlleles).                      */
int stf_read_data(stf_run *r);
/* Sizes after stf_read_data: NUMINDS, NUMLOCI, LINES, MAXALLELES.         */
int stf_dims(const stf_run *r, int dims[4]);
/* Recoded genotypes [N][LINES][L] (missing as the recoded MISSING value),
 * NumAlleles [L], Translation [L][MAXALLELES] (original allele values).    */
int stf_geno(const stf_run *r, int32_t *geno, int32_t *numalleles, int32_t *translation);
/* Per individual: population, popflag, location, phenotype [N] each (may
 * be NULL); labels as NUL-terminated strings of 12 bytes each [N][12].     */
int stf_individuals(const stf_run *r, int32_t *pop, int32_t *popflag, int32_t *location,
                    int32_t *phenotype, char *labels);

/* USEPOPINFO=1: the prior-population checks of src/Init.c:15-70
 * CheckPopPriors, after stf_read_data and before the popflags are taken
 * for the engine: everyone flagged when the file has no POPFLAG column,
 * flags dropped for populations outside 1..MAXPOPS (their number in
 * *dropped, may be NULL), INFERALPHA set to 0 when nobody is left without
 * prior information (NOALPHA).  STF_ERR_PARAMS for a MIGRPRIOR outside
 * [0, 1] or no POPDATA.  A no-op with USEPOPINFO=0.                        */
int stf_check_pop_priors(stf_run *r, int32_t *dropped);
/* USEPOPINFO=1: the UsePopProbs sums [N][MAXPOPS][GENSBACK+1] of the run
 * (copied), printed for flagged individuals in place of their Q
 * (src/output.c:800-829 PrintGeogQ).  Required before stf_write_results
 * with USEPOPINFO=1.                                                       */
int stf_set_usepopprobs(stf_run *r, const double *usepop);

/* LOCPRIOR=1: the number of locations (distinct location ids of the data,
 * numbered in increasing order as src/Util.c:237-275 GetNumLocations does),
 * and the LocPrior sums of the run, n = 1 with admixture or
 * 1 + MAXPOPS * (locations + 1) without (r, nu, gamma; st_get_state
 * ST_F_SUMLOCPRIOR).  Required before stf_write_results with LOCPRIOR=1,
 * where sumAlpha then holds MAXPOPS * (locations + 1) values with admixture. */
int stf_num_locations(const stf_run *r);
int stf_set_locprior_sums(stf_run *r, const double *sums, size_t n);

/* INTERMEDSAVE: with savenum > 0 the next stf_write_results writes the
 * intermediate file OUTFILE_<savenum> (src/output.c:1381-1385) and no
 * OUTFILE_q; 0 (the default) writes OUTFILE_f.                             */
int stf_set_save_number(stf_run *r, int savenum);

/* Writes OUTFILE_f (and OUTFILE_q when PRINTQHAT=1) from the run's sums, in
 * the reference layouts: QSum [N][K], PSum [L][K][MAXALLELES], SumEpsilon
 * [L][MAXALLELES] (may be NULL without FREQSCORR), FstSum [K], sumAlpha [K],
 * AncestDist [N][K][NUMBOXES] (may be NULL without ANCESTDIST).  rep is the
 * total number of sweeps (BURNIN + NUMREPS at the end of a run).            */
int stf_write_results(stf_run *r, int rep, const double *QSum, const double *PSum,
                      const double *SumEpsilon, const double *FstSum, const double *sumAlpha,
                      const double *sumlambda, const int32_t *AncestDist, double sumlikes,
                      double sumsqlikes);

/* The screen trace printed every UPDATEFREQ sweeps (src/output.c:218-374
 * PrintUpdate, called from src/structure.c:669-702 after sweep rep and once
 * more after the last sweep when BURNIN + NUMREPS is not a multiple of
 * UPDATEFREQ): the "BURNIN completed" and "Admixture Burnin complete" notes,
 * the column heads every 10 * UPDATEFREQ sweeps (PrintBanner, output.c:377-454)
 * preceded by the membership table of Q when PRINTQSUM=1 (PrintMembership),
 * and the line of rep, lambda, alpha, F, r (LOCPRIOR), the net distances of
 * P between clusters (PRINTNET or PRINTKLD) and Ln Like.  As in the
 * reference, the Est Ln P(D) column of the line holds 0 outside the linkage
 * model (output.c:258-279 evaluates it only there).  Q [N][K] and
 * P [L][K][MAXALLELES] may be NULL when the line does not print them;
 * alpha, F and lambda hold MAXPOPS values; locprior[0] is r (LOCPRIOR=1).
 * The text goes to buf as snprintf would put it (NUL-terminated, cut to
 * n - 1 bytes; buf may be NULL with n = 0); returns its full length, or a
 * negative status (STF_ERR_UNSUPPORTED with LINKAGE=1).                   */
int stf_format_update(const stf_run *r, int rep, const double *Q, const double *P,
                      const double *alpha, const double *F, const double *lambda, double like,
                      const double *locprior, char *buf, size_t n);

/* ECHODATA=1: the start and end of the data as read (src/datain.c:514-571
 * PrintSomeData, printed by ReadInputFile after the "Reading file" line):
 * the first four individuals and the last two (all of them when there are
 * six or fewer), each row with its label / population / popflag / phenotype
 * columns, its first loci up to nine columns in all, and its last locus.
 * Text as stf_format_update gives it.                                      */
int stf_echo_data(const stf_run *r, char *buf, size_t n);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
