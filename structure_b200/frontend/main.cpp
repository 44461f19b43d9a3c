// main.cpp -- stgpu_structure: the `structure` command line on the GPU sweep
// engine.  Reads mainparams / extraparams and the data file like the
// reference program (src/structure.c:155-700, with the same -m -e -i -o -K
// -L -N -D flags), runs BURNIN + NUMREPS sweeps of one chain on the GPU
// through libstgpu (include/stgpu.h), prints the reference's screen trace
// every UPDATEFREQ sweeps (and the data echo with ECHODATA=1) and writes
// OUTFILE_f (and OUTFILE_q with PRINTQHAT=1).
//
// USEPOPINFO=1 runs the migrant model for individuals with prior population
// information and prints its posterior in OUTFILE_f (src/output.c:800-829);
// LOCPRIOR=1 uses the sampling locations (LOCDATA column, or the population
// with LOCISPOP) and prints r, nu / gamma or the location alphas.
// Options the GPU path does not implement (LINKAGE, RECESSIVEALLELES, PLOIDY
// other than 2) stop the program with a message instead of running a
// different model.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "stfront.h"
#include "stgpu.h"

namespace {

int pi(stf_run* r, const char* k) {
  int v = 0;
  stf_param_int(r, k, &v);
  return v;
}

double pd(stf_run* r, const char* k) {
  double v = 0.0;
  stf_param_double(r, k, &v);
  return v;
}

int die(const char* what, const char* msg) {
  fprintf(stderr, "%s: %s\n\nExiting the program due to error(s) listed above.\n\n", what, msg);
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  stf_run* r = nullptr;
  if (stf_open(argc, argv, &r) != STF_OK) return die("parameters", stf_last_error(r));
  const char* unsupported[] = {"LINKAGE", "RECESSIVEALLELES"};
  for (const char* k : unsupported)
    if (pi(r, k)) {
      fprintf(stderr, "%s=1 is not available on the GPU path.\n", k);
      return 1;
    }
  if (pi(r, "MAXPOPS") < 1 || pi(r, "MAXPOPS") > 32)
    return die("parameters", "MAXPOPS must be in 1..32");
  char datafile[256];
  stf_param_str(r, "DATAFILE", datafile, sizeof datafile);
  printf("Reading file \"%s\".\n", datafile);
  if (stf_read_data(r) != STF_OK) return die("data", stf_last_error(r));
  if (pi(r, "ECHODATA")) {
    std::string echo((size_t)stf_echo_data(r, nullptr, 0) + 1, '\0');
    stf_echo_data(r, &echo[0], echo.size());
    fputs(echo.c_str(), stdout);
  }
  int dims[4];
  stf_dims(r, dims);
  const int N = dims[0], L = dims[1], A = dims[3], K = pi(r, "MAXPOPS");
  std::vector<int32_t> geno((size_t)N * 2 * L), na(L), tr((size_t)L * (A > 0 ? A : 1));
  stf_geno(r, geno.data(), na.data(), tr.data());
  for (int32_t& g : geno)
    if (g < 0) g = -9;   // the engine's missing code
  std::vector<int32_t> popflag(N), pop(N), flag_before(N), location(N);
  stf_individuals(r, nullptr, flag_before.data(), nullptr, nullptr, nullptr);
  if (stf_check_pop_priors(r, nullptr) != STF_OK) return die("parameters", stf_last_error(r));
  stf_individuals(r, pop.data(), popflag.data(), location.data(), nullptr, nullptr);
  if (pi(r, "USEPOPINFO"))
    for (int i = 0; i < N; i++)
      if (!popflag[i] && (flag_before[i] || !pi(r, "POPFLAG")))
        printf("Warning: population prior for individual %d is %d, which is not\n"
               "  in the range 1..%d.  Population prior for this individual will\n"
               "  be ignored\n", i + 1, pop[i], K);
  int amin = 1 << 30, amax = 0;
  double asum = 0.0;
  for (int v : na) {
    amin = v < amin ? v : amin;
    amax = v > amax ? v : amax;
    asum += v;
  }
  printf("Number of alleles per locus: min=%2d; ave=%2.1f; max=%2d\n", amin, asum / L, amax);

  // seed: RANDOMIZE=1 (or the example seed 2245) takes one from the clock,
  // and every seed used is appended to seed.txt (src/ran.c:114-126)
  int seed = pi(r, "SEED");
  if (pi(r, "RANDOMIZE") || seed == 2245) seed = (int)time(nullptr);
  stf_set_param_int(r, "SEED", seed);
  if (FILE* sf = fopen("seed.txt", "a")) {
    fprintf(sf, "%i\n", seed);
    fclose(sf);
  }

  st_ctx* ctx = nullptr;
  st_data* data = nullptr;
  st_chain* c = nullptr;
  int rc = st_ctx_create(0, 0, &ctx);
  if (rc != ST_OK) return die("GPU", "no CUDA device (st_ctx_create failed)");
  st_data_desc d{};
  d.num_inds = N;
  d.num_loci = L;
  d.lines = 2;
  d.layout = ST_LAYOUT_AUTO;
  d.geno = geno.data();
  d.num_alleles = na.data();
  d.popflags = popflag.data();
  d.population = pop.data();
  if (pi(r, "LOCPRIOR")) d.location = location.data();
  rc = st_data_upload(ctx, &d, &data);
  if (rc != ST_OK) return die("GPU", st_last_error(ctx));
  st_model m;
  st_model_defaults(&m);
  m.maxpops = K;
  m.burnin = pi(r, "BURNIN");
  m.numreps = pi(r, "NUMREPS");
  m.freqscorr = pi(r, "FREQSCORR");
  m.onefst = pi(r, "ONEFST");
  m.inferalpha = pi(r, "INFERALPHA");
  m.popalphas = pi(r, "POPALPHAS");
  m.noadmix = pi(r, "NOADMIX");
  m.admburnin = pi(r, "ADMBURNIN");
  m.inferlambda = pi(r, "INFERLAMBDA");
  m.popspecificlambda = pi(r, "POPSPECIFICLAMBDA");
  m.unifprioralpha = pi(r, "UNIFPRIORALPHA");
  m.computeprob = pi(r, "COMPUTEPROB");
  m.pfrompopflagonly = pi(r, "PFROMPOPFLAGONLY");
  m.ancestdist = pi(r, "ANCESTDIST");
  m.numboxes = pi(r, "NUMBOXES");
  m.metrofreq = pi(r, "METROFREQ");
  m.alpha = pd(r, "ALPHA");
  m.alphamax = pd(r, "ALPHAMAX");
  m.alphapropsd = pd(r, "ALPHAPROPSD");
  m.alphapriora = pd(r, "ALPHAPRIORA");
  m.alphapriorb = pd(r, "ALPHAPRIORB");
  m.lambda = pd(r, "LAMBDA");
  m.fpriormean = pd(r, "FPRIORMEAN");
  m.fpriorsd = pd(r, "FPRIORSD");
  m.usepopinfo = pi(r, "USEPOPINFO");
  m.popflag_given = 1;   // the flags above already hold CheckPopPriors' result
  m.gensback = pi(r, "GENSBACK");
  m.migrprior = pd(r, "MIGRPRIOR");
  m.startatpopinfo = pi(r, "STARTATPOPINFO");
  m.locprior = pi(r, "LOCPRIOR");
  m.updatelocprior = pi(r, "UPDATELOCPRIOR");
  m.locpriorinit = pd(r, "LOCPRIORINIT");
  m.maxlocprior = pd(r, "MAXLOCPRIOR");
  m.locpriorstep = pd(r, "LOCPRIORSTEP");
  rc = st_chain_create(ctx, data, &m, (uint64_t)seed, &c);
  if (rc != ST_OK) return die("GPU", st_last_error(ctx));

  printf("\n\n--------------------------------------\n\n");
  printf("Finished initialization; starting MCMC \n");
  printf("%d iterations + %d burnin\n\n", m.numreps, m.burnin);
  const int total = m.burnin + m.numreps, every = pi(r, "UPDATEFREQ") > 0 ? pi(r, "UPDATEFREQ") : 100;
  std::vector<double> alpha(K), F(K), stats(256);
  // results from the run's sums: OUTFILE_f at the end, OUTFILE_<n> for the
  // n-th intermediate save (src/structure.c:640-660)
  const size_t NK = (size_t)N * K, LKA = (size_t)L * K * A;
  auto write_results = [&](int rep, int savenum) -> int {
    std::vector<double> QSum(NK), PSum(LKA), SumEps((size_t)L * A), FstSum(K),
        sumAlpha(st_field_bytes(c, ST_F_SUMALPHA) / 8), sumlambda(K);
    std::vector<int32_t> AD;
    st_get_state(c, ST_F_QSUM, QSum.data(), NK * 8);
    st_get_state(c, ST_F_PSUM, PSum.data(), LKA * 8);
    st_get_state(c, ST_F_SUMEPS, SumEps.data(), SumEps.size() * 8);
    st_get_state(c, ST_F_FSTSUM, FstSum.data(), K * 8);
    st_get_state(c, ST_F_SUMALPHA, sumAlpha.data(), sumAlpha.size() * 8);
    st_get_state(c, ST_F_SUMLAMBDA, sumlambda.data(), K * 8);
    st_get_state(c, ST_F_STATS, stats.data(), stats.size() * 8);
    if (m.ancestdist) {
      AD.resize(NK * (size_t)m.numboxes);
      st_get_state(c, ST_F_ANCESTDIST, AD.data(), AD.size() * 4);
    }
    if (m.locprior) {
      std::vector<double> lp(st_field_bytes(c, ST_F_SUMLOCPRIOR) / 8);
      st_get_state(c, ST_F_SUMLOCPRIOR, lp.data(), lp.size() * 8);
      if (stf_set_locprior_sums(r, lp.data(), lp.size()) != STF_OK) return STF_ERR_ARG;
    }
    if (m.usepopinfo) {
      std::vector<double> up(NK * (size_t)(m.gensback + 1));
      st_get_state(c, ST_F_USEPOPPROBS, up.data(), up.size() * 8);
      stf_set_usepopprobs(r, up.data());
    }
    stf_set_save_number(r, savenum);
    const int wrc = stf_write_results(r, rep, QSum.data(), PSum.data(), SumEps.data(),
                                      FstSum.data(), sumAlpha.data(), sumlambda.data(),
                                      AD.empty() ? nullptr : AD.data(), stats[1], stats[2]);
    stf_set_save_number(r, 0);
    return wrc;
  };
  // INTERMEDSAVE: results every savefreq collected sweeps (src/Init.c:376-385)
  int savefreq = 0;
  if (pi(r, "INTERMEDSAVE") > 0) {
    savefreq = m.numreps / (pi(r, "INTERMEDSAVE") + 1);
    if (savefreq * (pi(r, "INTERMEDSAVE") + 1) < m.numreps) savefreq++;
  }
  const bool printlikes = pi(r, "PRINTLIKES") != 0;
  // the screen trace of src/output.c:218-374 PrintUpdate after every
  // UPDATEFREQ-th sweep and after the last one (src/structure.c:669-702),
  // from the chain's current state
  const size_t lp_n = m.locprior ? st_field_bytes(c, ST_F_LOCPRIOR) / 8 : 0;
  std::vector<double> lambda(K), Qd, Pd, locp(lp_n > 0 ? lp_n : 1);
  std::vector<float> Qf, Pf;
  const bool trace_q = pi(r, "PRINTQSUM") && K > 1, trace_p = pi(r, "PRINTNET") || pi(r, "PRINTKLD");
  std::string line;
  auto print_update = [&](int rep) -> int {
    alpha.assign(st_field_bytes(c, ST_F_ALPHA) / 8, 0.0);
    st_get_state(c, ST_F_ALPHA, alpha.data(), alpha.size() * 8);
    st_get_state(c, ST_F_F, F.data(), F.size() * 8);
    st_get_state(c, ST_F_LAMBDA, lambda.data(), lambda.size() * 8);
    if (lp_n > 0) st_get_state(c, ST_F_LOCPRIOR, locp.data(), lp_n * 8);
    if (trace_q) {
      Qf.resize(NK);
      st_get_state(c, ST_F_Q, Qf.data(), NK * 4);
      Qd.assign(Qf.begin(), Qf.end());
    }
    if (trace_p) {
      Pf.resize(LKA);
      st_get_state(c, ST_F_P, Pf.data(), LKA * 4);
      Pd.assign(Pf.begin(), Pf.end());
    }
    const int len = stf_format_update(r, rep, trace_q ? Qd.data() : nullptr,
                                      trace_p ? Pd.data() : nullptr, alpha.data(), F.data(),
                                      lambda.data(), stats[0], locp.data(), nullptr, 0);
    if (len < 0) return len;
    line.assign((size_t)len + 1, '\0');
    stf_format_update(r, rep, trace_q ? Qd.data() : nullptr, trace_p ? Pd.data() : nullptr,
                      alpha.data(), F.data(), lambda.data(), stats[0], locp.data(), &line[0],
                      line.size());
    fputs(line.c_str(), stdout);
    fflush(stdout);
    return STF_OK;
  };
  for (int done = 0; done < total;) {
    int next = std::min(total, (done / every + 1) * every);
    if (savefreq > 0 && savefreq <= m.numreps) {
      const int after = std::max(done + 1, m.burnin + 1);
      const int save = m.burnin + ((after - m.burnin + savefreq - 1) / savefreq) * savefreq;
      if (save < total) next = std::min(next, save);
    }
    if (printlikes) next = done + 1;
    rc = st_sweep(c, next - done);
    if (rc == ST_OK) rc = st_sync(c);
    if (rc != ST_OK) return die("GPU", st_last_error(ctx));
    done = next;
    st_get_state(c, ST_F_STATS, stats.data(), stats.size() * 8);
    if (printlikes) {
      // src/output.c:187-200 PrintLike: the sweep's ln P(D) once collecting,
      // else CalcLike of the current state
      double like = stats[0];
      if (done <= m.burnin && st_calc_like(c, &like) != ST_OK) return die("GPU", st_last_error(ctx));
      printf("%6.0f\n", like);
    }
    if (done % every == 0 || done == total)
      if (print_update(done) != STF_OK) return die("output", "screen trace");
    if (savefreq > 0 && done > m.burnin && (done - m.burnin) % savefreq == 0 && done != total)
      if (write_results(done, (done - m.burnin) / savefreq) != STF_OK)
        return die("output", stf_last_error(r));
  }
  printf("\nMCMC completed\n");
  rc = write_results(total, 0);
  if (rc != STF_OK) return die("output", stf_last_error(r));
  char outfile[256];
  stf_param_str(r, "OUTFILE", outfile, sizeof outfile);
  printf("Final results printed to file %s_f\n\n", outfile);
  printf("Structure seed: %d\n", seed);
  st_chain_destroy(c);
  st_data_destroy(data);
  st_ctx_destroy(ctx);
  stf_close(r);
  return 0;
}
