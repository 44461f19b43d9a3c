// front.cpp -- parameters, data file and result files of the `structure`
// program, for the GPU sweep engine (C ABI in include/stfront.h).
//
// Formats follow the reference so that a user's files and scripts keep
// working: parameter files are scanned for "#define KEY value"
// (src/params.c:222-330), the data file is read token by token in the order
// of src/datain.c:65-333, alleles are recoded in order of first appearance
// (src/datain.c:824-904), and OUTFILE_f carries the sections of
// src/output.c:1354-1423 in the reference's text layout.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "stfront.h"

namespace {

constexpr const char* kVersion = "2.3.4 (Jul 2012)";   // the release this front end mirrors
constexpr int kStrLen = 200;     // file names (DATAFILE, OUTFILE)
constexpr int kGeneLen = 15;     // marker names
constexpr int kLabelLen = 12;    // individual labels
constexpr int kAllelLen = 10;    // integer fields of the data file
constexpr int kMaxName = 30;     // parameter names

enum Kind { kInt, kIntAuto, kReal, kStr };

struct Key {
  const char* name;
  Kind kind;
  double def;        // numeric default
  const char* sdef;  // string default
};

// Every key the reference's SetValue accepts, with its PresetValues default
// (src/params.c:330-570).  kIntAuto keys are read like "%i" (base prefixes).
const Key kKeys[] = {
    {"DATAFILE", kStr, 0, ""}, {"OUTFILE", kStr, 0, "output"},
    {"NUMINDS", kInt, 0, nullptr}, {"NUMLOCI", kInt, 0, nullptr},
    {"MISSING", kInt, -9, nullptr}, {"LABEL", kInt, -1, nullptr},
    {"POPDATA", kInt, -1, nullptr}, {"MARKERNAMES", kInt, 0, nullptr},
    {"PHASEINFO", kInt, 0, nullptr}, {"MAPDISTANCES", kInt, 0, nullptr},
    {"MARKOVPHASE", kInt, -1, nullptr}, {"LINES", kInt, 2, nullptr},
    {"ONEROWPERIND", kInt, 0, nullptr}, {"RECESSIVEALLELES", kInt, 0, nullptr},
    {"NOTAMBIGUOUS", kInt, -939, nullptr}, {"POPFLAG", kInt, -1, nullptr},
    {"PHENOTYPE", kInt, -1, nullptr}, {"EXTRACOLS", kInt, -1, nullptr},
    {"MAXPOPS", kInt, -1, nullptr}, {"BURNIN", kInt, 10000, nullptr},
    {"NUMREPS", kInt, 20000, nullptr}, {"USEPOPINFO", kInt, 0, nullptr},
    {"PFROMPOPFLAGONLY", kInt, 0, nullptr}, {"INFERALPHA", kInt, 1, nullptr},
    {"INFERLAMBDA", kInt, 0, nullptr}, {"POPSPECIFICLAMBDA", kInt, 0, nullptr},
    {"POPALPHAS", kInt, 0, nullptr}, {"COMPUTEPROB", kInt, 1, nullptr},
    {"NOADMIX", kInt, 0, nullptr}, {"ADMBURNIN", kInt, 2500, nullptr},
    {"PHASED", kInt, 1, nullptr}, {"PRINTQHAT", kInt, 0, nullptr},
    {"PRINTQSUM", kInt, 0, nullptr}, {"UPDATEFREQ", kInt, 200, nullptr},
    {"PRINTLIKES", kInt, 0, nullptr}, {"INTERMEDSAVE", kInt, 0, nullptr},
    {"PRINTKLD", kInt, 0, nullptr}, {"PRINTNET", kInt, 0, nullptr},
    {"PRINTLAMBDA", kInt, 0, nullptr}, {"ECHODATA", kInt, 0, nullptr},
    {"ANCESTDIST", kInt, 0, nullptr}, {"NUMBOXES", kInt, 1000, nullptr},
    {"ANCESTPINT", kReal, 0.90, nullptr}, {"GENSBACK", kInt, 2, nullptr},
    {"MIGRPRIOR", kReal, 0.05, nullptr}, {"ALPHA", kReal, 1.0, nullptr},
    {"LOG10RPROPSD", kReal, 0.1, nullptr}, {"LOG10RMIN", kReal, -8, nullptr},
    {"LOG10RMAX", kReal, 2, nullptr}, {"LOG10RSTART", kReal, -4, nullptr},
    {"FREQSCORR", kInt, 1, nullptr}, {"ONEFST", kInt, 0, nullptr},
    {"FPRIORMEAN", kReal, 0.1, nullptr}, {"FPRIORSD", kReal, 0.1, nullptr},
    {"LAMBDA", kReal, 1.0, nullptr}, {"UNIFPRIORALPHA", kInt, 1, nullptr},
    {"ALPHAMAX", kReal, 10.0, nullptr}, {"ALPHAPRIORA", kReal, 1.0, nullptr},
    {"ALPHAPRIORB", kReal, 2.0, nullptr}, {"ALPHAPROPSD", kReal, 0.05, nullptr},
    {"STARTATPOPINFO", kInt, 0, nullptr}, {"RANDOMIZE", kInt, 1, nullptr},
    {"LINKAGE", kInt, 0, nullptr}, {"METROFREQ", kInt, 20, nullptr},
    {"REPORTHITRATE", kInt, 0, nullptr}, {"NOQS", kInt, 0, nullptr},
    {"POSTERIOR", kInt, 1, nullptr}, {"PICTUREFILE", kInt, 0, nullptr},
    {"INDIVIDUALR", kInt, 0, nullptr}, {"NUMSIMSTATS", kInt, 1000, nullptr},
    {"EMERROR", kReal, 0.001, nullptr}, {"POOLFREQ", kInt, 10, nullptr},
    {"LOCUSxONLY", kInt, 0, nullptr}, {"PHENOTYPECOL", kInt, -9, nullptr},
    {"MISSINGPHENO", kInt, -9, nullptr}, {"LOCPRIOR", kIntAuto, 0, nullptr},
    {"UPDATELOCPRIOR", kIntAuto, 1, nullptr}, {"LOCPRIORINIT", kReal, 1.0, nullptr},
    {"MAXLOCPRIOR", kReal, 20.0, nullptr}, {"LOCISPOP", kIntAuto, 0, nullptr},
    {"LOCDATA", kIntAuto, 0, nullptr}, {"LOCPRIORSTEP", kReal, 0.1, nullptr},
    {"PRINTLOCPRIOR", kInt, 1, nullptr}, {"SEED", kIntAuto, -1, nullptr},
};

// Names in the files that differ from the stored key.
const char* file_key(const std::string& w) {
  if (w == "INFILE") return "DATAFILE";
  if (w == "PLOIDY") return "LINES";
  return nullptr;
}

bool white(int c) { return c == ' ' || c == '\n' || c == '\t'; }

// A file read one character at a time, with the reference's tokenisers.
struct CharStream {
  std::string s;
  size_t p = 0;
  int get() { return p < s.size() ? (unsigned char)s[p++] : EOF; }
  int peek() const { return p < s.size() ? (unsigned char)s[p] : EOF; }

  // Next run of non-whitespace characters (space, newline, tab), at most
  // maxlength-1 of them; the rest of a longer run is skipped.  "" at EOF.
  std::string word(int maxlength) {
    std::string w;
    while ((int)w.size() < maxlength - 1) {
      const int c = get();
      if (c == EOF) break;
      if (!white(c)) {
        w.push_back((char)c);
      } else if (!w.empty()) {
        return w;
      }
    }
    if ((int)w.size() == maxlength - 1) {
      int c;
      do c = get(); while (c != EOF && !white(c));
    }
    return w;
  }

  // The rest of the line after leading blanks, up to a "//" comment or the
  // end of line, trailing blanks removed (file names may hold spaces).
  std::string rest_of_line(int maxlength) {
    std::string w;
    int last = 0;
    while ((int)w.size() < maxlength - 1) {
      const int c = get();
      if (c == EOF) break;
      if (last == '/' && c == '/') {
        w.pop_back();
        break;
      }
      if (last == 0 && isspace(c)) continue;
      if (c != '\n' && c != '\r') {
        w.push_back((char)c);
        last = c;
      } else if (!w.empty()) {
        break;
      }
    }
    while (!w.empty() && isspace((unsigned char)w.back())) w.pop_back();
    if ((int)w.size() + 1 == maxlength) {
      int c;
      do c = get(); while (c != EOF && !white(c));
    }
    return w;
  }

  // fscanf("%d") / ("%i") / ("%lf"): leading white space, then a number;
  // on failure nothing is assigned.
  bool number(Kind kind, double* out) {
    while (p < s.size() && isspace((unsigned char)s[p])) p++;
    const char* b = s.c_str() + p;
    char* e = nullptr;
    if (kind == kReal) {
      const double v = strtod(b, &e);
      if (e == b) return false;
      *out = v;
    } else {
      const long v = strtol(b, &e, kind == kIntAuto ? 0 : 10);
      if (e == b) return false;
      *out = (double)(int)v;
    }
    p += (size_t)(e - b);
    return true;
  }
};

struct Individual {
  std::string label;
  int population = 0, popflag = 0, phenotype = 0, location = 0;
};

}  // namespace

struct stf_run {
  std::map<std::string, double> num;
  std::map<std::string, std::string> str;
  std::vector<std::string> argv;
  std::string err;
  std::vector<std::string> warnings;
  // data
  bool have_data = false;
  int N = 0, L = 0, LINES = 2, MAXALLELES = 0, orig_missing = -9, missing = -9;
  std::vector<int32_t> geno, numalleles, translation;
  std::vector<std::string> markername;
  std::vector<Individual> ind;
  // USEPOPINFO (stf_check_pop_priors / stf_set_usepopprobs)
  bool noalpha = false;
  std::vector<double> usepop;   // [N][MAXPOPS][GENSBACK+1]
  // LOCPRIOR (stf_set_locprior_sums): sumLocPrior, the reference's layout
  std::vector<double> sumlocp;
  int savenum = 0;              // > 0: the next results go to OUTFILE_<savenum>
};

namespace {

int fail(stf_run* r, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  r->err = buf;
  return code;
}

const Key* find_key(const std::string& name) {
  for (const Key& k : kKeys)
    if (name == k.name) return &k;
  return nullptr;
}

int I(const stf_run* r, const char* k) { return (int)r->num.at(k); }
double D(const stf_run* r, const char* k) { return r->num.at(k); }
const std::string& S(const stf_run* r, const char* k) { return r->str.at(k); }

bool read_file(const std::string& path, std::string* out) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  char buf[1 << 16];
  size_t n;
  out->clear();
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) out->append(buf, n);
  fclose(f);
  return true;
}

// src/params.c:222-330: "#" then "define" then the name, then its value.
void read_params(stf_run* r, CharStream& cs) {
  int c;
  while ((c = cs.get()) != EOF) {
    if (c != '#') continue;
    std::string w = cs.word(kMaxName);
    if (w != "define") continue;
    w = cs.word(kMaxName);
    if (w.empty()) continue;
    const char* alias = file_key(w);
    const Key* k = find_key(alias ? alias : w);
    if (!k || w == "DATAFILE" || w == "LINES" || w == "PRINTLOCPRIOR") {
      r->warnings.push_back("Ignoring unrecognized parameter name (" + w + ")");
      continue;
    }
    if (k->kind == kStr) {
      r->str[k->name] = cs.rest_of_line(kStrLen);
    } else {
      double v;
      if (cs.number(k->kind, &v)) r->num[k->name] = v;
    }
  }
}

// src/params.c:147-220: the file named after a -m / -e flag (the words up to
// the next flag, joined by single spaces, quotes removed), else the default.
std::string param_file_name(const std::vector<std::string>& a, const char* flag,
                            const char* dflt) {
  for (size_t i = 0; i + 1 < a.size(); i++) {
    if (a[i] != flag) continue;
    std::string name;
    for (size_t j = i + 1; j < a.size() && a[j][0] != '-'; j++) {
      if (!name.empty()) name += ' ';
      name += a[j];
    }
    std::string out;
    for (char ch : name) {
      if (ch == '"') break;
      out += ch;
    }
    // a leading quote is dropped, the name ends at the closing one
    if (!name.empty() && name[0] == '"') {
      out.clear();
      for (size_t q = 1; q < name.size() && name[q] != '"'; q++) out += name[q];
    }
    return out;
  }
  return dflt;
}

bool valid_int_field(const std::string& w) {
  for (char ch : w)
    if ((ch < '0' || ch > '9') && ch != '-') return false;
  return true;
}

// src/params.c:744-770
int update_freq(const stf_run* r) {
  if (I(r, "UPDATEFREQ") > 0) return I(r, "UPDATEFREQ");
  const long numgens = (long)I(r, "LINES") * I(r, "NUMINDS") * I(r, "NUMLOCI");
  const int approx = numgens > 0 ? (int)(4000000 / numgens) : 0;
  if (approx <= 15) return 10;
  if (approx <= 37) return 25;
  if (approx <= 75) return 50;
  if (approx <= 250) return 100 * ((approx + 50) / 100);
  return 500 * ((approx + 250) / 500);
}

}  // namespace

// ===========================================================================
// parameters
// ===========================================================================
extern "C" int stf_open(int argc, char** argv, stf_run** out) {
  if (!out || argc < 1 || !argv) return STF_ERR_ARG;
  *out = nullptr;
  stf_run* r = new stf_run();
  for (int i = 0; i < argc; i++) r->argv.push_back(argv[i] ? argv[i] : "");
  for (const Key& k : kKeys) {
    if (k.kind == kStr) r->str[k.name] = k.sdef;
    else r->num[k.name] = k.def;
  }
  *out = r;
  for (const char* flag : {"-m", "-e"}) {
    const std::string path =
        param_file_name(r->argv, flag, flag[1] == 'm' ? "mainparams" : "extraparams");
    std::string text;
    if (!read_file(path, &text))
      return fail(r, STF_ERR_IO, "Can't open the file \"%s\".", path.c_str());
    CharStream cs;
    cs.s = std::move(text);
    read_params(r, cs);
  }
  // command-line values (src/params.c:87-145)
  const auto& a = r->argv;
  for (size_t i = 0; i + 1 < a.size(); i++) {
    const std::string& f = a[i];
    const char* map = f == "-K" ? "MAXPOPS" : f == "-L" ? "NUMLOCI" : f == "-N" ? "NUMINDS"
                    : f == "-r" ? "NUMSIMSTATS" : f == "-c" ? "PHENOTYPECOL" : nullptr;
    if (f == "-i") {
      r->str["DATAFILE"] = a[i + 1];
    } else if (f == "-o") {
      r->str["OUTFILE"] = a[i + 1];
    } else if (map) {
      if (!valid_int_field(a[i + 1]))
        return fail(r, STF_ERR_PARAMS, "Error in command-line data entry for %s: %s", map,
                    a[i + 1].c_str());
      r->num[map] = atoi(a[i + 1].c_str());
    } else if (f == "-D") {
      r->num["SEED"] = atoi(a[i + 1].c_str());
      i++;
    }
  }
  // src/params.c:680-742 CheckIfMissing
  std::string trouble;
  if (S(r, "DATAFILE").empty()) trouble += "Need to specify the name of the data file. ";
  if (I(r, "NUMINDS") < 1) trouble += "Need to set NUMINDS>0. ";
  if (I(r, "NUMLOCI") < 1) trouble += "Need to set NUMLOCI>0. ";
  if (I(r, "LABEL") == -1) trouble += "Need to set LABEL=0 or 1. ";
  if (I(r, "POPDATA") == -1) trouble += "Need to set POPDATA=0 or 1. ";
  if (I(r, "POPFLAG") == -1) trouble += "Need to set POPFLAG=0 or 1. ";
  if (I(r, "PHENOTYPE") == -1) trouble += "Need to set PHENOTYPE=0 or 1. ";
  if (I(r, "EXTRACOLS") < 0) trouble += "Need to set EXTRACOLS>=0. ";
  if (I(r, "LOCPRIOR") && I(r, "LOCDATA") < 0 && (I(r, "LOCISPOP") == 0 || I(r, "POPDATA") < 0))
    trouble += "Need to specify location data when LOCPRIOR is on. ";
  if (I(r, "LOCPRIOR") && I(r, "LINKAGE")) trouble += "Cannot run LOCPRIOR and LINKAGE together. ";
  if (!trouble.empty()) return fail(r, STF_ERR_PARAMS, "%s", trouble.c_str());
  r->num["UPDATEFREQ"] = update_freq(r);
  return STF_OK;
}

extern "C" int stf_close(stf_run* r) {
  if (!r) return STF_ERR_ARG;
  delete r;
  return STF_OK;
}

extern "C" const char* stf_last_error(const stf_run* r) { return r ? r->err.c_str() : ""; }

extern "C" int stf_param_int(const stf_run* r, const char* key, int* value) {
  if (!r || !key || !value) return STF_ERR_ARG;
  std::string k = key;
  if (const char* a = file_key(k)) k = a;
  auto it = r->num.find(k);
  if (it == r->num.end()) return STF_ERR_ARG;
  *value = (int)it->second;
  return STF_OK;
}

extern "C" int stf_set_param_int(stf_run* r, const char* key, int value) {
  if (!r || !key) return STF_ERR_ARG;
  std::string k = key;
  if (const char* a = file_key(k)) k = a;
  auto it = r->num.find(k);
  if (it == r->num.end()) return STF_ERR_ARG;
  it->second = value;
  return STF_OK;
}

extern "C" int stf_param_double(const stf_run* r, const char* key, double* value) {
  if (!r || !key || !value) return STF_ERR_ARG;
  auto it = r->num.find(key);
  if (it == r->num.end()) return STF_ERR_ARG;
  *value = it->second;
  return STF_OK;
}

extern "C" int stf_param_str(const stf_run* r, const char* key, char* buf, size_t n) {
  if (!r || !key || !buf || n == 0) return STF_ERR_ARG;
  std::string k = key;
  if (const char* a = file_key(k)) k = a;
  auto it = r->str.find(k);
  if (it == r->str.end()) return STF_ERR_ARG;
  snprintf(buf, n, "%s", it->second.c_str());
  return STF_OK;
}

// ===========================================================================
// data file (src/datain.c:65-333, 768-904)
// ===========================================================================
extern "C" int stf_read_data(stf_run* r) {
  if (!r) return STF_ERR_ARG;
  const int N = I(r, "NUMINDS"), L = I(r, "NUMLOCI"), LINES = I(r, "LINES");
  if (LINES != 2) return fail(r, STF_ERR_UNSUPPORTED, "PLOIDY=%d: the GPU path is diploid", LINES);
  if (I(r, "RECESSIVEALLELES"))
    return fail(r, STF_ERR_UNSUPPORTED, "RECESSIVEALLELES=1 is not on the GPU path");
  std::string text;
  if (!read_file(S(r, "DATAFILE"), &text))
    return fail(r, STF_ERR_IO, "Unable to open the file %s.", S(r, "DATAFILE").c_str());
  CharStream cs;
  cs.s = std::move(text);
  r->N = N; r->L = L; r->LINES = LINES;
  r->geno.assign((size_t)N * LINES * L, 0);
  r->markername.assign(L, "");
  r->ind.assign(N, Individual());
  const bool label = I(r, "LABEL") == 1, popdata = I(r, "POPDATA") == 1;
  const bool popflag = I(r, "POPFLAG") == 1, locdata = I(r, "LOCDATA") == 1;
  const bool phenotype = I(r, "PHENOTYPE") == 1;
  const int extracols = I(r, "EXTRACOLS");
  auto eof = [&](int i) {
    return fail(r, STF_ERR_DATA,
                "WARNING: Unexpected end of input file.  The data file ended while reading "
                "individual %d; check NUMINDS, NUMLOCI, ONEROWPERIND and the extra columns.",
                i + 1);
  };
  if (I(r, "MARKERNAMES"))
    for (int l = 0; l < L; l++) {
      std::string w = cs.word(kGeneLen);
      if (w.empty()) return eof(-1);
      r->markername[l] = w;
    }
  if (I(r, "MAPDISTANCES"))
    for (int l = 0; l < L; l++)
      if (cs.word(kAllelLen).empty()) return eof(-1);
  const bool onerow = I(r, "ONEROWPERIND") != 0;
  const int rows = onerow ? 1 : LINES, cols = onerow ? LINES : 1;
  int phencol = -1;
  if (phenotype) {
    const int pc = I(r, "PHENOTYPECOL");
    const int lo = (label ? 1 : 0) + (popdata ? 1 : 0) + (popflag ? 1 : 0);
    if (pc == -9) phencol = 0;
    else if (pc <= lo || pc > lo + 1 + extracols)
      return fail(r, STF_ERR_PARAMS, "PHENOTYPECOL=%d is outside %d..%d", pc, lo + 1,
                  lo + 1 + extracols);
    else phencol = pc - lo - 1;
  }
  bool valid = true;
  std::string bad;
  for (int i = 0; i < N; i++) {
    for (int line = 0; line < rows; line++) {
      std::string lab;
      int pop = -1, pf = -1, loc = -1, phen = -1;
      if (label) {
        lab = cs.word(kLabelLen);
        if (lab.empty()) return eof(i);
      }
      auto int_field = [&](int* v) -> bool {
        std::string w = cs.word(kAllelLen);
        if (w.empty()) return false;
        if (!valid_int_field(w)) {
          valid = false;
          if (bad.empty()) bad = "non-integer \"" + w + "\" for individual " + std::to_string(i + 1);
        }
        *v = atoi(w.c_str());
        return true;
      };
      if (popdata && !int_field(&pop)) return eof(i);
      if (popflag && !int_field(&pf)) return eof(i);
      if (locdata && !int_field(&loc)) return eof(i);
      if (phenotype) {
        for (int c = 0; c < extracols + 1; c++) {
          if (c == phencol) {
            if (!int_field(&phen)) return eof(i);
          } else {
            cs.word(kAllelLen);
          }
        }
      } else {
        for (int c = 0; c < extracols; c++) cs.word(kAllelLen);
      }
      Individual& d = r->ind[i];
      if (line == 0) {
        if (label) d.label = lab;
        if (popdata) d.population = pop;
        if (popflag) d.popflag = pf;
        if (phenotype) d.phenotype = phen;
        if (locdata) d.location = loc;
        if (I(r, "LOCISPOP")) d.location = pop;
      } else if (line > 1) {
        // the reference compares rows from the third on (src/datain.c:253),
        // so for diploid data the second row's fields are not checked
        if ((label && d.label != lab) || (popdata && d.population != pop) ||
            (popflag && d.popflag != pf) || (phenotype && d.phenotype != phen)) {
          valid = false;
          if (bad.empty())
            bad = "the rows of individual " + std::to_string(i + 1) + " disagree";
        }
      }
      for (int l = 0; l < L; l++)
        for (int c = 0; c < cols; c++) {
          int v;
          if (!int_field(&v)) return eof(i);
          r->geno[((size_t)i * LINES + (onerow ? c : line)) * L + l] = v;
        }
    }
    if (I(r, "PHASEINFO"))
      for (int l = 0; l < L; l++)
        if (cs.word(kAllelLen).empty()) return eof(i);
  }
  for (int c; (c = cs.get()) != EOF;)
    if (!white(c)) {
      valid = false;
      if (bad.empty()) bad = "data remain after the last individual (check NUMINDS/NUMLOCI)";
      break;
    }
  if (!valid) return fail(r, STF_ERR_DATA, "Error in the data file: %s", bad.c_str());

  // recoding: alleles 0..k-1 in order of first appearance (individuals, then
  // lines); a MISSING value that could collide with a code becomes -9
  const int missing = I(r, "MISSING");
  int maxk = 0;
  {
    std::vector<int> seen;
    for (int l = 0; l < L; l++) {
      seen.clear();
      for (int i = 0; i < N; i++)
        for (int line = 0; line < LINES; line++) {
          const int v = r->geno[((size_t)i * LINES + line) * L + l];
          if (v == missing) continue;
          bool found = false;
          for (int s : seen)
            if (s == v) { found = true; break; }
          if (!found) seen.push_back(v);
        }
      if ((int)seen.size() > maxk) maxk = (int)seen.size();
    }
  }
  const int A = maxk;
  const int newmissing = (missing >= 0 && missing < A + 1) ? -9 : missing;
  r->translation.assign((size_t)L * (A > 0 ? A : 1), 0);
  r->numalleles.assign(L, 0);
  for (int l = 0; l < L; l++) {
    int k = 0;
    for (int i = 0; i < N; i++)
      for (int line = 0; line < LINES; line++) {
        int32_t& g = r->geno[((size_t)i * LINES + line) * L + l];
        if (g == missing) {
          g = newmissing;
          continue;
        }
        int pos = 0;
        while (pos < k && r->translation[(size_t)l * A + pos] != g) pos++;
        if (pos == k) r->translation[(size_t)l * A + k++] = g;
        g = pos;
      }
    r->numalleles[l] = k;
  }
  r->MAXALLELES = A;
  r->orig_missing = missing;
  r->missing = newmissing;
  r->have_data = true;
  return STF_OK;
}

extern "C" int stf_dims(const stf_run* r, int dims[4]) {
  if (!r || !dims || !r->have_data) return STF_ERR_ARG;
  dims[0] = r->N; dims[1] = r->L; dims[2] = r->LINES; dims[3] = r->MAXALLELES;
  return STF_OK;
}

extern "C" int stf_geno(const stf_run* r, int32_t* geno, int32_t* numalleles,
                        int32_t* translation) {
  if (!r || !r->have_data) return STF_ERR_ARG;
  if (geno) memcpy(geno, r->geno.data(), r->geno.size() * 4);
  if (numalleles) memcpy(numalleles, r->numalleles.data(), r->numalleles.size() * 4);
  if (translation) memcpy(translation, r->translation.data(), r->translation.size() * 4);
  return STF_OK;
}

extern "C" int stf_individuals(const stf_run* r, int32_t* pop, int32_t* popflag,
                               int32_t* location, int32_t* phenotype, char* labels) {
  if (!r || !r->have_data) return STF_ERR_ARG;
  for (int i = 0; i < r->N; i++) {
    const Individual& d = r->ind[i];
    if (pop) pop[i] = d.population;
    if (popflag) popflag[i] = d.popflag;
    if (location) location[i] = d.location;
    if (phenotype) phenotype[i] = d.phenotype;
    if (labels) snprintf(labels + (size_t)i * kLabelLen, kLabelLen, "%s", d.label.c_str());
  }
  return STF_OK;
}

// The prior-population checks of src/Init.c:15-70 CheckPopPriors: MIGRPRIOR
// in [0, 1] and POPDATA present, every individual flagged when the file has
// no POPFLAG column, flags dropped where the population is outside
// 1..MAXPOPS, and alpha switched off (INFERALPHA=0) when no individual is
// left without prior information in the admixture model.
extern "C" int stf_check_pop_priors(stf_run* r, int32_t* dropped) {
  if (!r || !r->have_data) return STF_ERR_ARG;
  if (dropped) *dropped = 0;
  if (!I(r, "USEPOPINFO")) return STF_OK;
  const double migr = D(r, "MIGRPRIOR");
  if (migr < 0.0 || migr > 1.0)
    return fail(r, STF_ERR_PARAMS,
                "MIGRPRIOR (which is currently set to %1.3f) must be in the range [0.0, 1.0]",
                migr);
  if (!I(r, "POPDATA"))
    return fail(r, STF_ERR_PARAMS, "Can't apply USEPOPINFO because no POPDATA in input data file");
  const int K = I(r, "MAXPOPS");
  if (!I(r, "POPFLAG"))
    for (Individual& d : r->ind) d.popflag = 1;
  int nopop = 0;
  for (Individual& d : r->ind) {
    if (d.popflag && (d.population < 1 || d.population > K)) {
      d.popflag = 0;
      if (dropped) ++*dropped;
    }
    if (d.popflag == 0) nopop++;
  }
  if (I(r, "INFERALPHA") && !I(r, "NOADMIX") && nopop == 0) {
    r->noalpha = true;
    r->num["INFERALPHA"] = 0;
  }
  return STF_OK;
}

namespace {
// Location ids in increasing order: location l of the engine is ids[l]
// (src/Util.c:237-275 GetNumLocations; output.c:1009-1018 get_location_num).
std::vector<int> location_ids(const stf_run* r) {
  std::vector<int> ids;
  for (const Individual& d : r->ind) ids.push_back(d.location);
  std::sort(ids.begin(), ids.end());
  ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
  return ids;
}
}  // namespace

extern "C" int stf_num_locations(const stf_run* r) {
  if (!r || !r->have_data) return STF_ERR_ARG;
  return (int)location_ids(r).size();
}

extern "C" int stf_set_locprior_sums(stf_run* r, const double* sums, size_t n) {
  if (!r || !r->have_data) return STF_ERR_ARG;
  if (!sums) {
    r->sumlocp.clear();
    return STF_OK;
  }
  const size_t need = I(r, "NOADMIX") ? 1 + (size_t)I(r, "MAXPOPS") * (location_ids(r).size() + 1) : 1;
  if (n != need) return fail(r, STF_ERR_ARG, "sumLocPrior: %zu values given, %zu expected", n, need);
  r->sumlocp.assign(sums, sums + n);
  return STF_OK;
}

extern "C" int stf_set_save_number(stf_run* r, int savenum) {
  if (!r || savenum < 0) return STF_ERR_ARG;
  r->savenum = savenum;
  return STF_OK;
}

extern "C" int stf_set_usepopprobs(stf_run* r, const double* usepop) {
  if (!r || !r->have_data) return STF_ERR_ARG;
  if (!usepop) {
    r->usepop.clear();
    return STF_OK;
  }
  const size_t n = (size_t)r->N * I(r, "MAXPOPS") * (I(r, "GENSBACK") + 1);
  r->usepop.assign(usepop, usepop + n);
  return STF_OK;
}

// ===========================================================================
// results (src/output.c:1354-1423 and the printers it calls)
// ===========================================================================
namespace {

struct Out {
  std::string s;
  void f(const char* fmt, ...) {
    char buf[4096];
    va_list ap;
    va_start(ap, fmt);
    const int n = vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (n >= (int)sizeof buf) {
      std::vector<char> big((size_t)n + 1);
      va_start(ap, fmt);
      vsnprintf(big.data(), big.size(), fmt, ap);
      va_end(ap);
      s.append(big.data(), (size_t)n);
    } else if (n > 0) {
      s.append(buf, (size_t)n);
    }
  }
};

struct Sums {
  int rep;
  const double *QSum, *PSum, *SumEps, *FstSum, *sumAlpha, *sumlambda;
  const int32_t* AncestDist;
  double sumlikes, sumsqlikes;
};

double sample_var(double sumsq, double sum, long num) {
  return num == 1 ? 0.0 : (sumsq - sum * sum / num) / (num - 1);
}

void banner(Out& o) {
  o.f("\n\n");
  o.f("----------------------------------------------------\n");
  o.f("STRUCTURE by Pritchard, Stephens and Donnelly (2000)\n");
  o.f("     and Falush, Stephens and Pritchard (2003)\n");
  o.f("       Code by Pritchard, Falush and Hubisz\n");
  o.f("             Version %s\n", kVersion);
  o.f("----------------------------------------------------\n");
  o.f("\n\n");
}

void main_params(const stf_run* r, Out& o, int rep) {
  o.f("\n");
  if (r->argv.size() > 1) {
    o.f("Command line arguments:   ");
    for (const std::string& a : r->argv) o.f("%s ", a.c_str());
    o.f("\n");
  }
  o.f("Input File:    %s\n", S(r, "DATAFILE").c_str());
  o.f("\n");
  o.f("Run parameters:\n");
  o.f("   %d individuals\n", I(r, "NUMINDS"));
  o.f("   %d loci\n", I(r, "NUMLOCI"));
  o.f("   %d populations assumed\n", I(r, "MAXPOPS"));
  o.f("   %d Burn-in period\n", I(r, "BURNIN"));
  o.f("   %d Reps\n", rep - I(r, "BURNIN"));
  if (I(r, "USEPOPINFO")) {
    o.f("USEPOPINFO turned on\n");
    o.f("MIGRPRIOR = %1.4f\n", D(r, "MIGRPRIOR"));
  }
  if (I(r, "RECESSIVEALLELES")) o.f("RECESSIVE ALLELES model used\n");
  if (I(r, "NOADMIX")) o.f("NO ADMIXTURE model assumed\n");
  if (I(r, "STARTATPOPINFO")) o.f("STARTATPOPINFO turned on\n");
  if (I(r, "LOCPRIOR")) o.f("LOCPRIOR model used\n");
  if (!I(r, "RANDOMIZE")) o.f("RANDOMIZE turned off\n");
  o.f("\n");
}

void membership(const stf_run* r, Out& o, const double* QSum) {
  const int K = I(r, "MAXPOPS"), N = r->N;
  std::vector<double> sv(K);
  if (I(r, "POPDATA")) {
    int minp = r->ind[0].population, maxp = minp;
    for (int i = 1; i < N; i++) {
      minp = std::min(minp, r->ind[i].population);
      maxp = std::max(maxp, r->ind[i].population);
    }
    o.f("\n--------------------------------------------\n");
    o.f("Proportion of membership of each pre-defined\n");
    o.f(" population in each of the %d clusters\n\n", K);
    o.f("Given    Inferred Clusters");
    for (int k = 3; k < K; k++) o.f("       ");
    o.f("       Number of\n");
    o.f(" Pop    ");
    for (int k = 0; k < K; k++) o.f("  %2d   ", k + 1);
    for (int k = K; k < 3; k++) o.f("       ");
    o.f("   Individuals\n\n");
    for (int gp = minp; gp <= maxp; gp++) {
      std::fill(sv.begin(), sv.end(), 0.0);
      int n = 0;
      for (int i = 0; i < N; i++)
        if (r->ind[i].population == gp) {
          n++;
          for (int k = 0; k < K; k++) sv[k] += QSum[(size_t)i * K + k];
        }
      double rs = 0.0;
      for (int k = 0; k < K; k++) rs += sv[k];
      if (rs > 0.0) {
        o.f("%3d:     ", gp);
        for (int k = 0; k < K; k++) o.f("%1.3f  ", sv[k] / rs);
        for (int k = K; k < 3; k++) o.f("       ");
        o.f("    %3d\n", n);
      }
    }
  } else {
    for (int i = 0; i < N; i++)
      for (int k = 0; k < K; k++) sv[k] += QSum[(size_t)i * K + k];
    double rs = 0.0;
    for (int k = 0; k < K; k++) rs += sv[k];
    o.f("\n--------------------------------------------\n");
    o.f("Overall proportion of membership of the\n");
    o.f("sample in each of the %d clusters\n\n", K);
    o.f("Inferred Clusters\n");
    for (int k = 0; k < K; k++) o.f(" %2d    ", k + 1);
    o.f("\n");
    for (int k = 0; k < K; k++) o.f("%1.3f  ", sv[k] / rs);
    o.f("\n\n");
  }
  o.f("--------------------------------------------\n");
}

// Net and gross nucleotide distances between clusters from PSum / reps
// (src/output.c:470-520).
double net_d(const stf_run* r, int p1, int p2, const double* P, int reps) {
  const int K = I(r, "MAXPOPS"), A = r->MAXALLELES;
  double norm = (double)reps;
  norm *= norm;
  double sum = 0.0;
  for (int l = 0; l < r->L; l++) {
    double d1 = 0.0, d2 = 0.0, d12 = 0.0;
    for (int a = 0; a < r->numalleles[l]; a++) {
      const double x = P[((size_t)l * K + p1) * A + a], y = P[((size_t)l * K + p2) * A + a];
      d1 += x * x / norm;
      d2 += y * y / norm;
      d12 += x * y / norm;
    }
    sum += 0.5 * (d1 + d2) - d12;
  }
  return sum / r->L;
}

double gross_d(const stf_run* r, int p1, int p2, const double* P, int reps) {
  const int K = I(r, "MAXPOPS"), A = r->MAXALLELES;
  double norm = (double)reps;
  norm *= norm;
  double sum = 0.0;
  for (int l = 0; l < r->L; l++) {
    double d12 = 0.0;
    for (int a = 0; a < r->numalleles[l]; a++)
      d12 += P[((size_t)l * K + p1) * A + a] * P[((size_t)l * K + p2) * A + a] / norm;
    sum += 1.0 - d12;
  }
  return sum / r->L;
}

void net_table(const stf_run* r, Out& o, const double* P, int reps) {
  const int K = I(r, "MAXPOPS");
  o.f("\nAllele-freq. divergence among pops (Net nucleotide distance)");
  if (reps > 1) o.f(",\ncomputed using point estimates of P");
  o.f(".\n\n");
  o.f("     ");
  for (int j = 0; j < K; j++) o.f("%2d      ", j + 1);
  o.f("\n");
  for (int i = 0; i < K; i++) {
    o.f("%2d   ", i + 1);
    for (int j = 0; j < K; j++) {
      if (i == j) o.f("   -    ");
      else o.f("%1.4f  ", net_d(r, i, j, P, reps));
    }
    o.f("\n");
  }
  o.f("\nAverage distances (expected heterozygosity) between individuals in same cluster:\n");
  for (int i = 0; i < K; i++) o.f("cluster %2d  : %1.4f \n", i + 1, gross_d(r, i, i, P, reps));
  o.f("\n");
}

// The column heads of the screen trace (src/output.c:377-454 PrintBanner):
// one head per printed column of trace_line, widened by a space per digit of
// rep beyond five (and beyond nine before the likelihood heads).
void trace_banner(const stf_run* r, Out& o, int rep) {
  const int K = I(r, "MAXPOPS"), digits = (int)log10((double)rep);
  o.f("\n");
  for (int i = 4; i < digits; i++) o.f(" ");
  o.f(" Rep#:   ");
  if (I(r, "PRINTLAMBDA")) {
    if (I(r, "POPSPECIFICLAMBDA"))
      for (int k = 0; k < K; k++) o.f("Lambda%d ", k + 1);
    else
      o.f("Lambda  ");
  }
  if (!I(r, "NOADMIX") && !r->noalpha) {
    o.f(" ");
    if (I(r, "POPALPHAS"))
      for (int k = 0; k < K; k++) o.f("Alpha%d ", k + 1);
    else
      o.f("Alpha  ");
  }
  if (I(r, "FREQSCORR")) {
    o.f("   ");
    if (I(r, "ONEFST")) o.f("Fst   ");
    else
      for (int k = 0; k < K; k++) o.f(" F%d   ", k + 1);
    o.f(" ");
  } else {
    o.f(" ");
  }
  if (I(r, "LOCPRIOR")) o.f("  r     ");
  if (I(r, "PRINTKLD") || I(r, "PRINTNET"))
    for (int i = 0; i < K - 1; i++)
      for (int j = i + 1; j < K; j++) o.f(" D%d,%d ", i + 1, j + 1);
  if (I(r, "COMPUTEPROB")) {
    o.f("   Ln Like ");
    for (int i = 8; i < digits; i++) o.f(" ");
    if (rep >= I(r, "BURNIN")) o.f(" Est Ln P(D)");
  }
  o.f("\n");
}

void sums(const stf_run* r, Out& o, const Sums& s) {
  const int K = I(r, "MAXPOPS"), reps = s.rep - I(r, "BURNIN");
  o.f("--------------------------------------------\n");
  if (I(r, "COMPUTEPROB")) {
    if (reps > 2) {
      const double mean = s.sumlikes / reps;
      const double var = sample_var(s.sumsqlikes, s.sumlikes, reps);
      o.f("Estimated Ln Prob of Data   = %1.1f\n", mean - var / 2.0);
      o.f("Mean value of ln likelihood = %1.1f\n", s.sumlikes / reps);
      o.f("Variance of ln likelihood   = %1.1f\n", var);
    } else {
      o.f("Mean value of ln likelihood = %1.1f\n", s.sumlikes / reps);
    }
  }
  const bool locprior = I(r, "LOCPRIOR") != 0;
  const std::vector<int> ids = locprior ? location_ids(r) : std::vector<int>();
  if (!I(r, "NOADMIX") && !r->noalpha && K > 1) {
    if (I(r, "POPALPHAS")) {
      o.f("\n");
      for (int k = 0; k < K; k++)
        o.f("Mean value of alpha_%d       = %1.4f\n", k + 1, s.sumAlpha[k] / reps);
    } else {
      o.f("Mean value of alpha         = %1.4f\n", s.sumAlpha[0] / reps);
    }
    if (locprior) {
      // src/output.c:1061-1071: rows of alpha after the global one
      o.f("\nMean value of alpha_local for each location:\n");
      for (size_t l = 0; l < ids.size(); l++) {
        o.f("\tlocation %2i:", ids[l]);
        for (int k = 0; k < K; k++) o.f("  %1.4f", s.sumAlpha[(size_t)K * (l + 1) + k] / reps);
        o.f("\n");
      }
    }
  }
  if (I(r, "INFERLAMBDA")) {
    if (I(r, "POPSPECIFICLAMBDA"))
      for (int k = 0; k < K; k++)
        o.f("\nMean value of lambda%d       = %1.4f\n", k + 1, s.sumlambda[k] / reps);
    else
      o.f("\nMean value of lambda        = %1.4f\n", s.sumlambda[0] / reps);
  }
  if (I(r, "FREQSCORR")) {
    if (I(r, "ONEFST")) {
      o.f("Mean value of Fst           = %1.4f\n", s.FstSum[0] / reps);
    } else {
      o.f("\n");
      for (int k = 0; k < K; k++)
        o.f("Mean value of Fst_%d         = %1.4f\n", k + 1, s.FstSum[k] / reps);
    }
  } else {
    o.f("Allele frequencies uncorrelated\n");
  }
  if (I(r, "PFROMPOPFLAGONLY"))
    o.f("Allele frequencies updated using individuals with POPFLAG=1 ONLY.\n");
  o.f("\n");
  if (locprior) {
    // src/output.c:1120-1139
    const double* sl = r->sumlocp.data();
    o.f("Mean value of r = %1.4f\n", sl[0] / reps);
    if (I(r, "NOADMIX")) {
      o.f("Mean value of nu = ");
      for (int k = 0; k < K; k++) o.f(" %1.4f", sl[1 + k] / reps);
      o.f("\n");
      o.f("Mean value of gamma for each location:\n");
      for (size_t l = 0; l < ids.size(); l++) {
        o.f("\tlocation %2i:", ids[l]);
        for (int k = 0; k < K; k++) o.f("  %1.4f", sl[1 + (size_t)K * (l + 1) + k] / reps);
        o.f("\n");
      }
    }
  }
}

int missing_ind(const stf_run* r, int i) {
  int n = 0;
  for (int line = 0; line < r->LINES; line++)
    for (int l = 0; l < r->L; l++)
      if (r->geno[((size_t)i * r->LINES + line) * r->L + l] == r->missing) n++;
  return n;
}

int missing_loc(const stf_run* r, int l) {
  int n = 0;
  for (int i = 0; i < r->N; i++)
    for (int line = 0; line < r->LINES; line++)
      if (r->geno[((size_t)i * r->LINES + line) * r->L + l] == r->missing) n++;
  return n;
}

void ancest_interval(const stf_run* r, Out& o, const int32_t* AD, int i, int rep) {
  const int K = I(r, "MAXPOPS"), B = I(r, "NUMBOXES"), burn = I(r, "BURNIN");
  const double pint = D(r, "ANCESTPINT");
  o.f("    ");
  for (int k = 0; k < K; k++) {
    double sum = 0.0;
    int low = 0;
    for (int b = 0; b < B; b++) {
      sum += AD[((size_t)i * K + k) * B + b];
      if (low == 0 && sum > (int)((rep - burn) * (1.0 - pint) / 2.0)) {
        o.f("(%1.3f,", (double)(b + 0.0) / B);
        low = 1;
      }
      if (sum > ((rep - burn) * (1 + pint) / 2.0)) {
        o.f("%1.3f) ", (double)(b + 1.0) / B);
        break;
      }
    }
  }
}

// Posterior of the migrant model for an individual with prior information:
// P(from the given population) | for every other population, P(migrant
// ancestry from it) for 0..GENSBACK generations back, with one to three
// stars when P(given population) is below 0.5, 0.3, 0.1
// (src/output.c:800-829 PrintGeogQ).
void geog_q(const stf_run* r, Out& o, int i, int reps) {
  const int K = I(r, "MAXPOPS"), G = I(r, "GENSBACK") + 1;
  const int home = r->ind[i].population - 1;
  const double* u = r->usepop.data() + (size_t)i * K * G;
  const double ph = u[(size_t)home * G] / reps;
  o.f("%1.3f | ", ph);
  for (int k = 0; k < K; k++)
    if (k != home) {
      o.f("Pop %d: ", k + 1);
      for (int g = 0; g < G; g++) o.f("%1.3f ", u[(size_t)k * G + g] / reps);
      o.f(" | ");
    }
  o.f(" ");
  if (ph < 0.1) o.f("*");
  if (ph < 0.3) o.f("*");
  if (ph < 0.5) o.f("*");
}

void ancestry(const stf_run* r, Out& o, const Sums& s) {
  const int K = I(r, "MAXPOPS"), reps = s.rep - I(r, "BURNIN");
  const bool label = I(r, "LABEL") == 1, popdata = I(r, "POPDATA") == 1;
  const bool usepop = I(r, "USEPOPINFO") != 0;
  o.f("\n");
  o.f("Inferred ancestry of individuals:\n");
  if (usepop) o.f("Probability of being from assumed population | prob of other pops\n");
  o.f("    ");
  if (label) o.f(" %8s", "Label");
  o.f(" (%%Miss) ");
  if (popdata) o.f("Pop");
  if (!usepop) {
    o.f(":  ");
    o.f("Inferred clusters");
    if (I(r, "ANCESTDIST"))
      o.f(" (and %d%c probability intervals)", (int)(100.0 * D(r, "ANCESTPINT")), '%');
  }
  o.f("\n");
  for (int i = 0; i < r->N; i++) {
    const int miss = (100 * missing_ind(r, i)) / (r->LINES * r->L);
    o.f("%3d ", i + 1);
    if (label) o.f("%8s ", r->ind[i].label.c_str());
    if (miss < 10) o.f(" ");
    o.f("  (%d) ", miss);
    o.f("  ");
    if (popdata) o.f("%2d ", r->ind[i].population);
    o.f(":  ");
    if (usepop && r->ind[i].popflag) {
      geog_q(r, o, i, reps);
    } else {
      for (int k = 0; k < K; k++) o.f("%1.3f ", s.QSum[(size_t)i * K + k] / reps);
      if (I(r, "ANCESTDIST") && s.AncestDist) ancest_interval(r, o, s.AncestDist, i, s.rep);
    }
    o.f("\n");
  }
}

void gene_name(const stf_run* r, Out& o, int l) {
  const std::string& n = r->markername[l];
  if (n.empty()) o.f("XXX");
  else o.f("%s", n.c_str());
  o.f(" ");
}

void allele_freqs(const stf_run* r, Out& o, const Sums& s) {
  const int K = I(r, "MAXPOPS"), A = r->MAXALLELES, reps = s.rep - I(r, "BURNIN");
  const bool fc = I(r, "FREQSCORR") != 0;
  o.f("\n\nEstimated Allele Frequencies in each cluster\n");
  if (fc) o.f("First column gives estimated ancestral frequencies\n");
  o.f("\n\n");
  for (int l = 0; l < r->L; l++) {
    o.f("Locus %d : ", l + 1);
    if (I(r, "MARKERNAMES")) gene_name(r, o, l);
    o.f("\n");
    o.f("%d alleles\n", r->numalleles[l]);
    o.f("%2.1f%c missing data\n", (double)100.0 * missing_loc(r, l) / (r->LINES * r->N), '%');
    for (int a = 0; a < r->numalleles[l]; a++) {
      o.f("%4d   ", r->translation[(size_t)l * A + a]);
      if (fc) o.f("(%1.3f) ", (s.SumEps ? s.SumEps[(size_t)l * A + a] : 0.0) / reps);
      for (int k = 0; k < K; k++) o.f("%1.3f ", s.PSum[((size_t)l * K + k) * A + a] / reps);
      o.f("\n");
    }
    o.f("\n");
  }
}

void all_params(const stf_run* r, Out& o) {
  o.f("Values of parameters used in structure:\n");
  o.f("DATAFILE=%s,\t", S(r, "DATAFILE").c_str());
  o.f("OUTFILE=%s,\t", S(r, "OUTFILE").c_str());
  o.f("NUMINDS=%d,\t", I(r, "NUMINDS"));
  o.f("NUMLOCI=%d,\t", I(r, "NUMLOCI"));
  o.f("MISSING=%d,\t", r->have_data ? r->orig_missing : I(r, "MISSING"));
  const char* ints1[] = {"LABEL", "POPDATA", "POPFLAG", "PHENOTYPE", "EXTRACOLS", "MAXPOPS",
                         "BURNIN", "NUMREPS", "USEPOPINFO", "INFERALPHA", "INFERLAMBDA",
                         "POPSPECIFICLAMBDA", "POPALPHAS", "COMPUTEPROB", "NOADMIX",
                         "ADMBURNIN", "UPDATEFREQ", "PRINTLIKES", "INTERMEDSAVE", "PRINTKLD",
                         "PRINTNET", "PRINTLAMBDA", "ANCESTDIST", "NUMBOXES"};
  for (const char* k : ints1) o.f("%s=%d,\t", k, I(r, k));
  o.f("ANCESTPINT=%1.5f,\t", D(r, "ANCESTPINT"));
  o.f("GENSBACK=%d,\t", I(r, "GENSBACK"));
  o.f("MIGRPRIOR=%1.5f,\t", D(r, "MIGRPRIOR"));
  o.f("PRINTQHAT=%d,\t", I(r, "PRINTQHAT"));
  o.f("PRINTQSUM=%d,\t", I(r, "PRINTQSUM"));
  o.f("ALPHA=%1.4f,\t", D(r, "ALPHA"));
  o.f("FREQSCORR=%d,\t", I(r, "FREQSCORR"));
  o.f("FPRIORMEAN=%1.4f,\t", D(r, "FPRIORMEAN"));
  o.f("FPRIORSD=%1.4f,\t", D(r, "FPRIORSD"));
  o.f("ONEFST=%d,\t", I(r, "ONEFST"));
  o.f("LAMBDA=%1.4f,\t", D(r, "LAMBDA"));
  o.f("UNIFPRIORALPHA=%d,\t", I(r, "UNIFPRIORALPHA"));
  o.f("ALPHAMAX=%1.4f,\t", D(r, "ALPHAMAX"));
  o.f("ALPHAPRIORA=%1.4f,\t", D(r, "ALPHAPRIORA"));
  o.f("ALPHAPRIORB=%1.4f,\t", D(r, "ALPHAPRIORB"));
  o.f("ALPHAPROPSD=%1.4f,\t", D(r, "ALPHAPROPSD"));
  const char* ints2[] = {"STARTATPOPINFO", "RANDOMIZE", "LINKAGE", "METROFREQ",
                         "REPORTHITRATE", "MARKOVPHASE", "PHASED"};
  for (const char* k : ints2) o.f("%s=%d,\t", k, I(r, k));
  o.f("PLOIDY=%d,\t", I(r, "LINES"));
  o.f("PHASEINFO=%d\t", I(r, "PHASEINFO"));
  o.f("LOCPRIOR=%d, \t", I(r, "LOCPRIOR"));
  o.f("LOCPRIORINIT=%f, \t", D(r, "LOCPRIORINIT"));
  o.f("LOCDATA=%d, \t", I(r, "LOCDATA"));
  o.f("LOCISPOP=%d, \t", I(r, "LOCISPOP"));
  o.f("LOCPRIORSTEP=%f, \t", D(r, "LOCPRIORSTEP"));
  o.f("MAXLOCPRIOR=%f, \t", D(r, "MAXLOCPRIOR"));
  o.f("SEED=%d,\t", I(r, "SEED"));
  o.f("\n[STRAT parameters]:    ");
  o.f("NUMSIMSTATS=%d,\t", I(r, "NUMSIMSTATS"));
  o.f("PHENOTYPECOL=%d,\t", I(r, "PHENOTYPECOL"));
  o.f("POOLFREQ=%d,\t", I(r, "POOLFREQ"));
  o.f("LOCUSxONLY=%d,\t", I(r, "LOCUSxONLY"));
  o.f("EMERROR=%1.5f,\t", D(r, "EMERROR"));
  o.f("MISSINGPHENO=%d,\t", I(r, "MISSINGPHENO"));
}

bool write_text(const std::string& path, const std::string& text) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = fwrite(text.data(), 1, text.size(), f) == text.size();
  return fclose(f) == 0 && ok;
}

}  // namespace

extern "C" int stf_write_results(stf_run* r, int rep, const double* QSum, const double* PSum,
                                 const double* SumEpsilon, const double* FstSum,
                                 const double* sumAlpha, const double* sumlambda,
                                 const int32_t* AncestDist, double sumlikes,
                                 double sumsqlikes) {
  if (!r || !r->have_data || !QSum || !PSum || !FstSum || !sumAlpha) return STF_ERR_ARG;
  if (rep - I(r, "BURNIN") < 1) return fail(r, STF_ERR_ARG, "no collected sweeps to report");
  if (I(r, "USEPOPINFO") && r->usepop.empty())
    return fail(r, STF_ERR_ARG, "USEPOPINFO=1: give the UsePopProbs sums (stf_set_usepopprobs)");
  if (I(r, "LOCPRIOR") && r->sumlocp.empty())
    return fail(r, STF_ERR_ARG, "LOCPRIOR=1: give the LocPrior sums (stf_set_locprior_sums)");
  const Sums s{rep, QSum, PSum, SumEpsilon, FstSum, sumAlpha, sumlambda, AncestDist, sumlikes,
               sumsqlikes};
  Out o;
  banner(o);
  main_params(r, o, rep);
  membership(r, o, QSum);
  net_table(r, o, PSum, rep - I(r, "BURNIN"));
  sums(r, o, s);
  ancestry(r, o, s);
  allele_freqs(r, o, s);
  all_params(r, o);
  // src/output.c:1381-1385: OUTFILE_f at the end, OUTFILE_<n> for the n-th
  // intermediate save (INTERMEDSAVE); OUTFILE_q only at the end
  const std::string name =
      S(r, "OUTFILE") + (r->savenum > 0 ? "_" + std::to_string(r->savenum) : std::string("_f"));
  if (!write_text(name, o.s)) return fail(r, STF_ERR_IO, "Unable to open output file %s.", name.c_str());
  if (I(r, "PRINTQHAT") && r->savenum == 0) {
    // src/output.c:914-953 PrintQFile
    Out q;
    const int K = I(r, "MAXPOPS"), reps = rep - I(r, "BURNIN");
    for (int i = 0; i < r->N; i++) {
      if (I(r, "LABEL") == 1) q.f("%12s ", r->ind[i].label.c_str());
      else q.f("%4d ", i + 1);
      if (I(r, "POPDATA") == 1) q.f("%2d ", r->ind[i].population);
      for (int k = 0; k < K; k++) q.f("%1.4f ", QSum[(size_t)i * K + k] / reps);
      q.f("\n");
    }
    const std::string qn = S(r, "OUTFILE") + "_q";
    if (!write_text(qn, q.s)) return fail(r, STF_ERR_IO, "Unable to open output file %s.", qn.c_str());
  }
  return STF_OK;
}

namespace {

// Copies text into buf as snprintf would (NUL-terminated, truncated to n-1
// bytes) and returns its full length.
int give_text(const std::string& s, char* buf, size_t n) {
  if (buf && n > 0) {
    const size_t m = std::min(s.size(), n - 1);
    memcpy(buf, s.data(), m);
    buf[m] = '\0';
  }
  return (int)s.size();
}

}  // namespace

extern "C" int stf_format_update(const stf_run* r, int rep, const double* Q, const double* P,
                                 const double* alpha, const double* F, const double* lambda,
                                 double like, const double* locprior, char* buf, size_t n) {
  if (!r || !r->have_data || rep < 1 || !alpha || !F || !lambda) return STF_ERR_ARG;
  const int K = I(r, "MAXPOPS"), burnin = I(r, "BURNIN"), every = I(r, "UPDATEFREQ");
  const bool printnet = I(r, "PRINTKLD") || I(r, "PRINTNET");
  const bool banner_now = rep == every || (rep < burnin && rep % (10 * every) == 0) ||
                          (rep > burnin && (rep - burnin) % (10 * every) == 0);
  const bool membership_now = banner_now && rep != burnin + I(r, "NUMREPS") && rep > 1 &&
                              I(r, "PRINTQSUM") && K > 1;
  if (I(r, "LINKAGE")) return STF_ERR_UNSUPPORTED;
  if ((printnet && !P) || (membership_now && !Q) || (I(r, "LOCPRIOR") && !locprior))
    return STF_ERR_ARG;
  Out o;
  if (rep > burnin && rep < burnin + every) o.f("\nBURNIN completed");
  const int admburnin = I(r, "ADMBURNIN");
  if (I(r, "NOADMIX") && admburnin > 0 && !I(r, "LOCPRIOR") && rep >= admburnin &&
      rep < admburnin + every) {
    o.f("\nAdmixture Burnin complete.  Current alpha");
    if (I(r, "POPALPHAS")) {
      o.f("s = ");
      for (int k = 0; k < K; k++) o.f("%1.3f ", alpha[k]);
    } else {
      o.f(" = %1.3f ", alpha[0]);
    }
    o.f("\n\n");
  }
  if (banner_now && rep != burnin + I(r, "NUMREPS")) {
    if (membership_now) membership(r, o, Q);
    trace_banner(r, o, rep);
  }
  o.f("%5d:    ", rep);
  if (I(r, "PRINTLAMBDA")) {
    const int nl = I(r, "POPSPECIFICLAMBDA") ? K : 1;
    for (int k = 0; k < nl; k++) o.f("%1.2f    ", lambda[k]);
  }
  if (!I(r, "NOADMIX") && !r->noalpha) {
    if (I(r, "POPALPHAS"))
      for (int k = 0; k < K; k++) o.f(k > 8 ? "%1.3f   " : "%1.3f  ", alpha[k]);
    else
      o.f("%1.3f  ", alpha[0]);
  }
  if (I(r, "FREQSCORR")) {
    o.f("  ");
    const int nf = I(r, "ONEFST") ? 1 : K;
    for (int k = 0; k < nf; k++) o.f("%1.3f ", F[k]);
    o.f("   ");
  } else {
    o.f("  ");
  }
  if (I(r, "LOCPRIOR")) o.f("%1.3f    ", locprior[0]);
  if (printnet)
    for (int i = 0; i < K - 1; i++)
      for (int j = i + 1; j < K; j++) o.f("%1.3f ", net_d(r, i, j, P, 1));
  if (I(r, "COMPUTEPROB")) {
    // the reference evaluates Est Ln P(D) for this line only in its linkage
    // branch (src/output.c:258-279), so outside it the column holds 0
    if (rep > burnin + 2) o.f("  %.0f    %.0f ", like, 0.0);
    else o.f("  --  ");
  }
  o.f("\n");
  if (rep == burnin) {
    o.f("\nBURNIN completed");
    trace_banner(r, o, rep);
  }
  return give_text(o.s, buf, n);
}

extern "C" int stf_echo_data(const stf_run* r, char* buf, size_t n) {
  if (!r || !r->have_data) return STF_ERR_ARG;
  const int N = r->N, L = r->L, LINES = r->LINES, A = std::max(r->MAXALLELES, 1);
  const bool label = I(r, "LABEL") != 0, popdata = I(r, "POPDATA") != 0;
  const bool popflag = I(r, "POPFLAG") != 0, phenotype = I(r, "PHENOTYPE") != 0;
  const int precols = (int)label + (int)popdata + (int)popflag + (int)phenotype;
  Out o;
  o.f("\n\nData file \"%s\" (truncated) --\n\n", S(r, "DATAFILE").c_str());
  o.f("Ind:   ");
  if (label) o.f("%5s ", "Label");
  if (popdata) o.f("Pop ");
  if (popflag) o.f("Flag ");
  if (phenotype) o.f("Phen ");
  if (precols > 1) o.f(": ");
  o.f("Genotype_data . . . .\n");
  // the values as the file gives them: codes back through the allele table
  auto raw = [&](int i, int line, int l) {
    const int v = r->geno[((size_t)i * LINES + line) * L + l];
    return v == r->missing ? r->orig_missing : r->translation[(size_t)l * A + v];
  };
  // individuals 1..4 and the last two when there are more than 2 * LINES + 2
  // (src/structure.h:15 MAXINDS = 3, src/datain.c:566-570)
  const bool cut = N > 3 * LINES && N > 6;
  const int shown = std::min(L, 9 - precols);
  for (int i = 0; i < N; i++) {
    if (cut && i > 3 && i < N - 2) continue;
    for (int line = 0; line < LINES; line++) {
      o.f("%3d: ", i + 1);
      const Individual& d = r->ind[i];
      if (label) o.f("%5s ", d.label.c_str());
      if (popdata) o.f("%4d ", d.population);
      if (popflag) o.f("%4d ", d.popflag);
      if (phenotype) o.f("%4d ", d.phenotype);
      if (precols > 1) o.f(" :");
      for (int l = 0; l < shown; l++) o.f("%3d ", raw(i, line, l));
      if (L > shown) o.f(" . . . . %3d\n", raw(i, line, L - 1));
      else o.f("\n");
    }
    if (cut && i == 3) o.f("\n      *******   \n\n");
  }
  o.f("\n");
  return give_text(o.s, buf, n);
}
