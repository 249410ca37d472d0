// askja -- command-line driver of the B200 engine, a drop-in for the
// reference's `./askja params_file` (sun.cpp:1059-1373).
//
// Same params file, same output-DIM<D>/ directory, same constraints-/Wilson-
// diagnostics (every UPDATE steps), same U-*.conf configurations and
// master-*.params (every CONFTAKE trajectories), same step schedule: the first
// trajectory has UPDATE2-1 link updates, later ones UPDATE2 (sun.cpp:1212-1249),
// STEPS counts MD steps.  Differences, all documented:
//  - momenta and Metropolis uniforms come from Philox keyed by the seed
//    (RANDOM=0: 120351616, RANDOM=1 and every resume: time(NULL)), not GSL;
//  - the Wilson- file's eigenphase columns (never initialised by the
//    reference, sun.cpp:1119) are written as 0;
//  - `--fp32` selects the FP32 engine (default FP64, the reference's precision);
//    it projects every accepted configuration onto SU(NC) before saving it.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include <random>
#include <string>
#include <vector>

#include "../../include/askja_gpu.h"

namespace {

struct Files {
  FILE* constraints = nullptr;
  FILE* wilson = nullptr;
  ~Files() {
    if (constraints) fclose(constraints);
    if (wilson) fclose(wilson);
  }
};

int die(askja_ctx* ctx, const char* what) {
  fprintf(stderr, "ERROR: %s: %s\n", what, askja_last_error(ctx));
  printf("Finished with errors\n");
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  const char* paramsfile = nullptr;
  int precision = ASKJA_FP64;
  int device = 0;
  for (int i = 1; i < argc; i++) {
    if (!strcmp(argv[i], "--fp32"))
      precision = ASKJA_FP32;
    else if (!strcmp(argv[i], "--fp64"))
      precision = ASKJA_FP64;
    else if (!strcmp(argv[i], "--device") && i + 1 < argc)
      device = atoi(argv[++i]);
    else
      paramsfile = argv[i];
  }
  if (!paramsfile) {
    printf("ERROR please specify a params file name");
    printf("\nFinished with errors\n");
    return 1;
  }
  askja_run_params rp;
  const int prc = askja_params_load(paramsfile, &rp);
  if (prc == ASKJA_ERR_IO) {
    printf("\nERROR: params file %s could not be opened\n", paramsfile);
    printf("Finished with errors\n");
    return 1;
  }
  if (prc != ASKJA_OK) {
    printf("\nERROR: params file %s is malformed\n", paramsfile);
    printf("Finished with errors\n");
    return 1;
  }
  if (rp.update <= 0 || rp.update2 <= 0 || rp.conftake <= 0) {
    printf("\nERROR: UPDATE, UPDATE2 and CONFTAKE must be positive\n");
    printf("Finished with errors\n");
    return 1;
  }
  const int NC = rp.nc, DIM = rp.dim;
  const double BETA = rp.beta, dt = rp.dt;
  printf("DIM =%i\nBETA =%f\ndt =%f\nSTEPS =%i\nCONFTAKE =%i\n", DIM, BETA, dt, rp.steps, rp.conftake);
  if (rp.runcontinue)
    printf("===> Info: Continuing run at t=%f\nINFO: Taken=%i Nacc=%i Nac1=%i Nrec=%i Ntot=%i\n", rp.start * dt,
           rp.taken, rp.nacc, rp.nac1, rp.nrec, rp.ntot);
  printf("SU(%i) simulation in %i space dimensions\n", NC, DIM);

  askja_params p;
  memset(&p, 0, sizeof p);
  p.nc = NC;
  p.dim = DIM;
  for (int i = 0; i < DIM; i++) p.n[i] = rp.n[i];
  p.beta = BETA;
  p.dt = dt;
  p.level = rp.level;
  p.precision = precision;
  p.reunitarise = -1;
  p.device = device;
  uint64_t seed = rp.runcontinue ? (uint64_t)time(NULL) : (rp.random ? (uint64_t)time(NULL) : 120351616ull);
  p.seed = seed;
  askja_ctx* ctx = nullptr;
  if (askja_create(&p, &ctx) != ASKJA_OK) return die(nullptr, "engine");

  char outdir[255];
  snprintf(outdir, sizeof outdir, "output-DIM%i", DIM);
  struct stat st;
  if (stat(outdir, &st) != 0) {
    printf("===> Info: directory %s not present, creating it\n", outdir);
    mkdir(outdir, S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);
  }
  char stem[1024], path[1100];
  Files files;
  const char* mode = rp.runcontinue ? "a" : "w";
  askja_file_stem(&rp, outdir, "constraints", stem, sizeof stem);
  snprintf(path, sizeof path, "%s.dat", stem);
  files.constraints = fopen(path, mode);
  askja_file_stem(&rp, outdir, "Wilson", stem, sizeof stem);
  snprintf(path, sizeof path, "%s.dat", stem);
  files.wilson = fopen(path, mode);
  if (!files.constraints || !files.wilson) {
    askja_destroy(ctx);
    printf("\nERROR: cannot open output files in %s\nFinished with errors\n", outdir);
    return 1;
  }
  if (!rp.runcontinue) {
    fprintf(files.constraints, "#Time\t Gauss-law\t Total Energy\t E_L\t E_M\t Unitary-Violation\n");
    fprintf(files.wilson, "#Time\t <W>\t Wilson-Line-Phases\n");
  }

  const long V = askja_volume(ctx);
  const long ndoubles = V * DIM * NC * NC * 2;
  std::vector<double> conf;
  if (!rp.runcontinue) {
    if (askja_initializeU(ctx)) return die(ctx, "initializeU");
  } else {
    askja_file_stem(&rp, outdir, "U", stem, sizeof stem);
    snprintf(path, sizeof path, "%s-%i.conf", stem, rp.taken - 1);
    printf("===> Info: Attempting to load configuration %s\n", path);
    conf.resize(ndoubles);
    if (askja_conf_read(path, conf.data(), ndoubles) != ASKJA_OK) {
      printf("Error loading fields file %s ABORTED!\n", path);
      askja_destroy(ctx);
      printf("Finished with errors\n");
      return 1;
    }
    if (askja_set_links(ctx, conf.data())) return die(ctx, "set_links");
  }

  std::mt19937_64 uni_rng(seed ^ 0x5bd1e995ull);
  std::uniform_real_distribution<double> uni(0.0, 1.0);
  unsigned long long refresh_counter = 0;
  auto energy = [&](int which, double* h) -> int {
    double em = 0, k = 0;
    if (int rc = askja_EnergyMag(ctx, &em)) return rc;
    if (int rc = askja_simpleenergyEl(ctx, which, &k)) return rc;
    *h = (em + k / (2 * NC)) * BETA;
    return 0;
  };
  auto diagnostics = [&](double t, bool first) -> int {
    double em, ee, gauss, en, uv, w;
    if (askja_EnergyMag(ctx, &em) || askja_EnergyEl(ctx, &ee) || askja_GaussLaw(ctx, &gauss) ||
        askja_TotalEnergy(ctx, &en) || askja_UViol(ctx, &uv) || askja_WilsonLoop(ctx, &w))
      return -1;
    const double etot = first ? en / (2 * NC) * BETA : en * BETA / (2 * NC);
    if (rp.verbose)
      printf("t=%f Gauss Law =%g Energy=%g Wx=%g EL=%g EM=%g U-Viol=%g \n", t, gauss, etot, w, ee / (2 * NC) * BETA,
             em * BETA, uv);
    fprintf(files.constraints, "%f\t %g\t %g\t %g\t %f\t %g\n", t, gauss, etot, ee / (2 * NC) * BETA, em * BETA, uv);
    fflush(files.constraints);
    fprintf(files.wilson, "%f\t", t);
    fprintf(files.wilson, "%g\t", w);
    for (int i = 0; i < NC; i++) fprintf(files.wilson, "%g\t", 0.0);
    fprintf(files.wilson, "\n");
    fflush(files.wilson);
    return 0;
  };

  if (askja_initializeE(ctx, seed, refresh_counter++)) return die(ctx, "initializeE");
  double crit = 0;
  if (energy(0, &crit)) return die(ctx, "energy");
  printf("\t INFO: Initial energy =%f\n", crit);
  if (askja_updateE(ctx, dt / 2) || askja_copyDown(ctx)) return die(ctx, "first half step");
  if (!rp.runcontinue && diagnostics(0.0, true)) return die(ctx, "diagnostics");

  int taken = rp.taken;
  const int START = rp.start;
  const int last = rp.steps + START;
  int timekeep = START + 1;
  while (timekeep <= last) {
    // plain MD steps up to the next diagnostic or trajectory boundary
    int next = timekeep;
    while (next <= last && next % rp.update != 0 && next % rp.update2 != 0) next++;
    if (next > timekeep) {
      if (askja_md_steps(ctx, next - timekeep, dt)) return die(ctx, "md steps");
      timekeep = next;
      if (timekeep > last) break;
    }
    if (askja_updateUandcopyDown(ctx, dt)) return die(ctx, "updateUandcopyDown");
    if (timekeep % rp.update2 != 0)
      if (askja_updateE(ctx, dt)) return die(ctx, "updateE");
    if (timekeep % rp.update == 0)
      if (diagnostics(timekeep * dt, false)) return die(ctx, "diagnostics");
    if (timekeep % rp.update2 == 0) {
      if (askja_updateE(ctx, dt / 2)) return die(ctx, "updateE");
      double myenergy = 0;
      if (energy(1, &myenergy)) return die(ctx, "energy");
      printf("\t INFO: Final energy =%f\n", myenergy);
      rp.ntot++;
      bool accept = false;
      if (myenergy < crit) {
        printf("\t ACCEPT case 1: %f<%f\n", myenergy, crit);
        rp.nacc++;
        rp.nac1++;
        accept = true;
      } else {
        const double u = uni(uni_rng);
        if (u < exp(-myenergy + crit)) {
          printf("\t ACCEPT case 2: %f<%f\n", u, exp(-myenergy + crit));
          rp.nacc++;
          accept = true;
        } else {
          printf("\t REJECT %f>%f\n", u, exp(-myenergy + crit));
          rp.nrec++;
        }
      }
      // FP32: an accepted configuration is projected onto SU(NC) (in FP64 in the
      // residual-plane mode, whose link updates are not projected) before it is
      // saved, so every trajectory starts from projected links
      if (accept && precision == ASKJA_FP32 && askja_reunitarise(ctx)) return die(ctx, "reunitarise");
      if (accept ? askja_takeconfiguration(ctx) : askja_loadconfiguration(ctx)) return die(ctx, "configuration");
      if (askja_initializeE(ctx, seed, refresh_counter++)) return die(ctx, "initializeE");
      if (energy(0, &crit)) return die(ctx, "energy");
      printf("\t INFO: initial energy =%f\n", crit);
      if (askja_updateE(ctx, dt / 2)) return die(ctx, "updateE");
      if (rp.ntot % rp.conftake == 0) {
        askja_file_stem(&rp, outdir, "U", stem, sizeof stem);
        snprintf(path, sizeof path, "%s-%i.conf", stem, taken);
        printf("==>Info: storing configuration %s\n", path);
        conf.resize(ndoubles);
        if (askja_get_saved_links(ctx, conf.data())) return die(ctx, "get links");
        if (askja_conf_write(path, conf.data(), ndoubles) != ASKJA_OK) {
          printf("ERROR: could not write %s\n", path);
          askja_destroy(ctx);
          printf("Finished with errors\n");
          return 1;
        }
        taken++;
        askja_file_stem(&rp, outdir, "master", stem, sizeof stem);
        snprintf(path, sizeof path, "%s.params", stem);
        rp.taken = taken;
        if (askja_params_store(paramsfile, path, &rp, timekeep, taken) != ASKJA_OK) {
          printf("\nERROR: one of the params files %s,%s could not be opened\n", paramsfile, path);
          askja_destroy(ctx);
          printf("Finished with errors\n");
          return 1;
        }
      }
    }
    timekeep++;
  }
  askja_destroy(ctx);
  printf("===>Info: Statistics: acc=%i (%i) rec=%i, rate=%f\n", rp.nacc, rp.nac1, rp.nrec,
         rp.ntot ? (rp.nacc * 1.0) / rp.ntot : 0.0);
  printf("===>Took %i configurations\n", taken);
  printf("Finished successfully\n");
  return 0;
}
