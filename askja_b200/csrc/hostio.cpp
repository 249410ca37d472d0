// Host-side file formats of the askja drop-in (no GPU needed):
//   params file   positional "key value" tokens        (sun.cpp:803-938)
//   master params store_parameters rewrite + trailer   (sun.cpp:940-1057)
//   file stems    "...-N%i-Nt%i-Ns%i-BETA%.2f-DT%.4f-U%.4f-CT%i"  (sun.cpp:1124-1326)
//   U-conf        V*DIM*NC*NC complex doubles, [site][dir][row][col][re,im]
//                 native byte order, no header       (sun.cpp:289-302, 744-765)
// The reference's measure1d/2d/4d read these files unchanged.
#include <stdio.h>
#include <string.h>

#include <fstream>
#include <sstream>
#include <string>

#include "../../include/askja_gpu.h"

namespace {

bool read_int(std::istream& in, int& v) {
  std::string key;
  if (!(in >> key)) return false;
  return (bool)(in >> v);
}

bool read_double(std::istream& in, double& v) {
  std::string key;
  if (!(in >> key)) return false;
  return (bool)(in >> v);
}

}  // namespace

extern "C" {

int askja_params_load(const char* path, askja_run_params* p) {
  if (!path || !p) return ASKJA_ERR_ARG;
  std::ifstream in(path);
  if (!in.is_open()) return ASKJA_ERR_IO;
  memset(p, 0, sizeof *p);
  std::string header;
  if (!(in >> header)) return ASKJA_ERR_PARSE;
  if (!read_int(in, p->nc) || !read_int(in, p->dim)) return ASKJA_ERR_PARSE;
  if (p->dim < 1 || p->dim > ASKJA_MAX_DIM) return ASKJA_ERR_PARSE;
  for (int i = 0; i < p->dim; i++)
    if (!read_int(in, p->n[i])) return ASKJA_ERR_PARSE;
  if (!read_double(in, p->beta) || !read_double(in, p->dt)) return ASKJA_ERR_PARSE;
  if (!read_int(in, p->steps) || !read_int(in, p->update) || !read_int(in, p->update2) ||
      !read_int(in, p->conftake) || !read_int(in, p->level) || !read_int(in, p->verbose) ||
      !read_int(in, p->runcontinue) || !read_int(in, p->random))
    return ASKJA_ERR_PARSE;
  if (p->runcontinue) {
    if (!read_int(in, p->start) || !read_int(in, p->taken) || !read_int(in, p->nacc) || !read_int(in, p->nac1) ||
        !read_int(in, p->nrec) || !read_int(in, p->ntot))
      return ASKJA_ERR_PARSE;
    // correct for non-stored parts (sun.cpp:903-904)
    if (p->conftake > 0) p->nacc = (p->nacc / p->conftake) * p->conftake;
  } else {
    p->start = 1;
  }
  return ASKJA_OK;
}

int askja_params_store(const char* infile, const char* outfile, const askja_run_params* p, int timestep, int taken) {
  if (!infile || !outfile || !p) return ASKJA_ERR_ARG;
  // The input is read completely before the output is opened: on resume the
  // master params file is both (the reference copies it to <infile>-tmp first,
  // sun.cpp:945-949).
  std::stringstream in;
  {
    std::ifstream fin(infile);
    if (!fin.is_open()) return ASKJA_ERR_IO;
    in << fin.rdbuf();
  }
  {
    std::ofstream out(outfile, std::ios::out);
    if (!out.is_open()) return ASKJA_ERR_IO;
    std::string key;
    int iv;
    double dv;
    auto key_out = [&](const char* sep) -> bool {
      if (!(in >> key)) return false;
      out << key << sep;
      return true;
    };
    if (!(in >> key)) return ASKJA_ERR_PARSE;
    out << key << "\n";
    if (!key_out("\t\t") || !(in >> iv)) return ASKJA_ERR_PARSE;
    out << iv << "\n";  // NC as read
    if (!key_out("\t\t") || !(in >> iv)) return ASKJA_ERR_PARSE;
    out << iv << "\n";  // DIM as read
    for (int i = 0; i < p->dim; i++) {
      if (!key_out("\t\t") || !(in >> iv)) return ASKJA_ERR_PARSE;
      out << iv << "\n";
    }
    if (!key_out("\t\t") || !(in >> dv)) return ASKJA_ERR_PARSE;
    out << dv << "\n";  // BETA as read
    if (!key_out("\t\t") || !(in >> dv)) return ASKJA_ERR_PARSE;
    out << dv << "\n";  // DT as read
    if (!key_out("\t\t") || !(in >> iv)) return ASKJA_ERR_PARSE;
    out << p->steps << "\n";
    if (!key_out("\t\t") || !(in >> iv)) return ASKJA_ERR_PARSE;
    out << p->update << "\n";
    if (!key_out("\t\t") || !(in >> iv)) return ASKJA_ERR_PARSE;
    out << p->update2 << "\n";
    if (!key_out("\t\t") || !(in >> iv)) return ASKJA_ERR_PARSE;
    out << p->conftake << "\n";
    if (!key_out("\t") || !(in >> iv)) return ASKJA_ERR_PARSE;
    out << p->level << "\n";
    if (!key_out("\t\t") || !(in >> iv)) return ASKJA_ERR_PARSE;
    out << p->verbose << "\n";
    if (!key_out("\t") || !(in >> iv)) return ASKJA_ERR_PARSE;
    out << 1 << "\n";  // RUNCONTINUE
    if (!key_out("\t\t") || !(in >> iv)) return ASKJA_ERR_PARSE;
    out << p->random << "\n";
    out << "TIME-STEP\t" << timestep << "\n";
    out << "TAKEN\t\t" << taken << "\n";
    out << "NACC\t\t" << p->nacc << "\n";
    out << "NAC1\t\t" << p->nac1 << "\n";
    out << "NREC\t\t" << p->nrec << "\n";
    out << "NTOT\t\t" << p->ntot << "\n";
    if (!out.good()) return ASKJA_ERR_IO;
  }
  return ASKJA_OK;
}

int askja_file_stem(const askja_run_params* p, const char* dir, const char* kind, char* out, size_t cap) {
  if (!p || !dir || !kind || !out || cap == 0) return ASKJA_ERR_ARG;
  const int ns = p->dim > 1 ? p->n[1] : 1;
  const int n = snprintf(out, cap, "%s/%s-N%i-Nt%i-Ns%i-BETA%.2f-DT%.4f-U%.4f-CT%i", dir, kind, p->nc, p->n[0], ns,
                         p->beta, p->dt, p->update2 * p->dt, p->conftake);
  if (n < 0 || (size_t)n >= cap) return ASKJA_ERR_ARG;
  return ASKJA_OK;
}

int askja_conf_write(const char* path, const double* conf, long n_doubles) {
  if (!path || !conf || n_doubles <= 0) return ASKJA_ERR_ARG;
  FILE* f = fopen(path, "w");
  if (!f) return ASKJA_ERR_IO;
  const size_t w = fwrite(conf, sizeof(double), (size_t)n_doubles, f);
  const int rc = fclose(f);
  return (w == (size_t)n_doubles && rc == 0) ? ASKJA_OK : ASKJA_ERR_IO;
}

int askja_conf_read(const char* path, double* conf, long n_doubles) {
  if (!path || !conf || n_doubles <= 0) return ASKJA_ERR_ARG;
  FILE* f = fopen(path, "r");
  if (!f) return ASKJA_ERR_IO;
  const size_t r = fread(conf, sizeof(double), (size_t)n_doubles, f);
  fclose(f);
  return r == (size_t)n_doubles ? ASKJA_OK : ASKJA_ERR_IO;
}

}  // extern "C"
