// main.cpp -- MAIN: the reference's command line (maincode.cpp:56-770) on the
// B200 library.
//
//   MAIN onrate offrate V.dat E.dat T.dat Nknobs RBCdata.dat stl_flag
//
// Same arguments (maincode.cpp:73-74,174,230,259,394,456-457), the same
// set-up printout, knobs.dat in the working directory, a record of vertex
// x y z ix iy bondi in RBCdata.dat every out_every steps (first after step
// index out_every) and rbc<k>.stl beside it when stl_flag is 1.  The box and
// the other define.h parameters are irbc_params_default(); the vertex count
// is the vertex file's line count.  Not in the reference: IRBC_STEPS (total
// steps, default the reference's 4,000,000), IRBC_OUT_EVERY (default 5000),
// IRBC_SEED, IRBC_NS (solvent particles, default define.h's Ns: the
// reference's value is fixed at compile time), IRBC_PRECISION (fp64 /
// fp32) and IRBC_DEVICE in the environment.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "irbc.h"

namespace {

int64_t env_i64(const char* name, int64_t dflt) {
  const char* v = std::getenv(name);
  return v && *v ? std::strtoll(v, nullptr, 10) : dflt;
}

// whitespace-separated numbers, `per` to a line, until end of file
template <typename T>
bool read_table(const char* path, int per, std::vector<T>& out) {
  FILE* f = std::fopen(path, "r");
  if (!f) return false;
  out.clear();
  double v;
  while (std::fscanf(f, "%lf", &v) == 1) out.push_back((T)v);
  std::fclose(f);
  return !out.empty() && out.size() % per == 0;
}

int die(irbc_handle* h, const char* what) {
  std::fprintf(stderr, "MAIN: %s%s%s\n", what, h ? ": " : "", h ? irbc_last_error(h) : "");
  if (h) irbc_destroy(h);
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 9) {
    std::fprintf(stderr, "usage: %s onrate offrate V.dat E.dat T.dat Nknobs RBCdata.dat stl_flag\n", argv[0]);
    return 2;
  }
  std::vector<double> V;
  std::vector<int32_t> E, T;
  if (!read_table(argv[3], 3, V)) return die(nullptr, "cannot read the vertex file");
  if (!read_table(argv[4], 2, E)) return die(nullptr, "cannot read the edge file");
  if (!read_table(argv[5], 3, T)) return die(nullptr, "cannot read the triangle file");
  for (auto& e : E) e -= 1;  // the files are 1-based
  for (auto& t : T) t -= 1;
  const int32_t nv = (int32_t)(V.size() / 3), ne = (int32_t)(E.size() / 2), nt = (int32_t)(T.size() / 3);

  irbc_params p;
  irbc_params_default(&p);
  p.onrate = std::atof(argv[1]);
  p.offrate = std::atof(argv[2]);
  p.Nt = nv;
  p.seed = (uint64_t)env_i64("IRBC_SEED", (int64_t)p.seed);
  p.out_every = env_i64("IRBC_OUT_EVERY", p.out_every);
  p.Ns = env_i64("IRBC_NS", p.Ns);
  p.device = (int32_t)env_i64("IRBC_DEVICE", 0);
  const char* prec = std::getenv("IRBC_PRECISION");
  if (prec && std::strcmp(prec, "fp32") == 0) p.precision = IRBC_FP32;
  const int64_t total = env_i64("IRBC_STEPS", 4000000);
  const int32_t nknobs = std::atoi(argv[6]);
  const char* rbcdata = argv[7];
  const int stl = std::atoi(argv[8]);

  irbc_handle* h = nullptr;
  if (irbc_create(&p, &h)) return die(h, "cannot create the simulation");
  if (irbc_init(h, V.data(), nv, E.data(), ne, T.data(), nt, nknobs)) return die(h, "set-up failed");
  double rep[9];
  irbc_init_report(h, rep);
  std::printf("Mean edge is:\t%g\nStandard deviation is:\t%g\n", rep[0], rep[1]);
  std::printf("Sarea:\t%g\nVolume:\t%g\n", rep[2], rep[3]);
  std::printf("Shear modulus::\t%g\nYoung's modulus::\t%g\nPoisson's ratio::\t%g\n", rep[4], rep[5], rep[6]);

  // knobs.dat: the knob vertices' positions after placement (maincode.cpp:435-445)
  {
    std::vector<double> x(nv), y(nv), z(nv);
    std::vector<int32_t> knob(nv);
    irbc_view v;
    std::memset(&v, 0, sizeof(v));
    v.x = x.data(); v.y = y.data(); v.z = z.data(); v.knob = knob.data();
    if (irbc_get_state(h, &v)) return die(h, "cannot read the vertices");
    FILE* f = std::fopen("knobs.dat", "w");
    if (!f) return die(h, "cannot write knobs.dat");
    int cnt = 0;
    for (int i = 0; i < nv; ++i)
      if (knob[i] == 1) { std::fprintf(f, "%lf\t%lf\t%lf\n", x[i], y[i], z[i]); ++cnt; }
    std::fclose(f);
    std::printf("no of vertices selected:\t%d\n", cnt);
    std::fflush(stdout);
  }
  // RBCdata.dat is opened for writing at the start (maincode.cpp:456)
  {
    FILE* f = std::fopen(rbcdata, "w");
    if (!f) return die(h, "cannot write the RBCdata file");
    std::fclose(f);
  }
  // a record after the step that brings filecc to out_every (maincode.cpp:746)
  int64_t done = 0, next = p.out_every + 1;
  int filec = 0;
  while (done < total) {
    const int64_t n = std::min(next, total) - done;
    if (irbc_step(h, n)) return die(h, "step failed");
    done += n;
    if (done == next) {
      if (irbc_write_rbcdata(h, rbcdata, 1)) return die(h, "cannot append to the RBCdata file");
      ++filec;
      if (stl == 1) {
        char name[64];
        std::snprintf(name, sizeof(name), "rbc%d.stl", filec);
        if (irbc_write_stl(h, name)) return die(h, "cannot write the STL file");
      }
      next += p.out_every;
    }
  }
  irbc_destroy(h);
  return 0;
}
