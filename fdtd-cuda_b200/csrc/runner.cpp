// fdtd_runner -- the reference's program (main.cu main()) as a C++ host
// over the C ABI: read Input.txt (READ_DATA_FILE, setup.cu:10-133), set up
// and run t = 0 .. Tend (main.cu:2724-3175), write the centre-probe record
// OUT.txt (main.cu:2722-2732: t*dt, ex, ey, ez at the top of every step)
// and the spectra ScatAbs.<Tend>.txt (CalculateAbsScatt, Spectral.cu).
//
//   fdtd_runner [Input.txt] [--out DIR] [--fp32 | --fp64] [--device N]
//
// Exit status: 0 on success, 1 on a library error (its text on stderr), 2
// on bad arguments, 3 when the watchdog saw a non-finite field ("NAN
// Detected" ends OUT.txt, as in the reference).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fdtd_b200.h"

namespace {

void usage() {
  std::fprintf(stderr,
               "usage: fdtd_runner [Input.txt] [--out DIR] [--fp32 | --fp64] [--device N]\n"
               "  runs the reference's time loop on the GPU and writes OUT.txt and\n"
               "  ScatAbs.<Tend>.txt into DIR (default: the current directory)\n");
}

int fail(const char* what) {
  std::fprintf(stderr, "fdtd_runner: %s: %s\n", what, fdtd_last_error());
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  std::string input = "Input.txt", out = ".";
  int precision = -1, device = 0;
  for (int a = 1; a < argc; a++) {
    const char* s = argv[a];
    if (!std::strcmp(s, "--help") || !std::strcmp(s, "-h")) {
      usage();
      return 0;
    } else if (!std::strcmp(s, "--out") && a + 1 < argc) {
      out = argv[++a];
    } else if (!std::strcmp(s, "--device") && a + 1 < argc) {
      device = std::atoi(argv[++a]);
    } else if (!std::strcmp(s, "--fp32")) {
      precision = FDTD_FP32;
    } else if (!std::strcmp(s, "--fp64")) {
      precision = FDTD_FP64;
    } else if (s[0] == '-') {
      usage();
      return 2;
    } else {
      input = s;
    }
  }
  fdtd_params p;
  fdtd_params_default(&p);
  if (fdtd_load_input_txt(input.c_str(), &p) != FDTD_OK) return fail("reading the input");
  if (precision >= 0) p.precision = precision;
  fdtd_sim* sim = nullptr;
  if (fdtd_create(&p, device, &sim) != FDTD_OK) return fail("setting up");
  if (fdtd_run(sim, nullptr) != FDTD_OK) {
    fdtd_destroy(sim);
    return fail("running");
  }
  const fdtd_status chk = fdtd_check(sim);
  fdtd_dims d;
  if (fdtd_get_dims(sim, &d) != FDTD_OK) {
    fdtd_destroy(sim);
    return fail("reading the sizes");
  }
  // OUT.txt: row t holds E at the top of step t, i.e. the probe after step
  // t-1 (zero fields at t = 0)
  int n = 0;
  std::vector<double> probe((size_t)3 * (p.Tend + 1));
  if (fdtd_get_probe(sim, probe.data(), probe.size(), &n) != FDTD_OK) {
    fdtd_destroy(sim);
    return fail("reading the probe");
  }
  const std::string out_path = out + "/OUT.txt";
  FILE* f = std::fopen(out_path.c_str(), "w");
  if (!f) {
    std::fprintf(stderr, "fdtd_runner: cannot write %s\n", out_path.c_str());
    fdtd_destroy(sim);
    return 1;
  }
  for (int t = 0; t <= p.Tend; t++) {
    const double* e = t >= 1 && t - 1 < n ? &probe[(size_t)3 * (t - 1)] : nullptr;
    std::fprintf(f, "%e\t%e\t%e\t%e\n", t * d.dt, e ? e[0] : 0.0, e ? e[1] : 0.0, e ? e[2] : 0.0);
  }
  if (chk == FDTD_ERR_NONFINITE) std::fprintf(f, "NAN Detected\n");
  std::fclose(f);
  if (chk == FDTD_ERR_NONFINITE) {
    std::fprintf(stderr, "fdtd_runner: non-finite field values\n");
    fdtd_destroy(sim);
    return 3;
  }
  const std::string sca = out + "/ScatAbs." + std::to_string(p.Tend) + ".txt";
  if (fdtd_write_scatabs(sim, sca.c_str()) != FDTD_OK) {
    fdtd_destroy(sim);
    return fail("writing the spectra");
  }
  std::printf("fdtd_runner: %d x %d x %d cells, %d steps, %s; wrote %s and %s\n", d.nx, d.ny, d.nz, p.Tend + 1,
              p.precision == FDTD_FP64 ? "FP64" : "FP32", out_path.c_str(), sca.c_str());
  fdtd_destroy(sim);
  return 0;
}
