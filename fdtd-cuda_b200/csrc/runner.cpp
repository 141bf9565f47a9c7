// fdtd_runner -- the reference's program (main.cu main()) as a C++ host
// over the C ABI: read Input.txt (READ_DATA_FILE, setup.cu:10-133), set up
// and run t = 0 .. Tend (main.cu:2724-3175), and write what the reference
// writes:
//   OUT.txt              the centre probe (main.cu:2722-2732: t*dt, ex, ey,
//                        ez at the top of every step)
//   ScatAbs.<t>.txt      the spectra (CalculateAbsScatt, Spectral.cu) after
//                        every step t with t % (Tend/10) == 0
//                        (main.cu:3042-3172; at Tend only when Tend < 10)
//   Reflectivity{TE,TM}.<trial>.<t>.txt
//                        periodic_xy runs instead of ScatAbs: after every
//                        step t > 0 with t % (Tend/10) == 0 (main.cu:2994-
//                        3037), per frequency but the first: lambda (or
//                        the frequency), R, the reference's transmitted
//                        flux ratio (negative for a wave leaving through
//                        +z), |E_inc|^2, and the two fluxes over the area
//                        unnormalised (fdtd_reflectance)
//   aux_sim.<n>.txt, aux_sim.<n>_2.txt, videofiles/YZ_sim.<n>.txt,
//   videofiles/YZ_sim.<n>_N.txt
//                        the snapshots of Snap_in 1, 2, 3 every t_skip
//                        steps (main.cu:2948-2991, snapshot.cu), taken on
//                        the device and drained while the run goes on; n
//                        counts every file group written, as the
//                        reference's snapshot_count does
//
//   fdtd_runner [Input.txt] [--out DIR] [--fp32 | --fp64] [--device N]
//               [--periodic-xy]
//
// --periodic-xy switches on the reference's Periodic_XY path, which its
// Input.txt cannot select (main.cu:2398 forces it off); the deck must then
// set NcpmlX = NcpmlY = 0.
//
// Exit status: 0 on success, 1 on a library error (its text on stderr), 2
// on bad arguments, 3 when the watchdog saw a non-finite field ("NAN
// Detected" ends OUT.txt, as in the reference).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <string>
#include <vector>

#include "../../include/fdtd_b200.h"

namespace {

void usage() {
  std::fprintf(stderr,
               "usage: fdtd_runner [Input.txt] [--out DIR] [--fp32 | --fp64] [--device N] [--periodic-xy]\n"
               "  runs the reference's time loop on the GPU and writes OUT.txt, ScatAbs.<t>.txt\n"
               "  every Tend/10 steps and the Snap_in snapshots into DIR (default: the current\n"
               "  directory); --periodic-xy: periodic x and y, Reflectivity{TE,TM}.<trial>.<t>.txt\n"
               "  instead of ScatAbs\n");
}

int fail(const char* what) {
  std::fprintf(stderr, "fdtd_runner: %s: %s\n", what, fdtd_last_error());
  return 1;
}

// A one-value-per-line column (SNAPSHOT_1D).
bool write_column(const std::string& path, const double* v, int n) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  for (int i = 0; i < n; i++) std::fprintf(f, "%e\n", v[i]);
  std::fclose(f);
  return true;
}

// A plane, one row per line, values separated by a space (SNAPSHOT_2D).
bool write_plane(const std::string& path, const double* v, int rows, int cols) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  for (int r = 0; r < rows; r++) {
    for (int c = 0; c < cols; c++) std::fprintf(f, "%e ", v[(size_t)r * cols + c]);
    std::fprintf(f, "\n");
  }
  std::fclose(f);
  return true;
}

// The files of one snapshot record, named with the reference's counter.
bool write_snapshot(const std::string& out, const fdtd_snapshot_layout& L, const double* r, int& count) {
  const std::string vf = out + "/videofiles/YZ_sim.";
  auto aux = [&]() {
    const std::string b = out + "/aux_sim." + std::to_string(count);
    const bool ok = write_column(b + ".txt", r + L.off_aux, L.aux_len) &&
                    write_column(b + "_2.txt", r + L.off_line, L.line_len);
    count++;
    return ok;
  };
  auto plane = [&](int off, const char* suffix) {
    const bool ok = write_plane(vf + std::to_string(count) + suffix + ".txt", r + off, L.plane_rows, L.plane_cols);
    count++;
    return ok;
  };
  if (L.mode == 1) return aux();
  if (L.mode == 2) return plane(L.off_plane, "") && plane(L.off_plane2, "_N");
  return aux() && plane(L.off_plane, "");
}

// The periodic run's reflectivity file (main.cu:3026-3035): the columns
// the reference prints from its E_reflected / E_transmitted (P / A) and the
// incident amplitude |E_inc|^2.
bool write_reflectivity(fdtd_sim* sim, const fdtd_params& p, const std::string& path) {
  const int nf = p.NUM_freq;
  std::vector<double> rt((size_t)7 * nf), freq(nf);
  if (fdtd_reflectance(sim, rt.data()) != FDTD_OK || fdtd_get_freqs(sim, freq.data(), nf) != FDTD_OK) return false;
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  for (int m = 1; m < nf; m++) {
    const double* r = &rt[(size_t)7 * m];
    const double amp = r[4] * r[4];
    const double refl = r[1] * amp, trans = -r[2] * amp;  // P_refl / A, P_trans / A
    std::fprintf(f, "%e\t%e\t%e\t%e\t%e\t%e\n", p.WL_or_freq == 1 ? r[0] : freq[m], r[1], -r[2], amp, refl, trans);
  }
  std::fclose(f);
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  std::string input = "Input.txt", out = ".";
  int precision = -1, device = 0, periodic = 0;
  for (int a = 1; a < argc; a++) {
    const char* s = argv[a];
    if (!std::strcmp(s, "--help") || !std::strcmp(s, "-h")) {
      usage();
      return 0;
    } else if (!std::strcmp(s, "--out") && a + 1 < argc) {
      out = argv[++a];
    } else if (!std::strcmp(s, "--device") && a + 1 < argc) {
      device = std::atoi(argv[++a]);
    } else if (!std::strcmp(s, "--periodic-xy")) {
      periodic = 1;
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
  if (periodic) p.periodic_xy = 1;
  fdtd_sim* sim = nullptr;
  if (fdtd_create(&p, device, &sim) != FDTD_OK) return fail("setting up");
  // snapshots: taken on the device, drained after every chunk of steps
  fdtd_snapshot_layout lay{};
  const bool snaps = p.Snap_in >= 1 && p.Snap_in <= 3;
  const int cap = 130;  // a 128-step block of t_skip = 1 records between drains
  std::vector<double> recs;
  int snap_count = 0;
  if (snaps) {
    if (fdtd_snapshots_enable(sim, p.Snap_in, cap, &lay) != FDTD_OK) {
      fdtd_destroy(sim);
      return fail("enabling snapshots");
    }
    std::error_code ec;
    std::filesystem::create_directories(out + "/videofiles", ec);
    recs.resize((size_t)cap * lay.record);
  }
  // the time loop in chunks that end at every spectra dump and before the
  // snapshot ring fills
  const int total = p.Tend + 1;
  const int period = p.Tend / 10;
  std::vector<int> dumps;
  for (int t = 0; t <= p.Tend; t++) {
    if (p.periodic_xy) {
      if (t > 0 && period > 0 && t % period == 0) dumps.push_back(t);
    } else if (period > 0 ? t % period == 0 : t == p.Tend) {
      dumps.push_back(t);
    }
  }
  std::vector<std::string> written;
  int done = 0;
  size_t next_dump = 0;
  while (done < total) {
    int stop = total;
    if (next_dump < dumps.size()) stop = std::min(stop, dumps[next_dump] + 1);
    if (snaps) stop = std::min(stop, done + (cap - 1) * lay.t_skip);
    if (fdtd_step(sim, stop - done, nullptr) != FDTD_OK) {
      fdtd_destroy(sim);
      return fail("running");
    }
    done = stop;
    if (snaps) {
      int n = 0;
      if (fdtd_snapshots_drain(sim, recs.data(), cap, &n, nullptr) != FDTD_OK || fdtd_check(sim) == FDTD_ERR_CUDA) {
        fdtd_destroy(sim);
        return fail("draining snapshots");
      }
      for (int q = 0; q < n; q++)
        if (!write_snapshot(out, lay, recs.data() + (size_t)q * lay.record, snap_count)) {
          std::fprintf(stderr, "fdtd_runner: cannot write snapshot files under %s\n", out.c_str());
          fdtd_destroy(sim);
          return 1;
        }
    }
    if (next_dump < dumps.size() && done == dumps[next_dump] + 1) {
      const std::string t = std::to_string(dumps[next_dump]);
      std::string sca;
      bool ok;
      if (p.periodic_xy) {
        sca = out + "/Reflectivity" + (p.TE_TM == 1 ? "TM." : "TE.") + std::to_string(p.min_trials) + "." + t + ".txt";
        ok = write_reflectivity(sim, p, sca);
      } else {
        sca = out + "/ScatAbs." + t + ".txt";
        ok = fdtd_write_scatabs(sim, sca.c_str()) == FDTD_OK;
      }
      if (!ok) {
        fdtd_destroy(sim);
        return fail("writing the spectra");
      }
      written.push_back(sca);
      next_dump++;
    }
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
  std::printf("fdtd_runner: %d x %d x %d cells, %d steps, %s; wrote %s, %zu spectra (last %s), %d snapshot files\n",
              d.nx, d.ny, d.nz, p.Tend + 1, p.precision == FDTD_FP64 ? "FP64" : "FP32", out_path.c_str(),
              written.size(), written.empty() ? "-" : written.back().c_str(), snap_count);
  fdtd_destroy(sim);
  return 0;
}
