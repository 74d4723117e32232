// rpba_main.cpp -- the `rpba` executable: main() of rpba.cpp:45-176 on top of
// the C ABI.  Reads the INI file "parameters" from the working directory
// (keys Robust, Exteval, Threads, k2, k4, f, k24out, InputDir, File; all
// required, as rpba.cpp:56-64 reads them), loads InputDir/File as BAL text,
// runs CalcPLSA on the GPU and prints the reference's console lines.
// Threads selects the branch as in the reference (rpbacore.cpp:79-92): the
// partitioned RPBA when min(Threads, iround(images / 70)) > 1 and there are
// more than five images, else the global LSA; Threads = 0 means the host's
// hardware threads.  Extra optional keys: Solver (pcg | direct | learned),
// Precision (fp64 | mixed), MaxIterations, Output (write the adjusted block
// as BAL text; the reference has this call commented out, rpba.cpp:144-150).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rpba_b200.h"

namespace {

std::string trim(const std::string &s) {
  const size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  const size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

// Minimal INI reader: key=value lines, ';'/'#' comments, [sections] ignored
// (the reference's file has no sections, parameters:1-14).
bool read_ini(const char *path, std::map<std::string, std::string> &kv) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line;
  while (std::getline(in, line)) {
    line = trim(line);
    if (line.empty() || line[0] == ';' || line[0] == '#' || line[0] == '[') continue;
    const size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    kv[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
  }
  return true;
}

// stringstream >> bool / int, as rpba.cpp:69-80 parses the values.
template <typename T>
T parse(const std::string &s) {
  std::stringstream ss(s);
  T v{};
  ss >> v;
  return v;
}

}  // namespace

int main(int argc, char **argv) {
  (void)argv;
  if (argc > 1) {
    std::printf("Parameter file not used\n");
    return 1;
  }
  std::map<std::string, std::string> kv;
  if (!read_ini("parameters", kv)) {
    std::fprintf(stderr, "cannot read file \"parameters\"\n");
    return 1;
  }
  for (const char *key : {"InputDir", "File", "Robust", "Exteval", "k2", "k4", "f", "k24out", "Threads"})
    if (!kv.count(key)) {
      std::fprintf(stderr, "parameters: missing key %s\n", key);
      return 1;
    }
  const bool extevalflag = parse<bool>(kv["Exteval"]);
  const bool robustflag = parse<bool>(kv["Robust"]);
  const bool k2f = parse<bool>(kv["k2"]), k4f = parse<bool>(kv["k4"]), flf = parse<bool>(kv["f"]);
  const bool k24outflag = parse<bool>(kv["k24out"]);
  int mt = parse<int>(kv["Threads"]);
  const std::string inputfile = kv["InputDir"] + "/" + kv["File"];
  std::printf("Inputfile: %s\n\n", inputfile.c_str());
  std::printf("Robustflag: %d\n\n", (int)robustflag);
  if (mt < 1) mt = (int)std::thread::hardware_concurrency();
  std::printf("Threads: %d\n\n", mt);
  std::printf("K2: %d\nK4: %d\nFocal length: %d\n\nK24out: %d\n\n", (int)k2f, (int)k4f, (int)flf, (int)k24outflag);
  const int nraddpar = (int)k2f + (int)k4f + (int)flf;

  rpba_block blk;
  int st = rpba_input_block(inputfile.c_str(), nraddpar, k24outflag, &blk);
  if (st != RPBA_OK) {
    std::fprintf(stderr, "cannot read %s: %s\n", inputfile.c_str(), rpba_status_string(st));
    return 1;
  }
  const int nobs = blk.pt_obs_off[blk.n_points];
  std::printf("Cameras: %d  Points: %d Observations %d\n", blk.n_images, blk.n_points, nobs);
  const long long nrunknowns = 3ll * blk.n_points + (blk.n_images - 2) * 6 + 5 + (long long)blk.n_images * nraddpar;
  std::printf("Unknowns %lld  Redundancy %lld\n", nrunknowns, 2ll * nobs - nrunknowns);

  rpba_options opt{};
  opt.robust = robustflag;
  opt.exteval = extevalflag;
  opt.threads = mt;
  opt.k2 = k2f;
  opt.k4 = k4f;
  opt.f = flf;
  opt.solver = RPBA_SOLVER_PCG;
  if (kv.count("Solver")) {
    const std::string s = kv["Solver"];
    opt.solver = s == "direct" ? RPBA_SOLVER_DIRECT : (s == "learned" ? RPBA_SOLVER_LEARNED : RPBA_SOLVER_PCG);
  }
  opt.precision = kv.count("Precision") && kv["Precision"] == "mixed" ? RPBA_PREC_MIXED : RPBA_PREC_FP64;
  opt.max_lm_iterations = kv.count("MaxIterations") ? parse<int>(kv["MaxIterations"]) : -1;

  std::vector<char> log(1 << 20);
  rpba_report rep{};
  const auto t0 = std::chrono::steady_clock::now();
  // the branch (global or partitioned) follows the reference's rule inside
  // rpba_calc_plsa; the partitioned branch's lines are console output
  const bool partitioned = rpba_partition_count(blk.n_images, mt, extevalflag) > 1 &&
                           opt.precision == RPBA_PREC_FP64 && opt.solver != RPBA_SOLVER_LEARNED;
  st = rpba_calc_plsa(&blk, &opt, log.data(), log.size(), &rep);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  // the partitioned branch's progress lines are console output in the reference
  if (partitioned || blk.n_images < 50 || mt == 1 || extevalflag) std::printf("%s", log.data());
  if (st != RPBA_OK && st != RPBA_ERR_NO_OBS_IMAGE && st != RPBA_ERR_LOW_REDUNDANCY && st != RPBA_ERR_NAN_STEP)
    std::fprintf(stderr, "rpba: %s\n", rpba_status_string(st));
  std::printf("\n\nBundle adjustment runtime: %gs\n\n", (float)secs);
  if (kv.count("Output") && !extevalflag) {
    const std::string outfile = kv["InputDir"] + "/" + kv["Output"];
    rpba_output_block(outfile.c_str(), &blk, k24outflag);
  }
  rpba_block_free(&blk);
  return st == RPBA_OK ? 0 : 2;
}
