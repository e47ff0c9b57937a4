// A C++ caller of the library through include/pimc_b200.hpp, the way PIMC++
// code would use it.  Built and run by tests/test_cpp_host_cpu.py (no GPU:
// the header compiles, links, and a missing device is an exception) and by
// tests/test_gpu_cpp_host.py (on a GPU: actions and moves against the oracle).
//
//   host_cpp_check cpu
//   host_cpp_check gpu <dm> <tau> <box> <N> <S> <levels> <seed> <blocks> <path.bin> <out.bin>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "pimc_b200.hpp"

using namespace pimc_b200;

static std::vector<double> read_doubles(const char *file, size_t n) {
  std::vector<double> v(n);
  FILE *f = std::fopen(file, "rb");
  if (!f || std::fread(v.data(), sizeof(double), n, f) != n) {
    std::fprintf(stderr, "cannot read %s\n", file);
    std::exit(2);
  }
  std::fclose(f);
  return v;
}

int main(int argc, char **argv) {
  if (argc >= 2 && std::string(argv[1]) == "cpu") {
    try {
      PathData pd(4, 5, {9.0, 9.0, 9.0}, 0.01, 6.0596);
      std::printf("created\n");
    } catch (const Error &e) {
      std::printf("error %d\n", e.status());
    }
    return 0;
  }
  if (argc != 12) return 2;
  const char *dm = argv[2];
  const double tau = std::atof(argv[3]), L = std::atof(argv[4]);
  const int N = std::atoi(argv[5]), S = std::atoi(argv[6]), levels = std::atoi(argv[7]);
  const unsigned long long seed = std::strtoull(argv[8], nullptr, 10);
  const int blocks = std::atoi(argv[9]);
  std::vector<double> path = read_doubles(argv[10], (size_t)S * N * 3);
  std::vector<double> out;
  PathData pd(N, S, {L, L, L}, tau, 6.0596);
  pd.ReadDavidSquarerFile(dm);
  pd.SetPath(path);
  ShortRangeClass sr(pd);
  KineticClass kin(pd);
  struct Call {
    int s1, s2, level;
    std::vector<int> active;
  };
  const std::vector<Call> calls = {{0, 8, 0, {3}}, {4, 12, 1, {1, 5}}, {0, 16, 2, {0, 7, 9}}};
  for (const Call &c : calls) {
    out.push_back(sr.Action(c.s1, c.s2, c.active, c.level));
    out.push_back(kin.SingleAction(c.s1, c.s2, c.active, c.level));
  }
  out.push_back(sr.d_dBeta(0, S - 1, 0));
  BisectionBlockClass bb(pd, levels, 1);
  bb.Seed(seed);
  const std::vector<pimc_move_record> rec = bb.MakeMoves(blocks);
  for (const pimc_move_record &r : rec) {
    out.push_back(r.slice1);
    out.push_back(r.ptcl);
    out.push_back(r.accepted);
    out.push_back(r.stages_passed);
  }
  const std::vector<double> fin = pd.GetPath(OLDMODE);
  out.insert(out.end(), fin.begin(), fin.end());
  FILE *f = std::fopen(argv[11], "wb");
  if (!f || std::fwrite(out.data(), sizeof(double), out.size(), f) != out.size()) return 3;
  std::fclose(f);
  std::printf("ok %zu\n", out.size());
  return 0;
}
