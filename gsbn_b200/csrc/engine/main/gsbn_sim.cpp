/* gsbn_sim: the command line of gsbn (src/gsbn_sim/Main.cpp:1-88) over this
 * library's engine.
 *
 *   gsbn_sim -n net.prototxt [-s snapshot.bin] [-m GPU|CPU] [-l] [-t]
 *
 * -n network description (required), -s restore a SolverState snapshot,
 * -m mode (default GPU here: this build has no CPU path for ProcUpdLazy),
 * -l log procedure set-up and progress to stderr, -t tick-by-tick loop
 * instead of one device run per stimulus segment.  The solver prints
 * "Total time for [<simulated seconds>]: <wall seconds>" like gsbn.
 */
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <string>

#include "gsbn_engine.h"

int main(int argc, char* argv[]) {
  const char* n_path = nullptr;
  const char* s_path = nullptr;
  const char* m_mode = nullptr;
  bool log = false, ticks = false;
  int c;
  while ((c = getopt(argc, argv, "n:s:m:lt")) != -1) {
    switch (c) {
      case 'n': n_path = optarg; break;
      case 's': s_path = optarg; break;
      case 'm': m_mode = optarg; break;
      case 'l': log = true; break;
      case 't': ticks = true; break;
      default:
        std::cerr << "Arguments wrong, abort!\n"
                  << "usage: gsbn_sim -n net.prototxt [-s snapshot.bin] [-m GPU|CPU] [-l] [-t]\n";
        return 2;
    }
  }
  for (int i = optind; i < argc; i++) std::cerr << "WARNING: Non-option argument " << argv[i] << "\n";
  if (!n_path) {
    std::cerr << "Incompleted arguments!\n";
    return 2;
  }
  int mode = GSBN_MODE_GPU;
  if (m_mode) {
    if (!std::strcmp(m_mode, "CPU") || !std::strcmp(m_mode, "cpu"))
      mode = GSBN_MODE_CPU;
    else if (!std::strcmp(m_mode, "GPU") || !std::strcmp(m_mode, "gpu"))
      mode = GSBN_MODE_GPU;
    else {
      std::cerr << "Wrong mode!\n";
      return 2;
    }
  }
  gsbn_solver* s = nullptr;
  if (gsbn_solver_create(n_path, s_path, mode, &s) != 0) {
    std::cerr << "gsbn_sim: " << gsbn_engine_last_error() << "\n";
    return 1;
  }
  if (log) {
    char names[1024];
    if (gsbn_procedure_names(names, sizeof names) == 0) std::cerr << "registered procedures: " << names << "\n";
  }
  auto t0 = std::chrono::steady_clock::now();
  int st = gsbn_solver_run(s, ticks ? 0 : 1);
  auto t1 = std::chrono::steady_clock::now();
  if (st != 0) {
    std::cerr << "gsbn_sim: " << gsbn_engine_last_error() << "\n";
    gsbn_solver_destroy(s);
    return 1;
  }
  int64_t n_ticks = 0, n_windows = 0;
  gsbn_solver_stats(s, &n_ticks, &n_windows, nullptr, nullptr);
  if (log) std::cerr << "Simulation [ END ] " << n_ticks << " ticks in " << n_windows << " windows\n";
  if (log) std::cerr << "wall time " << std::chrono::duration<double>(t1 - t0).count() << " s\n";
  gsbn_solver_destroy(s);
  return 0;
}
