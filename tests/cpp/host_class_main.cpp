// Drives fdm::FastMonodomainSolver (include/fdm_b200.hpp) the way the reference's RepeatedCall and preCICE
// drive its FastMonodomainSolver: settings in, setTimeSpan/advanceTimeSpan twice with a checkpoint between,
// the checkpoint replayed, the states and the transferred algebraics written out.
//   host_class_main <settings file> <output file> <intermediate time>
// With a fifth argument "settings" it only writes what FiberSettings::load read (no device needed).
// With a fifth argument it otherwise advances [startTime, endTime] once: "log" records the stimulation log and
// writes it to the output file in the reference's format; a number is the outputInterval of an output writer
// whose callback writes one line per call (numbered name, current time, Vm sum) to the output file, and
// callOutputWriter(0, 0) is called once more.
// Exit status: 0 done, 2 fdm::Error (message on stderr), 3 the replay after the checkpoint differs.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>

#include "fdm_b200.hpp"

int main(int argc, char** argv)
{
  if (argc != 4 && argc != 5) {
    std::fprintf(stderr, "usage: %s settings output t_mid [output_interval]\n", argv[0]);
    return 1;
  }
  try {
    fdm::FiberSettings s = fdm::FiberSettings::load(argv[1]);
    if (argc == 5 && std::string(argv[4]) == "settings") { // host only: what FiberSettings::load read
      std::FILE* f = std::fopen(argv[2], "w");
      if (!f)
        return 1;
      std::fprintf(f, "n_fibers %d\nn_nodes %lld\nequilibrium %d %.17g\nfiber_numbers", s.n_fibers(),
                   (long long)s.n_nodes(), (int)s.initialize_states_to_equilibrium, s.equilibrium_dt);
      for (int x : s.fiber_numbers)
        std::fprintf(f, " %d", x);
      std::fprintf(f, "\nstates_for_transfer");
      for (int x : s.states_for_transfer)
        std::fprintf(f, " %d", x);
      std::fprintf(f, "\nalgebraics_for_transfer");
      for (int x : s.algebraics_for_transfer)
        std::fprintf(f, " %d", x);
      std::fprintf(f, "\n");
      std::fclose(f);
      return 0;
    }
    if (argc == 5 && std::string(argv[4]) == "log") {
      fdm::FastMonodomainSolver slv(s);
      slv.enableStimulationLog();
      slv.advanceTimeSpan();
      slv.writeStimulationLog(argv[2]);
      return 0;
    }
    if (argc == 5) {
      fdm::FastMonodomainSolver slv(s);
      std::FILE* f = std::fopen(argv[2], "w");
      if (!f)
        return 1;
      fdm::OutputWriter w;
      w.outputInterval = std::atoi(argv[4]);
      w.filename = "out/fiber";
      w.write = [&](const std::string& name, double t) {
        double sum = 0.0;
        for (double v : slv.data().vm)
          sum += v;
        std::fprintf(f, "%s %.17g %.17g\n", name.c_str(), t, sum);
      };
      slv.addOutputWriter(w);
      slv.advanceTimeSpan();
      slv.callOutputWriter(0, 0.0);
      std::fclose(f);
      return 0;
    }
    const double t_mid = std::atof(argv[3]);
    fdm::FastMonodomainSolver slv(s);
    slv.initialize();
    slv.setTimeSpan(s.start_time, t_mid);
    slv.advanceTimeSpan();
    slv.saveFiberDataCheckpoint();
    slv.setTimeSpan(t_mid, s.end_time);
    slv.advanceTimeSpan();
    const std::vector<double> a = slv.states();
    slv.restoreFiberDataCheckpoint();
    slv.advanceTimeSpan();
    const std::vector<double> b = slv.states();
    if (a != b) {
      std::fprintf(stderr, "the replay after restoreFiberDataCheckpoint differs\n");
      return 3;
    }
    // page-locked host memory (fdm::PinnedAllocator over fdm_host_alloc) holds the states like any vector
    const std::vector<double, fdm::PinnedAllocator<double>> pinned(a.begin(), a.end());
    if (!std::equal(a.begin(), a.end(), pinned.begin())) {
      std::fprintf(stderr, "the page-locked copy of the states differs\n");
      return 3;
    }
    const fdm::TransferData d = slv.data();
    std::ofstream out(argv[2], std::ios::binary);
    out.write(reinterpret_cast<const char*>(a.data()), (std::streamsize)(a.size() * sizeof(double)));
    out.write(reinterpret_cast<const char*>(d.algebraics.data()), (std::streamsize)(d.algebraics.size() * sizeof(double)));
    std::printf("startTime %g endTime %g nodes %lld\n", slv.startTime(), slv.endTime(), (long long)s.n_nodes());
    return 0;
  } catch (const fdm::Error& e) {
    std::fprintf(stderr, "fdm::Error %d: %s\n", e.code(), e.what());
    return 2;
  }
}
