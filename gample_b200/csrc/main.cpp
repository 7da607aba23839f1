// main.cpp -- command-line driver: gample_pic -i cond.json [-o tag]
//
// Restates src/main.mm:28-262: parse the condition, build the run objects,
// initial deposit + solve, then cycles Start+1..End with the XML log and the
// timeseries CSV "<Project>_<tag>_{log.xml,timeseries.csv}".
#include <chrono>
#include <ctime>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>

#include "simulation.hpp"

int main(int argc, char** argv) {
  std::map<std::string, std::string> args;  // src/main.mm:15-26
  for (int i = 1; i < argc - 1; ++i) {
    std::string k = argv[i];
    if (!k.empty() && k[0] == '-') {
      args[k] = argv[i + 1];
      ++i;
    }
  }
  if (!args.count("-i")) {
    std::cerr << "Usage: " << argv[0] << " -i inputfile.json [-o tag] [--reference-order 1]\n";
    return 1;
  }
  std::string tag;
  if (args.count("-o")) {
    tag = args["-o"];
  } else {
    auto now = std::chrono::system_clock::to_time_t(std::chrono::system_clock::now());
    std::tm tm = *std::localtime(&now);
    std::ostringstream oss;
    oss << std::put_time(&tm, "%Y%m%d%H%M%S");
    tag = oss.str();
  }
  const auto t0 = std::chrono::steady_clock::now();
  try {
    gample::Init init = gample::Init::parseInputFile(args["-i"]);
    const auto& T = init.paramForTimeIntegration;
    const bool fused = !(args.count("--reference-order") && args["--reference-order"] == "1");
    gample::Simulation sim(init, T.ProjectName + "_" + tag, fused);
    sim.initialize();
    for (int c = T.Start + 1; c <= T.End; ++c) {
      sim.cycle();
      if (T.LogOutput != 0 && c % T.LogOutput == 0) std::cerr << "Frame " << c << " completed\n";
    }
    GP_CUDA(cudaStreamSynchronize(sim.stream));
    const auto secs = std::chrono::duration_cast<std::chrono::seconds>(std::chrono::steady_clock::now() - t0);
    if (sim.logger)
      sim.logger->logComment("culculation end.\ntotal elapsed time: " + std::to_string(secs.count()) + " sec.\n");
  } catch (const std::exception& e) {
    std::cerr << "[Fatal] " << e.what() << "\n";
    return 1;
  }
  return 0;
}
