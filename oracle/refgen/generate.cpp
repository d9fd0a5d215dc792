// Runs the reference's own CellML code generator (CellmlSourceCodeGeneratorVc, compiled from the
// reference's sources against the stand-in headers in stubs/) and writes the FastMonodomainSolver source it
// emits for one model and parameter choice.  TEST INFRASTRUCTURE ONLY: the emitted compute0DInstance is the
// reference's Heun step (03_generator_vc.cpp:873-1163), which the oracle's restatement is checked against.
//
//   refgen <model.c> <nStates> <nAlgebraics> <approximateExponentialFunction 0|1> <output.cpp>
//          <parametersUsedAsAlgebraic, comma separated or -> <parametersUsedAsConstant, comma separated or ->
#include <Python.h>

#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "cellml/source_code_generator/03_generator_vc.h"

static std::vector<int> parse_list(const std::string& s)
{
  std::vector<int> out;
  if (s == "-")
    return out;
  std::stringstream ss(s);
  std::string item;
  while (std::getline(ss, item, ','))
    out.push_back(std::atoi(item.c_str()));
  return out;
}

int main(int argc, char** argv)
{
  if (argc != 8) {
    std::cerr << "usage: refgen model.c nStates nAlgebraics approx output.cpp algebraicParams constantParams\n";
    return 2;
  }
  const int n_states = std::atoi(argv[2]), n_algebraics = std::atoi(argv[3]);
  const bool approx = std::atoi(argv[4]) != 0;
  const std::vector<int> pa = parse_list(argv[6]), pc = parse_list(argv[7]);
  const int n_instances = 4;  // one point buffer of the vc path
  try {
    CellmlSourceCodeGeneratorVc g;
    g.initializeNames(argv[1], n_instances, n_states, n_algebraics);
    std::vector<double> initial;  // no parametersInitialValues: the generator fills zeros
    std::vector<double> values((size_t)n_algebraics * n_instances + 1, 0.0);
    g.initializeSourceCode(pa, pc, initial, n_algebraics, values.data());
    g.generateSourceFileFastMonodomain(argv[5], approx);
  } catch (const std::exception& e) {
    std::cerr << "refgen: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
