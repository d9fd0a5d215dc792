// Stand-in for the reference's OutputWriter::Generic (TEST INFRASTRUCTURE ONLY): the code generator only
// opens its output file through it.
#pragma once
#include <fstream>
#include <string>
namespace OutputWriter {
class Generic {
public:
  static void openFile(std::ofstream& file, std::string filename, bool append = false)
  {
    file.open(filename.c_str(), append ? std::ios::out | std::ios::app : std::ios::out);
  }
};
} // namespace OutputWriter
