// Stand-in for the reference's DihuContext (TEST INFRASTRUCTURE ONLY): the code generator only asks for
// the process's rank, and the cross-check runs as one process.
#pragma once
class DihuContext {
public:
  static int ownRankNoCommWorld() { return 0; }
};
