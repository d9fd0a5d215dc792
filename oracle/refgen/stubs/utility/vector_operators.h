// Stand-in for the reference's vector_operators.h (TEST INFRASTRUCTURE ONLY; the original pulls in PETSc):
// the code generator only streams vectors and sets into its (swallowed) log messages.
#pragma once
#include <ostream>
#include <set>
#include <vector>
template<class T>
std::ostream& operator<<(std::ostream& o, const std::vector<T>& v)
{
  for (const T& x : v)
    o << x << " ";
  return o;
}
template<class T>
std::ostream& operator<<(std::ostream& o, const std::set<T>& v)
{
  for (const T& x : v)
    o << x << " ";
  return o;
}
