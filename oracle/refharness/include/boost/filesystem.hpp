// Stand-in for boost/filesystem.hpp — TEST INFRASTRUCTURE ONLY: the one call
// the reference's file readers make (exists).
#pragma once
#include <string>
#include <sys/stat.h>

namespace boost {
namespace filesystem {
inline bool exists(const std::string& p) {
  struct stat st;
  return ::stat(p.c_str(), &st) == 0;
}
}  // namespace filesystem
}  // namespace boost
