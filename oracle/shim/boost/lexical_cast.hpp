// Compatibility header for compiling the reference's CPU sources without Boost.
// Only boost::lexical_cast<int>(std::string): the whole string must be an integer,
// otherwise boost::bad_lexical_cast is thrown.
#pragma once
#include <cerrno>
#include <cstdlib>
#include <string>
#include <typeinfo>
namespace boost {
class bad_lexical_cast : public std::bad_cast {
 public:
  const char* what() const noexcept override { return "bad lexical cast"; }
};
template <class T>
T lexical_cast(const std::string& s);
template <>
inline int lexical_cast<int>(const std::string& s) {
  if (s.empty()) throw bad_lexical_cast();
  char* end = nullptr;
  errno = 0;
  const long v = std::strtol(s.c_str(), &end, 10);
  if (*end != '\0' || errno != 0 || v < -2147483647L - 1 || v > 2147483647L) throw bad_lexical_cast();
  return (int)v;
}
}  // namespace boost
