// Stand-in for boost::lexical_cast<std::string>(number), the only use the
// reference's Diamond front-end makes of it (an error message).  Test
// infrastructure for building the reference oracle only.
#ifndef ORACLE_SHIM_LEXICAL_CAST_HPP
#define ORACLE_SHIM_LEXICAL_CAST_HPP
#include <sstream>
#include <string>

namespace boost {
template <class Target, class Source> Target lexical_cast(const Source &s) {
  std::ostringstream os;
  os << s;
  return os.str();
}
} // namespace boost
#endif
