/*
 * Minimal stand-in for boost::lexical_cast -- test infrastructure only.
 *
 * The CLAST reference uses boost::lexical_cast<int|double>(std::string) to
 * parse command-line values (listenCommandLine.cpp) and the '@startIdx'
 * lines of preprocessed FASTA (CFASTALoader.cpp:139).  Boost is not
 * installed here, so oracle/build_ref.py puts this header first on the
 * include path.  It keeps the behaviour the reference relies on: the whole
 * string must be one number, with no leading or trailing characters,
 * otherwise boost::bad_lexical_cast is thrown.
 */
#ifndef CLAST_REFSHIM_BOOST_LEXICAL_CAST_HPP_
#define CLAST_REFSHIM_BOOST_LEXICAL_CAST_HPP_

#include <cerrno>
#include <climits>
#include <cstdlib>
#include <stdexcept>
#include <string>

namespace boost {

class bad_lexical_cast : public std::bad_cast {};

namespace refshim_detail {
template <class T> struct parse;
template <> struct parse<int> {
  static int run(const std::string& s) {
    if (s.empty() || s[0] == ' ' || s[0] == '\t') throw bad_lexical_cast();
    errno = 0;
    char* end = nullptr;
    const long v = std::strtol(s.c_str(), &end, 10);
    if (end != s.c_str() + s.size() || errno == ERANGE || v < INT_MIN || v > INT_MAX)
      throw bad_lexical_cast();
    return static_cast<int>(v);
  }
};
template <> struct parse<double> {
  static double run(const std::string& s) {
    if (s.empty() || s[0] == ' ' || s[0] == '\t') throw bad_lexical_cast();
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (end != s.c_str() + s.size()) throw bad_lexical_cast();
    return v;
  }
};
}  // namespace refshim_detail

template <class T>
T lexical_cast(const std::string& s) { return refshim_detail::parse<T>::run(s); }

}  // namespace boost

#endif
