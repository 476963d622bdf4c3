// Read-only stand-in for <boost/algorithm/string.hpp>, for building the reference's
// ExtractOfftargets here (Boost.Algorithm is not installed). Test infrastructure only.
//
// The reference calls trim (remove leading and trailing whitespace in place) and to_upper (upper-
// case in place) on each input line, with the default "C" locale; split is named in a using
// declaration but not called. The same operations with <cctype>:
#pragma once
#include <cctype>
#include <string>

namespace boost {
namespace algorithm {

inline void trim(std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace(static_cast<unsigned char>(s[b]))) b++;
    while (e > b && std::isspace(static_cast<unsigned char>(s[e - 1]))) e--;
    s = s.substr(b, e - b);
}

inline void to_upper(std::string& s) {
    for (char& c : s) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
}

// named by the reference's using-declaration only
template <class SequenceT, class RangeT, class PredicateT>
SequenceT& split(SequenceT& out, RangeT& in, PredicateT pred);

}  // namespace algorithm
}  // namespace boost
