// Read-only stand-in for <boost/regex.hpp>, for building the reference's ExtractOfftargets here
// (Boost.Regex is not installed). Test infrastructure only: oracle/Makefile compiles the
// reference's own source against it to produce the extraction fixture.
//
// ExtractOfftargets uses regex, sregex_iterator and smatch with two patterns built from character
// classes, counted repeats and one lookahead group, "(?=([ACG][ACGT]{19}[ACGT][AG]G))" and
// "(?=(C[CT][ACGT][ACGT]{19}[TGC]))" (ExtractOfftargets.cpp:16-17). Those constructs mean the same
// in Boost's default Perl syntax and in std::regex's ECMAScript syntax, and both iterators step past
// an empty match by one character, so every overlapping site is reported once.
#pragma once
#include <regex>

namespace boost {
using std::regex;
using std::smatch;
using std::sregex_iterator;
}  // namespace boost
