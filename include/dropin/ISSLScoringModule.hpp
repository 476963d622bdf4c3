// Drop-in replacement for the reference's include/ISSLScoringModule.hpp.
//
// A Crackling++ pipeline built with this directory ahead of the reference's include directory
// (-I<this repo>/include/dropin -I<this repo>/include -I<reference>/include), without compiling
// the reference's lib/ISSLScoringModule.cpp and linked against libissl_b200.so, constructs and
// runs ISSLScoringModule exactly as src/CracklingPlusPlus.cpp:74-81 does:
//     ISSLScoringModule ISSLScoring(config);   ...   ISSLScoring.run(*currentBatch);
// with the reference's own cracklingConfig and guideResults (include/util.hpp).
#ifndef ISSLScoringModuleInclude
#define ISSLScoringModuleInclude
#include "util.hpp"
#define ISSL_B200_USE_REFERENCE_TYPES
#include "issl_b200_module.hpp"
#endif
