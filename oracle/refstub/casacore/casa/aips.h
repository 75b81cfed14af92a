// Test infrastructure: a minimal stand-in for casacore's aips.h, so that the
// reference's own GridKernel.cc compiles on its own (oracle/_ref).  Nothing
// of casacore is reproduced: only the names GridKernel.cc uses.
#ifndef ORACLE_REFSTUB_AIPS_H
#define ORACLE_REFSTUB_AIPS_H
#include <cstddef>
namespace casacore {
typedef float Float;
typedef double Double;
}  // namespace casacore
#endif
