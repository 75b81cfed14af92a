// Test infrastructure: casacore::Complex is std::complex<float> in casacore
// too; the reference builds with -fcx-limited-range, so products are the
// plain (ac - bd, ad + bc) formula.
#ifndef ORACLE_REFSTUB_COMPLEX_H
#define ORACLE_REFSTUB_COMPLEX_H
#include <complex>
namespace casacore {
typedef std::complex<float> Complex;
}  // namespace casacore
#endif
