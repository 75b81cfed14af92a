// Test infrastructure: the part of casacore::Matrix that GridKernel.cc uses,
// as a column-major view over caller-owned memory (element (i, j) at
// i + nrow * j, the casacore storage order).
#ifndef ORACLE_REFSTUB_MATRIX_H
#define ORACLE_REFSTUB_MATRIX_H
#include <cstddef>
namespace casacore {
template <class T>
class Matrix {
 public:
  Matrix(T* data, std::size_t nrow, std::size_t ncol) : p_(data), nr_(nrow), nc_(ncol) {}
  T& operator()(long i, long j) { return p_[i + (long)nr_ * j]; }
  const T& operator()(long i, long j) const { return p_[i + (long)nr_ * j]; }
  std::size_t nrow() const { return nr_; }
  std::size_t ncolumn() const { return nc_; }

 private:
  T* p_;
  std::size_t nr_, nc_;
};
}  // namespace casacore
#endif
