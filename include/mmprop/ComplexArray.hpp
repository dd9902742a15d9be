// ComplexArray.hpp — drop-in for the reference's ComplexArray
// (include/ComplexArray.hpp:12-60 of alexandreroget/MM_Propagation): a heap array of
// std::complex<double> with element-wise operators. Storage is a std::vector here;
// assignment resizes to the right-hand side (the reference copies only as many
// elements as the left-hand side already holds).
#ifndef MMPROP_B200_COMPLEX_ARRAY_HPP
#define MMPROP_B200_COMPLEX_ARRAY_HPP

#include <cmath>
#include <complex>
#include <vector>

typedef std::complex<double> Complex;

class ComplexArray {
 public:
  ComplexArray() {}
  explicit ComplexArray(unsigned int size) : data_(size, Complex(0., 0.)) {}
  ComplexArray(unsigned int size, Complex a) : data_(size, a) {}

  unsigned int getSize() const { return (unsigned int)data_.size(); }

  Complex& operator[](unsigned int i) const { return const_cast<Complex&>(data_[i]); }
  Complex& operator()(unsigned int i) const { return const_cast<Complex&>(data_[i]); }
  Complex* operator()() const { return const_cast<Complex*>(data_.data()); }
  operator Complex*() const { return const_cast<Complex*>(data_.data()); }

  ComplexArray& operator=(const ComplexArray& a) { data_ = a.data_; return *this; }
  ComplexArray& operator=(const ComplexArray* a) { data_ = a->data_; return *this; }
  ComplexArray& operator+=(const ComplexArray& a) { for (size_t i = 0; i < data_.size(); ++i) data_[i] += a.data_[i]; return *this; }
  ComplexArray& operator+=(const Complex a) { for (auto& x : data_) x += a; return *this; }
  ComplexArray& operator-=(const ComplexArray& a) { for (size_t i = 0; i < data_.size(); ++i) data_[i] -= a.data_[i]; return *this; }
  ComplexArray& operator*=(const ComplexArray& a) { for (size_t i = 0; i < data_.size(); ++i) data_[i] *= a.data_[i]; return *this; }
  ComplexArray& operator*=(const Complex a) { for (auto& x : data_) x *= a; return *this; }
  ComplexArray& operator*=(const double a) { for (auto& x : data_) x *= a; return *this; }
  ComplexArray& operator/=(const ComplexArray& a) { for (size_t i = 0; i < data_.size(); ++i) data_[i] /= a.data_[i]; return *this; }
  ComplexArray& operator/=(const Complex a) { for (auto& x : data_) x /= a; return *this; }
  ComplexArray& operator/=(const double a) { for (auto& x : data_) x /= a; return *this; }

 private:
  std::vector<Complex> data_;
};

inline ComplexArray operator+(ComplexArray const& a, ComplexArray const& b) { ComplexArray r(a); r += b; return r; }
inline ComplexArray operator-(ComplexArray const& a, ComplexArray const& b) { ComplexArray r(a); r -= b; return r; }
inline ComplexArray operator*(ComplexArray const& a, ComplexArray const& b) { ComplexArray r(a); r *= b; return r; }
inline ComplexArray operator*(ComplexArray const& a, Complex const& b) { ComplexArray r(a); r *= b; return r; }
inline ComplexArray operator*(ComplexArray const& a, double const& b) { ComplexArray r(a); r *= b; return r; }
inline ComplexArray operator/(ComplexArray const& a, ComplexArray const& b) { ComplexArray r(a); r /= b; return r; }
inline ComplexArray operator/(ComplexArray const& a, Complex const& b) { ComplexArray r(a); r /= b; return r; }
inline ComplexArray operator/(ComplexArray const& a, double const& b) { ComplexArray r(a); r /= b; return r; }

inline double sum(const std::vector<double> A) { double s = 0.; for (double x : A) s += x; return s; }
inline double norm(const ComplexArray A) {
  double s = 0.;
  for (unsigned int i = 0; i < A.getSize(); ++i) s += std::norm(A[i]);
  return std::sqrt(s);
}
inline std::vector<double> abs(const ComplexArray A) {
  std::vector<double> r(A.getSize());
  for (unsigned int i = 0; i < A.getSize(); ++i) r[i] = std::abs(A[i]);
  return r;
}
inline ComplexArray conj(const ComplexArray A) {
  ComplexArray r(A.getSize());
  for (unsigned int i = 0; i < A.getSize(); ++i) r[i] = std::conj(A[i]);
  return r;
}
inline ComplexArray exp(const ComplexArray A) {
  ComplexArray r(A.getSize());
  for (unsigned int i = 0; i < A.getSize(); ++i) r[i] = std::exp(A[i]);
  return r;
}

#endif
