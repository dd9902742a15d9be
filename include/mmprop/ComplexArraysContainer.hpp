// ComplexArraysContainer.hpp — drop-in for the reference's container of M complex
// arrays indexed [mode][sample] (include/ComplexArraysContainer.hpp:7-29). Constructor
// argument order is (array size, number of arrays), as in the reference.
#ifndef MMPROP_B200_COMPLEX_ARRAYS_CONTAINER_HPP
#define MMPROP_B200_COMPLEX_ARRAYS_CONTAINER_HPP

#include "ComplexArray.hpp"

class ComplexArraysContainer {
 public:
  ComplexArraysContainer() : M_(0), n_(0) {}
  ComplexArraysContainer(unsigned int arraySize, unsigned int numArrays)
      : M_(numArrays), n_(arraySize), arrays_(numArrays, ComplexArray(arraySize)) {}
  ComplexArraysContainer(unsigned int arraySize, std::complex<double> value, unsigned int numArrays)
      : M_(numArrays), n_(arraySize), arrays_(numArrays, ComplexArray(arraySize, value)) {}

  unsigned int getNumberOfArrays() const { return M_; }
  unsigned int getArraySize() const { return n_; }
  std::complex<double> getValue(const unsigned int arrayIndex, const unsigned int i) const {
    return arrays_[arrayIndex][i];
  }

  ComplexArray& operator[](unsigned int i) { return arrays_[i]; }
  ComplexArray& operator()(unsigned int i) { return arrays_[i]; }
  std::vector<ComplexArray> operator()() const { return arrays_; }
  operator std::vector<ComplexArray>() const { return arrays_; }

 private:
  unsigned int M_;
  unsigned int n_;
  std::vector<ComplexArray> arrays_;
};

#endif
