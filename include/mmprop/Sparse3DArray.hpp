// Sparse3DArray.hpp — drop-in for the reference's sparse coupling tensor Q^(p)_{k,l,m}
// (include/Sparse3DArray.hpp:7-30): non-zeros kept in insertion order, which decides
// the solver's pair table.
#ifndef MMPROP_B200_SPARSE_3D_ARRAY_HPP
#define MMPROP_B200_SPARSE_3D_ARRAY_HPP

#include <vector>

struct NonZeroValue {
  unsigned int index[3];  // k, l, m
  double value;
};

class Sparse3DArray {
 public:
  Sparse3DArray() {}
  NonZeroValue getNonZeroValue(const unsigned int i) const { return Q_[i]; }
  unsigned int getNumberOfNonZeroValues() const { return (unsigned int)Q_.size(); }
  void addNonZeroValue(const NonZeroValue nzv) { Q_.push_back(nzv); }
  void resetValue(const unsigned int i, const double Q_klm) { Q_[i].value = Q_klm; }

 private:
  std::vector<NonZeroValue> Q_;
};

#endif
