// MPStensor: one site of an MPS, storage[r + dimL * (c + dimR * sigma)].
// Interface of the reference's include/MPStensor.h:17-66.
#ifndef MPSTENSOR_H
#define MPSTENSOR_H

#include <fstream>
#include <iostream>

using std::ifstream;
using std::ostream;

#include "Random.h"

class MPStensor {
  friend ostream &operator<<(ostream &output, const MPStensor &tensor);

 public:
  MPStensor(const int dimL, const int dimR, const int phys_d, Random *RN);
  MPStensor(MPStensor *toCopy);
  MPStensor(const char *filename, Random *RN);
  ~MPStensor();
  int gDimL() const;
  int gDimR() const;
  int gPhys_d() const;
  int gStorageSize() const;
  double *gStorage();
  double *gStorage(const int d_val);
  Random *gRN();
  void QR(double *Rmx, double *mem, double *tau, double *work);
  void LQ(double *Lmx, double *tau, double *work);
  void LeftMultiply(double *Lmx, double *work);
  void RightMultiply(double *Rmx, double *work);
  void Reset(const int dimL, const int dimR);

 private:
  Random *RN;
  int dimL, dimR, phys_d;
  int storageSize;
  double *storage;
  void random();
};

#endif
