// TwoSiteObject: the two-site tensor of neighbouring MPS sites and its SVD split.
// Interface of the reference's include/TwoSiteObject.h:9-61.
#ifndef TWOSITEOBJECT_H
#define TWOSITEOBJECT_H

#include <vector>

#include "MPStensor.h"

class TwoSiteObject {
 public:
  TwoSiteObject(const int DimL, const int DimR, const int phys_d);
  ~TwoSiteObject();
  int gPhys_d() const;
  int gDimL() const;
  int gDimR() const;
  void Compose(MPStensor *MPSleft, MPStensor *MPSright);
  int gStorageSize() const;
  double *gStorage(const int d_left, const int d_right);
  double *gStorage();
  int Decompose(MPStensor *MPSleft, MPStensor *MPSright, const int Dtrunc, bool movingright,
                bool possiblyCompress);

 private:
  int phys_d, DimL, DimR;
  std::vector<double> storage;
  static const double SchmidtTrunc;
};

#endif
