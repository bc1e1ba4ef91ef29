// GridGenerator: points on the unit sphere of R^dim used as auxiliary fields.
// Interface of the reference's include/GridGenerator.h:8-55; point k, coordinate i is
// gCoOfPoint(k, i).
#ifndef GRIDGENERATOR_H
#define GRIDGENERATOR_H

#include <iostream>

using namespace std;

class GridGenerator {
 public:
  GridGenerator(const int dim);
  ~GridGenerator();
  int gDim() const;
  int gNPoints() const;
  double gCoOfPoint(const int point, const int index) const;
  friend ostream &operator<<(ostream &os, const GridGenerator &theGrid);
  void FillSimple(const int denominator);
  void FillMarsaglia(const int pointsPerCo);

 private:
  int dim;
  bool gridFilled;
  int nStates;
  double *grid;
  bool GenerateNextSimple(int *state, const int denominator);
};

#endif
