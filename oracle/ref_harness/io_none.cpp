/*
 * IO module for the oracle builds (takes the place of src/IO/text1d.cpp in the
 * Makefile's IO slot).  TEST INFRASTRUCTURE.
 *
 * The reference's printCols writes text snapshots under ../results/Last and, as
 * a side effect, stores isShocked in the advected tracer slot TR1+1
 * (src/IO/text1d.cpp:137-141).  The oracle drives the step without output, so
 * printCols here writes nothing and changes no state; the GPU path does the same.
 */
#include "grid.h"
#include "simu.h"

void Grid::printCols(int it, double t) {
  UNUSED(it);
  UNUSED(t);
}

void Simu::reinitialise(DIR *dir) {
  UNUSED(dir);
  fprintf(stderr, "oracle: resume from text snapshots is not part of the oracle\n");
  abort();
}
