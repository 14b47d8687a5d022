// ORACLE — test infrastructure only.  What the CPU build of the reference
// checker records from CUP2D's own code: the preconditioner P^-1 handed to
// the solver (ExpAMRSolver.cpp:86-98) and the linear system that
// LocalSpMatDnVec::make leaves for BiCGSTABSolver::updateAll
// (LocalSpMatDnVec.cpp:81-189, BiCGSTAB.cu:142-253): the local COO with int
// row/column indices, b, x0 and h^2 per block.
#pragma once

#include <vector>

struct RefCapture {
  std::vector<double> pinv;
  std::vector<int> row, col;
  std::vector<double> val, b, x0, h2;
  int m = 0;
  int mean_row = -1;
  bool have_system = false;
};

RefCapture& ref_capture();
