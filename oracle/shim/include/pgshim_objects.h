/*
 * pgshim_objects.h -- layouts of the stand-in PETSc objects (test infrastructure only), shared by
 * shim.cpp and the oracle driver so the driver can read assembled matrices and vectors directly.
 */
#pragma once
#include "pgshim.h"
#include <string>
#include <vector>

struct pg_Mat {
  int m = 0, n = 0;
  bool dense = false;
  std::vector<std::vector<int>> cols;     // sorted column indices per row
  std::vector<std::vector<double>> vals;  // values aligned with cols
  std::vector<double> dvals;              // dense storage (row-major) when dense
  std::vector<double> flat;               // MatSeqAIJGetArray: the values of all rows, in row order
};
struct pg_Vec { std::vector<double> a; };
struct pg_IS { std::vector<int> idx; };
struct pg_PC { std::string type; };
struct pg_KSP { Mat A = nullptr; pg_PC pc; std::string type; };
struct pg_SNES { int dummy; };
struct pg_VecScatter { int dummy; };

