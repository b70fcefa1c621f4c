/* Concrete PETSc-lite object layouts shared by the shim and the C driver
 * (test infrastructure only). */
#pragma once
#include <vector>
struct _p_Vec {
    double *a;
    int n;
};
struct _p_Mat {
    std::vector<int> r, c;
    std::vector<double> v;
};
