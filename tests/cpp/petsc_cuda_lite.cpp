/* PETSc-lite CUDA vectors and COO assembly for the boundary test (test
 * infrastructure only).  A Vec's device array is a staging copy: read access
 * uploads the host array, write access hands out a device buffer that is
 * copied back on restore.  MatSetPreallocationCOO keeps the (i, j) lists;
 * MatSetValuesCOO reads the device values back and appends one triplet per
 * non-negative (i, j), which the oracle's Mat sums as ADD_VALUES does. */
#include <cuda_runtime.h>
#include <map>
#include <vector>
#include "petsc_cuda_lite.h"
#include "shim_types.h"

namespace {
struct DevCopy {
    double *d = nullptr;
    int n = 0;
};
std::map<Vec, DevCopy> g_dev;
std::map<Mat, std::pair<std::vector<PetscInt>, std::vector<PetscInt>>> g_coo;

double *device_of(Vec v) {
    DevCopy &c = g_dev[v];
    if (c.n != v->n) {
        if (c.d) cudaFree(c.d);
        c.d = nullptr;
        if (cudaMalloc((void **)&c.d, (size_t)v->n * sizeof(double)) != cudaSuccess) return nullptr;
        c.n = v->n;
    }
    return c.d;
}
}  // namespace

PetscErrorCode VecCUDAGetArrayRead(Vec v, const PetscScalar **a) {
    double *d = device_of(v);
    if (!d || cudaMemcpy(d, v->a, (size_t)v->n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) return 1;
    *a = d;
    return 0;
}
PetscErrorCode VecCUDARestoreArrayRead(Vec, const PetscScalar **a) { *a = nullptr; return 0; }
PetscErrorCode VecCUDAGetArrayWrite(Vec v, PetscScalar **a) {
    double *d = device_of(v);
    if (!d) return 1;
    *a = d;
    return 0;
}
PetscErrorCode VecCUDARestoreArrayWrite(Vec v, PetscScalar **a) {
    cudaDeviceSynchronize();
    if (cudaMemcpy(v->a, *a, (size_t)v->n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
    *a = nullptr;
    return 0;
}
PetscErrorCode MatSetPreallocationCOO(Mat m, PetscCount n, PetscInt *i, PetscInt *j) {
    g_coo[m] = {std::vector<PetscInt>(i, i + n), std::vector<PetscInt>(j, j + n)};
    return 0;
}
PetscErrorCode MatSetValuesCOO(Mat m, const PetscScalar *d_vals, InsertMode) {
    auto it = g_coo.find(m);
    if (it == g_coo.end()) return 1;
    const std::vector<PetscInt> &I = it->second.first, &J = it->second.second;
    std::vector<double> v(I.size());
    if (cudaMemcpy(v.data(), d_vals, v.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
    m->r.clear();
    m->c.clear();
    m->v.clear();
    for (size_t k = 0; k < I.size(); k++)
        if (I[k] >= 0 && J[k] >= 0) {
            m->r.push_back(I[k]);
            m->c.push_back(J[k]);
            m->v.push_back(v[k]);
        }
    return 0;
}
