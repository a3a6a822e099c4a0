// MG_MODE pressure solve (PCG + red-black Gauss-Seidel multigrid); see tbfp_mg.cu.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "tbfp.h"
#include "tbfp_kernels.cuh"

namespace tbfp {

// One multigrid level as the kernels see it: sizes and FP32 tables.
struct MgLev {
  int nx, ny, nz;
  const float *invx1, *invx2, *invy1, *invy2, *invz1, *invz2;  // 1/(dc(i+1) df(i)), 1/(dc(i) df(i))
  const float *vx, *vy, *vz;                                     // df(i): cell volume factors
  const float *rx, *ry, *rz;  // restriction weights from the finer level, 2 per cell
  const float *px, *py, *pz;  // prolongation weights from the coarser level, 2 per cell
};

class MgSolver {
 public:
  struct Impl;
  MgSolver();
  ~MgSolver();
  MgSolver(const MgSolver &) = delete;
  MgSolver &operator=(const MgSolver &) = delete;
  // pcgCTOR (pcg.f90:62-99): the level hierarchy for an nx x ny x nz grid with
  // the caller's metrics (Fortran arrays dxf(1..nx), dxc(1..nx+1), ...).
  // Returns a TBFP_* status, with the message in *err.
  int init(const tbfp_mg_params &prm, int nx, int ny, int nz, const double *dxf, const double *dxc,
           const double *dyf, const double *dyc, const double *dzf, const double *dzc, std::string *err);
  // solvePCG (pcg.f90:103-140) on device arrays; psi is the initial guess and
  // the result (ghosts updated).  Returns TBFP_OK, TBFP_ENOTCONVERGED or an error.
  int solve(double *psi, Lay Lp, int hd_psi, const double *beta, Lay Lb, const double *q, Lay Lq, cudaStream_t st,
            int *iters, double *rel, int *mg_cycles, std::string *err);
  size_t device_bytes() const;

 private:
  Impl *d_;
};

}  // namespace tbfp
