// pcg.cuh - launch description of the pressure solver kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cfd2d_b200.h"

namespace cfd {

struct PcgLaunch {
    cfd2d_poisson op;
    int rhs_mode;              // 0: rhs array (nx*ny); 1: div(F, G) / dt from the padded F, G
    const double* rhs;
    const double* F;
    const double* G;
    double dx, dy;
    const double* dt_ptr;      // mode 1: dt read on the device (state->dt) ...
    double dt_const;           // ... or this constant when dt_ptr is null
    double rtol;
    int maxiter;
    double* p_out;             // nx*ny, or (nx+2)(ny+2) when p_padded
    int p_padded;
    int32_t* iters_out;        // device, may be null
    int32_t* iters_out2;       // device, may be null
    int32_t* status_out;       // device, may be null (atomicOr of CFD2D_S_* bits)
    const int32_t* active;     // device, may be null: skip when *active == 0
    int cap_cells;             // set by pcg_launch
    double* snap;              // grid solver: iterate snapshots (nullable)
    int snap_every, snap_max;
};

int pcg_cluster_plan(int nx, int ny);
bool pcg_var_cluster_fits(int nx, int ny, int C);
cudaError_t barrier_selftest(unsigned int* bar, int* status, int* ok_out, cudaStream_t s);
size_t pcg_grid_workspace_doubles(int nx, int ny);
cudaError_t pcg_launch(const PcgLaunch& L, cudaStream_t s);
cudaError_t pcg_matvec(const cfd2d_poisson& op, const double* x, double* y, cudaStream_t s);

}  // namespace cfd
