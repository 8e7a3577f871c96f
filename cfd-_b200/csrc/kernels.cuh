// kernels.cuh - host launchers of the stencil and bookkeeping kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cfd2d_b200.h"
#include "cellmath.cuh"

namespace cfd {

cudaError_t launch_momentum(const double* u, const double* v, const uint8_t* fl, int nx, int ny,
                            double dx, double dy, const double* nu, int variable, double gamma,
                            int periodic, double* hu, double* hv, const double* rho, int var_density,
                            cudaStream_t s);
cudaError_t launch_obstacle_bc(double* u, double* v, const uint8_t* fl, int nx, int ny, int periodic,
                               const cfd2d_state* st, cudaStream_t s);
cudaError_t launch_scalar_transport(const double* phi, const double* u, const double* v,
                                    const uint8_t* fl, int nx, int ny, double dx, double dy,
                                    const double* diff, int limiter, int periodic,
                                    const ScalarBCView& bc, int obs_t, double obs_v, double* out,
                                    cudaStream_t s);
cudaError_t launch_mask(int kind, int nx, int ny, double dx, double dy, const double* prm,
                        uint8_t* mask, cudaStream_t s);
cudaError_t launch_mask_polygon(int nx, int ny, double dx, double dy, const double* px, const double* py, int np,
                                uint8_t* mask, cudaStream_t s);
cudaError_t launch_mask_image(int nx, int ny, double dx, double dy, const uint8_t* solid, int h, int w, double x0,
                              double y0, double width, double height, uint8_t* mask, cudaStream_t s);

// step stages (all read step-varying scalars from S.state)
cudaError_t stage_domain_bc(const cfd2d_sim& S, double* u, double* v, int begin, cudaStream_t s);
cudaError_t stage_apply_bc(const cfd2d_sim& S, int begin, cudaStream_t s);
cudaError_t stage_sst_pre(const cfd2d_sim& S, cudaStream_t s);
cudaError_t stage_smag_pre(const cfd2d_sim& S, cudaStream_t s);
cudaError_t stage_vof_curvature(const cfd2d_sim& S, cudaStream_t s);
cudaError_t stage_monitors(const cfd2d_sim& S, cudaStream_t s);
int set_tile(int which, int tx, int ty);
int get_tile(int which, int* tx, int* ty);
cudaError_t stage_vof_operator(const cfd2d_sim& S, cudaStream_t s);
cudaError_t stage_vof_transport(const cfd2d_sim& S, cudaStream_t s);
cudaError_t stage_vof_properties(const cfd2d_sim& S, cudaStream_t s);
cudaError_t launch_vof_advect(const cfd2d_sim& S, double dt, double* out, cudaStream_t s);
cudaError_t stage_dt(const cfd2d_sim& S, cudaStream_t s);
cudaError_t stage_predictor(const cfd2d_sim& S, int copy_only, cudaStream_t s);
cudaError_t stage_correct(const cfd2d_sim& S, const double* p, int unit_dt, cudaStream_t s);
cudaError_t stage_flow_shift(const cfd2d_sim& S, cudaStream_t s);
cudaError_t stage_scalar(const cfd2d_sim& S, int slot, cudaStream_t s);
cudaError_t stage_scalar_ghosts(const cfd2d_sim& S, int slot, cudaStream_t s);
cudaError_t stage_end(const cfd2d_sim& S, cudaStream_t s);
cudaError_t stage_fill(const cfd2d_sim& S, double* a, int n, double value, cudaStream_t s);

int reduction_blocks(int ncell);

}  // namespace cfd
