// vof.cuh - device pieces of the two-phase VOF model used inside other kernels.
#pragma once

#include "../../include/cfd2d_b200.h"

namespace cfd {

// CSF surface-tension acceleration on u face (i, j) and v face (i, j):
// sigma kappa_f (grad alpha)_f / rho_f (cfd2d/vof.py:252-258)
__device__ __forceinline__ double csf_u(const cfd2d_sim& S, int i, int j) {
    const cfd2d_vof& V = S.vof;
    const int pc = S.ny + 2;
    const double fxs = ((V.sigma * 0.5) * (V.kappa[i * pc + j] + V.kappa[(i + 1) * pc + j])) *
                       (V.alpha[(i + 1) * pc + j] - V.alpha[i * pc + j]) / S.dx;
    const double rx = 0.5 * (V.rho[i * pc + j] + V.rho[(i + 1) * pc + j]);
    return fxs / rx;
}

__device__ __forceinline__ double csf_v(const cfd2d_sim& S, int i, int j) {
    const cfd2d_vof& V = S.vof;
    const int pc = S.ny + 2;
    const double fys = ((V.sigma * 0.5) * (V.kappa[i * pc + j] + V.kappa[i * pc + j + 1])) *
                       (V.alpha[i * pc + j + 1] - V.alpha[i * pc + j]) / S.dy;
    const double ry = 0.5 * (V.rho[i * pc + j] + V.rho[i * pc + j + 1]);
    return fys / ry;
}

}  // namespace cfd
