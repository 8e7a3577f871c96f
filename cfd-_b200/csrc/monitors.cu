// monitors.cu - per-step model monitors on the device.
//
// The reference appends every model's monitors to its history after each step
// (cfd2d/solver.py:441-443): scalar integrals, mean temperature and Nusselt
// numbers, k mean and nu_t max, the VOF volume, its error and the front position.
// One block evaluates them after the step and writes one record per step into a
// ring beside the history, so steps queued in a graph keep running without a host
// synchronisation. Sums run in a fixed block order (numpy's nansum adds pairwise:
// the values agree to rounding).

#include <cuda_runtime.h>
#include <math.h>

#include "device.cuh"
#include "kernels.cuh"

namespace cfd {
namespace {

constexpr int kMonThreads = 1024;

__device__ double monitor_value(const cfd2d_sim& S, const cfd2d_monitor& M, double* sred) {
    const int nx = S.nx, ny = S.ny, pc = ny + 2;
    const int tid = threadIdx.x;
    switch (M.kind) {
        case CFD2D_MON_SUM_FLUID:
        case CFD2D_MON_VOLUME_ERROR:
        case CFD2D_MON_MEAN_FLUID: {
            double v[2] = {0.0, 0.0};
            for (int q = tid; q < nx * ny; q += blockDim.x) {
                const int c = (q / ny + 1) * pc + q % ny + 1;
                if (S.fluid[c]) {
                    v[0] += M.data[c];
                    v[1] += 1.0;
                }
            }
            block_sum<2>(v, sred);
            if (M.kind == CFD2D_MON_MEAN_FLUID) return v[0] / v[1];
            const double vol = (v[0] * S.dx) * S.dy;
            if (M.kind == CFD2D_MON_SUM_FLUID) return vol;
            return vol / (M.param > 1e-300 ? M.param : 1e-300) - 1.0;
        }
        case CFD2D_MON_MAX_ALL: {
            double v[1] = {-INFINITY};
            for (int c = tid; c < (nx + 2) * (ny + 2); c += blockDim.x) v[0] = npmax(v[0], M.data[c]);
            block_max<1>(v, sred, -INFINITY);
            return v[0];
        }
        case CFD2D_MON_NUSSELT: {
            const cfd2d_scalar& sc = S.scalars[M.slot];
            const bool xs = M.side == CFD2D_LEFT || M.side == CFD2D_RIGHT;
            const int len = xs ? ny : nx;
            const double h = xs ? S.dx : S.dy;
            double v[1] = {0.0};
            for (int k = tid; k < len; k += blockDim.x) {
                int c;
                if (M.side == CFD2D_LEFT) c = 1 * pc + k + 1;
                else if (M.side == CFD2D_RIGHT) c = nx * pc + k + 1;
                else if (M.side == CFD2D_BOTTOM) c = (k + 1) * pc + 1;
                else c = (k + 1) * pc + ny;
                const int64_t code = sc.bt[M.side][k];
                const double val = sc.bv[M.side][k];
                double q = 0.0;
                if (code == 1) q = ((-sc.diff[c]) * (val - sc.phi[c])) / (0.5 * h);
                else if (code == 2) q = -val;
                v[0] += q;
            }
            block_sum<1>(v, sred);
            return fabs(v[0] / (double)len) * 1.0 / (M.param * 1.0);
        }
        case CFD2D_MON_FRONT_X:
        case CFD2D_MON_HEIGHT_LEFT: {
            const bool row = M.kind == CFD2D_MON_FRONT_X;
            const int len = row ? nx : ny;
            double v[1] = {-1.0};
            for (int k = tid; k < len; k += blockDim.x) {
                const int c = row ? (k + 1) * pc + 1 : 1 * pc + k + 1;
                if (M.data[c] > 0.5 && (double)k > v[0]) v[0] = (double)k;
            }
            block_max<1>(v, sred, -1.0);
            if (v[0] < 0.0) return 0.0;
            const double h = row ? S.dx : S.dy;
            return (v[0] + 0.5) * h + 0.5 * h;
        }
        default: return 0.0;
    }
}

__global__ void __launch_bounds__(kMonThreads) k_monitors(cfd2d_sim S) {
    const cfd2d_state* st = S.state;
    if (!st || !st->active) return;
    __shared__ double sred[64];
    double* rec = S.mon_ring + (size_t)((st->n - 1) % S.hist_cap) * CFD2D_MAX_MONITORS;
    for (int k = 0; k < S.nmon; ++k) {
        const double v = monitor_value(S, S.mon[k], sred);
        if (threadIdx.x == 0) rec[k] = v;
        __syncthreads();
    }
}

}  // namespace

cudaError_t stage_monitors(const cfd2d_sim& S, cudaStream_t s) {
    if (S.nmon <= 0 || !S.mon_ring || S.hist_cap <= 0 || !S.state) return cudaSuccess;
    k_monitors<<<1, kMonThreads, 0, s>>>(S);
    return cudaGetLastError();
}

}  // namespace cfd
