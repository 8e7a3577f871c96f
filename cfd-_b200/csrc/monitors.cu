// monitors.cu - per-step model monitors on the device.
//
// The reference appends every model's monitors to its history after each step
// (cfd2d/solver.py:441-443): scalar integrals, mean temperature and Nusselt
// numbers, k mean and nu_t max, the VOF volume, its error and the front position.
// One launch after the step evaluates them all: every block reduces its share of
// the cells for every monitor into a scratch slot, and the last block to finish
// adds the block partials in block order (so a run repeats itself bit for bit) and
// writes one record per step into a ring beside the history. Steps queued in a graph
// keep running without a host synchronisation. numpy's nansum adds pairwise: the
// values agree to rounding.

#include <cuda_runtime.h>
#include <math.h>

#include "device.cuh"
#include "kernels.cuh"

namespace cfd {
namespace {

constexpr int kMonThreads = 256;
constexpr int kMonBlocksMax = 296;  // CFD2D_MONITOR_SCRATCH / (2 CFD2D_MAX_MONITORS)
static_assert(CFD2D_MONITOR_SCRATCH == 2 * CFD2D_MAX_MONITORS * kMonBlocksMax, "monitor scratch size");

__device__ __forceinline__ int side_cell(const cfd2d_sim& S, int side, int k) {
    const int nx = S.nx, ny = S.ny, pc = ny + 2;
    if (side == CFD2D_LEFT) return 1 * pc + k + 1;
    if (side == CFD2D_RIGHT) return nx * pc + k + 1;
    if (side == CFD2D_BOTTOM) return (k + 1) * pc + 1;
    return (k + 1) * pc + ny;
}

// this block's share of monitor M: v[0] (sum, max or largest index), v[1] (count)
__device__ void block_partial(const cfd2d_sim& S, const cfd2d_monitor& M, double (&v)[2], double* sred) {
    const int nx = S.nx, ny = S.ny, pc = ny + 2;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    v[0] = 0.0;
    v[1] = 0.0;
    switch (M.kind) {
        case CFD2D_MON_SUM_FLUID:
        case CFD2D_MON_VOLUME_ERROR:
        case CFD2D_MON_MEAN_FLUID:
            for (int q = t0; q < nx * ny; q += stride) {
                const int c = (q / ny + 1) * pc + q % ny + 1;
                if (S.fluid[c]) {
                    v[0] += M.data[c];
                    v[1] += 1.0;
                }
            }
            block_sum<2>(v, sred);
            return;
        case CFD2D_MON_MAX_ALL: {
            double m[1] = {-INFINITY};
            for (int c = t0; c < (nx + 2) * (ny + 2); c += stride) m[0] = npmax(m[0], M.data[c]);
            block_max<1>(m, sred, -INFINITY);
            v[0] = m[0];
            return;
        }
        case CFD2D_MON_NUSSELT: {
            const cfd2d_scalar& sc = S.scalars[M.slot];
            const bool xs = M.side == CFD2D_LEFT || M.side == CFD2D_RIGHT;
            const int len = xs ? ny : nx;
            const double h = xs ? S.dx : S.dy;
            double s1[1] = {0.0};
            for (int k = t0; k < len; k += stride) {
                const int c = side_cell(S, M.side, k);
                const int64_t code = sc.bt[M.side][k];
                const double val = sc.bv[M.side][k];
                // -D (value - inner) / (h / 2) at a fixed value, -flux at a given flux
                // (cfd2d/models.py:245-249)
                if (code == 1) s1[0] += ((-sc.diff[c]) * (val - sc.phi[c])) / (0.5 * h);
                else if (code == 2) s1[0] += -val;
            }
            block_sum<1>(s1, sred);
            v[0] = s1[0];
            return;
        }
        case CFD2D_MON_FRONT_X:
        case CFD2D_MON_HEIGHT_LEFT: {
            const bool row = M.kind == CFD2D_MON_FRONT_X;
            const int len = row ? nx : ny;
            double m[1] = {-1.0};
            for (int k = t0; k < len; k += stride) {
                const int c = row ? (k + 1) * pc + 1 : 1 * pc + k + 1;
                if (M.data[c] > 0.5 && (double)k > m[0]) m[0] = (double)k;
            }
            block_max<1>(m, sred, -1.0);
            v[0] = m[0];
            return;
        }
        default: return;
    }
}

// the monitor's value from the block partials, added in block order
__device__ double finish(const cfd2d_sim& S, const cfd2d_monitor& M, const double* p0, const double* p1, int nb) {
    const int nx = S.nx, ny = S.ny;
    switch (M.kind) {
        case CFD2D_MON_SUM_FLUID:
        case CFD2D_MON_VOLUME_ERROR:
        case CFD2D_MON_MEAN_FLUID: {
            double s = 0.0, n = 0.0;
            for (int b = 0; b < nb; ++b) {
                s += ld_cg(p0 + b);
                n += ld_cg(p1 + b);
            }
            if (M.kind == CFD2D_MON_MEAN_FLUID) return s / n;
            const double vol = (s * S.dx) * S.dy;
            if (M.kind == CFD2D_MON_SUM_FLUID) return vol;
            return vol / (M.param > 1e-300 ? M.param : 1e-300) - 1.0;
        }
        case CFD2D_MON_MAX_ALL: {
            double m = -INFINITY;
            for (int b = 0; b < nb; ++b) m = npmax(m, ld_cg(p0 + b));
            return m;
        }
        case CFD2D_MON_NUSSELT: {
            const bool xs = M.side == CFD2D_LEFT || M.side == CFD2D_RIGHT;
            double s = 0.0;
            for (int b = 0; b < nb; ++b) s += ld_cg(p0 + b);
            // |mean(q)| L / (alpha dT) with L = dT = 1 (cfd2d/models.py:407-412)
            return fabs(s / (double)(xs ? ny : nx)) * 1.0 / (M.param * 1.0);
        }
        case CFD2D_MON_FRONT_X:
        case CFD2D_MON_HEIGHT_LEFT: {
            double m = -1.0;
            for (int b = 0; b < nb; ++b) m = fmax(m, ld_cg(p0 + b));
            if (m < 0.0) return 0.0;
            const double h = M.kind == CFD2D_MON_FRONT_X ? S.dx : S.dy;
            // cell centre (k + 1/2) h plus half a cell (cfd2d/vof.py:292-297)
            return (m + 0.5) * h + 0.5 * h;
        }
        default: return 0.0;
    }
}

__global__ void __launch_bounds__(kMonThreads) k_monitors(cfd2d_sim S) {
    cfd2d_state* st = S.state;
    if (!st || !st->active) return;
    __shared__ double sred[64];
    const int nb = gridDim.x;
    for (int k = 0; k < S.nmon; ++k) {
        double v[2];
        block_partial(S, S.mon[k], v, sred);
        if (threadIdx.x == 0) {
            S.mon_part[(2 * k) * nb + blockIdx.x] = v[0];
            S.mon_part[(2 * k + 1) * nb + blockIdx.x] = v[1];
        }
        __syncthreads();
    }
    if (!last_block(&st->ticket[3])) return;
    if (threadIdx.x == 0) {
        double* rec = S.mon_ring + (size_t)((st->n - 1) % S.hist_cap) * CFD2D_MAX_MONITORS;
        for (int k = 0; k < S.nmon; ++k)
            rec[k] = finish(S, S.mon[k], S.mon_part + (2 * k) * nb, S.mon_part + (2 * k + 1) * nb, nb);
        __threadfence();
        st->ticket[3] = 0u;
    }
}

}  // namespace

cudaError_t stage_monitors(const cfd2d_sim& S, cudaStream_t s) {
    if (S.nmon <= 0 || !S.mon_ring || !S.mon_part || S.hist_cap <= 0 || !S.state) return cudaSuccess;
    const long long cells = (long long)(S.nx + 2) * (S.ny + 2);
    long long nb = (cells + kMonThreads - 1) / kMonThreads;
    if (nb > kMonBlocksMax) nb = kMonBlocksMax;
    if (nb < 1) nb = 1;
    k_monitors<<<(unsigned)nb, kMonThreads, 0, s>>>(S);
    return cudaGetLastError();
}

}  // namespace cfd
