// walldist.cu - distance of every cell centre to the nearest wall, on the device.
//
// cfd2d/turbulence.py:43-70 (wall_distance) takes the exact Euclidean distance
// transform of the wall mask (scipy.ndimage.distance_transform_edt with sampling
// (dx, dy)) and moves it from the wall cell's centre to its face. Walls are the
// interior solid cells and the ghost layer of every no-slip side
// (turbulence.py:28-40); with periodicity in x the transform runs on three copies
// of the columns 1..nx side by side and keeps the middle one.
//
// Here the transform is separable. Pass 1 (one thread per grid row j) scans the
// row in x and stores the signed offset to its nearest wall cell. Pass 2 (one
// thread per cell) searches rows j' = j, j +- 1, j +- 2, ... for the smallest
// (off(j') dx)^2 + ((j - j') dy)^2 and stops once ((j - j') dy)^2 alone exceeds the
// best value found: every later row is farther, so the minimum is exact. The
// squared distance is formed from integer offsets in the order scipy uses
// (x term plus y term of float(offset) * spacing, squared), so the distance of
// the nearest wall cell is the same double.

#include <climits>
#include <cstdint>

#include "../../include/cfd2d_b200.h"

namespace cfd {
namespace {

constexpr int kNoWall = INT_MAX;
constexpr int kRowThreads = 128;
constexpr int kCellTX = 32, kCellTY = 8;

// Wall cell of the padded (nx+2) x (ny+2) grid (turbulence.py:28-40).
__device__ __forceinline__ bool is_wall(const uint8_t* fluid, const int* noslip, int nx, int ny, int i,
                                        int j) {
    if (i == 0 && noslip[0]) return true;
    if (i == nx + 1 && noslip[1]) return true;
    if (j == 0 && noslip[2]) return true;
    if (j == ny + 1 && noslip[3]) return true;
    const bool interior = i >= 1 && i <= nx && j >= 1 && j <= ny;
    return interior && !fluid[(size_t)i * (ny + 2) + j];
}

struct WallArgs {
    const uint8_t* fluid;
    int nx, ny;
    int periodic;
    int noslip[4];     // left, right, bottom, top
    double dx, dy;
    int* off;          // (nx+2)(ny+2) signed x offset to the row's nearest wall, kNoWall if none
    int* any;          // set to 1 when the grid has a wall
    double* dist;      // (nx+2)(ny+2) output
};

// Pass 1: row j, nearest wall cell in x. Non-periodic rows are i = 0..nx+1 of the
// padded grid; periodic rows are the columns 1..nx on a circle (three copies side
// by side reach every column's nearest periodic image).
__global__ void __launch_bounds__(kRowThreads) k_wall_rows(WallArgs A) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = A.nx, ny = A.ny;
    if (j >= ny + 2) return;
    const size_t stride = (size_t)ny + 2;
    const int lo = A.periodic ? 1 : 0;
    const int hi = A.periodic ? nx : nx + 1;
    const int n = hi - lo + 1;
    int first = -1, last = -1;
    for (int i = lo; i <= hi; ++i) {
        if (is_wall(A.fluid, A.noslip, nx, ny, i, j)) {
            if (first < 0) first = i;
            last = i;
        }
    }
    if (first < 0) {
        for (int i = lo; i <= hi; ++i) A.off[i * stride + j] = kNoWall;
        return;
    }
    atomicOr(A.any, 1);
    // forward: offset to the nearest wall at or before i (periodic: wrapped image of the last wall)
    int prev = A.periodic ? last - n : INT_MIN / 2;
    for (int i = lo; i <= hi; ++i) {
        if (is_wall(A.fluid, A.noslip, nx, ny, i, j)) prev = i;
        A.off[i * stride + j] = prev == INT_MIN / 2 ? kNoWall : prev - i;
    }
    // backward: keep the nearer of that and the nearest wall at or after i
    int next = A.periodic ? first + n : INT_MAX / 2;
    for (int i = hi; i >= lo; --i) {
        if (is_wall(A.fluid, A.noslip, nx, ny, i, j)) next = i;
        if (next == INT_MAX / 2) continue;
        const int o = A.off[i * stride + j];
        const int fwd = next - i;
        if (o == kNoWall || fwd < -o) A.off[i * stride + j] = fwd;
    }
}

__device__ __forceinline__ double sq_dist(int ox, int oy, double dx, double dy) {
    const double a = (double)ox * dx;
    const double b = (double)oy * dy;
    return a * a + b * b;
}

// Pass 2: per cell, the nearest wall over all rows, then the shift from the wall
// cell's centre to its face and the zero on non-fluid cells (turbulence.py:66-69).
__global__ void __launch_bounds__(kCellTX * kCellTY) k_wall_cells(WallArgs A) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = A.nx, ny = A.ny;
    if (j >= ny + 2 || i >= nx + 2) return;
    const size_t stride = (size_t)ny + 2;
    const size_t c = (size_t)i * stride + j;
    if (!*A.any) {  // no wall at all: 1e6 everywhere (turbulence.py:50-51)
        A.dist[c] = 1e6;
        return;
    }
    // periodic ghost columns take the values of the opposite columns (turbulence.py:60-61)
    const int si = A.periodic ? (i == 0 ? nx : (i == nx + 1 ? 1 : i)) : i;
    const int* row = A.off + (size_t)si * stride;
    double best = __longlong_as_double(0x7ff0000000000000LL);  // +inf
    for (int k = 0;; ++k) {
        const double b = (double)k * A.dy;
        if (b * b > best) break;
        const int up = j + k, dn = j - k;
        if (up > ny + 1 && dn < 0) break;
        if (up <= ny + 1) {
            const int o = row[up];
            if (o != kNoWall) best = fmin(best, sq_dist(o, k, A.dx, A.dy));
        }
        if (k > 0 && dn >= 0) {
            const int o = row[dn];
            if (o != kNoWall) best = fmin(best, sq_dist(o, -k, A.dx, A.dy));
        }
    }
    const double half = 0.5 * fmin(A.dx, A.dy);
    double d = sqrt(best) - half;
    d = d > half ? d : half;
    A.dist[c] = A.fluid[c] ? d : 0.0;
}

}  // namespace
}  // namespace cfd

extern "C" size_t cfd2d_wall_distance_workspace_bytes(int nx, int ny) {
    if (nx < 1 || ny < 1) return 0;
    return ((size_t)(nx + 2) * (ny + 2) + 4) * sizeof(int);
}

extern "C" int cfd2d_sim_wall_distance(const cfd2d_sim* sim, double* dist, void* work, size_t work_bytes,
                                       void* stream) {
    using namespace cfd;
    if (!sim || !dist || !work || !sim->fluid || sim->nx < 1 || sim->ny < 1) return CFD2D_E_ARG;
    if (work_bytes < cfd2d_wall_distance_workspace_bytes(sim->nx, sim->ny)) return CFD2D_E_ARG;
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    WallArgs A;
    A.fluid = sim->fluid;
    A.nx = sim->nx;
    A.ny = sim->ny;
    A.periodic = sim->periodic ? 1 : 0;
    for (int k = 0; k < 4; ++k) A.noslip[k] = sim->bc_kind[k] == CFD2D_BC_NOSLIP;
    A.dx = sim->dx;
    A.dy = sim->dy;
    A.any = static_cast<int*>(work);
    A.off = static_cast<int*>(work) + 4;
    A.dist = dist;
    if (cudaMemsetAsync(A.any, 0, sizeof(int), s) != cudaSuccess) return CFD2D_E_CUDA;
    k_wall_rows<<<(A.ny + 2 + kRowThreads - 1) / kRowThreads, kRowThreads, 0, s>>>(A);
    const dim3 blk(kCellTX, kCellTY);
    const dim3 grd((A.ny + 2 + kCellTX - 1) / kCellTX, (A.nx + 2 + kCellTY - 1) / kCellTY);
    k_wall_cells<<<grd, blk, 0, s>>>(A);
    return cudaGetLastError() == cudaSuccess ? CFD2D_OK : CFD2D_E_CUDA;
}
