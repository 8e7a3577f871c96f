// functions.cu - function objects fed from the device fields (cfd2d/functions.py).
//
// Probes, line samples, time averages and the VTK export of the reference read
// whole fields on the host after every step. Here they read the device fields:
//
//  * cfd2d_sample / cfd2d_probe_record: bilinear interpolation at a few points
//    (cfd2d/functions.py:24-39, cfd2d/solver.py:598-615). The cell value a
//    corner needs (pressure, cell velocity, speed, vorticity, a scalar) is formed
//    on the fly from the staggered fields, so a probe costs O(points), not a pass
//    over the grid. The arithmetic is scipy's RegularGridInterpolator(linear):
//    the cell index is the number of grid coordinates <= x minus one, clamped to
//    the grid, t = (x - x_i) / (x_{i+1} - x_i), and the four corners are added as
//    v00 (1-tx)(1-ty) + v01 (1-tx) ty + v10 tx (1-ty) + v11 tx ty, left to right.
//  * cfd2d_field_average_accumulate: the sums of cfd2d/functions.py:189-204 for
//    every cell, one pass per step.
//  * cfd2d_streamfunction: the running sums of cfd2d/solver.py:580-596, in order.
//  * cfd2d_vtk_pack: the VTK payload as big-endian float32 in VTK cell order.
//
// The recorders read t, dt and n from the simulation's state on the device and
// skip a call when no step ran since their last one, so they can be queued after
// every step without a host synchronisation.

#include <cstdint>

#include "../../include/cfd2d_b200.h"

namespace cfd {
namespace {

constexpr int kThreads = 256;

struct FieldSet {
    cfd2d_field f[CFD2D_MAX_FIELDS];
    int n;
};

__device__ __forceinline__ double qnan() { return __longlong_as_double(0x7ff8000000000000LL); }

// numpy.maximum: NaN if either operand is NaN
__device__ __forceinline__ double np_maximum(double a, double b) {
    if (a != a) return a;
    if (b != b) return b;
    return a > b ? a : b;
}

__device__ __forceinline__ double cell_u(const cfd2d_sim& S, int i, int j) {
    // 0.5 (u[i, j+1] + u[i+1, j+1]) (cfd2d/solver.py:528)
    const int ny = S.ny;
    return 0.5 * (S.u[(size_t)i * (ny + 2) + j + 1] + S.u[(size_t)(i + 1) * (ny + 2) + j + 1]);
}

__device__ __forceinline__ double cell_v(const cfd2d_sim& S, int i, int j) {
    // 0.5 (v[i+1, j] + v[i+1, j+1]) (cfd2d/solver.py:529)
    const int ny = S.ny;
    const size_t r = (size_t)(i + 1) * (ny + 1);
    return 0.5 * (S.v[r + j] + S.v[r + j + 1]);
}

// node vorticity dv/dx - du/dy at node (a, b), a in 0..nx, b in 0..ny (cfd2d/solver.py:569-573)
__device__ __forceinline__ double node_w(const cfd2d_sim& S, int a, int b) {
    const int ny = S.ny;
    const double dvdx = (S.v[(size_t)(a + 1) * (ny + 1) + b] - S.v[(size_t)a * (ny + 1) + b]) / S.dx;
    const double dudy = (S.u[(size_t)a * (ny + 2) + b + 1] - S.u[(size_t)a * (ny + 2) + b]) / S.dy;
    return dvdx - dudy;
}

// value of field F in interior cell (i, j), 0-based (cfd2d/visualization.py:50-73)
__device__ double cell_value(const cfd2d_sim& S, const cfd2d_field& F, int i, int j) {
    const int ny = S.ny;
    const size_t pc = (size_t)(i + 1) * (ny + 2) + (j + 1);
    const bool fluid = S.fluid[pc] != 0;
    if (F.kind == CFD2D_FIELD_FLUID) return fluid ? 1.0 : 0.0;
    if (!fluid) return qnan();
    switch (F.kind) {
        case CFD2D_FIELD_PRESSURE: return S.p[pc];
        case CFD2D_FIELD_UC: return cell_u(S, i, j);
        case CFD2D_FIELD_VC: return cell_v(S, i, j);
        case CFD2D_FIELD_SPEED: {
            const double a = cell_u(S, i, j), b = cell_v(S, i, j);
            return sqrt(a * a + b * b);
        }
        case CFD2D_FIELD_VORTICITY:
            return 0.25 * (((node_w(S, i, j) + node_w(S, i + 1, j)) + node_w(S, i, j + 1)) + node_w(S, i + 1, j + 1));
        case CFD2D_FIELD_CELL: return F.data[pc];
        case CFD2D_FIELD_CELL_LOG10: return log10(np_maximum(F.data[pc], 1e-30));
        case CFD2D_FIELD_NODE: {
            const double* d = F.data;
            const size_t r0 = (size_t)i * (ny + 1), r1 = (size_t)(i + 1) * (ny + 1);
            return 0.25 * (((d[r0 + j] + d[r1 + j]) + d[r0 + j + 1]) + d[r1 + j + 1]);
        }
        default: return qnan();
    }
}

// One axis of a sampling grid: n coordinates (k + off) h, k = 0..n-1.
struct Axis {
    int n;
    double off, h;
    __device__ __forceinline__ double at(int k) const { return ((double)k + off) * h; }
    // number of coordinates <= x, minus one, clamped to 0..n-2
    __device__ __forceinline__ int cell(double x) const {
        double kd = floor(x / h - off);
        kd = fmin(fmax(kd, -1.0), (double)(n - 1));
        int k = (int)kd;
        while (k + 1 <= n - 1 && at(k + 1) <= x) ++k;
        while (k >= 0 && at(k) > x) --k;
        return k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
    }
};

__device__ double sample_at(const cfd2d_sim& S, const cfd2d_field& F, double x, double y) {
    const int nx = S.nx, ny = S.ny;
    Axis ax, ay;
    const bool face_u = F.kind == CFD2D_FIELD_U, face_v = F.kind == CFD2D_FIELD_V;
    if (face_u) {
        ax = {nx + 1, 0.0, S.dx};
        ay = {ny + 2, -0.5, S.dy};
    } else if (face_v) {
        ax = {nx + 2, -0.5, S.dx};
        ay = {ny + 1, 0.0, S.dy};
    } else {
        ax = {nx, 0.5, S.dx};
        ay = {ny, 0.5, S.dy};
        // np.clip(x, xc[0], xc[-1]) = minimum(maximum(x, lo), hi)
        x = fmin(fmax(x, ax.at(0)), ax.at(nx - 1));
        y = fmin(fmax(y, ay.at(0)), ay.at(ny - 1));
    }
    const int i = ax.cell(x), j = ay.cell(y);
    const double tx = (x - ax.at(i)) / (ax.at(i + 1) - ax.at(i));
    const double ty = (y - ay.at(j)) / (ay.at(j + 1) - ay.at(j));
    double v00, v01, v10, v11;
    if (face_u || face_v) {
        const double* d = face_u ? S.u : S.v;
        const size_t st = face_u ? (size_t)ny + 2 : (size_t)ny + 1;
        v00 = d[(size_t)i * st + j];
        v01 = d[(size_t)i * st + j + 1];
        v10 = d[(size_t)(i + 1) * st + j];
        v11 = d[(size_t)(i + 1) * st + j + 1];
    } else {
        v00 = cell_value(S, F, i, j);
        v01 = cell_value(S, F, i, j + 1);
        v10 = cell_value(S, F, i + 1, j);
        v11 = cell_value(S, F, i + 1, j + 1);
    }
    const double sx = 1 - tx, sy = 1 - ty;
    return v00 * sx * sy + v01 * sx * ty + v10 * tx * sy + v11 * tx * ty;
}

__global__ void __launch_bounds__(kThreads) k_sample(cfd2d_sim S, FieldSet FS, const double* px,
                                                     const double* py, int npts, double* out) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long long)FS.n * npts) return;
    const int f = (int)(k / npts), q = (int)(k % npts);
    out[k] = sample_at(S, FS.f[f], px[q], py[q]);
}

__global__ void __launch_bounds__(kThreads) k_cell_values(cfd2d_sim S, cfd2d_field F, double* out) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)S.nx * S.ny) return;
    out[c] = cell_value(S, F, (int)(c / S.ny), (int)(c % S.ny));
}

// One block: thread 0 decides, every thread samples, thread 0 commits the row.
__global__ void __launch_bounds__(kThreads) k_probe_record(cfd2d_sim S, FieldSet FS, const double* px,
                                                           const double* py, int npts,
                                                           cfd2d_probe_series P) {
    __shared__ long long row;
    const cfd2d_state* st = S.state;
    const long long n = st->n;
    if (threadIdx.x == 0) {
        row = -1;
        if (n != P.count[1] && n % P.every == 0) {
            if (P.count[0] < P.cap) row = P.count[0];
            else P.count[2] = 1;
        }
    }
    __syncthreads();
    if (row < 0) return;
    const int total = FS.n * npts;
    double* dst = P.values + (size_t)row * total;
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int f = k / npts, q = k % npts;
        dst[k] = sample_at(S, FS.f[f], px[q], py[q]);
    }
    if (threadIdx.x == 0) {
        P.t[row] = st->t;
        P.count[0] = row + 1;
        P.count[1] = n;
    }
}

__device__ __forceinline__ bool average_due(const cfd2d_state* st, const cfd2d_field_average& A) {
    return !(st->t < A.t_start) && (double)st->n != A.T[1];
}

// cfd2d/functions.py:189-204: sum += a dt, sum2 += a a dt for a = uc, vc, p
__global__ void __launch_bounds__(kThreads) k_average_cells(cfd2d_sim S, cfd2d_field_average A) {
    const cfd2d_state* st = S.state;
    if (!average_due(st, A)) return;
    const int nx = S.nx, ny = S.ny;
    const int j = blockIdx.x * 32 + (threadIdx.x & 31);
    const int i = blockIdx.y * (kThreads / 32) + (threadIdx.x >> 5);
    if (i >= nx || j >= ny) return;
    const size_t N = (size_t)nx * ny, c = (size_t)i * ny + j;
    const double dt = st->dt;
    const bool fluid = S.fluid[(size_t)(i + 1) * (ny + 2) + j + 1] != 0;
    double a[3];
    a[0] = fluid ? cell_u(S, i, j) : qnan();
    a[1] = fluid ? cell_v(S, i, j) : qnan();
    a[2] = fluid ? S.p[(size_t)(i + 1) * (ny + 2) + j + 1] : qnan();
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        A.sum[k * N + c] = A.sum[k * N + c] + a[k] * dt;
        A.sum2[k * N + c] = A.sum2[k * N + c] + a[k] * a[k] * dt;
    }
}

__global__ void k_average_time(cfd2d_sim S, cfd2d_field_average A) {
    const cfd2d_state* st = S.state;
    if (!average_due(st, A)) return;
    A.T[0] = A.T[0] + st->dt;
    A.T[1] = (double)st->n;
}

// psi[a+1, 0] = -cumsum(v0)[a] dx along the bottom row (cfd2d/solver.py:590-593)
__global__ void k_psi_bottom(cfd2d_sim S, double* psi) {
    const int nx = S.nx, ny = S.ny;
    double acc = 0.0;
    psi[0] = 0.0;
    for (int a = 0; a < nx; ++a) {
        const size_t c0 = (size_t)(a + 1) * (ny + 2);
        const bool open = S.fluid[c0] || S.fluid[c0 + 1];
        acc = acc + (open ? S.v[(size_t)(a + 1) * (ny + 1)] : 0.0);
        psi[(size_t)(a + 1) * (ny + 1)] = -acc * S.dx;
    }
}

// psi[a, b+1] = psi[a, 0] + cumsum(u[a, 1:-1] on open faces)[b] dy (cfd2d/solver.py:594-595)
__global__ void __launch_bounds__(kThreads) k_psi_columns(cfd2d_sim S, double* psi) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = S.nx, ny = S.ny;
    if (a > nx) return;
    const double base = psi[(size_t)a * (ny + 1)];
    double acc = 0.0;
    for (int b = 0; b < ny; ++b) {
        const bool open = S.fluid[(size_t)a * (ny + 2) + b + 1] || S.fluid[(size_t)(a + 1) * (ny + 2) + b + 1];
        acc = acc + (open ? S.u[(size_t)a * (ny + 2) + b + 1] : 0.0);
        psi[(size_t)a * (ny + 1) + b + 1] = base + acc * S.dy;
    }
}

// big-endian float32 of x, NaN as 0 (np.nan_to_num(x, nan=0.0).astype(">f4"))
__device__ __forceinline__ uint32_t be_f32(double x) {
    if (x != x) x = 0.0;
    const uint32_t b = __float_as_uint(__double2float_rn(x));
    return __byte_perm(b, 0, 0x0123);
}

// VTK cell order: x fastest, cell index q = j nx + i
__global__ void __launch_bounds__(kThreads) k_vtk_pack(cfd2d_sim S, FieldSet FS, uint32_t* out) {
    const int nx = S.nx, ny = S.ny;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long N = (long long)nx * ny;
    if (q >= N) return;
    const int i = (int)(q % nx), j = (int)(q / nx);
    const bool fluid = S.fluid[(size_t)(i + 1) * (ny + 2) + j + 1] != 0;
    out[3 * q] = be_f32(fluid ? cell_u(S, i, j) : qnan());
    out[3 * q + 1] = be_f32(fluid ? cell_v(S, i, j) : qnan());
    out[3 * q + 2] = be_f32(0.0);
    for (int f = 0; f < FS.n; ++f) out[3 * N + f * N + q] = be_f32(cell_value(S, FS.f[f], i, j));
}

int load_fields(const cfd2d_field* fields, int nfields, FieldSet* fs) {
    if (nfields < 0 || nfields > CFD2D_MAX_FIELDS || (nfields > 0 && !fields)) return CFD2D_E_ARG;
    fs->n = nfields;
    for (int k = 0; k < nfields; ++k) {
        const int kind = fields[k].kind;
        if (kind < CFD2D_FIELD_U || kind > CFD2D_FIELD_FLUID) return CFD2D_E_ARG;
        const bool needs_data =
            kind == CFD2D_FIELD_CELL || kind == CFD2D_FIELD_CELL_LOG10 || kind == CFD2D_FIELD_NODE;
        if (needs_data && !fields[k].data) return CFD2D_E_ARG;
        fs->f[k] = fields[k];
    }
    return CFD2D_OK;
}

bool sim_ok(const cfd2d_sim* sim) {
    return sim && sim->nx >= 4 && sim->ny >= 4 && sim->u && sim->v && sim->p && sim->fluid && sim->state;
}

int launched() { return cudaGetLastError() == cudaSuccess ? CFD2D_OK : CFD2D_E_CUDA; }

}  // namespace
}  // namespace cfd

using namespace cfd;

extern "C" int cfd2d_sample(const cfd2d_sim* sim, const cfd2d_field* fields, int nfields, const double* px,
                            const double* py, int npts, double* out, void* stream) {
    FieldSet fs;
    if (!sim_ok(sim) || npts < 0) return CFD2D_E_ARG;
    if (const int rc = load_fields(fields, nfields, &fs)) return rc;
    const long long total = (long long)nfields * npts;
    if (total == 0) return CFD2D_OK;
    if (!px || !py || !out) return CFD2D_E_ARG;
    const unsigned blocks = (unsigned)((total + kThreads - 1) / kThreads);
    k_sample<<<blocks, kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(*sim, fs, px, py, npts, out);
    return launched();
}

extern "C" int cfd2d_cell_values(const cfd2d_sim* sim, const cfd2d_field* field, double* out, void* stream) {
    FieldSet fs;
    if (!sim_ok(sim) || !out) return CFD2D_E_ARG;
    if (const int rc = load_fields(field, 1, &fs)) return rc;
    const long long N = (long long)sim->nx * sim->ny;
    k_cell_values<<<(unsigned)((N + kThreads - 1) / kThreads), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        *sim, fs.f[0], out);
    return launched();
}

extern "C" int cfd2d_probe_record(const cfd2d_sim* sim, const cfd2d_field* fields, int nfields, const double* px,
                                  const double* py, int npts, const cfd2d_probe_series* series, void* stream) {
    FieldSet fs;
    if (!sim_ok(sim) || npts < 1 || !px || !py || !series) return CFD2D_E_ARG;
    if (const int rc = load_fields(fields, nfields, &fs)) return rc;
    if (nfields < 1 || !series->t || !series->values || !series->count || series->cap < 0 || series->every < 1)
        return CFD2D_E_ARG;
    k_probe_record<<<1, kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(*sim, fs, px, py, npts, *series);
    return launched();
}

extern "C" int cfd2d_field_average_accumulate(const cfd2d_sim* sim, const cfd2d_field_average* avg, void* stream) {
    if (!sim_ok(sim) || !avg || !avg->sum || !avg->sum2 || !avg->T) return CFD2D_E_ARG;
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const dim3 grd((sim->ny + 31) / 32, (sim->nx + kThreads / 32 - 1) / (kThreads / 32));
    k_average_cells<<<grd, kThreads, 0, s>>>(*sim, *avg);
    k_average_time<<<1, 1, 0, s>>>(*sim, *avg);
    return launched();
}

extern "C" int cfd2d_streamfunction(const cfd2d_sim* sim, double* psi, void* stream) {
    if (!sim_ok(sim) || !psi) return CFD2D_E_ARG;
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    k_psi_bottom<<<1, 1, 0, s>>>(*sim, psi);
    k_psi_columns<<<(sim->nx + 1 + kThreads - 1) / kThreads, kThreads, 0, s>>>(*sim, psi);
    return launched();
}

extern "C" int cfd2d_vtk_pack(const cfd2d_sim* sim, const cfd2d_field* fields, int nfields, uint8_t* out,
                              void* stream) {
    FieldSet fs;
    if (!sim_ok(sim) || !out || (reinterpret_cast<uintptr_t>(out) & 3)) return CFD2D_E_ARG;
    if (const int rc = load_fields(fields, nfields, &fs)) return rc;
    const long long N = (long long)sim->nx * sim->ny;
    const unsigned blocks = (unsigned)((N + kThreads - 1) / kThreads);
    k_vtk_pack<<<blocks, kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(*sim, fs,
                                                                                reinterpret_cast<uint32_t*>(out));
    return launched();
}
