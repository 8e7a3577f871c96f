// vof.cu - two-phase VOF on the device (cfd2d/vof.py, the variable-density parts of
// cfd2d/solver.py and cfd2d/pressure.py:187-244).
//
// Per step: the CSF curvature before the momentum update (smoothed alpha, node
// normals, cell curvature; the face force itself is added inside the predictor),
// the face coefficients b = 2 / (rho_L + rho_R) and the diagonal of the
// variable-coefficient operator before the pressure solve, and after the projection
// the alpha transport in sub-steps at the alpha Courant number, each followed by the
// ghost/solid fill, then the mixture density and viscosity.
//
// The transport is a gather: every cell adds the terms of its four faces in the
// order in which the reference's face loops reach it (west, east, south, north; with
// periodic x the wrapped face nx reaches cell 1 after its east face), each face term
// formed exactly as the reference forms it, so the result is bit-identical.

#include <cuda_runtime.h>
#include <math.h>

#include "device.cuh"
#include "kernels.cuh"

namespace cfd {
namespace {

constexpr int kTX = 32, kTY = 8;

__device__ __forceinline__ bool active(const cfd2d_state* st) { return st == nullptr || st->active != 0; }

dim3 tiles(int rows_j, int cols_i) { return dim3((rows_j + kTX - 1) / kTX, (cols_i + kTY - 1) / kTY); }

// cfd2d/vof.py:23-33: van Leer face value, first order without an upwind cell
__device__ __forceinline__ double vl_face(double a_up, double a_c, double a_d, bool has_up) {
    if (!has_up) return a_c;
    const double den = a_d - a_c;
    if (fabs(den) < 1e-300) return a_c;
    const double r = (a_c - a_up) / den;
    const double lim = (r <= 0.0) ? 0.0 : (2.0 * r) / (1.0 + r);
    return a_c + (0.5 * lim) * den;
}

// Flux through a face from its low cell to its high cell (cfd2d/vof.py:72-88, 113-124):
// bounded advection plus interface compression u_r a_c (1 - a_d).
__device__ __forceinline__ double face_flux(double vel, double a_lo, double a_hi, double a_up, bool has_up,
                                            double g_n, double g_t, double c_alpha) {
    const double af = (vel >= 0.0) ? vl_face(a_up, a_lo, a_hi, has_up) : vl_face(a_up, a_hi, a_lo, has_up);
    double flux = vel * af;
    const double gm = sqrt(g_n * g_n + g_t * g_t);
    if (gm > 1e-12 && c_alpha > 0.0) {
        const double ur = ((c_alpha * fabs(vel)) * g_n) / gm;
        const double ac = (ur >= 0.0) ? a_lo : a_hi;
        const double ad = (ur >= 0.0) ? a_hi : a_lo;
        flux = flux + (ur * ac) * (1.0 - ad);
    }
    return flux;
}

struct AdvectArgs {
    const double* a;
    const double* u;
    const double* v;
    const uint8_t* fl;
    int nx, ny, periodic;
    double dx, dy, c_alpha, a_in;
};

// flux of interior x face f (cells L = f and R = f + 1, or R = 1 for the periodic face nx)
__device__ double x_face_flux(const AdvectArgs& A, int f, int j) {
    const int nx = A.nx, ny = A.ny, pc = ny + 2;
    const int L = f, R = (f < nx) ? f + 1 : 1;
    const double uf = A.u[f * pc + j];
    int up;
    if (uf >= 0.0) up = (L - 1 >= 1) ? L - 1 : (A.periodic ? nx : -1);
    else up = (R + 1 <= nx) ? R + 1 : (A.periodic ? 1 : -1);
    const bool has_up = up >= 1 && A.fl[up * pc + j];
    const double gx = (A.a[R * pc + j] - A.a[L * pc + j]) / A.dx;
    const int jn = (j < ny) ? j + 1 : j, js = (j > 1) ? j - 1 : j;
    const double gy = (0.25 * ((A.a[L * pc + jn] - A.a[L * pc + js]) + (A.a[R * pc + jn] - A.a[R * pc + js]))) / A.dy;
    return face_flux(uf, A.a[L * pc + j], A.a[R * pc + j], has_up ? A.a[up * pc + j] : 0.0, has_up, gx, gy,
                     A.c_alpha);
}

// flux of interior y face f (cells B = f, T = f + 1) in column i
__device__ double y_face_flux(const AdvectArgs& A, int i, int f) {
    const int nx = A.nx, ny = A.ny, pc = ny + 2;
    const int B = f, T = f + 1;
    const double vf = A.v[i * (ny + 1) + f];
    const int up = (vf >= 0.0) ? B - 1 : T + 1;
    const bool has_up = up >= 1 && up <= ny && A.fl[i * pc + up];
    const double gy = (A.a[i * pc + T] - A.a[i * pc + B]) / A.dy;
    int ie = (i < nx || A.periodic) ? i + 1 : i;
    int iw = (i > 1 || A.periodic) ? i - 1 : i;
    if (ie > nx) ie = 1;
    if (iw < 1) iw = nx;
    const double gx = (0.25 * ((A.a[ie * pc + B] - A.a[iw * pc + B]) + (A.a[ie * pc + T] - A.a[iw * pc + T]))) / A.dx;
    return face_flux(vf, A.a[i * pc + B], A.a[i * pc + T], has_up ? A.a[i * pc + up] : 0.0, has_up, gy, gx,
                     A.c_alpha);
}

// inflow/outflow term of a boundary face: dt * into * a_b / h (cfd2d/vof.py:51-60)
__device__ __forceinline__ double open_term(double into, double a_in, double a_cell, double dt, double h) {
    const double ab = (into > 0) ? a_in : a_cell;
    return ((dt * into) * ab) / h;
}

__device__ double advect_cell(const AdvectArgs& A, double dt, int i, int j) {
    const int nx = A.nx, ny = A.ny, pc = ny + 2;
    const int c = i * pc + j;
    double val = A.a[c];
    if (!A.fl[c]) return val;
    const double dx = A.dx, dy = A.dy;
    // west face i - 1
    if (i == 1) {
        if (!A.periodic) val = val + open_term(A.u[j], A.a_in, A.a[c], dt, dx);
    } else if (A.fl[(i - 1) * pc + j]) {
        val = val + (dt * x_face_flux(A, i - 1, j)) / dx;
    }
    // east face i
    if (i == nx && !A.periodic) {
        val = val + open_term(-A.u[nx * pc + j], A.a_in, A.a[c], dt, dx);
    } else {
        const int R = (i < nx) ? i + 1 : 1;
        if (A.fl[R * pc + j]) val = val - (dt * x_face_flux(A, i, j)) / dx;
    }
    // periodic face nx reaches cell 1 last
    if (A.periodic && i == 1 && A.fl[nx * pc + j]) val = val + (dt * x_face_flux(A, nx, j)) / dx;
    // south face j - 1
    if (j == 1) {
        val = val + open_term(A.v[i * (ny + 1)], A.a_in, A.a[c], dt, dy);
    } else if (A.fl[c - 1]) {
        val = val + (dt * y_face_flux(A, i, j - 1)) / dy;
    }
    // north face j
    if (j == ny) {
        val = val + open_term(-A.v[i * (ny + 1) + ny], A.a_in, A.a[c], dt, dy);
    } else if (A.fl[c + 1]) {
        val = val - (dt * y_face_flux(A, i, j)) / dy;
    }
    if (val < 0.0) val = 0.0;
    else if (val > 1.0) val = 1.0;
    return val;
}

__global__ void __launch_bounds__(kTX * kTY) k_vof_advect(cfd2d_sim S, int k, double h_const, double* out) {
    if (!active(S.state)) return;
    const cfd2d_vof& V = S.vof;
    double h = h_const;
    if (k >= 0) {
        if ((double)k >= V.scal[1]) return;
        h = V.scal[2];
    }
    const int nx = S.nx, ny = S.ny;
    const int j = blockIdx.x * kTX + threadIdx.x;
    const int i = blockIdx.y * kTY + threadIdx.y;
    if (i >= nx + 2 || j >= ny + 2) return;
    const int c = i * (ny + 2) + j;
    AdvectArgs A{V.alpha, S.u, S.v, S.fluid, nx, ny, S.periodic, S.dx, S.dy, V.c_alpha, V.alpha_in};
    const bool interior = i >= 1 && i <= nx && j >= 1 && j <= ny;
    out[c] = interior ? advect_cell(A, h, i, j) : V.alpha[c];
}

// alpha from the transported field: side ghosts copy (periodic x wraps) the cell
// values before the solid fill, solid cells take the mean of their fluid
// neighbours (cfd2d/vof.py:200-220)
__global__ void __launch_bounds__(kTX * kTY) k_vof_ghosts(cfd2d_sim S, int k, const double* src, double* dst) {
    if (!active(S.state)) return;
    const cfd2d_vof& V = S.vof;
    if (k >= 0 && (double)k >= V.scal[1]) return;
    const int nx = S.nx, ny = S.ny, pc = ny + 2;
    const int j = blockIdx.x * kTX + threadIdx.x;
    const int i = blockIdx.y * kTY + threadIdx.y;
    if (i >= nx + 2 || j >= ny + 2) return;
    const int c = i * pc + j;
    const bool interior = i >= 1 && i <= nx && j >= 1 && j <= ny;
    if (!interior) {
        int si = i, sj = j;
        if (i == 0) si = S.periodic ? nx : 1;
        if (i == nx + 1) si = S.periodic ? 1 : nx;
        if (j == 0) sj = 1;
        if (j == ny + 1) sj = ny;
        dst[c] = src[si * pc + sj];
        return;
    }
    if (S.fluid[c]) {
        dst[c] = src[c];
        return;
    }
    // neighbour values after the side copies: periodic ghost columns hold columns nx and 1
    auto nb_val = [&](int ii, int jj) {
        int si = ii;
        if (ii == 0) si = S.periodic ? nx : 1;
        if (ii == nx + 1) si = S.periodic ? 1 : nx;
        int sj = jj < 1 ? 1 : (jj > ny ? ny : jj);
        return src[si * pc + sj];
    };
    const int nbs[4][2] = {{i + 1, j}, {i - 1, j}, {i, j + 1}, {i, j - 1}};
    double s = 0.0, cnt = 0.0;
    for (int q = 0; q < 4; ++q) {
        const bool f = S.fluid[nbs[q][0] * pc + nbs[q][1]] != 0;
        s = s + (f ? nb_val(nbs[q][0], nbs[q][1]) : 0.0);
    }
    for (int q = 0; q < 4; ++q) cnt = cnt + (S.fluid[nbs[q][0] * pc + nbs[q][1]] ? 1.0 : 0.0);
    dst[c] = (cnt > 0) ? s / (cnt > 1.0 ? cnt : 1.0) : 0.0;
}

// mixture density and dynamic viscosity (cfd2d/vof.py:222-227)
__global__ void k_vof_props(cfd2d_sim S) {
    if (!active(S.state)) return;
    const cfd2d_vof& V = S.vof;
    const int n = (S.nx + 2) * (S.ny + 2);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const double a = V.alpha[c];
        V.rho[c] = a * V.rho1 + (1 - a) * V.rho2;
        S.nu_eff[c] = a * V.mu1 + (1 - a) * V.mu2;
    }
}

// sub-step count and length from the corrected velocities (cfd2d/vof.py:262-265)
__global__ void __launch_bounds__(1024) k_vof_nsub(cfd2d_sim S) {
    cfd2d_state* st = S.state;
    if (!active(st)) return;
    const int nu = (S.nx + 1) * (S.ny + 2), nv = (S.nx + 2) * (S.ny + 1);
    double m[2] = {0.0, 0.0};
    for (int c = threadIdx.x; c < nu; c += blockDim.x) m[0] = npmax(m[0], fabs(S.u[c]));
    for (int c = threadIdx.x; c < nv; c += blockDim.x) m[1] = npmax(m[1], fabs(S.v[c]));
    __shared__ double sred[32 * 2];
    block_max<2>(m, sred);
    if (threadIdx.x != 0) return;
    const cfd2d_vof& V = S.vof;
    const double dt = st->dt;
    double um = m[0] / S.dx;
    const double vm = m[1] / S.dy;
    if (vm > um) um = vm;
    if (1e-12 > um) um = 1e-12;
    double ns = ceil((dt * um) / V.cfl);
    if (ns < 1.0) ns = 1.0;
    if (ns > (double)V.nsub_max) {
        atomicOr(&st->status, CFD2D_S_VOF_SUBSTEPS);
        ns = (double)V.nsub_max;
    }
    V.scal[1] = ns;
    V.scal[2] = dt / ns;
}

// ---------------------------------------------------------------- CSF curvature
// cfd2d/vof.py:240-249: smoothed alpha, unit normals at the nodes, kappa = -div(n)
__global__ void __launch_bounds__(kTX * kTY) k_csf_smooth(cfd2d_sim S) {
    if (!active(S.state)) return;
    const cfd2d_vof& V = S.vof;
    const int nx = S.nx, ny = S.ny, pc = ny + 2;
    const int j = blockIdx.x * kTX + threadIdx.x;
    const int i = blockIdx.y * kTY + threadIdx.y;
    if (i >= nx + 2 || j >= ny + 2) return;
    const int c = i * pc + j;
    const double* a = V.alpha;
    const bool interior = i >= 1 && i <= nx && j >= 1 && j <= ny;
    V.smooth[c] = interior ? ((((4 * a[c] + a[c + pc]) + a[c - pc]) + a[c + 1]) + a[c - 1]) / 8.0 : a[c];
}

__global__ void __launch_bounds__(kTX * kTY) k_csf_normals(cfd2d_sim S) {
    if (!active(S.state)) return;
    const cfd2d_vof& V = S.vof;
    const int nx = S.nx, ny = S.ny, pc = ny + 2, pn = ny + 1;
    const int b = blockIdx.x * kTX + threadIdx.x;
    const int a = blockIdx.y * kTY + threadIdx.y;
    if (a > nx || b > ny) return;
    const double* As = V.smooth;
    const double gx = (0.5 * ((As[(a + 1) * pc + b + 1] - As[a * pc + b + 1]) + (As[(a + 1) * pc + b] - As[a * pc + b]))) / S.dx;
    const double gy = (0.5 * ((As[(a + 1) * pc + b + 1] - As[(a + 1) * pc + b]) + (As[a * pc + b + 1] - As[a * pc + b]))) / S.dy;
    const double gm = sqrt(gx * gx + gy * gy) + 1e-8 / S.dx;
    V.nrm[a * pn + b] = gx / gm;
    V.nrm[(nx + 1) * pn + a * pn + b] = gy / gm;
}

__global__ void __launch_bounds__(kTX * kTY) k_csf_kappa(cfd2d_sim S) {
    if (!active(S.state)) return;
    const cfd2d_vof& V = S.vof;
    const int nx = S.nx, ny = S.ny, pc = ny + 2, pn = ny + 1;
    const int j = blockIdx.x * kTX + threadIdx.x;
    const int i = blockIdx.y * kTY + threadIdx.y;
    if (i >= nx + 2 || j >= ny + 2) return;
    const bool interior = i >= 1 && i <= nx && j >= 1 && j <= ny;
    if (!interior) {
        V.kappa[i * pc + j] = 0.0;
        return;
    }
    const double* nX = V.nrm;
    const double* nY = V.nrm + (nx + 1) * pn;
    const double ddx = (0.5 * ((nX[i * pn + j] - nX[(i - 1) * pn + j]) + (nX[i * pn + j - 1] - nX[(i - 1) * pn + j - 1]))) / S.dx;
    const double ddy = (0.5 * ((nY[i * pn + j] - nY[i * pn + j - 1]) + (nY[(i - 1) * pn + j] - nY[(i - 1) * pn + j - 1]))) / S.dy;
    V.kappa[i * pc + j] = -(ddx + ddy);
}

// ---------------------------------------------------------------- variable-density operator
// face coefficients b = 2 / (rho_L + rho_R), periodic face nx between columns nx and 1
// (cfd2d/solver.py:267-271)
__global__ void __launch_bounds__(kTX * kTY) k_vof_faces(cfd2d_sim S) {
    if (!active(S.state)) return;
    const cfd2d_vof& V = S.vof;
    const int nx = S.nx, ny = S.ny, pc = ny + 2;
    const int j = blockIdx.x * kTX + threadIdx.x;
    const int i = blockIdx.y * kTY + threadIdx.y;
    if (i >= nx + 2 || j >= ny + 2) return;
    const double* rho = V.rho;
    if (i <= nx) {
        const int r = (S.periodic && i == nx) ? 1 : i + 1;
        V.bx[i * pc + j] = 2.0 / (rho[i * pc + j] + rho[r * pc + j]);
    }
    if (j <= ny) V.by[i * (ny + 1) + j] = 2.0 / (rho[i * pc + j] + rho[i * pc + j + 1]);
}

// largest x-face coefficient over rows 1..ny (the pin weight of cfd2d/pressure.py:227-228)
__global__ void __launch_bounds__(1024) k_vof_bmax(cfd2d_sim S) {
    if (!active(S.state)) return;
    const cfd2d_vof& V = S.vof;
    const int nx = S.nx, ny = S.ny;
    const int n = (nx + 1) * ny;
    double m[1] = {-INFINITY};
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const double b = V.bx[(q / ny) * (ny + 2) + (q % ny) + 1];
        if (b > m[0]) m[0] = b;
    }
    __shared__ double sred[32];
    block_max<1>(m, sred, -INFINITY);
    if (threadIdx.x == 0) V.scal[0] = m[0];
}

// diagonal in the reference's accumulation order (cfd2d/pressure.py:197-228): interior
// x pairs (east, then west face), y pairs (north, south), the periodic pair, the
// outflow sides, the pinned cells
__global__ void __launch_bounds__(256) k_vof_diag(cfd2d_sim S) {
    if (!active(S.state)) return;
    const cfd2d_vof& V = S.vof;
    const cfd2d_poisson& op = S.pcg;
    const int nx = S.nx, ny = S.ny, pc = ny + 2, pv = ny + 1;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nx * ny) return;
    const uint8_t nb = op.nbr[c];
    if (!(nb & 0x80)) {
        V.vdiag[c] = 0.0;
        V.vdinv[c] = 0.0;
        return;
    }
    const int i = c / ny, j = c % ny;
    const double dx2 = op.dx2, dy2 = op.dy2;
    double d = 0.0;
    if (i < nx - 1 && (nb & 8)) d += V.bx[(i + 1) * pc + j + 1] * dx2;
    if (i > 0 && (nb & 1)) d += V.bx[i * pc + j + 1] * dx2;
    if (nb & 4) d += V.by[(i + 1) * pv + j + 1] * dy2;
    if (nb & 2) d += V.by[(i + 1) * pv + j] * dy2;
    if (S.periodic) {
        if (i == nx - 1 && (nb & 8)) d += V.bx[nx * pc + j + 1] * dx2;
        if (i == 0 && (nb & 1)) d += V.bx[nx * pc + j + 1] * dx2;
    }
    const uint8_t fl = V.vflags[c];
    if (fl & 1) d += (2 * dx2) * V.bx[j + 1];
    if (fl & 2) d += (2 * dx2) * V.bx[nx * pc + j + 1];
    if (fl & 4) d += (2 * dy2) * V.by[(i + 1) * pv];
    if (fl & 8) d += (2 * dy2) * V.by[(i + 1) * pv + ny];
    if (fl & 16) d += dx2 * (V.scal[0] > 1e-30 ? V.scal[0] : 1e-30);
    V.vdiag[c] = d;
    V.vdinv[c] = 1.0 / d;
}

}  // namespace

cudaError_t stage_vof_curvature(const cfd2d_sim& S, cudaStream_t s) {
    if (!(S.vof.sigma > 0)) return cudaSuccess;
    k_csf_smooth<<<tiles(S.ny + 2, S.nx + 2), dim3(kTX, kTY), 0, s>>>(S);
    k_csf_normals<<<tiles(S.ny + 1, S.nx + 1), dim3(kTX, kTY), 0, s>>>(S);
    k_csf_kappa<<<tiles(S.ny + 2, S.nx + 2), dim3(kTX, kTY), 0, s>>>(S);
    return cudaGetLastError();
}

cudaError_t stage_vof_operator(const cfd2d_sim& S, cudaStream_t s) {
    k_vof_faces<<<tiles(S.ny + 2, S.nx + 2), dim3(kTX, kTY), 0, s>>>(S);
    k_vof_bmax<<<1, 1024, 0, s>>>(S);
    k_vof_diag<<<(S.nx * S.ny + 255) / 256, 256, 0, s>>>(S);
    return cudaGetLastError();
}

cudaError_t stage_vof_transport(const cfd2d_sim& S, cudaStream_t s) {
    k_vof_nsub<<<1, 1024, 0, s>>>(S);
    const dim3 grd = tiles(S.ny + 2, S.nx + 2);
    for (int k = 0; k < S.vof.nsub_max; ++k) {
        k_vof_advect<<<grd, dim3(kTX, kTY), 0, s>>>(S, k, 0.0, S.vof.alpha_tmp);
        k_vof_ghosts<<<grd, dim3(kTX, kTY), 0, s>>>(S, k, S.vof.alpha_tmp, S.vof.alpha);
    }
    // cfd2d/vof.py:271: _update_properties fills the ghosts once more
    return stage_vof_properties(S, s);
}

cudaError_t stage_vof_properties(const cfd2d_sim& S, cudaStream_t s) {
    const dim3 grd = tiles(S.ny + 2, S.nx + 2);
    const int n = (S.nx + 2) * (S.ny + 2);
    cudaError_t e = cudaMemcpyAsync(S.vof.alpha_tmp, S.vof.alpha, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    k_vof_ghosts<<<grd, dim3(kTX, kTY), 0, s>>>(S, -1, S.vof.alpha_tmp, S.vof.alpha);
    k_vof_props<<<(n + 255) / 256, 256, 0, s>>>(S);
    return cudaGetLastError();
}

cudaError_t launch_vof_advect(const cfd2d_sim& S, double dt, double* out, cudaStream_t s) {
    k_vof_advect<<<tiles(S.ny + 2, S.nx + 2), dim3(kTX, kTY), 0, s>>>(S, -1, dt, out);
    return cudaGetLastError();
}

}  // namespace cfd
