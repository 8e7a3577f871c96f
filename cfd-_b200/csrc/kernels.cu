// kernels.cu - stencil and bookkeeping kernels of the projection step.
//
// All arithmetic goes through cellmath.cuh; this file maps threads to faces and
// cells and implements the per-step bookkeeping (time step, reductions,
// history) on the device. Compiled with -fmad=false so that every expression is
// rounded exactly as the reference's float64 code.
#include <cuda_runtime.h>
#include <math.h>

#include "device.cuh"
#include "kernels.cuh"
#include "vof.cuh"

namespace cfd {

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ bool is_active(const cfd2d_state* st) { return st == nullptr || st->active != 0; }

__device__ __forceinline__ bool u_fluid(const cfd2d_sim& S, Grid2 g, int i, int j) {
    // cfd2d/grid.py:138-142 and cfd2d/solver.py:134-135 (face 0 is a copy when periodic)
    if (S.periodic && i == 0) return false;
    return S.fluid[g.c(i, j)] && S.fluid[g.c(i + 1, j)];
}
__device__ __forceinline__ bool v_fluid(const cfd2d_sim& S, Grid2 g, int i, int j) {
    return S.fluid[g.c(i, j)] && S.fluid[g.c(i, j + 1)];
}

// ================================================================ drop-in kernels
// row kernels: 2D tiles of kTileX (along j, contiguous) x kTileY (along i) threads, so
// that the stencil rows a block reads are shared through L1 by its warps
constexpr int kTileX = 32, kTileY = 8;

// A block's copy of phi, diff and the fluid flags for the transport stencil: rows
// ib - 2 .. ib + TY + 1 and columns j0 - 2 .. j0 + kTileX + 1, every cell an interior
// face flux of the tile or its upwind neighbour reads. Periodic in x, the rows beyond
// 1..nx hold the rows they wrap to, so a wrapped index (L = nx for the face of cell 1,
// the upwind cell nx or 1) may be looked up at any of its copies; otherwise cells
// outside the grid hold 0 and are never read.
template <int TY>
struct TransportStage {
    static constexpr int kR = TY + 4, kC = kTileX + 4;
    double phi[kR][kC];
    double diff[kR][kC];
    uint8_t fl[kR][kC];
};

// TransportArrays' interface (cellmath.cuh) on a TransportStage; only a periodic grid
// has wrapped row indices to map back into the tile
template <int TY, bool PERIODIC>
struct TransportTileView {
    const TransportStage<TY>* s;
    int ib, j0, nx;
    __device__ __forceinline__ int r(int i) const {
        int d = i - ib + 2;
        if constexpr (PERIODIC) {
            if (d < 0) d += nx;
            else if (d >= TransportStage<TY>::kR) d -= nx;
        }
        return d;
    }
    __device__ __forceinline__ int c(int j) const { return j - j0 + 2; }
    __device__ __forceinline__ double ph(int i, int j) const { return s->phi[r(i)][c(j)]; }
    __device__ __forceinline__ bool f(int i, int j) const { return s->fl[r(i)][c(j)] != 0; }
    __device__ __forceinline__ double d(int i, int j) const { return s->diff[r(i)][c(j)]; }
};

// TVD transport (cfd2d/kernels.py:271-391) of the (kTileY * ROWS) x kTileX cells of
// one block, every interior face flux computed once and shared by its two cells.
// Thread (tx, ty) takes cells (ib + ty + kTileY r, j0 + tx), r < ROWS. The block first
// loads its tile of phi, diff and the flags with halo into shared memory (independent,
// coalesced loads; the upwind reads, whose addresses depend on the face velocity,
// then hit shared memory), each thread its face velocities into registers. FX[q][c]
// holds xflux/dx of the west face of cell (ib + q, j0 + c) (row kTileY ROWS: the east
// face of the tile's last row, which is also the periodic face nx -> 1); FY[q][c]
// holds yflux/dy of the south face of cell (ib + q, j0 + c). Each cell then assembles
// ((west + east) + south) + north exactly as transport_cell does, with -FX / -FY for
// its east and north faces, so the result is bit-identical. Every thread of the block
// must call it (it synchronises the block); res[r] receives the value of its row r.
template <int ROWS, bool PERIODIC>
__device__ __forceinline__ void transport_tile(const double* __restrict__ phi, const double* __restrict__ u,
                                               const double* __restrict__ v, const uint8_t* __restrict__ fl,
                                               const double* __restrict__ diff, Grid2 g, double dx, double dy,
                                               int lim, const ScalarBCView& bc, int obs_t, double obs_v,
                                               double (&res)[ROWS]) {
    constexpr int TY = kTileY * ROWS;
    constexpr bool periodic = PERIODIC;
    using Stage = TransportStage<TY>;
    __shared__ Stage st;
    __shared__ double FX[TY + 1][kTileX];
    __shared__ double FY[TY][kTileX + 1];
    const int nx = g.nx, ny = g.ny;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int j0 = blockIdx.x * kTileX;
    const int j = j0 + tx;
    const int ib = blockIdx.y * TY;
    const bool jin = (j >= 1 && j <= ny);
    // x face index of the west face of cell ii (1 <= ii <= nx + 1; periodic: the
    // domain faces are face nx), -1 for a domain face without flux
    auto west_face = [&](int ii) -> int {
        if (ii == 1 || ii == nx + 1) return periodic ? nx : -1;
        return ii - 1;
    };
    // this thread's face velocities
    double uW[ROWS], vS[ROWS], vN[ROWS], uE = 0.0;
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
        const int q = ty + kTileY * r;
        const int i = ib + q;
        uW[r] = 0.0;
        vS[r] = 0.0;
        vN[r] = 0.0;
        if (jin && i >= 1 && i <= nx + 1) {
            const int fi = west_face(i);
            if (fi >= 0) uW[r] = u[g.u(fi, j)];
            if (q == TY - 1 && i + 1 <= nx + 1) {
                const int fe = west_face(i + 1);
                if (fe >= 0) uE = u[g.u(fe, j)];
            }
        }
        if (i >= 1 && i <= nx && j >= 2 && j <= ny) vS[r] = v[g.v(i, j - 1)];
        if (tx == kTileX - 1 && i >= 1 && i <= nx && j + 1 >= 2 && j + 1 <= ny) vN[r] = v[g.v(i, j)];
    }
    // the tile with its halo
    {
        constexpr int kN = Stage::kR * Stage::kC;
        const int tid = ty * kTileX + tx;
#pragma unroll 4
        for (int k = tid; k < kN; k += kTileX * kTileY) {
            const int lr = k / Stage::kC, lc = k - lr * Stage::kC;
            int gi = ib - 2 + lr;
            const int gj = j0 - 2 + lc;
            if (periodic && (gi < 1 || gi > nx)) gi = ((gi - 1) % nx + nx) % nx + 1;
            double a = 0.0, b = 0.0;
            uint8_t f = 0;
            if (gi >= 0 && gi <= nx + 1 && gj >= 0 && gj <= ny + 1) {
                a = phi[g.c(gi, gj)];
                b = diff[g.c(gi, gj)];
                f = fl[g.c(gi, gj)];
            }
            st.phi[lr][lc] = a;
            st.diff[lr][lc] = b;
            st.fl[lr][lc] = f;
        }
    }
    __syncthreads();
    const TransportTileView<TY, PERIODIC> a{&st, ib, j0, nx};
    auto west = [&](int ii, double uf) -> double {
        int L, R;
        if (ii == 1 || ii == nx + 1) {
            L = nx; R = 1;
        } else {
            L = ii - 1; R = ii;
        }
        if (!(a.f(L, j) && a.f(R, j))) return 0.0;
        return xflux_at(a, uf, nx, dx, lim, periodic, L, R, j) / dx;
    };
    // south face of cell (ii, jj) (2 <= jj <= ny)
    auto south = [&](int ii, int jj, double vf) -> double {
        if (!(a.f(ii, jj - 1) && a.f(ii, jj))) return 0.0;
        return yflux_at(a, vf, ny, dy, lim, ii, jj - 1) / dy;
    };
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
        const int q = ty + kTileY * r;
        const int i = ib + q;
        if (jin && i >= 1 && i <= nx + 1) {
            FX[q][tx] = (west_face(i) >= 0) ? west(i, uW[r]) : 0.0;
            if (q == TY - 1 && i + 1 <= nx + 1) FX[TY][tx] = (west_face(i + 1) >= 0) ? west(i + 1, uE) : 0.0;
        }
        if (i >= 1 && i <= nx && j >= 2 && j <= ny) FY[q][tx] = south(i, j, vS[r]);
        if (tx == kTileX - 1 && i >= 1 && i <= nx && j + 1 >= 2 && j + 1 <= ny) FY[q][kTileX] = south(i, j + 1, vN[r]);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
        const int q = ty + kTileY * r;
        const int i = ib + q;
        res[r] = 0.0;
        if (!(jin && i >= 1 && i <= nx) || !a.f(i, j)) continue;
        const double phP = a.ph(i, j);
        const double DP = a.d(i, j);
        double xw = 0.0, xe = 0.0, ys = 0.0, yn = 0.0;
        if (i == 1 && !periodic) {
            xw = boundary_term(u[g.u(0, j)], phP, DP, bc.bt[0][j - 1], bc.bv[0][j - 1], dx);
        } else {
            const int L = (i == 1) ? nx : i - 1;
            if (a.f(L, j)) xw = FX[q][tx];
            else if (obs_t == 1) xw = ((DP * (obs_v - phP)) / (0.5 * dx)) / dx;
        }
        if (i == nx && !periodic) {
            xe = boundary_term(-u[g.u(nx, j)], phP, DP, bc.bt[1][j - 1], bc.bv[1][j - 1], dx);
        } else {
            const int R = (i == nx) ? 1 : i + 1;
            if (a.f(R, j)) xe = -FX[q + 1][tx];
            else if (obs_t == 1) xe = ((DP * (obs_v - phP)) / (0.5 * dx)) / dx;
        }
        if (j == 1) {
            ys = boundary_term(v[g.v(i, 0)], phP, DP, bc.bt[2][i - 1], bc.bv[2][i - 1], dy);
        } else {
            if (a.f(i, j - 1)) ys = FY[q][tx];
            else if (obs_t == 1) ys = ((DP * (obs_v - phP)) / (0.5 * dy)) / dy;
        }
        if (j == ny) {
            yn = boundary_term(-v[g.v(i, ny)], phP, DP, bc.bt[3][i - 1], bc.bv[3][i - 1], dy);
        } else {
            if (a.f(i, j + 1)) yn = -FY[q][tx + 1];
            else if (obs_t == 1) yn = ((DP * (obs_v - phP)) / (0.5 * dy)) / dy;
        }
        res[r] = ((xw + xe) + ys) + yn;
    }
}

// rows per thread of the transport tile
constexpr int kTransportRows = 2;

// Inputs and outputs never alias (the C ABI requires it): __restrict__ lets the
// compiler issue every stencil load of a thread before its stores.
constexpr int kMomRows = 4;
// The viscosity and density forms are template parameters, so each instance carries
// only the arithmetic it needs.
template <bool VARIABLE, bool VAR_DENSITY>
__global__ void __launch_bounds__(256) k_momentum(const double* __restrict__ u, const double* __restrict__ v,
                                                  const uint8_t* __restrict__ fl, int nx, int ny, InvSpacing inv,
                                                  const double* __restrict__ nu, double gamma, int periodic,
                                                  double* __restrict__ hu, double* __restrict__ hv,
                                                  const double* __restrict__ rho) {
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    // kMomRows consecutive rows per thread: a thread issues the loads of all its faces
    // before any arithmetic needs them (more bytes in flight per thread), and the rows
    // it shares with its own neighbours come from L1
    const int i0 = (blockIdx.y * blockDim.y + threadIdx.y) * kMomRows;
    if (j >= ny + 2 || i0 >= nx + 2) return;
    const MomCoef m = mom_coef_inv(inv, gamma, __ldg(&nu[g.c(1, 1)]));
    const int imax = periodic ? nx : nx - 1;
    // all tendencies first, then all stores
    double hU[kMomRows], hV[kMomRows];
#pragma unroll
    for (int r = 0; r < kMomRows; ++r) {
        const int i = i0 + r;
        hU[r] = 0.0;
        hV[r] = 0.0;
        if (i >= 1 && i <= imax && j >= 1 && j <= ny) hU[r] = mom_u(u, v, fl, nu, rho, g, m, VARIABLE, VAR_DENSITY, i, j);
        if (i >= 1 && i <= nx && j >= 1 && j <= ny - 1) hV[r] = mom_v(u, v, fl, nu, rho, g, m, VARIABLE, VAR_DENSITY, i, j);
    }
#pragma unroll
    for (int r = 0; r < kMomRows; ++r) {
        const int i = i0 + r;
        if (i <= nx) hu[g.u(i, j)] = hU[r];
        if (j <= ny && i <= nx + 1) hv[g.v(i, j)] = hV[r];
    }
}

__global__ void k_obstacle_bc(double* u, double* v, const uint8_t* fl, int nx, int ny,
                              int periodic, const cfd2d_state* st) {
    if (!is_active(st)) return;
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (blockIdx.y * blockDim.y + threadIdx.y);
    if (j >= ny + 2 || i >= nx + 1) return;
    const int imax = periodic ? nx : nx - 1;
    if (i >= 1 && i <= imax) {
        double nu_ = u[g.u(i, j)];
        if (j >= 1 && j <= ny) {
            nu_ = obc_u(u, fl, g, i, j);
            u[g.u(i, j)] = nu_;
        }
        // periodic: u[0, :] = u[nx, :] after the loop (cfd2d/kernels.py:188-190)
        if (periodic && i == nx) u[g.u(0, j)] = nu_;
    }
    if (i >= 1 && i <= nx && j >= 1 && j <= ny - 1) v[g.v(i, j)] = obc_v(v, fl, g, i, j);
}

template <bool PERIODIC>
__global__ void __launch_bounds__(256) k_scalar_transport(const double* __restrict__ phi,
                                                          const double* __restrict__ u,
                                                          const double* __restrict__ v,
                                                          const uint8_t* __restrict__ fl, int nx, int ny,
                                                          double dx, double dy, const double* __restrict__ diff,
                                                          int limiter, ScalarBCView bc, int obs_t,
                                                          double obs_v, double* __restrict__ out,
                                                          const cfd2d_state* st) {
    if (!is_active(st)) return;  // uniform over the grid
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double r[kTransportRows];
    transport_tile<kTransportRows, PERIODIC>(phi, u, v, fl, diff, g, dx, dy, limiter, bc, obs_t, obs_v, r);
#pragma unroll
    for (int k = 0; k < kTransportRows; ++k) {
        const int i = blockIdx.y * kTileY * kTransportRows + threadIdx.y + kTileY * k;
        if (j < ny + 2 && i < nx + 2) out[g.c(i, j)] = r[k];
    }
}

// cfd2d/geometry.py:17-22: (X - xc)**2 + (Y - yc)**2 <= r**2, X = (i + 0.5) * dx
__global__ void k_mask_circle(int nx, int ny, double dx, double dy, double xc, double yc, double r,
                              uint8_t* mask) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= ny || i >= nx) return;
    const double X = ((double)i + 0.5) * dx, Y = ((double)j + 0.5) * dy;
    const double a = X - xc, b = Y - yc;
    mask[i * ny + j] = (a * a + b * b <= r * r) ? 1 : 0;
}

// cfd2d/geometry.py:25-32
__global__ void k_mask_ellipse(int nx, int ny, double dx, double dy, double xc, double yc, double a,
                               double b, double cp, double sp, uint8_t* mask) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= ny || i >= nx) return;
    const double X = ((double)i + 0.5) * dx, Y = ((double)j + 0.5) * dy;
    const double xr = (X - xc) * cp + (Y - yc) * sp;
    const double yr = -(X - xc) * sp + (Y - yc) * cp;
    const double s = xr / a, t = yr / b;
    mask[i * ny + j] = (s * s + t * t <= 1.0) ? 1 : 0;
}

// cfd2d/geometry.py:35-40
__global__ void k_mask_rect(int nx, int ny, double dx, double dy, double xa, double ya, double xb,
                            double yb, uint8_t* mask) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= ny || i >= nx) return;
    const double X = ((double)i + 0.5) * dx, Y = ((double)j + 0.5) * dy;
    mask[i * ny + j] = (X >= xa && X <= xb && Y >= ya && Y <= yb) ? 1 : 0;
}

// Closed polygon (cfd2d/geometry.py:43-51, matplotlib Path.contains_points): crossing
// test of a ray from the cell centre towards +x against every edge, the edge counted
// when its end points lie on opposite sides of the centre's y (one side inclusive).
__global__ void k_mask_polygon(int nx, int ny, double dx, double dy, const double* px, const double* py, int np,
                               uint8_t* mask) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= ny || i >= nx) return;
    const double X = ((double)i + 0.5) * dx, Y = ((double)j + 0.5) * dy;
    bool inside = false;
    double x0 = px[np - 1], y0 = py[np - 1];
    bool above0 = y0 >= Y;
    for (int k = 0; k < np; ++k) {
        const double x1 = px[k], y1 = py[k];
        const bool above1 = y1 >= Y;
        if (above0 != above1) {
            // the edge crosses the centre's row: is the crossing right of the centre?
            if (((y1 - Y) * (x0 - x1) >= (x1 - X) * (y0 - y1)) == above1) inside = !inside;
        }
        x0 = x1;
        y0 = y1;
        above0 = above1;
    }
    mask[i * ny + j] = inside ? 1 : 0;
}

// Image obstacle (cfd2d/geometry.py:119-163): the cell centre's pixel of a solid
// bitmap (h rows from the top, w columns) placed on [x0, x0 + width] x [y0, y0 + height]
__global__ void k_mask_image(int nx, int ny, double dx, double dy, const uint8_t* solid, int h, int w, double x0,
                             double y0, double width, double height, uint8_t* mask) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= ny || i >= nx) return;
    const double X = ((double)i + 0.5) * dx, Y = ((double)j + 0.5) * dy;
    const double sx = (X - x0) / width, sy = (Y - y0) / height;
    const bool in = sx >= 0 && sx < 1 && sy >= 0 && sy < 1;
    uint8_t m = 0;
    if (in) {
        long long col = (long long)(sx * (double)w), row = (long long)((1.0 - sy) * (double)h);
        col = col < 0 ? 0 : (col > w - 1 ? w - 1 : col);
        row = row < 0 ? 0 : (row > h - 1 ? h - 1 : row);
        m = solid[row * w + col];
    }
    mask[i * ny + j] = m;
}

// ================================================================ domain boundary
// cfd2d/boundary.py:143-223 in one block: the statement groups of the reference
// (periodic copies; left/right; bottom/top; closing of blocked faces) depend on
// each other through the corners, so they run as barrier-separated phases.
// With begin != 0 the block first decides whether this step runs (run() stop
// conditions, cfd2d/solver.py:466-492).
__global__ void k_domain_bc(cfd2d_sim S, double* u, double* v, int begin) {
    cfd2d_state* st = S.state;
    __shared__ int act;
    if (threadIdx.x == 0) {
        int a = 1;
        if (st) {
            if (begin) {
                if (st->status & (CFD2D_S_NONFINITE | CFD2D_S_BARRIER_TIMEOUT)) a = 0;
                else if (st->stop_reason != 0) a = 0;
                else if (!(st->t < st->t_end - 1e-12)) { a = 0; st->stop_reason = 1; }
                else if (st->max_steps >= 0 && st->n >= st->max_steps) { a = 0; st->stop_reason = 2; }
                st->active = a;
            } else {
                a = st->active;
            }
        }
        act = a;
    }
    __syncthreads();
    if (!act) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int T = blockDim.x;
    if (S.periodic) {
        for (int j = threadIdx.x; j < ny + 2; j += T) u[g.u(0, j)] = u[g.u(nx, j)];
        for (int j = threadIdx.x; j < ny + 1; j += T) {
            v[g.v(0, j)] = v[g.v(nx, j)];
            v[g.v(nx + 1, j)] = v[g.v(1, j)];
        }
    }
    __syncthreads();
    // left (normal u[0, j], tangential ghost v[0, :]) and right
    for (int side = 0; side < 2; ++side) {
        const int kind = S.bc_kind[side];
        const int nrm = side == 0 ? 0 : nx;
        const int ghost = side == 0 ? 0 : nx + 1;
        const int inner = side == 0 ? 1 : nx;
        const double vel = S.bc_vel[side];
        const uint8_t* op = S.open[side];
        for (int j = threadIdx.x; j < ny + 1; j += T) {
            const double vi = v[g.v(inner, j)];
            if (kind == CFD2D_BC_NOSLIP) v[g.v(ghost, j)] = 2.0 * vel - vi;
            else if (kind == CFD2D_BC_SLIP || kind == CFD2D_BC_OUTFLOW) v[g.v(ghost, j)] = vi;
            else if (kind == CFD2D_BC_INFLOW) v[g.v(ghost, j)] = -vi;
        }
        for (int j = threadIdx.x + 1; j <= ny; j += T) {
            if (kind == CFD2D_BC_NOSLIP || kind == CFD2D_BC_SLIP) u[g.u(nrm, j)] = 0.0;
            else if (kind == CFD2D_BC_INFLOW) u[g.u(nrm, j)] = S.inflow[side][j - 1];
            else if (kind == CFD2D_BC_OUTFLOW) { if (!op[j - 1]) u[g.u(nrm, j)] = 0.0; }
        }
    }
    __syncthreads();
    // bottom (normal v[i, 0], tangential ghost u[:, 0]) and top
    for (int side = 2; side < 4; ++side) {
        const int kind = S.bc_kind[side];
        const int nrm = side == 2 ? 0 : ny;
        const int ghost = side == 2 ? 0 : ny + 1;
        const int inner = side == 2 ? 1 : ny;
        const double vel = S.bc_vel[side];
        const uint8_t* op = S.open[side];
        for (int i = threadIdx.x; i < nx + 1; i += T) {
            const double ui = u[g.u(i, inner)];
            if (kind == CFD2D_BC_NOSLIP) u[g.u(i, ghost)] = 2.0 * vel - ui;
            else if (kind == CFD2D_BC_SLIP || kind == CFD2D_BC_OUTFLOW) u[g.u(i, ghost)] = ui;
            else if (kind == CFD2D_BC_INFLOW) u[g.u(i, ghost)] = -ui;
        }
        for (int i = threadIdx.x + 1; i <= nx; i += T) {
            if (kind == CFD2D_BC_NOSLIP || kind == CFD2D_BC_SLIP) v[g.v(i, nrm)] = 0.0;
            else if (kind == CFD2D_BC_INFLOW) v[g.v(i, nrm)] = S.inflow[side][i - 1];
            else if (kind == CFD2D_BC_OUTFLOW) { if (!op[i - 1]) v[g.v(i, nrm)] = 0.0; }
        }
    }
    __syncthreads();
    // faces behind a blocked boundary cell are closed (cfd2d/boundary.py:218-223)
    if (!S.periodic) {
        for (int j = threadIdx.x + 1; j <= ny; j += T) {
            if (!S.open[0][j - 1]) u[g.u(0, j)] = 0.0;
            if (!S.open[1][j - 1]) u[g.u(nx, j)] = 0.0;
        }
    }
    for (int i = threadIdx.x + 1; i <= nx; i += T) {
        if (!S.open[2][i - 1]) v[g.v(i, 0)] = 0.0;
        if (!S.open[3][i - 1]) v[g.v(i, ny)] = 0.0;
    }
}

// ================================================================ SST pre-momentum
// cfd2d/turbulence.py:244-282 per interior cell: strain rate, blending, nu_t and
// the blended diffusivities of k and omega.
__global__ void k_sst_pre(cfd2d_sim S) {
    if (!is_active(S.state)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int i = (blockIdx.y * blockDim.y + threadIdx.y) + 1;
    if (j > ny || i > nx) return;
    const SSTConst K = sst_const();
    const cfd2d_scalar& ks = S.scalars[S.sst.k_index];
    const cfd2d_scalar& ws = S.scalars[S.sst.w_index];
    const int c = g.c(i, j);
    const int ci = (i - 1) * ny + (j - 1);
    const double nu = S.nu;
    const double k = npmax(ks.phi[c], 0.0);
    const double w = npmax(ws.phi[c], 1e-12);
    const double S2 = strain2(S.u, S.v, g, S.dx, S.dy, i, j);
    const double dkx = (ks.phi[g.c(i + 1, j)] - ks.phi[g.c(i - 1, j)]) / (2 * S.dx);
    const double dky = (ks.phi[g.c(i, j + 1)] - ks.phi[g.c(i, j - 1)]) / (2 * S.dy);
    const double dwx = (ws.phi[g.c(i + 1, j)] - ws.phi[g.c(i - 1, j)]) / (2 * S.dx);
    const double dwy = (ws.phi[g.c(i, j + 1)] - ws.phi[g.c(i, j - 1)]) / (2 * S.dy);
    const double cross = dkx * dwx + dky * dwy;
    const double CD = npmax(((2.0 * K.so2) / w) * cross, 1e-10);
    const double sk = sqrt(k);
    const double d = S.sst.d[ci];
    const double d2 = d * d;
    const double t1 = sk / ((K.beta_star * w) * d);
    const double t2 = (500 * nu) / (d2 * w);
    const double t3 = ((4 * K.so2) * k) / (CD * d2);
    const double arg1 = npmin(npmax(t1, t2), t3);
    const double F1 = tanh(pow(arg1, 4.0));
    const double arg2 = npmax((2 * sk) / ((K.beta_star * w) * d), t2);
    const double F2 = tanh(arg2 * arg2);
    const double nut = (K.a1 * k) / npmax(K.a1 * w, sqrt(S2) * F2);
    S.nu_t[c] = S.fluid[c] ? nut : 0.0;
    const double skb = F1 * K.sk1 + (1 - F1) * K.sk2;
    const double sob = F1 * K.so1 + (1 - F1) * K.so2;
    ks.diff[c] = nu + skb * nut;
    ws.diff[c] = nu + sob * nut;
    S.sst.F1[ci] = F1;
    S.sst.cross[ci] = cross;
}

// ================================================================ Smagorinsky
// cfd2d/turbulence.py:149-152 per interior cell: nu_t = l^2 sqrt(S^2) on fluid
// cells, 0 on solids (l^2 fixed at attach time, turbulence.py:137-147).
__global__ void k_smag_pre(cfd2d_sim S) {
    if (!is_active(S.state)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int i = (blockIdx.y * blockDim.y + threadIdx.y) + 1;
    if (j > ny || i > nx) return;
    const int c = g.c(i, j);
    const double S2 = strain2(S.u, S.v, g, S.dx, S.dy, i, j);
    const double nut = S.smag.l2[(i - 1) * ny + (j - 1)] * sqrt(S2);
    S.nu_t[c] = S.fluid[c] ? nut : 0.0;
}

// nu_t ghost values (cfd2d/turbulence.py:110-124) and nu_eff = nu + nu_t
// (cfd2d/solver.py:332-333) over every cell; with SST also the clamped ghost
// copies of the k and omega diffusivities (turbulence.py:278-282).
__device__ __forceinline__ double nut_col(const cfd2d_sim& S, Grid2 g, int i, int j) {
    // value of column i (0..nx+1) at row j (1..ny) after the column step
    const int nx = S.nx;
    if (i >= 1 && i <= nx) return S.nu_t[g.c(i, j)];
    if (i == 0) {
        if (S.periodic) return S.nu_t[g.c(nx, j)];
        return S.bc_kind[0] == CFD2D_BC_NOSLIP ? 0.0 : S.nu_t[g.c(1, j)];
    }
    if (S.periodic) return S.nu_t[g.c(1, j)];
    return S.bc_kind[1] == CFD2D_BC_NOSLIP ? 0.0 : S.nu_t[g.c(nx, j)];
}

template <bool SST>
__global__ void k_nut_ghosts(cfd2d_sim S) {
    if (!is_active(S.state)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (blockIdx.y * blockDim.y + threadIdx.y);
    if (j >= ny + 2 || i >= nx + 2) return;
    const int c = g.c(i, j);
    const bool ghost = (i == 0 || i == nx + 1 || j == 0 || j == ny + 1);
    double nut;
    if (!ghost) {
        nut = S.nu_t[c];
    } else {
        if (j == 0) nut = S.bc_kind[2] == CFD2D_BC_NOSLIP ? 0.0 : nut_col(S, g, i, 1);
        else if (j == ny + 1) nut = S.bc_kind[3] == CFD2D_BC_NOSLIP ? 0.0 : nut_col(S, g, i, ny);
        else nut = nut_col(S, g, i, j);
        if (SST) {
            // diffusivity ghosts: diff[i, j] = diff[clamp(i), clamp(j)]
            const int ii = i < 1 ? 1 : (i > nx ? nx : i);
            const int jj = j < 1 ? 1 : (j > ny ? ny : j);
            const cfd2d_scalar& ks = S.scalars[S.sst.k_index];
            const cfd2d_scalar& ws = S.scalars[S.sst.w_index];
            ks.diff[c] = ks.diff[g.c(ii, jj)];
            ws.diff[c] = ws.diff[g.c(ii, jj)];
        }
    }
    __syncwarp();
    if (ghost) S.nu_t[c] = nut;
    S.nu_eff[c] = S.nu + nut;
}

// ================================================================ time step
// Reductions for compute_dt / _auto_gamma (cfd2d/solver.py:209-253); the last
// block turns them into dt, gamma and the AB2 weights of this step.
__global__ void k_dt(cfd2d_sim S) {
    cfd2d_state* st = S.state;
    if (!is_active(st)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int ncell = (nx + 2) * (ny + 2);
    double m[3 + CFD2D_MAX_SCALARS];
    for (int k = 0; k < 3 + CFD2D_MAX_SCALARS; ++k) m[k] = 0.0;
    double numin = INFINITY;
    const bool need_nu = S.variable_viscosity != 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        const int i = c / (ny + 2), j = c % (ny + 2);
        if (i <= nx) m[0] = npmax(m[0], fabs(S.u[g.u(i, j)]));
        if (j <= ny) m[1] = npmax(m[1], fabs(S.v[g.v(i, j)]));
        if (need_nu) {
            if (S.vof_on) {
                // kinematic mixture viscosity over the fluid cells (cfd2d/solver.py:215-216, 248-249)
                if (S.fluid[c]) {
                    const double ne = S.nu_eff[c] / S.vof.rho[c];
                    m[2] = npmax(m[2], ne);
                    numin = npmin(numin, ne);
                }
            } else {
                const double ne = S.nu_eff[c];
                m[2] = npmax(m[2], ne);
                if (S.fluid[c]) numin = npmin(numin, ne);
            }
        }
        if (S.fluid[c]) {
            for (int s = 0; s < S.nscalars; ++s)
                if (S.scalar_dtlim_const[s] == 0.0) m[3 + s] = npmax(m[3 + s], S.scalars[s].diff[c]);
        }
    }
    __shared__ double sred[32 * (3 + CFD2D_MAX_SCALARS)];
    block_max<3 + CFD2D_MAX_SCALARS>(m, sred);
    {
        double mn[1] = {-numin};
        // min via max of the negation (all values finite or +inf)
        block_max<1>(mn, sred, -INFINITY);
        numin = -mn[0];
    }
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&st->umax_bits, m[0]);
        atomic_max_nonneg(&st->vmax_bits, m[1]);
        if (need_nu) {
            atomic_max_nonneg(&st->numax_bits, m[2]);
            atomic_min_nonneg(&st->numin_bits, numin);
        }
        for (int s = 0; s < S.nscalars; ++s) atomic_max_nonneg(&st->dmax_bits[s], m[3 + s]);
    }
    if (!last_block(&st->ticket[0])) return;
    if (threadIdx.x != 0) return;
    volatile cfd2d_state* vs = st;
    const double umax_raw = bitsd(vs->umax_bits);
    const double vmax_raw = bitsd(vs->vmax_bits);
    const double numax = bitsd(vs->numax_bits);
    const double numin_f = bitsd(vs->numin_bits);
    const double dx = S.dx, dy = S.dy;
    double dt;
    if (st->dt_fixed != 0.0) {
        dt = st->dt_fixed;
    } else {
        const double umax = pymax(umax_raw, 1e-12);
        const double vmax = pymax(vmax_raw, 1e-12);
        const double nu_max = need_nu ? numax : S.nu;
        double dt_visc = 0.5 / (nu_max * (1.0 / (dx * dx) + 1.0 / (dy * dy)));
        double dt_conv = pymin(dx / umax, dy / vmax);
        if (S.scheme_ab2) {
            dt_visc = dt_visc * 0.5;
            dt_conv = dt_conv * 0.8;
        }
        dt = S.tau * pymin(dt_visc, dt_conv);
        for (int s = 0; s < S.nscalars; ++s) {
            double lim = S.scalar_dtlim_const[s];
            if (lim == 0.0) {
                const double dmax = bitsd(vs->dmax_bits[s]);
                lim = (dmax <= 0.0) ? INFINITY : 0.5 / (dmax * (1.0 / (dx * dx) + 1.0 / (dy * dy)));
            }
            if (isfinite(lim)) dt = pymin(dt, S.tau * lim);
        }
        if (S.vof_on && S.vof.dt_limit > 0.0) dt = pymin(dt, S.tau * S.vof.dt_limit);
        // run(): shorten the last step to land on t_end (cfd2d/solver.py:470-480)
        if (st->t + dt > st->t_end) dt = st->t_end - st->t;
    }
    double gamma = S.gamma_fixed;
    if (S.gamma_auto) {
        if (!S.scheme_ab2) {
            const double cfl = pymax((umax_raw * dt) / dx, (vmax_raw * dt) / dy);
            gamma = pymin(1.0, pymax(0.05, 1.2 * cfl));
        } else {
            const double nu_ref = need_nu ? numin_f : S.nu;
            const double re_cell = pymax(umax_raw * dx, vmax_raw * dy) / nu_ref;
            gamma = pymin(1.0, pymax(0.05, 0.015 * re_cell));
        }
    }
    st->dt = dt;
    st->gamma = gamma;
    if (S.scheme_ab2 && st->have_old) {
        const double r = dt / st->dt_old;
        st->ab_a = 1.0 + 0.5 * r;
        st->ab_b = -0.5 * r;
    }
    st->umax_bits = 0ull;
    st->vmax_bits = 0ull;
    st->numax_bits = 0ull;
    st->numin_bits = dbits(INFINITY);
    for (int s = 0; s < CFD2D_MAX_SCALARS; ++s) st->dmax_bits[s] = 0ull;
    __threadfence();
    st->ticket[0] = 0u;
}

// ================================================================ predictor
// hu/hv (momentum_tendencies + Boussinesq source), AB2, F = u + dt H (+ body
// force), the outflow extrapolation of F, G and u_prev, v_prev
// (cfd2d/solver.py:338-368, cfd2d/models.py:386-396, cfd2d/boundary.py:225-245).
// With copy_only, F = u and G = v plus the extrapolation (solver.py:199-201, 417-419).
__global__ void k_predictor(cfd2d_sim S, int copy_only, InvSpacing inv) {
    cfd2d_state* st = S.state;
    if (!is_active(st)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (blockIdx.y * blockDim.y + threadIdx.y);
    if (j >= ny + 2 || i >= nx + 2) return;
    const double dt = copy_only ? 0.0 : st->dt;
    const bool ab2 = S.scheme_ab2 && st->have_old;
    const double a = st->ab_a, b = st->ab_b;
    const double fx = S.body_fx + st->flow_force;
    const double fy = S.body_fy;
    const MomCoef m = mom_coef_inv(inv, st->gamma, S.nu_eff[g.c(1, 1)]);
    const bool var = S.variable_viscosity != 0;
    // two-phase VOF: (1/rho) div(mu grad u) and the CSF surface-tension source
    const bool vd = S.vof_on != 0;
    const double* rho = vd ? S.vof.rho : nullptr;
    const bool csf = vd && S.vof.sigma > 0;
    const double* T = (S.thermal_index >= 0) ? S.scalars[S.thermal_index].phi : nullptr;
    const bool lo = S.bc_kind[0] == CFD2D_BC_OUTFLOW, ro = S.bc_kind[1] == CFD2D_BC_OUTFLOW;
    const bool bo = S.bc_kind[2] == CFD2D_BC_OUTFLOW, to = S.bc_kind[3] == CFD2D_BC_OUTFLOW;
    // ---- u face (i, j), i in 0..nx
    if (i <= nx) {
        const int f = g.u(i, j);
        const double uij = S.u[f];
        double Fv = uij;
        if (!copy_only) {
            double h = 0.0;
            if (u_fluid(S, g, i, j)) {
                h = mom_u(S.u, S.v, S.fluid, S.nu_eff, rho, g, m, var, vd, i, j);
                if (T && S.gx != 0.0) {
                    const double Tf = 0.5 * (T[g.c(i, j)] + T[g.c(i + 1, j)]) - S.T_ref;
                    h = h + (-S.gx) * Tf;
                }
                if (csf) h = h + csf_u(S, i, j);
                const double H = ab2 ? (a * h + b * S.hu[f]) : h;
                Fv = uij + dt * H;
                if (fx != 0.0) Fv = Fv + dt * fx;
            }
            S.hu[f] = h;
            S.u_prev[f] = uij;
        }
        const bool in_row = (j >= 1 && j <= ny);
        bool own = true;
        if (i == 0 && (S.periodic || (in_row && lo && S.open[0][j - 1]))) own = false;
        if (i == nx && in_row && ro && S.open[1][j - 1]) own = false;
        if (own) S.F[f] = Fv;
        if (S.periodic && i == nx) S.F[g.u(0, j)] = Fv;
        if (in_row && i == 1 && lo && S.open[0][j - 1]) S.F[g.u(0, j)] = Fv;
        if (in_row && i == nx - 1 && ro && S.open[1][j - 1]) S.F[g.u(nx, j)] = Fv;
    }
    // ---- v face (i, j), j in 0..ny
    if (j <= ny) {
        const int f = g.v(i, j);
        const double vij = S.v[f];
        double Gv = vij;
        if (!copy_only) {
            double h = 0.0;
            if (v_fluid(S, g, i, j)) {
                h = mom_v(S.u, S.v, S.fluid, S.nu_eff, rho, g, m, var, vd, i, j);
                if (T && S.gy != 0.0) {
                    const double Tf = 0.5 * (T[g.c(i, j)] + T[g.c(i, j + 1)]) - S.T_ref;
                    h = h + (-S.gy) * Tf;
                }
                if (csf) h = h + csf_v(S, i, j);
                const double H = ab2 ? (a * h + b * S.hv[f]) : h;
                Gv = vij + dt * H;
                if (fy != 0.0) Gv = Gv + dt * fy;
            }
            S.hv[f] = h;
            S.v_prev[f] = vij;
        }
        const bool in_col = (i >= 1 && i <= nx);
        bool own = true;
        if (j == 0 && in_col && bo && S.open[2][i - 1]) own = false;
        if (j == ny && in_col && to && S.open[3][i - 1]) own = false;
        if (own) S.G[f] = Gv;
        if (in_col && j == 1 && bo && S.open[2][i - 1]) S.G[g.v(i, 0)] = Gv;
        if (in_col && j == ny - 1 && to && S.open[3][i - 1]) S.G[g.v(i, ny)] = Gv;
    }
}

// ================================================================ correction
// u = F - dt grad p on fluid faces, outflow faces with 2 dt p / h
// (cfd2d/solver.py:277-321). unit_dt: dt = 1 (initial and flow-rate projections).
__global__ void k_correct(cfd2d_sim S, const double* p, int unit_dt) {
    cfd2d_state* st = S.state;
    if (!is_active(st)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (blockIdx.y * blockDim.y + threadIdx.y);
    if (j >= ny + 2 || i >= nx + 2) return;
    const double dt = unit_dt ? 1.0 : st->dt;
    const double dx = S.dx, dy = S.dy;
    const int pc = ny + 2;
    // variable density: dt b (dp/dh) with the face coefficient b (cfd2d/solver.py:284-321);
    // b = 1 gives the constant-density expressions bit for bit
    const bool vd = S.vof_on != 0;
    if (i <= nx && j >= 1 && j <= ny) {
        const int f = g.u(i, j);
        const double bu = vd ? S.vof.bx[f] : 1.0;
        if (i >= 1 && i <= nx - 1) {
            const double Fv = S.F[f];
            S.u[f] = u_fluid(S, g, i, j) ? Fv - ((dt * bu) * (p[(i + 1) * pc + j] - p[i * pc + j])) / dx : Fv;
        } else if (S.periodic) {
            if (i == nx) {
                const double Fv = S.F[f];
                S.u[f] = u_fluid(S, g, i, j) ? Fv - ((dt * bu) * (p[1 * pc + j] - p[nx * pc + j])) / dx : Fv;
            }
        } else if (i == 0) {
            const double Fv = S.F[f];
            const bool d = S.bc_kind[0] == CFD2D_BC_OUTFLOW && S.open[0][j - 1];
            S.u[f] = d ? Fv - (((2 * dt) * bu) * p[1 * pc + j]) / dx : Fv;
        } else {  // i == nx
            const double Fv = S.F[f];
            const bool d = S.bc_kind[1] == CFD2D_BC_OUTFLOW && S.open[1][j - 1];
            S.u[f] = d ? Fv + (((2 * dt) * bu) * p[nx * pc + j]) / dx : Fv;
        }
    }
    if (S.periodic && i == nx) {
        // u[0, :] = u[nx, :] after the correction (cfd2d/solver.py:305)
        S.u[g.u(0, j)] = S.u[g.u(nx, j)];
    }
    if (j <= ny && i >= 1 && i <= nx) {
        const int f = g.v(i, j);
        const double bv = vd ? S.vof.by[f] : 1.0;
        if (j >= 1 && j <= ny - 1) {
            const double Gv = S.G[f];
            S.v[f] = v_fluid(S, g, i, j) ? Gv - ((dt * bv) * (p[i * pc + j + 1] - p[i * pc + j])) / dy : Gv;
        } else if (!S.periodic) {
            const double Gv = S.G[f];
            if (j == 0) {
                const bool d = S.bc_kind[2] == CFD2D_BC_OUTFLOW && S.open[2][i - 1];
                S.v[f] = d ? Gv - (((2 * dt) * bv) * p[i * pc + 1]) / dy : Gv;
            } else {
                const bool d = S.bc_kind[3] == CFD2D_BC_OUTFLOW && S.open[3][i - 1];
                S.v[f] = d ? Gv + (((2 * dt) * bv) * p[i * pc + ny]) / dy : Gv;
            }
        }
    }
}

// p[:] = value (initial projection resets p to 0, cfd2d/solver.py:203)
__global__ void k_fill(double* a, int n, double value, const cfd2d_state* st) {
    if (!is_active(st)) return;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) a[c] = value;
}

// ================================================================ flow-rate control
// cfd2d/solver.py:405-425: bulk velocity over the fluid u faces of columns 1..nx,
// uniform shift, forcing update.
__global__ void k_bulk(cfd2d_sim S, double* red) {
    cfd2d_state* st = S.state;
    if (!is_active(st)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    double s[1] = {0.0};
    const int n = nx * ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c / ny + 1, j = c % ny + 1;
        if (u_fluid(S, g, i, j)) s[0] += S.u[g.u(i, j)];
    }
    __shared__ double sred[32];
    block_sum<1>(s, sred);
    if (threadIdx.x == 0) red[blockIdx.x] = s[0];
    if (!last_block(&st->ticket[1])) return;
    double t[1] = {0.0};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t[0] += ld_cg(&red[b]);
    block_sum<1>(t, sred);
    if (threadIdx.x == 0) {
        const double bulk = t[0] / S.flow_count;
        const double du = S.flow_rate - bulk;
        st->bulk_du = du;
        st->flow_force = st->flow_force + du / st->dt;
        st->ticket[1] = 0u;
    }
}

__global__ void k_shift_u(cfd2d_sim S) {
    cfd2d_state* st = S.state;
    if (!is_active(st)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (blockIdx.y * blockDim.y + threadIdx.y);
    if (j >= ny + 2 || i > nx) return;
    const double du = st->bulk_du;
    double val = S.u[g.u(i, j)];
    if (u_fluid(S, g, i, j)) {
        val = val + du;
        S.u[g.u(i, j)] = val;
    }
    if (S.periodic && i == nx) S.u[g.u(0, j)] = val;
}

// ================================================================ scalars
// diff = D0 + nu_t / Sc_t (cfd2d/models.py:320-322, 398-400)
__global__ void k_scalar_turb_diff(cfd2d_sim S, int s) {
    if (!is_active(S.state)) return;
    const cfd2d_scalar& sc = S.scalars[s];
    const int n = (S.nx + 2) * (S.ny + 2);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        sc.diff[c] = sc.D0 + S.nu_t[c] / sc.turb_div;
}

template <bool PERIODIC>
__global__ void k_scalar_rhs(cfd2d_sim S, int s) {
    if (!is_active(S.state)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const cfd2d_scalar& sc = S.scalars[s];
    ScalarBCView bc;
    for (int k = 0; k < 4; ++k) { bc.bt[k] = sc.bt[k]; bc.bv[k] = sc.bv[k]; }
    // rhs does not overlap phi, u, v, diff or the flags
    double r[kTransportRows];
    transport_tile<kTransportRows, PERIODIC>(sc.phi, S.u, S.v, S.fluid, sc.diff, g, S.dx, S.dy, sc.limiter, bc,
                                             sc.obs_t, sc.obs_v, r);
#pragma unroll
    for (int k = 0; k < kTransportRows; ++k) {
        const int i = blockIdx.y * kTileY * kTransportRows + threadIdx.y + kTileY * k;
        if (j < ny + 2 && i < nx + 2) sc.rhs[g.c(i, j)] = r[k];
    }
}

// Euler update with point-implicit source and clipping (cfd2d/models.py:196-207);
// SST sources cfd2d/turbulence.py:285-304, wall omega turbulence.py:239-242.
__global__ void k_scalar_update(cfd2d_sim S, int s) {
    cfd2d_state* st = S.state;
    if (!is_active(st)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int i = (blockIdx.y * blockDim.y + threadIdx.y) + 1;
    if (j > ny || i > nx) return;
    const cfd2d_scalar& sc = S.scalars[s];
    const int c = g.c(i, j);
    const int ci = (i - 1) * ny + (j - 1);
    const double dt = st->dt;
    const double phi_i = sc.phi[c];
    double nw = phi_i + dt * sc.rhs[c];
    if (sc.source == 1 || sc.source == 2) {
        const SSTConst K = sst_const();
        const double* kphi = S.scalars[S.sst.k_index].phi;
        const double* wphi = S.scalars[S.sst.w_index].phi;
        double s_exp, s_imp;
        if (sc.source == 1) {
            const double S2 = strain2(S.u, S.v, g, S.dx, S.dy, i, j);
            S.sst.S2[ci] = S2;
            const double k = npmax(kphi[c], 0.0);
            const double w = npmax(wphi[c], 1e-12);
            const double nut = S.nu_t[c];
            const double Pk = npmin(nut * S2, ((10.0 * K.beta_star) * k) * w);
            S.sst.Pk[ci] = Pk;
            s_exp = Pk;
            s_imp = K.beta_star * w;
        } else {
            const double F1 = S.sst.F1[ci];
            const double w = npmax(wphi[c], 1e-12);
            const double gam = F1 * K.gamma1 + (1 - F1) * K.gamma2;
            const double bet = F1 * K.beta1 + (1 - F1) * K.beta2;
            const double nut_raw = S.nu_t[c];
            const double nut = npmax(nut_raw, 1e-14);
            double Pw = (gam * S.sst.Pk[ci]) / nut;
            if (!(nut_raw > 1e-14)) Pw = gam * S.sst.S2[ci];
            const double CDw = (((2.0 * (1 - F1)) * K.so2) / w) * S.sst.cross[ci];
            s_exp = Pw + npmax(CDw, 0.0);
            s_imp = bet * w + npmax(-CDw, 0.0) / w;
        }
        nw = (nw + dt * s_exp) / (1.0 + dt * npmax(s_imp, 0.0));
    }
    if (sc.has_lower) nw = npmax(nw, sc.lower);
    if (sc.has_upper) nw = npmin(nw, sc.upper);
    sc.phi[c] = S.fluid[c] ? nw : phi_i;
}

// viscous omega in the wall-adjacent cells after the omega update
// (cfd2d/turbulence.py:239-242); the ghosts are filled before and after, as the
// reference does (a periodic corner keeps the value of the first fill)
__global__ void k_sst_wall_omega(cfd2d_sim S) {
    if (!is_active(S.state)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int i = (blockIdx.y * blockDim.y + threadIdx.y) + 1;
    if (j > ny || i > nx) return;
    const int ci = (i - 1) * ny + (j - 1);
    if (S.sst.wall_adj[ci]) S.scalars[S.sst.w_index].phi[g.c(i, j)] = S.sst.w_wall[ci];
}

// Domain ghost cells of a scalar (cfd2d/models.py:157-166). With periodic x the
// ghost columns copy the opposite columns over their full height; the corner
// entries take the old values of rows 0 and ny+1, which the same thread reads
// before recomputing them.
__global__ void k_scalar_ghost_domain(cfd2d_sim S, int s) {
    if (!is_active(S.state)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const cfd2d_scalar& sc = S.scalars[s];
    double* phi = sc.phi;
    const double* D = sc.diff;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    // threads 0..ny-1: left/right ghost columns at row j = t + 1
    if (t < ny) {
        const int j = t + 1;
        if (S.periodic) {
            phi[g.c(0, j)] = phi[g.c(nx, j)];
            phi[g.c(nx + 1, j)] = phi[g.c(1, j)];
        } else {
            phi[g.c(0, j)] = scalar_ghost(phi[g.c(1, j)], sc.bt[0][j - 1], sc.bv[0][j - 1], S.dx,
                                          npmax(D[g.c(1, j)], 1e-300));
            phi[g.c(nx + 1, j)] = scalar_ghost(phi[g.c(nx, j)], sc.bt[1][j - 1], sc.bv[1][j - 1], S.dx,
                                               npmax(D[g.c(nx, j)], 1e-300));
        }
    }
    // threads ny..ny+nx-1: bottom/top ghost rows at column i
    const int k = t - ny;
    if (k >= 0 && k < nx) {
        const int i = k + 1;
        if (S.periodic && i == nx) {
            phi[g.c(0, 0)] = phi[g.c(nx, 0)];
            phi[g.c(0, ny + 1)] = phi[g.c(nx, ny + 1)];
        }
        if (S.periodic && i == 1) {
            phi[g.c(nx + 1, 0)] = phi[g.c(1, 0)];
            phi[g.c(nx + 1, ny + 1)] = phi[g.c(1, ny + 1)];
        }
        phi[g.c(i, 0)] = scalar_ghost(phi[g.c(i, 1)], sc.bt[2][i - 1], sc.bv[2][i - 1], S.dy,
                                      npmax(D[g.c(i, 1)], 1e-300));
        phi[g.c(i, ny + 1)] = scalar_ghost(phi[g.c(i, ny)], sc.bt[3][i - 1], sc.bv[3][i - 1], S.dy,
                                           npmax(D[g.c(i, ny)], 1e-300));
    }
}

// Solid cells next to fluid take the mean of their fluid neighbours (mirrored
// about a fixed obstacle value), cfd2d/models.py:168-183.
__global__ void k_scalar_ghost_solid(cfd2d_sim S, int s, int obs_fixed, double obs_value) {
    if (!is_active(S.state)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int i = (blockIdx.y * blockDim.y + threadIdx.y) + 1;
    if (j > ny || i > nx) return;
    const int c = g.c(i, j);
    if (S.fluid[c]) return;
    const cfd2d_scalar& sc = S.scalars[s];
    double* phi = sc.phi;
    // neighbours E, W, N, S; the ghost columns of a periodic grid hold copies of the
    // opposite interior columns, read here directly
    int ie = i + 1, iw = i - 1;
    if (S.periodic) {
        if (ie == nx + 1) ie = 1;
        if (iw == 0) iw = nx;
    }
    const bool fe = S.fluid[g.c(i + 1, j)], fw = S.fluid[g.c(i - 1, j)];
    const bool fn = S.fluid[g.c(i, j + 1)], fs = S.fluid[g.c(i, j - 1)];
    const double pe = fe ? phi[g.c(ie, j)] : 0.0;
    const double pw = fw ? phi[g.c(iw, j)] : 0.0;
    const double pn = fn ? phi[g.c(i, j + 1)] : 0.0;
    const double ps = fs ? phi[g.c(i, j - 1)] : 0.0;
    const double sum = ((pe + pw) + pn) + ps;
    const double cnt = (((double)fe + (double)fw) + (double)fn) + (double)fs;
    if (cnt > 0) {
        const double avg = sum / pymax(cnt, 1.0);
        phi[c] = obs_fixed ? 2 * obs_value - avg : avg;
    } else if (obs_fixed) {
        phi[c] = obs_value;
    }
}

// ================================================================ end of step
// residual max|du|/dt (cfd2d/solver.py:390-399), time/step counters and the
// per-step history record (solver.py:427-443: max|div u|, kinetic energy,
// obstacle forces solver.py:542-567, forcing).
__global__ void k_end_step(cfd2d_sim S) {
    cfd2d_state* st = S.state;
    if (!is_active(st)) return;
    const int nx = S.nx, ny = S.ny;
    const Grid2 g{nx, ny};
    const double dx = S.dx, dy = S.dy;
    const int ncell = (nx + 2) * (ny + 2);
    double mx[3] = {0.0, 0.0, 0.0};  // du, dv, |div|
    double sm[9];                     // ke, pe, pw, pn, ps, un, us, ve, vw
    for (int k = 0; k < 9; ++k) sm[k] = 0.0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        const int i = c / (ny + 2), j = c % (ny + 2);
        if (i <= nx && u_fluid(S, g, i, j)) mx[0] = npmax(mx[0], fabs(S.u[g.u(i, j)] - S.u_prev[g.u(i, j)]));
        if (j <= ny && v_fluid(S, g, i, j)) mx[1] = npmax(mx[1], fabs(S.v[g.v(i, j)] - S.v_prev[g.v(i, j)]));
        if (i >= 1 && i <= nx && j >= 1 && j <= ny && S.fluid[c]) {
            const double div = (S.u[g.u(i, j)] - S.u[g.u(i - 1, j)]) / dx +
                               (S.v[g.v(i, j)] - S.v[g.v(i, j - 1)]) / dy;
            mx[2] = npmax(mx[2], fabs(div));
            const double uc = 0.5 * (S.u[g.u(i - 1, j)] + S.u[g.u(i, j)]);
            const double vc = 0.5 * (S.v[g.v(i, j - 1)] + S.v[g.v(i, j)]);
            sm[0] += uc * uc + vc * vc;
            if (S.compute_forces) {
                // solid neighbours inside the domain (the ghost frame is not solid here)
                const bool se = (i + 1 <= nx) && !S.fluid[g.c(i + 1, j)];
                const bool sw = (i - 1 >= 1) && !S.fluid[g.c(i - 1, j)];
                const bool sn = (j + 1 <= ny) && !S.fluid[g.c(i, j + 1)];
                const bool ss = (j - 1 >= 1) && !S.fluid[g.c(i, j - 1)];
                const double pv = S.p[c];
                if (se) sm[1] += pv;
                if (sw) sm[2] += pv;
                if (sn) sm[3] += pv;
                if (ss) sm[4] += pv;
                if (sn) sm[5] += uc;
                if (ss) sm[6] += uc;
                if (se) sm[7] += vc;
                if (sw) sm[8] += vc;
            }
        }
    }
    __shared__ double sred[32 * 9];
    block_max<3>(mx, sred);
    block_sum<9>(sm, sred);
    double* red = S.red;
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&st->du_bits, mx[0]);
        atomic_max_nonneg(&st->dv_bits, mx[1]);
        atomic_max_nonneg(&st->div_bits, mx[2]);
        for (int k = 0; k < 9; ++k) red[k * gridDim.x + blockIdx.x] = sm[k];
    }
    if (!last_block(&st->ticket[2])) return;
    double t[9];
    for (int k = 0; k < 9; ++k) {
        t[k] = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t[k] += ld_cg(&red[k * gridDim.x + b]);
    }
    block_sum<9>(t, sred);
    if (threadIdx.x != 0) return;
    volatile cfd2d_state* vs = st;
    const double du = bitsd(vs->du_bits), dv = bitsd(vs->dv_bits), dmax = bitsd(vs->div_bits);
    st->du_bits = 0ull;
    st->dv_bits = 0ull;
    st->div_bits = 0ull;
    const double dt = st->dt;
    st->dt_old = dt;
    if (S.scheme_ab2) st->have_old = 1;
    st->t = st->t + dt;
    st->n = st->n + 1;
    const double res = pymax(du, dv) / dt;
    st->residual = res;
    if (!isfinite(res) || res > 1e8) {
        if (st->status == 0) st->error_step = (int)st->n;
        st->status |= CFD2D_S_NONFINITE;
    }
    if (st->steady_tol > 0.0 && st->n > 10 && res < st->steady_tol) st->stop_reason = 3;
    const double ke = ((0.5 * t[0]) * dx) * dy;
    double fxo = 0.0, fyo = 0.0;
    if (S.compute_forces) {
        const double mu = S.nu;
        fxo = (t[1] - t[2]) * dy;
        fyo = (t[3] - t[4]) * dx;
        fxo = fxo + ((mu * (t[5] + t[6])) / (0.5 * dy)) * dx;
        fyo = fyo + ((mu * (t[7] + t[8])) / (0.5 * dx)) * dy;
    }
    if (S.hist && S.hist_cap > 0) {
        double* h = S.hist + (size_t)((st->n - 1) % S.hist_cap) * CFD2D_HIST_FIELDS;
        h[0] = st->t;
        h[1] = dt;
        h[2] = res;
        h[3] = dmax;
        h[4] = ke;
        h[5] = fxo;
        h[6] = fyo;
        h[7] = st->flow_force;
        h[8] = (double)st->cg_iters_step;
        h[9] = st->gamma;
    }
    __threadfence();
    st->ticket[2] = 0u;
}

// ================================================================ host launchers
namespace {
const dim3 kTile(kTileX, kTileY, 1);
inline dim3 grid_rows(int width, int rows) {
    return dim3((width + kTileX - 1) / kTileX, (rows + kTileY - 1) / kTileY, 1);
}
inline cudaError_t last() { return cudaGetLastError(); }

// Thread-block shapes of the row kernels that index by blockDim (every thread its own
// cells, so the shape changes only the speed): [0] the momentum_tendencies drop-in,
// [1] the step's row kernels. The transport kernels keep kTile (shared-memory tile).
int g_tile[2][2] = {{kTileX, kTileY}, {kTileX, kTileY}};
inline dim3 tile(int which) { return dim3(g_tile[which][0], g_tile[which][1], 1); }
inline dim3 grid_tile(int which, int width, int rows) {
    const int tx = g_tile[which][0], ty = g_tile[which][1];
    return dim3((width + tx - 1) / tx, (rows + ty - 1) / ty, 1);
}
constexpr int kMom = 0, kStep = 1;
}  // namespace

int set_tile(int which, int tx, int ty) {
    if (which < 0 || which > 1 || tx < 16 || tx % 16 != 0 || ty < 1 || tx * ty > 256) return -1;
    g_tile[which][0] = tx;
    g_tile[which][1] = ty;
    return 0;
}

int get_tile(int which, int* tx, int* ty) {
    if (which < 0 || which > 1 || !tx || !ty) return -1;
    *tx = g_tile[which][0];
    *ty = g_tile[which][1];
    return 0;
}

int reduction_blocks(int ncell) {
    int b = (ncell + kBlock - 1) / kBlock;
    if (b > 2 * 148) b = 2 * 148;
    if (b < 1) b = 1;
    return b;
}

cudaError_t launch_momentum(const double* u, const double* v, const uint8_t* fl, int nx, int ny,
                            double dx, double dy, const double* nu, int variable, double gamma,
                            int periodic, double* hu, double* hv, const double* rho, int var_density,
                            cudaStream_t s) {
    const InvSpacing inv = inv_spacing(dx, dy);
    const dim3 grd = grid_tile(kMom, ny + 2, (nx + 2 + kMomRows - 1) / kMomRows);
    const dim3 blk = tile(kMom);
    if (variable && var_density)
        k_momentum<true, true><<<grd, blk, 0, s>>>(u, v, fl, nx, ny, inv, nu, gamma, periodic, hu, hv, rho);
    else if (variable)
        k_momentum<true, false><<<grd, blk, 0, s>>>(u, v, fl, nx, ny, inv, nu, gamma, periodic, hu, hv, rho);
    else if (var_density)
        k_momentum<false, true><<<grd, blk, 0, s>>>(u, v, fl, nx, ny, inv, nu, gamma, periodic, hu, hv, rho);
    else
        k_momentum<false, false><<<grd, blk, 0, s>>>(u, v, fl, nx, ny, inv, nu, gamma, periodic, hu, hv, rho);
    return last();
}

cudaError_t launch_obstacle_bc(double* u, double* v, const uint8_t* fl, int nx, int ny, int periodic,
                               const cfd2d_state* st, cudaStream_t s) {
    k_obstacle_bc<<<grid_rows(ny + 2, nx + 1), kTile, 0, s>>>(u, v, fl, nx, ny, periodic, st);
    return last();
}

cudaError_t launch_scalar_transport(const double* phi, const double* u, const double* v,
                                    const uint8_t* fl, int nx, int ny, double dx, double dy,
                                    const double* diff, int limiter, int periodic,
                                    const ScalarBCView& bc, int obs_t, double obs_v, double* out,
                                    cudaStream_t s) {
    const dim3 grd = grid_rows(ny + 2, (nx + 2 + kTransportRows - 1) / kTransportRows);
    if (periodic)
        k_scalar_transport<true><<<grd, kTile, 0, s>>>(phi, u, v, fl, nx, ny, dx, dy, diff, limiter, bc, obs_t,
                                                        obs_v, out, nullptr);
    else
        k_scalar_transport<false><<<grd, kTile, 0, s>>>(phi, u, v, fl, nx, ny, dx, dy, diff, limiter, bc, obs_t,
                                                         obs_v, out, nullptr);
    return last();
}

cudaError_t launch_mask(int kind, int nx, int ny, double dx, double dy, const double* q,
                        uint8_t* mask, cudaStream_t s) {
    const dim3 grd = grid_rows(ny, nx);
    if (kind == 0) k_mask_circle<<<grd, kTile, 0, s>>>(nx, ny, dx, dy, q[0], q[1], q[2], mask);
    else if (kind == 1) k_mask_ellipse<<<grd, kTile, 0, s>>>(nx, ny, dx, dy, q[0], q[1], q[2], q[3], q[4], q[5], mask);
    else k_mask_rect<<<grd, kTile, 0, s>>>(nx, ny, dx, dy, q[0], q[1], q[2], q[3], mask);
    return last();
}

cudaError_t launch_mask_polygon(int nx, int ny, double dx, double dy, const double* px, const double* py, int np,
                                uint8_t* mask, cudaStream_t s) {
    k_mask_polygon<<<grid_rows(ny, nx), kTile, 0, s>>>(nx, ny, dx, dy, px, py, np, mask);
    return last();
}

cudaError_t launch_mask_image(int nx, int ny, double dx, double dy, const uint8_t* solid, int h, int w, double x0,
                              double y0, double width, double height, uint8_t* mask, cudaStream_t s) {
    k_mask_image<<<grid_rows(ny, nx), kTile, 0, s>>>(nx, ny, dx, dy, solid, h, w, x0, y0, width, height, mask);
    return last();
}

cudaError_t stage_domain_bc(const cfd2d_sim& S, double* u, double* v, int begin, cudaStream_t s) {
    k_domain_bc<<<1, 1024, 0, s>>>(S, u, v, begin);
    return last();
}

cudaError_t stage_apply_bc(const cfd2d_sim& S, int begin, cudaStream_t s) {
    cudaError_t e = stage_domain_bc(S, S.u, S.v, begin, s);
    if (e != cudaSuccess) return e;
    return launch_obstacle_bc(S.u, S.v, S.fluid, S.nx, S.ny, S.periodic, S.state, s);
}

cudaError_t stage_sst_pre(const cfd2d_sim& S, cudaStream_t s) {
    k_sst_pre<<<grid_tile(kStep, S.ny, S.nx), tile(kStep), 0, s>>>(S);
    k_nut_ghosts<true><<<grid_tile(kStep, S.ny + 2, S.nx + 2), tile(kStep), 0, s>>>(S);
    return last();
}

cudaError_t stage_smag_pre(const cfd2d_sim& S, cudaStream_t s) {
    k_smag_pre<<<grid_tile(kStep, S.ny, S.nx), tile(kStep), 0, s>>>(S);
    k_nut_ghosts<false><<<grid_tile(kStep, S.ny + 2, S.nx + 2), tile(kStep), 0, s>>>(S);
    return last();
}

cudaError_t stage_dt(const cfd2d_sim& S, cudaStream_t s) {
    k_dt<<<reduction_blocks((S.nx + 2) * (S.ny + 2)), kBlock, 0, s>>>(S);
    return last();
}

cudaError_t stage_predictor(const cfd2d_sim& S, int copy_only, cudaStream_t s) {
    k_predictor<<<grid_tile(kStep, S.ny + 2, S.nx + 2), tile(kStep), 0, s>>>(S, copy_only, inv_spacing(S.dx, S.dy));
    return last();
}

cudaError_t stage_correct(const cfd2d_sim& S, const double* p, int unit_dt, cudaStream_t s) {
    k_correct<<<grid_tile(kStep, S.ny + 2, S.nx + 2), tile(kStep), 0, s>>>(S, p, unit_dt);
    return last();
}

cudaError_t stage_flow_shift(const cfd2d_sim& S, cudaStream_t s) {
    k_bulk<<<reduction_blocks(S.nx * S.ny), kBlock, 0, s>>>(S, S.red);
    k_shift_u<<<grid_tile(kStep, S.ny + 2, S.nx + 1), tile(kStep), 0, s>>>(S);
    return last();
}

cudaError_t stage_scalar(const cfd2d_sim& S, int slot, cudaStream_t s) {
    const cfd2d_scalar& sc = S.scalars[slot];
    if (sc.turb_div > 0.0 && S.variable_viscosity)
        k_scalar_turb_diff<<<reduction_blocks((S.nx + 2) * (S.ny + 2)), kBlock, 0, s>>>(S, slot);
    const dim3 grd = grid_rows(S.ny + 2, (S.nx + 2 + kTransportRows - 1) / kTransportRows);
    if (S.periodic)
        k_scalar_rhs<true><<<grd, kTile, 0, s>>>(S, slot);
    else
        k_scalar_rhs<false><<<grd, kTile, 0, s>>>(S, slot);
    k_scalar_update<<<grid_tile(kStep, S.ny, S.nx), tile(kStep), 0, s>>>(S, slot);
    cudaError_t e = stage_scalar_ghosts(S, slot, s);
    if (e != cudaSuccess || sc.source != 2) return e;
    k_sst_wall_omega<<<grid_tile(kStep, S.ny, S.nx), tile(kStep), 0, s>>>(S);
    return stage_scalar_ghosts(S, slot, s);
}

cudaError_t stage_scalar_ghosts(const cfd2d_sim& S, int slot, cudaStream_t s) {
    const cfd2d_scalar& sc = S.scalars[slot];
    const int n = S.nx + S.ny;
    k_scalar_ghost_domain<<<(n + kBlock - 1) / kBlock, kBlock, 0, s>>>(S, slot);
    if (S.has_solid)
        k_scalar_ghost_solid<<<grid_tile(kStep, S.ny, S.nx), tile(kStep), 0, s>>>(S, slot, sc.obs_t == 1 ? 1 : 0, sc.obs_v);
    return last();
}

cudaError_t stage_end(const cfd2d_sim& S, cudaStream_t s) {
    k_end_step<<<reduction_blocks((S.nx + 2) * (S.ny + 2)), kBlock, 0, s>>>(S);
    return last();
}

cudaError_t stage_fill(const cfd2d_sim& S, double* a, int n, double value, cudaStream_t s) {
    k_fill<<<reduction_blocks(n), kBlock, 0, s>>>(a, n, value, S.state);
    return last();
}

}  // namespace cfd
