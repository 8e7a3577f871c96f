// cellmath.cuh - per-face / per-cell arithmetic of the projection step.
//
// Every function evaluates one face or one cell in exactly the operation order of
// the reference (Python/Numba, IEEE float64, no fused multiply-add), so results
// are bit-identical to cfd2d when compiled with -fmad=false (nvcc) or
// -ffp-contract=off (host compilers). The functions are __host__ __device__ so that
// host code can evaluate the same expressions.
//
// The stencil functions read their inputs through an accessor (by global face and
// cell index): the *Arrays views read the reference's arrays in HBM, the transport
// kernels' tile view reads a block's copy in shared memory. The arithmetic is
// written once.
//
// Layout (reference cfd2d/grid.py:1-18): p-like and u arrays have row pitch
// ny+2, v arrays ny+1; fluid flags (nx+2)(ny+2) bytes.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define CFD_HD __host__ __device__ __forceinline__
#else
#define CFD_HD inline
#endif

namespace cfd {

// Python's builtin min/max on two floats: min(a, b) keeps a unless b < a.
CFD_HD double pymin(double a, double b) { return (b < a) ? b : a; }
CFD_HD double pymax(double a, double b) { return (b > a) ? b : a; }
// numpy.minimum / numpy.maximum: NaN in either operand propagates.
CFD_HD double npmin(double a, double b) { return (a != a || b != b) ? (a + b) : ((b < a) ? b : a); }
CFD_HD double npmax(double a, double b) { return (a != a || b != b) ? (a + b) : ((b > a) ? b : a); }

struct Grid2 {
    int nx, ny;
    CFD_HD int pc() const { return ny + 2; }  // pitch of cell and u arrays
    CFD_HD int pv() const { return ny + 1; }  // pitch of v arrays
    CFD_HD int c(int i, int j) const { return i * (ny + 2) + j; }
    CFD_HD int u(int i, int j) const { return i * (ny + 2) + j; }
    CFD_HD int v(int i, int j) const { return i * (ny + 1) + j; }
};

struct MomCoef {
    double idx, idy, idx2, idy2, nu0, gx, gy;  // gx = gamma*idx, gy = gamma*idy
};

// Reciprocal spacings, computed once on the host: the kernels then divide by
// nothing per cell. Same IEEE operations as the reference's 1/dx, 1/dx**2.
struct InvSpacing {
    double idx, idy, idx2, idy2;
};
inline InvSpacing inv_spacing(double dx, double dy) {
    return InvSpacing{1.0 / dx, 1.0 / dy, 1.0 / (dx * dx), 1.0 / (dy * dy)};
}
CFD_HD MomCoef mom_coef_inv(const InvSpacing& s, double gamma, double nu0) {
    MomCoef m;
    m.idx2 = s.idx2;
    m.idy2 = s.idy2;
    m.idx = s.idx;
    m.idy = s.idy;
    m.nu0 = nu0;
    m.gx = gamma * m.idx;
    m.gy = gamma * m.idy;
    return m;
}

// The arrays of the momentum stencil in the reference's layout. ue(i, j) is u on the
// face east of face i, face 1 for i = nx (periodic; cfd2d/kernels.py:90).
struct MomArrays {
    const double *u, *v, *nu, *rho;
    const uint8_t* fl;
    Grid2 g;
    CFD_HD bool f(int i, int j) const { return fl[g.c(i, j)] != 0; }
    CFD_HD double U(int i, int j) const { return u[g.u(i, j)]; }
    CFD_HD double ue(int i, int j) const { return u[g.u((i < g.nx) ? i + 1 : 1, j)]; }
    CFD_HD double V(int i, int j) const { return v[g.v(i, j)]; }
    CFD_HD double Nu(int i, int j) const { return nu[g.c(i, j)]; }
    CFD_HD double Rho(int i, int j) const { return rho[g.c(i, j)]; }
};

// u-momentum tendency on face (i, j), i in 1..imax, j in 1..ny
// (cfd2d/kernels.py:85-119). Returns 0 for faces not between two fluid cells.
template <class A>
CFD_HD double mom_u_at(const A& a, const MomCoef& m, bool variable, bool var_density, int i, int j) {
    if (!(a.f(i, j) && a.f(i + 1, j))) return 0.0;
    const double uc = a.U(i, j), ue = a.ue(i, j), uw = a.U(i - 1, j);
    const double un = a.U(i, j + 1), us = a.U(i, j - 1);
    double diff;
    if (variable) {
        const double nu_e = a.Nu(i + 1, j);
        const double nu_w = a.Nu(i, j);
        const double nu_n = 0.25 * (((a.Nu(i, j) + a.Nu(i + 1, j)) + a.Nu(i, j + 1)) + a.Nu(i + 1, j + 1));
        const double nu_s = 0.25 * (((a.Nu(i, j) + a.Nu(i + 1, j)) + a.Nu(i, j - 1)) + a.Nu(i + 1, j - 1));
        const double vn = (a.V(i + 1, j) - a.V(i, j)) * m.idx;
        const double vs = (a.V(i + 1, j - 1) - a.V(i, j - 1)) * m.idx;
        diff = ((2.0 * nu_e) * (ue - uc) - (2.0 * nu_w) * (uc - uw)) * m.idx2 +
               m.idy * (nu_n * ((un - uc) * m.idy + vn) - nu_s * ((uc - us) * m.idy + vs));
    } else {
        diff = m.nu0 * (((ue - 2.0 * uc) + uw) * m.idx2 + ((un - 2.0 * uc) + us) * m.idy2);
    }
    if (var_density) diff = diff / (0.5 * (a.Rho(i, j) + a.Rho(i + 1, j)));
    const double a_e = 0.5 * (uc + ue);
    const double a_w = 0.5 * (uw + uc);
    const double du2dx = m.idx * (a_e * a_e - a_w * a_w) +
                         m.gx * ((fabs(a_e) * 0.5) * (uc - ue) - (fabs(a_w) * 0.5) * (uw - uc));
    const double v_n = 0.5 * (a.V(i, j) + a.V(i + 1, j));
    const double v_s = 0.5 * (a.V(i, j - 1) + a.V(i + 1, j - 1));
    const double duvdy = m.idy * ((v_n * 0.5) * (uc + un) - (v_s * 0.5) * (us + uc)) +
                         m.gy * ((fabs(v_n) * 0.5) * (uc - un) - (fabs(v_s) * 0.5) * (us - uc));
    return (diff - du2dx) - duvdy;
}

// v-momentum tendency on face (i, j), i in 1..nx, j in 1..ny-1 (cfd2d/kernels.py:122-155).
template <class A>
CFD_HD double mom_v_at(const A& a, const MomCoef& m, bool variable, bool var_density, int i, int j) {
    if (!(a.f(i, j) && a.f(i, j + 1))) return 0.0;
    const double vc = a.V(i, j), ve = a.V(i + 1, j), vw = a.V(i - 1, j);
    const double vn = a.V(i, j + 1), vs = a.V(i, j - 1);
    double diff;
    if (variable) {
        const double nu_n = a.Nu(i, j + 1);
        const double nu_s = a.Nu(i, j);
        const double nu_e = 0.25 * (((a.Nu(i, j) + a.Nu(i + 1, j)) + a.Nu(i, j + 1)) + a.Nu(i + 1, j + 1));
        const double nu_w = 0.25 * (((a.Nu(i, j) + a.Nu(i - 1, j)) + a.Nu(i, j + 1)) + a.Nu(i - 1, j + 1));
        const double ue_ = (a.U(i, j + 1) - a.U(i, j)) * m.idy;
        const double uw_ = (a.U(i - 1, j + 1) - a.U(i - 1, j)) * m.idy;
        diff = ((2.0 * nu_n) * (vn - vc) - (2.0 * nu_s) * (vc - vs)) * m.idy2 +
               m.idx * (nu_e * ((ve - vc) * m.idx + ue_) - nu_w * ((vc - vw) * m.idx + uw_));
    } else {
        diff = m.nu0 * (((ve - 2.0 * vc) + vw) * m.idx2 + ((vn - 2.0 * vc) + vs) * m.idy2);
    }
    if (var_density) diff = diff / (0.5 * (a.Rho(i, j) + a.Rho(i, j + 1)));
    const double b_n = 0.5 * (vc + vn);
    const double b_s = 0.5 * (vs + vc);
    const double dv2dy = m.idy * (b_n * b_n - b_s * b_s) +
                         m.gy * ((fabs(b_n) * 0.5) * (vc - vn) - (fabs(b_s) * 0.5) * (vs - vc));
    const double u_e = 0.5 * (a.U(i, j) + a.U(i, j + 1));
    const double u_w = 0.5 * (a.U(i - 1, j) + a.U(i - 1, j + 1));
    const double duvdx = m.idx * ((u_e * 0.5) * (vc + ve) - (u_w * 0.5) * (vw + vc)) +
                         m.gx * ((fabs(u_e) * 0.5) * (vc - ve) - (fabs(u_w) * 0.5) * (vw - vc));
    return (diff - duvdx) - dv2dy;
}

CFD_HD double mom_u(const double* u, const double* v, const uint8_t* fl, const double* nu,
                    const double* rho, Grid2 g, const MomCoef& m, bool variable, bool var_density,
                    int i, int j) {
    return mom_u_at(MomArrays{u, v, nu, rho, fl, g}, m, variable, var_density, i, j);
}
CFD_HD double mom_v(const double* u, const double* v, const uint8_t* fl, const double* nu,
                    const double* rho, Grid2 g, const MomCoef& m, bool variable, bool var_density,
                    int i, int j) {
    return mom_v_at(MomArrays{u, v, nu, rho, fl, g}, m, variable, var_density, i, j);
}

// New value of u face (i, j) after the obstacle condition (cfd2d/kernels.py:170-187);
// i in 1..imax, j in 1..ny. The neighbours read are both-fluid faces, which this
// condition never writes, so every face can be evaluated independently.
CFD_HD double obc_u(const double* u, const uint8_t* fl, Grid2 g, int i, int j) {
    const bool a = fl[g.c(i, j)], b = fl[g.c(i + 1, j)];
    if (a && b) return u[g.u(i, j)];
    if (a || b) return 0.0;
    double s = 0.0;
    int c = 0;
    if (fl[g.c(i, j + 1)] && fl[g.c(i + 1, j + 1)]) { s += u[g.u(i, j + 1)]; c += 1; }
    if (fl[g.c(i, j - 1)] && fl[g.c(i + 1, j - 1)]) { s += u[g.u(i, j - 1)]; c += 1; }
    return c > 0 ? -s / (double)c : 0.0;
}

// v face (i, j), i in 1..nx, j in 1..ny-1 (cfd2d/kernels.py:192-209).
CFD_HD double obc_v(const double* v, const uint8_t* fl, Grid2 g, int i, int j) {
    const bool a = fl[g.c(i, j)], b = fl[g.c(i, j + 1)];
    if (a && b) return v[g.v(i, j)];
    if (a || b) return 0.0;
    double s = 0.0;
    int c = 0;
    if (fl[g.c(i + 1, j)] && fl[g.c(i + 1, j + 1)]) { s += v[g.v(i + 1, j)]; c += 1; }
    if (fl[g.c(i - 1, j)] && fl[g.c(i - 1, j + 1)]) { s += v[g.v(i - 1, j)]; c += 1; }
    return c > 0 ? -s / (double)c : 0.0;
}

// ---------------------------------------------------------------- TVD transport
// cfd2d/kernels.py:215-235
CFD_HD double limiter(double r, int kind) {
    if (kind == 0) return 0.0;
    if (kind == 1) return (r <= 0.0) ? 0.0 : (2.0 * r) / (1.0 + r);
    if (kind == 2) return (r <= 0.0) ? 0.0 : pymin(r, 1.0);
    if (kind == 3) return (r <= 0.0) ? 0.0 : pymax(pymin(2.0 * r, 1.0), pymin(r, 2.0));
    if (kind == 5) return (r <= 0.0) ? 0.0 : pymin(2.0 * r, pymin(0.5 * (1.0 + r), 2.0));
    return 1.0;
}

// cfd2d/kernels.py:238-251: face value between C (upwind) and D, U further upstream.
CFD_HD double face_value(double phu, double phc, double phd, bool has_u, int kind) {
    if (kind == 0) return phc;
    if (kind == 4) return 0.5 * (phc + phd);
    if (!has_u) return phc;
    const double den = phd - phc;
    if (fabs(den) < 1e-300) return phc;
    const double r = (phc - phu) / den;
    return phc + (0.5 * limiter(r, kind)) * den;
}

CFD_HD double harmonic(double a, double b) {
    return (a + b > 0.0) ? ((2.0 * a) * b) / (a + b) : 0.0;
}

struct ScalarBCView {
    const int64_t* bt[4];
    const double* bv[4];
};

// The cell arrays the interior transport fluxes read, in the reference's layout.
struct TransportArrays {
    const double* phi;
    const uint8_t* fl;
    const double* diff;
    Grid2 g;
    CFD_HD double ph(int i, int j) const { return phi[g.c(i, j)]; }
    CFD_HD bool f(int i, int j) const { return fl[g.c(i, j)] != 0; }
    CFD_HD double d(int i, int j) const { return diff[g.c(i, j)]; }
};

// Flux F through an interior x face with velocity uf joining cells L (west) and R
// (east) (cfd2d/kernels.py:304-330). Both cells are fluid.
template <class A>
CFD_HD double xflux_at(const A& a, double uf, int nx, double dx, int limiter_kind, bool periodic, int L, int R,
                       int j) {
    int C, D, Ui;
    if (uf >= 0.0) {
        C = L; D = R; Ui = L - 1;
        if (Ui < 1) Ui = periodic ? nx : -1;
    } else {
        C = R; D = L; Ui = R + 1;
        if (Ui > nx) Ui = periodic ? 1 : -1;
    }
    const bool has_u = Ui >= 1 && a.f(Ui, j);
    const double phu = has_u ? a.ph(Ui, j) : 0.0;
    const double phf = face_value(phu, a.ph(C, j), a.ph(D, j), has_u, limiter_kind);
    const double df = harmonic(a.d(L, j), a.d(R, j));
    return uf * phf - (df * (a.ph(R, j) - a.ph(L, j))) / dx;
}

// Flux through the interior y face with velocity vf joining cells B (south) and
// T = B + 1 of row i (cfd2d/kernels.py:361-383).
template <class A>
CFD_HD double yflux_at(const A& a, double vf, int ny, double dy, int limiter_kind, int i, int B) {
    const int T = B + 1;
    int C, D, Uj;
    if (vf >= 0.0) { C = B; D = T; Uj = B - 1; }
    else { C = T; D = B; Uj = T + 1; }
    const bool has_u = Uj >= 1 && Uj <= ny && a.f(i, Uj);
    const double phu = has_u ? a.ph(i, Uj) : 0.0;
    const double phf = face_value(phu, a.ph(i, C), a.ph(i, D), has_u, limiter_kind);
    const double df = harmonic(a.d(i, B), a.d(i, T));
    return vf * phf - (df * (a.ph(i, T) - a.ph(i, B))) / dy;
}

// The same fluxes on the arrays in HBM, the x face with index fi
CFD_HD double xflux(const double* phi, const double* u, const uint8_t* fl, const double* diff,
                    Grid2 g, double dx, int limiter_kind, bool periodic, int fi, int L, int R,
                    int j) {
    return xflux_at(TransportArrays{phi, fl, diff, g}, u[g.u(fi, j)], g.nx, dx, limiter_kind, periodic, L, R, j);
}
CFD_HD double yflux(const double* phi, const double* v, const uint8_t* fl, const double* diff,
                    Grid2 g, double dy, int limiter_kind, int i, int B) {
    return yflux_at(TransportArrays{phi, fl, diff, g}, v[g.v(i, B)], g.ny, dy, limiter_kind, i, B);
}

// Boundary inflow term for a domain face (cfd2d/kernels.py:278-302, 338-359):
// un = velocity into the domain, ph = value of the adjacent cell P.
CFD_HD double boundary_term(double un, double ph, double Dp, int64_t t, double val, double h) {
    const double phb = (t == 1 && un > 0.0) ? val : ph;
    double flux = un * phb;
    if (t == 1) flux = flux + (Dp * (val - ph)) / (0.5 * h);
    else if (t == 2) flux = flux + val;
    return flux / h;
}

// out(i, j) of scalar_transport for an interior cell (i in 1..nx, j in 1..ny):
// the reference accumulates the two x-face terms, then the south and north terms
// onto 0, i.e. ((west + east) + south) + north (cfd2d/kernels.py:271-391).
CFD_HD double transport_cell(const double* phi, const double* u, const double* v,
                             const uint8_t* fl, const double* diff, Grid2 g, double dx, double dy,
                             int lim, bool periodic, const ScalarBCView& bc, int obs_t,
                             double obs_v, int i, int j) {
    const int nx = g.nx, ny = g.ny;
    if (!fl[g.c(i, j)]) return 0.0;
    const double phP = phi[g.c(i, j)];
    const double DP = diff[g.c(i, j)];
    double xw = 0.0, xe = 0.0, ys = 0.0, yn = 0.0;
    // west face: index i-1 joining (i-1, i); for i == 1 the domain face (or the
    // periodic face nx joining (nx, 1))
    if (i == 1 && !periodic) {
        xw = boundary_term(u[g.u(0, j)], phP, DP, bc.bt[0][j - 1], bc.bv[0][j - 1], dx);
    } else {
        const int L = (i == 1) ? nx : i - 1;
        const int fi = (i == 1) ? nx : i - 1;
        const bool fL = fl[g.c(L, j)];
        if (fL) xw = xflux(phi, u, fl, diff, g, dx, lim, periodic, fi, L, i, j) / dx;
        else if (obs_t == 1) xw = ((DP * (obs_v - phP)) / (0.5 * dx)) / dx;
    }
    // east face: index i joining (i, i+1); for i == nx the domain face (or periodic)
    if (i == nx && !periodic) {
        xe = boundary_term(-u[g.u(nx, j)], phP, DP, bc.bt[1][j - 1], bc.bv[1][j - 1], dx);
    } else {
        const int R = (i == nx) ? 1 : i + 1;
        const bool fR = fl[g.c(R, j)];
        if (fR) xe = -(xflux(phi, u, fl, diff, g, dx, lim, periodic, i, i, R, j) / dx);
        else if (obs_t == 1) xe = ((DP * (obs_v - phP)) / (0.5 * dx)) / dx;
    }
    // south face: y face j-1 joining (j-1, j); domain face for j == 1
    if (j == 1) {
        ys = boundary_term(v[g.v(i, 0)], phP, DP, bc.bt[2][i - 1], bc.bv[2][i - 1], dy);
    } else {
        if (fl[g.c(i, j - 1)]) ys = yflux(phi, v, fl, diff, g, dy, lim, i, j - 1) / dy;
        else if (obs_t == 1) ys = ((DP * (obs_v - phP)) / (0.5 * dy)) / dy;
    }
    // north face: y face j joining (j, j+1); domain face for j == ny
    if (j == ny) {
        yn = boundary_term(-v[g.v(i, ny)], phP, DP, bc.bt[3][i - 1], bc.bv[3][i - 1], dy);
    } else {
        if (fl[g.c(i, j + 1)]) yn = -(yflux(phi, v, fl, diff, g, dy, lim, i, j) / dy);
        else if (obs_t == 1) yn = ((DP * (obs_v - phP)) / (0.5 * dy)) / dy;
    }
    return ((xw + xe) + ys) + yn;
}

// ---------------------------------------------------------------- scalar ghosts
// ghost value for one boundary cell (cfd2d/models.py:150-155)
CFD_HD double scalar_ghost(double inner, int64_t code, double val, double h, double D) {
    if (code == 1) return 2.0 * val - inner;
    if (code == 2) return inner + (val * h) / D;
    return inner;
}

// ---------------------------------------------------------------- k-omega SST
struct SSTConst {
    double a1, beta_star, sk1, so1, beta1, gamma1, sk2, so2, beta2, gamma2;
};
CFD_HD SSTConst sst_const() {
    // cfd2d/turbulence.py:185-188
    SSTConst c;
    c.a1 = 0.31; c.beta_star = 0.09;
    c.sk1 = 0.85; c.so1 = 0.5; c.beta1 = 0.075; c.gamma1 = 5.0 / 9.0;
    c.sk2 = 1.0; c.so2 = 0.856; c.beta2 = 0.0828; c.gamma2 = 0.44;
    return c;
}

// S^2 = 2 S_ij S_ij at the centre of cell (i, j) (cfd2d/turbulence.py:89-100).
CFD_HD double strain2(const double* u, const double* v, Grid2 g, double dx, double dy, int i,
                      int j) {
    const double dudx = (u[g.u(i, j)] - u[g.u(i - 1, j)]) / dx;
    const double dvdy = (v[g.v(i, j)] - v[g.v(i, j - 1)]) / dy;
    // shear at node (a, b) = (u[a,b+1]-u[a,b])/dy + (v[a+1,b]-v[a,b])/dx; this cell uses
    // nodes (i-1, j-1), (i, j-1), (i-1, j), (i, j)
#define CFD_SH(a, b) ((u[g.u(a, (b) + 1)] - u[g.u(a, b)]) / dy + (v[g.v((a) + 1, b)] - v[g.v(a, b)]) / dx)
    const double s00 = CFD_SH(i - 1, j - 1);
    const double s10 = CFD_SH(i, j - 1);
    const double s01 = CFD_SH(i - 1, j);
    const double s11 = CFD_SH(i, j);
#undef CFD_SH
    const double sh2 = 0.25 * (((s00 * s00 + s10 * s10) + s01 * s01) + s11 * s11);
    return 2.0 * (dudx * dudx + dvdy * dvdy) + sh2;
}

}  // namespace cfd
