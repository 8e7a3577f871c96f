/*
 * cfd2d_b200.h - C ABI of the B200 (sm_100a) projection-step library.
 *
 * Every entry point takes plain pointers, sizes and a CUDA stream (as void*),
 * launches asynchronously on that stream and returns an int status
 * (CFD2D_OK or a negative CFD2D_E* code). Array pointers are DEVICE pointers
 * unless a comment says otherwise. Arrays use the reference's layout: cell
 * (i, j) with one ghost layer, row-major with j contiguous; p-like fields are
 * (nx+2) x (ny+2), u is (nx+1) x (ny+2), v is (nx+2) x (ny+1), float64;
 * fluid flags are one byte per cell (nonzero = fluid).
 *
 * The reference is the Python package cfd2d (kaeptnzursee1910/CFD-); each
 * declaration names the reference interface it replaces as file:line.
 */
#ifndef CFD2D_B200_H
#define CFD2D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define CFD2D_OK 0
#define CFD2D_E_ARG (-1)        /* invalid argument (sizes, null pointers) */
#define CFD2D_E_CUDA (-2)       /* a CUDA runtime call failed */
#define CFD2D_E_CAPACITY (-3)   /* problem larger than a fixed-capacity path supports */
#define CFD2D_E_UNSUPPORTED (-4)

/* device-side status bits, written into cfd2d_state.status by the kernels */
#define CFD2D_S_NONFINITE 1     /* residual not finite or > 1e8 (FloatingPointError) */
#define CFD2D_S_CG_MAXITER 2    /* CG stopped at maxiter (reference: warnings.warn) */
#define CFD2D_S_BARRIER_TIMEOUT 4 /* a bounded inter-block wait gave up */
#define CFD2D_S_COMPONENTS 8    /* more Neumann components than the solver tracks */
#define CFD2D_S_VOF_SUBSTEPS 16 /* the VOF transport needed more sub-steps than queued */

/* side order used by every per-side array: left, right, bottom, top */
#define CFD2D_LEFT 0
#define CFD2D_RIGHT 1
#define CFD2D_BOTTOM 2
#define CFD2D_TOP 3

/* boundary kinds, cfd2d/boundary.py:31 */
#define CFD2D_BC_NOSLIP 0
#define CFD2D_BC_SLIP 1
#define CFD2D_BC_INFLOW 2
#define CFD2D_BC_OUTFLOW 3
#define CFD2D_BC_PERIODIC 4

#define CFD2D_MAX_COMPONENTS 16
#define CFD2D_MAX_SCALARS 4
#define CFD2D_HIST_FIELDS 10

/* Device-resident per-simulation state: everything that changes from step to
 * step lives here so that a captured CUDA graph of one step can be replayed. */
typedef struct cfd2d_state {
    double t, dt, dt_old, gamma;
    double ab_a, ab_b;        /* AB2 weights of this step */
    double flow_force;        /* cfd2d/solver.py:152 */
    double residual;          /* max|du|/dt, cfd2d/solver.py:390-392 */
    double dt_fixed;          /* > 0: fixed step (cfd2d/solver.py:210-211) */
    double t_end;             /* run(): clamp the last step to land on t_end */
    double steady_tol;        /* run(): stop when residual < steady_tol after 10 steps */
    double bulk_du;           /* flow-rate correction of this step */
    int64_t n;                /* steps taken */
    int64_t max_steps;        /* run(): stop after this many steps (<0: none) */
    int32_t have_old;         /* hu_old valid (AB2 after the first step) */
    int32_t status;           /* CFD2D_S_* bits (sticky) */
    int32_t active;           /* this step runs (0 after a stop condition) */
    int32_t cg_iters;         /* iterations of the last pressure solve */
    int32_t cg_iters_step;    /* iterations of this step's main solve */
    int32_t error_step;       /* step number at which status first became nonzero */
    int32_t stop_reason;      /* 0 none, 1 t_end, 2 max_steps, 3 steady */
    int32_t pad0;
    /* reduction slots (bit patterns of non-negative doubles, max via atomicMax) */
    unsigned long long umax_bits, vmax_bits, numax_bits, numin_bits;
    unsigned long long dmax_bits[CFD2D_MAX_SCALARS];
    unsigned long long du_bits, dv_bits, div_bits;
    unsigned int ticket[8];   /* last-block-done counters */
} cfd2d_state;

/* Pressure operator on the interior cells (cfd2d/pressure.py:32-140), built by
 * the host in the reference's accumulation order. */
typedef struct cfd2d_poisson {
    int nx, ny, periodic;
    double dx2, dy2;          /* 1/dx^2, 1/dy^2 */
    const double* diag;       /* nx*ny, 0 in solid cells */
    const double* dinv;       /* nx*ny, 1/diag in fluid cells, 0 in solids */
    const uint8_t* nbr;       /* nx*ny: bit0 W, bit1 S, bit2 N, bit3 E coupled, bit7 fluid */
    const int16_t* label;     /* nx*ny: Neumann-component index (0..ncomp-1) or -1 */
    int ncomp;                /* Neumann-only components (mean removed before/after) */
    const double* comp_count; /* ncomp cell counts (as double) */
    double* x0;               /* nx*ny warm start, updated by every solve */
    double* work;             /* scratch, cfd2d_pcg_workspace_bytes() */
    size_t work_bytes;
    int cluster;              /* CTAs of the on-chip solver (0 = grid-persistent solver) */
    int mixed;                /* 1: FP32 iterations with FP64 residual refinement and FP64
                                 reductions (on-chip solver only; no reference counterpart);
                                 0: the FP64 scipy-form iteration */
    int grid_ctas;            /* cluster == 0: 0 = cooperative launch over every SM,
                                 each CTA holding a slab of rows in shared memory when the
                                 slabs fit (constant coefficients, even ny <= 1024), else
                                 vectors in the workspace; -2 = the slabs with one grid
                                 reduction per iteration (Chronopoulos-Gear recurrence instead
                                 of scipy's two); -1 = over every SM with the vectors
                                 in the workspace; 16 = one 16-CTA cluster (vectors in the
                                 workspace, cluster barriers), which leaves the other SMs to
                                 other solves. cluster > 0: -2 = the on-chip solver with one
                                 cluster reduction per iteration (same recurrence; FP64,
                                 constant coefficients, even ny, when its 14 ny extra
                                 doubles per CTA fit), any other value its default form */
    const double* bx;         /* NULL: constant coefficients. Else div(b grad p) with face
                                 coefficients b = 1/rho (cfd2d/pressure.py:187-244):
                                 bx (nx+1)(ny+2) on the x faces, periodic face nx coupling
                                 cells nx-1 and 0; needs cluster == 0 and diag/dinv of the
                                 variable operator */
    const double* by;         /* (nx+2)(ny+1) on the y faces */
} cfd2d_poisson;

/* One scalar transport equation (cfd2d/models.py:73-250). */
typedef struct cfd2d_scalar {
    double* phi;              /* (nx+2)(ny+2) */
    double* diff;             /* (nx+2)(ny+2) */
    double* rhs;              /* (nx+2)(ny+2) transport output */
    const int64_t* bt[4];     /* per-side BC codes: 0 zero-gradient, 1 fixed, 2 flux */
    const double* bv[4];      /* per-side BC values */
    int limiter;              /* cfd2d/kernels.py:33 */
    int obs_t;                /* 1: obstacle fixed value obs_v in the transport */
    double obs_v;
    double D0;                /* molecular diffusivity */
    double turb_div;          /* > 0: diff = D0 + nu_t / turb_div each step */
    int has_lower, has_upper;
    double lower, upper;
    int source;               /* 0 none, 1 SST k, 2 SST omega */
    int pad;
} cfd2d_scalar;

/* k-omega SST model data (cfd2d/turbulence.py:166-325). */
typedef struct cfd2d_sst {
    double* S2;               /* nx*ny strain rate squared */
    double* F1;               /* nx*ny */
    double* cross;            /* nx*ny */
    double* Pk;               /* nx*ny production (k source) */
    const double* d;          /* nx*ny wall distance (>= 1e-12) */
    const uint8_t* wall_adj;  /* nx*ny */
    const double* w_wall;     /* nx*ny */
    int k_index, w_index;     /* scalar slots of k and omega */
} cfd2d_sst;

/* LES Smagorinsky model data (cfd2d/turbulence.py:130-160): nu_t = l^2 |S| on fluid
 * cells, l = min(C_s sqrt(dx dy), kappa d) fixed when the model attaches. */
typedef struct cfd2d_smagorinsky {
    const double* l2;         /* nx*ny squared length scale l^2 */
} cfd2d_smagorinsky;

/* Two-phase VOF model data (cfd2d/vof.py:140-306): volume fraction transport with
 * interface compression, CSF surface tension, mixture density and viscosity, and
 * the variable-density projection (cfd2d/solver.py:267-321). */
typedef struct cfd2d_vof {
    double* alpha;            /* (nx+2)(ny+2) volume fraction of phase 1 */
    double* alpha_tmp;        /* (nx+2)(ny+2) */
    double* rho;              /* (nx+2)(ny+2) mixture density; the mixture dynamic viscosity
                                 is held in sim->nu_eff (cfd2d/vof.py:222-227) */
    double* smooth;           /* (nx+2)(ny+2) smoothed alpha of the curvature */
    double* nrm;              /* 2 (nx+1)(ny+1) interface normals at the nodes (x, then y) */
    double* kappa;            /* (nx+2)(ny+2) curvature, 0 on the ghost layer */
    double* bx;               /* (nx+1)(ny+2) face coefficients 2 / (rho_L + rho_R) */
    double* by;               /* (nx+2)(ny+1) */
    double* vdiag;            /* nx*ny diagonal of the variable-coefficient operator */
    double* vdinv;            /* nx*ny */
    double* scal;             /* 4 doubles: largest face coefficient, sub-steps, sub-step length */
    const uint8_t* vflags;    /* nx*ny: bit0-3 outflow (Dirichlet) at the left/right/bottom/top
                                 side, bit4 pinned cell of a Neumann component */
    double rho1, rho2, mu1, mu2;
    double sigma, c_alpha, cfl, alpha_in;
    double dt_limit;          /* capillary and gravity-wave limit (cfd2d/vof.py:273-284), 0: none */
    double rtol;              /* relative residual of the variable-coefficient solve */
    int maxiter;
    int nsub_max;             /* transport sub-steps queued per step; more needed sets
                                 CFD2D_S_VOF_SUBSTEPS */
} cfd2d_vof;

/* Per-step model monitors (the model part of cfd2d/solver.py:441-443 _record): one
 * value per monitor and step, written into sim->mon_ring after the step. */
#define CFD2D_MAX_MONITORS 12
#define CFD2D_MONITOR_SCRATCH (2 * CFD2D_MAX_MONITORS * 296)
#define CFD2D_MON_SUM_FLUID 0     /* (sum of data over fluid cells) dx dy: ScalarField.total,
                                     VOF volume (cfd2d/models.py:221-224, vof.py:229-231) */
#define CFD2D_MON_MEAN_FLUID 1    /* mean of data over fluid cells (np.nanmean of cell()) */
#define CFD2D_MON_MAX_ALL 2       /* max of data over all (nx+2)(ny+2) cells (nu_t_max) */
#define CFD2D_MON_NUSSELT 3       /* |mean wall flux of scalar `slot` at side `side`| / param
                                     (cfd2d/models.py:226-250, 407-412) */
#define CFD2D_MON_VOLUME_ERROR 4  /* (sum of data over fluid cells) dx dy / max(param, 1e-300) - 1 */
#define CFD2D_MON_FRONT_X 5       /* right face of the last cell of the first row with data > 0.5,
                                     0 if none (cfd2d/vof.py:292-294) */
#define CFD2D_MON_HEIGHT_LEFT 6   /* top face of the last cell of the first column with data > 0.5 */

typedef struct cfd2d_monitor {
    int kind;                 /* CFD2D_MON_* */
    int slot;                 /* NUSSELT: scalar slot */
    int side;                 /* NUSSELT: CFD2D_LEFT .. CFD2D_TOP */
    int pad;
    const double* data;       /* padded (nx+2)(ny+2) cell array */
    double param;
} cfd2d_monitor;

/* A whole simulation: geometry, boundary data, device fields and parameters.
 * Filled by the host once; every pointer is a device pointer. */
typedef struct cfd2d_sim {
    int nx, ny;
    double dx, dy;
    int periodic;
    int scheme_ab2;           /* 1 AB2, 0 explicit Euler */
    int gamma_auto;
    double gamma_fixed;
    double tau;
    double nu;
    double body_fx, body_fy;
    int has_flow_rate;
    double flow_rate;
    double flow_count;        /* number of fluid u faces in columns 1..nx (bulk mean) */
    int variable_viscosity;
    int compute_forces;
    int has_solid;            /* interior solids exist (flow-rate re-projection) */
    int bc_kind[4];
    double bc_vel[4];
    const double* inflow[4];  /* inflow values per side (NULL if not inflow) */
    const uint8_t* open[4];   /* open masks: left/right length ny, bottom/top length nx */
    const uint8_t* fluid;     /* (nx+2)(ny+2) */
    double *u, *v, *p, *F, *G, *hu, *hv, *u_prev, *v_prev, *nu_eff, *nu_t;
    cfd2d_poisson pcg;
    double cg_rtol;
    int cg_maxiter;
    int nscalars;
    cfd2d_scalar scalars[CFD2D_MAX_SCALARS];
    double scalar_dtlim_const[CFD2D_MAX_SCALARS]; /* > 0: constant diffusion dt limit */
    int thermal_index;        /* scalar slot of the Boussinesq temperature, -1 none */
    double gx, gy, T_ref;     /* buoyancy beta*g and reference temperature */
    int sst_on;
    cfd2d_sst sst;
    int smag_on;              /* Smagorinsky nu_t before the momentum update */
    cfd2d_smagorinsky smag;
    int vof_on;               /* two-phase VOF with variable density */
    cfd2d_vof vof;
    int nmon;                 /* model monitors recorded after every step */
    cfd2d_monitor mon[CFD2D_MAX_MONITORS];
    double* mon_ring;         /* hist_cap records of CFD2D_MAX_MONITORS doubles */
    double* mon_part;         /* scratch, CFD2D_MONITOR_SCRATCH doubles */
    cfd2d_state* state;
    double* red;              /* reduction scratch, cfd2d_sim_scratch_doubles() */
    double* hist;             /* history ring: hist_cap records of CFD2D_HIST_FIELDS doubles:
                                 t, dt, residual, max|div u|, kinetic energy, fx, fy,
                                 flow_force, CG iterations, gamma */
    int hist_cap;
    double* p_tmp;            /* (nx+2)(ny+2) scratch: pressure of the flow-rate re-projection */
} cfd2d_sim;

/* ---- kernel-level entry points (drop-in for cfd2d/kernels.py) ------------ */

/* hu, hv = diffusion - convection on fluid faces; zero elsewhere. hu and hv must
 * not overlap any input array. nu is a cell field of (nx+2)*(ny+2) doubles, as the
 * reference's; with variable = 0 only nu[1][1] is read.
 * Replaces cfd2d/kernels.py:44-46 momentum_tendencies(u, v, fluid, nx, ny, dx,
 * dy, nu, variable, gamma, periodic, hu, hv, rho, var_density). */
int cfd2d_momentum_tendencies(const double* u, const double* v, const uint8_t* fluid, int nx,
                              int ny, double dx, double dy, const double* nu, int variable,
                              double gamma, int periodic, double* hu, double* hv,
                              const double* rho, int var_density, void* stream);

/* Velocities on faces touching solid cells, in place.
 * Replaces cfd2d/kernels.py:158-159 obstacle_bc(u, v, fluid, nx, ny, periodic). */
int cfd2d_obstacle_bc(double* u, double* v, const uint8_t* fluid, int nx, int ny, int periodic,
                      void* stream);

/* out = -div(u phi) + div(D grad phi) on fluid cells (TVD faces); out must not
 * overlap any input array.
 * Replaces cfd2d/kernels.py:254-256 scalar_transport(phi, u, v, fluid, nx, ny,
 * dx, dy, diff, limiter, periodic, bt_l, bv_l, bt_r, bv_r, bt_b, bv_b, bt_t,
 * bv_t, obs_t, obs_v, out). bt_* are int64 arrays, bv_* float64 arrays of
 * length ny (left/right) or nx (bottom/top). */
int cfd2d_scalar_transport(const double* phi, const double* u, const double* v,
                           const uint8_t* fluid, int nx, int ny, double dx, double dy,
                           const double* diff, int limiter, int periodic, const int64_t* bt_l,
                           const double* bv_l, const int64_t* bt_r, const double* bv_r,
                           const int64_t* bt_b, const double* bv_b, const int64_t* bt_t,
                           const double* bv_t, int obs_t, double obs_v, double* out,
                           void* stream);

/* Domain boundary values on u and v (ghost cells and boundary faces).
 * Replaces cfd2d/boundary.py:143 DomainBoundary.apply(u, v). */
int cfd2d_domain_bc(const cfd2d_sim* sim, double* u, double* v, void* stream);

/* Cell-centre obstacle masks (nx, ny), one byte per cell, bit-exact with the
 * reference's float64 expressions. Replace cfd2d/geometry.py:17 circle,
 * :25 ellipse (cos/sin of the angle are passed in, computed by numpy as in the
 * reference) and :35 rectangle (corners already sorted). */
int cfd2d_mask_circle(int nx, int ny, double dx, double dy, double xc, double yc, double r,
                      uint8_t* mask, void* stream);
int cfd2d_mask_ellipse(int nx, int ny, double dx, double dy, double xc, double yc, double a,
                       double b, double cos_phi, double sin_phi, uint8_t* mask, void* stream);
int cfd2d_mask_rectangle(int nx, int ny, double dx, double dy, double xa, double ya, double xb,
                         double yb, uint8_t* mask, void* stream);

/* Closed polygon with npts vertices (device arrays px, py; the last vertex joins the
 * first): cell centres inside by the crossing test. Replaces cfd2d/geometry.py:43
 * polygon(grid, points) (matplotlib Path.contains_points); NACA profiles
 * (geometry.py:105 naca4) are polygons of their outline. */
int cfd2d_mask_polygon(int nx, int ny, double dx, double dy, const double* px, const double* py, int npts,
                       uint8_t* mask, void* stream);

/* Image obstacle: `solid` is the h x w solid-pixel bitmap (row 0 at the top, device),
 * placed on [x0, x0 + width] x [y0, y0 + height]; each cell centre takes its pixel.
 * Replaces the pixel lookup of cfd2d/geometry.py:119 from_image (the image is decoded
 * and thresholded on the host). */
int cfd2d_mask_image(int nx, int ny, double dx, double dy, const uint8_t* solid, int h, int w, double x0, double y0,
                     double width, double height, uint8_t* mask, void* stream);

/* ---- pressure Poisson (drop-in for cfd2d/pressure.py) -------------------- */

/* Bytes of scratch the solver needs for an nx x ny grid (cfd2d_poisson.work) on the
 * current device (its partial-sum arrays are sized by the device's SM count). */
size_t cfd2d_pcg_workspace_bytes(int nx, int ny);

/* Choose the solver variant for this grid on the current device: the number of
 * CTAs of the on-chip (cluster) solver, or 0 for the grid-persistent solver. */
int cfd2d_pcg_plan(int nx, int ny, int* cluster);

/* Solve Lap(p) = rhs on the fluid cells: Neumann-component mean removal, sign
 * flip, Jacobi-preconditioned CG in scipy's iteration form from the warm start
 * op->x0 (updated), then per-component mean removal of p. rhs and p are nx*ny
 * arrays (p is 0 in solid cells). iters_out (device int32, may be NULL) gets
 * the iteration count, status_out (device int32, may be NULL) gets
 * CFD2D_S_CG_MAXITER / CFD2D_S_BARRIER_TIMEOUT bits.
 * Replaces cfd2d/pressure.py:143 PressureSolver.solve(rhs) with
 * method="cg" (scipy.sparse.linalg.cg at cfd2d/pressure.py:171). */
int cfd2d_pressure_solve(const cfd2d_poisson* op, const double* rhs, double* p, double rtol,
                         int maxiter, int32_t* iters_out, int32_t* status_out, void* stream);

/* ---- whole projection step (drop-in for cfd2d/solver.py) ----------------- */

/* Doubles of reduction scratch a simulation needs (cfd2d_sim.red). */
size_t cfd2d_sim_scratch_doubles(int nx, int ny);

/* Boundary conditions on u, v: domain sides then obstacle faces.
 * Replaces cfd2d/solver.py:189 Simulation._apply_bc(). */
int cfd2d_sim_apply_bc(const cfd2d_sim* sim, void* stream);

/* Projection of the initial field with dt = 1, p reset to 0 afterwards.
 * Replaces cfd2d/solver.py:195 Simulation._project_initial() (the caller skips
 * it when u and v are zero, as the reference does). */
int cfd2d_sim_project_initial(const cfd2d_sim* sim, void* stream);

/* One projection time step, all on the device; skipped entirely when
 * state->active is 0 at its start (run() stop conditions).
 * Replaces cfd2d/solver.py:326 Simulation.step(). */
int cfd2d_sim_step(const cfd2d_sim* sim, void* stream);

/* Fill the ghost and solid cells of scalar slot `slot` from its interior values.
 * Replaces cfd2d/models.py:139 ScalarField.fill_ghosts(). */
int cfd2d_sim_scalar_fill_ghosts(const cfd2d_sim* sim, int slot, void* stream);

/* k-omega SST blending functions, nu_t, blended diffusivities and nu_eff.
 * Replaces cfd2d/turbulence.py:262 KOmegaSST.pre_momentum(sim). */
int cfd2d_sim_sst_pre_momentum(const cfd2d_sim* sim, void* stream);

/* Smagorinsky nu_t = l^2 sqrt(S^2) on fluid cells, its ghost values and nu_eff.
 * Replaces cfd2d/turbulence.py:149 Smagorinsky.pre_momentum(sim). */
int cfd2d_sim_smagorinsky_pre_momentum(const cfd2d_sim* sim, void* stream);

/* Bytes of device workspace cfd2d_sim_wall_distance needs for an nx x ny grid. */
size_t cfd2d_wall_distance_workspace_bytes(int nx, int ny);

/* Distance of every cell centre to the nearest wall face, (nx+2)(ny+2) doubles into
 * `dist`: the exact Euclidean distance transform of the wall cells (interior solids
 * and the ghost layer of no-slip sides; periodic in x when sim->periodic) minus half
 * a cell, at least half a cell, 0 on non-fluid cells, 1e6 everywhere when the grid
 * has no wall. Reads sim->nx, ny, dx, dy, periodic, bc_kind and fluid only.
 * Replaces cfd2d/turbulence.py:43 wall_distance(sim) (scipy.ndimage
 * distance_transform_edt). */
int cfd2d_sim_wall_distance(const cfd2d_sim* sim, double* dist, void* work, size_t work_bytes, void* stream);

/* One explicit, conservative transport step of the volume fraction with interface
 * compression: out = alpha after dt (out must not be alpha). Replaces
 * cfd2d/vof.py:36 vof_advect(a, u, v, fluid, nx, ny, dx, dy, dt, c_alpha, periodic,
 * a_in, out) with the same arguments (device arrays). */
int cfd2d_vof_advect(const double* a, const double* u, const double* v, const uint8_t* fluid, int nx, int ny,
                     double dx, double dy, double dt, double c_alpha, int periodic, double a_in, double* out,
                     void* stream);

/* Ghost and solid values of sim->vof.alpha, then the mixture density and viscosity.
 * Replaces cfd2d/vof.py:222 VOF._update_properties(). */
int cfd2d_sim_vof_properties(const cfd2d_sim* sim, void* stream);

/* Capture nsteps consecutive calls of cfd2d_sim_step on `stream` (a created,
 * non-default stream) into an instantiated CUDA graph returned as an opaque
 * handle; cfd2d_graph_launch replays it, cfd2d_graph_destroy frees it. The
 * graph reads every step-varying scalar from sim->state, so it may be replayed
 * any number of times while the device buffers named in *sim stay valid. */
int cfd2d_graph_capture_steps(const cfd2d_sim* sim, int nsteps, void* stream, void** graph_out);
int cfd2d_graph_launch(void* graph, void* stream);
int cfd2d_graph_destroy(void* graph);

/* As cfd2d_graph_capture_steps; with events != NULL (four cudaEvent_t, only for
 * nsteps == 1) the graph records them at step start, before and after the main
 * pressure solve, and at step end. kernel_nodes (may be NULL) receives the number
 * of kernel launches in the graph. */
int cfd2d_graph_capture_steps_ex(const cfd2d_sim* sim, int nsteps, void* stream, void* const* events,
                                 void** graph_out, int* kernel_nodes);

/* Timing events for the measurement harness (cudaEvent_t as void*). */
int cfd2d_events_create(int n, void** events);
int cfd2d_events_destroy(int n, void** events);
int cfd2d_event_elapsed_ms(void* start, void* end, float* ms);

/* ---- split step, for an external pressure solver ------------------------ */

/* First part of cfd2d_sim_step: boundary conditions, model pre-momentum hooks,
 * time step and predictor F, G (cfd2d/solver.py:326-368). */
int cfd2d_sim_step_begin(const cfd2d_sim* sim, void* stream);

/* Second part: with sim->p holding the pressure of this step, the correction,
 * boundary conditions, flow-rate control, scalar transport and the end-of-step
 * record (cfd2d/solver.py:277-403). */
int cfd2d_sim_step_finish(const cfd2d_sim* sim, void* stream);

/* y = A x for the pressure operator (nx*ny vectors, solid entries 0), rows summed
 * in increasing column order. No reference counterpart (scipy's A @ x). */
int cfd2d_poisson_matvec(const cfd2d_poisson* op, const double* x, double* y, void* stream);

/* Pressure solve that also records the iterate x every `every` iterations into
 * snap (up to max_snaps vectors of nx*ny), for harvesting training pairs of the
 * learned preconditioner; otherwise as cfd2d_pressure_solve. Grid-persistent
 * solver only (op->cluster == 0). No reference counterpart. */
int cfd2d_pressure_solve_snapshots(const cfd2d_poisson* op, const double* rhs, double* p, double rtol,
                                   int maxiter, double* snap, int every, int max_snaps, int32_t* iters_out,
                                   int32_t* status_out, void* stream);

/* ---- pressure solve without device allocation (no counterpart in the reference)
 *
 * For callers that cannot provide cfd2d_poisson.work: a C or ctypes host that owns
 * no device allocator, or a time loop that must not call cudaMalloc/cudaFree
 * between steps (both can synchronise the device). Same arguments, results and
 * error codes as cfd2d_pressure_solve, always on the grid-persistent solver as a
 * cooperative launch over every SM: op->cluster, op->grid_ctas, op->work and
 * op->work_bytes are ignored; every other field of *op is used as by
 * cfd2d_pressure_solve (constant or variable coefficients, Neumann components).
 * Its scratch is a static device array of the library (8.2 MiB per device), so
 * nothing is allocated.
 *  - Grids above CFD2D_STATIC_MAX_CELLS cells return CFD2D_E_CAPACITY.
 *  - The first call on each device looks the array up (cudaGetSymbolAddress, which
 *    can load the library's module on that device): make it outside any stream
 *    capture, with that device current. The address is kept for the life of the
 *    process: a cudaDeviceReset (or anything else that destroys the device's
 *    primary context) invalidates it, and the entry point must not be called on
 *    that device afterwards.
 *  - Nothing has to start at zero: each call clears the solver's barrier words on
 *    `stream` before its launch, and the solver writes the rest before reading it.
 *  - All calls on one device share the array: two calls whose kernels can overlap
 *    (different streams with no ordering between them) race on it and give wrong
 *    results. Order them on one stream or with events. */
#define CFD2D_STATIC_MAX_CELLS 262144 /* e.g. 512 x 512 */
int cfd2d_pressure_solve_static(const cfd2d_poisson* op, const double* rhs, double* p, double rtol,
                                int maxiter, int32_t* iters_out, int32_t* status_out, void* stream);

/* ---- learned Poisson preconditioner (no counterpart in the reference) ---- */
/* Activations: BF16, NHWC with 32 channels, pixel = cell (i, j) at i*W + j. */

/* Bytes of the packed weight image of one 32->32 3x3 convolution. */
size_t cfd2d_lpc_w32_bytes(void);
/* Pack w[32][32][3][3] (float32, out x in x kh x kw) into the tensor-core image. */
int cfd2d_lpc_pack_w32(const float* w, void* image, void* stream);
/* Pack the data-gradient convolution of the same layer (channels swapped, taps
 * mirrored): cfd2d_lpc_conv32 with this image maps dy to dx on the tensor cores. */
int cfd2d_lpc_pack_w32_adjoint(const float* w, void* image, void* stream);
/* y = act(conv3x3(x, w) + bias (+ skip)) masked; tcgen05 implicit GEMM. err: device
 * int set to 1 if the bounded wait for the accumulator gave up (may be NULL). */
int cfd2d_lpc_conv32(const void* x, const void* image, const float* bias, const void* skip,
                     const uint8_t* mask, void* y, int H, int W, int relu, int32_t* err, void* stream);
/* CUDA-core 3x3 convolution for cin, cout in {1, 32}: x and y FP32 or BF16
 * (x_bf16, y_bf16 flags); transposed != 0 applies the adjoint (data gradient). */
int cfd2d_lpc_conv(int cin, int cout, const void* x, int x_bf16, const float* w, const float* bias,
                   const uint8_t* mask, void* y, int y_bf16, int H, int W, int relu, int transposed,
                   void* stream);
int cfd2d_lpc_pool2(const void* x, void* y, int H, int W, void* stream);
int cfd2d_lpc_pool_mask(const uint8_t* m, uint8_t* mc, int H, int W, void* stream);
/* y = scale * upsample(coarse) + skip (nearest, (H+1)/2 x (W+1)/2 -> H x W, 32 channels,
 * BF16); the backward pass writes dcoarse = scale * (sum of the children of dy). */
int cfd2d_lpc_upadd(const void* coarse, const void* skip, void* y, int H, int W, float scale, void* stream);
int cfd2d_lpc_relu_bwd(const float* dy, const void* y, const uint8_t* mask, float* g, int npix, int ch,
                       int relu, void* stream);
int cfd2d_lpc_upadd_bwd(const float* dy, float* dcoarse, int H, int W, float scale, void* stream);
int cfd2d_lpc_pool_bwd(const float* dcoarse, float* dfine, int H, int W, void* stream);
size_t cfd2d_lpc_conv_dw_partial_floats(int cin, int cout, int H, int W, int pix_per_block);
/* weight and bias gradient: out = [dw (cout*cin*9), db (cout)] */
int cfd2d_lpc_conv_dw(int cin, int cout, const void* x, int x_bf16, const float* g, int H, int W,
                      int pix_per_block, float* partial, float* out, void* stream);

/* ---- flexible CG around a variable preconditioner (no reference counterpart) */
typedef struct cfd2d_fcg_scalars {
    double alpha, beta, rz, pq, rr, bb;
    int32_t iters;
    uint32_t ticket;
} cfd2d_fcg_scalars;

size_t cfd2d_fcg_partial_doubles(int n);
/* b = -(div(F,G)/dt) (or -rhs when rhs != NULL), r = b - A x, p_zero (may be NULL) = 0 */
int cfd2d_fcg_init(const cfd2d_poisson* op, const double* F, const double* G, const double* rhs, double dx,
                   double dy, const double* dt, double* b, double* x, double* r, double* p_zero,
                   cfd2d_fcg_scalars* s, double* partial, void* stream);
/* Notay's flexible CG with one stored direction (no reliance on r . M(r) > 0):
 * pq: q = A p, pq = p . q, alpha = (p . r) / pq;  update: x += alpha p, r -= alpha q,
 * rr = ||r||^2, iters += 1;  zr: beta = -(z . q) / pq with q = A p_old (0 when
 * first != 0, or when first < 0 and iters == 0);  dir: p = z + beta p. */
int cfd2d_fcg_pq(const cfd2d_poisson* op, const double* p, double* q, const double* r, cfd2d_fcg_scalars* s,
                 double* partial, void* stream);
int cfd2d_fcg_update(int n, double* x, double* r, const double* p, const double* q, cfd2d_fcg_scalars* s,
                     double* partial, void* stream);
int cfd2d_fcg_zr(int n, const double* z, const double* q, int first, cfd2d_fcg_scalars* s, double* partial,
                 void* stream);
int cfd2d_fcg_dir(int n, const double* z, double* p, const cfd2d_fcg_scalars* s, void* stream);
int cfd2d_fcg_net_in(int n, const double* r, const cfd2d_fcg_scalars* s, const uint8_t* mask, float* in,
                     void* stream);
/* z = ||r|| * scale * out + jacobi * r / diag (scale = h^2 of the dimensionless operator) */
int cfd2d_fcg_net_out(int n, const float* out, const double* r, const double* dinv, const uint8_t* mask,
                      const cfd2d_fcg_scalars* s, double scale, double jacobi, double* z, void* stream);
int cfd2d_fcg_scatter_p(const cfd2d_poisson* op, const double* x, double* p_padded, void* stream);

/* Device-driven flexible CG: the whole iteration runs inside one CUDA graph whose
 * WHILE node repeats the loop body (preconditioner, r.z, direction, A p, update,
 * gate) until the gate kernel stops it, so a solve needs no host round trip per
 * iteration. The control block lives in device memory. */
#define CFD2D_FCG_RUNNING 0
#define CFD2D_FCG_CONVERGED 1
#define CFD2D_FCG_MAXITER 2
#define CFD2D_FCG_STALLED 3   /* ||r|| > stall_factor * ||r|| of stall_window iterations ago */
#define CFD2D_FCG_NONFINITE 4
typedef struct cfd2d_fcg_control {
    double rtol;              /* stop when ||r|| < rtol ||b|| */
    double stall_factor;
    int32_t stall_window;
    int32_t maxiter;
    int32_t reason;           /* CFD2D_FCG_*, written by the gate */
    int32_t iters;            /* iterations done, written by the gate */
    int32_t calls;            /* gate invocations (set 0 before a solve); a hard bound
                                 on the loop independent of the iteration counter */
    int32_t pad;
    double* hist;             /* device, maxiter + 1 residual norms */
    int32_t* iters_out;       /* device, may be NULL: also receives the iteration count */
} cfd2d_fcg_control;

/* One thread: record ||r||, apply the stop tests, set the WHILE condition `handle`
 * (0 = no graph, only the tests). */
int cfd2d_fcg_gate(const cfd2d_fcg_scalars* s, cfd2d_fcg_control* ctl, uint64_t handle, void* stream);
/* x = b when ||b|| = 0 (read on the device). */
int cfd2d_fcg_zero_rhs(int n, const double* b, double* x, const cfd2d_fcg_scalars* s, void* stream);

/* Stream capture of a graph with one WHILE loop (no reference counterpart):
 * capture_begin starts a relaxed-mode capture of `stream`; capture_condition
 * creates the loop's condition (0 at every launch; a kernel captured before the
 * loop, such as cfd2d_fcg_gate, sets it); while_begin appends the WHILE node after
 * the work captured so far and starts capturing `body_stream` into the loop body,
 * which must end with a kernel that sets the condition again; while_end ends the
 * body; capture_end instantiates the graph (launch with cfd2d_graph_launch, free
 * with cfd2d_graph_destroy). No device memory may be allocated or freed while a
 * capture is open. */
int cfd2d_capture_begin(void* stream);
int cfd2d_capture_condition(void* stream, uint64_t* handle_out);
int cfd2d_capture_while_begin(void* stream, void* body_stream, uint64_t handle);
int cfd2d_capture_while_end(void* body_stream);
int cfd2d_capture_end(void* stream, void** graph_out);
/* Abandon a capture after an error (ends it and frees the partial graph). */
int cfd2d_capture_abort(void* stream);

/* ---- function objects fed from the device (drop-in for cfd2d/functions.py) ----
 * Probes, line samples, time averages and the VTK export read the device fields
 * directly: nothing copies a whole field to the host per step. */

/* Field selectors (cfd2d/visualization.py:50-73 field_data; cfd2d/solver.py:598-615
 * sample_u / sample_v). Face fields are interpolated on their own staggered grid and
 * extrapolated outside it; cell fields are NaN on solid cells and their sample
 * points are clipped to the first and last cell centre (cfd2d/functions.py:24-39). */
#define CFD2D_FIELD_U 0           /* face u, (nx+1)(ny+2) at (i dx, (j - 1/2) dy) */
#define CFD2D_FIELD_V 1           /* face v, (nx+2)(ny+1) at ((i - 1/2) dx, j dy) */
#define CFD2D_FIELD_PRESSURE 2    /* p of the cell */
#define CFD2D_FIELD_UC 3          /* mean of the two u faces (cfd2d/solver.py:526-533) */
#define CFD2D_FIELD_VC 4
#define CFD2D_FIELD_SPEED 5       /* sqrt(uc^2 + vc^2) */
#define CFD2D_FIELD_VORTICITY 6   /* mean of the 4 node vorticities (cfd2d/solver.py:569-578) */
#define CFD2D_FIELD_CELL 7        /* `data`: a padded (nx+2)(ny+2) cell array (scalar, nu_t) */
#define CFD2D_FIELD_CELL_LOG10 8  /* log10(max(data, 1e-30)) of a padded cell array */
#define CFD2D_FIELD_NODE 9        /* mean of the 4 corners of a (nx+1)(ny+1) node array (psi) */
#define CFD2D_FIELD_FLUID 10      /* 1 on fluid cells, 0 on solids (not NaN) */
#define CFD2D_MAX_FIELDS 16

typedef struct cfd2d_field {
    int kind;                 /* CFD2D_FIELD_* */
    int pad;
    const double* data;       /* CELL, CELL_LOG10, NODE: the device array; else NULL */
} cfd2d_field;

/* out[f * npts + k] = field f at (px[k], py[k]) (device arrays), bilinear
 * interpolation as scipy's RegularGridInterpolator(method="linear",
 * bounds_error=False, fill_value=None). `fields` is a host array of nfields <=
 * CFD2D_MAX_FIELDS. Replaces cfd2d/functions.py:24 sample_field(sim, field, x, y). */
int cfd2d_sample(const cfd2d_sim* sim, const cfd2d_field* fields, int nfields, const double* px,
                 const double* py, int npts, double* out, void* stream);

/* out[i ny + j] = field at interior cell (i, j), NaN on solids (FLUID: 1 or 0).
 * Replaces cfd2d/visualization.py:50 field_data(sim, field). */
int cfd2d_cell_values(const cfd2d_sim* sim, const cfd2d_field* field, double* out, void* stream);

/* Time series of a Probes object (cfd2d/functions.py:59-80): device buffers. */
typedef struct cfd2d_probe_series {
    double* t;                /* cap sample times */
    double* values;           /* cap rows of nfields * npts values (row, field, point) */
    int64_t* count;           /* [0] rows written, [1] step number of the last row,
                                 [2] 1 when a row did not fit (the host sizes cap ahead) */
    int cap;
    int every;                /* record when n % every == 0 */
} cfd2d_probe_series;

/* Append one row after a step: skipped when no step ran since the last row or
 * n % every != 0 (reads t and n from sim->state). One block, no host sync.
 * Replaces cfd2d/functions.py:70 Probes.execute(sim). */
int cfd2d_probe_record(const cfd2d_sim* sim, const cfd2d_field* fields, int nfields, const double* px,
                       const double* py, int npts, const cfd2d_probe_series* series, void* stream);

/* Time sums of the cell velocity and pressure (cfd2d/functions.py:180-224). */
typedef struct cfd2d_field_average {
    double t_start;           /* accumulate once t >= t_start */
    double* sum;              /* 3 nx*ny: uc, vc, p (NaN on solids), sum of value * dt */
    double* sum2;             /* 3 nx*ny: sum of value * value * dt */
    double* T;                /* device [0] summed time, [1] step number of the last sum (as double) */
} cfd2d_field_average;

/* Add this step's fields (skipped before t_start or when no step ran since the
 * last call). Replaces cfd2d/functions.py:189 FieldAverage.execute(sim). */
int cfd2d_field_average_accumulate(const cfd2d_sim* sim, const cfd2d_field_average* avg, void* stream);

/* Stream function psi, (nx+1)(ny+1) node values (cfd2d/solver.py:580-596, the same
 * running sums in the same order). */
int cfd2d_streamfunction(const cfd2d_sim* sim, double* psi, void* stream);

/* VTK payload (cfd2d/functions.py:244-287 write_vtk): big-endian float32, cells in
 * VTK order (x fastest), NaN written as 0. `out` receives the velocity vectors
 * (uc, vc, 0 per cell; 12 nx ny bytes) followed by one block of 4 nx ny bytes per
 * field. The host writes the text header lines around these blocks. */
int cfd2d_vtk_pack(const cfd2d_sim* sim, const cfd2d_field* fields, int nfields, uint8_t* out, void* stream);

/* Self-test of the bounded grid barrier the persistent solvers use (no reference
 * counterpart): one block runs it on the counter bar[0] as given, as if bar[1] CTAs
 * (at least 1) took part, and writes 1 to *ok_out when it passed and 0 when it gave
 * up. With bar[0] = 0 and bar[1] = 1 the single block is the last to arrive and passes
 * at once; with bar[1] > 1 the others never arrive, and after its spin limit (about a
 * second) it sets CFD2D_S_BARRIER_TIMEOUT in *status and returns, leaving the context
 * usable. */
int cfd2d_barrier_selftest(unsigned int* bar, int* status, int* ok_out, void* stream);

/* Thread-block shape (tx along j, ty along i) of the row kernels: which = 0 the
 * momentum_tendencies drop-in, 1 the step's row kernels (predictor, correction,
 * turbulence, scalar update and ghosts). tx a multiple of 16, tx * ty <= 256. Every
 * thread computes its own cells, so results do not depend on the shape; captured
 * step graphs keep the shape they were captured with. Default 32 x 8. No reference
 * counterpart: the knob of the tile autotuner (cfd2d_b200.autotune). */
int cfd2d_set_tile(int which, int tx, int ty);
int cfd2d_get_tile(int which, int* tx, int* ty);

/* Library version string (host memory, static). */
const char* cfd2d_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CFD2D_B200_H */
