// capi.cu - the extern "C" entry points declared in include/cfd2d_b200.h.
//
// Thin wrappers: argument checks, launch configuration, and the sequence of
// stage kernels that makes up one projection step (cfd2d/solver.py:326-403).
#include <cuda_runtime.h>

#include "../../include/cfd2d_b200.h"
#include "kernels.cuh"
#include "pcg.cuh"

using namespace cfd;

namespace {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }
inline int status_of(cudaError_t e) { return e == cudaSuccess ? CFD2D_OK : CFD2D_E_CUDA; }
#define CFD_TRY(x)                                   \
    do {                                             \
        cudaError_t e_ = (x);                        \
        if (e_ != cudaSuccess) return CFD2D_E_CUDA;  \
    } while (0)

bool grid_ok(int nx, int ny) { return nx >= 4 && ny >= 4 && (long long)(nx + 2) * (ny + 2) < (1LL << 31); }

// Main or auxiliary pressure projection inside a step: rhs = div(F, G)/dt.
int project(const cfd2d_sim* sim, double* p_out, bool unit_dt, bool main_solve, cudaStream_t s) {
    PcgLaunch L = {};
    L.op = sim->pcg;
    if (sim->vof_on) {
        // variable density: div(b grad p) with b = 1/rho on the faces, solved to the
        // tolerance of a direct solve (cfd2d/pressure.py:187-244 uses spsolve)
        const cfd2d_vof& V = sim->vof;
        L.op.bx = V.bx;
        L.op.by = V.by;
        L.op.diag = V.vdiag;
        L.op.dinv = V.vdinv;
        L.op.mixed = 0;
        // the on-chip solver of the plan when the four coefficient arrays fit beside it
        if (L.op.cluster > 0 && !pcg_var_cluster_fits(sim->nx, sim->ny, L.op.cluster)) L.op.cluster = 0;
        if (L.op.cluster == 0 && (long long)sim->nx * sim->ny <= 262144) L.op.grid_ctas = 16;
    }
    L.rhs_mode = 1;
    L.F = sim->F;
    L.G = sim->G;
    L.dx = sim->dx;
    L.dy = sim->dy;
    L.dt_ptr = unit_dt ? nullptr : &sim->state->dt;
    L.dt_const = 1.0;
    L.rtol = sim->vof_on ? sim->vof.rtol : sim->cg_rtol;
    L.maxiter = sim->vof_on ? sim->vof.maxiter : sim->cg_maxiter;
    L.p_out = p_out;
    L.p_padded = 1;
    L.iters_out = &sim->state->cg_iters;
    L.iters_out2 = main_solve ? &sim->state->cg_iters_step : nullptr;
    L.status_out = &sim->state->status;
    L.active = &sim->state->active;
    return status_of(pcg_launch(L, s));
}

}  // namespace

extern "C" {

const char* cfd2d_version(void) { return "cfd2d_b200 0.1 (sm_100a)"; }

int cfd2d_momentum_tendencies(const double* u, const double* v, const uint8_t* fluid, int nx,
                              int ny, double dx, double dy, const double* nu, int variable,
                              double gamma, int periodic, double* hu, double* hv,
                              const double* rho, int var_density, void* stream) {
    if (!u || !v || !fluid || !nu || !hu || !hv || !grid_ok(nx, ny)) return CFD2D_E_ARG;
    if (var_density && !rho) return CFD2D_E_ARG;
    return status_of(launch_momentum(u, v, fluid, nx, ny, dx, dy, nu, variable, gamma, periodic, hu, hv,
                                     rho, var_density, as_stream(stream)));
}

int cfd2d_obstacle_bc(double* u, double* v, const uint8_t* fluid, int nx, int ny, int periodic,
                      void* stream) {
    if (!u || !v || !fluid || !grid_ok(nx, ny)) return CFD2D_E_ARG;
    return status_of(launch_obstacle_bc(u, v, fluid, nx, ny, periodic, nullptr, as_stream(stream)));
}

int cfd2d_scalar_transport(const double* phi, const double* u, const double* v,
                           const uint8_t* fluid, int nx, int ny, double dx, double dy,
                           const double* diff, int limiter, int periodic, const int64_t* bt_l,
                           const double* bv_l, const int64_t* bt_r, const double* bv_r,
                           const int64_t* bt_b, const double* bv_b, const int64_t* bt_t,
                           const double* bv_t, int obs_t, double obs_v, double* out,
                           void* stream) {
    if (!phi || !u || !v || !fluid || !diff || !out || !grid_ok(nx, ny)) return CFD2D_E_ARG;
    if (!bt_l || !bv_l || !bt_r || !bv_r || !bt_b || !bv_b || !bt_t || !bv_t) return CFD2D_E_ARG;
    ScalarBCView bc;
    bc.bt[0] = bt_l; bc.bv[0] = bv_l;
    bc.bt[1] = bt_r; bc.bv[1] = bv_r;
    bc.bt[2] = bt_b; bc.bv[2] = bv_b;
    bc.bt[3] = bt_t; bc.bv[3] = bv_t;
    return status_of(launch_scalar_transport(phi, u, v, fluid, nx, ny, dx, dy, diff, limiter, periodic, bc,
                                             obs_t, obs_v, out, as_stream(stream)));
}

int cfd2d_domain_bc(const cfd2d_sim* sim, double* u, double* v, void* stream) {
    if (!sim || !u || !v) return CFD2D_E_ARG;
    cfd2d_sim S = *sim;
    S.state = nullptr;
    return status_of(stage_domain_bc(S, u, v, 0, as_stream(stream)));
}

int cfd2d_mask_circle(int nx, int ny, double dx, double dy, double xc, double yc, double r,
                      uint8_t* mask, void* stream) {
    if (!mask || nx < 1 || ny < 1) return CFD2D_E_ARG;
    const double q[3] = {xc, yc, r};
    return status_of(launch_mask(0, nx, ny, dx, dy, q, mask, as_stream(stream)));
}

int cfd2d_mask_ellipse(int nx, int ny, double dx, double dy, double xc, double yc, double a,
                       double b, double cos_phi, double sin_phi, uint8_t* mask, void* stream) {
    if (!mask || nx < 1 || ny < 1) return CFD2D_E_ARG;
    const double q[6] = {xc, yc, a, b, cos_phi, sin_phi};
    return status_of(launch_mask(1, nx, ny, dx, dy, q, mask, as_stream(stream)));
}

int cfd2d_mask_rectangle(int nx, int ny, double dx, double dy, double xa, double ya, double xb,
                         double yb, uint8_t* mask, void* stream) {
    if (!mask || nx < 1 || ny < 1) return CFD2D_E_ARG;
    const double q[4] = {xa, ya, xb, yb};
    return status_of(launch_mask(2, nx, ny, dx, dy, q, mask, as_stream(stream)));
}

int cfd2d_mask_polygon(int nx, int ny, double dx, double dy, const double* px, const double* py, int npts,
                       uint8_t* mask, void* stream) {
    if (!mask || !px || !py || npts < 3 || nx < 1 || ny < 1) return CFD2D_E_ARG;
    return status_of(launch_mask_polygon(nx, ny, dx, dy, px, py, npts, mask, as_stream(stream)));
}

int cfd2d_mask_image(int nx, int ny, double dx, double dy, const uint8_t* solid, int h, int w, double x0, double y0,
                     double width, double height, uint8_t* mask, void* stream) {
    if (!mask || !solid || h < 1 || w < 1 || nx < 1 || ny < 1 || !(width > 0) || !(height > 0)) return CFD2D_E_ARG;
    return status_of(launch_mask_image(nx, ny, dx, dy, solid, h, w, x0, y0, width, height, mask, as_stream(stream)));
}

size_t cfd2d_pcg_workspace_bytes(int nx, int ny) {
    return pcg_grid_workspace_doubles(nx, ny) * sizeof(double);
}

int cfd2d_pcg_plan(int nx, int ny, int* cluster) {
    if (!cluster || !grid_ok(nx, ny)) return CFD2D_E_ARG;
    *cluster = pcg_cluster_plan(nx, ny);
    return CFD2D_OK;
}

int cfd2d_pressure_solve(const cfd2d_poisson* op, const double* rhs, double* p, double rtol,
                         int maxiter, int32_t* iters_out, int32_t* status_out, void* stream) {
    if (!op || !rhs || !p || maxiter < 0 || !grid_ok(op->nx, op->ny)) return CFD2D_E_ARG;
    if (op->cluster < 0) return CFD2D_E_ARG;
    if (op->cluster == 0 && !op->work) return CFD2D_E_ARG;
    if (op->ncomp > CFD2D_MAX_COMPONENTS) return CFD2D_E_CAPACITY;
    PcgLaunch L = {};
    L.op = *op;
    L.rhs_mode = 0;
    L.rhs = rhs;
    L.rtol = rtol;
    L.maxiter = maxiter;
    L.p_out = p;
    L.p_padded = 0;
    L.iters_out = iters_out;
    L.status_out = status_out;
    return status_of(pcg_launch(L, as_stream(stream)));
}

size_t cfd2d_sim_scratch_doubles(int nx, int ny) {
    return (size_t)16 * reduction_blocks((nx + 2) * (ny + 2)) + 64;
}

int cfd2d_sim_apply_bc(const cfd2d_sim* sim, void* stream) {
    if (!sim || !sim->state) return CFD2D_E_ARG;
    return status_of(stage_apply_bc(*sim, 0, as_stream(stream)));
}

int cfd2d_sim_project_initial(const cfd2d_sim* sim, void* stream) {
    if (!sim || !sim->state) return CFD2D_E_ARG;
    if (sim->pcg.cluster == 0 && !sim->pcg.work) return CFD2D_E_ARG;
    const cudaStream_t s = as_stream(stream);
    // F = u, G = v, outflow extrapolation; solve with dt = 1; correct; p = 0; BCs
    // (cfd2d/solver.py:195-204)
    CFD_TRY(stage_predictor(*sim, 1, s));
    if (sim->vof_on) CFD_TRY(stage_vof_operator(*sim, s));
    int rc = project(sim, sim->p, true, false, s);
    if (rc) return rc;
    CFD_TRY(stage_correct(*sim, sim->p, 1, s));
    CFD_TRY(stage_fill(*sim, sim->p, (sim->nx + 2) * (sim->ny + 2), 0.0, s));
    return status_of(stage_apply_bc(*sim, 0, s));
}

}  // extern "C"

namespace {

// Event record that becomes an externally visible event node when the stream is
// being captured into a graph (plain record otherwise).
cudaError_t record(cudaEvent_t e, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t err = cudaStreamIsCapturing(s, &cs);
    if (err != cudaSuccess) return err;
    if (cs == cudaStreamCaptureStatusActive) return cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
    return cudaEventRecord(e, s);
}

int step_begin(const cfd2d_sim& S, cudaStream_t s);
int step_finish(const cfd2d_sim* sim, cudaStream_t s);

// One projection step; ev (may be null) gets four events recorded: step start,
// before and after the main pressure solve, step end.
int sim_step_impl(const cfd2d_sim* sim, cudaStream_t s, cudaEvent_t* ev) {
    if (!sim || !sim->state || !grid_ok(sim->nx, sim->ny)) return CFD2D_E_ARG;
    if (sim->pcg.cluster == 0 && !sim->pcg.work) return CFD2D_E_ARG;
    const cfd2d_sim& S = *sim;
    if (ev) CFD_TRY(record(ev[0], s));
    int rc = step_begin(S, s);
    if (rc) return rc;
    // 5. pressure Poisson (divergence fused into the solver prologue) and correction
    if (ev) CFD_TRY(record(ev[1], s));
    rc = project(sim, S.p, false, true, s);
    if (rc) return rc;
    if (ev) CFD_TRY(record(ev[2], s));
    rc = step_finish(sim, s);
    if (rc) return rc;
    if (ev) CFD_TRY(record(ev[3], s));
    return CFD2D_OK;
}

int step_begin(const cfd2d_sim& S, cudaStream_t s) {
    // 1. boundary conditions (and the run() stop decision for this step)
    CFD_TRY(stage_apply_bc(S, 1, s));
    // 2. model pre-momentum hooks: k-omega SST blending or Smagorinsky, nu_t, nu_eff
    if (S.sst_on) CFD_TRY(stage_sst_pre(S, s));
    if (S.smag_on) CFD_TRY(stage_smag_pre(S, s));
    // 3. time step and upwind fraction
    CFD_TRY(stage_dt(S, s));
    // 4. tendencies (with the VOF surface tension), AB2, predictor, outflow extrapolation
    if (S.vof_on) CFD_TRY(stage_vof_curvature(S, s));
    CFD_TRY(stage_predictor(S, 0, s));
    // variable-density operator of this step's projection
    if (S.vof_on) CFD_TRY(stage_vof_operator(S, s));
    return CFD2D_OK;
}

int step_finish(const cfd2d_sim* sim, cudaStream_t s) {
    const cfd2d_sim& S = *sim;
    int rc = CFD2D_OK;
    CFD_TRY(stage_correct(S, S.p, 0, s));
    CFD_TRY(stage_apply_bc(S, 0, s));
    // 6. volume-flow forcing (cfd2d/solver.py:410-425)
    if (S.has_flow_rate) {
        CFD_TRY(stage_flow_shift(S, s));
        if (S.has_solid) {
            CFD_TRY(stage_predictor(S, 1, s));
            rc = project(sim, S.p_tmp, true, false, s);
            if (rc) return rc;
            CFD_TRY(stage_correct(S, S.p_tmp, 1, s));
        }
        CFD_TRY(stage_apply_bc(S, 0, s));
    }
    // 7. model post-step hooks: scalar transport (k then omega for SST), VOF transport
    for (int k = 0; k < S.nscalars; ++k) CFD_TRY(stage_scalar(S, k, s));
    if (S.vof_on) CFD_TRY(stage_vof_transport(S, s));
    // 8. residual, counters, history record, model monitors
    CFD_TRY(stage_end(S, s));
    CFD_TRY(stage_monitors(S, s));
    return CFD2D_OK;
}

}  // namespace

extern "C" {

int cfd2d_sim_step(const cfd2d_sim* sim, void* stream) {
    return sim_step_impl(sim, as_stream(stream), nullptr);
}

int cfd2d_sim_step_begin(const cfd2d_sim* sim, void* stream) {
    if (!sim || !sim->state || !grid_ok(sim->nx, sim->ny)) return CFD2D_E_ARG;
    return step_begin(*sim, as_stream(stream));
}

int cfd2d_sim_step_finish(const cfd2d_sim* sim, void* stream) {
    if (!sim || !sim->state || !grid_ok(sim->nx, sim->ny)) return CFD2D_E_ARG;
    if (sim->pcg.cluster == 0 && !sim->pcg.work) return CFD2D_E_ARG;
    return step_finish(sim, as_stream(stream));
}

int cfd2d_poisson_matvec(const cfd2d_poisson* op, const double* x, double* y, void* stream) {
    if (!op || !x || !y || !grid_ok(op->nx, op->ny)) return CFD2D_E_ARG;
    return status_of(pcg_matvec(*op, x, y, as_stream(stream)));
}

int cfd2d_pressure_solve_snapshots(const cfd2d_poisson* op, const double* rhs, double* p, double rtol,
                                   int maxiter, double* snap, int every, int max_snaps, int32_t* iters_out,
                                   int32_t* status_out, void* stream) {
    if (!op || !rhs || !p || !snap || every < 1 || max_snaps < 1 || maxiter < 0) return CFD2D_E_ARG;
    if (op->cluster != 0 || !op->work) return CFD2D_E_ARG;
    PcgLaunch L = {};
    L.op = *op;
    L.rhs_mode = 0;
    L.rhs = rhs;
    L.rtol = rtol;
    L.maxiter = maxiter;
    L.p_out = p;
    L.iters_out = iters_out;
    L.status_out = status_out;
    L.snap = snap;
    L.snap_every = every;
    L.snap_max = max_snaps;
    return status_of(pcg_launch(L, as_stream(stream)));
}

int cfd2d_sim_scalar_fill_ghosts(const cfd2d_sim* sim, int slot, void* stream) {
    if (!sim || slot < 0 || slot >= sim->nscalars) return CFD2D_E_ARG;
    return status_of(stage_scalar_ghosts(*sim, slot, as_stream(stream)));
}

int cfd2d_sim_sst_pre_momentum(const cfd2d_sim* sim, void* stream) {
    if (!sim || !sim->sst_on) return CFD2D_E_ARG;
    return status_of(stage_sst_pre(*sim, as_stream(stream)));
}

int cfd2d_sim_smagorinsky_pre_momentum(const cfd2d_sim* sim, void* stream) {
    if (!sim || !sim->smag_on || !sim->smag.l2) return CFD2D_E_ARG;
    return status_of(stage_smag_pre(*sim, as_stream(stream)));
}

int cfd2d_vof_advect(const double* a, const double* u, const double* v, const uint8_t* fluid, int nx, int ny,
                     double dx, double dy, double dt, double c_alpha, int periodic, double a_in, double* out,
                     void* stream) {
    if (!a || !u || !v || !fluid || !out || !grid_ok(nx, ny) || a == out) return CFD2D_E_ARG;
    cfd2d_sim S = {};
    S.nx = nx;
    S.ny = ny;
    S.dx = dx;
    S.dy = dy;
    S.periodic = periodic ? 1 : 0;
    S.u = const_cast<double*>(u);
    S.v = const_cast<double*>(v);
    S.fluid = fluid;
    S.vof.alpha = const_cast<double*>(a);
    S.vof.c_alpha = c_alpha;
    S.vof.alpha_in = a_in;
    return status_of(launch_vof_advect(S, dt, out, as_stream(stream)));
}

int cfd2d_sim_vof_properties(const cfd2d_sim* sim, void* stream) {
    if (!sim || !sim->vof_on || !sim->vof.alpha || !sim->vof.alpha_tmp || !sim->vof.rho) return CFD2D_E_ARG;
    return status_of(stage_vof_properties(*sim, as_stream(stream)));
}

int cfd2d_barrier_selftest(unsigned int* bar, int* status, int* ok_out, void* stream) {
    if (!bar || !status || !ok_out) return CFD2D_E_ARG;
    return status_of(barrier_selftest(bar, status, ok_out, as_stream(stream)));
}

int cfd2d_set_tile(int which, int tx, int ty) { return set_tile(which, tx, ty) == 0 ? CFD2D_OK : CFD2D_E_ARG; }

int cfd2d_get_tile(int which, int* tx, int* ty) { return get_tile(which, tx, ty) == 0 ? CFD2D_OK : CFD2D_E_ARG; }

int cfd2d_graph_capture_steps_ex(const cfd2d_sim* sim, int nsteps, void* stream, void* const* events,
                                 void** graph_out, int* kernel_nodes) {
    if (!sim || nsteps < 1 || !graph_out) return CFD2D_E_ARG;
    if (events && nsteps != 1) return CFD2D_E_ARG;
    const cudaStream_t s = as_stream(stream);
    if (s == nullptr) return CFD2D_E_ARG;  // the legacy default stream cannot be captured
    cudaEvent_t ev[4];
    if (events)
        for (int k = 0; k < 4; ++k) ev[k] = (cudaEvent_t)events[k];
    CFD_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    int rc = CFD2D_OK;
    for (int k = 0; k < nsteps && rc == CFD2D_OK; ++k) rc = sim_step_impl(sim, s, events ? ev : nullptr);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (rc != CFD2D_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return CFD2D_E_CUDA;
    if (kernel_nodes) {
        size_t n = 0;
        if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) { cudaGraphDestroy(g); return CFD2D_E_CUDA; }
        cudaGraphNode_t* nodes = new cudaGraphNode_t[n > 0 ? n : 1];
        size_t m = n;
        int kn = 0;
        if (cudaGraphGetNodes(g, nodes, &m) == cudaSuccess) {
            for (size_t k = 0; k < m; ++k) {
                cudaGraphNodeType t;
                if (cudaGraphNodeGetType(nodes[k], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kn;
            }
        }
        delete[] nodes;
        *kernel_nodes = kn;
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return CFD2D_E_CUDA;
    *graph_out = (void*)exec;
    return CFD2D_OK;
}

int cfd2d_graph_capture_steps(const cfd2d_sim* sim, int nsteps, void* stream, void** graph_out) {
    return cfd2d_graph_capture_steps_ex(sim, nsteps, stream, nullptr, graph_out, nullptr);
}

int cfd2d_events_create(int n, void** events) {
    if (n < 0 || (n > 0 && !events)) return CFD2D_E_ARG;
    for (int k = 0; k < n; ++k) {
        cudaEvent_t e;
        CFD_TRY(cudaEventCreate(&e));
        events[k] = (void*)e;
    }
    return CFD2D_OK;
}

int cfd2d_events_destroy(int n, void** events) {
    for (int k = 0; k < n; ++k)
        if (events[k]) cudaEventDestroy((cudaEvent_t)events[k]);
    return CFD2D_OK;
}

int cfd2d_event_elapsed_ms(void* start, void* end, float* ms) {
    if (!start || !end || !ms) return CFD2D_E_ARG;
    CFD_TRY(cudaEventSynchronize((cudaEvent_t)end));
    return status_of(cudaEventElapsedTime(ms, (cudaEvent_t)start, (cudaEvent_t)end));
}

int cfd2d_graph_launch(void* graph, void* stream) {
    if (!graph) return CFD2D_E_ARG;
    return status_of(cudaGraphLaunch((cudaGraphExec_t)graph, as_stream(stream)));
}

int cfd2d_graph_destroy(void* graph) {
    if (!graph) return CFD2D_OK;
    return status_of(cudaGraphExecDestroy((cudaGraphExec_t)graph));
}

}  // extern "C"
