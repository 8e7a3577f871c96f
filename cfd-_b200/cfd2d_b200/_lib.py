"""ctypes binding of ``libcfd2d_b200.so`` (the C ABI in include/cfd2d_b200.h).

The structures below mirror the C structs field for field. Device memory is
owned by torch tensors on the Python side; only raw pointers cross the ABI.
There is no CPU fallback: if the library or a CUDA device is missing, every
entry point raises.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "lib" / "libcfd2d_b200.so"

OK = 0
E_ARG, E_CUDA, E_CAPACITY, E_UNSUPPORTED = -1, -2, -3, -4
S_NONFINITE, S_CG_MAXITER, S_BARRIER_TIMEOUT, S_COMPONENTS, S_VOF_SUBSTEPS = 1, 2, 4, 8, 16
MAX_COMPONENTS = 16
MAX_SCALARS = 4
HIST_FIELDS = 10
BC_CODES = {"noslip": 0, "slip": 1, "inflow": 2, "outflow": 3, "periodic": 4}

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p


class State(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("dt", C.c_double), ("dt_old", C.c_double), ("gamma", C.c_double),
        ("ab_a", C.c_double), ("ab_b", C.c_double), ("flow_force", C.c_double),
        ("residual", C.c_double), ("dt_fixed", C.c_double), ("t_end", C.c_double),
        ("steady_tol", C.c_double), ("bulk_du", C.c_double),
        ("n", C.c_int64), ("max_steps", C.c_int64),
        ("have_old", C.c_int32), ("status", C.c_int32), ("active", C.c_int32),
        ("cg_iters", C.c_int32), ("cg_iters_step", C.c_int32), ("error_step", C.c_int32),
        ("stop_reason", C.c_int32), ("pad0", C.c_int32),
        ("umax_bits", C.c_uint64), ("vmax_bits", C.c_uint64), ("numax_bits", C.c_uint64),
        ("numin_bits", C.c_uint64), ("dmax_bits", C.c_uint64 * MAX_SCALARS),
        ("du_bits", C.c_uint64), ("dv_bits", C.c_uint64), ("div_bits", C.c_uint64),
        ("ticket", C.c_uint32 * 8),
    ]


class Poisson(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("periodic", C.c_int),
        ("dx2", C.c_double), ("dy2", C.c_double),
        ("diag", _vp), ("dinv", _vp), ("nbr", _vp), ("label", _vp),
        ("ncomp", C.c_int), ("comp_count", _vp), ("x0", _vp), ("work", _vp),
        ("work_bytes", C.c_size_t), ("cluster", C.c_int), ("mixed", C.c_int),
        ("grid_ctas", C.c_int), ("bx", _vp), ("by", _vp),
    ]


class Scalar(C.Structure):
    _fields_ = [
        ("phi", _vp), ("diff", _vp), ("rhs", _vp), ("bt", _vp * 4), ("bv", _vp * 4),
        ("limiter", C.c_int), ("obs_t", C.c_int), ("obs_v", C.c_double), ("D0", C.c_double),
        ("turb_div", C.c_double), ("has_lower", C.c_int), ("has_upper", C.c_int),
        ("lower", C.c_double), ("upper", C.c_double), ("source", C.c_int), ("pad", C.c_int),
    ]


class SST(C.Structure):
    _fields_ = [
        ("S2", _vp), ("F1", _vp), ("cross", _vp), ("Pk", _vp), ("d", _vp), ("wall_adj", _vp),
        ("w_wall", _vp), ("k_index", C.c_int), ("w_index", C.c_int),
    ]


# field selectors of the device function objects
FIELD_U, FIELD_V, FIELD_PRESSURE, FIELD_UC, FIELD_VC, FIELD_SPEED, FIELD_VORTICITY = range(7)
FIELD_CELL, FIELD_CELL_LOG10, FIELD_NODE, FIELD_FLUID = 7, 8, 9, 10
MAX_FIELDS = 16


class Field(C.Structure):
    _fields_ = [("kind", C.c_int), ("pad", C.c_int), ("data", _vp)]


class ProbeSeries(C.Structure):
    _fields_ = [("t", _vp), ("values", _vp), ("count", _vp), ("cap", C.c_int), ("every", C.c_int)]


class FieldAverage(C.Structure):
    _fields_ = [("t_start", C.c_double), ("sum", _vp), ("sum2", _vp), ("T", _vp)]


class Smagorinsky(C.Structure):
    _fields_ = [("l2", _vp)]


class Vof(C.Structure):
    _fields_ = [
        ("alpha", _vp), ("alpha_tmp", _vp), ("rho", _vp), ("smooth", _vp), ("nrm", _vp), ("kappa", _vp),
        ("bx", _vp), ("by", _vp), ("vdiag", _vp), ("vdinv", _vp), ("scal", _vp), ("vflags", _vp),
        ("rho1", C.c_double), ("rho2", C.c_double), ("mu1", C.c_double), ("mu2", C.c_double),
        ("sigma", C.c_double), ("c_alpha", C.c_double), ("cfl", C.c_double), ("alpha_in", C.c_double),
        ("dt_limit", C.c_double), ("rtol", C.c_double), ("maxiter", C.c_int), ("nsub_max", C.c_int),
    ]


MAX_MONITORS = 12
MONITOR_SCRATCH = 2 * MAX_MONITORS * 296
MON_SUM_FLUID, MON_MEAN_FLUID, MON_MAX_ALL, MON_NUSSELT, MON_VOLUME_ERROR, MON_FRONT_X, MON_HEIGHT_LEFT = range(7)


class Monitor(C.Structure):
    _fields_ = [("kind", C.c_int), ("slot", C.c_int), ("side", C.c_int), ("pad", C.c_int), ("data", _vp),
                ("param", C.c_double)]


class Sim(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
        ("periodic", C.c_int), ("scheme_ab2", C.c_int), ("gamma_auto", C.c_int),
        ("gamma_fixed", C.c_double), ("tau", C.c_double), ("nu", C.c_double),
        ("body_fx", C.c_double), ("body_fy", C.c_double), ("has_flow_rate", C.c_int),
        ("flow_rate", C.c_double), ("flow_count", C.c_double),
        ("variable_viscosity", C.c_int), ("compute_forces", C.c_int), ("has_solid", C.c_int),
        ("bc_kind", C.c_int * 4), ("bc_vel", C.c_double * 4), ("inflow", _vp * 4),
        ("open", _vp * 4), ("fluid", _vp),
        ("u", _vp), ("v", _vp), ("p", _vp), ("F", _vp), ("G", _vp), ("hu", _vp), ("hv", _vp),
        ("u_prev", _vp), ("v_prev", _vp), ("nu_eff", _vp), ("nu_t", _vp),
        ("pcg", Poisson), ("cg_rtol", C.c_double), ("cg_maxiter", C.c_int),
        ("nscalars", C.c_int), ("scalars", Scalar * MAX_SCALARS),
        ("scalar_dtlim_const", C.c_double * MAX_SCALARS), ("thermal_index", C.c_int),
        ("gx", C.c_double), ("gy", C.c_double), ("T_ref", C.c_double), ("sst_on", C.c_int),
        ("sst", SST), ("smag_on", C.c_int), ("smag", Smagorinsky),
        ("vof_on", C.c_int), ("vof", Vof), ("nmon", C.c_int), ("mon", Monitor * MAX_MONITORS),
        ("mon_ring", _vp), ("mon_part", _vp), ("state", _vp), ("red", _vp), ("hist", _vp), ("hist_cap", C.c_int),
        ("p_tmp", _vp),
    ]


class FcgScalars(C.Structure):
    _fields_ = [("alpha", C.c_double), ("beta", C.c_double), ("rz", C.c_double), ("pq", C.c_double),
                ("rr", C.c_double), ("bb", C.c_double), ("iters", C.c_int32), ("ticket", C.c_uint32)]


class FcgControl(C.Structure):
    _fields_ = [("rtol", C.c_double), ("stall_factor", C.c_double), ("stall_window", C.c_int32),
                ("maxiter", C.c_int32), ("reason", C.c_int32), ("iters", C.c_int32), ("calls", C.c_int32),
                ("pad", C.c_int32), ("hist", C.c_void_p), ("iters_out", C.c_void_p)]


FCG_RUNNING, FCG_CONVERGED, FCG_MAXITER, FCG_STALLED, FCG_NONFINITE = 0, 1, 2, 3, 4


_LIB = None


class CudaPathError(RuntimeError):
    """The CUDA library or device is unavailable; the path has no CPU fallback."""


def lib():
    """Load the library once; raise if it was not built or cannot be loaded."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = Path(os.environ.get("CFD2D_B200_LIB", LIB_PATH))
    if not path.exists():
        raise CudaPathError(f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; "
                            f"g.build()'` (the CUDA library has no CPU fallback)")
    L = C.CDLL(str(path))
    i, d, vp, sz = C.c_int, C.c_double, C.c_void_p, C.c_size_t
    sig = {
        "cfd2d_version": ([], C.c_char_p),
        "cfd2d_momentum_tendencies": ([vp, vp, vp, i, i, d, d, vp, i, d, i, vp, vp, vp, i, vp], i),
        "cfd2d_obstacle_bc": ([vp, vp, vp, i, i, i, vp], i),
        "cfd2d_scalar_transport": ([vp, vp, vp, vp, i, i, d, d, vp, i, i] + [vp] * 8 + [i, d, vp, vp], i),
        "cfd2d_domain_bc": ([vp, vp, vp, vp], i),
        "cfd2d_mask_circle": ([i, i, d, d, d, d, d, vp, vp], i),
        "cfd2d_mask_ellipse": ([i, i, d, d, d, d, d, d, d, d, vp, vp], i),
        "cfd2d_mask_rectangle": ([i, i, d, d, d, d, d, d, vp, vp], i),
        "cfd2d_pcg_workspace_bytes": ([i, i], sz),
        "cfd2d_pcg_plan": ([i, i, C.POINTER(C.c_int)], i),
        "cfd2d_pressure_solve": ([vp, vp, vp, d, i, vp, vp, vp], i),
        "cfd2d_pressure_solve_static": ([vp, vp, vp, d, i, vp, vp, vp], i),
        "cfd2d_sim_scratch_doubles": ([i, i], sz),
        "cfd2d_sim_apply_bc": ([vp, vp], i),
        "cfd2d_sim_project_initial": ([vp, vp], i),
        "cfd2d_sim_step": ([vp, vp], i),
        "cfd2d_sim_scalar_fill_ghosts": ([vp, i, vp], i),
        "cfd2d_sim_sst_pre_momentum": ([vp, vp], i),
        "cfd2d_sim_smagorinsky_pre_momentum": ([vp, vp], i),
        "cfd2d_wall_distance_workspace_bytes": ([i, i], sz),
        "cfd2d_sim_wall_distance": ([vp, vp, vp, sz, vp], i),
        "cfd2d_sample": ([vp, vp, i, vp, vp, i, vp, vp], i),
        "cfd2d_set_tile": ([i, i, i], i),
        "cfd2d_mask_polygon": ([i, i, d, d, vp, vp, i, vp, vp], i),
        "cfd2d_mask_image": ([i, i, d, d, vp, i, i, d, d, d, d, vp, vp], i),
        "cfd2d_barrier_selftest": ([vp, vp, vp, vp], i),
        "cfd2d_get_tile": ([i, C.POINTER(C.c_int), C.POINTER(C.c_int)], i),
        "cfd2d_vof_advect": ([vp, vp, vp, vp, i, i, d, d, d, d, i, d, vp, vp], i),
        "cfd2d_sim_vof_properties": ([vp, vp], i),
        "cfd2d_cell_values": ([vp, vp, vp, vp], i),
        "cfd2d_probe_record": ([vp, vp, i, vp, vp, i, vp, vp], i),
        "cfd2d_field_average_accumulate": ([vp, vp, vp], i),
        "cfd2d_streamfunction": ([vp, vp, vp], i),
        "cfd2d_vtk_pack": ([vp, vp, i, vp, vp], i),
        "cfd2d_graph_capture_steps": ([vp, i, vp, C.POINTER(C.c_void_p)], i),
        "cfd2d_graph_launch": ([vp, vp], i),
        "cfd2d_graph_destroy": ([vp], i),
        "cfd2d_graph_capture_steps_ex": ([vp, i, vp, vp, C.POINTER(C.c_void_p), C.POINTER(C.c_int)], i),
        "cfd2d_events_create": ([i, vp], i),
        "cfd2d_events_destroy": ([i, vp], i),
        "cfd2d_event_elapsed_ms": ([vp, vp, C.POINTER(C.c_float)], i),
        "cfd2d_sim_step_begin": ([vp, vp], i),
        "cfd2d_sim_step_finish": ([vp, vp], i),
        "cfd2d_poisson_matvec": ([vp, vp, vp, vp], i),
        "cfd2d_pressure_solve_snapshots": ([vp, vp, vp, d, i, vp, i, i, vp, vp, vp], i),
        "cfd2d_lpc_w32_bytes": ([], sz),
        "cfd2d_lpc_pack_w32": ([vp, vp, vp], i),
        "cfd2d_lpc_pack_w32_adjoint": ([vp, vp, vp], i),
        "cfd2d_lpc_conv32": ([vp, vp, vp, vp, vp, vp, i, i, i, vp, vp], i),
        "cfd2d_lpc_conv": ([i, i, vp, i, vp, vp, vp, vp, i, i, i, i, i, vp], i),
        "cfd2d_lpc_pool2": ([vp, vp, i, i, vp], i),
        "cfd2d_lpc_pool_mask": ([vp, vp, i, i, vp], i),
        "cfd2d_lpc_upadd": ([vp, vp, vp, i, i, C.c_float, vp], i),
        "cfd2d_lpc_relu_bwd": ([vp, vp, vp, vp, i, i, i, vp], i),
        "cfd2d_lpc_upadd_bwd": ([vp, vp, i, i, C.c_float, vp], i),
        "cfd2d_lpc_pool_bwd": ([vp, vp, i, i, vp], i),
        "cfd2d_lpc_conv_dw_partial_floats": ([i, i, i, i, i], sz),
        "cfd2d_lpc_conv_dw": ([i, i, vp, i, vp, i, i, i, vp, vp, vp], i),
        "cfd2d_fcg_partial_doubles": ([i], sz),
        "cfd2d_fcg_init": ([vp, vp, vp, vp, d, d, vp, vp, vp, vp, vp, vp, vp, vp], i),
        "cfd2d_fcg_pq": ([vp, vp, vp, vp, vp, vp, vp], i),
        "cfd2d_fcg_update": ([i, vp, vp, vp, vp, vp, vp, vp], i),
        "cfd2d_fcg_zr": ([i, vp, vp, i, vp, vp, vp], i),
        "cfd2d_fcg_dir": ([i, vp, vp, vp, vp], i),
        "cfd2d_fcg_net_in": ([i, vp, vp, vp, vp, vp], i),
        "cfd2d_fcg_net_out": ([i, vp, vp, vp, vp, vp, d, d, vp, vp], i),
        "cfd2d_fcg_gate": ([vp, vp, C.c_uint64, vp], i),
        "cfd2d_fcg_zero_rhs": ([i, vp, vp, vp, vp], i),
        "cfd2d_capture_begin": ([vp], i),
        "cfd2d_capture_condition": ([vp, vp], i),
        "cfd2d_capture_while_begin": ([vp, vp, C.c_uint64], i),
        "cfd2d_capture_while_end": ([vp], i),
        "cfd2d_capture_end": ([vp, vp], i),
        "cfd2d_capture_abort": ([vp], i),
        "cfd2d_fcg_scatter_p": ([vp, vp, vp, vp], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _LIB = L
    return L


def exported_symbols():
    """Names of the entry points bound above (each must be exported by the library)."""
    return [
        "cfd2d_version", "cfd2d_momentum_tendencies", "cfd2d_obstacle_bc", "cfd2d_scalar_transport",
        "cfd2d_domain_bc", "cfd2d_mask_circle", "cfd2d_mask_ellipse", "cfd2d_mask_rectangle",
        "cfd2d_pcg_workspace_bytes", "cfd2d_pcg_plan", "cfd2d_pressure_solve",
        "cfd2d_sim_scratch_doubles", "cfd2d_sim_apply_bc", "cfd2d_sim_project_initial",
        "cfd2d_sim_step", "cfd2d_sim_scalar_fill_ghosts", "cfd2d_sim_sst_pre_momentum",
        "cfd2d_sim_smagorinsky_pre_momentum", "cfd2d_wall_distance_workspace_bytes",
        "cfd2d_sim_wall_distance", "cfd2d_sample", "cfd2d_mask_polygon", "cfd2d_mask_image", "cfd2d_barrier_selftest", "cfd2d_set_tile", "cfd2d_get_tile", "cfd2d_cell_values", "cfd2d_vof_advect", "cfd2d_sim_vof_properties", "cfd2d_probe_record", "cfd2d_field_average_accumulate",
        "cfd2d_streamfunction", "cfd2d_vtk_pack", "cfd2d_graph_capture_steps", "cfd2d_graph_launch", "cfd2d_graph_destroy",
        "cfd2d_graph_capture_steps_ex", "cfd2d_events_create", "cfd2d_events_destroy",
        "cfd2d_event_elapsed_ms", "cfd2d_sim_step_begin", "cfd2d_sim_step_finish", "cfd2d_poisson_matvec",
        "cfd2d_pressure_solve_snapshots", "cfd2d_lpc_w32_bytes", "cfd2d_lpc_pack_w32", "cfd2d_lpc_pack_w32_adjoint", "cfd2d_lpc_conv32",
        "cfd2d_lpc_conv", "cfd2d_lpc_pool2", "cfd2d_lpc_pool_mask", "cfd2d_lpc_upadd", "cfd2d_lpc_relu_bwd",
        "cfd2d_lpc_upadd_bwd", "cfd2d_lpc_pool_bwd", "cfd2d_lpc_conv_dw_partial_floats", "cfd2d_lpc_conv_dw",
        "cfd2d_fcg_partial_doubles", "cfd2d_fcg_init", "cfd2d_fcg_pq", "cfd2d_fcg_update", "cfd2d_fcg_zr",
        "cfd2d_fcg_dir", "cfd2d_fcg_net_in", "cfd2d_fcg_net_out", "cfd2d_fcg_scatter_p",
        "cfd2d_pressure_solve_static", "cfd2d_fcg_gate", "cfd2d_fcg_zero_rhs", "cfd2d_capture_begin",
        "cfd2d_capture_condition", "cfd2d_capture_while_begin", "cfd2d_capture_while_end", "cfd2d_capture_end",
        "cfd2d_capture_abort",
    ]


def check(rc: int, what: str) -> None:
    if rc != OK:
        names = {E_ARG: "invalid argument", E_CUDA: "CUDA error", E_CAPACITY: "capacity exceeded",
                 E_UNSUPPORTED: "unsupported"}
        detail = ""
        if rc == E_CUDA:
            import torch
            try:
                torch.cuda.synchronize()
            except Exception as exc:  # surface the CUDA error text
                detail = f": {exc}"
        raise RuntimeError(f"{what} failed ({names.get(rc, rc)}){detail}")


# ------------------------------------------------------------------ torch plumbing
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        raise CudaPathError("no CUDA device: the cfd2d_b200 path runs on the GPU only")
    return _t


def device():
    return torch().device("cuda", torch().cuda.current_device())


def stream_ptr(stream=None):
    t = torch()
    s = stream if stream is not None else t.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def ptr(t) -> C.c_void_p:
    """Raw device pointer of a CUDA tensor (None -> NULL)."""
    if t is None:
        return C.c_void_p(0)
    return C.c_void_p(t.data_ptr())


def to_dev(a, dtype=None):
    """numpy array (or CUDA tensor) -> contiguous CUDA tensor."""
    t = torch()
    if isinstance(a, t.Tensor):
        x = a if a.is_cuda else a.to(device())
        if dtype is not None and x.dtype != dtype:
            x = x.to(dtype)
        return x.contiguous()
    arr = np.ascontiguousarray(a)
    if arr.dtype == np.bool_:
        arr = arr.astype(np.uint8)
    x = t.from_numpy(arr).to(device())
    if dtype is not None and x.dtype != dtype:
        x = x.to(dtype)
    return x
