"""Pressure Poisson solver (drop-in for cfd2d/pressure.py).

The host assembles the operator data once, in the reference's accumulation order
(cfd2d/pressure.py:43-131): the diagonal of A = -Lap over the fluid cells
(neighbour couplings, +2/h^2 on outflow Dirichlet faces, +1/dx^2 on the first cell
of every component without a Dirichlet face), the coupling bits of every cell and
the Neumann-component labels. The solve itself is the on-chip Jacobi-PCG of
``cfd2d_pressure_solve`` (scipy's CG iteration form, warm-started from the
previous solution).

Methods: ``"cg"`` runs to the relative residual ``tol`` (reference default 1e-10).
``"direct"`` (alias ``"lu"``) has no GPU LU; it runs the same CG to a relative
residual of 1e-13, which agrees with a sparse LU solve to about 1e-15.
"""

from __future__ import annotations

import ctypes as C
import os
import warnings

import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components

from . import _lib
from .boundary import DomainBoundary
from .grid import Grid

DIRECT_RTOL = 1e-13
DIRECT_MAXITER = 50000
CG_MAXITER = 5000  # scipy cg's maxiter in cfd2d/pressure.py:171


class PressureSolver:
    METHODS = ("direct", "cg", "lu")

    def __init__(self, grid: Grid, boundary: DomainBoundary, method: str = "direct",
                 tol: float = 1e-10):
        if method not in self.METHODS:
            raise ValueError(f"Unbekannter Drucklöser {method!r}, erlaubt: {self.METHODS}")
        self.grid = grid
        self.method = "direct" if method == "lu" else method
        self._tol = float(tol)
        self._cg_maxiter = CG_MAXITER
        self.on_change = None
        nx, ny = grid.nx, grid.ny
        self.dx2 = dx2 = 1.0 / grid.dx ** 2
        self.dy2 = dy2 = 1.0 / grid.dy ** 2
        fluid = grid.fluid_interior.copy()
        self.fluid = fluid
        n = int(fluid.sum())
        if n == 0:
            raise ValueError("Das Gebiet enthält keine Fluidzellen.")
        idx = -np.ones((nx, ny), dtype=np.int64)
        idx[fluid] = np.arange(n)
        self.idx, self.n = idx, n
        bx = fluid[:-1, :] & fluid[1:, :]
        by = fluid[:, :-1] & fluid[:, 1:]
        self.periodic = boundary.periodic
        bp = (fluid[-1, :] & fluid[0, :]) if self.periodic else np.zeros(ny, dtype=bool)
        self._both = (bx, by, bp)
        diag = np.zeros((nx, ny))
        diag[:-1, :][bx] += dx2
        diag[1:, :][bx] += dx2
        diag[:, :-1][by] += dy2
        diag[:, 1:][by] += dy2
        if self.periodic:
            diag[-1, :][bp] += dx2
            diag[0, :][bp] += dx2
        self.dirichlet = {s: boundary.outflow_mask(s) for s in ("left", "right", "bottom", "top")}
        diag[0, :][self.dirichlet["left"]] += 2 * dx2
        diag[-1, :][self.dirichlet["right"]] += 2 * dx2
        diag[:, 0][self.dirichlet["bottom"]] += 2 * dy2
        diag[:, -1][self.dirichlet["top"]] += 2 * dy2
        has_dir = np.zeros((nx, ny), dtype=bool)
        has_dir[0, :] |= self.dirichlet["left"]
        has_dir[-1, :] |= self.dirichlet["right"]
        has_dir[:, 0] |= self.dirichlet["bottom"]
        has_dir[:, -1] |= self.dirichlet["top"]
        a = np.concatenate([idx[:-1, :][bx], idx[:, :-1][by], idx[-1, :][bp]])
        b = np.concatenate([idx[1:, :][bx], idx[:, 1:][by], idx[0, :][bp]])
        adj = sp.csr_matrix((np.ones(a.size), (a, b)), shape=(n, n))
        ncomp, comp_of = connected_components(adj, directed=False)
        labels = np.zeros((nx, ny), dtype=np.int64)
        labels[fluid] = comp_of + 1
        self.labels = labels
        dir_comps = set(np.unique(labels[has_dir & fluid]).tolist())
        self.neumann_components, self._pinned = [], []
        for c in range(1, ncomp + 1):
            if c not in dir_comps:
                first = int(np.argmax(comp_of == c - 1))
                fi, fj = np.argwhere(idx == first)[0]
                diag[fi, fj] += dx2
                self.neumann_components.append(c)
                self._pinned.append((int(fi), int(fj)))
        if len(self.neumann_components) > _lib.MAX_COMPONENTS:
            raise ValueError(f"{len(self.neumann_components)} Neumann-Komponenten; der GPU-Löser "
                             f"verfolgt höchstens {_lib.MAX_COMPONENTS}")
        self.diag = diag
        self.last_iterations = 0
        self._A = None
        self._upload()

    # ------------------------------------------------------------------ device
    def _upload(self):
        t = _lib.torch()
        g = self.grid
        nx, ny = g.nx, g.ny
        f = self.fluid
        bx, by, bp = self._both
        nbr = np.zeros((nx, ny), dtype=np.uint8)
        nbr[1:, :][bx] |= 1       # west neighbour coupled
        nbr[:, 1:][by] |= 2       # south
        nbr[:, :-1][by] |= 4      # north
        nbr[:-1, :][bx] |= 8      # east
        if self.periodic:
            nbr[0, :][bp] |= 1
            nbr[-1, :][bp] |= 8
        nbr[f] |= 0x80
        dinv = np.zeros((nx, ny))
        dinv[f] = 1.0 / self.diag[f]
        lab = -np.ones((nx, ny), dtype=np.int16)
        counts = []
        for k, c in enumerate(self.neumann_components):
            m = self.labels == c
            lab[m] = k
            counts.append(float(m.sum()))
        self._d_diag = _lib.to_dev(self.diag)
        self._d_dinv = _lib.to_dev(dinv)
        self._d_nbr = _lib.to_dev(nbr)
        self._d_lab = _lib.to_dev(lab)
        self._d_cnt = _lib.to_dev(np.array(counts + [1.0], dtype=np.float64))
        self._d_x0 = t.zeros((nx, ny), dtype=t.float64, device=_lib.device())
        cl = C.c_int(0)
        _lib.check(_lib.lib().cfd2d_pcg_plan(nx, ny, C.byref(cl)), "cfd2d_pcg_plan")
        # > 0: CTAs of the on-chip cluster solver; 0: grid-persistent solver with a workspace.
        # CFD2D_PCG_VARIANT=grid (or grid-l2, cluster-l2) selects the workspace solver for any size.
        variant = os.environ.get("CFD2D_PCG_VARIANT")
        self.cluster = 0 if variant in ("grid", "grid-slab1", "grid-l2", "cluster-l2") else cl.value
        self._work = None
        if self.cluster == 0:
            nbytes = int(_lib.lib().cfd2d_pcg_workspace_bytes(nx, ny))
            self._work = t.zeros(nbytes // 8, dtype=t.float64, device=_lib.device())
        self._d_iters = t.zeros(2, dtype=t.int32, device=_lib.device())
        P = _lib.Poisson()
        P.nx, P.ny, P.periodic = nx, ny, int(self.periodic)
        P.dx2, P.dy2 = self.dx2, self.dy2
        P.diag, P.dinv = self._d_diag.data_ptr(), self._d_dinv.data_ptr()
        P.nbr, P.label = self._d_nbr.data_ptr(), self._d_lab.data_ptr()
        P.ncomp = len(self.neumann_components)
        P.comp_count = self._d_cnt.data_ptr()
        P.x0 = self._d_x0.data_ptr()
        if self._work is not None:
            P.work, P.work_bytes = self._work.data_ptr(), self._work.numel() * 8
        else:
            P.work, P.work_bytes = 0, 0
        P.cluster = self.cluster
        P.mixed = 0
        # CFD2D_PCG_VARIANT=cluster-l2: the workspace solver on one 16-CTA cluster;
        # grid-l2: over every SM with the vectors in the workspace (no shared-memory slabs);
        # grid-slab1: the shared-memory slabs with one reduction per iteration;
        # single: the single-reduction form of whichever solver the grid takes
        P.grid_ctas = {"cluster-l2": 16, "grid-l2": -1, "grid-slab1": -2}.get(variant, 0) if self.cluster == 0 else 0
        if variant == "single":
            P.grid_ctas = -2
        self.op = P

    def ensure_workspace(self) -> None:
        """Allocate the workspace of the grid-persistent solver (the variable-density
        solve of the VOF model always runs there)."""
        if self._work is not None:
            return
        t = _lib.torch()
        nbytes = int(_lib.lib().cfd2d_pcg_workspace_bytes(self.grid.nx, self.grid.ny))
        self._work = t.zeros(nbytes // 8, dtype=t.float64, device=_lib.device())
        self.op.work, self.op.work_bytes = self._work.data_ptr(), self._work.numel() * 8
        if self.on_change is not None:
            self.on_change()

    @property
    def grid_ctas(self) -> int:
        """The solver form. -2 = the single-reduction form (Chronopoulos-Gear recurrence:
        one reduction per iteration, the same iteration counts, p rounded differently)
        of whichever solver the grid takes: the on-chip cluster solver (even ny) or the
        shared-memory slabs. For grids beyond one on-chip cluster: 0 = the solver spreads
        over every SM (cooperative launch; each CTA keeps a slab of rows in shared memory
        when the slabs fit, else the vectors live in the workspace); -1 = over every SM
        with the vectors in the workspace; 16 = on one 16-CTA cluster, leaving the other
        SMs to other solves (cfd2d_b200.batch). On a cluster grid 0, -1 and 16 all mean
        the on-chip solver."""
        return int(self.op.grid_ctas)

    @grid_ctas.setter
    def grid_ctas(self, value: int) -> None:
        if int(value) not in (0, 16, -1, -2):
            raise ValueError("grid_ctas must be 0, -1, -2 or 16")
        if self.cluster != 0 and int(value) != -2:
            value = 0  # the on-chip solver is used; only its form can be chosen
        self.op.grid_ctas = int(value)
        if self.on_change is not None:
            self.on_change()

    @property
    def precision(self) -> str:
        """"fp64": the reference's iteration (scipy's CG form) in FP64; "mixed": FP32
        iterations with FP64 residual refinement and FP64 reductions, to the same
        relative residual (on-chip solver only; no counterpart in the reference)."""
        return "mixed" if self.op.mixed else "fp64"

    @precision.setter
    def precision(self, value: str) -> None:
        if value not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', not {value!r}")
        if value == "mixed" and self.cluster == 0:
            raise ValueError("the mixed-precision solver runs on the on-chip (cluster) solver only")
        self.op.mixed = int(value == "mixed")
        if self.on_change is not None:
            self.on_change()

    @property
    def tol(self) -> float:
        return self._tol

    @tol.setter
    def tol(self, value: float) -> None:
        self._tol = float(value)
        if self.on_change is not None:
            self.on_change()

    @property
    def rtol(self) -> float:
        """Relative residual the CG runs to (``tol``, or 1e-13 for 'direct')."""
        return DIRECT_RTOL if self.method == "direct" else self._tol

    @property
    def maxiter(self) -> int:
        """Iteration cap of the CG: 5000 for 'cg' as the reference (settable, e.g. for
        grids whose solve needs more), 50000 for 'direct'."""
        return DIRECT_MAXITER if self.method == "direct" else self._cg_maxiter

    @maxiter.setter
    def maxiter(self, value: int) -> None:
        if int(value) < 1:
            raise ValueError("maxiter must be positive")
        self._cg_maxiter = int(value)
        if self.on_change is not None:
            self.on_change()

    @property
    def _x0(self) -> np.ndarray:
        return self._d_x0.cpu().numpy()[self.fluid]

    @_x0.setter
    def _x0(self, x) -> None:
        full = np.zeros(self.fluid.shape)
        full[self.fluid] = np.asarray(x, dtype=float)
        self._d_x0.copy_(_lib.to_dev(full))

    @property
    def A(self):
        """The assembled sparse operator (built on demand, for inspection)."""
        if self._A is None:
            bx, by, bp = self._both
            idx = self.idx
            rows = [idx[:-1, :][bx], idx[1:, :][bx], idx[:, :-1][by], idx[:, 1:][by],
                    idx[-1, :][bp], idx[0, :][bp], np.arange(self.n)]
            cols = [idx[1:, :][bx], idx[:-1, :][bx], idx[:, 1:][by], idx[:, :-1][by],
                    idx[0, :][bp], idx[-1, :][bp], np.arange(self.n)]
            vals = [np.full(bx.sum(), -self.dx2)] * 2 + [np.full(by.sum(), -self.dy2)] * 2 + \
                   [np.full(bp.sum(), -self.dx2)] * 2 + [self.diag[self.fluid]]
            self._A = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                                    shape=(self.n, self.n))
        return self._A

    def solve(self, rhs):
        """Solve Lap(p) = rhs (cfd2d/pressure.py:143-185); returns p (nx, ny), 0 in solids.

        rhs may be a host array (the result is a host array) or a CUDA tensor.
        """
        t = _lib.torch()
        host = not isinstance(rhs, t.Tensor)
        r = _lib.to_dev(rhs, t.float64)
        p = t.empty_like(r)
        st = t.zeros(1, dtype=t.int32, device=_lib.device())
        rc = _lib.lib().cfd2d_pressure_solve(C.byref(self.op), _lib.ptr(r), _lib.ptr(p), self.rtol,
                                             self.maxiter, _lib.ptr(self._d_iters), _lib.ptr(st),
                                             _lib.stream_ptr())
        _lib.check(rc, "cfd2d_pressure_solve")
        info = st.cpu().numpy()
        self.last_iterations = int(self._d_iters[0].item())
        if info[0] & _lib.S_BARRIER_TIMEOUT:
            raise RuntimeError("pressure solve abandoned: a bounded inter-block wait timed out")
        if info[0] & _lib.S_CG_MAXITER:
            warnings.warn(f"CG-Drucklöser nicht konvergiert ({self.maxiter} Iterationen)")
        return p.cpu().numpy() if host else p

    def variable_operator(self, bx, by):
        """The C-ABI operator of div(b grad p) with face coefficients bx (nx+1, ny) and
        by (nx, ny+1), the diagonal assembled on the host in the reference's order
        (cfd2d/pressure.py:187-236), with a zero warm start. Returns (op, tensors): the
        device tensors the operator points to, which must outlive its use."""
        t = _lib.torch()
        g = self.grid
        nx, ny = g.nx, g.ny
        bx = np.asarray(bx, dtype=np.float64)
        by = np.asarray(by, dtype=np.float64)
        dx2, dy2 = self.dx2, self.dy2
        f = self.fluid
        both_x = f[:-1, :] & f[1:, :]
        both_y = f[:, :-1] & f[:, 1:]
        diag = np.zeros((nx, ny))
        cxi = (bx[1:nx, :] * dx2)[both_x]
        diag[:-1, :][both_x] += cxi
        diag[1:, :][both_x] += cxi
        cyi = (by[:, 1:ny] * dy2)[both_y]
        diag[:, :-1][both_y] += cyi
        diag[:, 1:][both_y] += cyi
        if self.periodic:
            bp = f[-1, :] & f[0, :]
            cpi = (bx[nx, :] * dx2)[bp]
            diag[-1, :][bp] += cpi
            diag[0, :][bp] += cpi
        d = self.dirichlet
        diag[0, :][d["left"]] += 2 * dx2 * bx[0, :][d["left"]]
        diag[-1, :][d["right"]] += 2 * dx2 * bx[nx, :][d["right"]]
        diag[:, 0][d["bottom"]] += 2 * dy2 * by[:, 0][d["bottom"]]
        diag[:, -1][d["top"]] += 2 * dy2 * by[:, ny][d["top"]]
        for fi, fj in self._pinned:
            diag[fi, fj] += dx2 * max(float(bx.max()), 1e-30)
        dinv = np.where(f, 1.0 / np.where(f, diag, 1.0), 0.0)
        self.ensure_workspace()
        # the solver reads the coefficients on the padded face grids
        bxp = np.zeros((nx + 1, ny + 2))
        bxp[:, 1:-1] = bx
        byp = np.zeros((nx + 2, ny + 1))
        byp[1:-1, :] = by
        dev = [_lib.to_dev(a, t.float64) for a in (bxp, byp, np.where(f, diag, 0.0), dinv)]
        op = _lib.Poisson.from_buffer_copy(self.op)
        op.bx, op.by, op.diag, op.dinv = (a.data_ptr() for a in dev)
        x0 = t.zeros((nx, ny), dtype=t.float64, device=_lib.device())  # no warm start, as a direct solve
        op.x0 = x0.data_ptr()
        op.cluster, op.mixed = 0, 0
        op.grid_ctas = 16 if nx * ny <= 262144 else 0
        return op, dev + [x0]

    def solve_variable(self, rhs, bx, by):
        """Solve div(b grad p) = rhs with face coefficients b = 1/rho (cfd2d/pressure.py:187-244):
        bx (nx+1, ny) on the x faces (face nx couples columns nx-1 and 0 when periodic),
        by (nx, ny+1). The reference rebuilds the matrix and solves it directly on every
        call; here the diagonal is assembled in its order on the host and the system is
        solved by the variable-coefficient PCG on the device to a relative residual of
        1e-13. The time step itself builds the operator on the device."""
        t = _lib.torch()
        op, _keep = self.variable_operator(bx, by)
        r = _lib.to_dev(np.asarray(rhs, dtype=np.float64), t.float64)
        p = t.empty_like(r)
        st = t.zeros(1, dtype=t.int32, device=_lib.device())
        rc = _lib.lib().cfd2d_pressure_solve(C.byref(op), _lib.ptr(r), _lib.ptr(p), 1e-13, 20000,
                                             _lib.ptr(self._d_iters), _lib.ptr(st), _lib.stream_ptr())
        _lib.check(rc, "cfd2d_pressure_solve (variable coefficients)")
        info = st.cpu().numpy()
        self.last_iterations = int(self._d_iters[0].item())
        if info[0] & _lib.S_BARRIER_TIMEOUT:
            raise RuntimeError("pressure solve abandoned: a bounded inter-block wait timed out")
        if info[0] & _lib.S_CG_MAXITER:
            warnings.warn("CG-Drucklöser (variable Dichte) nicht konvergiert")
        return p.cpu().numpy()
