"""Host-side mirror of UBOLT's operator and preconditioner interface over the C ABI.

Names and argument meaning follow the reference classes the library stands
in for (stevendargaville/UBOLT):

    TransportOperator  - MatShell MULT / unscattered MULT / diagonal
                         (include/ubolt/transport_operator.hpp, src/transport_operatork.kokkos.cxx)
    ElementBlockInverse - removal stage blocks (include/ubolt/block_inverse.hpp)
    GroupTransfer      - external source, scalar-flux cache, group transfer
                         (include/ubolt/multigroup.hpp:103-182)
    angular_integral   - UboltAngularIntegral (include/ubolt/sn_quadrature.hpp:163-171)
    fill_inflow        - UboltFillInflow, ghost-flux path (include/ubolt/coo_pattern.hpp:68)

Vectors are torch CUDA tensors (float64, or float32 for the *_f32 paths)
in UBOLT's row layout; torch only supplies device memory and the stream.
Errors raise ubolt_b200._lib.UboltError carrying the library's status.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import lib, check


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class Context:
    """ubolt_ctx: geometry and ordinates on one device (the current one).

    A problem.Geometry gives the DG backend (UnstructuredDG); a
    problem.CGGeometry the CG-SUPG one (UnstructuredCG, zeta its thin-cell
    SUPG parameter), whose nodes are the mesh's vertices and whose cells -
    what cross sections and sources are given on - are its elements."""

    def __init__(self, geometry, quad, zeta=0.5):
        self.geometry, self.quad = geometry, quad
        h = _lib.vp()
        gs, qs = geometry.struct(), quad.struct()
        self.is_cg = isinstance(geometry.struct(), _lib.CGGeometry)
        if self.is_cg:
            check(lib.ubolt_ctx_create_cg(C.byref(gs), C.byref(qs), float(zeta), C.byref(h)))
        else:
            check(lib.ubolt_ctx_create(C.byref(gs), C.byref(qs), C.byref(h)))
        self.handle = h
        self.device = torch.device("cuda", torch.cuda.current_device())
        rows, nodes, cells = C.c_int64(), C.c_int64(), C.c_int64()
        nb, na = C.c_int32(), C.c_int32()
        check(lib.ubolt_ctx_sizes(h, C.byref(rows), C.byref(nodes), C.byref(cells), C.byref(nb), C.byref(na)))
        self.n_rows, self.n_nodes, self.n_cells = rows.value, nodes.value, cells.value
        self.n_basis, self.n_angles = nb.value, na.value
        self._group = None

    def close(self):
        if getattr(self, "handle", None):
            lib.ubolt_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def vector(self, dtype=torch.float64, fill=None):
        v = torch.empty(self.n_rows, dtype=dtype, device=self.device)
        if fill is not None:
            v.fill_(fill)
        return v

    def set_group(self, sigma_t, sigma_s_within, stream=None):
        """Point the terms at a group's cross sections (device float64, per cell).
        The tensors are referenced, not copied - keep them alive."""
        self._group = (sigma_t, sigma_s_within)
        check(lib.ubolt_set_group(self.handle, _p(sigma_t), _p(sigma_s_within), _stream(stream)))


class TransportOperator:
    """The shell operator A = L - S and its unscattered twin L."""

    def __init__(self, ctx):
        self.ctx = ctx

    def _call(self, fn64, fn32, x, y, stream):
        if y is None:
            y = torch.empty_like(x)
        fn = fn64 if x.dtype == torch.float64 else fn32
        check(fn(self.ctx.handle, _p(x), _p(y), _stream(stream)))
        return y

    def mult(self, x, y=None, stream=None):
        """y = (L - S) x (ShellMatMultApply)."""
        return self._call(lib.ubolt_apply, lib.ubolt_apply_f32, x, y, stream)

    def mult_unscattered(self, x, y=None, stream=None):
        """y = L x (UnscatteredMatMultApply)."""
        return self._call(lib.ubolt_apply_unscattered, lib.ubolt_apply_unscattered_f32, x, y, stream)

    def mult_transpose(self, x, y=None, stream=None):
        """y = (L - S)^T x."""
        return self._call(lib.ubolt_apply_adjoint, lib.ubolt_apply_adjoint_f32, x, y, stream)

    def diagonal(self, d=None, stream=None):
        d = self.ctx.vector() if d is None else d
        check(lib.ubolt_diagonal(self.ctx.handle, _p(d), _stream(stream)))
        return d


class ElementBlockInverse:
    """D^{-1} for the (cell, angle) element blocks of streaming + removal."""

    def __init__(self, ctx):
        self.ctx = ctx

    def setup(self, stream=None):
        """Check every block is invertible; raises UBOLT_ERR_SINGULAR otherwise."""
        n = C.c_int64()
        check(lib.ubolt_block_setup(self.ctx.handle, C.byref(n), _stream(stream)))
        return n.value

    def apply(self, x, y=None, stream=None):
        y = torch.empty_like(x) if y is None else y
        fn = lib.ubolt_block_apply if x.dtype == torch.float64 else lib.ubolt_block_apply_f32
        check(fn(self.ctx.handle, _p(x), _p(y), _stream(stream)))
        return y

    def apply_transpose(self, x, y=None, stream=None):
        y = torch.empty_like(x) if y is None else y
        check(lib.ubolt_block_apply_transpose(self.ctx.handle, _p(x), _p(y), _stream(stream)))
        return y

    def inverse(self, stream=None):
        c = self.ctx
        inv = torch.empty(c.n_cells * c.n_angles * c.n_basis * c.n_basis, dtype=torch.float64, device=c.device)
        check(lib.ubolt_block_inverse(c.handle, _p(inv), _stream(stream)))
        return inv


def angular_integral(ctx, psi, phi=None, stream=None):
    phi = torch.empty(ctx.n_nodes, dtype=psi.dtype, device=psi.device) if phi is None else phi
    fn = lib.ubolt_scalar_flux if psi.dtype == torch.float64 else lib.ubolt_scalar_flux_f32
    check(fn(ctx.handle, _p(psi), _p(phi), _stream(stream)))
    return phi


def current(ctx, psi, cur=None, stream=None):
    """J(node, d) = sum_a w_a Omega_a,d psi(node, a), as (n_nodes, dim)."""
    cur = torch.empty(ctx.n_nodes, ctx.geometry.dim, dtype=torch.float64, device=psi.device) if cur is None else cur
    check(lib.ubolt_current(ctx.handle, _p(psi), _p(cur), _stream(stream)))
    return cur


def expand_p1(ctx, phi, cur, psi=None, stream=None):
    """psi(node, a) = phi(node) / W + T^{-1} Omega_a . J(node): the P1 field with these moments."""
    psi = ctx.vector() if psi is None else psi
    check(lib.ubolt_expand_p1(ctx.handle, _p(phi), _p(cur), _p(psi), _stream(stream)))
    return psi


def fill_inflow(ctx, side_inflow, b, stream=None):
    """b += the ghost-flux vacuum inflow (side_inflow: angle-integrated, per side)."""
    s = np.zeros(6)
    s[:len(side_inflow)] = side_inflow
    check(lib.ubolt_add_ghost_inflow(ctx.handle, s.ctypes.data_as(_lib.dp), _p(b), _stream(stream)))
    return b


class GroupTransfer:
    """External source and group-to-group transfer of the per-node backends."""

    def __init__(self, ctx, sigma_s_table, source_table):
        """sigma_s_table[g_from][g_to], source_table[g]: device float64 per-cell tensors."""
        self.ctx = ctx
        self.sigma_s = sigma_s_table
        self.source = source_table
        self.phi = [None] * len(source_table)

    def add_external(self, g, b, stream=None):
        check(lib.ubolt_add_source(self.ctx.handle, _p(self.source[g]), _p(b), _stream(stream)))
        return b

    def set_scalar_flux(self, g, psi, stream=None):
        self.phi[g] = angular_integral(self.ctx, psi, self.phi[g], stream)
        return self.phi[g]

    def add_transfer(self, g_from, g_to, b, stream=None):
        if self.phi[g_from] is None:
            raise _lib.UboltError(4, f"no scalar flux cached for group {g_from}")
        check(lib.ubolt_add_transfer(self.ctx.handle, _p(self.phi[g_from]), _p(self.sigma_s[g_from][g_to]), _p(b),
                                     _stream(stream)))
        return b


class Sweep:
    """psi = L^{-1} q for every ordinate - the streaming stage (PCAIR's place)."""

    def __init__(self, ctx, patch_size=0, factor_limit=None):
        self.ctx = ctx
        check(lib.ubolt_sweep_setup(ctx.handle, patch_size))
        if factor_limit is not None:
            self.set_factor_limit(factor_limit)

    def set_factor_limit(self, nbytes):
        """Cache each cell-ordinate's B^{-1} and couplings (-1 automatic, 0 never, else a byte limit)."""
        check(lib.ubolt_sweep_set_factor_limit(self.ctx.handle, int(nbytes)))

    KERNELS = {"auto": _lib.SWEEP_AUTO, "tasks": _lib.SWEEP_TASKS, "wave": _lib.SWEEP_WAVE}

    def set_kernel(self, kind):
        """"tasks" (any mesh), "wave" (one block per ordinate; acyclic meshes) or "auto"."""
        check(lib.ubolt_sweep_set_kernel(self.ctx.handle, self.KERNELS[kind]))

    def apply(self, q, psi=None, stream=None):
        psi = torch.empty_like(q) if psi is None else psi
        fn = lib.ubolt_sweep if q.dtype == torch.float64 else lib.ubolt_sweep_f32
        check(fn(self.ctx.handle, _p(q), _p(psi), _stream(stream)))
        return psi

    def apply_iso(self, phi, psi, u=None, ordinate_major=False, stream=None):
        """psi = L^{-1} (u_a phi(node)): phi FP64 per node, psi in its own precision."""
        fn = lib.ubolt_sweep_iso if psi.dtype == torch.float64 else lib.ubolt_sweep_iso_f32
        check(fn(self.ctx.handle, _p(phi), _p(u), _p(psi), int(bool(ordinate_major)), _stream(stream)))
        return psi

    def status(self, stream=None):
        info = _lib.SweepInfo()
        check(lib.ubolt_sweep_status(self.ctx.handle, C.byref(info), _stream(stream)))
        return {k: getattr(info, k) for k, _ in info._fields_ if k != "pad_"}


class TransportSolver:
    """GMRES (right-preconditioned) on the current group: TransportSolver::solve."""

    def __init__(self, ctx, rtol=1e-8, precision="fp64", pc="sweep", restart=30, max_it=500, inner_rtol=1e-5,
                 max_outer=10, krylov="auto"):
        self.ctx = ctx
        o = _lib.SolveOptions()
        lib.ubolt_solve_defaults(C.byref(o))
        o.rtol, o.inner_rtol, o.max_it, o.restart, o.max_outer = rtol, inner_rtol, max_it, restart, max_outer
        o.krylov = {"auto": 0, "full": 1}[krylov]
        o.precision = {"fp64": _lib.PRECISION_FP64, "mixed": _lib.PRECISION_MIXED}[precision]
        o.pc = {"none": _lib.PC_NONE, "block": _lib.PC_BLOCK, "sweep": _lib.PC_SWEEP,
                "sweep+dsa": _lib.PC_SWEEP_DSA, "block+dsa": _lib.PC_BLOCK_DSA}[pc]
        self.opts = o
        check(lib.ubolt_solver_setup(ctx.handle, C.byref(o)))

    def solve(self, b, x=None, stream=None, x_zero=True):
        x = torch.zeros_like(b) if x is None else x
        self.opts.x_zero = 1 if x_zero else 0
        st = _lib.SolveStats()
        check(lib.ubolt_solve(self.ctx.handle, _p(b), _p(x), C.byref(self.opts), C.byref(st), _stream(stream)))
        return x, {k: getattr(st, k) for k, _ in st._fields_ if k != "pad_"}

    def solve_host_batch(self, bs, xs, stream=None):
        """x_i = A^{-1} b_i for CPU tensors b_i (pinned memory for the copies
        to overlap the solves), each solve from zero: the upload of the next
        b and the download of the previous x run while a solve runs. xs are
        filled once `stream` (default: the current one) is synchronised.
        Returns the per-solve stats."""
        n = len(bs)
        if n != len(xs):
            raise ValueError("solve_host_batch: as many x as b")
        for t in list(bs) + list(xs):
            if t.device.type != "cpu" or t.dtype != torch.float64 or not t.is_contiguous() or t.numel() != self.ctx.n_rows:
                raise ValueError("solve_host_batch: contiguous float64 CPU tensors of n_rows entries")
        bp = (C.c_void_p * n)(*[t.data_ptr() for t in bs])
        xp = (C.c_void_p * n)(*[t.data_ptr() for t in xs])
        st = (_lib.SolveStats * n)()
        check(lib.ubolt_solve_host_batch(self.ctx.handle, n, bp, xp, C.byref(self.opts), st, _stream(stream)))
        return [{k: getattr(s_, k) for k, _ in s_._fields_ if k != "pad_"} for s_ in st]

    def solve_adjoint(self, g, lam=None, stream=None, x_zero=True):
        """(L - S)^T lambda = g with the hand-written transpose operator."""
        lam = torch.zeros_like(g) if lam is None else lam
        self.opts.x_zero = 1 if x_zero else 0
        st = _lib.SolveStats()
        check(lib.ubolt_solve_adjoint(self.ctx.handle, _p(g), _p(lam), C.byref(self.opts), C.byref(st),
                                      _stream(stream)))
        return lam, {k: getattr(st, k) for k, _ in st._fields_ if k != "pad_"}


def response_source(ctx, detector, g=None, stream=None):
    """g += the adjoint source of J = sum_c detector(c) V_c phi(c, basis 0)."""
    g = ctx.vector(fill=0.0) if g is None else g
    check(lib.ubolt_add_response_source(ctx.handle, _p(detector), _p(g), _stream(stream)))
    return g


def gradient(ctx, psi, lam, stream=None):
    """(dJ/dsigma_t, dJ/dsigma_s) per cell from the forward and adjoint fluxes."""
    gt = torch.empty(ctx.n_cells, dtype=torch.float64, device=psi.device)
    gs = torch.empty_like(gt)
    check(lib.ubolt_gradient(ctx.handle, _p(psi), _p(lam), _p(gt), _p(gs), _stream(stream)))
    return gt, gs


class _Response(torch.autograd.Function):
    @staticmethod
    def forward(fctx, sigma_t, sigma_s, model):
        st = sigma_t.detach().contiguous().double()
        ss = sigma_s.detach().contiguous().double()
        model.ctx.set_group(st, ss)
        psi, stats = model.solver.solve(model.b)
        model.last_forward = stats
        J = torch.dot(model.g, psi)
        fctx.model = model
        fctx.keep = (st, ss)
        fctx.save_for_backward(psi)
        return J

    @staticmethod
    def backward(fctx, grad_J):
        (psi,) = fctx.saved_tensors
        model = fctx.model
        model.ctx.set_group(*fctx.keep)
        lam, stats = model.solver.solve_adjoint(model.g)
        model.last_adjoint = stats
        gt, gs = gradient(model.ctx, psi, lam)
        return grad_J * gt, grad_J * gs, None


class DetectorResponse:
    """J(sigma_t, sigma_s) = sum_c detector(c) V_c phi(c, 0) of the fixed-source
    solution, differentiable with respect to both per-cell cross sections
    through the adjoint solve (a torch.autograd.Function over the C ABI)."""

    def __init__(self, ctx, source_cell, detector_cell, side_inflow=None, **solver_opts):
        self.ctx = ctx
        dev = ctx.device
        self.source = torch.as_tensor(source_cell, dtype=torch.float64, device=dev)
        self.detector = torch.as_tensor(detector_cell, dtype=torch.float64, device=dev)
        self.b = ctx.vector(fill=0.0)
        if side_inflow is not None:
            fill_inflow(ctx, side_inflow, self.b)
        check(lib.ubolt_add_source(ctx.handle, _p(self.source), _p(self.b), _stream()))
        self.g = response_source(ctx, self.detector)
        self.solver = TransportSolver(ctx, **solver_opts)

    def __call__(self, sigma_t, sigma_s):
        return _Response.apply(sigma_t, sigma_s, self)


def group_tables(ctx, sigma_t, sigma_s, source):
    """The cross-section and source tables on the device, float64, contiguous:
    (st[g], ss[g][h], src[g]). NumPy arrays are uploaded; device tensors are
    used as they are (converted only if their dtype or layout differs)."""
    dev = ctx.device

    def as_dev(a):
        if isinstance(a, torch.Tensor):
            return a.to(device=dev, dtype=torch.float64).contiguous()
        return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)

    G = len(sigma_t)
    st = [as_dev(sigma_t[g]) for g in range(G)]
    ss = [[as_dev(sigma_s[g][h]) for h in range(G)] for g in range(G)]
    src = [as_dev(source[g]) for g in range(G)]
    return st, ss, src


def solve_groups(ctx, sigma_t, sigma_s, source, side_inflow=None, dsa=None, keep_psi=False, solver=None,
                 outer_rtol=1e-8, outer_max_it=1000, outer_inner_gamma=0.01, outer_store="angular",
                 outer_recon="tol", outer_info=None, **solver_opts):
    """The group loop of the reference driver (tests/transportk.kokkos.cxx:
    1036-1208): per group g, point the operator (and the DSA) at g's cross
    sections, build b = inflow + source + the transfer out of the other
    groups' cached scalar fluxes, solve, and cache phi_g.

    Downscatter only: one pass over the groups in order, exact
    (docs/architecture.md:362-364).

    With upscatter (some group scatters into a lower one), the reference's
    outer iteration, angular store (one psi per group, -outer_store angular):
    the first pass solves every group in order, a thermal group (from g_up,
    the lowest group anything scatters up into) reading zero for the groups
    not solved yet; each later pass re-solves the thermal block, every group
    warm-started from its own last psi and taking every other group's
    transfer. After a pass, change = ||phi_new - phi_old|| / ||phi_new||
    over the thermal block, rho the ratio of successive changes, and the
    error estimate change rho / (1 - rho); the iteration stops when that
    estimate is below outer_rtol (or the change is exactly zero), on a pass
    whose thermal solves ran at the solver's own rtol: the inner rtol of a
    thermal pass is max(rtol, outer_inner_gamma min(change, 1)) until the
    test first passes, then one more pass at rtol. outer_rtol below the
    solver's rtol is refused (a warm start that moves by less than its rtol
    takes no iterations, and the outer test would pass falsely).

    outer_store "moments" (-outer_store moments) keeps, in place of one psi
    per group, each thermal group's scalar flux and current and ONE psi that
    every solve reuses: a thermal solve after the first pass starts from the
    P1 expansion of the group's last moments, then (outer_recon) Richardson
    steps on L_g psi = c, c = b + the within-group scatter of the group's last
    phi, each step psi += sweep(c - L_g psi) - "tol": until ||c - L_g psi|| <=
    rtol ||c||, at most 40 steps; "none": the P1 guess alone; an int: that
    many steps. A step that does not reduce the residual is reverted and ends
    the reconstruction (tests/transportk.kokkos.cxx:282-334, 650-720). With the
    exact sweep as the streaming stage, one step solves L_g psi = c.

    sigma_t: (G, n_cells), sigma_s: (G, G, n_cells) [from, to], source:
    (G, n_cells) - NumPy arrays, or device tensors (used in place, as from
    group_tables). solver: a TransportSolver set up on ctx (else one is made
    from solver_opts; its workspace allocation is then part of the call).
    outer_info: a dict, filled with the outer iteration's record. Returns
    (phi per group, stats of each group's last solve[, psi per group])."""
    st, ss, src = group_tables(ctx, sigma_t, sigma_s, source)
    G = len(st)
    # Which transfers are nonzero, in one read-back for every pair
    nonzero = [[False] * G for _ in range(G)]
    if G > 1:
        pairs = [(g, h) for g in range(G) for h in range(G) if g != h]
        flags = torch.stack([torch.count_nonzero(ss[g][h]) for g, h in pairs]).tolist()
        for (g, h), n in zip(pairs, flags):
            nonzero[g][h] = n > 0
    g_up = min([h for g in range(G) for h in range(g) if nonzero[g][h]], default=G)
    transfer = GroupTransfer(ctx, ss, src)
    solver = TransportSolver(ctx, **solver_opts) if solver is None else solver
    b = ctx.vector()

    def rhs(g, from_all):
        ctx.set_group(st[g], ss[g][g])
        if dsa is not None:
            dsa.set_group()
        b.zero_()
        if side_inflow is not None:
            fill_inflow(ctx, side_inflow, b)
        transfer.add_external(g, b)
        for h in range(G if from_all else g):
            if h != g and nonzero[h][g]:
                transfer.add_transfer(h, g, b)

    if g_up == G:
        psi = ctx.vector(fill=0.0)
        phis, stats, psis = [], [], []
        for g in range(G):
            rhs(g, False)
            psi, s = solver.solve(b, psi)
            transfer.set_scalar_flux(g, psi)
            transfer.phi[g] = transfer.phi[g].clone()
            phis.append(transfer.phi[g])
            stats.append(s)
            if keep_psi:
                psis.append(psi.clone())
        if outer_info is not None:
            outer_info.update(upscatter=False, outer_iterations=1, converged=True)
        return (phis, stats, psis) if keep_psi else (phis, stats)

    if outer_store not in ("angular", "moments"):
        raise _lib.UboltError(1, f"outer_store is angular or moments, was given {outer_store!r}")
    if outer_recon == "tol":
        recon_steps, recon_tol = 40, True
    elif outer_recon == "none":
        recon_steps, recon_tol = 0, False
    elif isinstance(outer_recon, int) and outer_recon >= 0:
        recon_steps, recon_tol = outer_recon, False
    else:
        raise _lib.UboltError(1, f"outer_recon is 'tol', 'none' or a step count, was given {outer_recon!r}")
    moments = outer_store == "moments"
    inner_rtol = solver.opts.rtol
    if outer_rtol < inner_rtol:
        raise _lib.UboltError(1, f"outer_rtol {outer_rtol:g} is below the solver's rtol {inner_rtol:g}: a warm start "
                                 "that moves by less than its rtol takes no iterations and the outer test would pass "
                                 "falsely")
    if moments:
        # One psi for every solve, the three reconstruction vectors, and each
        # thermal group's current
        one = ctx.vector(fill=0.0)
        psis = [one] * G
        rv, tv, dz = (ctx.vector() for _ in range(3)) if recon_steps > 0 else (None, None, None)
        cur = [torch.zeros(ctx.n_nodes, ctx.geometry.dim, dtype=torch.float64, device=ctx.device)
               for _ in range(G)]
        op = TransportOperator(ctx)
        sw = Sweep.__new__(Sweep)
        sw.ctx = ctx
    else:
        psis = [ctx.vector(fill=0.0) for _ in range(G)]
    for g in range(g_up, G):
        transfer.phi[g] = torch.zeros(ctx.n_nodes, dtype=torch.float64, device=ctx.device)
    new_phi = torch.empty(ctx.n_nodes, dtype=torch.float64, device=ctx.device)
    stats = [None] * G
    outer_change, final_sweep, converged = 0.0, False, False
    changes, inner_its = [], 0
    recon = {"steps": 0, "solves": 0, "safeguarded": 0}
    err = float("inf")

    def reconstruct(g, rtol):
        """The moments store's starting psi for thermal group g (into psis[g]):
        Reconstruct, tests/transportk.kokkos.cxx:282-334."""
        psi = psis[g]
        expand_p1(ctx, transfer.phi[g], cur[g], psi)
        recon["solves"] += 1
        if recon_steps == 0:
            return
        # r = c - L psi, c = b + the within-group scatter at the last phi
        rv.copy_(b)
        transfer.add_transfer(g, g, rv)
        target = rtol * float(torch.linalg.norm(rv)) if recon_tol else -1.0
        op.mult_unscattered(psi, tv)
        rv.sub_(tv)
        r_norm = float(torch.linalg.norm(rv))
        k = 0
        while k < recon_steps and r_norm > target:
            sw.apply(rv, dz)          # dz = L^{-1} r (r is rebuilt below)
            k += 1
            torch.add(psi, dz, out=tv)
            op.mult_unscattered(tv, rv)
            torch.sub(b, rv, out=rv)
            transfer.add_transfer(g, g, rv)
            new_norm = float(torch.linalg.norm(rv))
            if not new_norm < r_norm:  # NaN too: the step is dropped
                recon["safeguarded"] += 1
                break
            psi.copy_(tv)
            r_norm = new_norm
        recon["steps"] += k

    try:
        for outer in range(outer_max_it):
            sweep_rtol = inner_rtol
            if outer_inner_gamma > 0.0 and not final_sweep:
                sweep_rtol = max(inner_rtol, outer_inner_gamma * (1.0 if outer == 0 else min(outer_change, 1.0)))
            sums = torch.zeros(2, dtype=torch.float64, device=ctx.device)
            for g in range(0 if outer == 0 else g_up, G):
                thermal = g >= g_up
                rhs(g, thermal)
                solver.opts.rtol = sweep_rtol if thermal else inner_rtol
                if moments and thermal and outer >= 1:
                    reconstruct(g, solver.opts.rtol)
                # From the second pass a thermal solve starts from its last psi
                # (angular) or the reconstruction (moments); the first from zero
                psis[g], s = solver.solve(b, psis[g], x_zero=(outer == 0 or not thermal))
                stats[g] = s
                inner_its += s["iterations"]
                if thermal:
                    angular_integral(ctx, psis[g], new_phi)
                    sums[0] += torch.sum((new_phi - transfer.phi[g]) ** 2)
                    sums[1] += torch.sum(new_phi * new_phi)
                    transfer.phi[g].copy_(new_phi)
                    if moments:
                        current(ctx, psis[g], cur[g])
                else:
                    transfer.set_scalar_flux(g, psis[g])
            change_sq, norm_sq = sums.tolist()
            change = (change_sq / norm_sq) ** 0.5 if norm_sq > 0.0 else change_sq ** 0.5
            have_rho = outer >= 2 and outer_change > 0.0
            rho = change / outer_change if have_rho else 0.0
            outer_change = change
            err = change * rho / (1.0 - rho) if have_rho and rho < 1.0 else float("inf")
            changes.append(change)
            if change == 0.0 or err < outer_rtol:
                if sweep_rtol == inner_rtol:
                    converged = True
                    break
                final_sweep = True
    finally:
        solver.opts.rtol = inner_rtol
    if outer_info is not None:
        outer_info.update(upscatter=True, g_up=g_up, outer_iterations=len(changes), changes=changes,
                          error_estimate=err, inner_iterations=inner_its, converged=converged, store=outer_store,
                          reconstruction_steps=recon["steps"], reconstructed_solves=recon["solves"],
                          reconstruction_safeguarded=recon["safeguarded"])
    if not converged:
        raise _lib.UboltError(5, f"outer iteration not converged after {len(changes)} passes: error estimate "
                                 f"{err:.3e}, outer_rtol {outer_rtol:g}")
    phis = [transfer.phi[g].clone() for g in range(G)]
    return (phis, stats, psis) if keep_psi else (phis, stats)


class DSAPrecon:
    """The diffusion correction y = P D^{-1} R x (include/ubolt/dsa.hpp)."""

    def __init__(self, ctx, penalty=4.0, consistent_d=True, consistent_power=1.5, inner_iterations=30,
                 void_sigma_t=0.0, void_bridge=True, void_d=0.0):
        self.ctx = ctx
        o = _lib.DsaOptions()
        lib.ubolt_dsa_defaults(C.byref(o))
        o.penalty, o.consistent_d, o.consistent_power = penalty, int(consistent_d), consistent_power
        o.inner_iterations = inner_iterations
        o.void_sigma_t, o.void_bridge, o.void_d = void_sigma_t, int(void_bridge), void_d
        if ctx.is_cg:
            # DSACG on the context's own tables (the penalty and consistent-D
            # options are the DG operators' and do not apply)
            check(lib.ubolt_dsa_setup(ctx.handle, None, C.byref(o)))
        else:
            gs = ctx.geometry.struct()
            check(lib.ubolt_dsa_setup(ctx.handle, C.byref(gs), C.byref(o)))

    def set_group(self, stream=None):
        """Refill D for the context's current group (call after Context.set_group)."""
        check(lib.ubolt_dsa_set_group(self.ctx.handle, _stream(stream)))

    def void_info(self):
        """The void policy's outcome for the current group: (void cells, bridged, mean chord)."""
        n, br, ch = C.c_int64(0), C.c_int32(0), C.c_double(0.0)
        check(lib.ubolt_dsa_void_info(self.ctx.handle, C.byref(n), C.byref(br), C.byref(ch)))
        return n.value, bool(br.value), ch.value

    def apply(self, x, y=None, stream=None):
        y = torch.empty_like(x) if y is None else y
        check(lib.ubolt_dsa_apply(self.ctx.handle, _p(x), _p(y), _stream(stream)))
        return y

    def spmv(self, u, v=None, stream=None):
        v = torch.empty_like(u) if v is None else v
        check(lib.ubolt_dsa_spmv(self.ctx.handle, _p(u), _p(v), _stream(stream)))
        return v

    def restrict(self, x, stream=None):
        rhs = torch.empty(self.ctx.n_nodes, dtype=torch.float64, device=x.device)
        check(lib.ubolt_dsa_restrict(self.ctx.handle, _p(x), _p(rhs), _stream(stream)))
        return rhs

    def prolong(self, u, stream=None):
        y = self.ctx.vector()
        check(lib.ubolt_dsa_prolong(self.ctx.handle, _p(u), _p(y), _stream(stream)))
        return y

    def matrix(self):
        """D as a SciPy CSR matrix over the nodes, from the assembled blocks."""
        import scipy.sparse as sp
        g = self.ctx.geometry
        nc, F, nb = g.n_cells, g.faces_per_cell, g.n_basis
        blocks = np.zeros(nc * (F + 1) * nb * nb)
        check(lib.ubolt_dsa_matrix(self.ctx.handle, blocks.ctypes.data_as(_lib.dp)))
        blocks = blocks.reshape(nc, F + 1, nb, nb)
        nbr = np.concatenate([g.face_neighbour.reshape(nc, F), np.arange(nc)[:, None]], axis=1)
        c = np.repeat(np.arange(nc), F + 1).reshape(nc, F + 1)
        rows = (c[:, :, None, None] * nb + np.arange(nb)[None, None, :, None]).repeat(nb, axis=3)
        cols = (nbr[:, :, None, None] * nb + np.arange(nb)[None, None, None, :]).repeat(nb, axis=2)
        keep = np.broadcast_to((nbr >= 0)[:, :, None, None], rows.shape)
        return sp.csr_matrix((blocks[keep], (rows[keep], cols[keep])), shape=(nc * nb, nc * nb))
