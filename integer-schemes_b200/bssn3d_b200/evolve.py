"""``BSSNEvolution`` — RK4 time integration (3D/src/bssn3d/evolve.py:24-194)
on the fused B200 stage kernel.

Each RK4 stage is ONE launch of ``bssn_b200_rk4_stage``: derivatives, KO
dissipation, the BSSN algebra and the stage update (with algebraic
enforcement after the last stage) in one kernel. A step is four launches
(+ a ghost sync per stage for periodic boundaries) and ``evolve`` replays the
step as a captured CUDA graph. Stage times are t, t+dt/2, t+dt/2, t+dt with
the full dt in the CAHD factor (evolve.py:121-131).

``integrator="rk4_2_1"`` or ``"rk4_2_2"`` selects the 2-step / 3-stage MSRK
recurrence instead (evolve.py:139-183; coefficients in ``msrk``): three
launches of ``bssn_b200_msrk_stage`` per step, each stage folding its rate
into every later combination it appears in, so no k_i is stored except
f(y_n), which the next step reuses.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib, msrk
from .fused_rhs import _stream_handle, as_device_state, device_scalars, scalars
from .grid import Grid
from .rhs import BSSNSolver
from .state import BSSNState, PhysicsParams


class BSSNEvolution:
    def __init__(self, grid: Grid, params: PhysicsParams = None, order: int = 6,
                 ko_sigma: float = 0.0, bc: str = "periodic", precision: str = "fp64",
                 scheme: str = "cuda_b200", ko_order: int = 8, integrator: str = "rk4"):
        self.grid = grid
        self.params = params or PhysicsParams()
        self.solver = BSSNSolver(grid, self.params, order, precision=precision,
                                 scheme=scheme, ko_order=ko_order)
        self.ng = grid.ng
        self.ko_sigma = float(ko_sigma)
        self.ko_order = ko_order
        if bc not in ("periodic", "none"):
            raise ValueError(f"unknown bc {bc!r} (periodic or none)")
        self.bc = bc
        self.integrator = integrator
        self._msrk = None
        if integrator != "rk4":
            self._msrk = msrk.get(integrator)
            self._coef = (ctypes.c_double * 9)(*self._msrk.coef)
        self._bufs = {}
        self._graph = None

    # ------------------------------------------------------------------
    def _buffers(self, U: torch.Tensor):
        key = (tuple(U.shape), U.device)
        b = self._bufs.get(key)
        if b is None:
            b = {name: torch.empty_like(U) for name in ("Ya", "Yb", "ACC")}
            if self.bc == "periodic":
                b["Ys"] = torch.empty_like(U)
            self._bufs = {key: b}
        return b

    def _S(self, t: float, dt: float, device) -> torch.Tensor:
        g = self.grid
        return device_scalars(scalars(self.params, g.dx, g.dy, g.dz, dt, t), device)

    def _stage(self, stage, U, Y, ACC, YNEXT, S):
        lib = _lib.load()
        _, Sx, Sy, Sz = U.shape
        src = Y
        if self.bc == "periodic":
            Ys = self._buffers(U)["Ys"]
            Ys.copy_(Y)
            _lib.check(lib.bssn_b200_periodic_sync(_stream_handle(U.device), Ys.data_ptr(),
                                                   Sx, Sy, Sz, self.ng))
            src = Ys
        p = self.params
        rc = lib.bssn_b200_rk4_stage(_stream_handle(U.device), stage, U.data_ptr(), src.data_ptr(),
                                     ACC.data_ptr(), YNEXT.data_ptr(), S.data_ptr(),
                                     self.ko_sigma, self.ko_order, p.chi_floor, p.alpha_floor,
                                     Sx, Sy, Sz)
        _lib.check(rc)

    def _mstage(self, stage, U, Y, ACC, OUT, OUT2, OUT3, S):
        lib = _lib.load()
        _, Sx, Sy, Sz = U.shape
        src = Y
        if self.bc == "periodic":
            Ys = self._buffers(U)["Ys"]
            Ys.copy_(Y)
            _lib.check(lib.bssn_b200_periodic_sync(_stream_handle(U.device), Ys.data_ptr(),
                                                   Sx, Sy, Sz, self.ng))
            src = Ys
        p = self.params
        ptr = lambda t: None if t is None else t.data_ptr()
        rc = lib.bssn_b200_msrk_stage(_stream_handle(U.device), stage, U.data_ptr(), src.data_ptr(),
                                      ptr(ACC), OUT.data_ptr(), ptr(OUT2), ptr(OUT3), S.data_ptr(),
                                      ctypes.cast(self._coef, ctypes.c_void_p), self.ko_sigma,
                                      self.ko_order, p.chi_floor, p.alpha_floor, Sx, Sy, Sz)
        _lib.check(rc)

    def _msrk_step_inplace(self, U: torch.Tensor, KP: torch.Tensor, S: torch.Tensor):
        """One MSRK step in place: U <- y_{n+1}, KP <- f(y_n) (was f(y_{n-1}))."""
        b = self._buffers(U)
        Y2, Q3, QF = b["Ya"], b["Yb"], b["ACC"]
        self._mstage(0, U, U, KP, Y2, Q3, QF, S)
        self._mstage(1, Q3, Y2, QF, Q3, None, None, S)
        self._mstage(2, QF, Q3, None, U, None, None, S)

    def _startup_inplace(self, U: torch.Tensor, KP: torch.Tensor, S: torch.Tensor):
        """The RK4 step that starts an MSRK run, keeping its stage-0 rate
        f(y_0) (evolve.py:173-175: f0 = rhs(y0), y1 = step(y0))."""
        b = self._buffers(U)
        self._stage(0, U, U, b["ACC"], b["Ya"], S)
        KP.copy_(b["ACC"])
        self._stage(1, U, b["Ya"], b["ACC"], b["Yb"], S)
        self._stage(2, U, b["Yb"], b["ACC"], b["Ya"], S)
        self._stage(3, U, b["Ya"], b["ACC"], U, S)

    def _advance_time(self, S: torch.Tensor):
        _lib.check(_lib.load().bssn_b200_advance_time(_stream_handle(S.device), S.data_ptr()))

    def _step_inplace(self, U: torch.Tensor, S: torch.Tensor):
        b = self._buffers(U)
        self._stage(0, U, U, b["ACC"], b["Ya"], S)
        self._stage(1, U, b["Ya"], b["ACC"], b["Yb"], S)
        self._stage(2, U, b["Yb"], b["ACC"], b["Ya"], S)
        self._stage(3, U, b["Ya"], b["ACC"], U, S)

    # ------------------------------------------------------------------
    def rhs(self, state: BSSNState, t: float = 0.0, dt: float = None) -> BSSNState:
        """rate = RHS + KO of ``state`` (evolve.py:86-91)."""
        U = as_device_state(state.data if isinstance(state, BSSNState) else state)
        dt = self.solver.dt if dt is None else dt
        S = self._S(t, dt, U.device)
        b = self._buffers(U)
        rate = torch.empty_like(U)
        self._stage(0, U, U, rate, b["Yb"], S)
        return BSSNState(rate)

    def enforce(self, state: BSSNState) -> BSSNState:
        U = as_device_state(state.data if isinstance(state, BSSNState) else state).clone()
        p = self.params
        n = U[0].numel()
        _lib.check(_lib.load().bssn_b200_enforce(_stream_handle(U.device), U.data_ptr(), n,
                                                 p.chi_floor, p.alpha_floor))
        return BSSNState(U)

    def step(self, state: BSSNState, t: float, dt: float) -> BSSNState:
        U = as_device_state(state.data if isinstance(state, BSSNState) else state).clone()
        self._step_inplace(U, self._S(t, dt, U.device))
        return BSSNState(U)

    def msrk_step(self, state: BSSNState, fprev, t: float, dt: float):
        """One MSRK step (evolve.py:139-153): returns (enforce(y_{n+1}), f(y_n)),
        the second being the next step's ``fprev``."""
        if self._msrk is None:
            raise ValueError("msrk_step needs an rk4_2_* integrator")
        U = as_device_state(state.data if isinstance(state, BSSNState) else state).clone()
        KP = as_device_state(fprev.data if isinstance(fprev, BSSNState) else fprev).clone()
        self._msrk_step_inplace(U, KP, self._S(t, dt, U.device))
        return BSSNState(U), BSSNState(KP)

    def evolve(self, state: BSSNState, dt: float, nsteps: int, t0: float = 0.0,
               use_graph: bool = True) -> BSSNState:
        """``nsteps`` steps from t0; the step is captured once as a CUDA graph
        and replayed, with the time advanced on the device (t <- t + dt).
        An MSRK integrator starts with one RK4 step that also keeps f(y_0),
        then runs the MSRK recurrence (evolve.py:167-183)."""
        U = as_device_state(state.data if isinstance(state, BSSNState) else state).clone()
        S = self._S(t0, dt, U.device)
        if nsteps <= 0:
            return BSSNState(U)
        if self._msrk is not None:
            KP = torch.empty_like(U)
            self._startup_inplace(U, KP, S)
            self._advance_time(S)
            if nsteps == 1:
                return BSSNState(U)
            if not use_graph:
                for _ in range(int(nsteps) - 1):
                    self._msrk_step_inplace(U, KP, S)
                    self._advance_time(S)
                return BSSNState(U)
            g, U_g, S_g, K_g = self.capture_msrk(U, S, KP)
            for _ in range(int(nsteps) - 1):
                g.replay()
            U.copy_(U_g)
            return BSSNState(U)
        if not use_graph:
            for _ in range(int(nsteps)):
                self._step_inplace(U, S)
                self._advance_time(S)
            return BSSNState(U)
        g, U_g, S_g = self.capture(U, S)
        for _ in range(int(nsteps)):
            g.replay()
        U.copy_(U_g)
        return BSSNState(U)

    def capture(self, U: torch.Tensor, S: torch.Tensor):
        """Capture one step (4 stages + time advance) on static buffers.
        Returns (graph, U_static, S_static); replay advances U_static by one step."""
        U_g = U.clone()
        S_g = S.clone()
        self._buffers(U_g)
        side = torch.cuda.Stream(U_g.device)
        side.wait_stream(torch.cuda.current_stream(U_g.device))
        with torch.cuda.stream(side):
            # warm the launch path (attributes, module load) outside the capture
            probe_U = U_g.clone()
            probe_S = S_g.clone()
            self._step_inplace(probe_U, probe_S)
        torch.cuda.current_stream(U_g.device).wait_stream(side)
        torch.cuda.synchronize(U_g.device)
        del probe_U, probe_S
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self._step_inplace(U_g, S_g)
            self._advance_time(S_g)
        # a graph does not own the memory it replays on: keep its static
        # tensors and stage buffers alive as long as the graph object is
        graph.static_tensors = (U_g, S_g, self._buffers(U_g))
        return graph, U_g, S_g

    def capture_msrk(self, U: torch.Tensor, S: torch.Tensor, KP: torch.Tensor):
        """Capture one MSRK step (3 stages + time advance) on static buffers.
        Returns (graph, U_static, S_static, KP_static); each replay advances
        U_static by one step and leaves f(y_n) in KP_static."""
        U_g, S_g, K_g = U.clone(), S.clone(), KP.clone()
        self._buffers(U_g)
        side = torch.cuda.Stream(U_g.device)
        side.wait_stream(torch.cuda.current_stream(U_g.device))
        with torch.cuda.stream(side):
            probe = (U_g.clone(), K_g.clone(), S_g.clone())
            self._msrk_step_inplace(*probe)
        torch.cuda.current_stream(U_g.device).wait_stream(side)
        torch.cuda.synchronize(U_g.device)
        del probe
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self._msrk_step_inplace(U_g, K_g, S_g)
            self._advance_time(S_g)
        graph.static_tensors = (U_g, S_g, K_g, self._buffers(U_g))
        return graph, U_g, S_g, K_g


class HostStepPipeline:
    """One RK4 step for each of a stream of HOST-resident states, with the
    copies overlapped with the compute: while step i runs on the device, the
    state of step i+1 is copied in and the result of step i-1 is copied out.

    ``nslots`` device slots (default 3), each with its own captured step
    graph (the stage buffers are shared: the steps themselves run one after
    another on the compute stream), and three streams (copy in, compute, copy
    out) ordered by events. A slot is refilled only after its previous result
    is out, so with two slots a step waits for the copy out and the copy in
    of its slot back to back; a third slot hides both behind the compute of
    the steps between. For pinned host tensors the throughput approaches the
    device step rate once each copy of a state takes less time than a step.
    Every item is advanced from the same start time ``t``.
    """

    def __init__(self, evo: BSSNEvolution, shape, dt: float, t: float = 0.0, device="cuda", nslots: int = 3):
        self.evo = evo
        self.device = torch.device(device)
        S = evo._S(t, dt, self.device)
        self.nslots = int(nslots)
        if self.nslots < 1:
            raise ValueError("nslots must be >= 1")
        self.slots = []
        for _ in range(self.nslots):
            U = torch.empty(tuple(shape), dtype=torch.float64, device=self.device)
            U.zero_()
            U[0].fill_(1.0)     # a harmless state for the capture's warm-up step
            U[1].fill_(1.0)
            for p in (3, 6, 8):
                U[p].fill_(1.0)
            self.slots.append(self._capture(U, S.clone()))
        self.s_in = torch.cuda.Stream(self.device)
        self.s_comp = torch.cuda.Stream(self.device)
        self.s_out = torch.cuda.Stream(self.device)
        self.ev_in = [torch.cuda.Event() for _ in range(self.nslots)]
        self.ev_comp = [torch.cuda.Event() for _ in range(self.nslots)]
        self.ev_out = [torch.cuda.Event() for _ in range(self.nslots)]

    def _capture(self, U, S):
        evo = self.evo
        evo._buffers(U)
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            probe = U.clone()
            evo._step_inplace(probe, S.clone())
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        del probe
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            evo._step_inplace(U, S)
        g.static_tensors = (U, S, evo._buffers(U))
        return g, U

    def run(self, host_in, host_out) -> None:
        """Advance host_in[i] by one step into host_out[i] for every i (pinned
        float64 host tensors of the pipeline's shape). Enqueues everything;
        the caller's current stream waits for the last copy out."""
        cur = torch.cuda.current_stream(self.device)
        for st in (self.s_in, self.s_comp, self.s_out):
            st.wait_stream(cur)
        for i, (hin, hout) in enumerate(zip(host_in, host_out)):
            k = i % self.nslots
            g, U = self.slots[k]
            if i >= self.nslots:
                self.s_in.wait_event(self.ev_out[k])      # slot k's previous result is out
            with torch.cuda.stream(self.s_in):
                U.copy_(hin, non_blocking=True)
                self.ev_in[k].record(self.s_in)
            self.s_comp.wait_event(self.ev_in[k])
            with torch.cuda.stream(self.s_comp):
                g.replay()
                self.ev_comp[k].record(self.s_comp)
            self.s_out.wait_event(self.ev_comp[k])
            with torch.cuda.stream(self.s_out):
                hout.copy_(U, non_blocking=True)
                self.ev_out[k].record(self.s_out)
        cur.wait_stream(self.s_out)
