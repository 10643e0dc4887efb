"""B200-native PPPM vortex-particle velocity evaluation (host-side mirror).

The compute path is libpppm_b200.so (hand-written sm_100a CUDA behind the C
ABI of include/pppm.h).  This module binds it with ctypes and mirrors the
reference's C++ interface for the path, using torch CUDA tensors only as
device buffers:

* ``BiotSavartSolver`` — hybridFastSummation/BiotSavartSolver.h:16-38
  (initializeSolver, setVortParameter, setEvalParameter, computeFarFieldBuffer,
  evaluateVelocity, getU, getVort, getSortVort, getSortPos, getVortStartTable,
  getVortEndTable, sortVort, getCellh, getOrigin, shutdown);
* ``ParticleManager`` — particle_hash/SpaceHashClass.h:10-84;
* ``MultiGridSolver3DPeriod_double`` — multigrid/MultiGrid.h:188-209;
* ``Scene`` — a direct wrapper of one pppm_scene.

There is no CPU fallback: without the library or a CUDA device every call
raises.
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import (DOMAIN_BBOX3X, DOMAIN_FIXED, GRID_FAR, GRID_PSI, GRID_VORT, MG_CONVERGED,
                   MG_REFERENCE, PppmBatchItem, PppmError, PppmParams, check, default_params, load)

__all__ = [
    "Scene", "BiotSavartSolver", "ParticleManager", "MultiGridSolver3DPeriod_double", "PppmError",
    "PppmParams", "default_params", "load", "direct_sum_fp64", "MG_REFERENCE", "MG_CONVERGED",
    "DOMAIN_BBOX3X", "DOMAIN_FIXED", "batch_run",
]


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("pppm_b200 needs a CUDA device (B200, sm_100a); no CPU path exists")


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream_handle(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _pos4(t: torch.Tensor) -> torch.Tensor:
    if t.dtype != torch.float32 or t.dim() != 2 or t.shape[1] != 4 or not t.is_cuda:
        raise ValueError("positions must be a CUDA float32 tensor of shape (N, 4)")
    return t.contiguous()


def _alpha3(t: torch.Tensor, N: int):
    """Accepts (N, 3) or (3, N) float64; returns three contiguous (N,) tensors."""
    if t.dtype != torch.float64 or not t.is_cuda:
        raise ValueError("strengths must be a CUDA float64 tensor")
    if t.shape == (N, 3):
        t = t.t()
    if t.shape != (3, N):
        raise ValueError(f"strengths must have shape (N, 3) or (3, N) with N={N}")
    return [t[c].contiguous() for c in range(3)]


def tuning_report() -> str:
    """The multigrid smoother autotuner's measurements (pppm_tuning_report)."""
    buf = C.create_string_buffer(8192)
    n = C.c_size_t()
    check(load().pppm_tuning_report(buf, 8192, C.byref(n)), "pppm_tuning_report")
    return buf.value.decode()


class Scene:
    """One resident PPPM scene (pppm_scene)."""

    def __init__(self, n: int, K: int = 1, a: float = 0.08, domain: str = "bbox3x",
                 fixed_origin=(0.0, 0.0, 0.0), fixed_length: float = 1.0, mg: str = "reference",
                 mg_tol: float = 1e-10, mg_max_cycles: int = 50, cap_vort: int = 1, cap_eval: int = 1,
                 stream: torch.cuda.Stream | None = None, a_cells: float = 0.0):
        """a_cells > 0 ties the smoothing radius to the cell size of each build
        (a = a_cells * h), overriding the absolute a."""
        _require_cuda()
        self._lib = load()
        self.params = default_params(
            n, K=K, a=a, domain_mode=DOMAIN_FIXED if domain == "fixed" else DOMAIN_BBOX3X,
            fixed_origin=fixed_origin, fixed_length=fixed_length,
            mg_mode=MG_CONVERGED if mg == "converged" else MG_REFERENCE, mg_tol=mg_tol,
            mg_max_cycles=mg_max_cycles, a_cells=a_cells)
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        h = C.c_void_p()
        check(self._lib.pppm_scene_create(C.byref(self.params), cap_vort, cap_eval,
                                          _stream_handle(self.stream), C.byref(h)), "pppm_scene_create")
        self._h = h
        self._keep = []
        self.N = 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pppm_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_vortices(self, pos4: torch.Tensor, alpha: torch.Tensor):
        pos4 = _pos4(pos4)
        N = pos4.shape[0]
        ax, ay, az = _alpha3(alpha, N)
        check(self._lib.pppm_set_vortices(self._h, N, _ptr(pos4), _ptr(ax), _ptr(ay), _ptr(az)),
              "pppm_set_vortices")
        self._keep = [pos4, ax, ay, az]  # copies are enqueued; keep sources alive until they land
        self.N = N

    def build_far_field(self):
        check(self._lib.pppm_build_far_field(self._h), "pppm_build_far_field")

    def eval(self, eval_a: torch.Tensor, eval_b: torch.Tensor | None = None, is_segment: int = 0,
             out: torch.Tensor | None = None) -> torch.Tensor:
        """Velocities (M, 3) float64... returned as a (3, M) tensor view transposed to (M, 3)."""
        ea = _pos4(eval_a)
        M = ea.shape[0]
        eb = _pos4(eval_b) if eval_b is not None else None
        if is_segment == 1 and eb is None:
            raise ValueError("is_segment=1 needs eval_b")
        if out is None:
            out = torch.empty((3, M), dtype=torch.float64, device=ea.device)
        check(self._lib.pppm_eval(self._h, M, _ptr(ea), _ptr(eb), int(is_segment), _ptr(out[0]),
                                  _ptr(out[1]), _ptr(out[2])), "pppm_eval")
        return out.t()

    def eval_f32(self, eval_a, eval_b=None, is_segment=0, out=None) -> torch.Tensor:
        ea = _pos4(eval_a)
        M = ea.shape[0]
        eb = _pos4(eval_b) if eval_b is not None else None
        if out is None:
            out = torch.empty((M, 3), dtype=torch.float32, device=ea.device)
        check(self._lib.pppm_eval_f32(self._h, M, _ptr(ea), _ptr(eb), int(is_segment), _ptr(out)),
              "pppm_eval_f32")
        return out

    def solve_host(self, pos4_host, alpha_host, eval_a_host=None, eval_b_host=None, is_segment=0,
                   out_host=None):
        """End to end on (pinned) host tensors; returns (3, M) float64 host tensor."""
        N = pos4_host.shape[0]
        ax, ay, az = [alpha_host[c] for c in range(3)] if alpha_host.shape[0] == 3 else \
            [alpha_host[:, c].contiguous() for c in range(3)]
        M = N if eval_a_host is None else eval_a_host.shape[0]
        if out_host is None:
            out_host = torch.empty((3, M), dtype=torch.float64, pin_memory=True)
        check(self._lib.pppm_solve_host(self._h, N, _ptr(pos4_host), _ptr(ax), _ptr(ay), _ptr(az), M,
                                        _ptr(eval_a_host), _ptr(eval_b_host), int(is_segment),
                                        _ptr(out_host[0]), _ptr(out_host[1]), _ptr(out_host[2])),
              "pppm_solve_host")
        return out_host

    def domain(self):
        o = (C.c_double * 3)()
        L = C.c_double()
        h = C.c_double()
        check(self._lib.pppm_get_domain(self._h, o, C.byref(L), C.byref(h)), "pppm_get_domain")
        return (o[0], o[1], o[2]), L.value, h.value

    def smoothing(self) -> float:
        """Smoothing radius a of the last far field (absolute, or a_cells x h)."""
        a = C.c_double()
        check(self._lib.pppm_get_smoothing(self._h, C.byref(a)), "pppm_get_smoothing")
        return a.value

    def cell_tables(self):
        """(start, end) as int64 CPU tensors of the uint32 tables (n^3 each)."""
        s = C.c_void_p()
        e = C.c_void_p()
        check(self._lib.pppm_get_cell_tables(self._h, C.byref(s), C.byref(e)), "pppm_get_cell_tables")
        return _copy_u32(s.value, self.params.n ** 3, self.stream), _copy_u32(e.value, self.params.n ** 3, self.stream)

    def sorted_index(self):
        k = C.c_void_p()
        i = C.c_void_p()
        check(self._lib.pppm_get_sorted_index(self._h, C.byref(k), C.byref(i)), "pppm_get_sorted_index")
        return _copy_u32(k.value, self.N, self.stream), _copy_u32(i.value, self.N, self.stream)

    def sorted_vortices(self):
        pos = torch.empty((self.N, 4), dtype=torch.float32, device="cuda")
        al = torch.empty((3, self.N), dtype=torch.float64, device="cuda")
        check(self._lib.pppm_get_sorted_vortices(self._h, _ptr(pos), _ptr(al[0]), _ptr(al[1]), _ptr(al[2])),
              "pppm_get_sorted_vortices")
        return pos, al

    def grid(self, which: int) -> torch.Tensor:
        p = C.c_void_p()
        check(self._lib.pppm_get_grid(self._h, which, C.byref(p)), "pppm_get_grid")
        n3 = self.params.n ** 3
        dt = torch.float64 if which == GRID_PSI else torch.float32
        return _copy_dev(p.value, 3 * n3, dt, self.stream).reshape(3, n3)

    def stats(self):
        pairs = C.c_uint64()
        cyc = C.c_int32()
        rr = C.c_double()
        check(self._lib.pppm_get_stats(self._h, C.byref(pairs), C.byref(cyc), C.byref(rr)), "pppm_get_stats")
        return {"mg_cycles": cyc.value, "mg_relres": rr.value}

    def advect(self, pos4: torch.Tensor, alpha: torch.Tensor, dt: float, method: str = "rk2"):
        """Moves pos4 (CUDA float32 (N, 4), in place) by one Euler or RK2 step."""
        if pos4.dtype != torch.float32 or not pos4.is_cuda or not pos4.is_contiguous() or pos4.shape[1] != 4:
            raise ValueError("pos4 must be a contiguous CUDA float32 (N, 4) tensor (updated in place)")
        N = pos4.shape[0]
        ax, ay, az = _alpha3(alpha, N)
        fn = self._lib.pppm_advect_rk2 if method == "rk2" else self._lib.pppm_advect_euler
        check(fn(self._h, N, _ptr(pos4), _ptr(ax), _ptr(ay), _ptr(az), float(dt)), f"pppm_advect_{method}")
        self._keep = [ax, ay, az]
        self.N = N
        return pos4

    def vortex_step(self, pos4: torch.Tensor, alpha: torch.Tensor, dt: float, h_seg: float = 0.1,
                    nu: float = 0.1, return_ends: bool = False, passive: torch.Tensor | None = None):
        """One vortex-segment time step of the reference's solveTimeStep (pppm_vortex_step).

        pos4 (CUDA float32 (N, 4)) and alpha (CUDA float64 (N, 3) or (3, N)) are
        updated in place.  passive (CUDA float32 (P, 4), tracers or heat
        particles) is moved in place with the velocity of the same far field.
        Returns (pos4, alpha), then (enda, endb) with return_ends, then the
        passive velocity (P, 3) float64 when passive points are given.
        """
        if pos4.dtype != torch.float32 or not pos4.is_cuda or not pos4.is_contiguous() or pos4.shape[1] != 4:
            raise ValueError("pos4 must be a contiguous CUDA float32 (N, 4) tensor (updated in place)")
        N = pos4.shape[0]
        P = 0 if passive is None else passive.shape[0]
        if P and (passive.dtype != torch.float32 or not passive.is_cuda or not passive.is_contiguous()
                  or passive.shape[1] != 4):
            raise ValueError("passive must be a contiguous CUDA float32 (P, 4) tensor (updated in place)")
        with torch.cuda.stream(self.stream):
            ax, ay, az = _alpha3(alpha, N)
            ea = eb = None
            if return_ends:
                ea = torch.empty((N, 4), dtype=torch.float32, device=pos4.device)
                eb = torch.empty((N, 4), dtype=torch.float32, device=pos4.device)
            pvel = torch.empty((3, max(P, 1)), dtype=torch.float64, device=pos4.device)
            check(self._lib.pppm_vortex_step(self._h, N, _ptr(pos4), _ptr(ax), _ptr(ay), _ptr(az), float(dt),
                                             float(h_seg), float(nu), _ptr(ea), _ptr(eb), P,
                                             _ptr(passive) if P else None, _ptr(pvel[0]) if P else None,
                                             _ptr(pvel[1]) if P else None, _ptr(pvel[2]) if P else None),
                  "pppm_vortex_step")
            if alpha.shape == (N, 3):
                alpha.copy_(torch.stack([ax, ay, az], dim=1))
            else:
                alpha.copy_(torch.stack([ax, ay, az], dim=0))
        self.N = N
        out = (pos4, alpha)
        if return_ends:
            out = out + (ea, eb)
        if P:
            out = out + (pvel.t()[:P].contiguous(),)
        return out

    def baroclinic(self, heat4: torch.Tensor, heat: torch.Tensor, pos4: torch.Tensor, alpha: torch.Tensor,
                   dt: float):
        """Buoyancy source (pppm_baroclinic): adds the baroclinic vorticity of the
        heat particles (heat4 (H, 4) float32, heat (H,) float32) to alpha (in place)."""
        N = pos4.shape[0]
        H = heat4.shape[0]
        for t, nm in ((heat4, "heat4"), (pos4, "pos4")):
            if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous() or t.shape[1] != 4:
                raise ValueError(f"{nm} must be a contiguous CUDA float32 (n, 4) tensor")
        if heat.dtype != torch.float32 or not heat.is_cuda or heat.shape != (H,):
            raise ValueError("heat must be a CUDA float32 (H,) tensor")
        hc = heat.contiguous()
        with torch.cuda.stream(self.stream):
            ax, ay, az = _alpha3(alpha, N)
            check(self._lib.pppm_baroclinic(self._h, H, _ptr(heat4), _ptr(hc), N, _ptr(pos4),
                                            _ptr(ax), _ptr(ay), _ptr(az), float(dt)), "pppm_baroclinic")
            if alpha.shape == (N, 3):
                alpha.copy_(torch.stack([ax, ay, az], dim=1))
            else:
                alpha.copy_(torch.stack([ax, ay, az], dim=0))
        return alpha

    def solve_time_step(self, pos4: torch.Tensor, alpha: torch.Tensor, dt: float, heat: torch.Tensor,
                        heat4: torch.Tensor | None = None, h_seg: float = 0.1, nu: float = 0.1):
        """One buoyant time step of VortexSimulationSystem::solveTimeStep without
        emitters or boundary (HFS/VortexSimulationSystemImp.cpp:90-125):
        addBaroclinicForce (:369-465), then the vortex-segment step
        (convertVortToSeg, computeURotation, applyFlow, convertSegToVort,
        computeStretching).

        heat (H,) float32 is the temperature of the heat particles heat4 (H, 4),
        which move with the flow in place; with heat4 None the vortex particles
        themselves carry it (H = N) and move as vortices.  pos4 and alpha are
        updated in place.  Returns (pos4, alpha)."""
        carried = heat4 is None
        self.baroclinic(pos4 if carried else heat4, heat, pos4, alpha, dt)
        self.vortex_step(pos4, alpha, dt, h_seg=h_seg, nu=nu, passive=None if carried else heat4)
        return pos4, alpha

    def density(self):
        """(dim, origin, h, rho (dim^3,) float32, grad (3, dim^3) float32) of the last pppm_baroclinic."""
        dim = C.c_uint32()
        org = (C.c_double * 3)()
        h = C.c_double()
        r = C.c_void_p()
        g = C.c_void_p()
        check(self._lib.pppm_get_density(self._h, C.byref(dim), org, C.byref(h), C.byref(r), C.byref(g)),
              "pppm_get_density")
        c = dim.value ** 3
        rho = _copy_dev(r.value, c, torch.float32, self.stream)
        grad = _copy_dev(g.value, 3 * c, torch.float32, self.stream).reshape(3, c)
        return dim.value, tuple(org), h.value, rho, grad

    def set_profiling(self, on: bool = True):
        check(self._lib.pppm_scene_set_profiling(self._h, int(on)), "pppm_scene_set_profiling")

    def stage_times(self) -> dict:
        """Last recorded duration (ms) of each stage; -1 for stages not run."""
        from ._lib import STAGES
        ms = (C.c_double * 16)()
        cnt = C.c_int()
        check(self._lib.pppm_get_stage_times(self._h, ms, 16, C.byref(cnt)), "pppm_get_stage_times")
        return {STAGES[i]: ms[i] for i in range(cnt.value)}

    def count_pairs(self, eval_a: torch.Tensor) -> int:
        ea = _pos4(eval_a)
        pairs = C.c_uint64()
        check(self._lib.pppm_count_pairs(self._h, ea.shape[0], _ptr(ea), C.byref(pairs)), "pppm_count_pairs")
        return int(pairs.value)


class _DevView:
    """Zero-copy view of device memory owned by the library."""

    def __init__(self, ptr: int, count: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False),
                                         "version": 2, "strides": None}


def _copy_dev(ptr: int, count: int, dtype, stream) -> torch.Tensor:
    """Copy `count` elements at a device address into a new CPU tensor."""
    typestr = {torch.float32: "<f4", torch.float64: "<f8", torch.int32: "<i4"}[dtype]
    torch.cuda.synchronize()
    view = torch.as_tensor(_DevView(ptr, count, typestr), device="cuda")
    return view.cpu()


def _copy_u32(ptr: int, count: int, stream) -> torch.Tensor:
    t = _copy_dev(ptr, count, torch.int32, stream)
    return t.to(torch.int64) & 0xFFFFFFFF


def direct_sum_fp64(vort_pos4, alpha, eval_a, a: float, eval_b=None, is_segment: int = 0, stream=None):
    """FP64 O(N*M) smoothed Biot-Savart sum on the GPU; returns (M, 3) float64."""
    _require_cuda()
    L = load()
    vp = _pos4(vort_pos4)
    N = vp.shape[0]
    ax, ay, az = _alpha3(alpha, N)
    ea = _pos4(eval_a)
    eb = _pos4(eval_b) if eval_b is not None else None
    M = ea.shape[0]
    out = torch.empty((3, M), dtype=torch.float64, device=ea.device)
    check(L.pppm_direct_sum_fp64(N, _ptr(vp), _ptr(ax), _ptr(ay), _ptr(az), M, _ptr(ea), _ptr(eb),
                                 int(is_segment), float(a), _ptr(out[0]), _ptr(out[1]), _ptr(out[2]),
                                 _stream_handle(stream)), "pppm_direct_sum_fp64")
    return out.t()


def batch_run(jobs, stream=None):
    """Runs several independent scenes at once (pppm_batch_run).

    jobs: list of (scene, pos4, alpha, eval_a or None, eval_b or None,
    is_segment).  eval_a None evaluates at the vortices against themselves.
    Returns a list of (M, 3) float64 velocity tensors, one per job."""
    _require_cuda()
    L = load()
    items = (PppmBatchItem * len(jobs))()
    keep, outs = [], []
    for q, (scene, pos4, alpha, ea, eb, seg) in enumerate(jobs):
        pos4 = _pos4(pos4)
        N = pos4.shape[0]
        ax, ay, az = _alpha3(alpha, N)
        if ea is None:
            ea, eb, seg = pos4, pos4, 1
        ea = _pos4(ea)
        eb = _pos4(eb) if eb is not None else None
        M = ea.shape[0]
        out = torch.empty((3, M), dtype=torch.float64, device=pos4.device)
        it = items[q]
        it.scene = scene.handle.value
        it.N, it.pos4_dev = N, pos4.data_ptr()
        it.ax_dev, it.ay_dev, it.az_dev = ax.data_ptr(), ay.data_ptr(), az.data_ptr()
        it.M, it.eval_a4_dev = M, ea.data_ptr()
        it.eval_b4_dev = eb.data_ptr() if eb is not None else None
        it.is_segment = int(seg)
        it.u_dev, it.v_dev, it.w_dev = out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr()
        keep += [pos4, ax, ay, az, ea, eb]
        outs.append(out)
        scene.N = N
    check(L.pppm_batch_run(items, len(jobs), _stream_handle(stream)), "pppm_batch_run")
    torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
    del keep
    return [o.t() for o in outs]


class BiotSavartSolver:
    """Mirror of hybridFastSummation/BiotSavartSolver.h:16-38 over one Scene.

    Inputs are torch CUDA tensors standing in for the reference's GpuArrayf4
    (float4 positions) and GpuArrayd (double per-component arrays).
    """

    def __init__(self):
        self._scene = None
        self._dims = None
        self._K = 1
        self._M = 0
        self._N = 0
        self._eval_pos = None
        self._U = None
        self._vort = None
        self._sorted = None

    def initializeSolver(self, gdx, gdy, gdz, isVIC, K, M, N, a=0.08, mg="reference"):
        """HFS/BiotSavartSolverImp.cpp:44-229.  Cubic grids only; isVIC=True
        (mesh-only velocities) is not part of the path and is rejected."""
        if not (gdx == gdy == gdz):
            raise ValueError("the hash and multigrid are cubic: gdx == gdy == gdz required")
        if isVIC:
            raise ValueError("isVIC is not supported (the reference ships with it off)")
        if self._scene is None or self._dims != (gdx, K):
            if self._scene is not None:
                self._scene.close()
            self._scene = Scene(gdx, K=K, a=a, mg=mg, cap_vort=max(N, 1), cap_eval=max(M, 1))
            self._dims = (gdx, K)
        self._K, self._M, self._N = K, M, N
        return True

    def setVortParameter(self, n, pos, omega):
        """HFS/BiotSavartSolverImp.cpp:318-360: omega is a list of 3 double arrays."""
        self._N = n
        self._vort = [o[:n] for o in omega]
        self._scene.set_vortices(pos[:n], torch.stack(self._vort))
        self._sorted = None
        return True

    def setEvalParameter(self, m, pos):
        """HFS/BiotSavartSolverImp.cpp:266-316."""
        self._M = m
        self._eval_pos = pos[:m]
        return True

    def computeFarFieldBuffer(self):
        """HFS/BiotSavartSolverImp.cpp:756-816."""
        self._scene.build_far_field()

    def evaluateVelocity(self, another_end, is_segment):
        """HFS/BiotSavartSolverImp.cpp:410-516."""
        eb = another_end[:self._M] if (is_segment == 1 and another_end is not None) else None
        self._U = self._scene.eval(self._eval_pos, eb, int(is_segment)).t()
        return True

    def getU(self, i):
        return self._U[i]

    def getVort(self, i):
        return self._vort[i]

    def sortVort(self):
        """HFS/BiotSavartSolverImp.cpp:733-753 (bounding box + hash + reorder);
        the far-field build performs the same steps, so this only refreshes the
        sorted copies."""
        self._scene.build_far_field()
        self._sorted = self._scene.sorted_vortices()

    def _sorted_copy(self):
        if self._sorted is None:
            self._sorted = self._scene.sorted_vortices()
        return self._sorted

    def getSortPos(self):
        return self._sorted_copy()[0]

    def getSortVort(self, i):
        return self._sorted_copy()[1][i]

    def getVortStartTable(self):
        return self._scene.cell_tables()[0]

    def getVortEndTable(self):
        return self._scene.cell_tables()[1]

    def getCellh(self):
        return self._scene.domain()[2]

    def getOrigin(self):
        o, _, _ = self._scene.domain()
        return (o[0], o[1], o[2], 0.0)

    def shutdown(self):
        if self._scene is not None:
            self._scene.close()
            self._scene = None
        return True


class ParticleManager:
    """Mirror of particle_hash/SpaceHashClass.h:10-84 (pppm_hasher)."""

    def __init__(self):
        self._h = None
        self._n = 0
        self._N = 0
        self._h_cell = 0.0
        self._origin = (0.0, 0.0, 0.0)

    def initSpatialHash(self, numParticles, dimx, dimy, dimz):
        _require_cuda()
        if not (dimx == dimy == dimz):
            raise ValueError("cubic hash grids only")
        self.endSpatialHash()
        L = load()
        h = C.c_void_p()
        check(L.pppm_hasher_create(numParticles, dimx, _stream_handle(None), C.byref(h)), "pppm_hasher_create")
        self._h = h
        self._n = dimx
        self._N = numParticles
        self._h_cell = 1.0 / dimx

    def endSpatialHash(self):
        if self._h is not None:
            load().pppm_hasher_destroy(self._h)
            self._h = None

    def setSpatialHashGrid(self, size0, h, bbmin, numParticles):
        self._h_cell = float(torch.tensor(h, dtype=torch.float32))
        self._origin = tuple(float(torch.tensor(v, dtype=torch.float32)) for v in bbmin)
        self._N = numParticles

    def setHashParam(self):
        pass  # parameters travel with each call; no global constant memory

    def doSpatialHash(self, pos, numParticles):
        pos = _pos4(pos)
        o = (C.c_float * 3)(*self._origin)
        check(load().pppm_hasher_run(self._h, numParticles, _ptr(pos), C.c_float(self._h_cell), o),
              "pppm_hasher_run")

    def _tables(self):
        k, i, s, e = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(load().pppm_hasher_tables(self._h, C.byref(k), C.byref(i), C.byref(s), C.byref(e)),
              "pppm_hasher_tables")
        return k.value, i.value, s.value, e.value

    def getHashTable(self):
        return _copy_u32(self._tables()[0], self._N, None)

    def getIndexTable(self):
        return _copy_u32(self._tables()[1], self._N, None)

    def getStartTable(self):
        return _copy_u32(self._tables()[2], self._n ** 3, None)

    def getEndTable(self):
        return _copy_u32(self._tables()[3], self._n ** 3, None)

    def reorderData(self, numParticles, data, dataReorder, stride, precision):
        check(load().pppm_hasher_reorder(self._h, numParticles, _ptr(data), _ptr(dataReorder), stride, precision),
              "pppm_hasher_reorder")

    def deorderData(self, numParticles, data, dataReorder, stride, precision):
        check(load().pppm_hasher_deorder(self._h, numParticles, _ptr(data), _ptr(dataReorder), stride, precision),
              "pppm_hasher_deorder")


class MultiGridSolver3DPeriod_double:
    """Mirror of multigrid/MultiGrid.h:188-209 (pppm_mg)."""

    def __init__(self):
        self._h = None
        self.n = 0

    def m_InitialSystem(self, gridx, gridy, gridz):
        _require_cuda()
        if not (gridx == gridy == gridz):
            raise ValueError("cubic grids only")
        self.m_FinalMemoryEachLevel()
        h = C.c_void_p()
        check(load().pppm_mg_create(gridx, _stream_handle(None), C.byref(h)), "pppm_mg_create")
        self._h = h
        self.n = gridx

    def m_FinalMemoryEachLevel(self):
        if self._h is not None:
            load().pppm_mg_destroy(self._h)
            self._h = None

    def m_FullMultiGrid(self, x: torch.Tensor, b: torch.Tensor, tol: float = 1e-10,
                        mode: int = MG_REFERENCE, max_cycles: int = 50) -> float:
        """Solves sum_nbr(x) - 6x = b (zero ghosts) into x, starting from the x
        given (x <- x + FMG(0, b - A x), as the reference's first residual is
        b - A x); returns the relative residual (-1 in reference mode, which
        does not measure it)."""
        if x.dtype != torch.float64 or b.dtype != torch.float64 or not x.is_cuda:
            raise ValueError("x and b must be CUDA float64 tensors")
        rr = C.c_double()
        check(load().pppm_mg_full_multigrid(self._h, _ptr(x), _ptr(b.contiguous()), mode, tol, max_cycles,
                                            C.byref(rr)), "pppm_mg_full_multigrid")
        return rr.value

    def m_Vcycle(self, x: torch.Tensor, b: torch.Tensor, tol: float = 1e-10, residual=None, level: int = 0):
        """One V(4,4) cycle from `level` down (multigrid/MultiGrid.cpp:128-201)
        on that level's float64 arrays (edge n >> level); tol and residual are
        unused, as in the reference."""
        if x.dtype != torch.float64 or b.dtype != torch.float64 or not x.is_cuda:
            raise ValueError("x and b must be CUDA float64 tensors")
        check(load().pppm_mg_vcycle(self._h, _ptr(x), _ptr(b.contiguous()), int(level)), "pppm_mg_vcycle")

    def levels(self):
        """Edges of the levels of the hierarchy, finest first."""
        cnt = C.c_int()
        edges = (C.c_uint32 * 16)()
        check(load().pppm_mg_levels(self._h, C.byref(cnt), edges, 16), "pppm_mg_levels")
        return [int(edges[i]) for i in range(cnt.value)]
