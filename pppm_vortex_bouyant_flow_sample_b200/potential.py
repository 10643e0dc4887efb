"""Scalar PPPM (pppm_potential_* in include/pppm.h): mirror of the reference's
PotentialFieldSolver (hybridFastSummation/PotentialFieldSolver.h:10-91) with
its method names.  Device tensors in, device tensors out; no CPU path.
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import check, load


def _f32x4(t: torch.Tensor, name: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32 or t.dim() != 2 \
            or t.shape[1] != 4:
        raise ValueError(f"{name} must be a CUDA float32 (n, 4) tensor")
    return t.contiguous()


def _f64(t: torch.Tensor, n: int, name: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float64 or t.numel() != n:
        raise ValueError(f"{name} must be a CUDA float64 tensor of {n} values")
    return t.contiguous().reshape(n)


class PotentialFieldSolver:
    """initializeSolver / setMassParameter / setEvalParameter /
    computeFarFieldBuffer + evaluateGradient / computeFarFieldPotentialBuffer +
    evaluateScalarPotential / computeDphiDn, as the reference names them."""

    def __init__(self, stream: torch.cuda.Stream | None = None):
        self._h = None
        self._lib = None
        self.stream = stream
        self._eval = None
        self._normals = None
        self._areas = None
        self._mass = None
        self.grad_phi = None
        self.scalar_phi = None
        self.dphidn = None

    def initializeSolver(self, gdx: int, gdy: int, gdz: int, K: int, M: int, N: int) -> bool:
        if not (gdx == gdy == gdz):
            raise ValueError("cubic grids only")
        if not torch.cuda.is_available():
            raise RuntimeError("the scalar PPPM needs a CUDA device (sm_100a); there is no CPU path")
        self.shutdown()
        self._lib = load()
        st = self.stream if self.stream is not None else torch.cuda.current_stream()
        self.stream = st
        h = C.c_void_p()
        check(self._lib.pppm_potential_create(gdx, K, max(N, 1), max(M, 1), C.c_void_p(st.cuda_stream),
                                              C.byref(h)), "pppm_potential_create")
        self._h = h
        self.n = gdx
        return True

    def shutdown(self) -> bool:
        if self._h is not None:
            self._lib.pppm_potential_destroy(self._h)
            self._h = None
        return True

    def __del__(self):
        try:
            self.shutdown()
        except Exception:
            pass

    def setMassParameter(self, n: int, pos: torch.Tensor, mass: torch.Tensor) -> bool:
        pos = _f32x4(pos, "pos")[:n]
        self._mass = _f64(mass[:n], n, "mass")
        self._pos = pos
        check(self._lib.pppm_potential_set_masses(self._h, n, C.c_void_p(pos.data_ptr()),
                                                  C.c_void_p(self._mass.data_ptr())), "pppm_potential_set_masses")
        return True

    def setEvalParameter(self, m: int, pos: torch.Tensor) -> bool:
        self._eval = _f32x4(pos, "pos")[:m]
        return True

    def setEvalNormals(self, m: int, normals: torch.Tensor) -> bool:
        self._normals = normals[:m].to(torch.float64).contiguous()
        return True

    def setEvalAreas(self, m: int, areas: torch.Tensor) -> bool:
        self._areas = _f64(areas[:m], m, "areas")
        return True

    def computeFarFieldBuffer(self) -> None:
        with torch.cuda.stream(self.stream):
            check(self._lib.pppm_potential_build(self._h, 0), "pppm_potential_build")

    def computeFarFieldPotentialBuffer(self) -> None:
        with torch.cuda.stream(self.stream):
            check(self._lib.pppm_potential_build(self._h, 1), "pppm_potential_build")

    def evaluateGradient(self, large_eval: bool = True) -> bool:
        m = self._eval.shape[0]
        g = torch.empty((3, max(m, 1)), dtype=torch.float64, device=self._eval.device)
        with torch.cuda.stream(self.stream):
            check(self._lib.pppm_potential_eval_gradient(self._h, m, C.c_void_p(self._eval.data_ptr()),
                                                         C.c_void_p(g[0].data_ptr()), C.c_void_p(g[1].data_ptr()),
                                                         C.c_void_p(g[2].data_ptr())),
                  "pppm_potential_eval_gradient")
        self.grad_phi = g[:, :m].t()
        return True

    def evaluateScalarPotential(self) -> None:
        m = self._eval.shape[0]
        out = torch.empty(max(m, 1), dtype=torch.float64, device=self._eval.device)
        with torch.cuda.stream(self.stream):
            check(self._lib.pppm_potential_eval_scalar(self._h, m, C.c_void_p(self._eval.data_ptr()),
                                                       C.c_void_p(out.data_ptr())), "pppm_potential_eval_scalar")
        self.scalar_phi = out[:m]

    def computeDphiDn(self) -> bool:
        m = self._eval.shape[0]
        g = self.grad_phi.t().contiguous()
        n = self._normals.t().contiguous()
        out = torch.empty(max(m, 1), dtype=torch.float64, device=g.device)
        with torch.cuda.stream(self.stream):
            ptr = lambda t: C.c_void_p(t.data_ptr())
            check(self._lib.pppm_potential_dphidn(self._h, m, ptr(n[0]), ptr(n[1]), ptr(n[2]), ptr(g[0]),
                                                  ptr(g[1]), ptr(g[2]), ptr(self._mass), ptr(self._areas),
                                                  ptr(out)), "pppm_potential_dphidn")
        self.dphidn = out[:m]
        return True

    def getGradPhi(self) -> torch.Tensor:
        return self.grad_phi

    def getScalarPhi(self) -> torch.Tensor:
        return self.scalar_phi

    def getDpDn(self) -> torch.Tensor:
        return self.dphidn

    def grids(self) -> dict:
        """Origin, L, monopole (centre, total mass) and host copies of the
        density, right-hand side, potential and far-field grids of the last build."""
        ol = (C.c_double * 4)()
        mono = (C.c_double * 4)()
        ptrs = [C.c_void_p() for _ in range(4)]
        check(self._lib.pppm_potential_grids(self._h, ol, *(C.byref(p) for p in ptrs), mono), "pppm_potential_grids")
        c3 = self.n ** 3
        torch.cuda.synchronize()
        def host(ptr, count):
            view = _Dev(ptr, count)
            return torch.as_tensor(view, device="cuda").cpu()
        return {"origin": tuple(ol[:3]), "length": ol[3], "monopole": tuple(mono),
                "density": host(ptrs[0].value, c3), "rhs": host(ptrs[1].value, c3), "phi": host(ptrs[2].value, c3),
                "far": host(ptrs[3].value, 3 * c3)}

    def getCellh(self) -> float:
        """The hash cell size as the solver stores it (float L / n)."""
        import numpy as np
        return float(np.float32(self.grids()["length"] / self.n))

    def getOrigin(self):
        return self.grids()["origin"]


class _Dev:
    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False), "version": 3}
