"""Host-side mirror of the reference's element assembler, backed by libfne_asm.so.

``CudaElementAssemblerBase`` keeps the public surface of
``ReorderedElementAssemblerBase`` (``src/core/petsc/reordered_element_base.py:642``):
``energy_fn(vec)`` (:1579), ``gradient_fn(vec, g)`` (:1613),
``assemble_hessian(u_owned, variant=2)`` (:1635), ``update_dirichlet(u0)``
(:1560), ``create_vec(full)`` (:1568), ``cleanup()`` (:1777),
``callback_summary()`` / ``setup_summary()`` / ``iter_timings``, and the same
layout (``self.layout``: ``perm, iperm, lo, hi, n_free, total_to_free_reord,
owned_rows, owned_cols``).  Vectors may be CUDA tensors (zero copy), NumPy
arrays, or objects with an ``.array`` attribute (PETSc ``Vec``).  The owned
Hessian values land in ``self.owned_values`` (a CUDA tensor, COO order of
``layout.owned_rows/owned_cols``); when a PETSc matrix is attached as
``self.A`` they are handed to ``A.setValuesCOO`` unchanged, as the reference
does (:1046-1050).

Family subclasses mirror the reference's ``_make_local_element_kernels``
implementations; the kernels themselves are in ``csrc/fne_asm.cu``.  The
layout is built on the device (``fne_layout_build_device``) unless
``layout_on_device=False`` selects the host build; both give the same arrays.
"""

from __future__ import annotations

import time
from types import SimpleNamespace

import numpy as np
import torch

from fenics_nonlinear_energies_b200 import _lib
from fenics_nonlinear_energies_b200._lib import check, lib

_DTYPES = {"fp64": _lib.FNE_FP64, "fp32": _lib.FNE_FP32}


def _comm_rank_size(comm):
    if comm is None:
        return 0, 1
    if hasattr(comm, "Get_rank"):
        return int(comm.Get_rank()), int(comm.Get_size())
    return int(getattr(comm, "rank", 0)), int(getattr(comm, "size", 1))


class CudaElementAssemblerBase:
    """Element energy / gradient / Hessian assembly on one CUDA device."""

    family = 0
    npe = 3
    block_size = 1
    coordinate_key = "nodes"
    dirichlet_key = "u_0"
    local_elem_data_keys: tuple[str, ...] = ()

    def __init__(self, params, comm=None, adjacency=None, *, reorder_mode="block_xyz", perm_override=None,
                 precision="fp64", hess_dtype=None, device=None, kernel_variant="auto", layout_on_device=True,
                 **_ignored_solver_kwargs):
        if not torch.cuda.is_available():
            raise RuntimeError("CudaElementAssemblerBase needs a CUDA device (no CPU fallback)")
        t_setup = time.perf_counter()
        self.params = params
        self.comm = comm
        self.rank, self.size = _comm_rank_size(comm)
        self.precision = str(precision)
        if self.precision not in _DTYPES:
            raise ValueError(f"precision must be 'fp64' or 'fp32', got {precision!r}")
        if hess_dtype is None:
            hess_dtype = torch.float64
        if self.precision == "fp64" and hess_dtype != torch.float64:
            raise ValueError("fp64 mode produces float64 Hessian values")
        self.hess_dtype = hess_dtype
        self.device = torch.device(device if device is not None else f"cuda:{torch.cuda.current_device()}")
        torch.cuda.set_device(self.device)
        self.iter_timings: list[dict] = []
        self._setup_timings: dict[str, float] = {}
        self._callback_stats = {
            "energy": {"calls": 0, "kernel": 0.0, "total": 0.0},
            "gradient": {"calls": 0, "kernel": 0.0, "total": 0.0},
            "hessian": {"calls": 0, "hvp_compute": 0.0, "extraction": 0.0, "coo_assembly": 0.0, "total": 0.0},
        }

        freedofs = np.asarray(params["freedofs"], dtype=np.int64)
        elems = np.asarray(params["elems"], dtype=np.int64)
        n_total = len(np.asarray(params[self.dirichlet_key]))
        t0 = time.perf_counter()
        lay = _lib.build_layout(
            freedofs=freedofs, elems=elems, n_total=n_total, block_size=self.block_size,
            reorder=reorder_mode, coords=np.asarray(params[self.coordinate_key], dtype=np.float64),
            perm_override=perm_override, adjacency=adjacency, rank=self.rank, size=self.size,
            device=bool(layout_on_device),
        )
        self._setup_timings["global_layout"] = time.perf_counter() - t0
        self.layout = SimpleNamespace(**lay)
        self.part = SimpleNamespace(perm=lay["perm"], iperm=lay["iperm"], lo=lay["lo"], hi=lay["hi"],
                                    n_free=lay["n_free"], n_owned=lay["hi"] - lay["lo"])
        self.n_owned = lay["hi"] - lay["lo"]
        self.dirichlet_full = np.asarray(params[self.dirichlet_key], dtype=np.float64).copy()
        weights = (lay["elem_owner"] == self.rank).astype(np.float64)

        t0 = time.perf_counter()
        keep = []
        d = _lib.Desc()
        d.family = self.family
        d.precision = _DTYPES[self.precision]
        d.hess_fp32 = 1 if hess_dtype == torch.float32 else 0
        el, d.elems = _lib.i64(elems)
        t2f, d.total_to_free_reord = _lib.i64(lay["total_to_free_reord"])
        orows, d.owned_rows = _lib.i64(lay["owned_rows"])
        ocols, d.owned_cols = _lib.i64(lay["owned_cols"])
        w, d.energy_weights = _lib.f64(weights)
        dirv, d.dirichlet = _lib.f64(self.dirichlet_full)
        keep += [el, t2f, orows, ocols, w, dirv]
        d.n_elem, d.npe, d.block_size = int(el.shape[0]), self.npe, self.block_size
        d.n_total, d.n_free = int(n_total), int(lay["n_free"])
        d.lo, d.hi, d.nnz = int(lay["lo"]), int(lay["hi"]), int(orows.size)
        rhs = self._build_rhs_owned()
        self._f_owned = rhs
        if rhs is not None:
            r, d.rhs_owned = _lib.f64(rhs)
            keep.append(r)
        for slot, arr in zip(("e0", "e1", "e2", "e3"), self._element_arrays()):
            if arr is None:
                continue
            a, p = _lib.f64(arr)
            keep.append(a)
            setattr(d, slot, p)
        for i, v in enumerate(self._scalars()):
            d.s[i] = float(v)
        d.nq = int(self._nq())
        d.dirichlet_only_energy = 1 if (self._adds_dirichlet_only_energy() and self.rank == 0) else 0
        d.kernel_variant = {"auto": 0, "cluster": 8, "row_gather": 1, "incidence": 2, "element": 2,
                            "cuda_cores": 1, "push": 3, "row_lanes_2": 4, "row_lanes_4": 5,
                            "row_lanes_8": 6, "sweep": 7}[kernel_variant]
        self._handle = _lib.C.c_void_p()
        check(lib.fne_create(_lib.C.byref(d), _lib.C.byref(self._handle)))
        del keep
        self._setup_timings["kernel_build"] = time.perf_counter() - t0
        info = _lib.Info()
        check(lib.fne_info_get(self._handle, _lib.C.byref(info)))
        self.info = {k: getattr(info, k) for k, _ in _lib.Info._fields_}

        dev = self.device
        self._u = torch.zeros(max(1, int(lay["n_free"])), dtype=torch.float64, device=dev)
        self._grad = torch.zeros(max(1, self.n_owned), dtype=torch.float64, device=dev)
        self._energy = torch.zeros(1, dtype=torch.float64, device=dev)
        self.owned_values = torch.zeros(int(orows.size), dtype=hess_dtype, device=dev)
        self.A = None  # optional PETSc Mat (drop-in handoff)
        self._ev0 = torch.cuda.Event(enable_timing=True)
        self._ev1 = torch.cuda.Event(enable_timing=True)
        self._setup_timings["total"] = time.perf_counter() - t_setup

    # ---- family hooks (overridden) -----------------------------------------
    def _element_arrays(self):
        return [np.asarray(self.params[k], dtype=np.float64) for k in self.local_elem_data_keys]

    def _scalars(self):
        return []

    def _nq(self):
        return 0

    def _build_rhs_owned(self):
        return None

    def _adds_dirichlet_only_energy(self):
        return False

    def check_device_status(self):
        """Raise if a bounded device wait of an earlier pass gave up (synchronous)."""
        check(lib.fne_check_device_status(self._handle))

    def _poll_status(self):
        """Raise ``FneError(FNE_ETIMEOUT)`` if the last pass gave up a bounded
        device wait (its values are then not valid).  Reads the pinned copy
        the pass left behind: call after the pass's stream has synchronised."""
        check(lib.fne_poll_device_status(self._handle))

    def launches_per_eval(self, flags):
        """Kernel launches one ``eval(u, flags)`` issues: one fused kernel for the
        triangle families and the tet row-gather kernel; element kernel plus one
        node-block gather for the element-parallel tet pass; for Mohr-Coulomb
        the element kernel, the Hessian gather or shared-block fix-up, and the
        gradient rows."""
        kv = self.info["kernel_variant"]
        if flags == _lib.FNE_ENERGY or kv not in (5, 6, 7, 9, 11):
            return 1
        if kv in (7, 11):
            return 2
        return 1 + bool(flags & _lib.FNE_HESS) + bool(flags & _lib.FNE_GRAD)

    # ---- vector helpers -----------------------------------------------------
    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _as_u(self, vec):
        """Device float64 view of the full reordered free vector."""
        arr = getattr(vec, "array", vec)
        if isinstance(arr, torch.Tensor):
            if arr.device == self.device and arr.dtype == torch.float64 and arr.is_contiguous():
                if arr.numel() == self.layout.n_free:
                    return arr
            self._u[: self.layout.n_free].copy_(arr.reshape(-1), non_blocking=True)
            return self._u
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        if a.size != self.layout.n_free:
            raise ValueError(f"vector has {a.size} entries, expected {self.layout.n_free}")
        self._u[: a.size].copy_(torch.from_numpy(a), non_blocking=False)
        return self._u

    def create_vec(self, full_array_reordered=None):
        """Device vector of the owned range (the reference returns a PETSc Vec)."""
        v = torch.zeros(self.n_owned, dtype=torch.float64, device=self.device)
        if full_array_reordered is not None:
            a = torch.as_tensor(np.asarray(full_array_reordered, dtype=np.float64))
            v.copy_(a[self.layout.lo: self.layout.hi])
        return v

    # ---- device-level API ---------------------------------------------------
    def eval(self, u, flags, *, energy=None, grad=None, hess=None):
        """One fused kernel pass on the current stream; returns the output tensors."""
        u = self._as_u(u)
        energy = self._energy if energy is None else energy
        grad = self._grad if grad is None else grad
        hess = self.owned_values if hess is None else hess
        check(lib.fne_eval(
            self._handle, u.data_ptr(), int(flags),
            energy.data_ptr() if flags & _lib.FNE_ENERGY else None,
            grad.data_ptr() if flags & _lib.FNE_GRAD else None,
            hess.data_ptr() if flags & _lib.FNE_HESS else None,
            self._stream(),
        ))
        return energy, grad, hess

    def energy_device(self, u):
        """Energy as a 1-element CUDA tensor (no host synchronisation)."""
        return self.eval(u, _lib.FNE_ENERGY)[0]

    # ---- reference callbacks ------------------------------------------------
    def energy_fn(self, vec):
        t = time.perf_counter()
        self._ev0.record()
        e = self.eval(vec, _lib.FNE_ENERGY)[0]
        self._ev1.record()
        val = float(e.item())
        self._poll_status()
        st = self._callback_stats["energy"]
        st["calls"] += 1
        st["kernel"] += self._ev0.elapsed_time(self._ev1) * 1e-3
        st["total"] += time.perf_counter() - t
        return val

    def gradient_fn(self, vec, g):
        t = time.perf_counter()
        self._ev0.record()
        _, grad, _ = self.eval(vec, _lib.FNE_GRAD)
        self._ev1.record()
        out = getattr(g, "array", g)
        if isinstance(out, torch.Tensor):
            out.copy_(grad[: self.n_owned])
        else:
            out[:] = grad[: self.n_owned].cpu().numpy()
        st = self._callback_stats["gradient"]
        st["calls"] += 1
        torch.cuda.current_stream(self.device).synchronize()
        self._poll_status()
        st["kernel"] += self._ev0.elapsed_time(self._ev1) * 1e-3
        st["total"] += time.perf_counter() - t

    def assemble_hessian(self, u_owned, variant=2):
        del variant
        return self.assemble_hessian_element(u_owned)

    def assemble_hessian_element(self, u_owned):
        t_total = time.perf_counter()
        self._ev0.record()
        self.eval(u_owned, _lib.FNE_HESS)
        self._ev1.record()
        self._ev1.synchronize()
        self._poll_status()
        t_k = self._ev0.elapsed_time(self._ev1) * 1e-3
        timings = {"elem_hessian_compute": t_k, "scatter": 0.0, "hvp_compute": t_k, "extraction": 0.0,
                   "allgatherv": 0.0, "ghost_exchange": 0.0, "build_v_local": 0.0, "p2p_exchange": 0.0,
                   "n_hvps": 0, "assembly_mode": "element_overlap_cuda"}
        t0 = time.perf_counter()
        if self.A is not None:
            self.A.setValuesCOO(self.owned_values.double().cpu().numpy(), addv=1)
            self.A.assemble()
        timings["coo_assembly"] = time.perf_counter() - t0
        timings["total"] = time.perf_counter() - t_total
        self.iter_timings.append(timings)
        st = self._callback_stats["hessian"]
        st["calls"] += 1
        st["hvp_compute"] += t_k
        st["coo_assembly"] += timings["coo_assembly"]
        st["total"] += timings["total"]
        return timings

    def update_dirichlet(self, u_0_new):
        self.dirichlet_full = np.ascontiguousarray(u_0_new, dtype=np.float64).copy()
        a, p = _lib.f64(self.dirichlet_full)
        check(lib.fne_set_dirichlet(self._handle, p))

    def owned_values_host(self):
        return self.owned_values.cpu().numpy()

    def setup_summary(self):
        return {k: float(v) for k, v in self._setup_timings.items()}

    def callback_summary(self):
        return {k: dict(v) for k, v in self._callback_stats.items()}

    def memory_summary(self):
        return {"device_bytes": int(self.info["device_bytes"]), "owned_nnz": int(self.layout.owned_rows.size),
                "local_elements": int(self.info["n_elem"])}

    def cleanup(self):
        if getattr(self, "_handle", None):
            lib.fne_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.cleanup()
        except Exception:
            pass


class PLaplaceCudaAssembler(CudaElementAssemblerBase):
    """``PLaplaceReorderedElementAssembler`` (plaplace/jax_petsc/reordered_element_assembler.py:22-72)."""

    family = _lib.FNE_PLAPLACE
    npe, block_size = 3, 1
    coordinate_key, dirichlet_key = "nodes", "u_0"
    local_elem_data_keys = ("dvx", "dvy", "vol")

    def _scalars(self):
        return [float(self.params["p"])]

    def _build_rhs_owned(self):
        """``_build_rhs_owned`` (:67-72): f[freedofs][perm][lo:hi]."""
        rhs = np.asarray(self.params["f"], dtype=np.float64)
        free = np.asarray(self.params["freedofs"], dtype=np.int64)
        return np.ascontiguousarray(rhs[free][self.layout.perm][self.layout.lo: self.layout.hi])


class GLCudaAssembler(CudaElementAssemblerBase):
    """``GLReorderedElementAssembler`` (ginzburg_landau/jax_petsc/reordered_element_assembler.py:27-97)."""

    family = _lib.FNE_GINZBURG_LANDAU
    npe, block_size = 3, 1
    coordinate_key, dirichlet_key = "nodes", "u_0"
    local_elem_data_keys = ("dvx", "dvy", "vol")

    def _scalars(self):
        ip = np.asarray(self.params["ip"], dtype=np.float64).reshape(3, 3)
        w = np.asarray(self.params["w"], dtype=np.float64).reshape(3)
        return [float(self.params["eps"]), *ip.ravel().tolist(), *w.tolist()]

    def _adds_dirichlet_only_energy(self):
        return True


class HECudaAssembler(CudaElementAssemblerBase):
    """``HEReorderedElementAssembler`` (hyperelasticity/jax_petsc/reordered_element_assembler.py:16-101)."""

    family = _lib.FNE_NEOHOOKEAN
    npe, block_size = 4, 3
    coordinate_key, dirichlet_key = "nodes2coord", "u_0_ref"
    local_elem_data_keys = ("dphix", "dphiy", "dphiz", "vol")

    def __init__(self, params, comm=None, adjacency=None, *, use_abs_det=False, **kw):
        self.use_abs_det = bool(use_abs_det)
        super().__init__(params, comm, adjacency, **kw)

    def _scalars(self):
        return [float(self.params["C1"]), float(self.params["D1"]), 1.0 if self.use_abs_det else 0.0]


class SlopeStabilityCudaAssembler(CudaElementAssemblerBase):
    """``SlopeStabilityReorderedElementAssembler``
    (slope_stability/jax_petsc/reordered_element_assembler.py:75-243), plane-strain
    Mohr-Coulomb (``constitutive_mode="mc"``) or linear elastic (``"elastic"``).

    The element operators are passed as the element map (inverse Jacobian,
    ``|det J|`` and the reference-element basis gradients at the quadrature
    points) instead of the reference's stored ``elem_B``: one map per element
    (``inv_jac (E, 4)``, ``det_j (E,)``; P4, affine), or one per quadrature
    point (``(E, nq, 4)``, ``(E, nq)``; the isoparametric P2 map).  Without
    ``inv_jac`` the per-point map is recovered from the reference's
    ``elem_B`` / ``quad_weight`` (``meshes.geometry_from_elem_B``), so the
    reference's own problem data can be passed as is (it must then also
    carry ``dhat1``, ``dhat2`` and ``quad_w``).  The load vector is the
    gravity ``force`` restricted to the owned DOFs.
    """

    family = _lib.FNE_MOHR_COULOMB
    block_size = 2
    coordinate_key, dirichlet_key = "nodes", "u_0"

    def __init__(self, params, comm=None, adjacency=None, *, constitutive_mode="mc", **kw):
        self.constitutive_mode = str(constitutive_mode)
        if self.constitutive_mode not in ("mc", "elastic"):
            raise ValueError(f"Unsupported constitutive_mode {constitutive_mode!r}")
        self.npe = int(np.asarray(params["elems_scalar"]).shape[1])
        super().__init__(params, comm, adjacency, **kw)

    def _geometry(self):
        p = self.params
        if "inv_jac" in p:
            return np.asarray(p["inv_jac"], dtype=np.float64), np.asarray(p["det_j"], dtype=np.float64)
        from fenics_nonlinear_energies_b200.meshes import geometry_from_elem_B

        return geometry_from_elem_B(np.asarray(p["elem_B"], dtype=np.float64),
                                    np.asarray(p["quad_weight"], dtype=np.float64),
                                    np.asarray(p["dhat1"]), np.asarray(p["dhat2"]), np.asarray(p["quad_w"]))

    def _element_arrays(self):
        p = self.params
        epsp = np.asarray(p["eps_p_old"], dtype=np.float64)
        tables = np.concatenate((np.ravel(p["dhat1"]), np.ravel(p["dhat2"]), np.ravel(p["quad_w"])))
        inv, det = self._geometry()
        return [inv, det, epsp if np.any(epsp) else None, tables]

    def _nq(self):
        return int(np.asarray(self.params["quad_w"]).size)

    def _scalars(self):
        p = self.params
        per_point = 1.0 if self._geometry()[1].ndim == 2 else 0.0
        return [float(p["E"]), float(p["nu"]), float(p["phi_deg"]), float(p["cohesion"]),
                float(p.get("reg", 1.0e-12)), 1.0 if self.constitutive_mode == "elastic" else 0.0, per_point]

    # ---- matrix-free Hessian products -----------------------------------------
    # prepare_matrix_free_operator / matrix_free_mult / matrix_free_get_diagonal
    # (slope_stability/jax_petsc/reordered_element_assembler.py:335-562): the
    # linearization is kept on the device (weighted tangent per quadrature
    # point); products never assemble K.  Vectors as in eval: CUDA tensors,
    # NumPy arrays or objects with ``.array``.
    _MATFREE_MODES = ("matfree_element", "matfree_overlap")

    def prepare_matrix_free_operator(self, u_owned, *, mode="matfree_element"):
        """Linearize at ``u`` (full reordered free vector on one rank); returns self."""
        if str(mode) not in self._MATFREE_MODES:
            raise ValueError(f"Unsupported matrix-free operator mode {mode!r}")
        u = self._as_u(u_owned)
        check(lib.fne_hvp_prepare(self._handle, u.data_ptr(), self._stream()))
        self._matfree_mode = str(mode)
        return self

    def _matfree_check(self, mode):
        if getattr(self, "_matfree_mode", None) != str(mode):
            raise RuntimeError(f"Matrix-free operator {mode!r} is missing a matching linearization point")

    def matrix_free_mult(self, mode, x, y=None):
        """``y[owned] = H(u) x``; ``x``'s Dirichlet components are zero by construction."""
        self._matfree_check(mode)
        arr = getattr(x, "array", x)
        xt = torch.as_tensor(np.asarray(arr) if not isinstance(arr, torch.Tensor) else arr)
        xt = xt.to(device=self.device, dtype=torch.float64).contiguous().reshape(-1)
        if xt.numel() != self.layout.n_free:
            raise ValueError(f"tangent has {xt.numel()} entries, expected {self.layout.n_free}")
        out = torch.empty(max(1, self.n_owned), dtype=torch.float64, device=self.device)
        check(lib.fne_hvp(self._handle, xt.data_ptr(), out.data_ptr(), self._stream()))
        return self._deliver(out[: self.n_owned], y)

    def matrix_free_get_diagonal(self, mode, diag=None):
        """Owned diagonal of H(u)."""
        self._matfree_check(mode)
        out = torch.empty(max(1, self.n_owned), dtype=torch.float64, device=self.device)
        check(lib.fne_hvp_diagonal(self._handle, out.data_ptr(), self._stream()))
        return self._deliver(out[: self.n_owned], diag)

    @staticmethod
    def _deliver(t, dest):
        if dest is None:
            return t
        arr = getattr(dest, "array", dest)
        if isinstance(arr, torch.Tensor):
            arr.copy_(t)
        else:
            arr[:] = t.cpu().numpy()
        return dest

    def _build_rhs_owned(self):
        force = np.asarray(self.params["force"], dtype=np.float64)
        free = np.asarray(self.params["freedofs"], dtype=np.int64)
        return np.ascontiguousarray(force[free][self.layout.perm][self.layout.lo: self.layout.hi])


class SlopeStability3DCudaAssembler(CudaElementAssemblerBase):
    """``SlopeStability3DReorderedElementAssembler``
    (slope_stability_3d/jax_petsc/reordered_element_assembler.py:189-206,
    377-560): 3-D Mohr-Coulomb (``constitutive_mode="mc"``, the reference's
    "plastic" mode) or linear elastic (``"elastic"``) on P1 / P2 tetrahedra.

    Takes the reference's local element data as is: ``dphix``, ``dphiy``,
    ``dphiz`` (E, nq, n_p), ``quad_weight`` and the per-point material fields
    ``c_bar_q``, ``sin_phi_q``, ``shear_q``, ``bulk_q``, ``lame_q`` (E, nq)
    (the names without the ``_q`` suffix are accepted too), and the gravity
    ``force`` as the load vector.
    """

    family = _lib.FNE_MOHR_COULOMB_3D
    block_size = 3
    coordinate_key, dirichlet_key = "nodes", "u_0"
    _MATERIAL = ("c_bar", "sin_phi", "shear", "bulk", "lame")

    def __init__(self, params, comm=None, adjacency=None, *, constitutive_mode="mc", **kw):
        self.constitutive_mode = {"plastic": "mc"}.get(str(constitutive_mode), str(constitutive_mode))
        if self.constitutive_mode not in ("mc", "elastic"):
            raise ValueError(f"Unsupported constitutive_mode {constitutive_mode!r}")
        self.npe = int(np.asarray(params["elems_scalar"]).shape[1])
        super().__init__(params, comm, adjacency, **kw)

    def _field(self, name):
        p = self.params
        return np.asarray(p[name + "_q"] if name + "_q" in p else p[name], dtype=np.float64)

    def _element_arrays(self):
        p = self.params
        w = np.asarray(p["quad_weight"], dtype=np.float64)
        pts = np.stack([w] + [np.broadcast_to(self._field(k), w.shape) for k in self._MATERIAL], axis=-1)
        return [np.asarray(p[k], dtype=np.float64) for k in ("dphix", "dphiy", "dphiz")] + [pts]

    def _nq(self):
        return int(np.asarray(self.params["quad_weight"]).shape[1])

    def _scalars(self):
        return [1.0e-15, 0.0, 0.0, 0.0, 0.0, 1.0 if self.constitutive_mode == "elastic" else 0.0]

    def _build_rhs_owned(self):
        force = np.asarray(self.params["force"], dtype=np.float64)
        free = np.asarray(self.params["freedofs"], dtype=np.int64)
        return np.ascontiguousarray(force[free][self.layout.perm][self.layout.lo: self.layout.hi])


class EnergyFunction(torch.autograd.Function):
    """``J(u)`` with ``dJ/du`` from the hand-written adjoint kernels.

    ``u`` is the full reordered free vector (``layout.n_free`` entries).
    forward: one fused ENERGY|GRAD pass (the gradient is kept for backward);
    backward: ``grad_out * gradient`` as a tensor shaped like ``u``: the owned
    rows ``[lo, hi)`` hold this rank's rows of dJ/du, the other rows are 0, so
    summing the ranks' results gives dJ/du (one rank: dJ/du itself).  The
    Hessian is not part of the autograd graph: call
    ``assembler.assemble_hessian`` explicitly.
    """

    @staticmethod
    def forward(ctx, u, assembler):
        if u.numel() != assembler.layout.n_free:
            raise ValueError(f"u has {u.numel()} entries, expected layout.n_free = {assembler.layout.n_free}")
        e, g, _ = assembler.eval(u.detach().contiguous(), _lib.FNE_ENERGY | _lib.FNE_GRAD,
                                 energy=torch.empty(1, dtype=torch.float64, device=assembler.device),
                                 grad=torch.empty(max(1, assembler.n_owned), dtype=torch.float64,
                                                  device=assembler.device))
        ctx.save_for_backward(g)
        ctx.lo, ctx.hi, ctx.shape = int(assembler.layout.lo), int(assembler.layout.hi), u.shape
        return e[0]

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        full = torch.zeros(ctx.shape, dtype=g.dtype, device=g.device)
        full.view(-1)[ctx.lo: ctx.hi] = g[: ctx.hi - ctx.lo]
        return grad_out * full, None


def energy(u, assembler):
    """Differentiable energy: ``energy(u, asm).backward()`` fills ``u.grad``."""
    return EnergyFunction.apply(u, assembler)
