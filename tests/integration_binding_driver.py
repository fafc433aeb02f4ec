"""Executes the drop-in subclass text of INTEGRATION.md section 1 under the
reference's own assembler classes (test infrastructure; run in a subprocess
by ``test_integration_binding.py``, because the stand-in modules it installs
-- torch for JAX, fakes for mpi4py / petsc4py -- must not leak into other
tests).

The library is replaced by ``FakeLib``: ``fne_create`` reads back every
array and scalar the mixin put into the ``fne_desc`` (so a wrong pointer,
size or slot shows up), and ``fne_eval_host`` computes the documented
``fne_eval`` outputs from them with the oracle's element derivatives.  Each
case builds the unmodified reference assembler and the mixin assembler on
the same problem and reports their energies, gradients, COO values handed to
``Mat.setValuesCOO``, ``iter_timings`` keys and callback statistics.

Usage: ``python tests/integration_binding_driver.py REFERENCE_ROOT`` prints one
JSON object.
"""

from __future__ import annotations

import json
import math
import re
import sys
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

from tests.golden import refshim  # noqa: E402

FAMILY_NAMES = {1: "plaplace", 2: "gl", 3: "he", 4: "mc"}


def snippet():
    text = (ROOT / "INTEGRATION.md").read_text()
    sec = text[text.index("## 1. Drop-in subclass"):]
    return re.search(r"```python\n(.*?)```", sec, re.S).group(1)


class _Handle:
    """What fne_create would have copied to the device, read back from the descriptor."""

    def __init__(self, d, real):
        from fenics_nonlinear_energies_b200 import meshes

        def arr(ptr, count, dt=np.float64):
            if not ptr:
                return None
            return np.ctypeslib.as_array(ptr, shape=(int(count),)).astype(dt).copy()

        ne, n = int(d.n_elem), int(d.npe) * int(d.block_size)
        self.family = FAMILY_NAMES[int(d.family)]
        self.elems = arr(d.elems, ne * n, np.int64).reshape(ne, n)
        self.t2f = arr(d.total_to_free_reord, d.n_total, np.int64)
        self.rows = arr(d.owned_rows, d.nnz, np.int64)
        self.cols = arr(d.owned_cols, d.nnz, np.int64)
        w = arr(d.energy_weights, ne)
        self.w = np.ones(ne) if w is None else w
        self.dir = arr(d.dirichlet, d.n_total)
        self.lo, self.hi, self.n_free = int(d.lo), int(d.hi), int(d.n_free)
        self.rhs = arr(d.rhs_owned, self.hi - self.lo)
        s = list(d.s)
        if self.family in ("plaplace", "gl"):
            self.data = {"dvx": arr(d.e0, ne * 3).reshape(ne, 3), "dvy": arr(d.e1, ne * 3).reshape(ne, 3),
                         "vol": arr(d.e2, ne)}
            self.params = ({"p": s[0]} if self.family == "plaplace" else
                           {"eps": s[0], "ip": np.array(s[1:10]).reshape(3, 3), "w": np.array(s[10:13])})
        elif self.family == "he":
            self.data = {k: arr(p, ne * 4).reshape(ne, 4) for k, p in (("dphix", d.e0), ("dphiy", d.e1),
                                                                      ("dphiz", d.e2))}
            self.data["vol"] = arr(d.e3, ne)
            self.params = {"C1": s[0], "D1": s[1], "use_abs_det": bool(s[2])}
        else:
            npe, nq = int(d.npe), int(d.nq)
            per_point = s[6] != 0.0
            inv = arr(d.e0, ne * (nq if per_point else 1) * 4).reshape((ne, nq, 4) if per_point else (ne, 4))
            det = arr(d.e1, ne * (nq if per_point else 1)).reshape((ne, nq) if per_point else (ne,))
            tab = arr(d.e3, 2 * nq * npe + nq)
            dh1, dh2, wq = tab[: nq * npe].reshape(nq, npe), tab[nq * npe: 2 * nq * npe].reshape(nq, npe), \
                tab[2 * nq * npe:]
            ep = arr(d.e2, ne * nq * 3)
            self.data = {"elem_B": meshes.slope_elem_B({"inv_jac": inv, "dhat1": dh1, "dhat2": dh2}),
                         "quad_weight": (det if per_point else det[:, None]) * wq[None, :],
                         "eps_p_old": np.zeros((ne, nq, 3)) if ep is None else ep.reshape(ne, nq, 3)}
            self.params = {"E": s[0], "nu": s[1], "phi_deg": s[2], "cohesion": s[3], "reg": s[4],
                           "elastic": bool(s[5])}
        keys = self.rows * np.int64(self.n_free) + self.cols
        self.order = np.argsort(keys, kind="mergesort")
        self.keys_sorted = keys[self.order]

    def set_dirichlet(self, ptr):
        self.dir = np.ctypeslib.as_array(ptr, shape=(self.dir.size,)).copy()

    def eval(self, u, flags, e_out, g_out, h_out):
        from oracle import energies

        er = self.t2f[self.elems]
        v = np.where(er >= 0, u[np.maximum(er, 0)], self.dir[self.elems])
        e, g_e, h_e = energies.element_derivatives(self.family, v, self.data, self.params,
                                                   want_hessian=bool(flags & 4))
        u_owned = u[self.lo: self.hi]
        if flags & 1:
            e_out[0] = float(np.sum(self.w * e)) - (float(self.rhs @ u_owned) if self.rhs is not None else 0.0)
        if flags & 2:
            own = (er >= self.lo) & (er < self.hi)
            g = np.zeros(self.hi - self.lo)
            np.add.at(g, er[own] - self.lo, g_e[own])
            g_out[:] = g - (self.rhs if self.rhs is not None else 0.0)
        if flags & 4:
            ei, li, lj = np.nonzero(((er >= self.lo) & (er < self.hi))[:, :, None] & (er[:, None, :] >= 0))
            kp = np.searchsorted(self.keys_sorted, er[ei, li] * np.int64(self.n_free) + er[ei, lj])
            vals = np.zeros(self.rows.size)
            np.add.at(vals, self.order[kp], h_e[ei, li, lj])
            h_out[:] = vals


def make_fake_lib():
    from fenics_nonlinear_energies_b200 import _lib as real

    fake = types.ModuleType("fenics_nonlinear_energies_b200._lib")
    for k in dir(real):
        if not k.startswith("__") and k != "lib":
            setattr(fake, k, getattr(real, k))
    handles = {}

    class Lib:
        calls = {"create": 0, "eval": 0, "set_dirichlet": 0, "destroy": 0}

        @staticmethod
        def fne_create(dref, href):
            h = _Handle(dref._obj, real)
            hid = len(handles) + 1
            handles[hid] = h
            href._obj.value = hid
            Lib.calls["create"] += 1
            return 0

        @staticmethod
        def fne_eval_host(hv, u, flags, e, g, hh):
            h = handles[hv.value]
            n = h.n_free
            u = np.ctypeslib.as_array(u, shape=(n,))
            view = lambda p, k: None if not p else np.ctypeslib.as_array(p, shape=(k,))  # noqa: E731
            h.eval(u, flags, view(e, 1), view(g, h.hi - h.lo),
                   None if not hh else np.ctypeslib.as_array(real.C.cast(hh, real._f64p), shape=(h.rows.size,)))
            Lib.calls["eval"] += 1
            return 0

        @staticmethod
        def fne_set_dirichlet(hv, ptr):
            handles[hv.value].set_dirichlet(ptr)
            Lib.calls["set_dirichlet"] += 1
            return 0

        @staticmethod
        def fne_destroy(hv):
            handles.pop(hv.value, None)
            Lib.calls["destroy"] += 1
            return 0

    fake.lib = Lib
    return fake


def run(reference):
    refshim.install()
    sys.path.insert(0, str(reference))
    import fenics_nonlinear_energies_b200 as pkg

    fake = make_fake_lib()
    pkg._lib = fake
    sys.modules["fenics_nonlinear_energies_b200._lib"] = fake
    ns = {"__name__": "cuda_element_kernels"}
    exec(compile(snippet(), "INTEGRATION.md", "exec"), ns)

    from src.problems.ginzburg_landau.jax_petsc.reordered_element_assembler import GLReorderedElementAssembler
    from src.problems.hyperelasticity.jax_petsc.reordered_element_assembler import HEReorderedElementAssembler
    from src.problems.plaplace.jax_petsc.reordered_element_assembler import PLaplaceReorderedElementAssembler
    from src.problems.plaplace_u3.support.mesh import _build_scalar_adjacency
    from src.problems.slope_stability.jax_petsc.reordered_element_assembler import (
        SlopeStabilityReorderedElementAssembler)
    from src.problems.slope_stability.support.mesh import _build_dof_adjacency

    gold = ROOT / "tests" / "golden"

    def fixture(name):
        fx = dict(np.load(gold / f"reference_{name}.npz"))
        params = {k[3:]: v for k, v in fx.items() if k.startswith("in_")}
        params.update({k[3:]: float(v) for k, v in fx.items() if k.startswith("sc_")})
        return fx, params

    results = []
    cases = [
        ("gl", GLReorderedElementAssembler, ns["GLCudaReorderedElementAssembler"], {}, (1, 2)),
        ("plaplace", PLaplaceReorderedElementAssembler, ns["PLaplaceCudaReorderedElementAssembler"], {}, (1, 2)),
        ("he", HEReorderedElementAssembler, ns["HECudaReorderedElementAssembler"], {"use_near_nullspace": False},
         (1, 2)),
        ("mc_p2", SlopeStabilityReorderedElementAssembler, ns["SlopeStabilityCudaReorderedElementAssembler"],
         {"use_near_nullspace": False}, (1,)),
    ]
    for name, ref_cls, cuda_cls, kw, sizes in cases:
        fx, params = fixture(name)
        if name in ("gl", "plaplace"):
            adj = _build_scalar_adjacency(params["elems"], params["freedofs"])
        else:
            adj = _build_dof_adjacency(params["elems"], params["freedofs"])
        u = fx["in_u"]
        for size in sizes:
            for rank in range(size):
                out = {"case": name, "rank": rank, "size": size}
                pair = []
                for cls in (ref_cls, cuda_cls):
                    comm = refshim.FakeComm(rank, size)
                    comm.full = u
                    asm = cls(params, comm, adj, **kw)
                    if "in_dirichlet" in fx:
                        asm.update_dirichlet(fx["in_dirichlet"])
                    vec = asm.create_vec(u)
                    e = asm.energy_fn(vec)
                    g = asm.create_vec()
                    asm.gradient_fn(vec, g)
                    t = asm.assemble_hessian(np.asarray(u[asm.layout.lo: asm.layout.hi]))
                    pair.append((asm, e, g.array.copy(), asm.A.values.copy(), t))
                (ra, re_, rg, rh, rt), (ca, ce, cg, ch, ct) = pair
                out["energy"] = [re_, ce]
                out["grad_rel"] = float(np.abs(cg - rg).max(initial=0.0) / max(np.abs(rg).max(initial=0.0), 1e-300))
                out["hess_rel"] = float(np.abs(ch - rh).max(initial=0.0) / max(np.abs(rh).max(initial=0.0), 1e-300))
                out["coo_inserts"] = [ra.A.inserts, ca.A.inserts]
                out["timing_keys_missing"] = sorted(set(rt) - set(ct))
                out["iter_timings"] = [len(ra.iter_timings), len(ca.iter_timings)]
                out["iter_timings_last_is_returned"] = ca.iter_timings[-1] is ct
                rs, cs = ra.callback_summary(), ca.callback_summary()
                out["callback_calls"] = [{k: v["calls"] for k, v in rs.items()}, {k: v["calls"] for k, v in cs.items()}]
                out["callback_keys_missing"] = {k: sorted(set(rs[k]) - set(cs[k])) for k in rs}
                try:
                    ca._energy_jit(np.zeros(3))
                    out["jit_stub_raises"] = False
                except RuntimeError:
                    out["jit_stub_raises"] = True
                ca.cleanup()
                results.append(out)
    print(json.dumps({"results": results, "calls": fake.lib.calls,
                      "finite": all(math.isfinite(r["energy"][1]) for r in results)}))


if __name__ == "__main__":
    run(Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference"))
