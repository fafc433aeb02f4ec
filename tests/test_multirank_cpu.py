"""Two-rank paths on the CPU (gloo, world size 2, spawned processes).

* ``bench.py``'s rank plumbing: process-group set-up from the environment,
  barrier, and the max-over-ranks reduction used for the timed region.
* The ownership decomposition the drop-in relies on for N > 1: every rank
  builds its own layout (C++ ``fne_layout_build`` and the oracle, which must
  agree) and evaluates its owned part of energy, gradient and Hessian; the
  sum of the rank energies and the union of the owned gradient rows and COO
  values equal the single-rank results
  (``src/core/petsc/reordered_element_base.py:509-597, 1579-1633, 1733-1775``).
"""

import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)


def _bench_worker(rank, world, port, out):
    _env(rank, world, port)
    import bench

    w, r, _ = bench._dist_setup()
    assert (w, r) == (world, rank)
    bench._barrier(w)
    m = bench._max_over_ranks(float(rank + 1) * 0.5, w)
    out[rank] = m
    dist.destroy_process_group()


def test_bench_rank_reduction_gloo():
    port = _free_port()
    out = mp.Manager().dict()
    mp.spawn(_bench_worker, args=(2, port, out), nprocs=2, join=True)
    assert out[0] == out[1] == 1.0


def _decomp_worker(rank, world, port, family, out):
    _env(rank, world, port)
    from fenics_nonlinear_energies_b200 import _lib, meshes
    from oracle.assembler import OracleAssembler

    dist.init_process_group("gloo", rank=rank, world_size=world)
    if family == "gl":
        params, u0 = meshes.gl_problem(n=12, seed=2)
        kw, bs, ck = {}, 1, "nodes"
    else:
        params, u0 = meshes.he_beam_problem(nx=6, ny=2, nz=2)
        kw, bs, ck = {"block_size": 3, "coordinate_key": "nodes2coord", "dirichlet_key": "u_0_ref"}, 3, "nodes2coord"
    ref = OracleAssembler(family, params, rank=rank, size=world, **kw)
    lay = _lib.build_layout(freedofs=params["freedofs"], elems=params["elems"],
                            n_total=len(ref.dirichlet_full), block_size=bs, coords=params[ck],
                            rank=rank, size=world)
    assert (lay["lo"], lay["hi"]) == (ref.layout.lo, ref.layout.hi)
    np.testing.assert_array_equal(lay["owned_rows"], ref.layout.owned_rows)
    np.testing.assert_array_equal(lay["owned_cols"], ref.layout.owned_cols)
    u = np.asarray(u0, dtype=np.float64)[np.asarray(ref.layout.perm)]
    if family == "he":
        u = u + 1e-3 * np.random.default_rng(3).standard_normal(u.size)
    e, g, h = ref.all_in_one(u)
    et = torch.tensor([e], dtype=torch.float64)
    dist.all_reduce(et)
    parts = [None] * world
    dist.all_gather_object(parts, (ref.layout.lo, np.asarray(g), np.asarray(ref.layout.owned_rows),
                                   np.asarray(ref.layout.owned_cols), np.asarray(h)))
    if rank == 0:
        out["energy"] = float(et.item())
        out["parts"] = parts
        out["u"] = u
    dist.destroy_process_group()


@pytest.mark.parametrize("family", ["gl", "he"])
def test_two_rank_decomposition_gloo(family):
    from fenics_nonlinear_energies_b200 import meshes
    from oracle.assembler import OracleAssembler

    port = _free_port()
    out = mp.Manager().dict()
    mp.spawn(_decomp_worker, args=(2, port, family, out), nprocs=2, join=True)
    if family == "gl":
        params, _ = meshes.gl_problem(n=12, seed=2)
        full = OracleAssembler("gl", params)
    else:
        params, _ = meshes.he_beam_problem(nx=6, ny=2, nz=2)
        full = OracleAssembler("he", params, block_size=3, coordinate_key="nodes2coord", dirichlet_key="u_0_ref")
    u = out["u"]
    e1, g1, h1 = full.all_in_one(u)
    assert abs(out["energy"] - e1) <= 1e-12 * max(1.0, abs(e1))
    g = np.zeros_like(g1)
    vals = {}
    for lo, gr, rows, cols, hv in out["parts"]:
        g[lo: lo + gr.size] = gr
        vals.update({(int(r), int(c)): v for r, c, v in zip(rows, cols, hv)})
    np.testing.assert_allclose(g, g1, rtol=0, atol=1e-12 * np.abs(g1).max())
    ref_vals = {(int(r), int(c)): v for r, c, v in zip(full.layout.owned_rows, full.layout.owned_cols, h1)}
    assert vals.keys() == ref_vals.keys()
    diff = max(abs(vals[k] - ref_vals[k]) for k in ref_vals)
    assert diff <= 1e-12 * max(abs(v) for v in ref_vals.values())
