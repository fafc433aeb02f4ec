"""Stand-in modules that let the reference's own assembly code run here.

Test infrastructure only: used by ``make_fixtures.py`` (in a container that
holds the reference sources) and by the binding test of the drop-in subclass;
nothing in the package imports it.

The reference's element assembly is plain NumPy plus JAX
(``jax.numpy``, ``jax.vmap``, ``jax.grad``, ``jax.hessian``, ``jax.jit``,
``lax.cond``) and talks to MPI and PETSc through ``mpi4py`` / ``petsc4py``.
None of these is installed, so ``install()`` puts stand-ins into
``sys.modules`` before the reference is imported:

* ``jax`` / ``jax.numpy`` / ``jax.lax``: torch (float64, CPU).  ``vmap``,
  ``grad``, ``hessian`` and ``jvp`` map to ``torch.func``; ``jit`` is the
  identity; ``lax.cond`` evaluates both branches and selects with
  ``torch.where`` (what JAX does for a batched predicate under ``vmap``);
  ``lax.stop_gradient`` detaches.  The derivatives are therefore torch's
  autodiff of the reference's own energy code, standing in for JAX's.
* ``mpi4py.MPI``: a communicator of a given rank / size whose collectives
  act on one process (``allreduce`` returns the local value, ``Allgatherv``
  copies a caller-provided full vector, see ``FakeComm.full``).
* ``petsc4py.PETSc``: ``Vec`` with an ``array``; ``Mat`` that records
  ``setPreallocationCOO`` / ``setValuesCOO``; inert KSP / PC / Options.
* ``basix``, ``h5py``, ``igraph``: empty modules (only import-time names).
"""

from __future__ import annotations

import sys
import types

import numpy as np
import torch
import torch.func as tfunc

F64 = torch.float64


# ----------------------------------------------------------------------------
# jax.numpy on torch
# ----------------------------------------------------------------------------
def _tensor(x, dtype=None):
    if isinstance(x, torch.Tensor):
        return x if dtype is None else x.to(_dt(dtype))
    if isinstance(x, (list, tuple)) and any(isinstance(v, (torch.Tensor, list, tuple)) for v in x):
        parts = [_tensor(v, dtype) for v in x]
        common = parts[0].dtype
        for p in parts[1:]:
            common = torch.promote_types(common, p.dtype)
        if dtype is None and not common.is_floating_point and any(p.dtype.is_floating_point for p in parts):
            common = F64
        return torch.stack([p.to(common if dtype is None else _dt(dtype)) for p in parts])
    a = np.asarray(x)
    if a.dtype == np.float32 and dtype is None:
        a = a.astype(np.float64)
    t = torch.as_tensor(a)
    return t if dtype is None else t.to(_dt(dtype))


def _dt(dtype):
    if isinstance(dtype, torch.dtype):
        return dtype
    return {np.dtype(np.float64): F64, np.dtype(np.float32): torch.float32,
            np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64,
            np.dtype(np.bool_): torch.bool}[np.dtype(dtype)]


def _pair(a, b):
    ta = a if isinstance(a, torch.Tensor) else None
    tb = b if isinstance(b, torch.Tensor) else None
    like = ta if ta is not None else tb
    if ta is None:
        ta = torch.as_tensor(a, dtype=like.dtype if like is not None else F64)
    if tb is None:
        tb = torch.as_tensor(b, dtype=like.dtype if like is not None else F64)
    return ta, tb


def _make_jnp():
    jnp = types.ModuleType("jax.numpy")
    jnp.float64, jnp.float32, jnp.int32, jnp.int64, jnp.bool_ = F64, torch.float32, torch.int32, torch.int64, torch.bool
    jnp.pi = float(np.pi)
    jnp.inf = float("inf")
    jnp.nan = float("nan")
    jnp.ndarray = torch.Tensor
    jnp.asarray = lambda x, dtype=None: _tensor(x, dtype)
    jnp.array = lambda x, dtype=None: _tensor(x, dtype)

    def _sum(x, axis=None, keepdims=False):
        x = _tensor(x)
        return x.sum() if axis is None else x.sum(dim=axis, keepdim=keepdims)

    jnp.sum = _sum
    for name in ("sqrt", "log", "exp", "abs", "sin", "cos", "tan", "arcsin", "arccos", "arctan", "tanh",
                 "deg2rad", "rad2deg", "square", "sign", "isfinite", "floor", "ceil", "cosh", "sinh", "log1p"):
        tname = {"arcsin": "asin", "arccos": "acos", "arctan": "atan"}.get(name, name)
        setattr(jnp, name, (lambda f: lambda x: f(_tensor(x) if not isinstance(x, torch.Tensor) else x))(
            getattr(torch, tname)))
    jnp.arctan2 = lambda y, x: torch.atan2(*_pair(y, x))
    jnp.maximum = lambda a, b: torch.maximum(*_pair(a, b))
    jnp.minimum = lambda a, b: torch.minimum(*_pair(a, b))

    def _where(c, a, b):
        c = _tensor(c)
        a, b = _pair(a, b)
        return torch.where(c, a, b)

    jnp.where = _where
    jnp.einsum = lambda spec, *ops, **_kw: torch.einsum(spec, *[_tensor(o) for o in ops])  # optimize= ignored
    jnp.stack = lambda xs, axis=0: torch.stack([_tensor(v) for v in xs], dim=axis)
    jnp.concatenate = lambda xs, axis=0: torch.cat([_tensor(v) for v in xs], dim=axis)
    jnp.zeros = lambda shape, dtype=F64: torch.zeros(shape, dtype=_dt(dtype))
    jnp.ones = lambda shape, dtype=F64: torch.ones(shape, dtype=_dt(dtype))
    jnp.zeros_like = lambda x, dtype=None: torch.zeros_like(_tensor(x), dtype=None if dtype is None else _dt(dtype))
    jnp.ones_like = lambda x, dtype=None: torch.ones_like(_tensor(x), dtype=None if dtype is None else _dt(dtype))
    jnp.dot = lambda a, b: torch.matmul(_tensor(a), _tensor(b))
    jnp.matmul = jnp.dot
    jnp.outer = lambda a, b: torch.outer(_tensor(a), _tensor(b))
    jnp.trace = lambda a: torch.trace(_tensor(a))
    jnp.clip = lambda x, lo=None, hi=None: torch.clamp(_tensor(x), lo, hi)
    linalg = types.ModuleType("jax.numpy.linalg")
    linalg.eigvalsh = lambda a: torch.linalg.eigvalsh(_tensor(a))
    linalg.det = lambda a: torch.linalg.det(_tensor(a))
    linalg.inv = lambda a: torch.linalg.inv(_tensor(a))
    linalg.norm = lambda a, *args, **kw: torch.linalg.norm(_tensor(a), *args, **kw)
    jnp.linalg = linalg
    return jnp, linalg


def _cond(pred, true_fn, false_fn, *operands, operand=None):
    args = operands if operands else (operand,)
    t = true_fn(*args)
    f = false_fn(*args)
    p = _tensor(pred)
    if isinstance(t, tuple):
        return tuple(torch.where(p, *_pair(a, b)) for a, b in zip(t, f))
    return torch.where(p, *_pair(t, f))


def _vmap(fun, in_axes=0, out_axes=0):
    return tfunc.vmap(fun, in_dims=in_axes if isinstance(in_axes, (tuple, int)) or in_axes is None else tuple(in_axes),
                      out_dims=out_axes)


def _jit(fun=None, **_kw):
    if fun is None:
        return lambda f: f
    return fun


def _make_jax():
    jax = types.ModuleType("jax")
    jnp, linalg = _make_jnp()
    lax = types.ModuleType("jax.lax")
    lax.cond = _cond
    lax.stop_gradient = lambda x: x.detach() if isinstance(x, torch.Tensor) else x
    config = types.SimpleNamespace(update=lambda *a, **k: None)
    jax.numpy, jax.lax, jax.config = jnp, lax, config
    jax.vmap = _vmap
    jax.grad = lambda f, argnums=0: tfunc.grad(f, argnums=argnums)
    jax.hessian = lambda f, argnums=0: tfunc.hessian(f, argnums=argnums)
    jax.jacfwd = lambda f, argnums=0: tfunc.jacfwd(f, argnums=argnums)
    jax.jacrev = lambda f, argnums=0: tfunc.jacrev(f, argnums=argnums)
    jax.jvp = lambda f, primals, tangents: tfunc.jvp(f, tuple(primals), tuple(tangents))
    jax.jit = _jit
    jax.block_until_ready = lambda x: x
    tree_util = types.ModuleType("jax.tree_util")
    tree_util.tree_map = lambda f, *trees: f(*trees)
    jax.tree_util = tree_util
    return {"jax": jax, "jax.numpy": jnp, "jax.numpy.linalg": linalg, "jax.lax": lax, "jax.tree_util": tree_util}


# ----------------------------------------------------------------------------
# mpi4py / petsc4py
# ----------------------------------------------------------------------------
class FakeComm:
    """One-process communicator playing rank ``rank`` of ``size``.

    ``full`` (set by the caller before a callback) is the full reordered free
    vector that ``Allgatherv`` hands back, i.e. what the other ranks' owned
    pieces would have filled in."""

    SUM, MAX, MIN = "sum", "max", "min"

    def __init__(self, rank=0, size=1):
        self.rank, self.size = int(rank), int(size)
        self.full = None

    def Get_rank(self):
        return self.rank

    def Get_size(self):
        return self.size

    def allreduce(self, value, op=None):
        return value

    def allgather(self, value):
        return [value] * self.size

    def bcast(self, value, root=0):
        return value

    def Barrier(self):
        return None

    barrier = Barrier

    def Allgatherv(self, send, recv):
        full = recv[0]
        if self.size == 1:
            full[:] = np.asarray(send, dtype=full.dtype)
        else:
            if self.full is None:
                raise RuntimeError("FakeComm.full must hold the full vector for a multi-rank Allgatherv")
            full[:] = self.full
        return None


def _make_mpi():
    mpi4py = types.ModuleType("mpi4py")
    MPI = types.ModuleType("mpi4py.MPI")
    MPI.COMM_WORLD = FakeComm()
    MPI.COMM_SELF = FakeComm()
    MPI.Comm = FakeComm
    MPI.SUM, MPI.MAX, MPI.MIN = FakeComm.SUM, FakeComm.MAX, FakeComm.MIN
    MPI.DOUBLE, MPI.INT, MPI.LONG, MPI.INT64_T = "double", "int", "long", "int64"
    mpi4py.MPI = MPI
    return {"mpi4py": mpi4py, "mpi4py.MPI": MPI}


class _Inert:
    """Accepts any call and returns itself (KSP, PC, Options, LGMap, events)."""

    def __getattr__(self, name):
        return self

    def __call__(self, *a, **k):
        return self

    def __setitem__(self, key, value):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


class FakeVec:
    def __init__(self, n=0):
        self.array = np.zeros(int(n), dtype=np.float64)

    def createMPI(self, sizes, comm=None):
        n = sizes[0] if isinstance(sizes, (tuple, list)) else sizes
        self.array = np.zeros(int(n), dtype=np.float64)
        return self

    def assemble(self):
        return None

    def getArray(self, readonly=False):
        return self.array

    def duplicate(self):
        v = FakeVec(self.array.size)
        return v

    def destroy(self):
        return None


class FakeMat:
    """Records the COO pattern and every ``setValuesCOO`` call."""

    class Type:
        MPIAIJ = "mpiaij"
        AIJ = "aij"
        PYTHON = "python"

    def __init__(self):
        self.coo_rows = self.coo_cols = None
        self.values = None
        self.inserts = 0
        self.type = None

    def create(self, comm=None):
        return self

    def setType(self, t):
        self.type = t

    def getType(self):
        return self.type

    def setSizes(self, *a, **k):
        pass

    def setBlockSize(self, *a):
        pass

    def setPreallocationCOO(self, rows, cols):
        self.coo_rows, self.coo_cols = np.array(rows), np.array(cols)

    def setValuesCOO(self, values, addv=None):
        self.values = np.array(values, dtype=np.float64)
        self.inserts += 1

    def assemble(self):
        pass

    def __getattr__(self, name):  # setOption, setNearNullSpace, destroy, ...
        return lambda *a, **k: None


def _make_petsc():
    petsc4py = types.ModuleType("petsc4py")
    PETSc = types.ModuleType("petsc4py.PETSc")
    PETSc.ScalarType = np.float64
    PETSc.IntType = np.int32
    PETSc.RealType = np.float64
    PETSc.InsertMode = types.SimpleNamespace(INSERT_VALUES=1, ADD_VALUES=2, INSERT=1, ADD=2)
    PETSc.Vec = FakeVec
    PETSc.Mat = FakeMat
    PETSc.KSP = _Inert
    PETSc.PC = _Inert
    PETSc.Options = _Inert
    PETSc.LGMap = _Inert
    PETSc.NullSpace = _Inert
    PETSc.LogEvent = _Inert
    PETSc.Log = types.SimpleNamespace(Event=_Inert())
    PETSc.Viewer = _Inert
    PETSc.COMM_WORLD = FakeComm()
    PETSc.Sys = _Inert()
    petsc4py.PETSc = PETSc
    petsc4py.init = lambda *a, **k: None
    return {"petsc4py": petsc4py, "petsc4py.PETSc": PETSc}


def install():
    """Put the stand-ins into ``sys.modules`` (idempotent)."""
    if getattr(sys.modules.get("jax"), "__fne_shim__", False):
        return
    mods = {}
    mods.update(_make_jax())
    mods.update(_make_mpi())
    mods.update(_make_petsc())
    for name in ("basix", "h5py", "igraph", "pyamg", "dolfinx"):
        mods[name] = types.ModuleType(name)
    mods["jax"].__fne_shim__ = True
    sys.modules.update(mods)
    if not hasattr(torch.Tensor, "block_until_ready"):
        torch.Tensor.block_until_ready = lambda self: self
    torch.set_default_dtype(torch.float64)
