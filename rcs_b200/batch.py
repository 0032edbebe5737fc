"""Batches of independent bodies: concurrent factorization and FGMRES solves
(aifmm_batch_factorize / aifmm_batch_solve_gmres), and the seeded ellipsoid
family of the batched benchmark configuration.

Each body needs its own Context (its own stream): the library's host threads
drive the bodies concurrently, so the small kernels of many bodies share the
GPU.  The reference solves one geometry per process (test/sphere.cpp); a batch
gives each body the result the one-body calls give it."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from . import mesh as M


def ellipsoid_family(n: int = 64, seed: int = 64, subdivisions=(3, 4)) -> list[tuple[M.Mesh, tuple]]:
    """n ellipsoids with semi-axes drawn from U[0.05, 0.3] m (numpy's MT19937
    generator seeded with `seed`, three draws per body), meshed as icospheres
    of subdivisions[b % len(subdivisions)] scaled by the semi-axes."""
    rng = np.random.Generator(np.random.MT19937(seed))
    out = []
    for b in range(n):
        axes = tuple(float(a) for a in rng.uniform(0.05, 0.3, size=3))
        out.append((M.ellipsoid(subdivisions[b % len(subdivisions)], axes), axes))
    return out


def _ptrs(objs) -> C.Array:
    return (C.c_void_p * len(objs))(*[o.h.value if isinstance(o.h, C.c_void_p) else o.h for o in objs])


def batch_factorize(solvers, threads: int = 16) -> float:
    """Factorize every solver (each on its own Context) concurrently; returns
    the batch's wall seconds."""
    sec = C.c_double()
    _lib.check(_lib.lib().aifmm_batch_factorize(_ptrs(solvers), len(solvers), int(threads), C.byref(sec)))
    return sec.value


def batch_solve_gmres(solvers, ops, rhs_list, tol: float = 1e-6, restart: int = 30, maxit: int = 200,
                      threads: int = 16):
    """FGMRES of every body (rhs_list[i]: N_i x nrhs_i); returns (solutions,
    records, seconds)."""
    n = len(solvers)
    bs = [np.ascontiguousarray(np.asarray(b, dtype=np.complex128).reshape(s.N, -1).T) for s, b in zip(solvers, rhs_list)]
    xs = [np.zeros_like(b) for b in bs]
    nr = (C.c_int * n)(*[b.shape[0] for b in bs])
    rp = (C.c_void_p * n)(*[b.ctypes.data for b in bs])
    xp = (C.c_void_p * n)(*[x.ctypes.data for x in xs])
    infos = (_lib.GmresInfo * n)()
    sec = C.c_double()
    _lib.check(_lib.lib().aifmm_batch_solve_gmres(_ptrs(solvers), _ptrs(ops), rp, nr, xp, n, float(tol), int(restart),
                                                  int(maxit), int(threads), C.cast(infos, C.c_void_p),
                                                  C.byref(sec)))
    sols = [x.T.copy() for x in xs]
    recs = [{f: getattr(g, f) for f, _ in g._fields_} for g in infos]
    return sols, recs, sec.value
