"""Shared test helpers: synthetic pieces, their oracle lattices and loads."""
import numpy as np

import statics_cuda as sc
from oracle import oracle as O


def piece(n, seed, k_dist=sc.K_UNIFORM, shape=None):
    nx, ny, nz = shape or (n, n, n)
    return sc.generate_piece(nx, ny, nz, seed, k_dist)


def oracle_lattice(state, k):
    return O.Lattice.grid(state, k, g_over_e=0.4, rho=512.0)


def z_loads(lat):
    """Gravity -1 along z per unit mass: loads(v) = [0, 0, -m_v, 0, 0, 0]."""
    ex = lat.export()
    loads = np.zeros((lat.n_nodes, 6))
    loads[:, 2] = -ex["m"]
    return loads, ex


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def lattice_dict(ex, level=0):
    return dict(x=ex["x"], held=ex["held"], around=ex["around"], bi=ex["bi"], bj=ex["bj"], p=ex["p"], n=ex["n"],
                a=ex["a"], d=ex["d"], e=ex["e"], g=ex["g"], level=level)
