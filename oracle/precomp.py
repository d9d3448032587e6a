"""Test infrastructure: the reference's adjacency precomputation restated in
numpy, and writers of its text files, for runs that must not load the
product library (the benchmark's reference arm prepares its inputs with
these and reads them back through the reference's own readers).

* ``build_con`` restates buildIncid + buildCon (vfRayPreComp.cc:219-501).
  Face f of tet t is its vertices (f, f+1, f+2) mod 4 (vfRayPreComp.cc:442-
  448).  The neighbour across it is the tet with the smallest id other than
  t among the tets holding the same vertex triple -- the first one the
  reference's incidence search meets, as it scans tets in ascending order --
  or t itself when there is none (a boundary face).  Returns (con (nT, 4),
  number of boundary faces).
* ``build_extf`` restates buildExtF (vfRayPreComp.cc:710-737): the boundary
  faces as (tet, face) pairs, tet-then-face order.
* ``write_off/con/extf/tf`` write the layouts readOff, readCon, readExtF and
  readTF parse (vfRayPreComp.cc:29-69, 375-420, 551-590).

Nothing in the vfray_b200 product imports this module.
"""
from __future__ import annotations

import numpy as np

# vertex k of face f is (f + k) mod 4
_FACE_VERTS = (np.arange(4)[:, None] + np.arange(3)[None, :]) % 4


def build_con(tet):
    tet = np.ascontiguousarray(tet, np.uint32).reshape(-1, 4)
    nT = tet.shape[0]
    tri = np.sort(tet[:, _FACE_VERTS], axis=2).reshape(-1, 3)  # face 4t+f
    owner = np.repeat(np.arange(nT, dtype=np.int64), 4)
    order = np.lexsort((owner, tri[:, 2], tri[:, 1], tri[:, 0]))
    st, tt = tri[order], owner[order]
    head = np.ones(len(order), bool)
    head[1:] = np.any(st[1:] != st[:-1], axis=1)
    start = np.flatnonzero(head)
    size = np.diff(np.append(start, len(order)))
    g = np.cumsum(head) - 1
    first = tt[start[g]]                                   # smallest tet of the triple
    second = tt[np.minimum(start[g] + 1, len(order) - 1)]  # the next smallest
    nb = np.where(size[g] == 1, tt, np.where(first != tt, first, second))
    con = np.empty(4 * nT, np.uint32)
    con[order] = nb.astype(np.uint32)
    con = con.reshape(nT, 4)
    n_ext = int(np.count_nonzero(con == np.arange(nT, dtype=np.uint32)[:, None]))
    return con, n_ext


def build_extf(con):
    con = np.asarray(con).reshape(-1, 4)
    t, f = np.nonzero(con == np.arange(con.shape[0], dtype=con.dtype)[:, None])
    return np.stack([t, f], axis=1).astype(np.uint32)


def _write_rows(f, a, fmt):
    np.savetxt(f, a, fmt=fmt)


def write_off(path, vert4, tet):
    with open(path, "w") as f:
        f.write(f"{len(vert4)} {len(tet)}\n")
        _write_rows(f, np.asarray(vert4, np.float32), "%.9g")
        _write_rows(f, np.asarray(tet, np.uint32), "%d")


def write_con(path, con, n_ext):
    with open(path, "w") as f:
        f.write(f"{n_ext}\n{len(con)}\n")
        _write_rows(f, np.asarray(con, np.uint32), "%d")


def write_extf(path, extf):
    with open(path, "w") as f:
        f.write(f"{len(extf)}\n")
        _write_rows(f, np.asarray(extf, np.uint32), "%d")


def write_tf(path, tf):
    with open(path, "w") as f:
        f.write("256\n")
        _write_rows(f, np.asarray(tf, np.float32), "%.9g")
