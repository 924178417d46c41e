"""Adaptive hyperoctree (oracle restatement of ``core/hypoct.m``).

Indices are 0-based here; the reference is 1-based.  A tree is a dict:

``nlvl``   number of levels
``lvp``    level pointer, length nlvl+1: boxes of level L (1-based) are
           ``range(lvp[L-1], lvp[L])``                       (hypoct.m:67,126)
``l``      d x nlvl box sizes                                 (hypoct.m:127)
``ctr``    nbox x d centres
``xi``     list of int64 arrays (point ids; empty for split boxes)
``prnt``   int array (-1 for the root)
``chld``   list of int arrays (ascending child key order)
``nbor``   list of int arrays (siblings, coarser leaves, then children of
           parent-neighbours, the order of hypoct.m:141-170)
"""
import math

import numpy as np


def mround(v):
    """MATLAB ``round``: halves away from zero (numpy rounds halves to even)."""
    v = np.asarray(v, dtype=np.float64)
    a = np.abs(v)
    f = np.floor(a)
    r = f + (a - f >= 0.5)
    return np.copysign(r, v)


def hypoct(x, occ, lvlmax=math.inf, ext=None):
    """Build the hyperoctree of points ``x`` (d x N).  core/hypoct.m:51-171."""
    x = np.asarray(x, dtype=np.float64)
    if lvlmax is None:
        lvlmax = math.inf
    if not occ >= 0:
        raise ValueError("FLAM:hypoct:invalidOcc: Leaf occupancy must be nonnegative.")
    if not lvlmax >= 1:
        raise ValueError("FLAM:hypoct:invalidLvlmax: Maximum tree depth must be at least 1.")
    d, n = x.shape
    # root node (hypoct.m:65-69)
    if ext is None or np.size(ext) == 0:
        ext = np.stack([x.min(axis=1), x.max(axis=1)], axis=1)
    ext = np.asarray(ext, dtype=np.float64).reshape(d, 2)
    l = ext[:, 1] - ext[:, 0]
    ctr0 = 0.5 * (ext[:, 0] + ext[:, 1])
    ctr = [ctr0]
    xi = [np.arange(n, dtype=np.int64)]
    prnt = [-1]
    chld = [[]]
    lvp = [0, 1]
    ls = [l.copy()]
    nlvl = 1
    nbox = 1
    pw = 2 ** np.arange(d)
    while True:
        if nlvl >= lvlmax:
            break
        nbox_ = nbox
        ldiv = l >= np.max(l) / math.sqrt(2)          # hypoct.m:81
        l = l.copy()
        l[ldiv] = 0.5 * l[ldiv]                         # hypoct.m:82
        for p in range(lvp[nlvl - 1], lvp[nlvl]):
            pts = xi[p]
            if len(pts) > occ:                          # hypoct.m:90
                c = ctr[p]
                side = (x[:, pts] > c[:, None]) & ldiv[:, None]
                key = pw @ side.astype(np.int64)        # hypoct.m:92-93
                for u in np.unique(key):                # ascending, hypoct.m:94
                    bits = ((u >> np.arange(d)) & 1).astype(np.float64)
                    ctr.append(c + (l * ldiv) * (bits - 0.5))   # hypoct.m:108
                    xi.append(pts[key == u])
                    prnt.append(p)
                    chld.append([])
                    chld[p].append(nbox)
                    nbox += 1
                xi[p] = np.zeros(0, dtype=np.int64)     # hypoct.m:116
        if nbox <= nbox_:                               # hypoct.m:121
            break
        nlvl += 1
        lvp.append(nbox)
        ls.append(l.copy())
    lvp = np.asarray(lvp, dtype=np.int64)
    lmat = np.stack(ls, axis=1)
    ctr = np.stack(ctr, axis=0)
    prnt = np.asarray(prnt, dtype=np.int64)
    chld = [np.asarray(c, dtype=np.int64) for c in chld]
    # box level (1-based) of every box
    boxlvl = np.zeros(nbox, dtype=np.int64)
    for L in range(1, nlvl + 1):
        boxlvl[lvp[L - 1]:lvp[L]] = L
    nbor = [np.zeros(0, dtype=np.int64) for _ in range(nbox)]
    # neighbours (hypoct.m:141-170)
    for L in range(2, nlvl + 1):
        lL = lmat[:, L - 1]
        for i in range(lvp[L - 1], lvp[L]):
            c = ctr[i]
            p = prnt[i]
            j = chld[p]
            nb = list(j[j != i])                        # hypoct.m:148-149
            for jj in nbor[p]:                          # hypoct.m:152-160
                if len(xi[jj]) > 0:
                    jl = lmat[:, boxlvl[jj] - 1]
                    dist = mround((np.abs(c - ctr[jj]) - 0.5 * (lL + jl)) / lL)
                    if np.max(dist) <= 0:
                        nb.append(jj)
            idx = [cc for q in nbor[p] for cc in chld[q]]   # hypoct.m:163
            if idx:
                idx = np.asarray(idx, dtype=np.int64)
                dist = mround(np.abs(c[:, None] - ctr[idx].T) / lL[:, None])
                nb.extend(idx[np.max(dist, axis=0) <= 1].tolist())
            nbor[i] = np.asarray(nb, dtype=np.int64)
    return dict(nlvl=nlvl, lvp=lvp, l=lmat, ctr=ctr, xi=xi, prnt=prnt,
                chld=chld, nbor=nbor, boxlvl=boxlvl, d=d, N=n)


def hypoct_perm(t):
    """Natural (pre-order) permutation, last child popped first.  core/hypoct_perm.m:11-39."""
    out = []
    stack = [0]
    while stack:
        i = stack.pop()
        out.extend(t["xi"][i].tolist())
        stack.extend(t["chld"][i].tolist())
    return np.asarray(out, dtype=np.int64)


def tree_arrays(t):
    """Flatten a tree into CSR arrays (the layout the device tree exports)."""
    nbox = len(t["xi"])

    def csr(lists):
        ptr = np.zeros(nbox + 1, dtype=np.int64)
        ptr[1:] = np.cumsum([len(a) for a in lists])
        ind = np.concatenate([np.asarray(a, dtype=np.int64) for a in lists]) if ptr[-1] else np.zeros(0, np.int64)
        return ptr, ind

    xp, xv = csr(t["xi"])
    cp, cv = csr(t["chld"])
    npt, nv = csr(t["nbor"])
    return dict(nlvl=t["nlvl"], lvp=t["lvp"], l=t["l"], ctr=t["ctr"], prnt=t["prnt"],
                xi_ptr=xp, xi=xv, chld_ptr=cp, chld=cv, nbor_ptr=npt, nbor=nv)
