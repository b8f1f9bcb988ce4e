"""Oracle helper (test infrastructure): box-scene pressure system in the reference's MacPressureInputs3D form
(mac_pressure_3d.h:14-61): fluid cells in (z,y,x) order, every incident face
with its link kind -- internal between fluid cells, Dirichlet p = 0 at
distance h against air, sealed against solid cells."""

import numpy as np

from fluidity_b200 import scenes


def box_pressure_system(box, cell_type, u_pred, density=scenes.DENSITY):
    n = [box.n[0], box.n[1], box.n[2]]
    h = box.h
    ct = np.asarray(cell_type)
    k, j, i = np.nonzero(ct == 1)
    order = np.lexsort((i, j, k))
    k, j, i = k[order], j[order], i[order]
    cells_idx = np.stack([i, j, k], 1).astype(np.int32)
    cells_val = np.zeros((len(i), 5))
    cells_val[:, 0] = h ** 3
    faces = []
    for a in range(3):
        shape = box.face_shape(a)
        fk, fj, fi = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
        head = [fi, fj, fk]
        tail = [fi.copy(), fj.copy(), fk.copy()]
        tail[a] = tail[a] - 1

        def typ(c):
            ok = (c[0] >= 0) & (c[1] >= 0) & (c[2] >= 0) & (c[0] < n[0]) & (c[1] < n[1]) & (c[2] < n[2])
            t = np.zeros(c[0].shape, np.int32)
            t[ok] = ct[c[2][ok], c[1][ok], c[0][ok]]
            return t

        th, tt = typ(head), typ(tail)
        inc = (th == 1) | (tt == 1)
        other = np.where(th == 1, tt, th)
        kind = np.where(other == 0, 0, np.where(other == 1, 1, 2))[inc]
        vals = np.zeros((inc.sum(), 6))
        open_ = kind != 0
        vals[open_, 0] = h * h
        vals[open_, 1] = 1.0 / density
        vals[open_, 2] = h
        vals[:, 3] = np.asarray(u_pred[a])[inc]
        idx = np.stack([np.full(inc.sum(), a), fi[inc], fj[inc], fk[inc]], 1)
        faces.append((idx, kind, vals))
    faces_idx = np.concatenate([f[0] for f in faces]).astype(np.int32)
    faces_kind = np.concatenate([f[1] for f in faces]).astype(np.int32)
    faces_val = np.concatenate([f[2] for f in faces])
    order = owned_slot_order(faces_idx)
    faces_idx, faces_kind, faces_val = faces_idx[order], faces_kind[order], faces_val[order]
    return dict(cells_idx=cells_idx, cells_val=cells_val, faces_idx=faces_idx, faces_kind=faces_kind,
                faces_val=faces_val)


def owned_slot_order(faces_idx):
    """Permutation putting faces (axis, x, y, z) in the reference's owned-slot
    order: 4^3 block (z, y, x), normal axis, local (z, y, x)
    (SparseMacGrid3D::FaceSlot, sparse_mac_grid_3d.cc:388-409)."""
    a, x, y, z = (faces_idx[:, k].astype(np.int64) for k in range(4))
    return np.lexsort((x % 4, y % 4, z % 4, a, x // 4, y // 4, z // 4))


def ref_blocks_for_box(n):
    """All 4^3 reference blocks of an n^3 box plus the high ring that owns the
    faces at index n."""
    nb = n // 4 + 1
    return np.array([[x, y, z] for z in range(nb) for y in range(nb) for x in range(nb)], np.int32)
