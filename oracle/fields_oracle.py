"""CPU oracle of the exported node fields (test infrastructure only).

A NumPy restatement of what chfem writes with -e for a solved load case:
  thermal  (chfem/src/femhmg/physical_phenomena/femhmg_thermal_3D.c:674-692 fluxFromTemp,
            :694-1111 saveFields_thermal_3D) -- per node, 3 heat-flux components q = k grad T;
  elastic  (femhmg_elastic_3D.c:1710-1750 stressFromDispl, :1800-2650 saveFields_elastic_3D) --
            per node, 6 stress components D(E, nu) B u, Voigt order xx yy zz yz xz xy with
            engineering shear strains.
Each voxel evaluates its field at each of its 8 corners and adds 1/8 of it into that corner's
node; a voxel on the +axis boundary of the periodic cell (x: last column, y: first row, z:
first layer) sees the load case's macroscopic jump (the cell length in voxels along the
axis) on its +face nodes, in the loaded component (femhmg_thermal_3D.c:827-1090 and
femhmg_elastic_3D.c:1973-2630, the "compensate for periodic borders" loops).

Node and voxel arrays here are indexed [layer][col][row] (node id = row + col*ny + layer*ny*nx,
C-order flattening), the order of chfem's DOF vectors and field files.  Used only by tests to
check the product's fields; nothing in the product imports this file.
"""
import numpy as np


def _drow(k):
    return -((k & 3) >> 1)


def _dcol(k):
    return 1 if (k & 3) in (1, 2) else 0


def _dlay(k):
    return k >> 2


def _corner(k):
    """Local coordinates of voxel node k: x right, y up, z towards the near face."""
    return _dcol(k), -_drow(k), 1 - _dlay(k)


def _grad_shape(j, px, py, pz):
    """Gradient of the trilinear shape function of local node j at the local point (px, py, pz)."""
    xj, yj, zj = _corner(j)
    fx, fy, fz = (px if xj else 1 - px), (py if yj else 1 - py), (pz if zj else 1 - pz)
    sx, sy, sz = (1 if xj else -1), (1 if yj else -1), (1 if zj else -1)
    return np.array([sx * fy * fz, fx * sy * fz, fx * fy * sz], dtype=np.float64)


def _face_nodes(axis):
    return [j for j in range(8) if _corner(j)[axis] == 1]


def elastic_D(E, nu):
    co = E / ((1 + nu) * (1 - 2 * nu))
    D = np.zeros((6, 6))
    D[:3, :3] = co * nu
    for i in range(3):
        D[i, i] = co * (1 - nu)
        D[3 + i, 3 + i] = co * 0.5 * (1 - 2 * nu)
    return D


def node_fields(x, mat, props, axis, comp, nd):
    """Nodal flux (nd == 1) or stress (nd == 3).

    x: solution, N*nd values in DOF order; mat: [layer][col][row] voxel material index;
    props: per material index, k (thermal) or (E, nu) (elastic); axis/comp: the load case
    (X 0/0, Y 1/1, Z 2/2, YZ 1/2, XZ 2/0, XY 1/0; thermal comp 0).  Returns N*nf values.
    """
    L, C, R = mat.shape
    X = np.asarray(x, np.float64).reshape(L, C, R, nd)
    jump = float((C, R, L)[axis])
    boundary = np.zeros((L, C, R), bool)
    if axis == 0:
        boundary[:, C - 1, :] = True
    elif axis == 1:
        boundary[:, :, 0] = True
    else:
        boundary[0, :, :] = True
    # the 8 local nodes' values of every voxel, plus the jump on its +face nodes
    U = []
    faces = _face_nodes(axis)
    for j in range(8):
        Uj = np.roll(X, shift=(-_dlay(j), -_dcol(j), -(1 + _drow(j))), axis=(0, 1, 2)).copy()
        if j in faces:
            Uj[..., comp] += np.where(boundary, jump, 0.0)
        U.append(Uj)
    nf = 3 if nd == 1 else 6
    out = np.zeros((L, C, R, nf))
    if nd == 1:
        kv = np.asarray([props[i] for i in range(len(props))], np.float64)[mat]
    else:
        Ds = np.stack([elastic_D(*props[i]) for i in range(len(props))])[mat]  # [L][C][R][6][6]
    for k in range(8):
        G = np.zeros((L, C, R, nd, 3))  # gradient of each component at corner k
        for j in range(8):
            G += U[j][..., :, None] * _grad_shape(j, *_corner(k))[None, None, None, None, :]
        if nd == 1:
            F = kv[..., None] * G[..., 0, :]
        else:
            strain = np.stack([G[..., 0, 0], G[..., 1, 1], G[..., 2, 2], G[..., 1, 2] + G[..., 2, 1],
                               G[..., 0, 2] + G[..., 2, 0], G[..., 0, 1] + G[..., 1, 0]], axis=-1)
            F = np.einsum("...ij,...j->...i", Ds, strain)
        # voxel corner k is the node at (row + 1 + drow(k), col + dcol(k), layer + dlay(k))
        out += 0.125 * np.roll(F, shift=(_dlay(k), _dcol(k), 1 + _drow(k)), axis=(0, 1, 2))
    return out.reshape(-1)


def materials_from_image(img, codes, refinement=1):
    """[layer][col][row] material index of a (z, y, x) image whose phase codes, in the .nf
    file's order, are `codes`; each voxel split into refinement^3 (femhmg.c:1644-1700)."""
    lut = np.full(256, -1, np.int64)
    for i, c in enumerate(codes):
        lut[c] = i
    m = lut[np.asarray(img, np.uint8)]
    assert (m >= 0).all()
    for ax in range(3):
        m = np.repeat(m, refinement, axis=ax)
    return np.ascontiguousarray(m.transpose(0, 2, 1))
