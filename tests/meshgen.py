"""Test-side mesh generators (numpy), restating the reference's generators:

* ``hole_plate`` -- Mesh::genRectWithHole (src/Mesh.cu:112-246) including the
  ring renumbering of Mesh::renumerateRing (src/Mesh.cu:332-380). ``rad_n``
  may be given explicitly (the O-grid of the benchmark configurations); by
  default it is tied to the perimeter count exactly as the reference does.
* ``ring`` -- Mesh::genRing (src/Mesh.cu:249-329).
* ``rect`` -- Mesh::genRectangle (src/Mesh.cu:17-110), order 1.
* ``split_t3`` -- splits every quad (n1,n2,n3,n4) into (n1,n2,n3),(n1,n3,n4).

They exist so tests can build identical inputs for the oracle, the reference
harness and the product; the product has its own generators in C++.
"""
import math

import numpy as np


def _renumerate_ring(node, elem4, borders, border_n):
    node_count = node.shape[0]
    rad_n = node_count // border_n
    new = np.zeros(node_count, dtype=np.int64)
    new_n = 0
    j_front, j_back = 0, border_n - 1
    while j_back > j_front:
        for i in range(rad_n):
            new[i * border_n + j_front] = new_n
            new_n += 1
        for i in range(rad_n):
            new[i * border_n + j_back] = new_n
            new_n += 1
        j_front += 1
        j_back -= 1
    if j_back == j_front:
        # the reference writes newNodes[newN++] = old index here (a bug for
        # odd column counts); reproduced so that odd counts match it too
        for i in range(rad_n):
            new[new_n] = i * border_n + j_front
            new_n += 1
    elem4 = new[elem4]
    borders = [new[b] for b in borders]
    nodes = np.zeros_like(node)
    nodes[new] = node
    return nodes, elem4, borders


def hole_plate(x1, x2, y1, y2, hole_rad, n1, n2, rad_n=None):
    """O-grid around a centred circular hole, Q4, order 1."""
    border_n = (n1 + n2) * 2
    if rad_n is None:
        rad_n = (n1 + n2) // 4
        rad_n = int(round(float(rad_n) * (x2 - x1 + y2 - y1 - 4.0 * hole_rad) * 2.0 / (x2 - x1 + y2 - y1)))
    node_count = border_n * (rad_n + 1)
    node = np.zeros((node_count, 2))
    blen = [n1 + 1, n2 + 1, n1 + 1, n2 + 1, border_n + 1]
    borders = [np.zeros(L, dtype=np.int64) for L in blen]
    nid = 0
    hx, hy = (x2 - x1) / n1, (y2 - y1) / n2
    for i in range(n1):
        node[nid] = (x1 + i * hx, y1)
        borders[0][i] = nid
        nid += 1
    borders[0][-1] = nid
    for j in range(n2):
        node[nid] = (x2, y1 + j * hy)
        borders[1][j] = nid
        nid += 1
    borders[1][-1] = nid
    for i in range(n1):
        node[nid] = (x2 - i * hx, y2)
        borders[2][i] = nid
        nid += 1
    borders[2][-1] = nid
    for j in range(n2):
        node[nid] = (x1, y2 - j * hy)
        borders[3][j] = nid
        nid += 1
    borders[3][-1] = 0
    pi = 3.141592653589793
    phi = 2.0 * pi / border_n
    nid = rad_n * border_n
    cx, cy = 0.5 * (x1 + x2), 0.5 * (y1 + y2)
    start = phi * (n1 + n2 * 1.5)
    for i in range(border_n):
        a = start + i * phi
        node[nid] = (cx + math.cos(a) * hole_rad, cy + math.sin(a) * hole_rad)
        borders[4][border_n - i - 1] = nid
        nid += 1
    borders[4][-1] = node_count - 1
    rh = (node[rad_n * border_n] - node[0]) / rad_n
    for i in range(1, rad_n):
        node[i * border_n] = node[0] + rh * i
    rh = (node[node_count - 1] - node[border_n - 1]) / rad_n
    for i in range(1, rad_n):
        node[i * border_n + border_n - 1] = node[border_n - 1] + rh * i
    for j in range(1, border_n):
        rh = (node[rad_n * border_n + j] - node[j]) / rad_n
        for i in range(1, rad_n):
            node[i * border_n + j] = node[j] + rh * i
    count4 = border_n * rad_n
    elem4 = np.zeros((count4, 4), dtype=np.int64)
    for i in range(rad_n):
        for j in range(border_n - 1):
            k = j * rad_n + i
            elem4[k] = ((i + 1) * border_n + j + 1, (i + 1) * border_n + j, i * border_n + j, i * border_n + j + 1)
        k = (border_n - 1) * rad_n + i
        elem4[k] = ((i + 1) * border_n, (i + 1) * border_n + border_n - 1, i * border_n + border_n - 1, i * border_n)
    node, elem4, borders = _renumerate_ring(node, elem4, borders, border_n)
    return dict(node_xy=node, elem4=elem4.astype(np.int32), elem3=np.zeros((0, 3), np.int32),
                borders=[b.astype(np.int32) for b in borders])


def ring(a, b, n_phi, n_r):
    node_count = (n_r + 1) * n_phi
    node = np.zeros((node_count, 2))
    borders = [np.zeros(n_phi + 1, dtype=np.int64), np.zeros(n_phi + 1, dtype=np.int64)]
    pi = 3.141592653589793
    h_r, h_phi = (b - a) / n_r, 2.0 * pi / n_phi
    for j in range(n_phi):
        for i in range(n_r + 1):
            r = b - h_r * i
            ph = h_phi * j
            node[i * n_phi + j] = (r * math.cos(ph), r * math.sin(ph))
        borders[1][n_phi - j] = j
        borders[0][j] = n_r * n_phi + j
    borders[1][0] = 0
    borders[0][n_phi] = n_r * n_phi
    count4 = n_r * n_phi
    elem4 = np.zeros((count4, 4), dtype=np.int64)
    for i in range(n_r):
        for j in range(n_phi - 1):
            k = j * n_r + i
            elem4[k] = ((i + 1) * n_phi + j + 1, (i + 1) * n_phi + j, i * n_phi + j, i * n_phi + j + 1)
        k = (n_phi - 1) * n_r + i
        elem4[k] = ((i + 1) * n_phi, (i + 1) * n_phi + n_phi - 1, i * n_phi + n_phi - 1, i * n_phi)
    node, elem4, borders = _renumerate_ring(node, elem4, borders, n_phi)
    return dict(node_xy=node, elem4=elem4.astype(np.int32), elem3=np.zeros((0, 3), np.int32),
                borders=[b.astype(np.int32) for b in borders])


def rect(x1, x2, y1, y2, n1, n2):
    node_count = (n1 + 1) * (n2 + 1)
    node = np.zeros((node_count, 2))
    h1, h2 = (x2 - x1) / n1, (y2 - y1) / n2
    for i in range(n1 + 1):
        for j in range(n2 + 1):
            node[i * (n2 + 1) + j] = (x1 + h1 * i, y1 + h2 * j)
    elem4 = np.zeros((n1 * n2, 4), dtype=np.int64)
    for i in range(n1):
        for j in range(n2):
            elem4[i * n2 + j] = ((i + 1) * (n2 + 1) + j + 1, i * (n2 + 1) + j + 1, i * (n2 + 1) + j, (i + 1) * (n2 + 1) + j)
    borders = [np.zeros(n2 + 1, np.int64), np.zeros(n1 + 1, np.int64), np.zeros(n2 + 1, np.int64), np.zeros(n1 + 1, np.int64)]
    for i in range(n2 + 1):
        borders[0][n2 - i] = (n1 + 1) * (n2 + 1) - i - 1
        borders[2][n2 - i] = i
    for i in range(n1 + 1):
        borders[1][n1 - i] = (i + 1) * (n2 + 1) - 1
        borders[3][n1 - i] = (n1 - i) * (n2 + 1)
    return dict(node_xy=node, elem4=elem4.astype(np.int32), elem3=np.zeros((0, 3), np.int32),
                borders=[b.astype(np.int32) for b in borders])


def split_t3(mesh):
    q = np.asarray(mesh["elem4"], dtype=np.int64)
    tri = np.empty((2 * q.shape[0], 3), dtype=np.int64)
    tri[0::2] = q[:, [0, 1, 2]]
    tri[1::2] = q[:, [0, 2, 3]]
    return dict(node_xy=mesh["node_xy"], elem4=np.zeros((0, 4), np.int32), elem3=tri.astype(np.int32),
                borders=mesh["borders"])


def axis_dofs(node_xy, tol=1e-9):
    """Symmetry constraints for a ring centred at the origin: u_y = 0 on the x
    axis, u_x = 0 on the y axis (removes the three rigid-body modes)."""
    xy = np.asarray(node_xy)
    r = np.hypot(xy[:, 0], xy[:, 1])
    on_x = np.where(np.abs(xy[:, 1]) <= tol * r)[0]
    on_y = np.where(np.abs(xy[:, 0]) <= tol * r)[0]
    return sorted([2 * int(n) + 1 for n in on_x] + [2 * int(n) for n in on_y])
