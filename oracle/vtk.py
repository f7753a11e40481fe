"""Minimal reader for the ASCII VTK POLYDATA files the reference writes
(PlasticitySolver::saveAsVtk, src/PlasticitySolver.cu:1784-1945): points,
polygons, the CELL_DATA field block and the POINT_DATA displacement block.

TEST INFRASTRUCTURE ONLY (golden-fixture extraction).
"""
import numpy as np


def read_solution_vtk(path):
    with open(path) as f:
        tok = f.read().split()
    i = 0
    out = {"cell_fields": {}, "point_fields": {}}
    n = len(tok)
    while i < n:
        t = tok[i]
        if t == "POINTS":
            npts = int(tok[i + 1])
            vals = np.array(tok[i + 3 : i + 3 + 3 * npts], dtype=np.float64)
            out["points"] = vals.reshape(npts, 3)[:, :2]
            i += 3 + 3 * npts
        elif t == "POLYGONS":
            ncell, total = int(tok[i + 1]), int(tok[i + 2])
            vals = np.array(tok[i + 3 : i + 3 + total], dtype=np.int64)
            cells, j = [], 0
            while j < total:
                k = vals[j]
                cells.append(vals[j + 1 : j + 1 + k])
                j += k + 1
            out["polygons"] = cells
            i += 3 + total
        elif t == "CELL_DATA":
            ncells = int(tok[i + 1])
            i += 2
            # skip "SCALARS ElementID int 1 LOOKUP_TABLE default" + ids
            if tok[i] == "SCALARS":
                i += 6 + ncells
            if tok[i] == "FIELD":
                nf = int(tok[i + 2])
                i += 3
                for _ in range(nf):
                    name, cnt = tok[i], int(tok[i + 2])
                    out["cell_fields"][name] = np.array(tok[i + 4 : i + 4 + cnt], dtype=np.float64)
                    i += 4 + cnt
        elif t == "POINT_DATA":
            npts = int(tok[i + 1])
            i += 2
            if tok[i] == "SCALARS":
                i += 6 + npts
            if tok[i] == "FIELD":
                nf = int(tok[i + 2])
                i += 3
                for _ in range(nf):
                    name, ncomp, cnt = tok[i], int(tok[i + 1]), int(tok[i + 2])
                    vals = np.array(tok[i + 4 : i + 4 + ncomp * cnt], dtype=np.float64)
                    out["point_fields"][name] = vals.reshape(cnt, ncomp)
                    i += 4 + ncomp * cnt
        else:
            i += 1
    return out
