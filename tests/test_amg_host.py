"""Host set-up of the aggregation multigrid hierarchy (cpx_amg_*), CPU only.

The hierarchy has no counterpart in the reference (its CG is unpreconditioned
or block-Jacobi, src/ConjGradSolver.h:52-101), so it is checked against a
numpy restatement of the same construction written here, and by its
properties: orthonormal prolongator blocks, rigid-body modes in the range of
the first prolongator, Galerkin blocks equal to the sparse triple product
T^T A T, and a V-cycle built on it that preconditions the elastic stiffness
of the reference's own assembly (the oracle's) far better than the 2x2
block-Jacobi of the device CG.
"""
import os

import numpy as np
import pytest
import scipy.linalg as sla
import scipy.sparse as sp

import meshgen
import oracle
import scenarios
from cudaplasticity_b200 import CuplastError, Hierarchy

# ------------------------------------------------------------ restatement --


def aggregate(adj_pos, adj, part_pos):
    """Greedy aggregation inside each partition: pass 1 takes a node and its
    neighbours when all are free; pass 2 joins each remaining node to its
    first aggregated neighbour or makes it a singleton. Edges between
    partitions are ignored; aggregates are renumbered partition by
    partition."""
    n = len(adj_pos) - 1
    part = np.searchsorted(part_pos, np.arange(n), side="right") - 1
    agg = -np.ones(n, np.int64)
    na = 0
    for i in range(n):
        nb = adj[adj_pos[i]:adj_pos[i + 1]]
        nb = nb[part[nb] == part[i]]
        if agg[i] < 0 and np.all(agg[nb] < 0):
            agg[i] = na
            agg[nb] = na
            na += 1
    for i in range(n):
        if agg[i] >= 0:
            continue
        nb = adj[adj_pos[i]:adj_pos[i + 1]]
        nb = nb[part[nb] == part[i]]
        got = agg[nb][agg[nb] >= 0]
        if len(got):
            agg[i] = got[0]
        else:
            agg[i] = na
            na += 1
    apart = np.zeros(na, np.int64)
    apart[agg] = part
    order = np.argsort(apart, kind="stable")
    renum = np.empty(na, np.int64)
    renum[order] = np.arange(na)
    cpart = np.concatenate([[0], np.cumsum(np.bincount(apart, minlength=len(part_pos) - 1))])
    return renum[agg], na, cpart


def mgs(B):
    """Modified Gram-Schmidt of B's 3 columns; dependent columns are zeroed."""
    B = B.copy()
    R = np.zeros((3, 3))
    ref = np.linalg.norm(B, axis=0)
    for c in range(3):
        for p in range(c):
            R[p, c] = B[:, p] @ B[:, c]
            B[:, c] -= R[p, c] * B[:, p]
        nrm = np.linalg.norm(B[:, c])
        if not nrm > 1e-10 * ref[c] or nrm == 0.0:
            B[:, c] = 0.0
            continue
        R[c, c] = nrm
        B[:, c] /= nrm
    return B, R


def merged_ranges(part_pos, min_range=16):
    """A coarse level aggregates inside its inherited ranges, each merged with
    its successors until it holds at least min_range nodes (a short last
    range joins the one before)."""
    out = [0]
    for p in range(1, len(part_pos)):
        if part_pos[p] - out[-1] >= min_range or p + 1 == len(part_pos):
            out.append(part_pos[p])
    if len(out) > 2 and out[-1] - out[-2] < min_range:
        del out[-2]
    return np.array(out)


def restate(adj_pos, adj, xy, mask, min_coarse_dofs, part_nodes=0):
    """Levels as dicts (graph, partitions, aggregates, prolongator blocks)."""
    levels = []
    n, fb = len(adj_pos) - 1, 2
    ns = None
    part_pos = np.array([0, n]) if part_nodes == 0 else np.append(np.arange(0, n, part_nodes), n)
    while True:
        lev = dict(nodes=n, dofs=fb, adj_pos=np.asarray(adj_pos), adj=np.asarray(adj), parts=part_pos)
        levels.append(lev)
        if n * fb <= min_coarse_dofs:
            break
        agg, na, cpart = aggregate(lev["adj_pos"], lev["adj"], part_pos if fb == 2 else merged_ranges(part_pos))
        if na >= n:
            break
        if ns is None:  # rigid-body modes about each aggregate's centroid
            ns = np.zeros((n, 2, 3))
            for a in range(na):
                mem = np.where(agg == a)[0]
                c = xy[mem].mean(axis=0)
                d = xy[mem] - c
                for i, (dx, dy) in zip(mem, d):
                    if mask[2 * i]:
                        ns[i, 0] = (1.0, 0.0, -dy)
                    if mask[2 * i + 1]:
                        ns[i, 1] = (0.0, 1.0, dx)
        T = np.zeros((n, fb, 3))
        ns_c = np.zeros((na, 3, 3))
        nb_c = [[] for _ in range(na)]
        for a in range(na):
            mem = np.where(agg == a)[0]
            Q, R = mgs(ns[mem].reshape(-1, 3))
            T[mem] = Q.reshape(len(mem), fb, 3)
            ns_c[a] = R
            for i in mem:
                for j in lev["adj"][lev["adj_pos"][i]:lev["adj_pos"][i + 1]]:
                    b = agg[j]
                    if b != a and b not in nb_c[a]:
                        nb_c[a].append(b)
        lev.update(agg=agg, aggregates=na, T=T)
        adj_pos = np.concatenate([[0], np.cumsum([len(x) for x in nb_c])])
        adj = np.array([b for x in nb_c for b in x], np.int64)
        n, fb, ns, part_pos = na, 3, ns_c, cpart
    return levels


# ----------------------------------------------------------------- inputs --


def elastic_system(name, workdir):
    """Graph, mask and the first (elastic) stiffness of a scenario, from the
    oracle's assembly."""
    path = os.path.join(workdir, f"{name}.bin")
    m, lines = scenarios.scenario_lines(name, path, mode="elastic", extra=["dump_k 1", "dump_csr 1"])
    oracle.write_mesh(path, m["node_xy"], elem3=m["elem3"], elem4=m["elem4"], borders=m["borders"],
                      elem8=m.get("elem8", ()))
    return m, oracle.run_oracle(lines)


def config1_system(workdir):
    """The 64x64 O-grid plate with a hole (8320 DOF), top traction, elastic."""
    m = meshgen.hole_plate(-100.0, 100.0, -100.0, 100.0, 20.0, 16, 16, rad_n=64)
    path = os.path.join(workdir, "plate64.bin")
    oracle.write_mesh(path, m["node_xy"], elem3=m["elem3"], elem4=m["elem4"], borders=m["borders"])
    lines = ["mode elastic", f"mesh file {path}", "cg_eps 1e-8", "material 210000 0.3 1",
             "diagram linear 210000 250 2000", "force 2 0 200 0", "fixborderhor 0", "fixpoint -100 -100",
             "dump_k 1", "dump_csr 1"]
    return m, oracle.run_oracle(lines)


def blocks_from_csr(r):
    """2x2 blocks of the reference CSR: row pair (2n, 2n+1) holds the blocks
    of columns (n, adj[adj_pos[n]], ...), two values per block per row."""
    ap, rows, k = r["adj_pos"], r["rows"], r["k_data"]
    out = []
    for i in range(len(ap) - 1):
        w = ap[i + 1] - ap[i] + 1
        r0 = k[rows[2 * i]:rows[2 * i] + 2 * w].reshape(w, 2)
        r1 = k[rows[2 * i + 1]:rows[2 * i + 1] + 2 * w].reshape(w, 2)
        out.append(np.stack([r0, r1], axis=1))
    return np.concatenate(out)


def block_matrix(adj_pos, adj, blocks, fb):
    n = len(adj_pos) - 1
    rows, cols = [], []
    for i in range(n):
        cs = [i] + list(adj[adj_pos[i]:adj_pos[i + 1]])
        for j in cs:
            rows.append(i)
            cols.append(j)
    return sp.bsr_matrix((blocks, np.asarray(cols), np.concatenate([[0], np.cumsum(np.diff(adj_pos) + 1)])),
                         shape=(fb * n, fb * n)).tocsr()


def t_matrix(lev):
    n, fb, na = lev["nodes"], lev["dofs"], lev["aggregates"]
    T = sp.lil_matrix((fb * n, 3 * na))
    for i in range(n):
        a = lev["agg"][i]
        T[fb * i:fb * i + fb, 3 * a:3 * a + 3] = lev["T"][i]
    return T.tocsr()


# ------------------------------------------------------------------ tests --

MESHES = ["hole12_pow", "ogrid16_bilin", "ring_pw", "hole12_q8_pow", "ogrid16_t3"]


@pytest.mark.parametrize("name,part", [(m, 0) for m in MESHES] + [("ogrid16_bilin", 32), ("hole12_q8_pow", 64)])
def test_hierarchy_matches_restatement(name, part, workdir):
    m, r = elastic_system(name, workdir)
    xy = np.asarray(m["node_xy"], np.float64).reshape(-1, 2)
    h = Hierarchy(r["adj_pos"], r["adj"], xy, r["mask"], min_coarse_dofs=40, part_nodes=part)
    ref = restate(r["adj_pos"], r["adj"], xy, r["mask"], 40, part)
    assert len(h) == len(ref) >= 2
    for lv in range(len(ref)):
        got, want = h.level(lv), ref[lv]
        assert got["nodes"] == want["nodes"] and got["dofs"] == want["dofs"]
        assert np.array_equal(h.parts(lv), want["parts"])
        assert np.array_equal(got["adj_pos"], want["adj_pos"])
        assert np.array_equal(got["adj"], want["adj"])
        if "agg" in want:
            assert got["aggregates"] == want["aggregates"]
            assert np.array_equal(got["agg"], want["agg"])
            assert np.max(np.abs(got["T"] - want["T"])) <= 1e-12
        else:
            assert got["aggregates"] == 0 and "agg" not in got


def test_partitioned_aggregates_stay_inside(workdir):
    m, r = elastic_system("ogrid16_bilin", workdir)
    xy = np.asarray(m["node_xy"], np.float64).reshape(-1, 2)
    h = Hierarchy(r["adj_pos"], r["adj"], xy, r["mask"], min_coarse_dofs=40, part_nodes=32)
    assert len(h.parts(0)) - 1 == -(-len(xy) // 32)
    lev, pp, cp_ = h.level(0), h.parts(0), h.parts(1)
    assert len(pp) == len(cp_)
    for p in range(len(pp) - 1):
        a = lev["agg"][pp[p]:pp[p + 1]]
        assert a.min() >= cp_[p] and a.max() < cp_[p + 1]
    for lv in range(1, len(h) - 1):
        # coarser levels: no aggregate crosses the merged inherited ranges
        lev, rg = h.level(lv), merged_ranges(h.parts(lv))
        for p in range(len(rg) - 1):
            a = lev["agg"][rg[p]:rg[p + 1]]
            if p + 1 < len(rg) - 1:
                assert a.max() < lev["agg"][rg[p + 1]]


def test_prolongator_properties(workdir):
    m, r = elastic_system("ogrid16_bilin", workdir)
    xy = np.asarray(m["node_xy"], np.float64).reshape(-1, 2)
    mask = r["mask"].astype(bool)
    h = Hierarchy(r["adj_pos"], r["adj"], xy, r["mask"], min_coarse_dofs=40)
    lev = h.level(0)
    T = t_matrix(lev).toarray()
    # orthonormal columns (or zero ones, dropped), zero rows on prescribed DOFs
    G = T.T @ T
    d = np.diag(G)
    assert np.all((np.abs(d - 1) < 1e-12) | (d == 0))
    assert np.max(np.abs(G - np.diag(d))) < 1e-12
    assert np.all(T[~mask] == 0)
    # the rigid-body modes restricted to the free DOFs lie in range(T)
    rb = np.zeros((2 * len(xy), 3))
    rb[0::2, 0] = 1
    rb[1::2, 1] = 1
    rb[0::2, 2] = -xy[:, 1]
    rb[1::2, 2] = xy[:, 0]
    rb[~mask] = 0
    assert np.max(np.abs(T @ (T.T @ rb) - rb)) < 1e-9 * np.max(np.abs(rb))


@pytest.mark.parametrize("name", ["ogrid16_bilin", "hole12_q8_pow", "ogrid16_t3"])
def test_galerkin_blocks_equal_triple_product(name, workdir):
    m, r = elastic_system(name, workdir)
    xy = np.asarray(m["node_xy"], np.float64).reshape(-1, 2)
    h = Hierarchy(r["adj_pos"], r["adj"], xy, r["mask"], min_coarse_dofs=20)
    assert len(h) >= 3
    blocks = blocks_from_csr(r)
    A = block_matrix(r["adj_pos"], r["adj"], blocks, 2)
    for lv in range(len(h) - 1):
        lev, nxt = h.level(lv), h.level(lv + 1)
        coarse = h.galerkin(lv, blocks)
        T = t_matrix(lev)
        Ac = (T.T @ A @ T).toarray()
        Ab = block_matrix(nxt["adj_pos"], nxt["adj"], coarse, 3).toarray()
        assert np.max(np.abs(Ab - Ac)) <= 1e-13 * np.max(np.abs(Ac))
        A, blocks = sp.csr_matrix(Ab), coarse


def _vcycle_levels(A0, h):
    levels = []
    A = A0
    for lv in range(len(h) - 1):
        T = t_matrix(h.level(lv))
        d = A.diagonal().copy()
        zero = d == 0
        dinv = np.where(zero, 0.0, 1.0 / np.where(zero, 1.0, d))
        # largest eigenvalue of D^-1 A by power iteration from a fixed vector
        v = np.cos(np.arange(A.shape[0]) * 0.37)
        for _ in range(60):
            w = dinv * (A @ v)
            lam = np.linalg.norm(w) / np.linalg.norm(v)
            v = w / np.linalg.norm(w)
        levels.append((A, T, 1.33 * dinv / (1.05 * lam)))
        A = (T.T @ A @ T).tocsr()
    Ad = A.toarray()
    z = np.diag(Ad) == 0
    Ad[z, z] = 1.0
    return levels, sla.cho_factor(Ad)


def _vcycle(levels, cf, b, lv=0):
    if lv == len(levels):
        return sla.cho_solve(cf, b)
    A, T, w = levels[lv]
    x = w * b
    x = x + w * (b - A @ x)
    x = x + T @ _vcycle(levels, cf, T.T @ (b - A @ x), lv + 1)
    x = x + w * (b - A @ x)
    return x + w * (b - A @ x)


def _pcg(A, b, M, tol=1e-10, cap=5000):
    x = np.zeros_like(b)
    r = b.copy()
    z = M(r)
    p = z.copy()
    rz = r @ z
    nb = np.linalg.norm(b)
    it = 0
    while np.linalg.norm(r) > tol * nb and it < cap:
        q = A @ p
        al = rz / (p @ q)
        x += al * p
        r -= al * q
        z = M(r)
        rz, rz_old = r @ z, rz
        p = z + (rz / rz_old) * p
        it += 1
    return x, it


def test_vcycle_preconditions_plate(workdir):
    """Elastic 8320-DOF plate: 8320 -> 1386 -> 168 DOF; the V-cycle (two
    damped-Jacobi sweeps around the coarse correction, Cholesky at the
    bottom) needs several times fewer CG iterations than 2x2 block-Jacobi and
    reaches the same solution."""
    m, r = config1_system(workdir)
    xy = np.asarray(m["node_xy"], np.float64).reshape(-1, 2)
    free = r["mask"].astype(bool)
    h = Hierarchy(r["adj_pos"], r["adj"], xy, r["mask"], min_coarse_dofs=400)
    assert [h.sizes(lv)[0] * h.sizes(lv)[1] for lv in range(len(h))] == [8320, 1386, 168]
    K = sp.csr_matrix((r["k_data"], r["cols"], r["rows"]), shape=(len(free), len(free)))
    Df = sp.diags(free.astype(float))
    A0 = (Df @ K @ Df + sp.diags((~free).astype(float))).tocsr()
    b = np.where(free, r["rp"], 0.0)
    levels, cf = _vcycle_levels(A0, h)
    x_mg, it_mg = _pcg(A0, b, lambda v: _vcycle(levels, cf, v))
    n = len(xy)
    inv = np.array([np.linalg.inv(A0[2 * i:2 * i + 2, 2 * i:2 * i + 2].toarray()) for i in range(n)])
    Bj = sp.bsr_matrix((inv, np.arange(n), np.arange(n + 1)), shape=(2 * n, 2 * n)).tocsr()
    x_bj, it_bj = _pcg(A0, b, lambda v: Bj @ v)
    assert it_mg * 5 < it_bj, (it_mg, it_bj)
    assert np.max(np.abs(x_mg - x_bj)) <= 1e-8 * np.max(np.abs(x_bj))


def test_invalid_inputs():
    ap = np.array([0, 1, 2], np.int32)
    xy = np.zeros((2, 2))
    mask = np.ones(4, np.uint8)
    with pytest.raises(CuplastError):
        Hierarchy(ap, np.array([1, 5], np.int32), xy, mask)  # neighbour out of range
    with pytest.raises(ValueError):
        Hierarchy(ap, np.array([1, 0], np.int32), np.zeros(2), mask)
    h = Hierarchy(ap, np.array([1, 0], np.int32), xy, mask, min_coarse_dofs=1)
    assert len(h) == 2 and h.sizes(1)[:2] == (1, 3)
    with pytest.raises(CuplastError):
        h.galerkin(1, np.zeros(9))  # the coarsest level has no next level
    with pytest.raises(ValueError):
        h.galerkin(0, np.zeros(3))


# ------------------------------------------- device-kernel emulation --


def sliced_layout(adj_pos, adj, blocks):
    """The level-0 sliced layout of the device CSR: nodes in slices of 32,
    slice s padded to the width max(deg + 1) of its nodes; block k of node
    32 s + t at slice_ptr[s] + 32 k + t; padding blocks zero with column = the
    node itself."""
    n = len(adj_pos) - 1
    deg = np.diff(adj_pos)
    ns = (n + 31) // 32
    widths = np.array([deg[32 * s:32 * s + 32].max() + 1 for s in range(ns)])
    slice_ptr = np.concatenate([[0], np.cumsum(32 * widths)]).astype(np.int32)
    val = np.zeros((slice_ptr[-1], 4))
    scol = np.zeros(slice_ptr[-1], np.int64)
    bp = np.concatenate([[0], np.cumsum(deg + 1)])
    for i in range(n):
        s, t = divmod(i, 32)
        cols = [i] + list(adj[adj_pos[i]:adj_pos[i + 1]])
        for k in range(widths[s]):
            q = slice_ptr[s] + 32 * k + t
            if k < len(cols):
                scol[q] = cols[k]
                val[q] = blocks[bp[i] + k].ravel()
            else:
                scol[q] = i
    return slice_ptr, scol, val


def masked_inv3(d):
    on = np.diag(d) != 0
    m = np.where(np.outer(on, on), d, np.eye(3))
    o = np.linalg.inv(m)
    o[~on, :] = 0
    o[:, ~on] = 0
    return o


class DeviceEmulation:
    """The kernels of the multigrid PCG, one numpy step per kernel, on the
    index arrays the device receives (Hierarchy.device_maps)."""

    def __init__(self, h, slice_ptr, scol, val, mask, omega=1.8):
        self.L = len(h)
        self.n = len(mask) // 2
        self.mask = mask.astype(bool).reshape(-1, 2)
        self.omega = omega
        # level-0 operator as the sliced kernels apply it
        ent_i, ent_j, ent_v = [], [], []
        for s in range(len(slice_ptr) - 1):
            w = (slice_ptr[s + 1] - slice_ptr[s]) // 32
            for t in range(32):
                i = 32 * s + t
                if i >= self.n:
                    continue
                for k in range(w):
                    q = slice_ptr[s] + 32 * k + t
                    ent_i.append(i)
                    ent_j.append(scol[q])
                    ent_v.append(val[q])
        ent_v = np.array(ent_v)
        rows = np.repeat(2 * np.array(ent_i), 4) + np.tile([0, 0, 1, 1], len(ent_i))
        cols = np.repeat(2 * np.array(ent_j), 4) + np.tile([0, 1, 0, 1], len(ent_j))
        self.K = sp.csr_matrix((ent_v.ravel(), (rows, cols)), shape=(2 * self.n, 2 * self.n))
        self.slice = (slice_ptr, scol, val)
        self.lev = [h.level(lv) for lv in range(self.L)]
        self.maps = [h.device_maps(lv, slice_ptr) for lv in range(self.L)]

    def setup(self):
        """diag0, galerkin, diag, coarse_inv."""
        L, n = self.L, self.n
        fm = self.mask.ravel()
        self.lam = np.zeros(L)
        d = np.zeros((n, 2, 2))
        Kd = self.K.tocsr()
        for c in range(2):
            for r in range(2):
                d[:, r, c] = Kd[r::2][:, c::2].diagonal()
        dinv = np.zeros((n, 2, 2))
        for i in range(n):
            mx, my = self.mask[i]
            if mx and my:
                dinv[i] = np.linalg.inv(d[i])
            elif mx:
                dinv[i, 0, 0] = 1 / d[i, 0, 0]
            elif my:
                dinv[i, 1, 1] = 1 / d[i, 1, 1]
        self.dinv = [sp.bsr_matrix((dinv, np.arange(n), np.arange(n + 1)), shape=(2 * n, 2 * n)).tocsr()]
        A0f = (self.dinv[0] @ self.K @ sp.diags(fm.astype(float))).tocsr()
        self.lam[0] = np.abs(A0f).sum(axis=1).max()
        self.A = [None]
        self.T = []
        fine_vals = self.slice[2]  # sliced, 4 per block
        for lv in range(L - 1):
            lev, mp = self.lev[lv], self.maps[lv]
            fb = lev["dofs"]
            nb_c = len(mp["gal_pos"]) - 1
            cval = np.zeros((nb_c, 3, 3))
            T = lev["T"]
            for c in range(nb_c):
                for q in range(mp["gal_pos"][c], mp["gal_pos"][c + 1]):
                    idx, i, j, _ = mp["gal"][q]
                    Kb = fine_vals[idx].reshape(fb, fb)
                    cval[c] += T[i].T @ Kb @ T[j]
            nxt = self.maps[lv + 1]
            rp, ci = nxt["rp"], nxt["ci"]
            n_c = len(rp) - 1
            Ac = sp.bsr_matrix((cval, ci, rp), shape=(3 * n_c, 3 * n_c)).tocsr()
            self.A.append(Ac)
            self.T.append(t_matrix(lev))
            if lv + 1 < L - 1:
                di = np.array([masked_inv3(cval[rp[a]]) for a in range(n_c)])
                Dm = sp.bsr_matrix((di, np.arange(n_c), np.arange(n_c + 1)), shape=(3 * n_c, 3 * n_c)).tocsr()
                self.dinv.append(Dm)
                self.lam[lv + 1] = np.abs(Dm @ Ac).sum(axis=1).max()
            fine_vals = cval.reshape(nb_c, 9)
        Ac = self.A[-1].toarray()
        z = np.diag(Ac) == 0
        Ac[z, z] = 1.0
        self.cinv = np.linalg.inv(Ac)

    def w(self, lv):
        return self.omega / self.lam[lv] if self.lam[lv] > 0 else 0.0

    def vcycle(self, r, y0):
        """R0..R_{L-2}, C, S_{L-2}..S1, S0 from U's y0; returns z."""
        L, fm = self.L, self.mask.ravel()
        b, y = [r], [y0]
        for lv in range(L - 1):
            A = self.K if lv == 0 else self.A[lv]
            res = b[lv] - A @ y[lv]
            if lv == 0:
                res = np.where(fm, res, 0.0)
            c = self.T[lv].T @ res
            b.append(c)
            y.append(self.w(lv + 1) * (self.dinv[lv + 1] @ c) if lv + 1 < L - 1 else None)
        e = self.cinv @ b[L - 1]
        for lv in range(L - 2, -1, -1):
            A = self.K if lv == 0 else self.A[lv]
            yp = y[lv] + self.T[lv] @ e
            s = b[lv] - A @ yp
            if lv == 0:
                s = np.where(fm, s, 0.0)
            e = yp + self.w(lv) * (self.dinv[lv] @ s)
        return e

    def solve(self, bvec, eps, cap=2000):
        fm = self.mask.ravel()
        x = np.zeros_like(bvec)
        r = np.where(fm, bvec - self.K @ x, 0.0)
        rr, bb = r @ r, bvec @ bvec
        p = [np.zeros_like(x), np.zeros_like(x)]
        y0 = self.w(0) * (self.dinv[0] @ r)
        z = self.vcycle(r, y0)
        rho, beta, it = r @ z, 0.0, 0
        parity = 0
        while not rr <= eps * eps * bb and it < cap:
            pn = z + beta * p[parity]                 # P
            q = self.K @ pn
            alpha = rho / (pn @ q)
            p[parity ^ 1] = pn
            x = x + alpha * pn                        # U
            r = r - alpha * np.where(fm, q, 0.0)
            rr = r @ r
            it += 1
            parity ^= 1
            if rr <= eps * eps * bb:
                break
            y0 = self.w(0) * (self.dinv[0] @ r)
            z = self.vcycle(r, y0)                    # R.., C, S.. (S0: rho, beta)
            rho_new = r @ z
            beta, rho = rho_new / rho, rho_new
        return x, it


def test_device_kernels_emulated(workdir):
    """The device multigrid PCG, kernel by kernel in numpy on the index arrays
    the device receives: the Galerkin blocks gathered through the sliced
    layout equal the host map's, and the solve converges to the direct
    solution in far fewer iterations than block-Jacobi PCG."""
    m, r = config1_system(workdir)
    xy = np.asarray(m["node_xy"], np.float64).reshape(-1, 2)
    free = r["mask"].astype(bool)
    blocks = blocks_from_csr(r)
    slice_ptr, scol, val = sliced_layout(r["adj_pos"], r["adj"], blocks)
    h = Hierarchy(r["adj_pos"], r["adj"], xy, r["mask"], min_coarse_dofs=150, part_nodes=256)
    assert 3 <= len(h) <= 8 and 3 * h.sizes(len(h) - 1)[0] <= 160
    # R0 runs one block per range of 256 level-0 nodes: every level-1 node of
    # range p has its members inside the range
    pp1 = h.parts(1)
    mp0 = h.device_maps(0, slice_ptr)
    assert len(pp1) - 1 == -(-len(xy) // 256)
    for p_ in range(len(pp1) - 1):
        mem = mp0["mem"][mp0["mem_pos"][pp1[p_]]:mp0["mem_pos"][pp1[p_ + 1]]]
        assert mem.min() >= 256 * p_ and mem.max() < 256 * (p_ + 1)
    em = DeviceEmulation(h, slice_ptr, scol, val, r["mask"])
    em.setup()
    # the sliced gather reproduces the host Galerkin product
    host = h.galerkin(0, blocks)
    nxt = h.device_maps(1)
    A1 = sp.bsr_matrix((host, nxt["ci"], nxt["rp"]), shape=em.A[1].shape).toarray()
    assert np.max(np.abs(A1 - em.A[1].toarray())) <= 1e-13 * np.max(np.abs(A1))
    b = np.where(free, r["rp"], 0.0)
    x, it = em.solve(b, 1e-10)
    K = sp.csr_matrix((r["k_data"], r["cols"], r["rows"]), shape=(len(free), len(free)))
    xd = np.zeros(len(free))
    xd[free] = sp.linalg.spsolve(K[free][:, free].tocsc(), b[free])
    assert np.max(np.abs(x - xd)) <= 1e-8 * np.max(np.abs(xd))
    # block-Jacobi PCG on the same system (the preconditioner of the other FP64 paths)
    fm = free.astype(float)
    A0 = (sp.diags(fm) @ em.K @ sp.diags(fm) + sp.diags(1 - fm)).tocsr()
    _, it_bj = _pcg(A0, b, lambda v: em.dinv[0] @ v + np.where(free, 0.0, v))
    assert it * 5 < it_bj, (it, it_bj)


@pytest.mark.parametrize("nodes,edges,fixed", [
    (4, [(0, 1), (1, 2), (2, 3), (3, 0), (0, 2), (1, 3)], ()),   # one 4-node element
    (5, [(0, 1), (1, 2), (2, 3), (3, 0), (0, 2), (1, 3)], ()),   # plus an isolated node
    (4, [(0, 1), (1, 2), (2, 3), (3, 0), (0, 2), (1, 3)], tuple(range(8))),  # every DOF prescribed
    (3, [(0, 1), (1, 2), (0, 2)], (0, 1)),                        # one triangle, one node fixed
])
def test_tiny_graphs_coarsen(nodes, edges, fixed):
    """The fallback the solver takes for meshes at or below the coarse size
    (min_coarse_dofs 0: coarsen while the graph shrinks) gives at least two
    levels with consistent maps, and zero prolongator rows on prescribed DOFs."""
    nb = [[] for _ in range(nodes)]
    for a, b in edges:
        nb[a].append(b)
        nb[b].append(a)
    adj_pos = np.concatenate([[0], np.cumsum([len(x) for x in nb])]).astype(np.int32)
    adj = np.array([j for x in nb for j in x] or [0], np.int32)[:adj_pos[-1]]
    xy = np.random.default_rng(nodes).uniform(size=(nodes, 2))
    mask = np.ones(2 * nodes, np.uint8)
    mask[list(fixed)] = 0
    h = Hierarchy(adj_pos, adj, xy, mask, min_coarse_dofs=0, part_nodes=256)
    assert len(h) >= 2
    lev = h.level(0)
    T = lev["T"].reshape(-1, 3)
    assert np.all(T[mask == 0] == 0)
    for lv in range(len(h) - 1):
        maps = h.device_maps(lv, np.array([0, 32 * (max(len(x) for x in nb) + 1)], np.int32))
        assert maps["mem_pos"][-1] == h.sizes(lv)[0]
        assert maps["gal_pos"][-1] == h.sizes(lv)[2]
        coarse = h.galerkin(lv, np.ones((h.sizes(lv)[2], h.sizes(lv)[1], h.sizes(lv)[1])))
        assert np.all(np.isfinite(coarse))
