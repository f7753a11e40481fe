"""A numpy model of the product's FP64 solve of a Q4 plate, used to study
how solver options change the CG iteration count without a GPU.

It restates, in plain numpy and scipy.sparse, what cp_solve does with the
benchmark's options: load levels with the level predictor, the secant
iteration with Aitken relaxation of psi (clamped to [0.1, 10], psi >= 1),
adaptive rule 2 for the linear tolerance, and 2x2 block-Jacobi PCG with the
masked residual and the stop rule ||r||^2 / ||b||^2 <= eps^2. The element
arithmetic follows the product's (and the reference's) Q4 formulas: 2x2
Gauss points, plane stress, bilinear hardening. Standard PCG stands in for
the device's Chronopoulos-Gear form; the iteration counts agree to a few per
cent with the B200's (185 / 39.3k against 187 / 40.1k on configuration 1).

``recycle = m`` models cp_solve_opts.recycle: before each linear solve the
warm start is corrected by the Galerkin projection onto the level's last m
solution increments, with the same Cholesky-with-drop small solve as the
device (csrc/recycle.cu).

This is test infrastructure: nothing in the product uses it.
"""
import numpy as np
import scipy.sparse as sp

_G = 1.0 / np.sqrt(3.0)


def _q4_grad(x, y, r, s):
    """Shape-function gradients and detJ at (r, s) for every element; local
    corners at (1, 1), (-1, 1), (-1, -1), (1, -1)."""
    j0 = 0.25 * ((1 + s) * x[:, 0] - (1 + s) * x[:, 1] - (1 - s) * x[:, 2] + (1 - s) * x[:, 3])
    j2 = 0.25 * ((1 + r) * x[:, 0] + (1 - r) * x[:, 1] - (1 - r) * x[:, 2] - (1 + r) * x[:, 3])
    j1 = 0.25 * ((1 + s) * y[:, 0] - (1 + s) * y[:, 1] - (1 - s) * y[:, 2] + (1 - s) * y[:, 3])
    j3 = 0.25 * ((1 + r) * y[:, 0] + (1 - r) * y[:, 1] - (1 - r) * y[:, 2] - (1 + r) * y[:, 3])
    det = j0 * j3 - j1 * j2
    i0, i1, i2, i3 = j3 / det, -j1 / det, -j2 / det, j0 / det
    bx = np.stack([0.25 * ((1 + s) * i0 + (1 + r) * i1), 0.25 * ((-1 - s) * i0 + (1 - r) * i1),
                   0.25 * ((-1 + s) * i0 - (1 - r) * i1), 0.25 * ((1 - s) * i0 - (1 + r) * i1)], 1)
    by = np.stack([0.25 * ((1 + s) * i2 + (1 + r) * i3), 0.25 * ((-1 - s) * i2 + (1 - r) * i3),
                   0.25 * ((-1 + s) * i2 - (1 - r) * i3), 0.25 * ((1 - s) * i2 - (1 + r) * i3)], 1)
    return bx, by, det


def chol_drop_solve(a, h, tol=1e-10):
    """(W^T K W) y = W^T r0 as the device solves it: Cholesky of the
    diagonally scaled matrix, increments with a pivot <= tol dropped (y = 0)."""
    m = len(h)
    d = np.sqrt(np.maximum(np.diag(a), 0.0))
    keep = d > 0
    dd = np.where(keep, d, 1.0)
    s = np.where(keep[:, None] & keep[None, :], a / np.outer(dd, dd), 0.0)
    low = np.zeros((m, m))
    ok = np.zeros(m, bool)
    for j in range(m):
        if not keep[j]:
            continue
        v = s[j, j] - sum(low[j, k] ** 2 for k in range(j) if ok[k])
        if not v > tol:
            continue
        low[j, j] = np.sqrt(v)
        ok[j] = True
        for i in range(j + 1, m):
            if keep[i]:
                low[i, j] = (s[i, j] - sum(low[i, k] * low[j, k] for k in range(j) if ok[k])) / low[j, j]
    z = np.zeros(m)
    for j in range(m):
        if ok[j]:
            z[j] = (h[j] / dd[j] - sum(low[j, k] * z[k] for k in range(j) if ok[k])) / low[j, j]
    y = np.zeros(m)
    for j in reversed(range(m)):
        if ok[j]:
            y[j] = (z[j] - sum(low[k, j] * y[k] for k in range(j + 1, m) if ok[k])) / low[j, j]
    return np.where(ok, y / dd, 0.0)


class PlateModel:
    """The FP64 solve of one Q4 mesh under a bilinear diagram (plane stress)."""

    def __init__(self, node_xy, elem4, rp, mask, uv, E, nu, sigma_t, k_t, h=1.0, diagram=None):
        self.xy = np.asarray(node_xy, float).reshape(-1, 2)
        self.el = np.asarray(elem4, np.int64).reshape(-1, 4)
        self.n, self.ne = self.xy.shape[0], self.el.shape[0]
        self.N = 2 * self.n
        self.E, self.nu, self.sy, self.kt, self.h = E, nu, sigma_t, k_t, h
        self.diagram = diagram  # f(eps_i) -> sigma; None: bilinear (sigma_t, k_t)
        self.rp = np.asarray(rp, float)
        self.mask = np.asarray(mask).astype(bool)
        self.uv = np.asarray(uv, float)
        x, y = self.xy[self.el, 0], self.xy[self.el, 1]
        self.gauss = []
        for r, s in ((-_G, -_G), (-_G, _G), (_G, -_G), (_G, _G)):
            bx, by, det = _q4_grad(x, y, r, s)
            b = np.zeros((self.ne, 3, 8))
            b[:, 0, 0::2] = bx
            b[:, 1, 1::2] = by
            b[:, 2, 0::2] = by
            b[:, 2, 1::2] = bx
            self.gauss.append((b, det))
        self.bmean = 0.25 * sum(b for b, _ in self.gauss)
        self.dofs = np.stack([2 * self.el, 2 * self.el + 1], 2).reshape(self.ne, 8)
        self.rows = np.repeat(self.dofs, 8, 1).ravel()
        self.cols = np.tile(self.dofs, (1, 8)).ravel()

    def _dmat(self, ec, nuc):
        c = ec / (1 - nuc * nuc)
        d = np.zeros((self.ne, 3, 3))
        d[:, 0, 0] = d[:, 1, 1] = c
        d[:, 0, 1] = d[:, 1, 0] = c * nuc
        d[:, 2, 2] = c * (1 - nuc) / 2
        return d

    def _assemble(self, ec, nuc):
        d = self._dmat(ec, nuc)
        ke = np.zeros((self.ne, 8, 8))
        for b, det in self.gauss:
            ke += np.einsum('eia,eij,ejb->eab', b, d, b) * (self.h * det)[:, None, None]
        return sp.csr_matrix((ke.ravel(), (self.rows, self.cols)), shape=(self.N, self.N))

    def _block_jacobi(self, k):
        diag = k.diagonal()
        off = np.asarray(k[np.arange(0, self.N, 2), np.arange(1, self.N, 2)]).ravel()
        a, c = diag[0::2], diag[1::2]
        mx, my = self.mask[0::2], self.mask[1::2]
        inv = np.zeros((self.n, 4))
        both = mx & my
        det = a * c - off * off
        inv[both, 0] = c[both] / det[both]
        inv[both, 1] = inv[both, 2] = -off[both] / det[both]
        inv[both, 3] = a[both] / det[both]
        ox, oy = mx & ~my, my & ~mx
        inv[ox, 0] = 1 / a[ox]
        inv[oy, 3] = 1 / c[oy]
        return inv

    def _pcg(self, k, b, x, eps, defl=None):
        """Block-Jacobi PCG; with ``defl`` (a matrix W of directions) the
        deflated variant: every search direction is made K-orthogonal to W
        (Saad, Yeung, Erhel and Guyomarc'h, 2000)."""
        inv = self._block_jacobi(k)

        def apply_m(v):
            v2 = v.reshape(self.n, 2)
            return np.stack([inv[:, 0] * v2[:, 0] + inv[:, 1] * v2[:, 1],
                             inv[:, 2] * v2[:, 0] + inv[:, 3] * v2[:, 1]], 1).ravel()

        project = None
        if defl is not None:
            kw = np.where(self.mask[:, None], k @ defl, 0.0)
            ev, vec = np.linalg.eigh(defl.T @ kw)
            keep = ev > 1e-10 * ev.max()
            ginv = (vec[:, keep] / ev[keep]) @ vec[:, keep].T

            def project(v):
                return v - defl @ (ginv @ (kw.T @ v))

        r = np.where(self.mask, b - k @ x, 0.0)
        nb = b @ b
        if r @ r == 0 or (r @ r) / nb <= eps * eps:
            return x, 0
        z = apply_m(r)
        p = project(z) if project else z.copy()
        rho = r @ z
        it = 0
        while True:
            q = np.where(self.mask, k @ p, 0.0)
            al = rho / (p @ q)
            x = x + al * p
            r = r - al * q
            it += 1
            if (r @ r) / nb <= eps * eps:
                return x, it
            z = apply_m(r)
            rn = r @ z
            p = (project(z) if project else z) + (rn / rho) * p
            rho = rn

    def _diagram(self, eps):
        if self.diagram is not None:
            return self.diagram(eps)
        et = self.sy / self.E
        return np.where(eps < et, eps * self.E, self.sy + (eps - et) * self.kt)

    def solve(self, levels=10, outer_tol=1e-6, cg_tol=1e-10, recycle=0, max_outer=2000, rule=2, deflate=False):
        """Returns (outer iterations, CG iterations, u) with the benchmark's
        options (Aitken, adaptive rule 2 or 1, level predictor, block-Jacobi).
        ``deflate`` (with ``recycle``): the linear solves also deflate the
        recycled increments (not in the product yet)."""
        E, nu = self.E, self.nu
        psi = np.ones(self.ne)
        ec, nuc = E / psi, 0.5 * (1 - (1 - 2 * nu) / psi)
        u = np.zeros(self.N)
        u_prev = psi_prev = None
        tot_cg = tot_outer = 0
        for lev in range(1, levels + 1):
            lam = lev / levels
            if lev >= 2:  # level predictor
                c, cpsi = u.copy(), psi.copy()
                if lev >= 3:
                    u = np.where(self.mask, 2 * c - u_prev, c)
                    psi = 2 * cpsi - psi_prev
                    psi[~(psi >= 1.0)] = 1.0
                    ec, nuc = E / psi, 0.5 * (1 - (1 - 2 * nu) / psi)
                u_prev, psi_prev = c, cpsi
            b = lam * self.rp
            u = np.where(self.mask, u, lam * self.uv)
            res_prev = np.zeros(self.ne)
            rel, w_prev = 1.0, 1.0
            incs = []
            for it in range(max_outer):
                if rule == 2:
                    eps = max(cg_tol, 0.2 * rel) if rel > outer_tol else cg_tol
                else:
                    eps = max(cg_tol, 1e-2 * rel) if rel > 10 * outer_tol else cg_tol
                k = self._assemble(ec, nuc)
                x0, w = u, None
                if recycle and incs:
                    w = np.stack(incs[::-1][:recycle], 1)  # newest first
                    r0 = np.where(self.mask, b - k @ u, 0.0)
                    y = chol_drop_solve(w.T @ (k @ w), w.T @ r0)
                    x0 = u + w @ y
                u_new, ncg = self._pcg(k, b, x0, eps, defl=w if deflate else None)
                incs.append(u_new - u)
                u = u_new
                tot_cg += ncg
                tot_outer += 1
                st = np.einsum('eia,ea->ei', self.bmean, u[self.dofs])
                sig = np.einsum('eij,ej->ei', self._dmat(ec, nuc), st)
                sx, sy_, t = sig[:, 0], sig[:, 1], sig[:, 2]
                si = np.sqrt(0.5 * (sx * sx + sy_ * sy_ + (sx - sy_) ** 2 + 6 * t * t))
                tab = self._diagram(si / ec)
                ps = E * (si / ec) / tab
                rel = np.sqrt(((si - tab) ** 2).sum() / (tab ** 2).sum())
                r = np.where(ps == ps, ps - psi, 0.0)
                dr = r - res_prev
                an, ad = (res_prev * dr).sum(), (dr * dr).sum()
                wgt = -w_prev * an / ad if it > 0 and ad > 0 else 1.0
                wgt = min(max(wgt, 0.1), 10.0)
                psi = psi + wgt * r
                psi[~(psi >= 1.0)] = 1.0
                ec, nuc = E / psi, 0.5 * (1 - (1 - 2 * nu) / psi)
                res_prev, w_prev = r, wgt
                if rel <= outer_tol and eps <= cg_tol:
                    break
        return tot_outer, tot_cg, u
