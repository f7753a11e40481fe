"""cudaplasticity_b200 -- Python front end of the B200 (sm_100a) implementation
of CudaPlasticity's 2D elasto-plastic FEM hot path.

Everything here calls the C ABI of the in-tree library libcuplast.so
(include/cuplast.h, include/cuplast_host.h); the work itself runs in the
library's CUDA kernels. Importing works without a GPU (mesh generation and
load building are host code); device calls raise CuplastError when no CUDA
device is present.
"""
import atexit
import ctypes
import os
import weakref

import numpy as np

from . import _capi as C
from ._capi import (CP_DIAGRAM_ELASTIC, CP_DIAGRAM_HOLLOMON, CP_DIAGRAM_LINEAR, CP_DIAGRAM_PIECEWISE,  # noqa: F401
                    CP_DIAGRAM_POWER, CP_PLANE_STRAIN, CP_PLANE_STRESS, CP_PREC_FLOAT_BOOST, CP_PREC_FP64, CP_PREC_MIXED)

FIELDS = ["exx", "eyy", "gamma", "eps_i", "sxx", "syy", "tau", "sig_i", "table_s", "psi", "E_c", "nu_c",
          "exx_p", "eyy_p", "gamma_p", "eps_p_i"]


class CuplastError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        text = C.lib().cp_status_string(status).decode()
        super().__init__(f"{text} ({status})" + (f": {msg}" if msg else ""))


def _dp(a):
    return a.ctypes.data_as(C.P_double)


def _ip(a):
    return a.ctypes.data_as(C.P_int)


def _up(a):
    return a.ctypes.data_as(C.P_ubyte)


def version():
    return C.lib().cp_version().decode()


def device_count():
    n = ctypes.c_int(0)
    C.lib().cp_device_count(ctypes.byref(n))
    return n.value


# ------------------------------------------------------------------ material --

def material(E, nu=0.3, h=1.0, rho=1.0, plane=CP_PLANE_STRESS, diagram="elastic", **kw):
    """cp_material. diagram: 'elastic'; 'linear' (sigma_t, k_t); 'power'
    (sigma_t, a, m); 'hollomon' (sigma_y, eps0, n); 'piecewise' (points:
    [(eps, sigma), ...], elastic up to the first point)."""
    m = C.cp_material()
    m.E, m.nu, m.h, m.rho, m.plane = float(E), float(nu), float(h), float(rho), int(plane)
    kind = {"elastic": CP_DIAGRAM_ELASTIC, "linear": CP_DIAGRAM_LINEAR, "power": CP_DIAGRAM_POWER,
            "hollomon": CP_DIAGRAM_HOLLOMON, "piecewise": CP_DIAGRAM_PIECEWISE}[diagram]
    m.diagram = kind
    if kind == CP_DIAGRAM_LINEAR:
        m.sigma_t, m.k_t = kw["sigma_t"], kw["k_t"]
    elif kind == CP_DIAGRAM_POWER:
        m.sigma_t, m.a, m.m = kw["sigma_t"], kw["a"], kw["m"]
    elif kind == CP_DIAGRAM_HOLLOMON:
        m.sigma_t, m.eps0, m.n = kw["sigma_y"], kw["eps0"], kw["n"]
    elif kind == CP_DIAGRAM_PIECEWISE:
        pts = kw["points"]
        m.n_points = len(pts)
        for i, (e, s) in enumerate(pts):
            m.pw_eps[i], m.pw_sig[i] = e, s
        m.sigma_t = pts[0][1]
    return m


# ---------------------------------------------------------------------- mesh --

class Mesh:
    """Host mesh (the drop-in Mesh class) with the reference's generators."""

    def __init__(self):
        self._h = C.c_p()
        self._check(C.lib().cpx_mesh_create(ctypes.byref(self._h)))

    def __del__(self):
        if getattr(self, "_h", None):
            C.lib().cpx_mesh_destroy(self._h)
            self._h = None

    @staticmethod
    def _check(st):
        if st != C.CP_OK:
            raise CuplastError(st)

    @classmethod
    def rect(cls, x1, x2, y1, y2, n1, n2, order=1):
        m = cls()
        m._check(C.lib().cpx_mesh_gen_rect(m._h, x1, x2, y1, y2, n1, n2, order))
        return m

    @classmethod
    def rect_with_hole(cls, x1, x2, y1, y2, hole_rad, n1, n2, rad_n=0, order=1):
        m = cls()
        m._check(C.lib().cpx_mesh_gen_rect_with_hole(m._h, x1, x2, y1, y2, hole_rad, n1, n2, rad_n, order))
        return m

    @classmethod
    def ring(cls, a, b, n_phi, n_r, order=1):
        m = cls()
        m._check(C.lib().cpx_mesh_gen_ring(m._h, a, b, n_phi, n_r, order))
        return m

    @classmethod
    def load(cls, path):
        """Mesh::loadFromFile: an .inp file (nodes, S3/S4 elements, *MPC borders)."""
        m = cls()
        m._check(C.lib().cpx_mesh_load_inp(m._h, os.fspath(path).encode()))
        return m

    @classmethod
    def from_arrays(cls, node_xy, elem3=None, elem4=None, borders=(), elem8=None):
        m = cls()
        xy = np.ascontiguousarray(node_xy, dtype=np.float64).ravel()
        e3 = np.ascontiguousarray(elem3 if elem3 is not None else np.zeros(0), dtype=np.int32).ravel()
        e4 = np.ascontiguousarray(elem4 if elem4 is not None else np.zeros(0), dtype=np.int32).ravel()
        e8 = np.ascontiguousarray(elem8 if elem8 is not None else np.zeros(0), dtype=np.int32).ravel()
        bl = np.array([len(b) for b in borders], dtype=np.int32)
        bn = np.ascontiguousarray(np.concatenate([np.asarray(b, np.int32) for b in borders]) if len(borders)
                                  else np.zeros(1, np.int32), dtype=np.int32)
        m._check(C.lib().cpx_mesh_set(m._h, xy.size // 2, _dp(xy), e3.size // 3, _ip(e3), e4.size // 4, _ip(e4),
                                      len(borders), _ip(bl) if len(bl) else None, _ip(bn), e8.size // 8,
                                      _ip(e8) if e8.size else None))
        return m

    def renum_by_direction(self, dx=1.0, dy=1.0):
        """Mesh::renumByDirection: nodes renumbered by projection on (dx, dy)."""
        self._check(C.lib().cpx_mesh_renum_by_direction(self._h, dx, dy))
        return self

    def smooth_ring(self, border_n):
        self._check(C.lib().cpx_mesh_smooth_ring(self._h, border_n))
        return self

    def quality(self):
        """aspect ratio and skew-angle sine per 4-node element, mean element area."""
        c4 = self.counts()[2]
        asp, skw, avr = np.zeros(max(c4, 1)), np.zeros(max(c4, 1)), ctypes.c_double()
        self._check(C.lib().cpx_mesh_quality(self._h, _dp(asp), _dp(skw), ctypes.byref(avr)))
        return dict(aspect=asp[:c4], skew_sin=skw[:c4], avr_elem_size=avr.value)

    def split_t3(self):
        self._check(C.lib().cpx_mesh_split_t3(self._h))
        return self

    def counts(self):
        """(nodes, triangles, quads, borders, border nodes in total)."""
        v = [ctypes.c_int() for _ in range(6)]
        self._check(C.lib().cpx_mesh_counts(self._h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v[:5])

    def count8(self):
        """8-node elements (meshes generated with order=2 or read from S8R blocks)."""
        v = ctypes.c_int()
        self._check(C.lib().cpx_mesh_counts(self._h, None, None, None, None, None, ctypes.byref(v)))
        return v.value

    def arrays(self):
        n, c3, c4, nb, bt = self.counts()
        c8 = self.count8()
        xy = np.zeros(2 * n)
        e3 = np.zeros(max(3 * c3, 1), np.int32)
        e4 = np.zeros(max(4 * c4, 1), np.int32)
        e8 = np.zeros(max(8 * c8, 1), np.int32)
        bl = np.zeros(max(nb, 1), np.int32)
        bn = np.zeros(max(bt, 1), np.int32)
        self._check(C.lib().cpx_mesh_get(self._h, _dp(xy), _ip(e3), _ip(e4), _ip(bl), _ip(bn), _ip(e8)))
        borders, off = [], 0
        for L in bl[:nb]:
            borders.append(bn[off:off + L].copy())
            off += L
        out = dict(node_xy=xy.reshape(-1, 2), elem3=e3[:3 * c3].reshape(-1, 3), elem4=e4[:4 * c4].reshape(-1, 4),
                   borders=borders)
        if c8:
            out["elem8"] = e8[:8 * c8].reshape(-1, 8)
        return out

    def max_index_diff(self):
        v = ctypes.c_int()
        self._check(C.lib().cpx_mesh_max_index_diff(self._h, ctypes.byref(v)))
        return v.value


class Loads:
    """LoadConditions of the drop-in API (constant-valued loads)."""

    def __init__(self):
        self._h = C.c_p()
        Mesh._check(C.lib().cpx_loads_create(ctypes.byref(self._h)))

    def __del__(self):
        if getattr(self, "_h", None):
            C.lib().cpx_loads_destroy(self._h)
            self._h = None

    def _do(self, name, *args):
        Mesh._check(getattr(C.lib(), name)(self._h, *args))
        return self

    def set_force(self, border, fx, fy, normal=False):
        return self._do("cpx_loads_set_force", border, fx, fy, int(normal))

    def set_displacement(self, border, ux, uy, fix_mid_x=False, fix_mid_y=False):
        return self._do("cpx_loads_set_displacement", border, ux, uy, int(fix_mid_x), int(fix_mid_y))

    def fix_border(self, b):
        return self._do("cpx_loads_fix_border", b)

    def fix_border_vert(self, b):
        return self._do("cpx_loads_fix_border_vert", b)

    def fix_border_hor(self, b):
        return self._do("cpx_loads_fix_border_hor", b)

    def fix_vert_axis(self, x):
        return self._do("cpx_loads_fix_vert_axis", x)

    def fix_hor_axis(self, y):
        return self._do("cpx_loads_fix_hor_axis", y)

    def fix_point(self, x, y):
        return self._do("cpx_loads_fix_point", x, y)

    def set_displ_point(self, x, y, ux, uy):
        return self._do("cpx_loads_set_displ_point", x, y, ux, uy)

    def set_force_point(self, x, y, fx, fy):
        return self._do("cpx_loads_set_force_point", x, y, fx, fy)

    def set_gravity(self, g=9.81, dx=0.0, dy=-1.0):
        return self._do("cpx_loads_set_gravity", g, dx, dy)

    def set_rotation(self, omega, ax=0.0, ay=0.0):
        return self._do("cpx_loads_set_rotation", omega, ax, ay)

    def fix_dof(self, dof):
        return self._do("cpx_loads_fix_dof", int(dof))

    def build(self, mesh, h=1.0, rho=1.0):
        n = mesh.counts()[0]
        rp, uv, mask = np.zeros(2 * n), np.zeros(2 * n), np.zeros(2 * n, np.uint8)
        Mesh._check(C.lib().cpx_loads_build(mesh._h, self._h, h, rho, _dp(rp), _up(mask), _dp(uv)))
        return rp, mask, uv


# ------------------------------------------------------------------- device --

class Context:
    """cp_context. Instances and batches made on it are closed with it
    (batches first), so no handle outlives its context."""

    def __init__(self, device=0):
        self._h = C.c_p()
        self._deps = weakref.WeakSet()
        st = C.lib().cp_context_create(device, ctypes.byref(self._h))
        if st != C.CP_OK:
            self._h = None
            raise CuplastError(st)

    def close(self):
        if getattr(self, "_h", None):
            deps = list(getattr(self, "_deps", ()))
            for d in deps:
                if isinstance(d, Batch):
                    d.close()
            for d in deps:
                if not isinstance(d, Batch):
                    d.close()
            C.lib().cp_context_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def error(self):
        return C.lib().cp_context_last_error(self._h).decode()

    def check(self, st):
        if st != C.CP_OK:
            raise CuplastError(st, self.error())
        return st


def mesh_view(arrays):
    """cp_mesh_view over numpy arrays (kept alive by the returned tuple)."""
    xy = np.ascontiguousarray(arrays["node_xy"], dtype=np.float64).ravel()
    e3 = np.ascontiguousarray(arrays.get("elem3", np.zeros(0)), dtype=np.int32).ravel()
    e4 = np.ascontiguousarray(arrays.get("elem4", np.zeros(0)), dtype=np.int32).ravel()
    e8 = np.ascontiguousarray(arrays.get("elem8", np.zeros(0)), dtype=np.int32).ravel()
    v = C.cp_mesh_view(xy.size // 2, _dp(xy), e3.size // 3, _ip(e3) if e3.size else None, e4.size // 4,
                       _ip(e4) if e4.size else None, e8.size // 8, _ip(e8) if e8.size else None)
    return v, (xy, e3, e4, e8)


def solve_opts(**kw):
    o = C.cp_solve_opts()
    C.lib().cp_solve_opts_default(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Instance:
    """One problem on the device (cp_instance)."""

    def __init__(self, ctx, mesh_arrays, mat):
        self.ctx = ctx
        self._h = C.c_p()
        v, keep = mesh_view(mesh_arrays)
        self.n_nodes = v.node_count
        self.n_elem = v.count3 + v.count4 + v.count8
        self.count3 = v.count3
        self.count4 = v.count4
        self.count8 = v.count8
        ctx.check(C.lib().cp_instance_create(ctx._h, ctypes.byref(v), ctypes.byref(mat), ctypes.byref(self._h)))
        ctx._deps.add(self)
        del keep

    def close(self):
        if getattr(self, "_h", None):
            C.lib().cp_instance_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def sizes(self):
        a, b, c, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong()
        self.ctx.check(C.lib().cp_instance_sizes(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                                 ctypes.byref(d)))
        return a.value, b.value, c.value, d.value

    def set_loads(self, rp, mask, uv=None):
        rp = np.ascontiguousarray(rp, np.float64)
        mask = np.ascontiguousarray(mask, np.uint8)
        uvp = None
        if uv is not None:
            uv = np.ascontiguousarray(uv, np.float64)
            uvp = _dp(uv)
        self.ctx.check(C.lib().cp_instance_set_loads(self._h, _dp(rp), _up(mask), uvp))

    def set_level(self, lam):
        self.ctx.check(C.lib().cp_instance_set_level(self._h, float(lam)))

    def reset_state(self):
        self.ctx.check(C.lib().cp_instance_reset_state(self._h))

    def assemble(self, precision=CP_PREC_FP64):
        self.ctx.check(C.lib().cp_assemble(self._h, precision))

    def cg_solve(self, eps, max_iter=10_000_000):
        it, rr = ctypes.c_longlong(), ctypes.c_double()
        st = C.lib().cp_cg_solve(self._h, eps, max_iter, ctypes.byref(it), ctypes.byref(rr))
        if st not in (C.CP_OK,):
            raise CuplastError(st, self.ctx.error())
        return it.value, rr.value

    def secant_update(self):
        r = ctypes.c_double()
        self.ctx.check(C.lib().cp_secant_update(self._h, ctypes.byref(r)))
        return r.value

    def plastic_strains(self):
        self.ctx.check(C.lib().cp_plastic_strains(self._h))

    def solve(self, allow_not_converged=False, **kw):
        o = solve_opts(**kw)
        rep = C.cp_solve_report()
        st = C.lib().cp_solve(self._h, ctypes.byref(o), ctypes.byref(rep))
        if st != C.CP_OK and not (allow_not_converged and st == C.CP_ERR_NOT_CONVERGED):
            raise CuplastError(st, self.ctx.error())
        return {k: getattr(rep, k) for k, _ in C.cp_solve_report._fields_}

    def csr(self):
        n, ne, nnz, nadj = self.sizes()
        rows, cols = np.zeros(2 * n + 1, np.int32), np.zeros(nnz, np.int32)
        adj_pos, adj = np.zeros(n + 1, np.int32), np.zeros(max(nadj, 1), np.int32)
        vals = np.zeros(nnz)
        self.ctx.check(C.lib().cp_get_csr(self._h, _ip(rows), _ip(cols), _ip(adj_pos), _ip(adj), _dp(vals)))
        return dict(rows=rows, cols=cols, adj_pos=adj_pos, adj=adj[:nadj], k_data=vals)

    def slot_map(self):
        ns = 9 * self.count3 + 16 * self.count4 + 64 * self.count8
        s = np.zeros(max(ns, 1), np.int32)
        self.ctx.check(C.lib().cp_get_slot_map(self._h, _ip(s)))
        return s[:ns]

    def field(self, name):
        n = 2 * self.n_nodes if name in ("uv", "rp") else self.n_elem
        out = np.zeros(n)
        self.ctx.check(C.lib().cp_get_field(self._h, name.encode(), _dp(out)))
        return out

    def set_field(self, name, values):
        v = np.ascontiguousarray(values, np.float64)
        self.ctx.check(C.lib().cp_set_field(self._h, name.encode(), _dp(v)))

    def state(self):
        d = {k: self.field(k) for k in FIELDS}
        d["uv"] = self.field("uv")
        return d


def _report(rep):
    return {k: getattr(rep, k) for k, _ in C.cp_solve_report._fields_}


class Batch:
    """Many instances solved together in mixed precision (cp_batch): one CUDA
    graph advances every instance's own state machine; instances join between
    runs and are harvested when done."""

    def __init__(self, ctx, **opts):
        self.ctx = ctx
        o = C.cp_batch_opts()
        C.lib().cp_batch_opts_default(ctypes.byref(o))
        for k, v in opts.items():
            setattr(o, k, v)
        self.opts = o
        self._h = C.c_p()
        ctx.check(C.lib().cp_batch_create(ctx._h, ctypes.byref(o), ctypes.byref(self._h)))
        ctx._deps.add(self)
        self._slots = {}

    def close(self):
        if getattr(self, "_h", None):
            C.lib().cp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def add(self, inst, **solve_kw):
        """Adds an Instance (loads set) with cp_solve options; mixed precision."""
        kw = dict(solve_kw)
        kw["precision"] = CP_PREC_MIXED
        o = solve_opts(**kw)
        slot = ctypes.c_int(-1)
        self.ctx.check(C.lib().cp_batch_add(self._h, inst._h, ctypes.byref(o), ctypes.byref(slot)))
        self._slots[slot.value] = inst
        return slot.value

    def launch(self, any_done=False, max_trips=0):
        until = C.CP_BATCH_RUN_ANY_DONE if any_done else C.CP_BATCH_RUN_ALL
        self.ctx.check(C.lib().cp_batch_launch(self._h, until, int(max_trips)))

    def wait(self):
        a, d = ctypes.c_int(), ctypes.c_int()
        self.ctx.check(C.lib().cp_batch_wait(self._h, ctypes.byref(a), ctypes.byref(d)))
        return a.value, d.value

    def interrupt(self):
        self.ctx.check(C.lib().cp_batch_interrupt(self._h))

    def run(self, any_done=False, max_trips=0):
        self.launch(any_done, max_trips)
        return self.wait()

    def harvest(self):
        """[(slot, Instance, report dict)] of the finished instances."""
        cap = max(len(self._slots), 1)
        slots = np.zeros(cap, np.int32)
        hs = (C.c_p * cap)()
        reps = (C.cp_solve_report * cap)()
        n = ctypes.c_int()
        self.ctx.check(C.lib().cp_batch_harvest(self._h, cap, _ip(slots), hs, reps, ctypes.byref(n)))
        out = []
        for i in range(n.value):
            inst = self._slots.pop(int(slots[i]))
            out.append((int(slots[i]), inst, _report(reps[i])))
        return out

    def progress(self, slot):
        """(phase, level, report dict) of the instance in slot, as of the last run."""
        ph, lv = ctypes.c_int(), ctypes.c_int()
        rep = C.cp_solve_report()
        self.ctx.check(C.lib().cp_batch_progress(self._h, slot, ctypes.byref(ph), ctypes.byref(lv), ctypes.byref(rep)))
        return ph.value, lv.value, _report(rep)

    def autotune(self):
        ms = ctypes.c_double()
        self.ctx.check(C.lib().cp_batch_autotune(self._h, ctypes.byref(ms)))
        return ms.value

    def tile(self, bucket):
        v = ctypes.c_int()
        self.ctx.check(C.lib().cp_batch_get_tile(self._h, bucket, ctypes.byref(v)))
        return v.value

    def set_tile(self, bucket, slices):
        self.ctx.check(C.lib().cp_batch_set_tile(self._h, bucket, slices))

    def last_run_ms(self):
        """Device time of the last run (CUDA events on the batch's stream)."""
        v = ctypes.c_double()
        self.ctx.check(C.lib().cp_batch_last_run_ms(self._h, ctypes.byref(v)))
        return v.value

    def stats(self):
        t, k, r = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        self.ctx.check(C.lib().cp_batch_stats(self._h, ctypes.byref(t), ctypes.byref(k), ctypes.byref(r)))
        return dict(trips=t.value, kernel_launches=k.value, runs=r.value)


class _Handed(Instance):
    """An instance created by the library (a server result). It lives on the
    server's streams: it is freed before the server (Server.close frees the
    ones still open)."""

    def __init__(self, server, handle, n_nodes, n_elem, count3, count4, count8=0):
        self.ctx = _HandedContext(server.ctx, handle)
        self._server = server
        self._h = handle
        self.n_nodes, self.n_elem, self.count3, self.count4, self.count8 = n_nodes, n_elem, count3, count4, count8


class _HandedContext:
    """Error reporting for a handed-back instance: its messages live on the
    service's context that the instance belongs to."""

    def __init__(self, ctx, handle):
        self._ctx, self._ih = ctx, handle

    def error(self):
        return C.lib().cp_instance_last_error(self._ih).decode()

    def check(self, st):
        if st != C.CP_OK:
            raise CuplastError(st, self.error())


_LIVE_SERVERS = weakref.WeakSet()


@atexit.register
def _close_servers():
    for srv in list(_LIVE_SERVERS):
        srv.close()


class Server:
    """Solve service (cp_server): requests are submitted as they arrive and
    solved on one GPU, mixed-precision ones with continuous batching, FP64
    ones concurrently on fp64_lanes lanes; wait() hands back each request's
    results."""

    def __init__(self, device=0, hbm_reserve=0.05, max_bytes=0, max_inflight=1024, trip_quantum=0, fp64_lanes=8,
                 **batch):
        o = C.cp_server_opts()
        C.lib().cp_server_opts_default(ctypes.byref(o))
        o.device, o.hbm_reserve, o.max_bytes = device, hbm_reserve, int(max_bytes)
        o.max_inflight, o.trip_quantum = max_inflight, int(trip_quantum)
        o.fp64_lanes = fp64_lanes
        for k, v in batch.items():
            setattr(o.batch, k, v)
        self._h = C.c_p()
        st = C.lib().cp_server_create(ctypes.byref(o), ctypes.byref(self._h))
        if st != C.CP_OK:
            self._h = None
            raise CuplastError(st)
        self.ctx = Context(device)  # for error strings
        self._meta = {}
        self._handed = weakref.WeakSet()
        _LIVE_SERVERS.add(self)

    def close(self):
        if getattr(self, "_h", None):
            for inst in list(self._handed):
                inst.close()
            C.lib().cp_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def submit(self, mesh_arrays, mat, rp, mask, uv=None, **solve_kw):
        """cp_solve options as keywords; precision defaults to CP_PREC_MIXED
        (the batch), CP_PREC_FP64 / CP_PREC_FLOAT_BOOST go to the lanes."""
        v, keep = mesh_view(mesh_arrays)
        rp = np.ascontiguousarray(rp, np.float64)
        mask = np.ascontiguousarray(mask, np.uint8)
        uvp = None
        if uv is not None:
            uv = np.ascontiguousarray(uv, np.float64)
            uvp = _dp(uv)
        kw = dict(solve_kw)
        kw.setdefault("precision", CP_PREC_MIXED)
        o = solve_opts(**kw)
        rid = ctypes.c_longlong()
        st = C.lib().cp_server_submit(self._h, ctypes.byref(v), ctypes.byref(mat), _dp(rp), _up(mask), uvp,
                                      ctypes.byref(o), ctypes.byref(rid))
        if st != C.CP_OK:
            raise CuplastError(st)
        self._meta[rid.value] = (v.node_count, v.count3 + v.count4 + v.count8, v.count3, v.count4, v.count8)
        del keep
        return rid.value

    def wait(self, rid, timeout=-1.0):
        """(Instance with the results, report dict, latency seconds)."""
        h = C.c_p()
        rep = C.cp_solve_report()
        lat = ctypes.c_double()
        st = C.lib().cp_server_wait(self._h, rid, float(timeout), ctypes.byref(h), ctypes.byref(rep),
                                    ctypes.byref(lat))
        if st != C.CP_OK:
            raise CuplastError(st)
        meta = self._meta.pop(rid)
        inst = _Handed(self, h, *meta)
        self._handed.add(inst)
        return inst, _report(rep), lat.value

    def stats(self):
        s = C.cp_server_stats()
        st = C.lib().cp_server_get_stats(self._h, ctypes.byref(s))
        if st != C.CP_OK:
            raise CuplastError(st)
        return {k: getattr(s, k) for k, _ in C.cp_server_stats._fields_}


class Hierarchy:
    """Aggregation multigrid hierarchy of a node graph (cpx_amg_build): level 0
    has 2 DOFs per node, every coarser level 3 per aggregate (its rigid-body
    modes). ``adj_pos`` / ``adj`` are the graph without the nodes themselves
    (``Instance.csr()``'s), ``mask`` 1 per free DOF; ``part_nodes`` > 0 cuts
    level 0 into node ranges that no level-0 aggregate crosses."""

    def __init__(self, adj_pos, adj, xy, mask, min_coarse_dofs=400, part_nodes=0):
        ap = np.ascontiguousarray(adj_pos, np.int32)
        aj = np.ascontiguousarray(adj, np.int32)
        if aj.size == 0:
            aj = np.zeros(1, np.int32)
        xy = np.ascontiguousarray(np.asarray(xy, np.float64).ravel())
        mk = np.ascontiguousarray(mask, np.uint8)
        n = ap.size - 1
        if xy.size != 2 * n or mk.size != 2 * n:
            raise ValueError("xy and mask need 2 values per node")
        self._h = C.c_p()
        Mesh._check(C.lib().cpx_amg_build(n, _ip(ap), _ip(aj), _dp(xy), _up(mk), min_coarse_dofs, part_nodes,
                                          ctypes.byref(self._h)))

    def __del__(self):
        if getattr(self, "_h", None):
            C.lib().cpx_amg_destroy(self._h)
            self._h = None

    def __len__(self):
        n = ctypes.c_int()
        Mesh._check(C.lib().cpx_amg_levels(self._h, ctypes.byref(n)))
        return n.value

    def sizes(self, level):
        """(nodes, DOFs per node, blocks, aggregates of the next level)."""
        out = [ctypes.c_int() for _ in range(4)]
        Mesh._check(C.lib().cpx_amg_level_sizes(self._h, level, *(ctypes.byref(x) for x in out)))
        return tuple(x.value for x in out)

    def parts(self, level):
        """Partition bounds of a level (n_parts + 1 node indices)."""
        np_ = ctypes.c_int()
        Mesh._check(C.lib().cpx_amg_level_parts(self._h, level, ctypes.byref(np_), None))
        out = np.zeros(np_.value + 1, np.int32)
        Mesh._check(C.lib().cpx_amg_level_parts(self._h, level, None, _ip(out)))
        return out

    def level(self, level):
        """Graph, aggregates and prolongator blocks (nodes x dofs x 3) of a level."""
        n, fb, nb, na = self.sizes(level)
        ap, aj = np.zeros(n + 1, np.int32), np.zeros(max(nb - n, 1), np.int32)
        agg, T = np.zeros(max(n, 1), np.int32), np.zeros(max(n * fb * 3, 1))
        last = na == 0
        Mesh._check(C.lib().cpx_amg_level_get(self._h, level, _ip(ap), _ip(aj), None if last else _ip(agg),
                                              None if last else _dp(T)))
        out = dict(nodes=n, dofs=fb, blocks=nb, aggregates=na, adj_pos=ap, adj=aj[:nb - n])
        if not last:
            out.update(agg=agg[:n], T=T[:n * fb * 3].reshape(n, fb, 3))
        return out

    def device_maps(self, level, slice_ptr=None):
        """Index arrays of the device kernels of a level (cpx_amg_device_maps):
        rp, ci, mem_pos, mem, gal_pos and gal (entries x 4)."""
        sp_ = None if slice_ptr is None else np.ascontiguousarray(slice_ptr, np.int32)
        counts = np.zeros(6, np.int32)
        spp = None if sp_ is None else _ip(sp_)
        Mesh._check(C.lib().cpx_amg_device_maps(self._h, level, spp, _ip(counts), *([None] * 6)))
        bufs = [np.zeros(max(int(c), 1), np.int32) for c in counts]
        Mesh._check(C.lib().cpx_amg_device_maps(self._h, level, spp, _ip(counts), *(_ip(b) for b in bufs)))
        names = ["rp", "ci", "mem_pos", "mem", "gal_pos", "gal"]
        out = {k: b[:int(c)] for k, b, c in zip(names, bufs, counts)}
        out["gal"] = out["gal"].reshape(-1, 4)
        return out

    def galerkin(self, level, fine_blocks):
        """Blocks of level + 1's operator from level's (blocks x dofs x dofs)."""
        n, fb, nb, na = self.sizes(level)
        f = np.ascontiguousarray(fine_blocks, np.float64).reshape(-1)
        if f.size != nb * fb * fb:
            raise ValueError(f"expected {nb} blocks of {fb}x{fb}")
        cb = self.sizes(level + 1)[2]
        out = np.zeros(9 * cb)
        Mesh._check(C.lib().cpx_amg_galerkin(self._h, level, _dp(f), _dp(out)))
        return out.reshape(cb, 3, 3)


def footprint(mesh_arrays, precision=CP_PREC_FP64):
    v, keep = mesh_view(mesh_arrays)
    out = ctypes.c_size_t()
    st = C.lib().cp_instance_footprint(ctypes.byref(v), precision, ctypes.byref(out))
    if st != C.CP_OK:
        raise CuplastError(st)
    return out.value
