"""Oracle package: the checkers the CUDA product is tested against.

TEST INFRASTRUCTURE ONLY. Importable by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, and nowhere else; the product never calls it.

* ``run_oracle(job, out)`` runs the C restatement (liboracle.so, built from
  cuplast_oracle.c) on a job description;
* ``run_reference(job, out)`` runs the reference implementation's own CPU path
  through the harness in ref_harness.cu (``_ref/cpref``, built from the
  reference sources; present only where they were available at build time).

A job is a list of lines in the harness syntax (see ref_harness.cu).
"""
import ctypes
import os
import subprocess
import tempfile

from . import cpbin

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "cpref")
# the same harness with the reference's Mesh.cu built at -O0, for its .inp
# loader (see the Makefile)
REF_BIN_INP = os.path.join(HERE, "_ref", "cpref_inp")
# the harness built with the solver's source for its phases_csr mode (the
# reference's element arithmetic added straight into CSR: meshes whose band
# matrix does not fit)
REF_BIN_CSR = os.path.join(HERE, "_ref", "cpref_csr")

_lib = None


def build(with_reference=None, ref_dir=None):
    """Builds liboracle.so, and _ref/cpref when the reference sources exist
    (ref_dir, else the CUPLAST_REFERENCE environment variable)."""
    ref_dir = ref_dir or os.environ.get("CUPLAST_REFERENCE", "")
    if with_reference is None:
        with_reference = bool(ref_dir) and os.path.isdir(os.path.join(ref_dir, "src"))
    targets = ["oracle"] + (["ref"] if with_reference else [])
    subprocess.run(["make", "-s", "-C", HERE, f"REF={ref_dir}"] + targets, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(with_reference=False)
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.orc_run_job.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        _lib.orc_run_job.restype = ctypes.c_int
    return _lib


def have_reference():
    return os.path.exists(REF_BIN)


def _write_job(lines, path):
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def run_oracle(lines, workdir=None):
    """Runs the C restatement; returns the output records as a dict."""
    with tempfile.TemporaryDirectory(dir=workdir) as d:
        job, out = os.path.join(d, "job.txt"), os.path.join(d, "out.bin")
        _write_job(lines, job)
        rc = lib().orc_run_job(job.encode(), out.encode())
        if rc != 0:
            raise RuntimeError(f"oracle job failed with code {rc}")
        return cpbin.read(out)


def run_reference(lines, threads=None, workdir=None, binary=None):
    """Runs the reference's CPU path through the harness (no GPU is used:
    the child sees no CUDA device, so the reference selects its CPU path)."""
    if not have_reference():
        raise FileNotFoundError("reference harness not built (oracle/_ref/cpref)")
    env = dict(os.environ)
    env["CUDA_VISIBLE_DEVICES"] = ""
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory(dir=workdir) as d:
        job, out = os.path.join(d, "job.txt"), os.path.join(d, "out.bin")
        _write_job(lines, job)
        subprocess.run([binary or REF_BIN, job, out], check=True, env=env, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL)
        return cpbin.read(out)


def write_mesh(path, node_xy, elem3=(), elem4=(), borders=(), elem8=()):
    """Writes a mesh in the layout the harness and the restatement read. The
    mid-side nodes of 8-node elements are the mesh's second-order nodes."""
    import numpy as np

    bl = [len(b) for b in borders]
    bn = np.concatenate([np.asarray(b, dtype=np.int32) for b in borders]) if borders else np.zeros(0, np.int32)
    cpbin.write(
        path,
        {
            "node_xy": np.asarray(node_xy, dtype=np.float64).ravel(),
            "elem3": np.asarray(elem3, dtype=np.int32).ravel(),
            "elem4": np.asarray(elem4, dtype=np.int32).ravel(),
            "elem8": np.asarray(elem8, dtype=np.int32).ravel(),
            "border_len": np.asarray(bl, dtype=np.int32),
            "border_nodes": bn,
        },
    )
