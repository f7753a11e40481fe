"""Shared parity measures for the tests.

Fields are compared in relative L2, each normalised by the larger of its own
norm and the norm of the quantity that sets its natural scale (strain
components by the strain intensity, stress components by the stress
intensity, plastic strains by the total strain intensity), so that a field
which is round-off noise in a scenario (e.g. a lateral strain at nu ~ 0) is
compared against the scale of the solution rather than against itself.
"""
import numpy as np

FIELDS = ["uv", "exx", "eyy", "gamma", "eps_i", "sxx", "syy", "tau", "sig_i", "table_s", "psi", "E_c", "nu_c",
          "exx_p", "eyy_p", "gamma_p", "eps_p_i"]

SCALE_OF = {"exx": "eps_i", "eyy": "eps_i", "gamma": "eps_i", "sxx": "sig_i", "syy": "sig_i", "tau": "sig_i",
            "table_s": "sig_i", "exx_p": "eps_i", "eyy_p": "eps_i", "gamma_p": "eps_i", "eps_p_i": "eps_i"}


def rel_l2(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def field_error(name, got, ref):
    """Relative L2 error of field ``name`` (dicts of arrays)."""
    a, b = np.asarray(got[name], dtype=np.float64), np.asarray(ref[name], dtype=np.float64)
    scale = np.linalg.norm(b)
    if name in SCALE_OF:
        scale = max(scale, np.linalg.norm(np.asarray(ref[SCALE_OF[name]], dtype=np.float64)))
    return float(np.linalg.norm(a - b) / (scale if scale > 0 else 1.0))


def yielded(state, margin=1e-12):
    """Elements on the plastic branch of the diagram (secant modulus below E)."""
    return np.asarray(state["psi"]) > 1.0 + margin


def worst(got, ref, fields=FIELDS):
    errs = {k: field_error(k, got, ref) for k in fields}
    k = max(errs, key=errs.get)
    return k, errs[k], errs
