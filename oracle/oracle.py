"""ORACLE — test infrastructure only.

ctypes bindings of ``oracle/_build/liboracle.so``, the CPU restatement of the
reference's element routines (see ``oracle_core.hpp``). Only the tests, the
smoke check and bench.py's CPU-baseline leg import this module; the product
never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
NF = 39  # per-point state layout: ep 6, beta 6, alpha 4x6, eqps, thick, loading

_lib = None
_libs = {}
# "strict": the parity build (-O2, no contraction: every product and sum
# separately rounded); "fast": the timed CPU baseline (-O3 -march=native,
# fused multiply-adds allowed), built for the CPU it runs on.
_variant = "strict"
FAST_FLAGS = "-O3 -march=native -fopenmp (fused multiply-adds allowed)"
STRICT_FLAGS = "-O2 -fopenmp -ffp-contract=off"


def build() -> str:
    """Compile the oracle (make in oracle/)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def cpu_key() -> str:
    """A name for this host's CPU (model and instruction-set flags), so that
    a -march=native build is only loaded on the CPU it was built for."""
    import hashlib
    import platform

    text = platform.machine()
    try:
        with open("/proc/cpuinfo") as f:
            lines = f.read().splitlines()
        model = next((ln for ln in lines if ln.startswith("model name")), "")
        flags = next((ln for ln in lines if ln.startswith("flags")), "")
        text += model + flags
    except OSError:
        pass
    return hashlib.sha1(text.encode()).hexdigest()[:12]


def fast_path() -> str:
    return os.path.join(HERE, "_build", "fast-" + cpu_key(), "liboracle.so")


def build_fast() -> str:
    """Compile the timed CPU baseline for this host's CPU (make fast)."""
    path = fast_path()
    subprocess.run(["make", "-s", "-C", HERE, "fast", f"FAST_OUT={path}"], check=True)
    return path


def use_variant(name: str) -> str:
    """Route every binding of this module through the "strict" (parity) or
    the "fast" (timed baseline) build; returns the previous variant."""
    global _variant, _lib
    if name not in ("strict", "fast"):
        raise ValueError(name)
    prev = _variant
    _variant = name
    _lib = None
    return prev


def lib():
    global _lib
    if _lib is None:
        if _variant == "fast":
            path = build_fast()
        else:
            path = LIB_PATH
            if not os.path.exists(LIB_PATH):
                build()
        if path not in _libs:
            handle = ctypes.CDLL(path)
            _declare(handle)
            _libs[path] = handle
        _lib = _libs[path]
    return _lib


_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)
_c = ctypes.POINTER(ctypes.c_char)
_ll = ctypes.c_longlong


def _declare(L):
    L.orc_set_element.argtypes = [ctypes.c_int, ctypes.c_int]
    L.orc_vjp_x.argtypes = [_d] + [ctypes.c_int] * 4 + [_ll, _d, _d, _d, _d, _d, _d, _i]
    L.orc_rule_size.argtypes = [ctypes.c_int] * 3
    L.orc_rule.argtypes = [ctypes.c_int] * 3 + [_d]
    L.orc_yield_matrix.argtypes = [_d, _d]
    L.orc_return.argtypes = [_d, _d, _d, ctypes.c_int, _d, _d, _d, _d, _i]
    L.orc_log_strain.argtypes = [_d, _d, _d, _d, _d, _d]
    L.orc_elements.argtypes = ([_d] + [ctypes.c_int] * 4 + [_ll, _d, _d, _d, _d, ctypes.c_int, ctypes.c_int]
                               + [_d, _d, _d, _d, _d, _i, _i, _i, ctypes.c_void_p])
    L.orc_element_stress.argtypes = [_d] + [ctypes.c_int] * 4 + [_ll, _d, _d, _d, _d, ctypes.c_int, _d, _i]
    L.orc_count_flops.restype = _ll
    L.orc_count_flops.argtypes = [_d] + [ctypes.c_int] * 4 + [_ll, _d, _d, _d, _d, ctypes.c_int]
    L.orc_pattern_nnz.restype = _ll
    L.orc_pattern_nnz.argtypes = [ctypes.c_int, ctypes.c_int, _i]
    L.orc_build_pattern.argtypes = [ctypes.c_int, ctypes.c_int, _i, _i, _i, _i]
    L.orc_scatter.argtypes = [ctypes.c_int, ctypes.c_int, _i, _i, _i, _d, _d, _ll]
    L.orc_system_evaluate.argtypes = ([_d] + [ctypes.c_int] * 6 + [_d, _i, _d, _d, _d, ctypes.c_int, ctypes.c_int,
                                      _i, _i, _ll, _d, _d, _d, _i, _d, _d, _d, _i])
    L.orc_add_node_blocks.argtypes = [_i, _i, _d, ctypes.c_int, _i, _d]
    L.orc_contact_create.restype = ctypes.c_void_p
    L.orc_contact_create.argtypes = [ctypes.c_int, _d, ctypes.c_int, _d, _d, _d, ctypes.c_int]
    L.orc_contact_destroy.argtypes = [ctypes.c_void_p]
    L.orc_contact_begin.argtypes = [ctypes.c_void_p, _d, ctypes.c_double, ctypes.c_double, _c, ctypes.c_double, _i]
    L.orc_contact_evaluate.argtypes = [ctypes.c_void_p, _d, ctypes.c_double, ctypes.c_int, _d, ctypes.c_int, _i,
                                       _d, _d, _d]
    L.orc_contact_anticipate.argtypes = [ctypes.c_void_p, _d, _d, ctypes.c_double, _d, ctypes.c_int, _i, _d]
    L.orc_contact_commit.argtypes = [ctypes.c_void_p]
    L.orc_contact_history.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _d]


class element:
    """Context: the calls inside evaluate the standard Hex8
    (Elastoplastic.cpp:226-340; `averaged`: with mean dilatation) instead of
    the incompatible-mode Hex8."""

    def __init__(self, standard: bool, averaged: bool = False):
        self.standard, self.averaged = bool(standard), bool(averaged)

    def __enter__(self):
        lib().orc_set_element(int(self.standard), int(self.averaged))
        return self

    def __exit__(self, *exc):
        lib().orc_set_element(0, 0)


def _p(a, kind=_d):
    if a is None:
        return None
    return a.ctypes.data_as(kind)


def material_record(m: dict) -> np.ndarray:
    """The oracle's flat material layout from a material dict (keys as in
    the product's Material: youngs_modulus, poisson_ratio, yield_stress,
    hardening_modulus, kinematic_hardening_modulus, saturation_stress,
    saturation_rate, criterion ('von_mises'|'hill48'), backstresses
    [(C, gamma)...], kinematic_integration ('exponential'|'backward_euler'),
    r0, r45, r90, shear_l, shear_m, rolling_direction, sheet_normal)."""
    r = np.zeros(32)
    r[0] = m["youngs_modulus"]
    r[1] = m["poisson_ratio"]
    r[2] = m.get("yield_stress", 0.0)
    r[3] = m.get("hardening_modulus", 0.0)
    r[4] = m.get("kinematic_hardening_modulus", 0.0)
    r[5] = m.get("saturation_stress", 0.0)
    r[6] = m.get("saturation_rate", 0.0)
    r[7] = 1.0 if m.get("criterion", "von_mises") == "hill48" else 0.0
    back = m.get("backstresses", [])
    r[8] = len(back)
    r[9] = 1.0 if m.get("kinematic_integration", "exponential") == "backward_euler" else 0.0
    for i, (c, g) in enumerate(back):
        r[10 + i] = c
        r[14 + i] = g
    r[18] = m.get("r0", 1.0)
    r[19] = m.get("r45", 1.0)
    r[20] = m.get("r90", 1.0)
    r[21] = m.get("shear_l", 1.5)
    r[22] = m.get("shear_m", 1.5)
    r[23:26] = m.get("rolling_direction", (1.0, 0.0, 0.0))
    r[26:29] = m.get("sheet_normal", (0.0, 0.0, 1.0))
    return r


KIN = {"small": 0, "finite": 1, "logarithmic": 2}


def rule_size(in_plane=2, thickness=0, axis=2) -> int:
    return int(lib().orc_rule_size(in_plane, thickness, axis))


def rule(in_plane=2, thickness=0, axis=2) -> np.ndarray:
    n = lib().orc_rule_size(in_plane, thickness, axis)
    out = np.zeros((n, 4))
    lib().orc_rule(in_plane, thickness, axis, _p(out))
    return out


def yield_matrix(m: dict) -> np.ndarray:
    rec = material_record(m)
    p = np.zeros(36)
    if lib().orc_yield_matrix(_p(rec), _p(p)) != 0:
        raise ValueError("invalid material")
    return p.reshape(6, 6)


def plastic_return(m: dict, strain, committed=None, want_tangent=True):
    rec = material_record(m)
    strain = np.ascontiguousarray(strain, dtype=np.float64)
    committed = np.zeros(NF) if committed is None else np.ascontiguousarray(committed, dtype=np.float64)
    stress, tangent, trial, energy = np.zeros(6), np.zeros(36), np.zeros(NF), np.zeros(1)
    y = ctypes.c_int(0)
    code = lib().orc_return(_p(rec), _p(strain), _p(committed), int(want_tangent), _p(stress), _p(tangent),
                            _p(trial), _p(energy), ctypes.byref(y))
    return dict(code=code, stress=stress, tangent=tangent.reshape(6, 6), state=trial, energy=energy[0],
                yielding=bool(y.value))


def log_strain(green, t=None):
    green = np.ascontiguousarray(green, dtype=np.float64)
    t = np.zeros(6) if t is None else np.ascontiguousarray(t, dtype=np.float64)
    s, p, c, st = np.zeros(6), np.zeros(36), np.zeros(36), np.zeros(6)
    code = lib().orc_log_strain(_p(green), _p(t), _p(s), _p(p), _p(c), _p(st))
    return dict(code=code, strain=s, projection=p.reshape(6, 6), curvature=c.reshape(6, 6), stress=st)


def elements(m: dict, X, ue, committed=None, alpha_n=None, kinematics="logarithmic", in_plane=2, thickness=0,
             axis=2, want_tangent=True, threads=0):
    """Evaluate a batch of independent IM Hex8 elements. X, ue: (ne, 24)
    node-major; committed: (ne, nq, 39) or None (virgin); alpha_n: (ne, 9)."""
    rec = material_record(m)
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 24)
    ne = X.shape[0]
    ue = np.ascontiguousarray(ue, dtype=np.float64).reshape(ne, 24)
    nq = lib().orc_rule_size(in_plane, thickness, axis)
    committed = (np.zeros((ne, nq, NF)) if committed is None
                 else np.ascontiguousarray(committed, dtype=np.float64).reshape(ne, nq, NF))
    alpha_n = (np.zeros((ne, 9)) if alpha_n is None
               else np.ascontiguousarray(alpha_n, dtype=np.float64).reshape(ne, 9))
    f = np.zeros((ne, 24))
    K = np.zeros((ne, 24, 24)) if want_tangent else None
    energy = np.zeros(ne)
    trial = np.zeros((ne, nq, NF))
    alpha = np.zeros((ne, 9))
    y = np.zeros(ne, dtype=np.int32)
    it = np.zeros(ne, dtype=np.int32)
    st = np.zeros(ne, dtype=np.int32)
    yf = np.zeros((ne, nq), dtype=np.int8)
    lib().orc_elements(_p(rec), in_plane, thickness, axis, KIN[kinematics], ne, _p(X), _p(ue), _p(committed),
                       _p(alpha_n), int(want_tangent), threads, _p(f), _p(K), _p(energy), _p(trial), _p(alpha),
                       _p(y, _i), _p(it, _i), _p(st, _i), yf.ctypes.data_as(ctypes.c_void_p))
    return dict(force=f, tangent=K, energy=energy, states=trial, alpha=alpha, yielding=y, iterations=it, status=st,
                yield_flags=yf.astype(bool))


def element_stress(m: dict, X, ue, committed=None, alpha=None, kinematics="logarithmic", in_plane=2, thickness=0,
                   axis=2, threads=0):
    """incompatible_elastoplastic_stress (IncompatibleModes.cpp:602-664) of
    a batch: (ne, 28) - Cauchy 6, second Piola-Kirchhoff 6, von Mises, max
    eqps, max strain, min det F, Kirchhoff 6, log strain 6 - and a status
    per element."""
    rec = material_record(m)
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 24)
    ne = X.shape[0]
    ue = np.ascontiguousarray(ue, dtype=np.float64).reshape(ne, 24)
    nq = lib().orc_rule_size(in_plane, thickness, axis)
    committed = (np.zeros((ne, nq, NF)) if committed is None
                 else np.ascontiguousarray(committed, dtype=np.float64).reshape(ne, nq, NF))
    out = np.zeros((ne, 28))
    st = np.zeros(ne, dtype=np.int32)
    al = None if alpha is None else np.ascontiguousarray(alpha, dtype=np.float64).reshape(ne, 9)
    lib().orc_element_stress(_p(rec), in_plane, thickness, axis, KIN[kinematics], ne, _p(X), _p(ue), _p(committed),
                             _p(al) if al is not None else None, threads, _p(out), _p(st, _i))
    return out, st


def count_flops(m: dict, X, ue, committed=None, alpha_n=None, kinematics="logarithmic", in_plane=2, thickness=0,
                axis=2, want_tangent=True) -> int:
    rec = material_record(m)
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 24)
    ne = X.shape[0]
    ue = np.ascontiguousarray(ue, dtype=np.float64).reshape(ne, 24)
    nq = lib().orc_rule_size(in_plane, thickness, axis)
    committed = (np.zeros((ne, nq, NF)) if committed is None
                 else np.ascontiguousarray(committed, dtype=np.float64).reshape(ne, nq, NF))
    alpha_n = (np.zeros((ne, 9)) if alpha_n is None
               else np.ascontiguousarray(alpha_n, dtype=np.float64).reshape(ne, 9))
    return int(lib().orc_count_flops(_p(rec), in_plane, thickness, axis, KIN[kinematics], ne, _p(X), _p(ue),
                                     _p(committed), _p(alpha_n), int(want_tangent)))


def vjp_x(m: dict, X, ue, lam, committed=None, alpha_n=None, kinematics="logarithmic", in_plane=2, thickness=0,
          axis=2):
    """lambda . d f*/d X per IM Hex8 (ne, 24) at fixed ue and committed
    history, the modes through their local equilibrium; and a status per
    element."""
    rec = material_record(m)
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 24)
    ne = X.shape[0]
    ue = np.ascontiguousarray(ue, dtype=np.float64).reshape(ne, 24)
    lam = np.ascontiguousarray(lam, dtype=np.float64).reshape(ne, 24)
    nq = lib().orc_rule_size(in_plane, thickness, axis)
    committed = (np.zeros((ne, nq, NF)) if committed is None
                 else np.ascontiguousarray(committed, dtype=np.float64).reshape(ne, nq, NF))
    alpha_n = (np.zeros((ne, 9)) if alpha_n is None
               else np.ascontiguousarray(alpha_n, dtype=np.float64).reshape(ne, 9))
    out = np.zeros((ne, 24))
    st = np.zeros(ne, dtype=np.int32)
    lib().orc_vjp_x(_p(rec), in_plane, thickness, axis, KIN[kinematics], ne, _p(X), _p(ue), _p(committed),
                    _p(alpha_n), _p(lam), _p(out), _p(st, _i))
    return out, st


def pattern(nn: int, conn) -> dict:
    conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1, 8)
    ne = conn.shape[0]
    nnz = lib().orc_pattern_nnz(nn, ne, _p(conn, _i))
    outer = np.zeros(3 * nn + 1, dtype=np.int32)
    inner = np.zeros(nnz, dtype=np.int32)
    bo = np.zeros(ne * 64, dtype=np.int32)
    lib().orc_build_pattern(nn, ne, _p(conn, _i), _p(outer, _i), _p(inner, _i), _p(bo, _i))
    return dict(outer=outer, inner=inner, block_offset=bo, nnz=nnz)


def scatter(nn: int, conn, pat: dict, K) -> np.ndarray:
    conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1, 8)
    K = np.ascontiguousarray(K, dtype=np.float64)
    values = np.zeros(pat["nnz"])
    lib().orc_scatter(nn, conn.shape[0], _p(conn, _i), _p(pat["outer"], _i), _p(pat["block_offset"], _i), _p(K),
                      _p(values), pat["nnz"])
    return values


def system_evaluate(m: dict, coords, conn, u, committed=None, alpha_n=None, kinematics="logarithmic", in_plane=2,
                    thickness=0, axis=2, want_tangent=True, threads=0, pat=None):
    rec = material_record(m)
    coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
    conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1, 8)
    nn, ne = coords.shape[0], conn.shape[0]
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(nn * 3)
    nq = lib().orc_rule_size(in_plane, thickness, axis)
    committed = (np.zeros((ne, nq, NF)) if committed is None
                 else np.ascontiguousarray(committed, dtype=np.float64).reshape(ne, nq, NF))
    alpha_n = (np.zeros((ne, 9)) if alpha_n is None
               else np.ascontiguousarray(alpha_n, dtype=np.float64).reshape(ne, 9))
    if pat is None:
        pat = pattern(nn, conn)
    internal = np.zeros(nn * 3)
    gross, energy = np.zeros(1), np.zeros(1)
    y = ctypes.c_int(0)
    values = np.zeros(pat["nnz"])
    trial = np.zeros((ne, nq, NF))
    alpha = np.zeros((ne, 9))
    failed = ctypes.c_int(-1)
    code = lib().orc_system_evaluate(_p(rec), in_plane, thickness, axis, KIN[kinematics], nn, ne, _p(coords),
                                     _p(conn, _i), _p(u), _p(committed), _p(alpha_n), int(want_tangent), threads,
                                     _p(pat["outer"], _i), _p(pat["block_offset"], _i), pat["nnz"], _p(internal),
                                     _p(gross), _p(energy), ctypes.byref(y), _p(values), _p(trial), _p(alpha),
                                     ctypes.byref(failed))
    return dict(code=code, failed_element=failed.value, internal=internal, gross=gross[0], energy=energy[0],
                yielding_points=y.value, values=values, states=trial, alpha=alpha, pattern=pat)


def add_node_blocks(pat: dict, values, nodes, blocks) -> np.ndarray:
    values = np.array(values, dtype=np.float64, copy=True)
    nodes = np.ascontiguousarray(nodes, dtype=np.int32)
    blocks = np.ascontiguousarray(blocks, dtype=np.float64).reshape(-1, 9)
    rc = lib().orc_add_node_blocks(_p(pat["outer"], _i), _p(pat["inner"], _i), _p(values), len(nodes),
                                   _p(nodes, _i), _p(blocks))
    if rc:
        raise ValueError("a node block lies outside the pattern")
    return values


def stiffness_product(pat: dict, values, u) -> np.ndarray:
    """|K| |u| per row as stiffness_gross forms it
    (src/fem/NonlinearSystem.hpp:55-67): the CSC columns in ascending order,
    columns of zero displacement skipped, each column's |K(r, c)| |u(c)|
    added to its rows."""
    outer, inner = pat["outer"], pat["inner"]
    values = np.asarray(values, dtype=np.float64)
    u = np.asarray(u, dtype=np.float64)
    product = np.zeros(len(outer) - 1)
    for col in range(len(outer) - 1):
        uc = abs(u[col])
        if uc == 0.0:
            continue
        lo, hi = outer[col], outer[col + 1]
        product[inner[lo:hi]] += np.abs(values[lo:hi]) * uc  # distinct rows within a column
    return product


def stiffness_gross(pat: dict, values, u, free) -> float:
    """stiffness_gross(K, u, free): the norm of |K| |u| over the free DOFs,
    summed in the order of `free` (NonlinearSystem.hpp:64-66)."""
    product = stiffness_product(pat, values, u)
    s = 0.0
    for d in free:
        s += product[d] * product[d]
    return float(np.sqrt(s))


def free_free_block(pat: dict, values, free):
    """The free-free block of a full CSC tangent as PartitionedFactor::reset
    and ::build (src/fem/Forming.cpp:73-84, 213-241) and
    Assembler::reduce_free_free (src/fem/Assembler.cpp:294-320) form it:
    for every free column in ascending order, the entries of its free rows in
    the full column's order. Returns the block's outer, inner, the full index
    of each entry (the inverse of the reference's positions_ map) and its
    values (assemble, Forming.cpp:89-98, copies them)."""
    outer, inner = pat["outer"], pat["inner"]
    n = len(outer) - 1
    free = [int(d) for d in free]
    mapping = [-1] * n  # reset: DOF -> free index
    for i, d in enumerate(free):
        mapping[d] = i
    ff_outer = [0] * (len(free) + 1)
    ff_inner, source = [], []
    for col in range(n):
        c = mapping[col]
        if c < 0:
            continue
        for k in range(int(outer[col]), int(outer[col + 1])):
            r = mapping[int(inner[k])]
            if r < 0:
                continue
            ff_inner.append(r)
            source.append(k)
        ff_outer[c + 1] = len(ff_inner)
    source = np.array(source, dtype=np.int64)
    return (np.array(ff_outer, dtype=np.int32), np.array(ff_inner, dtype=np.int32), source,
            np.asarray(values, dtype=np.float64)[source])


def restrict(full, free) -> np.ndarray:
    """restrict(full, dofs) (src/fem/NonlinearSystem.hpp:336-340)."""
    return np.asarray(full, dtype=np.float64)[np.asarray(free, dtype=np.int64)]


def add_to(full, free, part, factor) -> np.ndarray:
    """add_to(full, dofs, part, factor) (src/fem/NonlinearSystem.hpp:342-347):
    full[dofs[i]] += factor * part[i], returned as a new array."""
    out = np.array(full, dtype=np.float64, copy=True)
    for i, d in enumerate(free):
        out[int(d)] += factor * float(part[i])
    return out


def release_solve(m: dict, coords, conn, committed, alpha_n, free, u0, kinematics="logarithmic", tol=1e-10,
                  max_iterations=40, threads=0, increments=1):
    """The released equilibrium on the CPU: Newton on the free rows of
    f_int(u) = 0 from u0 (its held DOFs kept), every tangent the oracle's
    assembled CSC (NonlinearSystem::evaluate restated) and every correction
    a scipy sparse solve of its free-free block, a step halved while an
    element refuses it, until a full step is below `tol` of u, then one step
    more. `increments` > 1 takes the start's imbalance r0 off in equal
    steps (equilibrium of f_int(u) = (1 - k / increments) r0 at each k), as
    the device Release does. The frozen release passes a material whose
    yield stress no point reaches. Returns (u, Newton iterations)."""
    import scipy.sparse
    import scipy.sparse.linalg

    coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
    nn = coords.shape[0]
    pat = pattern(nn, conn)
    free = np.asarray(free, dtype=np.int64)
    u = np.array(u0, dtype=np.float64, copy=True)

    def evaluate(x):
        return system_evaluate(m, coords, conn, x, committed, alpha_n, kinematics=kinematics, threads=threads, pat=pat)

    r = evaluate(u)
    if r["code"] != 0:
        raise RuntimeError(f"the oracle's element {r['failed_element']} failed in the release")
    r0 = r["internal"][free].copy()
    total = 0
    for k in range(1, increments + 1):
        left = 1.0 - k / increments
        last = k == increments
        converged = False
        for _ in range(max_iterations):
            kk = scipy.sparse.csc_matrix((r["values"], pat["inner"], pat["outer"]), shape=(3 * nn, 3 * nn))
            du = scipy.sparse.linalg.spsolve(kk[free][:, free].tocsc(), -(r["internal"][free] - left * r0))
            step = 1.0
            while True:
                trial = u.copy()
                trial[free] += step * du
                rt = evaluate(trial)
                if rt["code"] == 0:
                    break
                step *= 0.5
                if step < 1.0 / 1024:
                    raise RuntimeError(f"the oracle's element {rt['failed_element']} failed in the release")
            u, r = trial, rt
            total += 1
            if converged:
                break
            converged = step == 1.0 and np.linalg.norm(du) <= tol * np.linalg.norm(u)
            if converged and not last:
                break
        else:
            raise RuntimeError("the oracle's release did not converge")
    return u, total


def release_adjoint(m: dict, coords, conn, committed, alpha_n, free, u, dj_du, kinematics="logarithmic",
                    threads=0) -> np.ndarray:
    """dJ/dX (nn, 3) of a functional J(u*) of the released equilibrium u* on
    the CPU: K_ff^T lambda_f = (dJ/du)_f with the oracle's tangent at u*
    (scipy sparse solve of the transposed block), lambda zero on the held
    DOFs, and -lambda . d f_int / d X from the oracle's per-element shape
    derivative (vjp_x), summed into the nodes in element order."""
    import scipy.sparse
    import scipy.sparse.linalg

    coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
    conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1, 8)
    nn = coords.shape[0]
    pat = pattern(nn, conn)
    free = np.asarray(free, dtype=np.int64)
    r = system_evaluate(m, coords, conn, u, committed, alpha_n, kinematics=kinematics, threads=threads, pat=pat)
    k = scipy.sparse.csc_matrix((r["values"], pat["inner"], pat["outer"]), shape=(3 * nn, 3 * nn))
    lam = np.zeros(3 * nn)
    lam[free] = scipy.sparse.linalg.spsolve(k[free][:, free].T.tocsc(), np.asarray(dj_du)[free])
    dofs = (3 * conn[:, :, None] + np.arange(3)).reshape(-1, 24)
    per, st = vjp_x(m, coords[conn].reshape(-1, 24), u[dofs], lam[dofs], committed, alpha_n, kinematics=kinematics)
    if (st != 0).any():
        raise RuntimeError("the oracle's shape derivative failed")
    gx = np.zeros(3 * nn)
    np.add.at(gx, dofs.reshape(-1), per.reshape(-1))
    return -gx.reshape(nn, 3)


class Contact:
    """ToolContact restated: tools = list of dicts with shape ('sphere',
    'plane', 'cylinder'), radius, friction, tangential_ratio, normal, axis,
    times, points, nodes, area, kappa."""

    SHAPES = {"sphere": 0, "plane": 1, "cylinder": 2}

    def __init__(self, coords, tools, friction_tangent="exact"):
        self.coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
        self.nn = self.coords.shape[0]
        self.ntools = len(tools)
        rec, knots, slaves = [], [], []
        for t in tools:
            rec += [self.SHAPES[t["shape"]], t.get("radius", 0.0), t.get("friction", 0.0),
                    t.get("tangential_ratio", 1.0), *t.get("normal", (0, 0, 1)), *t.get("axis", (0, 0, 1)),
                    len(t["times"]), len(t["nodes"])]
            for tt, p in zip(t["times"], t["points"]):
                knots += [tt, *p]
            for n, a, k in zip(t["nodes"], t["area"], t["kappa"]):
                slaves += [n, a, k]
        self._rec = np.array(rec, dtype=np.float64)
        self._knots = np.array(knots, dtype=np.float64)
        self._slaves = np.array(slaves, dtype=np.float64)
        self.max_blocks = sum(len(t["nodes"]) for t in tools)
        self.h = lib().orc_contact_create(self.nn, _p(self.coords), self.ntools, _p(self._rec), _p(self._knots),
                                          _p(self._slaves), 1 if friction_tangent == "symmetric" else 0)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_contact_destroy(self.h)
            self.h = None

    def begin_increment(self, u0, t0, t1, active, margin):
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        act = (ctypes.c_char * self.ntools)(*[bytes([1 if a else 0]) for a in active])
        counts = np.zeros(self.ntools, dtype=np.int32)
        lib().orc_contact_begin(self.h, _p(u0), t0, t1, act, margin, _p(counts, _i))
        return counts

    def evaluate(self, u, t, want_tangent=True):
        u = np.ascontiguousarray(u, dtype=np.float64)
        residual = np.zeros(self.nn * 3)
        nodes = np.zeros(max(self.max_blocks, 1), dtype=np.int32)
        blocks = np.zeros((max(self.max_blocks, 1), 9))
        res = np.zeros((self.ntools, 9))
        sc = np.zeros(4)
        nb = lib().orc_contact_evaluate(self.h, _p(u), t, int(want_tangent), _p(residual), self.max_blocks,
                                        _p(nodes, _i), _p(blocks), _p(res), _p(sc))
        if nb < 0:
            return dict(code=-1)
        return dict(code=0, residual=residual, nodes=nodes[:nb].copy(), blocks=blocks[:nb].reshape(-1, 3, 3).copy(),
                    tools=res, gross=sc[0], round_off=sc[1], force_norm=sc[2], symmetric=bool(sc[3]))

    def anticipate(self, u, du, t, residual):
        u = np.ascontiguousarray(u, dtype=np.float64)
        du = np.ascontiguousarray(du, dtype=np.float64)
        residual = np.array(residual, dtype=np.float64, copy=True)
        nodes = np.zeros(max(self.max_blocks, 1), dtype=np.int32)
        blocks = np.zeros((max(self.max_blocks, 1), 9))
        n = lib().orc_contact_anticipate(self.h, _p(u), _p(du), t, _p(residual), self.max_blocks, _p(nodes, _i),
                                         _p(blocks))
        return residual, nodes[:n].copy(), blocks[:n].reshape(-1, 3, 3).copy()

    def commit(self):
        lib().orc_contact_commit(self.h)

    def history(self, k):
        cap = self.max_blocks + 1
        out = np.zeros((cap, 7))
        n = lib().orc_contact_history(self.h, k, cap, _p(out))
        return out[:n].copy()


def oracle_to_device(st: np.ndarray, nterms: int) -> np.ndarray:
    """(ne, nq, 39) oracle states -> (nfields, ne, nq), the product's device
    layout (plastic strain, back stress, kinematic terms, eqps, loading)."""
    ne, nq, _ = st.shape
    out = np.zeros((14 + 6 * nterms, ne, nq))
    out[0:12] = np.moveaxis(st[..., 0:12], -1, 0)
    for t in range(nterms):
        out[12 + 6 * t:18 + 6 * t] = np.moveaxis(st[..., 12 + 6 * t:18 + 6 * t], -1, 0)
    out[12 + 6 * nterms] = st[..., 36]
    out[13 + 6 * nterms] = st[..., 38]
    return out


def device_to_oracle(st: np.ndarray, nterms: int) -> np.ndarray:
    """The inverse of oracle_to_device."""
    _, ne, nq = st.shape
    out = np.zeros((ne, nq, NF))
    out[..., 0:12] = np.moveaxis(st[0:12], 0, -1)
    for t in range(nterms):
        out[..., 12 + 6 * t:18 + 6 * t] = np.moveaxis(st[12 + 6 * t:18 + 6 * t], 0, -1)
    out[..., 36] = st[12 + 6 * nterms]
    out[..., 38] = st[13 + 6 * nterms]
    return out
