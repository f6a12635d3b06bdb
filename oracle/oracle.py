"""TEST INFRASTRUCTURE ONLY: the CPU oracle for the cut-scoring / local-search path.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this module. The product package never imports it and has no CPU
fallback through it.

Contents
--------
* ctypes bindings to ``oracle/libpqi_oracle.so`` (the plain-C restatement of the
  reference's dense OpenCL kernels, ``oracle/pqi_oracle.c``) and, when it has
  been built, to ``oracle/_ref/libpqi_ref.so`` (the reference's own
  ``pyqrackising/kernels.cl`` compiled for the host by ``oracle/build_ref.sh``).
* numpy restatements of the objective functions
  (``pyqrackising/maxcut_tfim_util.py:319-346,445-461``) in float64.
* bit packing in the reference's layout (``maxcut_tfim_util.py:276-316``).
* the launch geometry of the reference host glue (``maxcut_tfim_util.py:169-221``).
* a restatement of the GPU branch of the ``spin_glass_solver`` driver loop
  (``pyqrackising/spin_glass_solver.py:603-727``) on top of those kernels.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libpqi_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpqi_ref.so")

GRAY_NODE_LIMIT = 131072  # maxcut_tfim_util.py:11
HEURISTIC_THRESHOLD = 24  # maxcut_tfim_util.py:165
WORK_GROUP_MULTIPLE = 32  # PREFERRED_WORK_GROUP_SIZE_MULTIPLE on NVIDIA (maxcut_tfim_util.py:132)


def build_oracle(force: bool = False) -> str:
    """Compile ``pqi_oracle.c`` with gcc (no FMA contraction: float sums keep the
    reference's one-rounding-per-add behaviour; OpenMP only splits independent
    candidates across threads)."""
    src = os.path.join(HERE, "pqi_oracle.c")
    if force or not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.check_call(
            ["gcc", "-O2", "-fPIC", "-shared", "-std=gnu11", "-ffp-contract=off", "-fopenmp", "-o", ORACLE_SO, src, "-lm"]
        )
    return ORACLE_SO


def reference_root() -> str:
    """Where the reference checkout lies in the build container: the
    environment variable PQI_REFERENCE_ROOT, else the container's read-only
    mount. Only build recipes and fixture generators read it."""
    return os.environ.get("PQI_REFERENCE_ROOT", "/root/reference")


def build_ref(reference_root: str | None = None) -> str | None:
    """Build ``oracle/_ref/libpqi_ref.so`` from the reference's kernels.cl when the
    reference checkout is present; returns None otherwise."""
    if reference_root is None:
        reference_root = globals()["reference_root"]()
    if not os.path.exists(os.path.join(reference_root, "pyqrackising", "kernels.cl")):
        return None
    subprocess.check_call(["sh", os.path.join(HERE, "build_ref.sh"), reference_root])
    return REF_SO


_F32P = ctypes.POINTER(ctypes.c_float)
_F64P = ctypes.POINTER(ctypes.c_double)
_U32P = ctypes.POINTER(ctypes.c_uint32)
_U64P = ctypes.POINTER(ctypes.c_uint64)
_I32P = ctypes.POINTER(ctypes.c_int32)
_I64P = ctypes.POINTER(ctypes.c_int64)

_lib = None
_ref = None


def _p(a, t):
    return a.ctypes.data_as(t)


def lib():
    global _lib
    if _lib is None:
        build_oracle()
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_cut_values.argtypes = [_F32P, ctypes.c_int, _U32P, ctypes.c_int, ctypes.c_int, _F32P]
        L.orc_single_values.argtypes = [_F32P, ctypes.c_int, _U32P, ctypes.c_int, _F32P]
        L.orc_double_one.argtypes = [_F32P, ctypes.c_int, _U32P, ctypes.c_int, ctypes.c_int]
        L.orc_double_one.restype = ctypes.c_float
        L.orc_pair_decode.argtypes = [ctypes.c_int, ctypes.c_int, _I32P, _I32P]
        L.orc_select.argtypes = [_F32P, ctypes.c_long, ctypes.c_int, ctypes.c_int, _F32P, _I32P, _F32P, _I32P]
        L.orc_select.restype = ctypes.c_int
        L.orc_double_select.argtypes = [_F32P, ctypes.c_int, _U32P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _F32P, _I32P]
        L.orc_double_select.restype = ctypes.c_int
        L.orc_gray_seed.argtypes = [_U64P, ctypes.c_int, ctypes.c_long]
        L.orc_gray.argtypes = [_F32P, ctypes.c_int, _U64P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _U64P, _F32P, _I64P]
        L.orc_gray_margin.argtypes = [_F32P, ctypes.c_int, _U64P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _U64P, _F32P, _I64P, _F32P]
        L.orc_double_select_gains.argtypes = [_F64P, _F32P, ctypes.c_int, _U32P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _F32P, _I32P]
        L.orc_double_select_gains.restype = ctypes.c_int
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """The reference's own kernels.cl, compiled for the host (oracle/_ref)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError("oracle/_ref/libpqi_ref.so not built (oracle/build_ref.sh)")
        R = ctypes.CDLL(REF_SO)
        R.pqi_ref_calculate_cut.argtypes = [_F32P, ctypes.c_int, _U32P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _F32P, _I32P]
        R.pqi_ref_single_bit_flips.argtypes = [_F32P, ctypes.c_int, _U32P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _F32P, _I32P]
        R.pqi_ref_double_bit_flips.argtypes = [_F32P, ctypes.c_int, _U32P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _F32P, _I32P]
        R.pqi_ref_gray.argtypes = [_F32P, ctypes.c_int, _U64P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _U64P, _F32P]
        _ref = R
    return _ref


# --------------------------------------------------------------------------------------
# Bit layout (maxcut_tfim_util.py:276-316): node j -> word j >> 5 (or >> 6), bit j & 31.


def pack32(bits) -> np.ndarray:
    """bool[..., n] -> uint32[..., ceil(n/32)] (convert_bool_to_uint, util:304-316)."""
    b = np.asarray(bits, dtype=np.bool_)
    n = b.shape[-1]
    n32 = (n + 31) >> 5
    pad = np.zeros(b.shape[:-1] + (n32 * 32,), dtype=np.bool_)
    pad[..., :n] = b
    w = np.packbits(pad.reshape(b.shape[:-1] + (n32, 4, 8)), axis=-1, bitorder="little")
    return np.ascontiguousarray(w.reshape(b.shape[:-1] + (n32, 4))).view(np.uint32).reshape(b.shape[:-1] + (n32,))


def pack64(bits) -> np.ndarray:
    """bool[n] -> uint64[ceil(n/64)] (make_best_theta_buf_64, util:290-301)."""
    b = np.asarray(bits, dtype=np.bool_)
    n = b.shape[-1]
    n64 = (n + 63) >> 6
    w32 = pack32(np.concatenate([b, np.zeros(n64 * 64 - n, dtype=np.bool_)]) if n64 * 64 != n else b)
    return np.ascontiguousarray(w32).view(np.uint64)


def unpack64(words, n) -> np.ndarray:
    """uint64 words -> bool[n] (spin_glass_solver.py:296-305)."""
    w = np.ascontiguousarray(np.asarray(words, dtype=np.uint64))
    bits = np.unpackbits(w.view(np.uint8), bitorder="little")
    return bits[:n].astype(np.bool_)


def unpack32(words, n) -> np.ndarray:
    w = np.ascontiguousarray(np.asarray(words, dtype=np.uint32))
    bits = np.unpackbits(w.view(np.uint8), bitorder="little")
    return bits[:n].astype(np.bool_)


# --------------------------------------------------------------------------------------
# Objectives in float64 (maxcut_tfim_util.py:319-346, 445-461).


def compute_cut(bits, W) -> float:
    """Sum over all ordered pairs with differing bits, halved (util:327-331)."""
    s = np.asarray(bits, dtype=np.int64)
    d = s[:, None] ^ s[None, :]
    return float((d * W.astype(np.float64)).sum() / 2.0)


def compute_energy(bits, W) -> float:
    """Half the sum of W * (2[s_u != s_v] - 1) over ordered pairs (util:319-324)."""
    s = np.asarray(bits, dtype=np.int64)
    d = ((s[:, None] ^ s[None, :]) << 1) - 1
    return float((d * W.astype(np.float64)).sum() / 2.0)


def compute_cut_diff(u, bits, W) -> float:
    """Row-u gain against the state given (util:334-336)."""
    s = np.asarray(bits, dtype=np.int64)
    return float((W[u].astype(np.float64) * (((s[u] ^ s) << 1) - 1)).sum())


def compute_cut_diff_between(o_bits, n_bits, W) -> float:
    """Upper-triangle cut delta between two states (util:445-461)."""
    o = np.asarray(o_bits, dtype=np.bool_)
    nb = np.asarray(n_bits, dtype=np.bool_)
    od = o[:, None] != o[None, :]
    nd = nb[:, None] != nb[None, :]
    ch = np.triu(od != nd, 1)
    sgn = np.where(nd, 1.0, -1.0)
    return float((W.astype(np.float64) * sgn * ch).sum())


# --------------------------------------------------------------------------------------
# Launch geometry of the reference host glue (maxcut_tfim_util.py:169-221).


def geometry(l: int, g: int, max_gpu_proc_elem: int, wgs: int = WORK_GROUP_MULTIPLE):
    """Return (global_size, local_size) as setup_opencl computes them."""
    local = min(wgs, l)
    max_global = ((max_gpu_proc_elem + local - 1) // local) * local
    glob = min(((g + local - 1) // local) * local, max_global)
    return glob, local


def flip_geometry(n: int, mpe: int):
    """single/double flips: setup_opencl(min(wgs, n), n, ...) (spin_glass_solver.py:569-575)."""
    return geometry(min(WORK_GROUP_MULTIPLE, n), n, mpe)


def cut_geometry(shots: int, mpe: int):
    """calculate_cut: setup_opencl(shots, shots, ...) (maxcut_tfim.py:167-171)."""
    return geometry(shots, shots, mpe)


# --------------------------------------------------------------------------------------
# Kernel-level oracle calls.


def _w(W):
    return np.ascontiguousarray(W, dtype=np.float32)


def cut_values(W, theta32, shots, is_spin_glass) -> np.ndarray:
    W = _w(W)
    n = W.shape[0]
    th = np.ascontiguousarray(theta32, dtype=np.uint32)
    out = np.empty(shots, dtype=np.float32)
    lib().orc_cut_values(_p(W, _F32P), n, _p(th, _U32P), shots, int(bool(is_spin_glass)), _p(out, _F32P))
    return out


def single_values(W, theta32, is_spin_glass) -> np.ndarray:
    W = _w(W)
    n = W.shape[0]
    th = np.ascontiguousarray(theta32, dtype=np.uint32)
    out = np.empty(n, dtype=np.float32)
    lib().orc_single_values(_p(W, _F32P), n, _p(th, _U32P), int(bool(is_spin_glass)), _p(out, _F32P))
    return out


def double_value(W, theta32, k, l) -> float:
    W = _w(W)
    th = np.ascontiguousarray(theta32, dtype=np.uint32)
    return float(lib().orc_double_one(_p(W, _F32P), W.shape[0], _p(th, _U32P), int(k), int(l)))


def pair_decode(c, n):
    k = ctypes.c_int32()
    l = ctypes.c_int32()
    lib().orc_pair_decode(int(c), int(n), ctypes.byref(k), ctypes.byref(l))
    return k.value, l.value


def select(values, G, L, with_groups=False):
    v = np.ascontiguousarray(values, dtype=np.float32)
    e = ctypes.c_float()
    i = ctypes.c_int32()
    ge = np.empty(G // L, dtype=np.float32)
    gi = np.empty(G // L, dtype=np.int32)
    rc = lib().orc_select(_p(v, _F32P), v.size, G, L, ctypes.byref(e), ctypes.byref(i), _p(ge, _F32P), _p(gi, _I32P))
    if rc:
        raise ValueError("bad geometry")
    if with_groups:
        return np.float32(e.value), int(i.value), ge, gi
    return np.float32(e.value), int(i.value)


def single_select(W, theta32, is_spin_glass, G, L):
    return select(single_values(W, theta32, is_spin_glass), G, L)


def double_select(W, theta32, is_spin_glass, G, L):
    W = _w(W)
    th = np.ascontiguousarray(theta32, dtype=np.uint32)
    e = ctypes.c_float()
    i = ctypes.c_int32()
    rc = lib().orc_double_select(_p(W, _F32P), W.shape[0], _p(th, _U32P), int(bool(is_spin_glass)), G, L, ctypes.byref(e), ctypes.byref(i))
    if rc:
        raise ValueError("bad geometry")
    return np.float32(e.value), int(i.value)


def cut_select(W, theta32, shots, is_spin_glass, G, L):
    return select(cut_values(W, theta32, shots, is_spin_glass), G, L)


def gray_seed(theta64, n, gid) -> np.ndarray:
    w = np.array(theta64, dtype=np.uint64, copy=True)
    lib().orc_gray_seed(_p(w, _U64P), int(n), int(gid))
    return w


def gray(W, theta64, is_spin_glass, iters_bound, G, margins=False):
    """Returns (theta_out uint64[G, blocks], energy_out float32[G], skipped_oob_flips)
    and, with margins=True, a fourth item: float32[G], each work-item's smallest
    |gain| over its keep-or-revert decisions (inf when it made none)."""
    W = _w(W)
    n = W.shape[0]
    blocks = (n + 63) >> 6
    th = np.ascontiguousarray(theta64, dtype=np.uint64)
    tout = np.empty((G, blocks), dtype=np.uint64)
    eout = np.empty(G, dtype=np.float32)
    marg = np.empty(G, dtype=np.float32)
    oob = ctypes.c_int64()
    lib().orc_gray_margin(_p(W, _F32P), n, _p(th, _U64P), int(bool(is_spin_glass)), int(iters_bound), int(G),
                          _p(tout, _U64P), _p(eout, _F32P), ctypes.byref(oob), _p(marg, _F32P))
    if margins:
        return tout, eout, int(oob.value), marg
    return tout, eout, int(oob.value)


def double_select_gains(W, theta32, gains64, is_spin_glass, G, L):
    """The double-flip pass's selection (kernels.cl:186-231) with pair values
    from float64 gains, each rounded once to float32 (pqi_oracle.c
    orc_double_select_gains): the reference's exact result for integer
    weights, O(n^2) so it runs at full benchmark sizes."""
    W = _w(W)
    th = np.ascontiguousarray(theta32, dtype=np.uint32)
    g = np.ascontiguousarray(gains64, dtype=np.float64)
    e = ctypes.c_float()
    i = ctypes.c_int32()
    if lib().orc_double_select_gains(_p(g, _F64P), _p(W, _F32P), W.shape[0], _p(th, _U32P), int(bool(is_spin_glass)),
                                     int(G), int(L), ctypes.byref(e), ctypes.byref(i)) != 0:
        raise ValueError("bad geometry")
    return np.float32(e.value), int(i.value)


def gray_has_oob(n, iters_bound, G) -> bool:
    """True when some Gray flip of the reference schedule lands on k >= n (then the
    reference kernel reads outside W and has no defined result)."""
    rem = n & 63
    if rem == 0:
        return False
    # flip k = ctz(i+1) + 64*(blocks-1) >= n  <=>  ctz(i+1) >= rem, for some i < iters_bound
    return iters_bound >= (1 << rem)


# --------------------------------------------------------------------------------------
# The reference's own kernels (oracle/_ref), same call shapes.


def ref_single_select(W, theta32, is_spin_glass, G, L):
    W = _w(W)
    th = np.ascontiguousarray(theta32, dtype=np.uint32)
    ge = np.empty(G // L, dtype=np.float32)
    gi = np.empty(G // L, dtype=np.int32)
    ref().pqi_ref_single_bit_flips(_p(W, _F32P), W.shape[0], _p(th, _U32P), int(bool(is_spin_glass)), G, L, _p(ge, _F32P), _p(gi, _I32P))
    bx = int(np.argmax(ge))
    return ge[bx], int(gi[bx]), ge, gi


def ref_double_select(W, theta32, is_spin_glass, G, L):
    W = _w(W)
    th = np.ascontiguousarray(theta32, dtype=np.uint32)
    ge = np.empty(G // L, dtype=np.float32)
    gi = np.empty(G // L, dtype=np.int32)
    ref().pqi_ref_double_bit_flips(_p(W, _F32P), W.shape[0], _p(th, _U32P), int(bool(is_spin_glass)), G, L, _p(ge, _F32P), _p(gi, _I32P))
    bx = int(np.argmax(ge))
    return ge[bx], int(gi[bx]), ge, gi


def ref_cut_select(W, theta32, shots, is_spin_glass, G, L):
    W = _w(W)
    th = np.array(theta32, dtype=np.uint32, copy=True)
    ge = np.empty(G // L, dtype=np.float32)
    gi = np.empty(G // L, dtype=np.int32)
    ref().pqi_ref_calculate_cut(_p(W, _F32P), W.shape[0], _p(th, _U32P), int(shots), int(bool(is_spin_glass)), G, L, _p(ge, _F32P), _p(gi, _I32P))
    bx = int(np.argmax(ge))
    return ge[bx], int(gi[bx]), ge, gi


def ref_gray(W, theta64, is_spin_glass, iters_bound, G):
    W = _w(W)
    n = W.shape[0]
    if gray_has_oob(n, iters_bound, G):
        raise ValueError("reference gray kernel reads outside W for this schedule")
    blocks = (n + 63) >> 6
    th = np.ascontiguousarray(theta64, dtype=np.uint64)
    tout = np.empty((G, blocks), dtype=np.uint64)
    eout = np.empty(G, dtype=np.float32)
    ref().pqi_ref_gray(_p(W, _F32P), n, _p(th, _U64P), int(bool(is_spin_glass)), int(iters_bound), int(G), _p(tout, _U64P), _p(eout, _F32P))
    return tout, eout


# --------------------------------------------------------------------------------------
# Driver loop, GPU branch of spin_glass_solver (spin_glass_solver.py:603-727).


def spin_glass_gpu_path(W, best_theta, is_spin_glass, gray_iterations, mpe, gray_seeds, use_ref=False, reheat=True, trace=None):
    """Restates the while-improved loop of the reference's OpenCL path.

    ``mpe`` is MAX_GPU_PROC_ELEM (flip geometry); ``gray_seeds`` is the gray
    kernel's global size (the reference uses MAX_GPU_PROC_ELEM there,
    spin_glass_solver.py:587). Returns (theta bool[n], running max_energy).
    ``trace`` (a list) receives one tuple per accepted move.
    """
    W = _w(W)
    n = W.shape[0]
    theta = np.array(best_theta, dtype=np.bool_, copy=True)
    max_energy = compute_energy(theta, W) if is_spin_glass else compute_cut(theta, W)
    Gf, Lf = flip_geometry(n, mpe)
    iters_bound = (gray_iterations + gray_seeds - 1) // gray_seeds

    def single(th):
        if use_ref:
            e, i, _, _ = ref_single_select(W, pack32(th), is_spin_glass, Gf, Lf)
        else:
            e, i = single_select(W, pack32(th), is_spin_glass, Gf, Lf)
        if e <= 0.0:
            return 0.0, th
        th = th.copy()
        th[i] = not th[i]
        return e, th

    def double(th):
        if use_ref:
            e, c, _, _ = ref_double_select(W, pack32(th), is_spin_glass, Gf, Lf)
        else:
            e, c = double_select(W, pack32(th), is_spin_glass, Gf, Lf)
        if e <= 0.0:
            return 0.0, th
        k, l = pair_decode(c, n)
        th = th.copy()
        th[k] = not th[k]
        th[l] = not th[l]
        return e, th

    def gray_step(th):
        if use_ref:
            tout, eout = ref_gray(W, pack64(th), is_spin_glass, iters_bound, gray_seeds)
        else:
            tout, eout, _ = gray(W, pack64(th), is_spin_glass, iters_bound, gray_seeds)
        bx = int(np.argmax(eout))
        e = eout[bx]
        if e <= 0.0:
            return 0.0, th
        return e, unpack64(tout[bx], n)

    improved = True
    while improved:
        improved = False
        e, st = single(theta)
        if e > 0.0:
            max_energy += e
            theta = st
            improved = True
            if trace is not None:
                trace.append(("single", float(e)))
            continue
        e, st = double(theta)
        if e > 0.0:
            max_energy += e
            theta = st
            improved = True
            if trace is not None:
                trace.append(("double", float(e)))
            continue
        if n <= GRAY_NODE_LIMIT:
            e, st = gray_step(theta)
        else:  # pragma: no cover - the CPU gray of the reference, not restated
            raise NotImplementedError("n above the gray node limit")
        if e > 0.0:
            max_energy += e
            theta = st
            improved = True
            if trace is not None:
                trace.append(("gray", float(e)))
            continue
        if not reheat:
            break
        # Post-reheat phase (spin_glass_solver.py:670-717). On this path gray
        # returned (0.0, theta) so the reheat starts from the current theta.
        reheat_theta = st.copy()
        reheat_energy = e
        e, st = single(reheat_theta)
        if (e + reheat_energy) > 0.0:
            max_energy += reheat_energy + e
            theta = st
            improved = True
            continue
        if e > 0.0:
            reheat_theta = st.copy()
            reheat_energy += e
        e, st = double(reheat_theta)
        if (e + reheat_energy) > 0.0:
            max_energy += reheat_energy + e
            theta = st
            improved = True
    return theta, float(max_energy)


# --------------------------------------------------------------------------------------
# Batched form (no reference counterpart): steepest single-flip ascent with the
# batched kernel's rule -- the largest gain rounded to float32, lowest node on
# ties, accept while > 0 -- with float64 gains kept incrementally.


def steepest_ascent(W, bits, budget=None):
    """Returns (final bool[n], number of flips)."""
    Wd = np.asarray(W, dtype=np.float64).copy()
    np.fill_diagonal(Wd, 0.0)
    s = np.array(bits, dtype=np.bool_, copy=True)
    x = np.where(s, 1.0, -1.0)
    g = x * (Wd @ x)
    flips = 0
    budget = budget if budget is not None else 4 * len(s) + 64
    while True:
        g32 = g.astype(np.float32)
        k = int(np.argmax(g32))
        if not g32[k] > 0 or flips >= budget:
            break
        xk = x[k]
        g -= 2.0 * x * xk * Wd[k]
        g[k] = -g[k] - 2.0 * xk * xk * Wd[k, k]
        x[k] = -xk
        s[k] = not s[k]
        flips += 1
    return s, flips
