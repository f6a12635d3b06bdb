"""Device-resident graph state for the cut-scoring / local-search path.

``DeviceGraph`` owns the coupling matrix and its prepared copies in HBM (torch
tensors used as plain buffers) and a reusable workspace, and exposes the
library's kernels on them. It replaces the reference's OpenCL context and
buffer packers (``pyqrackising/maxcut_tfim_util.py:9-35,169-301``).

HBM layout per graph of n nodes (ld = n rounded up to 128):
  W       n*n   float32   caller's matrix, row-major (rescoring)
  W_f32z  n*ld  float32   zero diagonal, zero padding
  W_i8    n*ld  int8      integer weights in [-127, 127] (else absent)
  W_hi/lo n*ld  bf16 x2   split of float weights (else absent)
  W_d     4*n*ld int8    fixed-point digit planes of float weights (else absent)
"""

from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import _lib
from ._lib import PqiWeights, PqiWeightStats, call

WORK_GROUP_MULTIPLE = 32  # NVIDIA's PREFERRED_WORK_GROUP_SIZE_MULTIPLE (maxcut_tfim_util.py:132)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def default_device():
    if not torch.cuda.is_available():
        raise _lib.PQIUnavailable("no CUDA device: this package runs only on an sm_100 GPU")
    return torch.device("cuda", torch.cuda.current_device())


def max_gpu_proc_elem(device=None) -> int:
    """MAX_GPU_PROC_ELEM: env PYQRACKISING_MAX_GPU_PROC_ELEM, else the SM count
    (the reference uses the OpenCL MAX_COMPUTE_UNITS, maxcut_tfim_util.py:105-110)."""
    env = os.getenv("PYQRACKISING_MAX_GPU_PROC_ELEM")
    if env:
        return int(env)
    dev = device if device is not None else default_device()
    return torch.cuda.get_device_properties(dev).multi_processor_count


def geometry(l: int, g: int, mpe: int, wgs: int = WORK_GROUP_MULTIPLE):
    """(global_size, local_size) exactly as setup_opencl computes them
    (maxcut_tfim_util.py:179-184)."""
    local = min(wgs, l)
    max_global = ((mpe + local - 1) // local) * local
    return min(((g + local - 1) // local) * local, max_global), local


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def pack_bits(bits, n: int, device, stream=None) -> torch.Tensor:
    """bool[rows, n] (host or device) -> device int32 words, tight pitch
    ceil(n/32) per row (the reference layout), plus one spare zero word so a
    single state can also be read as ceil(n/64) 64-bit words."""
    if isinstance(bits, torch.Tensor):
        b = bits
    else:
        b = torch.from_numpy(np.ascontiguousarray(np.asarray(bits, dtype=np.uint8)))
    if b.dim() == 1:
        b = b[None, :]
    rows = int(b.shape[0])
    b = b.to(device=device, dtype=torch.uint8).contiguous()
    n32 = (n + 31) >> 5
    out = torch.zeros(rows * n32 + 1, dtype=torch.int32, device=device)
    call("pqi_pack_bits", _ptr(b), rows, n, _ptr(out), stream_ptr(stream))
    return out


def unpack_bits(words: torch.Tensor, n: int, rows: int = 1, pitch: int | None = None, device=None,
                stream=None) -> np.ndarray:
    """device words (row pitch `pitch`, default ceil(n/32)) -> host bool[rows, n]."""
    n32 = (n + 31) >> 5
    pitch = n32 if pitch is None else pitch
    w = words[: rows * pitch].view(rows, pitch)
    if pitch != n32:
        w = w[:, :n32]
    w = w.contiguous()
    out = torch.empty(rows * n, dtype=torch.uint8, device=words.device if device is None else device)
    call("pqi_unpack_bits", _ptr(w), rows, n, _ptr(out), stream_ptr(stream))
    return out.view(rows, n).cpu().numpy().astype(np.bool_)


class Workspace:
    """Grow-only device scratch buffer handed to the library calls."""

    def __init__(self, device):
        self.device = device
        self.buf = None

    def get(self, nbytes: int):
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, device=self.device)
        return ctypes.c_void_p(self.buf.data_ptr()), ctypes.c_size_t(self.buf.numel())


class DeviceGraph:
    """A prepared dense coupling matrix on one GPU."""

    def __init__(self, W, device=None, stream=None):
        _lib.load()
        self.device = torch.device(device) if device is not None else default_device()
        if isinstance(W, torch.Tensor):
            Wt = W.detach().to(device=self.device, dtype=torch.float32).contiguous()
        else:
            Wt = torch.from_numpy(np.ascontiguousarray(W, dtype=np.float32)).to(self.device)
        if Wt.dim() != 2 or Wt.shape[0] != Wt.shape[1]:
            raise ValueError("coupling matrix must be square")
        self.n = n = int(Wt.shape[0])
        self.W = Wt
        self.ws = Workspace(self.device)
        self.stream = stream
        st = PqiWeightStats()
        wsp, wsn = self.ws.get(_lib.load().pqi_workspace_bytes(n, 1))
        rc = _lib.status("pqi_scan_weights", _ptr(Wt), n, wsp, wsn, ctypes.byref(st), self.sp())
        if rc == _lib.PQI_EINVAL:
            if st.nonfinite:
                raise ValueError("coupling matrix has non-finite entries")
            if st.asym:
                raise ValueError("coupling matrix must be symmetric")
        if rc != _lib.PQI_OK:
            raise _lib.PQIError(rc, "pqi_scan_weights")
        self.stats = st
        ld = _lib.load().pqi_padded_ld(n)
        self.ld = ld
        self.W_f32z = torch.empty(n * ld, dtype=torch.float32, device=self.device)
        self.W_i8 = self.W_hi = self.W_lo = None
        if st.kind == _lib.PQI_W_I8:
            self.W_i8 = torch.empty(n * ld, dtype=torch.int8, device=self.device)
        else:
            self.W_hi = torch.empty(n * ld, dtype=torch.int16, device=self.device)
            self.W_lo = torch.empty(n * ld, dtype=torch.int16, device=self.device)
        self.w = PqiWeights()
        call(
            "pqi_prepare_weights",
            _ptr(Wt),
            n,
            ctypes.byref(st),
            _ptr(self.W_f32z),
            _ptr(self.W_i8),
            _ptr(self.W_hi),
            _ptr(self.W_lo),
            ctypes.byref(self.w),
            self.sp(),
        )
        self.W_d = None
        if st.kind != _lib.PQI_W_I8:
            # float weights: also their fixed-point digit planes (exact scoring)
            self.W_d = torch.empty(4 * n * ld, dtype=torch.int8, device=self.device)
            call("pqi_prepare_digits", ctypes.byref(self.w), ctypes.c_float(st.maxabs), _ptr(self.W_d), self.sp())
        self.n32 = (n + 31) >> 5
        self.n64 = (n + 63) >> 6

    # -- helpers ---------------------------------------------------------------------
    @property
    def is_integer(self) -> bool:
        return self.w.kind == _lib.PQI_W_I8

    @property
    def upper_sum(self) -> float:
        return float(self.w.upper_sum)

    def sp(self):
        return stream_ptr(self.stream)

    def wsp(self, count: int = 1):
        return self.ws.get(_lib.load().pqi_workspace_bytes(self.n, max(1, int(count))))

    def pack(self, bits) -> torch.Tensor:
        """bool[rows, n] (host or device) -> device int32 words, tight pitch
        ceil(n/32) per row (the reference layout), plus one spare zero word so a
        single state can also be read as ceil(n/64) 64-bit words."""
        return pack_bits(bits, self.n, self.device, self.stream)

    def unpack(self, words: torch.Tensor, rows: int = 1, pitch: int | None = None) -> np.ndarray:
        """device words (row pitch `pitch`, default ceil(n/32)) -> host bool[rows, n]."""
        return unpack_bits(words, self.n, rows, pitch, self.device, self.stream)

    # -- kernels ---------------------------------------------------------------------
    def gains(self, words: torch.Tensor, rows: int = 1, fp64: bool = True):
        """Gains of `rows` states given as tight [rows, n32] words."""
        src = words
        g32 = torch.empty(rows * self.n, dtype=torch.float32, device=self.device)
        g64 = torch.empty(rows * self.n, dtype=torch.float64, device=self.device) if fp64 else None
        wsp, wsn = self.wsp(rows)
        call("pqi_gains", ctypes.byref(self.w), _ptr(src), rows, _ptr(g32), _ptr(g64), wsp, wsn, self.sp())
        return g32, g64

    def calculate_cut(self, words: torch.Tensor, shots: int, is_spin_glass: bool, G: int, L: int, energies=True):
        """Batched scoring; words is tight [shots, n32]. Returns (energies|None, best_e, best_i) device tensors."""
        e = torch.empty(shots, dtype=torch.float32, device=self.device) if energies else None
        be = torch.empty(1, dtype=torch.float32, device=self.device)
        bi = torch.empty(1, dtype=torch.int32, device=self.device)
        wsp, wsn = self.wsp(shots)
        call(
            "pqi_calculate_cut",
            ctypes.byref(self.w),
            _ptr(words),
            shots,
            int(bool(is_spin_glass)),
            G,
            L,
            _ptr(e),
            _ptr(be),
            _ptr(bi),
            wsp,
            wsn,
            self.sp(),
        )
        return e, be, bi

    def single_bit_flips(self, words, is_spin_glass, G, L):
        be = torch.empty(1, dtype=torch.float32, device=self.device)
        bi = torch.empty(1, dtype=torch.int32, device=self.device)
        wsp, wsn = self.wsp(1)
        call("pqi_single_bit_flips", ctypes.byref(self.w), _ptr(words), int(bool(is_spin_glass)), G, L, _ptr(be), _ptr(bi), wsp, wsn, self.sp())
        return be, bi

    def double_bit_flips(self, words, g64, is_spin_glass, G, L, improving=False):
        """(best value, pair index) of one double-flip pass over all pairs
        (improving: accepted for the compressed-row graph's interface; the
        dense pass is always exact)."""
        be = torch.empty(1, dtype=torch.float32, device=self.device)
        bi = torch.empty(1, dtype=torch.int32, device=self.device)
        wsp, wsn = self.wsp(1)
        call("pqi_double_bit_flips", ctypes.byref(self.w), _ptr(words), _ptr(g64), int(bool(is_spin_glass)), G, L, _ptr(be), _ptr(bi), wsp, wsn, self.sp())
        return be, bi

    def select(self, values: torch.Tensor, G: int, L: int):
        be = torch.empty(1, dtype=torch.float32, device=self.device)
        bi = torch.empty(1, dtype=torch.int32, device=self.device)
        wsp, wsn = self.wsp(1)
        call("pqi_select", _ptr(values), values.numel(), G, L, _ptr(be), _ptr(bi), wsp, wsn, self.sp())
        return be, bi

    def gray(self, words64, g64, is_spin_glass, iters_bound, seeds):
        tout = torch.empty(seeds * self.n64 * 2, dtype=torch.int32, device=self.device)
        eout = torch.empty(seeds, dtype=torch.float32, device=self.device)
        wsp, wsn = self.wsp(seeds)
        call("pqi_gray", ctypes.byref(self.w), _ptr(words64), _ptr(g64), int(bool(is_spin_glass)), int(iters_bound), int(seeds), _ptr(tout), _ptr(eout), wsp, wsn, self.sp())
        return tout, eout

    def single_descent(self, words, g64, is_spin_glass, G, L, max_flips, trace=None):
        esum = torch.zeros(1, dtype=torch.float64, device=self.device)
        flips = torch.zeros(1, dtype=torch.int32, device=self.device)
        wsp, wsn = self.wsp(1)
        rc = _lib.status(
            "pqi_single_descent",
            ctypes.byref(self.w),
            _ptr(words),
            _ptr(g64),
            int(bool(is_spin_glass)),
            G,
            L,
            int(max_flips),
            _ptr(esum),
            _ptr(flips),
            _ptr(trace),
            wsp,
            wsn,
            self.sp(),
        )
        if rc not in (_lib.PQI_OK, _lib.PQI_ETIMEOUT):
            raise _lib.PQIError(rc, "pqi_single_descent")
        return esum, flips, rc

    def apply_flip(self, words, g64, k, l=-1):
        call("pqi_apply_flip", ctypes.byref(self.w), _ptr(words), _ptr(g64), int(k), int(l), self.sp())

    def rescore(self, words: torch.Tensor, rows: int = 1):
        """float64 (cut, energy) of `rows` states given as tight [rows, n32] words."""
        cut = torch.empty(rows, dtype=torch.float64, device=self.device)
        en = torch.empty(rows, dtype=torch.float64, device=self.device)
        wsp, wsn = self.wsp(rows)
        call("pqi_rescore_fp64", ctypes.byref(self.w), _ptr(words), rows, _ptr(cut), _ptr(en), wsp, wsn, self.sp())
        return cut, en
