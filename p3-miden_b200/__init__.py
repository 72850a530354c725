"""p3-miden_b200: B200-native lifted-STARK prover hot path.

Python mirror of the reference prover's public surface
(p3-miden-lifted-stark: ``prove_single`` / ``prove_multi``, ``PcsParams``,
``LmcsConfig``/``LmcsTree``, the DFT's ``coset_lde_batch``) over the C ABI
of ``libp3miden_b200.so`` (declared in include/p3g.h). All compute runs in
the CUDA library; this module only marshals arguments. If the library is
missing, every entry point raises: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import sys
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libp3miden_b200.so"
P = 0xFFFFFFFF00000001

AIR_CUBIC = 1
AIR_KECCAK = 2
KECCAK_NUM_COLS = 2633
KECCAK_ROWS_PER_HASH = 24

u64p = C.POINTER(C.c_uint64)

# status codes (include/p3g.h)
OK, ERR_INVALID, ERR_VALIDATION, ERR_OOM, ERR_TIMEOUT, ERR_CUDA = range(6)


class P3gError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"p3g status {status}: {what}")


_lib = None


def _load_build_module():
    spec = importlib.util.spec_from_file_location("p3g_build", HERE / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def build(force: bool = False) -> Path:
    return _load_build_module().build(force=force)


class PcsParamsC(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in (
        "log_blowup", "log_folding_arity", "log_final_degree",
        "folding_pow_bits", "deep_pow_bits", "num_queries", "query_pow_bits")]


class InstanceC(C.Structure):
    _fields_ = [("air", C.c_int32), ("trace_on_device", C.c_int32),
                ("height", C.c_uint64), ("width", C.c_uint64),
                ("trace", u64p), ("consts", u64p), ("n_consts", C.c_uint64)]


class ProofC(C.Structure):
    _fields_ = [("fields", u64p), ("n_fields", C.c_uint64),
                ("commits", u64p), ("n_commits", C.c_uint64),
                ("digest", C.c_uint64 * 12),
                ("stage_ms", C.c_double * 12),
                ("gpu_launches", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64)]


def lib():
    """Load the CUDA library; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run p3-miden_b200/build.py (no CPU fallback exists)")
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        sigs = {
            "p3g_ctx_create": (C.c_int, [C.c_int, u64p, C.POINTER(vp)]),
            "p3g_ctx_destroy": (None, [vp]),
            "p3g_last_error": (C.c_char_p, [vp]),
            "p3g_default_poseidon2_params": (None, [u64p]),
            "p3g_poseidon2_params_from_seed": (None, [C.c_uint64, u64p, u64p]),
            "p3g_coset_lde": (C.c_int, [vp, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint64, C.c_void_p]),
            "p3g_lmcs_build": (C.c_int, [vp, C.POINTER(C.c_void_p), u64p, u64p, C.c_uint64, C.c_uint32, C.POINTER(vp)]),
            "p3g_lmcs_root": (C.c_int, [vp, u64p]),
            "p3g_lmcs_layer": (C.c_int, [vp, vp, C.c_uint32, u64p]),
            "p3g_lmcs_free": (None, [vp]),
            "p3g_poseidon2_permute_batch": (C.c_int, [vp, C.c_void_p, C.c_uint64]),
        }
        optional = {
            "p3g_lmcs_prove_batch": (C.c_int, [vp, vp, u64p, C.c_uint64, u64p, u64p, u64p, u64p]),
            "p3g_grind": (C.c_int, [vp, u64p, u64p, C.c_uint32, C.c_uint32, u64p]),
            "p3g_prove": (C.c_int, [vp, C.POINTER(PcsParamsC), C.POINTER(InstanceC), C.c_uint64, C.POINTER(ProofC)]),
            "p3g_proof_free": (None, [C.POINTER(ProofC)]),
            "p3g_keccak_trace": (C.c_int, [u64p, C.c_uint64, C.c_uint32, u64p]),
            "p3g_keccak_inputs": (C.c_int, [C.c_uint64, C.c_uint64, u64p]),
            "p3g_cubic_trace": (C.c_int, [C.c_uint32, C.c_uint64, C.c_uint64, u64p, u64p]),
            "p3g_air_num_constraints": (C.c_uint64, [C.c_int32, C.c_uint64]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        for name, (res, args) in optional.items():
            if hasattr(L, name):
                fn = getattr(L, name)
                fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(u64p)


def default_poseidon2_params() -> np.ndarray:
    out = np.zeros(130, dtype=np.uint64)
    lib().p3g_default_poseidon2_params(_ptr(out))
    return out


def poseidon2_params_from_seed(seed: int, diag) -> np.ndarray:
    d = np.ascontiguousarray(np.array(diag, dtype=np.uint64))
    out = np.zeros(130, dtype=np.uint64)
    lib().p3g_poseidon2_params_from_seed(seed, _ptr(d), _ptr(out))
    return out


def _check(status: int, ctx=None):
    if status != OK:
        what = lib().p3g_last_error(ctx).decode() if ctx is not None else ""
        raise P3gError(status, what)


class Context:
    """One device, one stream; owns device memory between calls."""

    def __init__(self, device: int = 0, poseidon2_params: np.ndarray | None = None):
        params = default_poseidon2_params() if poseidon2_params is None else np.ascontiguousarray(poseidon2_params, dtype=np.uint64)
        assert params.shape == (130,)
        self._h = C.c_void_p()
        _check(lib().p3g_ctx_create(device, _ptr(params), C.byref(self._h)))
        self.device = device
        self.poseidon2_params = params

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().p3g_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, status: int):
        _check(status, self._h)


# ------------------------------------------------------------------ torch
def to_device(a: np.ndarray, device: int = 0):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64))
    return t.to(f"cuda:{device}")


def to_host(t) -> np.ndarray:
    return t.detach().cpu().numpy().view(np.uint64)


def empty_device(shape, device: int = 0):
    import torch
    return torch.empty(shape, dtype=torch.int64, device=f"cuda:{device}")


# ---------------------------------------------------------- stage seams
def coset_lde(ctx: Context, trace_dev, log_blowup: int, shift: int):
    """TwoAdicSubgroupDft::coset_lde_batch + bit_reverse_rows on a device matrix."""
    import torch
    h, w = trace_dev.shape
    torch.cuda.synchronize(ctx.device)
    out = empty_device((h << log_blowup, w), ctx.device)
    ctx.check(lib().p3g_coset_lde(ctx.handle, trace_dev.data_ptr(), h, w, log_blowup, shift, out.data_ptr()))
    return out


class LmcsTree:
    """LmcsTree over device matrices (ascending heights)."""

    def __init__(self, ctx: Context, mats_dev, alignment: int):
        import torch
        torch.cuda.synchronize(ctx.device)
        self.ctx = ctx
        self._keep = list(mats_dev)
        n = len(mats_dev)
        ptrs = (C.c_void_p * n)(*[m.data_ptr() for m in mats_dev])
        hs = np.array([m.shape[0] for m in mats_dev], dtype=np.uint64)
        ws = np.array([m.shape[1] for m in mats_dev], dtype=np.uint64)
        self._h = C.c_void_p()
        ctx.check(lib().p3g_lmcs_build(ctx.handle, ptrs, _ptr(hs), _ptr(ws), n, alignment, C.byref(self._h)))
        self.height = int(hs[-1])
        self.depth = self.height.bit_length() - 1

    def root(self) -> np.ndarray:
        r = np.zeros(4, dtype=np.uint64)
        _check(lib().p3g_lmcs_root(self._h, _ptr(r)))
        return r

    def layer(self, level: int) -> np.ndarray:
        n = self.height >> level
        out = np.zeros((n, 4), dtype=np.uint64)
        self.ctx.check(lib().p3g_lmcs_layer(self.ctx.handle, self._h, level, _ptr(out)))
        return out

    def prove_batch(self, indices):
        idx = np.array(sorted(set(int(i) for i in indices)), dtype=np.uint64)
        cap_f = len(idx) * sum(((m.shape[1] + 7) // 8) * 8 for m in self._keep) + 16
        cap_c = len(idx) * (self.depth + 1) + 4
        fields = np.zeros(cap_f, dtype=np.uint64)
        commits = np.zeros((cap_c, 4), dtype=np.uint64)
        nf = np.array([cap_f], dtype=np.uint64)
        nc = np.array([cap_c], dtype=np.uint64)
        self.ctx.check(lib().p3g_lmcs_prove_batch(self.ctx.handle, self._h, _ptr(idx), len(idx),
                                                  _ptr(fields), _ptr(nf), _ptr(commits.reshape(-1)), _ptr(nc)))
        return fields[: int(nf[0])], commits[: int(nc[0])]

    def __del__(self):
        try:
            if self._h:
                lib().p3g_lmcs_free(self._h)
        except Exception:
            pass


def poseidon2_permute_batch(ctx: Context, states_dev):
    import torch
    torch.cuda.synchronize(ctx.device)
    ctx.check(lib().p3g_poseidon2_permute_batch(ctx.handle, states_dev.data_ptr(), states_dev.shape[0]))
    return states_dev
