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

from . import symbolic
from .symbolic import AirDesc, SymbolicAirBuilder, build_air

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libp3miden_b200.so"
P = 0xFFFFFFFF00000001

AIR_CUBIC = 1
AIR_KECCAK = 2
AIR_SYMBOLIC = 3
KECCAK_NUM_COLS = 2633
KECCAK_ROWS_PER_HASH = 24

u64p = C.POINTER(C.c_uint64)

# status codes (include/p3g.h)
OK, ERR_INVALID, ERR_VALIDATION, ERR_OOM, ERR_TIMEOUT, ERR_CUDA, ERR_REJECTED = range(7)


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


# AuxBuilder::build_aux_trace (include/p3g.h, p3g_aux_build_fn)
AUX_BUILD_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(C.c_uint64), C.c_uint64,
                           C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64))


class InstanceC(C.Structure):
    _fields_ = [("air", C.c_int32), ("trace_on_device", C.c_int32),
                ("height", C.c_uint64), ("width", C.c_uint64),
                ("trace", u64p), ("consts", u64p), ("n_consts", C.c_uint64),
                ("sym", C.c_void_p), ("public_values", u64p), ("n_public_values", C.c_uint64),
                ("aux_build", AUX_BUILD_FN), ("aux_user", C.c_void_p)]


class AirDescC(C.Structure):
    _fields_ = [("main_width", C.c_uint32), ("aux_width", C.c_uint32), ("num_randomness", C.c_uint32),
                ("num_aux_values", C.c_uint32), ("num_public_values", C.c_uint32), ("num_periodic", C.c_uint32),
                ("periodic_lengths", u64p), ("periodic_values", u64p), ("nodes", C.c_void_p),
                ("n_nodes", C.c_uint64), ("constraints", C.POINTER(C.c_uint32)), ("is_ext", C.POINTER(C.c_uint8)),
                ("n_constraints", C.c_uint64)]


class ProofC(C.Structure):
    _fields_ = [("fields", u64p), ("n_fields", C.c_uint64),
                ("commits", u64p), ("n_commits", C.c_uint64),
                ("digest", C.c_uint64 * 12),
                ("stage_ms", C.c_double * 12),
                ("gpu_launches", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64)]


class VerifyStatsC(C.Structure):
    _fields_ = [("host_ms", C.c_double), ("device_ms", C.c_double), ("gpu_launches", C.c_uint64)]


class VerifyJobC(C.Structure):
    _fields_ = [("pcs", PcsParamsC), ("instances", C.POINTER(InstanceC)), ("n_instances", C.c_uint64),
                ("fields", u64p), ("n_fields", C.c_uint64), ("commits", u64p), ("n_commits", C.c_uint64),
                ("digest12", u64p)]


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
            "p3g_lmcs_build_hiding": (C.c_int, [vp, C.POINTER(C.c_void_p), u64p, u64p, C.c_uint64, C.c_uint32,
                                                C.c_void_p, C.c_uint64, C.POINTER(vp)]),
            "p3g_lmcs_open_batch": (C.c_int, [vp, u64p, u64p, C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, u64p,
                                              C.c_uint64, u64p, C.c_uint64, u64p, C.c_uint64, C.POINTER(C.c_int32)]),
            "p3g_lmcs_root": (C.c_int, [vp, u64p]),
            "p3g_periodic_lde": (C.c_int, [vp, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32,
                                           C.c_uint64, C.c_void_p]),
            "p3g_lmcs_layer": (C.c_int, [vp, vp, C.c_uint32, u64p]),
            "p3g_lmcs_free": (None, [vp]),
            "p3g_poseidon2_permute_batch": (C.c_int, [vp, C.c_void_p, C.c_uint64]),
        }
        optional = {
            "p3g_lmcs_prove_batch": (C.c_int, [vp, vp, u64p, C.c_uint64, u64p, u64p, u64p, u64p]),
            "p3g_grind": (C.c_int, [vp, u64p, u64p, C.c_uint32, C.c_uint32, u64p]),
            "p3g_prove": (C.c_int, [vp, C.POINTER(PcsParamsC), C.POINTER(InstanceC), C.c_uint64, C.POINTER(ProofC)]),
            "p3g_proof_free": (None, [C.POINTER(ProofC)]),
            "p3g_proof_wire_size": (C.c_uint64, [C.POINTER(ProofC)]),
            "p3g_proof_serialize": (C.c_int, [C.POINTER(ProofC), C.c_char_p, C.c_uint64, C.POINTER(C.c_uint64)]),
            "p3g_proof_deserialize": (C.c_int, [C.c_char_p, C.c_uint64, C.POINTER(ProofC)]),
            "p3g_keccak_trace": (C.c_int, [u64p, C.c_uint64, C.c_uint32, u64p]),
            "p3g_keccak_trace_device": (C.c_int, [vp, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]),
            "p3g_keccak_inputs": (C.c_int, [C.c_uint64, C.c_uint64, u64p]),
            "p3g_cubic_trace": (C.c_int, [C.c_uint32, C.c_uint64, C.c_uint64, u64p, u64p]),
            "p3g_air_num_constraints": (C.c_uint64, [C.c_int32, C.c_uint64]),
            "p3g_cubic_trace_device": (C.c_int, [vp, C.c_uint32, C.c_uint64, C.c_uint64, u64p, C.c_void_p]),
            "p3g_autotune_lde": (C.c_int, [vp, C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32,
                                           C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_double),
                                           C.POINTER(C.c_double)]),
            "p3g_autotune_slabs": (C.c_int, [vp, C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32,
                                             C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
            "p3g_ctx_set_lde_split": (C.c_int, [vp, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32]),
            "p3g_ctx_set_slab_columns": (C.c_int, [vp, C.c_uint64]),
            "p3g_ctx_memory_stats": (C.c_int, [vp, u64p, u64p, C.POINTER(C.c_double)]),
            "p3g_verify": (C.c_int, [vp, C.POINTER(PcsParamsC), C.POINTER(InstanceC), C.c_uint64, u64p, C.c_uint64,
                                     u64p, C.c_uint64, u64p, C.POINTER(C.c_int32), C.POINTER(VerifyStatsC)]),
            "p3g_verify_batch": (C.c_int, [vp, C.POINTER(VerifyJobC), C.c_uint64, C.c_uint32, C.POINTER(C.c_int32),
                                           C.POINTER(VerifyStatsC)]),
            "p3g_lmcs_rows": (C.c_int, [vp, vp, C.c_uint64, u64p, C.POINTER(C.c_uint64)]),
            "p3g_fri_fold": (C.c_int, [vp, C.c_void_p, C.c_uint32, C.c_uint32, u64p, C.c_void_p]),
            "p3g_deep_evals": (C.c_int, [vp, C.POINTER(C.c_void_p), u64p, u64p, C.c_uint64, C.c_uint32, u64p, u64p]),
            "p3g_deep_quotient": (C.c_int, [vp, C.POINTER(C.c_void_p), u64p, u64p, C.c_uint64, C.c_uint32, C.c_uint32,
                                            u64p, u64p, u64p, u64p, C.c_void_p]),
            "p3g_air_analyse": (C.c_int, [C.POINTER(AirDescC), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                          C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
            "p3g_air_generate_source": (C.c_int, [C.POINTER(AirDescC), C.c_char_p, C.c_uint64,
                                                  C.POINTER(C.c_uint64)]),
            "p3g_air_create": (C.c_int, [vp, C.POINTER(AirDescC), C.POINTER(vp)]),
            "p3g_air_compile_check": (C.c_int, [C.POINTER(AirDescC), C.c_int32, C.POINTER(C.c_uint64)]),
            "p3g_air_log_quotient_degree": (C.c_uint32, [vp]),
            "p3g_air_max_degree": (C.c_uint32, [vp]),
            "p3g_air_num_constraints_of": (C.c_uint64, [vp]),
            "p3g_air_num_kernels": (C.c_uint64, [vp]),
            "p3g_ctx_set_air_chunk_nodes": (C.c_int, [vp, C.c_uint64]),
            "p3g_air_layout": (C.c_int, [vp, u64p, C.POINTER(C.c_uint64), u64p, C.POINTER(C.c_uint64)]),
            "p3g_air_free": (None, [vp]),
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

    # ---- launch-shape tuning (p3g_autotune_*, p3g_ctx_set_*)
    def autotune_lde(self, log_h: int, width: int, log_blowup: int, reps: int = 3) -> dict:
        """Time the candidate bit-range splits of a 2^log_h x width coset LDE;
        the fastest is kept for this context. Returns it with both times."""
        sizes = (C.c_uint32 * 8)()
        n, best, dflt = C.c_uint32(8), C.c_double(), C.c_double()
        self.check(lib().p3g_autotune_lde(self._h, log_h, width, log_blowup, reps, sizes, C.byref(n), C.byref(best),
                                          C.byref(dflt)))
        return {"log_h": log_h, "width": width, "log_blowup": log_blowup, "split": list(sizes[:n.value]),
                "ms": best.value, "default_ms": dflt.value}

    def autotune_slabs(self, log_h: int, width: int, log_blowup: int, reps: int = 2) -> dict:
        """Time the main commit for several column-slab widths; the fastest is
        kept for this context (0 = the default rule)."""
        cols, best, dflt = C.c_uint64(), C.c_double(), C.c_double()
        self.check(lib().p3g_autotune_slabs(self._h, log_h, width, log_blowup, reps, C.byref(cols), C.byref(best),
                                            C.byref(dflt)))
        return {"log_h": log_h, "width": width, "log_blowup": log_blowup, "slab_cols": cols.value, "ms": best.value,
                "default_ms": dflt.value}

    def set_lde_split(self, log_h: int, sizes):
        arr = (C.c_uint32 * max(1, len(sizes)))(*sizes)
        self.check(lib().p3g_ctx_set_lde_split(self._h, log_h, arr, len(sizes)))

    def set_slab_columns(self, cols: int):
        self.check(lib().p3g_ctx_set_slab_columns(self._h, cols))

    def set_air_chunk_nodes(self, nodes: int):
        """DAG nodes per generated constraint kernel of symbolic AIRs created
        on this context from now on (0: the default)."""
        self.check(lib().p3g_ctx_set_air_chunk_nodes(self._h, nodes))

    def memory_stats(self) -> dict:
        """The context pool's reserved and used bytes, and the host ms spent in
        allocation calls since the context was created."""
        r, u, ms = C.c_uint64(), C.c_uint64(), C.c_double()
        self.check(lib().p3g_ctx_memory_stats(self._h, C.byref(r), C.byref(u), C.byref(ms)))
        return {"reserved_bytes": r.value, "used_bytes": u.value, "alloc_ms": ms.value}

    def load_tuning(self, table: dict):
        """Apply a saved tuning table ({"lde_split": {L: [..]}, "slab_cols": n})."""
        for L, sizes in table.get("lde_split", {}).items():
            self.set_lde_split(int(L), sizes)
        if table.get("slab_cols"):
            self.set_slab_columns(int(table["slab_cols"]))


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


def periodic_lde(ctx: Context, repeated_dev, log_blowup: int, log_trace_height: int, lde_shift: int = 7):
    """PeriodicLde::build (p3-miden-lifted-stark/src/prover/periodic.rs:49-81):
    periodic columns repeated to the largest period (a device matrix), extended
    on the period's coset in natural order; row i of the trace's LDE is row
    i mod the result's height."""
    import torch
    torch.cuda.synchronize(ctx.device)
    p, w = repeated_dev.shape
    out = empty_device((p << log_blowup, w), ctx.device)
    ctx.check(lib().p3g_periodic_lde(ctx.handle, repeated_dev.data_ptr(), p, w, log_blowup, log_trace_height,
                                     lde_shift, out.data_ptr()))
    return out


class LmcsTree:
    """LmcsTree over device matrices (ascending heights). With `salt_dev`
    (tree height x SALT, on the device) the hiding LMCS
    (p3-miden-lmcs/src/hiding_lmcs.rs): each leaf absorbs its salt row last,
    and openings carry the salt after the rows."""

    def __init__(self, ctx: Context, mats_dev, alignment: int, salt_dev=None):
        import torch
        torch.cuda.synchronize(ctx.device)
        self.ctx = ctx
        self._keep = list(mats_dev)
        n = len(mats_dev)
        ptrs = (C.c_void_p * n)(*[m.data_ptr() for m in mats_dev])
        hs = np.array([m.shape[0] for m in mats_dev], dtype=np.uint64)
        ws = np.array([m.shape[1] for m in mats_dev], dtype=np.uint64)
        self._h = C.c_void_p()
        self.salt_width = 0
        self.alignment = alignment
        self.widths = [int(w) for w in ws]
        if salt_dev is None:
            ctx.check(lib().p3g_lmcs_build(ctx.handle, ptrs, _ptr(hs), _ptr(ws), n, alignment, C.byref(self._h)))
        else:
            assert salt_dev.shape[0] == int(hs[-1])
            self._salt = salt_dev
            self.salt_width = int(salt_dev.shape[1])
            ctx.check(lib().p3g_lmcs_build_hiding(ctx.handle, ptrs, _ptr(hs), _ptr(ws), n, alignment,
                                                  salt_dev.data_ptr(), self.salt_width, C.byref(self._h)))
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

    def rows(self, index: int) -> np.ndarray:
        """LmcsTree::rows (p3-miden-lmcs/src/lifted_tree.rs:127-138): the row of
        every matrix at this leaf (lifted), each padded to the alignment."""
        n = C.c_uint64(0)
        lib().p3g_lmcs_rows(self.ctx.handle, self._h, index, _ptr(np.zeros(1, dtype=np.uint64)), C.byref(n))
        out = np.zeros(max(1, n.value), dtype=np.uint64)
        self.ctx.check(lib().p3g_lmcs_rows(self.ctx.handle, self._h, index, _ptr(out), C.byref(n)))
        return out[:n.value]

    def prove_batch(self, indices):
        idx = np.array(sorted(set(int(i) for i in indices)), dtype=np.uint64)
        cap_f = len(idx) * (sum(((m.shape[1] + 7) // 8) * 8 for m in self._keep) + self.salt_width) + 16
        cap_c = len(idx) * (self.depth + 1) + 4
        fields = np.zeros(cap_f, dtype=np.uint64)
        commits = np.zeros((cap_c, 4), dtype=np.uint64)
        nf = np.array([cap_f], dtype=np.uint64)
        nc = np.array([cap_c], dtype=np.uint64)
        self.ctx.check(lib().p3g_lmcs_prove_batch(self.ctx.handle, self._h, _ptr(idx), len(idx),
                                                  _ptr(fields), _ptr(nf), _ptr(commits.reshape(-1)), _ptr(nc)))
        return fields[: int(nf[0])], commits[: int(nc[0])]

    def open_batch(self, indices, fields, commits, commitment=None) -> int:
        """Lmcs::open_batch of hints from prove_batch against this tree's root
        (or `commitment`), hashed on the device; returns the verdict
        (0 = accepted, else VERDICTS: opening, root or transcript)."""
        idx = np.array(sorted(set(int(i) for i in indices)), dtype=np.uint64)
        root = np.ascontiguousarray(self.root() if commitment is None else commitment, dtype=np.uint64)
        w = np.array(self.widths, dtype=np.uint64)
        f = np.ascontiguousarray(fields, dtype=np.uint64).reshape(-1)
        c = np.ascontiguousarray(commits, dtype=np.uint64).reshape(-1)
        v = C.c_int32(-1)
        self.ctx.check(lib().p3g_lmcs_open_batch(self.ctx.handle, _ptr(root), _ptr(w), w.size, self.alignment,
                                                 self.salt_width, self.depth, _ptr(idx) if idx.size else None,
                                                 idx.size, _ptr(f) if f.size else None, f.size,
                                                 _ptr(c) if c.size else None, c.size // 4, C.byref(v)))
        return int(v.value)

    def __del__(self):
        try:
            if self._h:
                lib().p3g_lmcs_free(self._h)
        except Exception:
            pass


def fri_fold(ctx: Context, layer_dev, log_arity: int, beta) -> object:
    """FriFold::fold_matrix (p3-miden-lifted-fri/src/fri/fold/mod.rs:119-181) of a
    bit-reversed layer of n EF values (device tensor n x 2) with challenge beta
    (c0, c1): the n / 2^log_arity folded values."""
    n = layer_dev.shape[0]
    log_n = n.bit_length() - 1
    assert n == 1 << log_n and layer_dev.shape[1] == 2
    out = empty_device((n >> log_arity, 2), ctx.device)
    b = np.array(beta, dtype=np.uint64)
    import torch
    torch.cuda.synchronize(ctx.device)
    ctx.check(lib().p3g_fri_fold(ctx.handle, layer_dev.data_ptr(), log_n, log_arity, _ptr(b), out.data_ptr()))
    return out


def _mat_args(mats_dev):
    ptrs = (C.c_void_p * len(mats_dev))(*[m.data_ptr() for m in mats_dev])
    hs = np.array([m.shape[0] for m in mats_dev], dtype=np.uint64)
    ws = np.array([m.shape[1] for m in mats_dev], dtype=np.uint64)
    return ptrs, hs, ws


def deep_evals(ctx: Context, mats_dev, log_blowup: int, zs) -> np.ndarray:
    """DEEP openings: f(z_0), f(z_1) of every column of the committed
    (bit-reversed LDE) matrices, ascending heights; (total columns, 2 points, 2)."""
    import torch
    torch.cuda.synchronize(ctx.device)
    ptrs, hs, ws = _mat_args(mats_dev)
    z = np.array([zs[0][0], zs[0][1], zs[1][0], zs[1][1]], dtype=np.uint64)
    out = np.zeros(4 * int(ws.sum()), dtype=np.uint64)
    ctx.check(lib().p3g_deep_evals(ctx.handle, ptrs, _ptr(hs), _ptr(ws), len(mats_dev), log_blowup, _ptr(z), _ptr(out)))
    return out.reshape(-1, 2, 2)


def deep_quotient(ctx: Context, mats_dev, log_blowup: int, alignment: int, zs, evals, alpha, beta):
    """The DEEP quotient over the committed matrices (n EF on the LDE domain,
    bit-reversed; device tensor n x 2)."""
    import torch
    torch.cuda.synchronize(ctx.device)
    ptrs, hs, ws = _mat_args(mats_dev)
    z = np.array([zs[0][0], zs[0][1], zs[1][0], zs[1][1]], dtype=np.uint64)
    ev = np.ascontiguousarray(evals, dtype=np.uint64).reshape(-1)
    a = np.array(alpha, dtype=np.uint64)
    b = np.array(beta, dtype=np.uint64)
    out = empty_device((int(hs[-1]), 2), ctx.device)
    ctx.check(lib().p3g_deep_quotient(ctx.handle, ptrs, _ptr(hs), _ptr(ws), len(mats_dev), log_blowup, alignment,
                                      _ptr(z), _ptr(ev), _ptr(a), _ptr(b), out.data_ptr()))
    return out


def poseidon2_permute_batch(ctx: Context, states_dev):
    import torch
    torch.cuda.synchronize(ctx.device)
    ctx.check(lib().p3g_poseidon2_permute_batch(ctx.handle, states_dev.data_ptr(), states_dev.shape[0]))
    return states_dev


# -------------------------------------------------------------- prover
@dataclass(frozen=True)
class PcsParams:
    """PcsParams::new argument order (p3-miden-lifted-fri/src/params.rs:170-178)."""
    log_blowup: int
    log_folding_arity: int
    log_final_degree: int
    folding_pow_bits: int
    deep_pow_bits: int
    num_queries: int
    query_pow_bits: int

    def as_c(self) -> PcsParamsC:
        return PcsParamsC(self.log_blowup, self.log_folding_arity, self.log_final_degree,
                          self.folding_pow_bits, self.deep_pow_bits, self.num_queries, self.query_pow_bits)


def _desc_c(desc, keep) -> AirDescC:
    """p3g_air_desc of a symbolic.AirDesc (arrays kept alive in `keep`)."""
    nodes = np.ascontiguousarray(desc.nodes, dtype=symbolic.NODE_DTYPE)
    cons = np.ascontiguousarray(desc.constraints, dtype=np.uint32)
    ext = np.ascontiguousarray(desc.is_ext, dtype=np.uint8)
    pl = np.ascontiguousarray(desc.periodic_lengths, dtype=np.uint64)
    pv = np.ascontiguousarray(desc.periodic_values, dtype=np.uint64)
    keep += [nodes, cons, ext, pl, pv]
    return AirDescC(desc.width, desc.aux_width, desc.num_randomness, desc.num_aux_values, desc.num_public_values,
                    desc.num_periodic, _ptr(pl) if pl.size else None, _ptr(pv) if pv.size else None,
                    nodes.ctypes.data if nodes.size else None, nodes.size,
                    cons.ctypes.data_as(C.POINTER(C.c_uint32)) if cons.size else None,
                    ext.ctypes.data_as(C.POINTER(C.c_uint8)) if ext.size else None, cons.size)


def air_analyse(desc) -> dict:
    """Degree analysis of a symbolic AIR without a device: the maximal
    degree multiple, log_quotient_degree (air.rs:225-247) and the numbers of
    base and extension constraints (ConstraintLayout)."""
    keep = []
    d = _desc_c(desc, keep)
    md, lq, nb, ne = C.c_uint32(), C.c_uint32(), C.c_uint64(), C.c_uint64()
    _check(lib().p3g_air_analyse(C.byref(d), C.byref(md), C.byref(lq), C.byref(nb), C.byref(ne)))
    return {"max_degree": md.value, "log_quotient_degree": lq.value, "n_base": nb.value, "n_ext": ne.value}


def air_source(desc) -> str:
    """The CUDA source the library generates for this AIR's constraint kernel."""
    keep = []
    d = _desc_c(desc, keep)
    n = C.c_uint64()
    lib().p3g_air_generate_source(C.byref(d), None, 0, C.byref(n))
    buf = C.create_string_buffer(n.value)
    _check(lib().p3g_air_generate_source(C.byref(d), buf, n.value, C.byref(n)))
    return buf.value.decode()


def air_compile_check(desc, cc: int = 100) -> int:
    """Generate this AIR's constraint kernel and compile it with NVRTC for
    sm_<cc>a without a device; returns the cubin size."""
    keep = []
    d = _desc_c(desc, keep)
    n = C.c_uint64()
    _check(lib().p3g_air_compile_check(C.byref(d), cc, C.byref(n)))
    return n.value


class Air:
    """A symbolic AIR compiled for one device (p3g_air_create): the DAG of a
    symbolic.AirDesc, its degree analysis and its generated constraint
    kernel."""

    def __init__(self, ctx: "Context", desc):
        self.desc = desc
        keep = []
        d = _desc_c(desc, keep)
        self._h = C.c_void_p()
        ctx.check(lib().p3g_air_create(ctx.handle, C.byref(d), C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    @property
    def log_quotient_degree(self) -> int:
        return int(lib().p3g_air_log_quotient_degree(self._h))

    @property
    def max_degree(self) -> int:
        return int(lib().p3g_air_max_degree(self._h))

    @property
    def num_kernels(self) -> int:
        """Generated constraint kernels (chunks of the constraint DAG)."""
        return int(lib().p3g_air_num_kernels(self._h))

    def layout(self):
        """ConstraintLayout: (base_indices, ext_indices) in emission order."""
        nb, ne = C.c_uint64(self.desc.num_constraints), C.c_uint64(self.desc.num_constraints)
        b = np.zeros(max(1, nb.value), dtype=np.uint64)
        e = np.zeros(max(1, ne.value), dtype=np.uint64)
        _check(lib().p3g_air_layout(self._h, _ptr(b), C.byref(nb), _ptr(e), C.byref(ne)))
        return b[:nb.value].copy(), e[:ne.value].copy()

    def close(self):
        if self._h:
            lib().p3g_air_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def aux_builder_c(fn):
    """Wrap fn(instance, randomness, height) -> (aux, aux_values) as the
    C callback (AuxBuilder::build_aux_trace): randomness is a list of
    (c0, c1) extension elements; aux is height x (2 * aux_width) words (each
    EF column as its two coordinates), aux_values 2 words per value."""
    def cb(user, instance, main_trace, rnd, n_rnd, height, aux_out, vals_out):
        try:
            r = [(int(rnd[2 * i]), int(rnd[2 * i + 1])) for i in range(n_rnd)]
            aux, vals = fn(int(instance), r, int(height))
            aux = np.ascontiguousarray(aux, dtype=np.uint64).reshape(-1)
            vals = np.ascontiguousarray(vals, dtype=np.uint64).reshape(-1)
            C.memmove(aux_out, aux.ctypes.data, aux.nbytes)
            if vals.size:
                C.memmove(vals_out, vals.ctypes.data, vals.nbytes)
            return 0
        except Exception:
            return 1
    return AUX_BUILD_FN(cb)


@dataclass
class AirWitness:
    """One instance: the AIR (a built-in id, or an Air for a symbolic AIR),
    the row-major trace (numpy host array or torch CUDA tensor of int64 bit
    patterns), the AIR's constants (cubic: k[w]), its public values and its
    AuxBuilder, fn(instance, randomness, height) -> (aux, aux_values)
    (None: the all-zero aux trace)."""
    air: object
    trace: object
    consts: np.ndarray | None = None
    public_values: np.ndarray | None = None
    aux_builder: object = None


def _instance_c(air, height, width, trace_ptr, on_dev, consts, public_values, aux_builder, keep) -> InstanceC:
    c = np.ascontiguousarray(consts if consts is not None else np.zeros(0), dtype=np.uint64)
    pv = np.ascontiguousarray(public_values if public_values is not None else np.zeros(0), dtype=np.uint64)
    keep += [c, pv]
    sym = None
    if isinstance(air, Air):
        sym, air = air.handle, AIR_SYMBOLIC
    cb = AUX_BUILD_FN()
    if aux_builder is not None:
        cb = aux_builder_c(aux_builder)
        keep.append(cb)
    return InstanceC(air, on_dev, height, width, C.cast(C.c_void_p(trace_ptr), u64p) if trace_ptr else None,
                     c.ctypes.data_as(u64p) if c.size else None, c.size, sym,
                     pv.ctypes.data_as(u64p) if pv.size else None, pv.size, cb, None)


@dataclass
class TranscriptData:
    fields: np.ndarray
    commitments: np.ndarray  # (n, 4)

    def to_bytes(self) -> bytes:
        """Raw payload: field words then commitment words, little-endian u64."""
        return self.fields.astype("<u8").tobytes() + self.commitments.astype("<u8").tobytes()


def proof_to_wire(digest: np.ndarray, proof: TranscriptData) -> bytes:
    """p3g_proof_serialize: the library's wire format of a proof."""
    f = np.ascontiguousarray(proof.fields, dtype=np.uint64)
    c = np.ascontiguousarray(proof.commitments, dtype=np.uint64).reshape(-1)
    p = ProofC()
    p.fields, p.n_fields = f.ctypes.data_as(u64p), f.size
    p.commits, p.n_commits = c.ctypes.data_as(u64p), c.size // 4
    for i in range(12):
        p.digest[i] = int(digest[i])
    n = int(lib().p3g_proof_wire_size(C.byref(p)))
    buf = C.create_string_buffer(n)
    ln = C.c_uint64()
    _check(lib().p3g_proof_serialize(C.byref(p), buf, n, C.byref(ln)))
    return buf.raw[: ln.value]


def proof_from_wire(data: bytes) -> tuple[np.ndarray, TranscriptData]:
    """p3g_proof_deserialize: (digest, TranscriptData); raises on a malformed buffer."""
    p = ProofC()
    _check(lib().p3g_proof_deserialize(data, len(data), C.byref(p)))
    try:
        fields = np.ctypeslib.as_array(p.fields, shape=(p.n_fields,)).copy() if p.n_fields else np.zeros(0, np.uint64)
        commits = (np.ctypeslib.as_array(p.commits, shape=(p.n_commits * 4,)).reshape(-1, 4).copy()
                   if p.n_commits else np.zeros((0, 4), np.uint64))
        return np.array(p.digest[:], dtype=np.uint64), TranscriptData(fields, commits)
    finally:
        lib().p3g_proof_free(C.byref(p))


@dataclass
class StarkOutput:
    digest: np.ndarray
    proof: TranscriptData
    stage_ms: list
    gpu_launches: int
    h2d_bytes: int
    d2h_bytes: int
    device_ms: float  # whole proof on the device timeline (CUDA events)
    lde_kernel_ms: float = 0.0  # main-trace coset-LDE kernels (events on their stream)
    leaf_kernel_ms: float = 0.0  # main-tree leaf-sponge launches (events on the prover stream)
    leaf_launches: int = 0


# Device-timeline stages of one proof. "main LDE" ends when the last column
# slab of the main LDE is written (the leaf hash of earlier slabs runs
# concurrently); "main tree" is the remaining hash and the compression.
STAGES = ("main LDE", "main tree", "commit aux", "constraints", "commit quotient", "DEEP", "FRI commit", "queries")


def prove_multi(ctx: Context, pcs: PcsParams, instances: list[AirWitness]) -> StarkOutput:
    """prove_multi (p3-miden-lifted-stark/src/prover/mod.rs:223-461) on the GPU.

    Instances must be in ascending height order. The challenger starts from
    the configuration's fresh DuplexChallenger state."""
    n = len(instances)
    arr = (InstanceC * max(1, n))()
    keep = []
    for i, w in enumerate(instances):
        t = w.trace
        if isinstance(t, np.ndarray):
            t = np.ascontiguousarray(t, dtype=np.uint64)
            keep.append(t)
            ptr, on_dev = t.ctypes.data, 0
            h, wd = t.shape
        else:  # torch tensor (host pinned or CUDA)
            keep.append(t)
            ptr, on_dev = t.data_ptr(), int(t.is_cuda)
            h, wd = t.shape
        arr[i] = _instance_c(w.air, h, wd, ptr, on_dev, w.consts, w.public_values, w.aux_builder, keep)
    if any(not isinstance(w.trace, np.ndarray) and w.trace.is_cuda for w in instances):
        import torch
        torch.cuda.synchronize(ctx.device)
    pc = pcs.as_c()
    out = ProofC()
    ctx.check(lib().p3g_prove(ctx.handle, C.byref(pc), arr, n, C.byref(out)))
    try:
        fields = np.ctypeslib.as_array(out.fields, shape=(out.n_fields,)).copy()
        commits = np.ctypeslib.as_array(out.commits, shape=(out.n_commits * 4,)).reshape(-1, 4).copy()
        res = StarkOutput(np.array(out.digest[:], dtype=np.uint64), TranscriptData(fields, commits),
                          list(out.stage_ms[:len(STAGES)]), int(out.gpu_launches), int(out.h2d_bytes),
                          int(out.d2h_bytes), float(out.stage_ms[11]), float(out.stage_ms[8]),
                          float(out.stage_ms[9]), int(out.stage_ms[10]))
    finally:
        lib().p3g_proof_free(C.byref(out))
    return res


def prove_single(ctx: Context, pcs: PcsParams, witness: AirWitness) -> StarkOutput:
    return prove_multi(ctx, pcs, [witness])


# ------------------------------------------------------------- verifier
VERDICTS = ("accept", "shape", "opening", "root", "pow", "deep", "fri", "final", "quotient", "transcript",
            "digest")


@dataclass
class AirShape:
    """The verifier's view of one instance: the AIR (built-in id or Air),
    trace height and width, the AIR's constants (cubic: k[w]) and its public
    values."""
    air: object
    height: int
    width: int
    consts: np.ndarray | None = None
    public_values: np.ndarray | None = None


@dataclass
class VerifyResult:
    verdict: int  # 0 = accepted, else the first failing check (VERDICTS)
    host_ms: float
    device_ms: float
    gpu_launches: int

    @property
    def ok(self) -> bool:
        return self.verdict == 0

    @property
    def name(self) -> str:
        return VERDICTS[self.verdict]


def verify_multi(ctx: Context, pcs: PcsParams, shapes: list[AirShape], fields: np.ndarray,
                 commitments: np.ndarray, digest: np.ndarray) -> VerifyResult:
    """verify_multi (p3-miden-lifted-stark/src/verifier/mod.rs:170-364) of a
    proof of prove_multi, with the opening, DEEP and FRI query checks on the
    GPU. Raises on a bad argument (including a transcript word >= p); a
    rejected proof is a verdict, not an exception."""
    n = len(shapes)
    arr = (InstanceC * max(1, n))()
    keep = []
    for i, sh in enumerate(shapes):
        arr[i] = _instance_c(sh.air, sh.height, sh.width, 0, 0, sh.consts, sh.public_values, None, keep)
    f = np.ascontiguousarray(fields, dtype=np.uint64).reshape(-1)
    cm = np.ascontiguousarray(commitments, dtype=np.uint64).reshape(-1)
    dg = np.ascontiguousarray(digest, dtype=np.uint64).reshape(-1)
    assert dg.size == 12 and cm.size % 4 == 0
    pc = pcs.as_c()
    verdict = C.c_int32(-1)
    st = VerifyStatsC()
    ctx.check(lib().p3g_verify(ctx.handle, C.byref(pc), arr, n, _ptr(f), f.size, _ptr(cm), cm.size // 4, _ptr(dg),
                               C.byref(verdict), C.byref(st)))
    return VerifyResult(int(verdict.value), float(st.host_ms), float(st.device_ms), int(st.gpu_launches))


def verify_output(ctx: Context, pcs: PcsParams, shapes: list[AirShape], out: StarkOutput) -> VerifyResult:
    return verify_multi(ctx, pcs, shapes, out.proof.fields, out.proof.commitments, out.digest)


def verify_batch(ctx: Context, items, host_threads: int = 0) -> tuple[list[int], VerifyResult]:
    """verify_multi of several proofs in one call: items are
    (pcs, shapes, fields, commitments, digest); the host replays run on
    host_threads threads (0: all), then one device pass checks every proof.
    Returns the verdicts (0 = accepted) and the call's timing."""
    n = len(items)
    jobs = (VerifyJobC * max(1, n))()
    keep = []
    for i, (pcs, shapes, fields, commits, digest) in enumerate(items):
        arr = (InstanceC * max(1, len(shapes)))()
        for k, sh in enumerate(shapes):
            arr[k] = _instance_c(sh.air, sh.height, sh.width, 0, 0, sh.consts, sh.public_values, None, keep)
        f = np.ascontiguousarray(fields, dtype=np.uint64).reshape(-1)
        cm = np.ascontiguousarray(commits, dtype=np.uint64).reshape(-1)
        dg = np.ascontiguousarray(digest, dtype=np.uint64).reshape(-1)
        keep += [arr, f, cm, dg]
        jobs[i] = VerifyJobC(pcs.as_c(), arr, len(shapes), _ptr(f), f.size, _ptr(cm), cm.size // 4, _ptr(dg))
    verdicts = (C.c_int32 * max(1, n))()
    st = VerifyStatsC()
    ctx.check(lib().p3g_verify_batch(ctx.handle, jobs, n, host_threads, verdicts, C.byref(st)))
    return [int(verdicts[i]) for i in range(n)], VerifyResult(0, float(st.host_ms), float(st.device_ms),
                                                             int(st.gpu_launches))


# ------------------------------------------------------- trace builders
def keccak_inputs(seed: int, n_perms: int) -> np.ndarray:
    out = np.zeros((n_perms, 25), dtype=np.uint64)
    _check(lib().p3g_keccak_inputs(seed, n_perms, _ptr(out)))
    return out


def generate_keccak_trace(inputs: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
    """p3-miden-lifted-examples/src/keccak.rs:54-56: next_power_of_two(24 * n) rows."""
    inputs = np.ascontiguousarray(inputs, dtype=np.uint64).reshape(-1, 25)
    n = inputs.shape[0]
    h = max(1, n * KECCAK_ROWS_PER_HASH)
    log_h = (h - 1).bit_length()
    if out is None:
        out = np.empty((1 << log_h, KECCAK_NUM_COLS), dtype=np.uint64)
    _check(lib().p3g_keccak_trace(_ptr(inputs), n, log_h, out.ctypes.data_as(u64p)))
    return out


def generate_keccak_trace_device(ctx: Context, inputs_dev, log_h: int | None = None, out=None):
    """generate_trace_rows on the device: inputs_dev is a device tensor of
    n_perms x 25 words (int64 view); returns a device tensor of
    2^log_h x 2633 (default: the smallest height that holds the rows)."""
    import torch
    n = int(inputs_dev.shape[0])
    if log_h is None:
        log_h = max(0, (24 * n - 1).bit_length()) if n else 0
    if out is None:
        out = empty_device((1 << log_h, KECCAK_NUM_COLS), ctx.device)
    torch.cuda.synchronize(ctx.device)
    ctx.check(lib().p3g_keccak_trace_device(ctx.handle, inputs_dev.data_ptr() if n else None, n, log_h,
                                            out.data_ptr()))
    return out


def generate_cubic_trace_device(ctx: Context, log_h: int, width: int, seed: int, out=None):
    """The cubic AIR's trace generated on the device (forward iteration there;
    k and row 0 from the seeded RNG): returns (k, device tensor)."""
    if out is None:
        out = empty_device((1 << log_h, width), ctx.device)
    k = np.zeros(width, dtype=np.uint64)
    import torch
    torch.cuda.synchronize(ctx.device)
    ctx.check(lib().p3g_cubic_trace_device(ctx.handle, log_h, width, seed, _ptr(k), out.data_ptr()))
    return k, out


def generate_cubic_trace(log_h: int, width: int, seed: int, out: np.ndarray | None = None):
    k = np.zeros(width, dtype=np.uint64)
    if out is None:
        out = np.empty((1 << log_h, width), dtype=np.uint64)
    _check(lib().p3g_cubic_trace(log_h, width, seed, _ptr(k), out.ctypes.data_as(u64p)))
    return k, out


# ---------------------------------------------------- batched / serving
class JobC(C.Structure):
    _fields_ = [("pcs", PcsParamsC), ("instances", C.POINTER(InstanceC)), ("n_instances", C.c_uint64),
                ("arrival_s", C.c_double)]


class JobResultC(C.Structure):
    _fields_ = [("status", C.c_int32), ("verdict", C.c_int32), ("proof", ProofC),
                ("submit_s", C.c_double), ("start_s", C.c_double), ("end_s", C.c_double), ("verify_ms", C.c_double)]


@dataclass
class Job:
    pcs: PcsParams
    instances: list  # list[AirWitness]
    arrival_s: float = 0.0


@dataclass
class JobResult:
    status: int
    output: StarkOutput | None
    submit_s: float
    start_s: float
    end_s: float
    verdict: int = -1  # self-check verdict (VERDICTS index), -1 when not checked
    verify_ms: float = 0.0

    @property
    def latency_s(self) -> float:
        return self.end_s - self.submit_s


def _instances_c(instances, keep):
    arr = (InstanceC * max(1, len(instances)))()
    for i, w in enumerate(instances):
        t = w.trace
        if isinstance(t, np.ndarray):
            t = np.ascontiguousarray(t, dtype=np.uint64)
            ptr, on_dev = t.ctypes.data, 0
        else:
            ptr, on_dev = t.data_ptr(), int(t.is_cuda)
        keep.append(t)
        h, wd = t.shape
        arr[i] = _instance_c(w.air, h, wd, ptr, on_dev, w.consts, w.public_values, w.aux_builder, keep)
    keep.append(arr)
    return arr


def _result_from_c(r: JobResultC) -> JobResult:
    out = None
    if r.status == OK:
        p = r.proof
        fields = np.ctypeslib.as_array(p.fields, shape=(p.n_fields,)).copy()
        commits = np.ctypeslib.as_array(p.commits, shape=(p.n_commits * 4,)).reshape(-1, 4).copy()
        out = StarkOutput(np.array(p.digest[:], dtype=np.uint64), TranscriptData(fields, commits),
                          list(p.stage_ms[:len(STAGES)]), int(p.gpu_launches), int(p.h2d_bytes),
                          int(p.d2h_bytes), float(p.stage_ms[11]))
        lib().p3g_proof_free(C.byref(r.proof))
    return JobResult(int(r.status), out, r.submit_s, r.start_s, r.end_s, int(r.verdict), float(r.verify_ms))


class ProofServer:
    """Batched / continuous-batching prover: n_workers concurrent proofs on one
    device, admitted by estimated HBM footprint against hbm_budget bytes."""

    def __init__(self, device: int = 0, n_workers: int = 4, hbm_budget: int = 150 * 10**9,
                 poseidon2_params: np.ndarray | None = None, self_check: bool = False,
                 max_heavy: int = 1):
        L = lib()
        vp = C.c_void_p
        for name, res, args in [
            ("p3g_server_create", C.c_int, [C.c_int, u64p, C.c_uint32, C.c_uint64, C.POINTER(vp)]),
            ("p3g_server_destroy", None, [vp]),
            ("p3g_server_submit", C.c_int, [vp, C.POINTER(JobC), u64p]),
            ("p3g_server_wait", C.c_int, [vp, C.c_uint64, C.POINTER(JobResultC)]),
            ("p3g_server_run", C.c_int, [vp, C.POINTER(JobC), C.c_uint64, C.POINTER(JobResultC)]),
            ("p3g_server_peak_admitted_bytes", C.c_uint64, [vp]),
            ("p3g_server_set_self_check", C.c_int, [vp, C.c_int32]),
            ("p3g_server_set_lde_split", C.c_int, [vp, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32]),
            ("p3g_server_set_slab_columns", C.c_int, [vp, C.c_uint64]),
            ("p3g_server_set_max_heavy", C.c_int, [vp, C.c_uint32]),
            ("p3g_job_footprint_bytes", C.c_uint64, [C.POINTER(PcsParamsC), C.POINTER(InstanceC), C.c_uint64]),
        ]:
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        params = default_poseidon2_params() if poseidon2_params is None else np.ascontiguousarray(poseidon2_params, dtype=np.uint64)
        self._h = C.c_void_p()
        _check(L.p3g_server_create(device, _ptr(params), n_workers, int(hbm_budget), C.byref(self._h)))
        self.n_workers = n_workers
        self._pending = {}
        if self_check:
            _check(L.p3g_server_set_self_check(self._h, 1))
        if max_heavy != 1:  # heavy jobs (LDEs above 2^26 words) allowed at once; 0: no limit
            _check(L.p3g_server_set_max_heavy(self._h, max_heavy))

    def load_tuning(self, table: dict):
        """Apply a saved tuning table to every worker (Context.load_tuning's format)."""
        L = lib()
        for lh, sizes in table.get("lde_split", {}).items():
            arr = (C.c_uint32 * max(1, len(sizes)))(*sizes)
            _check(L.p3g_server_set_lde_split(self._h, int(lh), arr, len(sizes)))
        if table.get("slab_cols"):
            _check(L.p3g_server_set_slab_columns(self._h, int(table["slab_cols"])))

    def run(self, jobs: list[Job]) -> list[JobResult]:
        """Submit every job at its arrival time (seconds from now) and wait for all."""
        keep = []
        arr = (JobC * max(1, len(jobs)))()
        for i, j in enumerate(jobs):
            ins = _instances_c(j.instances, keep)
            arr[i] = JobC(j.pcs.as_c(), ins, len(j.instances), float(j.arrival_s))
        res = (JobResultC * max(1, len(jobs)))()
        _check(lib().p3g_server_run(self._h, arr, len(jobs), res))
        return [_result_from_c(res[i]) for i in range(len(jobs))]

    def submit(self, job: Job) -> int:
        keep = []
        ins = _instances_c(job.instances, keep)
        jc = JobC(job.pcs.as_c(), ins, len(job.instances), 0.0)
        t = C.c_uint64()
        _check(lib().p3g_server_submit(self._h, C.byref(jc), C.byref(t)))
        self._pending[t.value] = keep
        return t.value

    def wait(self, ticket: int) -> JobResult:
        r = JobResultC()
        lib().p3g_server_wait(self._h, ticket, C.byref(r))
        self._pending.pop(ticket, None)
        return _result_from_c(r)

    def peak_admitted_bytes(self) -> int:
        return int(lib().p3g_server_peak_admitted_bytes(self._h))

    @staticmethod
    def footprint_bytes(pcs: PcsParams, instances) -> int:
        keep = []
        ins = _instances_c(instances, keep)
        pc = pcs.as_c()
        return int(lib().p3g_job_footprint_bytes(C.byref(pc), ins, len(instances)))

    def close(self):
        if self._h:
            lib().p3g_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
