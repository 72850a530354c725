"""ctypes binding of the CPU oracle (oracle/build/liboracle.so).

Test infrastructure only: the oracle is the checker for the CUDA product and
is never part of the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
LIB_PATH = ORACLE_DIR / "build" / "liboracle.so"

P = 0xFFFFFFFF00000001
AIR_CUBIC = 1
AIR_KECCAK = 2

u64p = C.POINTER(C.c_uint64)


class PcsParams(C.Structure):
    _fields_ = [(n, C.c_uint) for n in (
        "log_blowup", "log_folding_arity", "log_final_degree",
        "folding_pow_bits", "deep_pow_bits", "num_queries", "query_pow_bits")]


AIR_SYMBOLIC = 3
# or_aux_fn: the AuxBuilder callback (same signature as the product's)
AUX_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(C.c_uint64), C.c_uint64, C.c_uint64,
                     C.POINTER(C.c_uint64), C.POINTER(C.c_uint64))


class EF(C.Structure):
    _fields_ = [("c0", C.c_uint64), ("c1", C.c_uint64)]


class SymAir(C.Structure):
    _fields_ = [("main_width", C.c_uint32), ("aux_width", C.c_uint32), ("num_randomness", C.c_uint32),
                ("num_aux_values", C.c_uint32), ("num_public_values", C.c_uint32), ("num_periodic", C.c_uint32),
                ("periodic_lengths", u64p), ("periodic_values", u64p), ("nodes", C.c_void_p),
                ("n_nodes", C.c_size_t), ("constraints", C.POINTER(C.c_uint32)), ("is_ext", C.POINTER(C.c_uint8)),
                ("n_constraints", C.c_size_t)]


class Instance(C.Structure):
    _fields_ = [("air", C.c_int), ("height", C.c_size_t), ("width", C.c_size_t),
                ("trace", u64p), ("consts", u64p), ("sym", C.POINTER(SymAir)), ("public_values", u64p),
                ("aux_build", AUX_FN), ("aux_user", C.c_void_p)]


class Proof(C.Structure):
    _fields_ = [("fields", u64p), ("n_fields", C.c_size_t),
                ("commits", u64p), ("n_commits", C.c_size_t),
                ("digest", C.c_uint64 * 12),
                ("main_root", C.c_uint64 * 4), ("aux_root", C.c_uint64 * 4),
                ("quot_root", C.c_uint64 * 4),
                ("alpha", C.c_uint64 * 2), ("beta", C.c_uint64 * 2), ("z", C.c_uint64 * 2),
                ("deep_alpha", C.c_uint64 * 2), ("deep_beta", C.c_uint64 * 2)]


class P2Params(C.Structure):
    _fields_ = [("rc_init", C.c_uint64 * 48), ("rc_term", C.c_uint64 * 48),
                ("rc_int", C.c_uint64 * 22), ("diag", C.c_uint64 * 12)]


class Matrix(C.Structure):
    _fields_ = [("data", u64p), ("height", C.c_size_t), ("width", C.c_size_t)]


class Tree(C.Structure):
    _fields_ = [("n_mats", C.c_size_t), ("mats", Matrix * 8), ("alignment", C.c_size_t),
                ("depth", C.c_uint), ("layers", u64p), ("layer_off", C.c_size_t * 40),
                ("salt", u64p), ("salt_width", C.c_size_t)]


class Challenger(C.Structure):
    _fields_ = [("pp", C.c_void_p), ("state", C.c_uint64 * 12), ("inp", C.c_uint64 * 8),
                ("out", C.c_uint64 * 8), ("n_in", C.c_int), ("n_out", C.c_int)]


class Transcript(C.Structure):
    _fields_ = [("ch", Challenger), ("fields", u64p), ("n_fields", C.c_size_t),
                ("cap_fields", C.c_size_t), ("commits", u64p), ("n_commits", C.c_size_t),
                ("cap_commits", C.c_size_t)]


_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in [
            ("or_x_mul", C.c_uint64, [C.c_uint64, C.c_uint64]),
            ("or_x_mul_ref", C.c_uint64, [C.c_uint64, C.c_uint64]),
            ("or_x_add", C.c_uint64, [C.c_uint64, C.c_uint64]),
            ("or_x_sub", C.c_uint64, [C.c_uint64, C.c_uint64]),
            ("or_x_inv", C.c_uint64, [C.c_uint64]),
            ("or_x_root", C.c_uint64, [C.c_uint]),
            ("or_x_ef_mul", None, [u64p, u64p, u64p]),
            ("or_x_ef_inv", None, [u64p, u64p]),
            ("or_p2_default_params", None, [C.POINTER(P2Params)]),
            ("or_p2_placeholder_diag", None, [u64p]),
            ("or_p2_params_from_seed", None, [C.POINTER(P2Params), C.c_uint64, u64p]),
            ("or_p2_permute", None, [C.POINTER(P2Params), u64p]),
            ("or_sponge_absorb", None, [C.POINTER(P2Params), u64p, u64p, C.c_size_t]),
            ("or_compress", None, [C.POINTER(P2Params), u64p, u64p, u64p]),
            ("or_rng_seed", None, [u64p, C.c_uint64]),
            ("or_rng_next", C.c_uint64, [u64p]),
            ("or_rng_field", C.c_uint64, [u64p]),
            ("or_ntt", None, [u64p, C.c_size_t]),
            ("or_intt", None, [u64p, C.c_size_t]),
            ("or_coset_lde_bitrev", None, [u64p, C.c_size_t, C.c_size_t, C.c_uint, C.c_uint64, u64p]),
            ("or_periodic_lde", None, [u64p, C.c_size_t, C.c_size_t, C.c_uint, C.c_uint, C.c_uint64, u64p]),
            ("or_tree_build", None, [C.POINTER(P2Params), C.POINTER(Tree), C.POINTER(Matrix), C.c_size_t, C.c_size_t]),
            ("or_tree_root", None, [C.POINTER(Tree), u64p]),
            ("or_tree_build_hiding", None, [C.POINTER(P2Params), C.POINTER(Tree), C.POINTER(Matrix), C.c_size_t,
                                            C.c_size_t, u64p, C.c_size_t]),
            ("or_tree_free", None, [C.POINTER(Tree)]),
            ("or_tree_prove_batch", None, [C.POINTER(Tree), C.POINTER(C.c_size_t), C.c_size_t, C.POINTER(Transcript)]),
            ("or_tr_init", None, [C.POINTER(Transcript), C.POINTER(P2Params)]),
            ("or_tr_free", None, [C.POINTER(Transcript)]),
            ("or_ch_init", None, [C.POINTER(Challenger), C.POINTER(P2Params)]),
            ("or_ch_observe", None, [C.POINTER(Challenger), C.c_uint64]),
            ("or_ch_sample", C.c_uint64, [C.POINTER(Challenger)]),
            ("or_ch_sample_bits", C.c_uint64, [C.POINTER(Challenger), C.c_uint]),
            ("or_ch_grind", C.c_uint64, [C.POINTER(Challenger), C.c_uint]),
            ("or_ch_finalize", None, [C.POINTER(Challenger), u64p]),
            ("or_air_num_constraints", C.c_size_t, [C.c_int, C.c_size_t]),
            ("or_air_eval", None, [C.c_int, C.c_size_t, u64p, u64p, u64p, u64p, u64p]),
            ("or_cubic_trace", None, [C.c_size_t, C.c_size_t, C.c_uint64, u64p, u64p]),
            ("or_keccak_num_cols", C.c_size_t, []),
            ("or_keccak_trace", None, [u64p, C.c_size_t, C.c_size_t, u64p]),
            ("or_keccak_inputs", None, [C.c_uint64, C.c_size_t, u64p]),
            ("or_check_constraints", C.c_size_t, [C.c_int, C.c_size_t, C.c_size_t, u64p, u64p]),
            ("or_prove", C.c_int, [C.POINTER(P2Params), C.POINTER(PcsParams), C.POINTER(Instance), C.c_size_t, C.POINTER(Proof)]),
            ("or_proof_free", None, [C.POINTER(Proof)]),
            ("or_last_stage_seconds", C.c_double, [C.c_int]),
            ("or_verify", C.c_int, [C.POINTER(P2Params), C.POINTER(PcsParams), C.POINTER(Instance), C.c_size_t,
                                    u64p, C.c_size_t, u64p, C.c_size_t, u64p]),
            ("or_sym_validate", C.c_int, [C.POINTER(SymAir)]),
            ("or_deep_evals", None, [C.POINTER(Matrix), C.c_size_t, C.c_uint, u64p, u64p]),
            ("or_deep_quotient", None, [C.POINTER(Matrix), C.c_size_t, C.c_uint, C.c_size_t, u64p, u64p,
                                        EF, EF, u64p]),
            ("or_fri_fold", None, [u64p, C.c_uint, C.c_uint, u64p, u64p]),
            ("or_sym_max_degree", C.c_uint, [C.POINTER(SymAir)]),
            ("or_sym_log_quotient_degree", C.c_uint, [C.POINTER(SymAir)]),
        ]:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(u64p)


def default_p2() -> P2Params:
    pp = P2Params()
    lib().or_p2_default_params(C.byref(pp))
    return pp


def p2_to_array(pp: P2Params) -> np.ndarray:
    """Flatten to the product's layout: rc_init[48], rc_term[48], rc_int[22], diag[12]."""
    return np.frombuffer(bytes(pp), dtype=np.uint64).copy()


def p2_from_array(a) -> P2Params:
    """The inverse of p2_to_array: 130 words -> oracle parameters."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    assert a.size == 130
    return P2Params.from_buffer_copy(a.tobytes())


def periodic_lde(repeated: np.ndarray, log_blowup: int, log_trace_height: int, lde_shift: int) -> np.ndarray:
    """PeriodicLde::build: natural-order LDE of the repeated periodic columns."""
    r = np.ascontiguousarray(repeated, dtype=np.uint64)
    p, w = r.shape
    out = np.zeros((p << log_blowup, w), dtype=np.uint64)
    lib().or_periodic_lde(ptr(r), p, w, log_blowup, log_trace_height, lde_shift, ptr(out))
    return out


def permute(pp: P2Params, st) -> np.ndarray:
    a = np.array(st, dtype=np.uint64)
    lib().or_p2_permute(C.byref(pp), ptr(a))
    return a


def coset_lde_bitrev(trace: np.ndarray, log_blowup: int, shift: int) -> np.ndarray:
    h, w = trace.shape
    out = np.zeros((h << log_blowup, w), dtype=np.uint64)
    t = np.ascontiguousarray(trace, dtype=np.uint64)
    lib().or_coset_lde_bitrev(ptr(t), h, w, log_blowup, shift, ptr(out))
    return out


class OracleTree:
    """LMCS tree over row-major matrices (ascending heights); with `salt`
    (tree height x SALT) the hiding LMCS."""

    def __init__(self, pp: P2Params, mats, alignment: int, salt=None):
        self._keep = [np.ascontiguousarray(m, dtype=np.uint64) for m in mats]
        arr = (Matrix * len(mats))()
        for i, m in enumerate(self._keep):
            arr[i] = Matrix(ptr(m), m.shape[0], m.shape[1])
        self.t = Tree()
        self.pp = pp
        if salt is None:
            lib().or_tree_build(C.byref(pp), C.byref(self.t), arr, len(mats), alignment)
        else:
            s = np.ascontiguousarray(salt, dtype=np.uint64)
            self._keep.append(s)
            lib().or_tree_build_hiding(C.byref(pp), C.byref(self.t), arr, len(mats), alignment, ptr(s), s.shape[1])

    def root(self) -> np.ndarray:
        r = np.zeros(4, dtype=np.uint64)
        lib().or_tree_root(C.byref(self.t), ptr(r))
        return r

    def layer(self, l: int) -> np.ndarray:
        n = 1 << (self.t.depth - l)
        off = self.t.layer_off[l]
        buf = np.ctypeslib.as_array(self.t.layers, shape=((2 << self.t.depth) * 4,))
        return buf[off * 4:(off + n) * 4].reshape(n, 4).copy()

    def prove_batch(self, indices) -> tuple[np.ndarray, np.ndarray]:
        idx = sorted(set(int(i) for i in indices))
        arr = (C.c_size_t * max(1, len(idx)))(*idx)
        tr = Transcript()
        lib().or_tr_init(C.byref(tr), C.byref(self.pp))
        lib().or_tree_prove_batch(C.byref(self.t), arr, len(idx), C.byref(tr))
        f = np.ctypeslib.as_array(tr.fields, shape=(tr.n_fields,)).copy() if tr.n_fields else np.zeros(0, np.uint64)
        c = (np.ctypeslib.as_array(tr.commits, shape=(tr.n_commits * 4,)).reshape(-1, 4).copy()
             if tr.n_commits else np.zeros((0, 4), np.uint64))
        lib().or_tr_free(C.byref(tr))
        return f, c

    def __del__(self):
        try:
            lib().or_tree_free(C.byref(self.t))
        except Exception:
            pass


def cubic_trace(log_h: int, width: int, seed: int):
    k = np.zeros(width, dtype=np.uint64)
    t = np.zeros((1 << log_h, width), dtype=np.uint64)
    lib().or_cubic_trace(log_h, width, seed, ptr(k), ptr(t))
    return k, t


def keccak_inputs(seed: int, n_perms: int) -> np.ndarray:
    out = np.zeros((n_perms, 25), dtype=np.uint64)
    lib().or_keccak_inputs(seed, n_perms, ptr(out))
    return out


def keccak_trace(inputs: np.ndarray, log_h: int) -> np.ndarray:
    w = lib().or_keccak_num_cols()
    t = np.zeros((1 << log_h, w), dtype=np.uint64)
    inp = np.ascontiguousarray(inputs, dtype=np.uint64)
    lib().or_keccak_trace(ptr(inp), inp.shape[0], log_h, ptr(t))
    return t


def check_constraints(air: int, trace: np.ndarray, consts=None) -> int:
    h, w = trace.shape
    c = np.ascontiguousarray(consts if consts is not None else np.zeros(1), dtype=np.uint64)
    t = np.ascontiguousarray(trace, dtype=np.uint64)
    return int(lib().or_check_constraints(air, h, w, ptr(c), ptr(t)))


def sym_air(desc, keep) -> SymAir:
    """The oracle's view of a symbolic AIR description (the product's
    symbolic.AirDesc: the same node layout)."""
    nodes = np.ascontiguousarray(desc.nodes)
    cons = np.ascontiguousarray(desc.constraints, dtype=np.uint32)
    ext = np.ascontiguousarray(desc.is_ext, dtype=np.uint8)
    pl = np.ascontiguousarray(desc.periodic_lengths, dtype=np.uint64)
    pv = np.ascontiguousarray(desc.periodic_values, dtype=np.uint64)
    keep += [nodes, cons, ext, pl, pv]
    a = SymAir(desc.width, desc.aux_width, desc.num_randomness, desc.num_aux_values, desc.num_public_values,
               pl.size, ptr(pl) if pl.size else None, ptr(pv) if pv.size else None, nodes.ctypes.data,
               nodes.size, cons.ctypes.data_as(C.POINTER(C.c_uint32)), ext.ctypes.data_as(C.POINTER(C.c_uint8)),
               cons.size)
    keep.append(a)
    return a


def sym_degree(desc):
    keep = []
    a = sym_air(desc, keep)
    return int(lib().or_sym_max_degree(C.byref(a))), int(lib().or_sym_log_quotient_degree(C.byref(a)))


def aux_fn(fn, keep):
    """fn(instance, randomness [(c0, c1)], height) -> (aux words h x 2*aux_width, aux value words)."""
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
    f = AUX_FN(cb)
    keep.append(f)
    return f


def _instance(air, h, w, trace_ptr, consts, extra, keep) -> Instance:
    """extra: None, or a dict with 'sym' (AirDesc), 'public_values', 'aux_builder'."""
    c = np.ascontiguousarray(consts if consts is not None else np.zeros(1), dtype=np.uint64)
    keep.append(c)
    extra = extra or {}
    sym = None
    if extra.get("sym") is not None:
        sym = C.pointer(sym_air(extra["sym"], keep))
        air = AIR_SYMBOLIC
    pv = np.ascontiguousarray(extra.get("public_values") if extra.get("public_values") is not None
                              else np.zeros(1), dtype=np.uint64)
    keep.append(pv)
    fb = aux_fn(extra["aux_builder"], keep) if extra.get("aux_builder") is not None else AUX_FN()
    return Instance(air, h, w, trace_ptr, ptr(c), sym, ptr(pv), fb, None)


def prove(pp: P2Params, pcs: dict, instances):
    """instances: list of (air, trace ndarray, consts ndarray|None[, extra])
    where extra holds a symbolic AIR ('sym'), its 'public_values' and its
    'aux_builder'. Returns a dict."""
    keep = []
    arr = (Instance * len(instances))()
    for i, inst in enumerate(instances):
        air, trace, consts = inst[:3]
        t = np.ascontiguousarray(trace, dtype=np.uint64)
        keep.append(t)
        arr[i] = _instance(air, t.shape[0], t.shape[1], ptr(t), consts, inst[3] if len(inst) > 3 else None, keep)
    pr = PcsParams(**pcs)
    proof = Proof()
    rc = lib().or_prove(C.byref(pp), C.byref(pr), arr, len(instances), C.byref(proof))
    if rc != 0:
        raise ValueError(f"oracle prove failed with status {rc}")
    out = {
        "fields": np.ctypeslib.as_array(proof.fields, shape=(proof.n_fields,)).copy(),
        "commits": np.ctypeslib.as_array(proof.commits, shape=(proof.n_commits * 4,)).reshape(-1, 4).copy(),
        "digest": np.array(proof.digest[:], dtype=np.uint64),
    }
    for k in ("main_root", "aux_root", "quot_root", "alpha", "beta", "z", "deep_alpha", "deep_beta"):
        out[k] = np.array(getattr(proof, k)[:], dtype=np.uint64)
    out["stage_seconds"] = [lib().or_last_stage_seconds(i) for i in range(7)]
    lib().or_proof_free(C.byref(proof))
    return out


VERIFY_ERRORS = {0: "accepted", 1: "shape", 2: "opening index", 3: "LMCS root", 4: "proof of work",
                 5: "DEEP point on domain", 6: "FRI row", 7: "final polynomial", 8: "quotient identity",
                 9: "transcript length", 10: "digest"}
VERIFY_ERRORS_CODE = {v: k for k, v in VERIFY_ERRORS.items()}


def verify(pp: P2Params, pcs: dict, instances, fields, commits, digest) -> int:
    """Verifier restatement: instances are (air, height, width, consts|None),
    in ascending height order; returns 0 when the proof is accepted, else an
    error code (VERIFY_ERRORS)."""
    keep = []
    arr = (Instance * len(instances))()
    dummy = np.zeros(1, dtype=np.uint64)
    for i, inst in enumerate(instances):
        air, h, w, consts = inst[:4]
        arr[i] = _instance(air, h, w, ptr(dummy), consts, inst[4] if len(inst) > 4 else None, keep)
    f = np.ascontiguousarray(fields, dtype=np.uint64)
    cm = np.ascontiguousarray(np.asarray(commits, dtype=np.uint64).reshape(-1))
    d = np.ascontiguousarray(digest, dtype=np.uint64)
    pr = PcsParams(**pcs)
    return int(lib().or_verify(C.byref(pp), C.byref(pr), arr, len(instances), ptr(f), f.size,
                               ptr(cm) if cm.size else ptr(dummy), cm.size // 4, ptr(d)))


def _mats(mats, keep):
    arr = (Matrix * len(mats))()
    for i, m in enumerate(mats):
        a = np.ascontiguousarray(m, dtype=np.uint64)
        keep.append(a)
        arr[i] = Matrix(ptr(a), a.shape[0], a.shape[1])
    return arr


def deep_evals(mats, log_blowup: int, zs) -> np.ndarray:
    """or_deep_evals: (total columns, 2 points, 2 words)."""
    keep = []
    arr = _mats(mats, keep)
    z = np.array([zs[0][0], zs[0][1], zs[1][0], zs[1][1]], dtype=np.uint64)
    out = np.zeros(4 * sum(m.shape[1] for m in mats), dtype=np.uint64)
    lib().or_deep_evals(arr, len(mats), log_blowup, ptr(z), ptr(out))
    return out.reshape(-1, 2, 2)


def deep_quotient(mats, log_blowup: int, alignment: int, zs, evals, alpha, beta) -> np.ndarray:
    keep = []
    arr = _mats(mats, keep)
    z = np.array([zs[0][0], zs[0][1], zs[1][0], zs[1][1]], dtype=np.uint64)
    ev = np.ascontiguousarray(evals, dtype=np.uint64).reshape(-1)
    out = np.zeros((mats[-1].shape[0], 2), dtype=np.uint64)
    lib().or_deep_quotient(arr, len(mats), log_blowup, alignment, ptr(z), ptr(ev), EF(*alpha), EF(*beta), ptr(out))
    return out


def fri_fold(layer: np.ndarray, log_arity: int, beta) -> np.ndarray:
    l = np.ascontiguousarray(layer, dtype=np.uint64)
    n = l.shape[0]
    out = np.zeros((n >> log_arity, 2), dtype=np.uint64)
    b = np.array(beta, dtype=np.uint64)
    lib().or_fri_fold(ptr(l), n.bit_length() - 1, log_arity, ptr(b), ptr(out))
    return out


def set_threads(n: int):
    os.environ["OMP_NUM_THREADS"] = str(n)
