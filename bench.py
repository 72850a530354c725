#!/usr/bin/env python3
"""Benchmark: proofs/s of the lifted-STARK prover on the Keccak workload.

Workload (one step = one full prove_multi of one proof): the Keccak-f[1600]
AIR with 10922 seeded random permutations padded to 2^18 rows x 2633
Goldilocks columns, Goldilocks/Poseidon2 configuration, log_blowup 1, FRI
arity 2, final degree 0, folding PoW 16 bits, 100 queries (the plain
prover-at-scale configuration). Synthetic, seeded inputs.

Arms:
  default          the CUDA prover (libp3miden_b200.so) on N GPUs, one
                   independent proof per GPU per step (replicas; weak scaling)
  --impl reference the CPU restatement of the reference prover (oracle/) on
                   the host cores, on a bounded sample of the same workload

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
N_PERMS = 10922
LOG_H = 18  # overridden by --log-h for small profiling cases
PCS = dict(log_blowup=1, log_folding_arity=1, log_final_degree=0, folding_pow_bits=16,
           deep_pow_bits=0, num_queries=100, query_pow_bits=0)
METRIC = "proofs/s"
# ncu summaries of the current kernels (profiles/): per-launch instruction
# counts, pipe utilisation and DRAM traffic, each with the command that made it
HASH_PROFILE = ROOT / "profiles" / "leaf_class_kernel_slab_2e18.json"
# the same kernel writing the column-major rows the generated constraint
# kernels read (the headline's main commit with a symbolic AIR)
HASH_PROFILE_CM = ROOT / "profiles" / "leaf_class_kernel_cm_2e15.json"
LDE_PROFILE = ROOT / "profiles" / "lde_kernels_slab_2e18.json"


def workload_name() -> str:
    return (f"keccak-f1600 AIR, {N_PERMS} perms -> 2^{LOG_H} x 2633 Goldilocks trace, "
            f"lifted STARK (Poseidon2-12 LMCS)")


def base_config() -> dict:
    """The workload description shared by both arms (the GPU prover and the
    CPU reference arm) so that their lines name the same configuration."""
    return {"workload": workload_name(), "pcs": PCS}


TUNING = ROOT / "p3-miden_b200" / "tuning" / "b200.json"


def apply_tuning(ctx):
    """Launch shapes chosen by p3-miden_b200/autotune.py on a B200, if saved
    (a Context or a ProofServer)."""
    try:
        table = json.loads(TUNING.read_text())
    except Exception:
        return None
    ctx.load_tuning(table)
    return str(TUNING.relative_to(ROOT))


def load_profile(path: Path):
    try:
        return json.loads(path.read_text())
    except Exception:
        return None


def load_product():
    pkg = ROOT / "p3-miden_b200"
    spec = importlib.util.spec_from_file_location("p3_miden_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["p3_miden_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        fd, name = tempfile.mkstemp(prefix=f"p3g_clocks_gpu{gpu}_", suffix=".csv")
        os.close(fd)
        self.path = Path(name)

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in self.path.read_text().strip().splitlines() if r.strip()]
            sm = [float(r[1]) for r in rows]
            mx = max(float(r[2]) for r in rows)
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        finally:
            try:
                self.path.unlink()
            except OSError:
                pass


def dist_setup(backend: str = "nccl"):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        # short timeout: a rank that never arrives ends the others' next collective with an error
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def _scalar(v: float, dev):
    import torch
    return torch.tensor([v], dtype=torch.float64, device="cpu" if dev is None else f"cuda:{dev}")


def barrier(pg, dev):
    """All ranks meet; dev None means a CPU (gloo) group."""
    if pg is not None:
        t = _scalar(0.0, dev)
        pg.all_reduce(t)
        if dev is not None:
            import torch
            torch.cuda.synchronize(dev)


def max_over_ranks(pg, v: float, dev) -> float:
    if pg is None:
        return v
    t = _scalar(v, dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, v: float, dev) -> float:
    if pg is None:
        return v
    t = _scalar(v, dev)
    pg.all_reduce(t)
    return float(t.item())


def aggregate(pg, proofs: float, device_s: float, dev):
    """Replica aggregation: whole-job proofs/s = proofs of all ranks / the
    slowest rank's device time (weak scaling, no data-path collective)."""
    t = max_over_ranks(pg, device_s, dev)
    total = sum_over_ranks(pg, proofs, dev)
    return total / t, t, total


# ---------------------------------------------------------------- CPU arm
def oracle_proof_seconds(log_h: int, threads: int) -> float:
    """One full oracle proof (the CPU restatement of the reference prover) of
    a 2^log_h-row Keccak trace with the workload's parameters."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ffi as O
    trace = O.keccak_trace(O.keccak_inputs(1, (1 << log_h) // 24), log_h)
    t0 = time.perf_counter()
    O.prove(O.default_p2(), PCS, [(O.AIR_KECCAK, trace, None)])
    return time.perf_counter() - t0


def affine_extrapolation(samples: dict) -> tuple[float, float, float]:
    """Proof time on the CPU as a + b * rows, fitted to sample proofs of two
    heights {log_h: seconds}; returns (seconds at 2^LOG_H, a, b). Fixed costs
    (grinding, the FRI tail, thread start-up) dominate small samples, so a
    linear scaling from one sample overstates the CPU's time; this model
    matched a measured 2^18 oracle proof within 6 % (421 s measured on 8
    cores, 433 s predicted from 2^12 and 2^13 samples)."""
    (l0, t0), (l1, t1) = sorted(samples.items())
    b = (t1 - t0) / ((1 << l1) - (1 << l0))
    a = t0 - b * (1 << l0)
    return a + b * (1 << LOG_H), a, b


def run_reference(args):
    """The CPU arm: the oracle (a plain-C restatement of the reference prover;
    the Rust reference cannot be built without a Rust toolchain) on all host
    cores. Steps alternate full oracle proofs of 2^12- and 2^13-row samples of
    the workload (the same parameters; about 10 and 14 s on 16 cores), so
    that the whole run ends within minutes; ms_per_step is the mean sample
    time, and value extrapolates the per-height medians to the 2^18 workload
    with the affine model of affine_extrapolation."""
    # CPU-only arm with no collectives: under torchrun, rank 0 alone runs and prints
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    threads = os.cpu_count() or 1
    sizes = (12, 13)
    for i in range(args.warmup):
        oracle_proof_seconds(sizes[i % 2], threads)
    times = {sz: [] for sz in sizes}
    all_t = []
    for i in range(args.steps):
        t = oracle_proof_seconds(sizes[i % 2], threads)
        times[sizes[i % 2]].append(t)
        all_t.append(t)
    if not times[sizes[1]]:  # a single step: time the other height once more
        times[sizes[1]].append(oracle_proof_seconds(sizes[1], threads))
    per_proof, a, b = affine_extrapolation({k: statistics.median(v) for k, v in times.items()})
    value = 1.0 / per_proof
    sample = (f"full oracle proofs of 2^12- and 2^13-row Keccak samples (170 and 341 perms, same parameters), "
              f"alternating per step on {threads} threads; medians "
              f"{statistics.median(times[12]):.2f} s and {statistics.median(times[13]):.2f} s, extrapolated as "
              f"{a:.1f} s + {b * 1e3:.3f} ms per row to 2^{LOG_H} rows ({per_proof:.0f} s per proof)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(all_t) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Goldilocks, exact)",
        "data": "synthetic (seeded Keccak-f inputs)",
        "config": base_config(),
        "arm": {"parallelism": f"{threads} host threads (OpenMP)", "ms_per_proof_extrapolated": per_proof * 1e3,
                "step": "a 2^12- or 2^13-row sample proof"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def slab_widths(w: int):
    """Column slabs of the main commit (prover.cuh commit_main_pipelined)."""
    sw = ((w + 7) // 8 + 7) // 8 * 8 if w >= 256 else w
    return [min(sw, w - c0) for c0 in range(0, w, sw)]


def hash_roofline(n_lde: int, w: int, leaf_ms: float, n_launches: int, hbm_peak: float, peak_src: str,
                  sm_mhz, profile: Path = HASH_PROFILE):
    """Roofline line of the dominant kernel, merkle::leaf_class_kernel (one
    launch per column slab). It is bound by the integer ALU pipe: achieved =
    this run's ALU-pipe warp instructions per second (the live launch time
    times the per-permutation ALU count of the committed ncu summary), peak =
    the pipe's rate at this run's SM clock (from the same summary's
    instruction count and % of peak). The HBM figures sit beside it."""
    n_launches = max(1, n_launches)
    launch_s = leaf_ms / 1e3 / n_launches
    perms = n_lde * sum((x + 7) // 8 for x in slab_widths(w))
    perms_per_launch = perms / n_launches
    alg_bytes = 8.0 * n_lde * w / n_launches
    hbm_gbs = alg_bytes / launch_s / 1e9
    hbm = {"achieved": hbm_gbs, "peak": hbm_peak, "unit": "GB/s", "frac": hbm_gbs / hbm_peak,
           "peak_source": peak_src, "algorithmic_bytes": alg_bytes}
    base = {"kernel": "merkle::leaf_class_kernel (LMCS leaf sponge, Poseidon2-12)", "kernel_ms": launch_s * 1e3,
            "launches_per_proof": n_launches, "perms_per_launch": perms_per_launch,
            "perms_per_s": perms_per_launch / launch_s, "algorithmic_bytes": alg_bytes}
    prof = load_profile(profile)
    if not prof:
        return {**base, "bound": "hbm", "achieved": hbm_gbs, "peak": hbm_peak, "unit": "GB/s",
                "frac": hbm_gbs / hbm_peak, "traffic": None, "peak_source": peak_src}
    alu_per_perm = prof["inst_alu"] / prof["perms_per_launch"]
    # the pipe's peak rate from the full-size slab capture (a small capture
    # leaves SMs idle in its tail, which understates the rate)
    pk = load_profile(HASH_PROFILE) or prof
    peak_rate = pk["inst_alu"] / (pk["duration_ns"] * 1e-9) / (pk["alu_pct_of_peak"] / 100.0)
    if sm_mhz and pk.get("sm_mhz"):
        peak_rate *= sm_mhz / pk["sm_mhz"]
    achieved = perms_per_launch * alu_per_perm / launch_s
    return {**base, "bound": "int_alu", "achieved": achieved / 1e9, "peak": peak_rate / 1e9,
            "unit": "G warp-instructions/s (ALU pipe)", "frac": achieved / peak_rate,
            "traffic": prof["dram_bytes"] / prof["perms_per_launch"] * perms_per_launch,
            "alu_inst_per_perm": alu_per_perm, "issue_frac_in_profile": prof["issue_pct"] / 100.0,
            "peak_source": f"ALU-pipe rate from {HASH_PROFILE.relative_to(ROOT)}; instructions per permutation "
                           f"and DRAM traffic from {profile.relative_to(ROOT)}", "hbm": hbm}


def lde_roofline(w: int, B: int, lde_ms: float, hbm_peak: float, sm_mhz):
    """The main-trace coset LDE (3 launches per column slab): HBM fraction of
    the algorithmic bytes 8*w*N*(1+B), and its binding resource, the integer
    ALU pipe, scaled from the committed ncu summary by algorithmic bytes."""
    lde_bytes = 8.0 * w * (1 << LOG_H) * (1 + B)
    gbs = lde_bytes / (lde_ms * 1e-3) / 1e9
    out = {"kernel": "lde::lde_pass_kernel + lde::lde_fused_kernel (coset LDE, 3 launches x 8 slabs)",
           "bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
           "algorithmic_bytes": lde_bytes, "kernel_ms": lde_ms, "traffic": None}
    prof = load_profile(LDE_PROFILE)
    if prof:
        per_byte = prof["inst_alu"] / prof["algorithmic_bytes"]
        peak_rate = prof["inst_alu"] / (prof["duration_ns"] * 1e-9) / (prof["alu_pct_of_peak"] / 100.0)
        if sm_mhz and prof.get("sm_mhz"):
            peak_rate *= sm_mhz / prof["sm_mhz"]
        achieved = per_byte * lde_bytes / (lde_ms * 1e-3)
        out.update({"bound": "int_alu", "traffic": prof["dram_bytes"] / prof["algorithmic_bytes"] * lde_bytes,
                    "alu_pipe": {"achieved": achieved / 1e9, "peak": peak_rate / 1e9,
                                 "unit": "G warp-instructions/s (ALU pipe)", "frac": achieved / peak_rate,
                                 "source": str(LDE_PROFILE.relative_to(ROOT))}})
    return out


# ---------------------------------------------------------------- GPU arm
def run_gpu(args):
    import torch
    world, rank, local, pg = dist_setup()
    dev = local
    torch.cuda.set_device(dev)
    P = load_product()
    ctx = P.Context(dev)
    tuning = apply_tuning(ctx)
    pcs = P.PcsParams(**PCS)
    # the Keccak AIR: by default given as its symbolic constraints, whose
    # constraint kernels the library generates and compiles once, here, before
    # any proof (the built-in AIR's hand-written kernel gives the same proof)
    air, air_setup = P.AIR_KECCAK, {"constraints": "hand-written kernel (built-in AIR)"}
    if args.constraints == "generated":
        import p3_miden_b200.airs as airs
        t0 = time.perf_counter()
        air = P.Air(ctx, P.build_air(airs.keccak_eval, airs.KC_NCOLS))
        air_setup = {"constraints": "generated from the AIR's symbolic constraints (p3_miden_b200.airs)",
                     "kernels": air.num_kernels, "compile_s": time.perf_counter() - t0}

    # trace: seeded inputs (one distinct seed per rank), host-generated
    inputs = P.keccak_inputs(1 + rank, N_PERMS)
    host = torch.empty((1 << LOG_H, P.KECCAK_NUM_COLS), dtype=torch.int64, pin_memory=True)
    P.generate_keccak_trace(inputs, out=host.numpy().view(np.uint64))
    dev_trace = host.to(f"cuda:{dev}", non_blocking=False)
    torch.cuda.synchronize(dev)
    wit_dev = [P.AirWitness(air, dev_trace)]
    wit_host = [P.AirWitness(air, host)]

    # ---- device-resident arm (value): trace already in HBM
    for _ in range(args.warmup):
        out = P.prove_multi(ctx, pcs, wit_dev)
    ref_digest = out.digest.copy()
    if air is not P.AIR_KECCAK:  # one untimed proof through the hand-written kernel: the same proof
        hw = P.prove_multi(ctx, pcs, [P.AirWitness(P.AIR_KECCAK, dev_trace)])
        assert np.array_equal(hw.digest, ref_digest), "generated and hand-written constraint kernels differ"
        air_setup["same_proof_as_hand_written"] = True
        del hw
    barrier(pg, dev)
    torch.cuda.synchronize(dev)
    lat, launches, stages, lde_k, leaf_k = [], 0, np.zeros(len(P.STAGES)), [], []
    with ClockSampler(dev) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            out = P.prove_multi(ctx, pcs, wit_dev)
            lat.append(out.device_ms)
            lde_k.append(out.lde_kernel_ms)
            leaf_k.append(out.leaf_kernel_ms)
            leaf_n = out.leaf_launches
            launches += out.gpu_launches
            stages += np.array(out.stage_ms)
            assert np.array_equal(out.digest, ref_digest), "non-deterministic proof"
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - t0
    barrier(pg, dev)
    value, dev_time, total_proofs = aggregate(pg, float(args.steps), sum(lat) / 1e3, dev)

    # ---- end-to-end arm: host (pinned) trace in, proof bytes out, per step
    for _ in range(max(1, args.warmup // 2)):
        P.prove_multi(ctx, pcs, wit_host)
    barrier(pg, dev)
    torch.cuda.synchronize(dev)
    e2e_lat, h2d, d2h = [], 0, 0
    for _ in range(args.steps):
        o = P.prove_multi(ctx, pcs, wit_host)
        e2e_lat.append(o.device_ms)
        h2d, d2h = o.h2d_bytes, o.d2h_bytes + o.proof.fields.nbytes + o.proof.commitments.nbytes
        assert np.array_equal(o.digest, ref_digest)
    barrier(pg, dev)
    e2e_time = max_over_ranks(pg, sum(e2e_lat) / 1e3, dev)
    e2e_value = total_proofs / e2e_time

    # ---- end-to-end from the permutation inputs: pinned inputs uploaded,
    # trace generated on the device (p3g_keccak_trace_device), proved, proof
    # returned; host wall clock around the public calls
    inputs_pinned = torch.from_numpy(inputs.reshape(-1, 25).view(np.int64)).pin_memory()
    inputs_dev = torch.empty_like(inputs_pinned, device=f"cuda:{dev}")
    trace_dev = torch.empty((1 << LOG_H, P.KECCAK_NUM_COLS), dtype=torch.int64, device=f"cuda:{dev}")

    def from_inputs():
        inputs_dev.copy_(inputs_pinned, non_blocking=True)
        P.generate_keccak_trace_device(ctx, inputs_dev, LOG_H, out=trace_dev)
        return P.prove_multi(ctx, pcs, [P.AirWitness(air, trace_dev)])

    for _ in range(max(1, args.warmup // 2)):
        from_inputs()
    barrier(pg, dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o = from_inputs()
        assert np.array_equal(o.digest, ref_digest)
    torch.cuda.synchronize(dev)
    inp_time = max_over_ranks(pg, time.perf_counter() - t0, dev)
    inp_value = total_proofs / inp_time
    inp_d2h = o.d2h_bytes + o.proof.fields.nbytes + o.proof.commitments.nbytes

    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return 0

    stages_ms = stages / args.steps
    pk = peaks()
    hbm_peak = pk.get("hbm_gbs", 6650.0)
    w = P.KECCAK_NUM_COLS
    B = 1 << PCS["log_blowup"]
    n_lde = (1 << LOG_H) * B
    tree_ms = float(stages_ms[1])
    perms = n_lde * ((w + 7) // 8) + n_lde - 1
    dominant = int(np.argmax(stages_ms))
    clk = clocks.summary()
    cm = air is not P.AIR_KECCAK and HASH_PROFILE_CM.exists()
    roofline = hash_roofline(n_lde, w, float(np.mean(leaf_k)), int(leaf_n), hbm_peak,
                             "measured" if "hbm_gbs" in pk else "fallback", clk.get("sm_mhz"),
                             HASH_PROFILE_CM if cm else HASH_PROFILE)
    if cm:
        roofline["kernel"] = ("merkle::leaf_class_kernel<true> (LMCS leaf sponge, Poseidon2-12; also writes "
                              "the column-major rows the generated constraint kernels read)")
    lde = lde_roofline(w, B, float(np.mean(lde_k)), hbm_peak, clk.get("sm_mhz"))
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_time / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Goldilocks, exact)",
        "data": "synthetic (seeded Keccak-f inputs)",
        "config": base_config(),
        "arm": {"parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (5.5 GB trace, 11 GB LDE)",
                "timing": "CUDA events on the prover stream", "tuning": tuning, "air": air_setup},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "wall_per_step": wall / args.steps * 1e3},
        "stage_ms": {n: float(v) for n, v in zip(P.STAGES, stages_ms)},
        "dominant_stage": P.STAGES[dominant],
        "roofline": roofline,
        "lde": lde,
        "hash": {"kernel": "LMCS leaf sponge + compress (Poseidon2-12)", "perms": perms,
                 "perms_per_s": perms / (tree_ms * 1e-3)},
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_time / args.steps * 1e3},
        "e2e_from_inputs": {"value": inp_value, "unit": METRIC, "h2d_bytes_per_step": int(inputs_pinned.numel() * 8),
                            "d2h_bytes_per_step": int(inp_d2h), "ms_per_step": inp_time / args.steps * 1e3,
                            "timing": "host wall clock around upload + device trace generation + prove_multi"},
        "gpu_launches": launches,
        "clocks": clk,
        "proof_bytes": int(out.proof.fields.nbytes + out.proof.commitments.nbytes),
    }
    if args.cpu_baseline and world == 1:
        # one oracle proof each of 2^12- and 2^13-row samples (about 24 s on 16 host cores)
        threads = os.cpu_count() or 1
        oracle_proof_seconds(10, threads)  # warm-up: thread pool, first-touch pages
        samples = {lh: oracle_proof_seconds(lh, threads) for lh in (12, 13)}
        per_proof, a, b = affine_extrapolation(samples)
        line["cpu_baseline"] = {
            "value": 1.0 / per_proof, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"one oracle proof each of 2^12- and 2^13-row Keccak samples (same parameters) in "
                      f"{samples[12]:.1f} s and {samples[13]:.1f} s, extrapolated as {a:.1f} s + "
                      f"{b * 1e3:.3f} ms per row to 2^{LOG_H} rows",
        }
    print(json.dumps(line), flush=True)
    ctx.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


# ------------------------------------------ other named configurations
LIFTED_PCS = dict(log_blowup=3, log_folding_arity=2, log_final_degree=0, folding_pow_bits=16,
                  deep_pow_bits=0, num_queries=100, query_pow_bits=0)
SMALL_PCS = PCS


def time_proofs(P, ctx, pcs, wits, steps, warmup, dev, per_proof=None):
    """Device-timed prove_multi on resident witnesses: per-proof ms, stage ms
    (mean), last output; per_proof, when given, receives per timed proof its
    8 stage ms, the context's cumulative host ms in allocation calls and its
    pool's reserved GB."""
    import torch
    ref = None
    for _ in range(warmup):
        out = P.prove_multi(ctx, pcs, wits)
        ref = out.digest.copy()
    torch.cuda.synchronize(dev)
    lat, stages, launches = [], np.zeros(len(P.STAGES)), 0
    with ClockSampler(dev) as clocks:
        for _ in range(steps):
            out = P.prove_multi(ctx, pcs, wits)
            lat.append(out.device_ms)
            stages += np.array(out.stage_ms)
            if per_proof is not None:
                m = ctx.memory_stats()
                per_proof.append([round(float(v), 2) for v in out.stage_ms[:8]] +
                                 [round(m["alloc_ms"], 2), round(m["reserved_bytes"] / 1e9, 2)])
            launches += out.gpu_launches
            if ref is None:
                ref = out.digest.copy()
            assert np.array_equal(out.digest, ref), "non-deterministic proof"
    return lat, stages / steps, launches, out, clocks.summary()


def run_named(args):
    """Config 1 (Keccak, 42 permutations, 2^10 rows: latency) or config 3
    (three cubic-AIR traces 2^20 x 64, 2^16 x 256, 2^12 x 1024 lifted to
    2^20, log_blowup 3, FRI arity 4)."""
    import torch
    dev = 0
    torch.cuda.set_device(dev)
    P = load_product()
    ctx = P.Context(dev)
    if args.workload == "small":
        inputs = P.keccak_inputs(1, 42)
        t = P.generate_keccak_trace(inputs)
        wits = [P.AirWitness(P.AIR_KECCAK, torch.from_numpy(t.view(np.int64)).to(f"cuda:{dev}"))]
        pcs_d, name = SMALL_PCS, "keccak-f1600 AIR, 42 perms -> 2^10 x 2633 trace, lifted STARK (Poseidon2-12 LMCS)"
    else:
        wits = []
        for i, (lh, w) in enumerate([(12, 1024), (16, 256), (20, 64)]):  # ascending heights
            k, t = P.generate_cubic_trace(lh, w, 300 + i)
            wits.append(P.AirWitness(P.AIR_CUBIC, torch.from_numpy(t.view(np.int64)).to(f"cuda:{dev}"), k))
        pcs_d, name = LIFTED_PCS, "cubic AIR x3 (2^12 x 1024, 2^16 x 256, 2^20 x 64) lifted to 2^20, log_blowup 3, arity 4"
    torch.cuda.synchronize(dev)
    lat, stages, launches, out, clk = time_proofs(P, ctx, P.PcsParams(**pcs_d), wits, args.steps, args.warmup, dev)
    line = {
        "metric": "proofs/s", "value": len(lat) / (sum(lat) / 1e3), "unit": "proofs/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(lat)), "higher_is_better": True,
        "dtype": "u64 (Goldilocks, exact)", "data": "synthetic (seeded traces), resident in HBM",
        "config": {"workload": name, "pcs": pcs_d, "timing": "CUDA events on the prover stream"},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "stage_ms": {n: float(v) for n, v in zip(P.STAGES, stages)},
        "gpu_launches": launches, "clocks": clk,
        "proof_bytes": int(out.proof.fields.nbytes + out.proof.commitments.nbytes),
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_symbolic(args):
    """The headline proof (Keccak AIR, 10922 permutations, 2^18 x 2633) with
    the AIR given as symbolic constraints (p3_miden_b200.airs, the AirBuilder
    form) and its constraint kernels generated and compiled by the library,
    next to the hand-written Keccak kernel on the same trace: per-stage
    device time of both, and the generated kernels' compile time."""
    import torch
    dev = 0
    torch.cuda.set_device(dev)
    P = load_product()
    import p3_miden_b200.airs as S
    ctx = P.Context(dev)
    tuning = apply_tuning(ctx)
    if args.chunk_nodes:
        ctx.set_air_chunk_nodes(args.chunk_nodes)
    t0 = time.perf_counter()
    air = P.Air(ctx, P.build_air(S.keccak_eval, S.KC_NCOLS))
    compile_s = time.perf_counter() - t0
    t = P.generate_keccak_trace(P.keccak_inputs(1, N_PERMS))
    d = torch.from_numpy(t.view(np.int64)).to(f"cuda:{dev}")
    del t
    pcs = P.PcsParams(**PCS)
    out = {}
    for name, a in (("generated", air), ("hand-written", P.AIR_KECCAK)):
        each = []
        lat, stages, launches, o, clk = time_proofs(P, ctx, pcs, [P.AirWitness(a, d)], args.steps, args.warmup, dev,
                                                    each)
        out[name] = {"ms_per_proof": float(np.mean(lat)), "stage_ms": {n: float(v) for n, v in zip(P.STAGES, stages)},
                     "ms_each": [round(float(v), 2) for v in lat], "stage_ms_each": each,
                     "digest": [int(x) for x in o.digest[:4]], "clocks": clk}
    assert out["generated"]["digest"] == out["hand-written"]["digest"], "generated and hand-written proofs differ"
    print(json.dumps({"workload": f"{workload_name()}, AIR as symbolic constraints (3182, 40470 DAG nodes)",
                      "compile_s": compile_s, "kernels": air.num_kernels, "tuning": tuning, **out}), flush=True)
    ctx.close()
    return 0


def run_verify(args):
    """Verification of the headline proof (2^18 x 2633 Keccak, the example's
    parameters) through the public call p3g_verify: transcript replay on the
    host, openings, DEEP and FRI query checks on the GPU. The proof is made
    once; each step verifies it from host memory (wall clock around the call,
    host and device parts reported). The verifier restatement (oracle) times
    the same check on one host core beside it."""
    import torch
    dev = 0
    torch.cuda.set_device(dev)
    P = load_product()
    ctx = P.Context(dev)
    t = P.generate_keccak_trace(P.keccak_inputs(1, N_PERMS))
    pcs = P.PcsParams(**PCS)
    out = P.prove_multi(ctx, pcs, [P.AirWitness(P.AIR_KECCAK, torch.from_numpy(t.view(np.int64)).to(f"cuda:{dev}"))])
    del t
    shapes = [P.AirShape(P.AIR_KECCAK, 1 << LOG_H, 2633)]
    B = max(1, args.batch)
    items = [(pcs, shapes, out.proof.fields, out.proof.commitments, out.digest)] * B

    def step():
        if B == 1:
            r = P.verify_output(ctx, pcs, shapes, out)
            assert r.ok, r.name
            return r
        verdicts, r = P.verify_batch(ctx, items)
        assert verdicts == [0] * B, verdicts
        return r

    for _ in range(args.warmup):
        step()
    wall, host, device, launches = [], [], [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = step()
        wall.append((time.perf_counter() - t0) * 1e3)
        host.append(r.host_ms), device.append(r.device_ms)
        launches += r.gpu_launches
    value = B * 1e3 / statistics.median(wall)
    line = {
        "metric": "verifications/s", "value": value, "unit": "verifications/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.median(wall), "higher_is_better": True,
        "dtype": "u64 (Goldilocks, exact)", "data": "synthetic (seeded Keccak-f inputs); proof from p3g_prove",
        "config": {"workload": f"verify_multi of the {workload_name()} proof", "pcs": PCS, "proofs_per_call": B,
                   "proof_bytes": int(out.proof.fields.nbytes + out.proof.commitments.nbytes)},
        "split_ms": {"host replay + layout (median)": statistics.median(host),
                     "device: upload, kernels, read-back (median)": statistics.median(device)},
        "gpu_launches": launches,
        "e2e": {"value": value, "unit": "verifications/s",
                "h2d_bytes_per_step": B * int(out.proof.fields.nbytes + out.proof.commitments.nbytes),
                "d2h_bytes_per_step": 0},
    }
    if args.cpu_baseline:
        sys.path.insert(0, str(ROOT / "tests"))
        import oracle_ffi as O
        times = []
        for _ in range(2):
            t0 = time.perf_counter()
            rc = O.verify(O.default_p2(), PCS, [(O.AIR_KECCAK, 1 << LOG_H, 2633, None)], out.proof.fields,
                          out.proof.commitments, out.digest)
            times.append(time.perf_counter() - t0)
            assert rc == 0
        line["cpu_baseline"] = {"value": 1.0 / min(times), "unit": "verifications/s", "cores": 1, "kind": "port",
                                "sample": "the verifier restatement on the same proof, one host thread"}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_slab(args):
    """One full-size column slab of the headline workload through the public
    LDE and LMCS entry points (2^18 x 336 seeded words, log_blowup 1, then the
    2^19-leaf tree): the launch shapes of one of the 8 main-trace slabs, for
    kernel-level profiling."""
    import torch
    dev = 0
    torch.cuda.set_device(dev)
    P = load_product()
    ctx = P.Context(dev)
    h, w = 1 << LOG_H, 336
    m = np.random.default_rng(1).integers(0, P.P, size=(h, w), dtype=np.uint64)
    d = P.to_device(m, dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    lde_ms, tree_ms = [], []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize(dev)
        ev[0].record()
        out = P.coset_lde(ctx, d, PCS["log_blowup"], 7)
        ev[1].record()
        torch.cuda.synchronize(dev)
        if i >= args.warmup:
            lde_ms.append(ev[0].elapsed_time(ev[1]))
        ev[0].record()
        root = P.LmcsTree(ctx, [out], 8).root()
        ev[1].record()
        torch.cuda.synchronize(dev)
        if i >= args.warmup:
            tree_ms.append(ev[0].elapsed_time(ev[1]))
    print(json.dumps({"workload": f"column slab 2^{LOG_H} x {w}, log_blowup {PCS['log_blowup']}",
                      "lde_ms": float(np.median(lde_ms)), "tree_ms": float(np.median(tree_ms)),
                      "root": [int(x) for x in root],
                      "timing": "CUDA events on the current stream around each synchronous call (includes host set-up)"}),
          flush=True)
    ctx.close()
    return 0


# ------------------------------------------------- batched and serving
MIX_PCS = dict(log_blowup=3, log_folding_arity=1, log_final_degree=0, folding_pow_bits=16,
               deep_pow_bits=0, num_queries=100, query_pow_bits=0)


def job_specs(n, seed, max_log_cubic=18, max_log_keccak=16):
    """Seeded uneven mix: 60% cubic AIR (height 2^12..2^max log-uniform, width
    in {16..512}), 40% Keccak AIR (2^12..2^16 rows)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        if rng.random() < 0.6:
            specs.append(("cubic", int(rng.integers(12, max_log_cubic + 1)),
                          int(rng.choice([16, 32, 64, 128, 256, 512])), 10_000 + i))
        else:
            specs.append(("keccak", int(rng.integers(12, max_log_keccak + 1)), 2633, 20_000 + i))
    return specs


def build_jobs(P, specs, device, pinned):
    import torch
    jobs = []
    for air, log_h, w, seed in specs:
        if air == "cubic":
            k, t = P.generate_cubic_trace(log_h, w, seed)
            inst_air, consts = P.AIR_CUBIC, k
        else:
            t = P.generate_keccak_trace(P.keccak_inputs(seed, (1 << log_h) // 24))
            inst_air, consts = P.AIR_KECCAK, None
        tt = torch.from_numpy(t.view(np.int64))
        tt = tt.pin_memory() if pinned else tt.to(f"cuda:{device}")
        jobs.append(P.Job(P.PcsParams(**MIX_PCS), [P.AirWitness(inst_air, tt, consts)]))
    torch.cuda.synchronize(device)
    return jobs


def run_pool(P, jobs, srv):
    """One pass of a job list through a running server (its workers, streams
    and memory pools persist across passes, as in a serving process)."""
    t0 = time.perf_counter()
    res = srv.run(jobs)
    wall = time.perf_counter() - t0
    peak = srv.peak_admitted_bytes()
    bad = [r.status for r in res if r.status != P.OK]
    assert not bad, f"failed jobs: {bad}"
    span = max(r.end_s for r in res) - min(r.submit_s for r in res)
    lat = [(r.end_s - (j.arrival_s)) * 1e3 for r, j in zip(res, jobs)]
    return res, span, wall, lat, peak


def run_batch(args):
    import torch
    dev = 0
    torch.cuda.set_device(dev)
    P = load_product()
    specs = job_specs(args.jobs, args.seed, args.max_log_cubic, args.max_log_keccak)
    jobs = build_jobs(P, specs, dev, pinned=False)
    srv_plain = P.ProofServer(dev, n_workers=1, hbm_budget=args.budget)
    srv_pool = P.ProofServer(dev, n_workers=args.workers, hbm_budget=args.budget)
    apply_tuning(srv_plain)
    tuning = apply_tuning(srv_pool)
    # warm-up over the whole list on both servers (twice), so that neither arm
    # pays for growing its memory pools or for first-use tables in the timed passes
    for _ in range(2):  # one pass left the plain arm's first timed pass slower on some boxes
        run_pool(P, jobs, srv_plain)
        run_pool(P, jobs, srv_pool)
    # alternate the two arms and keep the median pass of each: single passes
    # of the same list vary by several percent
    p_runs, b_runs, diag = [], [], []
    import psutil

    def note(arm, run):
        res, span = run[0], run[1]
        free, total = torch.cuda.mem_get_info(dev)
        diag.append({"arm": arm, "proofs_per_s": len(jobs) / span,
                     "device_ms_sum": float(sum(r.output.device_ms for r in res)),
                     "device_free_gb": free / 1e9, "host_rss_gb": psutil.Process().memory_info().rss / 1e9})

    with ClockSampler(dev) as clocks:
        for _ in range(args.reps):
            p_runs.append(run_pool(P, jobs, srv_plain))
            note("plain", p_runs[-1])
            b_runs.append(run_pool(P, jobs, srv_pool))
            note("pooled", b_runs[-1])
    srv_plain.close()
    srv_pool.close()
    p_runs.sort(key=lambda r: r[1])
    b_runs.sort(key=lambda r: r[1])
    plain, span1, _, lat1, _ = p_runs[len(p_runs) // 2]
    batched, spanK, _, latK, peak = b_runs[len(b_runs) // 2]
    for a, b in zip(plain, batched):
        assert np.array_equal(a.output.digest, b.output.digest), "batched proof differs from plain"
    line = {
        "metric": "proofs/s (uneven 64-proof batch)", "unit": "proofs/s", "value": len(jobs) / spanK,
        "plain_value": len(jobs) / span1, "speedup_vs_plain": span1 / spanK, "n_gpus": 1,
        "workers": args.workers, "jobs": len(jobs), "higher_is_better": True, "dtype": "u64 (Goldilocks, exact)",
        "data": "synthetic seeded job mix, traces resident in HBM",
        "config": {"workload": f"60% cubic AIR 2^12..2^{args.max_log_cubic} x {{16..512}}, "
                               f"40% Keccak AIR 2^12..2^{args.max_log_keccak}", "pcs": MIX_PCS,
                   "seed": args.seed, "hbm_budget": args.budget},
        "latency_ms": {"plain_p50": float(np.percentile(lat1, 50)), "plain_p99": float(np.percentile(lat1, 99)),
                       "batched_p50": float(np.percentile(latK, 50)), "batched_p99": float(np.percentile(latK, 99))},
        "peak_admitted_gb": peak / 1e9,
        "passes": {"plain_proofs_per_s": [len(jobs) / r[1] for r in p_runs],
                   "batched_proofs_per_s": [len(jobs) / r[1] for r in b_runs]},
        "bit_identical_to_plain": True,
        "tuning": tuning,
        "pass_diagnostics": diag,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def run_serve(args):
    import torch
    dev = 0
    torch.cuda.set_device(dev)
    P = load_product()
    specs = job_specs(args.pool, args.seed, max_log_cubic=20, max_log_keccak=16)
    pool = build_jobs(P, specs, dev, pinned=True)
    rng = np.random.default_rng(args.seed + 1)
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, size=args.jobs))
    picks = rng.integers(0, len(pool), size=args.jobs)
    stream = [P.Job(pool[k].pcs, pool[k].instances, float(a)) for k, a in zip(picks, arrivals)]
    # the server's heavy class: LDEs above 2^26 words (every Keccak job of the mix)
    heavy = [sum((i.trace.shape[0] << MIX_PCS["log_blowup"]) * i.trace.shape[1] for i in pool[k].instances) > 1 << 26
             for k in picks]
    out = {}
    arms = [("plain", 1, False, 1), ("served", args.workers, False, 1)]
    if args.self_check:  # every served proof verified on the device before it is returned
        arms.append(("served+self-check", args.workers, True, 1))
    for name, workers, check, max_heavy in arms:
        srv = P.ProofServer(dev, n_workers=workers, hbm_budget=args.budget, self_check=check, max_heavy=max_heavy)
        apply_tuning(srv)
        run_pool(P, pool, srv)  # warm-up over every distinct job
        res, span, wall, lat, peak = run_pool(P, stream, srv)
        srv.close()
        lat = np.asarray(lat)
        hv = np.asarray(heavy)
        out[name] = {"proofs_per_s": len(stream) / span, "p50_ms": float(np.percentile(lat, 50)),
                     "p99_ms": float(np.percentile(lat, 99)), "makespan_s": span, "peak_admitted_gb": peak / 1e9,
                     "workers": workers,
                     "by_class": {c: {"jobs": int(m.sum()), "p50_ms": float(np.percentile(lat[m], 50)),
                                      "p99_ms": float(np.percentile(lat[m], 99))}
                                  for c, m in (("heavy", hv), ("light", ~hv)) if m.any()}}
        if check:
            assert all(r.verdict == 0 for r in res)
            out[name]["verify_ms_mean"] = float(np.mean([r.verify_ms for r in res]))
    line = {
        "metric": "served proofs/s and p50/p99 latency", "unit": "proofs/s", "value": out["served"]["proofs_per_s"],
        "higher_is_better": True, "n_gpus": 1, "jobs": args.jobs, "arrival_rate_per_s": args.rate,
        "dtype": "u64 (Goldilocks, exact)", "data": "synthetic seeded job pool, Poisson arrivals, pinned host traces",
        "config": {"workload": "job pool: 60% cubic AIR 2^12..2^20 x {16..512}, 40% Keccak AIR 2^12..2^16",
                   "pool": args.pool, "pcs": MIX_PCS, "hbm_budget": args.budget},
        **out,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--log-h", type=int, default=18,
                    help="trace height (log2); 18 is the measured workload, smaller values are profiling cases")
    ap.add_argument("--workload", default="keccak", choices=["keccak", "small", "lifted", "batch", "serve", "slab", "verify", "symbolic"],
                    help="keccak: the plain prover at scale (headline); small: 42-permutation Keccak proof; "
                         "lifted: three cubic traces lifted to 2^20; batch: 64-proof uneven mix; serve: Poisson stream; "
                         "slab: one 2^18 x 336 column slab through the LDE and the tree (kernel profiling); "
                         "verify: the device-side verifier on the headline proof; "
                         "symbolic: the headline proof through generated constraint kernels")
    ap.add_argument("--jobs", type=int, default=64)
    ap.add_argument("--workers", type=int, default=2)
    ap.add_argument("--reps", type=int, default=3, help="batch: alternating passes per arm (median kept)")
    ap.add_argument("--pool", type=int, default=32)
    ap.add_argument("--rate", type=float, default=20.0, help="serve: arrivals per second")
    ap.add_argument("--budget", type=float, default=150e9, help="HBM admission budget in bytes")
    ap.add_argument("--seed", type=int, default=2025)
    ap.add_argument("--self-check", action="store_true", help="serve: add an arm that verifies every proof on the device")
    ap.add_argument("--batch", type=int, default=1, help="verify: proofs per p3g_verify_batch call")
    ap.add_argument("--max-log-cubic", type=int, default=18)
    ap.add_argument("--max-log-keccak", type=int, default=16)
    ap.add_argument("--constraints", default="generated", choices=["generated", "hand-written"],
                    help="keccak: the AIR as symbolic constraints with generated kernels (default) or the built-in "
                         "AIR's hand-written kernel (the same proof)")
    ap.add_argument("--chunk-nodes", type=int, default=0,
                    help="symbolic: DAG nodes per generated constraint kernel (0: the library default)")
    args = ap.parse_args()
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload in ("small", "lifted"):
        return run_named(args)
    global LOG_H, N_PERMS
    if args.log_h != LOG_H:
        LOG_H = args.log_h
        N_PERMS = (1 << LOG_H) // 24
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "slab":
        return run_slab(args)
    if args.workload == "verify":
        return run_verify(args)
    if args.workload == "symbolic":
        return run_symbolic(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
