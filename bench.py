#!/usr/bin/env python
"""Benchmark: atoms/s of the Matching Pursuit decomposition on B200.

Workload (the reference's headline multichannel configuration): MMP2,
19 channels x 8 epochs x 5120 float32 samples at 256 Hz, energyError 0.01,
100 iterations, energyPercent 99, seeded synthetic signals (20 shared Gabor
atoms per epoch with N(0,1) channel gains, white noise at 5 dB per channel).
One step = the whole decomposition of the 8 epochs (800 MP atoms) as one
device batch.  An MMP2 multichannel atom counts once.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU: one process per GPU (torchrun); each rank decomposes its own
8-epoch workload (weak scaling, no data-path collective); the timed region is
bracketed by a barrier and synchronize, and the max over ranks is reported.

--impl reference times the reference's own CPU code (empi's src/*.cpp built
by oracle/Makefile with the project FFT shim in place of FFTW) on one epoch
of the same workload per step, on rank 0 with all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = 1  # empi_b200.synth workload index


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    # small cases for profiling runs (not bench numbers)
    p.add_argument("--workload", type=int, default=WORKLOAD,
                   help="synthetic workload index (empi_b200.synth); the default is the headline one")
    p.add_argument("--epochs", type=int, default=0, help="decompose only the first E epochs (instances)")
    p.add_argument("--iterations", type=int, default=0, help="override the iteration count")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                   help="weak: every rank decomposes its own copy of the workload (the default); strong: one "
                        "workload split across the ranks by estimated cost (empi_b200.shard)")
    p.add_argument("--no-roofline", action="store_true")
    p.add_argument("--persistent", type=int, default=-1, choices=[-1, 0, 1],
                   help="the MP loop as one persistent kernel per chunk (1), as the CUDA graph (0), or by the "
                        "tune cache / batch size (-1, the default)")
    p.add_argument("--proposal", choices=["net", "last_atom", "none"],
                   help="time the block proposal too (same workload, plain and proposal back to back; the atoms "
                        "must be identical); net uses --proposal-weights")
    p.add_argument("--proposal-weights", default=os.path.join(ROOT, "empi_b200", "proposal_b200.bin"))
    p.add_argument("--proposal-k", type=int, default=16)
    p.add_argument("--proposal-probe", action="store_true",
                   help="also measure the refresh work no certified block proposal could skip (one extra run)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return rank, local, world


# ---------------------------------------------------------------- reference arm


def reference_config(d, w, epoch_index, iterations):
    path = os.path.join(d, "sig.bin")
    w.epochs[epoch_index].tofile(path)
    cfg = os.path.join(d, "cfg")
    with open(cfg, "w") as f:
        f.write(f"energyError {w.energy_error}\nmaximalNumberOfIterations {iterations}\n"
                f"energyPercent {w.energy_percent}\nMP {w.variant.upper()}\nnameOfDataFile sig.bin\n"
                f"nameOfOutputDirectory .\nsamplingFrequency {w.fs}\nnumberOfChannels {w.channels}\n"
                f"selectedChannels 1-{w.channels}\nnumberOfSamplesInEpoch {w.samples}\n")
    return cfg


def run_reference(w, iterations, threads):
    """Wall time and atom count of the reference CLI on epoch 0."""
    from oracle import oracle as O

    cli = O.ref_cli()
    if not os.path.exists(cli):
        return None
    with tempfile.TemporaryDirectory() as d:
        cfg = reference_config(d, w, 0, iterations)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
        t0 = time.perf_counter()
        p = subprocess.run([cli, cfg], cwd=d, env=env, capture_output=True, text=True, check=True)
        dt = time.perf_counter() - t0
    atoms = sum(1 for line in p.stdout.splitlines() if line.startswith("ATOM"))
    return dt, atoms


def reference_arm(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    from empi_b200 import synth

    w = synth.workload(args.workload, epochs=args.epochs or None, iterations=args.iterations or None)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        r = run_reference(w, 5, threads)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/empi not built (make -C oracle ref)"}))
            return
    times, atoms = [], 0
    for _ in range(args.steps):
        dt, n = run_reference(w, w.iterations, threads)
        times.append(dt)
        atoms += n
    total = sum(times)
    value = atoms / total
    sample = (f"epoch 0 of the workload per step ({w.channels}ch x {w.samples} @ {w.fs:g} Hz, "
              f"{w.variant.upper()}, {w.iterations} iterations), reference CLI built from empi src/*.cpp "
              f"-O3 -fopenmp with the {ref_fft_label()}")
    line = {
        "impl": "reference", "metric": "atoms/s", "value": value, "unit": "atoms/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(w, world),
        "cpu_baseline": {"value": value, "unit": "atoms/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "atoms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def workload_config(w, world, scaling="weak"):
    if len({e.shape for e in w.epochs}) > 1:
        shape = (f"{len(w.epochs)} uneven instances ({sum(e.shape[1] for e in w.epochs)} channels, "
                 f"{min(e.shape[0] for e in w.epochs)}-{max(e.shape[0] for e in w.epochs)} samples)")
    else:
        shape = f"{w.channels}ch x {len(w.epochs)} epochs x {w.samples}"
    return {"workload": f"{w.variant.upper()} {shape} "
                        f"float32 @ {w.fs:g} Hz, energyError {w.energy_error}, {w.iterations} iterations, "
                        f"energyPercent {w.energy_percent}",
            "variant": w.variant, "channels": w.channels, "epochs": len(w.epochs), "samples": w.samples,
            "fs": w.fs, "energy_error": w.energy_error, "iterations": w.iterations,
            "energy_percent": w.energy_percent, "parallelism": f"instances x{world} ({scaling})",
            "l2": "256 MiB buffer written between timed steps (inputs are smaller than L2)"}


# ---------------------------------------------------------------- clocks


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.file = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "-i", str(self.device),
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=self.file, stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- our arm


def cpu_baseline(w):
    threads = os.cpu_count() or 1
    r = run_reference(w, w.iterations, threads)
    if r is None:
        return None
    dt, atoms = r
    return {"value": atoms / dt, "unit": "atoms/s", "cores": threads, "kind": "reference",
            "sample": f"epoch 0 of the workload ({w.channels}ch x {w.samples} @ {w.fs:g} Hz, "
                      f"{w.variant.upper()}, {w.iterations} iterations, {dt:.2f} s), reference CLI from "
                      f"empi src/*.cpp -O3 -fopenmp with the {ref_fft_label()}"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def profiled_executed_fp32(w):
    """Executed FP32 FLOPs of the refresh as a fraction of the FP32 peak, from
    the committed ncu figure (profiles/refresh_traffic_mmp2_19x8x5120.json);
    None for other workloads."""
    if w.name != "mmp2-19x8x5120@256":
        return None
    try:
        with open(os.path.join(ROOT, "profiles", "refresh_traffic_mmp2_19x8x5120.json")) as f:
            return float(json.load(f)["executed_fp32_frac_of_peak"])
    except (OSError, KeyError, ValueError):
        return None


def profiled_traffic(w):
    """DRAM bytes of one refresh fork of the headline workload from the
    committed ncu figure (profiles/refresh_traffic_mmp2_19x8x5120.json);
    None for other workloads."""
    if w.name != "mmp2-19x8x5120@256" or len(w.epochs) != 8:
        return None
    try:
        with open(os.path.join(ROOT, "profiles", "refresh_traffic_mmp2_19x8x5120.json")) as f:
            return float(json.load(f)["dram_bytes_per_fork"])
    except (OSError, KeyError, ValueError):
        return None


def host_fftw():
    """Whether the host has FFTW3 (the reference's FFT library) installed."""
    try:
        out = subprocess.run(["ldconfig", "-p"], capture_output=True, text=True, timeout=10).stdout
    except (OSError, subprocess.SubprocessError):
        return False
    return "libfftw3" in out


def ref_fft_label():
    return ("project FP64 FFT shim in place of FFTW3 (" +
            ("FFTW3 is installed on this host, but the reference is built from its sources where they are, "
             "against the shim" if host_fftw() else "FFTW3 absent on this host") + ")")


def ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import empi_b200
    from empi_b200 import synth

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    if args.scaling == "strong":
        # one job for all ranks, its epochs split by estimated cost (no collective on the data path)
        from empi_b200 import shard

        w = synth.workload(args.workload, epochs=args.epochs or None, iterations=args.iterations or None)
        costs = [shard.epoch_cost(e.shape, w.fs, w.energy_error, w.iterations, w.variant) for e in w.epochs]
        job_epochs = len(w.epochs)
        w.epochs = [w.epochs[i] for i in shard.partition(costs, world)[rank]]
        if not w.epochs:
            raise SystemExit(f"strong scaling: {job_epochs} epochs for {world} ranks leaves rank {rank} idle")
    else:
        w = synth.workload(args.workload, seed=1000 + args.workload + 7919 * rank, epochs=args.epochs or None,
                           iterations=args.iterations or None)
    stream = torch.cuda.Stream()
    from empi_b200 import autotune

    # the committed autotuner cache: launch shapes tuned on a B200 per workload
    tune_cache = autotune.DEFAULT_CACHE if os.path.exists(autotune.DEFAULT_CACHE) else None
    eng = empi_b200.Engine(device=local, stream=stream.cuda_stream, tune_cache=tune_cache,
                           persistent=args.persistent)
    settings = empi_b200.DecompositionSettings(w.iterations, 1.0 - 0.01 * w.energy_percent)
    shapes = [e.shape for e in w.epochs]
    pinned = [torch.from_numpy(e).pin_memory() for e in w.epochs]
    host = [p.numpy() for p in pinned]
    batch = empi_b200.Batch(w.variant, w.energy_error, settings, shapes, w.fs, engine=eng)
    batch.load(host)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")

    def atoms_of():
        return sum(int(batch.result(e).counts[0]) if w.variant != "smp" else int(batch.result(e).counts.sum())
                   for e in range(len(w.epochs)))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        batch.run()
    atoms_per_step = atoms_of()

    # device-resident inputs: one step = batch.run()
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    total_ms = 0.0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        batch.run()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    barrier()
    clk = clocks.stop()
    bs = batch.stats()  # the timed batch's last run
    launches = bs.kernel_launches

    # end to end through the public API: pinned host inputs in, atoms out
    e2e_ms = 0.0
    d2h = 0
    barrier()
    for _ in range(0 if args.no_e2e else args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        batch.load(host)
        batch.run()
        d2h = 0
        for e in range(len(w.epochs)):
            r = batch.result(e)
            d2h += r.atoms.nbytes + r.counts.nbytes + r.energies.nbytes + r.indices.nbytes + r.totals.nbytes
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    barrier()
    h2d = sum(e.nbytes for e in host)

    t = torch.tensor([total_ms, e2e_ms], dtype=torch.float64, device=f"cuda:{local}")
    n_atoms = torch.tensor([float(atoms_per_step)], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(n_atoms, op=dist.ReduceOp.SUM)
    total_ms, e2e_ms = float(t[0]), float(t[1])
    atoms_all_ranks = float(n_atoms[0])  # weak: world x one workload's atoms; strong: the one job's
    units = atoms_all_ranks * args.steps
    value = units / (total_ms / 1e3)
    e2e_value = units / (e2e_ms / 1e3) if e2e_ms > 0 else None

    # dominant kernel (k_refresh): CUDA events around every refresh launch
    eng_t = empi_b200.Engine(device=local, stream=stream.cuda_stream, timing=True, tune_cache=tune_cache)
    bt = empi_b200.Batch(w.variant, w.energy_error, settings, shapes, w.fs, engine=eng_t)
    bt.load(host)
    for _ in range(0 if args.no_roofline else 2):
        bt.run()
    st = bt.stats()
    roofline = roofline_fp32 = None
    if st.refresh_launches:
        per_launch_ms = st.refresh_ms / max(1, st.refresh_launches)
        bytes_per_launch = st.algorithmic_bytes / max(1, st.refresh_launches)
        flops_per_launch = st.fft_flops / max(1, st.refresh_launches)
        peaks, peak_kind = measured_peaks()
        achieved_gbs = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
        tr = profiled_traffic(w)
        roofline = {"kernel": "k_refresh (windowed FFT + energy + slot max)", "bound": "hbm",
                    "achieved": achieved_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved_gbs / peaks["hbm_gbs"], "peak_source": f"{peak_kind} hbm_gbs",
                    "traffic": tr, "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum, cold "
                                                      "cache, one epoch scaled to 8 (profiles/"
                                                      "refresh_traffic_mmp2_19x8x5120.json)") if tr else None,
                    "limiter": "FP32/ALU instruction issue, not DRAM: the residual and tables are L2-resident "
                               "(roofline_fp32 is the binding roofline)",
                    "launch_ms": per_launch_ms, "launches": st.refresh_launches,
                    "algorithmic_bytes_per_launch": bytes_per_launch}
        fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12
        roofline_fp32 = {"achieved": flops_per_launch / (per_launch_ms * 1e-3) / 1e12, "unit": "TFLOP/s",
                         "peak": fp32_peak, "peak_source": "nominal FP32 CUDA-core (148 SMs x 128 x 2 x 1.965 GHz)",
                         "frac": flops_per_launch / (per_launch_ms * 1e-3) / 1e12 / fp32_peak,
                         "flops": "reference-equivalent 2.5 Nfft log2 Nfft per refreshed window",
                         "executed_frac": profiled_executed_fp32(w),
                         "executed_source": "ncu FP32 thread instructions of k_refresh<0, 12, 2> (profiles/"
                                            "refresh_traffic_mmp2_19x8x5120.json)" if profiled_executed_fp32(w)
                                            else None}
    bt.close()
    eng_t.close()

    proposal = None
    if args.proposal:
        # the same workload with the block proposal: device time per step, the
        # atoms compared with the plain run's, hit rate and refresh work
        bq = empi_b200.Batch(w.variant, w.energy_error, settings, shapes, w.fs, engine=eng)
        bq.set_proposal(args.proposal, args.proposal_k, args.proposal_weights if args.proposal == "net" else None)
        bq.load(host)
        for _ in range(args.warmup):
            bq.run()
        pq_ms = 0.0
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            torch.cuda.synchronize()
            bq.run()
            pq_ms += bq.stats().run_ms
        sq = bq.stats()
        same = all(np.array_equal(bq.result(e).indices, batch.result(e).indices) and
                   np.array_equal(bq.result(e).atoms, batch.result(e).atoms) for e in range(len(w.epochs)))
        bq.close()
        plain_ms = bs.run_ms
        proposal = {"source": args.proposal, "k": args.proposal_k,
                    "atoms_per_s": atoms_per_step * args.steps / (pq_ms * 1e-3),
                    "plain_atoms_per_s_same_run": atoms_per_step / (plain_ms * 1e-3),
                    "identical_atoms": bool(same),
                    "hit_rate": sq.proposal_hits / max(1, sq.proposal_iterations),
                    "refresh_flops_vs_plain": sq.fft_flops / max(bs.fft_flops, 1e-300),
                    "weights": os.path.basename(args.proposal_weights) if args.proposal == "net" else None}

    ceiling = None
    if args.proposal_probe:
        bp = empi_b200.Batch(w.variant, w.energy_error, settings, shapes, w.fs, engine=eng)
        bp.probe_proposal(True)
        bp.load(host)
        bp.run()
        sp = bp.stats()
        bp.close()
        frac = sp.probe_needed_work / max(sp.probe_dirty_work, 1e-300)
        ceiling = {"needed_work_fraction": frac, "needed_slot_fraction":
                   sp.probe_needed_slots / max(1, sp.probe_dirty_slots),
                   "refresh_speedup_ceiling": 1.0 / max(frac, 1e-300),
                   "what": "share of the refresh rule's FFT work whose upper bound, propagated through each "
                           "subtraction without recomputing, still reached the next certified best: no exact "
                           "block proposal could skip it (one-step bound; atoms unchanged)"}

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(w)
    if rank == 0:
        line = {
            "metric": "atoms/s", "value": value, "unit": "atoms/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": args.scaling, "vs_baseline": None,
            "dtype": "f32 (FFT maps) + f64 (rescore, residual, energies)",
            "data": "synthetic", "config": dict(workload_config(w, world, args.scaling),
                                                **({"job_epochs": job_epochs} if args.scaling == "strong" else {})),
            "e2e": {"value": e2e_value, "unit": "atoms/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches, "roofline": roofline, "roofline_fp32": roofline_fp32,
            "cpu_baseline": base, "clocks": clk, "atoms_per_step": atoms_per_step,
            "candidate_bins_per_atom": bs.candidate_bins / max(1, bs.atoms),
            "proposal_ceiling": ceiling, "proposal": proposal,
            "launch_shape": {"transform_cap": bs.transform_cap, "iterations_per_graph": bs.iterations_per_graph,
                             "wide_mask": bs.wide_mask, "tuned": bool(bs.tuned),
                             "persistent": bool(bs.persistent)},
        }
        print(json.dumps(line))
    batch.close()
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
