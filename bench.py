#!/usr/bin/env python
"""Benchmark of the DVB-S2 LDPC decoder on B200 (and of the reference's CPU
decoder on the same host).

Workload (the configuration the headline metric is quoted on): DVB-S2 normal
FECFRAMEs (n = 64800), code rate 3/5, 8PSK over AWGN with Es/N0 swept
5.0 - 6.5 dB in 0.25 dB steps, int8 LLRs, layered min-sum with at most 30
iterations and syndrome early stop, 4096 frames per launch.  One step = one
decode launch over one 4096-frame batch of one Es/N0 point; the steps cycle
through the seven points.  Inputs are seeded synthetic frames (the project's
encoder, interleaver, 8PSK mapper, AWGN and max-log demapper), generated on
the GPU before timing; each batch is 265 MB, above the 126 MB L2, so no L2
flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  Under torchrun every rank decodes its own
frames (weak scaling, no data-path collective); the time is the max over
ranks of the CUDA-event time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LDPC info Gbit/s at matched FER: learned vs plain min-sum, 1xB200 vs host CPU"
UNIT = "Gbit/s"
RATE, SHORT, CONST = "3_5", 0, "8PSK"
LEARNED_ITERS = 12
ESN0 = [5.0, 5.25, 5.5, 5.75, 6.0, 6.25, 6.5]
MAX_ITER = 30
SMEM_BYTES_PER_CLK = 128  # per SM


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=14)
    ap.add_argument("--warmup", type=int, default=7)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--frames", type=int, default=4096, help="frames per step (launch)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--e2e-steps", type=int, default=7)
    ap.add_argument("--no-learned", action="store_true", help="skip the learned decoder's line items")
    ap.add_argument("--no-bch", action="store_true", help="skip the BCH line item")
    ap.add_argument("--no-group", action="store_true", help="skip the 64-frame group-stopping line item")
    ap.add_argument("--no-dropin", action="store_true", help="skip the drop-in call line item")
    ap.add_argument("--dropin-calls", type=int, default=16, help="64-frame calls per worker thread")
    ap.add_argument("--mix-frames", type=int, default=16384,
                    help="frames of the mixed-MODCOD batch (0: skip that line item)")
    ap.add_argument("--variant", default="auto", choices=["auto", "frame"],
                    help="decoder kernel: automatic choice, or the one-frame kernel")
    ap.add_argument("--per-code", action="store_true",
                    help="print the per-code cost table (us per frame-iteration) instead of the JSON line")
    ap.add_argument("--rates", nargs="*", default=None, help="--per-code: the rates (default: every DVB-S2 rate)")
    ap.add_argument("--short", action="store_true", help="--per-code: short frames")
    ap.add_argument("--batches", type=int, default=len(ESN0),
                    help="Es/N0 points held on the device (small profiling cases use fewer)")
    return ap.parse_args()


def workload_config(frames, world):
    return {
        "workload": "dvbs2-normal-3_5-8psk-awgn-sweep",
        "code": "DVB-S2 normal FECFRAME n=64800 rate 3/5 (kldpc=38880 info bits)",
        "modulation": CONST,
        "esn0_db": ESN0,
        "frames_per_step": frames,
        "max_iter": MAX_ITER,
        "stopping": "per frame (syndrome before every iteration)",
        "llr": "int8, 2 x max-log LLR saturated to +-127",
        "l2": "inputs larger than L2 (265 MB per step), no flush",
        "parallelism": "frames across persistent CTAs; %d rank(s), independent frame shards" % world,
    }


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm),
                "reasons": sorted(reasons)}


def load_learned_table():
    """The committed learned table of the workload's code, or None."""
    from dvbrx_b200 import train as T
    return T.load_table(SHORT, RATE, CONST, LEARNED_ITERS)


def profiled_figures():
    """Figures of the committed ncu summary of the decode kernel: DRAM bytes
    read per frame and written per frame-iteration, issue and ALU-pipe
    utilisation (percent)."""
    path = os.path.join(ROOT, "profiles", "ldpc_decode_normal_3_5.txt")
    out = {}
    if not os.path.exists(path):
        return out
    keys = {"dram_read_bytes_per_frame": "read_per_frame",
            "dram_write_bytes_per_frame_iteration": "write_per_frame_iteration",
            "issue_active_pct": "issue_pct", "alu_pipe_pct": "alu_pct"}
    for line in open(path):
        k = line.split(":", 1)[0]
        if k in keys:
            try:
                out[keys[k]] = float(line.split(":", 1)[1].split()[0])
            except ValueError:
                pass
    return out


# ---------------------------------------------------------------------------
# CPU: the reference decoder compiled from its sources (oracle/_ref)
# ---------------------------------------------------------------------------

def cpu_description(ref):
    """The host CPU and the reference build that runs on it."""
    import oracle
    c = oracle.cpu_info()
    return {"cpu_model": c["model"], "physical_cores": c["physical_cores"], "logical_cpus": c["logical_cpus"],
            "ref_build": "libref_%s.so" % ref.flavour, "march": oracle.flavour_march(ref.flavour),
            "march_note": "compiled for this host's CPU (what -march=native gives here)"
                          if oracle.native_arch() == ref.flavour else
                          "portable ISA level (no build for this CPU model)",
            "lanes": ref.lanes}


def cpu_reference_run(pool, seconds, threads):
    """Reference production mode (rxmt.c:514-536): persistent worker
    threads, each with its own handle, decoding batches of `lanes` frames
    with drx_ldpc_decode (oracle/refbench.c, CLOCK_MONOTONIC) for about
    `seconds`.  Returns (frames/s, frames, RefCode)."""
    import oracle
    ref = oracle.RefCode(SHORT, RATE)
    ref.bench(pool, MAX_ITER, threads, seconds=min(1.0, seconds))  # warm-up: pages, caches, clocks
    step_s, calls = ref.bench(pool, MAX_ITER, threads, seconds=seconds)
    return calls * ref.lanes / step_s[0], calls * ref.lanes, ref


def host_llr_pool(frames_per_point, seed=99):
    """Input frames of the CPU-only arm, made on the CPU (numpy channel):
    the sweep's seven Es/N0 points, one after the other."""
    from oracle import OrcCode, datagen
    code = OrcCode(SHORT, RATE)
    out = []
    for k, es in enumerate(ESN0):
        d = datagen.make_frames(SHORT, RATE, frames_per_point, es, CONST, seed=seed + k, code=code)
        out.append(d["llr"])
    return np.concatenate(out)


def run_reference(args):
    """The reference's own CPU decoder on this host's cores: every step
    decodes as many frames as one GPU step (args.frames) in calls of `lanes`
    frames, shared by persistent worker threads (one handle each, one per
    logical CPU), steps separated by barriers; only rank 0 runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    lib = oracle.load_ref()
    if lib is None or not hasattr(lib, "refx_bench"):
        print(json.dumps({"impl": "reference", "unavailable": "reference decoder not built (oracle/_ref missing)"}))
        return
    threads = oracle.host_threads()
    ref = oracle.RefCode(SHORT, RATE)
    lanes = ref.lanes
    pool = host_llr_pool(128)
    calls = max(1, args.frames // lanes)
    step_s, ncalls = ref.bench(pool, MAX_ITER, threads, steps=args.warmup + args.steps, calls_per_step=calls)
    dt = float(step_s[args.warmup:].sum())
    frames = args.steps * calls * lanes
    gbps = frames * 38880 / dt / 1e9
    cpu = {"value": gbps, "unit": UNIT, "cores": threads, "kind": "reference",
           "sample": "%d steps x %d drx_ldpc_decode calls of %d frames (the sweep's 7 Es/N0 points, 128 "
                     "frames each), %d persistent threads" % (args.steps, calls, lanes, threads)}
    cpu.update(cpu_description(ref))
    line = {
        "metric": METRIC, "value": gbps, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int8", "data": "synthetic",
        "impl": "reference",
        "config": dict(workload_config(calls * lanes, 1),
                       stopping="per batch of %d frames (reference drx_ldpc_decode semantics)" % lanes,
                       frames_per_step=calls * lanes, l2="n/a (host CPU)",
                       parallelism="persistent worker threads, one decoder handle each, one per logical CPU"),
        "cpu_baseline": cpu,
        "e2e": {"value": gbps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

# ---------------------------------------------------------------------------
# ranks: one process per GPU, frames sharded by rank (weak scaling)
# ---------------------------------------------------------------------------

def rank_env():
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init_ranks(world, backend="nccl", timeout_s=120):
    """Process group for world > 1 (a short timeout: ranks that wait for a
    lost peer end with an error)."""
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def rank_seed(rank, k):
    """Seed of Es/N0 batch k on a rank: every rank decodes its own frames."""
    return 1000003 * (rank + 1) + k


def max_over_ranks(x, world, device):
    """The largest x over all ranks (a timed region's milliseconds)."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_gbps(world, frames_per_rank, kldpc, ms):
    """Whole-job information throughput: every rank's frames over the
    slowest rank's time."""
    return world * frames_per_rank * kldpc / (ms * 1e-3) / 1e9


def run_mix(args, world, rank, learned=False):
    """The mixed-MODCOD batch (80 % normal / 20 % short frames, the eleven
    DVB-S2 rates, every MODCOD of the rate, Es/N0 = the MODCOD's QEF value
    + 0.5 dB) as one planned device batch: the tuner's tiling, then timed
    replays of the CUDA graph.  learned: the learned 12-iteration tables of
    every code with the plain decoder as fallback (None if a table is
    missing)."""
    import numpy as np
    import torch

    import dvbrx_b200 as D
    from dvbrx_b200 import modcods as MC
    from dvbrx_b200 import train as T

    n = args.mix_frames
    spec = MC.mixed_batch(n, seed=4242 + rank)
    codes = sorted(set((s, r) for s, r, _, _ in spec))
    cidx = {c: k for k, c in enumerate(codes)}
    code = np.array([cidx[(s, r)] for s, r, _, _ in spec], np.int32)
    tables = {}
    if learned:
        for s, r in codes:
            t = T.load_table(s, r, "QPSK", LEARNED_ITERS) or T.load_table(s, r, "8PSK", LEARNED_ITERS)
            if t is None:
                return None
            tables[(s, r)] = t
    handles = {c: D.Ldpc(D.fec_lookup(*c), c[1]) for c in codes}
    maxb = max(h.nbytes for h in handles.values())
    llr = torch.zeros((n, 64800), dtype=torch.int8, device="cuda")
    info = torch.zeros((n, maxb), dtype=torch.uint8, device="cuda")
    groups = {}
    for f, (s, r, c, es) in enumerate(spec):
        groups.setdefault((s, r, c, es), []).append(f)
    for g, (key, rows) in enumerate(sorted(groups.items())):
        s, r, c, es = key
        h = handles[(s, r)]
        l, inf, _ = h.generate(len(rows), es, seed=rank_seed(rank, 100 + g), constellation=c, const_rate=r,
                               info=True)
        rt = torch.tensor(rows, dtype=torch.long, device="cuda")
        llr[rt, : h.N] = l
        info[rt, : h.nbytes] = inf
    out = torch.zeros((n, maxb), dtype=torch.uint8, device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    ok = torch.zeros(n, dtype=torch.uint8, device="cuda")
    fb = torch.zeros(n, dtype=torch.uint8, device="cuda")
    mix = D.LdpcMix(codes)
    if learned:
        for k, c in enumerate(codes):
            t = tables[c]
            mix.set_learned(k, t["scale"], t["offset"], t["class_of_degree"])
        mix.plan_learned(code, llr, out, it, ok, fb, LEARNED_ITERS, MAX_ITER)
    else:
        mix.plan(code, llr, out, it, ok, MAX_ITER)
    choice, t_one, t_per = mix.tune()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    reps = 3
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        mix.run()
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / reps, world, "cuda")
    bits = sum(handles[(s, r)].kldpc for s, r, _, _ in spec)
    errs = 0
    for c, h in handles.items():
        rows = torch.from_numpy(np.nonzero(code == cidx[c])[0]).cuda()
        errs += int((out[rows, : h.nbytes] != info[rows, : h.nbytes]).any(dim=1).sum())
    res = {"value": aggregate_gbps(world, 1, bits, ms), "unit": UNIT, "frames_per_rank": n, "codes": len(codes),
           "normal_share": float(np.mean([s == 0 for s, _, _, _ in spec])), "ms_per_batch": ms,
           "tiling": {D.TILING_ONE_LAUNCH: "one launch, one frame per CTA", D.TILING_PER_CODE: "per code",
                      D.TILING_ONE_LAUNCH_PAIR: "one launch, two frames per CTA"}[choice],
           "tune_ms": {"one_launch_one_frame_per_cta": t_one, "per_code": t_per,
                       "one_launch_two_frames_per_cta": mix.tuned_ms(D.TILING_ONE_LAUNCH_PAIR)},
           "fer": errs / n,
           "avg_iterations": float(it.float().mean()),
           "esn0": "QEF (EN 302 307-1 Table 13, normal-frame values for both sizes) + 0.5 dB",
           "max_iter": MAX_ITER}
    if learned:
        res.update({"learned_iters": LEARNED_ITERS, "fallback_frac": float(fb.float().mean())})
    mix.close()
    return res


def run_dropin(host_batches, threads, calls_per_thread, world):
    """The reference's own call pattern on the GPU: `threads` host threads
    (the reference receiver's LDPC workers, rxmt.c:514-536), each with its
    own handle, each decoding `calls_per_thread` drx_ldpc_decode calls of 64
    frames from host memory through per-frame pointer arrays (the drop-in
    entry point, reference batch semantics); wall clock over all threads."""
    import ctypes
    import threading

    import dvbrx_b200 as D

    p = D.fec_lookup(SHORT, RATE)
    pool = np.ascontiguousarray(np.concatenate(host_batches))
    handles = [D.Ldpc(p, RATE) for _ in range(threads)]
    nb = handles[0].nbytes
    outs = [np.zeros((64, nb), np.uint8) for _ in range(threads)]
    PtrArr = ctypes.c_void_p * 64

    def calls(w, n):
        out_ptrs = PtrArr(*[outs[w][k].ctypes.data for k in range(64)])
        for c in range(n):
            f0 = ((w * n + c) * 64) % (pool.shape[0] - 63)
            in_ptrs = PtrArr(*[pool[f0 + k].ctypes.data for k in range(64)])
            handles[w]._lib.drx_ldpc_decode(handles[w].h, in_ptrs, out_ptrs, 64, MAX_ITER)

    def run(n):
        ts = [threading.Thread(target=calls, args=(w, n)) for w in range(threads)]
        t0 = time.perf_counter()
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        return time.perf_counter() - t0

    run(2)  # warm-up: scratch, staging, streams
    dt = max_over_ranks(run(calls_per_thread), world, "cuda")
    for h in handles:
        h.close()
    frames = threads * calls_per_thread * 64
    return {"value": aggregate_gbps(world, frames, p.kldpc, dt * 1e3), "unit": UNIT, "threads": threads,
            "frames_per_call": 64, "calls": threads * calls_per_thread, "seconds": dt,
            "api": "drx_ldpc_decode (host per-frame pointers, 64 frames per call, one handle per thread; "
                   "the frames of one call stop together, as in the reference)"}


def run_demap(nframes, world, hbm_peak, reps=5):
    """The soft demapper ahead of the decoder: nframes 8PSK PLFRAMEs of the
    workload's MODCOD (random received symbols; the kernel's work does not
    depend on them) to int8 LLRs; CUDA-event time of the call; an HBM-bound
    kernel (8 bytes of symbol in, 3 LLR bytes out per symbol)."""
    import torch

    import dvbrx_b200 as D

    m = D.Demapper(CONST, RATE, SHORT)
    g = torch.Generator(device="cuda").manual_seed(5)
    sym = torch.randn((nframes, 2 * m.nsym), generator=g, device="cuda")
    n0 = torch.full((nframes,), 0.25, device="cuda")
    llr = torch.empty((nframes, m.nldpc), dtype=torch.int8, device="cuda")
    m.run(sym, n0, llr)
    ms = 0.0
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        m.run(sym, n0, llr)
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    ms = max_over_ranks(ms / reps, world, "cuda")
    nbytes = nframes * (8 * m.nsym + m.nldpc + 4)
    m.close()
    return {"frames_per_rank": nframes, "modcod": "%s %s %s" % (CONST, RATE, "short" if SHORT else "normal"),
            "ms_per_batch": ms, "msym_per_s": world * nframes * m.nsym / ms / 1e3,
            "roofline": {"bound": "hbm", "achieved": nbytes / ms / 1e6, "peak": hbm_peak,
                         "frac": nbytes / ms / 1e6 / hbm_peak, "unit": "GB/s",
                         "algorithmic_bytes_per_launch": nbytes}}


def run_bch(nframes, world, reps=5):
    """The BCH outer code of the workload on the device: nframes random
    BBFRAMEs encoded on the GPU, decoded clean (the receiver's common case,
    the remainder check only) and with t errors per frame at distinct
    positions (syndromes, Berlekamp-Massey and the Chien search for every
    frame); CUDA-event time of the decode calls only."""
    import torch

    import dvbrx_b200 as D

    p = D.fec_lookup(SHORT, RATE)
    b = D.Bch(p)
    nb, kb = p.kldpc // 8, p.kbch // 8
    g = torch.Generator(device="cuda").manual_seed(11)
    clean = torch.zeros((nframes, nb), dtype=torch.uint8, device="cuda")
    clean[:, :kb] = torch.randint(0, 256, (nframes, kb), generator=g, device="cuda", dtype=torch.uint8)
    b.encode_device(clean)
    base = torch.randint(0, p.kldpc, (nframes, 1), generator=g, device="cuda")
    pos = (base + torch.arange(p.t, device="cuda")[None, :] * (p.kldpc // p.t)) % p.kldpc
    masks = torch.zeros((nframes, nb), dtype=torch.int32, device="cuda")
    masks.scatter_add_(1, pos // 8, (1 << (7 - pos % 8)).to(torch.int32))
    noisy = clean ^ masks.to(torch.uint8)
    res = torch.empty(nframes, dtype=torch.int32, device="cuda")
    work = torch.empty_like(clean)
    out = {"frames_per_rank": nframes, "code": "DVB-S2 normal rate 3/5 BCH (nbch %d, kbch %d, t %d)" % (
        p.kldpc, p.kbch, p.t), "unit": UNIT}
    for name, src, want in (("no_error", clean, 0), ("t_errors", noisy, p.t)):
        work.copy_(src)
        b.decode_device(work, res)  # warm-up
        ms = 0.0
        ok = True
        for _ in range(reps):
            work.copy_(src)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            b.decode_device(work, res)
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            ok = ok and bool((res == want).all()) and bool(torch.equal(work, clean))
        ms = max_over_ranks(ms / reps, world, "cuda")
        out[name] = {"value": aggregate_gbps(world, nframes, p.kbch, ms), "ms_per_batch": ms, "all_corrected": ok}
    b.close()
    return out


def run_b200(args):
    import torch
    import torch.distributed as dist

    import dvbrx_b200 as D

    world, rank, local = rank_env()
    torch.cuda.set_device(local)
    init_ranks(world, "nccl")

    p = D.fec_lookup(SHORT, RATE)
    dec = D.Ldpc(p, RATE)
    variant = dec.set_variant(D.VARIANT_FRAME if args.variant == "frame" else D.VARIANT_AUTO)
    kernel_name = {D.VARIANT_PAIR: "drxg::k_decode_pair (two frames per CTA, 16x2 SIMD)",
                   D.VARIANT_FRAME: "drxg::k_decode (one frame per CTA)"}[variant]
    F = args.frames
    kldpc = p.kldpc
    stream = torch.cuda.current_stream()

    # inputs: one batch per Es/N0 point, resident in HBM
    llr, info = [], []
    for k, es in enumerate(ESN0[: args.batches]):
        l, inf, _ = dec.generate(F, es, seed=rank_seed(rank, k), constellation=CONST, info=True)
        llr.append(l)
        info.append(inf)
    outs = [torch.empty((F, dec.nbytes), dtype=torch.uint8, device="cuda") for _ in range(args.steps)]
    out = outs[0]
    iters = [torch.empty(F, dtype=torch.int32, device="cuda") for _ in range(args.steps)]
    oks = [torch.empty(F, dtype=torch.uint8, device="cuda") for _ in range(args.steps)]
    errs = torch.zeros(args.steps, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()

    def step(k, it_buf, ok_buf, out_buf=None):
        dec.decode_device(llr[k % len(llr)], MAX_ITER, out=out if out_buf is None else out_buf, iters=it_buf,
                          ok=ok_buf)

    for k in range(args.warmup):
        step(k, iters[0], oks[0])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    sampler = ClockSampler(local)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    for k in range(args.steps):
        ev[k][0].record(stream)
        step(args.warmup + k, iters[k], oks[k], outs[k])
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    # frame errors of every step, after the timed region
    for k in range(args.steps):
        errs[k] = (outs[k] != info[(args.warmup + k) % len(info)]).any(dim=1).sum()
    clocks = sampler.stop()
    launch_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(ev[0][0].elapsed_time(ev[-1][1]), world, "cuda")

    it_all = torch.stack(iters).to(torch.int64)
    iters_sum = int(it_all.sum().item())
    frames_rank = args.steps * F
    fer = float(errs.sum().item()) / frames_rank
    value = aggregate_gbps(world, frames_rank, kldpc, total_ms)

    # roofline of the decode kernel (one launch per step)
    edges = dec.info.edges
    kern_s = statistics.mean(launch_ms) * 1e-3
    smem_bytes = iters_sum / args.steps * 4 * edges
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    smem_peak = nsm * SMEM_BYTES_PER_CLK * 1965e6 / 1e9
    hbm_bytes = F * (dec.N + dec.nbytes + 5)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    prof = profiled_figures()
    traffic = None
    if "read_per_frame" in prof and "write_per_frame_iteration" in prof:
        traffic = prof["read_per_frame"] * F + prof["write_per_frame_iteration"] * iters_sum / args.steps
    roofline = {
        "bound": "smem",
        "kernel": kernel_name,
        "achieved": smem_bytes / kern_s / 1e9,
        "peak": smem_peak,
        "unit": "GB/s",
        "frac": smem_bytes / kern_s / 1e9 / smem_peak,
        "peak_source": "nominal: %d SMs x 128 B/clk x 1965 MHz (no shared-memory peak in MEASURED_PEAKS.json)" % nsm,
        "algorithmic_bytes_per_launch": smem_bytes,
        "bytes_per_unit": "4 x E = %d B per frame-iteration (E = %d edges)" % (4 * edges, edges),
        "traffic": traffic,
        "traffic_note": "DRAM bytes read + written per launch: ncu on a 2048-frame, 30-iteration launch, "
                        "reads scaled by this launch's frames and writes (L2 write-backs of the per-CTA "
                        "message slab) by its frame-iterations; against the HBM algorithmic bytes below",
        "issue": {"issue_active_pct": prof.get("issue_pct"), "alu_pipe_pct": prof.get("alu_pct"),
                  "note": "ncu on the profiled small case: integer issue on the ALU pipe binds"},
        "hbm": {"achieved": hbm_bytes / kern_s / 1e9, "peak": hbm_peak,
                "frac": hbm_bytes / kern_s / 1e9 / hbm_peak, "unit": "GB/s",
                "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback",
                "algorithmic_bytes_per_launch": hbm_bytes},
        "avg_launch_ms": statistics.mean(launch_ms),
        "gap_ms_per_step": (total_ms - sum(launch_ms)) / args.steps,
        "sm_mhz_median": sm_mhz,
    }

    # the same batches with the reference's batch semantics: groups of 64
    # frames (drx_ldpc_decode on 64 lanes) iterate until all their frames pass
    group64 = None
    if not args.no_group:
        g_it = [torch.empty(F, dtype=torch.int32, device="cuda") for _ in range(args.steps)]
        g_ok = [torch.empty(F, dtype=torch.uint8, device="cuda") for _ in range(args.steps)]
        for k in range(min(args.warmup, 3)):
            dec.decode_device(llr[k % len(llr)], MAX_ITER, out=outs[0], iters=g_it[0], ok=g_ok[0], stop=64)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        gev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            gev[k][0].record(stream)
            dec.decode_device(llr[(args.warmup + k) % len(llr)], MAX_ITER, out=outs[k], iters=g_it[k], ok=g_ok[k],
                              stop=64)
            gev[k][1].record(stream)
        torch.cuda.synchronize()
        g_ms = max_over_ranks(gev[0][0].elapsed_time(gev[-1][1]), world, "cuda")
        g_iters = torch.stack(g_it).to(torch.int64)
        group64 = {"value": aggregate_gbps(world, frames_rank, kldpc, g_ms), "unit": UNIT,
                   "ms_per_step": g_ms / args.steps,
                   "stopping": "groups of 64 consecutive frames stop together (the reference's "
                               "drx_ldpc_decode batch semantics on 64 lanes)",
                   "avg_iterations": float(g_iters.float().mean()),
                   "frame_iterations_vs_per_frame": float(g_iters.sum()) / max(1, iters_sum),
                   "launch": "one cooperative launch per step, teams of 32 co-resident CTAs per group"}

    # the learned decoder on the same batches and steps: the committed
    # 12-iteration table with the plain decoder as fallback (the plain
    # decoder's FER), and the 30-iteration table in one pass (the plain
    # decoder's iteration budget, its own FER)
    def per_point(errors):
        """frame error rate of each Es/N0 point over the timed steps"""
        n = [0] * len(llr)
        e = [0] * len(llr)
        for k in range(args.steps):
            b = (args.warmup + k) % len(llr)
            n[b] += F
            e[b] += int(errors[k])
        return [round(e[b] / n[b], 5) if n[b] else None for b in range(len(llr))]

    plain_fer_points = per_point(errs.tolist())

    def run_learned(table, fallback_iters):
        from dvbrx_b200 import train as T
        T.apply_table(dec, table)
        L = int(table["iters"])
        l_it = [torch.empty(F, dtype=torch.int32, device="cuda") for _ in range(args.steps)]
        l_ok = [torch.empty(F, dtype=torch.uint8, device="cuda") for _ in range(args.steps)]
        l_fb = [torch.empty(F, dtype=torch.uint8, device="cuda") for _ in range(args.steps)]
        for k in range(args.warmup):
            dec.decode_learned(llr[k % len(llr)], L, fallback_iters, out=outs[0], iters=l_it[0], ok=l_ok[0],
                               fallback=l_fb[0])
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        lev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            lev[k][0].record(stream)
            dec.decode_learned(llr[(args.warmup + k) % len(llr)], L, fallback_iters, out=outs[k], iters=l_it[k],
                               ok=l_ok[k], fallback=l_fb[k])
            lev[k][1].record(stream)
        torch.cuda.synchronize()
        l_ms = max_over_ranks(lev[0][0].elapsed_time(lev[-1][1]), world, "cuda")
        l_errs = [int((outs[k] != info[(args.warmup + k) % len(info)]).any(dim=1).sum()) for k in range(args.steps)]
        fb_all = torch.stack(l_fb).float()
        lval = aggregate_gbps(world, frames_rank, kldpc, l_ms)
        dec.set_learned(None, None, None)
        res = {
            "value": lval, "unit": UNIT, "vs_plain": lval / value, "fer": sum(l_errs) / frames_rank, "plain_fer": fer,
            "fer_per_point": per_point(l_errs), "plain_fer_per_point": plain_fer_points, "esn0_db": ESN0[: len(llr)],
            "avg_iterations": float(torch.stack(l_it).float().mean()),
            "plain_avg_iterations": iters_sum / frames_rank,
            "learned_iters": L, "ms_per_step": l_ms / args.steps,
            "table": "dvbrx_b200/learned_tables/" + os.path.basename(T.table_path(SHORT, RATE, CONST, L)),
        }
        if fallback_iters:
            res.update({
                "fallback_frac": float(fb_all.mean()),
                "avg_iterations_learned_pass": float(torch.stack(l_it).float()[fb_all == 0].mean())
                if bool((fb_all == 0).any()) else None,
                "plain_fallback_max_iter": fallback_iters, "launches_per_step": 3,
                "decoder": "learned scaled/offset min-sum at int8 (Q8 table per iteration and degree class), "
                           "frames failing the syndrome re-decoded by the plain decoder on the device"})
        else:
            res.update({
                "launches_per_step": 1,
                "decoder": "learned scaled/offset min-sum at int8 (Q8 table per iteration and degree class), "
                           "one pass of at most %d iterations with per-frame stopping, no plain decoder" % L})
        return res

    learned = learned30 = None
    if not args.no_learned:
        from dvbrx_b200 import train as T
        t12 = load_learned_table()
        if t12 is not None:
            learned = run_learned(t12, MAX_ITER)
        t30 = T.load_table(SHORT, RATE, CONST, MAX_ITER)
        if t30 is not None:
            learned30 = run_learned(t30, 0)

    # the drop-in call as the reference's workers make it: 16 threads, 64-frame calls, host memory
    dropin = None
    if not args.no_dropin:
        dropin = run_dropin([l[:1024].cpu().numpy() for l in llr], 16, args.dropin_calls, world)

    # the BCH outer code behind the decoder, the demapper ahead of it
    bch = None if args.no_bch else run_bch(F, world)
    demap = None if args.no_bch else run_demap(F, world, hbm_peak)

    # the mixed-MODCOD batch, plain and learned with fallback
    mix_res = mix_learned = None
    if args.mix_frames > 0:
        mix_res = run_mix(args, world, rank)
        if not args.no_learned:
            mix_learned = run_mix(args, world, rank, learned=True)
        torch.cuda.empty_cache()

    # end to end through the C ABI with host buffers (synchronous call)
    e2e = None
    if args.e2e_steps > 0:
        # pinned host rows in and out (the copy engines read and write them directly), the output
        # buffers allocated once and reused, as a receiver decoding batch after batch does
        host_t = [l.cpu().pin_memory() for l in llr]
        host = [t.numpy() for t in host_t]
        out_t = [torch.zeros((F, dec.nbytes), dtype=torch.uint8).pin_memory(),
                 torch.zeros(F, dtype=torch.int32).pin_memory(), torch.zeros(F, dtype=torch.uint8).pin_memory()]
        h_out, h_it, h_ok = (t.numpy() for t in out_t)
        for k in range(min(2, args.e2e_steps)):
            dec.decode_host(host[k % len(host)], MAX_ITER, out=h_out, iters=h_it, ok=h_ok)
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for k in range(args.e2e_steps):
            dec.decode_host(host[k % len(host)], MAX_ITER, out=h_out, iters=h_it, ok=h_ok)
        dt = max_over_ranks(time.perf_counter() - t0, world, "cuda")
        e2e = {"value": aggregate_gbps(world, args.e2e_steps * F, kldpc, dt * 1e3), "unit": UNIT,
               "h2d_bytes_per_step": F * dec.N,
               "d2h_bytes_per_step": F * (dec.nbytes + 4 + 1),
               "api": "drx_ldpc_decode_host (pinned host rows in, pinned host bits/iterations/flags out; "
                      "wall clock)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            import oracle
            pool = np.concatenate([l[:128].cpu().numpy() for l in llr])
            threads = oracle.host_threads()
            fps, nf, ref = cpu_reference_run(pool, args.cpu_seconds, threads)
            fps1, _, _ = cpu_reference_run(pool, min(3.0, args.cpu_seconds), 1)
            cpu = {"value": fps * kldpc / 1e9, "unit": UNIT, "cores": threads, "kind": "reference",
                   "value_1core": fps1 * kldpc / 1e9,
                   "sample": "%d frames in %.0f s: drx_ldpc_decode calls of %d frames by %d persistent "
                             "threads (one handle each), the same int8 LLRs as the GPU (128 frames of each "
                             "Es/N0 point)" % (nf, args.cpu_seconds, ref.lanes, threads)}
            cpu.update(cpu_description(ref))
        except Exception as e:  # the baseline is reported, not required
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": "failed: %s" % e}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int8", "data": "synthetic",
            "config": workload_config(F, world),
            "decoder": "plain layered offset min-sum (bit-exact to the reference)",
            "quality": {"fer": fer, "avg_iterations": iters_sum / frames_rank},
            "roofline": roofline, "clocks": clocks, "e2e": e2e, "cpu_baseline": cpu, "group64": group64,
            "dropin": dropin,
            "learned": learned, "learned_30it_one_pass": learned30,
            "mixed_modcod": mix_res, "mixed_modcod_learned": mix_learned, "bch": bch, "demapper": demap,
            "gpu_launches": args.steps,
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


NORMAL_RATES = ["1_4", "1_3", "2_5", "1_2", "3_5", "2_3", "3_4", "4_5", "5_6", "8_9", "9_10"]


def frame_iteration_us(dec, variant, n, seed=7):
    """Microseconds of the whole GPU per frame-iteration of one kernel on one
    code: n frames generated far below the code's threshold (no frame
    converges, every frame runs its iterations); (t(30) - t(10)) / 20 / n
    from CUDA events, best of five."""
    import torch

    import dvbrx_b200 as D

    dec.set_variant(variant)
    llr, _, _ = dec.generate(n, -6.0, seed=seed)
    t = {}
    for it in (10, 30):
        best = float("inf")
        for _ in range(5):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            _, _, ok = dec.decode_device(llr, it)
            b.record()
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        t[it] = best
    assert int(ok.sum()) == 0, "a frame converged: the case must stay below threshold"
    dec.set_variant(D.VARIANT_AUTO)
    return (t[30] - t[10]) / 20 * 1e3 / n


def run_per_code(args):
    """--per-code: decoder cost per DVB-S2 code (frame-pair kernel against
    the one-frame kernel), several full waves of frames per code (6 per SM
    for normal frames, 24 for short ones: every CTA of either kernel busy).
    Prints a table, not the JSON line."""
    import torch

    import dvbrx_b200 as D

    short = int(args.short)
    n = (24 if short else 6) * torch.cuda.get_device_properties(0).multi_processor_count
    print("%-6s %-6s %12s %12s %8s" % ("frame", "rate", "pair us", "frame us", "ratio"))
    for rate in args.rates or NORMAL_RATES:
        if short and rate == "9_10":
            continue
        dec = D.Ldpc(D.fec_lookup(short, rate), rate)
        pair = frame_iteration_us(dec, D.VARIANT_PAIR, n)
        one = frame_iteration_us(dec, D.VARIANT_FRAME, n)
        print("%-6s %-6s %12.3f %12.3f %8.2f" % ("short" if short else "normal", rate, pair, one, one / pair))
        dec.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.per_code:
        run_per_code(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
