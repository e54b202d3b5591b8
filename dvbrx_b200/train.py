"""Train the learned (neural offset / scaled) min-sum decoder on the GPU and
evaluate it against the plain decoder.

    python -m dvbrx_b200.train --rate 2_3 --iters 20 --batch 512 --es 6.0 7.5 --steps 300 \\
        --out table.json
    python -m dvbrx_b200.train --eval table.json --es-list 6.0 6.25 6.5 --frames 4096

Training data: the library's own frame generator (random information bits,
the DVB-S2 encoder, the MODCOD's constellation and interleaver, AWGN, the
max-log demapper) with FP16 LLRs on the int8 decoder's scale (2 x LLR,
unquantised); every minibatch is drawn in chunks, each at its own Es/N0
uniform in the given range.  Loss: mean binary cross-entropy of the
information-bit posteriors after every unrolled iteration, through the
hand-written forward and backward kernels (learned.LearnedMinSum).

The exported table (JSON: scale and offset [iters][classes], the class of
every check degree) is what Ldpc.set_learned / drx_ldpc_set_learned load;
the int8 decoders round it to Q8.

Data-parallel on several GPUs (one process per GPU, torchrun): every rank
draws its own minibatches (a rank-dependent seed) and the gradient of the
tables, a few hundred numbers, is averaged with one all-reduce per step, so
the ranks keep identical tables; rank 0 logs and writes the table.

    torchrun --nproc-per-node 8 -m dvbrx_b200.train --rate 3_5 --const 8PSK ...
"""
import argparse
import json
import os
import sys
import time

import numpy as np
import torch

from . import FecParams, Ldpc, code_info, fec_lookup
from .learned import LearnedDecoder, degree_classes, learned_posteriors

TABLES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "learned_tables")


def dist_world():
    """(world size, rank) of the initialised process group, (1, 0) without one."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def rank_seed(seed, rank):
    """Minibatch seed of a rank: distinct frames on every rank."""
    return seed + 1000003 * rank


def average_gradients(params, world):
    """Mean of every parameter's gradient over the ranks, in one all-reduce
    of the flattened gradients (the learned tables are small)."""
    import torch.distributed as dist

    grads = [p.grad for p in params if p.grad is not None]
    if world <= 1 or not grads:
        return
    flat = torch.cat([g.reshape(-1) for g in grads])
    dist.all_reduce(flat)
    flat /= world
    k = 0
    for g in grads:
        n = g.numel()
        g.copy_(flat[k:k + n].view_as(g))
        k += n


def table_path(short_frame, rate, constellation, iters):
    return os.path.join(TABLES, "%s_%s_%s_%dit.json" % ("short" if short_frame else "normal", rate,
                                                        constellation.lower(), iters))


def load_table(short_frame, rate, constellation, iters):
    """A committed learned table, or None."""
    path = table_path(short_frame, rate, constellation, iters)
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


def apply_table(dec, table):
    """Load a table (dict as exported) into a decoder handle."""
    dec.set_learned(np.asarray(table["scale"], np.float32), np.asarray(table["offset"], np.float32),
                    np.asarray(table["class_of_degree"], np.int8))


def _params(short_frame, rate):
    try:
        return fec_lookup(short_frame, rate)
    except KeyError:
        info = code_info(short_frame, rate)
        return FecParams(int(bool(short_frame)), info.nldpc, info.K, info.K, 0)


def minibatch(dec, n, es_lo, es_hi, constellation, rng, chunks=8):
    """n frames in `chunks` groups, each at an Es/N0 drawn uniformly in
    [es_lo, es_hi]: (FP16 LLRs [n, N], packed information bits [n, nbytes])."""
    sizes = [n // chunks + (1 if k < n % chunks else 0) for k in range(chunks)]
    llrs, infos = [], []
    for s in sizes:
        if s == 0:
            continue
        es = float(rng.uniform(es_lo, es_hi))
        _, info, h = dec.generate(s, es, seed=int(rng.integers(1, 2**62)), constellation=constellation, llr=False,
                                  info=True, llr_f16=True)
        llrs.append(h)
        infos.append(info)
    return torch.cat(llrs), torch.cat(infos)


def int8_minibatch(dec, n, es_lo, es_hi, constellation, rng, chunks=8, decodable_iters=0, max_draws=6):
    """n frames in `chunks` groups, each at an Es/N0 drawn uniformly in
    [es_lo, es_hi], as the int8 decoder receives them (the quantised int8
    LLRs, carried in FP16 exactly): (FP16 LLRs [n, N], packed information
    bits).  With the int8 inputs, the float model at scale 1 and offset 1 is
    the plain int8 decoder frame for frame.  decodable_iters > 0 keeps only
    the frames the plain int8 decoder decodes correctly within that many
    iterations (the loss then rewards reaching the right answer sooner, not
    lower confidence on frames no decoder recovers); the draw is repeated
    until n frames are kept (at most max_draws times, the kept frames then
    repeated to fill the batch)."""
    sizes = [n // chunks + (1 if k < n % chunks else 0) for k in range(chunks)]
    llrs, infos, have = [], [], 0
    for _ in range(max_draws):
        for s in sizes:
            if s == 0:
                continue
            es = float(rng.uniform(es_lo, es_hi))
            llr, info, _ = dec.generate(s, es, seed=int(rng.integers(1, 2**62)), constellation=constellation,
                                        info=True)
            if decodable_iters > 0:
                bits, _, _ = dec.decode_device(llr, decodable_iters)
                good = (bits == info).all(dim=1)
                llr, info = llr[good], info[good]
            llrs.append(llr)
            infos.append(info)
            have += llr.shape[0]
        if have >= n:
            break
    llr, info = torch.cat(llrs), torch.cat(infos)
    if llr.shape[0] == 0:
        raise RuntimeError("no decodable frame in the Es/N0 range")
    if llr.shape[0] < n:
        idx = torch.arange(n, device=llr.device) % llr.shape[0]
        llr, info = llr[idx], info[idx]
    return llr[:n].to(torch.float16), info[:n]


def int8_selection_set(dec, es_points, n, constellation, seed=4321):
    """Fixed frames for model selection: int8 LLRs and information bits per
    Es/N0 point."""
    out = []
    for k, es in enumerate(es_points):
        llr, info, _ = dec.generate(n, float(es), seed=seed + k, constellation=constellation, info=True)
        out.append((float(es), llr, info))
    return out


def int8_fer(dec, beta, alpha, cod, sset, iters):
    """FER of the int8 learned decoder (the table rounded to Q8 as the library
    does, no fallback) on a selection set, and its mean iterations."""
    dec.set_learned(beta.detach().float().cpu().numpy(), alpha.detach().float().cpu().numpy(), cod)
    errs = frames = 0
    its = 0.0
    for _, llr, info in sset:
        bits, it, _, _ = dec.decode_learned(llr, iters, 0)
        errs += int((bits != info).any(dim=1).sum())
        frames += llr.shape[0]
        its += float(it.float().sum())
    dec.set_learned(None, None, None)
    return errs / frames, its / frames


def loss_weights(kind, iters):
    """Per-iteration weights of the BCE sums: "uniform", "ramp" ((t + 1) / T)
    or "last" (the final iteration only)."""
    if kind == "uniform":
        return np.ones(iters, np.float32)
    if kind == "ramp":
        return (np.arange(iters, dtype=np.float32) + 1) / iters
    if kind == "last":
        w = np.zeros(iters, np.float32)
        w[-1] = 1.0
        return w
    raise ValueError(kind)


def validation_set(dec, es_points, n, constellation, seed=99):
    """Fixed frames: one (FP16 LLRs, info bits) pair per Es/N0 point."""
    out = []
    for k, es in enumerate(es_points):
        _, info, h = dec.generate(n, float(es), seed=seed + k, constellation=constellation, llr=False, info=True,
                                  llr_f16=True)
        out.append((float(es), h, info))
    return out


def validate(model, vset):
    """Per Es/N0 point: mean BCE of the last iteration and the FER of the
    float model's final hard decisions."""
    b, a = model.fp16_tables()
    res = []
    for es, h, info in vset:
        loss, post = learned_posteriors(model.dec, b, a, model.cod, h, info, model.iters)
        bits = torch.from_numpy(np.unpackbits(info.cpu().numpy(), axis=1)[:, : model.dec.kldpc]).cuda()
        err = ((post < 0).to(torch.uint8) != bits).any(dim=1).float().mean()
        res.append({"esn0_db": es, "bce_last": float(loss[-1]) / (h.shape[0] * model.dec.kldpc),
                    "float_fer": float(err)})
    return res


def train(short_frame, rate, constellation, iters, batch, es_lo, es_hi, steps, lr, seed, log=None,
          weights="uniform", val_points=None, int8_inputs=False, decodable_iters=0, select_points=None,
          select_frames=1024, eval_every=20, floor_points=None, floor_frames=4096, max_scale=4.0):
    """Adam on the fp32 masters of the FP16 tables, initialised to the
    plain decoder (scale 1, offset 1).  int8_inputs / decodable_iters: the
    minibatches of int8_minibatch.  select_points: Es/N0 points of a fixed
    selection set; every eval_every steps the int8 learned decoder's FER at
    `iters` iterations is measured there, and the model keeps the best tables
    seen (the plain decoder's to start with), so that the result is never
    worse than the plain decoder on that set.  floor_points: Es/N0 points above
    the waterfall (floor_frames frames each) where a table is kept only if it
    fails no more frames than the plain decoder does.  max_scale: the upper
    bound of every scale.  Returns (model, history)."""
    world, rank = dist_world()
    torch.manual_seed(seed)
    rng = np.random.default_rng(rank_seed(seed, rank))
    model = LearnedDecoder(short_frame, rate, iters=iters, params=_params(short_frame, rate),
                           weights=loss_weights(weights, iters))
    vset = validation_set(model.dec, val_points or [es_lo, (es_lo + es_hi) / 2, es_hi], 256, constellation)
    if log:
        log(json.dumps({"validation_init": validate(model, vset)}))
    opt = torch.optim.Adam(model.parameters(), lr=lr)
    hist = []
    sset = int8_selection_set(model.dec, select_points, select_frames, constellation) if select_points else None
    fset = int8_selection_set(model.dec, floor_points, floor_frames, constellation, seed=8765) if floor_points else None
    floor0 = int8_fer(model.dec, model.beta, model.alpha, model.cod, fset, iters)[0] if fset else 0.0
    best = None
    if sset:
        f0, i0 = int8_fer(model.dec, model.beta, model.alpha, model.cod, sset, iters)
        best = (f0, i0, model.beta.detach().clone(), model.alpha.detach().clone(), -1)
        model.selection = {"plain_fer": f0, "plain_avg_iters": i0}
        if log:
            log(json.dumps({"selection_plain": {"fer": f0, "avg_iters": i0}}))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for k in range(steps):
        if int8_inputs or decodable_iters:
            llr16, info = int8_minibatch(model.dec, batch, es_lo, es_hi, constellation, rng,
                                         decodable_iters=decodable_iters)
        else:
            llr16, info = minibatch(model.dec, batch, es_lo, es_hi, constellation, rng)
        torch.cuda.synchronize()
        ev0.record()
        loss = model(llr16, info)
        opt.zero_grad()
        loss.backward()
        average_gradients(list(model.parameters()), world)
        opt.step()
        with torch.no_grad():
            model.beta.clamp_(0.0, max_scale)
        ev1.record()
        torch.cuda.synchronize()
        rec = {"step": k, "loss": float(loss.detach()), "ms": ev0.elapsed_time(ev1)}
        if sset and ((k + 1) % eval_every == 0 or k == steps - 1):
            f, i = int8_fer(model.dec, model.beta, model.alpha, model.cod, sset, iters)
            rec.update({"select_fer": f, "select_avg_iters": i})
            ok = True
            if fset:
                ff = int8_fer(model.dec, model.beta, model.alpha, model.cod, fset, iters)[0]
                rec["floor_fer"] = ff
                ok = ff <= floor0
            if ok and (f, i) < (best[0], best[1]):
                best = (f, i, model.beta.detach().clone(), model.alpha.detach().clone(), k)
        hist.append(rec)
        if log and (k % 10 == 0 or k == steps - 1):
            log(json.dumps(rec))
    if best is not None:
        with torch.no_grad():
            model.beta.copy_(best[2])
            model.alpha.copy_(best[3])
        model.selection.update({"fer": best[0], "avg_iters": best[1], "step": best[4],
                                "points": list(select_points), "frames_per_point": select_frames})
        if fset:
            model.selection.update({"floor_points": list(floor_points), "floor_frames_per_point": floor_frames,
                                    "plain_floor_fer": floor0})
        if log:
            log(json.dumps({"selection_best": model.selection}))
    model.validation = validate(model, vset)
    if log:
        log(json.dumps({"validation_final": model.validation}))
    return model, hist


def export(model, meta):
    b, a = model.fp16_tables()
    t = dict(meta)
    t.update({"iters": model.iters, "degrees": model.degrees, "class_of_degree": [int(v) for v in model.cod],
              "scale": b.float().cpu().numpy().tolist(), "offset": a.float().cpu().numpy().tolist()})
    return t


def evaluate(short_frame, rate, constellation, table, es_list, nframes, learned_iters, plain_iters, seed=7):
    """FER of plain@plain_iters, plain@learned_iters, learned@learned_iters
    and learned + plain fallback on the same frames, with device-timed
    Gbit/s of the plain, the learned + fallback and the learned-only
    (one pass, no fallback) decodes."""
    p = _params(short_frame, rate)
    dec = Ldpc(p, rate)
    apply_table(dec, table)
    rows = []
    for k, es in enumerate(es_list):
        llr, info, _ = dec.generate(nframes, float(es), seed=seed + 1000 * k, constellation=constellation, info=True)
        res = {"esn0_db": float(es)}
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        dec.decode_device(llr, plain_iters)  # warm-up
        dec.decode_learned(llr, learned_iters, plain_iters)
        torch.cuda.synchronize()
        ev[0].record()
        pb, pi, po = dec.decode_device(llr, plain_iters)
        ev[1].record()
        lb, li, lo, fb = dec.decode_learned(llr, learned_iters, plain_iters)
        ev[2].record()
        torch.cuda.synchronize()
        sb, si, so = dec.decode_device(llr, learned_iters)
        ob, oi, oo, _ = dec.decode_learned(llr, learned_iters, 0)
        ev[3].record()
        dec.decode_learned(llr, learned_iters, 0, out=ob, iters=oi, ok=oo)
        ev[4].record()
        torch.cuda.synchronize()

        def fer(bits):
            return float((bits != info).any(dim=1).float().mean())

        def ber(bits):
            x = torch.bitwise_xor(bits, info)
            ones = sum(int(((x >> b) & 1).sum()) for b in range(8))
            return ones / float(nframes * p.kldpc)

        t_plain = ev[0].elapsed_time(ev[1]) * 1e-3
        t_learn = ev[1].elapsed_time(ev[2]) * 1e-3
        t_only = ev[3].elapsed_time(ev[4]) * 1e-3
        res.update({
            "plain_fer": fer(pb), "plain_ber": ber(pb), "plain_avg_iters": float(pi.float().mean()),
            "plain_short_fer": fer(sb),
            "learned_only_fer": fer(ob), "learned_only_avg_iters": float(oi.float().mean()),
            "learned_fer": fer(lb), "learned_ber": ber(lb), "fallback_frac": float(fb.float().mean()),
            "plain_gbps": nframes * p.kldpc / t_plain / 1e9, "learned_gbps": nframes * p.kldpc / t_learn / 1e9,
            "learned_only_gbps": nframes * p.kldpc / t_only / 1e9,
        })
        rows.append(res)
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--short", type=int, default=0)
    ap.add_argument("--rate", default="2_3")
    ap.add_argument("--const", default="8PSK")
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--es", type=float, nargs=2, default=[6.0, 7.5])
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--lr", type=float, default=0.02)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=None, help="table JSON (default: the package's table path)")
    ap.add_argument("--eval", default=None, help="evaluate this table JSON instead of training")
    ap.add_argument("--es-list", type=float, nargs="*", default=None)
    ap.add_argument("--frames", type=int, default=2048)
    ap.add_argument("--plain-iters", type=int, default=30)
    ap.add_argument("--weights", default="uniform", choices=["uniform", "ramp", "last"])
    ap.add_argument("--val", type=float, nargs="*", default=None, help="validation Es/N0 points")
    ap.add_argument("--int8-inputs", action="store_true",
                    help="train on the int8 LLRs the decoder receives (carried in FP16)")
    ap.add_argument("--decodable", type=int, default=0,
                    help="keep only frames the plain int8 decoder decodes within this many iterations")
    ap.add_argument("--select", type=float, nargs="*", default=None,
                    help="Es/N0 points of the model-selection set (int8 FER at --iters iterations)")
    ap.add_argument("--select-frames", type=int, default=1024)
    ap.add_argument("--select-floor", type=float, nargs="*", default=None,
                    help="Es/N0 points above the waterfall where a kept table fails no more frames than plain")
    ap.add_argument("--floor-frames", type=int, default=4096)
    ap.add_argument("--max-scale", type=float, default=4.0, help="upper bound of the trained scales")
    ap.add_argument("--select-offsets", type=float, nargs="*", default=None,
                    help="--all-s2: selection points as offsets (dB) from each rate's QEF Es/N0")
    ap.add_argument("--all-s2", action="store_true",
                    help="one table per DVB-S2 code (normal and short), trained on the rate's QPSK MODCOD over "
                         "[QEF - 0.25, QEF + 0.75] dB, into --out-dir")
    ap.add_argument("--out-dir", default=None)
    a = ap.parse_args(argv)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl")
    world, rank = dist_world()
    log = (lambda s: print(s, flush=True)) if rank == 0 else (lambda s: None)
    if a.all_s2:
        from .modcods import RATES, qef_db
        out_dir = a.out_dir or TABLES
        os.makedirs(out_dir, exist_ok=True)
        for short in (0, 1):
            for rate in RATES:
                if short and rate == "9_10":
                    continue
                q = qef_db("QPSK", rate)
                es = [q - 0.25, q + 0.75]
                t0 = time.time()
                # selection (with --select-offsets): the int8 learned FER at QEF + each offset
                sel = [q + o for o in a.select_offsets] if a.select_offsets else None
                model, hist = train(short, rate, "QPSK", a.iters, a.batch, es[0], es[1], a.steps, a.lr, a.seed,
                                    None, a.weights, [q, q + 0.25, q + 0.5], int8_inputs=a.int8_inputs,
                                    decodable_iters=a.decodable, select_points=sel, select_frames=a.select_frames)
                ms = [h["ms"] for h in hist[1:]] or [hist[0]["ms"]]
                meta = {"short": short, "rate": rate, "constellation": "QPSK", "es": es, "batch": a.batch,
                        "steps": a.steps, "lr": a.lr, "seed": a.seed, "weights": a.weights,
                        "validation": model.validation, "int8_inputs": a.int8_inputs,
                        "decodable_iters": a.decodable, "selection": getattr(model, "selection", None),
                        "loss_first": hist[0]["loss"],
                        "loss_last": float(np.mean([h["loss"] for h in hist[-10:]])),
                        "train_ms_per_step": float(np.median(ms)),
                        "train_frames_per_s": a.batch / (float(np.median(ms)) * 1e-3),
                        "train_wall_s": time.time() - t0}
                table = export(model, meta)
                path = os.path.join(out_dir, os.path.basename(table_path(short, rate, "QPSK", a.iters)))
                if rank == 0:
                    with open(path, "w") as f:
                        json.dump(table, f, indent=1)
                log(json.dumps({"table": os.path.basename(path), "wall_s": meta["train_wall_s"],
                                "validation": model.validation}))
                del model
                torch.cuda.empty_cache()
        return 0
    if a.eval:
        with open(a.eval) as f:
            table = json.load(f)
        es_list = a.es_list or list(np.arange(table["es"][0], table["es"][1] + 1e-6, 0.25))
        rows = evaluate(table["short"], table["rate"], table["constellation"], table, es_list, a.frames,
                        table["iters"], a.plain_iters)
        for r in rows:
            log(json.dumps(r))
        return 0
    t0 = time.time()
    model, hist = train(a.short, a.rate, a.const, a.iters, a.batch, a.es[0], a.es[1], a.steps, a.lr, a.seed, log,
                        a.weights, a.val, int8_inputs=a.int8_inputs, decodable_iters=a.decodable,
                        select_points=a.select, select_frames=a.select_frames, floor_points=a.select_floor,
                        floor_frames=a.floor_frames, max_scale=a.max_scale)
    wall = time.time() - t0
    ms = [h["ms"] for h in hist[1:]] or [hist[0]["ms"]]
    meta = {"short": a.short, "rate": a.rate, "constellation": a.const, "es": a.es, "batch": a.batch,
            "steps": a.steps, "lr": a.lr, "seed": a.seed, "weights": a.weights,
            "validation": model.validation, "int8_inputs": a.int8_inputs, "decodable_iters": a.decodable,
            "selection": getattr(model, "selection", None),
            "loss_first": hist[0]["loss"], "loss_last": float(np.mean([h["loss"] for h in hist[-10:]])),
            "train_ms_per_step": float(np.median(ms)), "train_frames_per_s": a.batch / (float(np.median(ms)) * 1e-3),
            "train_wall_s": wall}
    meta["ranks"] = world
    table = export(model, meta)
    out = a.out or table_path(a.short, a.rate, a.const, a.iters)
    if rank == 0:
        os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
        with open(out, "w") as f:
            json.dump(table, f, indent=1)
    log(json.dumps({k: v for k, v in meta.items()}))
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
