"""The learned-correction workloads, end to end.

Training (fine 256^3 vs coarse 128^3): pairs generated by the solver from
seeded KH layers (shear in [0.2, 0.8], density ratio in [1, 4]) and smooth
8-mode Fourier states; a 4-layer, 32-channel 3x3x3 CNN with GELU predicting
face fluxes (the correction is their divergence), trained by the library's
tensor-core kernels with Adam, batch 8 crops of 64^3.

Evaluation (coarse 256^3 corrected every step vs fine 512^3 plain): held-out
KH (shear 0.5, density ratio 2) and Fourier states, to the time the fine
grid reaches in 400 steps.  Reported: relative L1 density error of the
corrected and of the plain 256^3 solve against the coarsened 512^3 solve,
the fallback rate, and times to solution.

    python -m deepgreen.learned_workload --out results.json [--small]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import learned
from .net import Net


def rel_l1_density(coarse_ctx, truth_ctx):
    a = np.asarray(coarse_ctx.get_conserved()[0], np.float64)[2:-2, 2:-2, 2:-2]
    b = np.asarray(truth_ctx.get_conserved()[0], np.float64)[2:-2, 2:-2, 2:-2]
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def training(n_coarse, trajectories, pairs_per_traj, spacing, warmup_max, steps, batch, crop, lr, seed, log=print,
             balance=True):
    t0 = time.time()
    ps = learned.make_pairs(n_coarse, trajectories, pairs_per_traj, spacing, warmup_max, seed, log=log)
    t_pairs = time.time() - t0
    norm = learned.fit_norm(ps, samples=16, crop=min(48, n_coarse), seed=seed)
    net = Net(learned.INPUTS, learned.OUTPUTS, seed=seed, out_scale=0.1)
    t1 = time.time()
    hist = learned.train(net, ps, norm, steps, batch=batch, crop=crop, lr=lr, seed=seed, log=log, balance=balance)
    t_train = time.time() - t1
    return net, norm, ps, {"pairs": ps.count, "pair_seconds": t_pairs, "train_seconds": t_train,
                           "loss_first": float(np.mean(hist[:20])), "loss_last": float(np.mean(hist[-20:])),
                           "loss_history": [float(v) for v in hist[:: max(1, len(hist) // 100)]]}


def validation_loss(net, ps, norm, batches=8, batch=8, crop=64, seed=123):
    """Mean loss of the trained network, and of the zero correction, on
    crops of a pair set (the gain over the method without correction)."""
    b = learned.Batcher(ps, batch, crop, seed)
    zero = Net(learned.INPUTS, learned.OUTPUTS, seed=0, out_scale=0.0)
    lt, lz = [], []
    for _ in range(batches):
        b.fill(norm)
        lt.append(net.forward_backward_flux(b.feat, b.tgt))
        lz.append(zero.forward_backward_flux(b.feat, b.tgt))
    return float(np.mean(lt)), float(np.mean(lz))


def evaluate_case(net, norm, kind, seed, n_coarse, fine_steps, log=print, **kw):
    import torch
    n_fine = 2 * n_coarse
    prim, meta = learned.initial_state(kind, n_fine, seed, **kw)
    fine = learned.grid(n_fine)
    fine.set_primitives(prim)
    del prim
    plain = learned.grid(n_coarse)
    corr = learned.grid(n_coarse)
    warm = learned.grid(n_coarse)
    for g in (plain, corr, warm):
        learned.coarsen(fine, g)
    # two corrected steps outside the clocks: the network's workspace and the
    # kernels' launch attributes are set up once per shape
    cw = learned.Corrector(warm, net, norm)
    cw.step(2)
    warm.synchronize()
    cw.close()
    warm.close()
    # plain fine solve: the reference solution (reads dt every step, as the reference loop)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t_end = 0.0
    for _ in range(fine_steps):
        t_end += fine.next_dt()
        fine.enqueue_steps(1)
    fine.synchronize()
    t_fine = time.perf_counter() - t0
    truth = learned.grid(n_coarse)
    learned.coarsen(fine, truth)
    fine.close()
    steps_plain, t_plain = learned.solve_to_time(plain, t_end)
    cor = learned.Corrector(corr, net, norm)
    steps_corr, t_corr = learned.solve_to_time(corr, t_end, corrector=cor)
    st = cor.stats()
    res = dict(meta)
    res.update({
        "n_coarse": n_coarse, "n_fine": n_fine, "fine_steps": fine_steps, "t_end": t_end,
        "fine_seconds": t_fine, "plain_coarse_seconds": t_plain, "learned_coarse_seconds": t_corr,
        "plain_coarse_steps": steps_plain, "learned_coarse_steps": steps_corr,
        "l1_density_plain_coarse": rel_l1_density(plain, truth),
        "l1_density_learned_coarse": rel_l1_density(corr, truth),
        "fallback_step_rate": st["fallback_steps"] / max(1, st["steps"]),
        "masked_cell_rate": st["masked_cells"] / max(1, st["cells"]),
        "max_drift": st["max_drift"],
        "time_ratio_fine_over_learned": t_fine / t_corr,
    })
    log(json.dumps(res))
    return res


def _density_l1_device(ctx, ref):
    """Relative L1 of the density of ctx against ref (same grid size),
    computed on the GPU from the conserved totals (equal cell volumes)."""
    import torch
    shape = tuple(ctx.n)
    a = torch.empty((5,) + shape, dtype=torch.float32, device="cuda")
    b = torch.empty_like(a)
    ctx.get_conserved_device([a[f].data_ptr() for f in range(5)])
    ref.get_conserved_device([b[f].data_ptr() for f in range(5)])
    ctx.synchronize()
    ref.synchronize()
    ai = a[0, 2:-2, 2:-2, 2:-2].double()
    bi = b[0, 2:-2, 2:-2, 2:-2].double()
    return float((ai - bi).abs().sum() / bi.abs().sum())


def resolution_norm(norm, n_train, n_eval, order=2):
    """The normalisation of a network trained on n_train^3 coarse grids, with
    its output scale moved to n_eval^3.  Per step the correction is the
    coarse step's truncation error, which for smooth flow shrinks like
    dt ds^2 ~ ds^3 (second order in space, dt ~ ds), while the network's
    dominant input, the change over the step, shrinks like dt ~ ds: a network
    that responds in proportion to its inputs over-corrects by
    (n_eval / n_train)^order with order = 2.  The output scale is multiplied
    by (n_train / n_eval)^order."""
    s = learned.Norm.from_dict(norm.to_dict())
    f = (n_train / n_eval) ** order
    for c in range(16):
        s.out_std[c] = s.out_std[c] * f
    return s


def evaluate_truth(net, norm, kind, seed, n_coarse, fine_steps, log=print, threshold=0.02, train_n=None, **kw):
    """The learned-vs-plain comparison against a plain solve at FOUR times the
    coarse resolution (1024^3 for the 256^3 workload), which serves as the
    truth for every method, including the 512^3 plain solve.

    Every grid starts from the 2x2x2 sums of the next finer one, down from the
    truth's initial state (1024 -> 512 -> 256 -> 128 -> 64).  The 512^3 plain
    solve takes `fine_steps` CFL steps and defines the end time; every other
    method solves to that time (solve_to_time).  Each solution is compared
    with the truth summed to its own resolution, and the 512^3 solution also
    at the 256^3 resolution, where the workload's criterion compares it with
    the corrected 256^3 solve (error within 1.5x).  Time to L1 <= threshold:
    the fastest method whose density error is within the threshold.  With
    train_n (the coarse resolution of the training pairs) the corrected
    solves at other resolutions run twice: with the trained normalisation
    ("learned_n") and with its output scale moved to n (resolution_norm,
    "learned_rs_n")."""
    import torch
    n1, n2, n4 = n_coarse, 2 * n_coarse, 4 * n_coarse
    cons, meta = learned.device_initial_conserved(kind, n4, seed, **kw)
    truth = learned.grid(n4)
    truth.set_conserved_device([c.data_ptr() for c in cons])
    del cons
    torch.cuda.empty_cache()
    sizes = [n2, n1, n1 // 2, n1 // 4]
    plain, prev = {}, truth
    for n in sizes:
        plain[n] = learned.grid(n)
        learned.coarsen(prev, plain[n])
        prev = plain[n]
    # corrected solves: (name, resolution, normalisation)
    variants = [(f"learned_{n}", n, norm) for n in (n1, n1 // 2)]
    if train_n:
        variants += [(f"learned_rs_{n}", n, resolution_norm(norm, train_n, n)) for n in (n1, n1 // 2) if n != train_n]
    corr = {}
    for name, n, _ in variants:
        corr[name] = learned.grid(n)
        learned.coarsen(plain[2 * n], corr[name])
    # corrected steps on scratch grids outside the clocks: the network's
    # workspace and launch attributes are set up once per shape
    for n in (n1, n1 // 2):
        w = learned.grid(n)
        learned.coarsen(plain[2 * n], w)
        cw = learned.Corrector(w, net, norm)
        cw.step(2)
        w.synchronize()
        cw.close()
        w.close()
    torch.cuda.synchronize()
    times, steps = {}, {}
    # the 512^3 plain solve defines the end time (reads dt every step, as the
    # reference's time loop does)
    t0 = time.perf_counter()
    t_end = 0.0
    for _ in range(fine_steps):
        t_end += plain[n2].next_dt()
        plain[n2].enqueue_steps(1)
    plain[n2].synchronize()
    times[f"plain_{n2}"], steps[f"plain_{n2}"] = time.perf_counter() - t0, fine_steps
    steps[f"plain_{n4}"], times[f"plain_{n4}"] = learned.solve_to_time(truth, t_end)
    for n in sizes[1:]:
        steps[f"plain_{n}"], times[f"plain_{n}"] = learned.solve_to_time(plain[n], t_end)
    stats = {}
    for name, n, nm in variants:
        cor = learned.Corrector(corr[name], net, nm)
        steps[name], times[name] = learned.solve_to_time(corr[name], t_end, corrector=cor)
        st = cor.stats()
        stats[name] = {"fallback_step_rate": st["fallback_steps"] / max(1, st["steps"]),
                       "masked_cell_rate": st["masked_cells"] / max(1, st["cells"]),
                       "max_drift": st["max_drift"]}
        cor.close()
    # the truth summed to every resolution
    ref, prev = {}, truth
    for n in sizes:
        ref[n] = learned.grid(n)
        learned.coarsen(prev, ref[n])
        prev = ref[n]
    truth.close()
    err = {f"plain_{n}": _density_l1_device(plain[n], ref[n]) for n in sizes}
    for name, n, _ in variants:
        err[name] = _density_l1_device(corr[name], ref[n])
    c512 = learned.grid(n1)
    learned.coarsen(plain[n2], c512)
    err_512_at_256 = _density_l1_device(c512, ref[n1])
    meeting = {k: times[k] for k in err if err[k] <= threshold}
    best = min(meeting, key=meeting.get) if meeting else None
    res = dict(meta)
    res.update({
        "truth": f"plain {n4}^3 FP32 solve", "n_coarse": n1, "fine_steps": fine_steps, "t_end": t_end,
        "l1_density": err, "l1_density_plain_512_at_256": err_512_at_256,
        "seconds": times, "steps": steps, "corrector": stats,
        "criterion_learned_within_1p5x_of_plain_512": {
            "at_256": err[f"learned_{n1}"] <= 1.5 * err_512_at_256,
            "own_resolution": err[f"learned_{n1}"] <= 1.5 * err[f"plain_{n2}"]},
        "time_ratio_plain_512_over_learned_256": times[f"plain_{n2}"] / times[f"learned_{n1}"],
        "time_to_l1": {"threshold": threshold, "meeting": meeting, "fastest": best,
                       "fastest_seconds": meeting.get(best) if best else None},
        # every corrected solve at the workload's resolution against the criterion
        "by_method_at_256": {name: {"l1_density": err[name],
                                    "within_1p5x_of_plain_512_at_256": err[name] <= 1.5 * err_512_at_256,
                                    "time_ratio_plain_512_over_it": times[f"plain_{n2}"] / times[name]}
                             for name, n, _ in variants if n == n1},
    })
    for g in list(plain.values()) + list(corr.values()) + list(ref.values()) + [c512]:
        g.close()
    log(json.dumps(res))
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="learned_results.json")
    ap.add_argument("--small", action="store_true", help="reduced sizes for a quick end-to-end check")
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--save", default=None, help="write the trained network here (JSON)")
    ap.add_argument("--load", default=None, help="skip training, load a network")
    ap.add_argument("--no-eval", action="store_true")
    ap.add_argument("--no-balance", dest="balance", action="store_false",
                    help="plain MSE instead of weighing every training crop by its inverse target power")
    ap.add_argument("--truth", action="store_true",
                    help="evaluate against a plain solve at 4x the coarse resolution (1024^3 for the full workload)")
    ap.add_argument("--eval-train-res", action="store_true",
                    help="also evaluate at the training resolution (coarse = the pairs' coarse grid)")
    args = ap.parse_args(argv)
    if args.small:
        cfg = dict(n_coarse=32, traj=[("kh", 11), ("fourier", 12)], ppt=4, spacing=4, warm=8, steps=args.steps or 20,
                   batch=4, crop=16, eval_n=32, fine_steps=40)
    else:
        traj = [("kh", 100 + i) for i in range(8)] + [("fourier", 200 + i) for i in range(8)]
        cfg = dict(n_coarse=128, traj=traj, ppt=8, spacing=20, warm=40, steps=args.steps or 2000, batch=8, crop=64,
                   eval_n=256, fine_steps=400)
    out = {"config": {k: v for k, v in cfg.items() if k != "traj"} | {"balance": args.balance},
           "trajectories": cfg["traj"]}
    if args.load:
        net, norm, _ = learned.load(args.load)
    else:
        net, norm, ps, tr = training(cfg["n_coarse"], cfg["traj"], cfg["ppt"], cfg["spacing"], cfg["warm"],
                                     cfg["steps"], cfg["batch"], cfg["crop"], 1e-3, 0, balance=args.balance)
        out["training"] = tr
        lt, lz = validation_loss(net, ps, norm, batch=cfg["batch"], crop=cfg["crop"])
        out["training"]["crop_loss_trained"] = lt
        out["training"]["crop_loss_zero_correction"] = lz
        if args.save:
            learned.save(args.save, net, norm, {"training": {k: v for k, v in tr.items() if k != "loss_history"}})
        del ps
    if not args.no_eval and args.truth:
        out["evaluation_truth"] = [
            evaluate_truth(net, norm, "kh", 9001, cfg["eval_n"], cfg["fine_steps"], train_n=cfg["n_coarse"],
                           shear=0.5, ratio=2.0),
            evaluate_truth(net, norm, "fourier", 9002, cfg["eval_n"], cfg["fine_steps"], train_n=cfg["n_coarse"]),
        ]
    if not args.no_eval:
        out["evaluation"] = [
            evaluate_case(net, norm, "kh", 9001, cfg["eval_n"], cfg["fine_steps"], shear=0.5, ratio=2.0),
            evaluate_case(net, norm, "fourier", 9002, cfg["eval_n"], cfg["fine_steps"]),
        ]
        if args.eval_train_res:
            out["evaluation_training_resolution"] = [
                evaluate_case(net, norm, "kh", 9001, cfg["n_coarse"], cfg["fine_steps"] // 2, shear=0.5, ratio=2.0),
                evaluate_case(net, norm, "fourier", 9002, cfg["n_coarse"], cfg["fine_steps"] // 2),
            ]
    with open(args.out, "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps({k: v for k, v in out.items() if k != "training"} | {
        "training": {k: v for k, v in out.get("training", {}).items() if k != "loss_history"}}))


if __name__ == "__main__":
    main()
