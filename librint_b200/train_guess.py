"""Train the learned initial guess on densities the GPU SCF generates.

    python -m librint_b200.train_guess --train 2000 --test 200 --flakes 60 \
        --test-flakes 8 --gen-conv 1e-6 --gen-mixed --tau-prim 1e-15 \
        --out librint_b200/data/guess_ch.npz --summary summary.json

Data: seeded C6H6-like rings (``synthetic.benzene_like``: bonds +-0.05 A,
angles +-3 deg, the seed-3 per-element C 3s2p1d / H 2s1p basis with K =
1..6, 120 cartesian AOs), geometry seeds 10000 + i; optionally (``--flakes``)
small C/H flakes of the same lattice construction as the 660-AO cluster
(``synthetic.flake_like``, seeds 20000 + i), so that the network also sees
interior carbons.  Each density comes from this library's RHF
(core-Hamiltonian guess, DIIS, density change <= --gen-conv; with
--gen-mixed the mixed-precision schedule, which ends with FP64 builds).
After the first ``--bootstrap`` ring geometries a provisional network is
trained and used as the starting density for the rest, which only shortens
data generation (the converged densities do not depend on the start).  The
final network is trained on the GPU with this library's MLP kernels, then
judged on held-out geometries by FP64 SCF to --conv: energies against the
core-Hamiltonian start, iterations and wall time.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import synthetic
from .guess import LearnedGuess, PairModel, lowdin
from .scf import MolContext

SCF_OPTS = dict(guess=1, diis=8, tau=1e-12, max_iter=100)
# extra options of the SCFs that generate the training densities (--gen-mixed,
# --tau-prim); the held-out evaluation runs SCF_OPTS plus --tau-prim
GEN_OPTS: dict = {}


def geometry(i: int, family: str = "rings"):
    if family == "rings":
        return synthetic.benzene_like(seed=10000 + i)
    if family == "flakes":
        return synthetic.flake_like(20000 + i)
    raise ValueError(family)


def run_scf(m, conv, guess=None):
    """Converged density and its Loewdin transform S^(1/2) P S^(1/2).  A
    start from ``guess`` that does not converge is redone from the
    core-Hamiltonian start (the data must not depend on the start)."""
    ctx = MolContext(m)
    try:
        S = ctx.int1e(0)
        r = None
        if guess is not None:
            r, P = ctx.scf(conv=conv, P0=guess.predict(m, S=S), return_density=True, check=False,
                           **dict(SCF_OPTS, **GEN_OPTS))
        if r is None or not r.converged:
            r, P = ctx.scf(conv=conv, return_density=True, check=False,
                           **dict(SCF_OPTS, max_iter=300, **GEN_OPTS))
    finally:
        ctx.close()
    if not r.converged:          # no usable target (e.g. a near-degenerate flake)
        return r, None
    Sh, _ = lowdin(S)
    return r, Sh @ P @ Sh


def generate(ids, conv, guess=None, log=print):
    """ids: list of (family, index); returns the ids that converged, their
    Loewdin densities and (iterations, ms, E) per geometry."""
    kept, dens, stats = [], [], []
    for n, (fam, i) in enumerate(ids):
        m = geometry(i, fam)
        # the provisional network has seen rings only
        r, P = run_scf(m, conv, guess if fam == "rings" else None)
        if P is None:
            if log:
                log(f"  {fam} {i}: SCF did not converge from the core-Hamiltonian start; skipped")
            continue
        kept.append((fam, i))
        dens.append(P)
        stats.append((r.iterations, r.wall_ms, r.energy))
        if log and (n % 100 == 0):
            log(f"  scf {n}/{len(ids)} ({fam} {i}, {m.nao(0)} AOs): {r.iterations} it, "
                f"{r.wall_ms:.0f} ms, E={r.energy:.10f}")
    return kept, dens, stats


def fit(model, ids, dens, hidden, epochs, batch, lr, seed, log=print):
    g = LearnedGuess(model, hidden=hidden, seed=seed)
    X, Y, M, T = g.dataset([geometry(i, f) for f, i in ids], dens)
    g.fit_normalisation(X, Y, M, T)
    t = time.perf_counter()
    hist = g.train(X, Y, M, T, epochs=epochs, batch=batch, lr=lr, seed=seed, log=log)
    return g, hist, time.perf_counter() - t, len(X)


def evaluate_one(g, m, conv, scf_opts=None):
    """SCF from the core-Hamiltonian start and from the learned start."""
    opts = dict(SCF_OPTS, **(scf_opts or {}))
    ctx = MolContext(m)
    try:
        S = ctx.int1e(0)
        t0 = time.perf_counter()
        P0 = g.predict(m, S=S)
        t_pred = (time.perf_counter() - t0) * 1e3
        rb, Pb = ctx.scf(conv=conv, return_density=True, check=False, **opts)
        if not rb.converged:
            return None
        rl, _ = ctx.scf(conv=conv, P0=P0, return_density=True, check=False, **opts)
    finally:
        ctx.close()
    Sh, _ = lowdin(S)
    # guess error in the Loewdin metric, max |S^1/2 (P0 - P) S^1/2|
    return dict(nao=m.nao(0), e_core=rb.energy, e_learned=rl.energy,
                learned_converged=bool(rl.converged),
                it_core=rb.iterations, it_learned=rl.iterations,
                ms_core=rb.wall_ms, ms_learned=rl.wall_ms + t_pred, ms_predict=t_pred,
                guess_err=float(np.abs(Sh @ (P0 - Pb) @ Sh).max()))


def summarise(rows):
    de = np.array([abs(r["e_core"] - r["e_learned"]) for r in rows if r["learned_converged"]])
    mean = lambda k: float(np.mean([r[k] for r in rows]))  # noqa: E731
    return dict(n=len(rows), learned_not_converged=sum(not r["learned_converged"] for r in rows),
                max_abs_de=float(de.max()) if de.size else None, it_core=mean("it_core"),
                it_learned=mean("it_learned"), ms_core=mean("ms_core"),
                ms_learned=mean("ms_learned"), ms_predict=mean("ms_predict"),
                guess_err=mean("guess_err"))


def evaluate(g, ids, conv, log=print):
    rows = []
    for fam, i in ids:
        r = evaluate_one(g, geometry(i, fam), conv)
        if r is None:      # no converged reference for this geometry
            continue
        r.update(family=fam, index=i)
        rows.append(r)
    out = {}
    for fam in sorted(set(f for f, _ in ids)):
        out[fam] = summarise([r for r in rows if r["family"] == fam])
        if log:
            s = out[fam]
            log(f"held-out {fam} {s['n']}: iterations {s['it_core']:.2f} -> {s['it_learned']:.2f}, "
                f"wall {s['ms_core']:.1f} -> {s['ms_learned']:.1f} ms, max |dE| {s['max_abs_de']:.2e}")
    return out, rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--train", type=int, default=2000, help="ring geometries for training")
    ap.add_argument("--test", type=int, default=200, help="held-out ring geometries")
    ap.add_argument("--flakes", type=int, default=0, help="flake geometries for training")
    ap.add_argument("--test-flakes", type=int, default=0, help="held-out flake geometries")
    ap.add_argument("--bootstrap", type=int, default=200)
    ap.add_argument("--conv", type=float, default=1e-8,
                    help="density convergence of the held-out evaluation SCFs")
    ap.add_argument("--gen-conv", type=float, default=None,
                    help="density convergence of the training SCFs (default: --conv)")
    ap.add_argument("--gen-mixed", action="store_true",
                    help="training SCFs with the mixed-precision incremental schedule")
    ap.add_argument("--tau-prim", type=float, default=0.0,
                    help="primitive-quartet screening of every SCF (0: off)")
    ap.add_argument("--hidden", type=int, nargs="+", default=[256, 256, 256])
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "data", "guess_ch.npz"))
    ap.add_argument("--summary", default=None)
    ap.add_argument("--densities", default=None, help="cache file for the training densities")
    ap.add_argument("--evaluate-only", action="store_true",
                    help="load the network at --out and only run the held-out evaluation")
    a = ap.parse_args(argv)

    gen_conv = a.gen_conv if a.gen_conv else a.conv
    if a.gen_mixed:
        GEN_OPTS.update(mixed=1, tau_fp32=1e-11)
    if a.tau_prim > 0:
        GEN_OPTS["tau_prim"] = a.tau_prim
        SCF_OPTS["tau_prim"] = a.tau_prim
    model = PairModel.from_molecule(geometry(0))
    if a.evaluate_only:
        from .guess import LearnedGuess
        test_ids = [("rings", i) for i in range(a.train, a.train + a.test)] + \
                   [("flakes", i) for i in range(a.flakes, a.flakes + a.test_flakes)]
        ev, rows = evaluate(LearnedGuess.load(a.out), test_ids, a.conv)
        summary = dict(network=os.path.basename(a.out), test=a.test, test_flakes=a.test_flakes,
                       first_test_ring=a.train, first_test_flake=a.flakes, conv=a.conv,
                       scf_options=SCF_OPTS, heldout=ev, heldout_rows=rows[:40])
        if a.summary:
            with open(a.summary, "w") as fh:
                json.dump(summary, fh, indent=1)
        print(json.dumps({k: v for k, v in summary.items() if k != "heldout_rows"}))
        return
    train_ids = [("rings", i) for i in range(a.train)] + [("flakes", i) for i in range(a.flakes)]
    test_ids = [("rings", i) for i in range(a.train, a.train + a.test)] + \
               [("flakes", i) for i in range(a.flakes, a.flakes + a.test_flakes)]
    t0 = time.perf_counter()
    if a.densities and os.path.exists(a.densities):
        f = np.load(a.densities, allow_pickle=True)
        train_ids = [(str(fam), int(i)) for fam, i in f["ids"]]
        dens = list(f["Pt"])
        stats = [tuple(v) for v in f["stats"]]
        print(f"loaded {len(dens)} densities from {a.densities}")
    else:
        nb = min(a.bootstrap, a.train)
        print(f"generating {nb} densities from the core-Hamiltonian start")
        kept, dens, stats = generate(train_ids[:nb], gen_conv)
        if nb < len(train_ids):
            g0 = fit(model, kept, dens, a.hidden, max(40, a.epochs // 5),
                     a.batch, a.lr, a.seed, log=None)[0] if kept else None
            print(f"generating {len(train_ids) - nb} more from the provisional network")
            k2, d2, s2 = generate(train_ids[nb:], gen_conv, guess=g0)
            kept += k2
            dens += d2
            stats += s2
        print(f"{len(kept)} of {len(train_ids)} training geometries converged")
        train_ids = kept
        if a.densities:
            arr = np.empty(len(dens), dtype=object)
            arr[:] = dens
            ids = np.empty(len(train_ids), dtype=object)
            ids[:] = train_ids
            np.savez_compressed(a.densities, Pt=arr, stats=np.array(stats), ids=ids)
    t_gen = time.perf_counter() - t0
    g, hist, t_train, nsamp = fit(model, train_ids, dens, a.hidden, a.epochs, a.batch, a.lr, a.seed)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    g.save(a.out)
    ev, rows = evaluate(g, test_ids, a.conv)
    st = np.array(stats)
    summary = dict(train=a.train, flakes=a.flakes, test=a.test, test_flakes=a.test_flakes,
                   train_converged=len(train_ids),
                   samples=nsamp, hidden=a.hidden, epochs=a.epochs, batch=a.batch, lr=a.lr,
                   conv=a.conv, gen_conv=gen_conv, scf_options=SCF_OPTS, gen_options=GEN_OPTS,
                   gen_seconds=t_gen,
                   gen_iterations_mean=float(st[:, 0].mean()), gen_ms_mean=float(st[:, 1].mean()),
                   train_seconds=t_train, loss_first=hist[0], loss_last=hist[-1],
                   heldout=ev, heldout_rows=rows[:40])
    if a.summary:
        with open(a.summary, "w") as fh:
            json.dump(summary, fh, indent=1)
    print(json.dumps({k: v for k, v in summary.items() if k != "heldout_rows"}))


if __name__ == "__main__":
    main()
