"""Benchmark: Rys ERI sweep, shell quartets per second (FP64).

Workload: 21 angular classes (ss|ss) .. (dd|dd), ``--nq`` independent shell
quartets per class (default 2^20), every shell with its own centre uniform in
a 10 A cube, 1..6 primitives, exponents log-uniform in [0.05, 5000],
spherical output (seeded synthetic data of that distribution; no dataset).
One step = one pass of the batched ERI path over all 21 classes with inputs
resident in HBM.  Outputs (18 GB per step at 2^20) exceed the 126 MB L2, so
no explicit L2 flush is needed between steps.

Arms:
  default          the CUDA library (librint_b200), one process per GPU;
                   with torchrun each rank runs its own shard (weak scaling).
                   On one GPU the line also carries the RHF leg on the
                   60-atom C/H cluster (``rhf``: plain FP64 vs mixed precision
                   and the learned start) and the learned guess on held-out
                   C6H6-like rings (``guess``: SCF iterations and wall time
                   against the core-Hamiltonian start).
  --impl reference the reference algorithm on the host cores (the CPU
                   restatement in oracle/, since the Rust reference cannot be
                   built here), rank 0 only, on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from librint_b200 import shard, synthetic  # noqa: E402

CLASSES = synthetic.canonical_classes(2)
METRIC = "ERI shell quartets/s (FP64 Rys sweep, (ss|ss)..(dd|dd), K=1..6, spherical)"
UNIT = "quartets/s"
CPU_STEP_S = 3.0        # seconds of oracle work per CPU pass (bounded sample)


# ------------------------------------------------------------ workload
def _gen(args):
    cls, nq, seed = args
    m, shls = synthetic.eri_sweep(cls, nq, seed=seed)
    return cls, m.atm, m.bas, m.env, shls


def generate(nq, seed, procs):
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(procs, len(CLASSES))) as pool:
        return pool.map(_gen, [(c, nq, seed) for c in CLASSES])


def ncart(l):
    return (l + 1) * (l + 2) // 2


def nsph(l):
    return 2 * l + 1


def class_flops_bytes(cls, bas, shls):
    """Fixed algorithmic FLOP / byte convention per shell quartet.

    F = P [50 + n_r (64 + 15 (nmax+1)(mmax+1) + 6 H + 3 nf)] + C2S with
    P = Ki Kj Kk Kl (unscreened), n_r = L/2 + 1, nmax = li+lj, mmax = lk+ll,
    nf = prod ncart, H = sum_{i=1..li}(nmax-i+1)(mmax+1) + (lj+1)(li+1)
    sum_{k=1..lk}(mmax-k+1), C2S = 2 [nsi nci ncj nck ncl + nsj ncj nsi nck ncl
    + nsk nck nsi nsj ncl + nsl ncl nsi nsj nsk];
    B = 8 prod ns written + 8 sum_shells (3 + 2K) read.
    """
    li, lj, lk, ll = cls
    nmax, mmax = li + lj, lk + ll
    nr = (nmax + mmax) // 2 + 1
    nf = ncart(li) * ncart(lj) * ncart(lk) * ncart(ll)
    H = sum((nmax - i + 1) * (mmax + 1) for i in range(1, li + 1)) + \
        (lj + 1) * (li + 1) * sum(mmax - k + 1 for k in range(1, lk + 1))
    nc = [ncart(l) for l in cls]
    ns = [nsph(l) for l in cls]
    c2s = 2 * (ns[0] * nc[0] * nc[1] * nc[2] * nc[3] + ns[1] * nc[1] * ns[0] * nc[2] * nc[3] +
               ns[2] * nc[2] * ns[0] * ns[1] * nc[3] + ns[3] * nc[3] * ns[0] * ns[1] * ns[2])
    per_prim = 50 + nr * (64 + 15 * (nmax + 1) * (mmax + 1) + 6 * H + 3 * nf)
    k = bas.reshape(-1, 8)[:, 2].astype(np.float64)[shls]          # (nq, 4)
    P = k.prod(axis=1)
    flops = float((P * per_prim + c2s).sum())
    nbytes = float(8 * np.prod(ns) * shls.shape[0] + 8 * (3 + 2 * k).sum())
    return flops, nbytes


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per shell quartet
# of the output kernels, from one ncu capture of 65,536 quartets of the sweep
# class (K = 1..6, spherical output); traffic grows with the quartets processed
# (output block plus pair data), so a launch's traffic is this times its
# quartet count.
NCU_TRAFFIC_PER_QUARTET = {(2, 2, 2, 2): (81.393408e6 + 269.814016e6) / 65536}


def class_id(c):
    """Kernel class id of (li, lj, lk, ll): P(P+1)/2 + Q over pair indices."""
    P = c[0] * (c[0] + 1) // 2 + c[1]
    Q = c[2] * (c[2] + 1) // 2 + c[3]
    return P * (P + 1) // 2 + Q


def _pair_cce(bas, env, atm, si, sj, kmax=6):
    """libcint screening keys of all primitive pairs of shells si, sj (arrays
    of shell indices): cce = mu R^2 - log_rr - log|c_i| - log|c_j| (reference
    src/optimizer.rs:732-808); (n, kmax*kmax), +inf for absent primitives."""
    b = bas.reshape(-1, 8)
    a6 = atm.reshape(-1, 6)
    bi, bj = b[si], b[sj]
    ri = np.stack([env[a6[bi[:, 0], 1] + x] for x in range(3)], 1)
    rj = np.stack([env[a6[bj[:, 0], 1] + x] for x in range(3)], 1)
    rr = ((ri - rj) ** 2).sum(1)
    ki, kj = bi[:, 2], bj[:, 2]
    cols = np.arange(kmax)
    mi = cols[None, :] < ki[:, None]
    mj = cols[None, :] < kj[:, None]
    ei = np.where(mi, env[np.minimum(bi[:, 5:6] + cols, env.size - 1)], 1.0)
    ej = np.where(mj, env[np.minimum(bj[:, 5:6] + cols, env.size - 1)], 1.0)
    ci = np.where(mi, env[np.minimum(bi[:, 6:7] + cols, env.size - 1)], 1.0)
    cj = np.where(mj, env[np.minimum(bj[:, 6:7] + cols, env.size - 1)], 1.0)
    amin_i = env[bi[:, 5] + ki - 1]
    amin_j = env[bj[:, 5] + kj - 1]
    log_rr = 1.7 - 1.5 * np.log(amin_i + amin_j)
    lij = bi[:, 1] + bj[:, 1]
    log_rr = log_rr + np.where(lij > 0, lij * np.log(np.sqrt(rr) + 1.0), 0.0)
    mu = ei[:, :, None] * ej[:, None, :] / (ei[:, :, None] + ej[:, None, :])
    cce = (mu * rr[:, None, None] - log_rr[:, None, None] - np.log(np.abs(ci))[:, :, None]
           - np.log(np.abs(cj))[:, None, :])
    ok = mi[:, :, None] & mj[:, None, :]
    return np.where(ok, cce, np.inf).reshape(len(si), -1)


def screened_prim_quartets(atm, bas, env, shls, expcutoff=60.0, chunk=32768):
    """Primitive quartets that pass the reference's screening
    (src/cint2e.rs:367-393: ket cce <= cutoff and bra + ket <= cutoff),
    summed over all quartets of one sweep class."""
    total = 0
    for a in range(0, shls.shape[0], chunk):
        sh = shls[a:a + chunk]
        cb = _pair_cce(bas, env, atm, sh[:, 0], sh[:, 1])
        ck = _pair_cce(bas, env, atm, sh[:, 2], sh[:, 3])
        ck = np.where(ck <= expcutoff, ck, np.inf)
        total += int(np.count_nonzero(cb[:, :, None] + ck[:, None, :] <= expcutoff))
    return total


# Upper edges of the K^4 bins (P = Ki Kj Kk Kl primitive quartets per shell
# quartet, K = 1..6) of the screening profile.
K4_BINS = (1, 16, 81, 256, 625, 1296)


def screening_profile(atm, bas, env, shls, expcutoff=60.0, chunk=32768):
    """Per K^4 bin: shell quartets, primitive quartets, and primitive
    quartets that pass the reference's screening (the test of
    screened_prim_quartets), as rows of a (len(K4_BINS), 3) array."""
    b = bas.reshape(-1, 8)
    out = np.zeros((len(K4_BINS), 3))
    for a in range(0, shls.shape[0], chunk):
        sh = shls[a:a + chunk]
        cb = _pair_cce(bas, env, atm, sh[:, 0], sh[:, 1])
        ck = _pair_cce(bas, env, atm, sh[:, 2], sh[:, 3])
        ck = np.where(ck <= expcutoff, ck, np.inf)
        ok = (cb[:, :, None] + ck[:, None, :] <= expcutoff).reshape(sh.shape[0], -1)
        passed = np.count_nonzero(ok, axis=1)
        P = b[sh, 2].astype(np.int64).prod(axis=1)
        k = np.searchsorted(K4_BINS, P)
        np.add.at(out[:, 0], k, 1)
        np.add.at(out[:, 1], k, P)
        np.add.at(out[:, 2], k, passed)
    return out


def screening_summary(data, sample=65536):
    """Fraction of primitive quartets that pass the reference's screening,
    per class and per K^4 bin over all classes, on the first `sample`
    quartets of every class of the sweep."""
    tot = np.zeros((len(K4_BINS), 3))
    per_class = {}
    for cls, atm, bas, env, shls in data:
        prof = screening_profile(atm, bas, env, shls[:sample])
        tot += prof
        per_class["%d%d%d%d" % tuple(cls)] = round(float(prof[:, 2].sum() / prof[:, 1].sum()), 4)
    bins = [{"P_max": int(e), "quartets": int(r[0]), "prim_quartets": int(r[1]),
             "passed": int(r[2]), "fraction": round(float(r[2] / r[1]), 4) if r[1] else None}
            for e, r in zip(K4_BINS, tot)]
    return {"sample": f"first {sample} quartets of each class",
            "fraction_passed": round(float(tot[:, 2].sum() / tot[:, 1].sum()), 4),
            "classes": per_class, "k4_bins": bins}


def class_flops(cls, prim_quartets, nq):
    """class_flops_bytes' FLOP convention with a given primitive-quartet count."""
    li, lj, lk, ll = cls
    nmax, mmax = li + lj, lk + ll
    nr = (nmax + mmax) // 2 + 1
    nf = ncart(li) * ncart(lj) * ncart(lk) * ncart(ll)
    H = sum((nmax - i + 1) * (mmax + 1) for i in range(1, li + 1)) + \
        (lj + 1) * (li + 1) * sum(mmax - k + 1 for k in range(1, lk + 1))
    nc = [ncart(l) for l in cls]
    ns = [nsph(l) for l in cls]
    c2s = 2 * (ns[0] * nc[0] * nc[1] * nc[2] * nc[3] + ns[1] * nc[1] * ns[0] * nc[2] * nc[3] +
               ns[2] * nc[2] * ns[0] * ns[1] * nc[3] + ns[3] * nc[3] * ns[0] * ns[1] * ns[2])
    per_prim = 50 + nr * (64 + 15 * (nmax + 1) * (mmax + 1) + 6 * H + 3 * nf)
    return float(prim_quartets) * per_prim + float(c2s) * nq


# ------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-i", str(self.idx), "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def link_bandwidth(dev, nbytes=1 << 30, reps=3):
    """Pinned host <-> device copy bandwidth (GB/s per direction), measured
    with CUDA events on one stream: the ceiling of the end-to-end path."""
    import torch
    h = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    out = {}
    for name, fn in (("h2d_gbs", lambda: d.copy_(h, non_blocking=True)),
                     ("d2h_gbs", lambda: h.copy_(d, non_blocking=True))):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        out[name] = nbytes * reps / (a.elapsed_time(b) * 1e-3) / 1e9
    del h, d
    return out


# ------------------------------------------------------------ CPU arms
def _prefix_molecule(atm, bas, env, nshell):
    """The first nshell shells of a sweep (one atom per shell, env laid out
    shell after shell), so the host call does not carry the whole class."""
    from librint_b200.basis import Molecule
    b = bas.reshape(-1, 8)[:nshell]
    a = atm.reshape(-1, 6)[:nshell]
    end = int(max((b[:, 6] + b[:, 2]).max(), (a[:, 1] + 3).max()))
    return Molecule(np.ascontiguousarray(a.ravel()), np.ascontiguousarray(b.ravel()),
                    np.ascontiguousarray(env[:end]))


def cpu_sample(data, sample, threads):
    """Oracle on the first `sample` quartets of every class; (quartets/s, s)."""
    import oracle
    tot_q, tot_t = 0, 0.0
    for cls, atm, bas, env, shls in data:
        sh = np.ascontiguousarray(shls[:sample])
        m = _prefix_molecule(atm, bas, env, int(sh.max()) + 1)
        t0 = time.perf_counter()
        oracle.int2e_batch(m, sh, 1, nthreads=threads)
        tot_t += time.perf_counter() - t0
        tot_q += sh.shape[0]
    return tot_q / tot_t, tot_t


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def pick_sample(data, threads, budget_s=CPU_STEP_S):
    """Sample size per class so one oracle pass takes about budget_s (two
    probes: a small one, then one of about a tenth of the budget)."""
    nmax = data[0][4].shape[0]
    s = 64
    for frac in (None, 0.1):
        if frac is not None:
            s = max(64, min(int(s * frac), nmax))
        _, t = cpu_sample(data, s, threads)
        s = int(s * budget_s / max(t, 1e-4))
    return max(64, min(s, nmax))


def cpu_rate(data, threads, steps, warmup, sample=None):
    """The CPU restatement on the first ``sample`` quartets of every class
    (sized by pick_sample when None): ``warmup`` untimed passes, then
    ``steps`` timed passes.  The cpu_baseline leg and ``--impl reference``
    both measure through this function on the same generated workload, so
    their figures are the same measurement.  Returns (quartets/s, sample,
    seconds timed)."""
    s = sample or pick_sample(data, threads)
    for _ in range(warmup):
        cpu_sample(data, s, threads)
    tt = 0.0
    for _ in range(steps):
        tt += cpu_sample(data, s, threads)[1]
    return steps * len(data) * s / tt, s, tt


# ------------------------------------------------------------ end to end
def merged_layout(data):
    """Sizes and offsets of the sweep's classes placed back to back in one
    molecule: per class its first atom, shell and env entry and its first
    output element; totals last."""
    na = nb = ne = no = 0
    offs = []
    for cls, atm, bas, env, shls in data:
        b = bas.reshape(-1, 8)
        l = b[:, 1][shls]
        nout = int(((2 * l + 1).prod(axis=1)).sum())
        offs.append((na, nb, ne, no))
        na += atm.size // 6
        nb += b.shape[0]
        ne += env.size
        no += nout
    # the atm/bas/env pointers are int32; the kernels index bas and atm rows
    # with 32-bit products
    if ne >= 2 ** 31 or 8 * nb >= 2 ** 31 or 6 * na >= 2 ** 31:
        raise ValueError("sweep too large for one molecule (int32 pointers)")
    return offs, (na, nb, ne, no)


def fill_merged(data, offs, atm_all, bas_all, env_all, shls_all):
    """Writes the classes into the merged arrays (numpy views), shifting
    atom, shell and env pointers by each class's offsets."""
    A = atm_all.reshape(-1, 6)
    Bv = bas_all.reshape(-1, 8)
    S = shls_all.reshape(-1, 4)
    q = 0
    for (cls, atm, bas, env, shls), (oa, ob, oe, _) in zip(data, offs):
        a = atm.reshape(-1, 6)
        b = bas.reshape(-1, 8)
        A[oa:oa + a.shape[0]] = a
        A[oa:oa + a.shape[0], 1] += oe
        A[oa:oa + a.shape[0], 3] += oe
        Bv[ob:ob + b.shape[0]] = b
        Bv[ob:ob + b.shape[0], 0] += oa
        Bv[ob:ob + b.shape[0], 5] += oe
        Bv[ob:ob + b.shape[0], 6] += oe
        env_all[oe:oe + env.size] = env
        S[q:q + shls.shape[0]] = shls
        S[q:q + shls.shape[0]] += ob
        q += shls.shape[0]


def e2e_one_call(L, data, dev_data):
    """Step function of the end-to-end leg as one lrb_int2e_batch call over
    all classes (page-locked inputs and output); (step, h2d bytes, d2h
    bytes).  step.out is the output tensor."""
    import ctypes
    import torch
    from librint_b200 import _bindings as B
    offs, (na, nb, ne, no) = merged_layout(data)
    nq = sum(d[4].shape[0] for d in data)
    atm = torch.empty(6 * na, dtype=torch.int32, pin_memory=True)
    bas = torch.empty(8 * nb, dtype=torch.int32, pin_memory=True)
    env = torch.empty(ne, dtype=torch.float64, pin_memory=True)
    shl = torch.empty(4 * nq, dtype=torch.int32, pin_memory=True)
    out = torch.empty(no, dtype=torch.float64, pin_memory=True)
    fill_merged(data, offs, atm.numpy(), bas.numpy(), env.numpy(), shl.numpy())
    P_i, P_d = B.P_i, B.P_d

    def step():
        rc = L.lrb_int2e_batch(ctypes.cast(out.data_ptr(), P_d), 1,
                               ctypes.cast(shl.data_ptr(), P_i), nq,
                               ctypes.cast(atm.data_ptr(), P_i), na,
                               ctypes.cast(bas.data_ptr(), P_i), nb,
                               ctypes.cast(env.data_ptr(), P_d), ne)
        B.check(rc, "lrb_int2e_batch")
    step.out = out
    step.keep = (atm, bas, env, shl)
    h2d = 4 * (6 * na + 8 * nb + 4 * nq) + 8 * ne
    return step, h2d, 8 * no


def e2e_check_one_call(data, dev_data, out, n=4096):
    """The one-call output equals the device-resident leg's class outputs
    (the same kernels on the same quartets), bit for bit, on the first,
    middle and last n elements of every class."""
    import torch
    o = 0
    for t in dev_data:
        ref = t["out"]
        m = ref.numel()
        for a in (0, max(0, m // 2 - n // 2), max(0, m - n)):
            b = min(m, a + n)
            if not torch.equal(out[o + a:o + b], ref[a:b].cpu()):
                raise AssertionError("one-call output differs from the device-resident leg in "
                                     "class %s" % (t["cls"],))
        o += m
    if o != out.numel():
        raise AssertionError("one-call output length %d, classes %d" % (out.numel(), o))


def e2e_per_class(L, data, dev_data):
    """Step function of the end-to-end leg as one lrb_int2e_batch call per
    class (page-locked inputs and outputs); (step, h2d bytes, d2h bytes)."""
    import ctypes
    import torch
    from librint_b200 import _bindings as B
    host = []
    h2d = d2h = 0
    for (cls, atm, bas, env, shls), t in zip(data, dev_data):
        pin = lambda a: torch.from_numpy(a).pin_memory()  # noqa: E731
        out = torch.empty(t["out"].numel(), dtype=torch.float64, pin_memory=True)
        host.append((pin(atm), pin(bas), pin(env), pin(shls), out))
        h2d += atm.nbytes + bas.nbytes + env.nbytes + shls.nbytes
        d2h += out.numel() * 8
    P_i, P_d = B.P_i, B.P_d

    def step():
        for (a, b, e, s, o) in host:
            rc = L.lrb_int2e_batch(ctypes.cast(o.data_ptr(), P_d), 1,
                                   ctypes.cast(s.data_ptr(), P_i), s.numel() // 4,
                                   ctypes.cast(a.data_ptr(), P_i), a.numel() // 6,
                                   ctypes.cast(b.data_ptr(), P_i), b.numel() // 8,
                                   ctypes.cast(e.data_ptr(), P_d), e.numel())
            B.check(rc, "lrb_int2e_batch")
    return step, h2d, d2h


# ------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--nq", type=int, default=1 << 20, help="quartets per class per rank")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--rhf", type=int, default=1,
                    help="time RHF on the 60-atom C/H cluster (plain FP64 vs mixed / learned); "
                         "single-GPU runs only")
    ap.add_argument("--guess", default=os.path.join(ROOT, "librint_b200", "data", "guess_ch.npz"),
                    help="learned-guess network for the --rhf runs")
    ap.add_argument("--rhf-reference-run", action="store_true",
                    help="compute the RHF reference energy on the GPU (plain run continued to "
                         "1e-8) instead of reading the recorded one")
    ap.add_argument("--rhf-ablations", action="store_true",
                    help="also run the learned FP64 and learned fractional-occupation mixed RHF "
                         "legs (the mixed core-H leg runs first then)")
    ap.add_argument("--guess-rings", type=int, default=50,
                    help="held-out C6H6-like ring geometries on which the learned guess is "
                         "compared with the core-Hamiltonian start (0 skips)")
    ap.add_argument("--classes", default="",
                    help="comma list of classes to run, e.g. 2222,2221 (default: all 21)")
    args = ap.parse_args()
    global CLASSES
    if args.classes:
        CLASSES = [tuple(int(ch) for ch in c.strip()) for c in args.classes.split(",")]

    world, rank, local = shard.world_info()
    threads = host_threads()

    if args.impl == "reference":
        return run_reference(args, rank, world, threads)

    # inputs generated on the host before any CUDA call (spawn pool)
    data = generate(args.nq, shard.shard_seed(2, rank), procs=max(1, threads // max(world, 1)))

    import torch
    import torch.distributed as dist
    from librint_b200 import _bindings as B
    from librint_b200 import eri

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", world_size=world, rank=rank,
                                timeout=__import__("datetime").timedelta(seconds=120))
    L = B.lib()

    # device-resident inputs and outputs
    dev_data = []
    flops, nbytes = {}, {}
    for cls, atm, bas, env, shls in data:
        from librint_b200.basis import Molecule
        n = eri.batch_len(Molecule(atm, bas, env), shls, 1)
        t = dict(cls=cls, atm=torch.from_numpy(atm).to(dev), bas=torch.from_numpy(bas).to(dev),
                 env=torch.from_numpy(env).to(dev), shls=torch.from_numpy(shls).to(dev),
                 out=torch.empty(n, dtype=torch.float64, device=dev))
        dev_data.append(t)
        flops[cls], nbytes[cls] = class_flops_bytes(cls, bas, shls)
    stream = torch.cuda.current_stream()

    def step():
        for t in dev_data:
            eri.int2e_batch_device(t["out"], 1, t["shls"], t["atm"], t["bas"], t["env"], stream)

    fp64_peak = L.lrb_fp64_peak_probe(300)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    phys = vis.split(",")[local] if vis and vis.split(",")[local].strip().isdigit() else str(local)
    sampler = ClockSampler(phys)
    L.lrb_profile_read((__import__("ctypes").c_double * 64)(), 64)
    L.lrb_profile_enable(1)
    n0 = L.lrb_launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    L.lrb_profile_enable(0)
    launches = L.lrb_launch_count() - n0
    ms_arr = (__import__("ctypes").c_double * 64)()
    L.lrb_profile_read(ms_arr, 64)
    elapsed = shard.max_over_ranks(ev0.elapsed_time(ev1) / 1e3, dev)
    nq_total = world * len(CLASSES) * args.nq * args.steps
    value = nq_total / elapsed

    # dominant kernel: the class with the largest share of kernel time
    cls_ms = {cls: ms_arr[class_id(cls)] / args.steps for cls in CLASSES}
    top = max(cls_ms, key=cls_ms.get)
    top_ms = cls_ms[top]
    total_kernel_ms = sum(cls_ms.values())
    # algorithmic FLOPs of the top class: primitive quartets that pass the
    # reference's screening (exact count over the whole class)
    d_top = next(d for d in data if tuple(d[0]) == tuple(top))
    prim_top = screened_prim_quartets(*d_top[1:])
    flops_top = class_flops(top, prim_top, d_top[4].shape[0])
    achieved_tf = flops_top / (top_ms * 1e-3) / 1e12

    # end to end through the host API (pinned host buffers, copies timed)
    e2e = None
    if args.e2e_steps > 0:
        import torch.distributed as tdist
        form, err = "one call", None
        try:
            step_fn, h2d, d2h = e2e_one_call(L, data, dev_data)
            step_fn()                                   # warm-up, then checked
            torch.cuda.synchronize()
            e2e_check_one_call(data, dev_data, step_fn.out)
        except Exception as exc:   # noqa: BLE001
            err = "%s: %s" % (type(exc).__name__, exc)
        if world > 1:
            flag = torch.tensor([0 if err else 1], device=dev)
            tdist.all_reduce(flag, op=tdist.ReduceOp.MIN)
            if int(flag.item()) == 0 and err is None:
                err = "another rank's one-call form failed"
        if err is not None:
            step_fn = h2d = d2h = None
            form = "one call per class"
            step_fn, h2d, d2h = e2e_per_class(L, data, dev_data)
            step_fn()
            torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            step_fn()
        torch.cuda.synchronize()
        te = shard.max_over_ranks(time.perf_counter() - t0, dev)
        bw = link_bandwidth(dev)
        step_s = te / args.e2e_steps
        bound = {"h2d": h2d / bw["h2d_gbs"] / 1e9, "d2h": d2h / bw["d2h_gbs"] / 1e9,
                 "device": elapsed / args.steps}
        e2e = {"value": world * len(CLASSES) * args.nq * args.e2e_steps / te, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "step_s": step_s, "link": bw, "bound_s": bound,
               "frac_of_overlapped_bound": max(bound.values()) / step_s,
               "form": form,
               "note": "lrb_int2e_batch with pinned host buffers; all %d classes per step (%s: "
                       "one call over the classes' quartets back to back, its output checked "
                       "against the device-resident leg's, or one call per class); bound_s = "
                       "bytes / measured pinned copy bandwidth per direction, and the "
                       "device-resident step time; a fully overlapped pipeline takes the largest"
                       % (len(CLASSES), form)}
        if err is not None:
            e2e["one_call_error"] = err

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            v, s, tcpu = cpu_rate(data, threads, steps=3, warmup=1)
            cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"first {s} quartets of each of the {len(CLASSES)} classes of the "
                             f"same workload, 1 untimed + 3 timed passes ({3 * len(CLASSES) * s} "
                             f"quartets, {tcpu:.1f} s), oracle/ C++ restatement, OpenMP over "
                             f"quartets"}
        except Exception as exc:   # noqa: BLE001
            cpu = {"error": "%s: %s" % (type(exc).__name__, exc)}

    screening = None
    if rank == 0:
        try:
            screening = screening_summary(data)
        except Exception as exc:   # noqa: BLE001
            screening = {"error": "%s: %s" % (type(exc).__name__, exc)}

    rhf = None
    if args.rhf and world == 1:
        # single-process leg (no collectives): a failure is reported in its
        # key and does not cost the sweep's line
        try:
            rhf = run_rhf(args.guess, threads, fp64_peak, cpu=not args.no_cpu,
                          ablations=args.rhf_ablations, reference_run=args.rhf_reference_run)
        except Exception as exc:   # noqa: BLE001
            rhf = {"error": "%s: %s" % (type(exc).__name__, exc)}

    guess = None
    if args.guess_rings > 0 and world == 1:
        try:
            guess = run_guess_rings(args.guess, args.guess_rings)
        except Exception as exc:   # noqa: BLE001
            guess = {"error": "%s: %s" % (type(exc).__name__, exc)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded, distribution of the ERI sweep config)",
            "config": sweep_config(args, world,
                                   sum(t['out'].numel() for t in dev_data) * 8 / 1e9),
            "roofline": {"bound": "fp64", "kernel": "k_eri<%d,%d,%d,%d,0,double>" % top,
                         "achieved": achieved_tf, "peak": fp64_peak, "unit": "TFLOP/s",
                         "frac": achieved_tf / fp64_peak if fp64_peak > 0 else None,
                         "peak_source": "measured FP64 FMA probe (lrb_fp64_peak_probe) on this "
                                        "GPU (the measured copy and GEMM peaks have no FP64 figure)",
                         "kernel_ms": top_ms, "kernel_share": top_ms / total_kernel_ms,
                         "flop_convention": "fixed per-quartet count, see class_flops_bytes",
                         "traffic": (NCU_TRAFFIC_PER_QUARTET[tuple(top)] * d_top[4].shape[0]
                                     if tuple(top) in NCU_TRAFFIC_PER_QUARTET else None),
                         "algorithmic_bytes": class_flops_bytes(top, d_top[2], d_top[4])[1],
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of "
                                           "65,536 quartets of this class, scaled per quartet"},
            "class_kernel_ms": {"%d%d%d%d" % c: round(v, 4) for c, v in cls_ms.items()},
            "screening": screening,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "rhf": rhf,
            "guess": guess,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# Screening threshold of the FP32 SCF phases (learned + mixed): the FP32
# phases skip quartets whose Schwarz x density bound is below it; the FP64
# phase screens at TAU after a full rebuild, so the fixed point is the FP64
# operator's.
TAU_FP32 = 1e-11
TAU = 1e-13
TAU_PRIM = 1e-15        # primitive-quartet screening of every leg's Fock builds
RHF_TARGET_EH = 1e-6     # |E - E_FP64| a leg must reach to count


def fock_flops(cls, prim_quartets, quartets):
    """FLOPs of Fock-mode work of one class: the per-primitive convention of
    class_flops_bytes for the screened primitive quartets, plus 8 prod(nc)
    per shell quartet for the J/K digestion (cartesian blocks, no cart2sph)."""
    li, lj, lk, ll = cls
    nmax, mmax = li + lj, lk + ll
    nr = (nmax + mmax) // 2 + 1
    nf = ncart(li) * ncart(lj) * ncart(lk) * ncart(ll)
    H = sum((nmax - i + 1) * (mmax + 1) for i in range(1, li + 1)) + \
        (lj + 1) * (li + 1) * sum(mmax - k + 1 for k in range(1, lk + 1))
    per_prim = 50 + nr * (64 + 15 * (nmax + 1) * (mmax + 1) + 6 * H + 3 * nf)
    return float(prim_quartets) * per_prim + 8.0 * nf * float(quartets)


NCLASS_FOCK = 55        # Fock class ids: canonical class id, + 55 for the FP32 kernels


def lane_class(c, prec):
    """Classes with the lane-per-primitive Fock kernel (csrc/eri_kernel.cuh
    lp_passes): at most 27 cartesian elements, (ds|pp), (ds|ds), and (pp|pp)
    in FP64."""
    nf = ncart(c[0]) * ncart(c[1]) * ncart(c[2]) * ncart(c[3])
    return nf <= 27 or tuple(c) in ((2, 0, 1, 1), (2, 0, 2, 0)) or \
        (tuple(c) == (1, 1, 1, 1) and prec == 0)


def fock_kernel_name(c, prec):
    r = "double" if prec == 0 else "float"
    slot = "k_eri<%d,%d,%d,%d,1,%s>" % (tuple(c) + (r,))
    if lane_class(c, prec):
        return "k_fock_lp<%d,%d,%d,%d,%s> (quartets with >= 32 primitive quartets) + %s" % (
            tuple(c) + (r, slot))
    return slot


def fock_measure(ctx, P, fp64_peak, builds=1):
    """Fock builds G(P) of the cluster at its converged density: FP64 and
    all-FP32 builds per second (host wall clock around lrb_fock_G_prec,
    copies of P and G included), per-class kernel times (CUDA events) and
    counts, and the FP64 roofline of the dominant FP64 class."""
    import ctypes
    import torch
    from librint_b200 import _bindings as B
    L = B.lib()
    out = {"tau": TAU, "tau_prim": TAU_PRIM}
    ctx.set_tau_prim(TAU_PRIM)
    for prec, name in ((0, "fp64"), (1, "fp32")):
        ctx.fock_G_prec(P, prec, tau=TAU)          # warm
        torch.cuda.synchronize()
        L.lrb_profile_read((ctypes.c_double * 128)(), 128)
        L.lrb_fock_class_counts((ctypes.c_longlong * 128)(), (ctypes.c_longlong * 128)(), 128)
        L.lrb_profile_enable(1)
        t0 = time.perf_counter()
        for _ in range(builds):
            _, nq, _ = ctx.fock_G_prec(P, prec, tau=TAU)
        dt = (time.perf_counter() - t0) / builds
        L.lrb_profile_enable(0)
        ms = (ctypes.c_double * 128)()
        L.lrb_profile_read(ms, 128)
        qn, pn = (ctypes.c_longlong * 128)(), (ctypes.c_longlong * 128)()
        L.lrb_fock_class_counts(qn, pn, 128)
        off = 0 if prec == 0 else NCLASS_FOCK
        cls_rows = {}
        for c in CLASSES:
            i = class_id(c) + off
            if qn[i] == 0:
                continue
            k_ms = ms[i] / builds
            fl = fock_flops(c, pn[i] / builds, qn[i] / builds)
            cls_rows["%d%d%d%d" % c] = {"ms": round(k_ms, 3), "quartets": qn[i] // builds,
                                        "prim_quartets": pn[i] // builds,
                                        "tflops": round(fl / (k_ms * 1e-3) / 1e12, 3) if k_ms > 0 else None}
        kern = sum(v["ms"] for v in cls_rows.values())
        out[name] = {"build_s": dt, "builds_per_s": 1.0 / dt, "quartets": nq,
                     "kernel_ms": round(kern, 2), "classes": cls_rows}
        if prec == 0:
            top = max(cls_rows, key=lambda k: cls_rows[k]["ms"])
            r = cls_rows[top]
            out["roofline"] = {"bound": "fp64", "kernel": fock_kernel_name(tuple(int(x) for x in top), 0),
                               "achieved": r["tflops"], "peak": fp64_peak, "unit": "TFLOP/s",
                               "frac": r["tflops"] / fp64_peak if fp64_peak > 0 else None,
                               "kernel_ms": r["ms"], "kernel_share": r["ms"] / kern,
                               "flop_convention": "fock_flops: screened primitive quartets x "
                                                 "per-primitive count + 8 nf per quartet",
                               "peak_source": "lrb_fp64_peak_probe (measured FP64 FMA rate)"}
    return out


def rhf_cpu_baseline(mol, P, threads, iterations, budget_s=10.0, seed=7):
    """The reference's Fock build (src/scf.rs:316-410: every one of the
    nbas^4 shell quartets, digested into G) restated by the oracle on the
    host cores, timed on a uniform random sample of those quartets and
    extrapolated to one build and to the plain schedule's iteration count."""
    import oracle
    nb = mol.nbas
    rng = np.random.default_rng(seed)
    n = 2048
    for _ in range(3):
        sh = rng.integers(0, nb, size=(n, 4)).astype(np.int32)
        t0 = time.perf_counter()
        oracle.fock_G_quartets(mol, P, sh, nthreads=threads)
        t = time.perf_counter() - t0
        if t >= 0.5 * budget_s:
            break
        n = int(min(n * budget_s / max(t, 1e-3), 50_000_000))
    rate = n / t
    build_s = float(nb) ** 4 / rate
    return {"value": build_s * iterations, "unit": "s", "cores": threads, "kind": "port",
            "fock_build_s": build_s, "iterations": iterations,
            "sample": f"{n} shell quartets drawn uniformly from the nbas^4 = {nb ** 4} of one "
                      f"Fock build of this system ({t:.1f} s, {rate:.0f} quartets/s), oracle/ "
                      f"restatement of the reference's build, OpenMP; one build = nbas^4 / rate, "
                      f"times the {iterations} iterations of the plain GPU schedule (the "
                      f"reference's own P = I Roothaan loop needs more)"}


C3_FIXTURE = os.path.join(ROOT, "tests", "golden", "c3_energy.npz")


def run_rhf(guess_file=None, threads=1, fp64_peak=0.0, cpu=True, ablations=False,
            reference_run=False):
    """RHF wall time on the 60-atom C/H cluster (synthetic.c3_cluster: 36 C +
    24 H, 660 cartesian AOs, the seed-3 per-element C 3s2p1d / H 2s1p basis
    with K = 1..6).

    plain:     FP64 GPU path: core-H guess, DIIS(8), full Fock builds with
               Schwarz x density screening at tau = 1e-13 and primitive
               screening at TAU_PRIM, stopped at ||dP||/2 <= 1e-5;
    reference: the FP64 energy every leg is judged against: the converged
               (||dP||/2 <= 1e-8) FP64 SCF energy of this system recorded
               in tests/golden/c3_energy.npz (tests/test_gpu_configs.py
               checks that the GPU SCF reaches it again, and the energy
               functional at its density against the oracle); with
               reference_run, or without that file, the plain run continued
               from its density to 1e-8 on this GPU;
    mixed:     core-H start, incremental Fock builds with FP32 quartets
               (FP32 phases screened at tau_fp32 = 1e-11), FP64 finish at
               1e-13;
    learned_mixed: the same from the learned guess (when its network
               applies to this basis; the host prediction is timed in);
    with ablations also learned_fp64 and learned_fractional_mixed (the
               learned start with fractional occupations at its occupation
               cut, guess.density_from_lowdin).
    chosen = the fastest leg within 1e-6 Eh of the reference.  Times exclude
    the one-off pair table / Schwarz set-up (setup_s)."""
    import torch
    from librint_b200 import scf as S
    mol = synthetic.c3_cluster()
    t0 = time.perf_counter()
    ctx = S.MolContext(mol)
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    base = dict(guess=1, diis=8, tau=TAU, max_iter=300, check=False, tau_prim=TAU_PRIM)

    def run(conv, P0=None, extra_ms=0.0, density=False, **kw):
        t0 = time.perf_counter()
        r, Pc = ctx.scf(conv=conv, P0=P0, return_density=True, **dict(base, **kw))
        dt = time.perf_counter() - t0 + extra_ms / 1e3
        res = {"wall_s": dt, "energy": r.energy, "iterations": r.iterations,
               "converged": bool(r.converged), "delta": r.delta, "fock_s": r.fock_ms / 1e3,
               "quartets": r.quartets, "fp32_quartets": r.fp32_quartets}
        return (res, Pc) if density else res

    out = {"system": "c3_cluster seed 3: %d atoms, %d cartesian AOs, %d shells, %d electrons"
                     % (mol.natm, ctx.nao, mol.nbas, mol.nelec), "setup_s": setup,
           "target_eh": RHF_TARGET_EH, "tau": TAU, "tau_prim": TAU_PRIM, "tau_fp32": TAU_FP32}
    out["plain"], P_plain = run(1e-5, density=True)
    if reference_run or not os.path.exists(C3_FIXTURE):
        out["reference"], P_ref = run(1e-8, P0=P_plain, density=True)
        out["reference"]["note"] = "plain FP64 continued from the plain run's density to 1e-8"
    else:
        f = np.load(C3_FIXTURE)
        out["reference"] = {"energy": float(f["E_scf"]), "energy_oracle_functional": float(f["E_oracle"]),
                            "note": "recorded converged FP64 SCF energy (tests/golden/c3_energy.npz)"}
        P_ref = P_plain
    legs = ["plain"]
    if ablations:
        out["mixed"] = run(1e-5, mixed=1, tau_fp32=TAU_FP32)
        legs.append("mixed")
    if guess_file and os.path.exists(guess_file):
        from librint_b200.guess import LearnedGuess
        g = LearnedGuess.load(guess_file)
        if g.applies(mol):
            S_ov = ctx.int1e(0)
            tp = time.perf_counter()
            P0 = g.predict(mol, S=S_ov)
            t_pred = (time.perf_counter() - tp) * 1e3
            if ablations:
                out["learned_fp64"] = run(1e-5, P0=P0, extra_ms=t_pred)
                legs.append("learned_fp64")
                # fractional occupations at the predicted occupation cut
                tp = time.perf_counter()
                P0f = g.predict(mol, S=S_ov, fractional=True)
                t_f = (time.perf_counter() - tp) * 1e3
                out["learned_fractional_mixed"] = run(1e-5, P0=P0f, extra_ms=t_f, mixed=1,
                                                      tau_fp32=TAU_FP32)
                legs.append("learned_fractional_mixed")
            out["learned_mixed"] = run(1e-5, P0=P0, extra_ms=t_pred, mixed=1, tau_fp32=TAU_FP32)
            legs.append("learned_mixed")
            out["predict_ms"] = t_pred
        else:
            out["learned"] = "network does not apply to this basis"
    if "mixed" not in out:
        out["mixed"] = run(1e-5, mixed=1, tau_fp32=TAU_FP32)
        legs.append("mixed")
    e_ref = out["reference"]["energy"]
    for k in legs:
        out[k]["dE_vs_reference"] = out[k]["energy"] - e_ref
        out[k]["speedup_vs_plain"] = out["plain"]["wall_s"] / out[k]["wall_s"]
    ok = [k for k in legs if out[k]["converged"] and abs(out[k]["dE_vs_reference"]) <= RHF_TARGET_EH]
    if ok:
        best = min(ok, key=lambda k: out[k]["wall_s"])
        out["chosen"] = best
        out["chosen_wall_s"] = out[best]["wall_s"]
        out["plain_wall_s"] = out["plain"]["wall_s"]
        out["speedup_chosen_vs_plain"] = out["plain"]["wall_s"] / out[best]["wall_s"]
    out["fock"] = fock_measure(ctx, P_ref, fp64_peak)
    out["fock"]["density"] = "converged plain-run density"
    ctx.close()
    if cpu:
        out["cpu_baseline"] = rhf_cpu_baseline(mol, P_ref, threads, out["plain"]["iterations"])
    return out


def run_guess_rings(guess_file, n, first=2000, conv=1e-8):
    """The learned-guess configuration: C6H6-like rings (synthetic.benzene_like,
    seeds 10000 + i) held out of the network's training set (rings 0..1999),
    each converged from the core-Hamiltonian start and from the learned start
    (train_guess.evaluate_one: DIIS(8), tau 1e-12, primitive screening
    TAU_PRIM, ||dP||/2 <= conv, the settings of the recorded evaluation); SCF
    iterations and wall time per start (the prediction timed into the
    learned one) and the largest energy difference between the two."""
    from librint_b200 import train_guess
    from librint_b200.guess import LearnedGuess
    g = LearnedGuess.load(guess_file)
    t0 = time.perf_counter()
    rows = [r for r in (train_guess.evaluate_one(g, train_guess.geometry(i, "rings"), conv,
                                                 {"tau_prim": TAU_PRIM})
                        for i in range(first, first + n)) if r is not None]
    out = train_guess.summarise(rows)
    out.update(config="C6H6-like rings %d..%d (held out of training), 120 cartesian AOs"
                      % (first, first + n - 1),
               conv=conv, tau_prim=TAU_PRIM, wall_s=time.perf_counter() - t0,
               iterations_saved=out["it_core"] - out["it_learned"])
    return out


def run_reference(args, rank, world, threads):
    """The reference arm: the CPU restatement of the reference algorithm
    (oracle/, OpenMP on every host thread) on the same generated workload as
    the GPU arm, each step one bounded pass over the first quartets of every
    class (cpu_rate, the same measurement as the GPU arm's cpu_baseline)."""
    if rank != 0:
        return
    data = generate(args.nq, shard.shard_seed(2, 0), procs=threads)
    value, s, tt = cpu_rate(data, threads, steps=args.steps, warmup=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded, distribution of the ERI sweep config)",
        "config": sweep_config(args, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"each step: the first {s} quartets of each of the "
                                   f"{len(CLASSES)} classes of this workload; the reference "
                                   f"(Rust, nightly Enzyme toolchain) cannot be built here, so "
                                   f"its CPU restatement in oracle/ runs with OpenMP over quartets"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def sweep_config(args, world, out_gb=None):
    cfg = {"workload": "ERI sweep: %s x %d quartets per class per GPU, K=1..6, exponents "
                       "log-uniform [0.05,5000], centres in a 10 A cube, spherical output"
                       % ("21 classes (ss|ss)..(dd|dd)" if len(CLASSES) == 21 else
                          "classes " + ",".join("%d%d%d%d" % c for c in CLASSES), args.nq),
           "quartets_per_step": len(CLASSES) * args.nq * world,
           "parallelism": f"dp{world} (independent quartet shards)"}
    if out_gb is not None:
        cfg["l2"] = "outputs (%.1f GB/step) exceed L2; no flush needed" % out_gb
    return cfg


if __name__ == "__main__":
    main()
