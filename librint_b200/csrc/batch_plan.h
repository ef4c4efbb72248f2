// Host-side planning of lrb_int2e_batch (plain C++, no CUDA): the checks of
// the quartet list and of the molecule that must pass before any device
// work, the split of the quartets into chunks, and the part of the molecule
// each chunk reaches.  Kept apart from the CUDA host code so that CPU tests
// can compile it with a host compiler and compare it with a serial
// restatement.
#pragma once

#include <sched.h>

#include <algorithm>
#include <atomic>
#include <memory>
#include <thread>
#include <vector>

#include "../../include/librint_b200.h"

namespace lrb {
namespace plan {

// Host threads this process may run on (its CPU affinity), at least 1.
inline int host_threads() {
  cpu_set_t set;
  if (sched_getaffinity(0, sizeof set, &set) == 0) return std::max(1, CPU_COUNT(&set));
  return std::max(1u, std::thread::hardware_concurrency());
}

// fn(begin, end) over contiguous parts of [0, n), each of at least `grain`
// items, on up to 32 host threads (the caller's thread takes the first
// part); one part when n <= grain.  A thread that cannot be started runs its
// part on the caller's thread.
template <class F>
void host_parallel(long long n, long long grain, F &&fn) {
  if (n <= 0) return;
  const long long nt = std::min<long long>({(long long)host_threads(), 32, (n + grain - 1) / grain});
  if (nt <= 1) {
    fn(0LL, n);
    return;
  }
  const long long per = (n + nt - 1) / nt;
  std::vector<std::thread> th;
  th.reserve((size_t)nt);
  for (long long t = 1; t < nt; ++t) {
    const long long b = t * per, e = std::min(n, b + per);
    if (b >= e) break;
    try {
      th.emplace_back([&fn, b, e] { fn(b, e); });
    } catch (...) {
      fn(b, e);
    }
  }
  fn(0LL, std::min(n, per));
  for (std::thread &x : th) x.join();
}

// Items per host thread below which a loop stays on one thread.
constexpr long long HOST_GRAIN = 1 << 16;

// Rows of a shell's block: cartesian (coord 0) or spherical components times
// contractions.
inline long long shell_rows(int coord, const int *bas, int s) {
  const int l = bas[8 * s + 1];
  return (long long)(coord == 0 ? (l + 1) * (l + 2) / 2 : 2 * l + 1) * bas[8 * s + 3];
}

// A bas entry whose primitive count, contraction count or env pointers are
// out of range (the check every shell must pass).
inline bool bad_shell_entry(const int *b, long long nenv) {
  return b[3] < 1 || b[2] < 1 || b[5] < 0 || b[6] < 0 || (long long)b[5] + b[2] > nenv ||
         (long long)b[6] + (long long)b[2] * b[3] > nenv;
}

// Shells, atoms and env entries (half-open ranges) that one chunk's quartets
// can reach: every shell between the lowest and highest index it names,
// their atoms, and the env entries of those shells and atoms.
struct ChunkRange {
  int s0, s1, a0, a1;
  long long e0, e1;
};

struct BatchPlan {
  std::vector<long long> qb, ob;   // chunk c: quartets [qb[c], qb[c+1]), output from ob[c]
  long long max_q = 0, max_len = 1;
  bool gc = false;                 // a shell has nctr > 1 (the plan is then not used)
  bool streamed = false;           // chunks may upload their own ranges (rg)
  std::vector<ChunkRange> rg;
  int nchunk() const { return (int)qb.size() - 1; }
};

// Checks and plans a batch:
//  * every shell index of shls in [0, nbas), else LRB_ERR_INPUT "shell index
//    out of range";
//  * every shell's bas entry (bad_shell_entry), else LRB_ERR_INPUT "bas entry
//    out of range (nprim, nctr or env pointers)";
//  * chunks of at most chunk_q quartets and, past the first quartet of a
//    chunk, at most chunk_out output doubles;
//  * per chunk its ChunkRange; streamed when there are at least two chunks,
//    every chunk's shells name atoms in [0, natm) whose coordinates lie in
//    env, the ranges start at or after env[head] and each chunk's ranges lie
//    after the previous chunk's.
// The shells inside the chunks' ranges are checked in the same pass that
// finds the ranges; the others in a pass of their own.  A bad atom index or
// coordinate pointer is left to the device-side check (it only makes the
// batch not streamed).  *msg receives the error text.
inline int plan_batch(int coord, const int *shls, long long nq, const int *atm, int natm,
                      const int *bas, int nbas, long long nenv, long long head, long long chunk_q,
                      long long chunk_out, BatchPlan &p, const char **msg) {
  p = BatchPlan();
  *msg = "";
  // shell indices and block sizes, one pass over the quartets
  std::unique_ptr<long long[]> blen(new long long[(size_t)std::max(nq, 1LL)]);
  std::atomic<bool> bad_index{false};
  host_parallel(nq, HOST_GRAIN, [&](long long b, long long e) {
    for (long long q = b; q < e; ++q) {
      const int *s4 = shls + 4 * q;
      if (s4[0] < 0 || s4[0] >= nbas || s4[1] < 0 || s4[1] >= nbas || s4[2] < 0 ||
          s4[2] >= nbas || s4[3] < 0 || s4[3] >= nbas) {
        bad_index.store(true, std::memory_order_relaxed);
        return;
      }
      // unsigned: the entries are checked only later, and a plan from
      // unchecked entries is never used
      const unsigned long long d = (unsigned long long)shell_rows(coord, bas, s4[0]) *
                                   (unsigned long long)shell_rows(coord, bas, s4[1]) *
                                   (unsigned long long)shell_rows(coord, bas, s4[2]) *
                                   (unsigned long long)shell_rows(coord, bas, s4[3]);
      blen[q] = (long long)d;
    }
  });
  if (bad_index.load()) {
    *msg = "shell index out of range";
    return LRB_ERR_INPUT;
  }
  // chunks (greedy, in quartet order)
  p.qb.push_back(0);
  p.ob.push_back(0);
  {
    long long cq = 0, co = 0, tot = 0;
    for (long long q = 0; q < nq; ++q) {
      const long long b = blen[q];
      if (cq > 0 && (cq == chunk_q || co + b > chunk_out)) {
        p.qb.push_back(q);
        p.ob.push_back(tot);
        p.max_q = std::max(p.max_q, cq);
        p.max_len = std::max(p.max_len, co);
        cq = co = 0;
      }
      ++cq;
      co += b;
      tot += b;
    }
    p.qb.push_back(nq);
    p.ob.push_back(tot);
    p.max_q = std::max(p.max_q, cq);
    p.max_len = std::max(p.max_len, co);
  }
  blen.reset();
  // per chunk: its shell range, the checks of those shells, its atom and env
  // ranges
  const int nchunk = p.nchunk();
  p.rg.assign(nchunk, ChunkRange{0, 0, 0, 0, 0, 0});
  std::vector<char> ok_atoms(nchunk, 0);
  std::atomic<bool> bad_entry{false}, any_gc{false};
  host_parallel(nchunk, 1, [&](long long b, long long e) {
    for (long long c = b; c < e; ++c) {
      ChunkRange r{nbas, -1, natm, -1, nenv, -1};
      for (long long q = 4 * p.qb[c]; q < 4 * p.qb[c + 1]; ++q) {
        r.s0 = std::min(r.s0, shls[q]);
        r.s1 = std::max(r.s1, shls[q] + 1);
      }
      bool atoms = true, gc = false;
      for (int sh = r.s0; sh < r.s1; ++sh) {
        const int *bs = bas + 8 * sh;
        if (bad_shell_entry(bs, nenv)) {
          bad_entry.store(true, std::memory_order_relaxed);
          return;
        }
        gc = gc || bs[3] > 1;
        if (bs[0] < 0 || bs[0] >= natm) {
          atoms = false;
          continue;
        }
        r.a0 = std::min(r.a0, bs[0]);
        r.a1 = std::max(r.a1, bs[0] + 1);
        r.e0 = std::min({r.e0, (long long)bs[5], (long long)bs[6]});
        r.e1 = std::max({r.e1, (long long)bs[5] + bs[2], (long long)bs[6] + (long long)bs[2] * bs[3]});
      }
      if (gc) any_gc.store(true, std::memory_order_relaxed);
      for (int a = r.a0; atoms && a < r.a1; ++a) {
        const long long pc = atm[6 * a + 1];
        if (pc < 0 || pc + 3 > nenv) {
          atoms = false;
          break;
        }
        r.e0 = std::min(r.e0, pc);
        r.e1 = std::max(r.e1, pc + 3);
      }
      p.rg[c] = r;
      ok_atoms[c] = atoms;
    }
  });
  if (bad_entry.load()) {
    *msg = "bas entry out of range (nprim, nctr or env pointers)";
    return LRB_ERR_INPUT;
  }
  // the shells outside every chunk's range
  {
    std::vector<std::pair<int, int>> iv;
    iv.reserve(nchunk);
    for (const ChunkRange &r : p.rg)
      if (r.s1 > r.s0) iv.emplace_back(r.s0, r.s1);
    std::sort(iv.begin(), iv.end());
    std::vector<std::pair<int, int>> gaps;
    int next = 0;
    for (const auto &v : iv) {
      if (v.first > next) gaps.emplace_back(next, v.first);
      next = std::max(next, v.second);
    }
    if (next < nbas) gaps.emplace_back(next, nbas);
    for (const auto &g : gaps) {
      host_parallel(g.second - g.first, HOST_GRAIN, [&](long long b, long long e) {
        bool gc = false;
        for (long long s = g.first + b; s < g.first + e; ++s) {
          const int *bs = bas + 8 * s;
          if (bad_shell_entry(bs, nenv)) {
            bad_entry.store(true, std::memory_order_relaxed);
            return;
          }
          gc = gc || bs[3] > 1;
        }
        if (gc) any_gc.store(true, std::memory_order_relaxed);
      });
    }
  }
  if (bad_entry.load()) {
    *msg = "bas entry out of range (nprim, nctr or env pointers)";
    return LRB_ERR_INPUT;
  }
  p.gc = any_gc.load();
  // streamed layout: every chunk's ranges valid and after the previous chunk's
  p.streamed = nchunk >= 2;
  for (int c = 0; c < nchunk && p.streamed; ++c) {
    const ChunkRange &r = p.rg[c];
    const ChunkRange *prev = c > 0 ? &p.rg[c - 1] : nullptr;
    if (!ok_atoms[c] || r.e0 < head ||
        (prev && (r.s0 < prev->s1 || r.a0 < prev->a1 || r.e0 < prev->e1)))
      p.streamed = false;
  }
  return LRB_OK;
}

}  // namespace plan
}  // namespace lrb
