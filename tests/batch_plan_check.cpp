// CPU check of librint_b200/csrc/batch_plan.h (built and run by
// tests/test_batch_plan.py): plan_batch against a serial restatement of the
// same rules, one check at a time, on random batches -- the sweep layout
// (every quartet with its own shells, atoms and env entries; also with each
// atom's coordinates after its shell's data, and with the atom indices
// reversed), quartets over a small shared molecule, generally contracted
// shells, unreferenced shells, and single corruptions (a shell index, a bas entry, an atom index or a
// coordinate pointer out of range) -- with small and large chunk limits.
// Prints "ok <cases>" or the first difference and exits non-zero.
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../librint_b200/csrc/batch_plan.h"

using lrb::plan::BatchPlan;
using lrb::plan::ChunkRange;

namespace {

struct Batch {
  std::vector<int> atm, bas, shls;
  std::vector<double> env;
  int natm() const { return (int)atm.size() / 6; }
  int nbas() const { return (int)bas.size() / 8; }
  long long nq() const { return (long long)shls.size() / 4; }
};

// Serial restatement: index check, check of every shell entry and the
// contraction scan, greedy chunks, then per chunk its ranges; the batch is
// streamed only if every range is valid and each lies after the previous.
int ref_plan(int coord, const Batch &b, long long head, long long cq_max, long long co_max,
             BatchPlan &p, std::string &msg) {
  p = BatchPlan();
  const int nbas = b.nbas(), natm = b.natm();
  const long long nenv = (long long)b.env.size(), nq = b.nq();
  for (long long q = 0; q < 4 * nq; ++q)
    if (b.shls[q] < 0 || b.shls[q] >= nbas) return msg = "shell index out of range", LRB_ERR_INPUT;
  for (int s = 0; s < nbas; ++s) {
    const int *e = &b.bas[8 * s];
    if (e[3] < 1 || e[2] < 1 || e[5] < 0 || e[6] < 0 || (long long)e[5] + e[2] > nenv ||
        (long long)e[6] + (long long)e[2] * e[3] > nenv)
      return msg = "bas entry out of range (nprim, nctr or env pointers)", LRB_ERR_INPUT;
    p.gc = p.gc || e[3] > 1;
  }
  if (p.gc) return msg = "", LRB_OK;
  auto rows = [&](int s) {
    const int l = b.bas[8 * s + 1];
    return (long long)(coord == 0 ? (l + 1) * (l + 2) / 2 : 2 * l + 1) * b.bas[8 * s + 3];
  };
  p.qb = {0};
  p.ob = {0};
  long long cq = 0, co = 0, tot = 0;
  for (long long q = 0; q < nq; ++q) {
    long long d = 1;
    for (int a = 0; a < 4; ++a) d *= rows(b.shls[4 * q + a]);
    if (cq > 0 && (cq == cq_max || co + d > co_max)) {
      p.qb.push_back(q);
      p.ob.push_back(tot);
      p.max_q = std::max(p.max_q, cq);
      p.max_len = std::max(p.max_len, co);
      cq = co = 0;
    }
    ++cq;
    co += d;
    tot += d;
  }
  p.qb.push_back(nq);
  p.ob.push_back(tot);
  p.max_q = std::max(p.max_q, cq);
  p.max_len = std::max(p.max_len, co);
  const int nchunk = (int)p.qb.size() - 1;
  p.streamed = nchunk >= 2;
  p.rg.assign(nchunk, ChunkRange{0, 0, 0, 0, 0, 0});
  for (int c = 0; c < nchunk && p.streamed; ++c) {
    ChunkRange r{nbas, -1, natm, -1, nenv, -1};
    for (long long q = 4 * p.qb[c]; q < 4 * p.qb[c + 1]; ++q) {
      r.s0 = std::min(r.s0, b.shls[q]);
      r.s1 = std::max(r.s1, b.shls[q] + 1);
    }
    for (int sh = r.s0; sh < r.s1 && p.streamed; ++sh) {
      const int *e = &b.bas[8 * sh];
      if (e[0] < 0 || e[0] >= natm) {
        p.streamed = false;
        break;
      }
      r.a0 = std::min(r.a0, e[0]);
      r.a1 = std::max(r.a1, e[0] + 1);
      r.e0 = std::min({r.e0, (long long)e[5], (long long)e[6]});
      r.e1 = std::max({r.e1, (long long)e[5] + e[2], (long long)e[6] + (long long)e[2] * e[3]});
    }
    for (int a = r.a0; a < r.a1 && p.streamed; ++a) {
      const long long pc = b.atm[6 * a + 1];
      if (pc < 0 || pc + 3 > nenv) p.streamed = false;
      r.e0 = std::min(r.e0, pc);
      r.e1 = std::max(r.e1, pc + 3);
    }
    const ChunkRange *prev = c > 0 ? &p.rg[c - 1] : nullptr;
    if (r.e0 < head || (prev && (r.s0 < prev->s1 || r.a0 < prev->a1 || r.e0 < prev->e1)))
      p.streamed = false;
    p.rg[c] = r;
  }
  return msg = "", LRB_OK;
}

// One shell with its own atom appended: l, K primitives, nctr contractions.
void add_shell(Batch &b, int l, int k, int nctr, int atom) {
  b.bas.insert(b.bas.end(), {atom, l, k, nctr, 0, (int)b.env.size(),
                             (int)b.env.size() + k, 0});
  b.env.resize(b.env.size() + k + (size_t)k * nctr, 0.5);
}

void add_atom(Batch &b) {
  b.atm.insert(b.atm.end(), {6, (int)b.env.size(), 1, 0, 0, 0});
  b.env.resize(b.env.size() + 3, 0.1);
}

Batch sweep(std::mt19937 &g, int nq, int extra_unreferenced, bool gc) {
  Batch b;
  b.env.assign(20, 0.0);
  std::uniform_int_distribution<int> L(0, 3), K(1, 6);
  for (int q = 0; q < nq; ++q)
    for (int a = 0; a < 4; ++a) {
      add_atom(b);
      add_shell(b, L(g), K(g), gc && (g() % 7 == 0) ? 2 : 1, b.natm() - 1);
      b.shls.push_back(b.nbas() - 1);
    }
  for (int e = 0; e < extra_unreferenced; ++e) {
    add_atom(b);
    add_shell(b, L(g), K(g), 1, b.natm() - 1);
  }
  return b;
}

// The sweep layout with each atom's coordinates after its shell's data in
// env (the chunk's env range then ends at an atom), or with the atom
// indices reversed (env and shells in order, atoms not).
Batch sweep_variant(std::mt19937 &g, int nq, bool atoms_after, bool reverse_atoms) {
  Batch b;
  b.env.assign(20, 0.0);
  std::uniform_int_distribution<int> L(0, 3), K(1, 6);
  for (int q = 0; q < nq; ++q)
    for (int a = 0; a < 4; ++a) {
      if (atoms_after) {
        add_shell(b, L(g), K(g), 1, b.natm());
        add_atom(b);
      } else {
        add_atom(b);
        add_shell(b, L(g), K(g), 1, b.natm() - 1);
      }
      b.shls.push_back(b.nbas() - 1);
    }
  if (reverse_atoms) {
    const int n = b.natm();
    std::vector<int> atm(b.atm.size());
    for (int a = 0; a < n; ++a)
      std::copy(&b.atm[6 * a], &b.atm[6 * a] + 6, &atm[6 * (n - 1 - a)]);
    b.atm = atm;
    for (int s = 0; s < b.nbas(); ++s) b.bas[8 * s] = n - 1 - b.bas[8 * s];
  }
  return b;
}

Batch shared(std::mt19937 &g, int nbas, int nq, bool gc) {
  Batch b;
  b.env.assign(20, 0.0);
  std::uniform_int_distribution<int> L(0, 3), K(1, 6);
  const int natm = std::max(1, nbas / 3);
  for (int a = 0; a < natm; ++a) add_atom(b);
  for (int s = 0; s < nbas; ++s) add_shell(b, L(g), K(g), gc && s == nbas / 2 ? 3 : 1, s % natm);
  std::uniform_int_distribution<int> S(0, nbas - 1);
  for (int q = 0; q < 4 * nq; ++q) b.shls.push_back(S(g));
  return b;
}

// One corruption of kind k at a random place.
void corrupt(std::mt19937 &g, Batch &b, int k) {
  const int nbas = b.nbas(), natm = b.natm();
  switch (k) {
    case 0: b.shls[g() % b.shls.size()] = (g() & 1) ? nbas + (int)(g() % 5) : -1 - (int)(g() % 3); break;
    case 1: b.bas[8 * (g() % nbas) + 2] = 0; break;                                  // nprim
    case 2: b.bas[8 * (g() % nbas) + 6] = (int)b.env.size(); break;                  // coefficients past env
    case 3: b.bas[8 * (g() % nbas) + 3] = 0; break;                                  // nctr
    case 4: b.bas[8 * (g() % nbas) + 0] = (g() & 1) ? natm : -1; break;              // atom index
    case 5: b.atm[6 * (g() % natm) + 1] = (int)b.env.size() - 1; break;              // coordinates past env
    default: break;
  }
}

bool same(const BatchPlan &a, const BatchPlan &b, std::string &why) {
  if (a.gc != b.gc) return why = "gc", false;
  if (a.gc) return true;
  if (a.qb != b.qb) return why = "chunk boundaries", false;
  if (a.ob != b.ob) return why = "output offsets", false;
  if (a.max_q != b.max_q || a.max_len != b.max_len) return why = "chunk maxima", false;
  if (a.streamed != b.streamed) return why = "streamed", false;
  if (a.streamed)
    for (size_t c = 0; c < a.rg.size(); ++c)
      if (std::memcmp(&a.rg[c], &b.rg[c], sizeof(ChunkRange)) != 0) return why = "ranges", false;
  return true;
}

}  // namespace

int main() {
  std::mt19937 g(12345);
  int cases = 0;
  const long long limits[][2] = {{1, 1LL << 25}, {3, 1LL << 25}, {64, 300}, {1 << 18, 1LL << 25},
                                 {1 << 18, 5000}, {7, 1}};
  for (int rep = 0; rep < 60; ++rep) {
    for (int kind = -1; kind < 6; ++kind) {
      for (int layout = 0; layout < 6; ++layout) {
        Batch b;
        if (layout == 4) b = sweep_variant(g, 1 + (int)(g() % 300), true, false);
        if (layout == 5) b = sweep_variant(g, 1 + (int)(g() % 300), false, true);
        if (layout == 0) b = sweep(g, 1 + (int)(g() % 300), 0, false);
        if (layout == 1) b = sweep(g, 1 + (int)(g() % 300), 1 + (int)(g() % 5), rep % 5 == 0);
        if (layout == 2) b = shared(g, 2 + (int)(g() % 40), 1 + (int)(g() % 400), rep % 5 == 1);
        if (layout == 3) b = sweep(g, rep == 0 ? 150000 : 20000, 3, false);   // several threads
        if (layout == 3 && rep % 10 != 0) continue;
        if (kind >= 0) corrupt(g, b, kind);
        for (const auto &lim : limits) {
          for (int coord = 0; coord < 2; ++coord) {
            BatchPlan pr, pp;
            std::string mr;
            const char *mp = "";
            const int rr = ref_plan(coord, b, 20, lim[0], lim[1], pr, mr);
            const int rp = lrb::plan::plan_batch(coord, b.shls.data(), b.nq(), b.atm.data(),
                                                 b.natm(), b.bas.data(), b.nbas(),
                                                 (long long)b.env.size(), 20, lim[0], lim[1], pp, &mp);
            std::string why;
            if (rr != rp || mr != mp) why = "status " + mr + " / " + mp;
            else if (rr == LRB_OK && !same(pr, pp, why)) why = "plan: " + why;
            if (!why.empty()) {
              std::printf("difference: layout %d corruption %d limits %lld %lld coord %d: %s\n",
                          layout, kind, lim[0], lim[1], coord, why.c_str());
              return 1;
            }
            ++cases;
          }
        }
      }
    }
  }
  std::printf("ok %d\n", cases);
  return 0;
}
