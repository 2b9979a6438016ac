// rotate_check.cpp -- CPU check of the pair-rotate launch planning (no GPU).
//
// Plans random runs of one-qubit gates with rbk::plan_rotations, with and
// without an owed diagonal (one-bit phases and controlled Zs) and Z-type
// overlaps, and executes the planned launches with a plain C++ model of what
// pair_rotate_kernel does with a pair_rotate_set: per tile and thread the load
// layout, the owed diagonal from the kernel's decomposition of the factor and
// sign, the Z sums in the kernel's per-thread / per-warp bookkeeping, the
// register phases through swizzled shared-memory slots, the overlaps in the
// arithmetic the per-gate kinds select, the gates, and the store.  Where a
// phase exchange waits only on a warp barrier, the model checks that every warp
// reads back only slots it wrote.  States, overlaps and Z sums must equal the
// gates applied directly.  Test code only; built and run by
// tests/test_rotate_plan.py.
#include <algorithm>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "rbk_rotate_plan.h"

using cplx = std::complex<double>;
using namespace rbk;

namespace {

int failures = 0;

void fail(const char* what, int seed)
{
  std::printf("FAIL seed=%d: %s\n", seed, what);
  ++failures;
}

// rbk::smem_slot for complex<double> (VBITS = 0).
uint32_t slot_of(uint32_t j)
{
  uint32_t u = j;
  const uint32_t f = (u >> 3) ^ (u >> 6) ^ (u >> 9) ^ (u >> 12);
  u ^= f & 7u;
  return u;
}

int parity(uint64_t x) { return __builtin_popcountll(x) & 1; }

cplx mat(const double* m, int k) { return {m[2 * k], m[2 * k + 1]}; }

// Runs the planned launches on (lam, psi); overlap results by slot (imaginary
// parts, as the kernel's finish writes them) in ov.
void run_model(int n, const std::vector<pair_rotate_set>& sets, std::vector<cplx>& lam, std::vector<cplx>& psi,
               std::vector<double>& ov, int seed)
{
  constexpr int RB = kPairRegBits, NE = 1 << RB, KT = 8 + RB, NT = 256;
  for (const pair_rotate_set& S : sets) {
    const spin_group& g = S.g;
    if (g.K != KT || g.nphases < 1 || g.nphases > kSpinPhases || g.nflips != g.nphases * RB || g.nflips > kMaxRotFlips) {
      fail("launch shape", seed);
      return;
    }
    for (int b = 0; b < RB; ++b) if (g.phase_reg[0][b] != 8 + b) fail("phase 0 is not the load layout", seed);
    for (int b = 0; b < 8; ++b) if (g.phase_thr[0][b] != b) fail("phase 0 is not the load layout", seed);
    for (int p = 0; p < g.nphases; ++p) {
      uint32_t seen = 0;
      for (int k = 0; k < RB; ++k) seen |= 1u << g.phase_reg[p][k];
      for (int b = 0; b < 8; ++b) seen |= 1u << g.phase_thr[p][b];
      if (seen != (1u << KT) - 1) fail("a phase layout is not a permutation of the tile bits", seed);
    }
    uint64_t tmask = 0;
    for (int b = 0; b < KT; ++b) tmask |= 1ull << g.tile_phys[b];
    if (__builtin_popcountll(tmask) != KT || (tmask >> n) != 0 || (tmask & 7) != 7) fail("tile bits", seed);
    const pre_diag& D = S.pre;
    const uint64_t tiles = 1ull << (n - KT);
    // Pre-step bookkeeping of the kernel: per-thread factor over thread bits, partner row and pair parity.
    std::vector<cplx> fthr(NT), freg(NE);
    std::vector<uint64_t> mthr(NT);
    std::vector<uint32_t> qthr(NT);
    if (D.active) {
      for (int t = 0; t < NT; ++t) {
        cplx f{1.0, 0.0};
        uint64_t tphys = 0, m = 0;
        for (int b = 0; b < 8; ++b) if ((t >> b) & 1) tphys |= 1ull << g.tile_phys[b];
        uint32_t q = 0;
        for (int b = 0; b < 8; ++b)
          if ((t >> b) & 1) {
            f *= cplx{D.u[g.tile_phys[b]][0], D.u[g.tile_phys[b]][1]};
            m ^= D.full[g.tile_phys[b]];
            q ^= static_cast<uint32_t>(__builtin_popcountll(tphys & D.adj[g.tile_phys[b]]));
          }
        fthr[static_cast<size_t>(t)] = f;
        mthr[static_cast<size_t>(t)] = m;
        qthr[static_cast<size_t>(t)] = q & 1u;
      }
      for (int it = 0; it < NE; ++it) {
        cplx r{1.0, 0.0};
        for (int b = 0; b < RB; ++b) if ((it >> b) & 1) r *= cplx{D.u[g.tile_phys[8 + b]][0], D.u[g.tile_phys[8 + b]][1]};
        freg[static_cast<size_t>(it)] = r;
      }
    }
    std::vector<double> acc(kMaxRotFlips, 0.0);
    std::vector<double> zt(NT, 0.0), zr0(NT, 0.0), zr1(NT, 0.0), zr2(NT, 0.0);
    std::vector<double> zh(static_cast<size_t>(kMaxQubits) * 8, 0.0);
    for (uint64_t t = 0; t < tiles; ++t) {
      std::vector<cplx> tl(1u << KT), tp(1u << KT);
      std::vector<int> owner(1u << KT, -1);
      std::vector<cplx> el(NT * NE), ep(NT * NE);
      std::vector<uint64_t> bases(NT);
      for (int tid = 0; tid < NT; ++tid) {
        uint64_t tphys = 0;
        for (int b = 0; b < 8; ++b) if ((tid >> b) & 1) tphys |= 1ull << g.tile_phys[b];
        uint64_t base = tphys;
        for (int r = 0; r < g.num_runs; ++r) base |= ((t >> g.run_src[r]) & ((1ull << g.run_len[r]) - 1)) << g.run_dst[r];
        bases[static_cast<size_t>(tid)] = base;
        for (int it = 0; it < NE; ++it) {
          uint64_t p = base;
          for (int b = 0; b < RB; ++b) if ((it >> b) & 1) p |= 1ull << g.tile_phys[8 + b];
          el[static_cast<size_t>(tid * NE + it)] = lam[p];
          ep[static_cast<size_t>(tid * NE + it)] = psi[p];
        }
        if (D.active) {
          if (D.nz > 0) {
            double tot = 0, r0 = 0, r1 = 0, r2 = 0;
            for (int it = 0; it < NE; ++it) {
              const double c = (std::conj(el[static_cast<size_t>(tid * NE + it)]) * ep[static_cast<size_t>(tid * NE + it)]).imag();
              tot += c;
              if (it & 1) r0 += c;
              if (it & 2) r1 += c;
              if (it & 4) r2 += c;
            }
            zt[static_cast<size_t>(tid)] += tot;
            zr0[static_cast<size_t>(tid)] += r0;
            zr1[static_cast<size_t>(tid)] += r1;
            zr2[static_cast<size_t>(tid)] += r2;
            for (uint64_t hb = base ^ tphys; hb; hb &= hb - 1)
              zh[static_cast<size_t>(__builtin_ctzll(hb)) * 8 + static_cast<size_t>(tid >> 5)] += tot;
          }
          cplx f{D.g[0], D.g[1]};
          const uint64_t hbase = base ^ tphys;
          for (uint64_t hb = hbase; hb; hb &= hb - 1) {
            const int q = __builtin_ctzll(hb);
            f *= cplx{D.u[q][0], D.u[q][1]};
          }
          f *= fthr[static_cast<size_t>(tid)];
          uint32_t qb = 0;
          for (uint64_t hb = hbase; hb; hb &= hb - 1) qb ^= static_cast<uint32_t>(__builtin_popcountll(hbase & D.adj[__builtin_ctzll(hb)]));
          qb ^= qthr[static_cast<size_t>(tid)] ^ static_cast<uint32_t>(parity(hbase & mthr[static_cast<size_t>(tid)]));
          for (int it = 0; it < NE; ++it) {
            cplx fi = f * freg[static_cast<size_t>(it)];
            if ((qb ^ (D.qr >> it) ^ static_cast<uint32_t>(parity(base & D.mr[it]))) & 1) fi = -fi;
            el[static_cast<size_t>(tid * NE + it)] *= fi;
            ep[static_cast<size_t>(tid * NE + it)] *= fi;
          }
        }
      }
      for (int p = 0; p < g.nphases; ++p) {
        // Slots of this phase's layout per thread and register slot.
        auto slot_at = [&](int lp, int tid, int i) {
          uint32_t j = 0;
          for (int b = 0; b < 8; ++b) j |= ((uint32_t(tid) >> b) & 1u) << g.phase_thr[lp][b];
          for (int k = 0; k < RB; ++k) j |= ((uint32_t(i) >> k) & 1u) << g.phase_reg[lp][k];
          return slot_of(j);
        };
        for (int tid = 0; tid < NT; ++tid) {
          cplx* E = &el[static_cast<size_t>(tid * NE)];
          cplx* P = &ep[static_cast<size_t>(tid * NE)];
          if (p > 0)
            for (int i = 0; i < NE; ++i) {
              const uint32_t s = slot_at(p, tid, i);
              if (owner[s] >= 0 && owner[s] != (tid >> 5) && !S.block_sync[p - 1]) fail("a warp reads a slot another warp wrote behind a warp barrier", seed);
              E[i] = tl[s];
              P[i] = tp[s];
            }
          for (int k = 0; k < RB; ++k) {
            const int f = p * RB + k;
            const auto& F = S.flip[f];
            if (F.okind != 0) {
              const double sg = F.minus ? -1.0 : 1.0;
              double xr = 0, xi = 0;
              for (int i = 0; i < NE; ++i) {
                if ((i >> k) & 1) continue;
                const cplx A = std::conj(E[i]) * P[i | (1 << k)], B = std::conj(E[i | (1 << k)]) * P[i];
                if (F.okind & 1) xr += (A + sg * B).real();
                if (F.okind & 2) xi += (A + sg * B).imag();
              }
              acc[static_cast<size_t>(f)] += F.wi * xr + F.wr * xi;
            }
            if (F.mkind != 2) {
              const cplx m00 = F.mkind == 1 ? cplx{F.m[0], 0} : mat(F.m, 0), m01 = F.mkind == 1 ? cplx{F.m[2], 0} : mat(F.m, 1);
              const cplx m10 = F.mkind == 1 ? cplx{F.m[4], 0} : mat(F.m, 2), m11 = F.mkind == 1 ? cplx{F.m[6], 0} : mat(F.m, 3);
              for (int i = 0; i < NE; ++i) {
                if ((i >> k) & 1) continue;
                for (cplx* X : {E, P}) {
                  const cplx a0 = X[i], a1 = X[i | (1 << k)];
                  X[i] = m00 * a0 + m01 * a1;
                  X[i | (1 << k)] = m10 * a0 + m11 * a1;
                }
              }
            }
          }
          for (int i = 0; i < NE; ++i) {
            const uint32_t s = slot_at(p, tid, i);
            tl[s] = E[i];
            tp[s] = P[i];
            owner[s] = tid >> 5;
          }
        }
      }
      // The store reads the load layout (phase 0's).
      for (int tid = 0; tid < NT; ++tid)
        for (int it = 0; it < NE; ++it) {
          const uint32_t s = slot_of(uint32_t(tid) | (uint32_t(it) << 8));
          if (owner[s] != (tid >> 5) && !S.block_sync[g.nphases - 1]) fail("the store reads a slot another warp wrote behind a warp barrier", seed);
          uint64_t ph = bases[static_cast<size_t>(tid)];
          for (int b = 0; b < RB; ++b) if ((it >> b) & 1) ph |= 1ull << g.tile_phys[8 + b];
          lam[ph] = tl[s];
          psi[ph] = tp[s];
        }
    }
    for (int f = 0; f < g.nflips; ++f)
      if (S.flip[f].out_slot >= 0) ov[static_cast<size_t>(S.flip[f].out_slot)] = acc[static_cast<size_t>(f)];
    if (D.active && D.nz > 0) {
      // The kernel's block reduction: total, thread bits from thread totals, register bits, then warps' sums.
      double total = 0;
      for (int t = 0; t < NT; ++t) total += zt[static_cast<size_t>(t)];
      for (int k = 0; k < D.nz; ++k) {
        const int q = D.z[k].bit;
        double o = 0;
        int col = -1;
        for (int b = 0; b < KT; ++b) if (g.tile_phys[b] == q) col = b;
        if (col >= 0 && col < 8) {
          for (int t = 0; t < NT; ++t) if ((t >> col) & 1) o += zt[static_cast<size_t>(t)];
        } else if (col >= 8) {
          const std::vector<double>& zr = col == 8 ? zr0 : col == 9 ? zr1 : zr2;
          for (int t = 0; t < NT; ++t) o += zr[static_cast<size_t>(t)];
        } else {
          for (int w = 0; w < 8; ++w) o += zh[static_cast<size_t>(q) * 8 + static_cast<size_t>(w)];
        }
        ov[static_cast<size_t>(D.z[k].out_slot)] = D.z[k].wr * (total - 2.0 * o);
      }
    }
  }
}

cplx random_unit(std::mt19937_64& rng)
{
  std::uniform_real_distribution<double> u(0.0, 6.283185307179586);
  return std::polar(1.0, u(rng));
}

}  // namespace

int main(int argc, char** argv)
{
  const int rounds = argc > 1 ? std::atoi(argv[1]) : 60;
  int launches = 0, owed_runs = 0, multi = 0;
  for (int seed = 0; seed < rounds; ++seed) {
    std::mt19937_64 rng(static_cast<uint64_t>(seed) * 7919u + 17u);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    const int n = 11 + static_cast<int>(rng() % 4);
    const size_t N = size_t(1) << n;
    std::vector<cplx> psi(N), lam(N);
    for (size_t i = 0; i < N; ++i) { psi[i] = {U(rng), U(rng)}; lam[i] = {U(rng), U(rng)}; }
    // A run: distinct bits, random matrices (real for some), overlaps for some.
    std::vector<int> bits(static_cast<size_t>(n));
    for (int b = 0; b < n; ++b) bits[static_cast<size_t>(b)] = b;
    std::shuffle(bits.begin(), bits.end(), rng);
    const int count = 1 + static_cast<int>(rng() % static_cast<uint64_t>(n));
    std::vector<rotate_item> items;
    int slots = 0;
    for (int k = 0; k < count; ++k) {
      rotate_item it{};
      it.bit = bits[static_cast<size_t>(k)];
      const double th = U(rng) * 3.0;
      if (rng() % 2) {  // real rotation [[c, s], [-s, c]]
        it.m[0] = std::cos(th); it.m[2] = std::sin(th); it.m[4] = -std::sin(th); it.m[6] = std::cos(th);
      } else {  // a general unitary: phases around a rotation
        const cplx a = random_unit(rng), b = random_unit(rng), c = random_unit(rng);
        const cplx m[4] = {a * std::cos(th), b * std::sin(th), -std::conj(b) * c * std::sin(th), std::conj(a) * c * std::cos(th)};
        for (int e = 0; e < 4; ++e) { it.m[2 * e] = m[e].real(); it.m[2 * e + 1] = m[e].imag(); }
      }
      it.slot = -1;
      it.spec = overlap_spec{0, 0, 1.0, 0.0};
      const int kind = static_cast<int>(rng() % 3);  // 0 none, 1 X type, 2 Y type
      if (kind) {
        it.slot = slots++;
        it.spec.flip = 1ull << it.bit;
        if (kind == 2) { it.spec.sign = 1ull << it.bit; it.spec.wr = 0.0; it.spec.wi = -1.0; }
      }
      items.push_back(it);
    }
    // An owed diagonal on half of the runs, with Z-type overlaps.
    pre_diag owed{};
    const bool with_owed = rng() % 2;
    std::vector<cplx> dfac(N, cplx{1.0, 0.0});
    std::vector<int> zbits;
    if (with_owed) {
      const cplx g0 = random_unit(rng);
      owed.g[0] = g0.real();
      owed.g[1] = g0.imag();
      for (int b = 0; b < kMaxQubits; ++b) { owed.u[b][0] = 1.0; owed.u[b][1] = 0.0; }
      for (int b = 0; b < n; ++b)
        if (rng() % 2) {
          const cplx u = (rng() % 4 == 0) ? cplx{-1.0, 0.0} : random_unit(rng);
          owed.u[b][0] = u.real();
          owed.u[b][1] = u.imag();
        }
      for (int e = 0; e < n; ++e) {  // a ring of controlled Zs and a few random pairs
        int a = e, b = (e + 1) % n;
        if (rng() % 3 == 0) b = static_cast<int>(rng() % static_cast<uint64_t>(n));
        if (a == b) continue;
        owed.adj[std::min(a, b)] ^= 1ull << std::max(a, b);
        owed.full[a] ^= 1ull << b;
        owed.full[b] ^= 1ull << a;
      }
      const int nz = static_cast<int>(rng() % static_cast<uint64_t>(n + 1));
      for (int k = 0; k < nz; ++k) {
        owed.z[k].bit = static_cast<int>(rng() % static_cast<uint64_t>(n));
        owed.z[k].out_slot = slots++;
        owed.z[k].wr = 1.0;
        zbits.push_back(owed.z[k].bit);
      }
      owed.nz = nz;
      for (size_t j = 0; j < N; ++j) {
        cplx f = g0;
        int par = 0;
        for (int b = 0; b < n; ++b)
          if ((j >> b) & 1) {
            f *= cplx{owed.u[b][0], owed.u[b][1]};
            par ^= parity(j & owed.adj[b]);
          }
        dfac[j] = par ? -f : f;
      }
      ++owed_runs;
    }
    const std::vector<pair_rotate_set> sets = plan_rotations(n, items, with_owed ? &owed : nullptr);
    launches += static_cast<int>(sets.size());
    multi += sets.size() > 1;
    // Reference: the owed diagonal, then the overlaps (the gates commute), then the gates.
    std::vector<cplx> rpsi(psi), rlam(lam);
    std::vector<double> ref(static_cast<size_t>(slots), 0.0);
    for (size_t k = 0; k < zbits.size(); ++k) {
      double s = 0;
      for (size_t j = 0; j < N; ++j) s += (((j >> zbits[k]) & 1) ? -1.0 : 1.0) * (std::conj(lam[j]) * psi[j]).imag();
      ref[static_cast<size_t>(owed.z[k].out_slot)] = s;
    }
    for (size_t j = 0; j < N; ++j) { rpsi[j] *= dfac[j]; rlam[j] *= dfac[j]; }
    for (const rotate_item& it : items) {
      if (it.slot < 0) continue;
      cplx o = 0;
      for (size_t j = 0; j < N; ++j)
        o += std::conj(rlam[j]) * (parity(j & it.spec.sign) ? -1.0 : 1.0) * rpsi[j ^ it.spec.flip];
      ref[static_cast<size_t>(it.slot)] = (cplx{it.spec.wr, it.spec.wi} * o).imag();
    }
    for (const rotate_item& it : items) {
      const uint64_t t = 1ull << it.bit;
      for (size_t j = 0; j < N; ++j) {
        if (j & t) continue;
        for (std::vector<cplx>* X : {&rpsi, &rlam}) {
          const cplx a0 = (*X)[j], a1 = (*X)[j | t];
          (*X)[j] = mat(it.m, 0) * a0 + mat(it.m, 1) * a1;
          (*X)[j | t] = mat(it.m, 2) * a0 + mat(it.m, 3) * a1;
        }
      }
    }
    std::vector<double> ov(static_cast<size_t>(slots), 0.0);
    run_model(n, sets, lam, psi, ov, seed);
    double err = 0, oerr = 0;
    for (size_t j = 0; j < N; ++j) err = std::max({err, std::abs(psi[j] - rpsi[j]), std::abs(lam[j] - rlam[j])});
    for (int k = 0; k < slots; ++k) oerr = std::max(oerr, std::abs(ov[static_cast<size_t>(k)] - ref[static_cast<size_t>(k)]));
    if (!(err <= 1e-12)) fail("states differ from the gates applied directly", seed);
    if (!(oerr <= 1e-9)) fail("overlaps or Z sums differ", seed);
    if (seed < 3 || !(err <= 1e-12 && oerr <= 1e-9))
      std::printf("seed=%d n=%d gates=%d owed=%d z=%zu launches=%zu err=%.3e overlap err=%.3e\n", seed, n, count,
                  with_owed ? 1 : 0, zbits.size(), sets.size(), err, oerr);
  }
  std::printf("launches planned: %d (runs with an owed diagonal: %d, runs in more than one launch: %d)\n", launches,
              owed_runs, multi);
  if (owed_runs == 0 || multi == 0) fail("the random runs did not cover owed diagonals and multi-launch runs", -1);
  if (failures == 0) std::printf("ALL OK\n");
  return failures == 0 ? 0 : 1;
}
