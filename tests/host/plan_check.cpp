// plan_check.cpp -- CPU check of the host-side fusion planner (no GPU).
//
// Plans random gate queues with rbk::plan_passes / rbk::plan_canonicalize and
// executes the resulting pass programs with a plain C++ model of what
// tile_pass_kernel does with a dev_pass (load the tile, per phase gather the
// registers, apply the ops with their register / thread / outside-tile
// predicates, scatter back with the write positions, store).  The result,
// read back through the final layout map, must equal the gates applied one by
// one in logical order.  Test code only; built and run by tests/test_planner.py.
#include <algorithm>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <set>
#include <vector>

#include "rbk_internal.h"
#include "rbk_plan.h"

using cplx = std::complex<double>;
using namespace rbk;

static void apply_direct(std::vector<cplx>& a, const hgate& g)
{
  const uint64_t N = a.size();
  if (g.kind == HK_SWAP) {
    const uint64_t m1 = 1ull << g.target, m2 = 1ull << g.target2;
    for (uint64_t i = 0; i < N; ++i)
      if ((i & m1) && !(i & m2)) std::swap(a[i], a[(i & ~m1) | m2]);
    return;
  }
  const cplx m00{g.m[0], g.m[1]}, m01{g.m[2], g.m[3]}, m10{g.m[4], g.m[5]}, m11{g.m[6], g.m[7]};
  for (uint64_t i = 0; i < N; ++i) {
    if ((i & g.cmask) != g.cmask) continue;
    if (g.kind == OPK_NEG) { a[i] = -a[i]; continue; }
    const uint64_t tm = 1ull << g.target;
    if (g.kind == OPK_DIAG) { a[i] *= (i & tm) ? m01 : m00; continue; }
    if (i & tm) continue;
    const cplx a0 = a[i], a1 = a[i | tm];
    if (g.kind == OPK_X) { a[i] = a1; a[i | tm] = a0; }
    else if (g.kind == OPK_Y) { a[i] = cplx{0, -1} * a1; a[i | tm] = cplx{0, 1} * a0; }
    else { a[i] = m00 * a0 + m01 * a1; a[i | tm] = m10 * a0 + m11 * a1; }
  }
}

static uint32_t slot_of(uint32_t j, int vbits)
{
  uint32_t u = j >> vbits;
  const uint32_t f = (u >> 3) ^ (u >> 6) ^ (u >> 9) ^ (u >> 12);
  u ^= f & 7u;
  return (u << vbits) | (j & ((1u << vbits) - 1));
}

// The kernel's apply_folds: folded CNOTs that hold on this tile move write positions.
static void apply_folds(const dev_phase& D, uint64_t base, int tid, int R, uint64_t& thr, uint64_t* reg)
{
  if (D.num_folds > kMaxFolds) { std::fprintf(stderr, "too many folds\n"); std::exit(11); }
  for (int f = 0; f < D.num_folds; ++f) {
    const dev_fold& F = D.folds[f];
    if ((base & F.cout) != F.cout) continue;
    if (F.kind == 0) thr ^= F.x;
    else if (F.kind == 2) { if ((tid >> F.bit) & 1) thr ^= F.x; }
    else if (F.bit < R) reg[F.bit] ^= F.x;
    else { std::fprintf(stderr, "bad fold register\n"); std::exit(13); }
  }
}

// Model of tile_pass_kernel for one pass: shared memory is indexed by slot and
// every address comes from the precomputed tables, as in the kernel.  Each
// phase completes all threads' reads before any write, which is what the
// kernel's barriers guarantee (including the one before the direct store of a
// one-phase pass that also loaded straight from HBM).
// Direct HBM layouts.  Mode 1 moves 16-byte vectors: complex<float> must have
// the pair bit (physical bit 0) on register bit 0 and nowhere else, and the five
// lanes on the next physical bits (one 512-byte run per warp).  Mode 2
// (complex<float> only) moves 8-byte amplitudes with the lanes on physical bits
// 0-4.  Lane l is thread bit l: its contribution is tphys_lo[1 << l] ^
// tphys_lo[0] (l < 4), tphys_hi[1] ^ tphys_hi[0] (l = 4).
static void check_direct_layout(const plan_params& p, const dev_hbm_layout& L, int mode)
{
  if (mode != 1 && !(mode == 2 && p.vbits)) { std::fprintf(stderr, "bad direct mode\n"); std::exit(19); }
  bool ok = true;
  if (p.vbits && mode == 1) {
    ok = L.rphys[0] == 1;
    for (int b = 1; b < p.R; ++b) ok = ok && !(L.rphys[b] & 1);
    for (int x = 0; x < 16; ++x) ok = ok && !((L.tphys_lo[x] ^ L.tphys_lo[0]) & 1);
    for (int x = 0; x < 32; ++x) ok = ok && !((L.tphys_hi[x] ^ L.tphys_hi[0]) & 1);
    if (!ok) { std::fprintf(stderr, "direct layout splits a 16-byte pair\n"); std::exit(10); }
  }
  const int lane0 = mode == 1 ? p.vbits : 0;
  uint64_t lanes = 0;
  for (int l = 0; l < 4; ++l) lanes |= L.tphys_lo[1 << l] ^ L.tphys_lo[0];
  lanes |= L.tphys_hi[1] ^ L.tphys_hi[0];
  if (lanes != (31ull << lane0)) { std::fprintf(stderr, "direct layout lanes are not one contiguous run\n"); std::exit(20); }
}

static void run_pass(std::vector<cplx>& st, const plan_params& p, const dev_pass& P)
{
  if (P.direct_load) check_direct_layout(p, P.load, P.direct_load);
  if (P.direct_store) check_direct_layout(p, P.store, P.direct_store);
  const int K = p.K, R = p.R, T = K - R, NR = 1 << R, NT = 1 << T;
  const uint64_t blocks = 1ull << (p.n - K);
  std::vector<cplx> smem(1u << K);
  std::vector<cplx> regs(size_t(NT) * NR);
  for (uint64_t b = 0; b < blocks; ++b) {
    uint64_t base = 0;
    for (int r = 0; r < P.num_runs; ++r)
      base |= ((b >> P.run_src[r]) & ((1ull << P.run_len[r]) - 1)) << P.run_dst[r];
    auto phys_of = [&](uint32_t j) {
      uint64_t ph = base;
      for (int t = 0; t < K; ++t) if ((j >> t) & 1) ph |= 1ull << P.tile_phys[t];
      return ph;
    };
    std::set<uint64_t> touched, stored;  // direct HBM accesses of this tile
    auto in_state = [&](uint64_t phys) {
      if (phys >= st.size()) { std::fprintf(stderr, "HBM access out of range\n"); std::exit(9); }
      return phys;
    };
    if (!P.direct_load)
      for (uint32_t j = 0; j < (1u << K); ++j) smem[slot_of(j, p.vbits)] = st[in_state(phys_of(j))];
    for (int ph = 0; ph < P.num_phases; ++ph) {
      const dev_phase& D = P.phases[ph];
      for (int tid = 0; tid < NT; ++tid) {
        cplx* a = &regs[size_t(tid) * NR];
        if (ph == 0 && P.direct_load) {
          const uint64_t tp = base | P.load.tphys_lo[tid & 15] | P.load.tphys_hi[tid >> 4];
          for (int i = 0; i < NR; ++i) {
            uint64_t phys = tp;
            for (int x = 0; x < R; ++x) if (i & (1 << x)) phys |= P.load.rphys[x];
            if (!touched.insert(phys).second) { std::fprintf(stderr, "direct load reads an amplitude twice\n"); std::exit(4); }
            a[i] = st[in_state(phys)];
          }
        } else {
          const uint32_t ts = D.tslot_lo[tid & 15] ^ D.tslot_hi[tid >> 4];
          for (int i = 0; i < NR; ++i) {
            uint32_t sidx = ts;
            for (int x = 0; x < R; ++x) if (i & (1 << x)) sidx ^= D.rslot[x];
            if (sidx >= (1u << K)) { std::fprintf(stderr, "bad read position\n"); std::exit(3); }
            a[i] = smem[sidx];
          }
        }
        for (int o = D.op_begin; o < D.op_end; ++o) {
          const dev_op& op = P.ops[o];
          const uint32_t want_code = op.kind == OPK_MAT ? op_code(OPK_MAT, op.real, op.creg != 0, op.treg)
                                   : (op.kind == OPK_X || op.kind == OPK_Y) ? op_code(op.kind, 0, true, op.treg)
                                   : op.kind == OPK_LAYER ? op_code(OPK_LAYER, op.real, op.dreg == (1u << R) - 1, 0)
                                   : op_code(op.kind, 0, true, 0);
          if (op.code != want_code || op.code >= kNumOpCodes || op.treg >= R) { std::fprintf(stderr, "bad dispatch code\n"); std::exit(8); }
          if (op.kind == OPK_PHASES) {  // a run header: the run's gates follow, each a factor on the amplitudes whose bits are all one
            if (op.run < 1 || o + static_cast<int>(op.run) >= D.op_end) { std::fprintf(stderr, "bad phase run\n"); std::exit(14); }
            // class sizes (no register bit, register bit 0 .. R-1; the rest: two or more register bits)
            int bound[9], sum = 0;
            for (int c = 0; c <= R; ++c) { sum += static_cast<int>((op.dout >> (8 * c)) & 0xff); bound[c] = sum; }
            if (sum > static_cast<int>(op.run) || (op.dout >> (8 * (R + 1))) != 0) { std::fprintf(stderr, "bad phase run classes\n"); std::exit(18); }
            for (int k = 1; k <= static_cast<int>(op.run); ++k) {
              const dev_op& g = P.ops[o + k];
              int c = 0;
              while (c <= R && k - 1 >= bound[c]) ++c;  // the class member k - 1 belongs to
              const int nr = __builtin_popcount(g.creg);
              const bool ok_class = c == 0 ? nr == 0 : c <= R ? g.creg == (1u << (c - 1)) : nr >= 2;
              if (g.kind != OPK_DIAG || g.dreg || g.dthr || g.dout || g.creg >= (1u << R) || !ok_class) {
                std::fprintf(stderr, "phase run holds a gate out of its form or class\n");
                std::exit(15);
              }
              if ((uint32_t(tid) & g.cthr) != g.cthr || (base & g.cout) != g.cout) continue;
              const cplx d{g.m[2], g.m[3]};
              for (int i = 0; i < NR; ++i)
                if ((uint32_t(i) & g.creg) == g.creg) a[i] *= d;
            }
            o += static_cast<int>(op.run);
            continue;
          }
          if (op.kind == OPK_LAYER) {  // a layer header: one uncontrolled 2x2 gate per bit of dreg follows, in bit order
            if (op.run < 2 || o + static_cast<int>(op.run) >= D.op_end || op.real > kLayerFactored || op.dreg >= (1u << R) ||
                __builtin_popcount(op.dreg) != static_cast<int>(op.run) || op.creg || op.cthr || op.cout) {
              std::fprintf(stderr, "bad layer header\n");
              std::exit(16);
            }
            uint32_t bits = op.dreg;
            for (int k = 1; k <= static_cast<int>(op.run); ++k) {
              const dev_op& g = P.ops[o + k];
              const int want = __builtin_ctz(bits);
              bits &= bits - 1;
              // the layer's form must compute each matrix exactly: real only with real,
              // general with general or m00-real; factored members carry t0, t1 only
              const bool form_ok = op.real == kLayerFactored ? (g.m[2] == 0.0 && g.m[7] == 0.0)
                                 : op.real == g.real || (op.real == 0 && g.real == 2);
              if (g.kind != OPK_MAT || g.creg || g.cthr || g.cout || g.treg != want || !form_ok) {
                std::fprintf(stderr, "layer holds a gate it cannot run\n");
                std::exit(17);
              }
            }
            if (op.real == kLayerFactored) {
              // pre factors, each member's middle factor [[1, t0], [t1, 1]], post factors; the
              // slot holds pre_lo[4], pre_hi[H], post_lo[4], post_hi[H], H = 2^(R-2)
              if (op.dthr >= static_cast<uint32_t>(kMaxLayerTabs)) { std::fprintf(stderr, "bad layer table\n"); std::exit(19); }
              const int H = NR / 4;
              auto entry = [&](int i) {
                const double* t = P.tabs + op.dthr * kTabDoubles;
                if (p.vbits == 0) return cplx{t[2 * i], t[2 * i + 1]};
                const float* f = reinterpret_cast<const float*>(t);
                return cplx{f[2 * i], f[2 * i + 1]};
              };
              if (entry(0) != cplx{1.0, 0.0} || entry(4) != cplx{1.0, 0.0} || entry(8 + H) != cplx{1.0, 0.0}) {
                std::fprintf(stderr, "a layer factor that the kernel skips is not 1 (%.17g %.17g / %.17g %.17g / %.17g %.17g)\n",
                             entry(0).real(), entry(0).imag(), entry(4).real(), entry(4).imag(), entry(8 + H).real(), entry(8 + H).imag());
                std::exit(19);
              }
              if (op.diag_one)
                for (int i = 0; i < NR; ++i) a[i] *= entry(i & 3) * entry(4 + (i >> 2));
              for (int k = 1; k <= static_cast<int>(op.run); ++k) {
                const dev_op& g = P.ops[o + k];
                const int tb = 1 << g.treg;
                for (int i = 0; i < NR; ++i) {
                  if (i & tb) continue;
                  const cplx a0 = a[i], a1 = a[i | tb];
                  a[i] = a0 + g.m[0] * a1;
                  a[i | tb] = g.m[1] * a0 + a1;
                }
              }
              for (int i = 0; i < NR; ++i) a[i] *= entry(4 + H + (i & 3)) * entry(8 + H + (i >> 2));
              o += static_cast<int>(op.run);
            }
            continue;
          }
          if ((uint32_t(tid) & op.cthr) != op.cthr || (base & op.cout) != op.cout) continue;
          const cplx m00{op.m[0], op.m[1]}, m01{op.m[2], op.m[3]}, m10{op.m[4], op.m[5]}, m11{op.m[6], op.m[7]};
          for (int i = 0; i < NR; ++i) {
            if ((uint32_t(i) & op.creg) != op.creg) continue;
            if (op.kind == OPK_NEG) { a[i] = -a[i]; continue; }
            if (op.kind == OPK_DIAG) {
              const bool bit = (uint32_t(tid) & op.dthr) || (base & op.dout) || (uint32_t(i) & op.dreg);
              if (bit) a[i] *= m01; else if (!op.diag_one) a[i] *= m00;
              continue;
            }
            const int tb = 1 << op.treg;
            if (i & tb) continue;
            const cplx a0 = a[i], a1 = a[i | tb];
            if (op.kind == OPK_X) { a[i] = a1; a[i | tb] = a0; }
            else if (op.kind == OPK_Y) { a[i] = cplx{0, -1} * a1; a[i | tb] = cplx{0, 1} * a0; }
            else { a[i] = m00 * a0 + m01 * a1; a[i | tb] = m10 * a0 + m11 * a1; }
          }
        }
      }
      const bool last = ph + 1 == P.num_phases;
      std::vector<char> written(1u << K, 0);
      for (int tid = 0; tid < NT; ++tid) {
        const cplx* a = &regs[size_t(tid) * NR];
        if (last && P.direct_store) {
          uint64_t tp = base ^ P.store.tphys_lo[tid & 15] ^ P.store.tphys_hi[tid >> 4];
          uint64_t rp[8];
          for (int x = 0; x < R; ++x) rp[x] = P.store.rphys[x];
          apply_folds(D, base, tid, R, tp, rp);
          for (int i = 0; i < NR; ++i) {
            uint64_t phys = tp;
            for (int x = 0; x < R; ++x) if (i & (1 << x)) phys ^= rp[x];
            if (!stored.insert(phys).second) { std::fprintf(stderr, "direct store writes an amplitude twice\n"); std::exit(5); }
            st[in_state(phys)] = a[i];
          }
          continue;
        }
        uint64_t ts = D.wtslot_lo[tid & 15] ^ D.wtslot_hi[tid >> 4];
        uint64_t rs[8];
        for (int x = 0; x < R; ++x) rs[x] = D.wslot[x];
        apply_folds(D, base, tid, R, ts, rs);
        for (int i = 0; i < NR; ++i) {
          uint32_t sidx = static_cast<uint32_t>(ts);
          for (int x = 0; x < R; ++x) if (i & (1 << x)) sidx ^= static_cast<uint32_t>(rs[x]);
          if (sidx >= (1u << K) || written[sidx]) { std::fprintf(stderr, "bad write position\n"); std::exit(3); }
          written[sidx] = 1;
          smem[sidx] = a[i];
        }
      }
    }
    if (!P.direct_store)
      for (uint32_t j = 0; j < (1u << K); ++j) st[in_state(phys_of(j))] = smem[slot_of(j, p.vbits)];
    if ((P.direct_load && touched.size() != (1u << K)) || (P.direct_store && stored.size() != (1u << K))) {
      std::fprintf(stderr, "direct HBM access does not cover the tile\n");
      std::exit(6);
    }
    for (uint64_t ph : stored) if ((ph & ~((1ull << p.n) - 1)) != 0) { std::fprintf(stderr, "store out of range\n"); std::exit(7); }
  }
}

// A random U3(theta, phi, lambda) = [[c, -e^{i lambda} s], [e^{i phi} s, e^{i (phi + lambda)} c]]
// (c = cos theta/2, s = sin theta/2): unitary, so layers of them take the factored form.
static void unitary_u3(std::mt19937_64& rng, double* m)
{
  std::uniform_real_distribution<double> ang(0.0, 6.283185307179586);
  const double th = ang(rng), ph = ang(rng), la = ang(rng);
  const cplx c{std::cos(th / 2), 0.0}, s{std::sin(th / 2), 0.0};
  const cplx v[4] = {c, -std::polar(1.0, la) * s, std::polar(1.0, ph) * s, std::polar(1.0, ph + la) * c};
  for (int i = 0; i < 4; ++i) { m[2 * i] = v[i].real(); m[2 * i + 1] = v[i].imag(); }
}

// A brick: U3 on every qubit, then CNOTs on alternate neighbour pairs, `depth` times.
static std::vector<hgate> brick_gates(std::mt19937_64& rng, int n, int depth)
{
  std::vector<hgate> out;
  for (int l = 0; l < depth; ++l) {
    for (int q = 0; q < n; ++q) {
      hgate g{};
      g.kind = OPK_MAT;
      g.target = static_cast<int8_t>(q);
      g.target2 = -1;
      unitary_u3(rng, g.m);
      out.push_back(g);
    }
    for (int q = l % 2; q + 1 < n; q += 2) {
      hgate g{};
      g.kind = OPK_X;
      g.target = static_cast<int8_t>(q + 1);
      g.target2 = -1;
      g.cmask = 1ull << q;
      out.push_back(g);
    }
  }
  return out;
}

// The adjoint ansatz: EY (real rotation) and EZ (diagonal) on every qubit, then a CZ ring.
static std::vector<hgate> ansatz_gates(std::mt19937_64& rng, int n, int depth)
{
  std::uniform_real_distribution<double> ang(-3.0, 3.0);
  std::vector<hgate> out;
  for (int l = 0; l < depth; ++l) {
    for (int q = 0; q < n; ++q) {
      hgate g{};
      g.kind = OPK_MAT;
      g.target = static_cast<int8_t>(q);
      g.target2 = -1;
      const double t = ang(rng);
      g.m[0] = std::cos(t); g.m[2] = std::sin(t); g.m[4] = -std::sin(t); g.m[6] = std::cos(t);
      out.push_back(g);
    }
    for (int q = 0; q < n; ++q) {
      hgate g{};
      g.kind = OPK_DIAG;
      g.target = static_cast<int8_t>(q);
      g.target2 = -1;
      const double t = ang(rng);
      g.m[0] = std::cos(t); g.m[1] = std::sin(t); g.m[2] = std::cos(t); g.m[3] = -std::sin(t);
      out.push_back(g);
    }
    for (int q = 0; q < n; ++q) {
      hgate g{};
      g.kind = OPK_NEG;
      g.target = -1;
      g.target2 = -1;
      g.cmask = (1ull << q) | (1ull << ((q + 1) % n));
      out.push_back(g);
    }
  }
  return out;
}

// phase_heavy: mostly diagonal gates and sign flips between dense ones, so
// that register phases hold many short runs of phase gates.
static hgate random_gate(std::mt19937_64& rng, int n, bool phase_heavy = false)
{
  hgate g{};
  g.target2 = -1;
  std::uniform_int_distribution<int> kind(0, 9), q(0, n - 1), nc(0, 2);
  std::uniform_real_distribution<double> u(-1, 1);
  int k = kind(rng);
  if (phase_heavy) k = (k < 2) ? 0 : (k < 4) ? 4 : (k < 7) ? 6 : 7;  // MAT, X, DIAG, NEG
  g.target = static_cast<int8_t>(q(rng));
  const int ncontrols = nc(rng) == 2 ? 1 + (rng() % 2) : 0;
  for (int c = 0; c < ncontrols; ++c) {
    const int cq = q(rng);
    if (cq != g.target) g.cmask |= 1ull << cq;
  }
  for (double& x : g.m) x = u(rng);
  if (k == 3) unitary_u3(rng, g.m);
  if (k <= 3) g.kind = OPK_MAT;
  else if (k == 4) g.kind = OPK_X;
  else if (k == 5) g.kind = OPK_Y;
  else if (k == 6) { g.kind = OPK_DIAG; g.diag_one = rng() % 2; if (g.diag_one) { g.m[0] = 1; g.m[1] = 0; } }
  else if (k == 7) { g.kind = OPK_NEG; g.cmask |= 1ull << g.target; g.target = -1; }
  else {
    g.kind = HK_SWAP;
    g.cmask = 0;
    do g.target2 = static_cast<int8_t>(q(rng)); while (g.target2 == g.target);
  }
  return g;
}

int main(int argc, char** argv)
{
  const int seeds = argc > 1 ? std::atoi(argv[1]) : 20;
  int failures = 0, factored_layers = 0;
  for (int prec = 0; prec < 2; ++prec)
  for (int shape = 0; shape < kNumShapes; ++shape) {
    plan_params p{};
    shape_bits(prec, shape, &p.K, &p.R);
    p.vbits = prec;
    for (int seed = 0; seed < seeds; ++seed) {
      std::mt19937_64 rng(1000 * prec + 100 * shape + seed);
      // the precision's coalescing run (512 bytes), or 128-byte runs on every fourth seed
      p.LOW = (seed % 4 == 3) ? 3 : (prec == 0 ? 5 : 6);
      p.n = p.K + static_cast<int>(rng() % 4);
      p.dense_budget = 1 + static_cast<int>(rng() % 16);
      const uint64_t N = 1ull << p.n;
      std::vector<cplx> init(N);
      std::normal_distribution<double> nd;
      for (auto& x : init) x = cplx{nd(rng), nd(rng)};
      std::vector<hgate> gates;
      const int count = 50 + static_cast<int>(rng() % 300);
      const bool phase_heavy = seed % 2 == 1;
      if (seed % 6 == 5) gates = ansatz_gates(rng, p.n, 1 + static_cast<int>(rng() % 4));
      else if (seed % 3 == 2) gates = brick_gates(rng, p.n, 2 + static_cast<int>(rng() % 6));
      else for (int i = 0; i < count; ++i) gates.push_back(random_gate(rng, p.n, phase_heavy));

      std::vector<cplx> want = init;
      for (const auto& g : gates) apply_direct(want, g);

      std::vector<int> perm(p.n), inv(p.n);
      for (int i = 0; i < p.n; ++i) perm[i] = inv[i] = i;
      std::vector<dev_pass> passes;
      plan_passes(p, gates, perm, inv, passes);
      std::vector<cplx> st = init;
      for (const auto& P : passes) run_pass(st, p, P);
      // A detour through a random layout, then home: both are data moves only.
      std::vector<int> target(p.n);
      for (int i = 0; i < p.n; ++i) target[i] = i;
      std::shuffle(target.begin(), target.end(), rng);
      std::vector<dev_pass> detour;
      plan_layout(p, perm, inv, target, detour);
      for (const auto& P : detour) run_pass(st, p, P);
      if (perm != target) { std::printf("layout not reached\n"); ++failures; }
      std::vector<dev_pass> canon;
      plan_canonicalize(p, perm, inv, canon);
      for (const auto& P : canon) run_pass(st, p, P);
      for (int i = 0; i < p.n; ++i) if (perm[i] != i) { std::printf("layout not canonical\n"); ++failures; break; }
      // Random (non-unitary) matrices let amplitudes grow: the error is relative to the largest.
      // complex<float> plans hold the factored layers' tables in float, so 1e-12 there would test
      // the rounding of the tables, not the program; a wrong program is off by O(1) either way.
      double err = 0, scale = 1;
      for (uint64_t i = 0; i < N; ++i) scale = std::max(scale, std::abs(want[i]));
      for (uint64_t i = 0; i < N; ++i) err = std::max(err, std::abs(st[i] - want[i]) / scale);
      std::printf("prec=%d shape=%d seed=%d n=%d gates=%d budget=%d passes=%zu detour=%zu canon=%zu err=%.3e\n", prec, shape, seed,
                  p.n, count, p.dense_budget, passes.size(), detour.size(), canon.size(), err);
      if (!(err < (prec == 0 ? 1e-12 : 1e-5))) ++failures;
      for (const auto& P : passes)
        for (const auto& o : P.ops) factored_layers += o.kind == OPK_LAYER && o.real == kLayerFactored;
    }
  }
  std::printf("factored layers planned: %d\n", factored_layers);
  if (factored_layers == 0) { std::printf("no factored layer was planned\n"); ++failures; }
  std::printf(failures ? "FAILED %d\n" : "ALL OK\n", failures);
  return failures ? 1 : 0;
}
