// rbk_plan.cpp -- host-side fusion planner.
//
// The reference applies each gate as one sweep over the state
// (ket/include/ket/gate/*.hpp) or, inside BEGIN/END FUSION, replays a recorded
// gate list on every 2^k chunk of the fused qubits
// (bra/src/nompi_state.cpp:1285-1357).  Here the whole queue of gates is cut
// into tile passes instead:
//
//  * A pass owns a set of K physical bits (the tile bits).  The low LOW
//    physical bits are always tile bits, so that every tile is made of
//    contiguous 512-byte runs in HBM (coalesced 16-byte accesses).
//  * Walking the queue in order, a gate is taken into the pass when its
//    non-diagonal target fits in the tile and it commutes with every earlier
//    gate that was left behind (on each shared qubit both act diagonally:
//    control, phase or Z-type).  Controls and diagonal qubits need not be
//    tile bits: outside the tile they are a per-tile predicate.
//  * Inside the pass, gates are grouped into register phases: R tile bits are
//    held in each thread's registers, and a gate can run once its target is
//    one of them.  Changing phase costs one shared-memory exchange.
//  * At the end of a pass the tile bits are relabelled: the logical qubits
//    that the queue needs next are written into the low physical bits.  This
//    is the layout map of ket::mpi::qubit_permutation
//    (ket/include/ket/mpi/qubit_permutation.hpp:242-252 `permutate`) with the
//    swap of swap_permutated_local_qubits
//    (ket/include/ket/mpi/utility/detail/swap_permutated_local_qubits.hpp:26-81)
//    folded into a pass that moves the data anyway.
//  * Uncontrolled SWAP gates only change the layout map.
#include "rbk_plan.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <limits>
#include <stdexcept>

namespace rbk {
namespace {

inline uint64_t bit(int q) { return 1ull << q; }
inline int popc(uint64_t v) { return __builtin_popcountll(v); }

uint64_t map_mask(uint64_t logical, const std::vector<int>& perm)
{
  uint64_t r = 0;
  while (logical) {
    const int q = __builtin_ctzll(logical);
    logical &= logical - 1;
    r |= bit(perm[q]);
  }
  return r;
}

// A selected gate in physical bits.
struct pop {
  uint8_t kind;
  uint8_t diag_one;
  int target;       // physical; -1 for NEG
  uint64_t cmask;   // physical
  double m[8];
};

bool is_target_kind(uint8_t k) { return k == OPK_MAT || k == OPK_X || k == OPK_Y; }

// Tracks register phases while gates are added (same greedy as build_pass).
struct phase_tracker {
  int R;
  std::vector<int> cur;  // physical bits held in registers in the current phase
  int phases = 1;

  bool would_fit(int t, int max_phases) const
  {
    if (std::find(cur.begin(), cur.end(), t) != cur.end()) return true;
    if (static_cast<int>(cur.size()) < R) return true;
    return phases + 1 <= max_phases;
  }
  void add(int t)
  {
    if (std::find(cur.begin(), cur.end(), t) != cur.end()) return;
    if (static_cast<int>(cur.size()) < R) { cur.push_back(t); return; }
    cur.assign(1, t);
    ++phases;
  }
};

// Orders the thread bits of a phase so that the lowest lanes fall on tile bits
// that map to distinct shared-memory bank groups (see smem_slot in
// rbk_device.cuh: vector-index bit b contributes to slot bit b mod 3): the
// lanes of one 128-byte wavefront then touch 8 distinct 16-byte bank groups.
// wmap (the last phase of a pass, which writes the tile back relabelled): the
// write puts thread bit b at tile bit wmap[b], so the lanes are chosen to be
// conflict-free for that write too where the thread bits allow it.
void order_thread_bits(std::vector<int>& thr, int vbits, const int* wmap)
{
  std::vector<int> out;
  std::vector<int> rest(thr);
  auto take = [&](int b) {
    out.push_back(b);
    rest.erase(std::find(rest.begin(), rest.end(), b));
  };
  if (vbits == 1 && std::find(rest.begin(), rest.end(), 0) != rest.end()) take(0);
  auto residue = [&](int b) { return b < vbits ? -1 : (b - vbits) % 3; };
  bool done = false;
  if (wmap) {  // three lanes with distinct residues both where they are read and where they are written
    const std::vector<int> cand(rest);
    const size_t m = cand.size();
    for (size_t i = 0; i < m && !done; ++i)
      for (size_t j = i + 1; j < m && !done; ++j)
        for (size_t k = j + 1; k < m && !done; ++k) {
          const int b[3] = {cand[i], cand[j], cand[k]};
          bool rd[3] = {false, false, false}, wr[3] = {false, false, false}, ok = true;
          for (int x : b) {
            const int r = residue(x), w = residue(wmap[x]);
            if (r < 0 || w < 0 || rd[r] || wr[w]) { ok = false; break; }
            rd[r] = wr[w] = true;
          }
          if (ok) {
            for (int x : b) take(x);
            done = true;
          }
        }
  }
  if (!done) {
    bool used[3] = {false, false, false};
    for (int pass = 0; pass < 3; ++pass) {
      for (int b : std::vector<int>(rest)) {
        if (b < vbits) continue;
        const int res = residue(b);
        if (!used[res]) { used[res] = true; take(b); break; }
      }
    }
  }
  std::sort(rest.begin(), rest.end());
  out.insert(out.end(), rest.begin(), rest.end());
  thr = out;
}

// Host copy of smem_slot in rbk_device.cuh (shared-memory slot of tile index j).
uint32_t smem_slot_host(uint32_t j, int vbits)
{
  uint32_t u = j >> vbits;
  const uint32_t f = (u >> 3) ^ (u >> 6) ^ (u >> 9) ^ (u >> 12);
  u ^= f & 7u;
  return (u << vbits) | (j & ((1u << vbits) - 1));
}

// Qubits an op acts on non-diagonally (the target of MAT/X/Y) and diagonally
// (controls, DIAG target, NEG bits), as physical masks.
inline uint64_t n_mask(const pop& o) { return is_target_kind(o.kind) ? bit(o.target) : 0; }
inline uint64_t z_mask(const pop& o) { return o.cmask | (o.kind == OPK_DIAG ? bit(o.target) : 0); }
inline bool conflict(const pop& a, const pop& b)
{
  return (n_mask(a) & (n_mask(b) | z_mask(b))) || (z_mask(a) & n_mask(b));
}

struct phase_build { std::vector<int> reg; std::vector<int> ops; };

// Register phases in program order: a new phase whenever a target misses the
// current register set (the same rule as phase_tracker).
std::vector<phase_build> phases_in_order(const std::vector<pop>& ops, const int* tile_of_phys, int R)
{
  std::vector<phase_build> phases(1);
  for (int i = 0; i < static_cast<int>(ops.size()); ++i) {
    const pop& o = ops[i];
    if (is_target_kind(o.kind)) {
      const int tb = tile_of_phys[o.target];
      auto& cur = phases.back().reg;
      if (std::find(cur.begin(), cur.end(), tb) == cur.end()) {
        if (static_cast<int>(cur.size()) < R) cur.push_back(tb);
        else { phases.emplace_back(); phases.back().reg.push_back(tb); }
      }
    }
    phases.back().ops.push_back(i);
  }
  return phases;
}

// Register phases over the dependency graph of the pass: each phase sweeps
// the ops in order and takes every op whose predecessors are done and whose
// target is (or can still join) the phase's register set.  Gates that commute
// are thereby gathered per register set (a light cone inside the registers).
std::vector<phase_build> phases_by_dag(const std::vector<pop>& ops, const int* tile_of_phys, int R, bool defer_x)
{
  const int m = static_cast<int>(ops.size());
  std::vector<std::vector<int>> preds(m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < j; ++i)
      if (conflict(ops[i], ops[j])) preds[j].push_back(i);
  std::vector<char> done(m, 0);
  int remaining = m;
  std::vector<phase_build> phases;
  while (remaining > 0) {
    phase_build pb;
    // defer_x: the phase first takes every other ready op, then the ready
    // CNOT / X gates, and closes -- so that those end the phase and fold into
    // its write layout (fold_trailing_x); their dependents start the next phase.
    for (int stage = defer_x ? 0 : 1; stage < 2; ++stage) {
    bool progress = true;
    while (progress) {
      progress = false;
      for (int j = 0; j < m; ++j) {
        if (done[j]) continue;
        if (stage == 0 && ops[j].kind == OPK_X) continue;
        if (defer_x && stage == 1 && ops[j].kind != OPK_X) continue;
        bool ready = true;
        for (int i : preds[j]) if (!done[i]) { ready = false; break; }
        if (!ready) continue;
        if (is_target_kind(ops[j].kind)) {
          const int tb = tile_of_phys[ops[j].target];
          if (std::find(pb.reg.begin(), pb.reg.end(), tb) == pb.reg.end()) {
            if (static_cast<int>(pb.reg.size()) >= R) continue;
            pb.reg.push_back(tb);
          }
        }
        done[j] = 1;
        --remaining;
        pb.ops.push_back(j);
        progress = true;
      }
    }
    }
    phases.push_back(pb);  // never empty: a fresh register set takes at least one ready op
  }
  if (phases.empty()) phases.emplace_back();
  return phases;
}

// CNOT / X gates at the end of a phase permute the tile's indices GF(2)-affinely:
// instead of running them, the write-back layout absorbs them.  A gate X_t
// controlled by one bit c (a register bit, a warp-uniform thread bit, or none)
// moves the value of register slot i of thread tid by W(e_t) -- the write
// position of register bit t -- where c holds: register control c adds W(e_t)
// to wslot[c], a thread control adds it to the thread tables' entries with
// that bit, no control adds it to every thread.  Gates that also have controls
// outside the tile hold on some tiles only and go to dp.folds for the kernel.
// A gate folds when no later kept op of the phase touches its target or acts
// non-diagonally on its control, and no later folded gate is controlled by its
// target (so every folded gate reads its control before any fold moved it and
// their contributions add up).  direct_store (the store's mode, 0 when the
// phase writes to shared memory): the phase stores straight to HBM and the
// contributions are physical offsets (store layout); for complex<float> in
// 16-byte vectors (mode 1) the pair (register bit 0) must then stay out of the folds.
void fold_trailing_x(const plan_params& p, dev_pass& out, dev_phase& dp, int& op_end, int direct_store)
{
  const int begin = dp.op_begin, count = op_end - begin;
  std::vector<char> folded(static_cast<size_t>(count), 0);
  uint32_t later_target = 0, later_diag = 0, later_fold_ctl = 0;
  int conditional = 0;
  for (int k = op_end - 1; k >= begin; --k) {
    const dev_op& d = out.ops[k];
    bool ok = d.kind == OPK_X;
    if (ok) {
      const uint32_t t = 1u << d.treg;
      const int nctl = __builtin_popcount(d.creg) + __builtin_popcount(d.cthr);
      // a lane-bit control would split a warp's direct HBM store; shared-memory writes take it
      ok = nctl <= 1 && (d.cthr == 0 || !direct_store || __builtin_ctz(d.cthr) >= 5) &&
           !((later_target | later_diag | later_fold_ctl) & t) && !(later_target & d.creg);
      if (ok && direct_store == 1 && p.vbits) ok = d.treg != 0 && !(d.creg & 1u);
      if (ok && d.cout) ok = conditional < kMaxFolds;
    }
    if (ok) {
      folded[static_cast<size_t>(k - begin)] = 1;
      later_fold_ctl |= d.creg;
      if (d.cout) ++conditional;
      continue;
    }
    if (is_target_kind(d.kind)) later_target |= 1u << d.treg;
    later_diag |= d.creg | d.dreg;
  }
  // Contributions use the unfolded write positions of the target bits.
  uint16_t wslot0[8];
  uint64_t rphys0[8];
  std::memcpy(wslot0, dp.wslot, sizeof(wslot0));
  std::memcpy(rphys0, out.store.rphys, sizeof(rphys0));
  int kept = begin;
  for (int k = begin; k < op_end; ++k) {
    const dev_op d = out.ops[k];
    if (!folded[static_cast<size_t>(k - begin)]) {
      out.ops[kept++] = d;
      continue;
    }
    const uint64_t x = direct_store ? rphys0[d.treg] : wslot0[d.treg];
    const uint8_t kind = d.creg ? 1 : d.cthr ? 2 : 0;
    const uint8_t bitpos = static_cast<uint8_t>(d.creg ? __builtin_ctz(d.creg) : d.cthr ? __builtin_ctz(d.cthr) : 0);
    if (d.cout) {
      dev_fold& f = dp.folds[dp.num_folds++];
      f.cout = d.cout;
      f.x = x;
      f.kind = kind;
      f.bit = bitpos;
      continue;
    }
    // thread bit b: entry e of the low table (tid & 15) when b < 4, of the high table (tid >> 4) otherwise
    if (direct_store) {
      if (kind == 0) for (int e = 0; e < 16; ++e) out.store.tphys_lo[e] ^= x;
      else if (kind == 1) out.store.rphys[bitpos] ^= x;
      else if (bitpos < 4) for (int e = 0; e < 16; ++e) { if ((e >> bitpos) & 1) out.store.tphys_lo[e] ^= x; }
      else for (int e = 0; e < 32; ++e) if ((e >> (bitpos - 4)) & 1) out.store.tphys_hi[e] ^= x;
    } else {
      const uint16_t xs = static_cast<uint16_t>(x);
      if (kind == 0) for (int e = 0; e < 16; ++e) dp.wtslot_lo[e] ^= xs;
      else if (kind == 1) dp.wslot[bitpos] ^= xs;
      else if (bitpos < 4) for (int e = 0; e < 16; ++e) { if ((e >> bitpos) & 1) dp.wtslot_lo[e] ^= xs; }
      else for (int e = 0; e < 32; ++e) if ((e >> (bitpos - 4)) & 1) dp.wtslot_hi[e] ^= xs;
    }
  }
  for (int k = kept; k < op_end; ++k) out.ops[k] = dev_op{};
  op_end = kept;
}

// Runs of phase gates -- DIAG with d0 == 1 exactly, NEG: a factor on the
// amplitudes whose bits of the gate are all one -- go to the kernel behind one
// PHASES header: it multiplies each gate's factor into a per-thread
// accumulator (the whole thread's, or that of one register bit) and applies
// the products once, instead of running every gate over the registers.
// The members are rewritten in the run's own form: all the gate's bits in
// creg / cthr / cout (controls and target alike), the factor in (m[2], m[3]).
// They are sorted by accumulator -- no register bit, register bit 0, ..., R-1,
// then two or more register bits (gates that multiply amplitudes directly) --
// and the header's dout holds the class sizes, one byte each in that order
// (the last class takes the rest of `run`).  The gates of a run commute, so
// their order is free.
// A diagonal gate diag(d0, d1) with d0 != 1 (EZ: d0 = e^{i theta}) joins a run
// as two members: d0 on its controls alone (an empty condition: every
// amplitude) and d1 / d0 on its controls and target.  Members with the same
// condition are then multiplied into one, and members whose factor is exactly
// 1 dropped.  (A per-member sign parity for the factor -1, two multiply chains
// and branch-free selects in the kernel's run loop were measured too: the
// adjoint sweep gained nothing from them and the QFT workload lost 6-9 %.)
bool is_phase_op(const dev_op& d, bool general)
{
  if (d.kind == OPK_NEG || (d.kind == OPK_DIAG && d.diag_one && d.m[0] == 1.0 && d.m[1] == 0.0)) return true;
  return general && d.kind == OPK_DIAG && (d.m[0] != 0.0 || d.m[1] != 0.0);
}

// The members of a run of phase ops list[i..j) (see is_phase_op).
std::vector<dev_op> phase_members(const std::vector<dev_op>& list, size_t i, size_t j)
{
  using cd = std::complex<double>;
  std::vector<dev_op> members;
  auto add = [&](dev_op g, cd f) {
    for (dev_op& m : members)
      if (m.creg == g.creg && m.cthr == g.cthr && m.cout == g.cout) {
        const cd v = cd{m.m[2], m.m[3]} * f;
        m.m[2] = v.real();
        m.m[3] = v.imag();
        return;
      }
    g.m[2] = f.real();
    g.m[3] = f.imag();
    members.push_back(g);
  };
  for (size_t k = i; k < j; ++k) {
    dev_op g = list[k];
    const dev_op orig = g;
    g.kind = OPK_DIAG;
    g.diag_one = 1;
    g.m[0] = 1.0;
    g.m[1] = 0.0;
    g.m[4] = g.m[5] = g.m[6] = g.m[7] = 0.0;
    if (orig.kind == OPK_NEG) {
      add(g, cd{-1.0, 0.0});
      continue;
    }
    const cd d0{orig.m[0], orig.m[1]}, d1{orig.m[2], orig.m[3]};
    if (!orig.diag_one || d0 != cd{1.0, 0.0}) {  // d0 on the controls alone
      dev_op c = g;
      c.dreg = c.dthr = 0;
      c.dout = 0;
      add(c, d0);
    }
    g.creg |= g.dreg;
    g.cthr |= g.dthr;
    g.cout |= g.dout;
    g.dreg = g.dthr = 0;
    g.dout = 0;
    add(g, (!orig.diag_one || d0 != cd{1.0, 0.0}) ? d1 / d0 : d1);
  }
  std::vector<dev_op> kept;
  for (const dev_op& m : members)
    if (!(m.m[2] == 1.0 && m.m[3] == 0.0)) kept.push_back(m);
  return kept;
}

// headers_left: headers the pass may still add (kMaxPassOps - kMaxPassGates in
// all), so that the gates of later phases still fit in the op records.
void group_phase_runs(const plan_params& p, dev_pass& out, dev_phase& dp, int& op_end, int& headers_left)
{
  const int begin = dp.op_begin;
  std::vector<dev_op> list(out.ops + begin, out.ops + op_end);
  std::vector<dev_op> grouped;
  for (size_t i = 0; i < list.size();) {
    // Runs take general diagonals when the extra member records fit in the
    // records kept back for headers; otherwise only the phase form.
    size_t j = i;
    while (j < list.size() && is_phase_op(list[j], true)) ++j;
    std::vector<dev_op> members;
    if (j - i >= 2 && headers_left > 0) {
      members = phase_members(list, i, j);
      if (static_cast<int>(members.size()) - static_cast<int>(j - i) > headers_left - 1 || members.empty()) {
        j = i;
        while (j < list.size() && is_phase_op(list[j], false)) ++j;
        members = j - i >= 2 ? phase_members(list, i, j) : std::vector<dev_op>{};
      }
    }
    if (j - i >= 2 && headers_left > 0 && !members.empty()) {
      auto cls = [&](const dev_op& g) {
        const int c = __builtin_popcount(g.creg);
        return c == 0 ? 0 : c == 1 ? 1 + __builtin_ctz(g.creg) : 1 + p.R;
      };
      std::stable_sort(members.begin(), members.end(), [&](const dev_op& x, const dev_op& y) { return cls(x) < cls(y); });
      dev_op h{};
      h.kind = OPK_PHASES;
      h.run = static_cast<uint32_t>(members.size());
      h.code = op_code(OPK_PHASES, 0, true, 0);
      for (const dev_op& g : members) {
        const int c = cls(g);
        if (c <= p.R) h.dout += 1ull << (8 * c);
      }
      grouped.push_back(h);
      headers_left -= 1 + std::max(0, static_cast<int>(members.size()) - static_cast<int>(j - i));
      grouped.insert(grouped.end(), members.begin(), members.end());
    } else {
      if (j == i) ++j;  // a gate that is not a phase
      for (size_t k = i; k < j; ++k) grouped.push_back(list[k]);
    }
    i = j;
  }
  if (begin + static_cast<int>(grouped.size()) > kMaxPassOps) throw std::logic_error("planner: too many op records");
  for (size_t k = 0; k < grouped.size(); ++k) out.ops[begin + static_cast<int>(k)] = grouped[k];
  op_end = begin + static_cast<int>(grouped.size());
}

// Consecutive uncontrolled MAT ops of a phase on distinct register bits go to
// the kernel behind one LAYER header, sorted by register bit (gates on distinct
// qubits commute): the kernel applies them as one straight-line block, with no
// dispatch between the gates.  Form: the matrices' common form, where m00-real
// ones may join general ones (the general update computes the same values);
// real ones join only real ones.
int layer_form(int a, int b)
{
  if (a == b) return a;
  if ((a == 0 && b == 2) || (a == 2 && b == 0)) return 0;
  return -1;
}

// M = diag(p0, p1) * [[1, t0], [t1, 1]] * diag(1, q) for the factored layer
// (kLayerFactored in rbk_internal.h): q = e^{i (arg b - arg a)} makes
// t0 = |b| / |a| real, and t1 = c q / d is real when b c / (a d) is, as for every
// unitary.  When b / a is already real (real matrices: H, EY) q = 1 and t0 = b / a,
// so that a layer of such gates needs no pre factors.  false: a or d is zero, t1 is not real to 4e-15, or |t0| or |t1|
// exceeds 2^10 (a gate close to an X: the middle factor would grow the
// amplitudes by up to that much per gate; complex<float> has the smaller range).
struct gate_factors {
  double t0, t1;
  std::complex<double> p0, p1, q;
};

bool factor_gate(const double* m, gate_factors& f)
{
  using cd = std::complex<double>;
  const cd a{m[0], m[1]}, b{m[2], m[3]}, c{m[4], m[5]}, d{m[6], m[7]};
  const double na = std::abs(a), nb = std::abs(b), nd = std::abs(d);
  if (na == 0.0 || nd == 0.0) return false;
  const cd r = b / a;
  if (nb == 0.0 || std::abs(r.imag()) <= 4e-15 * std::abs(r.real())) {
    f.q = cd{1.0, 0.0};
    f.t0 = r.real();
  } else {
    f.q = r / std::abs(r);
    f.t0 = nb / na;
  }
  f.p0 = a;
  f.p1 = d / f.q;
  const cd w1 = c * f.q / d;
  if (!(std::abs(w1.imag()) <= 4e-15 * std::max(1.0, std::abs(w1)))) return false;
  f.t1 = w1.real();
  constexpr double kMaxT = 1024.0;
  return std::abs(f.t0) <= kMaxT && std::abs(f.t1) <= kMaxT;
}

// Rewrites the LAYER whose header is ops[0] (its members follow) into the
// factored form when every member factors and a table slot is free.  The slot
// is written in the state's precision (complex<float> entries for vbits 1).
bool factor_layer(const plan_params& p, dev_pass& out, dev_op* ops, int& tabs_used)
{
  dev_op& h = ops[0];
  const int run = static_cast<int>(h.run);
  if (run < p.factored_min || tabs_used + 1 > kMaxLayerTabs) return false;
  const int H = 1 << (p.R - 2);
  if ((8 + 2 * H) * (p.vbits == 0 ? 16 : 8) > kTabDoubles * 8) throw std::logic_error("planner: layer table too small");
  std::vector<gate_factors> f(static_cast<size_t>(run));
  for (int k = 0; k < run; ++k)
    if (!factor_gate(ops[1 + k].m, f[static_cast<size_t>(k)])) return false;
  // Per register bit: q, p0, p1 (1 for bits outside the layer).
  using cd = std::complex<double>;
  std::vector<cd> q(static_cast<size_t>(p.R), 1.0), p0(static_cast<size_t>(p.R), 1.0), p1(static_cast<size_t>(p.R), 1.0);
  bool any_q = false;
  for (int k = 0; k < run; ++k) {
    const gate_factors& g = f[static_cast<size_t>(k)];
    const size_t b = ops[1 + k].treg;
    q[b] = g.q;
    p0[b] = g.p0;
    p1[b] = g.p1;
    any_q = any_q || g.q != cd{1.0, 0.0};
  }
  // Products over bits [lo, lo + count) of the entry's index bits.
  auto pre_part = [&](int lo, int count, int x) {
    cd v = 1.0;
    for (int b = 0; b < count; ++b) if ((x >> b) & 1) v *= q[static_cast<size_t>(lo + b)];
    return v;
  };
  auto post_part = [&](int lo, int count, int x) {
    cd v = 1.0;
    for (int b = 0; b < count; ++b) v *= ((x >> b) & 1) ? p1[static_cast<size_t>(lo + b)] : p0[static_cast<size_t>(lo + b)];
    return v;
  };
  std::vector<cd> slot;  // pre_lo[4], pre_hi[H], post_lo[4], post_hi[H]
  for (int l = 0; l < 4; ++l) slot.push_back(pre_part(0, 2, l));
  for (int h = 0; h < H; ++h) slot.push_back(pre_part(2, p.R - 2, h));
  const cd hi0 = post_part(2, p.R - 2, 0);
  for (int l = 0; l < 4; ++l) slot.push_back(post_part(0, 2, l) * hi0);
  slot.push_back(1.0);  // post_hi[0] is exactly 1: the kernel skips it
  for (int h = 1; h < H; ++h) slot.push_back(post_part(2, p.R - 2, h) / hi0);
  double* tab = out.tabs + tabs_used * kTabDoubles;
  float* t32 = reinterpret_cast<float*>(tab);
  for (size_t i = 0; i < slot.size(); ++i) {
    if (p.vbits == 0) { tab[2 * i] = slot[i].real(); tab[2 * i + 1] = slot[i].imag(); }
    else { t32[2 * i] = static_cast<float>(slot[i].real()); t32[2 * i + 1] = static_cast<float>(slot[i].imag()); }
  }
  for (int k = 0; k < run; ++k) {
    dev_op& g = ops[1 + k];
    std::memset(g.m, 0, sizeof(g.m));
    g.m[0] = f[static_cast<size_t>(k)].t0;
    g.m[1] = f[static_cast<size_t>(k)].t1;
  }
  h.real = kLayerFactored;
  h.dthr = static_cast<uint32_t>(tabs_used);
  h.diag_one = any_q ? 1 : 0;
  h.code = op_code(OPK_LAYER, kLayerFactored, h.dreg == (1u << p.R) - 1, 0);
  tabs_used += 1;
  return true;
}

void group_layers(const plan_params& p, dev_pass& out, dev_phase& dp, int& op_end, int& headers_left, int& tabs_used)
{
  const int begin = dp.op_begin;
  std::vector<dev_op> list(out.ops + begin, out.ops + op_end);
  auto layer_op = [](const dev_op& d) { return d.kind == OPK_MAT && d.creg == 0 && d.cthr == 0 && d.cout == 0; };
  std::vector<dev_op> grouped;
  for (size_t i = 0; i < list.size();) {
    size_t j = i;
    uint32_t mask = 0;
    int form = layer_op(list[i]) ? list[i].real : -1;
    while (j < list.size() && layer_op(list[j]) && !((mask >> list[j].treg) & 1u)) {
      const int f = layer_form(form, list[j].real);
      if (f < 0) break;
      form = f;
      mask |= 1u << list[j].treg;
      ++j;
    }
    if (j - i >= 2 && headers_left > 0) {
      dev_op h{};
      h.kind = OPK_LAYER;
      h.run = static_cast<uint32_t>(j - i);
      h.dreg = mask;
      h.real = static_cast<uint8_t>(form);
      h.code = op_code(OPK_LAYER, form, mask == (1u << p.R) - 1, 0);
      grouped.push_back(h);
      --headers_left;
      std::vector<dev_op> run(list.begin() + static_cast<long>(i), list.begin() + static_cast<long>(j));
      std::sort(run.begin(), run.end(), [](const dev_op& x, const dev_op& y) { return x.treg < y.treg; });
      grouped.insert(grouped.end(), run.begin(), run.end());
      if (p.factored_min > 0) factor_layer(p, out, &grouped[grouped.size() - run.size() - 1], tabs_used);
    } else {
      if (j == i) ++j;
      for (size_t k = i; k < j; ++k) grouped.push_back(list[k]);
    }
    i = j;
  }
  if (begin + static_cast<int>(grouped.size()) > kMaxPassOps) throw std::logic_error("planner: too many op records");
  for (size_t k = 0; k < grouped.size(); ++k) out.ops[begin + static_cast<int>(k)] = grouped[k];
  op_end = begin + static_cast<int>(grouped.size());
}

void build_pass(const plan_params& p, uint64_t tile_mask, const std::vector<pop>& ops,
                const int* relabel_to, const int* tile_phys, dev_pass& out)
{
  std::memset(&out, 0, sizeof(out));
  const int K = p.K, R = p.R, T = K - R;
  int tile_of_phys[64];
  for (int i = 0; i < 64; ++i) tile_of_phys[i] = -1;
  for (int b = 0; b < K; ++b) {
    out.tile_phys[b] = static_cast<uint8_t>(tile_phys[b]);
    tile_of_phys[tile_phys[b]] = b;
  }
  // Non-tile physical bits as runs of consecutive bits.
  {
    int runs = 0, src = 0;
    for (int q = 0; q < p.n;) {
      if (tile_mask & bit(q)) { ++q; continue; }
      int len = 0;
      while (q + len < p.n && !(tile_mask & bit(q + len))) ++len;
      out.run_src[runs] = static_cast<uint8_t>(src);
      out.run_len[runs] = static_cast<uint8_t>(len);
      out.run_dst[runs] = static_cast<uint8_t>(q);
      ++runs;
      src += len;
      q += len;
    }
    out.num_runs = static_cast<uint8_t>(runs);
  }

  std::vector<phase_build> phases = phases_by_dag(ops, tile_of_phys, R, false);
  if (p.defer_x) {  // taking CNOT / X gates last lets them fold; keep it unless it costs register phases
    std::vector<phase_build> deferred = phases_by_dag(ops, tile_of_phys, R, true);
    if (deferred.size() <= phases.size()) phases.swap(deferred);
  }
  if (static_cast<int>(phases.size()) > kMaxPhases) phases = phases_in_order(ops, tile_of_phys, R);
  if (static_cast<int>(phases.size()) > kMaxPhases) throw std::logic_error("planner: too many phases");

  // Tile bits lane0 .. lane0+4 are contiguous in HBM (512-byte runs); for c64
  // tile bit 0 is the amplitude pair inside one 16-byte vector.
  const int lane0 = p.vbits;
  int relabel_from[16];
  for (int b = 0; b < K; ++b) relabel_from[relabel_to[b]] = b;
  auto contains = [](const std::vector<int>& v, int x) { return std::find(v.begin(), v.end(), x) != v.end(); };

  int op_index = 0;
  int headers_left = kMaxPassOps - kMaxPassGates;
  int tabs_used = 0;
  for (size_t ph = 0; ph < phases.size(); ++ph) {
    auto& pb = phases[ph];
    const bool first = ph == 0, last = ph + 1 == phases.size();
    // Direct HBM access modes of the first phase's load and the last phase's
    // store.  Mode 1: 16-byte vectors, lanes on HBM bits lane0 .. lane0+4 (a
    // warp touches one 512-byte run) and, for c64, the amplitude pair bit
    // (HBM bit 0) on register bit 0.  Mode 2 (c64 only): 8-byte amplitudes,
    // lanes on HBM bits 0..4 (256-byte runs), for phases whose gates act on the
    // pair bit or leave no register for it.  map[x]: tile bit at HBM bit x
    // (identity for the load; for the store, after the pass's relabelling).
    int identity[16];
    for (int b = 0; b < 16; ++b) identity[b] = b;
    auto lanes_of = [&](int mode, const int* map) {
      std::vector<int> l;
      const int first_lane = mode == 2 ? 0 : lane0;
      for (int x = 0; x < 5; ++x) l.push_back(map[first_lane + x]);
      return l;
    };
    auto mode_for = [&](const int* map) {
      auto off = [&](const std::vector<int>& bits) {
        for (int b : bits) if (contains(pb.reg, b)) return false;
        return true;
      };
      // the lanes' HBM bits must be tile bits in every tile: the fixed low bits
      if (lane0 + 5 <= p.LOW && off(lanes_of(1, map)) && (!p.vbits || contains(pb.reg, map[0]) || static_cast<int>(pb.reg.size()) < R)) return 1;
      if (p.vbits && 5 <= p.LOW && off(lanes_of(2, map))) return 2;
      return 0;
    };
    const int lmode = first ? mode_for(identity) : 0;
    const int smode = last ? mode_for(relabel_from) : 0;
    // Bits the fill should keep out of (or bring into) the registers for those modes.
    std::vector<int> keep_out, bring_in;
    if (lmode) {
      for (int b : lanes_of(lmode, identity)) keep_out.push_back(b);
      if (p.vbits && lmode == 1) bring_in.push_back(0);
    }
    if (smode) {
      for (int b : lanes_of(smode, relabel_from)) keep_out.push_back(b);
      if (p.vbits && smode == 1) bring_in.push_back(relabel_from[0]);
    }
    for (int b : bring_in)
      if (!contains(pb.reg, b) && !contains(keep_out, b) && static_cast<int>(pb.reg.size()) < R) pb.reg.push_back(b);
    for (int b = K - 1; b >= 0 && static_cast<int>(pb.reg.size()) < R; --b)
      if (!contains(pb.reg, b) && !contains(keep_out, b)) pb.reg.push_back(b);
    for (int b = K - 1; b >= 0 && static_cast<int>(pb.reg.size()) < R; --b)
      if (!contains(pb.reg, b)) pb.reg.push_back(b);

    auto holds = [&](int mode, const int* map) {
      if (!mode) return false;
      for (int b : lanes_of(mode, map)) if (contains(pb.reg, b)) return false;
      return !(p.vbits && mode == 1) || contains(pb.reg, map[0]);
    };
    bool dl = holds(lmode, identity), ds = holds(smode, relabel_from);
    if (dl && ds) {  // one layout must serve both: the same mode, with its lanes (and the c64 pair bit) in place
      ds = lmode == smode;
      for (int x = 0; x < 5 && ds; ++x) ds = lanes_of(lmode, identity)[x] == lanes_of(smode, relabel_from)[x];
      if (ds && p.vbits && lmode == 1) ds = relabel_from[0] == 0;
    }
    std::vector<int> thr;
    for (int b = 0; b < K; ++b) if (!contains(pb.reg, b)) thr.push_back(b);
    // The five lanes of a direct HBM access may come in any order (a warp
    // still touches one 512-byte run); the order puts three tile bits with
    // distinct bank residues on lanes 0-2 where it can, for the phase's
    // shared-memory accesses in the same layout.
    auto lanes_first = [&](const std::vector<int>& lanes) {
      std::vector<int> o(lanes);
      if (!p.vbits) {
        bool used[3] = {false, false, false};
        std::vector<int> front, back;
        for (int b : o) {
          if (front.size() < 3 && !used[b % 3]) { used[b % 3] = true; front.push_back(b); }
          else back.push_back(b);
        }
        o = front;
        o.insert(o.end(), back.begin(), back.end());
      }
      for (int b : thr) if (!contains(lanes, b)) o.push_back(b);
      thr = o;
    };
    if (dl) lanes_first(lanes_of(lmode, identity));
    else if (ds) lanes_first(lanes_of(smode, relabel_from));
    else order_thread_bits(thr, p.vbits, last ? relabel_to : nullptr);
    // c64 16-byte vectors: register index bit 0 must be the amplitude pair bit.
    if (p.vbits && ((dl && lmode == 1) || (ds && smode == 1))) {
      const int want = (dl && lmode == 1) ? 0 : relabel_from[0];
      auto it = std::find(pb.reg.begin(), pb.reg.end(), want);
      std::iter_swap(pb.reg.begin(), it);
    }
    if (first) out.direct_load = static_cast<uint8_t>(dl ? lmode : 0);
    if (last) out.direct_store = static_cast<uint8_t>(ds ? smode : 0);

    dev_phase& dp = out.phases[ph];
    int reg_index[64], thr_index[64];
    for (int i = 0; i < 64; ++i) reg_index[i] = thr_index[i] = -1;
    for (int b = 0; b < R; ++b) { dp.reg_pos[b] = static_cast<uint8_t>(pb.reg[b]); reg_index[pb.reg[b]] = b; }
    for (int b = 0; b < T; ++b) { dp.thr_pos[b] = static_cast<uint8_t>(thr[b]); thr_index[thr[b]] = b; }
    for (int b = 0; b < R; ++b) dp.wreg_pos[b] = static_cast<uint8_t>(last ? relabel_to[pb.reg[b]] : pb.reg[b]);
    for (int b = 0; b < T; ++b) dp.wthr_pos[b] = static_cast<uint8_t>(last ? relabel_to[thr[b]] : thr[b]);

    // Precomputed shared-memory slots (the slot map is linear) and HBM offsets.
    if (T < 5 || T > 9) throw std::logic_error("planner: layout tables hold 5 to 9 thread bits");
    for (int b = 0; b < R; ++b) {
      dp.rslot[b] = static_cast<uint16_t>(smem_slot_host(1u << dp.reg_pos[b], p.vbits));
      dp.wslot[b] = static_cast<uint16_t>(smem_slot_host(1u << dp.wreg_pos[b], p.vbits));
    }
    for (int x = 0; x < 32; ++x) {
      uint32_t lo = 0, hi = 0, wlo = 0, whi = 0;
      for (int k = 0; k < 5; ++k) {
        if (!((x >> k) & 1)) continue;
        if (k < 4) { lo |= 1u << dp.thr_pos[k]; wlo |= 1u << dp.wthr_pos[k]; }
        if (4 + k < T) { hi |= 1u << dp.thr_pos[4 + k]; whi |= 1u << dp.wthr_pos[4 + k]; }
      }
      if (x < 16) {
        dp.tslot_lo[x] = static_cast<uint16_t>(smem_slot_host(lo, p.vbits));
        dp.wtslot_lo[x] = static_cast<uint16_t>(smem_slot_host(wlo, p.vbits));
      }
      dp.tslot_hi[x] = static_cast<uint16_t>(smem_slot_host(hi, p.vbits));
      dp.wtslot_hi[x] = static_cast<uint16_t>(smem_slot_host(whi, p.vbits));
    }
    auto hbm = [&](dev_hbm_layout& L, const uint8_t* rpos, const uint8_t* tpos) {
      for (int b = 0; b < R; ++b) L.rphys[b] = bit(tile_phys[rpos[b]]);
      for (int x = 0; x < 32; ++x) {
        uint64_t lo = 0, hi = 0;
        for (int k = 0; k < 5; ++k) {
          if (!((x >> k) & 1)) continue;
          if (k < 4) lo |= bit(tile_phys[tpos[k]]);
          if (4 + k < T) hi |= bit(tile_phys[tpos[4 + k]]);
        }
        if (x < 16) L.tphys_lo[x] = lo;
        L.tphys_hi[x] = hi;
      }
    };
    if (first && dl) hbm(out.load, dp.reg_pos, dp.thr_pos);
    if (last && ds) hbm(out.store, dp.wreg_pos, dp.wthr_pos);

    dp.op_begin = static_cast<uint16_t>(op_index);
    for (int oi : pb.ops) {
      const pop& o = ops[oi];
      if (op_index >= kMaxPassOps) throw std::logic_error("planner: too many op records");
      dev_op& d = out.ops[op_index++];
      d = dev_op{};  // the slot may hold an op of an earlier phase that folding removed
      d.kind = o.kind;
      d.diag_one = o.diag_one;
      std::memcpy(d.m, o.m, sizeof(d.m));
      // 1: all four entries real; 2: m00 real (U3, U2); 0: general.
      if (o.kind == OPK_MAT && o.m[1] == 0.0 && o.m[3] == 0.0 && o.m[5] == 0.0 && o.m[7] == 0.0) d.real = 1;
      else if (o.kind == OPK_MAT && o.m[1] == 0.0) d.real = 2;
      else d.real = 0;
      auto classify = [&](uint64_t phys_mask, uint32_t& reg, uint32_t& thrm, uint64_t& outm) {
        while (phys_mask) {
          const int q = __builtin_ctzll(phys_mask);
          phys_mask &= phys_mask - 1;
          const int tb = tile_of_phys[q];
          if (tb < 0) outm |= bit(q);
          else if (reg_index[tb] >= 0) reg |= 1u << reg_index[tb];
          else thrm |= 1u << thr_index[tb];
        }
      };
      classify(o.cmask, d.creg, d.cthr, d.cout);
      if (is_target_kind(o.kind)) {
        const int tb = tile_of_phys[o.target];
        if (tb < 0 || reg_index[tb] < 0) throw std::logic_error("planner: target not in registers");
        d.treg = static_cast<uint8_t>(reg_index[tb]);
      } else if (o.kind == OPK_DIAG) {
        classify(bit(o.target), d.dreg, d.dthr, d.dout);
      }
    }
    for (int k = dp.op_begin; k < op_index; ++k) {
      dev_op& d = out.ops[k];
      d.code = d.kind == OPK_MAT ? op_code(OPK_MAT, d.real, d.creg != 0, d.treg)
             : (d.kind == OPK_X || d.kind == OPK_Y) ? op_code(d.kind, 0, true, d.treg)
             : op_code(d.kind, 0, true, 0);
    }
    if (p.fold_x) fold_trailing_x(p, out, dp, op_index, last && ds ? smode : 0);
    if (p.phase_runs) group_phase_runs(p, out, dp, op_index, headers_left);
    if (p.layers) group_layers(p, out, dp, op_index, headers_left, tabs_used);
    dp.op_end = static_cast<uint16_t>(op_index);
  }
  out.num_phases = static_cast<uint8_t>(phases.size());
}

// Single-qubit gates without controls as 2x2 matrices (row-major, re/im pairs).
bool single_qubit_matrix(const pop& o, double* m)
{
  std::memset(m, 0, 8 * sizeof(double));
  if (o.kind == OPK_MAT && o.cmask == 0) { std::memcpy(m, o.m, 8 * sizeof(double)); return true; }
  if (o.kind == OPK_X && o.cmask == 0) { m[2] = 1; m[4] = 1; return true; }
  if (o.kind == OPK_Y && o.cmask == 0) { m[3] = -1; m[5] = 1; return true; }
  if (o.kind == OPK_DIAG && o.cmask == 0) { m[0] = o.m[0]; m[1] = o.m[1]; m[6] = o.m[2]; m[7] = o.m[3]; return true; }
  return false;
}

bool touches(const pop& o, int q)
{
  return o.target == q || ((o.cmask >> q) & 1);
}

// Merges an uncontrolled single-qubit gate into the last op of the pass that
// touches its qubit when that op is an uncontrolled single-qubit gate too and
// one of the two is non-diagonal (so the qubit is a tile bit): the ops between
// them act on other qubits, so the new gate can move back to it and the two
// become one 2x2 matrix (later gate times earlier).  allow_dense: the merge may
// turn two sparse gates (X, Y, diagonal) into a dense one.
bool merge_single_qubit(std::vector<pop>& ops, const pop& o, bool allow_dense)
{
  double b[8];
  if (o.target < 0 || !single_qubit_matrix(o, b)) return false;
  for (size_t j = ops.size(); j-- > 0;) {
    if (!touches(ops[j], o.target)) continue;
    double a[8];
    if (ops[j].target != o.target || !single_qubit_matrix(ops[j], a)) return false;
    if (!is_target_kind(ops[j].kind) && !is_target_kind(o.kind)) return false;
    if (ops[j].kind != OPK_MAT && o.kind != OPK_MAT && !allow_dense) return false;
    double c[8];
    for (int r = 0; r < 2; ++r)
      for (int k = 0; k < 2; ++k) {
        double re = 0, im = 0;
        for (int l = 0; l < 2; ++l) {
          const double xr = b[2 * (2 * r + l)], xi = b[2 * (2 * r + l) + 1];
          const double yr = a[2 * (2 * l + k)], yi = a[2 * (2 * l + k) + 1];
          re += xr * yr - xi * yi;
          im += xr * yi + xi * yr;
        }
        c[2 * (2 * r + k)] = re;
        c[2 * (2 * r + k) + 1] = im;
      }
    ops[j].kind = OPK_MAT;
    ops[j].diag_one = 0;
    std::memcpy(ops[j].m, c, sizeof(c));
    return true;
  }
  return false;
}

// Tile bit order: physical bits 0..LOW-1 first, then the others ascending.
void tile_order(const plan_params& p, uint64_t tile_mask, int* tile_phys)
{
  int k = 0;
  for (int q = 0; q < p.LOW; ++q) tile_phys[k++] = q;
  for (int q = p.LOW; q < p.n; ++q)
    if (tile_mask & bit(q)) tile_phys[k++] = q;
}

// Applies a physical relabelling new_phys_of_old (for tile bits) to perm/inv
// and returns it as tile-bit -> tile-bit.
void apply_relabel(const plan_params& p, const int* tile_phys, const int* new_phys_of_tile_bit,
                   std::vector<int>& perm, std::vector<int>& inv, int* relabel_to)
{
  int tile_of_phys[64];
  for (int i = 0; i < 64; ++i) tile_of_phys[i] = -1;
  for (int b = 0; b < p.K; ++b) tile_of_phys[tile_phys[b]] = b;
  std::vector<int> moved_logical(p.K);
  for (int b = 0; b < p.K; ++b) moved_logical[b] = inv[tile_phys[b]];
  for (int b = 0; b < p.K; ++b) {
    const int np = new_phys_of_tile_bit[b];
    relabel_to[b] = tile_of_phys[np];
    perm[moved_logical[b]] = np;
    inv[np] = moved_logical[b];
  }
}

}  // namespace

gate_rec to_physical(const hgate& g, const std::vector<int>& perm)
{
  gate_rec r{};
  r.kind = g.kind;
  r.diag_one = g.diag_one;
  r.target = static_cast<uint8_t>(g.target >= 0 ? perm[g.target] : 0);
  r.cmask = map_mask(g.cmask, perm);
  std::memcpy(r.m, g.m, sizeof(r.m));
  return r;
}

void plan_passes(const plan_params& p, const std::vector<hgate>& gates, std::vector<int>& perm,
                 std::vector<int>& inv, std::vector<dev_pass>& out)
{
  const uint64_t all = p.n >= 64 ? ~0ull : bit(p.n) - 1;
  const uint64_t low_mask = bit(p.LOW) - 1;
  std::vector<char> taken(gates.size(), 0);
  size_t first = 0;
  const int budget = p.dense_budget > 0 ? p.dense_budget : 1;

  while (true) {
    while (first < gates.size() && taken[first]) ++first;
    if (first >= gates.size()) break;

    uint64_t tile = low_mask;
    uint64_t blockN = 0, blockZ = 0;
    std::vector<pop> ops;
    int dense = 0;
    phase_tracker tracker{p.R};

    for (size_t i = first; i < gates.size(); ++i) {
      if (taken[i]) continue;
      const hgate& g = gates[i];
      if (g.kind == HK_SWAP) {
        const uint64_t m = bit(g.target) | bit(g.target2);
        if ((blockN | blockZ) & m) { blockN |= m; continue; }
        const int pa = perm[g.target], pb = perm[g.target2];
        perm[g.target] = pb; perm[g.target2] = pa;
        inv[pa] = g.target2; inv[pb] = g.target;
        taken[i] = 1;
        continue;
      }
      const uint64_t Nq = is_target_kind(g.kind) ? bit(g.target) : 0;
      const uint64_t Zq = g.cmask | (g.kind == OPK_DIAG ? bit(g.target) : 0);
      if ((Nq & (blockN | blockZ)) || (Zq & blockN)) {
        blockN |= Nq; blockZ |= Zq;
        if (((blockN | blockZ) & all) == all) break;
        continue;
      }
      bool ok = static_cast<int>(ops.size()) < kMaxPassGates;
      const int t = Nq ? perm[g.target] : -1;
      if (ok && t >= 0 && !(tile & bit(t)) && popc(tile) >= p.K) ok = false;
      if (ok && is_dense(g) && dense >= budget) ok = false;
      if (ok && t >= 0 && !tracker.would_fit(t, kMaxPhases)) ok = false;
      if (!ok) {
        blockN |= Nq; blockZ |= Zq;
        if (((blockN | blockZ) & all) == all) break;
        continue;
      }
      if (t >= 0) { tile |= bit(t); tracker.add(t); }
      pop o{};
      o.kind = g.kind;
      o.diag_one = g.diag_one;
      o.target = g.target >= 0 ? perm[g.target] : -1;
      o.cmask = map_mask(g.cmask, perm);
      std::memcpy(o.m, g.m, sizeof(o.m));
      taken[i] = 1;
      if (p.merge_1q) {
        // the merged op is dense; it adds to the pass's dense count unless the op it replaces was dense
        bool was_dense = false;
        for (size_t j = ops.size(); j-- > 0;)
          if (touches(ops[j], o.target)) { was_dense = ops[j].kind == OPK_MAT; break; }
        if (merge_single_qubit(ops, o, dense < budget)) {
          dense += was_dense ? 0 : 1;
          continue;
        }
      }
      ops.push_back(o);
      dense += is_dense(g) ? 1 : 0;
    }
    if (ops.empty()) continue;  // only swaps were taken: layout map updated, no data moved

    // Next use (queue position) of each logical qubit as a non-diagonal target.
    const int INF = std::numeric_limits<int>::max();
    std::vector<int> next_use(p.n, INF);
    bool remaining = false;
    for (size_t i = first; i < gates.size(); ++i) {
      if (taken[i]) continue;
      remaining = true;
      const hgate& g = gates[i];
      if (g.kind == HK_SWAP) {
        next_use[g.target] = std::min(next_use[g.target], static_cast<int>(i));
        next_use[g.target2] = std::min(next_use[g.target2], static_cast<int>(i));
      } else if (is_target_kind(g.kind)) {
        next_use[g.target] = std::min(next_use[g.target], static_cast<int>(i));
      }
    }
    // Fill the tile to K bits with the qubits needed soonest.
    while (popc(tile) < p.K) {
      int best = -1;
      for (int q = 0; q < p.n; ++q) {
        if (tile & bit(perm[q])) continue;
        if (best < 0 || next_use[q] < next_use[best] ||
            (next_use[q] == next_use[best] && perm[q] < perm[best])) best = q;
      }
      tile |= bit(perm[best]);
    }
    int tile_phys[16];
    tile_order(p, tile, tile_phys);

    // Relabel: the soonest-needed logical qubits go to the low physical bits;
    // with nothing left in the queue, qubits go home where the tile allows.
    int new_phys[16];
    {
      std::vector<int> logical(p.K);
      for (int b = 0; b < p.K; ++b) logical[b] = inv[tile_phys[b]];
      std::vector<int> assign(p.K, -1);  // tile bit -> new physical bit
      std::vector<char> phys_used(64, 0);
      if (remaining) {
        std::vector<int> order(p.K);
        for (int b = 0; b < p.K; ++b) order[b] = b;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b2) {
          return next_use[logical[a]] < next_use[logical[b2]];
        });
        for (int r = 0; r < p.LOW; ++r) {
          if (next_use[logical[order[r]]] == INF) break;
          assign[order[r]] = r;
          phys_used[r] = 1;
        }
        // Others keep their position when it is free.
        for (int b = 0; b < p.K; ++b)
          if (assign[b] < 0 && !phys_used[tile_phys[b]]) { assign[b] = tile_phys[b]; phys_used[tile_phys[b]] = 1; }
      } else {
        for (int b = 0; b < p.K; ++b) {
          const int home = logical[b];
          if ((tile & bit(home)) && !phys_used[home]) { assign[b] = home; phys_used[home] = 1; }
        }
        for (int b = 0; b < p.K; ++b)
          if (assign[b] < 0 && !phys_used[tile_phys[b]]) { assign[b] = tile_phys[b]; phys_used[tile_phys[b]] = 1; }
      }
      for (int b = 0; b < p.K; ++b) {
        if (assign[b] >= 0) continue;
        for (int c = 0; c < p.K; ++c)
          if (!phys_used[tile_phys[c]]) { assign[b] = tile_phys[c]; phys_used[tile_phys[c]] = 1; break; }
      }
      for (int b = 0; b < p.K; ++b) new_phys[b] = assign[b];
    }
    int relabel_to[16];
    apply_relabel(p, tile_phys, new_phys, perm, inv, relabel_to);
    out.emplace_back();
    build_pass(p, tile, ops, relabel_to, tile_phys, out.back());
  }
}

void plan_layout(const plan_params& p, std::vector<int>& perm, std::vector<int>& inv, const std::vector<int>& target,
                 std::vector<dev_pass>& out)
{
  const uint64_t low_mask = bit(p.LOW) - 1;
  for (int guard = 0; guard < 4 * p.n + 4; ++guard) {
    bool done = true;
    for (int q = 0; q < p.n; ++q) if (perm[q] != target[q]) { done = false; break; }
    if (done) return;

    // Tile bits: the physical bits of as many misplaced qubits and of their
    // homes as fit, then any others up to K.
    uint64_t tile = low_mask;
    for (int q = 0; q < p.n; ++q) {
      if (perm[q] == target[q]) continue;
      const uint64_t need = bit(perm[q]) | bit(target[q]);
      if (popc(tile | need) <= p.K) tile |= need;
    }
    for (int q = 0; q < p.n && popc(tile) < p.K; ++q) tile |= bit(q);
    int tile_phys[16];
    tile_order(p, tile, tile_phys);

    int new_phys[16];
    std::vector<char> used(64, 0);
    std::vector<int> assign(p.K, -1);
    for (int b = 0; b < p.K; ++b) {
      const int home = target[inv[tile_phys[b]]];  // where the qubit on this tile bit belongs
      if ((tile & bit(home)) && !used[home]) { assign[b] = home; used[home] = 1; }
    }
    for (int b = 0; b < p.K; ++b) {
      if (assign[b] >= 0) continue;
      for (int c = 0; c < p.K; ++c)
        if (!used[tile_phys[c]]) { assign[b] = tile_phys[c]; used[tile_phys[c]] = 1; break; }
    }
    for (int b = 0; b < p.K; ++b) new_phys[b] = assign[b];
    int relabel_to[16];
    apply_relabel(p, tile_phys, new_phys, perm, inv, relabel_to);
    out.emplace_back();
    build_pass(p, tile, std::vector<pop>{}, relabel_to, tile_phys, out.back());
  }
  throw std::logic_error("planner: layout change did not converge");
}

void plan_canonicalize(const plan_params& p, std::vector<int>& perm, std::vector<int>& inv,
                       std::vector<dev_pass>& out)
{
  std::vector<int> identity(static_cast<size_t>(p.n));
  for (int q = 0; q < p.n; ++q) identity[static_cast<size_t>(q)] = q;
  plan_layout(p, perm, inv, identity, out);
}

}  // namespace rbk
