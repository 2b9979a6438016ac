// rbk_rotate_plan.cpp -- see rbk_rotate_plan.h.
#include "rbk_rotate_plan.h"

#include <algorithm>
#include <cstring>

namespace rbk {

namespace {
// The tiles of launch_paired_overlaps: the low 3 physical bits (128-byte runs
// of complex<double>) plus 8 more, 8 thread bits and kPairRegBits register bits.
constexpr int kLowBits = 3;
constexpr int kTileBits = 8 + kPairRegBits;
}  // namespace

std::vector<pair_rotate_set> plan_rotations(int n, const std::vector<rotate_item>& items, const pre_diag* owed)
{
  std::vector<pair_rotate_set> out;
  bool first_launch = true;
  constexpr int RB = kPairRegBits, KT = kTileBits;
  size_t next = 0;
  while (next < items.size()) {
    std::vector<int> tile_bits;
    for (int b = 0; b < kLowBits; ++b) tile_bits.push_back(b);
    std::vector<size_t> mine;
    while (next < items.size() && static_cast<int>(mine.size()) < kMaxRotFlips) {
      const int b = items[next].bit;
      const bool in = std::find(tile_bits.begin(), tile_bits.end(), b) != tile_bits.end();
      if (!in && static_cast<int>(tile_bits.size()) >= KT) break;
      if (!in) tile_bits.push_back(b);
      mine.push_back(next++);
    }
    for (int b = 0; static_cast<int>(tile_bits.size()) < KT; ++b)  // fillers
      if (std::find(tile_bits.begin(), tile_bits.end(), b) == tile_bits.end()) tile_bits.push_back(b);
    std::sort(tile_bits.begin(), tile_bits.end());
    pair_rotate_set set{};
    spin_group& g = set.g;
    g.K = KT;
    uint64_t mask = 0;
    for (int b = 0; b < KT; ++b) { g.tile_phys[b] = static_cast<uint8_t>(tile_bits[static_cast<size_t>(b)]); mask |= 1ull << tile_bits[static_cast<size_t>(b)]; }
    // Register phases, by groups of tile bits: A = 8..10 (the load layout),
    // B = 0..2, C = 3, 4 and a spare, D = 5..7.  A, B and C keep tile bits 5..7
    // on the warp index, so moving between them (and from C to the store) stays
    // inside each warp; only entering and leaving D needs the whole CTA.
    // Groups without a gate are left out, except A.  In every layout the tile
    // bits on lanes 0-2 reach distinct low bits of the swizzled shared-memory
    // slot (smem_slot), so that the 8 lanes of a 128-byte wavefront hit
    // distinct bank groups (c128).
    std::vector<int> local;      // tile bit of each register position
    std::vector<long> pos_item;  // index into items, -1 for a filler
    {
      std::vector<long> gate_at(KT, -1);
      for (size_t y : mine)
        gate_at[static_cast<size_t>(std::find(tile_bits.begin(), tile_bits.end(), items[y].bit) - tile_bits.begin())] =
          static_cast<long>(y);
      static const int groups[4][3] = {{8, 9, 10}, {0, 1, 2}, {3, 4, 0}, {5, 6, 7}};
      static const int thr_of[4][8] = {{0, 1, 2, 3, 4, 5, 6, 7}, {3, 4, 8, 9, 10, 5, 6, 7},
                                       {1, 2, 9, 8, 10, 5, 6, 7}, {0, 1, 2, 3, 4, 8, 9, 10}};
      int p = 0;
      int warps_of[kSpinPhases + 1] = {};
      for (int gi = 0; gi < 4; ++gi) {
        const int nreal = gi == 2 ? 2 : 3;  // group C's third bit is a spare
        bool any = gi == 0;
        for (int k = 0; k < nreal; ++k) any = any || gate_at[static_cast<size_t>(groups[gi][k])] >= 0;
        if (!any) continue;
        for (int k = 0; k < RB; ++k) {
          local.push_back(groups[gi][k]);
          pos_item.push_back(k < nreal ? gate_at[static_cast<size_t>(groups[gi][k])] : -1);
          g.phase_reg[p][k] = static_cast<uint8_t>(groups[gi][k]);
        }
        for (int b = 0; b < 8; ++b) g.phase_thr[p][b] = static_cast<uint8_t>(thr_of[gi][b]);
        warps_of[p] = gi == 3 ? 1 : 0;
        ++p;
      }
      g.nphases = p;
      warps_of[p] = 0;  // the store reads in the load layout
      for (int q = 0; q < p; ++q) set.block_sync[q] = warps_of[q] != warps_of[q + 1] ? 1 : 0;
    }
    g.nflips = static_cast<int>(local.size());
    int runs = 0, src = 0;
    for (int q = 0; q < n;) {
      if ((mask >> q) & 1) { ++q; continue; }
      int len = 0;
      while (q + len < n && !((mask >> (q + len)) & 1)) ++len;
      g.run_src[runs] = static_cast<uint8_t>(src);
      g.run_len[runs] = static_cast<uint8_t>(len);
      g.run_dst[runs] = static_cast<uint8_t>(q);
      ++runs;
      src += len;
      q += len;
    }
    g.num_runs = runs;
    for (size_t f = 0; f < local.size(); ++f) {
      auto& fl = set.flip[f];
      if (pos_item[f] < 0) {
        fl.out_slot = -1;
        fl.okind = 0;
        fl.mkind = 2;
        continue;
      }
      const rotate_item& it = items[static_cast<size_t>(pos_item[f])];
      fl.out_slot = it.slot;
      fl.minus = it.spec.sign != 0 ? 1 : 0;
      fl.wr = it.spec.wr;
      fl.wi = it.spec.wi;
      fl.okind = it.slot < 0 ? 0 : (it.spec.wr == 0.0 ? 1 : 0) | (it.spec.wi == 0.0 ? 2 : 0);
      if (it.slot >= 0 && fl.okind == 0) fl.okind = 3;
      std::memcpy(fl.m, it.m, sizeof(fl.m));
      fl.mkind = (it.m[1] == 0.0 && it.m[3] == 0.0 && it.m[5] == 0.0 && it.m[7] == 0.0) ? 1 : 0;
    }
    if (owed && first_launch) {
      set.pre = *owed;
      set.pre.active = 1;
      // The register slots' partner rows and their pairs among themselves.
      set.pre.qr = 0;
      for (int it = 0; it < (1 << RB); ++it) {
        uint64_t mr = 0;
        uint32_t par = 0;
        for (int k = 0; k < RB; ++k) {
          if (!((it >> k) & 1)) continue;
          const int a = g.tile_phys[8 + k];
          mr ^= owed->full[a];
          for (int k2 = k + 1; k2 < RB; ++k2)
            if ((it >> k2) & 1) par ^= static_cast<uint32_t>((owed->full[a] >> g.tile_phys[8 + k2]) & 1);
        }
        set.pre.mr[it] = mr;
        set.pre.qr |= par << it;
      }
    }
    first_launch = false;
    out.push_back(set);
  }
  return out;
}

}  // namespace rbk
