// ketref_driver.cpp -- TEST INFRASTRUCTURE ONLY (the oracle's reference leg).
//
// Runs the reference's own C++ code for the state-vector hot path:
// the header-only ket gate / observable functions from ket/include and bra's
// fused-gate classes from bra/src/fused_*.cpp, compiled unchanged against the
// project-written Boost stand-ins in riken-braket_b200/bra/shim.  bra itself (bra::state,
// bra::nompi_state, the interpreter) needs Boost.Variant, fmt and cxxopts, which
// are absent, so this file restates only the dispatch that bra::nompi_state
// performs for each instruction and calls exactly the ket function it calls:
//
//   H      -> ket::gate::ranges::hadamard            (bra/src/nompi_state.cpp:326-337)
//   X/Y/Z  -> ket::gate::ranges::pauli_{x,y,z}
//   U1     -> ket::gate::ranges::phase_shift         (bra/src/nompi_state.cpp do_u1)
//   U2     -> ket::gate::ranges::phase_shift2
//   U3     -> ket::gate::ranges::phase_shift3        (bra/src/nompi_state.cpp:681-694)
//   CNOT   -> ket::gate::ranges::not_ with a control (bra/src/nompi_state.cpp:1415-1431)
//   CZ     -> ket::gate::ranges::pauli_z on two controls
//   U c1 c2 k -> ket::gate::ranges::phase_shift_coeff with the bra phase table
//             (bra/src/state.cpp:148 generate_phase_coefficients; :2650-2669)
//   EX/EY/EZ -> ket::gate::ranges::exponential_pauli_{x,y,z}
//   BEGIN/END FUSION -> bra::fused_gate objects replayed per fused index by
//             ket::gate::runtime::ranges::gate (bra/src/nompi_state.cpp:1285-1357,
//             found-qubit bookkeeping of bra/include/bra/state.hpp:126-173)
//
// Observables: ket::ranges::all_spin_expectation_values (DO MEASUREMENT,
// bra/src/nompi_state.cpp:1105-1106), ket::runtime::ranges::expectation_value
// with the Pauli-string lambda of bra/src/nompi_state.cpp:1155-1202, and
// ket::ranges::inner_product.
//
// The product never links or loads this library; only tests, golden-fixture
// generation and bench.py's CPU reference arm do.

#include <algorithm>
#include <chrono>
#include <complex>
#include <cstdint>
#include <cstring>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include <ket/qubit.hpp>
#include <ket/control.hpp>
#include <ket/gate/gate.hpp>
#include <ket/gate/hadamard.hpp>
#include <ket/gate/not_.hpp>
#include <ket/gate/pauli_x.hpp>
#include <ket/gate/pauli_y.hpp>
#include <ket/gate/pauli_z.hpp>
#include <ket/gate/phase_shift.hpp>
#include <ket/gate/swap.hpp>
#include <ket/gate/exponential_pauli_x.hpp>
#include <ket/gate/exponential_pauli_y.hpp>
#include <ket/gate/exponential_pauli_z.hpp>
#include <ket/gate/exponential_swap.hpp>
#include <ket/gate/sqrt_pauli_x.hpp>
#include <ket/gate/sqrt_pauli_y.hpp>
#include <ket/gate/sqrt_pauli_z.hpp>
#include <ket/gate/x_rotation_half_pi.hpp>
#include <ket/gate/y_rotation_half_pi.hpp>
#include <ket/gate/toffoli.hpp>
#include <ket/gate/clear.hpp>
#include <ket/gate/set.hpp>
#include <ket/shor_box.hpp>
#include <ket/gate/utility/index_with_qubits.hpp>
#include <ket/gate/utility/pauli_index_coeff.hpp>
#include <ket/all_spin_expectation_values.hpp>
#include <ket/generate_events.hpp>
#include <ket/measure.hpp>
#include <ket/gate/projective_measurement.hpp>
#include <random>
#include <ket/expectation_value.hpp>
#include <ket/inner_product.hpp>
#include <ket/utility/generate_phase_coefficients.hpp>
#include <ket/utility/loop_n.hpp>
#include <ket/utility/parallel/loop_n.hpp>

#include <bra/types.hpp>
#include <bra/fused_gate/fused_gate.hpp>
#include <bra/fused_gate/fused_hadamard.hpp>
#include <bra/fused_gate/fused_pauli_x.hpp>
#include <bra/fused_gate/fused_pauli_y.hpp>
#include <bra/fused_gate/fused_pauli_z.hpp>
#include <bra/fused_gate/fused_u1.hpp>
#include <bra/fused_gate/fused_u2.hpp>
#include <bra/fused_gate/fused_u3.hpp>
#include <bra/fused_gate/fused_controlled_not.hpp>
#include <bra/fused_gate/fused_controlled_pauli_z.hpp>
#include <bra/fused_gate/fused_controlled_phase_shift.hpp>
#include <bra/fused_gate/fused_exponential_pauli_x.hpp>
#include <bra/fused_gate/fused_exponential_pauli_y.hpp>
#include <bra/fused_gate/fused_exponential_pauli_z.hpp>
#include <bra/fused_gate/fused_swap.hpp>

#include "oracle_ops.h"

namespace {

using complex_t = bra::complex_type;
using data_t = bra::data_type;
using qubit_t = bra::qubit_type;
using control_t = bra::control_qubit_type;
using plain_it = data_t::iterator;
#ifdef KET_USE_BIT_MASKS_EXPLICITLY
using cache_it = ket::gate::utility::cache_aware_iterator<plain_it, bra::state_integer_type>;
#else
using cache_it = ket::gate::utility::cache_aware_iterator<plain_it, qubit_t>;
#endif

enum class found : int { none = 0, control = 1, ez = 2, cez = 3, target = 4 };

struct ref_state
{
  unsigned n;
  ket::utility::policy::parallel<unsigned int> policy;
  data_t data;
  std::vector<complex_t> phase_table;
  bool in_fusion = false;
  std::vector<found> found_qubits;
  std::vector<std::unique_ptr<bra::fused_gate::fused_gate<plain_it>>> fused_plain;
  std::vector<std::unique_ptr<bra::fused_gate::fused_gate<cache_it>>> fused_cache;
  std::mt19937_64 rng{1};  // bra::state's random_number_generator_ (bra/include/bra/state.hpp:459-479)

  ref_state(unsigned nq, unsigned threads, std::uint64_t initial)
    : n{nq}, policy{threads}, data(std::size_t{1} << nq), found_qubits(nq, found::none)
  {
    data[initial] = complex_t{1.0, 0.0};
    ket::utility::generate_phase_coefficients(phase_table, n);
  }
};

// bra marks a target qubit unconditionally and a control/EZ qubit only when it
// is not already marked by something stronger (bra/include/bra/state.hpp:126-173).
void mark(ref_state& s, unsigned q, found kind)
{
  if (kind == found::target || static_cast<int>(s.found_qubits[q]) < static_cast<int>(kind))
    s.found_qubits[q] = kind;
}

template <template <typename> class Fused, typename... Args>
void push_fused(ref_state& s, Args const&... args)
{
  s.fused_plain.push_back(std::make_unique<Fused<plain_it>>(args...));
  s.fused_cache.push_back(std::make_unique<Fused<cache_it>>(args...));
}

struct fused_caller
{
  ref_state const* s;
  std::vector<bra::bit_integer_type> const* remap;

  template <typename First, typename A, typename B>
  auto operator()(First const first, bra::state_integer_type const index_wo_qubits,
                  A const& qubits_or_masks, B const& sorted_or_index_masks, int const) const
    -> typename std::enable_if<std::is_same<typename std::decay<First>::type, plain_it>::value>::type
  {
    for (auto const& g: s->fused_plain)
      g->call(first, index_wo_qubits, qubits_or_masks, sorted_or_index_masks, *remap);
  }

  template <typename First, typename A, typename B>
  auto operator()(First const first, bra::state_integer_type const index_wo_qubits,
                  A const& qubits_or_masks, B const& sorted_or_index_masks, int const) const
    -> typename std::enable_if<std::is_same<typename std::decay<First>::type, cache_it>::value>::type
  {
    for (auto const& g: s->fused_cache)
      g->call(first, index_wo_qubits, qubits_or_masks, sorted_or_index_masks, *remap);
  }
};

// END FUSION: targets (target/EZ/CEZ marks) first in ascending order, then the
// pure control qubits; every recorded gate is replayed on each 2^k chunk.
void end_fusion(ref_state& s)
{
  std::vector<qubit_t> targets;
  std::vector<qubit_t> controls;
  for (unsigned q = 0; q < s.n; ++q)
  {
    switch (s.found_qubits[q])
    {
     case found::control: controls.push_back(ket::make_qubit<bra::state_integer_type>(q)); break;
     case found::ez: case found::cez: case found::target:
      targets.push_back(ket::make_qubit<bra::state_integer_type>(q)); break;
     case found::none: break;
    }
  }
  std::vector<bra::bit_integer_type> remap(s.n);
  std::iota(remap.begin(), remap.end(), bra::bit_integer_type{0});
  bra::bit_integer_type slot = 0;
  for (auto const q: targets) remap[static_cast<bra::bit_integer_type>(q)] = slot++;
  for (auto const q: controls) remap[static_cast<bra::bit_integer_type>(q)] = slot++;

  std::vector<qubit_t> operated(targets);
  operated.insert(operated.end(), controls.begin(), controls.end());

  ket::gate::runtime::ranges::gate(s.policy, s.data, fused_caller{&s, &remap}, operated);

  s.fused_plain.clear();
  s.fused_cache.clear();
  std::fill(s.found_qubits.begin(), s.found_qubits.end(), found::none);
  s.in_fusion = false;
}

qubit_t qb(int q) { return ket::make_qubit<bra::state_integer_type>(static_cast<unsigned>(q)); }
control_t cq(int q) { return ket::make_control(qb(q)); }

void apply_one(ref_state& s, oracle_op const& op)
{
  auto const q0 = op.q[0];
  auto const q1 = op.q[1];
  bool const f = s.in_fusion;
  switch (op.code)
  {
   case ORC_H:
    if (f) { mark(s, q0, found::target); push_fused<bra::fused_gate::fused_hadamard>(s, qb(q0)); }
    else ket::gate::ranges::hadamard(s.policy, s.data, qb(q0));
    break;
   case ORC_X:
    if (f) { mark(s, q0, found::target); push_fused<bra::fused_gate::fused_pauli_x>(s, qb(q0)); }
    else ket::gate::ranges::pauli_x(s.policy, s.data, qb(q0));
    break;
   case ORC_Y:
    if (f) { mark(s, q0, found::target); push_fused<bra::fused_gate::fused_pauli_y>(s, qb(q0)); }
    else ket::gate::ranges::pauli_y(s.policy, s.data, qb(q0));
    break;
   case ORC_Z:
    if (f) { mark(s, q0, found::control); push_fused<bra::fused_gate::fused_pauli_z>(s, cq(q0)); }
    else ket::gate::ranges::pauli_z(s.policy, s.data, cq(q0));
    break;
   case ORC_U1:
    if (f) { mark(s, q0, found::control); push_fused<bra::fused_gate::fused_u1>(s, op.p[0], cq(q0)); }
    else ket::gate::ranges::phase_shift(s.policy, s.data, op.p[0], cq(q0));
    break;
   case ORC_U2:
    if (f) { mark(s, q0, found::target); push_fused<bra::fused_gate::fused_u2>(s, op.p[0], op.p[1], qb(q0)); }
    else ket::gate::ranges::phase_shift2(s.policy, s.data, op.p[0], op.p[1], qb(q0));
    break;
   case ORC_U3:
    if (f) { mark(s, q0, found::target); push_fused<bra::fused_gate::fused_u3>(s, op.p[0], op.p[1], op.p[2], qb(q0)); }
    else ket::gate::ranges::phase_shift3(s.policy, s.data, op.p[0], op.p[1], op.p[2], qb(q0));
    break;
   case ORC_CNOT:  // q0 = control, q1 = target ("CNOT c t")
    if (f)
    {
      mark(s, q1, found::target); mark(s, q0, found::control);
      push_fused<bra::fused_gate::fused_controlled_not>(s, qb(q1), cq(q0));
    }
    else ket::gate::ranges::not_(s.policy, s.data, qb(q1), cq(q0));
    break;
   case ORC_CZ:
    if (f)
    {
      mark(s, q0, found::control); mark(s, q1, found::control);
      push_fused<bra::fused_gate::fused_controlled_pauli_z>(s, cq(q0), cq(q1));
    }
    else ket::gate::ranges::pauli_z(s.policy, s.data, cq(q0), cq(q1));
    break;
   case ORC_CPHASE_K:  // "U c1 c2 k": phase 2*pi/2^k on |11>; negative k = adjoint
   {
    int const k = op.k;
    complex_t const coeff = k >= 0 ? s.phase_table.at(static_cast<std::size_t>(k))
                                   : std::conj(s.phase_table.at(static_cast<std::size_t>(-k)));
    if (f)
    {
      mark(s, q0, found::control); mark(s, q1, found::control);
      push_fused<bra::fused_gate::fused_controlled_phase_shift>(s, coeff, cq(q0), cq(q1));
    }
    else ket::gate::ranges::phase_shift_coeff(s.policy, s.data, coeff, cq(q0), cq(q1));
    break;
   }
   case ORC_EX:
    if (f) { mark(s, q0, found::target); push_fused<bra::fused_gate::fused_exponential_pauli_x>(s, op.p[0], qb(q0)); }
    else ket::gate::ranges::exponential_pauli_x(s.policy, s.data, op.p[0], qb(q0));
    break;
   case ORC_EY:
    if (f) { mark(s, q0, found::target); push_fused<bra::fused_gate::fused_exponential_pauli_y>(s, op.p[0], qb(q0)); }
    else ket::gate::ranges::exponential_pauli_y(s.policy, s.data, op.p[0], qb(q0));
    break;
   case ORC_EZ:
    if (f) { mark(s, q0, found::ez); push_fused<bra::fused_gate::fused_exponential_pauli_z>(s, op.p[0], qb(q0)); }
    else ket::gate::ranges::exponential_pauli_z(s.policy, s.data, op.p[0], qb(q0));
    break;
   case ORC_SWAP:
    if (f)
    {
      mark(s, q0, found::target); mark(s, q1, found::target);
      push_fused<bra::fused_gate::fused_swap>(s, qb(q0), qb(q1));
    }
    else ket::gate::ranges::swap(s.policy, s.data, qb(q0), qb(q1));
    break;
   case ORC_BEGIN_FUSION:
    s.in_fusion = true;
    std::fill(s.found_qubits.begin(), s.found_qubits.end(), found::none);
    break;
   case ORC_END_FUSION:
    if (s.in_fusion) end_fusion(s);
    break;
   default:
    throw std::invalid_argument("ketref: unsupported op code");
  }
}

// The wider instruction set, unfused, following bra's nompi_state dispatch
// (bra/src/nompi_state.cpp:326-1280 and :1359-2600): one target and at most one
// control use ket::gate::ranges::X, everything else the runtime forms
// ket::gate::runtime::ranges::X(targets, controls).
struct gate_args
{
  std::vector<qubit_t> t;
  std::vector<control_t> c;
  double const* p;
};

template <typename One, typename OneCtl, typename Many>
void dispatch_target(gate_args const& a, One one, OneCtl one_ctl, Many many)
{
  if (a.t.size() == 1 && a.c.empty()) one(a.t[0]);
  else if (a.t.size() == 1 && a.c.size() == 1) one_ctl(a.t[0], a.c[0]);
  else many(a.t, a.c);
}

// Gates on control-type qubits only (Z, SZ, U1, R): 1 or 2 qubits use the
// variadic forms, more the runtime form over all of them.
template <typename One, typename Two, typename Many>
void dispatch_controls(gate_args const& a, One one, Two two, Many many)
{
  if (a.c.size() == 1) one(a.c[0]);
  else if (a.c.size() == 2) two(a.c[0], a.c[1]);
  else many(a.c);
}

#define KR ket::gate::ranges
#define KRT ket::gate::runtime::ranges

void apply_gate(ref_state& s, int kind, gate_args const& a)
{
  auto& P = s.policy;
  auto& D = s.data;
  double const* p = a.p;
  switch (kind)
  {
   case KG_H:
    dispatch_target(a, [&](qubit_t t) { KR::hadamard(P, D, t); }, [&](qubit_t t, control_t c) { KR::hadamard(P, D, t, c); },
                    [&](auto const& t, auto const& c) { KRT::hadamard(P, D, t.at(0), c); });
    break;
   case KG_NOT:
    dispatch_target(a, [&](qubit_t t) { KR::not_(P, D, t); }, [&](qubit_t t, control_t c) { KR::not_(P, D, t, c); },
                    [&](auto const& t, auto const& c) { KRT::not_(P, D, t.at(0), c); });
    break;
   case KG_X:
    if (a.c.empty() && a.t.size() == 2) KR::pauli_x(P, D, a.t[0], a.t[1]);
    else if (a.c.empty() && a.t.size() > 2) KRT::pauli_x(P, D, a.t);
    else dispatch_target(a, [&](qubit_t t) { KR::pauli_x(P, D, t); }, [&](qubit_t t, control_t c) { KR::pauli_x(P, D, t, c); },
                         [&](auto const& t, auto const& c) { KRT::pauli_x(P, D, t, c); });
    break;
   case KG_Y:
    if (a.c.empty() && a.t.size() == 2) KR::pauli_y(P, D, a.t[0], a.t[1]);
    else if (a.c.empty() && a.t.size() > 2) KRT::pauli_y(P, D, a.t);
    else dispatch_target(a, [&](qubit_t t) { KR::pauli_y(P, D, t); }, [&](qubit_t t, control_t c) { KR::pauli_y(P, D, t, c); },
                         [&](auto const& t, auto const& c) { KRT::pauli_y(P, D, t, c); });
    break;
   case KG_Z:
    if (a.t.empty())
      dispatch_controls(a, [&](control_t c) { KR::pauli_z(P, D, c); }, [&](control_t c1, control_t c2) { KR::pauli_z(P, D, c1, c2); },
                        [&](auto const& c) { KRT::pauli_z(P, D, c); });
    else if (a.c.empty() && a.t.size() == 2) KR::pauli_z(P, D, a.t[0], a.t[1]);
    else if (a.c.empty()) KRT::pauli_z(P, D, a.t);
    else KRT::pauli_z(P, D, a.t, a.c);
    break;
   case KG_SWAP:
    if (a.c.empty()) KR::swap(P, D, a.t.at(0), a.t.at(1));
    else KRT::swap(P, D, a.t.at(0), a.t.at(1), a.c);
    break;
#define KG_TARGET_GATE(CODE, NAME)                                                                                       \
   case CODE:                                                                                                            \
    dispatch_target(a, [&](qubit_t t) { KR::NAME(P, D, t); }, [&](qubit_t t, control_t c) { KR::NAME(P, D, t, c); },       \
                    [&](auto const& t, auto const& c) { KRT::NAME(P, D, t.at(0), c); });                                \
    break;
   KG_TARGET_GATE(KG_SX, sqrt_pauli_x)
   KG_TARGET_GATE(KG_SX_ADJ, adj_sqrt_pauli_x)
   KG_TARGET_GATE(KG_SY, sqrt_pauli_y)
   KG_TARGET_GATE(KG_SY_ADJ, adj_sqrt_pauli_y)
   KG_TARGET_GATE(KG_ROTX, x_rotation_half_pi)
   KG_TARGET_GATE(KG_ROTX_ADJ, adj_x_rotation_half_pi)
   KG_TARGET_GATE(KG_ROTY, y_rotation_half_pi)
   KG_TARGET_GATE(KG_ROTY_ADJ, adj_y_rotation_half_pi)
#undef KG_TARGET_GATE
   case KG_SZ: case KG_SZ_ADJ:
   {
    bool const adj = kind == KG_SZ_ADJ;
    if (a.t.empty())
      dispatch_controls(a,
                        [&](control_t c) { if (adj) KR::adj_sqrt_pauli_z(P, D, c); else KR::sqrt_pauli_z(P, D, c); },
                        [&](control_t c1, control_t c2) { if (adj) KR::adj_sqrt_pauli_z(P, D, c1, c2); else KR::sqrt_pauli_z(P, D, c1, c2); },
                        [&](auto const& c) { if (adj) KRT::adj_sqrt_pauli_z(P, D, c); else KRT::sqrt_pauli_z(P, D, c); });
    else if (a.c.empty() && a.t.size() == 2)
    { if (adj) KR::adj_sqrt_pauli_z(P, D, a.t[0], a.t[1]); else KR::sqrt_pauli_z(P, D, a.t[0], a.t[1]); }
    else if (a.c.empty())
    { if (adj) KRT::adj_sqrt_pauli_z(P, D, a.t); else KRT::sqrt_pauli_z(P, D, a.t); }
    else
    { if (adj) KRT::adj_sqrt_pauli_z(P, D, a.t, a.c); else KRT::sqrt_pauli_z(P, D, a.t, a.c); }
    break;
   }
   case KG_U1: case KG_U1_ADJ:
   {
    bool const adj = kind == KG_U1_ADJ;
    dispatch_controls(a,
                      [&](control_t c) { if (adj) KR::adj_phase_shift(P, D, p[0], c); else KR::phase_shift(P, D, p[0], c); },
                      [&](control_t c1, control_t c2) { if (adj) KR::adj_phase_shift(P, D, p[0], c1, c2); else KR::phase_shift(P, D, p[0], c1, c2); },
                      [&](auto const& c) { if (adj) KRT::adj_phase_shift(P, D, p[0], c); else KRT::phase_shift(P, D, p[0], c); });
    break;
   }
   case KG_R: case KG_R_ADJ:  // bra::state::phase_shift: phase_coefficients_[k], negative k = adjoint
   {
    int k = static_cast<int>(p[0]);
    bool adj = kind == KG_R_ADJ;
    if (k < 0) { k = -k; adj = !adj; }
    complex_t const coeff = s.phase_table.at(static_cast<std::size_t>(k));
    dispatch_controls(a,
                      [&](control_t c) { if (adj) KR::adj_phase_shift_coeff(P, D, coeff, c); else KR::phase_shift_coeff(P, D, coeff, c); },
                      [&](control_t c1, control_t c2) { if (adj) KR::adj_phase_shift_coeff(P, D, coeff, c1, c2); else KR::phase_shift_coeff(P, D, coeff, c1, c2); },
                      [&](auto const& c) { if (adj) KRT::adj_phase_shift_coeff(P, D, coeff, c); else KRT::phase_shift_coeff(P, D, coeff, c); });
    break;
   }
   case KG_U2: case KG_U2_ADJ:
   {
    bool const adj = kind == KG_U2_ADJ;
    dispatch_target(a,
                    [&](qubit_t t) { if (adj) KR::adj_phase_shift2(P, D, p[0], p[1], t); else KR::phase_shift2(P, D, p[0], p[1], t); },
                    [&](qubit_t t, control_t c) { if (adj) KR::adj_phase_shift2(P, D, p[0], p[1], t, c); else KR::phase_shift2(P, D, p[0], p[1], t, c); },
                    [&](auto const& t, auto const& c) { if (adj) KRT::adj_phase_shift2(P, D, p[0], p[1], t.at(0), c); else KRT::phase_shift2(P, D, p[0], p[1], t.at(0), c); });
    break;
   }
   case KG_U3: case KG_U3_ADJ:
   {
    bool const adj = kind == KG_U3_ADJ;
    dispatch_target(a,
                    [&](qubit_t t) { if (adj) KR::adj_phase_shift3(P, D, p[0], p[1], p[2], t); else KR::phase_shift3(P, D, p[0], p[1], p[2], t); },
                    [&](qubit_t t, control_t c) { if (adj) KR::adj_phase_shift3(P, D, p[0], p[1], p[2], t, c); else KR::phase_shift3(P, D, p[0], p[1], p[2], t, c); },
                    [&](auto const& t, auto const& c) { if (adj) KRT::adj_phase_shift3(P, D, p[0], p[1], p[2], t.at(0), c); else KRT::phase_shift3(P, D, p[0], p[1], p[2], t.at(0), c); });
    break;
   }
#define KG_EXP_GATE(CODE, ADJCODE, NAME)                                                                                 \
   case CODE: case ADJCODE:                                                                                              \
   {                                                                                                                     \
    bool const adj = kind == ADJCODE;                                                                                    \
    if (a.c.empty() && a.t.size() == 1)                                                                                  \
    { if (adj) KR::adj_##NAME(P, D, p[0], a.t[0]); else KR::NAME(P, D, p[0], a.t[0]); }                                  \
    else if (a.c.empty() && a.t.size() == 2)                                                                             \
    { if (adj) KR::adj_##NAME(P, D, p[0], a.t[0], a.t[1]); else KR::NAME(P, D, p[0], a.t[0], a.t[1]); }                  \
    else if (a.c.size() == 1 && a.t.size() == 1)                                                                         \
    { if (adj) KR::adj_##NAME(P, D, p[0], a.t[0], a.c[0]); else KR::NAME(P, D, p[0], a.t[0], a.c[0]); }                  \
    else if (a.c.empty())                                                                                                \
    { if (adj) KRT::adj_##NAME(P, D, p[0], a.t); else KRT::NAME(P, D, p[0], a.t); }                                      \
    else                                                                                                                 \
    { if (adj) KRT::adj_##NAME(P, D, p[0], a.t, a.c); else KRT::NAME(P, D, p[0], a.t, a.c); }                            \
    break;                                                                                                               \
   }
   KG_EXP_GATE(KG_EX, KG_EX_ADJ, exponential_pauli_x)
   KG_EXP_GATE(KG_EY, KG_EY_ADJ, exponential_pauli_y)
   KG_EXP_GATE(KG_EZ, KG_EZ_ADJ, exponential_pauli_z)
#undef KG_EXP_GATE
   case KG_ESWAP: case KG_ESWAP_ADJ:
   {
    bool const adj = kind == KG_ESWAP_ADJ;
    if (a.c.empty())
    { if (adj) KR::adj_exponential_swap(P, D, p[0], a.t.at(0), a.t.at(1)); else KR::exponential_swap(P, D, p[0], a.t.at(0), a.t.at(1)); }
    else
    { if (adj) KRT::adj_exponential_swap(P, D, p[0], a.t.at(0), a.t.at(1), a.c); else KRT::exponential_swap(P, D, p[0], a.t.at(0), a.t.at(1), a.c); }
    break;
   }
   case KG_TOFFOLI:
    KR::toffoli(P, D, a.t.at(0), a.c.at(0), a.c.at(1));
    break;
   case KG_CLEAR:
    KR::clear(P, D, a.t.at(0));
    break;
   case KG_SET:
    KR::set(P, D, a.t.at(0));
    break;
   case KG_SHORBOX:  // p = {nx, divisor, base}; exponent qubits on top (bra/src/state.cpp shor_box)
   {
    auto const nx = static_cast<unsigned>(p[0]);
    std::vector<qubit_t> ex, mod;
    for (unsigned q = s.n - nx; q < s.n; ++q) ex.push_back(qb(static_cast<int>(q)));
    for (unsigned q = 0; q < s.n - nx; ++q) mod.push_back(qb(static_cast<int>(q)));
    ket::ranges::shor_box(P, D, static_cast<bra::state_integer_type>(p[2]), static_cast<bra::state_integer_type>(p[1]), ex, mod);
    break;
   }
   default:
    throw std::invalid_argument("ketref: unsupported gate kind");
  }
}

#undef KR
#undef KRT

thread_local std::string g_error;

} // namespace

extern "C" {

void* ketref_create(int num_qubits, int num_threads, std::uint64_t initial_index)
{
  try { return new ref_state(static_cast<unsigned>(num_qubits), static_cast<unsigned>(num_threads), initial_index); }
  catch (std::exception const& e) { g_error = e.what(); return nullptr; }
}

void ketref_destroy(void* h) { delete static_cast<ref_state*>(h); }

const char* ketref_last_error(void) { return g_error.c_str(); }

void ketref_set_amplitudes(void* h, double const* interleaved)
{
  auto& s = *static_cast<ref_state*>(h);
  std::memcpy(static_cast<void*>(s.data.data()), interleaved, s.data.size() * sizeof(complex_t));
}

void ketref_get_amplitudes(void* h, double* interleaved)
{
  auto const& s = *static_cast<ref_state*>(h);
  std::memcpy(interleaved, static_cast<void const*>(s.data.data()), s.data.size() * sizeof(complex_t));
}

// Applies ops in order.  Returns 0 on success, -1 on error (message in ketref_last_error).
int ketref_apply(void* h, oracle_op const* ops, int num_ops)
{
  auto& s = *static_cast<ref_state*>(h);
  try { for (int i = 0; i < num_ops; ++i) apply_one(s, ops[i]); }
  catch (std::exception const& e) { g_error = e.what(); return -1; }
  return 0;
}

// Same as ketref_apply, returning the wall time in seconds (bench CPU arm).
double ketref_apply_timed(void* h, oracle_op const* ops, int num_ops)
{
  auto const t0 = std::chrono::steady_clock::now();
  if (ketref_apply(h, ops, num_ops) != 0) return -1.0;
  auto const t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// DO MEASUREMENT: out[3*q + {0,1,2}] = <S_x>, <S_y>, <S_z> of qubit q (spin-1/2 units).
void ketref_spins(void* h, double* out)
{
  auto& s = *static_cast<ref_state*>(h);
  auto const spins = ket::ranges::all_spin_expectation_values<qubit_t>(s.policy, s.data);
  for (std::size_t q = 0; q < spins.size(); ++q)
    for (int c = 0; c < 3; ++c) out[3 * q + c] = spins[q][c];
}

// EXPECTATION over all qubits 0..n-1: sum_t coeff_t <psi| P_t |psi>, where
// pauli_strings holds num_terms strings of n characters from "IXYZ" (character
// k acts on qubit k) and coeffs holds num_terms complex coefficients.
void ketref_expectation(void* h, int num_terms, char const* pauli_strings, double const* coeffs, double* out)
{
  auto& s = *static_cast<ref_state*>(h);
  std::vector<std::pair<std::string, complex_t>> terms;
  for (int t = 0; t < num_terms; ++t)
    terms.emplace_back(std::string(pauli_strings + static_cast<std::size_t>(t) * s.n, s.n),
                       complex_t{coeffs[2 * t], coeffs[2 * t + 1]});
  std::vector<qubit_t> qubits;
  for (unsigned q = 0; q < s.n; ++q) qubits.push_back(qb(static_cast<int>(q)));
  auto const nq = qubits.size();

  auto const value = ket::runtime::ranges::expectation_value(
    s.policy, s.data,
    [&terms, nq](auto const first, auto const index_wo_qubits,
                 auto const& unsorted_qubits_or_masks, auto const& sorted_qubits_or_index_masks)
    {
      complex_t acc{};
      auto const last_index = bra::state_integer_type{1} << nq;
      for (auto index = bra::state_integer_type{0}; index < last_index; ++index)
      {
        auto const it = first + ket::gate::utility::index_with_qubits(
          index_wo_qubits, index,
          std::begin(unsorted_qubits_or_masks), std::end(unsorted_qubits_or_masks),
          std::begin(sorted_qubits_or_index_masks), std::end(sorted_qubits_or_index_masks));
        for (auto const& term: terms)
        {
          auto const other = ket::gate::utility::pauli_index_coeff<complex_t>(term.first, index);
          auto const other_it = first + ket::gate::utility::index_with_qubits(
            index_wo_qubits, other.first,
            std::begin(unsorted_qubits_or_masks), std::end(unsorted_qubits_or_masks),
            std::begin(sorted_qubits_or_index_masks), std::end(sorted_qubits_or_index_masks));
          acc += term.second * (std::conj(*it) * (other.second * *other_it));
        }
      }
      return acc;
    },
    qubits);
  out[0] = value.real();
  out[1] = value.imag();
}

// ket::inner_product(state_a, state_b) = <b|a> = sum conj(b_i) a_i
// (ket/include/ket/inner_product.hpp:30-56).
void ketref_inner_product(void* a, void* b, double* out)
{
  auto& sa = *static_cast<ref_state*>(a);
  auto& sb = *static_cast<ref_state*>(b);
  auto const v = ket::ranges::inner_product(sa.policy, sa.data, sb.data);
  out[0] = v.real();
  out[1] = v.imag();
}

void ketref_seed(void* h, std::uint64_t seed) { static_cast<ref_state*>(h)->rng.seed(seed); }

// GENERATE EVENTS (bra/src/nompi_state.cpp:1143-1153): seed < 0 uses the
// state's generator, else ket's seeded overload.  Like the reference, this
// overwrites the amplitudes with the prefix sums.
void ketref_generate_events(void* h, int num_events, long long seed, std::uint64_t* out)
{
  auto& s = *static_cast<ref_state*>(h);
  std::vector<std::uint64_t> events;
  if (seed < 0)
    ket::ranges::generate_events(ket::utility::policy::make_sequential(), events, s.data, num_events, s.rng);
  else
    ket::ranges::generate_events(ket::utility::policy::make_sequential(), events, s.data, num_events, s.rng,
                                 static_cast<std::mt19937_64::result_type>(seed));
  for (int i = 0; i < num_events; ++i) out[i] = events[i];
}

// ket::ranges::measure with the state's generator (bra/src/nompi_state.cpp do_measure).
std::uint64_t ketref_measure(void* h)
{
  auto& s = *static_cast<ref_state*>(h);
  return static_cast<std::uint64_t>(ket::ranges::measure(ket::utility::policy::make_sequential(), s.data, s.rng));
}

// EXPECTATION :PAULIS:<s> q_0 ... q_{m-1}: bra::nompi_state::do_expectation_value
// (bra/src/nompi_state.cpp:1155-1202) with the operated qubits as listed.
void ketref_expectation_on(void* h, char const* pauli, int num_qubits, int const* qubits, double* out)
{
  auto& s = *static_cast<ref_state*>(h);
  std::string const str(pauli, static_cast<std::size_t>(num_qubits));
  std::vector<qubit_t> operated;
  for (int i = 0; i < num_qubits; ++i) operated.push_back(qb(qubits[i]));
  auto const nq = operated.size();
  auto const value = ket::runtime::ranges::expectation_value(
    s.policy, s.data,
    [&str, nq](auto const first, auto const index_wo_qubits,
               auto const& unsorted_qubits_or_masks, auto const& sorted_qubits_or_index_masks)
    {
      complex_t acc{};
      auto const last_index = bra::state_integer_type{1} << nq;
      for (auto index = bra::state_integer_type{0}; index < last_index; ++index)
      {
        auto const it = first + ket::gate::utility::index_with_qubits(
          index_wo_qubits, index,
          std::begin(unsorted_qubits_or_masks), std::end(unsorted_qubits_or_masks),
          std::begin(sorted_qubits_or_index_masks), std::end(sorted_qubits_or_index_masks));
        auto const other = ket::gate::utility::pauli_index_coeff<complex_t>(str, index);
        auto const other_it = first + ket::gate::utility::index_with_qubits(
          index_wo_qubits, other.first,
          std::begin(unsorted_qubits_or_masks), std::end(unsorted_qubits_or_masks),
          std::begin(sorted_qubits_or_index_masks), std::end(sorted_qubits_or_index_masks));
        acc += std::conj(*it) * (other.second * *other_it);
      }
      return acc;
    },
    operated);
  out[0] = value.real();
  out[1] = value.imag();
}

// INNERPROD n :PAULIS:<s> q_0 ... q_{m-1} with one Pauli string of coefficient 1:
// bra::inner_product_op (bra/src/nompi_state.cpp:2602-2648) through
// ket::runtime::ranges::inner_product(state_a, state_b, observable, qubits)
// = <b| P |a> (ket/include/ket/inner_product.hpp:223-258).
void ketref_inner_product_on(void* a, void* b, char const* pauli, int num_qubits, int const* qubits, double* out)
{
  auto& sa = *static_cast<ref_state*>(a);
  auto& sb = *static_cast<ref_state*>(b);
  std::string const str(pauli, static_cast<std::size_t>(num_qubits));
  std::vector<qubit_t> operated;
  for (int i = 0; i < num_qubits; ++i) operated.push_back(qb(qubits[i]));
  auto const nq = operated.size();
  auto const value = ket::runtime::ranges::inner_product(
    sa.policy, sa.data, sb.data,
    [&str, nq](auto const ket_first, auto const bra_first, auto const index_wo_qubits,
               auto const& unsorted_qubits_or_masks, auto const& sorted_qubits_or_index_masks)
    {
      complex_t acc{};
      auto const last_index = bra::state_integer_type{1} << nq;
      for (auto bra_index = bra::state_integer_type{0}; bra_index < last_index; ++bra_index)
      {
        auto const bra_it = bra_first + ket::gate::utility::index_with_qubits(
          index_wo_qubits, bra_index,
          std::begin(unsorted_qubits_or_masks), std::end(unsorted_qubits_or_masks),
          std::begin(sorted_qubits_or_index_masks), std::end(sorted_qubits_or_index_masks));
        auto const ket_index_coeff = ket::gate::utility::pauli_index_coeff<complex_t>(str, bra_index);
        auto const ket_it = ket_first + ket::gate::utility::index_with_qubits(
          index_wo_qubits, ket_index_coeff.first,
          std::begin(unsorted_qubits_or_masks), std::end(unsorted_qubits_or_masks),
          std::begin(sorted_qubits_or_index_masks), std::end(sorted_qubits_or_index_masks));
        acc += std::conj(*bra_it) * (ket_index_coeff.second * *ket_it);
      }
      return acc;
    },
    operated);
  out[0] = value.real();
  out[1] = value.imag();
}

// One gate of the wider instruction set (kinds in oracle_ops.h).
int ketref_gate(void* h, int kind, int num_targets, int const* targets, int num_controls, int const* controls,
                double const* params)
{
  auto& s = *static_cast<ref_state*>(h);
  try
  {
    gate_args a;
    for (int i = 0; i < num_targets; ++i) a.t.push_back(qb(targets[i]));
    for (int i = 0; i < num_controls; ++i) a.c.push_back(cq(controls[i]));
    a.p = params;
    apply_gate(s, kind, a);
  }
  catch (std::exception const& e) { g_error = e.what(); return -1; }
  return 0;
}

// M q (bra/src/nompi_state.cpp:1102-1103).
int ketref_projective_measurement(void* h, int qubit)
{
  auto& s = *static_cast<ref_state*>(h);
  auto const r = ket::gate::ranges::projective_measurement(s.policy, s.data, s.rng, qb(qubit));
  return r == ket::gate::outcome::one ? 1 : 0;
}

} // extern "C"
