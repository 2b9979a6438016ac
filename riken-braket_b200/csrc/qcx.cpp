// qcx.cpp -- bra's .qcx interpreter over the C ABI of the engine (rbk_qcx.h).
//
// Parsing restates bra::interpreter::invoke (bra/src/interpreter.cpp:372-826)
// and its column readers; the controlled-gate prefixes C..C / Cn follow
// interpret_controlled_gates (:3341-3508).  Execution restates the nompi
// bra::state methods (bra/src/state.cpp:1980-2110) on an rbk_state: every gate
// becomes one or a few queued engine gates, and the printing reproduces bra's
// text line for line.
#include "rbk_qcx.h"

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <map>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace rbk {
int set_last_error(int code, const char* msg);
}

struct rbk_qcx_program {
  int num_qubits = -1;
  int num_circuits = 1;
  uint64_t initial_state = 0;
  std::vector<rbk_qcx_instruction> code;
  std::vector<std::vector<uint64_t>> amplitude_lists;  // DO AMPLITUDES index lists, by instruction
};

namespace {

using columns = std::vector<std::string>;

struct qcx_error : std::runtime_error {
  int code;
  qcx_error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void bad(const std::string& m) { throw qcx_error(RBK_ERR_INVALID, m); }
[[noreturn]] void unsupported(const std::string& m) { throw qcx_error(RBK_ERR_UNSUPPORTED, m); }

std::string upper(std::string s)
{
  for (auto& c : s) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
  return s;
}

bool all_of_char(const std::string& s, size_t from, char c)
{
  return s.size() > from && std::all_of(s.begin() + from, s.end(), [c](char x) { return x == c; });
}

bool all_digits(const std::string& s, size_t from, size_t to)
{
  return to > from && std::all_of(s.begin() + from, s.begin() + to, [](char x) { return std::isdigit(static_cast<unsigned char>(x)); });
}

// boost::lexical_cast<unsigned> / <int> / <double>: the whole column must convert.
uint64_t to_unsigned(const std::string& s)
{
  if (s.empty() || !std::all_of(s.begin(), s.end(), [](char x) { return std::isdigit(static_cast<unsigned char>(x)); }))
    bad("expected a non-negative integer, got '" + s + "'");
  errno = 0;
  const unsigned long long v = std::strtoull(s.c_str(), nullptr, 10);
  if (errno) bad("integer out of range: '" + s + "'");
  return v;
}

int64_t to_int(const std::string& s)
{
  size_t i = (!s.empty() && (s[0] == '+' || s[0] == '-')) ? 1 : 0;
  if (s.size() == i || !std::all_of(s.begin() + i, s.end(), [](char x) { return std::isdigit(static_cast<unsigned char>(x)); }))
    bad("expected an integer, got '" + s + "'");
  return std::strtoll(s.c_str(), nullptr, 10);
}

double parse_double(const std::string& s)
{
  char* end = nullptr;
  const double v = std::strtod(s.c_str(), &end);
  if (s.empty() || end != s.c_str() + s.size()) bad("expected a number, got '" + s + "'");
  return v;
}

// bra::state::to_real (bra/src/state.cpp:771-800) for literals and built-in constants.
double to_real(const std::string& s)
{
  if (s.empty()) bad("empty value");
  const char f = s.front();
  if (std::isdigit(static_cast<unsigned char>(f)) || f == '+' || f == '-' || f == '.') return parse_double(s);
  if (s == ":REAL" || s == ":IMAG") return 0.0;
  if (s == ":PI") return 3.141592653589793238462643383279502884;
  if (s == ":HALF_PI") return 1.570796326794896619231321691639751442;
  if (s == ":TWO_PI") return 6.283185307179586476925286766559005768;
  if (s == ":ROOT_TWO") return 1.414213562373095048801688724209698079;
  if (s == ":HALF_ROOT_TWO") return 0.7071067811865475244008443621048490393;
  if (s.rfind(":REAL:", 0) == 0 && s.size() > 6) {
    const std::string rest = s.substr(6);
    const char g = rest.front();
    if (std::isdigit(static_cast<unsigned char>(g)) || g == '+' || g == '-' || g == '.') return parse_double(rest);
  }
  unsupported("classical variables are not supported ('" + s + "')");
}

// Phase exponent of R / U / T: an integer literal (bra's int_visitor).
int64_t to_phase_exponent(const std::string& s)
{
  if (!s.empty() && s.front() == ':') unsupported("classical variables are not supported ('" + s + "')");
  return to_int(s);
}

// A variable reference: a letter, then letters, digits or '_', optionally
// followed by ':<index>' (bra's NAME:index element access).
bool valid_name(const std::string& s)
{
  if (s.empty() || !std::isalpha(static_cast<unsigned char>(s.front()))) return false;
  const size_t colon = s.find(':');
  for (size_t i = 0; i < std::min(colon, s.size()); ++i)
    if (!std::isalnum(static_cast<unsigned char>(s[i])) && s[i] != '_') return false;
  if (colon == std::string::npos) return true;
  const std::string idx = s.substr(colon + 1);
  return !idx.empty() && std::all_of(idx.begin(), idx.end(), [](char ch) { return std::isdigit(static_cast<unsigned char>(ch)) != 0; });
}

rbk_qcx_instruction blank(int op, int line)
{
  rbk_qcx_instruction in;
  std::memset(&in, 0, sizeof(in));
  in.op = op;
  in.line = line;
  return in;
}

struct parser {
  rbk_qcx_program& prog;
  int line = 0;
  bool done = false;
  int circuit = 0;          // BEGIN CIRCUIT k ... END CIRCUIT (bra/src/interpreter.cpp:672-745)
  bool in_circuit = false;

  uint32_t qubit(const std::string& s)
  {
    const uint64_t q = to_unsigned(s);
    if (prog.num_qubits < 0) bad("QUBITS must come before the first gate");
    if (q >= static_cast<uint64_t>(prog.num_qubits)) bad("qubit " + s + " is out of range");
    return static_cast<uint32_t>(q);
  }

  void expect(const columns& c, size_t n)
  {
    if (c.size() != n) bad("'" + c[0] + "' expects " + std::to_string(n - 1) + " operands, got " + std::to_string(c.size() - 1));
  }

  // A gate: controls first, then targets, then nparams angle columns (or a phase exponent).
  void gate(const columns& c, int kind, int nc, int nt, int nparams, bool exponent = false, bool all_controls = false)
  {
    expect(c, 1 + nc + nt + nparams);
    auto in = blank(RBK_QCX_GATE, line);
    in.kind = kind;
    if (nc + nt > RBK_QCX_MAX_QUBITS) bad("too many qubits");
    std::vector<uint32_t> seen;
    for (int i = 0; i < nc + nt; ++i) {
      const uint32_t q = qubit(c[1 + i]);
      if (std::find(seen.begin(), seen.end(), q) != seen.end()) bad("qubit " + c[1 + i] + " appears twice");
      seen.push_back(q);
      if (i < nc || all_controls) in.controls[in.num_controls++] = q;
      else in.targets[in.num_targets++] = q;
    }
    for (int k = 0; k < nparams; ++k) {
      const std::string& v = c[1 + nc + nt + k];
      in.params[k] = exponent ? static_cast<double>(to_phase_exponent(v)) : to_real(v);
    }
    prog.code.push_back(in);
  }

  void copy_text(rbk_qcx_instruction& in, const std::string& s)
  {
    if (s.size() >= sizeof(in.text)) bad("operand too long");
    std::memcpy(in.text, s.c_str(), s.size() + 1);
  }

  // The operator column of EXPECTATION / INNERPROD / FIDELITY: a :PAULIS:<s>
  // literal whose length must equal the number of operated qubits (returns
  // false), or a PAULISS variable NAME / NAME:index whose length is checked
  // when it runs (returns true).  Either goes to in.text.
  bool operator_column(const std::string& col, size_t num_qubits, rbk_qcx_instruction& in)
  {
    const std::string u = upper(col);
    if (u.rfind(":PAULIS:", 0) == 0 && u.size() > 8) {
      const std::string str = u.substr(8);
      if (str.size() != num_qubits) bad("the Pauli string length must equal the number of qubits");
      if (str.size() > RBK_QCX_MAX_QUBITS) bad("Pauli string too long");
      for (char ch : str)
        if (ch != 'I' && ch != 'X' && ch != 'Y' && ch != 'Z') bad("Pauli strings use I, X, Y, Z");
      copy_text(in, str);
      return false;
    }
    if (!valid_name(u)) unsupported("the operator must be a :PAULIS:<string> literal or a PAULISS variable");
    copy_text(in, u);
    return true;
  }

  void noop(const columns& c, int nqubits)
  {
    expect(c, 1 + nqubits);
    for (int i = 0; i < nqubits; ++i) qubit(c[1 + i]);
    prog.code.push_back(blank(RBK_QCX_NOOP, line));
  }

  // Number of repeated letters ("XXX" -> 3) or explicit count ("X3" -> 3) after the
  // first `skip` characters; 0 if the mnemonic has neither form.
  static int multiplicity(const std::string& m, size_t skip, char letter, bool adjoint)
  {
    const size_t end = m.size() - (adjoint ? 1 : 0);
    if (end <= skip) return 0;
    const std::string body = m.substr(skip, end - skip);
    if (body.empty() || body[0] != letter) return 0;
    if (all_of_char(body, 0, letter)) return static_cast<int>(body.size());
    if (all_digits(body, 1, body.size())) return std::atoi(body.c_str() + 1);
    return 0;
  }

  // Gates that can carry control prefixes; nc = number of controls (0: plain).
  // Returns false if the mnemonic is not a gate.
  bool gate_mnemonic(const columns& c, const std::string& m, int nc)
  {
    const bool adj = m.size() > 1 && m.back() == '+';
    const std::string base = adj ? m.substr(0, m.size() - 1) : m;
    if (base == "I") { noop(c, nc + 1); return true; }
    if (base == "IC") { noop(c, nc + 1); return true; }
    if (int k = multiplicity(m, 0, 'I', false); k >= 2 && !adj) { noop(c, nc + k); return true; }
    if (base == "H" && !adj) { gate(c, RBK_QCX_H, nc, 1, 0); return true; }
    if (base == "NOT" && !adj) { gate(c, RBK_QCX_NOT, nc, 1, 0); return true; }
    for (char p : {'X', 'Y'}) {
      if (adj) break;
      const int kind = p == 'X' ? RBK_QCX_X : RBK_QCX_Y;
      if (base.size() == 1 && base[0] == p) { gate(c, kind, nc, 1, 0); return true; }
      if (int k = multiplicity(m, 0, p, false); k >= 1) { gate(c, kind, nc, k, 0); return true; }
    }
    if (!adj && base == "Z") {  // Z c, CZ c1 c2, CnZ: every qubit of control type
      gate(c, RBK_QCX_Z, nc, 1, 0, false, true);
      return true;
    }
    if (!adj) {
      if (int k = multiplicity(m, 0, 'Z', false); k >= 1) { gate(c, RBK_QCX_Z, nc, k, 0); return true; }
    }
    if (base == "SWAP" && !adj) { gate(c, RBK_QCX_SWAP, nc, 2, 0); return true; }
    if (base == "S" || base == "SZ") { gate(c, adj ? RBK_QCX_SZ_ADJ : RBK_QCX_SZ, nc, 1, 0, false, true); return true; }
    if (int k = multiplicity(m, 1, 'Z', adj); k >= 1 && m[0] == 'S') {  // SZZ, SZ..Z, SZn (+)
      gate(c, adj ? RBK_QCX_SZ_ADJ : RBK_QCX_SZ, nc, k, 0, false, k == 1);
      return true;
    }
    if (base == "T") {  // bra::gate::t_gate: phase_shift(3, c) (bra/src/t_gate.cpp)
      gate(c, adj ? RBK_QCX_R_ADJ : RBK_QCX_R, nc, 1, 0, false, true);
      prog.code.back().params[0] = 3;
      return true;
    }
    if (base == "SX") { gate(c, adj ? RBK_QCX_SX_ADJ : RBK_QCX_SX, nc, 1, 0); return true; }
    if (base == "SY") { gate(c, adj ? RBK_QCX_SY_ADJ : RBK_QCX_SY, nc, 1, 0); return true; }
    if (base == "U1") { gate(c, adj ? RBK_QCX_U1_ADJ : RBK_QCX_U1, nc, 1, 1, false, true); return true; }
    if (base == "U2") { gate(c, adj ? RBK_QCX_U2_ADJ : RBK_QCX_U2, nc, 1, 2); return true; }
    if (base == "U3") { gate(c, adj ? RBK_QCX_U3_ADJ : RBK_QCX_U3, nc, 1, 3); return true; }
    if (base == "R") { gate(c, adj ? RBK_QCX_R_ADJ : RBK_QCX_R, nc, 1, 1, true, true); return true; }
    if (base == "+X" && !adj) { gate(c, RBK_QCX_ROTX, nc, 1, 0); return true; }
    if (base == "-X" && !adj) { gate(c, RBK_QCX_ROTX_ADJ, nc, 1, 0); return true; }
    if (base == "+Y" && !adj) { gate(c, RBK_QCX_ROTY, nc, 1, 0); return true; }
    if (base == "-Y" && !adj) { gate(c, RBK_QCX_ROTY_ADJ, nc, 1, 0); return true; }
    if (base == "ESWAP") { gate(c, adj ? RBK_QCX_ESWAP_ADJ : RBK_QCX_ESWAP, nc, 2, 1); return true; }
    if (m.size() >= 2 && m[0] == 'E') {
      const int kinds[3][2] = {{RBK_QCX_EX, RBK_QCX_EX_ADJ}, {RBK_QCX_EY, RBK_QCX_EY_ADJ}, {RBK_QCX_EZ, RBK_QCX_EZ_ADJ}};
      const char letters[3] = {'X', 'Y', 'Z'};
      for (int l = 0; l < 3; ++l) {
        if (int k = multiplicity(m, 1, letters[l], adj); k >= 1) {
          gate(c, kinds[l][adj ? 1 : 0], nc, k, 1);
          return true;
        }
      }
    }
    return false;
  }

  // Control prefixes (interpret_controlled_gates, interpreter.cpp:3341-3370):
  // "CC..C<gate>" has one control per C; "C<n><gate>" has n; a single "C" has one.
  bool controlled(const columns& c, const std::string& m)
  {
    size_t cs = 0;
    while (cs < m.size() && m[cs] == 'C') ++cs;
    size_t digits_end = 1;
    while (digits_end < m.size() && std::isdigit(static_cast<unsigned char>(m[digits_end]))) ++digits_end;
    int nc;
    std::string rest;
    if (cs > 1) {
      nc = static_cast<int>(cs);
      rest = m.substr(cs);
    } else if (digits_end > 1) {
      nc = std::atoi(m.substr(1, digits_end - 1).c_str());
      rest = m.substr(digits_end);
    } else {
      nc = 1;
      rest = m.substr(1);
    }
    if (nc <= 0 || rest.empty()) return false;
    return gate_mnemonic(c, rest, nc);
  }

  void statement(columns c)
  {
    c[0] = upper(c[0]);
    const std::string& m = c[0];
    auto word = [&](size_t i) { return i < c.size() ? upper(c[i]) : std::string{}; };
    if (m == "QUBITS") {
      expect(c, 2);
      const uint64_t n = to_unsigned(c[1]);
      if (n < 1 || n > 34) bad("QUBITS must be between 1 and 34");
      prog.num_qubits = static_cast<int>(n);
      return;
    }
    if (m == "CIRCUITS") {  // bra resizes its circuit list (interpreter.cpp:411-419)
      expect(c, 2);
      const uint64_t n = to_unsigned(c[1]);
      if (n < 1 || n > 64) bad("CIRCUITS must be between 1 and 64");
      if (static_cast<int>(n) <= circuit) bad("CIRCUITS leaves out the current circuit");
      prog.num_circuits = static_cast<int>(n);
      return;
    }
    if (m == "INITIAL") {  // INITIAL STATE v
      if (c.size() != 3 || word(1) != "STATE") bad("expected INITIAL STATE <value>");
      prog.initial_state = to_unsigned(c[2]);
      return;
    }
    if (m == "BIT") {  // BIT ASSIGNMENT: the initial permutation of MPI builds; nompi ignores it
      if (c.size() < 2 || word(1) != "ASSIGNMENT") bad("expected BIT ASSIGNMENT <qubits>");
      if (prog.num_qubits >= 0 && c.size() != 2 + static_cast<size_t>(prog.num_qubits))
        bad("BIT ASSIGNMENT needs one entry per qubit");
      for (size_t i = 2; i < c.size(); ++i) qubit(c[i]);
      return;
    }
    if (m == "MPIPROCESSES" || m == "MPISWAPBUFFER") return;
    if (m == "DEPOLARIZING" || m == "PERMUTATION" || m == "RANDOM" || m == "SEND" ||
        m == "RECEIVE" || m == "BROADCAST" || m == "GATHER" || m == "SCATTER" || m == "JUMP" || m == "JUMPIF" ||
        m.front() == '@')
      unsupported("'" + m + "' is not supported");
    if (prog.num_qubits < 0) bad("QUBITS must come first");
    if (m == "EXIT") {
      expect(c, 1);
      prog.code.push_back(blank(RBK_QCX_EXIT, line));
      done = true;  // bra stops reading at EXIT (interpreter.cpp:579-590)
      return;
    }
    if (m == "BEGIN") {
      const std::string w = word(1);
      if (w == "MEASUREMENT") {
        auto in = blank(RBK_QCX_MEASUREMENT, line);
        in.ints[0] = 3;
        prog.code.push_back(in);
      } else if (w == "FUSION") {
        prog.code.push_back(blank(RBK_QCX_BEGIN_FUSION, line));
      } else if (w == "CIRCUIT") {
        if (c.size() != 3 || in_circuit) bad("expected BEGIN CIRCUIT <index> outside another circuit block");
        const uint64_t k = to_unsigned(c[2]);
        if (k >= static_cast<uint64_t>(prog.num_circuits)) bad("circuit index " + c[2] + " is not below CIRCUITS");
        circuit = static_cast<int>(k);
        in_circuit = true;
      } else if (w == "LEARNING") {
        unsupported("BEGIN " + w + " is not supported");
      } else {
        bad("unknown BEGIN statement");
      }
      return;
    }
    if (m == "END") {
      const std::string w = word(1);
      if (w == "FUSION") prog.code.push_back(blank(RBK_QCX_END_FUSION, line));
      else if (w == "CIRCUIT") {
        if (!in_circuit) bad("END CIRCUIT without BEGIN CIRCUIT");
        circuit = 0;
        in_circuit = false;
      }
      else bad("unknown END statement");
      return;
    }
    if (m == "DO") {
      const std::string w = word(1);
      if (w == "MEASUREMENT") {
        if (c.size() > 3) bad("DO MEASUREMENT takes at most one precision");
        auto in = blank(RBK_QCX_MEASUREMENT, line);
        in.ints[0] = c.size() == 3 ? to_int(c[2]) : 3;
        prog.code.push_back(in);
      } else if (w == "AMPLITUDES") {
        auto in = blank(RBK_QCX_AMPLITUDES, line);
        std::vector<uint64_t> idx;
        for (size_t i = 2; i < c.size(); ++i) {
          const uint64_t v = to_unsigned(c[i]);
          if (v >= (1ull << prog.num_qubits)) bad("amplitude index " + c[i] + " is out of range");
          idx.push_back(v);
        }
        in.num_values = static_cast<int32_t>(idx.size());
        for (size_t i = 0; i < idx.size() && i < RBK_QCX_MAX_VALUES; ++i) in.values[i] = idx[i];
        prog.amplitude_lists.resize(prog.code.size() + 1);
        prog.amplitude_lists[prog.code.size()] = std::move(idx);
        prog.code.push_back(in);
      } else {
        bad("unknown DO statement");
      }
      return;
    }
    if (m == "GENERATE") {  // GENERATE EVENTS n seed; bra stops reading here (interpreter.cpp:764-785)
      if (c.size() != 4 || word(1) != "EVENTS") bad("expected GENERATE EVENTS <events> <seed>");
      auto in = blank(RBK_QCX_GENERATE_EVENTS, line);
      in.ints[0] = to_int(c[2]);
      in.ints[1] = to_int(c[3]);
      if (in.ints[0] < 0 || in.ints[0] > (1 << 30)) bad("number of events out of range");
      prog.code.push_back(in);
      done = true;
      return;
    }
    if (m == "VAR") {  // VAR name PAULISS [size] (interpreter.cpp:1966-1994)
      if (c.size() != 3 && c.size() != 4) bad("expected VAR <name> <type> [<size>]");
      const std::string name = upper(c[1]), type = upper(c[2]);
      if (type != "PAULISS") unsupported("VAR of type " + type + " (only PAULISS variables are supported)");
      if (!valid_name(name) || name.find(':') != std::string::npos) bad("'" + c[1] + "' is not a variable name");
      auto in = blank(RBK_QCX_VAR, line);
      in.ints[0] = c.size() == 4 ? to_int(c[3]) : 1;
      if (in.ints[0] <= 0) bad("the size of a variable must be positive");
      copy_text(in, name);
      prog.code.push_back(in);
      return;
    }
    if (m == "LET") {  // LET lhs op rhs (interpreter.cpp:1996-2027)
      expect(c, 4);
      const std::string lhs = upper(c[1]), rhs = upper(c[3]);
      auto in = blank(RBK_QCX_LET, line);
      const std::string& op = c[2];
      in.ints[0] = op == ":=" ? RBK_QCX_ASSIGN : op == "+=" ? RBK_QCX_PLUS : op == "-=" ? RBK_QCX_MINUS
                 : op == "*=" ? RBK_QCX_TIMES : op == "/=" ? RBK_QCX_DIVIDE : -1;
      if (in.ints[0] < 0) bad("unknown LET operation '" + op + "'");
      if (!valid_name(lhs)) bad("'" + c[1] + "' is not a variable");
      copy_text(in, lhs + " " + rhs);
      prog.code.push_back(in);
      return;
    }
    if (m == "EXPECTATION") {  // EXPECTATION <operator> q1 q2 ... (interpreter.cpp:3218-3240)
      if (c.size() < 3) bad("expected EXPECTATION <operator> <qubits>");
      auto in = blank(RBK_QCX_EXPECTATION, line);
      in.ints[1] = operator_column(c[1], c.size() - 2, in) ? 1 : 0;
      std::vector<uint32_t> seen;
      for (size_t i = 2; i < c.size(); ++i) {
        const uint32_t q = qubit(c[i]);
        if (std::find(seen.begin(), seen.end(), q) != seen.end()) bad("qubit " + c[i] + " appears twice");
        seen.push_back(q);
        in.targets[in.num_targets++] = q;
      }
      prog.code.push_back(in);
      return;
    }
    if (m == "INNERPROD" || m == "FIDELITY") {  // interpreter.cpp:3253-3330
      if (c.size() != 2 && c.size() < 4) bad("expected " + m + " (<circuit> | ALL) [<operator> <qubits>]");
      auto in = blank(m == "INNERPROD" ? RBK_QCX_INNERPROD : RBK_QCX_FIDELITY, line);
      const std::string& who = c[1];
      if (std::isdigit(static_cast<unsigned char>(who.front()))) {
        const uint64_t k = to_unsigned(who);
        if (k >= static_cast<uint64_t>(prog.num_circuits)) bad("circuit " + who + " is not below CIRCUITS");
        in.ints[0] = static_cast<int>(k) == circuit ? RBK_QCX_NONE : static_cast<int64_t>(k);
      } else {
        in.ints[0] = upper(who) == "ALL" ? RBK_QCX_ALL : RBK_QCX_NONE;
      }
      if (c.size() >= 4) {
        in.ints[1] = operator_column(c[2], c.size() - 3, in) ? 1 : 0;
        std::vector<uint32_t> seen;
        for (size_t i = 3; i < c.size(); ++i) {
          const uint32_t q = qubit(c[i]);
          if (std::find(seen.begin(), seen.end(), q) != seen.end()) bad("qubit " + c[i] + " appears twice");
          seen.push_back(q);
          in.targets[in.num_targets++] = q;
        }
      }
      prog.code.push_back(in);
      return;
    }
    if (m == "PRINT" || m == "PRINTLN") {
      auto in = blank(RBK_QCX_PRINT, line);
      std::string joined;
      for (size_t i = 1; i < c.size(); ++i) joined += (i > 1 ? " " : "") + c[i];
      if (joined.size() >= sizeof(in.text)) bad("PRINT arguments too long");
      std::memcpy(in.text, joined.c_str(), joined.size() + 1);
      in.ints[0] = m == "PRINTLN";
      prog.code.push_back(in);
      return;
    }
    if (m == "U" || m == "U+") {  // "U c1 c2 k" = CR c1 c2 k (docs/bra.md; interpreter.cpp:2747-2765)
      gate(c, m == "U" ? RBK_QCX_R : RBK_QCX_R_ADJ, 0, 2, 1, true, true);
      return;
    }
    if (m == "TOFFOLI") {  // TOFFOLI c1 c2 t (interpreter.cpp:3189-3197)
      gate(c, RBK_QCX_TOFFOLI, 2, 1, 0);
      return;
    }
    if (m == "M") {
      expect(c, 2);
      auto in = blank(RBK_QCX_PROJECTIVE, line);
      in.targets[in.num_targets++] = qubit(c[1]);
      prog.code.push_back(in);
      return;
    }
    if (m == "CLEAR" || m == "SET") {
      gate(c, m == "CLEAR" ? RBK_QCX_CLEAR : RBK_QCX_SET, 0, 1, 0);
      return;
    }
    if (m == "SHORBOX") {  // SHORBOX nx divisor base (interpreter.cpp:3208-3216)
      expect(c, 4);
      auto in = blank(RBK_QCX_GATE, line);
      in.kind = RBK_QCX_SHORBOX;
      const uint64_t nx = to_unsigned(c[1]);
      if (nx > static_cast<uint64_t>(prog.num_qubits)) bad("SHORBOX has more exponent qubits than qubits");
      in.params[0] = static_cast<double>(nx);
      in.params[1] = static_cast<double>(to_unsigned(c[2]));
      in.params[2] = static_cast<double>(to_unsigned(c[3]));
      in.ints[0] = static_cast<int64_t>(to_unsigned(c[2]));
      in.ints[1] = static_cast<int64_t>(to_unsigned(c[3]));
      prog.code.push_back(in);
      return;
    }
    if (gate_mnemonic(c, m, 0)) return;
    if (m.size() >= 2 && m[0] == 'C' && controlled(c, m)) return;
    bad("unknown mnemonic '" + m + "'");
  }

  void run(const std::string& text)
  {
    std::istringstream in(text);
    std::string raw;
    while (!done && std::getline(in, raw)) {
      ++line;
      raw.erase(std::find(raw.begin(), raw.end(), '!'), raw.end());
      columns c;
      std::istringstream ls(raw);
      std::string tok;
      while (ls >> tok) c.push_back(tok);
      if (c.empty()) continue;
      try {
        const size_t before = prog.code.size();
        statement(std::move(c));
        for (size_t i = before; i < prog.code.size(); ++i) prog.code[i].circuit = circuit;
      } catch (qcx_error const& e) {
        throw qcx_error(e.code, "line " + std::to_string(line) + ": " + e.what());
      }
    }
    if (prog.num_qubits < 0) bad("no QUBITS statement");
    if (prog.initial_state >= (1ull << prog.num_qubits)) bad("INITIAL STATE is out of range");
    for (const auto& in : prog.code)
      if ((in.op == RBK_QCX_INNERPROD || in.op == RBK_QCX_FIDELITY) && in.ints[0] >= prog.num_circuits)
        throw qcx_error(RBK_ERR_INVALID, "line " + std::to_string(in.line) + ": circuit index is not below CIRCUITS");
  }
};

}  // namespace

// ---- execution ---------------------------------------------------------------

namespace {

using clock_type = std::chrono::steady_clock;
using cplx = std::complex<double>;

// bra::state_detail::duration_to_second (bra/include/bra/state.hpp:118-123).
double seconds(clock_type::time_point from, clock_type::time_point to)
{
  return 0.000001 * static_cast<double>(std::chrono::duration_cast<std::chrono::microseconds>(to - from).count());
}

// bra::state_detail::integer_to_bits_string (bra/include/bra/state.hpp:100-117): most significant qubit first.
std::string bits(uint64_t v, int n)
{
  std::string s(static_cast<size_t>(n), '0');
  for (int b = 0; b < n; ++b)
    if ((v >> b) & 1) s[static_cast<size_t>(n - 1 - b)] = '1';
  return s;
}

// fmt's "{:^W}" centring: the odd padding character goes to the right.
std::string centre(const std::string& s, int width)
{
  const int pad = width - static_cast<int>(s.size());
  if (pad <= 0) return s;
  return std::string(static_cast<size_t>(pad / 2), ' ') + s + std::string(static_cast<size_t>(pad - pad / 2), ' ');
}

std::string fixed_with_space_sign(double v, int precision)
{
  char buf[64];
  std::snprintf(buf, sizeof(buf), "% .*f", precision, v);
  return buf;
}

void check(int rc)
{
  if (rc != RBK_OK) throw qcx_error(rc, rbk_last_error());
}

// bra::pauli_string_space (bra/include/bra/pauli_string_space.hpp:25-153): a
// linear combination of Pauli strings of one length; a new variable is the
// zero-qubit space {"" : 0}.
struct pauliss {
  size_t num_qubits = 0;
  std::map<std::string, cplx> terms{{std::string(), cplx{0.0, 0.0}}};
};

// One circuit of the program: bra's nompi_state with its wait reason
// (bra/include/bra/state.hpp wait_reason; bra/src/nompi_state.cpp:1204-1275).
struct circuit_ctx {
  rbk_state* s = nullptr;
  std::vector<size_t> code;  // indices into the program, in order
  size_t pc = 0;             // next instruction
  clock_type::time_point start, last;
  std::vector<int> last_outcomes;
  int last_measured = 0;
  cplx result{0.0, 0.0};
  bool in_fusion = false;
  const rbk_qcx_instruction* wait = nullptr;  // INNERPROD / FIDELITY this circuit waits on
  std::map<std::string, std::vector<pauliss>> variables;  // VAR name PAULISS [size]
};

struct runner {
  const rbk_qcx_program& prog;
  const rbk_qcx_options& opt;
  std::ostringstream out;
  std::vector<circuit_ctx> circ;
  circuit_ctx* cur = nullptr;  // the running circuit
  rbk_state* s = nullptr;      // its state

  runner(const rbk_qcx_program& p, const rbk_qcx_options& o) : prog(p), opt(o) {}

  void select(circuit_ctx& c)
  {
    cur = &c;
    s = c.s;
  }

  void mark(const char* what)
  {
    check(rbk_state_synchronize(s));
    const auto now = clock_type::now();
    if (opt.print_timing) out << what << " finished: " << seconds(cur->start, now) << " (" << seconds(cur->last, now) << ")\n";
    cur->last = now;
  }

  void gate(const rbk_qcx_instruction& g)
  {
    const uint32_t* t = g.targets;
    const uint32_t* c = g.num_controls ? g.controls : nullptr;
    const int nt = g.num_targets, nc = g.num_controls;
    const double* p = g.params;
    const bool adj = g.kind == RBK_QCX_SX_ADJ || g.kind == RBK_QCX_SY_ADJ || g.kind == RBK_QCX_SZ_ADJ ||
                     g.kind == RBK_QCX_U1_ADJ || g.kind == RBK_QCX_U2_ADJ || g.kind == RBK_QCX_U3_ADJ ||
                     g.kind == RBK_QCX_R_ADJ || g.kind == RBK_QCX_ROTX_ADJ || g.kind == RBK_QCX_ROTY_ADJ ||
                     g.kind == RBK_QCX_EX_ADJ || g.kind == RBK_QCX_EY_ADJ || g.kind == RBK_QCX_EZ_ADJ ||
                     g.kind == RBK_QCX_ESWAP_ADJ;
    switch (g.kind) {
      case RBK_QCX_H: check(rbk_hadamard(s, t[0], c, nc)); break;
      case RBK_QCX_NOT: check(rbk_pauli_x(s, t[0], c, nc)); break;
      case RBK_QCX_X: case RBK_QCX_Y: {
        if (nt == 1) check(g.kind == RBK_QCX_X ? rbk_pauli_x(s, t[0], c, nc) : rbk_pauli_y(s, t[0], c, nc));
        else check(rbk_pauli_string(s, std::string(static_cast<size_t>(nt), g.kind == RBK_QCX_X ? 'X' : 'Y').c_str(), t, nt, c, nc));
        break;
      }
      case RBK_QCX_Z:
        if (nt == 0) check(rbk_pauli_z(s, g.controls, nc));
        else check(rbk_pauli_string(s, std::string(static_cast<size_t>(nt), 'Z').c_str(), t, nt, c, nc));
        break;
      case RBK_QCX_SWAP: check(rbk_swap(s, t[0], t[1], c, nc)); break;
      case RBK_QCX_SX: case RBK_QCX_SX_ADJ: check(rbk_sqrt_pauli_x(s, adj, t[0], c, nc)); break;
      case RBK_QCX_SY: case RBK_QCX_SY_ADJ: check(rbk_sqrt_pauli_y(s, adj, t[0], c, nc)); break;
      case RBK_QCX_SZ: case RBK_QCX_SZ_ADJ:
        if (nt == 0) check(rbk_phase_shift_coeff(s, 0.0, adj ? -1.0 : 1.0, g.controls, nc));
        else check(rbk_sqrt_pauli_z(s, adj, t, nt, c, nc));
        break;
      case RBK_QCX_U1: case RBK_QCX_U1_ADJ: {
        // ket::gate::phase_shift(phase) multiplies by exp_i(phase); adj_ by its conjugate
        const cplx e = std::exp(cplx{0.0, p[0]});
        const cplx coeff = adj ? std::conj(e) : e;
        check(rbk_phase_shift_coeff(s, coeff.real(), coeff.imag(), g.controls, nc));
        break;
      }
      case RBK_QCX_U2:
        check(rbk_phase_shift2(s, p[0], p[1], t[0], c, nc));
        break;
      case RBK_QCX_U3:
        check(rbk_phase_shift3(s, p[0], p[1], p[2], t[0], c, nc));
        break;
      case RBK_QCX_U2_ADJ: case RBK_QCX_U3_ADJ: {
        // U3(theta, phi, lambda)^dagger = [[cos, e^{-i phi} sin], [-e^{-i lambda} sin, e^{-i(phi+lambda)} cos]]
        // (theta/2 inside cos, sin; U2 is U3 with theta = pi/2, phase_shift.hpp:660-709, :1200-1254)
        const double half = g.kind == RBK_QCX_U2_ADJ ? 0.25 * 3.141592653589793238462643383279502884 : 0.5 * p[0];
        const double phi = g.kind == RBK_QCX_U2_ADJ ? p[0] : p[1];
        const double lam = g.kind == RBK_QCX_U2_ADJ ? p[1] : p[2];
        const double cs = g.kind == RBK_QCX_U2_ADJ ? 0.7071067811865475244008443621048490393 : std::cos(half);
        const double sn = g.kind == RBK_QCX_U2_ADJ ? 0.7071067811865475244008443621048490393 : std::sin(half);
        const cplx m00{cs, 0.0}, m01 = std::exp(cplx{0.0, -phi}) * sn, m10 = -std::exp(cplx{0.0, -lam}) * sn,
                   m11 = std::exp(cplx{0.0, -(phi + lam)}) * cs;
        const double m[8] = {m00.real(), m00.imag(), m01.real(), m01.imag(), m10.real(), m10.imag(), m11.real(), m11.imag()};
        check(rbk_apply_matrix2(s, m, t[0], c, nc));
        break;
      }
      case RBK_QCX_R: case RBK_QCX_R_ADJ: {
        const int k = static_cast<int>(p[0]);
        check(rbk_controlled_phase_shift_k(s, adj ? -k : k, g.controls, nc));
        break;
      }
      case RBK_QCX_ROTX: case RBK_QCX_ROTX_ADJ: check(rbk_x_rotation_half_pi(s, adj, t[0], c, nc)); break;
      case RBK_QCX_ROTY: case RBK_QCX_ROTY_ADJ: check(rbk_y_rotation_half_pi(s, adj, t[0], c, nc)); break;
      case RBK_QCX_EX: case RBK_QCX_EX_ADJ: case RBK_QCX_EY: case RBK_QCX_EY_ADJ: case RBK_QCX_EZ: case RBK_QCX_EZ_ADJ: {
        const double phase = adj ? -p[0] : p[0];  // adj_exponential_pauli_*: exp(-i theta P)
        const char letter = (g.kind <= RBK_QCX_EX_ADJ) ? 'X' : (g.kind <= RBK_QCX_EY_ADJ) ? 'Y' : 'Z';
        if (nt == 1) {
          if (letter == 'X') check(rbk_exponential_pauli_x(s, phase, t[0], c, nc));
          else if (letter == 'Y') check(rbk_exponential_pauli_y(s, phase, t[0], c, nc));
          else check(rbk_exponential_pauli_z(s, phase, t[0], c, nc));
        } else {
          check(rbk_exponential_pauli_string(s, phase, std::string(static_cast<size_t>(nt), letter).c_str(), t, nt, c, nc));
        }
        break;
      }
      case RBK_QCX_ESWAP: case RBK_QCX_ESWAP_ADJ: check(rbk_exponential_swap(s, adj ? -p[0] : p[0], t[0], t[1], c, nc)); break;
      case RBK_QCX_TOFFOLI: check(rbk_pauli_x(s, t[0], g.controls, 2)); break;
      case RBK_QCX_CLEAR: check(rbk_clear(s, t[0])); break;
      case RBK_QCX_SET: check(rbk_set(s, t[0])); break;
      case RBK_QCX_SHORBOX:
        check(rbk_shor_box(s, static_cast<uint32_t>(p[0]), static_cast<uint64_t>(g.ints[0]), static_cast<uint64_t>(g.ints[1])));
        break;
      default: throw qcx_error(RBK_ERR_INVALID, "unknown gate kind");
    }
  }

  // bra::state::measurement (bra/src/state.cpp:1980-2034): the printed numbers are
  // 0.5 - <S> of each axis, i.e. the probability-like "qubit value" in [0, 1].
  void measurement(int precision)
  {
    mark("Operations");
    std::vector<double> spins(static_cast<size_t>(3 * prog.num_qubits));
    check(rbk_spin_expectation_values(s, spins.data()));
    out << "Expectation values of spins:\n";
    if (precision > 0) {
      const int width = std::max(precision + 3, 8);
      out << centre("<Qx>", width) << ' ' << centre("<Qy>", width) << ' ' << centre("<Qz>", width) << '\n';
      for (int q = 0; q < prog.num_qubits; ++q)
        out << centre(fixed_with_space_sign(0.5 - spins[3 * q], precision), width) << ' '
            << centre(fixed_with_space_sign(0.5 - spins[3 * q + 1], precision), width) << ' '
            << centre(fixed_with_space_sign(0.5 - spins[3 * q + 2], precision), width) << '\n';
    } else {
      out << "<Qx> <Qy> <Qz>\n";
      std::ostringstream vals;
      if (precision < 0) vals << std::setprecision(-precision);
      for (int q = 0; q < prog.num_qubits; ++q)
        vals << (0.5 - spins[3 * q]) << ' ' << (0.5 - spins[3 * q + 1]) << ' ' << (0.5 - spins[3 * q + 2]) << '\n';
      out << vals.str();
    }
    mark("Expectation values");
  }

  // bra::nompi_state::do_amplitudes (bra/src/nompi_state.cpp:1108-1133): "bits => re + im i".
  void amplitudes(const std::vector<uint64_t>& indices)
  {
    mark("Operations");
    const uint64_t size = 1ull << prog.num_qubits;
    int precision = RBK_C128;
    check(rbk_state_precision(s, &precision));
    auto print_range = [&](uint64_t first, uint64_t count, bool newline_each) {
      std::vector<double> buf(2 * count);
      std::vector<float> fbuf;
      if (precision == RBK_C128) check(rbk_state_download(s, buf.data(), first, count));
      else {
        fbuf.resize(2 * count);
        check(rbk_state_download(s, fbuf.data(), first, count));
      }
      for (uint64_t i = 0; i < count; ++i) {
        if (!newline_each && first + i > 0) out << '\n';
        out << bits(first + i, prog.num_qubits) << " => ";
        if (precision == RBK_C128) out << buf[2 * i] << " + " << buf[2 * i + 1] << " i";
        else out << fbuf[2 * i] << " + " << fbuf[2 * i + 1] << " i";
        if (newline_each) out << '\n';
      }
    };
    if (indices.empty()) {
      const uint64_t chunk = 1ull << 20;
      for (uint64_t first = 0; first < size; first += chunk) print_range(first, std::min(chunk, size - first), false);
      out << '\n';
    } else {
      for (uint64_t idx : indices) print_range(idx, 1, true);
    }
    mark("Amplitudes");
  }

  void generate_events(int num, int64_t seed)
  {
    mark("Operations");
    std::vector<uint64_t> ev(static_cast<size_t>(num));
    check(rbk_generate_events(s, num, seed, ev.data()));
    out << "Events:\n";
    for (int i = 0; i < num; ++i) out << i << ' ' << bits(ev[static_cast<size_t>(i)], prog.num_qubits) << '\n';
    mark("Events");
  }

  void exit_measure()
  {
    mark("Operations");
    uint64_t v = 0;
    check(rbk_measure(s, &v));
    out << "Measurement result: " << v << '\n';
    mark("Measurement");
  }

  // ---- PAULISS variables (bra/src/state.cpp:400-490, :977-998) ----
  // NAME or NAME:index of circuit c.
  pauliss& variable(circuit_ctx& c, const std::string& ref)
  {
    const size_t colon = ref.find(':');
    const std::string name = ref.substr(0, colon);
    const auto it = c.variables.find(name);
    if (it == c.variables.end()) throw qcx_error(RBK_ERR_UNSUPPORTED, "'" + name + "' is not a PAULISS variable of this circuit");
    const int64_t index = colon == std::string::npos ? 0 : to_int(ref.substr(colon + 1));
    if (index < 0 || static_cast<size_t>(index) >= it->second.size())
      throw qcx_error(RBK_ERR_INVALID, "index of '" + name + "' out of range");
    return it->second[static_cast<size_t>(index)];
  }

  // bra::state::to_pauli_string_space: a :PAULIS:<s> literal (coefficient 1) or a variable.
  pauliss pauli_value(circuit_ctx& c, const std::string& rhs)
  {
    if (rhs.rfind(":PAULIS:", 0) == 0 && rhs.size() > 8) {
      pauliss v;
      const std::string str = rhs.substr(8);
      for (char ch : str)
        if (ch != 'I' && ch != 'X' && ch != 'Y' && ch != 'Z') throw qcx_error(RBK_ERR_INVALID, "Pauli strings use I, X, Y, Z");
      v.num_qubits = str.size();
      v.terms = {{str, cplx{1.0, 0.0}}};
      return v;
    }
    if (rhs.front() == ':') throw qcx_error(RBK_ERR_UNSUPPORTED, "'" + rhs + "' is not a Pauli-string-space value");
    return variable(c, rhs);
  }

  // bra::state::to_complex for the literal forms.
  cplx complex_value(const circuit_ctx& c, const std::string& rhs) const
  {
    if (rhs == ":COMPLEX") return cplx{0.0, 0.0};
    if (rhs == ":I") return cplx{0.0, 1.0};
    if (rhs == ":MINUS_I") return cplx{0.0, -1.0};
    if (rhs == ":RESULT") return c.result;
    if (rhs.rfind(":COMPLEX:", 0) == 0 && rhs.size() > 9) {
      const std::string v = rhs.substr(9);
      const char f = v.front();
      if (std::isdigit(static_cast<unsigned char>(f)) || f == '+' || f == '-' || f == '.') return cplx{to_real(v), 0.0};
    }
    throw qcx_error(RBK_ERR_UNSUPPORTED, "'" + rhs + "' is not a supported complex value (:COMPLEX:<literal>, :I, :MINUS_I, :RESULT)");
  }

  void declare(const rbk_qcx_instruction& in)
  {
    const std::string name(in.text);
    if (cur->variables.count(name)) throw qcx_error(RBK_ERR_INVALID, "variable '" + name + "' is declared twice");
    cur->variables[name] = std::vector<pauliss>(static_cast<size_t>(in.ints[0]));
  }

  // bra::state::invoke_assign_operation on a PAULISS left side.
  void let(const rbk_qcx_instruction& in)
  {
    const std::string text(in.text);
    const size_t space = text.find(' ');
    const std::string lhs_ref = text.substr(0, space), rhs = text.substr(space + 1);
    pauliss& lhs = variable(*cur, lhs_ref);
    const int op = static_cast<int>(in.ints[0]);
    if (op == RBK_QCX_ASSIGN) {
      lhs = pauli_value(*cur, rhs);
    } else if (op == RBK_QCX_PLUS || op == RBK_QCX_MINUS) {
      for (const auto& term : pauli_value(*cur, rhs).terms) {
        if (term.first.size() != lhs.num_qubits)
          throw qcx_error(RBK_ERR_INVALID, term.first + " is not a valid Pauli string or has wrong length");
        if (op == RBK_QCX_PLUS) lhs.terms[term.first] += term.second;
        else lhs.terms[term.first] -= term.second;
      }
    } else {
      const cplx v = complex_value(*cur, rhs);
      for (auto& term : lhs.terms) term.second = op == RBK_QCX_TIMES ? term.second * v : term.second / v;
    }
  }

  // The operator of EXPECTATION / INNERPROD / FIDELITY as terms over all
  // qubits: character k of each string acts on the k-th listed qubit.
  void operator_terms(circuit_ctx& c, const rbk_qcx_instruction& in, std::string& strings, std::vector<double>& coeffs)
  {
    pauliss op;
    if (in.ints[1]) {
      op = variable(c, in.text);
      if (op.num_qubits != static_cast<size_t>(in.num_targets))
        throw qcx_error(RBK_ERR_INVALID, "the operator has " + std::to_string(op.num_qubits) + " qubits, " +
                                           std::to_string(in.num_targets) + " are listed");
    } else {
      op.num_qubits = static_cast<size_t>(in.num_targets);
      op.terms = {{std::string(in.text), cplx{1.0, 0.0}}};
    }
    strings.clear();
    coeffs.clear();
    for (const auto& term : op.terms) {
      std::string full(static_cast<size_t>(prog.num_qubits), 'I');
      for (int k = 0; k < in.num_targets; ++k) full[in.targets[k]] = term.first[static_cast<size_t>(k)];
      strings += full;
      coeffs.push_back(term.second.real());
      coeffs.push_back(term.second.imag());
    }
  }

  // EXPECTATION <operator> q...: sum over the operator's terms of coefficient x <psi|P|psi>.
  void expectation(const rbk_qcx_instruction& in)
  {
    std::string strings;
    std::vector<double> coeffs;
    operator_terms(*cur, in, strings, coeffs);
    double r[2];
    check(rbk_expectation_pauli(s, static_cast<int>(coeffs.size() / 2), strings.c_str(), coeffs.data(), r));
    cur->result = cplx{r[0], r[1]};
  }

  // bra::state::generate_print_string (bra/src/state.cpp:495-538) for literals and built-ins.
  void print(const rbk_qcx_instruction& in)
  {
    std::istringstream args(in.text);
    std::string a;
    bool first = true;
    while (args >> a) {
      if (!first) out << ' ';
      first = false;
      const char f = a.front();
      if (std::isdigit(static_cast<unsigned char>(f)) || f == '+' || f == '-' || f == '.') { out << a; continue; }
      if (f != ':') continue;  // classical variables do not exist here
      if (a == ":RESULT") out << cur->result;
      else if (a == ":I") out << cplx{0.0, 1.0};
      else if (a == ":MINUS_I") out << cplx{0.0, -1.0};
      else if (a == ":COMPLEX") out << cplx{0.0, 0.0};
      else if (a == ":INT") out << 0;
      else if (a == ":OUTCOME") out << cur->last_outcomes[static_cast<size_t>(cur->last_measured)];
      else if (a == ":OUTCOMES") out << cur->last_outcomes.front();
      else if (a.rfind(":OUTCOMES:", 0) == 0) {
        const int64_t q = to_int(a.substr(10));
        if (q < 0 || q >= prog.num_qubits) throw qcx_error(RBK_ERR_INVALID, "line " + std::to_string(in.line) + ": qubit out of range");
        out << cur->last_outcomes[static_cast<size_t>(q)];
      } else {
        out << to_real(a);
      }
    }
    if (in.ints[0]) out << '\n';
  }

  // ket::inner_product(a, b[, H]) = <b| [H] |a>, or its squared modulus; the
  // operator is circuit owner's.
  cplx overlap(rbk_state* a, rbk_state* b, circuit_ctx& owner, const rbk_qcx_instruction& in)
  {
    double r[2] = {0.0, 0.0};
    try {
      if (in.text[0]) {
        std::string strings;
        std::vector<double> coeffs;
        operator_terms(owner, in, strings, coeffs);
        check(rbk_inner_product_pauli(a, b, static_cast<int>(coeffs.size() / 2), strings.c_str(), coeffs.data(), r));
      } else {
        check(rbk_inner_product(a, b, r));
      }
    } catch (qcx_error const& e) {
      throw qcx_error(e.code, "line " + std::to_string(in.line) + ": " + e.what());
    }
    if (in.op == RBK_QCX_FIDELITY) return cplx{r[0] * r[0] + r[1] * r[1], 0.0};
    return cplx{r[0], r[1]};
  }

  // Runs the selected circuit until it finishes or waits (bra::interpreter::apply_circuit,
  // bra/src/interpreter.cpp:851-871).
  void run_circuit()
  {
    circuit_ctx& c = *cur;
    while (c.pc < c.code.size() && !c.wait) {
      const size_t i = c.code[c.pc++];
      const auto& in = prog.code[i];
      try {
        switch (in.op) {
          case RBK_QCX_GATE: gate(in); break;
          case RBK_QCX_BEGIN_FUSION: check(rbk_begin_fusion(s)); c.in_fusion = true; break;
          case RBK_QCX_END_FUSION: check(rbk_end_fusion(s)); c.in_fusion = false; break;
          case RBK_QCX_MEASUREMENT: measurement(static_cast<int>(in.ints[0])); break;
          case RBK_QCX_AMPLITUDES:
            amplitudes(i < prog.amplitude_lists.size() ? prog.amplitude_lists[i] : std::vector<uint64_t>{});
            break;
          case RBK_QCX_GENERATE_EVENTS: generate_events(static_cast<int>(in.ints[0]), in.ints[1]); break;
          case RBK_QCX_EXIT: exit_measure(); break;
          case RBK_QCX_PROJECTIVE: {
            int outcome = 0;
            check(rbk_projective_measurement(s, in.targets[0], &outcome));
            c.last_outcomes[in.targets[0]] = outcome;
            c.last_measured = static_cast<int>(in.targets[0]);
            break;
          }
          case RBK_QCX_EXPECTATION: expectation(in); break;
          case RBK_QCX_PRINT: print(in); break;
          case RBK_QCX_VAR: declare(in); break;
          case RBK_QCX_LET: let(in); break;
          case RBK_QCX_INNERPROD: case RBK_QCX_FIDELITY:
            // bra::state::inner_product / fidelity refuse a fused block (bra/src/state.cpp:2133-2170)
            if (c.in_fusion) throw qcx_error(RBK_ERR_UNSUPPORTED, "INNERPROD / FIDELITY inside BEGIN/END FUSION");
            if (in.ints[0] != RBK_QCX_NONE) c.wait = &in;
            break;
          case RBK_QCX_NOOP: break;
          default: throw qcx_error(RBK_ERR_INVALID, "unknown instruction");
        }
      } catch (qcx_error const& e) {
        throw qcx_error(e.code, "line " + std::to_string(in.line) + ": " + e.what());
      }
    }
  }

  // bra's nompi scheduler (bra/src/bra.cpp:329-760): run every circuit that is
  // not waiting; then evaluate the pairs that wait on each other (the lower
  // circuit index first, as the scan meets it), or, when every circuit waits
  // on the same ALL instruction, that collective.
  void execute()
  {
    const int nc = static_cast<int>(circ.size());
    auto kind_of = [](const rbk_qcx_instruction* w) {
      // 0: pair INNERPROD, 1: pair INNERPROD with operator, 2/3: FIDELITY; +4: ALL
      return (w->op == RBK_QCX_FIDELITY ? 2 : 0) + (w->text[0] ? 1 : 0) + (w->ints[0] == RBK_QCX_ALL ? 4 : 0);
    };
    while (true) {
      for (auto& c : circ)
        if (!c.wait) {
          select(c);
          run_circuit();
        }
      if (std::none_of(circ.begin(), circ.end(), [](const circuit_ctx& c) { return c.wait != nullptr; })) break;
      bool progress = false;
      int all_kind = -1;  // the ALL kind every circuit waits on, if any
      bool all_same = true;
      for (int k = 0; k < nc; ++k) {
        circuit_ctx& c = circ[static_cast<size_t>(k)];
        if (!c.wait) { all_same = false; continue; }
        const int kind = kind_of(c.wait);
        if (kind >= 4) {
          if (all_kind < 0) all_kind = kind;
          else if (all_kind != kind) all_same = false;
          continue;
        }
        all_same = false;
        const int other = static_cast<int>(c.wait->ints[0]);
        circuit_ctx& o = circ[static_cast<size_t>(other)];
        if (!o.wait || kind_of(o.wait) != kind || o.wait->ints[0] != k) continue;
        const cplx r = overlap(c.s, o.s, c, *c.wait);  // <Psi_other| [H] |Psi_k>
        c.result = r;
        o.result = std::conj(r);
        c.wait = o.wait = nullptr;
        progress = true;
      }
      if (!progress && all_same && all_kind >= 0) {
        const rbk_qcx_instruction& in = *circ.front().wait;  // the operator comes from circuit 0
        for (auto& c : circ) c.result = overlap(circ.front().s, c.s, circ.front(), in);  // <Psi_c| [H] |Psi_0>
        for (auto& c : circ) c.wait = nullptr;
        progress = true;
      }
      if (!progress) throw qcx_error(RBK_ERR_STATE, "circuits wait on INNERPROD / FIDELITY partners that never arrive");
    }
  }
};

template <typename F>
int guard(F&& f)
{
  try {
    return f();
  } catch (qcx_error const& e) {
    return rbk::set_last_error(e.code, e.what());
  } catch (std::bad_alloc const&) {
    return rbk::set_last_error(RBK_ERR_OOM, "host memory exhausted");
  } catch (std::exception const& e) {
    return rbk::set_last_error(RBK_ERR_STATE, e.what());
  }
}

}  // namespace

extern "C" {

void rbk_qcx_default_options(rbk_qcx_options* o)
{
  if (!o) return;
  o->precision = RBK_C128;
  o->device = 0;
  o->seed = 1;
  o->deferred = 1;
  o->print_timing = 1;
}

int rbk_qcx_parse(const char* text, size_t length, rbk_qcx_program** out)
{
  return guard([&]() -> int {
    if (!out || (!text && length)) return rbk::set_last_error(RBK_ERR_INVALID, "null argument");
    *out = nullptr;
    auto* p = new rbk_qcx_program;
    try {
      parser ps{*p};
      ps.run(std::string(text ? text : "", length));
    } catch (...) {
      delete p;
      throw;
    }
    p->amplitude_lists.resize(p->code.size());
    *out = p;
    return RBK_OK;
  });
}

int rbk_qcx_destroy(rbk_qcx_program* p)
{
  delete p;
  return RBK_OK;
}

int rbk_qcx_num_qubits(const rbk_qcx_program* p, int* out)
{
  if (!p || !out) return rbk::set_last_error(RBK_ERR_INVALID, "null argument");
  *out = p->num_qubits;
  return RBK_OK;
}

int rbk_qcx_num_circuits(const rbk_qcx_program* p, int* out)
{
  if (!p || !out) return rbk::set_last_error(RBK_ERR_INVALID, "null argument");
  *out = p->num_circuits;
  return RBK_OK;
}

int rbk_qcx_initial_state(const rbk_qcx_program* p, uint64_t* out)
{
  if (!p || !out) return rbk::set_last_error(RBK_ERR_INVALID, "null argument");
  *out = p->initial_state;
  return RBK_OK;
}

int rbk_qcx_num_instructions(const rbk_qcx_program* p, int* out)
{
  if (!p || !out) return rbk::set_last_error(RBK_ERR_INVALID, "null argument");
  *out = static_cast<int>(p->code.size());
  return RBK_OK;
}

int rbk_qcx_get_instruction(const rbk_qcx_program* p, int index, rbk_qcx_instruction* out)
{
  if (!p || !out) return rbk::set_last_error(RBK_ERR_INVALID, "null argument");
  if (index < 0 || static_cast<size_t>(index) >= p->code.size()) return rbk::set_last_error(RBK_ERR_INVALID, "index out of range");
  *out = p->code[static_cast<size_t>(index)];
  return RBK_OK;
}

int rbk_qcx_run(const rbk_qcx_program* p, const rbk_qcx_options* options, char** text, rbk_state** state_out)
{
  return guard([&]() -> int {
    if (!p || !text) return rbk::set_last_error(RBK_ERR_INVALID, "null argument");
    *text = nullptr;
    if (state_out) *state_out = nullptr;
    rbk_qcx_options opt;
    rbk_qcx_default_options(&opt);
    if (options) opt = *options;
    runner r(*p, opt);
    r.circ.resize(static_cast<size_t>(p->num_circuits));
    for (size_t i = 0; i < p->code.size(); ++i) r.circ[static_cast<size_t>(p->code[i].circuit)].code.push_back(i);
    auto release = [&] {
      for (auto& c : r.circ)
        if (c.s) rbk_state_destroy(c.s);
    };
    try {
      // Circuit 0 takes the given seed, circuit k >= 1 the k-th draw of
      // std::mt19937_64(seed) (bra/src/bra.cpp:300-326).
      std::mt19937_64 seeds(opt.seed);
      const auto now = clock_type::now();
      for (size_t k = 0; k < r.circ.size(); ++k) {
        auto& c = r.circ[k];
        c.last_outcomes.assign(static_cast<size_t>(p->num_qubits), -1);  // ket::gate::outcome::unspecified
        c.start = c.last = now;
        check(rbk_state_create(p->num_qubits, opt.precision, p->initial_state, opt.device, &c.s));
        check(rbk_state_seed(c.s, k == 0 ? opt.seed : seeds()));
        check(rbk_state_set_deferred(c.s, opt.deferred));
      }
      r.execute();
      for (auto& c : r.circ) check(rbk_state_synchronize(c.s));
    } catch (...) {
      release();
      throw;
    }
    const std::string o = r.out.str();
    char* buf = static_cast<char*>(std::malloc(o.size() + 1));
    if (!buf) {
      release();
      return rbk::set_last_error(RBK_ERR_OOM, "host memory exhausted");
    }
    std::memcpy(buf, o.c_str(), o.size() + 1);
    *text = buf;
    if (state_out) {
      *state_out = r.circ.front().s;
      r.circ.front().s = nullptr;
    }
    release();
    return RBK_OK;
  });
}

void rbk_qcx_free_text(char* text) { std::free(text); }

}  // extern "C"
