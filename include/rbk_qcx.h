/* rbk_qcx.h -- bra's .qcx interpreter on the B200 engine (librbk.so).
 *
 * Replaces the nompi build of bra (bra/src/bra.cpp:290-330, bra::interpreter in
 * bra/src/interpreter.cpp:372-826, the output of bra::state::measurement /
 * amplitudes / generate_events / exit in bra/src/state.cpp:1980-2110): the same
 * .qcx text runs unchanged and prints what bra prints, with the state vector in
 * HBM.  Parsing follows bra: everything from '!' to the end of a line is a
 * comment, columns are split on white space, the mnemonic is case-insensitive,
 * qubits are unsigned integers, angles are decimal literals or the constants
 * :PI :HALF_PI :TWO_PI :ROOT_TWO :HALF_ROOT_TWO (also :REAL:<literal>).
 *
 * Supported: QUBITS, CIRCUITS n, BEGIN CIRCUIT k / END CIRCUIT, INITIAL STATE,
 * BIT ASSIGNMENT (accepted; the nompi build ignores it), MPIPROCESSES /
 * MPISWAPBUFFER (ignored), the gate set of docs/bra.md (I.., H, NOT, X/Y/Z and
 * their multi-qubit forms, SWAP, S/T, SX/SY/SZ.., U1/U2/U3, R, U,
 * +X/-X/+Y/-Y, EX/EY/EZ.., ESWAP, TOFFOLI, with "+" adjoints and C../Cn control
 * prefixes), M, CLEAR, SET, SHORBOX, BEGIN/END FUSION, BEGIN MEASUREMENT, DO
 * MEASUREMENT [p], DO AMPLITUDES [i ...], GENERATE EVENTS n seed, EXPECTATION
 * <operator> q..., INNERPROD / FIDELITY (k | ALL) [<operator> q...], PRINT /
 * PRINTLN of literals and built-in symbols (:RESULT, :OUTCOME, :OUTCOMES:i,
 * ...), EXIT.
 * Operators are Pauli-string-space values (bra/include/bra/pauli_string_space.hpp:25-153):
 * a :PAULIS:<s> literal, or a PAULISS variable (NAME or NAME:index) declared
 * with VAR name PAULISS [size] and built with LET (bra/src/state.cpp:400-490):
 * LET H := <pauliss>, LET H += <pauliss>, LET H -= <pauliss> (the strings of
 * the right side, all of H's length, added or subtracted term by term), LET H
 * *= <complex>, LET H /= <complex> (every coefficient; <complex> is
 * :COMPLEX:<literal>, :COMPLEX, :I, :MINUS_I or :RESULT).  Variables belong
 * to the circuit that declares them; an INNERPROD / FIDELITY operator is the
 * running circuit's (circuit 0's for ALL).
 * Several circuits run as bra's nompi build runs them (bra/src/bra.cpp:299-760):
 * one state each, circuit 0 seeded with the given seed and circuit k >= 1 with
 * the k-th draw of std::mt19937_64(seed); each circuit runs until it finishes or
 * reaches an INNERPROD / FIDELITY, and those are evaluated when their partner
 * (or, for ALL, every circuit) waits on the matching instruction.  Their value
 * goes to :RESULT: <Psi_k|Psi_c> (c the running circuit, k the partner; circuit
 * 0 for ALL), with <Psi_k| H |Psi_c> when an operator is given, and the squared
 * modulus for FIDELITY.
 * Not supported (RBK_ERR_UNSUPPORTED naming the line): the rest of the
 * classical layer -- INT / REAL / COMPLEX variables and LET on them, @label,
 * JUMP, JUMPIF, SEND, RECEIVE, BROADCAST, GATHER, SCATTER, PRINT of variables
 * -- DEPOLARIZING, PERMUTATION, RANDOM PERMUTATION.
 */
#ifndef RBK_QCX_H_INCLUDED
#define RBK_QCX_H_INCLUDED

#include <stddef.h>
#include <stdint.h>

#include "rbk.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct rbk_qcx_program rbk_qcx_program;

/* Instruction kinds after parsing. */
enum {
  RBK_QCX_GATE = 1,             /* gate: kind, targets, controls, params */
  RBK_QCX_BEGIN_FUSION = 2,
  RBK_QCX_END_FUSION = 3,
  RBK_QCX_MEASUREMENT = 4,      /* DO MEASUREMENT p / BEGIN MEASUREMENT: ints[0] = p */
  RBK_QCX_AMPLITUDES = 5,       /* DO AMPLITUDES: values[] (none: all) */
  RBK_QCX_GENERATE_EVENTS = 6,  /* ints[0] = events, ints[1] = seed */
  RBK_QCX_EXIT = 7,
  RBK_QCX_PROJECTIVE = 8,       /* M t */
  RBK_QCX_EXPECTATION = 9,      /* text = Pauli string, or with ints[1] = 1 the name of a PAULISS
                                   variable (NAME or NAME:index); targets = operated qubits */
  RBK_QCX_PRINT = 10,           /* text = arguments separated by one space; ints[0] = 1 for PRINTLN */
  RBK_QCX_NOOP = 11,            /* I, IC, C..I: MPI-only identities */
  RBK_QCX_INNERPROD = 12,       /* ints[0] = partner circuit, RBK_QCX_ALL or RBK_QCX_NONE; text = Pauli
                                   string (empty: no operator) or, with ints[1] = 1, a PAULISS variable
                                   as for EXPECTATION; targets = operated qubits */
  RBK_QCX_FIDELITY = 13,        /* as RBK_QCX_INNERPROD */
  RBK_QCX_VAR = 14,             /* VAR name PAULISS [size]: text = name, ints[0] = size */
  RBK_QCX_LET = 15              /* LET lhs op rhs on a PAULISS variable: text = "LHS RHS", ints[0] =
                                   RBK_QCX_ASSIGN ... RBK_QCX_DIVIDE */
};

/* LET operations (bra/include/bra/state.hpp assign_operation_type). */
enum { RBK_QCX_ASSIGN = 0, RBK_QCX_PLUS = 1, RBK_QCX_MINUS = 2, RBK_QCX_TIMES = 3, RBK_QCX_DIVIDE = 4 };

/* Partner of INNERPROD / FIDELITY: every circuit (ALL), or none -- bra does
 * nothing for the running circuit's own index or a column that is neither a
 * number nor ALL (bra/src/nompi_state.cpp:1204-1220). */
#define RBK_QCX_ALL (-1)
#define RBK_QCX_NONE (-2)

/* Gate kinds (the numbering of the oracle's reference leg, for tests). */
enum {
  RBK_QCX_H = 1, RBK_QCX_NOT = 2, RBK_QCX_X = 3, RBK_QCX_Y = 4, RBK_QCX_Z = 5, RBK_QCX_SWAP = 6,
  RBK_QCX_SX = 7, RBK_QCX_SX_ADJ = 8, RBK_QCX_SY = 9, RBK_QCX_SY_ADJ = 10, RBK_QCX_SZ = 11, RBK_QCX_SZ_ADJ = 12,
  RBK_QCX_U1 = 13, RBK_QCX_U1_ADJ = 14, RBK_QCX_U2 = 15, RBK_QCX_U2_ADJ = 16, RBK_QCX_U3 = 17, RBK_QCX_U3_ADJ = 18,
  RBK_QCX_R = 19, RBK_QCX_R_ADJ = 20, RBK_QCX_ROTX = 21, RBK_QCX_ROTX_ADJ = 22, RBK_QCX_ROTY = 23,
  RBK_QCX_ROTY_ADJ = 24, RBK_QCX_EX = 25, RBK_QCX_EX_ADJ = 26, RBK_QCX_EY = 27, RBK_QCX_EY_ADJ = 28,
  RBK_QCX_EZ = 29, RBK_QCX_EZ_ADJ = 30, RBK_QCX_ESWAP = 31, RBK_QCX_ESWAP_ADJ = 32, RBK_QCX_TOFFOLI = 33,
  RBK_QCX_CLEAR = 34, RBK_QCX_SET = 35, RBK_QCX_SHORBOX = 36
};

#define RBK_QCX_MAX_QUBITS 40
#define RBK_QCX_MAX_VALUES 40

/* One parsed instruction.  Gates whose qubits are all of control type in ket
 * (Z c, CZ, S, T, U1, R, U) hold every qubit in controls[] and none in
 * targets[].  Angles are in params[] as written (R / U / T: params[0] = k). */
typedef struct rbk_qcx_instruction {
  int32_t op;
  int32_t kind;
  int32_t line;
  int32_t num_targets;
  int32_t num_controls;
  int32_t num_values;
  int32_t circuit;     /* circuit the instruction belongs to (BEGIN CIRCUIT k; 0 outside) */
  uint32_t targets[RBK_QCX_MAX_QUBITS];
  uint32_t controls[RBK_QCX_MAX_QUBITS];
  double params[3];
  int64_t ints[2];
  uint64_t values[RBK_QCX_MAX_VALUES]; /* first RBK_QCX_MAX_VALUES amplitude indices */
  char text[256];
} rbk_qcx_instruction;

typedef struct rbk_qcx_options {
  int precision;     /* RBK_C128 (default) or RBK_C64 */
  int device;        /* CUDA device */
  uint64_t seed;     /* bra --seed: the state's generator (default 1) */
  int deferred;      /* 1: fused passes (default); 0: one pass per gate */
  int print_timing;  /* 1: bra's "... finished: t (dt)" lines (default); 0: leave them out */
} rbk_qcx_options;

/* Fills the defaults above. */
void rbk_qcx_default_options(rbk_qcx_options* options);

/* Parses .qcx text.  Errors: RBK_ERR_INVALID / RBK_ERR_UNSUPPORTED with
 * rbk_last_error() = "line N: ...". */
int rbk_qcx_parse(const char* text, size_t length, rbk_qcx_program** out);
int rbk_qcx_destroy(rbk_qcx_program* program);
int rbk_qcx_num_qubits(const rbk_qcx_program* program, int* out);
int rbk_qcx_num_circuits(const rbk_qcx_program* program, int* out);
int rbk_qcx_initial_state(const rbk_qcx_program* program, uint64_t* out);
int rbk_qcx_num_instructions(const rbk_qcx_program* program, int* out);
int rbk_qcx_get_instruction(const rbk_qcx_program* program, int index, rbk_qcx_instruction* out);

/* Runs the program on new states (one per circuit) and returns bra's standard
 * output in *text (NUL-terminated; release with rbk_qcx_free_text).
 * state_out, if not NULL, receives circuit 0's final state (release with
 * rbk_state_destroy); if the program ends with GENERATE EVENTS the state is
 * intact (bra leaves prefix sums in its buffer).  Circuits that wait on each
 * other in a way that never resolves (bra loops forever) give RBK_ERR_STATE. */
int rbk_qcx_run(const rbk_qcx_program* program, const rbk_qcx_options* options, char** text, rbk_state** state_out);
void rbk_qcx_free_text(char* text);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* RBK_QCX_H_INCLUDED */
