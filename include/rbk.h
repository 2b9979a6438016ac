/* rbk.h -- C ABI of the B200 state-vector engine (librbk.so).
 *
 * One state vector of 2^n amplitudes lives in one GPU's HBM, as
 * complex<double> (RBK_C128, n <= 33) or complex<float> (RBK_C64, n <= 34).
 * Gates are the ones of RIKEN-braket's ket library and bra's .qcx
 * instruction set; each entry point below names the reference function it
 * replaces.  Reference paths are relative to the RIKEN-braket project root.
 *
 * Conventions
 *  - Every function returns an rbk_status; 0 (RBK_OK) is success.  On failure
 *    rbk_last_error() returns a message for the calling thread.  No C++
 *    exception crosses this interface.
 *  - Qubit q is bit q of the amplitude index (ket::qubit, ket/include/ket/qubit.hpp:10-53).
 *    Control qubits are given as an array of qubit indices (ket::control).
 *  - Gate angles and coefficients are turned into gate coefficients on the
 *    host in double precision, with the same formulas as ket (std::sin,
 *    std::cos, std::exp(i theta)); kernels receive coefficients, never angles.
 *  - Gates are queued on the state and executed in fused passes when a result
 *    is read (download, reductions, rbk_state_synchronize, rbk_flush).  The
 *    queue is invisible except through timing: every read sees all gates
 *    issued before it.  rbk_state_set_deferred(s, 0) executes each gate as
 *    soon as it is issued (one pass per gate, like ket).
 *  - A state is used from one host thread at a time.  Every state has its own
 *    CUDA stream.  Host waits are bounded (RBK_ERR_TIMEOUT).
 */
#ifndef RBK_H
#define RBK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef enum rbk_status {
  RBK_OK = 0,
  RBK_ERR_INVALID = 1,      /* bad argument: qubit out of range, repeated qubit, null pointer, size */
  RBK_ERR_CUDA = 2,         /* a CUDA call failed (message has the CUDA error string) */
  RBK_ERR_OOM = 3,          /* device memory exhausted */
  RBK_ERR_TIMEOUT = 4,      /* a bounded host wait expired */
  RBK_ERR_UNSUPPORTED = 5,  /* operation not available for this precision / size */
  RBK_ERR_STATE = 6         /* call out of order, e.g. END FUSION without BEGIN FUSION */
} rbk_status;

typedef enum rbk_precision { RBK_C128 = 0, RBK_C64 = 1 } rbk_precision;

typedef struct rbk_state rbk_state;

/* Execution statistics of one state since creation (or the last reset_stats). */
typedef struct rbk_stats {
  uint64_t gates_issued;     /* gate calls accepted */
  uint64_t passes;           /* fused read+write passes over the whole state */
  uint64_t gate_launches;    /* unfused single-gate kernel launches */
  uint64_t reduction_passes; /* read-only passes (observables) */
  uint64_t relabel_passes;   /* passes that only moved qubits (layout changes) */
  uint64_t kernel_launches;  /* all kernels launched */
} rbk_stats;

const char* rbk_last_error(void);
int rbk_version(void);
/* Bytes of the parameter block that one fused-pass launch carries from the
 * host: the pass descriptor, passed by value as the kernel's constant
 * parameter.  No reference counterpart (the reference has no device); it
 * lets a caller account for the host->device bytes of a circuit, which are
 * passes x this figure plus the smaller parameters of other launches. */
int rbk_pass_descriptor_bytes(uint64_t* out);

/* ---- state lifecycle ------------------------------------------------------
 * Replaces std::vector<complex> state creation in bra::nompi_state
 * (bra/src/nompi_state.cpp:120-137, make_initial_data) and the single-process
 * ket::mpi::state<Complex, false> (ket/include/ket/mpi/state.hpp:1973-2100,
 * ctor :1990-2000): the state is |initial_index>. */
int rbk_state_create(int num_qubits, int precision, uint64_t initial_index, int device, rbk_state** out);
int rbk_state_destroy(rbk_state* s);
int rbk_state_num_qubits(const rbk_state* s, int* out);
int rbk_state_precision(const rbk_state* s, int* out);
/* Sets the state to |index> (drops queued gates). */
int rbk_state_reset(rbk_state* s, uint64_t index);
/* Copies count amplitudes starting at logical index offset from / to host
 * memory (interleaved re, im of the state's precision).  Logical order: the
 * layout permutation is undone first (see rbk_state_get_permutation). */
int rbk_state_upload(rbk_state* s, const void* host, uint64_t offset, uint64_t count);
int rbk_state_download(rbk_state* s, void* host, uint64_t offset, uint64_t count);
/* Executes queued gates and waits for the device (bounded wait). */
int rbk_state_synchronize(rbk_state* s);
int rbk_flush(rbk_state* s);
/* 1: queue gates and fuse them (default); 0: one pass per gate as issued. */
int rbk_state_set_deferred(rbk_state* s, int deferred);
/* Upper bound on dense 2x2 gates per fused pass (0 = built-in default). */
int rbk_state_set_pass_budget(rbk_state* s, int max_dense_gates_per_pass);
/* Tile shape of the fused passes: 0 = 2^12 amplitudes (c128; 2^13 for c64)
 * with 16 (c64: 32) per thread, 2 = 2^11 (c128; 2^12 for c64) with 16 (32)
 * per thread (the default), 3 = the tile of shape 2 in persistent CTAs that
 * copy their next tile into shared memory while they work on the current one.
 * Shape 1 (the tile of shape 0 with half the amplitudes per thread) is not
 * built: RBK_ERR_INVALID.  Results do not depend on the shape. */
int rbk_state_set_tile_shape(rbk_state* s, int shape);
int rbk_state_get_stats(const rbk_state* s, rbk_stats* out);
int rbk_state_reset_stats(rbk_state* s);
/* Milliseconds of device time spent in this state's kernels since the last
 * reset_stats (CUDA events around each executed queue). */
int rbk_state_device_ms(rbk_state* s, double* out);

/* ---- layout map ----------------------------------------------------------
 * The single-device use of ket::mpi::qubit_permutation
 * (ket/include/ket/mpi/qubit_permutation.hpp:40-302): perm[q] is the physical
 * bit that holds logical qubit q.  SWAP gates and pass relabelling only change
 * the map.  rbk_state_canonicalize moves the data so that perm is the
 * identity (the in-place swap of swap_permutated_local_qubits,
 * ket/include/ket/mpi/utility/detail/swap_permutated_local_qubits.hpp:26-81,
 * done several qubits per pass). */
int rbk_state_get_permutation(rbk_state* s, uint32_t* perm);
int rbk_state_canonicalize(rbk_state* s);
/* Declares the layout map without moving data: from now on logical qubit q
 * is the one held by physical bit perm[q] of the amplitudes as they lie in
 * device memory (queued gates run first, under the old map).  The logical
 * state changes unless perm equals rbk_state_get_permutation's map.  This is
 * what ket::mpi::permutate does to a qubit_permutation
 * (ket/include/ket/mpi/qubit_permutation.hpp:242-252): the labels change,
 * the local data stays.  perm must be a permutation of 0..n-1. */
int rbk_state_set_permutation(rbk_state* s, const uint32_t* perm);
/* Moves the data so that the layout map becomes perm (logical qubit q on
 * physical bit perm[q]), in relabel-only passes; the logical state is
 * unchanged.  rbk_state_canonicalize is set_layout to the identity.  With
 * perm = a ket::mpi::qubit_permutation's map, the device memory holds
 * ket::mpi's local data order: amplitude i of the state at physical index
 * permutate_bits(permutation, i) (qubit_permutation.hpp:470-491). */
int rbk_state_set_layout(rbk_state* s, const uint32_t* perm);
/* Device pointer to the amplitudes in physical order (after a flush). */
int rbk_state_device_pointer(rbk_state* s, void** out);

/* ---- fusion (bra BEGIN FUSION / END FUSION, bra/src/state.cpp:2193-2217,
 *      bra/src/nompi_state.cpp:1285-1357) --------------------------------- */
int rbk_begin_fusion(rbk_state* s);
int rbk_end_fusion(rbk_state* s);

/* ---- gates -----------------------------------------------------------------
 * `controls` may be NULL when num_controls is 0. */

/* ket::gate::hadamard (ket/include/ket/gate/hadamard.hpp:34-140) */
int rbk_hadamard(rbk_state* s, uint32_t target, const uint32_t* controls, int num_controls);
/* ket::gate::pauli_x / not_ / controlled_not (pauli_x.hpp:34-165, not_.hpp:33-51) */
int rbk_pauli_x(rbk_state* s, uint32_t target, const uint32_t* controls, int num_controls);
/* ket::gate::pauli_y (pauli_y.hpp:36-134) */
int rbk_pauli_y(rbk_state* s, uint32_t target, const uint32_t* controls, int num_controls);
/* ket::gate::pauli_z on control qubits: Z c = pauli_z(c), CZ c1 c2 = pauli_z(c1, c2)
 * (pauli_z.hpp:58-137).  qubits holds 1 + num_controls qubit indices. */
int rbk_pauli_z(rbk_state* s, const uint32_t* qubits, int num_qubits);
/* ket::gate::phase_shift_coeff: multiplies the amplitudes whose listed qubits
 * are all one by (re, im) (phase_shift.hpp:63-142); U1, CU1, S, T, "U c1 c2 k". */
int rbk_phase_shift_coeff(rbk_state* s, double re, double im, const uint32_t* qubits, int num_qubits);
/* ket::gate::phase_shift (U1 with a real phase; phase_shift.hpp:513-521) */
int rbk_phase_shift(rbk_state* s, double phase, const uint32_t* qubits, int num_qubits);
/* "U c1 c2 k" / "R c k": phase 2 pi / 2^k from bra's phase table
 * (bra/src/state.cpp:148 and :2650-2669, generate_phase_coefficients.hpp:20-39);
 * negative k applies the adjoint. */
int rbk_controlled_phase_shift_k(rbk_state* s, int k, const uint32_t* qubits, int num_qubits);
/* ket::gate::phase_shift2 = U2 (phase_shift.hpp:660-709) */
int rbk_phase_shift2(rbk_state* s, double phase1, double phase2, uint32_t target, const uint32_t* controls, int num_controls);
/* ket::gate::phase_shift3 = U3 (phase_shift.hpp:1200-1332) */
int rbk_phase_shift3(rbk_state* s, double phase1, double phase2, double phase3, uint32_t target,
                     const uint32_t* controls, int num_controls);
/* ket::gate::exponential_pauli_{x,y,z}: exp(i theta P) (exponential_pauli_y.hpp:40-85,
 * :473-481; exponential_pauli_z.hpp:40-78, :369-377) */
int rbk_exponential_pauli_x(rbk_state* s, double phase, uint32_t target, const uint32_t* controls, int num_controls);
int rbk_exponential_pauli_y(rbk_state* s, double phase, uint32_t target, const uint32_t* controls, int num_controls);
int rbk_exponential_pauli_z(rbk_state* s, double phase, uint32_t target, const uint32_t* controls, int num_controls);
/* ket::gate::swap (swap.hpp:34-75).  Uncontrolled swaps only relabel the layout map. */
int rbk_swap(rbk_state* s, uint32_t qubit1, uint32_t qubit2, const uint32_t* controls, int num_controls);
/* Any 2x2 unitary: m = {m00re, m00im, m01re, m01im, m10re, m10im, m11re, m11im}
 * (the generic 1-target form of ket::gate::gate, ket/include/ket/gate/gate.hpp). */
int rbk_apply_matrix2(rbk_state* s, const double* m, uint32_t target, const uint32_t* controls, int num_controls);
/* diag(d0, d1) on target: d = {d0re, d0im, d1re, d1im}. */
int rbk_apply_diagonal2(rbk_state* s, const double* d, uint32_t target, const uint32_t* controls, int num_controls);

/* ---- further gate families of ket / bra's instruction set -------------------
 * adjoint = 0 applies the gate, 1 its adjoint (bra's "+" mnemonics). */
/* +X / -X: ket::gate::x_rotation_half_pi / adj_ (ket/include/ket/gate/x_rotation_half_pi.hpp:34, :254) */
int rbk_x_rotation_half_pi(rbk_state* s, int adjoint, uint32_t target, const uint32_t* controls, int num_controls);
/* +Y / -Y: ket::gate::y_rotation_half_pi / adj_ (y_rotation_half_pi.hpp:33, :251) */
int rbk_y_rotation_half_pi(rbk_state* s, int adjoint, uint32_t target, const uint32_t* controls, int num_controls);
/* SX / SX+: ket::gate::sqrt_pauli_x (sqrt_pauli_x.hpp:32, :259) */
int rbk_sqrt_pauli_x(rbk_state* s, int adjoint, uint32_t target, const uint32_t* controls, int num_controls);
/* SY / SY+: ket::gate::sqrt_pauli_y (sqrt_pauli_y.hpp:33, :256) */
int rbk_sqrt_pauli_y(rbk_state* s, int adjoint, uint32_t target, const uint32_t* controls, int num_controls);
/* SZ, S, SZZ, SZn and their controlled forms: ket::gate::sqrt_pauli_z (sqrt_pauli_z.hpp:55-205,
 * :428-520): |1> of each target times i (adjoint: -i) where all controls are one. */
int rbk_sqrt_pauli_z(rbk_state* s, int adjoint, const uint32_t* targets, int num_targets, const uint32_t* controls,
                     int num_controls);
/* XX, Xn, YY, ZZ, ... and C...C forms: the product of single-qubit Paulis paulis[k] (one of
 * "IXYZ") on targets[k] (ket::gate::runtime::ranges::pauli_x/_y/_z, pauli_x.hpp:288-572). */
int rbk_pauli_string(rbk_state* s, const char* paulis, const uint32_t* targets, int num_targets,
                     const uint32_t* controls, int num_controls);
/* EXX, EXn, EYn, EZn, ... and C...C forms: exp(i phase P) for the Pauli product P
 * (exponential_pauli_x.hpp / _y.hpp / _z.hpp, runtime forms). */
int rbk_exponential_pauli_string(rbk_state* s, double phase, const char* paulis, const uint32_t* targets, int num_targets,
                                 const uint32_t* controls, int num_controls);
/* ESWAP and C...CESWAP: exp(i phase SWAP) (ket/include/ket/gate/exponential_swap.hpp:37-40, :103). */
int rbk_exponential_swap(rbk_state* s, double phase, uint32_t qubit1, uint32_t qubit2, const uint32_t* controls,
                         int num_controls);
/* CLEAR i / SET i: ket::gate::clear / set (clear.hpp, set.hpp): the qubit projected onto
 * |0> / |1> and the state renormalised. */
int rbk_clear(rbk_state* s, uint32_t qubit);
int rbk_set(rbk_state* s, uint32_t qubit);
/* SHORBOX nx N a: ket::ranges::shor_box (ket/include/ket/shor_box.hpp) with the exponent
 * register on the top nx qubits; replaces the state.  0 < divisor <= 2^32, base < 2^32. */
int rbk_shor_box(rbk_state* s, uint32_t num_exponent_qubits, uint64_t divisor, uint64_t base);

/* ---- dense unitaries --------------------------------------------------------
 * u is 2^k x 2^k complex (re, im), row-major: u[r][c] = <r|U|c>, where bit i of
 * the basis index is qubits[i].  The qubits are first moved onto the low
 * physical bits by relabelling passes.  complex<float> states with k = 5 or 6
 * (and n >= k + 7) run on the tensor cores as 3xTF32 split-precision GEMMs with
 * FP32 accumulation (tcgen05, accumulator in TMEM); other cases on CUDA cores.
 * No counterpart in ket beyond the fused blocks below; k <= 10. */
int rbk_apply_unitary(rbk_state* s, const double* u, const uint32_t* qubits, int k);
/* 0 (default): BEGIN/END FUSION blocks run gate by gate inside the fused passes.
 * 1: on complex<float> states, a block that touches 5 or 6 qubits becomes its
 *    2^k x 2^k unitary (built on the host in FP64) applied by rbk_apply_unitary,
 *    i.e. on the tensor cores -- the bra-fused unitary of
 *    bra/src/nompi_state.cpp:1285-1357 as one GEMM; other blocks stay gate by gate. */
int rbk_state_set_fusion_mode(rbk_state* s, int mode);

/* ---- observables ---------------------------------------------------------- */
/* sum |a_i|^2 */
int rbk_norm2(rbk_state* s, double* out);
/* |a_i|^2 for logical indices [offset, offset + count) into host memory
 * (measure.hpp:16-46, generate_events.hpp:18-51 use these). */
int rbk_probabilities(rbk_state* s, double* host_out, uint64_t offset, uint64_t count);
/* DO MEASUREMENT: ket::all_spin_expectation_values (all_spin_expectation_values.hpp:22-42,
 * spin_expectation_value.hpp:21-80): out[3q + {0,1,2}] = <S_x>, <S_y>, <S_z> of
 * logical qubit q, in spin-1/2 units (half the Pauli expectation). */
int rbk_spin_expectation_values(rbk_state* s, double* out);
/* EXPECTATION: sum_t coeff_t <psi|P_t|psi> (bra/src/nompi_state.cpp:1155-1202,
 * ket/include/ket/gate/utility/pauli_index_coeff.hpp:17-59).  strings holds
 * num_terms strings of n characters from "IXYZ", character k acting on
 * logical qubit k; coeffs holds num_terms (re, im) pairs; out = (re, im). */
int rbk_expectation_pauli(rbk_state* s, int num_terms, const char* strings, const double* coeffs, double* out);
/* ket::inner_product(a, b) = <b|a> = sum conj(b_i) a_i (inner_product.hpp:30-56); out = (re, im).
 * Both states must have the same size and precision. */
int rbk_inner_product(rbk_state* a, rbk_state* b, double* out);
/* ket::fidelity: |<b|a>|^2 (fidelity.hpp) */
int rbk_fidelity(rbk_state* a, rbk_state* b, double* out);
/* <b| H |a> for H = sum_t coeffs[t] P_t given like rbk_expectation_pauli:
 * ket::inner_product(a, b, observable) as bra's INNERPROD n <operator> calls it
 * (bra/src/nompi_state.cpp:2602-2648; the observable's Pauli action follows
 * pauli_index_coeff.hpp:17-59).  Same state requirements as rbk_inner_product. */
int rbk_inner_product_pauli(rbk_state* a, rbk_state* b, int num_terms, const char* strings, const double* coeffs, double* out);
/* |<b| H |a>|^2 (ket::fidelity with an observable; bra's FIDELITY n <operator>). */
int rbk_fidelity_pauli(rbk_state* a, rbk_state* b, int num_terms, const char* strings, const double* coeffs, double* out);

/* ---- sampling and measurement -------------------------------------------
 * Random numbers come from a std::mt19937_64 per state, seeded with 1 at
 * creation (bra's random_number_generator_, bra/include/bra/state.hpp:459-479,
 * fed by --seed). */
int rbk_state_seed(rbk_state* s, uint64_t seed);
/* GENERATE EVENTS: num_events basis-state indices drawn from |a_i|^2 as
 * ket::generate_events does (ket/include/ket/generate_events.hpp:18-66):
 * uniform_real_distribution(0, total) and upper_bound over the inclusive prefix
 * sums.  seed < 0 uses (and advances) the state's generator; otherwise a fresh
 * generator built from seed.  Unlike the reference, the state is left intact. */
int rbk_generate_events(rbk_state* s, int num_events, int64_t seed, uint64_t* events);
/* ket::measure (ket/include/ket/measure.hpp:16-46): sample one index with the
 * state's generator; the state becomes that basis state. */
int rbk_measure(rbk_state* s, uint64_t* outcome);
/* M q: ket::gate::projective_measurement (ket/include/ket/gate/projective_measurement.hpp):
 * outcome 0/1 with probabilities p0/p1, the kept half scaled by p^(-1/2). */
int rbk_projective_measurement(rbk_state* s, uint32_t qubit, int* outcome);
/* The same three with the caller's random numbers.  ket's sampling functions take
 * the caller's engine and draw from it with ket::utility::positive_random_value_upto,
 * a uniform_real_distribution on [0, upper) (ket/include/ket/utility/
 * positive_random_value_upto.hpp): draw(context, upper) must return such a value.
 * It is called on the calling thread, once per event in order (generate_events.hpp:
 * 18-48), once for measure (measure.hpp:16-46) and once for the projective
 * measurement with upper = p0 + p1 (projective_measurement.hpp:154-186), so an
 * engine shared with ket's CPU code advances exactly as it would there.  The state's
 * own generator is not used. */
typedef double (*rbk_uniform_fn)(void* context, double upper);
int rbk_generate_events_with(rbk_state* s, int num_events, rbk_uniform_fn draw, void* context, uint64_t* events);
int rbk_measure_with(rbk_state* s, rbk_uniform_fn draw, void* context, uint64_t* outcome);
int rbk_projective_measurement_with(rbk_state* s, uint32_t qubit, rbk_uniform_fn draw, void* context, int* outcome);

/* ---- adjoint gradient (no counterpart in the reference) --------------------
 * One gate of a parametrised circuit, in bra's terms.  qubits[0] is the target
 * (CNOT: qubits[0] = control, qubits[1] = target, as in "CNOT c t"; CZ, SWAP and
 * "U c1 c2 k" use both).  EX/EY/EZ apply exp(i phi P) with
 * phi = scale * theta[param] + angles[0] (param = -1: a fixed angle); U1 takes
 * angles[0]; U2 angles[0..1]; U3 angles[0..2]; U takes k in angles[0]. */
typedef struct rbk_circuit_gate {
  int32_t kind;
  int32_t qubits[2];
  int32_t param;
  double scale;
  double angles[3];
} rbk_circuit_gate;

enum {
  RBK_GATE_H = 1, RBK_GATE_X = 2, RBK_GATE_Y = 3, RBK_GATE_Z = 4, RBK_GATE_U1 = 5, RBK_GATE_U2 = 6,
  RBK_GATE_U3 = 7, RBK_GATE_CNOT = 8, RBK_GATE_CZ = 9, RBK_GATE_U = 10, RBK_GATE_EX = 11, RBK_GATE_EY = 12,
  RBK_GATE_EZ = 13, RBK_GATE_SWAP = 14
};

/* Energy E = <psi|H|psi> of psi = U(theta)|0...0> and dE/dtheta for every
 * parameter, from one forward pass and one reverse sweep that un-applies each
 * gate on psi and on lambda = H psi (exact gate inverses; no stored
 * intermediate states).  Only EX/EY/EZ gates take parameters (RY(t) = EY with
 * scale -1/2).  H is given like rbk_expectation_pauli (strings over all
 * num_qubits qubits, complex coeffs); at most 128 strings in 64 X/Y patterns.
 * The reference has no differentiation support; the tests check these
 * gradients against the parameter-shift rule evaluated with the reference
 * ket code and against central finite differences. */
int rbk_adjoint_gradient(int num_qubits, int precision, int device, const rbk_circuit_gate* gates, int num_gates,
                         const double* theta, int num_params, int num_terms, const char* strings,
                         const double* coeffs, double* energy, double* grad);

/* ---- batches of parametrised circuits (no counterpart in the reference) -----
 * Energies and adjoint gradients of many independent circuits of uneven size,
 * each with its own parameters and observable (same conventions as
 * rbk_adjoint_gradient).  Instances with n <= 12 (c128) / n <= 13 (c64) run in
 * one persistent kernel launch, replayed from a CUDA graph, one CTA per
 * instance with both state vectors in shared memory; the CTA size is chosen by
 * timing the candidates at rbk_batch_create.  Larger instances run through
 * rbk_adjoint_gradient.  Parameters and gradients are concatenated in instance
 * order. */
typedef struct rbk_batch rbk_batch;
typedef struct rbk_batch_instance {
  int32_t num_qubits;
  int32_t num_gates;
  const rbk_circuit_gate* gates;
  int32_t num_params;
  int32_t num_terms;
  const char* strings;   /* num_terms strings of num_qubits characters */
  const double* coeffs;  /* num_terms (re, im) */
} rbk_batch_instance;
typedef struct rbk_batch_stats {
  int num_small;       /* instances in the persistent launch */
  int num_large;       /* instances through rbk_adjoint_gradient */
  int threads;         /* CTA size picked by the autotuner */
  float small_ms;      /* device time of the persistent launch when tuned */
  double last_run_ms;  /* host wall time of the last rbk_batch_run */
} rbk_batch_stats;
int rbk_batch_create(int precision, int device, int num_instances, const rbk_batch_instance* instances, rbk_batch** out);
int rbk_batch_run(rbk_batch* batch, const double* theta, double* energies, double* grads);
/* Host threads that drive the larger instances concurrently (default 8). */
int rbk_batch_set_workers(rbk_batch* batch, int workers);
int rbk_batch_get_stats(const rbk_batch* batch, rbk_batch_stats* out);
/* Tile shape (rbk_state_set_tile_shape: the fusion width of the fused passes)
 * that the batch's autotuner picked for its instances of num_qubits qubits,
 * or -1 where the default is kept (fewer than 16 qubits, or no such instance). */
int rbk_batch_tuned_shape(const rbk_batch* batch, int num_qubits, int* shape);
int rbk_batch_destroy(rbk_batch* batch);

/* The same sweep on a context that keeps its two state vectors and buffers
 * between calls (optimiser loops): create once per qubit count and precision,
 * then rbk_adjoint_run with the arguments of rbk_adjoint_gradient. */
typedef struct rbk_adjoint_ctx rbk_adjoint_ctx;
int rbk_adjoint_create(int num_qubits, int precision, int device, rbk_adjoint_ctx** out);
int rbk_adjoint_run(rbk_adjoint_ctx* ctx, const rbk_circuit_gate* gates, int num_gates, const double* theta,
                    int num_params, int num_terms, const char* strings, const double* coeffs, double* energy, double* grad);
int rbk_adjoint_destroy(rbk_adjoint_ctx* ctx);

/* Pauli-string expectation value of a caller-owned device state, with no
 * device memory allocated.  No counterpart in the reference: it exists for
 * callers that cannot allocate when they need the value -- a process whose
 * HBM another allocator (a framework's caching allocator, a 128 GiB state)
 * has already reserved in full, or a loop that must not take the device
 * synchronisation of cudaMalloc / cudaFree.  It makes CUDA runtime calls
 * (launches, a copy, stream queries), so it must not be called from a CUDA
 * stream callback or host function.  Same meaning and arguments as
 * rbk_expectation_pauli, except: device_amps points to 2^num_qubits
 * amplitudes of the given precision in logical order (e.g.
 * rbk_state_canonicalize + rbk_state_device_pointer); stream is a
 * cudaStream_t (NULL: the legacy default stream); out is a host pointer to
 * (re, im).  The call reads the amplitudes on `stream` only: the caller
 * orders it after every write to them (for a library state,
 * rbk_state_synchronize first, since the state's own stream does not order
 * against other streams).  Its scratch is one fixed device array of about
 * 10 KB, shared by all calls: calls that overlap on the GPU race.  The array
 * takes device memory when the library's device code is loaded on a device
 * (with CUDA's lazy loading, at the first launch or symbol lookup there), so
 * on a device whose HBM will be reserved in full, make one call before that
 * happens.  At most 64 groups of strings with distinct X/Y positions
 * (RBK_ERR_INVALID beyond).  The first call on a device looks up the array's
 * device address and keeps it for the process; make that first call before
 * any stream capture, and do not use the function on a device after
 * cudaDeviceReset of that device. */
int rbk_expectation_pauli_noalloc(const void* device_amps, int num_qubits, int precision, int num_terms,
                                  const char* strings, const double* coeffs, double* out, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* RBK_H */
