/* rbk_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU restatement of the
 * reference's state-vector hot path, used by tests/, by smoke() in
 * __graft_entry__.py and by bench.py's cpu_baseline leg, as the checker.  The
 * product (the CUDA library) never calls, links or loads it.
 *
 * Each function restates the loop of one reference ket function with the same
 * floating-point operation order, so that this file agrees with the reference
 * itself (oracle/_ref/libketref.so, built from the reference's own sources) to
 * the last bit on the gate paths; tests/test_oracle_pins.py checks exactly that
 * against tests/golden/.
 *
 * Amplitudes are stored interleaved (re, im) as double, like std::complex<double>.
 * Index conventions follow ket: qubit q is bit q of the amplitude index.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_ops.h"

typedef struct { double re, im; } cplx;

/* MT19937-64 (Matsumoto & Nishimura, 64-bit variant): the engine behind
 * std::mt19937_64, which bra::state uses (bra/include/bra/state.hpp:459). */
typedef struct mt64 { uint64_t x[312]; int i; } mt64;

static void mt64_seed(mt64* g, uint64_t seed)
{
  g->x[0] = seed;
  for (int k = 1; k < 312; ++k)
    g->x[k] = UINT64_C(6364136223846793005) * (g->x[k - 1] ^ (g->x[k - 1] >> 62)) + (uint64_t)k;
  g->i = 312;
}

static uint64_t mt64_next(mt64* g)
{
  if (g->i >= 312) {
    for (int k = 0; k < 312; ++k) {
      uint64_t y = (g->x[k] & UINT64_C(0xFFFFFFFF80000000)) | (g->x[(k + 1) % 312] & UINT64_C(0x7FFFFFFF));
      uint64_t v = g->x[(k + 156) % 312] ^ (y >> 1);
      if (y & 1) v ^= UINT64_C(0xB5026F5AA96619E9);
      g->x[k] = v;
    }
    g->i = 0;
  }
  uint64_t z = g->x[g->i++];
  z ^= (z >> 29) & UINT64_C(0x5555555555555555);
  z ^= (z << 17) & UINT64_C(0x71D67FFFEDA60000);
  z ^= (z << 37) & UINT64_C(0xFFF7EEE000000000);
  z ^= z >> 43;
  return z;
}

/* std::uniform_real_distribution<double>(0, maximum) over a 64-bit engine:
 * one draw scaled to [0, 1) with 53 significant bits, times the width. */
static double mt64_upto(mt64* g, double maximum)
{
  double u = (double)mt64_next(g) / 18446744073709551616.0;
  if (u >= 1.0) u = nextafter(1.0, 0.0);
  return u * maximum;
}

typedef struct orc_state {
  int n;
  uint64_t size;
  cplx* a;
  cplx phase_table[65];
  mt64 rng;
} orc_state;

static inline cplx c_mul(cplx x, cplx y)
{
  cplx r = { x.re * y.re - x.im * y.im, x.re * y.im + x.im * y.re };
  return r;
}
static inline cplx c_scale(cplx x, double s) { cplx r = { x.re * s, x.im * s }; return r; }
static inline cplx c_add(cplx x, cplx y) { cplx r = { x.re + y.re, x.im + y.im }; return r; }
static inline cplx c_sub(cplx x, cplx y) { cplx r = { x.re - y.re, x.im - y.im }; return r; }
static inline cplx c_conj(cplx x) { cplx r = { x.re, -x.im }; return r; }

/* ket::utility::exp_i (ket/include/ket/utility/exp_i.hpp:21-36): std::exp of i*theta. */
static cplx exp_i(double theta)
{
  double complex z = cexp(CMPLX(0.0, theta));
  cplx r = { creal(z), cimag(z) };
  return r;
}

static const double ONE_DIV_ROOT_TWO = 0.707106781186547524400844362104849039284835937688474036588;
static const double TWO_PI = 6.28318530717958647692528676655900576839433879875021164195;

/* Inserts a zero bit at position q of v:  ((v & ~low) << 1) | (v & low)
 * (ket/include/ket/gate/hadamard.hpp:57-59). */
static inline uint64_t insert0(uint64_t v, int q)
{
  uint64_t low = (UINT64_C(1) << q) - 1;
  return ((v & ~low) << 1) | (v & low);
}
/* Inserts zero bits at two distinct positions (ket two-qubit loops, e.g.
 * ket/include/ket/gate/pauli_x.hpp:145-160). */
static inline uint64_t insert00(uint64_t v, int q1, int q2)
{
  int lo = q1 < q2 ? q1 : q2, hi = q1 < q2 ? q2 : q1;
  return insert0(insert0(v, lo), hi);
}

orc_state* orc_create(int n, uint64_t initial_index)
{
  orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
  if (!s) return NULL;
  s->n = n;
  s->size = UINT64_C(1) << n;
  s->a = (cplx*)calloc(s->size, sizeof(cplx));
  if (!s->a) { free(s); return NULL; }
  s->a[initial_index].re = 1.0;
  mt64_seed(&s->rng, 1);
  /* ket::utility::generate_phase_coefficients (ket/include/ket/utility/generate_phase_coefficients.hpp:20-39),
   * called with num_qubits = n by bra (bra/src/state.cpp:148): entry k = exp_i(2 pi / 2^k). */
  for (int k = 0; k <= n && k < 65; ++k)
    s->phase_table[k] = exp_i(TWO_PI / (double)(UINT64_C(1) << k));
  return s;
}

void orc_destroy(orc_state* s) { if (s) { free(s->a); free(s); } }
void orc_set_amplitudes(orc_state* s, const double* in) { memcpy(s->a, in, s->size * sizeof(cplx)); }
void orc_get_amplitudes(const orc_state* s, double* out) { memcpy(out, s->a, s->size * sizeof(cplx)); }

/* H: ket/include/ket/gate/hadamard.hpp:52-71 */
static void gate_h(orc_state* s, int q)
{
  uint64_t half = s->size >> 1, m = UINT64_C(1) << q;
  #pragma omp parallel for schedule(static)
  for (uint64_t v = 0; v < half; ++v) {
    uint64_t i0 = insert0(v, q), i1 = i0 | m;
    cplx a0 = s->a[i0], a1 = s->a[i1];
    s->a[i0] = c_scale(c_add(a0, a1), ONE_DIV_ROOT_TWO);
    s->a[i1] = c_scale(c_sub(a0, a1), ONE_DIV_ROOT_TWO);
  }
}

/* X: pauli_x.hpp:34-61 (swap);  CNOT: pauli_x.hpp:116-165 via not_.hpp:33-51 */
static void gate_x(orc_state* s, int t, int c)
{
  if (c < 0) {
    uint64_t half = s->size >> 1, m = UINT64_C(1) << t;
    #pragma omp parallel for schedule(static)
    for (uint64_t v = 0; v < half; ++v) {
      uint64_t i0 = insert0(v, t), i1 = i0 | m;
      cplx tmp = s->a[i0]; s->a[i0] = s->a[i1]; s->a[i1] = tmp;
    }
  } else {
    uint64_t quarter = s->size >> 2, mt = UINT64_C(1) << t, mc = UINT64_C(1) << c;
    #pragma omp parallel for schedule(static)
    for (uint64_t v = 0; v < quarter; ++v) {
      uint64_t i0 = insert00(v, t, c) | mc, i1 = i0 | mt;
      cplx tmp = s->a[i0]; s->a[i0] = s->a[i1]; s->a[i1] = tmp;
    }
  }
}

/* Y: pauli_y.hpp:36-70 -- swap, then a0 *= -i, a1 *= i */
static void gate_y(orc_state* s, int q)
{
  uint64_t half = s->size >> 1, m = UINT64_C(1) << q;
  const cplx mi = { 0.0, -1.0 }, pi = { 0.0, 1.0 };
  #pragma omp parallel for schedule(static)
  for (uint64_t v = 0; v < half; ++v) {
    uint64_t i0 = insert0(v, q), i1 = i0 | m;
    cplx a0 = s->a[i0], a1 = s->a[i1];
    s->a[i0] = c_mul(a1, mi);
    s->a[i1] = c_mul(a0, pi);
  }
}

/* Multiplies the amplitudes whose bits in `mask` are all one by a real factor
 * (Z / CZ: pauli_z.hpp:58-137, `*= real_type(-1)`) or a complex one
 * (U1 / CU1 / U c1 c2 k: phase_shift.hpp:63-142). */
static void gate_phase_real(orc_state* s, uint64_t mask, double f)
{
  #pragma omp parallel for schedule(static)
  for (uint64_t i = 0; i < s->size; ++i)
    if ((i & mask) == mask) s->a[i] = c_scale(s->a[i], f);
}
static void gate_phase_coeff(orc_state* s, uint64_t mask, cplx coeff)
{
  #pragma omp parallel for schedule(static)
  for (uint64_t i = 0; i < s->size; ++i)
    if ((i & mask) == mask) s->a[i] = c_mul(s->a[i], coeff);
}

/* U2: phase_shift.hpp:660-709 */
static void gate_u2(orc_state* s, int q, double phase1, double phase2)
{
  cplx c1 = exp_i(phase1), c2 = exp_i(phase2);
  cplx mc1 = { ONE_DIV_ROOT_TWO * c1.re, ONE_DIV_ROOT_TWO * c1.im };
  uint64_t half = s->size >> 1, m = UINT64_C(1) << q;
  #pragma omp parallel for schedule(static)
  for (uint64_t v = 0; v < half; ++v) {
    uint64_t i0 = insert0(v, q), i1 = i0 | m;
    cplx a0 = s->a[i0], a1 = s->a[i1];
    cplx z = c_sub(a0, c_mul(c2, a1));
    z = c_scale(z, ONE_DIV_ROOT_TWO);
    cplx o = c_mul(a1, c2);
    o = c_add(o, a0);
    o = c_mul(o, mc1);
    s->a[i0] = z; s->a[i1] = o;
  }
}

/* U3: phase_shift.hpp:1200-1254 (uncontrolled) */
static void gate_u3(orc_state* s, int q, double theta, double phi, double lambda)
{
  double sine = sin(0.5 * theta), cosine = cos(0.5 * theta);
  cplx c2 = exp_i(phi), c3 = exp_i(lambda);
  cplx sc3 = { sine * c3.re, sine * c3.im }, cc3 = { cosine * c3.re, cosine * c3.im };
  uint64_t half = s->size >> 1, m = UINT64_C(1) << q;
  #pragma omp parallel for schedule(static)
  for (uint64_t v = 0; v < half; ++v) {
    uint64_t i0 = insert0(v, q), i1 = i0 | m;
    cplx a0 = s->a[i0], a1 = s->a[i1];
    cplx z = c_scale(a0, cosine);
    z = c_sub(z, c_mul(sc3, a1));
    cplx o = c_mul(a1, cc3);
    o = c_add(o, c_scale(a0, sine));
    o = c_mul(o, c2);
    s->a[i0] = z; s->a[i1] = o;
  }
}

/* EY: exponential_pauli_y.hpp:40-85 with coeff = exp_i(theta) (:473-481) */
static void gate_ey(orc_state* s, int q, double theta)
{
  cplx coeff = exp_i(theta);
  double cs = coeff.re, sn = coeff.im;
  uint64_t half = s->size >> 1, m = UINT64_C(1) << q;
  #pragma omp parallel for schedule(static)
  for (uint64_t v = 0; v < half; ++v) {
    uint64_t i0 = insert0(v, q), i1 = i0 | m;
    cplx a0 = s->a[i0], a1 = s->a[i1];
    cplx z = c_scale(a0, cs);
    z = c_add(z, c_scale(a1, sn));
    cplx o = c_scale(a1, cs);
    o = c_sub(o, c_scale(a0, sn));
    s->a[i0] = z; s->a[i1] = o;
  }
}

/* EX: exponential_pauli_x.hpp (coeff form): a0 = a0 cos + a1 (i sin), a1 = a1 cos + a0 (i sin) */
static void gate_ex(orc_state* s, int q, double theta)
{
  cplx coeff = exp_i(theta);
  double cs = coeff.re;
  cplx isn = { 0.0 * coeff.im, 1.0 * coeff.im };
  uint64_t half = s->size >> 1, m = UINT64_C(1) << q;
  #pragma omp parallel for schedule(static)
  for (uint64_t v = 0; v < half; ++v) {
    uint64_t i0 = insert0(v, q), i1 = i0 | m;
    cplx a0 = s->a[i0], a1 = s->a[i1];
    cplx z = c_scale(a0, cs);
    z = c_add(z, c_mul(a1, isn));
    cplx o = c_scale(a1, cs);
    o = c_add(o, c_mul(a0, isn));
    s->a[i0] = z; s->a[i1] = o;
  }
}

/* EZ: exponential_pauli_z.hpp:40-78 with coeff = exp_i(theta) (:369-377) */
static void gate_ez(orc_state* s, int q, double theta)
{
  cplx coeff = exp_i(theta), cc = c_conj(coeff);
  uint64_t half = s->size >> 1, m = UINT64_C(1) << q;
  #pragma omp parallel for schedule(static)
  for (uint64_t v = 0; v < half; ++v) {
    uint64_t i0 = insert0(v, q), i1 = i0 | m;
    s->a[i0] = c_mul(s->a[i0], coeff);
    s->a[i1] = c_mul(s->a[i1], cc);
  }
}

/* SWAP: swap.hpp:34-75 */
static void gate_swap(orc_state* s, int q1, int q2)
{
  uint64_t quarter = s->size >> 2, m1 = UINT64_C(1) << q1, m2 = UINT64_C(1) << q2;
  #pragma omp parallel for schedule(static)
  for (uint64_t v = 0; v < quarter; ++v) {
    uint64_t b = insert00(v, q1, q2);
    cplx tmp = s->a[b | m1]; s->a[b | m1] = s->a[b | m2]; s->a[b | m2] = tmp;
  }
}

/* Applies ops in order.  BEGIN/END FUSION markers are no-ops here: bra's fused
 * execution (bra/src/nompi_state.cpp:1285-1357) replays the recorded gates in
 * order on each 2^k chunk, which is the same per-amplitude arithmetic as
 * applying them one by one; tests/test_oracle_pins.py checks that against the
 * reference's own fused path.  Returns 0, or -1 for an unknown code. */
int orc_apply(orc_state* s, const oracle_op* ops, int num_ops)
{
  for (int i = 0; i < num_ops; ++i) {
    const oracle_op* op = &ops[i];
    int q0 = op->q[0], q1 = op->q[1];
    switch (op->code) {
      case ORC_H: gate_h(s, q0); break;
      case ORC_X: gate_x(s, q0, -1); break;
      case ORC_Y: gate_y(s, q0); break;
      case ORC_Z: gate_phase_real(s, UINT64_C(1) << q0, -1.0); break;
      case ORC_U1: gate_phase_coeff(s, UINT64_C(1) << q0, exp_i(op->p[0])); break;
      case ORC_U2: gate_u2(s, q0, op->p[0], op->p[1]); break;
      case ORC_U3: gate_u3(s, q0, op->p[0], op->p[1], op->p[2]); break;
      case ORC_CNOT: gate_x(s, q1, q0); break;
      case ORC_CZ: gate_phase_real(s, (UINT64_C(1) << q0) | (UINT64_C(1) << q1), -1.0); break;
      case ORC_CPHASE_K: {
        int k = op->k;
        cplx coeff = k >= 0 ? s->phase_table[k] : c_conj(s->phase_table[-k]);
        gate_phase_coeff(s, (UINT64_C(1) << q0) | (UINT64_C(1) << q1), coeff);
        break;
      }
      case ORC_EY: gate_ey(s, q0, op->p[0]); break;
      case ORC_EZ: gate_ez(s, q0, op->p[0]); break;
      case ORC_EX: gate_ex(s, q0, op->p[0]); break;
      case ORC_SWAP: gate_swap(s, q0, q1); break;
      case ORC_BEGIN_FUSION: case ORC_END_FUSION: break;
      default: return -1;
    }
  }
  return 0;
}

/* DO MEASUREMENT: ket::spin_expectation_value per qubit
 * (ket/include/ket/spin_expectation_value.hpp:21-80): long double partials of
 * Re/Im conj(a0) a1 and (|a0|^2 - |a1|^2), the last one halved. */
void orc_spins(const orc_state* s, double* out)
{
  for (int q = 0; q < s->n; ++q) {
    long double sx = 0, sy = 0, sz = 0;
    uint64_t half = s->size >> 1, m = UINT64_C(1) << q;
    for (uint64_t v = 0; v < half; ++v) {
      uint64_t i0 = insert0(v, q), i1 = i0 | m;
      cplx c0 = c_conj(s->a[i0]), a1 = s->a[i1];
      cplx p = c_mul(c0, a1);
      sx += p.re; sy += p.im;
      sz += (long double)(c0.re * c0.re + c0.im * c0.im) - (long double)(a1.re * a1.re + a1.im * a1.im);
    }
    out[3 * q + 0] = (double)sx;
    out[3 * q + 1] = (double)sy;
    out[3 * q + 2] = (double)sz * 0.5;
  }
}

/* sum_t coeff_t <psi|P_t|psi> with P_t given as n characters of "IXYZ"
 * (character k acts on qubit k).  P|psi> follows
 * ket/include/ket/gate/utility/pauli_index_coeff.hpp:17-59:
 * (P psi)(i) = C(i) psi(i ^ flip), C multiplies -i / +i for Y on a 0 / 1 bit
 * and -1 for Z on a 1 bit. */
void orc_expectation(const orc_state* s, int num_terms, const char* strings, const double* coeffs, double* out)
{
  long double re = 0, im = 0;
  for (int t = 0; t < num_terms; ++t) {
    const char* p = strings + (size_t)t * s->n;
    uint64_t flip = 0, ymask = 0, zmask = 0;
    int ny = 0;
    for (int k = 0; k < s->n; ++k) {
      if (p[k] == 'X') flip |= UINT64_C(1) << k;
      else if (p[k] == 'Y') { flip |= UINT64_C(1) << k; ymask |= UINT64_C(1) << k; ++ny; }
      else if (p[k] == 'Z') zmask |= UINT64_C(1) << k;
    }
    /* (-i)^ny */
    static const double pow_mi[4][2] = { { 1, 0 }, { 0, -1 }, { -1, 0 }, { 0, 1 } };
    cplx base = { pow_mi[ny & 3][0], pow_mi[ny & 3][1] };
    long double tre = 0, tim = 0;
    for (uint64_t i = 0; i < s->size; ++i) {
      cplx v = c_mul(c_conj(s->a[i]), s->a[i ^ flip]);
      if (__builtin_popcountll(i & (ymask | zmask)) & 1) { v.re = -v.re; v.im = -v.im; }
      tre += v.re; tim += v.im;
    }
    cplx term = { (double)tre, (double)tim };
    term = c_mul(term, base);
    cplx c = { coeffs[2 * t], coeffs[2 * t + 1] };
    term = c_mul(term, c);
    re += term.re; im += term.im;
  }
  out[0] = (double)re; out[1] = (double)im;
}

/* ket::inner_product(state_a, state_b) = <b|a> (ket/include/ket/inner_product.hpp:30-56). */
void orc_inner_product(const orc_state* a, const orc_state* b, double* out)
{
  long double re = 0, im = 0;
  for (uint64_t i = 0; i < a->size; ++i) {
    cplx v = c_mul(c_conj(b->a[i]), a->a[i]);
    re += v.re; im += v.im;
  }
  out[0] = (double)re; out[1] = (double)im;
}

/* |a_i|^2 for every i (measure.hpp:16-46 / generate_events.hpp:18-51 use std::norm). */
void orc_probabilities(const orc_state* s, double* out)
{
  for (uint64_t i = 0; i < s->size; ++i) out[i] = s->a[i].re * s->a[i].re + s->a[i].im * s->a[i].im;
}

/* std::norm of the reference's complex<double>: libstdc++ computes x*x + y*y
 * for the builtin floating types (the product is not contracted: no FMA on
 * the x86-64 baseline the reference is built for here). */
static double ref_norm(cplx z) { return z.re * z.re + z.im * z.im; }

void orc_seed(orc_state* s, uint64_t seed) { mt64_seed(&s->rng, seed); }

/* ket::generate_events (generate_events.hpp:18-66): inclusive prefix sums of
 * |a|^2, r = uniform(0, total), upper_bound.  seed < 0: the state's generator;
 * else a fresh one.  The state itself is not modified here. */
int orc_generate_events(orc_state* s, int num_events, long long seed, uint64_t* out)
{
  double* prefix = (double*)malloc(s->size * sizeof(double));
  if (!prefix) return -1;
  double run = 0;
  for (uint64_t i = 0; i < s->size; ++i) { run = run + ref_norm(s->a[i]); prefix[i] = run; }
  mt64 fresh;
  mt64* g = &s->rng;
  if (seed >= 0) { mt64_seed(&fresh, (uint64_t)seed); g = &fresh; }
  for (int k = 0; k < num_events; ++k) {
    double r = mt64_upto(g, prefix[s->size - 1]);
    uint64_t lo = 0, hi = s->size;
    while (lo < hi) { uint64_t mid = lo + ((hi - lo) >> 1); if (prefix[mid] > r) hi = mid; else lo = mid + 1; }
    out[k] = lo;
  }
  free(prefix);
  return 0;
}

/* ket::gate::projective_measurement (projective_measurement.hpp): long double
 * sums of |a|^2 per outcome, r = uniform(0, p0 + p1) < p0 -> 0, the kept half
 * scaled by pow(p, -1/2), the other half zeroed. */
int orc_projective_measurement(orc_state* s, int q)
{
  long double z = 0, o = 0;
  uint64_t half = s->size >> 1, m = UINT64_C(1) << q;
  for (uint64_t v = 0; v < half; ++v) {
    uint64_t i0 = insert0(v, q), i1 = i0 | m;
    z += (long double)ref_norm(s->a[i0]);
    o += (long double)ref_norm(s->a[i1]);
  }
  double p0 = (double)z, p1 = (double)o;
  int one = !(mt64_upto(&s->rng, p0 + p1) < p0);
  double mult = pow(one ? p1 : p0, -0.5);
  for (uint64_t v = 0; v < half; ++v) {
    uint64_t i0 = insert0(v, q), i1 = i0 | m;
    uint64_t keep = one ? i1 : i0, drop = one ? i0 : i1;
    s->a[keep] = c_scale(s->a[keep], mult);
    s->a[drop].re = 0; s->a[drop].im = 0;
  }
  return one;
}

/* ket::measure (measure.hpp): one event from the state's generator, then the
 * state becomes the basis vector of that index. */
uint64_t orc_measure(orc_state* s)
{
  uint64_t idx = 0;
  if (orc_generate_events(s, 1, -1, &idx) != 0) return UINT64_MAX;
  memset(s->a, 0, s->size * sizeof(cplx));
  s->a[idx].re = 1.0;
  return idx;
}
