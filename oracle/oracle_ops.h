/* oracle_ops.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Instruction encoding shared by the two oracle legs: the reference's own ket /
 * bra code (oracle/ketref_driver.cpp, built into oracle/_ref/) and the C
 * restatement (oracle/rbk_oracle.c).  One record per bra .qcx instruction of
 * the hot path (mnemonics from bra/src/interpreter.cpp:513-640).
 */
#ifndef RBK_ORACLE_OPS_H
#define RBK_ORACLE_OPS_H

#include <stdint.h>

enum oracle_code {
  ORC_H = 1,            /* H t                       q[0]=t                         */
  ORC_X = 2,            /* X t                                                      */
  ORC_Y = 3,            /* Y t                                                      */
  ORC_Z = 4,            /* Z c                                                      */
  ORC_U1 = 5,           /* U1 c lambda               p[0]=lambda                    */
  ORC_U2 = 6,           /* U2 t phi lambda           p[0]=phi p[1]=lambda           */
  ORC_U3 = 7,           /* U3 t theta phi lambda     p[0..2]                        */
  ORC_CNOT = 8,         /* CNOT c t                  q[0]=c q[1]=t                  */
  ORC_CZ = 9,           /* CZ c1 c2                                                 */
  ORC_CPHASE_K = 10,    /* U c1 c2 k                 k (negative: adjoint, U+)      */
  ORC_EY = 11,          /* EY t theta                exp(i theta Y), p[0]=theta     */
  ORC_EZ = 12,          /* EZ t theta                exp(i theta Z)                 */
  ORC_SWAP = 13,        /* SWAP t1 t2                                               */
  ORC_BEGIN_FUSION = 14,
  ORC_END_FUSION = 15,
  ORC_EX = 16           /* EX t theta                exp(i theta X), p[0]=theta     */
};

/* The rest of bra's instruction set, for the reference leg's generic entry
 * ketref_gate (targets t[], controls c[], parameters p[]).  Gates whose qubits
 * are all of control type in ket (Z, S/SZ, U1, R, T) take every qubit in c[]. */
enum oracle_gate_kind {
  KG_H = 1, KG_NOT = 2, KG_X = 3, KG_Y = 4, KG_Z = 5, KG_SWAP = 6,
  KG_SX = 7, KG_SX_ADJ = 8, KG_SY = 9, KG_SY_ADJ = 10, KG_SZ = 11, KG_SZ_ADJ = 12,
  KG_U1 = 13, KG_U1_ADJ = 14, KG_U2 = 15, KG_U2_ADJ = 16, KG_U3 = 17, KG_U3_ADJ = 18,
  KG_R = 19, KG_R_ADJ = 20, KG_ROTX = 21, KG_ROTX_ADJ = 22, KG_ROTY = 23, KG_ROTY_ADJ = 24,
  KG_EX = 25, KG_EX_ADJ = 26, KG_EY = 27, KG_EY_ADJ = 28, KG_EZ = 29, KG_EZ_ADJ = 30,
  KG_ESWAP = 31, KG_ESWAP_ADJ = 32, KG_TOFFOLI = 33, KG_CLEAR = 34, KG_SET = 35, KG_SHORBOX = 36
};

typedef struct oracle_op {
  int32_t code;
  int32_t q[2];
  int32_t k;
  double p[3];
} oracle_op;

#endif
