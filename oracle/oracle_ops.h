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

typedef struct oracle_op {
  int32_t code;
  int32_t q[2];
  int32_t k;
  double p[3];
} oracle_op;

#endif
