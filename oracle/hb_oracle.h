/*
 * hb_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of HasteBoots' TFHE gate-bootstrapping path (tfhe crate evaluator,
 * fhe_core modulus switch / binary and ternary blind rotation / RLWE key switching, lattice
 * RLWE/RGSW external product, algebra Goldilocks/BabyBear/DefaultFieldU32 arithmetic and unsigned
 * gadget decomposition).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg and reference arm
 * (--impl reference, the timed CPU restatement) may load this library, tests and smoke() only as
 * the checker. The product (hasteboots_b200/, libhb_gpu.so) never links it.
 *
 * Parity status: the reference (pure Rust, NTT in the un-vendored `concrete-ntt` git
 * dependency, branch `dev`, no pinned commit) cannot be built or run in this environment
 * and ships no golden vectors. This oracle is pinned against every known-answer test the
 * reference's own tests hold for this path (monomial products in
 * algebra/src/baby_bear/babybear_ntt.rs:185-213, decomposition/recomposition, NTT round
 * trips) and against the reference's properties (schoolbook product, truth tables,
 * noise < Q/16). Bit-exactness with the live Rust binary is therefore "parity unpinned".
 *
 * All buffers hold canonical little-endian field values: uint64_t words for Goldilocks,
 * uint32_t words for BabyBear and DefaultFieldU32 (Q = 132120577).
 */
#ifndef HB_ORACLE_H
#define HB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_FIELD_BABYBEAR = 0, ORC_FIELD_GOLDILOCKS = 1, ORC_FIELD_DEFAULT_U32 = 2 };

enum {
  ORC_GATE_NAND = 0,
  ORC_GATE_AND = 1,
  ORC_GATE_OR = 2,
  ORC_GATE_NOR = 3,
  ORC_GATE_XOR = 4,
  ORC_GATE_XNOR = 5,
  ORC_GATE_MAJORITY = 6,
  ORC_GATE_NOT = 7,
  ORC_GATE_MUX = 8
};

/* Mirrors fhe_core::ConstParameters (fhe_core/src/parameter.rs:81-107) for RLWE bootstrapping
 * with the RLWE key switch. */
typedef struct orc_params {
  int32_t field_id;      /* ORC_FIELD_* */
  uint32_t ring_dim;     /* N */
  uint32_t lwe_dim;      /* n, next_pow2(n) <= N */
  uint32_t br_bits;      /* blind_rotation_basis_bits */
  uint32_t br_len;       /* ceil(bits(Q)/br_bits) */
  uint32_t ks_bits;      /* key_switching_basis_bits */
  uint32_t ks_len;       /* ceil(bits(Q)/ks_bits) */
  uint32_t ring_ternary; /* 1: ternary ring key, 0: binary */
  uint32_t lwe_ternary;  /* 1: ternary LWE key (DefaultFieldU32 only), 0: binary */
  double lwe_noise_std;
  double ring_noise_std;
  double ks_noise_std;
} orc_params;

/* 0: BABYBEAR_BINARY_128_BITS, 1: GOLDILOCKS_BINARY_128_BITS, 2: ZAMA_BINARY_128_BITS,
 * 3: DEFAULT_TERNARY_128_BITS, 4: CUSTOM_TERNARY_128_BITS (tfhe/src/bfhe/parameters.rs:7-117).
 * Returns 0 or -1 for an unknown id. */
int orc_params_preset(int preset, orc_params *out);

/* The splitmix-style counter PRG that defines the project's seeded key convention. */
uint64_t orc_prg(uint64_t seed, uint64_t stream, uint64_t ctr);

/* Key generation from a seed. Output sizes (words): lwe_sk n, ring_sk N,
 * bsk n*pairs*2*br_len*2*N (layout [i][pair][part: 0=c_neg_s_m, 1=c_m][j][0=a,1=b][k]; one pair
 * for a binary LWE key, two -- RGSW(s_i == 1), RGSW(s_i == -1) -- for a ternary one),
 * ksk ks_len*2*N (layout [c][j][0=a,1=b][k < n'], n' = next_pow2(n), c < N/n'). All coefficient
 * domain. */
int orc_keygen(const orc_params *p, uint64_t seed, void *lwe_sk, void *ring_sk, void *bsk,
               void *ksk, int threads);

/* Encrypt bits[i] (0/1) as LWE ciphertext with index index0+i. lwe_out: count*(n+1) words. */
int orc_encrypt(const orc_params *p, const void *lwe_sk, uint64_t seed, uint64_t index0,
                const uint8_t *bits, size_t count, void *lwe_out);

/* Decrypt; noise_out (optional) receives min(|p - encode(m)|) per ciphertext. */
int orc_decrypt(const orc_params *p, const void *lwe_sk, const void *lwe, size_t count,
                uint8_t *bits_out, uint64_t *noise_out);

/* Homomorphic gate on count independent ciphertext tuples (c2 used by MAJORITY and MUX). */
int orc_gate(const orc_params *p, const void *bsk, const void *ksk, int gate, const void *c0,
             const void *c1, const void *c2, void *out, size_t count, int threads);

/* Evaluator::new (tfhe/src/bfhe/evaluate.rs:65-96): the bootstrapping and key-switching keys
 * transformed once into an opaque handle, so that gates on it skip the key transform. */
typedef struct orc_eval orc_eval;
int orc_eval_create(const orc_params *p, const void *bsk, const void *ksk, int threads, orc_eval **out);
void orc_eval_free(orc_eval *e);
/* orc_gate on a transformed key. */
int orc_eval_gate(const orc_eval *e, int gate, const void *c0, const void *c1, const void *c2,
                  void *out, size_t count, int threads);

/* EvaluationKey::bootstrap(c, lut) on count ciphertexts sharing one LUT polynomial (N words). */
int orc_bootstrap_lut(const orc_params *p, const void *bsk, const void *ksk, const void *c,
                      const void *lut, void *out, size_t count, int threads);

/* Stage probes for tests: modulus switch output ([n+1] values in [0,2N)), and the RLWE
 * accumulator after `steps` blind-rotation steps (2*N words: a then b, reference representation
 * canonicalised). */
int orc_modswitch(const orc_params *p, const void *c, uint32_t *out);
int orc_blind_rotate(const orc_params *p, const void *bsk, const void *c, const void *lut,
                     uint32_t steps, void *acc_out);
/* The accumulator after every one of the n steps in one pass: n rows of 2N words (a then b,
 * canonical), the rows of the AccTrace that vfhe's traced bootstrap records. digits_out (may be
 * NULL; binary LWE keys with B <= 2^8): every step's unsigned gadget digits of E.a then E.b,
 * [n][2][l][N] bytes, the bit polynomials of its SumHadamardTrace (zero for a step with a_i = 0). */
int orc_blind_rotate_trace(const orc_params *p, const void *bsk, const void *c, const void *lut,
                           void *trace_out, void *digits_out);

/* Negacyclic NTT round trip / product checks (N = 1<<log_n). */
int orc_ntt_roundtrip(int field_id, uint32_t log_n, const void *in, void *out);
int orc_negacyclic_mul(int field_id, uint32_t log_n, const void *x, const void *y, void *out,
                       int schoolbook);

/* RLWE x RGSW external product (lattice/src/rlwe.rs:573-596) in the coefficient domain.
 * rlwe: count*2*N words (a then b); rgsw: 2*len*2*N words (layout as one BSK entry);
 * out: count*2*N words. */
int orc_external_product(int field_id, uint32_t log_n, uint32_t bits, uint32_t len,
                         const void *rlwe, const void *rgsw, void *out, size_t count,
                         int threads);

#ifdef __cplusplus
}
#endif

#endif
