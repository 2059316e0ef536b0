// hb_gl_ptx.cuh -- Goldilocks arithmetic written with PTX carry chains so that carries and borrows
// come from the add/sub instructions themselves instead of 64-bit compares and selects.
// Multiplies are kept for the products themselves: multiplications by 2^32 - 1 and the carry
// corrections are ALU carry chains. With them as multiply-adds the bootstrapping kernel was bound by
// the integer multiply-add pipe (ncu: sm__pipe_fmaheavy_cycles_active 81 % against 59 % for the
// ALU); with the ALU forms the two read 69 % and 76 % and the launch is 7.5 % shorter.
// All functions accept any 64-bit word as a representative of its residue mod Q = 2^64 - 2^32 + 1.
#pragma once

#include <cstdint>

namespace hb {
namespace glx {

constexpr uint64_t P = 0xFFFFFFFF00000001ULL;

__device__ __forceinline__ void split(uint64_t x, uint32_t &lo, uint32_t &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=r"(lo), "=r"(hi) : "l"(x));
}
__device__ __forceinline__ uint64_t join(uint32_t lo, uint32_t hi) {
  uint64_t x;
  asm("mov.b64 %0, {%1, %2};" : "=l"(x) : "r"(lo), "r"(hi));
  return x;
}

// A = x2 (2^32 - 1) + (2^32 - 1 - x3) = x2 2^32 + (2^32 - 1 - x3) - x2 for 32-bit limbs x2, x3
// (A < 2^64): the low word (2^32 - 1 - x3) - x2, its borrow taken from x2. On the ALU (a multiply-add
// x2 (2^32 - 1) + ~x3 with ~x3 also formed on the multiply pipe measured 6.0 % slower on 16384
// GOLDILOCKS gates, 1925.2 vs 1809.5 ms: the multiply pipe is the bound one).
__device__ __forceinline__ uint64_t fold_hi(uint32_t x2, uint32_t x3) {
  uint32_t a0, a1;
  asm("sub.cc.u32 %0, %2, %3;\n\t"
      "subc.u32   %1, %3, 0;"
      : "=&r"(a0), "=r"(a1)
      : "r"(~x3), "r"(x2));
  return join(a0, a1);
}
// z (2^32 - 1) = z 2^32 - z as limbs: low word -z, its borrow (z != 0) taken from z (two ALU
// instructions instead of a wide multiply: 1788.6 -> 1780.1 ms on 16384 GOLDILOCKS gates).
__device__ __forceinline__ void times_eps(uint32_t z, uint32_t &lo, uint32_t &hi) {
  asm("sub.cc.u32 %0, 0, %2;\n\t"
      "subc.u32   %1, %2, 0;"
      : "=&r"(lo), "=r"(hi)
      : "r"(z));
}
// c (2^32 - 1) for a carry c in {0, 1}, added to (r0, r1) with carry: -c in the low word (an ALU
// negation instead of two multiply-adds c (2^32 - 1): with fold_hi's ALU form, 1809.5 -> 1789.2 ms).
#define HB_GL_ADD_EPS_C \
  "neg.s32        c, c;\n\t" \
  "add.cc.u32     %0, %0, c;\n\t" \
  "addc.u32       %1, %1, 0;\n\t"

// a * b folded to [0, 2^64) (not necessarily canonical).
// Product limbs x0..x3, then x = lo + x2 2^64 + x3 2^96 = lo + x2 (2^32 - 1) - x3 (mod Q):
//   A = x2 (2^32 - 1) + (2^32 - 1 - x3)  (fits 64 bits), r = lo + A = x + (2^32 - 1) + c 2^64,
//   so x = r - (1 - c)(2^32 - 1) mod Q, with one more -(2^32 - 1) if that subtraction borrows.
__device__ __forceinline__ uint64_t mul_lazy(uint64_t a, uint64_t b) {
  uint32_t a0, a1, b0, b1;
  split(a, a0, a1);
  split(b, b0, b1);
  uint32_t x0, x1, x2, x3;
  asm("mul.lo.u32     %0, %4, %6;\n\t"
      "mul.hi.u32     %1, %4, %6;\n\t"
      "mad.lo.cc.u32  %1, %4, %7, %1;\n\t"
      "madc.hi.u32    %2, %4, %7, 0;\n\t"
      "mad.lo.cc.u32  %1, %5, %6, %1;\n\t"
      "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
      "madc.hi.u32    %3, %5, %7, 0;\n\t"
      "mad.lo.cc.u32  %2, %5, %7, %2;\n\t"
      "addc.u32       %3, %3, 0;"
      : "=&r"(x0), "=&r"(x1), "=&r"(x2), "=&r"(x3)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
  const uint64_t A = fold_hi(x2, x3);
  uint32_t A0, A1;
  split(A, A0, A1);
  uint32_t r0, r1;
  asm("{\n\t.reg .u32 c, m, bw;\n\t"
      "add.cc.u32  %0, %2, %4;\n\t"
      "addc.cc.u32 %1, %3, %5;\n\t"
      "addc.u32    c, 0, 0;\n\t"
      "add.u32     m, c, 0xFFFFFFFF;\n\t"  // c - 1: 0 when carried, 2^32-1 otherwise
      "sub.cc.u32  %0, %0, m;\n\t"
      "subc.cc.u32 %1, %1, 0;\n\t"
      "subc.u32    bw, 0, 0;\n\t"
      "sub.cc.u32  %0, %0, bw;\n\t"
      "subc.u32    %1, %1, 0;\n\t}"
      : "=&r"(r0), "=&r"(r1)
      : "r"(x0), "r"(x1), "r"(A0), "r"(A1));
  return join(r0, r1);
}

// Canonical residue of the 128-bit value x0 + x1 2^32 + x2 2^64 + x3 2^96 (32-bit limbs). With
// A = x2 (2^32 - 1) + (2^32 - 1 - x3) (fits 64 bits, A <= 2^64 - 2^32 < Q), lo + A = r + c 2^64 and
// the value is r + (c - 1)(2^32 - 1) (mod Q):
//  * c = 1: r < A <= Q - 1, so r is the canonical result;
//  * c = 0: r - (2^32 - 1) <= Q - 1 when that does not borrow, and r - 2 (2^32 - 1) + 2^64 < Q
//    when it does (then r < 2^32 - 1).
// m = c - 1 (0 or 2^32 - 1) makes both cases one subtraction of m with a borrow fix-up. (Adding
// c (2^32 - 1) with two multiply-adds first and subtracting the constant measured 2.7 % slower in
// the bootstrapping kernel: one more instruction.)
__device__ __forceinline__ uint64_t reduce_canon_lo(uint32_t x0, uint32_t x1, uint64_t A) {
  uint32_t A0, A1;
  split(A, A0, A1);
  uint32_t r0, r1;
  asm("{\n\t.reg .u32 c, m, bw;\n\t"
      "add.cc.u32  %0, %2, %4;\n\t"
      "addc.cc.u32 %1, %3, %5;\n\t"
      "addc.u32    c, 0, 0;\n\t"
      "add.u32     m, c, 0xFFFFFFFF;\n\t"
      "sub.cc.u32  %0, %0, m;\n\t"
      "subc.cc.u32 %1, %1, 0;\n\t"
      "subc.u32    bw, 0, 0;\n\t"
      "sub.cc.u32  %0, %0, bw;\n\t"
      "subc.u32    %1, %1, 0;\n\t}"
      : "=&r"(r0), "=&r"(r1)
      : "r"(x0), "r"(x1), "r"(A0), "r"(A1));
  return join(r0, r1);
}
__device__ __forceinline__ uint64_t reduce_canon(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3) {
  return reduce_canon_lo(x0, x1, fold_hi(x2, x3));
}
// reduce_canon with x3 = 0: A = x2 (2^32 - 1) + (2^32 - 1) = x2 2^32 + (2^32 - 1 - x2), no borrow.
__device__ __forceinline__ uint64_t reduce_canon_x3zero(uint32_t x0, uint32_t x1, uint32_t x2) {
  return reduce_canon_lo(x0, x1, join(~x2, x2));
}

// reduce_canon with x0 = 0: the low limb of lo + A is A0 and cannot carry (one instruction fewer
// than reduce_canon; with the x3 = 0 form above, 1.0 % off the bootstrapping kernel).
__device__ __forceinline__ uint64_t reduce_canon_x0zero(uint32_t x1, uint32_t x2, uint32_t x3) {
  const uint64_t A = fold_hi(x2, x3);
  uint32_t A0, A1;
  split(A, A0, A1);
  uint32_t r0, r1;
  asm("{\n\t.reg .u32 c, m, bw;\n\t"
      "add.cc.u32  %1, %2, %3;\n\t"
      "addc.u32    c, 0, 0;\n\t"
      "add.u32     m, c, 0xFFFFFFFF;\n\t"
      "sub.cc.u32  %0, %4, m;\n\t"
      "subc.cc.u32 %1, %1, 0;\n\t"
      "subc.u32    bw, 0, 0;\n\t"
      "sub.cc.u32  %0, %0, bw;\n\t"
      "subc.u32    %1, %1, 0;\n\t}"
      : "=&r"(r0), "=&r"(r1)
      : "r"(x1), "r"(A1), "r"(A0));
  return join(r0, r1);
}

// a * b mod Q, canonical: the 128-bit product's limbs, then reduce_canon. The product is left to
// the compiler's 64-bit multiply lowering (measured faster here than a hand-written chain of
// 32-bit mad.lo.cc / madc.hi.cc, whose single carry flag serialises it, and than four
// mad.wide.u32 with 64-bit addends and no carry flags: 1.4 % slower in the bootstrapping kernel).
__device__ __forceinline__ uint64_t mul_canon(uint64_t a, uint64_t b) {
  const uint64_t lo = a * b, hi = __umul64hi(a, b);
  return reduce_canon((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
}

// Lazy multiply-accumulate for sums of products: (acc + cnt 2^64) += lo + A, where lo, x2, x3 are
// the 128-bit product's limbs and A = x2 (2^32 - 1) + (2^32 - 1 - x3), so lo + A = a b + (2^32 - 1)
// (mod Q) and nothing is reduced per product; cnt counts the carries out of 64 bits. After m calls
// the sum of the products is acc + cnt (2^32 - 1) - m (2^32 - 1) (mod Q): mac_lazy_value.
__device__ __forceinline__ void mac_lazy(uint64_t &acc, uint32_t &cnt, uint64_t a, uint64_t b) {
  uint32_t x0, x1, x2, x3;
  uint32_t a0, a1, b0, b1;
  split(a, a0, a1);
  split(b, b0, b1);
  asm("mul.lo.u32     %0, %4, %6;\n\t"
      "mul.hi.u32     %1, %4, %6;\n\t"
      "mad.lo.cc.u32  %1, %4, %7, %1;\n\t"
      "madc.hi.u32    %2, %4, %7, 0;\n\t"
      "mad.lo.cc.u32  %1, %5, %6, %1;\n\t"
      "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
      "madc.hi.u32    %3, %5, %7, 0;\n\t"
      "mad.lo.cc.u32  %2, %5, %7, %2;\n\t"
      "addc.u32       %3, %3, 0;"
      : "=&r"(x0), "=&r"(x1), "=&r"(x2), "=&r"(x3)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
  const uint64_t A = fold_hi(x2, x3);
  uint32_t A0, A1, c0, c1;
  split(A, A0, A1);
  split(acc, c0, c1);
  asm("add.cc.u32  %0, %0, %3;\n\t"
      "addc.cc.u32 %1, %1, %4;\n\t"
      "addc.u32    %2, %2, 0;\n\t"
      "add.cc.u32  %0, %0, %5;\n\t"
      "addc.cc.u32 %1, %1, %6;\n\t"
      "addc.u32    %2, %2, 0;"
      : "+r"(c0), "+r"(c1), "+r"(cnt)
      : "r"(x0), "r"(x1), "r"(A0), "r"(A1));
  acc = join(c0, c1);
}

// y * 2^E mod Q, canonical, for a compile-time 0 < E < 96 (the twiddles of the first forward
// stages are such powers of two). The limbs of y 2^E come from shifts instead of multiplies:
//  * E < 64: y 2^E < 2^128, reduced by reduce_canon;
//  * E >= 64: y 2^E = z 2^64 + H 2^96 with z = (y 2^(E-64)) mod 2^32 and H = y >> (96 - E), so the
//    value is z (2^32 - 1) - H. z (2^32 - 1) < Q; when the subtraction borrows, the wrapped word
//    is at least 2^64 - H and removing one more 2^32 - 1 lands in [0, Q).
template <int E>
__device__ __forceinline__ uint64_t mul_pow2(uint64_t y) {
  static_assert(E > 0 && E < 96, "exponent out of range");
  uint32_t y0, y1;
  split(y, y0, y1);
  if constexpr (E < 32) {
    return reduce_canon_x3zero(y0 << E, __funnelshift_l(y0, y1, E), y1 >> (32 - E));
  } else if constexpr (E == 32) {
    return reduce_canon_x0zero(y0, y1, 0u);
  } else if constexpr (E < 64) {
    constexpr int e = E - 32;
    return reduce_canon_x0zero(y0 << e, __funnelshift_l(y0, y1, e), y1 >> (32 - e));
  } else {
    constexpr int e = E - 64;
    const uint32_t z = y0 << e;
    const uint64_t H = y >> (96 - E);
    uint32_t h0, h1;
    split(H, h0, h1);
    uint32_t A0, A1;
    times_eps(z, A0, A1);
    uint32_t d0, d1;
    asm("{\n\t.reg .u32 bw;\n\t"
        "sub.cc.u32  %0, %2, %4;\n\t"
        "subc.cc.u32 %1, %3, %5;\n\t"
        "subc.u32    bw, 0, 0;\n\t"
        "sub.cc.u32  %0, %0, bw;\n\t"
        "subc.u32    %1, %1, 0;\n\t}"
        : "=&r"(d0), "=&r"(d1)
        : "r"(A0), "r"(A1), "r"(h0), "r"(h1));
    return join(d0, d1);
  }
}

// Canonical representative: r >= Q exactly when r + (2^32 - 1) carries out of 64 bits.
__device__ __forceinline__ uint64_t canon(uint64_t r) {
  uint32_t r0, r1;
  split(r, r0, r1);
  asm("{\n\t.reg .u32 t0, t1, c;\n\t"
      "add.cc.u32     t0, %0, 0xFFFFFFFF;\n\t"
      "addc.cc.u32    t1, %1, 0;\n\t"
      "addc.u32       c, 0, 0;\n\t"
      HB_GL_ADD_EPS_C "}"
      : "+r"(r0), "+r"(r1));
  return join(r0, r1);
}

__device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) { return canon(mul_lazy(a, b)); }

// a + b with b < Q: at most one carry, worth 2^32 - 1, and adding it cannot carry again.
__device__ __forceinline__ uint64_t add_c(uint64_t a, uint64_t b) {
  uint32_t a0, a1, b0, b1;
  split(a, a0, a1);
  split(b, b0, b1);
  uint32_t s0, s1;
  asm("{\n\t.reg .u32 c;\n\t"
      "add.cc.u32     %0, %2, %4;\n\t"
      "addc.cc.u32    %1, %3, %5;\n\t"
      "addc.u32       c, 0, 0;\n\t"
      HB_GL_ADD_EPS_C "}"
      : "=&r"(s0), "=&r"(s1)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
  return join(s0, s1);
}

// a - b with b < Q: at most one borrow, worth -(2^32 - 1), and removing it cannot borrow again.
__device__ __forceinline__ uint64_t sub_c(uint64_t a, uint64_t b) {
  uint32_t a0, a1, b0, b1;
  split(a, a0, a1);
  split(b, b0, b1);
  uint32_t d0, d1;
  asm("{\n\t.reg .u32 bw;\n\t"
      "sub.cc.u32  %0, %2, %4;\n\t"
      "subc.cc.u32 %1, %3, %5;\n\t"
      "subc.u32    bw, 0, 0;\n\t"
      "sub.cc.u32  %0, %0, bw;\n\t"
      "subc.u32    %1, %1, 0;\n\t}"
      : "=&r"(d0), "=&r"(d1)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
  return join(d0, d1);
}

// Value of a lazy accumulator as a 64-bit representative: acc + cnt (2^32 - 1) + off, where
// off = Q - m (2^32 - 1) removes the offsets of the m products (cnt (2^32 - 1) < 2^38 and off < Q,
// so both additions take the one-carry form).
__device__ __forceinline__ uint64_t mac_lazy_value(uint64_t acc, uint32_t cnt, uint64_t off) {
  uint32_t t0, t1;
  times_eps(cnt, t0, t1);
  const uint64_t t = join(t0, t1);
  return add_c(add_c(acc, t), off);
}

}  // namespace glx
}  // namespace hb
