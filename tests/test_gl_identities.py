"""The carry-chain forms of hasteboots_b200/csrc/hb_gl_ptx.cuh modelled limb by limb with PTX's
add.cc / addc / sub.cc / subc semantics (32-bit limbs, one carry or borrow flag) and checked
against exact arithmetic mod Q = 2^64 - 2^32 + 1 on random and edge words: fold_hi (A = x2 (2^32 - 1)
+ (2^32 - 1 - x3)), times_eps (z (2^32 - 1)), the ALU carry correction of add_c / canon, and the
canonical reduction of a 128-bit product built on them. The GPU parity tests check the compiled
code bit-exactly against the oracle; this pins the identities the forms rely on."""

import random

Q = (1 << 64) - (1 << 32) + 1
M32 = (1 << 32) - 1


class Chain:
    """One PTX carry flag over 32-bit limbs."""

    def __init__(self):
        self.cf = 0

    def add_cc(self, a, b, carry_in=False):
        s = a + b + (self.cf if carry_in else 0)
        self.cf = s >> 32
        return s & M32

    def addc(self, a, b):
        return (a + b + self.cf) & M32

    def sub_cc(self, a, b, borrow_in=False):
        d = a - b - (self.cf if borrow_in else 0)
        self.cf = 1 if d < 0 else 0
        return d & M32

    def subc(self, a, b):
        return (a - b - self.cf) & M32


def fold_hi(x2, x3):
    c = Chain()
    a0 = c.sub_cc((~x3) & M32, x2)
    a1 = c.subc(x2, 0)
    return a0 | (a1 << 32)


def times_eps(z):
    c = Chain()
    lo = c.sub_cc(0, z)
    hi = c.subc(z, 0)
    return lo | (hi << 32)


def add_eps_c(r0, r1, carry):
    # neg.s32 c; add.cc r0, r0, c; addc r1, r1, 0
    c = Chain()
    m = (-carry) & M32
    r0 = c.add_cc(r0, m)
    r1 = c.addc(r1, 0)
    return r0 | (r1 << 32)


def add_c(a, b):
    c = Chain()
    s0 = c.add_cc(a & M32, b & M32)
    s1 = c.add_cc(a >> 32, b >> 32, carry_in=True)
    carry = c.cf
    return add_eps_c(s0, s1, carry)


def canon(r):
    c = Chain()
    c.add_cc(r & M32, M32)
    c.add_cc(r >> 32, 0, carry_in=True)
    return add_eps_c(r & M32, r >> 32, c.cf)


def reduce_canon(x0, x1, x2, x3):
    A = fold_hi(x2, x3)
    c = Chain()
    r0 = c.add_cc(x0, A & M32)
    r1 = c.add_cc(x1, A >> 32, carry_in=True)
    carry = c.cf
    m = (carry + M32) & M32  # c - 1
    r0 = c.sub_cc(r0, m)
    r1 = c.sub_cc(r1, 0, borrow_in=True)
    bw = c.subc(0, 0)
    r0 = c.sub_cc(r0, bw)
    r1 = c.subc(r1, 0)
    return r0 | (r1 << 32)


def words(rng, n):
    edges = [0, 1, 2, M32 - 1, M32, M32 + 1, Q - 2, Q - 1, Q, Q + 1, (1 << 64) - 2, (1 << 64) - 1]
    return edges + [rng.randrange(1 << 64) for _ in range(n)]


def test_fold_hi_and_times_eps():
    rng = random.Random(5)
    limbs = [0, 1, M32 - 1, M32] + [rng.randrange(1 << 32) for _ in range(3000)]
    for x2 in limbs[:60]:
        for x3 in limbs:
            assert fold_hi(x2, x3) == x2 * M32 + (M32 - x3)
    for z in limbs:
        assert times_eps(z) == z * M32


def test_add_c_and_canon():
    rng = random.Random(6)
    ws = words(rng, 2000)
    canon_ws = [w for w in ws if w < Q]
    for a in ws:
        r = canon(a)
        assert r < Q and r == a % Q
        for b in canon_ws[:40]:
            s = add_c(a, b)
            assert s < (1 << 64) and s % Q == (a + b) % Q


def test_reduce_canon_of_products():
    rng = random.Random(7)
    ws = words(rng, 3000)
    for a, b in zip(ws, reversed(ws)):
        x = a * b
        limbs = [(x >> (32 * i)) & M32 for i in range(4)]
        r = reduce_canon(*limbs)
        assert r < Q and r == x % Q, (a, b)
    # the extreme 128-bit values
    for x in ((1 << 128) - 1, (1 << 64) * ((1 << 64) - 1), Q * Q, (Q - 1) * (Q - 1)):
        limbs = [(x >> (32 * i)) & M32 for i in range(4)]
        assert reduce_canon(*limbs) == x % Q
