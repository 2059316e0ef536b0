"""The 32-bit fields' arithmetic (hasteboots_b200/csrc/hb_field.cuh, Mont32) compiled for the host
with g++ and checked against exact integer arithmetic: the multiply-accumulate (DefaultFieldU32's
64-bit unreduced sums with residue-keeping folds, forced here at every spacing up to FOLD and at the
extreme word values, and BabyBear's per-product reduction; the value of a sum of products x k is
sum(x k) 2^-32 mod P, since the keys it multiplies are stored in Montgomery form), and the Shoup
twiddle product and butterflies of the NTT tables (Mont32::make_tw, shoup, ct, gs)."""

import os
import random
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "hasteboots_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include "hb_field.cuh"
template <class F>
void run() {
  using W = typename F::W;
  unsigned n, fold;
  while (scanf("%u %u", &n, &fold) == 2) {
    typename F::Acc a;
    F::acc_clear(a);
    for (unsigned i = 0; i < n; ++i) {
      unsigned x, k;
      if (scanf("%u %u", &x, &k) != 2) return;
      if (fold && i && i % fold == 0) F::acc_fold(a);
      F::acc_mac(a, (W)x, (W)k);
    }
    printf("%u\n", (unsigned)F::acc_value(a, 0));
  }
}
template <class F>
void run_shoup() {
  using W = typename F::W;
  unsigned a, w, x, y;
  // "a w x y": shoup(a, w) and the CT / GS butterflies of (x, y) with twiddle w
  while (scanf("%u %u %u %u", &a, &w, &x, &y) == 4) {
    const typename F::Tw t = F::make_tw((W)w);
    W cx = (W)x, cy = (W)y, gx = (W)x, gy = (W)y;
    F::ct(cx, cy, t);
    F::gs(gx, gy, t);
    printf("%u %u %u %u %u\n", (unsigned)F::shoup((W)a, t.w, t.q), (unsigned)cx, (unsigned)cy, (unsigned)gx,
           (unsigned)gy);
  }
}
template <class F>
void run_pairs() {
  using W = typename F::W;
  unsigned n;
  // "n x1 k1 y1 l1 ...": n pair steps a += x k + y l from zero
  while (scanf("%u", &n) == 1) {
    typename F::Acc a;
    F::acc_clear(a);
    for (unsigned i = 0; i < n; ++i) {
      unsigned x, k, y, l;
      if (scanf("%u %u %u %u", &x, &k, &y, &l) != 4) return;
      F::acc_mac2(a, (W)x, (W)k, (W)y, (W)l);
    }
    printf("%u\n", (unsigned)F::acc_value(a, 0));
  }
}
int main(int argc, char **argv) {
  if (argv[1][0] == 'p') {
    if (argv[1][1] == 'd') run_pairs<hb::DefaultFieldU32>(); else run_pairs<hb::BabyBear>();
    return 0;
  }
  if (argv[1][0] == 's') {
    if (argv[1][1] == 'd') run_shoup<hb::DefaultFieldU32>(); else run_shoup<hb::BabyBear>();
    return 0;
  }
  if (argv[1][0] == 'd') run<hb::DefaultFieldU32>(); else run<hb::BabyBear>();
  printf("FOLD %d\n", argv[1][0] == 'd' ? hb::DefaultFieldU32::FOLD : hb::BabyBear::FOLD);
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver():
    d = tempfile.mkdtemp()
    src, exe = os.path.join(d, "acc.cpp"), os.path.join(d, "acc")
    open(src, "w").write(DRIVER)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, src, "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("field,P", [("d", 132120577), ("b", 0x78000001)])
def test_accumulate_matches_exact_sums(driver, field, P):
    rng = random.Random(7)
    cases = []
    for n in (1, 2, 3, 8, 18, 27, 64):
        for fold in (0, 1, 2, 5, 16, 30):
            rows = [(rng.randrange(P), rng.randrange(P)) for _ in range(n)]
            cases.append((n, fold, rows))
    # the largest words, where the bounds are tight
    cases.append((40, 30, [(P - 1, P - 1)] * 40))
    cases.append((27, 0, [(P - 1, P - 1)] * 27))
    text = "".join(f"{n} {fold} " + " ".join(f"{x} {k}" for x, k in rows) + "\n" for n, fold, rows in cases)
    out = subprocess.run([driver, field], input=text, capture_output=True, text=True, check=True).stdout.split()
    fold_max = int(out[-1])
    assert out[-2] == "FOLD"
    rinv = pow(1 << 32, -1, P)
    for (n, fold, rows), got in zip(cases, out[:-2]):
        if field == "d":
            # a case only makes sense where the products between folds stay within FOLD
            span = fold if fold else n
            if span > fold_max:
                continue
        expect = sum(x * k for x, k in rows) * rinv % P
        assert int(got) == expect, (n, fold)
    if field == "d":
        assert fold_max >= 27  # DEFAULT_TERNARY's key switch sums 27 products without a fold


@pytest.mark.parametrize("field,P", [("d", 132120577), ("b", 0x78000001)])
def test_shoup_twiddle_products_are_exact(driver, field, P):
    rng = random.Random(11)
    M = 1 << 32
    cases = [(rng.randrange(M), rng.randrange(P), rng.randrange(P), rng.randrange(P)) for _ in range(4000)]
    for a in (0, 1, P - 1, P, M - 1):
        for w in (0, 1, P - 1):
            cases.append((a, w, P - 1, P - 1))
            cases.append((a, w, 0, P - 1))
    text = "".join(f"{a} {w} {x} {y}\n" for a, w, x, y in cases)
    out = subprocess.run([driver, "s" + field], input=text, capture_output=True, text=True, check=True).stdout.split("\n")
    for (a, w, x, y), line in zip(cases, out):
        r, cx, cy, gx, gy = map(int, line.split())
        assert r == a * w % P, (a, w)
        # CT: (x + w y, x - w y); GS: (x + y, (x - y) w), canonical
        assert (cx, cy) == ((x + w * y) % P, (x - w * y) % P), (x, y, w)
        assert (gx, gy) == ((x + y) % P, (x - y) * w % P), (x, y, w)


@pytest.mark.parametrize("field,P", [("d", 132120577), ("b", 0x78000001)])
def test_pair_accumulate_matches_exact_sums(driver, field, P):
    """Mont32::acc_mac2: the two products of a pair share one reduction (BabyBear) or add to the
    64-bit sum (DefaultFieldU32); value sum(x k + y l) 2^-32 mod P."""
    rng = random.Random(13)
    cases = []
    for n in (1, 2, 4, 7, 13):
        cases.append([tuple(rng.randrange(P) for _ in range(4)) for _ in range(n)])
    cases.append([(P - 1, P - 1, P - 1, P - 1)] * 13)
    cases.append([(P - 1, P - 1, 0, 0), (0, 0, P - 1, P - 1)])
    text = "".join(f"{len(c)} " + " ".join(" ".join(map(str, q)) for q in c) + "\n" for c in cases)
    out = subprocess.run([driver, "p" + field], input=text, capture_output=True, text=True, check=True).stdout.split()
    rinv = pow(1 << 32, -1, P)
    for c, got in zip(cases, out):
        expect = sum(x * k + y * l for x, k, y, l in c) * rinv % P
        assert int(got) == expect, c[:2]

