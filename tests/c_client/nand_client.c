/* A C client of libhb_gpu.so, the binding a C or Rust caller writes against include/hb_gpu.h: the
 * NAND gate of the reference's nand_babybear example (tfhe/examples/nand_babybear.rs) over the C ABI.
 *
 *   nand_client <preset> <count> <c0 file> <c1 file> <out file>
 *
 * Generates the preset's keys on the device from seed 0 (hb_keys_generate), reads count
 * ciphertext pairs (canonical little-endian words), bootstraps NAND on host buffers (hb_gate),
 * writes the output ciphertexts and prints the decrypted bits. Returns 0 on success. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "hb_gpu.h"

static int fail(hb_ctx *ctx, int rc, const char *what) {
  char msg[512] = "";
  if (ctx) hb_last_error(ctx, msg, sizeof(msg));
  fprintf(stderr, "%s failed with status %d: %s\n", what, rc, msg);
  return 1;
}

static void *read_file(const char *path, size_t bytes) {
  FILE *f = fopen(path, "rb");
  void *buf = f ? malloc(bytes) : NULL;
  if (!f || !buf || fread(buf, 1, bytes, f) != bytes) {
    free(buf);
    buf = NULL;
  }
  if (f) fclose(f);
  return buf;
}

int main(int argc, char **argv) {
  if (argc != 6) {
    fprintf(stderr, "usage: nand_client <preset> <count> <c0> <c1> <out>\n");
    return 2;
  }
  const int preset = atoi(argv[1]);
  const size_t count = (size_t)atol(argv[2]);
  hb_params p;
  int rc = hb_params_preset(preset, &p);
  if (rc) return fail(NULL, rc, "hb_params_preset");
  size_t n_lwe_sk = 0, n_ring_sk = 0, width = 0;
  rc = hb_params_sizes(&p, &n_lwe_sk, &n_ring_sk, NULL, NULL, &width);
  if (rc) return fail(NULL, rc, "hb_params_sizes");
  const size_t ws = p.field_id == HB_FIELD_GOLDILOCKS ? 8 : 4, bytes = count * width * ws;

  hb_ctx *ctx = NULL;
  rc = hb_ctx_create(0, 0, &ctx);
  if (rc) return fail(NULL, rc, "hb_ctx_create");
  void *lwe_sk = malloc(n_lwe_sk * ws), *ring_sk = malloc(n_ring_sk * ws);
  hb_keys *keys = NULL;
  rc = hb_keys_generate(ctx, &p, 0, lwe_sk, ring_sk, &keys);
  if (rc) return fail(ctx, rc, "hb_keys_generate");

  void *c0 = read_file(argv[3], bytes), *c1 = read_file(argv[4], bytes), *out = malloc(bytes);
  if (!c0 || !c1 || !out) {
    fprintf(stderr, "cannot read %zu bytes of ciphertexts\n", bytes);
    return 1;
  }
  rc = hb_gate(ctx, keys, HB_GATE_NAND, c0, c1, NULL, out, count);
  if (rc) return fail(ctx, rc, "hb_gate");

  uint8_t *bits = malloc(count);
  rc = hb_decrypt(&p, lwe_sk, out, count, bits, NULL);
  if (rc) return fail(ctx, rc, "hb_decrypt");
  for (size_t i = 0; i < count; ++i) printf("%u", (unsigned)bits[i]);
  printf("\n");

  FILE *f = fopen(argv[5], "wb");
  if (!f || fwrite(out, 1, bytes, f) != bytes) return fail(ctx, -1, "writing the outputs");
  fclose(f);
  hb_keys_free(ctx, keys);
  hb_ctx_destroy(ctx);
  free(lwe_sk);
  free(ring_sk);
  free(c0);
  free(c1);
  free(out);
  free(bits);
  return 0;
}
