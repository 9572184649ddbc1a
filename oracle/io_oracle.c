/*
 * io_oracle.c -- CPU restatement of the checksums of gauge-field files.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for qex_b200/csrc/gaugeio.cu.
 *
 * Follows (paths relative to the QEX source tree):
 *  - CRC-32, reflected polynomial 0xEDB88320, table per byte, initial value
 *    and final complement all ones: src/io/crc32.nim:1-40; its known answer
 *    crc32("The quick brown fox jumps over the lazy dog") = 0x414FA339 is
 *    src/io/crc32.nim:103-106, checked in tests/test_gaugeio.py.
 *  - MILC checksum, word k rotated left by k mod 29 and k mod 31 and XORed:
 *    src/new/milcIO.nim:44-55.  milcIO.nim writes the rotation as
 *    (t shl k) + (t shr (32-k)), which for k = 0 shifts a 32-bit word by 32
 *    (undefined in the C it compiles to); MILC's own format rotates, so
 *    k = 0 leaves the word unchanged here.
 *  - SciDAC checksum: the SciDAC reader and writer QEX uses live in the
 *    third-party qiolite package (required at "#head", unpinned, in
 *    qex.nimble; not vendored), which follows the USQCD QIO format: the
 *    CRC-32 of each site's bytes as stored, rotated left by (site rank
 *    mod 29) into suma and (mod 31) into sumb, XORed over sites.  Parity is
 *    anchored on QEX's call sites (src/gauge/gaugeUtils.nim:96-131,
 *    src/io/readerQiolite.nim, src/io/writerQiolite.nim) and the CRC known
 *    answer; no SciDAC file from QEX is available to pin it further.
 */
#include <stdint.h>
#include <stddef.h>

static uint32_t crc_table[256];
static int crc_ready = 0;

static void crc_init(void) {
  for (uint32_t i = 0; i < 256; i++) {
    uint32_t r = i;
    for (int j = 0; j < 8; j++) r = (r & 1u) ? (r >> 1) ^ 0xEDB88320u : r >> 1;
    crc_table[i] = r;
  }
  crc_ready = 1;
}

/* updateCrc32 over n bytes from crc (crc32.nim:18-25) */
uint32_t or_crc32_update(uint32_t crc, const uint8_t *p, size_t n) {
  if (!crc_ready) crc_init();
  for (size_t i = 0; i < n; i++) crc = (crc >> 8) ^ crc_table[(crc ^ p[i]) & 0xffu];
  return crc;
}

/* crc32 (crc32.nim:35-38): initial all ones, final complement */
uint32_t or_crc32(const uint8_t *p, size_t n) { return ~or_crc32_update(0xffffffffu, p, n); }

static uint32_t rotl(uint32_t x, unsigned k) { return k ? (x << k) | (x >> (32 - k)) : x; }

/* SciDAC checksum of nsites records of size bytes each, site rank = index */
void or_scidac_checksum(const uint8_t *data, long nsites, long size, uint32_t *suma, uint32_t *sumb) {
  uint32_t a = 0, b = 0;
  for (long r = 0; r < nsites; r++) {
    const uint32_t c = or_crc32(data + (size_t)r * size, (size_t)size);
    a ^= rotl(c, (unsigned)(r % 29));
    b ^= rotl(c, (unsigned)(r % 31));
  }
  *suma = a;
  *sumb = b;
}

/* MILC checksum of n 32-bit words (milcIO.nim:44-55) */
void or_milc_checksum(const uint32_t *w, long n, uint32_t *sum29, uint32_t *sum31) {
  uint32_t a = 0, b = 0;
  for (long k = 0; k < n; k++) {
    a ^= rotl(w[k], (unsigned)(k % 29));
    b ^= rotl(w[k], (unsigned)(k % 31));
  }
  *sum29 = a;
  *sum31 = b;
}
