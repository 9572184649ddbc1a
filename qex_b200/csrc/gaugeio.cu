// gaugeio.cu -- gauge-field files into and out of the device link layout.
//
// Formats (QEX reads and writes gauge fields with loadGauge / saveGauge,
// src/gauge/gaugeUtils.nim:96-131, through src/io/readerQiolite.nim and
// src/io/writerQiolite.nim over the third-party qiolite package; MILC
// binary files with src/new/milcIO.nim):
//  - SciDAC single-file (LIME records, the USQCD QIO layout), also ILDG:
//    big-endian IEEE F32 or F64, sites in lexicographic order (x0 fastest),
//    per site the 4 directions' 3x3 complex matrices, row-major.  Checksum:
//    CRC-32 of each site's bytes as stored, XORed over sites after a left
//    rotation by (site rank mod 29) for suma and (mod 31) for sumb.
//  - MILC binary (version 5): a 96-byte header (magic 20103, dims, time
//    stamp, order, sum29, sum31) then F32 links in the writer's byte order,
//    same site order; checksum over the 32-bit words, word k rotated left
//    by k mod 29 / k mod 31 (milcIO.nim:44-55).
//
// The host parses records and moves bytes; one kernel per direction of
// transfer does the byte order, the precision, the reordering into QEX's
// checkerboard site index and the checksum, with each block staging a
// contiguous run of sites through shared memory so that the file-order
// reads and the field writes are both coalesced.
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "lib.cuh"

namespace qs {

constexpr int kIoSites = 64;  // sites per block

// ---- CRC-32 (reflected, polynomial 0xEDB88320), slicing by 8 ----

struct CrcTables {
  uint32_t t[8][256];
};

static void make_crc_tables(CrcTables &c) {
  for (uint32_t i = 0; i < 256; i++) {
    uint32_t r = i;
    for (int j = 0; j < 8; j++) r = (r & 1u) ? (r >> 1) ^ 0xEDB88320u : r >> 1;
    c.t[0][i] = r;
  }
  for (int k = 1; k < 8; k++)
    for (int i = 0; i < 256; i++) c.t[k][i] = (c.t[k - 1][i] >> 8) ^ c.t[0][c.t[k - 1][i] & 0xffu];
}

// CRC-32 of n bytes (n a multiple of 8) at p in shared memory
__device__ __forceinline__ uint32_t crc32_smem(const uint32_t (*T)[256], const uint8_t *p, int n) {
  uint32_t crc = 0xffffffffu;
  for (int i = 0; i < n; i += 8) {
    const uint32_t lo = (uint32_t)p[i] | ((uint32_t)p[i + 1] << 8) | ((uint32_t)p[i + 2] << 16) |
                        ((uint32_t)p[i + 3] << 24);
    const uint32_t a = crc ^ lo;
    crc = T[7][a & 0xff] ^ T[6][(a >> 8) & 0xff] ^ T[5][(a >> 16) & 0xff] ^ T[4][a >> 24] ^ T[3][p[i + 4]] ^
          T[2][p[i + 5]] ^ T[1][p[i + 6]] ^ T[0][p[i + 7]];
  }
  return ~crc;
}

__device__ __forceinline__ uint32_t rotl32(uint32_t x, int k) { return k ? (x << k) | (x >> (32 - k)) : x; }

// QEX's checkerboard index of lexicographic site lex (all L even)
__device__ __forceinline__ int qex_index_of_lex(const Geom &g, int lex) {
  int t = fdiv(g, 0, lex);
  const int x0 = lex - t * g.L[0];
  int t2 = fdiv(g, 1, t);
  const int x1 = t - t2 * g.L[1];
  const int t3 = fdiv(g, 2, t2);
  const int x2 = t2 - t3 * g.L[2];
  const int par = (x0 + x1 + x2 + t3) & 1;
  return (lex >> 1) + (par ? g.nh : 0);
}

__device__ __forceinline__ double load_real(const uint8_t *p, int prec, bool swap) {
  if (prec == 8) {
    uint64_t u = 0;
#pragma unroll
    for (int b = 0; b < 8; b++) u |= (uint64_t)p[b] << (8 * (swap ? 7 - b : b));
    return __longlong_as_double((long long)u);
  }
  uint32_t u = 0;
#pragma unroll
  for (int b = 0; b < 4; b++) u |= (uint32_t)p[b] << (8 * (swap ? 3 - b : b));
  return (double)__uint_as_float(u);
}

__device__ __forceinline__ void store_real(uint8_t *p, double v, int prec, bool swap) {
  if (prec == 8) {
    const uint64_t u = (uint64_t)__double_as_longlong(v);
#pragma unroll
    for (int b = 0; b < 8; b++) p[b] = (uint8_t)(u >> (8 * (swap ? 7 - b : b)));
  } else {
    const uint32_t u = __float_as_uint((float)v);
#pragma unroll
    for (int b = 0; b < 4; b++) p[b] = (uint8_t)(u >> (8 * (swap ? 3 - b : b)));
  }
}

struct IoArgs {
  Geom g;
  uint8_t *payload;    // V * 4 * 18 * prec bytes, file order
  double2 *links;      // [4][9][V]
  const uint32_t *crc_tables;  // [8][256]
  unsigned *sums;      // [2] XOR accumulators
  int prec;            // 4 or 8 bytes per real
  int swap;            // file byte order differs from the device's
  int milc;            // MILC word checksum instead of SciDAC site CRCs
};

// XOR-reduce a and b over the block, then into sums (XOR is associative and
// commutative, so the result does not depend on the order of the atomics)
__device__ __forceinline__ void xor_sums(uint32_t a, uint32_t b, unsigned *sums) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a ^= __shfl_xor_sync(0xffffffffu, a, o);
    b ^= __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicXor(sums, a);
    atomicXor(sums + 1, b);
  }
}

__device__ __forceinline__ void site_sums(const IoArgs &A, const uint32_t (*T)[256], const uint8_t *sp,
                                          int sitebytes, int lex, uint32_t &a, uint32_t &b) {
  if (A.milc) {
    // words as numbers in the file's byte order, word k = lex * 72 + j
    const uint64_t k0 = (uint64_t)lex * 72;
    for (int j = 0; j < 72; j++) {
      uint32_t w = 0;
#pragma unroll
      for (int q = 0; q < 4; q++) w |= (uint32_t)sp[4 * j + q] << (8 * (A.swap ? 3 - q : q));
      const uint64_t k = k0 + j;
      a ^= rotl32(w, (int)(k % 29));
      b ^= rotl32(w, (int)(k % 31));
    }
  } else {
    const uint32_t crc = crc32_smem(T, sp, sitebytes);
    a ^= rotl32(crc, lex % 29);
    b ^= rotl32(crc, lex % 31);
  }
}

// file bytes -> device links, with the checksum of the bytes as read
__global__ void __launch_bounds__(kIoSites) gauge_unpack_kernel(const IoArgs A) {
  extern __shared__ __align__(16) uint8_t sm[];
  uint32_t(*T)[256] = (uint32_t(*)[256])sm;
  uint8_t *buf = sm + sizeof(uint32_t) * 8 * 256;
  const int sitebytes = 72 * A.prec;
  const int lex0 = blockIdx.x * kIoSites;
  const int nsite = min(kIoSites, A.g.V - lex0);
  for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&T[0][0])[i] = A.crc_tables[i];
  // the block's sites are one contiguous run of the payload
  const uint4 *src = (const uint4 *)(A.payload + (size_t)lex0 * sitebytes);
  uint4 *dst = (uint4 *)buf;
  const int nvec = nsite * sitebytes / 16;
  for (int i = threadIdx.x; i < nvec; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  uint32_t a = 0, b = 0;
  if (threadIdx.x < nsite) {
    const int lex = lex0 + threadIdx.x;
    const uint8_t *sp = buf + threadIdx.x * sitebytes;
    site_sums(A, T, sp, sitebytes, lex, a, b);
    const int idx = qex_index_of_lex(A.g, lex);
    const size_t V = (size_t)A.g.V;
    for (int mu = 0; mu < 4; mu++)
#pragma unroll
      for (int e = 0; e < 9; e++) {
        const uint8_t *q = sp + (size_t)(mu * 18 + 2 * e) * A.prec;
        A.links[((size_t)mu * 9 + e) * V + idx] =
            make_double2(load_real(q, A.prec, A.swap), load_real(q + A.prec, A.prec, A.swap));
      }
  }
  xor_sums(a, b, A.sums);
}

// device links -> file bytes, with the checksum of the bytes written
__global__ void __launch_bounds__(kIoSites) gauge_pack_kernel(const IoArgs A) {
  extern __shared__ __align__(16) uint8_t sm[];
  uint32_t(*T)[256] = (uint32_t(*)[256])sm;
  uint8_t *buf = sm + sizeof(uint32_t) * 8 * 256;
  const int sitebytes = 72 * A.prec;
  const int lex0 = blockIdx.x * kIoSites;
  const int nsite = min(kIoSites, A.g.V - lex0);
  for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&T[0][0])[i] = A.crc_tables[i];
  __syncthreads();
  uint32_t a = 0, b = 0;
  if (threadIdx.x < nsite) {
    const int lex = lex0 + threadIdx.x;
    uint8_t *sp = buf + threadIdx.x * sitebytes;
    const int idx = qex_index_of_lex(A.g, lex);
    const size_t V = (size_t)A.g.V;
    for (int mu = 0; mu < 4; mu++)
#pragma unroll
      for (int e = 0; e < 9; e++) {
        const double2 v = A.links[((size_t)mu * 9 + e) * V + idx];
        uint8_t *q = sp + (size_t)(mu * 18 + 2 * e) * A.prec;
        store_real(q, v.x, A.prec, A.swap);
        store_real(q + A.prec, v.y, A.prec, A.swap);
      }
    site_sums(A, T, sp, sitebytes, lex, a, b);
  }
  __syncthreads();
  uint4 *dst = (uint4 *)(A.payload + (size_t)lex0 * sitebytes);
  const uint4 *src = (const uint4 *)buf;
  const int nvec = nsite * sitebytes / 16;
  for (int i = threadIdx.x; i < nvec; i += blockDim.x) dst[i] = src[i];
  xor_sums(a, b, A.sums);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static bool host_little_endian() {
  const uint16_t x = 1;
  uint8_t b;
  std::memcpy(&b, &x, 1);
  return b == 1;
}

static uint64_t be64(const uint8_t *p) {
  uint64_t v = 0;
  for (int i = 0; i < 8; i++) v = (v << 8) | p[i];
  return v;
}
static uint32_t be32(const uint8_t *p) { return ((uint32_t)p[0] << 24) | (p[1] << 16) | (p[2] << 8) | p[3]; }
static void put_be64(uint8_t *p, uint64_t v) {
  for (int i = 7; i >= 0; i--) {
    p[i] = (uint8_t)v;
    v >>= 8;
  }
}
static void put_be32(uint8_t *p, uint32_t v) {
  for (int i = 3; i >= 0; i--) {
    p[i] = (uint8_t)v;
    v >>= 8;
  }
}

constexpr uint32_t kLimeMagic = 0x456789abu;
constexpr int kMilcMagic = 20103;

struct LimeRecord {
  std::string type;
  uint64_t offset;  // of the data
  uint64_t length;
};

static bool lime_scan(FILE *f, std::vector<LimeRecord> &recs) {
  uint8_t h[144];
  uint64_t pos = 0;
  while (std::fread(h, 1, 144, f) == 144) {
    if (be32(h) != kLimeMagic) return false;
    LimeRecord r;
    r.length = be64(h + 8);
    char type[129];
    std::memcpy(type, h + 16, 128);
    type[128] = 0;
    r.type = type;
    r.offset = pos + 144;
    recs.push_back(r);
    pos = r.offset + ((r.length + 7) / 8) * 8;
    if (fseeko(f, (off_t)pos, SEEK_SET) != 0) return false;
  }
  return !recs.empty();
}

static std::string read_text(FILE *f, const LimeRecord &r) {
  std::string s(r.length, '\0');
  if (fseeko(f, (off_t)r.offset, SEEK_SET) != 0 || std::fread(&s[0], 1, r.length, f) != r.length) return "";
  const size_t z = s.find('\0');
  if (z != std::string::npos) s.resize(z);
  return s;
}

// text between <tag> and </tag> (the first occurrence), or "" when absent
static std::string xml_tag(const std::string &x, const std::string &tag) {
  const size_t a = x.find("<" + tag + ">");
  if (a == std::string::npos) return "";
  const size_t b = x.find("</" + tag + ">", a);
  if (b == std::string::npos) return "";
  return x.substr(a + tag.size() + 2, b - a - tag.size() - 2);
}

static const LimeRecord *find_rec(const std::vector<LimeRecord> &recs, const char *type) {
  for (const auto &r : recs)
    if (r.type == type) return &r;
  return nullptr;
}

static void fill_text(char *dst, size_t n, const std::string &s) {
  if (!dst || n == 0) return;
  const size_t m = std::min(n - 1, s.size());
  std::memcpy(dst, s.data(), m);
  dst[m] = 0;
}

struct FileCloser {
  FILE *f;
  ~FileCloser() {
    if (f) std::fclose(f);
  }
};

struct DevBuf {
  void *p = nullptr;
  ~DevBuf() {
    if (p) {
      cudaStreamSynchronize(stream());
      cudaFree(p);
    }
  }
};

static int crc_tables_dev(uint32_t **out) {
  // built once per device and kept for the process
  static uint32_t *tables[64] = {nullptr};
  int dev = 0;
  QS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(QEXSTAG_ERR_ARG, "gauge I/O: device index out of range");
  if (!tables[dev]) {
    CrcTables h;
    make_crc_tables(h);
    void *p;
    if (cudaMalloc(&p, sizeof h) != cudaSuccess) {
      cudaGetLastError();
      return fail(QEXSTAG_ERR_ALLOC, "gauge I/O: table allocation failed");
    }
    QS_CUDA(cudaMemcpy(p, &h, sizeof h, cudaMemcpyHostToDevice));
    tables[dev] = (uint32_t *)p;
  }
  *out = tables[dev];
  return QEXSTAG_OK;
}

// run the unpack (to_device) or pack kernel over a device payload
static int run_io_kernel(const Geom &g, uint8_t *payload, double2 *links, int prec, bool swap, bool milc,
                         bool unpack, uint32_t sums_out[2]) {
  uint32_t *tables;
  int rc;
  if ((rc = crc_tables_dev(&tables))) return rc;
  DevBuf sums;
  if (cudaMalloc(&sums.p, 2 * sizeof(unsigned)) != cudaSuccess) {
    cudaGetLastError();
    return fail(QEXSTAG_ERR_ALLOC, "gauge I/O: allocation failed");
  }
  QS_CUDA(cudaMemsetAsync(sums.p, 0, 2 * sizeof(unsigned), stream()));
  IoArgs A;
  A.g = g;
  A.payload = payload;
  A.links = links;
  A.crc_tables = tables;
  A.sums = (unsigned *)sums.p;
  A.prec = prec;
  A.swap = swap ? 1 : 0;
  A.milc = milc ? 1 : 0;
  const size_t smem = sizeof(uint32_t) * 8 * 256 + (size_t)kIoSites * 72 * prec;
  const int grid = (g.V + kIoSites - 1) / kIoSites;
  if (unpack) {
    QS_CUDA(cudaFuncSetAttribute(gauge_unpack_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    gauge_unpack_kernel<<<grid, kIoSites, smem, stream()>>>(A);
  } else {
    QS_CUDA(cudaFuncSetAttribute(gauge_pack_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    gauge_pack_kernel<<<grid, kIoSites, smem, stream()>>>(A);
  }
  note_launch();
  QS_LAUNCH_CHECK();
  QS_CUDA(cudaMemcpyAsync(sums_out, sums.p, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, stream()));
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

// move n bytes between a file position and device memory in pinned chunks
static int file_to_dev(FILE *f, uint64_t off, uint8_t *dev, uint64_t n) {
  const size_t chunk = 64u << 20;
  void *pin = nullptr;
  if (cudaHostAlloc(&pin, chunk, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return fail(QEXSTAG_ERR_ALLOC, "gauge I/O: pinned allocation failed");
  }
  int rc = QEXSTAG_OK;
  if (fseeko(f, (off_t)off, SEEK_SET) != 0) rc = fail(QEXSTAG_ERR_IO, "gauge read: seek failed");
  for (uint64_t done = 0; !rc && done < n;) {
    const size_t m = (size_t)std::min<uint64_t>(chunk, n - done);
    if (std::fread(pin, 1, m, f) != m) {
      rc = fail(QEXSTAG_ERR_IO, "gauge read: file shorter than its records say");
      break;
    }
    cudaError_t e = cudaMemcpyAsync(dev + done, pin, m, cudaMemcpyHostToDevice, stream());
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream());
    if (e != cudaSuccess) rc = cuda_fail(e, "gauge read: copy to device");
    done += m;
  }
  cudaFreeHost(pin);
  return rc;
}

static int dev_to_file(FILE *f, const uint8_t *dev, uint64_t n) {
  const size_t chunk = 64u << 20;
  void *pin = nullptr;
  if (cudaHostAlloc(&pin, chunk, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return fail(QEXSTAG_ERR_ALLOC, "gauge I/O: pinned allocation failed");
  }
  int rc = QEXSTAG_OK;
  for (uint64_t done = 0; !rc && done < n;) {
    const size_t m = (size_t)std::min<uint64_t>(chunk, n - done);
    cudaError_t e = cudaMemcpyAsync(pin, dev + done, m, cudaMemcpyDeviceToHost, stream());
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream());
    if (e != cudaSuccess) {
      rc = cuda_fail(e, "gauge write: copy from device");
      break;
    }
    if (std::fwrite(pin, 1, m, f) != m) rc = fail(QEXSTAG_ERR_IO, "gauge write: write failed");
    done += m;
  }
  cudaFreeHost(pin);
  return rc;
}

// links given by the caller (host AoS or device) <-> device [4][9][V]
static int links_in(const Geom &g, const double *links, int mem, DevBuf &own, double2 **dev) {
  const size_t per = sizeof(double2) * 9 * (size_t)g.V;
  if (mem == QEXSTAG_MEM_DEVICE) {
    *dev = (double2 *)links;
    return QEXSTAG_OK;
  }
  if (cudaMalloc(&own.p, 5 * per) != cudaSuccess) {
    cudaGetLastError();
    return fail(QEXSTAG_ERR_ALLOC, "gauge I/O: allocation failed");
  }
  double2 *soa = (double2 *)own.p;
  if (links) {
    double2 *aos = soa + 4 * 9 * (size_t)g.V;
    for (int d = 0; d < 4; d++) {
      QS_CUDA(cudaMemcpyAsync(aos, links + (size_t)d * 18 * g.V, per, cudaMemcpyHostToDevice, stream()));
      int rc = aos_to_soa((const double *)aos, soa + (size_t)d * 9 * g.V, g.V, g.V, 9);
      if (rc) return rc;
    }
  }
  *dev = soa;
  return QEXSTAG_OK;
}

static int links_out(const Geom &g, const double2 *soa, double *links) {
  const size_t per = sizeof(double2) * 9 * (size_t)g.V;
  double2 *aos = (double2 *)soa + 4 * 9 * (size_t)g.V;
  for (int d = 0; d < 4; d++) {
    int rc = soa_to_aos(soa + (size_t)d * 9 * g.V, (double *)aos, g.V, g.V, 9);
    if (rc) return rc;
    QS_CUDA(cudaMemcpyAsync(links + (size_t)d * 18 * g.V, aos, per, cudaMemcpyDeviceToHost, stream()));
  }
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

// header of a MILC file in its own byte order
struct MilcHeaderRaw {
  int32_t magic;
  int32_t dims[4];
  char stamp[64];
  int32_t order;
  uint32_t sum29, sum31;
};
static_assert(sizeof(MilcHeaderRaw) == 96, "MILC header is 96 bytes");

static uint32_t bswap32(uint32_t v) {
  return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24);
}

struct FileInfo {
  int format = 0;  // QEXSTAG_GAUGE_*
  int dims[4] = {0, 0, 0, 0};
  int prec = 0;
  bool swap = false;  // file byte order is not the device's
  bool has_sums = false;
  uint32_t suma = 0, sumb = 0;
  uint64_t data_off = 0, data_len = 0;
  std::string date, file_md, record_md;
};

static int probe_file(FILE *f, FileInfo &fi) {
  uint8_t head[96];
  if (std::fread(head, 1, 96, f) != 96) return fail(QEXSTAG_ERR_IO, "gauge read: file too short");
  const bool le = host_little_endian();
  if (be32(head) == kLimeMagic) {
    std::vector<LimeRecord> recs;
    if (fseeko(f, 0, SEEK_SET) != 0 || !lime_scan(f, recs))
      return fail(QEXSTAG_ERR_IO, "gauge read: malformed LIME records");
    const LimeRecord *bin = find_rec(recs, "scidac-binary-data");
    if (!bin) bin = find_rec(recs, "ildg-binary-data");
    if (!bin) return fail(QEXSTAG_ERR_IO, "gauge read: no binary-data record");
    fi.data_off = bin->offset;
    fi.data_len = bin->length;
    fi.swap = le;  // SciDAC and ILDG data are big-endian
    const LimeRecord *r;
    if ((r = find_rec(recs, "scidac-private-file-xml"))) {
      fi.format = QEXSTAG_GAUGE_SCIDAC;
      const std::string x = read_text(f, *r);
      if (std::sscanf(xml_tag(x, "dims").c_str(), "%d %d %d %d", &fi.dims[0], &fi.dims[1], &fi.dims[2],
                      &fi.dims[3]) != 4)
        return fail(QEXSTAG_ERR_IO, "gauge read: no lattice dimensions in scidac-private-file-xml");
    }
    if ((r = find_rec(recs, "ildg-format"))) {
      const std::string x = read_text(f, *r);
      if (fi.format == 0) {
        const char *t[4] = {"lx", "ly", "lz", "lt"};
        for (int d = 0; d < 4; d++) fi.dims[d] = std::atoi(xml_tag(x, t[d]).c_str());
      }
      fi.format = QEXSTAG_GAUGE_ILDG;  // ILDG files carry SciDAC records too
      const int p = std::atoi(xml_tag(x, "precision").c_str());
      if (p == 32 || p == 64) fi.prec = p / 8;
    }
    if ((r = find_rec(recs, "scidac-private-record-xml"))) {
      const std::string x = read_text(f, *r);
      const std::string p = xml_tag(x, "precision");
      if (p == "F") fi.prec = 4;
      if (p == "D") fi.prec = 8;
      fi.date = xml_tag(x, "date");
      const std::string dc = xml_tag(x, "datacount"), ts = xml_tag(x, "typesize");
      if (!dc.empty() && std::atoi(dc.c_str()) != 4)
        return fail(QEXSTAG_ERR_IO, "gauge read: record does not hold 4 colour matrices per site");
      if (!ts.empty() && fi.prec && std::atoi(ts.c_str()) != 18 * fi.prec)
        return fail(QEXSTAG_ERR_IO, "gauge read: record type size is not a 3x3 complex matrix");
    }
    if ((r = find_rec(recs, "scidac-file-xml"))) fi.file_md = read_text(f, *r);
    if ((r = find_rec(recs, "scidac-record-xml"))) fi.record_md = read_text(f, *r);
    if ((r = find_rec(recs, "scidac-checksum"))) {
      const std::string x = read_text(f, *r);
      const std::string a = xml_tag(x, "suma"), b = xml_tag(x, "sumb");
      if (!a.empty() && !b.empty()) {
        fi.suma = (uint32_t)std::strtoul(a.c_str(), nullptr, 16);
        fi.sumb = (uint32_t)std::strtoul(b.c_str(), nullptr, 16);
        fi.has_sums = true;
      }
    }
    if (fi.format == 0) return fail(QEXSTAG_ERR_IO, "gauge read: neither SciDAC nor ILDG metadata found");
    if (fi.prec == 0) return fail(QEXSTAG_ERR_IO, "gauge read: precision not stated");
    return QEXSTAG_OK;
  }
  MilcHeaderRaw h;
  std::memcpy(&h, head, 96);
  bool swap;
  if (h.magic == kMilcMagic)
    swap = false;
  else if ((int32_t)bswap32((uint32_t)h.magic) == kMilcMagic)
    swap = true;
  else
    return fail(QEXSTAG_ERR_IO, "gauge read: not a LIME (SciDAC/ILDG) or MILC file");
  fi.format = QEXSTAG_GAUGE_MILC;
  fi.swap = swap;
  fi.prec = 4;
  for (int d = 0; d < 4; d++) fi.dims[d] = swap ? (int)bswap32((uint32_t)h.dims[d]) : h.dims[d];
  const int32_t order = swap ? (int32_t)bswap32((uint32_t)h.order) : h.order;
  if (order != 0) return fail(QEXSTAG_ERR_IO, "gauge read: MILC files with a site list are not supported");
  fi.suma = swap ? bswap32(h.sum29) : h.sum29;
  fi.sumb = swap ? bswap32(h.sum31) : h.sum31;
  fi.has_sums = true;
  char stamp[65];
  std::memcpy(stamp, h.stamp, 64);
  stamp[64] = 0;
  fi.date = stamp;
  fi.data_off = 96;
  long long v = 1;
  for (int d = 0; d < 4; d++) v *= fi.dims[d];
  fi.data_len = (uint64_t)v * 72 * 4;
  return QEXSTAG_OK;
}

static void put_info(const FileInfo &fi, qexstag_gauge_info *info, bool checked, uint32_t a, uint32_t b) {
  if (!info) return;
  std::memset(info, 0, sizeof(*info));
  info->format = fi.format;
  for (int d = 0; d < 4; d++) info->dims[d] = fi.dims[d];
  info->precision = fi.prec;
  info->has_checksum = fi.has_sums ? 1 : 0;
  info->file_checksum[0] = fi.suma;
  info->file_checksum[1] = fi.sumb;
  info->data_checksum[0] = checked ? a : 0;
  info->data_checksum[1] = checked ? b : 0;
  fill_text(info->date, sizeof info->date, fi.date);
  fill_text(info->file_metadata, sizeof info->file_metadata, fi.file_md);
  fill_text(info->record_metadata, sizeof info->record_metadata, fi.record_md);
}

static void lime_header(uint8_t *h, const char *type, uint64_t len, bool mb, bool me) {
  std::memset(h, 0, 144);
  put_be32(h, kLimeMagic);
  h[4] = 0;
  h[5] = 1;  // version 1
  h[6] = (uint8_t)((mb ? 0x80 : 0) | (me ? 0x40 : 0));
  put_be64(h + 8, len);
  std::strncpy((char *)h + 16, type, 127);
}

static int lime_write(FILE *f, const char *type, const void *data, uint64_t len, bool mb, bool me) {
  uint8_t h[144];
  lime_header(h, type, len, mb, me);
  if (std::fwrite(h, 1, 144, f) != 144) return fail(QEXSTAG_ERR_IO, "gauge write: write failed");
  if (data && len && std::fwrite(data, 1, len, f) != len) return fail(QEXSTAG_ERR_IO, "gauge write: write failed");
  static const uint8_t zeros[8] = {0};
  const size_t pad = (size_t)((8 - len % 8) % 8);
  if (pad && std::fwrite(zeros, 1, pad, f) != pad) return fail(QEXSTAG_ERR_IO, "gauge write: write failed");
  return QEXSTAG_OK;
}

static std::string now_text() {
  char b[64];
  const time_t t = std::time(nullptr);
  struct tm tmv;
  gmtime_r(&t, &tmv);
  std::strftime(b, sizeof b, "%a %b %d %H:%M:%S %Y UTC", &tmv);
  return b;
}

}  // namespace qs

using namespace qs;

extern "C" {

int qexstag_gauge_file_info(const char *path, qexstag_gauge_info *info) {
  if (!path || !info) return fail(QEXSTAG_ERR_ARG, "gauge_file_info: null argument");
  FileCloser fc{std::fopen(path, "rb")};
  if (!fc.f) return fail(QEXSTAG_ERR_IO, std::string("gauge_file_info: cannot open ") + path);
  FileInfo fi;
  int rc = probe_file(fc.f, fi);
  if (rc) return rc;
  put_info(fi, info, false, 0, 0);
  return QEXSTAG_OK;
}

int qexstag_gauge_read(qexstag_layout *l, const char *path, double *links, int mem, qexstag_gauge_info *info) {
  if (!l || !path || !links) return fail(QEXSTAG_ERR_ARG, "gauge_read: null argument");
  if (mem != QEXSTAG_MEM_HOST && mem != QEXSTAG_MEM_DEVICE) return fail(QEXSTAG_ERR_ARG, "gauge_read: bad memory kind");
  int rc = runtime_ready();
  if (rc) return rc;
  const Geom &g = l->g;
  FileCloser fc{std::fopen(path, "rb")};
  if (!fc.f) return fail(QEXSTAG_ERR_IO, std::string("gauge_read: cannot open ") + path);
  FileInfo fi;
  if ((rc = probe_file(fc.f, fi))) return rc;
  for (int d = 0; d < 4; d++)
    if (fi.dims[d] != g.L[d]) return fail(QEXSTAG_ERR_IO, "gauge_read: file lattice differs from the layout's");
  const uint64_t want = (uint64_t)g.V * 72 * fi.prec;
  if (fi.data_len != want) return fail(QEXSTAG_ERR_IO, "gauge_read: binary record has the wrong length");
  DevBuf payload, own;
  if (cudaMalloc(&payload.p, want) != cudaSuccess) {
    cudaGetLastError();
    return fail(QEXSTAG_ERR_ALLOC, "gauge_read: allocation failed");
  }
  double2 *dev;
  if ((rc = links_in(g, mem == QEXSTAG_MEM_DEVICE ? links : nullptr, mem, own, &dev))) return rc;
  if ((rc = file_to_dev(fc.f, fi.data_off, (uint8_t *)payload.p, want))) return rc;
  uint32_t sums[2];
  const bool milc = fi.format == QEXSTAG_GAUGE_MILC;
  if ((rc = run_io_kernel(g, (uint8_t *)payload.p, dev, fi.prec, fi.swap, milc, true, sums))) return rc;
  put_info(fi, info, true, sums[0], sums[1]);
  if (mem == QEXSTAG_MEM_HOST && (rc = links_out(g, dev, links))) return rc;
  if (fi.has_sums && (sums[0] != fi.suma || sums[1] != fi.sumb)) {
    char b[160];
    std::snprintf(b, sizeof b, "gauge_read: checksum mismatch (file %08x %08x, data %08x %08x)", fi.suma, fi.sumb,
                  sums[0], sums[1]);
    return fail(QEXSTAG_ERR_IO, b);
  }
  return QEXSTAG_OK;
}

int qexstag_gauge_write(qexstag_layout *l, const char *path, const double *links, int mem, int format,
                        int precision, const char *file_md, const char *record_md) {
  if (!l || !path || !links) return fail(QEXSTAG_ERR_ARG, "gauge_write: null argument");
  if (mem != QEXSTAG_MEM_HOST && mem != QEXSTAG_MEM_DEVICE) return fail(QEXSTAG_ERR_ARG, "gauge_write: bad memory kind");
  if (format != QEXSTAG_GAUGE_SCIDAC && format != QEXSTAG_GAUGE_ILDG && format != QEXSTAG_GAUGE_MILC)
    return fail(QEXSTAG_ERR_ARG, "gauge_write: unknown format");
  if (precision != 4 && precision != 8) return fail(QEXSTAG_ERR_ARG, "gauge_write: precision must be 4 or 8 bytes");
  if (format == QEXSTAG_GAUGE_MILC && precision != 4)
    return fail(QEXSTAG_ERR_ARG, "gauge_write: MILC files hold single precision");
  int rc = runtime_ready();
  if (rc) return rc;
  const Geom &g = l->g;
  const uint64_t nbytes = (uint64_t)g.V * 72 * precision;
  DevBuf payload, own;
  if (cudaMalloc(&payload.p, nbytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(QEXSTAG_ERR_ALLOC, "gauge_write: allocation failed");
  }
  double2 *dev;
  if ((rc = links_in(g, links, mem, own, &dev))) return rc;
  const bool milc = format == QEXSTAG_GAUGE_MILC;
  // MILC files are written in this machine's byte order, LIME data big-endian
  const bool swap = milc ? false : host_little_endian();
  uint32_t sums[2];
  if ((rc = run_io_kernel(g, (uint8_t *)payload.p, dev, precision, swap, milc, false, sums))) return rc;
  FileCloser fc{std::fopen(path, "wb")};
  if (!fc.f) return fail(QEXSTAG_ERR_IO, std::string("gauge_write: cannot create ") + path);
  const std::string date = now_text();
  if (milc) {
    MilcHeaderRaw h;
    std::memset(&h, 0, sizeof h);
    h.magic = kMilcMagic;
    for (int d = 0; d < 4; d++) h.dims[d] = g.L[d];
    std::strncpy(h.stamp, date.c_str(), 63);
    h.order = 0;
    h.sum29 = sums[0];
    h.sum31 = sums[1];
    if (std::fwrite(&h, 1, sizeof h, fc.f) != sizeof h) return fail(QEXSTAG_ERR_IO, "gauge_write: write failed");
    if ((rc = dev_to_file(fc.f, (const uint8_t *)payload.p, nbytes))) return rc;
  } else {
    char x[1024];
    std::snprintf(x, sizeof x,
                  "<?xml version=\"1.0\" encoding=\"UTF-8\"?><scidacFile><version>1.1</version>"
                  "<spacetime>4</spacetime><dims>%d %d %d %d </dims><volfmt>0</volfmt></scidacFile>",
                  g.L[0], g.L[1], g.L[2], g.L[3]);
    const std::string fmd = file_md ? file_md : "";
    const std::string rmd = record_md ? record_md : "";
    if ((rc = lime_write(fc.f, "scidac-private-file-xml", x, std::strlen(x), true, false)) ||
        (rc = lime_write(fc.f, "scidac-file-xml", fmd.data(), fmd.size(), false, true)))
      return rc;
    std::snprintf(x, sizeof x,
                  "<?xml version=\"1.0\" encoding=\"UTF-8\"?><scidacRecord><version>1.1</version>"
                  "<date>%s</date><recordtype>0</recordtype><datatype>QDP_%c3_ColorMatrix</datatype>"
                  "<precision>%c</precision><colors>3</colors><spins>4</spins><typesize>%d</typesize>"
                  "<datacount>4</datacount></scidacRecord>",
                  date.c_str(), precision == 8 ? 'D' : 'F', precision == 8 ? 'D' : 'F', 18 * precision);
    if ((rc = lime_write(fc.f, "scidac-private-record-xml", x, std::strlen(x), true, false)) ||
        (rc = lime_write(fc.f, "scidac-record-xml", rmd.data(), rmd.size(), false, false)))
      return rc;
    if (format == QEXSTAG_GAUGE_ILDG) {
      std::snprintf(x, sizeof x,
                    "<?xml version=\"1.0\" encoding=\"UTF-8\"?><ildgFormat><version>1.0</version>"
                    "<field>su3gauge</field><precision>%d</precision><lx>%d</lx><ly>%d</ly><lz>%d</lz>"
                    "<lt>%d</lt></ildgFormat>",
                    8 * precision, g.L[0], g.L[1], g.L[2], g.L[3]);
      if ((rc = lime_write(fc.f, "ildg-format", x, std::strlen(x), false, false))) return rc;
    }
    uint8_t h[144];
    lime_header(h, format == QEXSTAG_GAUGE_ILDG ? "ildg-binary-data" : "scidac-binary-data", nbytes, false, false);
    if (std::fwrite(h, 1, 144, fc.f) != 144) return fail(QEXSTAG_ERR_IO, "gauge_write: write failed");
    if ((rc = dev_to_file(fc.f, (const uint8_t *)payload.p, nbytes))) return rc;  // nbytes is a multiple of 8
    std::snprintf(x, sizeof x,
                  "<?xml version=\"1.0\" encoding=\"UTF-8\"?><scidacChecksum><version>1.0</version>"
                  "<suma>%x</suma><sumb>%x</sumb></scidacChecksum>",
                  sums[0], sums[1]);
    if ((rc = lime_write(fc.f, "scidac-checksum", x, std::strlen(x), false, true))) return rc;
  }
  if (std::fflush(fc.f) != 0) return fail(QEXSTAG_ERR_IO, "gauge_write: write failed");
  return QEXSTAG_OK;
}

}  // extern "C"
