// VTK output of a grid field, formatted on the GPU and written to disk in
// overlapped chunks.
//
// The reference writes its legacy ASCII file value by value through an
// ostream (WriteVtkStructuredPoints, src/vtk_writer.cpp:28-82: each value cast
// to float and printed fixed with 6 decimals, one space after each value, one
// newline after each x row) and its XML image data by base64-encoding a
// float32 copy of the field and of the derived fields (WriteVtkXmlImageData,
// src/vtk_writer.cpp:176-268; ComputeDerivedFields, :365-440; field list of
// BuildDerivedFieldVectors, src/main.cpp:255-288). Both are single-threaded
// host loops. Here the text is made on the device:
//  - legacy: every value's text length is computed (1024 values per tile),
//    the tile lengths are scanned into byte offsets, then each tile formats its
//    values into shared memory and stores its bytes at its offset;
//  - XML: one thread per 3 source bytes emits 4 base64 characters, reading the
//    field (or evaluating a derived-field stencil) on the fly.
// The host writes chunk c to the file while the device formats chunk c+1.
// Headers are formatted on the host with the same ostream settings as the
// reference, so the files are byte-identical.
//
// Fixed-point formatting: a float is m * 2^e exactly (m < 2^24). Its integer
// part fits in 128 bits, and its fraction times 10^6 is m' * 10^6 / 2^s with
// m' * 10^6 < 2^44, so the six decimals are an exact integer division with
// the remainder compared against half the divisor; exact ties round to the
// even last digit, as the C library's printf rounds under round-to-nearest.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iomanip>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "host.h"

namespace pdeb {

namespace {

constexpr int kVtThreads = 256;
constexpr int kVtPerThread = 4;
constexpr int kVtTile = kVtThreads * kVtPerThread;  // values per tile
constexpr int kVtMaxChars = 49;                      // longest value text incl. space and newline
constexpr size_t kVtChunkBytes = size_t(64) << 20;   // text per pipelined chunk (target)
constexpr long long kB64ChunkGroups = 16ll << 20;    // base64 groups (4 chars each) per chunk

// Fixed six-decimal text of f (no terminator); returns its length (<= 47).
__host__ __device__ inline int fmt_fixed6(float f, char* out) {
  uint32_t bits;
  memcpy(&bits, &f, 4);
  const bool neg = (bits >> 31) != 0;
  const uint32_t ex = (bits >> 23) & 0xffu, mant = bits & 0x7fffffu;
  int p = 0;
  if (neg) out[p++] = '-';
  if (ex == 0xffu) {
    const char* w = mant ? "nan" : "inf";
    out[p++] = w[0];
    out[p++] = w[1];
    out[p++] = w[2];
    return p;
  }
  const uint64_t m = ex ? (uint64_t(mant) | 0x800000u) : uint64_t(mant);
  const int e2 = (ex ? int(ex) : 1) - 150;
  uint64_t lo = 0;              // integer part when it fits 64 bits
  unsigned __int128 big = 0;    // integer part for e2 > 39
  bool wide = false;
  uint32_t q = 0;               // six decimals
  if (e2 >= 0) {
    if (e2 <= 39) {
      lo = m << e2;  // m < 2^24: below 2^64
    } else {
      big = (unsigned __int128)m << e2;
      wide = true;
    }
  } else {
    const int s = -e2;
    const uint64_t ip = s < 64 ? (m >> s) : 0;
    const uint64_t r = s < 64 ? m - (ip << s) : m;
    const uint64_t num = r * 1000000ull;  // < 2^44
    uint64_t qq = 0;
    if (s < 64) {
      qq = num >> s;
      const uint64_t rem = num - (qq << s);
      const uint64_t half = 1ull << (s - 1);
      if (rem > half || (rem == half && (qq & 1))) ++qq;
    }
    lo = ip;
    if (qq == 1000000ull) {
      qq = 0;
      ++lo;
    }
    q = uint32_t(qq);
  }
  char tmp[40];
  int nd = 0;
  if (wide) {
    do {
      tmp[nd++] = char('0' + int(big % 10));
      big /= 10;
    } while (big);
  } else {
    do {
      tmp[nd++] = char('0' + int(lo % 10));
      lo /= 10;
    } while (lo);
  }
  while (nd) out[p++] = tmp[--nd];
  out[p++] = '.';
  for (int d = 5; d >= 0; --d) {
    out[p + d] = char('0' + q % 10);
    q /= 10;
  }
  return p + 6;
}

// double -> float as cvtsd2ss does it: round to nearest, and a NaN keeps its
// sign and the top 22 bits of its payload with the quiet bit set.
__host__ __device__ inline float to_float_host_rule(double d) {
  if (d != d) {
    uint64_t b;
    memcpy(&b, &d, 8);
    const uint32_t f = uint32_t(b >> 63) << 31 | 0x7fc00000u | uint32_t((b >> 29) & 0x3fffffu);
    float r;
    memcpy(&r, &f, 4);
    return r;
  }
  return float(d);
}

// Text of value `idx`: the number, a space, and a newline at the end of a row.
__host__ __device__ inline int value_text(double v, long long idx, int nx, char* out) {
  int len = fmt_fixed6(to_float_host_rule(v), out);
  out[len++] = ' ';
  if (idx % nx == nx - 1) out[len++] = '\n';
  return len;
}

__device__ inline int block_exclusive_scan(int v, int* warp_tot, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    int x = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += t;
    }
    if (lane < nw) warp_tot[lane] = x;  // inclusive warp prefix
  }
  __syncthreads();
  const int before = w ? warp_tot[w - 1] : 0;
  if (total) *total = warp_tot[(blockDim.x >> 5) - 1];
  return before + incl - v;
}

// Text bytes of every tile of kVtTile values.
__global__ void __launch_bounds__(kVtThreads) k_vtk_len(const double* __restrict__ field, long long n, int nx,
                                                        int* __restrict__ tile_len) {
  __shared__ int warp_tot[kVtThreads / 32];
  const long long base = (long long)blockIdx.x * kVtTile + (long long)threadIdx.x * kVtPerThread;
  char buf[kVtMaxChars];
  int len = 0;
#pragma unroll
  for (int v = 0; v < kVtPerThread; ++v) {
    const long long idx = base + v;
    if (idx < n) len += value_text(field[idx], idx, nx, buf);
  }
  int total = 0;
  block_exclusive_scan(len, warp_tot, &total);
  if (threadIdx.x == 0) tile_len[blockIdx.x] = total;
}

// Exclusive byte offsets of the tiles (one block; tiles split into equal runs).
__global__ void __launch_bounds__(1024) k_vtk_scan(const int* __restrict__ tile_len, long long ntiles,
                                                   long long* __restrict__ tile_off) {
  __shared__ long long part[1024];
  const long long per = (ntiles + blockDim.x - 1) / blockDim.x;
  const long long t0 = (long long)threadIdx.x * per;
  const long long t1 = t0 + per < ntiles ? t0 + per : ntiles;
  long long s = 0;
  for (long long t = t0; t < t1; ++t) s += tile_len[t];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    const long long add = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += add;
    __syncthreads();
  }
  long long off = part[threadIdx.x] - s;
  for (long long t = t0; t < t1; ++t) {
    tile_off[t] = off;
    off += tile_len[t];
  }
  if (threadIdx.x == blockDim.x - 1) tile_off[ntiles] = part[threadIdx.x];
}

// Formats tiles [tile0, tile0 + gridDim.x) into out (offsets relative to out_base).
__global__ void __launch_bounds__(kVtThreads) k_vtk_text(const double* __restrict__ field, long long n, int nx,
                                                         long long tile0, const long long* __restrict__ tile_off,
                                                         long long out_base, char* __restrict__ out) {
  extern __shared__ char text[];
  __shared__ int warp_tot[kVtThreads / 32];
  const long long tile = tile0 + blockIdx.x;
  const long long base = tile * kVtTile + (long long)threadIdx.x * kVtPerThread;
  char buf[kVtPerThread * kVtMaxChars];
  int len = 0;
#pragma unroll
  for (int v = 0; v < kVtPerThread; ++v) {
    const long long idx = base + v;
    if (idx < n) len += value_text(field[idx], idx, nx, buf + len);
  }
  int total = 0;
  const int at = block_exclusive_scan(len, warp_tot, &total);
  for (int c = 0; c < len; ++c) text[at + c] = buf[c];
  __syncthreads();
  char* dst = out + (tile_off[tile] - out_base);
  for (int c = threadIdx.x; c < total; c += blockDim.x) dst[c] = text[c];
}

// Source of the float32 array behind a base64 DataArray: the field itself or
// one derived field of ComputeDerivedFields, evaluated at a node.
struct B64Src {
  const double* u;
  int kind;  // 0 solution, 1 grad x, 2 grad y, 3 grad z, 4 laplacian, 5 flux x, 6 flux y, 7 flux z, 8 energy
  int nx, ny, nz;
  bool three_d;
  double inv_dx, inv_dy, inv_dz, inv_dx2, inv_dy2, inv_dz2;
  double a, b, c;
  long long n;
};

// Arithmetic with the host's NaN results. The reference runs on x86-64 SSE2,
// where an operation with a NaN operand returns the first NaN operand
// (quieted) and an invalid operation (inf - inf, 0 * inf) returns the default
// NaN with the sign bit set; the GPU returns one canonical NaN instead. The
// derived fields are computed with these wrappers so that NaN bits, and so the
// encoded bytes, are the host's too; the first operand is the left operand
// of the source expression.
__device__ inline double x86_nan(double a, double b) {
  const long long quiet = 0x0008000000000000ll;
  if (isnan(a)) return __longlong_as_double(__double_as_longlong(a) | quiet);
  if (isnan(b)) return __longlong_as_double(__double_as_longlong(b) | quiet);
  return __longlong_as_double((long long)0xfff8000000000000ull);
}
__device__ inline double xadd(double a, double b) {
  const double r = __dadd_rn(a, b);
  return isnan(r) ? x86_nan(a, b) : r;
}
__device__ inline double xsub(double a, double b) {
  const double r = __dsub_rn(a, b);
  return isnan(r) ? x86_nan(a, b) : r;
}
__device__ inline double xmul(double a, double b) {
  const double r = __dmul_rn(a, b);
  return isnan(r) ? x86_nan(a, b) : r;
}

// ComputeDerivedFields (src/vtk_writer.cpp:365-440) at one node, in the
// reference's operation order with no contraction; boundary nodes are 0.
__device__ inline double derived_at(const B64Src& S, long long idx) {
  if (S.kind == 0) return S.u[idx];
  const int i = int(idx % S.nx), j = int((idx / S.nx) % S.ny), k = int(idx / ((long long)S.nx * S.ny));
  if (i < 1 || i > S.nx - 2 || j < 1 || j > S.ny - 2) return 0.0;
  if (S.three_d && (k < 1 || k > S.nz - 2)) return 0.0;
  const double u = S.u[idx];
  const long long sx = 1, sy = S.nx, sz = (long long)S.nx * S.ny;
  switch (S.kind) {
    case 1:
    case 5: {
      const double g = xmul(xmul(xsub(S.u[idx + sx], S.u[idx - sx]), 0.5), S.inv_dx);
      return S.kind == 1 ? g : xmul(-S.a, g);
    }
    case 2:
    case 6: {
      const double g = xmul(xmul(xsub(S.u[idx + sy], S.u[idx - sy]), 0.5), S.inv_dy);
      return S.kind == 2 ? g : xmul(-S.b, g);
    }
    case 3:
    case 7: {
      const double g = xmul(xmul(xsub(S.u[idx + sz], S.u[idx - sz]), 0.5), S.inv_dz);
      return S.kind == 3 ? g : xmul(-S.c, g);
    }
    case 4: {
      const double two_u = xmul(2.0, u);
      const double lx = xmul(xadd(xsub(S.u[idx + sx], two_u), S.u[idx - sx]), S.inv_dx2);
      const double ly = xmul(xadd(xsub(S.u[idx + sy], two_u), S.u[idx - sy]), S.inv_dy2);
      double l = xadd(lx, ly);
      if (S.three_d) {
        const double lz = xmul(xadd(xsub(S.u[idx + sz], two_u), S.u[idx - sz]), S.inv_dz2);
        l = xadd(l, lz);
      }
      return l;
    }
    default:
      return xmul(u, u);
  }
}

// Byte p of the encoded buffer [uint64 8][uint64 4n][float32 x n].
__device__ inline uint32_t b64_byte(const B64Src& S, long long p) {
  if (p < 8) return p == 0 ? 8u : 0u;
  if (p < 16) {
    const unsigned long long sz = (unsigned long long)S.n * 4ull;
    return uint32_t((sz >> (8 * (p - 8))) & 0xffu);
  }
  const long long idx = (p - 16) >> 2;
  const float f = to_float_host_rule(derived_at(S, idx));
  uint32_t bits;
  memcpy(&bits, &f, 4);
  return (bits >> (8 * ((p - 16) & 3))) & 0xffu;
}

__global__ void __launch_bounds__(256) k_b64(B64Src S, long long g0, long long ng, char* __restrict__ out) {
  const char* tbl = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
  const long long len = 16 + 4 * S.n;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ng; t += (long long)gridDim.x * blockDim.x) {
    const long long g = g0 + t;
    const long long p = 3 * g;
    // consecutive bytes of one float come from one source value: read it once
    uint32_t b0, b1 = 0, b2 = 0;
    if (p >= 16 && ((p - 16) & 3) <= 1 && p + 2 < len) {
      const long long idx = (p - 16) >> 2;
      const float f = to_float_host_rule(derived_at(S, idx));
      uint32_t bits;
      memcpy(&bits, &f, 4);
      const int sh = 8 * int((p - 16) & 3);
      b0 = (bits >> sh) & 0xffu;
      b1 = (bits >> (sh + 8)) & 0xffu;
      b2 = (bits >> (sh + 16)) & 0xffu;
    } else {
      b0 = b64_byte(S, p);
      if (p + 1 < len) b1 = b64_byte(S, p + 1);
      if (p + 2 < len) b2 = b64_byte(S, p + 2);
    }
    const uint32_t w = (b0 << 16) | (b1 << 8) | b2;
    char4 c;
    c.x = tbl[(w >> 18) & 63];
    c.y = tbl[(w >> 12) & 63];
    c.z = p + 1 < len ? tbl[(w >> 6) & 63] : '=';
    c.w = p + 2 < len ? tbl[w & 63] : '=';
    reinterpret_cast<char4*>(out)[t] = c;
  }
}

void copy_msg(char* dst, size_t len, const std::string& m) {
  if (!dst || len == 0) return;
  std::strncpy(dst, m.c_str(), len - 1);
  dst[len - 1] = '\0';
}

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

struct Geometry {
  int nx, ny, nz;
  long long n;
  double dx, dy, dz;
};

Geometry geometry(const pdeb200_problem* g) {
  Geometry G;
  G.nx = g->nx;
  G.ny = g->ny;
  G.nz = g->nz > 1 ? g->nz : 1;
  G.n = (long long)G.nx * G.ny * G.nz;
  G.dx = (g->xmax - g->xmin) / double(G.nx - 1 > 1 ? G.nx - 1 : 1);
  G.dy = (g->ymax - g->ymin) / double(G.ny - 1 > 1 ? G.ny - 1 : 1);
  G.dz = (g->zmax - g->zmin) / double(G.nz - 1 > 1 ? G.nz - 1 : 1);
  return G;
}

// A device copy of the field when it lives on the host.
const double* device_field(Context* ctx, const double* field, int mem_space, long long n, Buf* keep) {
  if (mem_space == PDEB200_MEM_DEVICE) return field;
  *keep = Buf(sizeof(double) * n, ctx->stream);
  PDEB_CUDA(cudaMemcpyAsync(keep->as<double>(), field, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  return keep->as<double>();
}

bool write_all(FILE* f, const char* p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f) == n; }

// Two device and two pinned host buffers of one chunk each: chunk c is
// formatted (launch(c, dst)) while chunk c-1 is written to the file. Kept in
// the device context between writes (allocating pinned memory costs more
// than formatting a chunk).
struct Staging {
  char* dev[2] = {nullptr, nullptr};
  char* host[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  size_t cap = 0;
  explicit Staging(size_t bytes) : cap(bytes) {
    for (int q = 0; q < 2; ++q) {
      cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&dev[q]), bytes);
      if (e == cudaErrorMemoryAllocation) throw StatusFailure{PDEB200_ERR_OOM, "device memory exhausted"};
      PDEB_CUDA(e);
      PDEB_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&host[q]), bytes, cudaHostAllocDefault));
      PDEB_CUDA(cudaEventCreateWithFlags(&done[q], cudaEventDisableTiming));
    }
  }
  ~Staging() {
    for (int q = 0; q < 2; ++q) {
      if (dev[q]) cudaFree(dev[q]);
      if (host[q]) cudaFreeHost(host[q]);
      if (done[q]) cudaEventDestroy(done[q]);
    }
  }
  Staging(const Staging&) = delete;
  Staging& operator=(const Staging&) = delete;

  // The context's staging, grown to at least `bytes` per buffer.
  static Staging* of(Context* ctx, size_t bytes) {
    bytes = bytes < 4096 ? 4096 : bytes;
    Staging* s = static_cast<Staging*>(ctx->io_staging.get());
    if (!s || s->cap < bytes) {
      ctx->io_staging.reset();
      auto fresh = std::make_shared<Staging>(bytes);
      ctx->io_staging = std::static_pointer_cast<void>(fresh);
      s = fresh.get();
    }
    return s;
  }

  template <class Launch>
  bool run(Context* ctx, FILE* f, int chunks, const std::vector<size_t>& bytes, Launch&& launch,
           pdeb200_write_progress progress, void* user) {
    bool ok = true;
    for (int c = 0; c <= chunks; ++c) {
      if (c < chunks) {
        char* d = dev[c & 1];
        launch(c, d);
        PDEB_CUDA(cudaMemcpyAsync(host[c & 1], d, bytes[c], cudaMemcpyDeviceToHost, ctx->stream));
        PDEB_CUDA(cudaEventRecord(done[c & 1], ctx->stream));
      }
      if (c > 0) {
        const int q = (c - 1) & 1;
        PDEB_CUDA(cudaEventSynchronize(done[q]));
        if (ok) ok = write_all(f, host[q], bytes[c - 1]);
        if (progress) progress(double(c) / double(chunks), user);
      }
    }
    return ok;
  }
};

}  // namespace
}  // namespace pdeb

extern "C" {

pdeb200_status pdeb200_write_vtk(const char* path, const pdeb200_problem* grid, const double* field,
                                 int32_t mem_space, int32_t device, pdeb200_write_progress progress, void* user,
                                 char* message, size_t message_len) {
  using namespace pdeb;
  copy_msg(message, message_len, "");
  if (!path || !grid || !field) return PDEB200_ERR_INVALID;
  if (grid->nx < 1 || grid->ny < 1) {
    copy_msg(message, message_len, "invalid grid dimensions");
    return PDEB200_ERR_INVALID;
  }
  const Geometry G = geometry(grid);
  File out;
  out.f = std::fopen(path, "wb");
  if (!out.f) {
    copy_msg(message, message_len, "failed to open output file");
    return PDEB200_ERR_INVALID;
  }
  std::ostringstream h;
  h << "# vtk DataFile Version 3.0\n"
    << "pde_solution\n"
    << "ASCII\n"
    << "DATASET STRUCTURED_POINTS\n"
    << "DIMENSIONS " << G.nx << " " << G.ny << " " << G.nz << "\n"
    << "ORIGIN " << grid->xmin << " " << grid->ymin << " " << grid->zmin << "\n"
    << "SPACING " << G.dx << " " << G.dy << " " << G.dz << "\n"
    << "POINT_DATA " << (G.nx * G.ny * G.nz) << "\n"
    << "SCALARS solution float 1\n"
    << "LOOKUP_TABLE default\n";
  const std::string head = h.str();
  if (!write_all(out.f, head.data(), head.size())) {
    copy_msg(message, message_len, "failed to write output file");
    return PDEB200_ERR_INVALID;
  }
  if (progress) progress(0.0, user);
  try {
    Context* ctx = get_context(device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    Buf keep;
    const double* u = device_field(ctx, field, mem_space, G.n, &keep);
    const long long ntiles = (G.n + kVtTile - 1) / kVtTile;
    Buf tile_len(sizeof(int) * ntiles, ctx->stream);
    Buf tile_off(sizeof(long long) * (ntiles + 1), ctx->stream);
    k_vtk_len<<<(unsigned)ntiles, kVtThreads, 0, ctx->stream>>>(u, G.n, G.nx, tile_len.as<int>());
    PDEB_CUDA(cudaGetLastError());
    k_vtk_scan<<<1, 1024, 0, ctx->stream>>>(tile_len.as<int>(), ntiles, tile_off.as<long long>());
    PDEB_CUDA(cudaGetLastError());
    ctx->count(2);
    std::vector<long long> off(ntiles + 1);
    PDEB_CUDA(cudaMemcpyAsync(off.data(), tile_off.as<long long>(), sizeof(long long) * (ntiles + 1),
                              cudaMemcpyDeviceToHost, ctx->stream));
    PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
    // chunks of whole tiles, about kVtChunkBytes of text each
    std::vector<long long> first{0};
    std::vector<size_t> bytes;
    size_t max_bytes = 0;
    for (long long t = 0; t < ntiles;) {
      long long e = t + 1;
      while (e < ntiles && size_t(off[e + 1] - off[t]) <= kVtChunkBytes) ++e;
      bytes.push_back(size_t(off[e] - off[t]));
      max_bytes = std::max(max_bytes, bytes.back());
      first.push_back(e);
      t = e;
    }
    static bool attr_set[64] = {};
    if (device >= 0 && device < 64 && !attr_set[device]) {
      PDEB_CUDA(cudaFuncSetAttribute(k_vtk_text, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kVtTile * kVtMaxChars));
      attr_set[device] = true;
    }
    const int chunks = int(bytes.size());
    Staging& stage = *Staging::of(ctx, max_bytes);
    const bool ok = stage.run(
        ctx, out.f, chunks, bytes,
        [&](int c, char* dst) {
          const long long t0 = first[c], t1 = first[c + 1];
          k_vtk_text<<<(unsigned)(t1 - t0), kVtThreads, kVtTile * kVtMaxChars, ctx->stream>>>(
              u, G.n, G.nx, t0, tile_off.as<long long>(), off[t0], dst);
          PDEB_CUDA(cudaGetLastError());
          ctx->count();
        },
        progress, user);
    if (!ok) {
      copy_msg(message, message_len, "failed to write output file");
      return PDEB200_ERR_INVALID;
    }
  } catch (const StatusFailure& s) {
    copy_msg(message, message_len, s.what);
    return s.status;
  } catch (const CudaFailure& c) {
    copy_msg(message, message_len, c.what);
    cudaGetLastError();
    return PDEB200_ERR_CUDA;
  }
  return PDEB200_OK;
}

pdeb200_status pdeb200_write_vti(const char* path, const pdeb200_problem* grid, const double* field,
                                 int32_t derived, int32_t mem_space, int32_t device, pdeb200_write_progress progress,
                                 void* user, char* message, size_t message_len) {
  using namespace pdeb;
  copy_msg(message, message_len, "");
  if (!path || !grid || !field) return PDEB200_ERR_INVALID;
  if (grid->nx < 1 || grid->ny < 1) {
    copy_msg(message, message_len, "invalid grid dimensions");
    return PDEB200_ERR_INVALID;
  }
  const Geometry G = geometry(grid);
  File out;
  out.f = std::fopen(path, "wb");
  if (!out.f) {
    copy_msg(message, message_len, "failed to open output file");
    return PDEB200_ERR_INVALID;
  }
  std::ostringstream h;
  h << std::setprecision(9) << std::scientific;
  h << "<?xml version=\"1.0\"?>\n"
    << "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
    << "  <ImageData WholeExtent=\"0 " << (G.nx - 1) << " 0 " << (G.ny - 1) << " 0 " << (G.nz - 1)
    << "\" Origin=\"" << grid->xmin << " " << grid->ymin << " " << grid->zmin << "\" Spacing=\"" << G.dx << " "
    << G.dy << " " << G.dz << "\">\n"
    << "    <Piece Extent=\"0 " << (G.nx - 1) << " 0 " << (G.ny - 1) << " 0 " << (G.nz - 1) << "\">\n"
    << "      <PointData>\n";
  // DataArrays: the solution, then BuildDerivedFieldVectors' list
  const bool three_d = grid->nz > 1;
  std::vector<std::pair<int, const char*>> arrays{{0, "solution"}};
  if (derived) {
    arrays.push_back({1, "gradient_x"});
    arrays.push_back({2, "gradient_y"});
    if (three_d) arrays.push_back({3, "gradient_z"});
    arrays.push_back({4, "laplacian"});
    arrays.push_back({5, "flux_x"});
    arrays.push_back({6, "flux_y"});
    if (three_d) arrays.push_back({7, "flux_z"});
    arrays.push_back({8, "energy_norm"});
  }
  try {
    Context* ctx = get_context(device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    Buf keep;
    const double* u = device_field(ctx, field, mem_space, G.n, &keep);
    B64Src S{};
    S.u = u;
    S.nx = G.nx;
    S.ny = G.ny;
    S.nz = G.nz;
    S.three_d = three_d;
    S.inv_dx = G.dx > 0.0 ? 1.0 / G.dx : 0.0;
    S.inv_dy = G.dy > 0.0 ? 1.0 / G.dy : 0.0;
    S.inv_dz = G.dz > 0.0 ? 1.0 / G.dz : 0.0;
    S.inv_dx2 = G.dx > 0.0 ? 1.0 / (G.dx * G.dx) : 0.0;
    S.inv_dy2 = G.dy > 0.0 ? 1.0 / (G.dy * G.dy) : 0.0;
    S.inv_dz2 = G.dz > 0.0 ? 1.0 / (G.dz * G.dz) : 0.0;
    S.a = grid->a;
    S.b = grid->b;
    S.c = grid->az;
    S.n = G.n;
    const long long groups = (16 + 4 * G.n + 2) / 3;
    const int per_array = int((groups + kB64ChunkGroups - 1) / kB64ChunkGroups);
    std::string head = h.str();
    Staging& stage = *Staging::of(ctx, size_t(4 * std::min(groups, kB64ChunkGroups)));
    for (size_t a = 0; a < arrays.size(); ++a) {
      std::ostringstream open;
      open << "        <DataArray type=\"Float32\" Name=\"" << arrays[a].second
           << "\" NumberOfComponents=\"1\" format=\"binary\">\n";
      head += open.str();
      if (!write_all(out.f, head.data(), head.size())) {
        copy_msg(message, message_len, "failed to write output file");
        return PDEB200_ERR_INVALID;
      }
      S.kind = arrays[a].first;
      std::vector<size_t> bytes(per_array);
      for (int c = 0; c < per_array; ++c) {
        const long long g0 = c * kB64ChunkGroups;
        const long long g1 = std::min(groups, g0 + kB64ChunkGroups);
        bytes[c] = size_t(4 * (g1 - g0));
      }
      const bool ok = stage.run(
          ctx, out.f, per_array, bytes,
          [&](int c, char* dst) {
            const long long g0 = c * kB64ChunkGroups;
            const long long ng = std::min(groups, g0 + kB64ChunkGroups) - g0;
            const int blocks = (int)std::min<long long>((ng + 255) / 256, (long long)ctx->num_sms * 16);
            k_b64<<<blocks, 256, 0, ctx->stream>>>(S, g0, ng, dst);
            PDEB_CUDA(cudaGetLastError());
            ctx->count();
          },
          nullptr, nullptr);
      if (!ok) {
        copy_msg(message, message_len, "failed to write output file");
        return PDEB200_ERR_INVALID;
      }
      head = "\n        </DataArray>\n";
      if (progress) progress(double(a + 1) / double(arrays.size()), user);
    }
    head += "      </PointData>\n      <CellData/>\n    </Piece>\n  </ImageData>\n</VTKFile>\n";
    if (!write_all(out.f, head.data(), head.size())) {
      copy_msg(message, message_len, "failed to write output file");
      return PDEB200_ERR_INVALID;
    }
  } catch (const StatusFailure& s) {
    copy_msg(message, message_len, s.what);
    return s.status;
  } catch (const CudaFailure& c) {
    copy_msg(message, message_len, c.what);
    cudaGetLastError();
    return PDEB200_ERR_CUDA;
  }
  return PDEB200_OK;
}

pdeb200_status pdeb200_vtk_values_host(const double* field, int64_t n, int32_t nx, char* out, size_t capacity,
                                       size_t* length) {
  using namespace pdeb;
  if (!field || !length || nx < 1 || n < 0) return PDEB200_ERR_INVALID;
  size_t len = 0;
  char buf[kVtMaxChars];
  for (long long q = 0; q < n; ++q) {
    const int l = value_text(field[q], q, nx, buf);
    if (out && len + l <= capacity) std::memcpy(out + len, buf, l);
    len += l;
  }
  *length = len;
  return (out && len > capacity) ? PDEB200_ERR_INVALID : PDEB200_OK;
}

}  // extern "C"
