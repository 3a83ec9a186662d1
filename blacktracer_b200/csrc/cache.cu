// cache.cu -- the reference's cache files and its perfect spatial hash of
// the grid, plus the perspective camera view.
//
// * Grid files (Grid::serialize, BT/Grid.h:36-39) hold MAXLEVEL, N, M and a
//   perfect spatial hash (PSH) of the grid's vertices (PSHOffsetTable,
//   BT/PSHOffsetTable.h:44-48, built by saveAsGpuHash, BT/Grid.h:642-654).
//   The reference renders from the PSH: makeGrid (BT/MakeImageKernel.cu
//   :369-384) looks every lattice vertex up (hashLookup, BT/kernel.cuh
//   :713-733).  Here the PSH exists only at the file boundary: a built grid is
//   hashed on the host when saved, and a loaded file is expanded on the device
//   (k_psh_map) into the same float2 map grid bt_grid_map_export produces.
// * Star files (StarProcessor::serialize, BT/StarProcessor.h:21-23) hold the
//   star tree in the layout bt_stars_create takes.
//
// Both are cereal (v1.2.2) binary archives: raw little-endian values in
// serialisation order, each std::vector as a uint64 element count followed by
// its elements, no headers.  They are read and written here without cereal.
//
// The PSH is built by the method of Lefebvre and Hoppe ("Perfect Spatial
// Hashing", 2006) that the reference follows: keys fall into buckets of an
// offset table (key mod offset width); buckets are placed largest first, each
// at an offset under which all its keys land on free slots of the hash table
// (key mod hash width, plus the offset).  The reference searches offsets from
// a time-seeded rand(); this search is deterministic: it walks the table from
// a start slot derived from the bucket's index.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "bt_internal.h"

using bt::clear_error;
using bt::set_error;

#if !defined(__BYTE_ORDER__) || __BYTE_ORDER__ != __ORDER_LITTLE_ENDIAN__
#error "cache files are little-endian; this build assumes a little-endian host"
#endif

namespace {

// ------------------------------------------------------------ archives
struct FileWriter {
  FILE* f = nullptr;
  bool ok = true;
  explicit FileWriter(const char* path) : f(std::fopen(path, "wb")) { ok = f != nullptr; }
  ~FileWriter() {
    if (f) std::fclose(f);
  }
  bool close() {
    if (f && std::fclose(f) != 0) ok = false;
    f = nullptr;
    return ok;
  }
  void raw(const void* p, size_t n) {
    if (ok && n && std::fwrite(p, 1, n, f) != n) ok = false;
  }
  void i32(int32_t v) { raw(&v, 4); }
  template <class T>
  void vec(const T* p, uint64_t n) {
    raw(&n, 8);
    raw(p, (size_t)n * sizeof(T));
  }
};

struct Reader {
  std::vector<unsigned char> buf;
  size_t off = 0;
  bool ok = true;
  bool raw(void* dst, size_t k) {
    if (!ok || k > buf.size() - off) return ok = false;
    if (dst && k) std::memcpy(dst, buf.data() + off, k);
    off += k;
    return true;
  }
  bool i32(int32_t& v) { return raw(&v, 4); }
  // A vector's element count, checked against the bytes left in the file.
  bool count(uint64_t& c, size_t elem) {
    if (!raw(&c, 8)) return false;
    if (c > (buf.size() - off) / elem) return ok = false;
    return true;
  }
  bool at_end() const { return ok && off == buf.size(); }
};

int read_file(const char* path, Reader& r) {
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("cannot open %s", path);
    return BT_ERR_ARG;
  }
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz < 0) {
    std::fclose(f);
    set_error("cannot size %s", path);
    return BT_ERR_ARG;
  }
  r.buf.resize((size_t)sz);
  const size_t got = sz ? std::fread(r.buf.data(), 1, (size_t)sz, f) : 0;
  std::fclose(f);
  if (got != (size_t)sz) {
    set_error("short read of %s", path);
    return BT_ERR_ARG;
  }
  return BT_OK;
}

// ------------------------------------------------------------ PSH
int gcd(int a, int b) { return b == 0 ? a : gcd(b, a % b); }

// Table widths of the reference (BT/PSHOffsetTable.h:59-79).
int hash_width_for(size_t n) {
  const float d = (float)std::pow((float)n * 1.1f, 0.5f);
  return (int)(d + 1.1f);
}
int offset_width_for(size_t n, int hw) {
  const float d = (float)std::pow((float)n / 4.f, 0.5f);
  int w = (int)(d + 1.1f);
  while (gcd(w, hw) > 1) w++;
  return w;
}

uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

enum PlaceResult { kPlaced, kRetry, kDuplicate };

// One attempt at offset width ow.  Fills ht/tag/ot on success.
PlaceResult psh_attempt(const int32_t* keys, const float* vals, size_t n, int hw, int ow,
                        std::vector<float>& ht, std::vector<int32_t>& tag,
                        std::vector<int32_t>& ot) {
  const size_t hw2 = (size_t)hw * hw, ow2 = (size_t)ow * ow;
  std::vector<uint32_t> start(ow2 + 1, 0), order(n);
  for (size_t k = 0; k < n; k++)
    start[(size_t)(keys[2 * k] % ow) * ow + (size_t)(keys[2 * k + 1] % ow) + 1]++;
  for (size_t b = 0; b < ow2; b++) start[b + 1] += start[b];
  {
    std::vector<uint32_t> fill(start.begin(), start.end() - 1);
    for (size_t k = 0; k < n; k++)
      order[fill[(size_t)(keys[2 * k] % ow) * ow + (size_t)(keys[2 * k + 1] % ow)]++] =
          (uint32_t)k;
  }
  // buckets largest first, ties by bucket index
  std::vector<uint32_t> buckets;
  buckets.reserve(ow2);
  for (size_t b = 0; b < ow2; b++)
    if (start[b + 1] > start[b]) buckets.push_back((uint32_t)b);
  std::stable_sort(buckets.begin(), buckets.end(), [&](uint32_t x, uint32_t y) {
    return start[x + 1] - start[x] > start[y + 1] - start[y];
  });
  ht.assign(2 * hw2, 0.f);
  tag.assign(2 * hw2, 0);
  ot.assign(2 * ow2, 0);
  std::vector<unsigned char> filled(hw2, 0);
  std::vector<int> hx, hy;
  size_t free_scan = 0;  // singletons take free slots in table order
  for (uint32_t b : buckets) {
    const uint32_t b0 = start[b], sz = start[b + 1] - b0;
    hx.resize(sz);
    hy.resize(sz);
    for (uint32_t e = 0; e < sz; e++) {
      const uint32_t k = order[b0 + e];
      hx[e] = keys[2 * k] % hw;
      hy[e] = keys[2 * k + 1] % hw;
      for (uint32_t f = 0; f < e; f++) {
        if (hx[f] == hx[e] && hy[f] == hy[e]) {
          const uint32_t k2 = order[b0 + f];
          if (keys[2 * k] == keys[2 * k2] && keys[2 * k + 1] == keys[2 * k2 + 1])
            return kDuplicate;
          return kRetry;  // congruent keys: no offset separates them
        }
      }
    }
    size_t placed = hw2;
    if (sz == 1) {
      while (free_scan < hw2 && filled[free_scan]) free_scan++;
      placed = free_scan;
    } else {
      const size_t s0 = mix64(b) % hw2;
      for (size_t t = 0; t < hw2 && placed == hw2; t++) {
        size_t p = s0 + t;
        if (p >= hw2) p -= hw2;
        if (filled[p]) continue;
        const int dx = ((int)(p / hw) - hx[0] + hw) % hw;
        const int dy = ((int)(p % hw) - hy[0] + hw) % hw;
        bool ok = true;
        for (uint32_t e = 1; e < sz && ok; e++) {
          const size_t s = (size_t)((hx[e] + dx) % hw) * hw + (size_t)((hy[e] + dy) % hw);
          ok = !filled[s];
        }
        if (ok) placed = p;
      }
    }
    if (placed >= hw2) return kRetry;
    const int dx = ((int)(placed / hw) - hx[0] + hw) % hw;
    const int dy = ((int)(placed % hw) - hy[0] + hw) % hw;
    ot[2 * b] = dx;
    ot[2 * b + 1] = dy;
    for (uint32_t e = 0; e < sz; e++) {
      const uint32_t k = order[b0 + e];
      const size_t s = (size_t)((hx[e] + dx) % hw) * hw + (size_t)((hy[e] + dy) % hw);
      filled[s] = 1;
      ht[2 * s] = vals[2 * k];
      ht[2 * s + 1] = vals[2 * k + 1];
      tag[2 * s] = keys[2 * k];
      tag[2 * s + 1] = keys[2 * k + 1];
    }
  }
  return kPlaced;
}

// The first kPshSameWidth attempts keep the reference's hash width (only the
// offset table grows, as the reference's retry does); later ones also lower
// the load factor, which regular key sets (a uniform lattice) need.
constexpr int kPshAttempts = 24;
constexpr int kPshSameWidth = 3;

int psh_build(const int32_t* keys, const float* vals, size_t n, int& hw, int& ow,
              std::vector<float>& ht, std::vector<int32_t>& tag, std::vector<int32_t>& ot) {
  if (n == 0) {
    hw = 1;
    ow = 1;
    ht.assign(2, 0.f);
    tag.assign(2, 0);
    ot.assign(2, 0);
    return BT_OK;
  }
  for (size_t k = 0; k < 2 * n; k++)
    if (keys[k] < 0) {
      set_error("invalid argument: negative key at %zu", k / 2);
      return BT_ERR_ARG;
    }
  hw = hash_width_for(n);
  ow = offset_width_for(n, hw);
  for (int att = 0; att < kPshAttempts; att++) {
    const PlaceResult r = psh_attempt(keys, vals, n, hw, ow, ht, tag, ot);
    if (r == kPlaced) return BT_OK;
    if (r == kDuplicate) {
      set_error("invalid argument: duplicate keys");
      return BT_ERR_ARG;
    }
    if (att + 1 < kPshSameWidth) {
      ow += 5;  // more, smaller buckets
    } else {
      hw += std::max(1, hw / 16);
      ow += std::max(5, ow / 8);
    }
    while (gcd(ow, hw) > 1) ow++;
  }
  set_error("no perfect hash found for %zu keys after %d attempts", n, kPshAttempts);
  return BT_ERR_NUMERIC;
}

int copy_out(const std::vector<float>& ht, const std::vector<int32_t>& tag,
             const std::vector<int32_t>& ot, int hw, int ow, bt_psh* out) {
  out->hash_width = hw;
  out->offset_width = ow;
  if (out->cap_hash < ht.size() || out->cap_offset < ot.size()) {
    set_error("PSH capacity too small: need %zu hash and %zu offset elements", ht.size(),
              ot.size());
    return BT_ERR_ARG;
  }
  if (out->hash_table) std::memcpy(out->hash_table, ht.data(), ht.size() * 4);
  if (out->pos_tag) std::memcpy(out->pos_tag, tag.data(), tag.size() * 4);
  if (out->offset_table) std::memcpy(out->offset_table, ot.data(), ot.size() * 4);
  return BT_OK;
}

// Non-negative remainder of a 64-bit value.
__device__ __forceinline__ int wrap_mod(long long v, int w) {
  long long r = v % w;
  return (int)(r < 0 ? r + w : r);
}

// makeGrid with hashLookup (BT/MakeImageKernel.cu:369-384, BT/kernel.cuh
// :713-733) for one grid: thread (j, i) looks up key (i, j).
__global__ void k_psh_map(const float2* __restrict__ ht, const int2* __restrict__ tag,
                          const int2* __restrict__ ot, int hw, int ow, int N, int M,
                          float2* __restrict__ grid, int rows, int sym) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (j >= M || i >= N) return;
  const int2 o = ot[(size_t)(i % ow) * ow + (j % ow)];
  const int hx = wrap_mod((long long)(i % hw) + o.x, hw);
  const int hy = wrap_mod((long long)(j % hw) + o.y, hw);
  const size_t s = (size_t)hx * hw + hy;
  const int2 t = tag[s];
  float2 v = (t.x == i && t.y == j) ? ht[s] : make_float2(-2.f, -2.f);
  grid[(size_t)i * M + j] = v;
  if (sym) {
    if (v.x != -1 && v.x != -2) v.x = bt::kPiF - v.x;
    grid[(size_t)(rows - i - 1) * M + j] = v;
  }
}

// Reads a .grid file; tables into vectors.
int grid_file_parse(const char* path, int32_t& maxlevel, int32_t& N, int32_t& M,
                    std::vector<float>& ht, std::vector<int32_t>& ot,
                    std::vector<int32_t>& tag, int32_t& hw, int32_t& ow) {
  Reader r;
  if (int rc = read_file(path, r)) return rc;
  uint64_t c = 0;
  r.i32(maxlevel);
  r.i32(N);
  r.i32(M);
  if (r.count(c, 4)) {
    ht.resize(c);
    r.raw(ht.data(), c * 4);
  }
  if (r.count(c, 4)) {
    ot.resize(c);
    r.raw(ot.data(), c * 4);
  }
  if (r.count(c, 4)) {
    tag.resize(c);
    r.raw(tag.data(), c * 4);
  }
  r.i32(hw);
  r.i32(ow);
  if (!r.at_end()) {
    set_error("%s is not a grid file (truncated or trailing bytes)", path);
    return BT_ERR_ARG;
  }
  int32_t n0 = 0, m0 = 0, n1 = 0, m1 = 0;
  const bool lvl_ok = maxlevel >= 1 && maxlevel <= 14 &&
                      bt_grid_dims(maxlevel, 0, &n0, &m0) == BT_OK &&
                      bt_grid_dims(maxlevel, 1, &n1, &m1) == BT_OK;
  if (!lvl_ok || !((N == n0 && M == m0) || (N == n1 && M == m1))) {
    set_error("%s: lattice %d x %d does not match max level %d", path, N, M, maxlevel);
    return BT_ERR_ARG;
  }
  if (hw <= 0 || ow <= 0 || hw > (1 << 15) || ow > (1 << 15) ||
      ht.size() != 2 * (size_t)hw * hw || tag.size() != ht.size() ||
      ot.size() != 2 * (size_t)ow * ow) {
    set_error("%s: hash table sizes do not match their widths (%d, %d)", path, hw, ow);
    return BT_ERR_ARG;
  }
  return BT_OK;
}

int map_rows_of(int N, int M) { return (float)M / (float)N > 3 ? 2 * N - 1 : N; }

int launch_psh_map(const float* ht, const int32_t* tag, const int32_t* ot, int hw, int ow,
                   int N, int M, float* grid, int rows, cudaStream_t s) {
  const int sym = (float)M / (float)N > 3 ? 1 : 0;  // dev_sym, BT/MakeImageKernel.cu:1259
  dim3 blk(256), grd((M + 255) / 256, N);
  k_psh_map<<<grd, blk, 0, s>>>((const float2*)ht, (const int2*)tag, (const int2*)ot, hw,
                                ow, N, M, (float2*)grid, rows, sym);
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}

// Perspective view: each output corner's theta depends only on its row and
// its phi only on its column, so both are evaluated on the host with the
// reference's expressions (BT/Viewer.h:115-131) and broadcast on the device.
__global__ void k_view_outer(const float* __restrict__ th, const float* __restrict__ ph,
                             int W1, int H1, float2* __restrict__ view) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (j < W1 && i < H1) view[(size_t)i * W1 + j] = make_float2(th[i], ph[j]);
}

}  // namespace

// ------------------------------------------------------------ C ABI
int bt_psh_build(const int32_t* keys, const float* values, size_t n, bt_psh* out) {
  clear_error();
  BT_ARG_CHECK(out && (n == 0 || (keys && values)), "NULL pointer");
  BT_ARG_CHECK(n < (size_t)1 << 28, "too many keys");
  int hw = 0, ow = 0;
  std::vector<float> ht;
  std::vector<int32_t> tag, ot;
  if (int rc = psh_build(keys, values, n, hw, ow, ht, tag, ot)) return rc;
  return copy_out(ht, tag, ot, hw, ow, out);
}

int bt_grid_map_from_psh(const float* hash_table, const int32_t* pos_tag,
                         const int32_t* offset_table, int hash_width, int offset_width,
                         int N, int M, float* grid, int rows, void* stream) {
  clear_error();
  BT_ARG_CHECK(hash_table && pos_tag && offset_table && grid, "NULL pointer");
  BT_ARG_CHECK(hash_width > 0 && offset_width > 0 && N > 0 && M > 0, "invalid widths");
  BT_ARG_CHECK(rows == map_rows_of(N, M), "rows must be 2N-1 when M/N > 3, else N");
  BT_ARG_CHECK((((uintptr_t)hash_table | (uintptr_t)pos_tag | (uintptr_t)offset_table |
                 (uintptr_t)grid) & 7) == 0,
               "tables and grid must be 8-byte aligned");
  return launch_psh_map(hash_table, pos_tag, offset_table, hash_width, offset_width, N, M,
                        grid, rows, (cudaStream_t)stream);
}

int bt_grid_file_write(const char* path, int maxlevel, int N, int M, const bt_psh* t) {
  clear_error();
  BT_ARG_CHECK(path && t && t->hash_table && t->pos_tag && t->offset_table, "NULL pointer");
  BT_ARG_CHECK(t->hash_width > 0 && t->offset_width > 0, "invalid widths");
  const uint64_t nh = 2 * (uint64_t)t->hash_width * t->hash_width;
  const uint64_t no = 2 * (uint64_t)t->offset_width * t->offset_width;
  BT_ARG_CHECK(t->cap_hash >= nh && t->cap_offset >= no, "tables smaller than their widths");
  FileWriter w(path);
  // Grid::serialize then PSHOffsetTable::serialize (BT/Grid.h:38,
  // BT/PSHOffsetTable.h:47)
  w.i32(maxlevel);
  w.i32(N);
  w.i32(M);
  w.vec(t->hash_table, nh);
  w.vec(t->offset_table, no);
  w.vec(t->pos_tag, nh);
  w.i32(t->hash_width);
  w.i32(t->offset_width);
  if (!w.close()) {
    set_error("cannot write %s", path);
    return BT_ERR_ARG;
  }
  return BT_OK;
}

int bt_grid_file_read(const char* path, int32_t* maxlevel, int32_t* N, int32_t* M,
                      bt_psh* t) {
  clear_error();
  BT_ARG_CHECK(path && maxlevel && N && M && t, "NULL pointer");
  std::vector<float> ht;
  std::vector<int32_t> ot, tag;
  int32_t hw = 0, ow = 0;
  if (int rc = grid_file_parse(path, *maxlevel, *N, *M, ht, ot, tag, hw, ow)) return rc;
  return copy_out(ht, tag, ot, hw, ow, t);
}

int bt_grid_save(bt_grid* g, const char* path, void* stream) {
  clear_error();
  BT_ARG_CHECK(g && path, "NULL pointer");
  bt_grid_info info;
  if (int rc = bt_grid_query(g, &info, stream)) return rc;
  bt_grid_export_t ex;
  std::memset(&ex, 0, sizeof(ex));
  int rc = bt_grid_export(g, &ex, stream);  // counts only (capacities 0)
  if (rc != BT_OK && rc != BT_ERR_ARG) return rc;
  const size_t nv = ex.n_vertices;
  std::vector<uint32_t> vi(nv + 1), vj(nv + 1);
  std::vector<double> th(nv + 1), ph(nv + 1);
  std::memset(&ex, 0, sizeof(ex));
  ex.vi = vi.data();
  ex.vj = vj.data();
  ex.theta = th.data();
  ex.phi = ph.data();
  ex.cap_vertices = nv + 1;
  ex.cap_blocks = (size_t)-1;  // blocks are not exported (NULL arrays)
  if ((rc = bt_grid_export(g, &ex, stream))) return rc;
  BT_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  // CamToCel -> (elements, data) of saveAsGpuHash (BT/Grid.h:645-650)
  std::vector<int32_t> keys(2 * nv);
  std::vector<float> vals(2 * nv);
  for (size_t k = 0; k < nv; k++) {
    keys[2 * k] = (int32_t)vi[k];
    keys[2 * k + 1] = (int32_t)vj[k];
    vals[2 * k] = (float)th[k];
    vals[2 * k + 1] = (float)ph[k];
  }
  int hw = 0, ow = 0;
  std::vector<float> ht;
  std::vector<int32_t> tag, ot;
  if ((rc = psh_build(keys.data(), vals.data(), nv, hw, ow, ht, tag, ot))) return rc;
  bt_psh t;
  t.hash_table = ht.data();
  t.pos_tag = tag.data();
  t.offset_table = ot.data();
  t.cap_hash = ht.size();
  t.cap_offset = ot.size();
  t.hash_width = hw;
  t.offset_width = ow;
  return bt_grid_file_write(path, info.maxlevel, info.N, info.M, &t);
}

int bt_grid_file_map_shape(const char* path, int32_t* maxlevel, int32_t* rows,
                           int32_t* cols, int32_t* sym) {
  clear_error();
  BT_ARG_CHECK(path, "NULL pointer");
  std::vector<float> ht;
  std::vector<int32_t> ot, tag;
  int32_t ml = 0, N = 0, M = 0, hw = 0, ow = 0;
  if (int rc = grid_file_parse(path, ml, N, M, ht, ot, tag, hw, ow)) return rc;
  if (maxlevel) *maxlevel = ml;
  if (rows) *rows = map_rows_of(N, M);
  if (cols) *cols = M;
  if (sym) *sym = map_rows_of(N, M) != N ? 1 : 0;
  return BT_OK;
}

int bt_grid_file_load_map(const char* path, float* grid, int rows, int cols, void* stream) {
  clear_error();
  BT_ARG_CHECK(path && grid, "NULL pointer");
  std::vector<float> ht;
  std::vector<int32_t> ot, tag;
  int32_t ml = 0, N = 0, M = 0, hw = 0, ow = 0;
  if (int rc = grid_file_parse(path, ml, N, M, ht, ot, tag, hw, ow)) return rc;
  if (rows != map_rows_of(N, M) || cols != M) {
    set_error("invalid argument: map grid %d x %d, the file needs %d x %d", rows, cols,
              map_rows_of(N, M), M);
    return BT_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const size_t bh = ht.size() * 4, bo = ot.size() * 4;
  char* dev = nullptr;
  BT_CUDA_TRY(cudaMallocAsync((void**)&dev, 2 * bh + bo, s));
  int rc = BT_OK;
  cudaError_t e = cudaMemcpyAsync(dev, ht.data(), bh, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dev + bh, tag.data(), bh, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dev + 2 * bh, ot.data(), bo, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) {
    set_error("table upload failed: %s", cudaGetErrorString(e));
    rc = BT_ERR_CUDA;
  } else {
    rc = launch_psh_map((const float*)dev, (const int32_t*)(dev + bh),
                        (const int32_t*)(dev + 2 * bh), hw, ow, N, M, grid, rows, s);
  }
  // pageable sources: the copies above have consumed them before returning
  cudaError_t ef = cudaFreeAsync(dev, s);
  if (rc == BT_OK && ef != cudaSuccess) {
    set_error("cudaFreeAsync: %s", cudaGetErrorString(ef));
    rc = BT_ERR_CUDA;
  }
  return rc;
}

int bt_stars_file_write(const char* path, const float* star_pos, const float* star_mag,
                        int n, const int* tree, int treeLevel) {
  clear_error();
  BT_ARG_CHECK(path && tree && (n == 0 || (star_pos && star_mag)), "NULL pointer");
  BT_ARG_CHECK(n >= 0 && treeLevel >= 1 && treeLevel <= 24, "invalid star set");
  const int tsize = bt_stars_tree_size(treeLevel);
  FileWriter w(path);
  // StarProcessor::serialize (BT/StarProcessor.h:22)
  w.vec(tree, (uint64_t)tsize);
  w.vec(star_pos, 2 * (uint64_t)n);
  w.vec(star_mag, 2 * (uint64_t)n);
  w.i32(n);
  w.i32(tsize);
  w.i32(treeLevel);
  if (!w.close()) {
    set_error("cannot write %s", path);
    return BT_ERR_ARG;
  }
  return BT_OK;
}

namespace {
int stars_parse(const char* path, std::vector<int32_t>& tree, std::vector<float>& pos,
                std::vector<float>& mag, int32_t& n, int32_t& tsize, int32_t& level) {
  Reader r;
  if (int rc = read_file(path, r)) return rc;
  uint64_t c = 0;
  if (r.count(c, 4)) {
    tree.resize(c);
    r.raw(tree.data(), c * 4);
  }
  if (r.count(c, 4)) {
    pos.resize(c);
    r.raw(pos.data(), c * 4);
  }
  if (r.count(c, 4)) {
    mag.resize(c);
    r.raw(mag.data(), c * 4);
  }
  r.i32(n);
  r.i32(tsize);
  r.i32(level);
  if (!r.at_end() || n < 0 || level < 1 || level > 24 ||
      tsize != bt_stars_tree_size(level) || tree.size() != (size_t)tsize ||
      pos.size() != 2 * (size_t)n || mag.size() != 2 * (size_t)n) {
    set_error("%s is not a star file (sizes do not match)", path);
    return BT_ERR_ARG;
  }
  return BT_OK;
}
}  // namespace

int bt_stars_file_info(const char* path, int* n, int* treeLevel) {
  clear_error();
  BT_ARG_CHECK(path && n && treeLevel, "NULL pointer");
  std::vector<int32_t> tree;
  std::vector<float> pos, mag;
  int32_t nn = 0, ts = 0, lv = 0;
  if (int rc = stars_parse(path, tree, pos, mag, nn, ts, lv)) return rc;
  *n = nn;
  *treeLevel = lv;
  return BT_OK;
}

int bt_stars_file_read(const char* path, float* star_pos, float* star_mag, int n_cap,
                       int* tree, int tree_cap) {
  clear_error();
  BT_ARG_CHECK(path && star_pos && star_mag && tree, "NULL pointer");
  std::vector<int32_t> tr;
  std::vector<float> pos, mag;
  int32_t nn = 0, ts = 0, lv = 0;
  if (int rc = stars_parse(path, tr, pos, mag, nn, ts, lv)) return rc;
  if (n_cap < nn || tree_cap < ts) {
    set_error("invalid argument: capacities %d, %d; the file holds %d stars, %d tree nodes",
              n_cap, tree_cap, nn, ts);
    return BT_ERR_ARG;
  }
  std::memcpy(star_pos, pos.data(), pos.size() * 4);
  std::memcpy(star_mag, mag.data(), mag.size() * 4);
  std::memcpy(tree, tr.data(), tr.size() * 4);
  return BT_OK;
}

int bt_view_camera(float* view, int width, int height, double view_angle,
                   double offset_ver, double offset_hor, void* stream) {
  clear_error();
  BT_ARG_CHECK(view, "NULL pointer");
  BT_ARG_CHECK(width >= 1 && height >= 1 && width <= (1 << 16) && height <= (1 << 16),
               "invalid size");
  BT_ARG_CHECK(view_angle > 0 && view_angle < bt::kPi, "view angle outside (0, pi)");
  // Viewer::Viewer (BT/Viewer.h:28-30) and makeCameraView (:109-133)
  const double angle_up = 1. * height * view_angle / (1. * width);
  BT_ARG_CHECK(std::fabs(offset_ver) <= (bt::kPi - angle_up) / 2.,
               "offset_ver above (pi - vertical view angle) / 2");
  const double PI = bt::kPi, PI1_2 = bt::kPi / 2.;
  const float yleft = std::tan(view_angle / 2.f);
  const float step = (2.f * yleft) / width;
  const float zup = yleft * height / width;
  std::vector<float> th(height + 1), ph(width + 1);
  for (int i = 0; i < height + 1; i++) {
    const float zval = zup - i * step;
    const float halfH = i * 1.f / (height / 2.f);
    th[i] = halfH == 1.f ? PI1_2 - offset_ver
                         : std::atan(1. / zval) + (halfH > 1.f) * PI - offset_ver;
  }
  // column j of the output holds the reference's index W - j
  for (int j = 0; j < width + 1; j++) {
    const float yval = yleft - j * step;
    const float halfV = j * 1.f / (width / 2.f);
    ph[width - j] = halfV == 1.f ? PI - offset_hor
                                 : std::atan(1. / yval) + (halfV > 1.f) * PI + PI1_2 - offset_hor;
  }
  cudaStream_t s = (cudaStream_t)stream;
  float* dev = nullptr;
  const size_t bytes = (size_t)(height + 1 + width + 1) * sizeof(float);
  BT_CUDA_TRY(cudaMallocAsync((void**)&dev, bytes, s));
  std::vector<float> both(th);
  both.insert(both.end(), ph.begin(), ph.end());
  int rc = BT_OK;
  cudaError_t e = cudaMemcpyAsync(dev, both.data(), bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    dim3 grd((width + 1 + 127) / 128, height + 1);
    k_view_outer<<<grd, 128, 0, s>>>(dev, dev + height + 1, width + 1, height + 1,
                                     (float2*)view);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_error("camera view: %s", cudaGetErrorString(e));
    rc = BT_ERR_CUDA;
  }
  cudaError_t ef = cudaFreeAsync(dev, s);
  if (rc == BT_OK && ef != cudaSuccess) {
    set_error("cudaFreeAsync: %s", cudaGetErrorString(ef));
    rc = BT_ERR_CUDA;
  }
  return rc;
}
