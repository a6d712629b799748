// Host-side graph construction and I/O: seeded RMAT and grid generators,
// COO -> CSR (io/read_csr.hpp:260-300), CSR transpose (formats/csr.hpp:179-209),
// the "SYGRCSR" binary layout (io/read_csr.hpp:22-25, 316-411) and Matrix
// Market coordinate files (io/read_csr.hpp:88-192, io/matrix_market.hpp:45-151).
// OpenMP; no device code.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "sygraph_b200.h"

namespace sgb {
sg_status fail(sg_status s, const std::string& msg);
void clear_error();

// Structure check of a host CSR before anything indexes with it: offsets
// start at 0, never decrease and end at m, and every column is a vertex id.
// A graph that fails it would make every kernel read and write outside its
// per-vertex arrays.  O(n + m), OpenMP.
sg_status check_csr(const uint32_t* ro, const uint32_t* col, uint32_t n, uint64_t m) {
  if (ro[0] != 0 || ro[n] != m) return fail(SG_ERR_INVALID, "row_offsets must start at 0 and end at m");
  int64_t bad_row = -1, bad_edge = -1;
#pragma omp parallel for schedule(static) reduction(max : bad_row)
  for (int64_t v = 0; v < (int64_t)n; v++)
    if (ro[v + 1] < ro[v]) bad_row = std::max(bad_row, v);
  if (bad_row >= 0)
    return fail(SG_ERR_INVALID, "row_offsets decrease at row " + std::to_string(bad_row));
#pragma omp parallel for schedule(static) reduction(max : bad_edge)
  for (int64_t e = 0; e < (int64_t)m; e++)
    if (col[e] >= n) bad_edge = std::max(bad_edge, e);
  if (bad_edge >= 0)
    return fail(SG_ERR_INVALID, "column index out of range at edge " + std::to_string(bad_edge));
  return SG_OK;
}
}  // namespace sgb

namespace {

using sgb::fail;

// splitmix64 finaliser (Steele, Lea, Flood 2014): a counter-based generator,
// so every edge / weight draw depends only on (seed, index).
inline uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
inline uint64_t hash2(uint64_t seed, uint64_t i) { return mix64(mix64(seed) ^ i); }

// Weight of the unordered pair {u, v}: identical for (u,v) and (v,u).
inline uint32_t pair_weight_bits(uint64_t seed, uint32_t u, uint32_t v, int value_type) {
  const uint32_t a = u < v ? u : v, b = u < v ? v : u;
  const uint64_t h = hash2(seed, ((uint64_t)a << 32) | b);
  if (value_type == SG_WEIGHT_F32) {
    // ((h >> 40) + 1) * 2^-24: uniform on (0, 1], exactly representable in fp32.
    float w = (float)((h >> 40) + 1) * (1.0f / 16777216.0f);
    uint32_t bits;
    memcpy(&bits, &w, 4);
    return bits;
  }
  return (uint32_t)(h >> 58) + 1u;  // uniform on [1, 64]
}

// Parallel LSD radix sort of 64-bit keys over the low `key_bits` bits.
void radix_sort_u64(std::vector<uint64_t>& keys, int key_bits) {
  const size_t n = keys.size();
  if (n < 2) return;
  std::vector<uint64_t> tmp(n);
  const int digit = 11, buckets = 1 << digit;
  const int nt = omp_get_max_threads();
  std::vector<size_t> hist((size_t)nt * buckets);
  uint64_t* src = keys.data();
  uint64_t* dst = tmp.data();
  int passes = 0;
  for (int shift = 0; shift < key_bits; shift += digit, passes++) {
    std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nt)
    {
      const int t = omp_get_thread_num();
      const size_t lo = n * t / nt, hi = n * (t + 1) / nt;
      size_t* h = &hist[(size_t)t * buckets];
      for (size_t i = lo; i < hi; i++) h[(src[i] >> shift) & (buckets - 1)]++;
#pragma omp barrier
#pragma omp single
      {
        size_t sum = 0;
        for (int b = 0; b < buckets; b++)
          for (int tt = 0; tt < nt; tt++) {
            size_t c = hist[(size_t)tt * buckets + b];
            hist[(size_t)tt * buckets + b] = sum;
            sum += c;
          }
      }
      for (size_t i = lo; i < hi; i++) dst[h[(src[i] >> shift) & (buckets - 1)]++] = src[i];
    }
    std::swap(src, dst);
  }
  if (passes & 1) keys.swap(tmp);
}

// Sorted, de-duplicated (src << shift | dst) keys -> CSR with pair weights.
sg_status keys_to_csr(std::vector<uint64_t>& keys, int shift, uint32_t n, int value_type, uint64_t weight_seed,
                      uint32_t flags, sg_host_csr* out) {
  const size_t m = keys.size();
  if (m >= (1ull << 32)) return fail(SG_ERR_INVALID, "graph has 2^32 or more edges");
  memset(out, 0, sizeof(*out));
  out->n = n;
  out->m = m;
  out->flags = flags | (value_type != SG_WEIGHT_NONE ? SG_GRAPH_WEIGHTED : 0u);
  out->value_type = value_type;
  out->row_offsets = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)n + 1));
  out->column_indices = (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1));
  if (value_type != SG_WEIGHT_NONE) out->values = malloc(sizeof(uint32_t) * (m ? m : 1));
  if (!out->row_offsets || !out->column_indices || (value_type != SG_WEIGHT_NONE && !out->values)) {
    sg_host_csr_free(out);
    return fail(SG_ERR_NOMEM, "host allocation failed");
  }
  uint32_t* ro = out->row_offsets;
  std::fill(ro, ro + (size_t)n + 1, 0u);
  const uint64_t low = (1ull << shift) - 1;
  for (size_t i = 0; i < m; i++) ro[(keys[i] >> shift) + 1]++;
  for (uint32_t v = 0; v < n; v++) ro[v + 1] += ro[v];
  uint32_t* col = out->column_indices;
  uint32_t* val = (uint32_t*)out->values;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)m; i++) {
    const uint32_t s = (uint32_t)(keys[i] >> shift), d = (uint32_t)(keys[i] & low);
    col[i] = d;
    if (val) val[i] = pair_weight_bits(weight_seed, s, d, value_type);
  }
  return SG_OK;
}

void unique_sorted(std::vector<uint64_t>& keys) {
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
}

// Drops the ~0 entries that mark self-loops (order is not kept; the keys are
// sorted afterwards).
void drop_marked(std::vector<uint64_t>& keys) {
  size_t w = 0;
  for (size_t i = 0; i < keys.size(); i++)
    if (keys[i] != ~0ull) keys[w++] = keys[i];
  keys.resize(w);
}

int bits_for(uint64_t x) {
  int b = 1;
  while (b < 64 && (1ull << b) <= x) b++;
  return b;
}

}  // namespace

extern "C" {

void sg_host_csr_free(sg_host_csr* csr) {
  if (!csr) return;
  free(csr->row_offsets);
  free(csr->column_indices);
  free(csr->values);
  csr->row_offsets = nullptr;
  csr->column_indices = nullptr;
  csr->values = nullptr;
}

sg_status sg_rmat_generate(const sg_rmat_params* p, sg_host_csr* out) {
  sgb::clear_error();
  if (!p || !out) return fail(SG_ERR_INVALID, "NULL argument");
  if (p->scale < 1 || p->scale > 30) return fail(SG_ERR_INVALID, "scale must be in [1, 30]");
  const double d = 1.0 - p->a - p->b - p->c;
  if (p->a < 0 || p->b < 0 || p->c < 0 || d < -1e-12) return fail(SG_ERR_INVALID, "invalid RMAT probabilities");
  const uint32_t n = 1u << p->scale;
  const uint64_t pairs = (uint64_t)p->edge_factor * n;
  const uint32_t scale = p->scale;
  const double ab = p->a + p->b, abc = p->a + p->b + p->c;
  // Seeded relabelling (Fisher-Yates driven by the counter generator).
  std::vector<uint32_t> perm(n);
  for (uint32_t i = 0; i < n; i++) perm[i] = i;
  if (p->perm_seed) {
    for (uint32_t i = n - 1; i > 0; i--) {
      uint32_t j = (uint32_t)(hash2(p->perm_seed, i) % ((uint64_t)i + 1));
      std::swap(perm[i], perm[j]);
    }
  }
  std::vector<uint64_t> keys(2 * pairs);
  uint64_t* kp = keys.data();
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)pairs; i++) {
    uint64_t st = hash2(p->seed, (uint64_t)i);
    uint32_t u = 0, v = 0;
    uint64_t r = 0;
    for (uint32_t lvl = 0; lvl < scale; lvl++) {
      if ((lvl & 1) == 0) r = mix64(st + lvl);
      const double x = (double)((lvl & 1) ? (r & 0xffffffffu) : (r >> 32)) * (1.0 / 4294967296.0);
      const uint32_t bit = 1u << (scale - 1 - lvl);
      if (x < p->a) {
      } else if (x < ab) {
        v |= bit;
      } else if (x < abc) {
        u |= bit;
      } else {
        u |= bit;
        v |= bit;
      }
    }
    u = perm[u];
    v = perm[v];
    // self-loops are marked and dropped before the sort
    if (u == v) {
      kp[2 * i] = kp[2 * i + 1] = ~0ull;
    } else {
      kp[2 * i] = ((uint64_t)u << scale) | v;
      kp[2 * i + 1] = ((uint64_t)v << scale) | u;
    }
  }
  drop_marked(keys);
  radix_sort_u64(keys, 2 * (int)scale);
  unique_sorted(keys);
  return keys_to_csr(keys, (int)scale, n, p->value_type, p->weight_seed, 0u, out);
}

sg_status sg_grid_generate(uint32_t side, double long_range_frac, uint64_t seed, uint64_t weight_seed, int value_type,
                           sg_host_csr* out) {
  sgb::clear_error();
  if (!out || side < 2) return fail(SG_ERR_INVALID, "side must be >= 2");
  const uint64_t n64 = (uint64_t)side * side;
  if (n64 >= 0xffffffffull) return fail(SG_ERR_INVALID, "grid too large");
  const uint32_t n = (uint32_t)n64;
  const uint64_t grid_pairs = 2ull * side * (side - 1);
  const uint64_t lr = (uint64_t)std::llround(long_range_frac * (double)grid_pairs);
  const int sh = bits_for(n - 1);
  std::vector<uint64_t> keys(2 * (grid_pairs + lr));
  uint64_t* kp = keys.data();
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < (int64_t)side; r++) {
    for (uint32_t c = 0; c < side; c++) {
      const uint32_t v = (uint32_t)r * side + c;
      // right neighbour pairs occupy [0, side*(side-1)), down pairs the rest
      if (c + 1 < side) {
        const uint64_t idx = (uint64_t)r * (side - 1) + c;
        kp[2 * idx] = ((uint64_t)v << sh) | (v + 1);
        kp[2 * idx + 1] = ((uint64_t)(v + 1) << sh) | v;
      }
      if ((uint32_t)r + 1 < side) {
        const uint64_t idx = (uint64_t)side * (side - 1) + (uint64_t)r * side + c;
        kp[2 * idx] = ((uint64_t)v << sh) | (v + side);
        kp[2 * idx + 1] = ((uint64_t)(v + side) << sh) | v;
      }
    }
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)lr; i++) {
    const uint64_t h = hash2(seed, (uint64_t)i);
    const uint32_t u = (uint32_t)((h >> 32) % n), v = (uint32_t)((h & 0xffffffffu) % n);
    const uint64_t idx = grid_pairs + i;
    if (u == v) {
      kp[2 * idx] = kp[2 * idx + 1] = ~0ull;
    } else {
      kp[2 * idx] = ((uint64_t)u << sh) | v;
      kp[2 * idx + 1] = ((uint64_t)v << sh) | u;
    }
  }
  drop_marked(keys);
  radix_sort_u64(keys, 2 * sh);
  unique_sorted(keys);
  return keys_to_csr(keys, sh, n, value_type, weight_seed, 0u, out);
}

sg_status sg_csr_from_edges(uint32_t n, const uint32_t* src, const uint32_t* dst, const void* values, int value_type,
                            uint64_t count, int symmetrize, int dedupe, int drop_self_loops, sg_host_csr* out) {
  sgb::clear_error();
  if (!out || (count && (!src || !dst))) return fail(SG_ERR_INVALID, "NULL argument");
  struct E {
    uint64_t key;
    uint64_t order;
    uint32_t val;
  };
  std::vector<E> es;
  es.reserve(symmetrize ? 2 * count : count);
  const uint32_t* vb = (const uint32_t*)values;
  for (uint64_t i = 0; i < count; i++) {
    if (src[i] >= n || dst[i] >= n) return fail(SG_ERR_INVALID, "edge endpoint out of range");
    if (drop_self_loops && src[i] == dst[i]) continue;
    const uint32_t w = vb ? vb[i] : 1u;
    es.push_back({((uint64_t)src[i] << 32) | dst[i], 2 * i, w});
    if (symmetrize && src[i] != dst[i]) es.push_back({((uint64_t)dst[i] << 32) | src[i], 2 * i + 1, w});
  }
  std::stable_sort(es.begin(), es.end(), [](const E& a, const E& b) { return a.key < b.key; });
  if (dedupe) es.erase(std::unique(es.begin(), es.end(), [](const E& a, const E& b) { return a.key == b.key; }), es.end());
  const uint64_t m = es.size();
  memset(out, 0, sizeof(*out));
  out->n = n;
  out->m = m;
  out->value_type = value_type;
  out->flags = (symmetrize ? 0u : SG_GRAPH_DIRECTED) | (value_type != SG_WEIGHT_NONE ? SG_GRAPH_WEIGHTED : 0u);
  out->row_offsets = (uint32_t*)calloc((size_t)n + 1, sizeof(uint32_t));
  out->column_indices = (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1));
  if (value_type != SG_WEIGHT_NONE) out->values = malloc(sizeof(uint32_t) * (m ? m : 1));
  for (uint64_t i = 0; i < m; i++) {
    out->row_offsets[(es[i].key >> 32) + 1]++;
    out->column_indices[i] = (uint32_t)es[i].key;
    if (out->values) ((uint32_t*)out->values)[i] = es[i].val;
  }
  for (uint32_t v = 0; v < n; v++) out->row_offsets[v + 1] += out->row_offsets[v];
  return SG_OK;
}

sg_status sg_csr_invert(const sg_host_csr* in, sg_host_csr* out) {
  sgb::clear_error();
  if (!in || !out) return fail(SG_ERR_INVALID, "NULL argument");
  const uint32_t n = in->n;
  const uint64_t m = in->m;
  if (!in->row_offsets || (m && !in->column_indices)) return fail(SG_ERR_INVALID, "NULL CSR array");
  if (sgb::check_csr(in->row_offsets, in->column_indices, n, m) != SG_OK) return SG_ERR_INVALID;
  memset(out, 0, sizeof(*out));
  out->n = n;
  out->m = m;
  out->value_type = in->value_type;
  out->flags = in->flags;
  out->row_offsets = (uint32_t*)calloc((size_t)n + 1, sizeof(uint32_t));
  out->column_indices = (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1));
  if (in->values) out->values = malloc(sizeof(uint32_t) * (m ? m : 1));
  for (uint64_t e = 0; e < m; e++) out->row_offsets[(size_t)in->column_indices[e] + 1]++;
  for (uint32_t v = 0; v < n; v++) out->row_offsets[v + 1] += out->row_offsets[v];
  std::vector<uint32_t> cursor(out->row_offsets, out->row_offsets + n);
  for (uint32_t r = 0; r < n; r++)
    for (uint32_t e = in->row_offsets[r]; e < in->row_offsets[r + 1]; e++) {
      const uint32_t c = in->column_indices[e];
      const uint32_t d = cursor[c]++;
      out->column_indices[d] = r;
      if (in->values) ((uint32_t*)out->values)[d] = ((const uint32_t*)in->values)[e];
    }
  return SG_OK;
}

// Binary layout (io/read_csr.hpp:316-349): u64 magic "SYGRCSR\x01", u8 version,
// u8 flags (1 directed, 2 weighted), u16 + u32 reserved, u64 num_rows (the
// length of the row-offset array, n+1), u64 nnz, then the three arrays.
static const uint64_t kMagic = 0x5359475243535201ull;

sg_status sg_csr_write_binary(const sg_host_csr* csr, const char* path) {
  sgb::clear_error();
  if (!csr || !path) return fail(SG_ERR_INVALID, "NULL argument");
  FILE* f = fopen(path, "wb");
  if (!f) return fail(SG_ERR_INVALID, std::string("cannot open ") + path);
  const uint8_t version = 1;
  const uint8_t flags = (uint8_t)(csr->flags & 3u);
  const uint16_t r16 = 0;
  const uint32_t r32 = 0;
  const uint64_t rows = (uint64_t)csr->n + 1, nnz = csr->m;
  bool ok = fwrite(&kMagic, 8, 1, f) == 1 && fwrite(&version, 1, 1, f) == 1 && fwrite(&flags, 1, 1, f) == 1 &&
            fwrite(&r16, 2, 1, f) == 1 && fwrite(&r32, 4, 1, f) == 1 && fwrite(&rows, 8, 1, f) == 1 &&
            fwrite(&nnz, 8, 1, f) == 1 && fwrite(csr->row_offsets, 4, rows, f) == rows &&
            fwrite(csr->column_indices, 4, nnz, f) == nnz;
  if (ok) {
    if (csr->values) {
      ok = fwrite(csr->values, 4, nnz, f) == nnz;
    } else {
      std::vector<uint32_t> ones(nnz, 1u);
      if (csr->value_type == SG_WEIGHT_F32) {
        float one = 1.0f;
        uint32_t b;
        memcpy(&b, &one, 4);
        std::fill(ones.begin(), ones.end(), b);
      }
      ok = fwrite(ones.data(), 4, nnz, f) == nnz;
    }
  }
  fclose(f);
  return ok ? SG_OK : fail(SG_ERR_INVALID, "short write");
}

sg_status sg_csr_read_binary(const char* path, int value_type, sg_host_csr* out) {
  sgb::clear_error();
  if (!path || !out) return fail(SG_ERR_INVALID, "NULL argument");
  FILE* f = fopen(path, "rb");
  if (!f) return fail(SG_ERR_INVALID, std::string("cannot open ") + path);
  uint64_t first = 0, rows = 0, nnz = 0;
  uint32_t flags = SG_GRAPH_DIRECTED | SG_GRAPH_WEIGHTED;  // legacy layout: io/read_csr.hpp:393-399
  bool ok = fread(&first, 8, 1, f) == 1;
  if (ok && first == kMagic) {
    uint8_t version = 0, fl = 0;
    uint16_t r16;
    uint32_t r32;
    ok = fread(&version, 1, 1, f) == 1 && fread(&fl, 1, 1, f) == 1 && fread(&r16, 2, 1, f) == 1 &&
         fread(&r32, 4, 1, f) == 1 && fread(&rows, 8, 1, f) == 1 && fread(&nnz, 8, 1, f) == 1;
    flags = fl & 3u;
  } else if (ok) {
    rows = first;
    ok = fread(&nnz, 8, 1, f) == 1;
  }
  if (!ok || rows == 0 || rows > (1ull << 32) || nnz >= (1ull << 32)) {
    fclose(f);
    return fail(SG_ERR_INVALID, "malformed binary CSR header");
  }
  memset(out, 0, sizeof(*out));
  out->n = (uint32_t)(rows - 1);
  out->m = nnz;
  out->flags = flags;
  out->value_type = value_type;
  out->row_offsets = (uint32_t*)malloc(4 * rows);
  out->column_indices = (uint32_t*)malloc(4 * (nnz ? nnz : 1));
  out->values = malloc(4 * (nnz ? nnz : 1));
  ok = fread(out->row_offsets, 4, rows, f) == rows && fread(out->column_indices, 4, nnz, f) == nnz &&
       fread(out->values, 4, nnz, f) == nnz;
  fclose(f);
  if (!ok) {
    sg_host_csr_free(out);
    return fail(SG_ERR_INVALID, "malformed binary CSR body");
  }
  if (sgb::check_csr(out->row_offsets, out->column_indices, out->n, nnz) != SG_OK) {
    sg_host_csr_free(out);
    return SG_ERR_INVALID;  // the message names the first bad row or edge
  }
  if (value_type == SG_WEIGHT_NONE) {
    free(out->values);
    out->values = nullptr;
  }
  return SG_OK;
}

sg_status sg_csr_read_mm(const char* path, int value_type, sg_host_csr* out) {
  sgb::clear_error();
  if (!path || !out) return fail(SG_ERR_INVALID, "NULL argument");
  std::ifstream in(path);
  if (!in.is_open()) return fail(SG_ERR_INVALID, std::string("Failed to open file: ") + path);
  std::string line;
  bool banner_read = false, dims = false, pattern = false, symmetric = false;
  uint64_t rows = 0, cols = 0, nnz = 0;
  std::vector<std::tuple<uint32_t, uint32_t, uint32_t>> entries;
  while (std::getline(in, line)) {
    if (line.empty()) continue;
    if (line[0] == '%') {
      if (!banner_read) {
        banner_read = true;
        std::istringstream b(line);
        std::string tag, object, format, field, symmetry;
        b >> tag >> object >> format >> field >> symmetry;
        if (tag != "%%MatrixMarket") return fail(SG_ERR_INVALID, "Invalid MatrixMarket banner");
        if (object != "matrix") return fail(SG_ERR_INVALID, "Invalid MatrixMarket object type");
        if (format != "coordinate") return fail(SG_ERR_INVALID, "Invalid MatrixMarket format type");
        if (field == "pattern") pattern = true;
        else if (field == "real" && value_type == SG_WEIGHT_U32)
          return fail(SG_ERR_INVALID, "Invalid MatrixMarket field type");
        else if (field == "integer" && value_type == SG_WEIGHT_F32)
          return fail(SG_ERR_INVALID, "Invalid MatrixMarket field type");
        else if (field != "real" && field != "integer")
          return fail(SG_ERR_INVALID, "Invalid field type in MatrixMarket banner");
        if (symmetry == "symmetric") symmetric = true;
        else if (symmetry != "general") return fail(SG_ERR_INVALID, "Invalid symmetry type in MatrixMarket banner");
      }
      continue;
    }
    std::istringstream ls(line);
    if (!dims) {
      ls >> rows >> cols >> nnz;
      dims = true;
      if (rows >= 0xffffffffull) return fail(SG_ERR_INVALID, "matrix too large");
      entries.reserve(symmetric ? 2 * nnz : nnz);
      continue;
    }
    uint64_t r, c;
    ls >> r >> c;
    uint32_t bits = 1u;
    if (value_type == SG_WEIGHT_F32) {
      float v = 1.0f;
      if (!pattern) ls >> v;
      memcpy(&bits, &v, 4);
    } else if (!pattern) {
      double v = 1;
      ls >> v;
      bits = (uint32_t)v;
    }
    if (r < 1 || c < 1 || r > rows || c > rows) return fail(SG_ERR_INVALID, "entry out of range");
    entries.emplace_back((uint32_t)(r - 1), (uint32_t)(c - 1), bits);
    // Symmetric storage adds the transpose of every stored entry (io/read_csr.hpp:130-131).
    if (symmetric) entries.emplace_back((uint32_t)(c - 1), (uint32_t)(r - 1), bits);
  }
  std::stable_sort(entries.begin(), entries.end(), [](const auto& a, const auto& b) {
    return std::get<0>(a) < std::get<0>(b) || (std::get<0>(a) == std::get<0>(b) && std::get<1>(a) < std::get<1>(b));
  });
  memset(out, 0, sizeof(*out));
  out->n = (uint32_t)rows;
  out->m = entries.size();
  out->value_type = value_type;
  out->flags = (symmetric ? 0u : SG_GRAPH_DIRECTED) | (pattern ? 0u : SG_GRAPH_WEIGHTED);
  out->row_offsets = (uint32_t*)calloc(rows + 1, sizeof(uint32_t));
  out->column_indices = (uint32_t*)malloc(4 * (out->m ? out->m : 1));
  if (value_type != SG_WEIGHT_NONE) out->values = malloc(4 * (out->m ? out->m : 1));
  for (size_t i = 0; i < entries.size(); i++) {
    out->row_offsets[std::get<0>(entries[i]) + 1]++;
    out->column_indices[i] = std::get<1>(entries[i]);
    if (out->values) ((uint32_t*)out->values)[i] = std::get<2>(entries[i]);
  }
  for (uint64_t v = 0; v < rows; v++) out->row_offsets[v + 1] += out->row_offsets[v];
  return SG_OK;
}

sg_status sg_sample_sources(const sg_host_csr* csr, uint32_t k, uint64_t seed, uint32_t* out_sources) {
  sgb::clear_error();
  if (!csr || !out_sources) return fail(SG_ERR_INVALID, "NULL argument");
  uint64_t nonzero = 0;
  for (uint32_t v = 0; v < csr->n; v++) nonzero += csr->row_offsets[v + 1] > csr->row_offsets[v];
  if (nonzero < k) return fail(SG_ERR_INVALID, "fewer vertices with edges than requested sources");
  std::vector<uint8_t> taken(csr->n, 0);
  uint32_t got = 0;
  for (uint64_t i = 0; got < k; i++) {
    const uint32_t v = (uint32_t)(hash2(seed, i) % csr->n);
    if (taken[v] || csr->row_offsets[v + 1] == csr->row_offsets[v]) continue;
    taken[v] = 1;
    out_sources[got++] = v;
  }
  return SG_OK;
}

}  // extern "C"
