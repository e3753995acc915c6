// sk_text.cu — the input and output contracts on the device: Soufflé TSV
// parsing with first-seen symbol interning, and the canonical text rendering
// of a relation.
//
// Input (strata-k/src/input.rs:53-197, 216-232).  The file's lines are split
// on '\n' (str::lines), trailing '\r's dropped, empty lines skipped; a row
// splits on '\t' into exactly `arity` symbol cells (+ one trailing weight
// cell for a Trop predicate); an empty symbol cell, a wrong cell count or a
// trailing cell that `trim().parse::<i64>()` rejects is an error reported
// with the 1-based line of the first failing row.  Symbol cells are interned
// first-seen (strata-ir/src/dict.rs:35-43) in row order, column order, after
// the symbols the dictionary already holds.
//
// Device interning: every cell (the dictionary's strings first, then the
// file's cells in interning order) gets a seeded 64-bit hash; a stable radix
// sort of (hash, position) puts equal strings next to each other with their
// first occurrence first; adjacent equal hashes are verified byte by byte
// (a mismatch — a hash collision — reruns with another seed, at most four
// times, so every id returned is exact); the first occurrences that are new
// to the dictionary are ranked by position, which is the first-seen order.
//
// Output (strata-cli/src/render.rs:29-54, 87-92): one line per tuple,
// `name(a, b)` with ` = w` or ` = inf` for Trop, tuples in id order.  The
// line lengths are computed, scanned and the bytes written in parallel.
#include "sk_ops.cuh"
#include "sk_prims.cuh"
#include "sk_rel.cuh"

#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace sk {
namespace {

constexpr int NT = 256;
constexpr int TX_ITEMS = 16;  // bytes per thread in the byte-flag passes
constexpr uint32_t TX_TILE = NT * TX_ITEMS;

inline unsigned gridn(uint64_t n, uint64_t per) { return (unsigned)ceil_div(n ? n : 1, per); }

// ---- flagged positions of a byte, in order (newlines, tabs) ----------------
__global__ void __launch_bounds__(NT) k_byte_count(const uint8_t* __restrict__ t, uint64_t n, uint8_t c,
                                                   uint64_t* __restrict__ tile_cnt) {
  __shared__ uint32_t s_red[NT / 32];
  const uint64_t b = (uint64_t)blockIdx.x * TX_TILE + (uint64_t)threadIdx.x * TX_ITEMS;
  uint32_t k = 0;
#pragma unroll
  for (int j = 0; j < TX_ITEMS; j++) k += (b + j < n && t[b + j] == c) ? 1u : 0u;
  k = warp_sum(k);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = k;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t s = 0;
    for (int w = 0; w < NT / 32; w++) s += s_red[w];
    tile_cnt[blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(NT) k_byte_write(const uint8_t* __restrict__ t, uint64_t n, uint8_t c,
                                                   const uint64_t* __restrict__ tile_off, uint64_t* __restrict__ pos) {
  __shared__ uint32_t s_scan[NT / 32 + 1];
  const uint64_t b = (uint64_t)blockIdx.x * TX_TILE + (uint64_t)threadIdx.x * TX_ITEMS;
  uint32_t m = 0;
#pragma unroll
  for (int j = 0; j < TX_ITEMS; j++)
    if (b + j < n && t[b + j] == c) m |= 1u << j;
  uint32_t tot;
  const uint32_t ex = block_excl_sum<NT>((uint32_t)__popc(m), s_scan, &tot);
  uint64_t at = tile_off[blockIdx.x] + ex;
  for (int j = 0; j < TX_ITEMS; j++)
    if ((m >> j) & 1u) pos[at++] = b + j;
}

// ---- rows --------------------------------------------------------------------
// Line i spans [i == 0 ? 0 : nl[i-1] + 1, i < n_nl ? nl[i] : n).  A row is a
// line that is not empty once its trailing '\r's are dropped.
__device__ __forceinline__ void line_span(const uint8_t* t, uint64_t n, const uint64_t* nl, uint64_t n_nl, uint64_t i,
                                          uint64_t* s, uint64_t* e) {
  uint64_t a = i == 0 ? 0 : nl[i - 1] + 1;
  uint64_t z = i < n_nl ? nl[i] : n;
  while (z > a && t[z - 1] == '\r') z--;
  *s = a;
  *e = z;
}

__global__ void __launch_bounds__(NT) k_rows_count(const uint8_t* __restrict__ t, uint64_t n,
                                                   const uint64_t* __restrict__ nl, uint64_t n_lines, uint64_t n_nl,
                                                   uint64_t* __restrict__ tile_cnt) {
  __shared__ uint32_t s_red[NT / 32];
  const uint64_t b = (uint64_t)blockIdx.x * TX_TILE + (uint64_t)threadIdx.x * TX_ITEMS;
  uint32_t k = 0;
  for (int j = 0; j < TX_ITEMS; j++) {
    if (b + j >= n_lines) break;
    uint64_t s, e;
    line_span(t, n, nl, n_nl, b + j, &s, &e);
    k += e > s ? 1u : 0u;
  }
  k = warp_sum(k);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = k;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t sum = 0;
    for (int w = 0; w < NT / 32; w++) sum += s_red[w];
    tile_cnt[blockIdx.x] = sum;
  }
}

__global__ void __launch_bounds__(NT) k_rows_write(const uint8_t* __restrict__ t, uint64_t n,
                                                   const uint64_t* __restrict__ nl, uint64_t n_lines, uint64_t n_nl,
                                                   const uint64_t* __restrict__ tile_off, uint64_t* __restrict__ rs,
                                                   uint64_t* __restrict__ re, uint64_t* __restrict__ rline) {
  __shared__ uint32_t s_scan[NT / 32 + 1];
  const uint64_t b = (uint64_t)blockIdx.x * TX_TILE + (uint64_t)threadIdx.x * TX_ITEMS;
  uint32_t m = 0;
  for (int j = 0; j < TX_ITEMS; j++) {
    if (b + j >= n_lines) break;
    uint64_t s, e;
    line_span(t, n, nl, n_nl, b + j, &s, &e);
    if (e > s) m |= 1u << j;
  }
  uint32_t tot;
  const uint32_t ex = block_excl_sum<NT>((uint32_t)__popc(m), s_scan, &tot);
  uint64_t at = tile_off[blockIdx.x] + ex;
  for (int j = 0; j < TX_ITEMS; j++) {
    if ((m >> j) & 1u) {
      uint64_t s, e;
      line_span(t, n, nl, n_nl, b + j, &s, &e);
      rs[at] = s;
      re[at] = e;
      rline[at] = b + j + 1;
      at++;
    }
  }
}

__device__ __forceinline__ uint64_t lower_bound_u64(const uint64_t* a, uint64_t n, uint64_t x) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Rust's char::is_whitespace (White_Space) at byte i of t[a, e): the length
// of the whitespace character starting there, 0 if none.
__device__ __forceinline__ int ws_len_fwd(const uint8_t* t, uint64_t i, uint64_t e) {
  const uint8_t c = t[i];
  if (c == ' ' || (c >= 0x09 && c <= 0x0d)) return 1;
  if (c == 0xc2 && i + 1 < e && (t[i + 1] == 0x85 || t[i + 1] == 0xa0)) return 2;
  if (c == 0xe1 && i + 2 < e && t[i + 1] == 0x9a && t[i + 2] == 0x80) return 3;  // U+1680
  if (c == 0xe2 && i + 2 < e) {
    const uint8_t d = t[i + 1], f = t[i + 2];
    if (d == 0x80 && ((f >= 0x80 && f <= 0x8a) || f == 0xa8 || f == 0xa9 || f == 0xaf)) return 3;  // U+2000-200A,2028,2029,202F
    if (d == 0x81 && f == 0x9f) return 3;  // U+205F
  }
  if (c == 0xe3 && i + 2 < e && t[i + 1] == 0x80 && t[i + 2] == 0x80) return 3;  // U+3000
  return 0;
}
// The same for the character that ends at byte e - 1 of t[a, e).
__device__ __forceinline__ int ws_len_back(const uint8_t* t, uint64_t a, uint64_t e) {
  if (e > a && ws_len_fwd(t, e - 1, e) == 1) return 1;
  if (e >= a + 2 && ws_len_fwd(t, e - 2, e) == 2) return 2;
  if (e >= a + 3 && ws_len_fwd(t, e - 3, e) == 3) return 3;
  return 0;
}

// `s.trim().parse::<i64>()`: optional sign, at least one digit, no overflow.
__device__ bool parse_i64(const uint8_t* t, uint64_t a, uint64_t e, int64_t* out) {
  for (int k; a < e && (k = ws_len_fwd(t, a, e)) > 0;) a += k;
  for (int k; e > a && (k = ws_len_back(t, a, e)) > 0;) e -= k;
  if (a >= e) return false;
  bool neg = false;
  if (t[a] == '+' || t[a] == '-') {
    neg = t[a] == '-';
    a++;
  }
  if (a >= e) return false;
  // accumulate as a negative number so i64::MIN parses
  long long v = 0;
  for (uint64_t i = a; i < e; i++) {
    const uint8_t c = t[i];
    if (c < '0' || c > '9') return false;
    const long long d = c - '0';
    if (v < (LLONG_MIN + d) / 10) return false;
    v = v * 10 - d;
  }
  if (!neg) {
    if (v == LLONG_MIN) return false;
    v = -v;
  }
  *out = v;
  return true;
}

// One thread per row: split on the tabs, check, record cells and the weight.
// err = (line << 8) | order (order 0 column count, 1 + c empty column c,
// 255 weight) keeps the first failing row and its first failing check.
__global__ void k_rows_split(const uint8_t* __restrict__ t, const uint64_t* __restrict__ rs,
                             const uint64_t* __restrict__ re, const uint64_t* __restrict__ rline, uint64_t rows,
                             const uint64_t* __restrict__ tabs, uint64_t n_tabs, uint32_t arity, int trop,
                             uint64_t text_base, uint64_t* __restrict__ cell_off, uint32_t* __restrict__ cell_len,
                             int64_t* __restrict__ w, unsigned long long* err) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const uint64_t s = rs[r], e = re[r];
  const uint64_t k0 = lower_bound_u64(tabs, n_tabs, s), k1 = lower_bound_u64(tabs, n_tabs, e);
  const uint32_t ncols = arity + (trop ? 1u : 0u);
  const unsigned long long line = rline[r];
  if (k1 - k0 != (uint64_t)ncols - 1) {
    atomicMin(err, (line << 8) | 0ull);
    return;
  }
  for (uint32_t c = 0; c < ncols; c++) {
    const uint64_t a = c == 0 ? s : tabs[k0 + c - 1] + 1;
    const uint64_t z = c + 1 == ncols ? e : tabs[k0 + c];
    if (c < arity) {
      if (z == a) {
        atomicMin(err, (line << 8) | (unsigned long long)(1 + c));
        return;
      }
      cell_off[r * arity + c] = text_base + a;
      cell_len[r * arity + c] = (uint32_t)(z - a);
    } else {
      int64_t v;
      if (!parse_i64(t, a, z, &v)) {
        atomicMin(err, (line << 8) | 255ull);
        return;
      }
      w[r] = v;
    }
  }
}

// ---- interning ---------------------------------------------------------------
__device__ __forceinline__ uint64_t mix_h(uint64_t z) {
  z ^= z >> 33;
  z *= 0xff51afd7ed558ccdull;
  z ^= z >> 33;
  z *= 0xc4ceb9fe1a85ec53ull;
  z ^= z >> 33;
  return z;
}

// Seeded hash of a byte string: 8-byte little-endian words folded through a
// multiply-xorshift mixer (MurmurHash3's 64-bit finalizer), length last.
__global__ void k_cell_hash(const uint8_t* __restrict__ B, const uint64_t* __restrict__ off,
                            const uint32_t* __restrict__ len, uint64_t n, uint64_t seed, uint64_t* __restrict__ h,
                            uint32_t* __restrict__ pos) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t* p = B + off[i];
  const uint32_t L = len[i];
  uint64_t acc = seed ^ 0x9e3779b97f4a7c15ull;
  uint32_t k = 0;
  for (; k + 8 <= L; k += 8) {
    uint64_t wv = 0;
#pragma unroll
    for (int b = 0; b < 8; b++) wv |= (uint64_t)p[k + b] << (8 * b);
    acc = mix_h(acc ^ wv) + 0x9e3779b97f4a7c15ull;
  }
  uint64_t wv = 0;
  for (uint32_t b = 0; k + b < L; b++) wv |= (uint64_t)p[k + b] << (8 * b);
  acc = mix_h(acc ^ wv ^ ((uint64_t)L << 56));
  h[i] = acc;
  pos[i] = (uint32_t)i;
}

__device__ __forceinline__ bool bytes_equal(const uint8_t* B, uint64_t oa, uint32_t la, uint64_t ob, uint32_t lb) {
  if (la != lb) return false;
  for (uint32_t k = 0; k < la; k++)
    if (B[oa + k] != B[ob + k]) return false;
  return true;
}

// Adjacent equal hashes must be equal strings; head flags of the runs.
__global__ void k_cell_verify(const uint8_t* __restrict__ B, const uint64_t* __restrict__ off,
                              const uint32_t* __restrict__ len, const uint64_t* __restrict__ h,
                              const uint32_t* __restrict__ pos, uint64_t n, uint32_t* __restrict__ head,
                              uint32_t* collision) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool hd = i == 0 || h[i] != h[i - 1];
  head[i] = hd ? 1u : 0u;
  if (!hd && !bytes_equal(B, off[pos[i]], len[pos[i]], off[pos[i - 1]], len[pos[i - 1]])) atomicOr(collision, 1u);
}

// newhead[p] = 1 for the first occurrence (by position) of a string the
// dictionary does not hold.
__global__ void k_new_heads(const uint32_t* __restrict__ head, const uint32_t* __restrict__ pos, uint64_t n,
                            uint64_t n_dict, uint32_t* __restrict__ newhead) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (head[i] && pos[i] >= n_dict) newhead[pos[i]] = 1u;
}

// run_of[i] = the inclusive count of heads up to sorted element i (its run's
// index + 1): the id of each run, then the id of every position.
__global__ void k_run_ids(const uint32_t* __restrict__ head, const uint64_t* __restrict__ run_of,
                          const uint32_t* __restrict__ pos, const uint64_t* __restrict__ rank, uint64_t n,
                          uint64_t n_dict, uint32_t* __restrict__ run_id) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !head[i]) return;
  const uint64_t p = pos[i];
  run_id[run_of[i] - 1] = p < n_dict ? (uint32_t)p : (uint32_t)(n_dict + rank[p]);
}

__global__ void k_pos_ids(const uint64_t* __restrict__ run_of, const uint32_t* __restrict__ pos,
                          const uint32_t* __restrict__ run_id, uint64_t n, uint32_t* __restrict__ id_of_pos) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) id_of_pos[pos[i]] = run_id[run_of[i] - 1];
}

// New symbols in id order: their byte ranges (positions of the new heads).
__global__ void k_new_syms(const uint32_t* __restrict__ newhead, const uint64_t* __restrict__ rank, uint64_t n,
                           uint64_t n_dict, const uint64_t* __restrict__ off, const uint32_t* __restrict__ len,
                           uint64_t* __restrict__ new_src, uint32_t* __restrict__ new_len) {
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || p < n_dict || !newhead[p]) return;
  new_src[rank[p]] = off[p];
  new_len[rank[p]] = len[p];
}

__global__ void k_gather_bytes(const uint8_t* __restrict__ B, const uint64_t* __restrict__ src,
                               const uint32_t* __restrict__ len, const uint64_t* __restrict__ dst_off, uint64_t n,
                               uint8_t* __restrict__ out) {
  const uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  for (uint32_t k = lane; k < len[i]; k += 32) out[dst_off[i] + k] = B[src[i] + k];
}

__global__ void k_cols_out(const uint32_t* __restrict__ id_of_pos, uint64_t n_dict, uint64_t rows, uint32_t arity,
                           uint32_t* __restrict__ cols) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= rows * arity) return;
  const uint64_t r = q / arity, c = q - r * arity;
  cols[c * rows + r] = id_of_pos[n_dict + q];
}

__global__ void k_u32_to_u64(const uint32_t* __restrict__ a, uint64_t n, uint64_t* __restrict__ b) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}

// ---- rendering ----------------------------------------------------------------
__device__ __forceinline__ uint32_t dec_len(uint64_t m) {
  uint32_t k = 1;
  while (m >= 10) {
    m /= 10;
    k++;
  }
  return k;
}
__device__ __forceinline__ uint32_t i64_len(int64_t v) {
  return v < 0 ? 1 + dec_len(v == INT64_MIN ? 9223372036854775808ull : (uint64_t)(-v)) : dec_len((uint64_t)v);
}
__device__ __forceinline__ void i64_write(int64_t v, uint8_t* o) {
  uint64_t m;
  if (v < 0) {
    *o++ = '-';
    m = v == INT64_MIN ? 9223372036854775808ull : (uint64_t)(-v);
  } else {
    m = (uint64_t)v;
  }
  const uint32_t L = dec_len(m);
  for (uint32_t k = 0; k < L; k++) {
    o[L - 1 - k] = (uint8_t)('0' + m % 10);
    m /= 10;
  }
}

struct RenderSpec {
  const uint8_t* dict;
  const uint64_t* dict_off;  // n_dict + 1
  uint64_t n_dict;
  const uint8_t* name;
  uint32_t name_len;
  uint32_t arity;
  int trop;
};

// line = name '(' s0 [', ' s1] ')' [' = ' w|inf] '\n'
__device__ __forceinline__ uint64_t sym_len(const RenderSpec& R, uint32_t id) {
  return id < R.n_dict ? R.dict_off[id + 1] - R.dict_off[id] : 1;  // '?' for an id the dictionary lacks
}

__global__ void k_render_len(RenderSpec R, const uint32_t* __restrict__ c0, const uint32_t* __restrict__ c1,
                             const int64_t* __restrict__ w, const uint8_t* __restrict__ inf, uint64_t n,
                             uint64_t* __restrict__ len) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t L = R.name_len + 2 + 1 + sym_len(R, c0[i]);
  if (R.arity == 2) L += 2 + sym_len(R, c1[i]);
  if (R.trop) L += 3 + ((inf && inf[i]) ? 3 : i64_len(w[i]));
  len[i] = L;
}

__device__ __forceinline__ uint8_t* put_sym(const RenderSpec& R, uint32_t id, uint8_t* o) {
  if (id >= R.n_dict) {
    *o++ = '?';
    return o;
  }
  for (uint64_t k = R.dict_off[id]; k < R.dict_off[id + 1]; k++) *o++ = R.dict[k];
  return o;
}

__global__ void k_render_write(RenderSpec R, const uint32_t* __restrict__ c0, const uint32_t* __restrict__ c1,
                               const int64_t* __restrict__ w, const uint8_t* __restrict__ inf, uint64_t n,
                               const uint64_t* __restrict__ start, uint8_t* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint8_t* o = out + start[i];
  for (uint32_t k = 0; k < R.name_len; k++) *o++ = R.name[k];
  *o++ = '(';
  o = put_sym(R, c0[i], o);
  if (R.arity == 2) {
    *o++ = ',';
    *o++ = ' ';
    o = put_sym(R, c1[i], o);
  }
  *o++ = ')';
  if (R.trop) {
    *o++ = ' ';
    *o++ = '=';
    *o++ = ' ';
    if (inf && inf[i]) {
      *o++ = 'i';
      *o++ = 'n';
      *o++ = 'f';
    } else {
      i64_write(w[i], o);
      o += i64_len(w[i]);
    }
  }
  *o = '\n';
}

// Ordered positions of byte `c` in t[0, n).
uint64_t byte_positions(strata_ctx* ctx, const uint8_t* t, uint64_t n, uint8_t c, DBuf<uint64_t>& pos) {
  const uint64_t tiles = ceil_div(n ? n : 1, TX_TILE);
  DBuf<uint64_t> tc(ctx, tiles + 1);
  k_byte_count<<<(unsigned)tiles, NT, 0, ctx->stream>>>(t, n, c, tc.p);
  after_launch(ctx, "k_byte_count");
  scan_tile_sums(ctx, tc.p, tiles);
  uint64_t m;
  read_u64(ctx, tc.p + tiles, &m, 1);
  pos.reserve(m + 1);
  k_byte_write<<<(unsigned)tiles, NT, 0, ctx->stream>>>(t, n, c, tc.p, pos.p);
  after_launch(ctx, "k_byte_write");
  return m;
}

}  // namespace

TsvResult tsv_load(strata_ctx* ctx, const char* text, uint64_t text_len, uint32_t arity, bool trop,
                   const char* dict_bytes, const uint64_t* dict_off, uint64_t n_dict) {
  TsvResult R;
  const uint64_t dict_len = n_dict ? dict_off[n_dict] : 0;
  const uint64_t total_bytes = dict_len + text_len;
  DBuf<uint8_t> B(ctx, total_bytes + 1);
  if (dict_len) SK_CUDA(cudaMemcpyAsync(B.p, dict_bytes, dict_len, cudaMemcpyHostToDevice, ctx->stream));
  if (text_len) SK_CUDA(cudaMemcpyAsync(B.p + dict_len, text, text_len, cudaMemcpyHostToDevice, ctx->stream));
  const uint8_t* T = B.p + dict_len;
  // rows
  DBuf<uint64_t> nl, tabs;
  nl.ctx = tabs.ctx = ctx;
  const uint64_t n_nl = byte_positions(ctx, T, text_len, '\n', nl);
  const uint64_t n_tabs = byte_positions(ctx, T, text_len, '\t', tabs);
  // lines: n_nl + 1 (the last one after the final '\n', possibly empty)
  const uint64_t n_lines = n_nl + 1;
  const uint64_t ltiles = ceil_div(n_lines, TX_TILE);
  DBuf<uint64_t> lt(ctx, ltiles + 1);
  k_rows_count<<<(unsigned)ltiles, NT, 0, ctx->stream>>>(T, text_len, nl.p, n_lines, n_nl, lt.p);
  after_launch(ctx, "k_rows_count");
  scan_tile_sums(ctx, lt.p, ltiles);
  uint64_t rows;
  read_u64(ctx, lt.p + ltiles, &rows, 1);
  DBuf<uint64_t> rs(ctx, rows + 1), re(ctx, rows + 1), rl(ctx, rows + 1);
  k_rows_write<<<(unsigned)ltiles, NT, 0, ctx->stream>>>(T, text_len, nl.p, n_lines, n_nl, lt.p, rs.p, re.p, rl.p);
  after_launch(ctx, "k_rows_write");
  // cells: dictionary strings first, then the file's symbol cells in interning order
  const uint64_t n_cells = n_dict + rows * arity;
  if (n_cells > kMaxSortN) fail(STRATA_E_UNSUPPORTED, "more than 2^30 - 1 symbol cells (dictionary + file) in one load");
  DBuf<uint64_t> coff(ctx, n_cells + 1);
  DBuf<uint32_t> clen(ctx, n_cells + 1);
  DBuf<int64_t> w(ctx, trop ? rows + 1 : 1);
  if (n_dict) {
    std::vector<uint64_t> ho(n_dict);
    std::vector<uint32_t> hl(n_dict);
    for (uint64_t i = 0; i < n_dict; i++) {
      ho[i] = dict_off[i];
      hl[i] = (uint32_t)(dict_off[i + 1] - dict_off[i]);
    }
    SK_CUDA(cudaMemcpyAsync(coff.p, ho.data(), n_dict * 8, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(clen.p, hl.data(), n_dict * 4, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaStreamSynchronize(ctx->stream));  // the host staging vectors go out of scope
  }
  DBuf<unsigned long long> err(ctx, 1);
  const unsigned long long no_err = ~0ull;
  SK_CUDA(cudaMemcpyAsync(err.p, &no_err, 8, cudaMemcpyHostToDevice, ctx->stream));
  if (rows) {
    k_rows_split<<<gridn(rows, NT), NT, 0, ctx->stream>>>(T, rs.p, re.p, rl.p, rows, tabs.p, n_tabs, arity, trop ? 1 : 0,
                                                          dict_len, coff.p + n_dict, clen.p + n_dict, w.p, err.p);
    after_launch(ctx, "k_rows_split");
  }
  uint64_t e;
  read_u64(ctx, reinterpret_cast<uint64_t*>(err.p), &e, 1);
  sync_and_check(ctx);
  if (e != ~0ull) {
    R.err_line = e >> 8;
    const uint32_t order = (uint32_t)(e & 0xff);
    R.err_kind = order == 0 ? 1 : order == 255 ? 3 : 2;
    R.err_col = (order >= 1 && order <= 254) ? order : 0;
    return R;
  }
  R.rows = rows;
  // intern: hash, sort, verify (reseed on a collision)
  DBuf<uint64_t> h(ctx, n_cells + 1), h2(ctx, n_cells + 1);
  DBuf<uint32_t> pos(ctx, n_cells + 1), pos2(ctx, n_cells + 1), head(ctx, n_cells + 1);
  DBuf<uint32_t> coll(ctx, 1);
  uint64_t* hp = nullptr;
  uint32_t* pp = nullptr;
  bool ok = false;
  for (int attempt = 0; attempt < 4 && !ok; attempt++) {
    const uint64_t seed = 0x2545F4914F6CDD1Dull * (uint64_t)(attempt + 1);
    k_cell_hash<<<gridn(n_cells, NT), NT, 0, ctx->stream>>>(B.p, coff.p, clen.p, n_cells, seed, h.p, pos.p);
    after_launch(ctx, "k_cell_hash");
    hp = h.p;
    uint64_t* ha = h2.p;
    pp = pos.p;
    uint32_t* pa = pos2.p;
    radix_sort<uint64_t, uint32_t>(ctx, &hp, &ha, &pp, &pa, true, n_cells, 64, true);
    SK_CUDA(cudaMemsetAsync(coll.p, 0, 4, ctx->stream));
    k_cell_verify<<<gridn(n_cells, NT), NT, 0, ctx->stream>>>(B.p, coff.p, clen.p, hp, pp, n_cells, head.p, coll.p);
    after_launch(ctx, "k_cell_verify");
    uint32_t c = 0;
    SK_CUDA(cudaMemcpyAsync(&c, coll.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    ok = c == 0;
  }
  if (!ok) fail(STRATA_E_UNSUPPORTED, "symbol interning met a 64-bit hash collision under four seeds");
  // run index of every sorted cell; first-seen rank of the new strings
  DBuf<uint64_t> h64(ctx, n_cells + 1), run_of(ctx, n_cells + 1), nh64(ctx, n_cells + 1), rank(ctx, n_cells + 1);
  DBuf<uint32_t> newhead(ctx, n_cells + 1), run_id(ctx, n_cells + 1), id_of_pos(ctx, n_cells + 1);
  k_u32_to_u64<<<gridn(n_cells, NT), NT, 0, ctx->stream>>>(head.p, n_cells, h64.p);
  after_launch(ctx, "k_u32_to_u64");
  // run_of[i] = heads at or before sorted position i = the run's index + 1
  scan_u64(ctx, h64.p, n_cells, run_of.p, true, nullptr);
  SK_CUDA(cudaMemsetAsync(newhead.p, 0, (n_cells + 1) * 4, ctx->stream));
  k_new_heads<<<gridn(n_cells, NT), NT, 0, ctx->stream>>>(head.p, pp, n_cells, n_dict, newhead.p);
  after_launch(ctx, "k_new_heads");
  k_u32_to_u64<<<gridn(n_cells, NT), NT, 0, ctx->stream>>>(newhead.p, n_cells, nh64.p);
  after_launch(ctx, "k_u32_to_u64");
  uint64_t n_new;
  scan_u64(ctx, nh64.p, n_cells, rank.p, false, &n_new);
  R.n_new = n_new;
  k_run_ids<<<gridn(n_cells, NT), NT, 0, ctx->stream>>>(head.p, run_of.p, pp, rank.p, n_cells, n_dict, run_id.p);
  after_launch(ctx, "k_run_ids");
  k_pos_ids<<<gridn(n_cells, NT), NT, 0, ctx->stream>>>(run_of.p, pp, run_id.p, n_cells, id_of_pos.p);
  after_launch(ctx, "k_pos_ids");
  // outputs: columns, weights, new symbols
  DBuf<uint32_t> cols(ctx, rows * arity + 1);
  if (rows) {
    k_cols_out<<<gridn(rows * arity, NT), NT, 0, ctx->stream>>>(id_of_pos.p, n_dict, rows, arity, cols.p);
    after_launch(ctx, "k_cols_out");
  }
  DBuf<uint64_t> nsrc(ctx, n_new + 1), noff(ctx, n_new + 2), nlen64(ctx, n_new + 1);
  DBuf<uint32_t> nlen(ctx, n_new + 1);
  uint64_t new_bytes = 0;
  if (n_new) {
    k_new_syms<<<gridn(n_cells, NT), NT, 0, ctx->stream>>>(newhead.p, rank.p, n_cells, n_dict, coff.p, clen.p, nsrc.p,
                                                           nlen.p);
    after_launch(ctx, "k_new_syms");
    k_u32_to_u64<<<gridn(n_new, NT), NT, 0, ctx->stream>>>(nlen.p, n_new, nlen64.p);
    after_launch(ctx, "k_u32_to_u64");
    scan_u64(ctx, nlen64.p, n_new, noff.p, false, &new_bytes);
  }
  DBuf<uint8_t> nbytes(ctx, new_bytes + 1);
  if (n_new) {
    k_gather_bytes<<<gridn(n_new * 32, NT), NT, 0, ctx->stream>>>(B.p, nsrc.p, nlen.p, noff.p, n_new, nbytes.p);
    after_launch(ctx, "k_gather_bytes");
  }
  sync_and_check(ctx);
  R.cols = static_cast<uint32_t*>(std::malloc(std::max<uint64_t>(1, rows * arity) * 4));
  R.w = trop ? static_cast<int64_t*>(std::malloc(std::max<uint64_t>(1, rows) * 8)) : nullptr;
  R.new_bytes = static_cast<char*>(std::malloc(new_bytes + 1));
  R.new_off = static_cast<uint64_t*>(std::malloc((n_new + 1) * 8));
  if (!R.cols || (trop && !R.w) || !R.new_bytes || !R.new_off) fail(STRATA_E_OOM, "host allocation failed");
  if (rows * arity) SK_CUDA(cudaMemcpyAsync(R.cols, cols.p, rows * arity * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (trop && rows) SK_CUDA(cudaMemcpyAsync(R.w, w.p, rows * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (new_bytes) SK_CUDA(cudaMemcpyAsync(R.new_bytes, nbytes.p, new_bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (n_new) SK_CUDA(cudaMemcpyAsync(R.new_off, noff.p, n_new * 8, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  R.new_off[n_new] = new_bytes;
  R.new_bytes[new_bytes] = 0;
  return R;
}

uint64_t render_rel(strata_ctx* ctx, const strata_rel* rel, const char* name, const char* dict_bytes,
                    const uint64_t* dict_off, uint64_t n_dict, char** out_text) {
  const uint64_t n = rel->n;
  const uint64_t name_len = std::strlen(name);
  const uint64_t dict_len = n_dict ? dict_off[n_dict] : 0;
  DBuf<uint8_t> D(ctx, dict_len + name_len + 1);
  DBuf<uint64_t> DO(ctx, n_dict + 1);
  if (dict_len) SK_CUDA(cudaMemcpyAsync(D.p, dict_bytes, dict_len, cudaMemcpyHostToDevice, ctx->stream));
  if (name_len) SK_CUDA(cudaMemcpyAsync(D.p + dict_len, name, name_len, cudaMemcpyHostToDevice, ctx->stream));
  SK_CUDA(cudaMemcpyAsync(DO.p, dict_off, (n_dict + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
  DBuf<uint32_t> c0(ctx, n + 1), c1(ctx, n + 1);
  DBuf<int64_t> w(ctx, rel->trop ? n + 1 : 1);
  DBuf<uint8_t> inf(ctx, rel->trop ? n + 1 : 1);
  const int arity = 2;
  if (n) {
    ctx->wshift = rel->wshift;
    if (rel->key_bytes == 4) {
      const uint32_t* k = static_cast<const uint32_t*>(rel->keys);
      if (!rel->trop) unpack_pairs<uint32_t, int32_t, false>(ctx, k, nullptr, n, rel->shift, c0.p, c1.p, nullptr, nullptr);
      else if (rel->w_bytes == 4) unpack_pairs<uint32_t, int32_t, true>(ctx, k, (const int32_t*)rel->w, n, rel->shift, c0.p, c1.p, w.p, inf.p);
      else unpack_pairs<uint32_t, int64_t, true>(ctx, k, (const int64_t*)rel->w, n, rel->shift, c0.p, c1.p, w.p, inf.p);
    } else {
      const uint64_t* k = static_cast<const uint64_t*>(rel->keys);
      if (!rel->trop) unpack_pairs<uint64_t, int32_t, false>(ctx, k, nullptr, n, rel->shift, c0.p, c1.p, nullptr, nullptr);
      else if (rel->w_bytes == 4) unpack_pairs<uint64_t, int32_t, true>(ctx, k, (const int32_t*)rel->w, n, rel->shift, c0.p, c1.p, w.p, inf.p);
      else unpack_pairs<uint64_t, int64_t, true>(ctx, k, (const int64_t*)rel->w, n, rel->shift, c0.p, c1.p, w.p, inf.p);
    }
  }
  RenderSpec R{D.p, DO.p, n_dict, D.p + dict_len, (uint32_t)name_len, (uint32_t)arity, rel->trop ? 1 : 0};
  DBuf<uint64_t> len(ctx, n + 1), start(ctx, n + 1);
  uint64_t total = 0;
  if (n) {
    k_render_len<<<gridn(n, NT), NT, 0, ctx->stream>>>(R, c0.p, c1.p, rel->trop ? w.p : nullptr,
                                                       rel->trop ? inf.p : nullptr, n, len.p);
    after_launch(ctx, "k_render_len");
    scan_u64(ctx, len.p, n, start.p, false, &total);
  }
  DBuf<uint8_t> out(ctx, total + 1);
  if (n) {
    k_render_write<<<gridn(n, NT), NT, 0, ctx->stream>>>(R, c0.p, c1.p, rel->trop ? w.p : nullptr,
                                                         rel->trop ? inf.p : nullptr, n, start.p, out.p);
    after_launch(ctx, "k_render_write");
  }
  char* h = static_cast<char*>(std::malloc(total + 1));
  if (!h) fail(STRATA_E_OOM, "host allocation failed");
  if (total) SK_CUDA(cudaMemcpyAsync(h, out.p, total, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  h[total] = 0;
  *out_text = h;
  return total;
}

}  // namespace sk
