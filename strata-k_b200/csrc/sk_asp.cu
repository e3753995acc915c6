// sk_asp.cu — the ASP grounding-simplify filter on the device
// (strata-gpu/src/asp.rs:53-100 gives its semantics; the reference runs it
// with host-scanned block sums).
//
// A ground rule  h :- pos, not neg  (body literals +(a+1) / -(a+1)) dies when
// a positive atom is impossible or a negative atom is certain; in a rule that
// lives, certain positive atoms and impossible negative atoms are dropped
// (trivially true).  `poss` / `cert` are the caller's bitsets, one byte per
// atom, read as the CPU reference reads them (keep_literal, asp.rs:53-67):
// a positive literal dies on !poss and is dropped on cert; a negative one
// dies on cert and is dropped on !poss.
//
// One thread per rule decides life and its kept-literal count; two device
// scans give each surviving rule its output index and literal offset; the
// write pass copies heads and kept literals.  No host round trip between
// passes.
#include "sk_ops.cuh"
#include "sk_prims.cuh"

#include <cstdlib>

namespace sk {
namespace {

constexpr int NT = 256;

// 0: the literal kills its rule; 1: kept; 2: dropped (trivially true).
__device__ __forceinline__ int asp_lit(int32_t l, const uint8_t* poss, const uint8_t* cert) {
  const uint64_t a = (uint64_t)(l > 0 ? (int64_t)l : -(int64_t)l) - 1;
  if (l > 0) return !poss[a] ? 0 : (cert[a] ? 2 : 1);
  return cert[a] ? 0 : (poss[a] ? 1 : 2);
}

// -1: the rule dies; else the number of literals it keeps.
__device__ __forceinline__ int64_t asp_rule(const int32_t* lit, uint32_t s, uint32_t e, const uint8_t* poss,
                                            const uint8_t* cert, uint64_t n_atoms, uint32_t* flags) {
  int64_t kept = 0;
  for (uint32_t k = s; k < e; k++) {
    const int32_t l = lit[k];
    const uint64_t a = (uint64_t)(l > 0 ? (int64_t)l : -(int64_t)l) - 1;
    if (l == 0 || a >= n_atoms) {
      *flags |= ST_BOUNDS;
      return -1;
    }
    const int x = asp_lit(l, poss, cert);
    if (x == 0) return -1;  // an impossible positive or a certain negative atom: the body is false
    kept += x == 1;
  }
  return kept;
}

__global__ void k_asp_count(const uint32_t* __restrict__ bstart, const int32_t* __restrict__ lit, uint64_t n_rules,
                            const uint8_t* __restrict__ poss, const uint8_t* __restrict__ cert, uint64_t n_atoms,
                            uint64_t* __restrict__ alive,
                            uint64_t* __restrict__ kept, uint32_t* status) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rules) return;
  uint32_t flags = 0;
  const uint32_t s = bstart[r], e = bstart[r + 1];
  if (e < s) flags |= ST_BOUNDS;
  const int64_t k = e < s ? -1 : asp_rule(lit, s, e, poss, cert, n_atoms, &flags);
  alive[r] = k >= 0 ? 1 : 0;
  kept[r] = k >= 0 ? (uint64_t)k : 0;
  if (flags) atomicOr(status, flags);
}

__global__ void k_asp_write(const int32_t* __restrict__ head, const uint32_t* __restrict__ bstart,
                            const int32_t* __restrict__ lit, uint64_t n_rules, const uint8_t* __restrict__ poss,
                            const uint8_t* __restrict__ cert, const uint64_t* __restrict__ alive, const uint64_t* __restrict__ rule_at,
                            const uint64_t* __restrict__ lit_at, int32_t* __restrict__ ohead,
                            uint32_t* __restrict__ ostart, int32_t* __restrict__ olit) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rules || !alive[r]) return;
  const uint64_t o = rule_at[r];
  uint64_t at = lit_at[r];
  ohead[o] = head[r];
  ostart[o] = (uint32_t)at;
  for (uint32_t k = bstart[r]; k < bstart[r + 1]; k++) {
    const int32_t l = lit[k];
    if (asp_lit(l, poss, cert) == 1) olit[at++] = l;
  }
}

inline unsigned grid_n(uint64_t n) { return (unsigned)ceil_div(n ? n : 1, NT); }

}  // namespace

AspResult asp_simplify(strata_ctx* ctx, uint64_t n_rules, const int32_t* head, const uint32_t* bstart,
                       const int32_t* lit, uint64_t n_atoms, const uint8_t* poss, const uint8_t* cert) {
  AspResult R;
  const uint64_t n_lit = n_rules ? bstart[n_rules] : 0;
  DBuf<int32_t> dh(ctx, n_rules + 1), dl(ctx, n_lit + 1);
  DBuf<uint32_t> ds(ctx, n_rules + 1);
  DBuf<uint8_t> dp(ctx, n_atoms + 1), dc(ctx, n_atoms + 1);
  if (n_rules) {
    SK_CUDA(cudaMemcpyAsync(dh.p, head, n_rules * 4, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(ds.p, bstart, (n_rules + 1) * 4, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (n_lit) SK_CUDA(cudaMemcpyAsync(dl.p, lit, n_lit * 4, cudaMemcpyHostToDevice, ctx->stream));
  if (n_atoms) {
    SK_CUDA(cudaMemcpyAsync(dp.p, poss, n_atoms, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(dc.p, cert, n_atoms, cudaMemcpyHostToDevice, ctx->stream));
  }
  DBuf<uint64_t> alive(ctx, n_rules + 1), kept(ctx, n_rules + 1), rule_at(ctx, n_rules + 1), lit_at(ctx, n_rules + 1);
  uint64_t n_out = 0, n_out_lit = 0;
  if (n_rules) {
    k_asp_count<<<grid_n(n_rules), NT, 0, ctx->stream>>>(ds.p, dl.p, n_rules, dp.p, dc.p, n_atoms, alive.p, kept.p,
                                                          ctx->d_status);
    after_launch(ctx, "k_asp_count");
    scan_u64(ctx, alive.p, n_rules, rule_at.p, false, &n_out);
    scan_u64(ctx, kept.p, n_rules, lit_at.p, false, &n_out_lit);
    sync_and_check(ctx);  // a literal naming no atom: STRATA_E_CUDA (bounds) before anything is written
  }
  DBuf<int32_t> oh(ctx, n_out + 1), ol(ctx, n_out_lit + 1);
  DBuf<uint32_t> os(ctx, n_out + 1);
  if (n_out) {
    k_asp_write<<<grid_n(n_rules), NT, 0, ctx->stream>>>(dh.p, ds.p, dl.p, n_rules, dp.p, dc.p, alive.p, rule_at.p,
                                                          lit_at.p, oh.p, os.p, ol.p);
    after_launch(ctx, "k_asp_write");
  }
  R.n_rules = n_out;
  R.head = static_cast<int32_t*>(std::malloc((n_out + 1) * 4));
  R.body_start = static_cast<uint32_t*>(std::malloc((n_out + 1) * 4));
  R.body_lit = static_cast<int32_t*>(std::malloc((n_out_lit + 1) * 4));
  if (!R.head || !R.body_start || !R.body_lit) fail(STRATA_E_OOM, "host allocation failed");
  if (n_out) {
    SK_CUDA(cudaMemcpyAsync(R.head, oh.p, n_out * 4, cudaMemcpyDeviceToHost, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(R.body_start, os.p, n_out * 4, cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (n_out_lit) SK_CUDA(cudaMemcpyAsync(R.body_lit, ol.p, n_out_lit * 4, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  R.body_start[n_out] = (uint32_t)n_out_lit;
  return R;
}

}  // namespace sk
