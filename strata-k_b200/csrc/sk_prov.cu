// sk_prov.cu — Prov_k provenance capture for the reachability program
//
//     path(X,Y) :- edge(X,Y).        path(X,Z) :- edge(X,Y), path(Y,Z).
//
// with every edge a probabilistic fact (edge i carries the proof {i+1}) and
// path annotated Prov_k(k), k <= 8.  It follows the reference's capture
// (strata-eval/src/provenance.rs:286-362) exactly: naive Jacobi rounds; each
// round every derivation is re-derived from the previous round's relation;
// the derived batches of a tuple are applied in the reference's order — the
// rule-1 batch, then one rule-2 batch per edge (X, Y) in ascending (X, Y)
// order — each with insert_minimal (absorption, provenance.rs:136-143) and
// then pruned to the k best proofs by (weight desc, literals asc)
// (prune_top_k, :195-212), the weight being the product of the literal
// probabilities in ascending literal order in FP64 (proof_weight, :179-192).
// Rounds continue until no tuple changes.
//
// Only the queried targets are evaluated: path(., t) depends only on
// path(., t) and edge, so restricting the saturation to the targets of the
// query pairs yields the same proof sets for the queried tuples.  Targets
// are processed in memory-bounded waves; a target none of whose tuples
// changed in a round is final (both state buffers then hold it) and is
// skipped from then on.  Within a live target, a tuple that did not change
// in the previous round and none of whose inputs did is skipped for the
// round: under the Jacobi schedule its derivation would repeat the previous
// one exactly, and the buffer being written already holds its set.
//
// Mapping: a half-warp (16 lanes, its own shuffle group) owns one tuple
// (target, X).  Lanes 0..7 hold the current proof set S, lanes 8..15 the
// candidates of the batch being applied; each lane keeps its proof's sorted
// literals in shared memory (double-buffered for the compaction), a 64-bit
// signature for quick subset rejection, the length and the FP64 weight.
#include "sk_ops.cuh"
#include "sk_prims.cuh"
#include "sk_rel.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

namespace sk {
namespace {

constexpr int PV_NT = 128;  // 8 half-warps (tuples in flight) per block
constexpr uint32_t PV_KMAX = 8;
constexpr uint32_t PV_LMAX = 32;

struct ProofRec {
  uint32_t lit[PV_LMAX];
  double w;
  uint64_t sig;
  uint32_t len;
  uint32_t pad;
};

__device__ __forceinline__ uint64_t lit_sig(uint32_t l) { return 1ull << ((l * 0x9E3779B1u) >> 26); }

// a ⊆ b over sorted lists
__device__ __forceinline__ bool sub_list(const uint32_t* a, uint32_t la, const uint32_t* b, uint32_t lb) {
  uint32_t i = 0, j = 0;
  while (i < la) {
    if (lb - j < la - i) return false;
    const uint32_t x = a[i], y = b[j];
    if (x == y) {
      i++;
      j++;
    } else if (x > y) {
      j++;
    } else {
      return false;
    }
  }
  return true;
}

// a < b in the order of ordered sets (element-wise, a proper prefix first)
__device__ __forceinline__ bool lex_less(const uint32_t* a, uint32_t la, const uint32_t* b, uint32_t lb) {
  const uint32_t n = la < lb ? la : lb;
  for (uint32_t i = 0; i < n; i++)
    if (a[i] != b[i]) return a[i] < b[i];
  return la < lb;
}

struct PvView {
  uint32_t n;              // nodes
  const uint32_t* off;     // out-CSR over X, neighbours sorted by Y
  const uint32_t* nbr;     // Y
  const uint32_t* eid;     // edge fact index i (literal i + 1)
  const double* prob;      // probability of edge fact i
  const uint32_t* tgt;     // targets of the wave
  uint32_t n_tgt;
  uint32_t k;
  const uint8_t* cnt_prev; // [τ * n + X]
  const ProofRec* rec_prev;// [(τ * n + X) * KMAX + j]
  uint8_t* cnt_next;
  ProofRec* rec_next;
  const uint32_t* live;    // [τ] target still changing
  uint32_t* changed;       // [τ] a tuple of τ changed this round
  uint32_t* status;
  uint32_t* last;          // [τ * n + X] last round in which (τ, X) changed (0: never)
  uint32_t round;          // this round, 1-based
};

__global__ void __launch_bounds__(PV_NT) k_prov_round(PvView v) {
  __shared__ uint32_t s_lists[PV_NT / 16][2][16][PV_LMAX];
  const int lane = threadIdx.x & 31;
  const int hw = threadIdx.x >> 4;    // half-warp in the block
  const int hl = lane & 15;           // lane in the half-warp
  const int hbase = lane & 16;
  const unsigned hmask = 0xffffu << hbase;
  const uint64_t pairs = (uint64_t)v.n_tgt * v.n;
  const uint64_t stride = (uint64_t)gridDim.x * (PV_NT / 16);
  uint32_t flags = 0;
  for (uint64_t pair = (uint64_t)blockIdx.x * (PV_NT / 16) + hw; pair < pairs; pair += stride) {
    const uint32_t tau = (uint32_t)(pair / v.n);
    const uint32_t X = (uint32_t)(pair - (uint64_t)tau * v.n);
    if (!v.live[tau]) continue;  // uniform per half-warp
    // A tuple none of whose inputs — itself and path(Y, t) for its edges
    // (X, Y); the rule-1 edge never changes — changed in the previous round
    // re-derives exactly what it derived then, and its slot in the buffer
    // being written still holds that set (it did not change either): skip
    // it.  A stamp read while another half-warp raises it to this round is
    // >= round - 1 and only makes the test conservative.
    if (v.round >= 2) {
      const uint32_t lim = v.round - 1;
      bool hot = hl == 0 && v.last[pair] >= lim;
      for (uint32_t e = v.off[X] + hl; e < v.off[X + 1]; e += 16) {
        const uint32_t y = v.nbr[e];
        if (y < v.n && v.last[(uint64_t)tau * v.n + y] >= lim) hot = true;
      }
      if ((__ballot_sync(hmask, hot) & hmask) == 0u) continue;
    }
    const uint32_t t = v.tgt[tau];
    int bank = 0;
    uint32_t s_cnt = v.cnt_prev[pair];
    bool valid = false;
    uint32_t len = 0;
    uint64_t sig = 0;
    double w = 0.0;
    if (hl < (int)s_cnt) {
      const ProofRec& r = v.rec_prev[pair * PV_KMAX + hl];
      len = r.len;
      sig = r.sig;
      w = r.w;
      for (uint32_t q = 0; q < len; q++) s_lists[hw][0][hl][q] = r.lit[q];
      valid = true;
    }
    bool changed = false;
    const uint32_t e0 = v.off[X], e1 = v.off[X + 1];
    for (uint32_t en = 0; en <= e1 - e0; en++) {
      // ---- the batch of this entry (uniform per half-warp)
      uint32_t b_cnt = 0, lit_e = 0, y = 0;
      if (en == 0) {
        uint32_t lo = e0, hi = e1;  // rule 1: is (X, t) an edge?
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (v.nbr[mid] < t) lo = mid + 1; else hi = mid;
        }
        if (lo < e1 && v.nbr[lo] == t) {
          b_cnt = 1;
          lit_e = v.eid[lo] + 1;
        }
      } else {
        const uint32_t q = e0 + en - 1;
        y = v.nbr[q];
        lit_e = v.eid[q] + 1;
        b_cnt = y < v.n ? v.cnt_prev[(uint64_t)tau * v.n + y] : 0;
      }
      if (b_cnt == 0) continue;
      uint32_t* Lc = s_lists[hw][bank][hl];
      // ---- candidates {e} ∪ P_j into lanes 8..15
      if (hl >= 8) {
        valid = false;
        const uint32_t j = (uint32_t)hl - 8;
        if (j < b_cnt) {
          if (en == 0) {
            Lc[0] = lit_e;
            len = 1;
            sig = lit_sig(lit_e);
            w = 1.0 * v.prob[lit_e - 1];
            valid = true;
          } else {
            const ProofRec& r = v.rec_prev[((uint64_t)tau * v.n + y) * PV_KMAX + j];
            const uint32_t pl = r.len;
            uint32_t o = 0;
            bool placed = false;
            for (uint32_t q = 0; q < pl; q++) {
              const uint32_t l = r.lit[q];
              if (!placed && lit_e <= l) {
                if (lit_e != l) {
                  if (o < PV_LMAX) Lc[o] = lit_e;
                  o++;
                }
                placed = true;
              }
              if (o < PV_LMAX) Lc[o] = l;
              o++;
            }
            if (!placed) {
              if (o < PV_LMAX) Lc[o] = lit_e;
              o++;
            }
            if (o > PV_LMAX) {
              flags |= ST_PROOF_LEN;
            } else {
              len = o;
              sig = r.sig | lit_sig(lit_e);
              double ww = 1.0;
              for (uint32_t q = 0; q < len; q++) ww = ww * v.prob[Lc[q] - 1];
              w = ww;
              valid = true;
            }
          }
        }
      }
      __syncwarp(hmask);
      // ---- subset matrix: bit y of subof = proof(y) ⊆ proof(me); eqof = equal
      // (only the valid lanes are visited: the set bits of the half-warp's
      // ballot, the same on all its lanes)
      uint32_t subof = 0, eqof = 0;
      const uint32_t vmask = (__ballot_sync(hmask, valid) >> hbase) & 0xffffu;
      for (uint32_t vm = vmask; vm; vm &= vm - 1) {
        const int yl = __ffs(vm) - 1;
        const uint32_t ly = __shfl_sync(hmask, len, yl, 16);
        const uint64_t sy = __shfl_sync(hmask, sig, yl, 16);
        if (valid && yl != hl && ly <= len && (sy & ~sig) == 0 &&
            sub_list(s_lists[hw][bank][yl], ly, Lc, len)) {
          subof |= 1u << yl;
          if (ly == len) eqof |= 1u << yl;
        }
      }
      // ---- insert_minimal of the batch: within-batch minimal (equal sets
      // keep the lowest lane), then rejected by any S proof it contains
      bool accepted = false;
      if (valid && hl >= 8) {
        const uint32_t below = (1u << hl) - 1u;
        const bool dom = ((subof & ~eqof) & 0xff00u) != 0u || (eqof & 0xff00u & below) != 0u;
        const bool rej = (subof & 0x00ffu) != 0u;
        accepted = !dom && !rej;
      }
      const uint32_t acc = (__ballot_sync(hmask, accepted) >> hbase) & 0xffffu;
      const uint32_t s_mask = (1u << s_cnt) - 1u;
      // S proofs absorbed by an accepted candidate (strictly: equal ones were rejected)
      const bool removed = hl < 8 && valid && (subof & acc) != 0u;
      const bool surv = (hl < 8 && valid && !removed) || accepted;
      const uint32_t sv = (__ballot_sync(hmask, surv) >> hbase) & 0xffffu;
      uint32_t keep = acc ? sv : s_mask;
      const uint32_t ns = __popc(sv);
      if (acc && ns > v.k) {
        // prune_top_k: rank by (weight desc, literals asc)
        uint32_t rank = 0;
        for (uint32_t vm = sv; vm; vm &= vm - 1) {
          const int yl = __ffs(vm) - 1;
          const double wy = __shfl_sync(hmask, w, yl, 16);
          const uint32_t ly = __shfl_sync(hmask, len, yl, 16);
          if (!surv || yl == hl) continue;
          if (wy > w || (wy == w && lex_less(s_lists[hw][bank][yl], ly, Lc, len))) rank++;
        }
        keep = (__ballot_sync(hmask, surv && rank < v.k) >> hbase) & 0xffffu;
      }
      if (keep == s_mask) {  // S unchanged: drop the candidates
        if (hl >= 8) {
          valid = false;
          len = 0;
          sig = 0;
          w = 0.0;
        }
        __syncwarp(hmask);
        continue;
      }
      changed = true;
      // ---- compaction: survivor d moves to lane d, lists to the other bank
      const uint32_t cnt = __popc(keep);
      const int src = hl < (int)cnt ? (int)(__fns(keep, 0, hl + 1)) : hl;
      const uint32_t nlen = __shfl_sync(hmask, len, src & 15, 16);
      const uint64_t nsig = __shfl_sync(hmask, sig, src & 15, 16);
      const double nw = __shfl_sync(hmask, w, src & 15, 16);
      __syncwarp(hmask);
      if (hl < (int)cnt) {
        const uint32_t* from = s_lists[hw][bank][src & 15];
        uint32_t* to = s_lists[hw][bank ^ 1][hl];
        for (uint32_t q = 0; q < nlen; q++) to[q] = from[q];
      }
      __syncwarp(hmask);
      bank ^= 1;
      s_cnt = cnt;
      valid = hl < (int)cnt;
      len = valid ? nlen : 0;
      sig = valid ? nsig : 0;
      w = valid ? nw : 0.0;
    }
    // ---- write the tuple's new proof set
    if (hl == 0) v.cnt_next[pair] = (uint8_t)s_cnt;
    if (hl < (int)s_cnt) {
      ProofRec* r = &v.rec_next[pair * PV_KMAX + hl];
      const uint32_t* from = s_lists[hw][bank][hl];
      for (uint32_t q = 0; q < len; q++) r->lit[q] = from[q];
      r->len = len;
      r->sig = sig;
      r->w = w;
    }
    if (changed && hl == 0) {
      atomicOr(&v.changed[tau], 1u);
      v.last[pair] = v.round;
    }
    __syncwarp(hmask);
  }
  if (flags) atomicOr(v.status, flags);
}

// Gather the queried tuples' proof sets: query q reads (qtau[q], qs[q]).
__global__ void k_prov_gather(const uint8_t* cnt, const ProofRec* rec, uint32_t n, const uint32_t* qtau,
                              const uint32_t* qs, uint32_t nq, uint8_t* out_cnt, ProofRec* out_rec) {
  const uint32_t q = blockIdx.x;
  if (q >= nq) return;
  const uint64_t pair = (uint64_t)qtau[q] * n + qs[q];
  const uint32_t c = qs[q] < n ? cnt[pair] : 0;
  if (threadIdx.x == 0) out_cnt[q] = (uint8_t)c;
  for (uint32_t j = threadIdx.x; j < c; j += blockDim.x) out_rec[(uint64_t)q * PV_KMAX + j] = rec[pair * PV_KMAX + j];
}

__global__ void k_edge_keys(const uint32_t* src, const uint32_t* dst, uint64_t m, int b, uint64_t* keys,
                            uint32_t* idx) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  keys[i] = ((uint64_t)src[i] << b) | dst[i];
  idx[i] = (uint32_t)i;
}

__global__ void k_dup_check(const uint64_t* keys, uint64_t m, uint32_t* dup) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  if (i > 0 && keys[i] == keys[i - 1]) *dup = 1u;
}

}  // namespace

// Host driver: see strata_prov_tc_capture in include/strata_b200.h.
void prov_tc_capture(strata_ctx* ctx, uint32_t n, const uint32_t* d_src, const uint32_t* d_dst, uint64_t m,
                     const double* d_prob, uint32_t k, uint32_t nq, const uint32_t* qs, const uint32_t* qt,
                     std::vector<std::vector<std::vector<uint32_t>>>& out, std::vector<uint32_t>& rounds_out,
                     strata_prov_stats* st) {
  if (st) std::memset(st, 0, sizeof(*st));
  reset_status(ctx);
  if (k == 0 || k > PV_KMAX) fail(STRATA_E_INVALID, "Prov_k capture supports 1 <= k <= 8");
  for (uint32_t q = 0; q < nq; q++)
    if (qs[q] >= n || qt[q] >= n) fail(STRATA_E_INVALID, "a query node is outside [0, n)");
  cudaEvent_t e0, e1;
  check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
  check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
  check_cuda(cudaEventRecord(e0, ctx->stream), "cudaEventRecord");
  const uint64_t l0 = ctx->launches;
  // ---- out-CSR sorted by (X, Y), edge fact ids as values; distinct edges
  if (m && (max_u32(ctx, d_src, m) >= n || max_u32(ctx, d_dst, m) >= n))
    fail(STRATA_E_INVALID, "an edge endpoint is outside [0, n)");
  const int b = std::max(1, bits_for(n ? n - 1 : 0));
  DBuf<uint64_t> keys(ctx, m + 1), kalt(ctx, m + 1);
  DBuf<uint32_t> idx(ctx, m + 1), ialt(ctx, m + 1), nbr(ctx, m + 1), off(ctx, (uint64_t)n + 1), flag(ctx, 1);
  SK_CUDA(cudaMemsetAsync(flag.p, 0, 4, ctx->stream));
  if (m) {
    // endpoints are checked against n by the CSR build below
    k_edge_keys<<<(unsigned)ceil_div(m, 256), 256, 0, ctx->stream>>>(d_src, d_dst, m, b, keys.p, idx.p);
    after_launch(ctx, "k_edge_keys");
    uint64_t* kp = keys.p;
    uint64_t* ka = kalt.p;
    uint32_t* vp = idx.p;
    uint32_t* va = ialt.p;
    radix_sort<uint64_t, uint32_t>(ctx, &kp, &ka, &vp, &va, true, m, 2 * b, false);
    k_dup_check<<<(unsigned)ceil_div(m, 256), 256, 0, ctx->stream>>>(kp, m, flag.p);
    after_launch(ctx, "k_dup_check");
    build_csr<uint64_t>(ctx, kp, m, b, n, off.p, nbr.p);
    if (vp != idx.p) std::swap(idx, ialt);
  } else {
    SK_CUDA(cudaMemsetAsync(off.p, 0, ((uint64_t)n + 1) * 4, ctx->stream));
  }
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, flag.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  if ((uint32_t)ctx->h_scalar[0])
    fail(STRATA_E_UNSUPPORTED, "duplicate probabilistic edge facts (X, Y): each edge tuple must be one leaf");
  // ---- targets and waves
  std::vector<uint32_t> targets(qt, qt + nq);
  std::sort(targets.begin(), targets.end());
  targets.erase(std::unique(targets.begin(), targets.end()), targets.end());
  const uint64_t per_target = 2ull * n * (PV_KMAX * sizeof(ProofRec) + 1) + 4ull * n;
  release_all_cached(ctx);
  uint64_t budget = (uint64_t)((double)reusable_device_bytes(ctx) * 0.5);
  if (ctx->cap && ctx->cap > ctx->in_use) budget = std::min<uint64_t>(budget, ctx->cap - ctx->in_use);
  if (ctx->tune_bs_budget_mb > 0) budget = std::min<uint64_t>(budget, ctx->tune_bs_budget_mb << 20);
  const uint64_t tw = std::max<uint64_t>(1, std::min<uint64_t>(targets.size() ? targets.size() : 1,
                                                                budget / std::max<uint64_t>(per_target, 1)));
  if (per_target > budget) fail(STRATA_E_OOM, "one target's proof states exceed the memory budget");
  DBuf<uint8_t> cntA(ctx, tw * n + 1), cntB(ctx, tw * n + 1);
  DBuf<ProofRec> recA(ctx, tw * n * PV_KMAX + 1), recB(ctx, tw * n * PV_KMAX + 1);
  DBuf<uint32_t> d_tgt(ctx, tw), d_live(ctx, tw), d_changed(ctx, tw), d_last(ctx, tw * n + 1);
  DBuf<uint32_t> d_qtau(ctx, nq + 1), d_qs(ctx, nq + 1);
  DBuf<uint8_t> d_ocnt(ctx, nq + 1);
  DBuf<ProofRec> d_orec(ctx, (uint64_t)nq * PV_KMAX + 1);
  int per_sm = 0;
  check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_prov_round, PV_NT, 0), "occupancy");
  const unsigned grid = (unsigned)(std::max(1, per_sm) * ctx->num_sms);
  out.assign(nq, {});
  rounds_out.assign(targets.size(), 0);
  std::map<uint32_t, uint32_t> tindex;
  for (size_t i = 0; i < targets.size(); i++) tindex[targets[i]] = (uint32_t)i;
  uint64_t total_rounds = 0, waves = 0, max_len_seen = 0;
  std::vector<uint32_t> h_changed(tw), h_live(tw);
  std::vector<uint8_t> h_cnt;
  std::vector<ProofRec> h_rec;
  const int kh = kprof_begin(ctx, K_PROV_ROUND);
  for (size_t w0 = 0; w0 < targets.size(); w0 += tw) {
    const uint32_t nt = (uint32_t)std::min<uint64_t>(tw, targets.size() - w0);
    SK_CUDA(cudaMemcpyAsync(d_tgt.p, targets.data() + w0, nt * 4, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemsetAsync(cntA.p, 0, (uint64_t)nt * n, ctx->stream));
    SK_CUDA(cudaMemsetAsync(cntB.p, 0, (uint64_t)nt * n, ctx->stream));
    SK_CUDA(cudaMemsetAsync(d_last.p, 0, (uint64_t)nt * n * 4, ctx->stream));
    std::fill(h_live.begin(), h_live.end(), 1u);
    SK_CUDA(cudaMemcpyAsync(d_live.p, h_live.data(), nt * 4, cudaMemcpyHostToDevice, ctx->stream));
    PvView v{n, off.p, nbr.p, idx.p, d_prob, d_tgt.p, nt, k, cntA.p, recA.p, cntB.p, recB.p,
             d_live.p, d_changed.p, ctx->d_status, d_last.p, 0};
    bool a_is_prev = true;
    uint32_t live_count = nt;
    uint32_t r = 0;
    while (live_count) {
      r++;
      v.round = r;
      v.cnt_prev = a_is_prev ? cntA.p : cntB.p;
      v.rec_prev = a_is_prev ? recA.p : recB.p;
      v.cnt_next = a_is_prev ? cntB.p : cntA.p;
      v.rec_next = a_is_prev ? recB.p : recA.p;
      SK_CUDA(cudaMemsetAsync(d_changed.p, 0, nt * 4, ctx->stream));
      k_prov_round<<<grid, PV_NT, 0, ctx->stream>>>(v);
      after_launch(ctx, "k_prov_round");
      SK_CUDA(cudaMemcpyAsync(h_changed.data(), d_changed.p, nt * 4, cudaMemcpyDeviceToHost, ctx->stream));
      sync_and_check(ctx);
      live_count = 0;
      for (uint32_t i = 0; i < nt; i++) {
        if (h_live[i] && !h_changed[i]) rounds_out[w0 + i] = r;  // converged this round
        h_live[i] = h_live[i] && h_changed[i];
        live_count += h_live[i];
      }
      SK_CUDA(cudaMemcpyAsync(d_live.p, h_live.data(), nt * 4, cudaMemcpyHostToDevice, ctx->stream));
      a_is_prev = !a_is_prev;
    }
    total_rounds = std::max<uint64_t>(total_rounds, r);
    // ---- the wave's queries
    std::vector<uint32_t> qi, qtau, qsv;
    for (uint32_t q = 0; q < nq; q++) {
      auto it = tindex.find(qt[q]);
      if (it->second >= w0 && it->second < w0 + nt) {
        qi.push_back(q);
        qtau.push_back(it->second - (uint32_t)w0);
        qsv.push_back(qs[q]);
      }
    }
    if (!qi.empty()) {
      const uint32_t nw = (uint32_t)qi.size();
      SK_CUDA(cudaMemcpyAsync(d_qtau.p, qtau.data(), nw * 4, cudaMemcpyHostToDevice, ctx->stream));
      SK_CUDA(cudaMemcpyAsync(d_qs.p, qsv.data(), nw * 4, cudaMemcpyHostToDevice, ctx->stream));
      // after the last swap the final state is the "prev" buffer
      const uint8_t* fc = a_is_prev ? cntA.p : cntB.p;
      const ProofRec* fr_ = a_is_prev ? recA.p : recB.p;
      k_prov_gather<<<nw, 32, 0, ctx->stream>>>(fc, fr_, n, d_qtau.p, d_qs.p, nw, d_ocnt.p, d_orec.p);
      after_launch(ctx, "k_prov_gather");
      h_cnt.resize(nw);
      h_rec.resize((size_t)nw * PV_KMAX);
      SK_CUDA(cudaMemcpyAsync(h_cnt.data(), d_ocnt.p, nw, cudaMemcpyDeviceToHost, ctx->stream));
      SK_CUDA(cudaMemcpyAsync(h_rec.data(), d_orec.p, (size_t)nw * PV_KMAX * sizeof(ProofRec),
                              cudaMemcpyDeviceToHost, ctx->stream));
      sync_and_check(ctx);
      for (uint32_t j = 0; j < nw; j++) {
        auto& ps = out[qi[j]];
        for (uint32_t s = 0; s < h_cnt[j]; s++) {
          const ProofRec& pr = h_rec[(size_t)j * PV_KMAX + s];
          ps.emplace_back(pr.lit, pr.lit + pr.len);
          max_len_seen = std::max<uint64_t>(max_len_seen, pr.len);
        }
        std::sort(ps.begin(), ps.end());  // the proof set's order
      }
    }
    waves++;
  }
  kprof_end(ctx, kh, 0);
  check_cuda(cudaEventRecord(e1, ctx->stream), "cudaEventRecord");
  sync_and_check(ctx);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  kprof_collect(ctx);
  if (st) {
    st->queries = nq;
    st->targets = targets.size();
    st->waves = waves;
    st->rounds_max = total_rounds;
    st->max_proof_len = max_len_seen;
    st->device_ms = ms;
    st->launches = ctx->launches - l0;
  }
}

}  // namespace sk
