// sk_circuit.cu — exact compilation of proof DNFs and the circuit kernels.
//
// Compilation (host, once per query): a proof DNF over signed literals
// ±(leaf+1) is normalised (contradictions dropped, absorption-minimal) and
// expanded by Shannon decomposition on the most frequent variable (ties to
// the smallest), memoising cofactors, into the decision DAG
//     Or(And(Leaf v, hi), And(NegLeaf v, lo))
// whose disjuncts are mutually exclusive, so the weighted model count is
// exact (strata-prob/src/compile.rs:30-172, circuit.rs:14-41).  Nodes are
// then levelled (a node's level is one above its highest child) and laid out
// level by level per query.
//
// Kernels (one thread block per query circuit, levels separated by block
// barriers):
//   forward  — node values: Leaf p, NegLeaf 1-p, And product, Or sum
//              (circuit.rs:43-63), each a compensated pair of FP32 values
//              (float-float: an unevaluated sum hi + lo, kept exact to about
//              2^-44 relative by the error-free TwoSum and FMA-based
//              TwoProduct transformations, Dekker 1971 / Knuth TAOCP 4.2.2);
//              the root's own sum/product is formed in FP64 from its
//              children's pairs;
//   adjoint  — reverse sweep from a per-query seed: And children receive
//              g · Π(siblings) (siblings' product formed without the child,
//              exact when a child is zero), Or children g, Leaf += g,
//              NegLeaf -= g (circuit.rs:68-106); node adjoints in FP32.
//              A Leaf / NegLeaf child of an And takes g times its sibling's
//              float-float value straight into its FP64 leaf gradient: the
//              leaf's gradient from a decision node is g·(hi − lo), the
//              difference of the two cofactors, and plain FP32 cofactor
//              values lose most of their digits in that difference when the
//              cofactors are close.  Every other term of a gradient is
//              non-negative for the monotone proof DNFs here, so the FP32
//              adjoints add no cancellation of their own.
// A vector-Jacobian product (seeds = dL/dP per query, one leaf-gradient
// vector) serves torch.autograd; per-query gradient rows serve `?grad`.
#include "sk_ops.cuh"
#include "sk_prims.cuh"
#include "sk_rel.cuh"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <exception>
#include <map>
#include <thread>
#include <unordered_map>
#include <vector>


namespace sk {
namespace {

using Lits = std::vector<int64_t>;
using Dnf = std::vector<Lits>;  // sorted, absorption-minimal, ordered

inline bool subset_of(const Lits& a, const Lits& b) { return std::includes(b.begin(), b.end(), a.begin(), a.end()); }

struct DnfHash {
  size_t operator()(const std::vector<std::vector<int64_t>>& d) const {
    uint64_t h = 0x9e3779b97f4a7c15ull ^ d.size();
    for (auto& p : d) {
      h = (h ^ (0x100000001b3ull * p.size())) * 0xbf58476d1ce4e5b9ull;
      for (auto l : p) h = (h ^ (uint64_t)l) * 0x94d049bb133111ebull;
    }
    return (size_t)(h ^ (h >> 31));
  }
};

struct HNode {
  uint8_t kind;
  uint32_t leaf;
  std::vector<uint32_t> ch;
};

struct Compiler {
  std::vector<HNode> nodes;
  std::unordered_map<Dnf, uint32_t, DnfHash> memo;
  uint64_t max_nodes;
  uint32_t num_leaves = 0;

  uint32_t push(HNode n) {
    nodes.push_back(std::move(n));
    return (uint32_t)(nodes.size() - 1);
  }

  static Dnf normalize(std::vector<Lits> proofs) {
    std::vector<Lits> sets;
    for (auto& p : proofs) {
      std::sort(p.begin(), p.end());
      p.erase(std::unique(p.begin(), p.end()), p.end());
      bool contra = false;
      for (auto l : p)
        if (std::binary_search(p.begin(), p.end(), -l)) contra = true;
      if (!contra) sets.push_back(p);
    }
    std::stable_sort(sets.begin(), sets.end(), [](const Lits& x, const Lits& y) { return x.size() < y.size(); });
    std::vector<Lits> keep;
    for (auto& p : sets) {
      bool absorbed = false;
      for (auto& k : keep)
        if (subset_of(k, p)) {
          absorbed = true;
          break;
        }
      if (!absorbed) keep.push_back(p);
    }
    std::sort(keep.begin(), keep.end());
    return keep;
  }

  static Dnf restrict_dnf(const Dnf& dnf, int64_t var, bool value) {
    const int64_t dies = value ? -var : var, gone = value ? var : -var;
    std::vector<Lits> out;  // kept ordered at the end
    for (auto& p : dnf) {
      if (std::binary_search(p.begin(), p.end(), dies)) continue;
      Lits q;
      q.reserve(p.size());
      for (auto l : p)
        if (l != gone) q.push_back(l);
      bool absorbed = false;
      for (auto& k : out)
        if (subset_of(k, q)) {
          absorbed = true;
          break;
        }
      if (absorbed) continue;
      out.erase(std::remove_if(out.begin(), out.end(), [&](const Lits& k) { return subset_of(q, k); }), out.end());
      out.push_back(std::move(q));
    }
    std::sort(out.begin(), out.end());
    return out;
  }

  uint32_t shannon(const Dnf& dnf) {
    if (nodes.size() > max_nodes)
      fail(STRATA_E_UNSUPPORTED, "a provenance circuit exceeded its node budget (exact compilation is #P-hard)");
    if (dnf.empty()) return push(HNode{5, 0, {}});
    for (auto& p : dnf)
      if (p.empty()) return push(HNode{4, 0, {}});
    auto it = memo.find(dnf);
    if (it != memo.end()) return it->second;
    std::map<int64_t, uint64_t> count;
    for (auto& p : dnf)
      for (auto l : p) count[l < 0 ? -l : l]++;
    int64_t v = 0;
    uint64_t best = 0;
    for (auto& kv : count)
      if (kv.second > best) {
        best = kv.second;
        v = kv.first;
      }
    const Dnf hi = restrict_dnf(dnf, v, true), lo = restrict_dnf(dnf, v, false);
    const uint32_t hi_n = shannon(hi);
    const uint32_t lo_n = shannon(lo);
    const uint32_t leaf = (uint32_t)(v - 1);
    num_leaves = std::max(num_leaves, leaf + 1);
    const uint32_t pos = push(HNode{0, leaf, {}});
    const uint32_t neg = push(HNode{1, leaf, {}});
    const uint32_t and_hi = push(HNode{2, 0, {pos, hi_n}});
    const uint32_t and_lo = push(HNode{2, 0, {neg, lo_n}});
    const uint32_t node = push(HNode{3, 0, {and_hi, and_lo}});
    memo.emplace(dnf, node);
    return node;
  }
};

constexpr int CK_NT = 256;

// ---- float-float arithmetic (a value is the unevaluated sum hi + lo) -------
struct ff {
  float hi, lo;
};
// Knuth's TwoSum: s + e == a + b exactly.
__device__ __forceinline__ ff ff_two_sum(float a, float b) {
  const float s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  const float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return ff{s, e};
}
// Dekker's FastTwoSum (|a| >= |b|): s + e == a + b exactly.
__device__ __forceinline__ ff ff_fast_two_sum(float a, float b) {
  const float s = __fadd_rn(a, b);
  return ff{s, __fsub_rn(b, __fsub_rn(s, a))};
}
__device__ __forceinline__ ff ff_add(ff x, ff y) {
  ff s = ff_two_sum(x.hi, y.hi);
  const float e = __fadd_rn(s.lo, __fadd_rn(x.lo, y.lo));
  return ff_fast_two_sum(s.hi, e);
}
// TwoProduct with an FMA: p + e == a * b exactly.
__device__ __forceinline__ ff ff_mul(ff x, ff y) {
  const float p = __fmul_rn(x.hi, y.hi);
  const float e = __fmaf_rn(x.hi, y.hi, -p);
  const float t = __fadd_rn(e, __fadd_rn(__fmul_rn(x.hi, y.lo), __fmul_rn(x.lo, y.hi)));
  return ff_fast_two_sum(p, t);
}
__device__ __forceinline__ ff ff_load(const strata_circuits& c, uint64_t i) { return ff{c.val[i], c.val_lo[i]}; }
__device__ __forceinline__ double ff_to_f64(ff x) { return (double)x.hi + (double)x.lo; }

__global__ void __launch_bounds__(CK_NT) k_circuit_forward(strata_circuits c, const float* __restrict__ p,
                                                           float* out32, double* out64) {
  const uint32_t q = blockIdx.x;
  const uint64_t n0 = c.qnode[q];
  const uint64_t l0 = c.qlevel[q], l1 = c.qlevel[q + 1];
  for (uint64_t L = l0; L + 1 < l1; L++) {
    const uint64_t a = n0 + c.lvl[L], b = n0 + c.lvl[L + 1];
    for (uint64_t i = a + threadIdx.x; i < b; i += CK_NT) {
      const uint8_t kd = c.kind[i];
      ff x;
      if (kd == 0) {
        x = ff{p[c.a[i]], 0.0f};
      } else if (kd == 1) {
        x = ff_two_sum(1.0f, -p[c.a[i]]);  // 1 - p, exactly
      } else if (kd == 2) {
        x = ff{1.0f, 0.0f};
        for (uint32_t j = 0; j < c.b[i]; j++) x = ff_mul(x, ff_load(c, c.ch[c.a[i] + j]));
      } else if (kd == 3) {
        x = ff{0.0f, 0.0f};
        for (uint32_t j = 0; j < c.b[i]; j++) x = ff_add(x, ff_load(c, c.ch[c.a[i] + j]));
      } else {
        x = ff{kd == 4 ? 1.0f : 0.0f, 0.0f};
      }
      c.val[i] = x.hi;
      c.val_lo[i] = x.lo;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const uint32_t r = c.root[q];
    const uint8_t kd = c.kind[r];
    double x = ff_to_f64(ff_load(c, r));
    if (kd == 2) {
      x = 1.0;
      for (uint32_t j = 0; j < c.b[r]; j++) x = x * ff_to_f64(ff_load(c, c.ch[c.a[r] + j]));
    } else if (kd == 3) {
      x = 0.0;
      for (uint32_t j = 0; j < c.b[r]; j++) x = x + ff_to_f64(ff_load(c, c.ch[c.a[r] + j]));
    }
    if (out32) out32[q] = (float)x;
    if (out64) out64[q] = x;
  }
}

// Reverse sweep; leaf gradients go to grad + (per_query ? q * n_leaves : 0).
__global__ void __launch_bounds__(CK_NT) k_circuit_adjoint(strata_circuits c, const float* __restrict__ seed,
                                                           double* grad, int per_query) {
  const uint32_t q = blockIdx.x;
  const uint64_t n0 = c.qnode[q], n1 = c.qnode[q + 1];
  const uint64_t l0 = c.qlevel[q], l1 = c.qlevel[q + 1];
  double* g_out = grad + (per_query ? (uint64_t)q * c.n_leaves : 0);
  const float s = seed ? seed[q] : 1.0f;
  for (uint64_t i = n0 + threadIdx.x; i < n1; i += CK_NT) c.adj[i] = 0.0f;
  __syncthreads();
  if (threadIdx.x == 0) c.adj[c.root[q]] = s;
  __syncthreads();
  for (uint64_t L = l1 - 1; L > l0; L--) {
    const uint64_t a = n0 + c.lvl[L - 1], b = n0 + c.lvl[L];
    for (uint64_t i = a + threadIdx.x; i < b; i += CK_NT) {
      const float gi = c.adj[i];
      if (gi == 0.0f) continue;
      const uint8_t kd = c.kind[i];
      if (kd == 0) {
        atomicAdd(&g_out[c.a[i]], (double)gi);
      } else if (kd == 1) {
        atomicAdd(&g_out[c.a[i]], -(double)gi);
      } else if (kd == 2) {
        const uint32_t f = c.a[i], nc = c.b[i];
        for (uint32_t j = 0; j < nc; j++) {
          const uint32_t cj = c.ch[f + j];
          const uint8_t kj = c.kind[cj];
          if (kj == 0 || kj == 1) {
            // a leaf child: its gradient term in FP64 from the siblings'
            // float-float product (no FP32 rounding before the cofactor
            // difference forms in the leaf's sum)
            ff sib{1.0f, 0.0f};
            for (uint32_t k = 0; k < nc; k++)
              if (k != j) sib = ff_mul(sib, ff_load(c, c.ch[f + k]));
            const double t = (double)gi * ff_to_f64(sib);
            atomicAdd(&g_out[c.a[cj]], kj == 0 ? t : -t);
          } else {
            float sib = 1.0f;
            for (uint32_t k = 0; k < nc; k++)
              if (k != j) sib = sib * c.val[c.ch[f + k]];
            atomicAdd(&c.adj[cj], gi * sib);
          }
        }
      } else if (kd == 3) {
        const uint32_t f = c.a[i], nc = c.b[i];
        for (uint32_t j = 0; j < nc; j++) atomicAdd(&c.adj[c.ch[f + j]], gi);
      }
    }
    __syncthreads();
  }
}

__global__ void k_f64_to_f32(const double* a, float* b, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

template <class T>
T* dev_upload(strata_ctx* ctx, const std::vector<T>& h) {
  T* d = static_cast<T*>(dev_alloc(ctx, std::max<size_t>(1, h.size()) * sizeof(T)));
  if (!h.empty()) check_cuda(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream),
                             "cudaMemcpyAsync");
  return d;
}

}  // namespace

// One query's circuit, levelled, with query-local node indices.
struct QCircuit {
  std::vector<uint8_t> kind;
  std::vector<uint32_t> A, B, CH, lvl;
  uint32_t root = 0, levels = 0;
};

static void compile_query(const uint64_t* proof_off, const uint64_t* lit_off, const int64_t* lits, uint32_t q,
                          uint32_t n_leaves, uint64_t max_nodes, QCircuit& out) {
  std::vector<Lits> proofs;
  for (uint64_t pi = proof_off[q]; pi < proof_off[q + 1]; pi++) {
    Lits p(lits + lit_off[pi], lits + lit_off[pi + 1]);
    for (auto l : p)
      if (l == 0 || (uint64_t)(l < 0 ? -l : l) > n_leaves)
        fail(STRATA_E_INVALID, "a literal is 0 or names a leaf beyond n_leaves");
    proofs.push_back(std::move(p));
  }
  Compiler cp;
  cp.max_nodes = max_nodes;
  const uint32_t r = cp.shannon(Compiler::normalize(proofs));
  const uint32_t nn = (uint32_t)cp.nodes.size();
  std::vector<uint32_t> level(nn, 0);
  uint32_t top = 0;
  for (uint32_t i = 0; i < nn; i++) {
    uint32_t lv = 0;
    for (auto c : cp.nodes[i].ch) lv = std::max(lv, level[c] + 1);
    level[i] = lv;
    top = std::max(top, lv);
  }
  // counting sort by level (stable)
  std::vector<uint32_t> start(top + 2, 0), pos(nn);
  for (uint32_t i = 0; i < nn; i++) start[level[i] + 1]++;
  for (uint32_t L = 0; L <= top; L++) start[L + 1] += start[L];
  out.lvl.assign(start.begin(), start.end());
  {
    std::vector<uint32_t> fill(start.begin(), start.end() - 1);
    for (uint32_t i = 0; i < nn; i++) pos[i] = fill[level[i]]++;
  }
  std::vector<uint32_t> order(nn);
  for (uint32_t i = 0; i < nn; i++) order[pos[i]] = i;
  out.kind.resize(nn);
  out.A.resize(nn);
  out.B.resize(nn);
  for (uint32_t j = 0; j < nn; j++) {
    const HNode& h = cp.nodes[order[j]];
    out.kind[j] = h.kind;
    if (h.kind <= 1) {
      out.A[j] = h.leaf;
      out.B[j] = 0;
    } else {
      out.A[j] = (uint32_t)out.CH.size();
      out.B[j] = (uint32_t)h.ch.size();
      for (auto c : h.ch) out.CH.push_back(pos[c]);
    }
  }
  out.root = pos[r];
  out.levels = top + 1;
}

// Host part of the compilation: every query's levelled circuit, queries in
// parallel on the host threads (no device work; safe beside other calls).
void circuits_compile_host(uint32_t nq, const uint64_t* proof_off, const uint64_t* lit_off, const int64_t* lits,
                           uint32_t n_leaves, uint64_t max_nodes, std::vector<QCircuit>& qc) {
  qc.assign(nq, QCircuit{});
  const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  const unsigned T = std::min<unsigned>(hw, std::max<uint32_t>(1, nq));
  std::atomic<uint32_t> next{0};
  std::vector<std::exception_ptr> errs(T);
  std::vector<std::thread> th;
  for (unsigned t = 0; t < T; t++)
    th.emplace_back([&, t]() {
      try {
        while (true) {
          const uint32_t q = next.fetch_add(1);
          if (q >= nq) break;
          compile_query(proof_off, lit_off, lits, q, n_leaves, max_nodes, qc[q]);
        }
      } catch (...) {
        errs[t] = std::current_exception();
        next.store(nq);
      }
    });
  for (auto& x : th) x.join();
  for (auto& e : errs)
    if (e) std::rethrow_exception(e);
}

// Device part: concatenate host-compiled query circuits (parts in order) into
// one levelled DAG on the device.
strata_circuits* circuits_upload(strata_ctx* ctx, const std::vector<const std::vector<QCircuit>*>& parts,
                                 uint32_t n_leaves) {
  std::vector<const QCircuit*> all;
  for (auto* p : parts)
    for (auto& q : *p) all.push_back(&q);
  const uint32_t nq = (uint32_t)all.size();
  std::vector<uint64_t> qnode(nq + 1, 0), qlevel(nq + 1, 0);
  uint64_t total_ch = 0, total_lvl = 0;
  uint32_t max_levels = 0;
  for (uint32_t q = 0; q < nq; q++) {
    qnode[q + 1] = qnode[q] + all[q]->kind.size();
    qlevel[q + 1] = qlevel[q] + all[q]->lvl.size();
    total_ch += all[q]->CH.size();
    max_levels = std::max(max_levels, all[q]->levels);
  }
  total_lvl = qlevel[nq];
  if (qnode[nq] >= (1ull << 32) || total_ch >= (1ull << 32))
    fail(STRATA_E_UNSUPPORTED, "circuits limited to 2^32 nodes in total");
  std::vector<uint8_t> kind(qnode[nq]);
  std::vector<uint32_t> A(qnode[nq]), B(qnode[nq]), CH(total_ch), root(nq), lvl(total_lvl);
  uint64_t chb = 0;
  for (uint32_t q = 0; q < nq; q++) {
    const QCircuit& c = *all[q];
    const uint64_t nb = qnode[q];
    std::copy(c.kind.begin(), c.kind.end(), kind.begin() + (long)nb);
    for (size_t j = 0; j < c.kind.size(); j++) {
      A[nb + j] = c.kind[j] <= 1 ? c.A[j] : (uint32_t)(chb + c.A[j]);
      B[nb + j] = c.B[j];
    }
    for (size_t j = 0; j < c.CH.size(); j++) CH[chb + j] = (uint32_t)(nb + c.CH[j]);
    chb += c.CH.size();
    root[q] = (uint32_t)(nb + c.root);
    std::copy(c.lvl.begin(), c.lvl.end(), lvl.begin() + (long)qlevel[q]);
  }
  auto* c = new strata_circuits();
  c->n_queries = nq;
  c->n_leaves = n_leaves;
  c->n_nodes = qnode[nq];
  c->max_levels = max_levels;
  c->n_children = CH.size();
  try {
    c->kind = dev_upload(ctx, kind);
    c->a = dev_upload(ctx, A);
    c->b = dev_upload(ctx, B);
    c->ch = dev_upload(ctx, CH);
    c->qnode = dev_upload(ctx, qnode);
    c->root = dev_upload(ctx, root);
    c->qlevel = dev_upload(ctx, qlevel);
    c->lvl = dev_upload(ctx, lvl);
    c->val = static_cast<float*>(dev_alloc(ctx, std::max<uint64_t>(1, c->n_nodes) * 4));
    c->val_lo = static_cast<float*>(dev_alloc(ctx, std::max<uint64_t>(1, c->n_nodes) * 4));
    c->adj = static_cast<float*>(dev_alloc(ctx, std::max<uint64_t>(1, c->n_nodes) * 4));
    sync_and_check(ctx);
  } catch (...) {
    circuits_free(ctx, c);
    throw;
  }
  return c;
}

strata_circuits* circuits_compile(strata_ctx* ctx, uint32_t nq, const uint64_t* proof_off, const uint64_t* lit_off,
                                  const int64_t* lits, uint32_t n_leaves, uint64_t max_nodes) {
  std::vector<QCircuit> qc;
  circuits_compile_host(nq, proof_off, lit_off, lits, n_leaves, max_nodes, qc);
  return circuits_upload(ctx, {&qc}, n_leaves);
}

struct CircuitParts {
  std::vector<QCircuit> q;
};

CircuitParts* circuit_parts_compile(uint32_t nq, const uint64_t* proof_off, const uint64_t* lit_off,
                                    const int64_t* lits, uint32_t n_leaves, uint64_t max_nodes) {
  auto* cp = new CircuitParts();
  try {
    circuits_compile_host(nq, proof_off, lit_off, lits, n_leaves, max_nodes, cp->q);
  } catch (...) {
    delete cp;
    throw;
  }
  return cp;
}

void circuit_parts_free(CircuitParts* p) { delete p; }

uint32_t circuit_parts_queries(const CircuitParts* p) { return (uint32_t)p->q.size(); }

uint64_t circuit_parts_nodes(const CircuitParts* p, uint32_t* max_levels) {
  uint64_t n = 0;
  uint32_t lv = 0;
  for (auto& q : p->q) {
    n += q.kind.size();
    lv = std::max(lv, q.levels);
  }
  if (max_levels) *max_levels = lv;
  return n;
}

// FP64 evaluation of the host-compiled circuits (node order = a valid
// topological order; And/Or fold their children in stored order), used to
// check the compiler on machines without a GPU.
void circuit_parts_eval64(const CircuitParts* p, const double* prob, double* out) {
  for (size_t q = 0; q < p->q.size(); q++) {
    const QCircuit& c = p->q[q];
    std::vector<double> val(c.kind.size(), 0.0);
    for (size_t i = 0; i < c.kind.size(); i++) {
      const uint8_t k = c.kind[i];
      if (k == 0) val[i] = prob[c.A[i]];
      else if (k == 1) val[i] = 1.0 - prob[c.A[i]];
      else if (k == 2) {
        double a = 1.0;
        for (uint32_t j = 0; j < c.B[i]; j++) a = a * val[c.CH[c.A[i] + j]];
        val[i] = a;
      } else if (k == 3) {
        double a = 0.0;
        for (uint32_t j = 0; j < c.B[i]; j++) a = a + val[c.CH[c.A[i] + j]];
        val[i] = a;
      } else {
        val[i] = k == 4 ? 1.0 : 0.0;
      }
    }
    out[q] = c.kind.empty() ? 0.0 : val[c.root];
  }
}

strata_circuits* circuit_parts_upload(strata_ctx* ctx, uint32_t n_parts, CircuitParts* const* parts,
                                      uint32_t n_leaves) {
  std::vector<const std::vector<QCircuit>*> v;
  for (uint32_t i = 0; i < n_parts; i++) v.push_back(&parts[i]->q);
  return circuits_upload(ctx, v, n_leaves);
}

void circuits_free(strata_ctx* ctx, strata_circuits* c) {
  if (!c) return;
  for (void* p : {(void*)c->kind, (void*)c->a, (void*)c->b, (void*)c->ch, (void*)c->qnode, (void*)c->root,
                  (void*)c->qlevel, (void*)c->lvl, (void*)c->val, (void*)c->val_lo, (void*)c->adj})
    if (p) dev_free(ctx, p);
  delete c;
}

void circuits_forward(strata_ctx* ctx, const strata_circuits* c, const float* d_p, float* out32, double* out64) {
  if (!c->n_queries) return;
  const int kh = kprof_begin(ctx, K_CIRCUIT);
  k_circuit_forward<<<c->n_queries, CK_NT, 0, ctx->stream>>>(*c, d_p, out32, out64);
  kprof_end(ctx, kh, c->n_nodes * (1 + 4 + 4 + 4) + c->n_children * 8);
  after_launch(ctx, "k_circuit_forward");
}

// seed null = 1 per query.  per_query: grad is [n_queries][n_leaves] FP64,
// else one FP64 vector of n_leaves; both are zeroed here.  grad32 (optional)
// receives the FP32 copy of the vector form.
void circuits_adjoint(strata_ctx* ctx, const strata_circuits* c, const float* d_p, const float* seed, double* grad,
                      int per_query, float* grad32) {
  const uint64_t n = per_query ? (uint64_t)c->n_queries * c->n_leaves : c->n_leaves;
  SK_CUDA(cudaMemsetAsync(grad, 0, std::max<uint64_t>(n, 1) * 8, ctx->stream));
  if (c->n_queries) {
    k_circuit_forward<<<c->n_queries, CK_NT, 0, ctx->stream>>>(*c, d_p, nullptr, nullptr);
    after_launch(ctx, "k_circuit_forward");
    const int kh = kprof_begin(ctx, K_CIRCUIT);
    k_circuit_adjoint<<<c->n_queries, CK_NT, 0, ctx->stream>>>(*c, seed, grad, per_query);
    kprof_end(ctx, kh, c->n_nodes * (1 + 4 + 4 + 4 + 4) + c->n_children * 12);
    after_launch(ctx, "k_circuit_adjoint");
  }
  if (grad32 && !per_query && n) {
    k_f64_to_f32<<<(unsigned)ceil_div(n, 256), 256, 0, ctx->stream>>>(grad, grad32, n);
    after_launch(ctx, "k_f64_to_f32");
  }
}

}  // namespace sk
