// sk_oracle.cpp — CPU restatement of the Strata/K reference semantics.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine:
// tests/, the smoke check and bench.py's CPU baseline may load it; the
// engine never does.  It is a plain restatement of the reference algorithms,
// each function citing the reference file it follows; the reference itself
// (Rust) cannot be built in this environment.
//
// Three layers:
//   A. `interp_*`: the reference interpreter itself — Core-IR rules over
//      BTreeMap relations, the recursive nested-loop `solve`, naive and
//      semi-naive drivers, Bool/Trop annotations with checked ⊗, stratified
//      negation, aggregates.  Follows strata-eval/src/{naive,seminaive,store,
//      value}.rs and strata-ir/src/trop.rs.
//   B. `fast_*`: the same semi-naive schedule for the config rule shapes (TC,
//      Trop all-pairs, MSSP) with indexed joins — same rounds, same Δ, same
//      overflow/cap behaviour — so parity can be checked at sizes where the
//      nested loop is hopeless.  Cross-checked against layer A in the tests.
//   C. independent oracles: per-source BFS closure, Dijkstra multi-source
//      (non-negative weights), brute-force and merge-based triangle/K4 counts,
//      order-independent fingerprints (same mixing as the device's).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <iterator>
#include <optional>
#include <queue>
#include <set>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

// ===========================================================================
// A. The reference interpreter
// ===========================================================================

// GroundVal (strata-ir/src/value.rs:19-24): Sym < Int < Term, then payload.
struct GV {
  uint8_t tag;  // 0 = Sym, 1 = Int
  int64_t v;
  bool operator<(const GV& o) const { return tag != o.tag ? tag < o.tag : v < o.v; }
  bool operator==(const GV& o) const { return tag == o.tag && v == o.v; }
  bool operator!=(const GV& o) const { return !(*this == o); }
};
using Tuple = std::vector<GV>;

// Weight (strata-ir/src/trop.rs:35-40): Finite(i64) < PosInf.
struct Weight {
  bool inf;
  int64_t v;
  bool operator<(const Weight& o) const {
    if (inf != o.inf) return !inf;
    return inf ? false : v < o.v;
  }
  bool operator==(const Weight& o) const { return inf == o.inf && (inf || v == o.v); }
};

// Ann (strata-eval/src/value.rs:16-19): Unit (Bool) or W (Trop).
struct Ann {
  bool trop;
  Weight w;
};

enum Err : int {
  OK = 0,
  E_OVERFLOW = 4,        // EvalError::Overflow (naive.rs:31)
  E_NEG_CYCLE = 5,       // EvalError::NegativeWeightCycle (naive.rs:45)
  E_UNKNOWN_PRED = 10,
  E_UNSAFE_HEAD = 11,
  E_UNSAFE_NEG = 12,
  E_NEG_NOT_STRAT = 13,
  E_AGG_RECURSION = 14,
  E_MALFORMED_AGG = 15,
  E_NON_INT_AGG = 16,
  E_ANN_MISMATCH = 17,   // the reference panics (value.rs:51,60)
  E_ROUND_LIMIT = 18,    // a bounded sample stopped early (not an error of the reference)
};

struct EvalError {
  int code;
};

// Checked ⊗ (trop.rs:52-62).
inline Weight w_otimes(Weight a, Weight b) {
  if (a.inf || b.inf) return Weight{true, 0};
  int64_t r;
  if (__builtin_add_overflow(a.v, b.v, &r)) throw EvalError{E_OVERFLOW};
  return Weight{false, r};
}

inline Ann ann_otimes(Ann a, Ann b) {  // value.rs:56-62
  if (a.trop != b.trop) throw EvalError{E_ANN_MISMATCH};
  if (!a.trop) return a;
  return Ann{true, w_otimes(a.w, b.w)};
}

// ⊕ with the change flag (value.rs:43-53): min, changed iff strictly smaller.
inline Ann ann_oplus(Ann a, Ann b, bool* changed) {
  if (a.trop != b.trop) throw EvalError{E_ANN_MISMATCH};
  if (!a.trop) {
    *changed = false;
    return a;
  }
  const Weight m = b.w < a.w ? b.w : a.w;
  *changed = m < a.w;
  return Ann{true, m};
}

struct Term {
  int kind;  // 0 var(slot), 1 sym, 2 int
  int64_t v;
};
struct Atom {
  int pred;
  std::vector<Term> args;
};
struct Lit {
  bool neg;
  Atom atom;
};
struct Rule {
  int var_count;
  Atom head;
  int agg_op;   // -1 none, 0 count, 1 sum, 2 min, 3 max (AggOp, naive.rs:370-391)
  int agg_slot;
  int agg_pos;  // head position of the aggregate term
  std::vector<Lit> body;
};
struct Pred {
  int arity;
  bool trop;
  int stratum;
};
struct Relation {  // store.rs:17-49
  bool trop;
  std::map<Tuple, Ann> rows;
  bool combine(const Tuple& t, Ann a) {
    auto it = rows.find(t);
    if (it == rows.end()) {
      rows.emplace(t, a);
      return true;
    }
    bool changed;
    Ann m = ann_oplus(it->second, a, &changed);
    if (changed) it->second = m;
    return changed;
  }
};

struct Program {
  std::vector<Pred> preds;
  std::vector<Rule> rules;
  int num_strata = 0;
};

using Binding2 = std::vector<std::optional<GV>>;

struct Interp {
  const Program& P;
  std::vector<Relation> db;
  int cur_stratum = 0;
  explicit Interp(const Program& p) : P(p) {
    for (auto& pr : p.preds) db.push_back(Relation{pr.trop, {}});
  }

  static bool unify(const std::vector<Term>& args, const Tuple& t, Binding2& b) {  // naive.rs:407-455
    if (args.size() != t.size()) return false;
    for (size_t i = 0; i < args.size(); i++) {
      const Term& a = args[i];
      const GV v = t[i];
      if (a.kind == 0) {
        auto& slot = b[(size_t)a.v];
        if (slot) {
          if (*slot != v) return false;
        } else {
          slot = v;
        }
      } else if (a.kind == 1) {
        if (!(v == GV{0, a.v})) return false;
      } else {
        if (!(v == GV{1, a.v})) return false;
      }
    }
    return true;
  }

  static Tuple ground(const std::vector<Term>& args, const Binding2& b, bool negated) {  // naive.rs:466-520
    Tuple t;
    t.reserve(args.size());
    for (auto& a : args) {
      if (a.kind == 0) {
        if (!b[(size_t)a.v]) throw EvalError{negated ? E_UNSAFE_NEG : E_UNSAFE_HEAD};
        t.push_back(*b[(size_t)a.v]);
      } else {
        t.push_back(GV{(uint8_t)(a.kind == 1 ? 0 : 1), a.v});
      }
    }
    return t;
  }

  bool negation_holds(const Atom& atom, const Binding2& b) {  // naive.rs:538-561
    if (P.preds[atom.pred].stratum >= cur_stratum) throw EvalError{E_NEG_NOT_STRAT};
    Tuple t = ground(atom.args, b, true);
    return db[atom.pred].rows.find(t) == db[atom.pred].rows.end();
  }

  // The recursive nested-loop join (seminaive.rs:215-298 / naive.rs:237-298).
  // `delta_pos` < 0: every literal scans its full relation.
  void solve(const std::vector<Lit>& body, size_t idx, Binding2& binding, Ann acc, int delta_pos,
             const std::vector<std::pair<Tuple, Ann>>* delta,
             std::vector<std::pair<Binding2, Ann>>& out) {
    if (idx == body.size()) {
      out.emplace_back(binding, acc);
      return;
    }
    const Lit& lit = body[idx];
    if (!lit.neg) {
      if ((int)idx == delta_pos) {
        for (auto& row : *delta) {
          Binding2 b = binding;
          if (unify(lit.atom.args, row.first, b)) {
            Ann na = ann_otimes(acc, row.second);
            solve(body, idx + 1, b, na, delta_pos, delta, out);
          }
        }
      } else {
        for (auto& row : db[lit.atom.pred].rows) {
          Binding2 b = binding;
          if (unify(lit.atom.args, row.first, b)) {
            Ann na = ann_otimes(acc, row.second);
            solve(body, idx + 1, b, na, delta_pos, delta, out);
          }
        }
      }
    } else {
      if (negation_holds(lit.atom, binding)) solve(body, idx + 1, binding, acc, delta_pos, delta, out);
    }
  }

  size_t universe() const {  // naive.rs:143-155
    std::set<int64_t> s;
    for (auto& r : db)
      for (auto& kv : r.rows)
        for (auto& v : kv.first)
          if (v.tag == 0) s.insert(v.v);
    return s.size();
  }

  static Ann otimes_id(bool trop) { return trop ? Ann{true, Weight{false, 0}} : Ann{false, Weight{false, 0}}; }

  void eval_aggregate(const Rule& r) {  // naive.rs:300-369
    for (auto& l : r.body)
      if (P.preds[l.atom.pred].stratum >= cur_stratum) throw EvalError{E_AGG_RECURSION};
    Binding2 b((size_t)r.var_count);
    std::vector<std::pair<Binding2, Ann>> solved;
    solve(r.body, 0, b, Ann{false, Weight{false, 0}}, -1, nullptr, solved);
    std::map<Tuple, std::vector<GV>> groups;
    for (auto& sb : solved) {
      Tuple key;
      for (size_t i = 0; i < r.head.args.size(); i++) {
        if ((int)i == r.agg_pos) continue;
        Tuple one = ground({r.head.args[i]}, sb.first, false);
        key.push_back(one[0]);
      }
      if (!sb.first[(size_t)r.agg_slot]) throw EvalError{E_UNSAFE_HEAD};
      groups[key].push_back(*sb.first[(size_t)r.agg_slot]);
    }
    for (auto& g : groups) {
      int64_t res = 0;
      const auto& vals = g.second;
      if (r.agg_op == 0) {
        res = (int64_t)vals.size();
      } else {
        std::vector<int64_t> ints;
        for (auto& v : vals) {
          if (v.tag != 1) throw EvalError{E_NON_INT_AGG};
          ints.push_back(v.v);
        }
        if (r.agg_op == 1) {
          uint64_t s = 0;
          for (auto x : ints) s += (uint64_t)x;
          res = (int64_t)s;
        } else if (r.agg_op == 2) {
          res = *std::min_element(ints.begin(), ints.end());
        } else {
          res = *std::max_element(ints.begin(), ints.end());
        }
      }
      Tuple t;
      size_t ki = 0;
      for (size_t i = 0; i < r.head.args.size(); i++) {
        if ((int)i == r.agg_pos) t.push_back(GV{1, res});
        else t.push_back(g.first[ki++]);
      }
      db[r.head.pred].combine(t, Ann{false, Weight{false, 0}});
    }
  }

  // The literal at `pos` ranges over `rows`, split across threads; each
  // thread runs the identical nested loop on its slice (same derivations).
  template <class Emit>
  void par_solve(const Rule& r, Ann id, int pos, const std::vector<std::pair<Tuple, Ann>>& rows,
                 int threads, Emit& emit) {
    const int T = std::min<int>(threads, (int)rows.size());
    std::vector<std::vector<std::pair<Tuple, Ann>>> parts(T);
    for (size_t k = 0; k < rows.size(); k++) parts[k % T].push_back(rows[k]);
    std::vector<std::vector<std::pair<Binding2, Ann>>> outs(T);
    std::vector<int> errs(T, 0);
    std::vector<std::thread> th;
    for (int q = 0; q < T; q++) {
      th.emplace_back([&, q]() {
        try {
          Binding2 b((size_t)r.var_count);
          solve(r.body, 0, b, id, pos, &parts[q], outs[q]);
        } catch (const EvalError& e) {
          errs[q] = e.code;
        }
      });
    }
    for (auto& t : th) t.join();
    for (int q = 0; q < T; q++)
      if (errs[q]) throw EvalError{errs[q]};
    for (int q = 0; q < T; q++) emit(outs[q]);
  }

  // One semi-naive round (seminaive.rs:114-210).  `idb` non-null = delta round.
  using Delta = std::vector<std::vector<std::pair<Tuple, Ann>>>;
  Delta apply_round(int stratum, const std::vector<char>* idb, const Delta* delta, int threads) {
    std::vector<std::tuple<int, Tuple, Ann>> derived;
    for (auto& r : P.rules) {
      if (P.preds[r.head.pred].stratum != stratum || r.agg_op >= 0) continue;
      const Ann id = otimes_id(P.preds[r.head.pred].trop);
      auto emit = [&](std::vector<std::pair<Binding2, Ann>>& solved) {
        for (auto& s : solved) derived.emplace_back(r.head.pred, ground(r.head.args, s.first, false), s.second);
      };
      if (!idb) {
        if (threads > 1 && !r.body.empty() && !r.body[0].neg && db[r.body[0].atom.pred].rows.size() > 1) {
          // Scanning the first literal's relation row by row is the same
          // nested loop; its rows are split across threads.
          std::vector<std::pair<Tuple, Ann>> rows(db[r.body[0].atom.pred].rows.begin(),
                                                  db[r.body[0].atom.pred].rows.end());
          par_solve(r, id, 0, rows, threads, emit);
        } else {
          std::vector<std::pair<Binding2, Ann>> solved;
          Binding2 b((size_t)r.var_count);
          solve(r.body, 0, b, id, -1, nullptr, solved);
          emit(solved);
        }
      } else {
        for (size_t i = 0; i < r.body.size(); i++) {
          const Lit& l = r.body[i];
          if (l.neg || !(*idb)[l.atom.pred]) continue;
          const auto& rows = (*delta)[l.atom.pred];
          if (rows.empty()) continue;
          if (threads <= 1 || rows.size() < 2) {
            std::vector<std::pair<Binding2, Ann>> solved;
            Binding2 b((size_t)r.var_count);
            solve(r.body, 0, b, id, (int)i, &rows, solved);
            emit(solved);
          } else {
            par_solve(r, id, (int)i, rows, threads, emit);
          }
        }
      }
    }
    std::set<std::pair<int, Tuple>> changed;
    for (auto& d : derived) {
      if (db[std::get<0>(d)].combine(std::get<1>(d), std::get<2>(d))) changed.emplace(std::get<0>(d), std::get<1>(d));
    }
    Delta next(P.preds.size());
    for (auto& c : changed) next[c.first].emplace_back(c.second, db[c.first].rows.at(c.second));
    return next;
  }

  // run_semi_naive (seminaive.rs:29-106).  max_rounds < 0: unbounded.
  int run_semi_naive(int threads, long max_rounds, long* rounds_out) {
    const size_t U = universe();
    long total_rounds = 0;
    for (int k = 0; k < P.num_strata; k++) {
      cur_stratum = k;
      bool is_trop = false;
      for (auto& r : P.rules)
        if (P.preds[r.head.pred].stratum == k && P.preds[r.head.pred].trop) is_trop = true;
      for (auto& r : P.rules)
        if (P.preds[r.head.pred].stratum == k && r.agg_op >= 0) eval_aggregate(r);
      std::vector<char> idb(P.preds.size(), 0);
      for (auto& r : P.rules)
        if (P.preds[r.head.pred].stratum == k && r.agg_op < 0) idb[r.head.pred] = 1;
      Delta delta = apply_round(k, nullptr, nullptr, threads);
      const size_t cap = U + 2;
      size_t iters = 0;
      auto nonempty = [&]() {
        for (auto& d : delta)
          if (!d.empty()) return true;
        return false;
      };
      while (nonempty()) {
        if (max_rounds >= 0 && total_rounds >= max_rounds) {
          if (rounds_out) *rounds_out = total_rounds;
          return E_ROUND_LIMIT;
        }
        delta = apply_round(k, &idb, &delta, threads);
        iters++;
        total_rounds++;
        if (is_trop && iters > cap) throw EvalError{E_NEG_CYCLE};
      }
    }
    if (rounds_out) *rounds_out = total_rounds;
    return OK;
  }

  // Naive run (naive.rs:96-233).
  int run_naive() {
    const size_t U = universe();
    for (int k = 0; k < P.num_strata; k++) {
      cur_stratum = k;
      bool is_trop = false;
      for (auto& r : P.rules)
        if (P.preds[r.head.pred].stratum == k && P.preds[r.head.pred].trop) is_trop = true;
      for (auto& r : P.rules)
        if (P.preds[r.head.pred].stratum == k && r.agg_op >= 0) eval_aggregate(r);
      const size_t cap = U + 2;
      size_t iters = 0;
      while (true) {
        std::vector<std::tuple<int, Tuple, Ann>> derived;
        for (auto& r : P.rules) {
          if (P.preds[r.head.pred].stratum != k || r.agg_op >= 0) continue;
          std::vector<std::pair<Binding2, Ann>> solved;
          Binding2 b((size_t)r.var_count);
          solve(r.body, 0, b, otimes_id(P.preds[r.head.pred].trop), -1, nullptr, solved);
          for (auto& s : solved) derived.emplace_back(r.head.pred, ground(r.head.args, s.first, false), s.second);
        }
        bool changed = false;
        for (auto& d : derived) changed |= db[std::get<0>(d)].combine(std::get<1>(d), std::get<2>(d));
        iters++;
        if (!changed) break;
        if (is_trop && iters > cap) throw EvalError{E_NEG_CYCLE};
      }
    }
    return OK;
  }
};

// Program blob decoding (layout documented in oracle.py).
struct Reader {
  const int64_t* p;
  size_t i = 0, n;
  int64_t next() {
    if (i >= n) throw EvalError{E_MALFORMED_AGG};
    return p[i++];
  }
};

Term read_term(Reader& r) {
  Term t;
  t.kind = (int)r.next();
  t.v = r.next();
  return t;
}

Atom read_atom(Reader& r) {
  Atom a;
  a.pred = (int)r.next();
  const int ar = (int)r.next();
  for (int k = 0; k < ar; k++) a.args.push_back(read_term(r));
  return a;
}

Program parse_program(Reader& R) {
  Program P;
  const int np = (int)R.next();
  for (int k = 0; k < np; k++) {
    Pred p;
    p.arity = (int)R.next();
    p.trop = R.next() != 0;
    p.stratum = (int)R.next();
    P.preds.push_back(p);
  }
  P.num_strata = (int)R.next();
  const int nr = (int)R.next();
  for (int k = 0; k < nr; k++) {
    Rule r;
    r.var_count = (int)R.next();
    r.head = read_atom(R);
    r.agg_op = (int)R.next();
    r.agg_slot = (int)R.next();
    r.agg_pos = (int)R.next();
    const int nb = (int)R.next();
    for (int q = 0; q < nb; q++) {
      Lit l;
      l.neg = R.next() != 0;
      l.atom = read_atom(R);
      r.body.push_back(l);
    }
    P.rules.push_back(r);
  }
  return P;
}

// ===========================================================================
// A'. Provenance capture (strata-eval/src/provenance.rs) and exact
//     compilation + weighted model counting (strata-prob/src/compile.rs,
//     circuit.rs), all in FP64: the oracle of the probabilistic path.
// ===========================================================================
enum ProvErr : int {
  E_NOT_BOOL = 20,       // ProvError::NotBool (provenance.rs:63)
  E_BAD_PROB = 21,       // ProvError::BadProbability
  E_PROOF_BUDGET = 22,   // ProvError::ProofBudget
  E_SOFT_AGG = 23,       // ProvError::SoftAggregate
  E_CIRCUIT_BUDGET = 24, // compile.rs BudgetExceeded
};

// A proof: sorted signed literals ±(i+1) (a BTreeSet<i64>); a proof set is an
// ordered set of proofs (BTreeSet<BTreeSet<i64>>: lexicographic order).
using Proof = std::vector<int64_t>;
using ProofSet = std::set<Proof>;

inline bool is_subset(const Proof& a, const Proof& b) {  // a ⊆ b
  return std::includes(b.begin(), b.end(), a.begin(), a.end());
}

// insert_minimal (provenance.rs:136-143).
bool insert_minimal(ProofSet& set, const Proof& proof) {
  for (auto& kept : set)
    if (is_subset(kept, proof)) return false;
  for (auto it = set.begin(); it != set.end();) {
    if (is_subset(proof, *it)) it = set.erase(it);
    else ++it;
  }
  set.insert(proof);
  return true;
}

inline Proof proof_union(const Proof& a, const Proof& b) {
  Proof u;
  u.reserve(a.size() + b.size());
  std::set_union(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(u));
  return u;
}

inline bool contradictory(const Proof& p) {
  for (auto l : p)
    if (std::binary_search(p.begin(), p.end(), -l)) return true;
  return false;
}

// product (provenance.rs:147-158).
ProofSet product(const ProofSet& acc, const ProofSet& other) {
  ProofSet out;
  for (auto& a : acc)
    for (auto& b : other) {
      Proof j = proof_union(a, b);
      if (!contradictory(j)) insert_minimal(out, j);
    }
  return out;
}

// complement (provenance.rs:166-176); false = over budget.
bool complement(const ProofSet& proofs, size_t max_proofs, ProofSet* out) {
  ProofSet acc{Proof{}};
  for (auto& p : proofs) {
    ProofSet neg;
    for (auto l : p) neg.insert(Proof{-l});
    acc = product(acc, neg);
    if (acc.size() > max_proofs) return false;
  }
  *out = acc;
  return true;
}

// proof_weight (provenance.rs:179-192): ascending literals, left fold from 1.
double proof_weight(const Proof& proof, const std::vector<double>& prob) {
  double w = 1.0;
  for (auto l : proof) {
    const double p = prob[(size_t)(std::llabs(l) - 1)];
    w = w * (l > 0 ? p : 1.0 - p);
  }
  return w;
}

// prune_top_k (provenance.rs:195-212): (weight desc, literals asc), stable.
void prune_top_k(ProofSet& set, size_t k, const std::vector<double>& prob) {
  if (set.size() <= k) return;
  std::vector<std::pair<double, Proof>> scored;
  for (auto& p : set) scored.emplace_back(proof_weight(p, prob), p);
  std::stable_sort(scored.begin(), scored.end(), [](const auto& a, const auto& b) {
    if (b.first < a.first) return true;
    if (a.first < b.first) return false;
    return a.second < b.second;
  });
  scored.resize(k);
  set.clear();
  for (auto& s : scored) set.insert(s.second);
}

struct ProvInterp {
  const Program& P;
  std::vector<std::map<Tuple, ProofSet>> db;
  std::vector<double> prob;
  std::vector<int64_t> modes;  // per predicate: 0 exact, k > 0 top-k
  size_t max_proofs;
  int cur_stratum = 0;
  ProvInterp(const Program& p, std::vector<double> probs, std::vector<int64_t> m, size_t maxp)
      : P(p), db(p.preds.size()), prob(std::move(probs)), modes(std::move(m)), max_proofs(maxp) {}

  // solve_prov (provenance.rs:368-507).
  void solve(const Rule& r, size_t idx, Binding2& binding, const ProofSet& acc,
             std::vector<std::tuple<int, Tuple, ProofSet>>& out) {
    if (idx == r.body.size()) {
      out.emplace_back(r.head.pred, Interp::ground(r.head.args, binding, false), acc);
      return;
    }
    const Lit& lit = r.body[idx];
    if (!lit.neg) {
      for (auto& row : db[lit.atom.pred]) {
        Binding2 b = binding;
        if (Interp::unify(lit.atom.args, row.first, b)) {
          ProofSet next = product(acc, row.second);
          if (next.empty()) continue;
          if (next.size() > max_proofs) throw EvalError{E_PROOF_BUDGET};
          solve(r, idx + 1, b, next, out);
        }
      }
    } else {
      if (P.preds[lit.atom.pred].stratum >= cur_stratum) throw EvalError{E_NEG_NOT_STRAT};
      Tuple t = Interp::ground(lit.atom.args, binding, true);
      auto it = db[lit.atom.pred].find(t);
      if (it == db[lit.atom.pred].end()) {
        solve(r, idx + 1, binding, acc, out);
        return;
      }
      if (it->second.count(Proof{})) return;  // certainly present
      ProofSet negated;
      if (!complement(it->second, max_proofs, &negated)) throw EvalError{E_PROOF_BUDGET};
      ProofSet next = product(acc, negated);
      if (next.empty()) return;
      if (next.size() > max_proofs) throw EvalError{E_PROOF_BUDGET};
      solve(r, idx + 1, binding, next, out);
    }
  }

  // saturate (provenance.rs:286-362): naive Jacobi rounds per stratum.
  long saturate() {
    long rounds = 0;
    for (int k = 0; k < P.num_strata; k++) {
      cur_stratum = k;
      for (auto& r : P.rules)
        if (P.preds[r.head.pred].stratum == k && r.agg_op >= 0) throw EvalError{E_SOFT_AGG};
      while (true) {
        std::vector<std::tuple<int, Tuple, ProofSet>> derived;
        for (auto& r : P.rules) {
          if (P.preds[r.head.pred].stratum != k || r.agg_op >= 0) continue;
          Binding2 b((size_t)r.var_count);
          solve(r, 0, b, ProofSet{Proof{}}, derived);
        }
        rounds++;
        bool changed = false;
        for (auto& d : derived) {
          const int pred = std::get<0>(d);
          const int64_t topk = modes[(size_t)pred];
          ProofSet& set = db[(size_t)pred][std::get<1>(d)];
          ProofSet before;
          if (topk > 0) before = set;
          bool local = false;
          for (auto& proof : std::get<2>(d)) local |= insert_minimal(set, proof);
          if (local && topk > 0) {
            prune_top_k(set, (size_t)topk, prob);
            local = set != before;
          } else if (local && set.size() > max_proofs) {
            throw EvalError{E_PROOF_BUDGET};
          }
          changed |= local;
        }
        if (!changed) break;
      }
    }
    return rounds;
  }
};

// ---- exact compilation (compile.rs) and the circuit (circuit.rs) ----------
struct CNode {
  int kind;  // 0 leaf, 1 neg leaf, 2 and, 3 or, 4 true, 5 false
  int64_t leaf;
  std::vector<size_t> ch;
};

struct CircuitBuilder {
  std::vector<CNode> nodes;
  size_t num_leaves = 0;
  size_t push(CNode n) {
    nodes.push_back(std::move(n));
    return nodes.size() - 1;
  }
};

// normalize (compile.rs:30-47).
std::vector<Proof> dnf_normalize(const std::vector<Proof>& proofs) {
  std::vector<Proof> sets;
  for (auto& p : proofs) {
    Proof q = p;
    std::sort(q.begin(), q.end());
    q.erase(std::unique(q.begin(), q.end()), q.end());
    if (!contradictory(q)) sets.push_back(q);
  }
  std::stable_sort(sets.begin(), sets.end(), [](const Proof& a, const Proof& b) { return a.size() < b.size(); });
  ProofSet min;
  for (auto& p : sets) {
    bool absorbed = false;
    for (auto& kept : min)
      if (is_subset(kept, p)) { absorbed = true; break; }
    if (!absorbed) min.insert(p);
  }
  return std::vector<Proof>(min.begin(), min.end());
}

// restrict (compile.rs:153-172).
ProofSet dnf_restrict(const std::vector<Proof>& dnf, int64_t var, bool value) {
  const int64_t dies = value ? -var : var, discharged = value ? var : -var;
  ProofSet out;
  for (auto& p : dnf) {
    if (std::binary_search(p.begin(), p.end(), dies)) continue;
    Proof q;
    for (auto l : p)
      if (l != discharged) q.push_back(l);
    bool absorbed = false;
    for (auto& kept : out)
      if (is_subset(kept, q)) { absorbed = true; break; }
    if (absorbed) continue;
    for (auto it = out.begin(); it != out.end();) {
      if (is_subset(q, *it)) it = out.erase(it);
      else ++it;
    }
    out.insert(q);
  }
  return out;
}

struct Shannon {
  CircuitBuilder& b;
  std::map<std::vector<Proof>, size_t> memo;
  size_t max_nodes;
  size_t run(const std::vector<Proof>& dnf) {  // shannon (compile.rs:103-150)
    if (b.nodes.size() > max_nodes) throw EvalError{E_CIRCUIT_BUDGET};
    if (dnf.empty()) return b.push(CNode{5, 0, {}});
    for (auto& p : dnf)
      if (p.empty()) return b.push(CNode{4, 0, {}});
    auto m = memo.find(dnf);
    if (m != memo.end()) return m->second;
    std::map<int64_t, size_t> count;
    for (auto& p : dnf)
      for (auto l : p) count[std::llabs(l)]++;
    // most frequent variable; ties to the smallest variable
    int64_t v = 0;
    size_t best = 0;
    for (auto& kv : count)
      if (kv.second > best) { best = kv.second; v = kv.first; }
    ProofSet hi_s = dnf_restrict(dnf, v, true), lo_s = dnf_restrict(dnf, v, false);
    std::vector<Proof> hi(hi_s.begin(), hi_s.end()), lo(lo_s.begin(), lo_s.end());
    const size_t hi_n = run(hi);
    const size_t lo_n = run(lo);
    const size_t leaf = (size_t)(v - 1);
    b.num_leaves = std::max(b.num_leaves, leaf + 1);
    const size_t pos = b.push(CNode{0, (int64_t)leaf, {}});
    const size_t neg = b.push(CNode{1, (int64_t)leaf, {}});
    const size_t and_hi = b.push(CNode{2, 0, {pos, hi_n}});
    const size_t and_lo = b.push(CNode{2, 0, {neg, lo_n}});
    const size_t node = b.push(CNode{3, 0, {and_hi, and_lo}});
    memo.emplace(dnf, node);
    return node;
  }
};

// Circuit::eval / grad (circuit.rs:43-106), FP64.
void circuit_grad(const std::vector<CNode>& nodes, size_t root, const std::vector<double>& p, double* value,
                  std::vector<double>* leaf_g) {
  std::vector<double> val(nodes.size(), 0.0);
  for (size_t i = 0; i < nodes.size(); i++) {
    const CNode& n = nodes[i];
    switch (n.kind) {
      case 0: val[i] = p[(size_t)n.leaf]; break;
      case 1: val[i] = 1.0 - p[(size_t)n.leaf]; break;
      case 2: { double a = 1.0; for (auto c : n.ch) a = a * val[c]; val[i] = a; break; }
      case 3: { double a = 0.0; for (auto c : n.ch) a = a + val[c]; val[i] = a; break; }
      case 4: val[i] = 1.0; break;
      default: val[i] = 0.0; break;
    }
  }
  *value = nodes.empty() ? 0.0 : val[root];
  if (!leaf_g || nodes.empty()) return;
  std::vector<double> g(nodes.size(), 0.0);
  g[root] = 1.0;
  for (size_t i = nodes.size(); i-- > 0;) {
    const double gi = g[i];
    if (gi == 0.0) continue;
    const CNode& n = nodes[i];
    if (n.kind == 0) (*leaf_g)[(size_t)n.leaf] += gi;
    else if (n.kind == 1) (*leaf_g)[(size_t)n.leaf] -= gi;
    else if (n.kind == 2) {
      for (size_t j = 0; j < n.ch.size(); j++) {
        double sib = 1.0;
        for (size_t q = 0; q < n.ch.size(); q++)
          if (q != j) sib = sib * val[n.ch[q]];
        g[n.ch[j]] += gi * sib;
      }
    } else if (n.kind == 3) {
      for (auto c : n.ch) g[c] += gi;
    }
  }
}

struct ProvHandle {
  Program P;
  std::unique_ptr<ProvInterp> I;
  long rounds = 0;
};

// ---- the TC-shaped capture restricted to queried targets -------------------
// path(X,Y) :- edge(X,Y).  path(X,Z) :- edge(X,Y), path(Y,Z).  with `path`
// Prov_k(k) and every edge fact probabilistic (literal = edge index + 1).
// For a fixed target t, path(., t) depends only on path(., t) and edge, so
// the saturation restricted to the queried targets yields the same proof
// sets for those tuples.  The per-tuple update follows saturate's order:
// the rule-1 entry, then rule-2 entries by ascending (X, Y) edge order, each
// inserted with insert_minimal and pruned after its batch.
struct TcProv {
  uint32_t n;
  // out-CSR over distinct edge tuples sorted by (X, Y); each tuple carries
  // the proofs {i+1} of its edge facts (duplicates give several)
  std::vector<uint32_t> off, nbr;
  std::vector<ProofSet> eproofs;
  std::vector<double> prob;
  size_t k;
  void build(uint32_t nodes, const uint32_t* src, const uint32_t* dst, size_t m) {
    n = nodes;
    std::vector<uint64_t> key(m);
    for (size_t i = 0; i < m; i++) key[i] = ((uint64_t)src[i] << 32) | dst[i];
    std::vector<size_t> ord(m);
    for (size_t i = 0; i < m; i++) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return key[a] < key[b]; });
    off.assign(n + 1, 0);
    nbr.clear();
    eproofs.clear();
    for (size_t q = 0; q < m; q++) {
      const size_t i = ord[q];
      if (q == 0 || key[i] != key[ord[q - 1]]) {
        nbr.push_back(dst[i]);
        eproofs.push_back(ProofSet{});
        off[src[i] + 1]++;
      }
      eproofs.back().insert(Proof{(int64_t)i + 1});
    }
    for (uint32_t v = 0; v < n; v++) off[v + 1] += off[v];
  }
  // Saturate path(., t); returns rounds.  state[X] = proof set of path(X, t).
  long run_target(uint32_t t, std::vector<ProofSet>& state) const {
    state.assign(n, ProofSet{});
    long rounds = 0;
    while (true) {
      rounds++;
      std::vector<ProofSet> next = state;
      bool changed = false;
      for (uint32_t x = 0; x < n; x++) {
        ProofSet& set = next[x];
        auto entry = [&](const ProofSet& batch) {
          ProofSet before = set;
          bool local = false;
          for (auto& pr : batch) local |= insert_minimal(set, pr);
          if (local) {
            prune_top_k(set, k, prob);
            local = set != before;
          }
          changed |= local;
        };
        // rule 1: path(X, t) :- edge(X, t)
        for (uint32_t q = off[x]; q < off[x + 1]; q++)
          if (nbr[q] == t) entry(product(ProofSet{Proof{}}, eproofs[q]));
        // rule 2: path(X, t) :- edge(X, Y), path(Y, t)
        for (uint32_t q = off[x]; q < off[x + 1]; q++) {
          const uint32_t y = nbr[q];
          if (state[y].empty()) continue;
          entry(product(product(ProofSet{Proof{}}, eproofs[q]), state[y]));
        }
      }
      state.swap(next);
      if (!changed) break;
    }
    return rounds;
  }
};

}  // namespace

// ===========================================================================
// C ABI of the oracle
// ===========================================================================
extern "C" {

// Run the interpreter.  Program blob:
//   npreds, {arity, trop, stratum}*, num_strata,
//   nrules, {var_count, head_atom, agg_op, agg_slot, agg_pos, nbody, {neg, atom}*}*,
//   nfacts, {pred, arity, {tag, val}*, wkind(0 none,1 finite,2 inf), wval}*
// atom = pred, arity, {kind, val}*.  mode: 0 naive, 1 semi-naive.
// Result blob (malloc'd, free with sko_free): for each pred in order:
//   count, {arity values as (tag,val)*, wkind, wval}*
int sko_interp(const int64_t* blob, size_t n, int mode, int threads, long max_rounds, int64_t** out,
               size_t* out_n, long* rounds) {
  try {
    Reader R{blob, 0, n};
    Program P;
    const int np = (int)R.next();
    for (int k = 0; k < np; k++) {
      Pred p;
      p.arity = (int)R.next();
      p.trop = R.next() != 0;
      p.stratum = (int)R.next();
      P.preds.push_back(p);
    }
    P.num_strata = (int)R.next();
    const int nr = (int)R.next();
    for (int k = 0; k < nr; k++) {
      Rule r;
      r.var_count = (int)R.next();
      r.head = read_atom(R);
      r.agg_op = (int)R.next();
      r.agg_slot = (int)R.next();
      r.agg_pos = (int)R.next();
      const int nb = (int)R.next();
      for (int q = 0; q < nb; q++) {
        Lit l;
        l.neg = R.next() != 0;
        l.atom = read_atom(R);
        r.body.push_back(l);
      }
      P.rules.push_back(r);
    }
    Interp I(P);
    const long nf = (long)R.next();
    for (long k = 0; k < nf; k++) {
      const int pred = (int)R.next();
      const int ar = (int)R.next();
      Tuple t;
      for (int q = 0; q < ar; q++) {
        GV g;
        g.tag = (uint8_t)R.next();
        g.v = R.next();
        t.push_back(g);
      }
      const int wk = (int)R.next();
      const int64_t wv = R.next();
      Ann a = wk == 0 ? Ann{false, Weight{false, 0}} : Ann{true, Weight{wk == 2, wk == 2 ? 0 : wv}};
      if (a.trop != P.preds[pred].trop) throw EvalError{E_ANN_MISMATCH};
      I.db[pred].combine(t, a);  // Db::insert (store.rs:88-93)
    }
    int rc = mode == 0 ? I.run_naive() : I.run_semi_naive(threads, max_rounds, rounds);
    std::vector<int64_t> res;
    for (size_t k = 0; k < P.preds.size(); k++) {
      res.push_back((int64_t)I.db[k].rows.size());
      for (auto& kv : I.db[k].rows) {
        for (auto& v : kv.first) {
          res.push_back(v.tag);
          res.push_back(v.v);
        }
        res.push_back(kv.second.trop ? (kv.second.w.inf ? 2 : 1) : 0);
        res.push_back(kv.second.trop && !kv.second.w.inf ? kv.second.w.v : 0);
      }
    }
    int64_t* buf = (int64_t*)malloc(sizeof(int64_t) * (res.size() + 1));
    std::memcpy(buf, res.data(), sizeof(int64_t) * res.size());
    *out = buf;
    *out_n = res.size();
    return rc;
  } catch (const EvalError& e) {
    *out = nullptr;
    *out_n = 0;
    return e.code;
  }
}

void sko_free(void* p) { free(p); }

// A loaded program kept between runs (the timed CPU baseline re-runs the
// fixpoint without re-loading the EDB).  Each run starts from the EDB alone.
struct SkoSession {
  Program P;
  std::vector<Relation> edb;
};

static Program decode_program(Reader& R, std::vector<Relation>* edb_out) {
  Program P;
  const int np = (int)R.next();
  for (int k = 0; k < np; k++) {
    Pred p;
    p.arity = (int)R.next();
    p.trop = R.next() != 0;
    p.stratum = (int)R.next();
    P.preds.push_back(p);
  }
  P.num_strata = (int)R.next();
  const int nr = (int)R.next();
  for (int k = 0; k < nr; k++) {
    Rule r;
    r.var_count = (int)R.next();
    r.head = read_atom(R);
    r.agg_op = (int)R.next();
    r.agg_slot = (int)R.next();
    r.agg_pos = (int)R.next();
    const int nb = (int)R.next();
    for (int q = 0; q < nb; q++) {
      Lit l;
      l.neg = R.next() != 0;
      l.atom = read_atom(R);
      r.body.push_back(l);
    }
    P.rules.push_back(r);
  }
  edb_out->clear();
  for (auto& pr : P.preds) edb_out->push_back(Relation{pr.trop, {}});
  const long nf = (long)R.next();
  for (long k = 0; k < nf; k++) {
    const int pred = (int)R.next();
    const int ar = (int)R.next();
    Tuple t;
    for (int q = 0; q < ar; q++) {
      GV g;
      g.tag = (uint8_t)R.next();
      g.v = R.next();
      t.push_back(g);
    }
    const int wk = (int)R.next();
    const int64_t wv = R.next();
    Ann a = wk == 0 ? Ann{false, Weight{false, 0}} : Ann{true, Weight{wk == 2, wk == 2 ? 0 : wv}};
    if (a.trop != P.preds[pred].trop) throw EvalError{E_ANN_MISMATCH};
    (*edb_out)[pred].combine(t, a);
  }
  return P;
}

void* sko_session_new(const int64_t* blob, size_t n) {
  try {
    Reader R{blob, 0, n};
    auto* s = new SkoSession();
    s->P = decode_program(R, &s->edb);
    return s;
  } catch (...) {
    return nullptr;
  }
}

// Run the semi-naive fixpoint (at most max_rounds delta rounds; < 0 = all)
// from the session's EDB.  counts[k] = |relation k| afterwards; *secs = the
// wall time of run_semi_naive itself (the EDB copy is not timed).
int sko_session_run(void* h, int threads, long max_rounds, int64_t* counts, long* rounds, double* secs) {
  auto* s = static_cast<SkoSession*>(h);
  try {
    Interp I(s->P);
    I.db = s->edb;
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = I.run_semi_naive(threads, max_rounds, rounds);
    const auto t1 = std::chrono::steady_clock::now();
    *secs = std::chrono::duration<double>(t1 - t0).count();
    for (size_t k = 0; k < s->P.preds.size(); k++) counts[k] = (int64_t)I.db[k].rows.size();
    return rc;
  } catch (const EvalError& e) {
    return e.code;
  }
}

void sko_session_free(void* h) { delete static_cast<SkoSession*>(h); }

}  // extern "C"

// ===========================================================================
// B. Fast restatements of the config rule shapes (same semi-naive schedule)
// ===========================================================================
namespace {

inline uint64_t key2(uint32_t a, uint32_t b) { return ((uint64_t)a << 32) | b; }

struct WeightMapEntry {
  bool inf;
  int64_t v;
};

inline bool wless(bool ai, int64_t av, bool bi, int64_t bv) {  // Weight a < b
  if (ai != bi) return !ai;
  return ai ? false : av < bv;
}

}  // namespace

extern "C" {

// Bool TC, right-linear:  path(X,Y) :- edge(X,Y).  path(X,Z) :- edge(X,Y), path(Y,Z).
// Output sorted by (src, dst) into malloc'd arrays.  Returns rounds via *rounds.
int sko_fast_tc(const uint32_t* src, const uint32_t* dst, size_t n, uint32_t** os, uint32_t** od,
                size_t* on, long* rounds) {
  std::unordered_set<uint64_t> path;
  path.reserve(n * 4 + 16);
  std::vector<uint64_t> delta;
  std::unordered_map<uint32_t, std::vector<uint32_t>> in;  // y -> xs with edge(x,y)
  for (size_t i = 0; i < n; i++) {
    const uint64_t k = key2(src[i], dst[i]);
    if (path.insert(k).second) {
      delta.push_back(k);
      in[dst[i]].push_back(src[i]);
    }
  }
  long r = 0;
  while (!delta.empty()) {
    r++;
    std::vector<uint64_t> next;
    for (uint64_t d : delta) {
      const uint32_t y = (uint32_t)(d >> 32), z = (uint32_t)d;
      auto it = in.find(y);
      if (it == in.end()) continue;
      for (uint32_t x : it->second) {
        const uint64_t k = key2(x, z);
        if (path.insert(k).second) next.push_back(k);
      }
    }
    delta.swap(next);
  }
  std::vector<uint64_t> v(path.begin(), path.end());
  std::sort(v.begin(), v.end());
  *os = (uint32_t*)malloc(4 * (v.size() + 1));
  *od = (uint32_t*)malloc(4 * (v.size() + 1));
  for (size_t i = 0; i < v.size(); i++) {
    (*os)[i] = (uint32_t)(v[i] >> 32);
    (*od)[i] = (uint32_t)v[i];
  }
  *on = v.size();
  if (rounds) *rounds = r;
  return 0;
}

// Trop, both config shapes, the interpreter's schedule:
//   shape 0:  h(X,Y) :- edge(X,Y).          h(X,Z) :- edge(X,Y), h(Y,Z).
//   shape 1:  h(S,Y) :- src(S), edge(S,Y).  h(S,Z) :- h(S,Y), edge(Y,Z).
// Δ' = tuples new or strictly improved in the round, with their merged value;
// a finite overflow anywhere in the round is an error; the stratum fails with
// a negative cycle after `universe + 2` delta rounds.
int sko_fast_trop(int shape, const uint32_t* sources, const int64_t* sw, const uint8_t* sinf, size_t ns,
                  const uint32_t* src, const uint32_t* dst, const int64_t* w, const uint8_t* winf, size_t n,
                  uint32_t** os, uint32_t** od, int64_t** ow, uint8_t** oi, size_t* on, long* rounds) {
  struct WV {
    bool inf;
    int64_t v;
  };
  auto mul = [](WV a, WV b) -> WV {
    if (a.inf || b.inf) return WV{true, 0};
    int64_t r;
    if (__builtin_add_overflow(a.v, b.v, &r)) throw EvalError{E_OVERFLOW};
    return WV{false, r};
  };
  auto lt = [](WV a, WV b) { return wless(a.inf, a.v, b.inf, b.v); };
  // EDB: edge min-merged per (x,y); src min-merged per s.
  std::unordered_map<uint64_t, WV> edge;
  edge.reserve(n * 2 + 16);
  std::set<uint32_t> uni;
  for (size_t i = 0; i < n; i++) {
    const WV x{winf && winf[i] != 0, winf && winf[i] ? 0 : w[i]};
    auto it = edge.find(key2(src[i], dst[i]));
    if (it == edge.end()) edge.emplace(key2(src[i], dst[i]), x);
    else if (lt(x, it->second)) it->second = x;
    uni.insert(src[i]);
    uni.insert(dst[i]);
  }
  std::unordered_map<uint32_t, WV> srcm;
  if (shape == 1) {
    for (size_t i = 0; i < ns; i++) {
      const WV x{sinf && sinf[i] != 0, sw ? (sinf && sinf[i] ? 0 : sw[i]) : 0};
      auto it = srcm.find(sources[i]);
      if (it == srcm.end()) srcm.emplace(sources[i], x);
      else if (lt(x, it->second)) it->second = x;
      uni.insert(sources[i]);
    }
  }
  const size_t cap = uni.size() + 2;
  // Index: shape 0 joins Δ(Y,Z) with edge(X,Y) on Y (in-edges);
  //        shape 1 joins Δ(S,Y) with edge(Y,Z) on Y (out-edges).
  std::unordered_map<uint32_t, std::vector<std::pair<uint32_t, WV>>> idx;
  for (auto& kv : edge) {
    const uint32_t x = (uint32_t)(kv.first >> 32), y = (uint32_t)kv.first;
    if (shape == 0) idx[y].emplace_back(x, kv.second);
    else idx[x].emplace_back(y, kv.second);
  }
  std::unordered_map<uint64_t, WV> full;
  full.reserve(n * 4 + 16);
  std::vector<std::pair<uint64_t, WV>> delta;
  try {
    // Bootstrap (seminaive.rs:90): every derivation of the full step.
    std::unordered_map<uint64_t, WV> boot;
    if (shape == 0) {
      for (auto& kv : edge) boot.emplace(kv.first, mul(WV{false, 0}, kv.second));
    } else {
      for (auto& s : srcm) {
        auto it = idx.find(s.first);
        if (it == idx.end()) continue;
        for (auto& e : it->second) {
          const WV x = mul(mul(WV{false, 0}, s.second), e.second);
          const uint64_t k = key2(s.first, e.first);
          auto b = boot.find(k);
          if (b == boot.end()) boot.emplace(k, x);
          else if (lt(x, b->second)) b->second = x;
        }
      }
    }
    for (auto& kv : boot) {
      full.emplace(kv.first, kv.second);
      delta.emplace_back(kv.first, kv.second);
    }
    long r = 0;
    size_t iters = 0;
    while (!delta.empty()) {
      r++;
      std::unordered_map<uint64_t, WV> best;  // min derivation per key this round
      for (auto& d : delta) {
        const uint32_t a = (uint32_t)(d.first >> 32), b = (uint32_t)d.first;
        const uint32_t j = shape == 0 ? a : b;
        auto it = idx.find(j);
        if (it == idx.end()) continue;
        for (auto& e : it->second) {
          // body order: shape 0 edge then Δ; shape 1 Δ then edge (same sum).
          const WV x = shape == 0 ? mul(mul(WV{false, 0}, e.second), d.second) : mul(mul(WV{false, 0}, d.second), e.second);
          const uint64_t k = shape == 0 ? key2(e.first, b) : key2(a, e.first);
          auto bb = best.find(k);
          if (bb == best.end()) best.emplace(k, x);
          else if (lt(x, bb->second)) bb->second = x;
        }
      }
      std::vector<std::pair<uint64_t, WV>> next;
      for (auto& kv : best) {
        auto f = full.find(kv.first);
        if (f == full.end()) {
          full.emplace(kv.first, kv.second);
          next.emplace_back(kv.first, kv.second);
        } else if (lt(kv.second, f->second)) {
          f->second = kv.second;
          next.emplace_back(kv.first, kv.second);
        }
      }
      delta.swap(next);
      iters++;
      if (iters > cap) throw EvalError{E_NEG_CYCLE};
    }
    if (rounds) *rounds = r;
  } catch (const EvalError& e) {
    *on = 0;
    *os = *od = nullptr;
    *ow = nullptr;
    *oi = nullptr;
    return e.code;
  }
  std::vector<std::pair<uint64_t, WV>> v(full.begin(), full.end());
  std::sort(v.begin(), v.end(), [](auto& a, auto& b) { return a.first < b.first; });
  *os = (uint32_t*)malloc(4 * (v.size() + 1));
  *od = (uint32_t*)malloc(4 * (v.size() + 1));
  *ow = (int64_t*)malloc(8 * (v.size() + 1));
  *oi = (uint8_t*)malloc(v.size() + 1);
  for (size_t i = 0; i < v.size(); i++) {
    (*os)[i] = (uint32_t)(v[i].first >> 32);
    (*od)[i] = (uint32_t)v[i].first;
    (*ow)[i] = v[i].second.inf ? 0 : v[i].second.v;
    (*oi)[i] = v[i].second.inf ? 1 : 0;
  }
  *on = v.size();
  return 0;
}

// ===========================================================================
// C. Independent oracles
// ===========================================================================

static inline uint64_t mix64(uint64_t z) {  // splitmix64 finalizer (same as the device)
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Fingerprint of tuples (src, dst[, w, inf]): Σ mix(...) mod 2^64.
uint64_t sko_fingerprint(const uint32_t* s, const uint32_t* d, const int64_t* w, const uint8_t* inf, size_t n) {
  uint64_t acc = 0;
  for (size_t i = 0; i < n; i++) {
    uint64_t h = mix64(((uint64_t)s[i] << 32) | d[i]);
    if (w) {
      const uint64_t wv = (inf && inf[i]) ? 0xfffffffffffffffull : (uint64_t)w[i];
      h = mix64(h ^ mix64(wv + 0x51ull));
    }
    acc += h;
  }
  return acc;
}

// Closure by BFS from every source node (multi-threaded): count + fingerprint.
void sko_bfs_closure(const uint32_t* src, const uint32_t* dst, size_t n, int threads, uint64_t* count,
                     uint64_t* fp) {
  uint32_t maxid = 0;
  for (size_t i = 0; i < n; i++) maxid = std::max(maxid, std::max(src[i], dst[i]));
  const size_t N = n ? (size_t)maxid + 1 : 0;
  std::vector<uint32_t> off(N + 1, 0), adj(n);
  for (size_t i = 0; i < n; i++) off[src[i] + 1]++;
  for (size_t v = 0; v < N; v++) off[v + 1] += off[v];
  std::vector<uint32_t> fill(off.begin(), off.end() - (N ? 1 : 0));
  for (size_t i = 0; i < n; i++) adj[fill[src[i]]++] = dst[i];
  std::atomic<uint64_t> c{0}, f{0};
  std::atomic<size_t> next{0};
  auto work = [&]() {
    std::vector<uint32_t> seen(N, 0xffffffffu), q;
    uint64_t lc = 0, lf = 0;
    while (true) {
      const size_t s = next.fetch_add(1);
      if (s >= N) break;
      q.clear();
      for (uint32_t k = off[s]; k < off[s + 1]; k++) {
        const uint32_t v = adj[k];
        if (seen[v] != s) { seen[v] = (uint32_t)s; q.push_back(v); }
      }
      for (size_t h = 0; h < q.size(); h++) {
        const uint32_t u = q[h];
        for (uint32_t k = off[u]; k < off[u + 1]; k++) {
          const uint32_t v = adj[k];
          if (seen[v] != s) { seen[v] = (uint32_t)s; q.push_back(v); }
        }
      }
      for (uint32_t v : q) {
        lc++;
        lf += mix64(((uint64_t)s << 32) | v);
      }
    }
    c += lc;
    f += lf;
  };
  std::vector<std::thread> th;
  for (int t = 0; t < std::max(1, threads); t++) th.emplace_back(work);
  for (auto& t : th) t.join();
  *count = c;
  *fp = f;
}

// ---- per-instance closure count + row-polynomial fingerprint --------------
// For the batched reachability form the closure of an instance is summarised
// by |path| and  fp = Σ_{(X,Z) ∈ path} mix64(X) · c^Z  (mod 2^64), c the odd
// constant kPolyC — order-independent, and computable from bit rows one word
// at a time.  This oracle is independent of the engine's round structure:
// strongly connected components (iterative Tarjan, components complete in
// reverse topological order), then per component C the set R(C) of nodes
// reachable by a path of length >= 1:
//   R(C) = (C if C has a cycle) ∪ ⋃_{C -> C'} (C' ∪ R(C')).
static const uint64_t kPolyC = 0x9e3779b97f4a7c15ull;

struct PolyTables {
  uint64_t tb[8][256];  // tb[b][v] = Σ_{j ∈ bits(v)} c^(8b + j)
  PolyTables() {
    uint64_t pw[64];
    pw[0] = 1;
    for (int j = 1; j < 64; j++) pw[j] = pw[j - 1] * kPolyC;
    for (int b = 0; b < 8; b++)
      for (int v = 0; v < 256; v++) {
        uint64_t a = 0;
        for (int j = 0; j < 8; j++)
          if (v >> j & 1) a += pw[8 * b + j];
        tb[b][v] = a;
      }
  }
};

static void closure_count_fp(uint32_t n, const uint32_t* src, const uint32_t* dst, uint64_t m,
                             const PolyTables& T, uint64_t* count, uint64_t* fp) {
  std::vector<uint32_t> off(n + 1, 0), adj(m);
  for (uint64_t i = 0; i < m; i++) off[src[i] + 1]++;
  for (uint32_t v = 0; v < n; v++) off[v + 1] += off[v];
  {
    std::vector<uint32_t> fill(off.begin(), off.end() - 1);
    for (uint64_t i = 0; i < m; i++) adj[fill[src[i]]++] = dst[i];
  }
  // iterative Tarjan
  std::vector<int64_t> idx(n, -1), low(n, 0);
  std::vector<int64_t> comp(n, -1);
  std::vector<uint32_t> stk;
  std::vector<char> on(n, 0);
  struct Frame { uint32_t v; uint32_t e; };
  std::vector<Frame> cs;
  int64_t next_idx = 0, ncomp = 0;
  for (uint32_t s0 = 0; s0 < n; s0++) {
    if (idx[s0] >= 0) continue;
    idx[s0] = low[s0] = next_idx++;
    stk.push_back(s0);
    on[s0] = 1;
    cs.push_back({s0, off[s0]});
    while (!cs.empty()) {
      const uint32_t v = cs.back().v;
      if (cs.back().e < off[v + 1]) {
        const uint32_t w = adj[cs.back().e++];
        if (idx[w] < 0) {
          idx[w] = low[w] = next_idx++;
          stk.push_back(w);
          on[w] = 1;
          cs.push_back({w, off[w]});
        } else if (on[w]) {
          low[v] = std::min(low[v], idx[w]);
        }
      } else {
        if (low[v] == idx[v]) {
          while (true) {
            const uint32_t x = stk.back();
            stk.pop_back();
            on[x] = 0;
            comp[x] = ncomp;
            if (x == v) break;
          }
          ncomp++;
        }
        cs.pop_back();
        if (!cs.empty()) {
          const uint32_t p = cs.back().v;
          low[p] = std::min(low[p], low[v]);
        }
      }
    }
  }
  // members per component, cycle flag, pending predecessor edges
  std::vector<uint32_t> moff(ncomp + 1, 0), mem(n);
  for (uint32_t v = 0; v < n; v++) moff[comp[v] + 1]++;
  for (int64_t c = 0; c < ncomp; c++) moff[c + 1] += moff[c];
  {
    std::vector<uint32_t> fill(moff.begin(), moff.end() - 1);
    for (uint32_t v = 0; v < n; v++) mem[fill[comp[v]]++] = v;
  }
  std::vector<char> cyc(ncomp, 0);
  std::vector<uint64_t> pend(ncomp, 0);
  for (uint32_t x = 0; x < n; x++)
    for (uint32_t k = off[x]; k < off[x + 1]; k++) {
      const uint32_t y = adj[k];
      if (comp[y] == comp[x]) cyc[comp[x]] = 1;  // an edge inside C (self-loop or cycle)
      else pend[comp[y]]++;
    }
  for (int64_t c = 0; c < ncomp; c++)
    if (moff[c + 1] - moff[c] > 1) cyc[c] = 1;
  const size_t W = ((size_t)n + 63) / 64;
  std::vector<uint64_t> cw(W);  // c^(64 w)
  {
    uint64_t c64 = 1;
    for (int j = 0; j < 64; j++) c64 *= kPolyC;
    uint64_t a = 1;
    for (size_t w = 0; w < W; w++) { cw[w] = a; a *= c64; }
  }
  std::vector<std::vector<uint64_t>> rstar(ncomp);
  uint64_t cnt = 0, f = 0;
  std::vector<uint64_t> R(W);
  for (int64_t c = 0; c < ncomp; c++) {
    std::fill(R.begin(), R.end(), 0ull);
    if (cyc[c])
      for (uint32_t k = moff[c]; k < moff[c + 1]; k++) R[mem[k] >> 6] |= 1ull << (mem[k] & 63);
    for (uint32_t k = moff[c]; k < moff[c + 1]; k++) {
      const uint32_t x = mem[k];
      for (uint32_t e = off[x]; e < off[x + 1]; e++) {
        const int64_t c2 = comp[adj[e]];
        if (c2 == c) continue;
        const std::vector<uint64_t>& r2 = rstar[c2];
        for (size_t w = 0; w < W; w++) R[w] |= r2[w];
        if (--pend[c2] == 0) std::vector<uint64_t>().swap(rstar[c2]);
      }
    }
    uint64_t pc = 0, poly = 0;
    for (size_t w = 0; w < W; w++) {
      const uint64_t x = R[w];
      if (!x) continue;
      pc += (uint64_t)__builtin_popcountll(x);
      uint64_t t = 0;
      for (int b = 0; b < 8; b++) t += T.tb[b][(x >> (8 * b)) & 255];
      poly += cw[w] * t;
    }
    uint64_t msum = 0;
    for (uint32_t k = moff[c]; k < moff[c + 1]; k++) msum += mix64(mem[k]);
    cnt += (uint64_t)(moff[c + 1] - moff[c]) * pc;
    f += msum * poly;
    if (pend[c]) {
      rstar[c] = R;
      for (uint32_t k = moff[c]; k < moff[c + 1]; k++) rstar[c][mem[k] >> 6] |= 1ull << (mem[k] & 63);
    }
  }
  *count = cnt;
  *fp = f;
}

// Multi-source shortest non-empty paths by Dijkstra (non-negative finite
// weights): dist(S, Y) for every Y reachable from S by >= 1 edge, seeded with
// the source weight.  Count + fingerprint (same mixing as the device).
int sko_dijkstra_mssp(const uint32_t* sources, const int64_t* sw, size_t ns, const uint32_t* src,
                      const uint32_t* dst, const int64_t* w, size_t n, int threads, uint64_t* count,
                      uint64_t* fp) {
  uint32_t maxid = 0;
  for (size_t i = 0; i < n; i++) {
    maxid = std::max(maxid, std::max(src[i], dst[i]));
    if (w[i] < 0) return 1;
  }
  const size_t N = (size_t)maxid + 1;
  std::vector<uint32_t> off(N + 1, 0), adj(n);
  std::vector<int64_t> aw(n);
  for (size_t i = 0; i < n; i++) off[src[i] + 1]++;
  for (size_t v = 0; v < N; v++) off[v + 1] += off[v];
  std::vector<uint32_t> fill(off.begin(), off.end() - 1);
  for (size_t i = 0; i < n; i++) {
    const uint32_t p = fill[src[i]]++;
    adj[p] = dst[i];
    aw[p] = w[i];
  }
  // distinct sources, min seed weight
  std::map<uint32_t, int64_t> seeds;
  for (size_t i = 0; i < ns; i++) {
    const int64_t x = sw ? sw[i] : 0;
    auto it = seeds.find(sources[i]);
    if (it == seeds.end() || x < it->second) seeds[sources[i]] = x;
  }
  std::vector<std::pair<uint32_t, int64_t>> sv(seeds.begin(), seeds.end());
  std::atomic<uint64_t> c{0}, f{0};
  std::atomic<size_t> next{0};
  auto work = [&]() {
    std::vector<int64_t> dist(N, INT64_MAX);
    std::vector<uint32_t> touched;
    uint64_t lc = 0, lf = 0;
    using QE = std::pair<int64_t, uint32_t>;
    while (true) {
      const size_t qi = next.fetch_add(1);
      if (qi >= sv.size()) break;
      const uint32_t s = sv[qi].first;
      const int64_t base = sv[qi].second;
      std::priority_queue<QE, std::vector<QE>, std::greater<QE>> pq;
      if (s < N) {
        for (uint32_t k = off[s]; k < off[s + 1]; k++) {
          const int64_t d = base + aw[k];
          if (d < dist[adj[k]]) {
            if (dist[adj[k]] == INT64_MAX) touched.push_back(adj[k]);
            dist[adj[k]] = d;
            pq.emplace(d, adj[k]);
          }
        }
      }
      while (!pq.empty()) {
        auto [d, u] = pq.top();
        pq.pop();
        if (d != dist[u]) continue;
        for (uint32_t k = off[u]; k < off[u + 1]; k++) {
          const int64_t nd = d + aw[k];
          if (nd < dist[adj[k]]) {
            if (dist[adj[k]] == INT64_MAX) touched.push_back(adj[k]);
            dist[adj[k]] = nd;
            pq.emplace(nd, adj[k]);
          }
        }
      }
      for (uint32_t v : touched) {
        lc++;
        uint64_t h = mix64(((uint64_t)s << 32) | v);
        h = mix64(h ^ mix64((uint64_t)dist[v] + 0x51ull));
        lf += h;
        dist[v] = INT64_MAX;
      }
      touched.clear();
    }
    c += lc;
    f += lf;
  };
  std::vector<std::thread> th;
  for (int t = 0; t < std::max(1, threads); t++) th.emplace_back(work);
  for (auto& t : th) t.join();
  *count = c;
  *fp = f;
  return 0;
}

// The same shortest paths as rows: every (S, Z, dist) with a finite distance,
// sorted by (S, Z), in malloc'd arrays (free with sko_free).  Independent of
// the interpreter (layer C); with non-negative weights the semi-naive
// fixpoint's minima are exactly these distances.
int sko_dijkstra_mssp_rows(const uint32_t* sources, const int64_t* sw, size_t ns, const uint32_t* src,
                           const uint32_t* dst, const int64_t* w, size_t n, int threads, uint32_t** out_s,
                           uint32_t** out_d, int64_t** out_w, size_t* out_n) {
  uint32_t maxid = 0;
  for (size_t i = 0; i < n; i++) {
    maxid = std::max(maxid, std::max(src[i], dst[i]));
    if (w[i] < 0) return 1;
  }
  const size_t N = (size_t)maxid + 1;
  std::vector<uint32_t> off(N + 1, 0), adj(n);
  std::vector<int64_t> aw(n);
  for (size_t i = 0; i < n; i++) off[src[i] + 1]++;
  for (size_t v = 0; v < N; v++) off[v + 1] += off[v];
  std::vector<uint32_t> fill(off.begin(), off.end() - 1);
  for (size_t i = 0; i < n; i++) {
    const uint32_t p = fill[src[i]]++;
    adj[p] = dst[i];
    aw[p] = w[i];
  }
  std::map<uint32_t, int64_t> seeds;
  for (size_t i = 0; i < ns; i++) {
    const int64_t x = sw ? sw[i] : 0;
    auto it = seeds.find(sources[i]);
    if (it == seeds.end() || x < it->second) seeds[sources[i]] = x;
  }
  std::vector<std::pair<uint32_t, int64_t>> sv(seeds.begin(), seeds.end());
  std::vector<std::vector<std::pair<uint32_t, int64_t>>> res(sv.size());
  std::atomic<size_t> next{0};
  auto work = [&]() {
    std::vector<int64_t> dist(N, INT64_MAX);
    std::vector<uint32_t> touched;
    using QE = std::pair<int64_t, uint32_t>;
    while (true) {
      const size_t qi = next.fetch_add(1);
      if (qi >= sv.size()) break;
      const uint32_t s0 = sv[qi].first;
      std::priority_queue<QE, std::vector<QE>, std::greater<QE>> pq;
      auto relax = [&](uint32_t u, int64_t d) {
        for (uint32_t k = off[u]; k < off[u + 1]; k++) {
          const int64_t nd = d + aw[k];
          if (nd < dist[adj[k]]) {
            if (dist[adj[k]] == INT64_MAX) touched.push_back(adj[k]);
            dist[adj[k]] = nd;
            pq.emplace(nd, adj[k]);
          }
        }
      };
      if (s0 < N) relax(s0, sv[qi].second);
      while (!pq.empty()) {
        auto [d, u] = pq.top();
        pq.pop();
        if (d == dist[u]) relax(u, d);
      }
      std::sort(touched.begin(), touched.end());
      auto& r = res[qi];
      r.reserve(touched.size());
      for (uint32_t v : touched) {
        r.emplace_back(v, dist[v]);
        dist[v] = INT64_MAX;
      }
      touched.clear();
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < std::max(1, threads); t++) th.emplace_back(work);
  for (auto& t : th) t.join();
  size_t total = 0;
  for (auto& r : res) total += r.size();
  *out_s = (uint32_t*)std::malloc(std::max<size_t>(1, total) * 4);
  *out_d = (uint32_t*)std::malloc(std::max<size_t>(1, total) * 4);
  *out_w = (int64_t*)std::malloc(std::max<size_t>(1, total) * 8);
  size_t k = 0;
  for (size_t qi = 0; qi < sv.size(); qi++)
    for (auto& [v, d] : res[qi]) {
      (*out_s)[k] = sv[qi].first;
      (*out_d)[k] = v;
      (*out_w)[k] = d;
      k++;
    }
  *out_n = total;
  return 0;
}

// Count aggregate  n(count<X>) :- e(X,Y), e(Y,Z), e(X,Z)  over the set e:
// the number of bindings, by sorted-list intersection per edge (threads).
uint64_t sko_count_pattern(const uint32_t* x, const uint32_t* y, size_t n, int threads) {
  std::vector<uint64_t> k(n);
  for (size_t i = 0; i < n; i++) k[i] = key2(x[i], y[i]);
  std::sort(k.begin(), k.end());
  k.erase(std::unique(k.begin(), k.end()), k.end());
  uint32_t maxid = 0;
  for (auto v : k) maxid = std::max(maxid, std::max((uint32_t)(v >> 32), (uint32_t)v));
  const size_t N = k.empty() ? 0 : (size_t)maxid + 1;
  std::vector<uint64_t> off(N + 1, 0);
  std::vector<uint32_t> adj(k.size());
  for (size_t i = 0; i < k.size(); i++) {
    off[(k[i] >> 32) + 1]++;
    adj[i] = (uint32_t)k[i];
  }
  for (size_t v = 0; v < N; v++) off[v + 1] += off[v];
  std::atomic<uint64_t> total{0};
  std::atomic<size_t> next{0};
  auto work = [&]() {
    uint64_t c = 0;
    while (true) {
      const size_t b = next.fetch_add(4096);
      if (b >= k.size()) break;
      const size_t e = std::min(k.size(), b + 4096);
      for (size_t i = b; i < e; i++) {
        const uint32_t u = (uint32_t)(k[i] >> 32), v = (uint32_t)k[i];
        uint64_t a = off[u], ae = off[u + 1], p = off[v], pe = off[v + 1];
        while (a < ae && p < pe) {
          if (adj[a] < adj[p]) a++;
          else if (adj[a] > adj[p]) p++;
          else { c++; a++; p++; }
        }
      }
    }
    total += c;
  };
  std::vector<std::thread> th;
  for (int t = 0; t < std::max(1, threads); t++) th.emplace_back(work);
  for (auto& t : th) t.join();
  return total;
}

// Triangles of the undirected simple graph by checking every triple (tiny n).
uint64_t sko_brute_triangles(const uint32_t* a, const uint32_t* b, size_t n, uint32_t nodes) {
  std::set<uint64_t> es;
  for (size_t i = 0; i < n; i++) {
    if (a[i] == b[i]) continue;
    es.insert(key2(std::min(a[i], b[i]), std::max(a[i], b[i])));
  }
  uint64_t t = 0;
  for (uint32_t x = 0; x < nodes; x++)
    for (uint32_t y = x + 1; y < nodes; y++) {
      if (!es.count(key2(x, y))) continue;
      for (uint32_t z = y + 1; z < nodes; z++)
        if (es.count(key2(x, z)) && es.count(key2(y, z))) t++;
    }
  return t;
}

uint64_t sko_brute_4cliques(const uint32_t* a, const uint32_t* b, size_t n, uint32_t nodes) {
  std::set<uint64_t> es;
  for (size_t i = 0; i < n; i++) {
    if (a[i] == b[i]) continue;
    es.insert(key2(std::min(a[i], b[i]), std::max(a[i], b[i])));
  }
  auto e = [&](uint32_t x, uint32_t y) { return es.count(key2(std::min(x, y), std::max(x, y))) > 0; };
  uint64_t t = 0;
  for (uint32_t p = 0; p < nodes; p++)
    for (uint32_t q = p + 1; q < nodes; q++) {
      if (!e(p, q)) continue;
      for (uint32_t r = q + 1; r < nodes; r++) {
        if (!(e(p, r) && e(q, r))) continue;
        for (uint32_t s = r + 1; s < nodes; s++)
          if (e(p, s) && e(q, s) && e(r, s)) t++;
      }
    }
  return t;
}


// Closure count + row-polynomial fingerprint of one graph on nodes [0, n).
int sko_closure_count_fp(uint32_t n, const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t* count,
                         uint64_t* fp) {
  for (uint64_t i = 0; i < m; i++)
    if (src[i] >= n || dst[i] >= n) return 1;
  static const PolyTables T;
  closure_count_fp(n, src, dst, m, T, count, fp);
  return 0;
}

// The same for a batch of instances (instance i: nodes[i], edges
// [edge_off[i], edge_off[i+1])), largest first across `threads` threads.
int sko_closure_batch(uint32_t n_inst, const uint32_t* nodes, const uint64_t* edge_off, const uint32_t* src,
                      const uint32_t* dst, int threads, uint64_t* counts, uint64_t* fps) {
  static const PolyTables T;
  std::vector<uint32_t> order(n_inst);
  for (uint32_t i = 0; i < n_inst; i++) order[i] = i;
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return nodes[a] > nodes[b]; });
  std::atomic<uint32_t> next{0};
  std::atomic<int> bad{0};
  auto work = [&]() {
    while (true) {
      const uint32_t k = next.fetch_add(1);
      if (k >= n_inst) break;
      const uint32_t i = order[k];
      const uint64_t a = edge_off[i], b = edge_off[i + 1];
      bool ok = true;
      for (uint64_t e = a; e < b; e++)
        if (src[e] >= nodes[i] || dst[e] >= nodes[i]) ok = false;
      if (!ok) { bad = 1; continue; }
      closure_count_fp(nodes[i], src + a, dst + a, b - a, T, &counts[i], &fps[i]);
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < std::max(1, threads); t++) th.emplace_back(work);
  for (auto& t : th) t.join();
  return bad.load();
}


// ---- provenance capture, compilation and WMC (FP64) ------------------------
static void put_proofs(const ProofSet& ps, std::vector<int64_t>& out) {
  out.push_back((int64_t)ps.size());
  for (auto& p : ps) {
    out.push_back((int64_t)p.size());
    for (auto l : p) out.push_back(l);
  }
}

// Capture over a program blob whose facts with weight kind 3 are the
// probabilistic leaves (in blob order, probabilities in `probs`); `modes[p]`
// is 0 (exact) or k (Prov_k) per predicate.  Returns a handle or null with
// *err set.
void* sko_prov_run(const int64_t* blob, size_t n, const double* probs, size_t n_prob, const int64_t* modes,
                   size_t max_proofs, long* rounds, int* err) {
  *err = 0;
  try {
    Reader R{blob, 0, n};
    auto* h = new ProvHandle();
    h->P = parse_program(R);
    for (auto& pr : h->P.preds)
      if (pr.trop) { delete h; *err = E_NOT_BOOL; return nullptr; }
    std::vector<double> pv(probs, probs + n_prob);
    for (double p : pv)
      if (!(p >= 0.0 && p <= 1.0)) { delete h; *err = E_BAD_PROB; return nullptr; }
    h->I.reset(new ProvInterp(h->P, pv, std::vector<int64_t>(modes, modes + h->P.preds.size()), max_proofs));
    const long nf = (long)R.next();
    int64_t leaf = 0;
    for (long q = 0; q < nf; q++) {
      const int pred = (int)R.next();
      const int ar = (int)R.next();
      Tuple t;
      for (int c = 0; c < ar; c++) {
        GV g;
        g.tag = (uint8_t)R.next();
        g.v = R.next();
        t.push_back(g);
      }
      const int wk = (int)R.next();
      (void)R.next();
      if (wk == 3) {
        if ((size_t)leaf >= n_prob) { delete h; *err = E_BAD_PROB; return nullptr; }
        insert_minimal(h->I->db[(size_t)pred][t], Proof{leaf + 1});
        leaf++;
      } else {
        insert_minimal(h->I->db[(size_t)pred][t], Proof{});
      }
    }
    h->rounds = h->I->saturate();
    if (rounds) *rounds = h->rounds;
    return h;
  } catch (const EvalError& e) {
    *err = e.code;
    return nullptr;
  }
}

void sko_prov_free(void* h) { delete static_cast<ProvHandle*>(h); }

// Proofs of pred(tuple) serialized as [n, (len, lits...)*]; -1 = no tuple.
long sko_prov_proofs(void* hv, int pred, const int64_t* vals, int arity, int64_t* out, size_t cap) {
  auto* h = static_cast<ProvHandle*>(hv);
  Tuple t;
  for (int c = 0; c < arity; c++) t.push_back(GV{(uint8_t)vals[2 * c], vals[2 * c + 1]});
  auto it = h->I->db[(size_t)pred].find(t);
  if (it == h->I->db[(size_t)pred].end()) return -1;
  std::vector<int64_t> buf;
  put_proofs(it->second, buf);
  if (buf.size() <= cap) std::copy(buf.begin(), buf.end(), out);
  return (long)buf.size();
}

// Every tuple of a predicate: [n_tuples, (arity values as tag,val..., proofs)*].
long sko_prov_relation(void* hv, int pred, int64_t* out, size_t cap) {
  auto* h = static_cast<ProvHandle*>(hv);
  std::vector<int64_t> buf;
  buf.push_back((int64_t)h->I->db[(size_t)pred].size());
  for (auto& kv : h->I->db[(size_t)pred]) {
    for (auto& v : kv.first) {
      buf.push_back(v.tag);
      buf.push_back(v.v);
    }
    put_proofs(kv.second, buf);
  }
  if (buf.size() <= cap) std::copy(buf.begin(), buf.end(), out);
  return (long)buf.size();
}

// compile_exact + Circuit::grad on serialized proofs [n, (len, lits...)*].
int sko_compile_grad(const int64_t* ser, size_t n_leaves, const double* probs, size_t max_nodes, double* p_out,
                     double* grad_out, int64_t* nodes_out) {
  try {
    std::vector<Proof> proofs;
    size_t i = 0;
    const int64_t np = ser[i++];
    for (int64_t q = 0; q < np; q++) {
      const int64_t len = ser[i++];
      proofs.emplace_back(ser + i, ser + i + len);
      i += (size_t)len;
    }
    std::vector<Proof> dnf = dnf_normalize(proofs);
    CircuitBuilder b;
    Shannon sh{b, {}, max_nodes};
    const size_t root = sh.run(dnf);
    const size_t nl = std::max(n_leaves, b.num_leaves);
    std::vector<double> pv(probs, probs + n_leaves);
    pv.resize(nl, 0.0);
    std::vector<double> g(nl, 0.0);
    circuit_grad(b.nodes, root, pv, p_out, grad_out ? &g : nullptr);
    if (grad_out) std::copy(g.begin(), g.begin() + (long)n_leaves, grad_out);
    if (nodes_out) *nodes_out = (int64_t)b.nodes.size();
    return 0;
  } catch (const EvalError& e) {
    return e.code;
  }
}

// The TC-shaped capture restricted to `targets` (edge i has probability
// probs[i] and literal i+1).  For each query q = (qs[q], qt[q]) writes the
// serialized proofs of path(qs, qt) into a buffer (offsets in q_off, n+1).
// Per-target rounds go to rounds[t].  Returns 0, or -1 when `cap` is short
// (*need gets the size).
long sko_prov_tc(uint32_t n, const uint32_t* src, const uint32_t* dst, size_t m, const double* probs, size_t k,
                 const uint32_t* targets, size_t n_targets, const uint32_t* qs, const uint32_t* qt, size_t nq,
                 int threads, int64_t* out, size_t cap, int64_t* q_off, long* rounds, size_t* need) {
  TcProv tp;
  tp.build(n, src, dst, m);
  tp.prob.assign(probs, probs + m);
  tp.k = k;
  std::vector<std::vector<int64_t>> per_q(nq);
  std::atomic<size_t> next{0};
  auto work = [&]() {
    std::vector<ProofSet> state;
    while (true) {
      const size_t ti = next.fetch_add(1);
      if (ti >= n_targets) break;
      const uint32_t t = targets[ti];
      const long r = tp.run_target(t, state);
      if (rounds) rounds[ti] = r;
      for (size_t q = 0; q < nq; q++)
        if (qt[q] == t) put_proofs(qs[q] < n ? state[qs[q]] : ProofSet{}, per_q[q]);
    }
  };
  std::vector<std::thread> th;
  for (int q = 0; q < std::max(1, threads); q++) th.emplace_back(work);
  for (auto& x : th) x.join();
  size_t total = 0;
  for (size_t q = 0; q < nq; q++) {
    q_off[q] = (int64_t)total;
    total += per_q[q].size();
  }
  q_off[nq] = (int64_t)total;
  *need = total;
  if (total > cap) return -1;
  for (size_t q = 0; q < nq; q++) std::copy(per_q[q].begin(), per_q[q].end(), out + q_off[q]);
  return 0;
}

}  // extern "C"
