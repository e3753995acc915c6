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

}  // extern "C"
